"""gb_linked_cell_sort_static: the linked-cell sort without device allocation.

Callers that cannot call cudaMalloc where they need the broad phase -- their
device memory is wholly reserved by another allocator in the process, or
their time loop must not block on an allocation -- use this entry point; its
scratch is a static device array of the library.  Its sort order and
cell-start table must equal those of the existing gb_update_links, on two
calls in a row (the second call reuses the scratch left by the first).
"""
import ctypes as C

import numpy as np
import pytest

from grains3dgpu_b200 import abi, engine, scenes

pytestmark = pytest.mark.gpu

MAX_PARTICLES = 262_144


def static_sort_fn():
    fn = engine.load().lib.gb_linked_cell_sort_static
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.c_double,
                   C.POINTER(C.c_int32), C.c_void_p, C.c_void_p, C.c_void_p]
    return fn


def static_sort_scene(kind):
    if kind == "one-tile":
        return scenes.superquadric_column(n=1500, pitch=2.05e-3)
    # the size limit: 128 tiles of the radix sort and, on the workload's
    # 0.3 x 0.3 x 1.2 m grid (~2.8e5 cells, 19 key bits), three radix passes
    return scenes.polydisperse_superquadrics(seed=7, n=MAX_PARTICLES)


@pytest.mark.parametrize("kind", ["one-tile", "max-size"])
def test_static_sort_matches_update_links(gb, kind):
    import torch
    fn = static_sort_fn()
    scene = static_sort_scene(kind)
    s = scenes.System(gb, scene, precision=abi.GB_FP64)
    assert gb.update_links(s.ctx) == abi.GB_OK
    ref_ids = s.dump(abi.GB_DUMP_SORTED_IDS)
    ref_start = s.dump(abi.GB_DUMP_CELL_START)
    st = s.stats()
    if kind == "max-size":
        assert s.n == MAX_PARTICLES and st.key_bits > 16
    origin = (C.c_double * 3)(*scene.config["origin"])
    dims = (C.c_int32 * 3)(*st.cells_per_dir)
    pos = C.c_void_p()
    assert gb.device_pointer(s.ctx, b"pos_x", C.byref(pos)) == abi.GB_OK  # x, y, z follow
    assert gb.synchronize(s.ctx) == abi.GB_OK
    out_ids = torch.empty(s.n, dtype=torch.int32, device="cuda")
    out_start = torch.empty(st.n_cells + 1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        out_ids.fill_(-1)
        out_start.fill_(-1)
        rc = fn(pos, s.n, origin, st.cell_size, dims, out_ids.data_ptr(), out_start.data_ptr(),
                stream)
        assert rc == abi.GB_OK, engine.status_string(rc)
        torch.cuda.synchronize()
        assert np.array_equal(out_ids.cpu().numpy().view(np.uint32), ref_ids)
        assert np.array_equal(out_start.cpu().numpy().view(np.uint32), ref_start)
    s.close()


def test_static_sort_rejects_oversize(gb):
    fn = static_sort_fn()
    origin = (C.c_double * 3)(0.0, 0.0, 0.0)
    dims = (C.c_int32 * 3)(4, 4, 4)
    dummy = C.c_void_p(16)  # never dereferenced: the size check comes first
    rc = fn(dummy, MAX_PARTICLES + 1, origin, 1e-3, dims, dummy, dummy, None)
    assert rc == abi.GB_E_CAPACITY
