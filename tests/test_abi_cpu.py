"""The C ABI and the host-side logic, without a GPU.

No test here launches device work: the library is loaded, its exports are
checked against include/grains_b200.h, struct layouts are checked against a
C compiler's, and the host-only set-up functions are compared with the
oracle.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from grains3dgpu_b200 import abi, engine, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol():
    lib = engine.load()
    missing = [s for s in engine.declared_symbols() if not hasattr(lib.lib, s)]
    assert not missing, missing


def test_library_has_no_exit_path():
    """No host code path may terminate the process (every call returns a status)."""
    out = subprocess.run(["nm", "-D", "--undefined-only", engine.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    names = {line.split()[-1].split("@")[0] for line in out.splitlines() if line.strip()}
    assert not names & {"exit", "_exit", "abort", "quick_exit"}


def test_status_strings_and_version():
    lib = engine.load()
    assert lib.abi_version() == 1
    for st in range(0, -10, -1):
        assert lib.status_string(st)
    assert lib.status_string(-1).decode() == "invalid argument"


def test_struct_layouts_match_the_c_compiler(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text("""
#include <stdio.h>
#include <stddef.h>
#include "grains_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(gb_convex), sizeof(gb_rigid_body_desc),
         sizeof(gb_rigid_body_props), sizeof(gb_contact_model), sizeof(gb_config),
         sizeof(gb_stats));
  printf("%zu %zu %zu %zu\\n", offsetof(gb_config, dt), offsetof(gb_config, pair_capacity),
         offsetof(gb_config, flags), offsetof(gb_stats, kernel_launches));
  return 0; }
""")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    sizes, offs = subprocess.run([str(exe)], capture_output=True, text=True,
                                 check=True).stdout.split("\n")[:2]
    assert [int(x) for x in sizes.split()] == [
        C.sizeof(abi.Convex), C.sizeof(abi.RigidBodyDesc), C.sizeof(abi.RigidBodyProps),
        C.sizeof(abi.ContactModel), C.sizeof(abi.Config), C.sizeof(abi.Stats)]
    assert [int(x) for x in offs.split()] == [
        abi.Config.dt.offset, abi.Config.pair_capacity.offset, abi.Config.flags.offset,
        abi.Stats.kernel_launches.offset]
    assert scenes.RB_DTYPE.itemsize == C.sizeof(abi.RigidBodyDesc)


def test_create_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = engine.load()
    cfg = abi.make_config(n_particles=10, dt=1e-6, max_coordinate=(1, 1, 1))
    st = C.c_int32(0)
    ctx = lib.create(C.byref(cfg), C.byref(st))
    assert not ctx and st.value == abi.GB_E_NO_DEVICE


def test_component_manager_adapter_fails_cleanly_without_device():
    """ComponentManagerB200 (C++ adapter over the C ABI) turns the engine's
    status into an exception, which the drop-in driver reports as JSON."""
    import json
    import torch
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "oracle", "_ref", "adapter_drive")
    if torch.cuda.is_available() or not os.path.exists(exe):
        pytest.skip("needs the built driver and no GPU")
    out = subprocess.run([exe, "1"], capture_output=True, text=True, timeout=120)
    assert out.returncode == 2
    assert "no usable CUDA device" in json.loads(out.stdout.strip())["error"]


def test_invalid_config_is_rejected():
    lib = engine.load()
    st = C.c_int32(0)
    cfg = abi.make_config(n_particles=10, dt=-1.0)
    assert not lib.create(C.byref(cfg), C.byref(st)) and st.value == abi.GB_E_INVALID_ARG
    cfg = abi.make_config(n_particles=10, dt=1e-6, precision=7)
    assert not lib.create(C.byref(cfg), C.byref(st)) and st.value == abi.GB_E_INVALID_ARG


def cube_vertices(h):
    return np.array([[sx * h[0], sy * h[1], sz * h[2]] for sx in (-1, 1) for sy in (-1, 1)
                     for sz in (-1, 1)])


def test_polyhedron_cube_equals_box(oracle):
    """A box given as the polyhedron of its 8 corners has the Box's support
    points and mass properties: the polyhedron's anchor to the reference's
    Box::support (Box.cpp:129-134) and Box::computeInertia (Box.cpp:88-107)."""
    lib = engine.load()
    rng = np.random.default_rng(3)
    for _ in range(20):
        h = rng.uniform(0.4e-3, 1.5e-3, 3)
        verts = np.ascontiguousarray(cube_vertices(h))
        poly = abi.rigid_body(abi.GB_POLYHEDRON, [], crust=5e-5, density=2500, n_vertices=8)
        box = abi.rigid_body(abi.GB_BOX, list(h), crust=5e-5, density=2500)
        for _ in range(20):
            d = rng.normal(size=3)
            a, b = np.zeros(3), np.zeros(3)
            oracle.support(C.byref(poly.convex), abi.dptr(verts), abi.dptr(d), abi.dptr(a))
            oracle.support(C.byref(box.convex), None, abi.dptr(d), abi.dptr(b))
            assert np.array_equal(a, b)
        pe, po, pb = abi.RigidBodyProps(), abi.RigidBodyProps(), abi.RigidBodyProps()
        assert lib.rigid_body_properties(C.byref(poly), abi.dptr(verts), C.byref(pe)) == 0
        assert oracle.rigid_body_properties(C.byref(poly), abi.dptr(verts), C.byref(po)) == 0
        assert lib.rigid_body_properties(C.byref(box), None, C.byref(pb)) == 0
        scale = max(abs(x) for x in pb.inertia)
        for p in (pe, po):
            assert np.isclose(p.volume, pb.volume, rtol=1e-13)
            assert np.allclose(list(p.inertia), list(pb.inertia), rtol=1e-12, atol=1e-13 * scale)
            assert np.allclose(list(p.bounding_box), list(pb.bounding_box), rtol=1e-15)
            assert np.isclose(p.circumscribed_radius, pb.circumscribed_radius, rtol=1e-15)


def test_polyhedron_hull_engine_vs_oracle(oracle):
    """Mass properties of random ellipsoid hulls: the engine's incremental hull
    and the oracle's exhaustive plane search agree."""
    lib = engine.load()
    rng = np.random.default_rng(5)
    for _ in range(40):
        k = int(rng.integers(8, 33))
        pts = scenes.ellipsoid_points(rng, (1e-3, rng.uniform(0.6e-3, 1.4e-3),
                                            rng.uniform(0.6e-3, 1.4e-3)), k)
        c = np.zeros(3)
        vol = C.c_double(0)
        assert lib.convex_hull_centroid(abi.dptr(np.ascontiguousarray(pts)), k, abi.dptr(c),
                                        C.byref(vol)) == 0
        pts = np.ascontiguousarray(pts - c)
        rb = abi.rigid_body(abi.GB_POLYHEDRON, [], crust=5e-5, density=2500, n_vertices=k)
        a, b = abi.RigidBodyProps(), abi.RigidBodyProps()
        assert lib.rigid_body_properties(C.byref(rb), abi.dptr(pts), C.byref(a)) == 0
        assert oracle.rigid_body_properties(C.byref(rb), abi.dptr(pts), C.byref(b)) == 0
        assert np.isclose(a.volume, b.volume, rtol=1e-12)
        assert np.allclose(list(a.inertia), list(b.inertia), rtol=1e-10, atol=1e-22)
        assert np.allclose(list(a.inertia_inv), list(b.inertia_inv), rtol=1e-9)
        # centred on the hull centroid: first moments vanish, so the
        # inertia about the origin is the central inertia
        assert abs(vol.value - a.volume) <= 1e-12 * a.volume


def test_scene_generators_are_seeded():
    a, b = scenes.polydisperse_superquadrics(n=2000), scenes.polydisperse_superquadrics(n=2000)
    assert np.array_equal(a.transforms, b.transforms) and np.array_equal(a.rbs, b.rbs)
    c = scenes.polydisperse_superquadrics(n=2000, seed=5)
    assert not np.array_equal(a.transforms, c.transforms)
