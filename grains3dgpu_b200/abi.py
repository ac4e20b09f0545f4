"""ctypes mirror of include/grains_b200.h.

The same function table is bound for the GPU engine (prefix ``gb_``) and,
in tests, for the CPU oracles (``or_``, ``ref_``), which export the same
signatures.  Nothing here loads a library by itself.
"""
import ctypes as C

import numpy as np

GB_OK = 0
GB_E_INVALID_ARG = -1
GB_E_CUDA = -2
GB_E_OUT_OF_MEMORY = -3
GB_E_NOT_READY = -4
GB_E_OUT_OF_DOMAIN = -5
GB_E_NONFINITE = -6
GB_E_NO_DEVICE = -7
GB_E_CAPACITY = -8
GB_E_UNSUPPORTED = -9

GB_SPHERE, GB_BOX, GB_CYLINDER, GB_CONE = 0, 1, 2, 3
GB_SUPERQUADRIC, GB_POLYHEDRON, GB_RECTANGLE, GB_DRUM = 4, 5, 6, 7
GB_MAX_POLY_VERTICES = 64

GB_FP64, GB_MIXED, GB_FP64_STRICT = 0, 1, 2
GB_FLAG_RECORD_CONTACT_INFO = 1
GB_FLAG_PHASE_TIMING = 2
GB_FLAG_CRUST_BOUNDS = 4
GB_RAW_COORDINATION_NUMBER = 1
PHASES = ["hash", "sort", "cell_start", "pair_count", "pair_fill", "narrow", "particle"]
GB_N_PHASES = len(PHASES)
GB_LAW_HOOKE, GB_LAW_HOOKE_HISTORY = 0, 1
GB_FIRST_ORDER_EXPLICIT, GB_VELOCITY_VERLET = 0, 1
GB_GJK_JH, GB_GJK_SV, GB_GJK_NESTEROV = 0, 1, 2

GB_DUMP_CELL_HASH = 0
GB_DUMP_SORTED_IDS = 1
GB_DUMP_CELL_START = 2
GB_DUMP_CANDIDATE_PAIRS = 3
GB_DUMP_CONTACT_PAIRS = 4
GB_DUMP_CONTACT_INFO = 5
GB_DUMP_NEIGHBORS = 6
GB_DUMP_CONTACT_FORCES = 7


class Convex(C.Structure):
    _fields_ = [("type", C.c_int32), ("n_vertices", C.c_int32),
                ("first_vertex", C.c_int64), ("p", C.c_double * 5)]


class RigidBodyDesc(C.Structure):
    _fields_ = [("convex", Convex), ("crust_thickness", C.c_double),
                ("density", C.c_double), ("material", C.c_int32),
                ("reserved", C.c_int32)]


class RigidBodyProps(C.Structure):
    _fields_ = [("volume", C.c_double), ("mass", C.c_double),
                ("circumscribed_radius", C.c_double),
                ("bounding_box", C.c_double * 3), ("inertia", C.c_double * 6),
                ("inertia_inv", C.c_double * 6)]


class ContactModel(C.Structure):
    _fields_ = [("kn", C.c_double), ("en", C.c_double), ("etat", C.c_double),
                ("muc", C.c_double), ("kr", C.c_double), ("kt", C.c_double)]


class Config(C.Structure):
    _fields_ = [("n_particles", C.c_int32), ("n_rigid_bodies", C.c_int32),
                ("n_obstacles", C.c_int32), ("n_materials", C.c_int32),
                ("origin", C.c_double * 3), ("max_coordinate", C.c_double * 3),
                ("cell_size_factor", C.c_double), ("pad_grid", C.c_int32),
                ("precision", C.c_int32), ("dt", C.c_double),
                ("gravity", C.c_double * 3), ("contact_law", C.c_int32),
                ("integrator", C.c_int32), ("gjk_variant", C.c_int32),
                ("device", C.c_int32), ("pair_capacity", C.c_int64),
                ("flags", C.c_int32), ("reserved", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("steps_done", C.c_int64), ("candidate_pairs", C.c_int64),
                ("contacts", C.c_int64), ("obstacle_contacts", C.c_int64),
                ("gjk_calls", C.c_int64), ("gjk_iterations", C.c_int64),
                ("status_flags", C.c_int32), ("n_cells", C.c_int32),
                ("cells_per_dir", C.c_int32 * 3), ("key_bits", C.c_int32),
                ("cell_size", C.c_double), ("grid_max", C.c_double * 3),
                ("kernel_launches", C.c_int64), ("gjk_fp64_calls", C.c_int64),
                ("fine_grid_cells", C.c_int64), ("obstacle_candidates", C.c_int64)]


class Contact(C.Structure):
    """or_contact of oracle/oracle.h (ContactInfo: point, vector, overlap)."""
    _fields_ = [("pt", C.c_double * 3), ("vec", C.c_double * 3),
                ("overlap", C.c_double)]


_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)
_U32 = C.POINTER(C.c_uint32)
_I64 = C.POINTER(C.c_int64)

# name -> (restype, argtypes) of the system API shared by gb_/or_/ref_
SYSTEM_API = {
    "create": (_P, [C.POINTER(Config), _I32]),
    "destroy": (C.c_int, [_P]),
    "set_rigid_bodies": (C.c_int, [_P, C.POINTER(RigidBodyDesc), _D, C.c_int64]),
    "get_rigid_body_props": (C.c_int, [_P, C.c_int32, C.POINTER(RigidBodyProps)]),
    "set_contact_models": (C.c_int, [_P, C.POINTER(ContactModel)]),
    "set_obstacles": (C.c_int, [_P, C.POINTER(RigidBodyDesc), _D]),
    "set_obstacle_velocities": (C.c_int, [_P, _D]),
    "set_rigid_body_ids": (C.c_int, [_P, _U32]),
    "set_transforms": (C.c_int, [_P, _D]),
    "set_velocities": (C.c_int, [_P, _D]),
    "get_transforms": (C.c_int, [_P, _D]),
    "get_velocities": (C.c_int, [_P, _D]),
    "get_torces": (C.c_int, [_P, _D]),
    "set_torces": (C.c_int, [_P, _D]),
    "adjoint_step": (C.c_int, [_P, _D, _D, _D]),
    "update_links": (C.c_int, [_P]),
    "detect_collision_and_compute_contact_forces": (C.c_int, [_P, _I32]),
    "add_external_forces": (C.c_int, [_P]),
    "move_particles": (C.c_int, [_P]),
    "step": (C.c_int, [_P, C.c_int32]),
    "get_stats": (C.c_int, [_P, C.POINTER(Stats)]),
    "debug_dump": (C.c_int, [_P, C.c_int32, _P, C.c_int64, _I64]),
}

# per-function entry points shared by or_/ref_ (known-answer tests)
FUNCTION_API = {
    "support": (C.c_int, [C.POINTER(Convex), _D, _D, _D]),
    "rigid_body_properties": (C.c_int, [C.POINTER(RigidBodyDesc), _D,
                                        C.POINTER(RigidBodyProps)]),
    "obb": (C.c_int, [_D, _D, _D, _D]),
    "gjk": (C.c_double, [C.c_int, C.POINTER(Convex), _D, C.POINTER(Convex), _D,
                         _D, _D, _D, _D, _I32]),
    "closest_points": (C.c_int, [C.POINTER(RigidBodyDesc), _D,
                                 C.POINTER(RigidBodyDesc), _D, _D, _D, C.c_int,
                                 C.POINTER(Contact)]),
    "hooke": (C.c_int, [C.POINTER(ContactModel), C.POINTER(Contact), _D, _D,
                        C.c_double, C.c_double, _D, _D, _D]),
    "linked_cell_dims": (C.c_int, [_D, _D, C.c_double, _U32]),
    "cell_hash": (C.c_int, [_D, _D, C.c_double, C.c_int64, _D, _U32]),
}

# entry points only the GPU engine exports
ENGINE_API = {
    "status_string": (C.c_char_p, [C.c_int]),
    "abi_version": (C.c_int, []),
    "rigid_body_properties": (C.c_int, [C.POINTER(RigidBodyDesc), _D,
                                        C.POINTER(RigidBodyProps)]),
    "convex_hull_centroid": (C.c_int, [_D, C.c_int32, _D, _D]),
    "device_pointer": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_void_p)]),
    "synchronize": (C.c_int, [_P]),
    "set_stream": (C.c_int, [_P, _P]),
    "get_phase_times": (C.c_int, [_P, _D, _I64, C.c_int32]),
    "rawdata_open": (C.c_int, [_P, C.c_char_p, C.c_char_p, C.c_int32, C.POINTER(C.c_void_p)]),
    "rawdata_write": (C.c_int, [C.c_void_p, C.c_double]),
    "rawdata_close": (C.c_int, [C.c_void_p]),
    "save_state": (C.c_int, [_P, C.c_void_p]),
    "load_state": (C.c_int, [_P, C.c_void_p]),
    "save_contacts": (C.c_int, [_P, C.c_void_p, C.c_int64, _I64]),
    "load_contacts": (C.c_int, [_P, C.c_void_p]),
    "set_integrator_phase": (C.c_int, [_P, C.c_int32]),
}


class Bound:
    """Functions of one library with a common prefix, callable without it."""

    def __init__(self, lib, prefix, tables):
        self.lib = lib
        self.prefix = prefix
        for table in tables:
            for name, (res, args) in table.items():
                fn = getattr(lib, prefix + name, None)
                if fn is None:
                    continue
                fn.restype = res
                fn.argtypes = args
                setattr(self, name, fn)


def dptr(a):
    """double* of a C-contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def u32ptr(a):
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(_U32)


def i32ptr(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_I32)


def make_config(**kw):
    cfg = Config()
    cfg.cell_size_factor = 1.0
    cfg.pad_grid = 1
    cfg.precision = GB_FP64
    cfg.contact_law = GB_LAW_HOOKE
    cfg.integrator = GB_FIRST_ORDER_EXPLICIT
    cfg.gjk_variant = GB_GJK_JH
    cfg.n_materials = 1
    cfg.n_rigid_bodies = 1
    for k, v in kw.items():
        if k in ("origin", "max_coordinate", "gravity"):
            getattr(cfg, k)[:] = list(v)
        else:
            setattr(cfg, k, v)
    return cfg


def rigid_body(convex_type, params, crust=0.0, density=0.0, material=0,
               n_vertices=0, first_vertex=0):
    rb = RigidBodyDesc()
    rb.convex.type = convex_type
    rb.convex.n_vertices = n_vertices
    rb.convex.first_vertex = first_vertex
    p = list(params) + [0.0] * (5 - len(params))
    rb.convex.p[:] = p
    rb.crust_thickness = crust
    rb.density = density
    rb.material = material
    return rb


def rigid_body_array(descs):
    arr = (RigidBodyDesc * max(1, len(descs)))()
    for i, d in enumerate(descs):
        arr[i] = d
    return arr


def contact_model_array(models):
    arr = (ContactModel * len(models))()
    for i, m in enumerate(models):
        for k, v in m.items():
            setattr(arr[i], k, v)
    return arr
