"""Loaders for the CPU oracles (TEST INFRASTRUCTURE).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  ``load_oracle()`` binds liboracle.so (the FP64 C restatement,
prefix ``or_``); ``load_reference()`` binds _ref/libgrainsref.so (the
reference's own CPU path, prefix ``ref_``) when it has been built.
"""
import ctypes as C
import os
import subprocess

from grains3dgpu_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libgrainsref.so")


def build(reference=True):
    """Builds liboracle.so (and the reference library when its sources exist)."""
    target = "all" if reference else "oracle"
    subprocess.run(["make", "-s", "-j16", "-C", HERE, target], check=True)


def _bind(path, prefix):
    lib = C.CDLL(path)
    return abi.Bound(lib, prefix, [abi.SYSTEM_API, abi.FUNCTION_API,
                                   {"set_threads": (C.c_int, [C.c_void_p, C.c_int32]),
                                    "set_rigid_body_props": (C.c_int, [C.c_void_p, C.c_int32,
                                                                       C.POINTER(abi.RigidBodyProps)])}])


_cache = {}


def load_oracle():
    if "or" not in _cache:
        if not os.path.exists(ORACLE_SO):
            build(reference=False)
        _cache["or"] = _bind(ORACLE_SO, "or_")
    return _cache["or"]


def reference_available():
    return os.path.exists(REF_SO)


def load_reference():
    if "ref" not in _cache:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO + " is not built (needs the reference sources)")
        _cache["ref"] = _bind(REF_SO, "ref_")
    return _cache["ref"]
