"""Loader of the in-tree CUDA engine (libgrains_b200.so).

The engine is the only compute path: there is no CPU fallback.  If the
library is missing or cannot be loaded, :func:`load` raises.
"""
import ctypes as C
import os
import subprocess

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgrains_b200.so")
CSRC = os.path.join(HERE, "csrc")

_lib = None


def build(jobs=8):
    """Compiles the sm_100a kernels and the C ABI into libgrains_b200.so."""
    subprocess.run(["make", "-s", f"-j{jobs}", "-C", CSRC], check=True)


def load():
    """Returns the bound ``gb_`` functions of the engine library."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is not built; run grains3dgpu_b200.engine.build() "
                "(needs nvcc) -- the engine has no CPU fallback")
        lib = C.CDLL(LIB_PATH)
        _lib = abi.Bound(lib, "gb_", [abi.SYSTEM_API, abi.ENGINE_API])
    return _lib


def status_string(st):
    return load().status_string(st).decode()


def declared_symbols(header=None):
    """Names of every function declared in include/grains_b200.h."""
    import re
    header = header or os.path.join(HERE, "..", "include", "grains_b200.h")
    text = open(header).read()
    return sorted(set(re.findall(r"\b(gb_[a-z0-9_]+)\s*\(", text)))
