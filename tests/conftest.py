import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    return pyoracle.load_oracle()


@pytest.fixture(scope="session")
def reference():
    import pyoracle
    if not pyoracle.reference_available():
        pytest.skip("compiled reference (oracle/_ref) not built here")
    return pyoracle.load_reference()


@pytest.fixture(scope="session")
def gb():
    """The CUDA engine; only for tests marked gpu."""
    import torch
    from grains3dgpu_b200 import engine
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected without a GPU")
    torch.cuda.init()
    return engine.load()


def share_props(src_sys, dst_sys, oracle_lib):
    """Copies the engine's rigid-body properties into an oracle system so both
    integrate with identical masses and inertias."""
    from grains3dgpu_b200 import abi
    for i in range(src_sys.cfg.n_rigid_bodies):
        p = src_sys.rb_props(i)
        oracle_lib.set_rigid_body_props(dst_sys.ctx, i, abi.C.byref(p))


def rel_err(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)
