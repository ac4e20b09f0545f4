"""Failure detection on the GPU, with no GPU fault: every wait in the
engine's kernels is bounded and reports a status, and bad input is reported
by the host call.

* The one-pass scans wait for their predecessor tiles' sums (a decoupled
  look-back) for at most GB_DEBUG_SCAN_SPIN_LIMIT polls (2^20 by default).
  With the limit at 0 the wait runs out as soon as a predecessor is still
  working; the step then reports GB_E_CUDA, every later kernel of the step
  returns at entry (no kernel uses the stalled scan's offsets), the state is
  the one before the step, and a context made without the knob steps on.
* A non-finite particle state is reported as GB_E_NONFINITE and a centre
  outside the linked-cell grid as GB_E_OUT_OF_DOMAIN (host-injected).
"""
import numpy as np
import pytest

from grains3dgpu_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def test_scan_wait_that_runs_out_is_reported(gb, monkeypatch):
    scene = scenes.polydisperse_superquadrics(n=1_000_000)  # ~500 tiles per scan
    monkeypatch.setenv("GB_DEBUG_SCAN_SPIN_LIMIT", "0")
    s = scenes.System(gb, scene, precision=abi.GB_MIXED)
    monkeypatch.delenv("GB_DEBUG_SCAN_SPIN_LIMIT")
    tr0, kin0 = s.transforms(), s.velocities()
    statuses = [gb.step(s.ctx, 1) for _ in range(3)]
    assert abi.GB_E_CUDA in statuses, statuses
    assert all(st in (abi.GB_OK, abi.GB_E_CUDA) for st in statuses)
    if all(st == abi.GB_E_CUDA for st in statuses):
        assert np.array_equal(s.transforms(), tr0) and np.array_equal(s.velocities(), kin0)
    s.close()
    fresh = scenes.System(gb, scene, precision=abi.GB_MIXED)
    assert gb.step(fresh.ctx, 2) == abi.GB_OK
    assert np.isfinite(fresh.transforms()).all()
    fresh.close()


def test_nonfinite_state_is_reported(gb):
    scene = scenes.superquadric_column(n=1500, pitch=2.05e-3)
    for prec in (abi.GB_MIXED, abi.GB_FP64):
        s = scenes.System(gb, scene, precision=prec)
        tr = scene.transforms.copy()
        tr[17, 10] = np.nan
        s.set_transforms(tr)
        assert gb.detect_collision_and_compute_contact_forces(s.ctx, None) == abi.GB_E_NONFINITE
        kin = scene.velocities.copy()
        kin[3, 0] = np.inf
        s.set_transforms(scene.transforms)
        s.set_velocities(kin)
        assert gb.step(s.ctx, 1) == abi.GB_E_NONFINITE
        s.close()


def test_out_of_domain_is_reported(gb):
    scene = scenes.superquadric_column(n=1500, pitch=2.05e-3)
    s = scenes.System(gb, scene, precision=abi.GB_FP64)
    tr = scene.transforms.copy()
    tr[5, 9] = -0.5  # half a metre outside the box
    s.set_transforms(tr)
    assert gb.detect_collision_and_compute_contact_forces(s.ctx, None) == abi.GB_E_OUT_OF_DOMAIN
    assert gb.step(s.ctx, 1) == abi.GB_E_OUT_OF_DOMAIN
    s.set_transforms(scene.transforms)
    assert gb.step(s.ctx, 1) == abi.GB_OK
    s.close()
