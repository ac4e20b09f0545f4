"""Long-run statistics of the mixed mode against the FP64 mode: 10,000
superquadrics falling in a column onto a plate for 5,000 steps (10 ms), with
the tangential-history law.  Trajectories of individual grains separate
slowly (contact events amplify rounding), so the check is on the ensemble:
mean height, translational and rotational kinetic energy, and the number of
wall contacts, sampled every 1,000 steps.

The Hooke law is not used here: its relative velocity takes the absolute
contact point as lever arm (Kinematics::kinematicsAtPoint as the reference
calls it), so the normal damping of a spinning grain acts on omega x x_world
and this column gains energy and blows apart after ~3,500 steps in every
precision mode alike.
"""
import numpy as np
import pytest

from grains3dgpu_b200 import abi, scenes

pytestmark = pytest.mark.gpu


def _run(gb, scene, precision, blocks=5, steps=1000):
    s = scenes.System(gb, scene, precision=precision, contact_law=abi.GB_LAW_HOOKE_HISTORY)
    out = []
    for _ in range(blocks):
        assert s.step(steps) in (abi.GB_OK, abi.GB_E_OUT_OF_DOMAIN)
        tr, kin = s.transforms(), s.velocities()
        assert np.isfinite(tr).all() and np.isfinite(kin).all()
        out.append(dict(z=tr[:, 11].mean(), v2=(kin[:, :3] ** 2).sum(),
                        w2=(kin[:, 3:] ** 2).sum(), walls=s.stats().obstacle_contacts))
    s.close()
    return out


def test_mixed_statistics_follow_fp64(gb):
    scene = scenes.superquadric_column_on_plate(n=10_000)
    ref = _run(gb, scene, abi.GB_FP64)
    mix = _run(gb, scene, abi.GB_MIXED)
    assert ref[-1]["walls"] > 1000  # the column does reach the walls
    for a, b in zip(ref, mix):
        assert abs(a["z"] - b["z"]) < 1e-6                      # m
        assert abs(a["v2"] - b["v2"]) <= 1e-3 * a["v2"]
        assert abs(a["w2"] - b["w2"]) <= 0.1 * a["w2"]
        assert abs(a["walls"] - b["walls"]) <= 0.03 * max(a["walls"], 100)
