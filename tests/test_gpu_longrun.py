"""Long-run statistics.  The mixed mode against the FP64 mode: 10,000 and
100,000 superquadrics falling in a column onto a plate for 5,000 steps (10 ms), with
the tangential-history law.  Trajectories of individual grains separate
slowly (contact events amplify rounding), so the check is on the ensemble:
mean height, translational and rotational kinetic energy, and the number of
wall contacts of the step, sampled every 1,000 steps.

The Hooke law is not used here: its relative velocity takes the absolute
contact point as lever arm (Kinematics::kinematicsAtPoint as the reference
calls it), so the normal damping of a spinning grain acts on omega x x_world
and this column gains energy and blows apart after ~3,500 steps in every
precision mode alike.
"""
import os
import sys

import numpy as np
import pytest

from grains3dgpu_b200 import abi, scenes

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLDEN)


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


@pytest.mark.parametrize("n", [10_000, 100_000])
def test_mixed_statistics_follow_fp64(gb, n):
    scene = scenes.superquadric_column_on_plate(n=n)
    ref = _run(gb, scene, abi.GB_FP64)
    mix = _run(gb, scene, abi.GB_MIXED)
    assert max(r["walls"] for r in ref) > 0  # the column does reach the plate
    for a, b in zip(ref, mix):
        assert abs(a["z"] - b["z"]) < 1e-6                      # m
        assert abs(a["v2"] - b["v2"]) <= 1e-3 * a["v2"]
        assert abs(a["w2"] - b["w2"]) <= 0.1 * a["w2"]
        assert abs(a["walls"] - b["walls"]) <= 0.1 * max(a["walls"], 100)


@pytest.mark.parametrize("precision", [abi.GB_FP64_STRICT, abi.GB_FP64, abi.GB_MIXED])
def test_statistics_follow_the_oracle(gb, precision):
    """2,000 superquadrics settling into a five-layer bed for 20,000 steps
    against the FP64 oracle's run of the same scene (tests/golden/
    longrun_column.npz, from tests/golden/make_longrun.py), sampled every
    2,000 steps.

    Up to 6,000 steps every statistic agrees within 1 %: mean height,
    translational and rotational kinetic energy, coordination number, the
    packing fraction of the bed's interior, and the wall contacts within one.
    Past ~8,000 steps the grains' trajectories have separated (each contact
    amplifies last-bit differences; FP64-strict, which repeats the oracle's
    operation order, separates as fast as the others because the
    superquadric support's pow differs from the host's in the last bit), so
    the later samples are compared as an ensemble: mean height and packing
    fraction still within 1 % at every sample; kinetic energies, the
    coordination number and the wall contacts averaged over the last five
    samples within 10 %, 10 % and 15 % (about 140 particle contacts and 65
    wall contacts per sample: a few percent of counting noise per sample)."""
    import make_longrun as ml
    want = dict(np.load(os.path.join(GOLDEN, "longrun_column.npz")))
    got = ml.run(gb, precision=precision)
    early = slice(0, 3)
    for k in ("z", "ke_t", "ke_r", "z_coord", "phi"):
        a, b = got[k][early], want[k][early]
        assert np.all(np.abs(a - b) <= 0.01 * np.abs(want[k]).max()), (k, a, b)
    assert np.all(np.abs(got["walls"][early] - want["walls"][early]) <= 1), got["walls"]
    for k in ("z", "phi"):
        assert np.all(np.abs(got[k] - want[k]) <= 0.01 * np.abs(want[k])), (k, got[k], want[k])
    late = slice(5, None)
    for k, tol in (("ke_t", 0.10), ("ke_r", 0.10), ("z_coord", 0.10), ("walls", 0.15)):
        a, b = got[k][late].mean(), want[k][late].mean()
        assert abs(a - b) <= tol * b, (k, a, b)
