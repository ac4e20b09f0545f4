"""GPU parity of the laws that extend the reference: the Coulomb-capped
tangential-history contact law (GB_LAW_HOOKE_HISTORY) and the
velocity-Verlet integrator (GB_VELOCITY_VERLET), each against the FP64
oracle's restatement over a multi-step trajectory.

The history law carries per-pair state from step to step, so one wrong
history lookup shows up as a force error of order kt * xi; the bound below
(1e-7 of the largest velocity) is far under that.
"""
import numpy as np
import pytest

from grains3dgpu_b200 import abi, scenes

from conftest import rel_err
from test_gpu_parity import make_scene, pair

pytestmark = pytest.mark.gpu


def _run(g, o, steps):
    for _ in range(steps):
        for s in (g, o):
            s.detect()
            s.add_external_forces()
            s.move()


def _with_tangential(scene):
    # one law per material pair: keep the table's length, add tangential damping
    scene.contact_models = [dict(m, etat=0.3) for m in scene.contact_models]
    return scene


@pytest.mark.parametrize("kind", ["sphere", "polyhedron", "superquadric"])
def test_history_law_trajectory(gb, oracle, kind):
    scene = _with_tangential(make_scene(kind))
    g, o = pair(gb, oracle, scene, contact_law=abi.GB_LAW_HOOKE_HISTORY)
    _run(g, o, 3)
    g.step(12)
    o.step(12)
    assert np.array_equal(g.dump(abi.GB_DUMP_CONTACT_PAIRS), o.dump(abi.GB_DUMP_CONTACT_PAIRS))
    assert g.stats().contacts > 0
    assert np.abs(g.transforms() - o.transforms()).max() < 1e-12
    assert rel_err(g.velocities(), o.velocities()) < 1e-7


@pytest.mark.parametrize("kind", ["sphere", "superquadric"])
def test_velocity_verlet_trajectory(gb, oracle, kind):
    g, o = pair(gb, oracle, make_scene(kind), integrator=abi.GB_VELOCITY_VERLET)
    _run(g, o, 3)
    g.step(12)
    o.step(12)
    assert np.abs(g.transforms() - o.transforms()).max() < 1e-12
    assert rel_err(g.velocities(), o.velocities()) < 1e-7


def test_history_law_mixed_precision(gb):
    """Mixed mode with the history law, from one state: the FP64 mode's
    contact set, forces within 1e-5 of the largest."""
    scene = _with_tangential(make_scene("superquadric"))
    m = scenes.System(gb, scene, precision=abi.GB_MIXED, contact_law=abi.GB_LAW_HOOKE_HISTORY)
    f = scenes.System(gb, scene, precision=abi.GB_FP64, contact_law=abi.GB_LAW_HOOKE_HISTORY)
    m.detect()
    f.detect()
    assert np.array_equal(m.dump(abi.GB_DUMP_CONTACT_PAIRS), f.dump(abi.GB_DUMP_CONTACT_PAIRS))
    a, b = m.torces(), f.torces()
    assert np.abs(a[:, :3] - b[:, :3]).max() <= 1e-5 * np.abs(b[:, :3]).max()
