"""The rotating drum on the GPU (GB_DRUM wall, end caps, surface velocity;
NEW features) against the FP64 oracle's restatement: a drum of radius 12 mm
turning at 300 rpm with a mix of spheres, cubes (polyhedra) and
superquadrics, the outer grains pressed on its wall.  FP64-strict: the
contact pairs equal and the trajectories within 1e-12 over 20 steps (the
superquadric supports differ from the host's pow in the last bits); mixed
against FP64: per particle torces within 1e-5."""
import numpy as np
import pytest

from grains3dgpu_b200 import abi, metrics, scenes

from conftest import rel_err, share_props

pytestmark = pytest.mark.gpu


def drum(rpm=300.0):
    return scenes.rotating_drum(n=300, radius=0.012, pitch=2.3e-3, margin=0.99e-3, rpm=rpm)


@pytest.mark.parametrize("flags", [0, abi.GB_FLAG_CRUST_BOUNDS])
@pytest.mark.parametrize("law", [abi.GB_LAW_HOOKE, abi.GB_LAW_HOOKE_HISTORY])
def test_drum_matches_oracle(gb, oracle, law, flags):
    sc = drum()
    g = scenes.System(gb, sc, precision=abi.GB_FP64_STRICT, contact_law=law, flags=flags)
    o = scenes.System(oracle, sc, contact_law=law, flags=flags)
    share_props(g, o, oracle)
    g.detect()
    o.detect()
    assert g.stats().obstacle_contacts == o.stats().obstacle_contacts > 3
    assert rel_err(g.torces(), o.torces()) < 1e-9
    g.add_external_forces()
    o.add_external_forces()
    g.move()
    o.move()
    g.step(19)
    o.step(19)
    assert np.abs(g.transforms() - o.transforms()).max() < 1e-12
    assert rel_err(g.velocities(), o.velocities()) < 1e-9


def test_drum_mixed_against_fp64(gb):
    sc = drum()
    law = abi.GB_LAW_HOOKE_HISTORY
    m = scenes.System(gb, sc, precision=abi.GB_MIXED, contact_law=law)
    f = scenes.System(gb, sc, precision=abi.GB_FP64, contact_law=law)
    m.detect()
    f.detect()
    assert m.stats().obstacle_contacts == f.stats().obstacle_contacts > 3
    e = metrics.particle_torce_errors(m, f)
    assert e["force"] <= 1e-5 and e["torque"] <= 1e-5, e


@pytest.mark.parametrize("shape", ["polyhedron", "box"])
def test_cube_collision_with_crust_bounds(gb, oracle, shape):
    """Two cubes meeting head on (scenes.cube_collision) under
    GB_FLAG_CRUST_BOUNDS with the signed-volume GJK, through the whole
    collision (600 steps): FP64-strict equals the oracle's trajectory to
    1e-12 m; FP64 and mixed stay finite and part at the oracle's speeds
    within 1e-3 (relative)."""
    sc = scenes.cube_collision(shape=shape, gap=0.2e-3, tilt=0.05)
    kw = dict(contact_law=abi.GB_LAW_HOOKE_HISTORY, gjk_variant=abi.GB_GJK_SV,
              flags=abi.GB_FLAG_CRUST_BOUNDS)
    o = scenes.System(oracle, sc, **kw)
    share_props(scenes.System(gb, sc, **kw), o, oracle)
    o.step(600)
    want_tr, want_kin = o.transforms(), o.velocities()
    assert np.isfinite(want_kin).all() and want_kin[0, 0] < 0.0 < want_kin[1, 0]
    for prec in (abi.GB_FP64_STRICT, abi.GB_FP64, abi.GB_MIXED):
        g = scenes.System(gb, sc, precision=prec, **kw)
        assert g.step(600) == abi.GB_OK
        tr, kin = g.transforms(), g.velocities()
        if prec == abi.GB_FP64_STRICT:
            assert np.abs(tr - want_tr).max() < 1e-12
            assert rel_err(kin, want_kin) < 1e-9
        else:
            assert np.isfinite(kin).all()
            assert rel_err(kin[:, :3], want_kin[:, :3]) < 1e-3, prec
        g.close()
