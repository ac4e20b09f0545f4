"""Obstacles past the 32 that the per-particle wall mask covers: their
candidates come from linked-cell bins built on the host when the obstacles
are set (the reference tests every particle against every obstacle,
ComponentManagerCPU.cpp:301-351).  A peg board (scenes.peg_board: 2,000
spheres among 64 fixed spherical pegs and the six box walls) against the
FP64 oracle: the same obstacle contacts and torces bit for bit in
FP64-strict, trajectories within 1e-12 m over 20 steps, the mixed mode per
contact within 1e-5 (of the larger of the contact's force and 1e-3 of the
step's largest), and far fewer candidate records than particles times
obstacles."""
import numpy as np
import pytest

from grains3dgpu_b200 import abi, metrics, scenes

from conftest import share_props

pytestmark = pytest.mark.gpu


def test_peg_board_matches_oracle(gb, oracle):
    sc = scenes.peg_board()
    n_obs = sc.obstacles.shape[0]
    assert n_obs > 32
    g = scenes.System(gb, sc, precision=abi.GB_FP64_STRICT)
    o = scenes.System(oracle, sc)
    share_props(g, o, oracle)
    g.detect()
    o.detect()
    st = g.stats()
    assert st.obstacle_contacts == o.stats().obstacle_contacts > 100
    assert st.contacts == o.stats().contacts
    assert np.array_equal(g.torces(), o.torces())
    assert 0 < st.obstacle_candidates < 0.1 * sc.n * n_obs
    g.add_external_forces()
    o.add_external_forces()
    g.move()
    o.move()
    g.step(19)
    o.step(19)
    assert np.abs(g.transforms() - o.transforms()).max() < 1e-12
    assert g.stats().obstacle_contacts == o.stats().obstacle_contacts


def test_peg_board_mixed_per_contact(gb):
    sc = scenes.peg_board()
    m = scenes.System(gb, sc, precision=abi.GB_MIXED)
    f = scenes.System(gb, sc, precision=abi.GB_FP64)
    m.detect()
    f.detect()
    assert m.stats().obstacle_contacts == f.stats().obstacle_contacts > 100
    # per contact (a sphere's torques are zero up to rounding, and a grain
    # squeezed between pegs sums large forces to a small one, so per-particle
    # relative errors say little here)
    e = metrics.contact_force_errors(m, f)
    assert e["matched"] == e["contacts_ref"] == e["contacts_run"], e
    assert e["force_scaled"]["max"] <= 1e-5 and e["force"]["p99"] <= 1e-5, e
