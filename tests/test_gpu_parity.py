"""GPU parity: the CUDA engine through the C ABI against the FP64 oracle.

Integer outputs (cell hashes, sort order, cell starts, candidate and contact
pair sets) must be bit-identical.  In GB_FP64_STRICT the engine evaluates the
reference's operation order with IEEE intrinsics, so contact information and
torces are bit-identical for shapes whose support needs no transcendental
function (boxes, spheres, polyhedra) and agree to 1e-9 relative for
superquadrics (CUDA's pow and the host libm's differ in the last ulp).
"""
import numpy as np
import pytest

from grains3dgpu_b200 import abi, engine, metrics, scenes

from conftest import rel_err, share_props

pytestmark = pytest.mark.gpu

BROAD_DUMPS = [abi.GB_DUMP_CELL_HASH, abi.GB_DUMP_SORTED_IDS, abi.GB_DUMP_CELL_START,
               abi.GB_DUMP_NEIGHBORS, abi.GB_DUMP_CANDIDATE_PAIRS]


def hull_centroid(v):
    c = np.zeros(3)
    vol = abi.C.c_double(0)
    st = engine.load().convex_hull_centroid(abi.dptr(np.ascontiguousarray(v)), v.shape[0],
                                           abi.dptr(c), abi.C.byref(vol))
    assert st == 0
    return c


def make_scene(kind):
    if kind == "superquadric":
        return scenes.superquadric_column(n=1500, pitch=2.05e-3)
    if kind == "sphere":
        return scenes.superquadric_column(n=1500, pitch=2.05e-3, shape="sphere")
    if kind == "box-on-walls":
        # boxes touch each other only through the walls in the reference: its
        # OBB pre-filter is the exact box, so box-box pairs never reach a contact
        s = scenes.superquadric_column(n=1500, pitch=2.05e-3, shape="box", tilt=0.3)
        s.transforms[:, 9:] -= 1.6e-3 - 0.79e-3
        return s
    if kind == "polyhedron":
        return scenes.polyhedra_box(n=1200, box=(0.030, 0.030, 0.030), pitch=1.9e-3,
                              hull_centroid=hull_centroid)
    raise ValueError(kind)


def pair(gb, oracle, scene, precision=abi.GB_FP64_STRICT, **kw):
    g = scenes.System(gb, scene, precision=precision,
                      flags=abi.GB_FLAG_RECORD_CONTACT_INFO, **kw)
    o = scenes.System(oracle, scene, **kw)
    share_props(g, o, oracle)
    return g, o


@pytest.mark.parametrize("kind", ["superquadric", "sphere", "box-on-walls", "polyhedron"])
def test_broad_phase_and_pairs_bit_exact(gb, oracle, kind):
    scene = make_scene(kind)
    g, o = pair(gb, oracle, scene)
    g.detect()
    o.detect()
    for kind_ in BROAD_DUMPS + [abi.GB_DUMP_CONTACT_PAIRS]:
        a, b = g.dump(kind_), o.dump(kind_)
        assert a.shape == b.shape and np.array_equal(a, b), f"dump {kind_} differs"
    assert g.stats().contacts == o.stats().contacts
    assert g.stats().obstacle_contacts == o.stats().obstacle_contacts
    assert g.stats().contacts + g.stats().obstacle_contacts > 0


@pytest.mark.parametrize("precision", [abi.GB_FP64_STRICT, abi.GB_MIXED])
def test_broad_phase_and_pairs_bit_exact_large(gb, oracle, precision):
    """The benchmark packing, 1,000,000 polydisperse superquadrics: ~500 tiles
    in each one-pass scan, so the look-back across tiles is exercised; cell
    hashes, sorted ids, cell starts, neighbour counts, candidate and contact
    pairs equal the oracle's, and so do the mixed mode's (its FP32 pre-test
    is certified)."""
    scene = scenes.polydisperse_superquadrics(n=1_000_000)
    g = scenes.System(gb, scene, precision=precision, flags=abi.GB_FLAG_RECORD_CONTACT_INFO)
    o = scenes.System(oracle, scene)
    share_props(g, o, oracle)
    g.detect()
    o.detect()
    for kind_ in BROAD_DUMPS + [abi.GB_DUMP_CONTACT_PAIRS]:
        a, b = g.dump(kind_), o.dump(kind_)
        assert a.shape == b.shape and np.array_equal(a, b), f"dump {kind_} differs"
    assert g.dump(abi.GB_DUMP_CANDIDATE_PAIRS).shape[0] > 1000
    assert g.stats().contacts == o.stats().contacts
    g.close()
    o.close()


def test_broad_phase_and_pairs_bit_exact_polyhedra_200k(gb, oracle):
    """The polyhedra configuration at its full size: 200,000 convex hulls of
    8-32 points on ellipsoids, seeded on the 2.6 mm jittered lattice of a
    100 x 100 x 400 mm box.  Cell hashes, sorted ids, cell starts, neighbour
    table, candidate pairs and contact pairs equal the oracle's (FP64 strict),
    and the mixed mode's candidate and contact pairs equal them too."""
    scene = scenes.polyhedra_box(n=200_000, hull_centroid=hull_centroid)
    systems = [scenes.System(gb, scene, precision=p) for p in (abi.GB_FP64_STRICT, abi.GB_MIXED)]
    o = scenes.System(oracle, scene)
    share_props(systems[0], o, oracle)  # the same hull volumes and radii
    o.detect()
    want = {k: o.dump(k) for k in BROAD_DUMPS + [abi.GB_DUMP_CONTACT_PAIRS]}
    assert want[abi.GB_DUMP_CANDIDATE_PAIRS].shape[0] > 100_000
    for g in systems:
        g.detect()
        for kind_, b in want.items():
            a = g.dump(kind_)
            assert a.shape == b.shape and np.array_equal(a, b), f"dump {kind_} differs"
        g.close()
    o.close()


@pytest.mark.parametrize("workload,knob", [("bed", None), ("dilute", "1"), ("bed", "0")])
def test_fine_grid_pairs_bit_exact(gb, oracle, monkeypatch, workload, knob):
    """Candidates of a polydisperse packing on the finer grid (cell twice the
    95th-percentile bounding radius; the largest 5 % of grains by warp): the
    dense bed of the headline workload (200,000 of its grains on the 2.2 mm
    lattice) takes it by itself, the dilute packing when forced, and the bed
    can be held to the linked cells alone.  Either way the cell starts,
    candidate and contact pairs equal the oracle's, in both FP64-strict and
    mixed precision."""
    if knob is not None:
        monkeypatch.setenv("GB_DEBUG_FINE_GRID", knob)
    # the bed on its 2.2 mm lattice; the dilute packing at the 1,000,000-grain
    # workload's spacing (a fifth of its box)
    kw = {"pitch": 2.2e-3} if workload == "bed" else {"box": (0.3, 0.3, 0.24)}
    scene = scenes.polydisperse_superquadrics(seed=5, n=200_000, **kw)
    systems = [scenes.System(gb, scene, precision=p) for p in (abi.GB_FP64_STRICT, abi.GB_MIXED)]
    o = scenes.System(oracle, scene)
    share_props(systems[0], o, oracle)
    o.detect()
    dumps = [abi.GB_DUMP_CELL_START, abi.GB_DUMP_CANDIDATE_PAIRS, abi.GB_DUMP_CONTACT_PAIRS]
    want = {k: o.dump(k) for k in dumps}
    assert want[abi.GB_DUMP_CANDIDATE_PAIRS].shape[0] > (100_000 if workload == "bed" else 100)
    for g in systems:
        g.detect()
        fine = g.stats().fine_grid_cells
        assert (fine > 0) == (knob != "0"), fine
        for kind_, b in want.items():
            a = g.dump(kind_)
            assert a.shape == b.shape and np.array_equal(a, b), f"dump {kind_} differs"
        g.close()
    o.close()


@pytest.mark.parametrize("kind", ["sphere", "box-on-walls", "polyhedron"])
def test_single_step_torce_bit_exact(gb, oracle, kind):
    scene = make_scene(kind)
    g, o = pair(gb, oracle, scene)
    g.detect()
    o.detect()
    assert np.array_equal(g.dump(abi.GB_DUMP_CONTACT_INFO), o.dump(abi.GB_DUMP_CONTACT_INFO),
                          equal_nan=True)
    assert np.array_equal(g.torces(), o.torces())


def test_single_step_torce_superquadric(gb, oracle):
    g, o = pair(gb, oracle, make_scene("superquadric"))
    g.detect()
    o.detect()
    assert np.array_equal(g.dump(abi.GB_DUMP_CONTACT_PAIRS), o.dump(abi.GB_DUMP_CONTACT_PAIRS))
    assert rel_err(g.dump(abi.GB_DUMP_CONTACT_INFO), o.dump(abi.GB_DUMP_CONTACT_INFO)) < 1e-9
    assert rel_err(g.torces(), o.torces()) < 1e-9


@pytest.mark.parametrize("precision", [abi.GB_FP64_STRICT, abi.GB_FP64])
def test_trajectory_fp64(gb, oracle, precision):
    g, o = pair(gb, oracle, make_scene("superquadric"), precision=precision)
    for _ in range(3):
        for s in (g, o):
            s.detect()
            s.add_external_forces()
            s.move()
    g.step(10)
    o.step(10)
    assert np.abs(g.transforms() - o.transforms()).max() < 1e-12
    assert rel_err(g.velocities(), o.velocities()) < 1e-7


def crowded_cell_scene():
    """One 5 mm sphere sets a 10 mm cell; 600 spheres of 0.13 mm radius on a
    0.25 mm lattice all sit in the first cell, more than the counting sort's
    rank pass takes, so the engine falls back to its radix sort."""
    rng = np.random.default_rng(5)
    n_small = 600
    rbs = np.zeros(2, scenes.RB_DTYPE)
    for k, r in enumerate((0.13e-3, 5e-3)):
        rbs[k]["type"] = abi.GB_SPHERE
        rbs[k]["p"][0] = r
        rbs[k]["crust"] = 0.05 * r
        rbs[k]["density"] = 2500.0
    ix = np.arange(n_small)
    pos = np.stack([1e-3 + (ix % 10) * 0.25e-3, 1e-3 + (ix // 10 % 10) * 0.25e-3,
                    1e-3 + (ix // 100) * 0.25e-3], 1)
    pos += rng.uniform(-2e-5, 2e-5, pos.shape)
    pos = np.concatenate([pos, [[0.02, 0.02, 0.02]]])
    n = n_small + 1
    tr = np.zeros((n, 12))
    tr[:, :9] = scenes.random_rotations(rng, n)
    tr[:, 9:] = pos
    box = (0.04, 0.04, 0.04)
    walls, wtr = scenes.box_walls(box)
    cfg = dict(n_particles=n, n_rigid_bodies=2, n_obstacles=6, n_materials=2, origin=(0, 0, 0),
               max_coordinate=box, dt=1e-6, gravity=(0, 0, -9.81))
    ids = np.zeros(n, np.uint32)
    ids[-1] = 1
    return scenes.Scene("crowded-cell", cfg, rbs, np.zeros((0, 3)), ids, tr, np.zeros((n, 6)),
                        walls, wtr, [scenes.law()] * 3)


@pytest.mark.parametrize("precision", [abi.GB_FP64_STRICT, abi.GB_MIXED])
def test_crowded_cell_falls_back_to_radix_sort(gb, oracle, precision):
    scene = crowded_cell_scene()
    g, o = pair(gb, oracle, scene, precision=precision)
    for s in (g, o):
        s.detect()
    assert np.diff(o.dump(abi.GB_DUMP_CELL_START)).max() > 512
    for kind_ in BROAD_DUMPS + [abi.GB_DUMP_CONTACT_PAIRS]:
        assert np.array_equal(g.dump(kind_), o.dump(kind_)), f"dump {kind_} differs"
    assert g.stats().contacts == o.stats().contacts > 0
    g.step(3)
    o.step(3)
    assert np.abs(g.transforms()[:, 9:] - o.transforms()[:, 9:]).max() < 1e-9


@pytest.mark.parametrize("law", [abi.GB_LAW_HOOKE, abi.GB_LAW_HOOKE_HISTORY])
def test_pair_capacity_overflow_is_replayed(gb, law):
    """A pair capacity far too small makes steps abort on the device; the
    engine grows it and replays them.  The trajectory (and, with the history
    law, the tangential springs carried across the regrowth) equals the one
    of a context that never overflowed."""
    scene = make_scene("sphere")
    scene.contact_models = [dict(m, etat=0.3) for m in scene.contact_models]
    small = scenes.System(gb, scene, precision=abi.GB_FP64_STRICT, contact_law=law,
                          pair_capacity=64)
    large = scenes.System(gb, scene, precision=abi.GB_FP64_STRICT, contact_law=law)
    for s in (small, large):
        s.step(2)
        s.detect()
        s.add_external_forces()
        s.move()
        s.step(6)
    assert small.stats().candidate_pairs > 64
    assert np.array_equal(small.transforms(), large.transforms())
    assert np.array_equal(small.velocities(), large.velocities())


@pytest.mark.parametrize("precision", [abi.GB_FP64_STRICT, abi.GB_MIXED])
def test_torce_accumulation(gb, oracle, precision):
    """set_torces, two detects and gravity add onto one torce; the move (and
    a fused step after separate calls) consumes and resets it."""
    scene = make_scene("sphere")
    g, o = pair(gb, oracle, scene, precision=precision)
    t0 = np.random.default_rng(3).normal(size=(scene.n, 6)) * 1e-4
    for s in (g, o):
        s.set_torces(t0)
        s.detect()
        s.detect()
        s.add_external_forces()
    if precision == abi.GB_FP64_STRICT:
        assert np.array_equal(g.torces(), o.torces())
    else:
        assert np.abs(g.torces() - o.torces()).max() <= 1e-5 * np.abs(o.torces()).max()
    for s in (g, o):
        s.set_torces(t0)
        s.step(2)
    assert not g.torces().any()
    d = np.abs(g.transforms() - o.transforms())
    if precision == abi.GB_FP64_STRICT:
        assert d.max() < 1e-12
        assert rel_err(g.velocities(), o.velocities()) < 1e-12
    else:
        # FP32 angular velocity and torques: basis entries to ~1e-7, FP64 centres
        assert d[:, 9:].max() < 1e-9 and d[:, :9].max() < 1e-6
        assert rel_err(g.velocities(), o.velocities()) < 1e-4


def test_separate_calls_equal_fused_step(gb):
    scene = make_scene("superquadric")
    a = scenes.System(gb, scene, precision=abi.GB_FP64_STRICT)
    b = scenes.System(gb, scene, precision=abi.GB_FP64_STRICT)
    for _ in range(4):
        a.detect()
        a.add_external_forces()
        a.move()
    b.step(4)
    assert np.array_equal(a.transforms(), b.transforms())
    assert np.array_equal(a.velocities(), b.velocities())


def test_rerun_is_bitwise_deterministic(gb):
    scene = make_scene("polyhedron")
    out = []
    for _ in range(2):
        s = scenes.System(gb, scene, precision=abi.GB_FP64)
        s.step(5)
        out.append((s.transforms(), s.velocities()))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("kind", ["superquadric", "polyhedron", "box-on-walls"])
def test_mixed_precision_single_step(gb, kind):
    """Mixed mode (FP32 bulk, FP64 positions, compensated FP32 quaternion,
    FP64 GJK past the bounding tests) against the FP64 mode, both given the
    same FP64 pose: the same contact pairs, and per contact a force and a
    torque within 1e-5 relative of the FP64 mode's."""
    scene = make_scene(kind)
    m = scenes.System(gb, scene, precision=abi.GB_MIXED)
    f = scenes.System(gb, scene, precision=abi.GB_FP64)
    m.detect()
    f.detect()
    assert np.array_equal(m.dump(abi.GB_DUMP_CONTACT_PAIRS), f.dump(abi.GB_DUMP_CONTACT_PAIRS))
    if kind != "box-on-walls":  # boxes touch only the walls (the exact-box OBB test)
        e = metrics.contact_force_errors(m, f)
        assert e["matched"] == e["contacts_ref"] > 0
        assert e["force"]["max"] <= 1e-5 and e["torque"]["max"] <= 1e-5, e
    # and per particle, walls included
    e = metrics.particle_torce_errors(m, f)
    assert e["particles"] > 0
    assert e["force"] <= 1e-5 and e["torque"] <= 1e-5, e


def test_mixed_precision_single_step_dense_polydisperse(gb):
    """The polydisperse superquadrics of the 1,000,000-grain workload,
    200,000 of them packed on a 2.2 mm lattice (a dense bed), with the
    workload's tangential-history law: mixed against FP64 from the same FP64
    pose, per contact, within 1e-5 relative."""
    scene = scenes.polydisperse_superquadrics(seed=5, n=200_000, pitch=2.2e-3)
    law = abi.GB_LAW_HOOKE_HISTORY
    m = scenes.System(gb, scene, precision=abi.GB_MIXED, contact_law=law)
    f = scenes.System(gb, scene, precision=abi.GB_FP64, contact_law=law)
    m.detect()
    f.detect()
    e = metrics.contact_force_errors(m, f)
    assert e["contacts_ref"] > 1000
    assert e["matched"] == e["contacts_ref"] == e["contacts_run"], e
    assert e["force"]["max"] <= 1e-5 and e["torque"]["max"] <= 1e-5, e
