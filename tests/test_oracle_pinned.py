"""The FP64 oracle pinned to the reference (CPU only).

1. Against the golden fixtures in tests/golden/, generated from the
   reference's own compiled CPU code by tests/golden/make_golden.py.
2. Directly against that compiled reference (oracle/_ref) when it is built.

The restatement follows the reference's operation order, so on one machine
the outputs are bit-identical; the only tolerance is for the superquadric
mass properties (the oracle uses tgamma where the reference host code uses
std::beta) and for values that pass through libm's pow/sin/cos when the
fixture was made on another CPU.
"""
import ctypes as C
import os

import numpy as np
import pytest

from grains3dgpu_b200 import abi, scenes

from conftest import rel_err

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))


def desc(row):
    return abi.rigid_body(int(row["type"]), list(row["p"]), crust=float(row["crust"]),
                          density=float(row["density"]))


def same(a, b, tol=0.0):
    a, b = np.asarray(a, float), np.asarray(b, float)
    if tol == 0.0:
        return np.array_equal(a, b, equal_nan=True)
    ok = np.isclose(a, b, rtol=tol, atol=0.0) | (np.isnan(a) & np.isnan(b))
    return bool(ok.all())


def test_support_and_properties_vs_golden(oracle):
    g = load("functions")
    for i in range(len(g["ka"])):
        A = desc(g["da"][i])
        o = np.zeros(3)
        oracle.support(C.byref(A.convex), None, abi.dptr(g["dirs"][i].copy()), abi.dptr(o))
        tol = 1e-15 if g["ka"][i] == abi.GB_SUPERQUADRIC else 0.0
        assert same(o, g["support"][i], tol), (i, o, g["support"][i])
        P = abi.RigidBodyProps()
        assert oracle.rigid_body_properties(C.byref(A), None, C.byref(P)) == 0
        props = [P.volume, P.mass, P.circumscribed_radius, *P.bounding_box, *P.inertia,
                 *P.inertia_inv]
        assert same(props, g["props"][i], 1e-13)


def test_gjk_closest_points_obb_vs_golden(oracle):
    g = load("functions")
    for i in range(len(g["ka"])):
        A, B = desc(g["da"][i]), desc(g["db"][i])
        ta, tb = g["ta"][i].copy(), g["tb"][i].copy()
        x, y = np.zeros(3), np.zeros(3)
        it = C.c_int32(0)
        d = oracle.gjk(abi.GB_GJK_JH, C.byref(A.convex), None, C.byref(B.convex), None,
                       abi.dptr(ta), abi.dptr(tb), abi.dptr(x), abi.dptr(y), C.byref(it))
        assert same([d, *x, *y], g["gjk"][i][:7], 1e-12)
        assert it.value == int(g["gjk"][i][7])
        ci = abi.Contact()
        oracle.closest_points(C.byref(A), None, C.byref(B), None, abi.dptr(ta), abi.dptr(tb),
                              abi.GB_GJK_JH, C.byref(ci))
        assert same([*ci.pt, *ci.vec, ci.overlap], g["closest"][i], 1e-12)
        ext_a = g["props"][i][3:6].copy()
        ext_b = g["pb"][i].copy()
        assert oracle.obb(abi.dptr(ext_a), abi.dptr(ext_b), abi.dptr(ta), abi.dptr(tb)) \
            == g["obb"][i]


def test_hooke_vs_golden(oracle):
    g = load("hooke")
    for row, out in zip(g["inputs"], g["outputs"]):
        kn, en, etat, muc, kr = row[:5]
        cm = abi.ContactModel(kn=kn, en=en, etat=etat, muc=muc, kr=kr, kt=0.0)
        ci = abi.Contact()
        ci.pt[:] = list(row[5:8])
        ci.vec[:] = list(row[8:11])
        ci.overlap = row[11]
        rv, rw = row[12:15].copy(), row[15:18].copy()
        m1, m2 = row[18], row[19]
        org = row[20:23].copy()
        f, t = row[23:26].copy(), row[26:29].copy()
        oracle.hooke(C.byref(cm), C.byref(ci), abi.dptr(rv), abi.dptr(rw), m1, m2,
                     abi.dptr(org), abi.dptr(f), abi.dptr(t))
        assert same([*f, *t], out, 1e-14)


@pytest.mark.parametrize("name,shape", [("superquadric", "superquadric"), ("sphere", "sphere")])
def test_system_vs_golden(oracle, name, shape):
    g = load("system_" + name)
    scene = scenes.superquadric_column(n=400, pitch=2.05e-3, box=(0.012, 0.012, 0.036), shape=shape)
    s = scenes.System(oracle, scene)
    p = abi.RigidBodyProps()
    v = g["props"][0]
    p.volume, p.mass, p.circumscribed_radius = v[0], v[1], v[2]
    p.bounding_box[:] = list(v[3:6])
    p.inertia[:] = list(v[6:12])
    p.inertia_inv[:] = list(v[12:18])
    oracle.set_rigid_body_props(s.ctx, 0, C.byref(p))
    s.detect()
    for k in ["GB_DUMP_CELL_HASH", "GB_DUMP_SORTED_IDS", "GB_DUMP_CELL_START",
              "GB_DUMP_CANDIDATE_PAIRS", "GB_DUMP_CONTACT_PAIRS"]:
        assert np.array_equal(s.dump(getattr(abi, k)), g[k]), k
    assert same(s.dump(abi.GB_DUMP_CONTACT_INFO), g["GB_DUMP_CONTACT_INFO"], 1e-12)
    assert same(s.torces(), g["torce_after_detect"], 1e-12)
    s.add_external_forces()
    s.move()
    s.step(int(g["steps"]) - 1)
    assert np.abs(s.transforms() - g["transforms"]).max() <= 1e-15
    assert rel_err(s.velocities(), g["velocities"]) <= 1e-11


# ---- direct comparison with the compiled reference ------------------------------
def _rot(rng):
    q = rng.normal(size=4)
    return scenes.quat_to_matrix((q / np.linalg.norm(q))[None])[0]


def test_functions_bit_exact_vs_reference(oracle, reference):
    rng = np.random.default_rng(7)
    for it in range(400):
        kind = [abi.GB_SUPERQUADRIC, abi.GB_BOX, abi.GB_SPHERE][it % 3]
        p = (list(rng.uniform(0.5e-3, 1.5e-3, 3)) + list(rng.uniform(2, 10, 2))
             if kind == abi.GB_SUPERQUADRIC else list(rng.uniform(0.5e-3, 1.5e-3, 3)))
        A = abi.rigid_body(kind, p, crust=5e-5, density=2500)
        B = abi.rigid_body(abi.GB_SUPERQUADRIC,
                           list(rng.uniform(0.5e-3, 1.5e-3, 3)) + list(rng.uniform(2, 10, 2)),
                           crust=5e-5, density=2500)
        ta, tb = np.zeros(12), np.zeros(12)
        ta[:9], tb[:9] = _rot(rng), _rot(rng)
        ta[9:] = rng.uniform(-1e-3, 1e-3, 3)
        tb[9:] = ta[9:] + rng.normal(size=3) * 1.6e-3
        outs = []
        for lib in (oracle, reference):
            o = np.zeros(3)
            lib.support(C.byref(A.convex), None, abi.dptr(rng.normal(size=3)), abi.dptr(o))
            ci = abi.Contact()
            lib.closest_points(C.byref(A), None, C.byref(B), None, abi.dptr(ta), abi.dptr(tb),
                               abi.GB_GJK_JH, C.byref(ci))
            outs.append([*ci.pt, *ci.vec, ci.overlap])
        assert same(outs[0], outs[1])


def test_system_bit_exact_vs_reference(oracle, reference):
    scene = scenes.superquadric_column(n=600, pitch=2.05e-3, box=(0.014, 0.014, 0.040))
    o = scenes.System(oracle, scene)
    r = scenes.System(reference, scene)
    p = r.rb_props(0)
    oracle.set_rigid_body_props(o.ctx, 0, C.byref(p))
    for _ in range(10):
        o.step(1)
        r.step(1)
    assert np.array_equal(o.transforms(), r.transforms())
    assert np.array_equal(o.velocities(), r.velocities())


def _random_pair(rng, offset=None):
    kind = [abi.GB_SUPERQUADRIC, abi.GB_BOX, abi.GB_SPHERE][int(rng.integers(3))]
    p = (list(rng.uniform(0.5e-3, 1.5e-3, 3)) + list(rng.uniform(2, 10, 2))
         if kind == abi.GB_SUPERQUADRIC else list(rng.uniform(0.5e-3, 1.5e-3, 3)))
    A = abi.rigid_body(kind, p, crust=5e-5, density=2500)
    B = abi.rigid_body(abi.GB_SUPERQUADRIC,
                       list(rng.uniform(0.5e-3, 1.5e-3, 3)) + list(rng.uniform(2, 10, 2)),
                       crust=5e-5, density=2500)
    ta, tb = np.zeros(12), np.zeros(12)
    ta[:9], tb[:9] = _rot(rng), _rot(rng)
    ta[9:] = rng.uniform(-1e-3, 1e-3, 3)
    if offset is None:
        tb[9:] = ta[9:] + rng.normal(size=3) * 1.6e-3
    else:
        u = rng.normal(size=3)
        tb[9:] = ta[9:] + offset * u / np.linalg.norm(u)
    return A, B, ta, tb


def _gjk(lib, variant, A, B, ta, tb):
    pa, pb, n = np.zeros(3), np.zeros(3), C.c_int(0)
    d = lib.gjk(variant, C.byref(A.convex), None, C.byref(B.convex), None, abi.dptr(ta),
                abi.dptr(tb), abi.dptr(pa), abi.dptr(pb), C.byref(n))
    return d, pa, pb, n.value


def test_signed_volume_gjk_bit_exact_vs_reference(oracle, reference):
    """GB_GJK_SV restates computeClosestPoints_GJK_AY (GJK_AY.cpp:392-469)."""
    rng = np.random.default_rng(21)
    for _ in range(400):
        A, B, ta, tb = _random_pair(rng)
        d0, pa0, pb0, n0 = _gjk(oracle, abi.GB_GJK_SV, A, B, ta, tb)
        d1, pa1, pb1, n1 = _gjk(reference, abi.GB_GJK_SV, A, B, ta, tb)
        assert same([d0, *pa0, *pb0], [d1, *pa1, *pb1]) and n0 == n1


def test_nesterov_gjk_converges_to_the_signed_volume_distance(oracle):
    """Nesterov-accelerated GJK (no reference counterpart) on separated pairs:
    the distance within the reference's relative tolerance (LOWEPS = 1e-5) of
    the signed-volume GJK's, and witness points that realise it."""
    rng = np.random.default_rng(22)
    checked = 0
    for _ in range(300):
        A, B, ta, tb = _random_pair(rng, offset=5e-3)
        ds, *_ = _gjk(oracle, abi.GB_GJK_SV, A, B, ta, tb)
        dn, pa, pb, n = _gjk(oracle, abi.GB_GJK_NESTEROV, A, B, ta, tb)
        if A.convex.type == abi.GB_SPHERE:
            # Sphere::support(0) = radius * normalized(0) is NaN (Sphere.cpp:111-114),
            # so every GJK of the reference starts from NaN with a sphere
            assert ds != ds and dn != dn
            continue
        checked += 1
        assert abs(dn - ds) <= 2e-5 * ds and 0 < n < 1000
        wa = ta[:9].reshape(3, 3) @ pa + ta[9:]
        wb = tb[:9].reshape(3, 3) @ pb + tb[9:]
        assert abs(np.linalg.norm(wa - wb) - dn) <= 1e-9 * dn + 1e-15
    assert checked > 150


def test_torce_accumulation_vs_reference(oracle, reference):
    """setTorce, two detects and gravity accumulate onto one torce, which the
    move consumes (ComponentManagerCPU: addForce onto m_torce, reset in
    moveParticles)."""
    scene = scenes.superquadric_column(n=400, pitch=2.05e-3, box=(0.012, 0.012, 0.036),
                                       shape="sphere")
    o = scenes.System(oracle, scene)
    r = scenes.System(reference, scene)
    oracle.set_rigid_body_props(o.ctx, 0, C.byref(r.rb_props(0)))
    t0 = np.random.default_rng(3).normal(size=(scene.n, 6)) * 1e-4
    for s in (o, r):
        s.set_torces(t0)
        s.detect()
        s.detect()
        s.add_external_forces()
    assert np.array_equal(o.torces(), r.torces())
    for s in (o, r):
        s.move()
    assert np.array_equal(o.torces(), r.torces()) and not o.torces().any()
    assert np.array_equal(o.transforms(), r.transforms())
    assert np.array_equal(o.velocities(), r.velocities())


def test_engine_host_properties_match_reference(reference):
    """The engine computes rigid-body properties on the host with the
    reference's formulas and std::beta: bit-identical."""
    from grains3dgpu_b200 import engine
    lib = engine.load()
    rng = np.random.default_rng(11)
    for it in range(300):
        kind = [abi.GB_SUPERQUADRIC, abi.GB_BOX, abi.GB_SPHERE, abi.GB_RECTANGLE][it % 4]
        p = (list(rng.uniform(0.5e-3, 1.5e-3, 3)) + list(rng.uniform(2, 10, 2))
             if kind == abi.GB_SUPERQUADRIC else list(rng.uniform(0.5e-3, 1.5e-3, 3)))
        rb = abi.rigid_body(kind, p, crust=5e-5, density=float(rng.choice([0.0, 2500.0])))
        a, b = abi.RigidBodyProps(), abi.RigidBodyProps()
        assert lib.rigid_body_properties(C.byref(rb), None, C.byref(a)) == 0
        assert reference.rigid_body_properties(C.byref(rb), None, C.byref(b)) == 0
        assert bytes(a) == bytes(b)
