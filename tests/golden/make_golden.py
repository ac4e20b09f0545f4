"""Generates the golden fixtures in this directory from the reference's own
CPU code (oracle/_ref/libgrainsref.so, built by oracle/Makefile from the
reference sources).  Run from the repository root after building:

    make -C oracle all && python tests/golden/make_golden.py

Every fixture is seeded, so a rerun reproduces the files.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from grains3dgpu_b200 import abi, scenes  # noqa: E402
import pyoracle  # noqa: E402


def rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    return scenes.quat_to_matrix(q[None])[0]


def transform(rng, spread):
    t = np.zeros(12)
    t[:9] = rotation(rng)
    t[9:] = rng.uniform(-spread, spread, 3)
    return t


def random_shape(rng, kind):
    if kind == abi.GB_SUPERQUADRIC:
        return list(rng.uniform(0.6e-3, 1.4e-3, 3)) + list(rng.uniform(2.0, 10.0, 2))
    if kind == abi.GB_BOX:
        return list(rng.uniform(0.5e-3, 1.2e-3, 3))
    if kind == abi.GB_SPHERE:
        return [rng.uniform(0.5e-3, 1.5e-3)]
    if kind == abi.GB_RECTANGLE:
        return list(rng.uniform(1e-3, 5e-3, 2))
    raise ValueError(kind)


def desc_array(kinds, params, crust, density):
    a = np.zeros(len(kinds), scenes.RB_DTYPE)
    for i, (k, p) in enumerate(zip(kinds, params)):
        a[i]["type"] = k
        a[i]["p"][:len(p)] = p
        a[i]["crust"] = crust[i]
        a[i]["density"] = density[i]
    return a


def as_desc(row):
    return abi.rigid_body(int(row["type"]), list(row["p"]), crust=float(row["crust"]),
                          density=float(row["density"]))


def functions(R, rng, count=600):
    kinds = [abi.GB_SUPERQUADRIC, abi.GB_BOX, abi.GB_SPHERE]
    ka = np.array([kinds[i % 3] for i in range(count)], np.int32)
    kb = np.full(count, abi.GB_SUPERQUADRIC, np.int32)
    pa = [random_shape(rng, k) for k in ka]
    pb = [random_shape(rng, k) for k in kb]
    da = desc_array(ka, pa, rng.uniform(2e-5, 8e-5, count), np.full(count, 2500.0))
    db = desc_array(kb, pb, rng.uniform(2e-5, 8e-5, count), np.full(count, 2500.0))
    dirs = rng.normal(size=(count, 3))
    dirs[::7, 0] = 0.0
    dirs[::11, :2] = 0.0
    ta = np.stack([transform(rng, 1e-3) for _ in range(count)])
    tb = np.stack([transform(rng, 1e-3) for _ in range(count)])
    tb[:, 9:] += rng.normal(size=(count, 3)) * 1.5e-3
    sup = np.zeros((count, 3))
    props = np.zeros((count, 18))
    gjk = np.zeros((count, 8))
    closest = np.zeros((count, 7))
    obb = np.zeros(count, np.int32)
    for i in range(count):
        A, B = as_desc(da[i]), as_desc(db[i])
        o = np.zeros(3)
        R.support(C.byref(A.convex), None, abi.dptr(dirs[i].copy()), abi.dptr(o))
        sup[i] = o
        P = abi.RigidBodyProps()
        R.rigid_body_properties(C.byref(A), None, C.byref(P))
        props[i] = [P.volume, P.mass, P.circumscribed_radius, *P.bounding_box, *P.inertia,
                    *P.inertia_inv]
        x, y = np.zeros(3), np.zeros(3)
        it = C.c_int32(0)
        d = R.gjk(abi.GB_GJK_JH, C.byref(A.convex), None, C.byref(B.convex), None,
                  abi.dptr(ta[i]), abi.dptr(tb[i]), abi.dptr(x), abi.dptr(y), C.byref(it))
        gjk[i] = [d, *x, *y, it.value]
        ci = abi.Contact()
        R.closest_points(C.byref(A), None, C.byref(B), None, abi.dptr(ta[i]), abi.dptr(tb[i]),
                         abi.GB_GJK_JH, C.byref(ci))
        closest[i] = [*ci.pt, *ci.vec, ci.overlap]
        obb[i] = R.obb(abi.dptr(props[i, 3:6].copy()), abi.dptr(np.array(pb[i][:3])),
                       abi.dptr(ta[i]), abi.dptr(tb[i]))
    np.savez_compressed(os.path.join(HERE, "functions.npz"), ka=ka, kb=kb, da=da, db=db,
                        dirs=dirs, ta=ta, tb=tb, support=sup, props=props, gjk=gjk,
                        closest=closest, obb=obb, pb=np.array([p[:3] for p in pb]))


def hooke_cases(R, rng, count=400):
    rows, outs = [], []
    for _ in range(count):
        kn, en, etat, muc = rng.uniform(1e3, 1e5), rng.uniform(0.3, 0.95), rng.uniform(0, 2), \
            rng.uniform(0.1, 0.9)
        kr = float(rng.choice([0.0, 1e-3]))
        pt = rng.normal(size=3) * 1e-3
        vec = rng.normal(size=3) * 1e-5
        rv, rw, org = rng.normal(size=3) * 0.1, rng.normal(size=3), rng.normal(size=3) * 1e-3
        m1, m2 = 1.6e-5, float(rng.choice([0.0, 2e-5]))
        f0, t0 = rng.normal(size=3), rng.normal(size=3)
        cm = abi.ContactModel(kn=kn, en=en, etat=etat, muc=muc, kr=kr, kt=0.0)
        ci = abi.Contact()
        ci.pt[:] = list(pt)
        ci.vec[:] = list(vec)
        ci.overlap = -float(np.linalg.norm(vec))
        f, t = f0.copy(), t0.copy()
        R.hooke(C.byref(cm), C.byref(ci), abi.dptr(rv), abi.dptr(rw), m1, m2, abi.dptr(org),
                abi.dptr(f), abi.dptr(t))
        rows.append([kn, en, etat, muc, kr, *pt, *vec, ci.overlap, *rv, *rw, m1, m2, *org,
                     *f0, *t0])
        outs.append([*f, *t])
    np.savez_compressed(os.path.join(HERE, "hooke.npz"), inputs=np.array(rows),
                        outputs=np.array(outs))


def system(R, name, scene, steps):
    s = scenes.System(R, scene)
    props = np.array([[p.volume, p.mass, p.circumscribed_radius, *p.bounding_box, *p.inertia,
                       *p.inertia_inv] for p in (s.rb_props(i)
                                                 for i in range(scene.config["n_rigid_bodies"]))])
    s.detect()
    out = {k: s.dump(getattr(abi, k)) for k in
           ["GB_DUMP_CELL_HASH", "GB_DUMP_SORTED_IDS", "GB_DUMP_CELL_START",
            "GB_DUMP_CANDIDATE_PAIRS", "GB_DUMP_CONTACT_PAIRS", "GB_DUMP_CONTACT_INFO"]}
    out["torce_after_detect"] = s.torces()
    s.add_external_forces()
    s.move()
    s.step(steps - 1)
    out["transforms"] = s.transforms()
    out["velocities"] = s.velocities()
    st = s.stats()
    np.savez_compressed(os.path.join(HERE, f"system_{name}.npz"), props=props, steps=steps,
                        cells_per_dir=np.array(list(st.cells_per_dir)),
                        cell_size=st.cell_size, **out)


def main():
    R = pyoracle.load_reference()
    rng = np.random.default_rng(20261203)
    functions(R, rng)
    hooke_cases(R, rng)
    system(R, "superquadric", scenes.superquadric_column(n=400, pitch=2.05e-3,
                                             box=(0.012, 0.012, 0.036)), 20)
    s = scenes.superquadric_column(n=400, pitch=2.05e-3, box=(0.012, 0.012, 0.036), shape="sphere")
    system(R, "sphere", s, 20)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
