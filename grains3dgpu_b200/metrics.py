"""Error and bulk statistics of DEM states, computed on the host from what the
C ABI returns.

* :func:`contact_force_errors` -- single-step error of one run against
  another from an identical state, per contact: for every particle-particle
  contact pair (A, B) found by both, |F_run - F_ref| / |F_ref| of the force
  that the pair puts on A, and the same for its torque.
* :func:`particle_torce_errors` -- the same per particle, on the torces
  accumulated over all of a particle's contacts (walls included).
* :func:`kinetic_energy`, :func:`coordination_number`,
  :func:`packing_fraction` -- the long-run statistics that compare chaotic
  trajectories: translational and rotational kinetic energy, mean number of
  particle-particle contacts per particle, and solid volume fraction of a
  region of the bed.
"""
import numpy as np

from . import abi


def _pair_keys(pairs):
    return pairs[:, 0].astype(np.uint64) << np.uint64(32) | pairs[:, 1].astype(np.uint64)


def contact_force_errors(run, ref):
    """Per-contact relative force and torque error of System `run` against
    System `ref`, both after a detect from the same state.

    Returns a dict: the contact counts of both, the number matched by pair,
    and for force and torque the max, 99th percentile and median of
    |x_run - x_ref| / |x_ref| over the matched contacts.  A contact whose
    reference force is exactly zero is compared against the largest force of
    the step instead (its relative error is undefined).  `force_scaled` and
    `torque_scaled` divide by max(|x_ref|, 1e-3 of the step's largest): a
    contact whose spring and damping nearly cancel (|F| a millionth of the
    typical) has a relative error set by the rounding of the cancelling
    terms, which this scale keeps from dominating the maximum."""
    pr, pf = run.dump(abi.GB_DUMP_CONTACT_PAIRS), ref.dump(abi.GB_DUMP_CONTACT_PAIRS)
    fr, ff = run.dump(abi.GB_DUMP_CONTACT_FORCES), ref.dump(abi.GB_DUMP_CONTACT_FORCES)
    kr, kf = _pair_keys(pr), _pair_keys(pf)
    common, ir, jf = np.intersect1d(kr, kf, assume_unique=True, return_indices=True)
    out = {"contacts_run": int(pr.shape[0]), "contacts_ref": int(pf.shape[0]),
           "matched": int(common.size)}
    for name, sl in (("force", slice(0, 3)), ("torque", slice(3, 6))):
        a, b = fr[ir, sl], ff[jf, sl]
        nb = np.linalg.norm(b, axis=1)
        floor = max(float(nb.max()) if nb.size else 0.0, 1e-300)
        d = np.linalg.norm(a - b, axis=1)
        for key, den in ((name, np.where(nb > 0, nb, floor)),
                         (name + "_scaled", np.maximum(nb, 1e-3 * floor))):
            e = d / den
            out[key] = ({"max": float(e.max()), "p99": float(np.percentile(e, 99)),
                         "median": float(np.median(e))} if e.size else
                        {"max": 0.0, "p99": 0.0, "median": 0.0})
    return out


def particle_torce_errors(run, ref):
    """Per-particle relative error of the accumulated torces (force and
    torque) of System `run` against System `ref`, over the particles whose
    reference force is non-zero: max of |x_run - x_ref| / |x_ref|."""
    a, b = run.torces(), ref.torces()
    out = {}
    for name, sl in (("force", slice(0, 3)), ("torque", slice(3, 6))):
        nb = np.linalg.norm(b[:, sl], axis=1)
        sel = nb > 0
        e = np.linalg.norm(a[sel, sl] - b[sel, sl], axis=1) / nb[sel]
        out[name] = float(e.max()) if e.size else 0.0
    out["particles"] = int((np.linalg.norm(b[:, :3], axis=1) > 0).sum())
    return out


def kinetic_energy(system):
    """Translational and rotational kinetic energy of all particles:
    sum m v^2 / 2 and sum w^T I w / 2, with I the world-frame inertia
    R I_body R^T from the rigid-body table."""
    kin = system.velocities()
    tr = system.transforms()
    ids = system.scene.rb_ids
    nrb = int(system.cfg.n_rigid_bodies)
    mass = np.empty(nrb)
    inert = np.empty((nrb, 6))
    for r in range(nrb):
        p = system.rb_props(r)
        mass[r] = p.mass
        inert[r] = list(p.inertia)
    m = mass[ids]
    ib = inert[ids]  # xx xy xz yy yz zz
    Ib = np.stack([ib[:, 0], ib[:, 1], ib[:, 2], ib[:, 1], ib[:, 3], ib[:, 4],
                   ib[:, 2], ib[:, 4], ib[:, 5]], 1).reshape(-1, 3, 3)
    R = tr[:, :9].reshape(-1, 3, 3)
    w = kin[:, 3:]
    wb = np.einsum("nji,nj->ni", R, w)  # body-frame angular velocity R^T w
    trans = 0.5 * float((m * (kin[:, :3] ** 2).sum(1)).sum())
    rot = 0.5 * float(np.einsum("ni,nij,nj->n", wb, Ib, wb).sum())
    return trans, rot


def coordination_number(system, select=None):
    """Mean number of particle-particle contacts per particle in the last
    detect (each contact counted once for each of its two particles), over
    the particles `select` (a boolean mask or index array; all by default)."""
    pairs = system.dump(abi.GB_DUMP_CONTACT_PAIRS)
    n = system.n
    z = np.bincount(pairs[:, 0].astype(np.int64), minlength=n)  # ordered pairs: once per side
    if select is None:
        return float(z.mean())
    return float(z[select].mean())


def particle_volumes(system):
    ids = system.scene.rb_ids
    vol = np.array([system.rb_props(r).volume for r in range(int(system.cfg.n_rigid_bodies))])
    return vol[ids]


def packing_fraction(system, lo, hi):
    """Solid volume fraction of the axis-aligned region [lo, hi]: the volume of
    the particles whose centres lie in it over the region's volume (a
    centre-count estimate, accurate when the region is many grains wide)."""
    x = system.transforms()[:, 9:]
    lo, hi = np.asarray(lo, float), np.asarray(hi, float)
    inside = np.all((x >= lo) & (x < hi), axis=1)
    return float(particle_volumes(system)[inside].sum() / np.prod(hi - lo))
