"""Generates tests/golden/longrun_column.npz: ensemble statistics of 2,000
superquadrics of the column configuration (a = b = c = 1 mm, n1 = n2 = 4,
density 2500, crust 5% of the semi-axis, dt 2e-6 s) settling into a bed, run
for 20,000 steps (40 ms) by the FP64 oracle (oracle/liboracle.so, the CPU
restatement) with the tangential-history law and the signed-volume GJK,
sampled every 2,000 steps.

The grains start on a 2.7 mm jittered lattice (+-0.03 mm) in a 60 x 60 x 30
mm box, five layers deep.  Three choices keep the run inside what the
reference's algorithms resolve: bounding spheres disjoint at the start (at
the configuration's 2.4 mm pitch randomly oriented grains start with
intersecting cores, which the closest-point solvers answer with a NaN
normal); drops of at most ~2.5 mm (impacts of ~0.2 m/s, whose overlap stays
well inside the crusts; the configuration's 60 mm column reaches ~1 m/s and
its bed goes non-finite); and the signed-volume GJK (GJK-JH's absolute
determinant threshold misses most contacts of mm grains, so they would pass
through one another).  Statistics:

  z        mean height of the grains
  ke_t     translational kinetic energy
  ke_r     rotational kinetic energy
  z_coord  coordination number (particle contacts per grain) of the last detect
  phi      packing fraction of the bed's interior, 3 mm from the side walls,
           0.5 < z < 4.5 mm
  walls    wall contacts

Run from the repository root:  python tests/golden/make_longrun.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from grains3dgpu_b200 import abi, metrics, scenes  # noqa: E402

STEPS, EVERY = 20_000, 2_000
SLAB = ((0.003, 0.003, 0.0005), (0.057, 0.057, 0.0045))


def column():
    return scenes.superquadric_column(n=2000, pitch=2.7e-3, jitter=0.03e-3,
                                      box=(0.060, 0.060, 0.030))


def sample(system):
    kt, kr = metrics.kinetic_energy(system)
    tr = system.transforms()
    return dict(z=float(tr[:, 11].mean()), ke_t=kt, ke_r=kr,
                z_coord=metrics.coordination_number(system),
                phi=metrics.packing_fraction(system, *SLAB),
                walls=float(system.stats().obstacle_contacts))


def run(lib, precision=None, threads=None):
    kw = {} if precision is None else {"precision": precision}
    s = scenes.System(lib, column(), contact_law=abi.GB_LAW_HOOKE_HISTORY,
                      gjk_variant=abi.GB_GJK_SV, **kw)
    if threads:
        lib.set_threads(s.ctx, threads)
    out = []
    for _ in range(STEPS // EVERY):
        assert s.step(EVERY) in (abi.GB_OK, abi.GB_E_OUT_OF_DOMAIN)
        out.append(sample(s))
    s.close()
    return {k: np.array([o[k] for o in out]) for k in out[0]}


if __name__ == "__main__":
    import pyoracle
    stats = run(pyoracle.load_oracle(), threads=os.cpu_count())
    for k, v in stats.items():
        print(k, v)
    np.savez(os.path.join(ROOT, "tests", "golden", "longrun_column.npz"), **stats)
