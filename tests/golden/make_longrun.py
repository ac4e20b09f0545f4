"""Generates tests/golden/longrun_column.npz: ensemble statistics of the
2,000-superquadric column (a = b = c = 1 mm, n1 = n2 = 4, dt 2e-6 s) run for
100,000 steps (0.2 s) by the FP64 oracle (oracle/liboracle.so, the CPU restatement)
with the tangential-history law and the signed-volume GJK, sampled every
10,000 steps.  The lattice pitch is 2.7 mm (jitter +-0.03 mm) in a
20 x 20 x 120 mm box: at the configuration's 2.4 mm, randomly oriented
grains start with intersecting cores, and at mm scale GJK-JH's absolute
determinant threshold misses most contacts, so grains would pass through one
another; with disjoint bounding spheres at the start and the signed-volume
GJK the column falls and stacks into a bed.  Statistics:

  z        mean height of the grains
  ke_t     translational kinetic energy
  ke_r     rotational kinetic energy
  z_coord  coordination number (particle contacts per grain) of the last detect
  phi      packing fraction of the slab 0 < z < 12 mm
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

STEPS, EVERY = 100_000, 10_000
SLAB = ((0.0, 0.0, 0.0), (0.020, 0.020, 0.012))


def column():
    return scenes.superquadric_column(n=2000, pitch=2.7e-3, jitter=0.03e-3,
                                      box=(0.020, 0.020, 0.120))


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
