"""GPU parity of the two other GJK variants through the whole step:
GB_GJK_SV (the reference's computeClosestPoints_GJK_AY, GJK_AY.cpp:392-469;
the oracle's restatement is pinned to it bit for bit) and GB_GJK_NESTEROV
(Nesterov-accelerated GJK on the signed-volume sub-algorithm, no reference
counterpart; the oracle restates it), against the FP64 oracle.

FP64-strict results are bit-identical for shapes without transcendental
supports and within 1e-9 for superquadrics; the mixed mode keeps the FP64
mode's contact set.

The signed-volume GJK finds the many shallow contacts that the reference's
Johnson GJK misses, and -- like GJK_AY.cpp -- returns coincident witness
points when two cores intersect, so those contacts carry a NaN normal and NaN
forces (in the oracle as on the GPU).  The comparisons below therefore treat
NaN as a value (strict) or compare the finite rows (mixed against FP64).
"""
import numpy as np
import pytest

from grains3dgpu_b200 import abi, scenes

from conftest import rel_err
from test_gpu_parity import make_scene, pair

pytestmark = pytest.mark.gpu

VARIANTS = [abi.GB_GJK_SV, abi.GB_GJK_NESTEROV]


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("kind", ["polyhedron", "box-on-walls"])
def test_variant_single_step_bit_exact(gb, oracle, variant, kind):
    g, o = pair(gb, oracle, make_scene(kind), gjk_variant=variant)
    g.detect()
    o.detect()
    assert np.array_equal(g.dump(abi.GB_DUMP_CONTACT_PAIRS), o.dump(abi.GB_DUMP_CONTACT_PAIRS))
    assert g.stats().contacts + g.stats().obstacle_contacts > 0
    assert np.array_equal(g.dump(abi.GB_DUMP_CONTACT_INFO), o.dump(abi.GB_DUMP_CONTACT_INFO),
                          equal_nan=True)
    assert np.array_equal(g.torces(), o.torces(), equal_nan=True)


def _finite_rows(*arrays):
    return np.all([np.isfinite(a).all(1) for a in arrays], axis=0)


def _rows_within(a, b, tol):
    """Fraction of particles whose force (first 3 columns) agrees to `tol` of
    the largest force.  Nearly touching cores leave the contact normal to the
    rounding of coincident witness points, so a few ill-conditioned contacts
    differ by O(1) between two correct evaluations."""
    ok = _finite_rows(a, b)
    scale = np.abs(b[ok, :3]).max()
    err = np.abs(a[ok, :3] - b[ok, :3]).max(1)
    return ok.mean(), (err <= tol * scale).mean()


def shallow_superquadrics():
    """Superquadrics 2.62 mm apart (2 R_circ = 2.63 mm): contacts are mostly
    shallow, and cores rarely intersect."""
    return scenes.superquadric_column(n=1000, pitch=2.62e-3, jitter=0.02e-3)


@pytest.mark.parametrize("variant", VARIANTS)
def test_variant_superquadric_single_step(gb, oracle, variant):
    g, o = pair(gb, oracle, shallow_superquadrics(), gjk_variant=variant)
    g.detect()
    o.detect()
    assert np.array_equal(g.dump(abi.GB_DUMP_CONTACT_PAIRS), o.dump(abi.GB_DUMP_CONTACT_PAIRS))
    assert g.stats().contacts > 100
    # CUDA's pow and the host's differ in the last ulp; the GJK's relative
    # stopping tolerance (1e-5 of the core distance, itself ~ the crust) turns
    # that into force differences up to ~1e-5 of the largest force
    finite, close = _rows_within(g.torces(), o.torces(), 1e-4)
    assert finite > 0.98 and close > 0.98


@pytest.mark.parametrize("variant", VARIANTS)
def test_variant_mixed_precision_contact_set(gb, variant):
    scene = shallow_superquadrics()
    m = scenes.System(gb, scene, precision=abi.GB_MIXED, gjk_variant=variant)
    f = scenes.System(gb, scene, precision=abi.GB_FP64, gjk_variant=variant)
    m.detect()
    f.detect()
    assert np.array_equal(m.dump(abi.GB_DUMP_CONTACT_PAIRS), f.dump(abi.GB_DUMP_CONTACT_PAIRS))
    # the mixed mode's FP32 quaternion is a 6e-8 rotation away from the FP64
    # basis; nearly coincident witness points (cores almost touching) turn that
    # into O(1) changes of a few contact normals
    finite, close = _rows_within(m.torces(), f.torces(), 1e-4)
    assert finite > 0.98 and close > 0.9
