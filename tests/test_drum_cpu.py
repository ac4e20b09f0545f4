"""The drum wall (GB_DRUM, NEW) and moving walls in the FP64 oracle, on the
CPU: known answers of the wall contact, and the wall's surface velocity in
both contact laws."""
import numpy as np
import pytest

from grains3dgpu_b200 import abi, scenes


def drum_contact(oracle, radius, centre_offset, sphere_r=1e-3):
    """A sphere at `centre_offset` (drum frame) from the axis of a drum of
    radius `radius` whose frame is the identity (axis = world z)."""
    a = abi.rigid_body(abi.GB_SPHERE, [sphere_r], crust=5e-5, density=2500.0)
    b = abi.rigid_body(abi.GB_DRUM, [radius, 0.05])
    a2w = np.zeros(12)
    a2w[[0, 4, 8]] = 1.0
    a2w[9:] = centre_offset
    b2w = np.zeros(12)
    b2w[[0, 4, 8]] = 1.0
    ci = abi.Contact()
    st = oracle.closest_points(abi.C.byref(a), None, abi.C.byref(b), None, abi.dptr(a2w),
                               abi.dptr(b2w), abi.GB_GJK_JH, abi.C.byref(ci))
    assert st == 0
    return ci


def test_drum_wall_contact_known_answer(oracle):
    R, r = 0.01, 1e-3
    # centre 9.2 mm from the axis along (3, 4)/5: the sphere reaches 10.2 mm
    e = np.array([0.6, 0.8, 0.0])
    ci = drum_contact(oracle, R, 9.2e-3 * e + [0, 0, 0.004], r)
    assert ci.overlap == pytest.approx(-0.2e-3, rel=1e-12)
    pt = np.array(ci.pt)
    assert np.allclose(pt, 0.5 * (10.2e-3 + 10e-3) * e + [0, 0, 0.004], rtol=0, atol=1e-15)
    vec = np.array(ci.vec)  # from the wall into the sphere: inwards, |vec| = overlap
    assert np.allclose(vec, -0.2e-3 * e, rtol=0, atol=1e-15)
    # clear of the wall, and a centre on the axis: no contact
    assert drum_contact(oracle, R, 8.9e-3 * e).overlap == 0.0
    assert drum_contact(oracle, R, [0.0, 0.0, 0.001]).overlap == 0.0


@pytest.mark.parametrize("law", [abi.GB_LAW_HOOKE, abi.GB_LAW_HOOKE_HISTORY])
def test_wall_surface_velocity_enters_the_law(oracle, law):
    """Grains pressed on the wall of a drum at rest and of the same drum
    turning: the same contacts, different tangential forces; and a drum
    whose velocities are set to zero equals one never given velocities."""
    sc = scenes.rotating_drum(n=300, radius=0.012, pitch=2.3e-3, margin=0.99e-3, rpm=300.0)
    still = scenes.rotating_drum(n=300, radius=0.012, pitch=2.3e-3, margin=0.99e-3, rpm=0.0)
    bare = scenes.rotating_drum(n=300, radius=0.012, pitch=2.3e-3, margin=0.99e-3)
    bare.obstacle_velocities = None
    out = []
    for s in (sc, still, bare):
        sysm = scenes.System(oracle, s, contact_law=law)
        sysm.detect()
        out.append((sysm.torces(), sysm.stats().obstacle_contacts))
        sysm.close()
    assert out[0][1] == out[1][1] > 3
    assert np.array_equal(out[1][0], out[2][0])
    assert np.abs(out[0][0] - out[1][0]).max() > 1e-3 * np.abs(out[1][0]).max()


def run_cubes(oracle, flags, shape, steps=600):
    """The head-on cube collision (scenes.cube_collision) in the oracle with the
    signed-volume GJK: the first contact's overlap, the steps in contact, and
    the final velocities (NaN once the state is non-finite)."""
    sc = scenes.cube_collision(shape=shape, gap=0.2e-3, tilt=0.05)
    s = scenes.System(oracle, sc, flags=flags | abi.GB_FLAG_RECORD_CONTACT_INFO,
                      contact_law=abi.GB_LAW_HOOKE_HISTORY, gjk_variant=abi.GB_GJK_SV)
    first, in_contact = None, 0
    for k in range(steps):
        s.step(1)
        if s.stats().contacts:
            in_contact += 1
            if first is None:
                first = s.dump(abi.GB_DUMP_CONTACT_INFO)[0, 6]
        kin = s.velocities()
        if not np.isfinite(kin).all():
            break
    s.close()
    return first, in_contact, kin


@pytest.mark.parametrize("shape", ["polyhedron", "box"])
def test_cube_contact_needs_the_crust_in_the_bounding_tests(oracle, shape):
    """The reference's OBB pre-filter bounds a cube by the cube itself, while
    the contact starts once the cubes come within the crusts' sum: the pair
    first reaches GJK with the cubes intersecting (overlap = -crust sum), whose
    normal is 0/0, and the state turns non-finite.  With GB_FLAG_CRUST_BOUNDS
    the contact starts at an overlap of less than a step's approach (0.4 um)
    and the cubes part again, slower (restitution 0.7; some of the energy
    goes into the spin the tilted faces give them)."""
    first, _, kin = run_cubes(oracle, 0, shape)
    assert first == pytest.approx(-0.08e-3, rel=1e-3)
    assert not np.isfinite(kin).all()
    first, in_contact, kin = run_cubes(oracle, abi.GB_FLAG_CRUST_BOUNDS, shape)
    assert -0.4e-6 < first < 0.0
    assert 50 < in_contact < 400
    assert np.isfinite(kin).all()
    assert kin[0, 0] < 0.0 < kin[1, 0]                 # moving apart
    assert abs(kin[1, 0] - kin[0, 0]) < 0.4            # slower than they met
