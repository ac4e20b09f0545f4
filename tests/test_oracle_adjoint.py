"""The oracle's adjoint of the time step (or_adjoint_step) against central
finite differences of the oracle's own FP64 forward, over a 6-step trajectory
of a sphere bed with sphere-sphere and sphere-wall contacts, viscous and
Coulomb-capped tangential forces and spinning particles.  This is the check
that makes the oracle's adjoint a trustworthy reference for the engine's."""
import numpy as np

from grains3dgpu_b200 import abi, scenes

T = 6
LAW_PARAMS = ("kn", "en", "etat", "muc")


sphere_bed = scenes.sphere_bed  # 60 spheres in a 9 x 9 x 16 mm box


def _state(s):
    tr, kin = s.transforms(), s.velocities()
    return np.concatenate([tr[:, 9:].T, kin[:, :3].T, kin[:, 3:].T])


def _loss(oracle, scene, w):
    s = scenes.System(oracle, scene)
    s.step(T)
    out = float((w * _state(s)).sum())
    s.close()
    return out


def _adjoint(oracle, scene, w):
    s = scenes.System(oracle, scene)
    states = []
    for _ in range(T):
        states.append((s.transforms().copy(), s.velocities().copy()))
        s.step(1)
    adj, grad = w.copy(), np.zeros(4 * len(scene.contact_models))
    for t in reversed(range(T)):
        s.set_transforms(states[t][0])
        s.set_velocities(states[t][1])
        prev = np.zeros_like(adj)
        assert oracle.adjoint_step(s.ctx, abi.dptr(adj), abi.dptr(prev), abi.dptr(grad)) == 0
        adj = prev
    s.close()
    return adj, grad


def _with(scene, **kw):
    return scenes.Scene(**{**scene.__dict__, **kw})


def test_adjoint_matches_finite_differences(oracle):
    scene = sphere_bed()
    n = scene.n
    rng = np.random.default_rng(1)
    w = rng.normal(size=(9, n))
    adj, grad = _adjoint(oracle, scene, w)
    checked = 0
    for l, m in enumerate(scene.contact_models):
        for k, name in enumerate(LAW_PARAMS):
            h = 1e-5 * abs(m[name])
            models = []
            for sign in (1, -1):
                ms = [dict(x) for x in scene.contact_models]
                ms[l][name] += sign * h
                models.append(ms)
            fd = (_loss(oracle, _with(scene, contact_models=models[0]), w)
                  - _loss(oracle, _with(scene, contact_models=models[1]), w)) / (2 * h)
            g = grad[4 * l + k]
            if fd == 0.0:
                assert g == 0.0, (l, name)
                continue
            assert abs(g - fd) <= 1e-6 * abs(fd), (l, name, g, fd)
            checked += 1
    assert checked == 8  # particle and wall laws; the third law has no contact
    dv = rng.normal(size=(n, 6))
    h = 1e-7
    fd = (_loss(oracle, _with(scene, velocities=scene.velocities + h * dv), w)
          - _loss(oracle, _with(scene, velocities=scene.velocities - h * dv), w)) / (2 * h)
    ad = (adj[3:6] * dv[:, :3].T).sum() + (adj[6:9] * dv[:, 3:].T).sum()
    assert abs(ad - fd) <= 1e-6 * abs(fd)
    dx = rng.normal(size=(n, 3))
    h = 1e-9
    tp, tm = scene.transforms.copy(), scene.transforms.copy()
    tp[:, 9:] += h * dx
    tm[:, 9:] -= h * dx
    fd = (_loss(oracle, _with(scene, transforms=tp), w)
          - _loss(oracle, _with(scene, transforms=tm), w)) / (2 * h)
    assert abs((adj[0:3] * dx.T).sum() - fd) <= 1e-6 * abs(fd)


def test_adjoint_rejects_out_of_scope(oracle):
    """Superquadrics are outside the adjoint's scope: the call says so."""
    scene = scenes.superquadric_column(n=40, box=(0.01, 0.01, 0.02))
    s = scenes.System(oracle, scene)
    adj = np.zeros((9, scene.n))
    prev = np.zeros_like(adj)
    grad = np.zeros(4 * len(scene.contact_models))
    assert oracle.adjoint_step(s.ctx, abi.dptr(adj), abi.dptr(prev),
                               abi.dptr(grad)) == abi.GB_E_UNSUPPORTED
    s.close()
