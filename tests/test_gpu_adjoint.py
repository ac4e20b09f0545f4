"""The hand-written adjoint of the time step on the GPU (gb_adjoint_step) and
the differentiable trajectory built on it (grains3dgpu_b200.adjoint): against
the oracle's adjoint (or_adjoint_step), against central finite differences of
the engine's own forward, and against finite differences of the FP64 CPU
oracle.  The scene has sphere-sphere and sphere-wall contacts, viscous and
Coulomb-capped tangential forces and spinning particles.
"""
import ctypes as C

import numpy as np
import pytest

from grains3dgpu_b200 import abi, scenes

from test_gpu_parity import pair

pytestmark = pytest.mark.gpu

T = 6


sphere_bed = scenes.sphere_bed  # 60 spheres in a 9 x 9 x 16 mm box


def _torch():
    import torch
    return torch


def test_adjoint_step_matches_oracle(gb, oracle):
    torch = _torch()
    scene = sphere_bed()
    g, o = pair(gb, oracle, scene, precision=abi.GB_FP64)
    n = scene.n
    rng = np.random.default_rng(3)
    adj = rng.normal(size=(9, n))
    prev_o, grad_o = np.zeros((9, n)), np.zeros(12)
    assert oracle.adjoint_step(o.ctx, abi.dptr(adj), abi.dptr(prev_o), abi.dptr(grad_o)) == 0
    d_adj = torch.tensor(adj, dtype=torch.float64, device="cuda")
    d_prev = torch.empty_like(d_adj)
    d_grad = torch.zeros(12, dtype=torch.float64, device="cuda")
    dp = lambda t: C.cast(C.c_void_p(t.data_ptr()), abi._D)
    torch.cuda.synchronize()
    assert gb.adjoint_step(g.ctx, dp(d_adj), dp(d_prev), dp(d_grad)) == 0
    prev_g, grad_g = d_prev.cpu().numpy(), d_grad.cpu().numpy()
    assert np.abs(prev_g - prev_o).max() <= 1e-9 * np.abs(prev_o).max()
    assert np.abs(grad_g - grad_o).max() <= 1e-9 * np.abs(grad_o).max()
    assert (grad_o != 0).sum() >= 7  # both laws; the particle friction is capped


def _loss_and_grads(scene, every, weights, **config):
    torch = _torch()
    from grains3dgpu_b200 import adjoint
    sim = adjoint.Simulation(scene, precision=abi.GB_FP64, **config)
    x0 = torch.tensor(scene.transforms[:, 9:], device="cuda", requires_grad=True)
    v0 = torch.tensor(scene.velocities[:, :3], device="cuda", requires_grad=True)
    w0 = torch.tensor(scene.velocities[:, 3:], device="cuda", requires_grad=True)
    laws = sim.law_tensor().requires_grad_(True)
    x, v, w = adjoint.trajectory(sim, x0, v0, w0, laws, T, every)
    loss = sum((wt * s).sum() for wt, s in zip(weights, (x, v, w)))
    loss.backward()
    out = (float(loss.detach()), x0.grad.cpu().numpy(), v0.grad.cpu().numpy(), w0.grad.cpu().numpy(),
           laws.grad.numpy().copy())
    sim.sys.close()
    return out


def _weights(n):
    torch = _torch()
    rng = np.random.default_rng(7)
    return [torch.tensor(rng.normal(size=(n, 3)), device="cuda") for _ in range(3)]


@pytest.mark.parametrize("integrator", [abi.GB_FIRST_ORDER_EXPLICIT, abi.GB_VELOCITY_VERLET])
def test_checkpoint_interval_does_not_change_gradients(integrator):
    scene = sphere_bed()
    wts = _weights(scene.n)
    ref = _loss_and_grads(scene, T, wts, integrator=integrator)
    for every in (1, 3):
        out = _loss_and_grads(scene, every, wts, integrator=integrator)
        for a, b in zip(ref[1:], out[1:]):
            assert np.array_equal(a, b)


def _fd_loss(lib, scene, weights, **config):
    """the same loss from a plain forward run of `lib` (engine or oracle)"""
    s = scenes.System(lib, scene, precision=abi.GB_FP64, **config) if lib.prefix == "gb_" else \
        scenes.System(lib, scene, **config)
    s.step(T)
    tr, kin = s.transforms(), s.velocities()
    s.close()
    w = [wt.cpu().numpy() for wt in weights]
    return float((w[0] * tr[:, 9:]).sum() + (w[1] * kin[:, :3]).sum() + (w[2] * kin[:, 3:]).sum())


def _perturbed(scene, law=None, name=None, h=0.0, dv=None, dx=None):
    s = scenes.Scene(**scene.__dict__)
    if law is not None:
        s.contact_models = [dict(m) for m in scene.contact_models]
        s.contact_models[law][name] += h
    if dv is not None:
        s.velocities = scene.velocities + dv
    if dx is not None:
        s.transforms = scene.transforms.copy()
        s.transforms[:, 9:] += dx
    return s


@pytest.mark.parametrize("fd_lib,integrator", [
    ("engine", abi.GB_FIRST_ORDER_EXPLICIT), ("oracle", abi.GB_FIRST_ORDER_EXPLICIT),
    ("engine", abi.GB_VELOCITY_VERLET), ("oracle", abi.GB_VELOCITY_VERLET)])
def test_trajectory_gradient_vs_finite_differences(gb, oracle, fd_lib, integrator):
    """Central differences of the engine's forward (GPU) and of the FP64 CPU
    oracle's forward agree with the adjoint gradients to 1e-4, with
    first-order explicit and with velocity-Verlet integration (whose first
    step is the leapfrog's half kick)."""
    lib = gb if fd_lib == "engine" else oracle
    scene = sphere_bed()
    wts = _weights(scene.n)
    cfg = {"integrator": integrator}
    _, gx, gv, gw, glaw = _loss_and_grads(scene, 3, wts, **cfg)
    checked = 0
    for l in range(glaw.shape[0]):
        for k, name in enumerate(("kn", "en", "etat", "muc")):
            if glaw[l, k] == 0.0:
                continue
            h = 1e-5 * abs(scene.contact_models[l][name])
            fd = (_fd_loss(lib, _perturbed(scene, l, name, h), wts, **cfg)
                  - _fd_loss(lib, _perturbed(scene, l, name, -h), wts, **cfg)) / (2 * h)
            assert abs(glaw[l, k] - fd) <= 1e-4 * abs(fd), (l, name, glaw[l, k], fd)
            checked += 1
    assert checked == 8
    rng = np.random.default_rng(11)
    dv = rng.normal(size=(scene.n, 6))
    h = 1e-7
    fd = (_fd_loss(lib, _perturbed(scene, dv=h * dv), wts, **cfg)
          - _fd_loss(lib, _perturbed(scene, dv=-h * dv), wts, **cfg)) / (2 * h)
    ad = (gv * dv[:, :3]).sum() + (gw * dv[:, 3:]).sum()
    assert abs(ad - fd) <= 1e-4 * abs(fd)
    dx = rng.normal(size=(scene.n, 3))
    h = 1e-9
    fd = (_fd_loss(lib, _perturbed(scene, dx=h * dx), wts, **cfg)
          - _fd_loss(lib, _perturbed(scene, dx=-h * dx), wts, **cfg)) / (2 * h)
    assert abs((gx * dx).sum() - fd) <= 1e-4 * abs(fd)
