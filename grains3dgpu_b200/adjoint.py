"""Differentiable trajectories: a torch.autograd.Function around the engine's
hand-written adjoint step (gb_adjoint_step).

A trajectory of n_steps maps the initial positions, velocities and angular
velocities of the particles and the contact-law parameters (kn, en, etat,
muc per material-pair law) to the final positions, velocities and angular
velocities.  The forward pass stores the state every `every` steps; the
backward pass replays each segment from its checkpoint, keeping the segment's
states and the contact set each replayed step found (gb_save_contacts), and
runs the adjoint steps backwards through it: a replayed step's adjoint takes
its saved contacts (gb_load_contacts) instead of detecting again, so a
checkpoint interval costs one forward step per replayed step and no more.
Device memory is (n_steps / every + every - 1) states of 18 doubles per
particle plus every - 1 contact sets; with every = 1 (the default while the
states fit in a quarter of the free device memory) nothing is replayed.

Scope of the adjoint: spheres, the Hooke law with kr = 0, Rectangle walls,
first-order explicit or velocity-Verlet integration (a trajectory starts with
the leapfrog's half kick), FP64 (GB_FP64 or GB_FP64_STRICT).  The contacts
of each step are those found at its start.
"""
import ctypes as C

import numpy as np
import torch

from . import abi, engine, scenes

LAW_PARAMS = ("kn", "en", "etat", "muc")


def _dp(t):
    return C.cast(C.c_void_p(t.data_ptr()), abi._D)


class Simulation:
    """One engine context for a scene, with device-side state access."""

    def __init__(self, scene, precision=abi.GB_FP64, device=0, **config):
        self.lib = engine.load()
        self.scene = scene
        self.sys = scenes.System(self.lib, scene, precision=precision, device=device, **config)
        self.n = scene.n
        self.laws = [dict(m) for m in scene.contact_models]
        self.dev = torch.device("cuda", device)
        # the engine works on torch's current stream, so that the state
        # tensors written by torch and the engine's copies are ordered
        stream = torch.cuda.current_stream(self.dev)
        self._check(self.lib.set_stream(self.sys.ctx, C.c_void_p(stream.cuda_stream)),
                    "set_stream")

    def _check(self, st, what):
        if st not in (abi.GB_OK, abi.GB_E_OUT_OF_DOMAIN):
            raise RuntimeError(f"gb_{what} returned {st}: "
                               f"{self.lib.status_string(st).decode()}")

    def save(self, out=None):
        out = out if out is not None else torch.empty((18, self.n), dtype=torch.float64,
                                                      device=self.dev)
        self._check(self.lib.save_state(self.sys.ctx, C.c_void_p(out.data_ptr())), "save_state")
        return out

    def load(self, state):
        self._check(self.lib.load_state(self.sys.ctx, C.c_void_p(state.data_ptr())), "load_state")

    def save_contacts(self, buf=None):
        """The last detect's contact set in a device byte tensor (reused when
        it is large enough)."""
        size = C.c_int64(0)
        self._check(self.lib.save_contacts(self.sys.ctx, None, 0, C.byref(size)), "save_contacts")
        if buf is None or buf.numel() < size.value:
            buf = torch.empty(size.value + size.value // 4, dtype=torch.uint8, device=self.dev)
        self._check(self.lib.save_contacts(self.sys.ctx, C.c_void_p(buf.data_ptr()), buf.numel(),
                                           C.byref(size)), "save_contacts")
        return buf

    def load_contacts(self, buf):
        self._check(self.lib.load_contacts(self.sys.ctx, C.c_void_p(buf.data_ptr())),
                    "load_contacts")

    def set_laws(self, params):
        """params: (n_laws, 4) tensor of kn, en, etat, muc."""
        p = params.detach().cpu().numpy()
        for m, row in zip(self.laws, p):
            m.update(zip(LAW_PARAMS, map(float, row)))
        self._check(self.lib.set_contact_models(self.sys.ctx, abi.contact_model_array(self.laws)),
                    "set_contact_models")

    def step(self, k=1):
        self._check(self.lib.step(self.sys.ctx, k), "step")

    def set_phase(self, started):
        """Velocity Verlet: whether the next step is past a trajectory's first
        (a full kick) or its first (a half kick)."""
        self._check(self.lib.set_integrator_phase(self.sys.ctx, 1 if started else 0),
                    "set_integrator_phase")

    def adjoint_step(self, adj_next, adj_prev, grad_laws):
        self._check(self.lib.adjoint_step(self.sys.ctx, _dp(adj_next), _dp(adj_prev),
                                          _dp(grad_laws)), "adjoint_step")

    def law_tensor(self):
        return torch.tensor([[m[k] for k in LAW_PARAMS] for m in self.laws], dtype=torch.float64)


class Trajectory(torch.autograd.Function):
    """(x0, v0, w0, laws) -> (x, v, w) after n_steps; x0, v0, w0 are (n, 3)
    float64 tensors on the simulation's device, laws (n_laws, 4)."""

    @staticmethod
    def forward(ctx, sim, x0, v0, w0, laws, n_steps, every):
        sim.set_laws(laws)
        state = sim.save()
        state[0:3] = x0.detach().T
        state[12:15] = v0.detach().T
        state[15:18] = w0.detach().T
        sim.load(state)
        sim.set_phase(False)  # the trajectory's first step (velocity Verlet's half kick)
        checkpoints = []
        for t in range(n_steps):
            if t % every == 0:
                checkpoints.append(state if t == 0 else sim.save())
            sim.step(1)
        final = sim.save()
        ctx.sim, ctx.n_steps, ctx.every, ctx.checkpoints = sim, n_steps, every, checkpoints
        ctx.n_laws = laws.shape[0]
        ctx.laws_device = laws.device
        return final[0:3].T.clone(), final[12:15].T.clone(), final[15:18].T.clone()

    @staticmethod
    def backward(ctx, gx, gv, gw):
        sim, n = ctx.sim, ctx.sim.n
        dev = sim.dev
        z = torch.zeros((n, 3), dtype=torch.float64, device=dev)
        adj = torch.cat([(g if g is not None else z).T for g in (gx, gv, gw)]).contiguous()
        prev = torch.empty_like(adj)
        grad = torch.zeros(4 * ctx.n_laws, dtype=torch.float64, device=dev)
        seg_states = [torch.empty((18, n), dtype=torch.float64, device=dev)
                      for _ in range(ctx.every - 1)]
        seg_contacts = [None] * (ctx.every - 1)
        for seg in reversed(range(len(ctx.checkpoints))):
            t0 = seg * ctx.every
            t1 = min(t0 + ctx.every, ctx.n_steps)
            # the segment's states: its checkpoint, then the replayed steps;
            # stepping from state t found its contacts, kept for its adjoint
            states = [ctx.checkpoints[seg]]
            contacts = [None] * (t1 - t0)
            if t1 - t0 > 1:
                sim.load(states[0])
                sim.set_phase(t0 > 0)
                for t in range(t0 + 1, t1):
                    sim.step(1)
                    k = t - t0 - 1
                    seg_contacts[k] = sim.save_contacts(seg_contacts[k])
                    contacts[k] = seg_contacts[k]
                    states.append(sim.save(seg_states[k]))
            for t in reversed(range(t0, t1)):
                sim.load(states[t - t0])
                sim.set_phase(t > 0)
                if contacts[t - t0] is not None:
                    sim.load_contacts(contacts[t - t0])
                sim.adjoint_step(adj, prev, grad)
                adj, prev = prev, adj
        torch.cuda.synchronize(dev)
        return (None, adj[0:3].T.clone(), adj[3:6].T.clone(), adj[6:9].T.clone(),
                grad.view(ctx.n_laws, 4).to(ctx.laws_device), None, None)


def checkpoint_interval(sim, n_steps, budget_fraction=0.25):
    """The smallest checkpoint interval whose states (n_steps / every
    checkpoints plus every - 1 replayed states, 144 bytes per particle each)
    fit in `budget_fraction` of the device's free memory: every step is kept
    while that fits, so the backward pass replays nothing."""
    free, _ = torch.cuda.mem_get_info(sim.dev)
    per_state = 18 * 8 * sim.n
    budget = budget_fraction * free
    for every in range(1, n_steps + 1):
        if (-(-n_steps // every) + every - 1) * per_state <= budget:
            return every
    return n_steps


def trajectory(sim, x0, v0, w0, laws, n_steps, every=None):
    """(x, v, w) after n_steps from (x0, v0, w0) under `laws`, differentiable
    in all four; `every` is the checkpoint interval (None: checkpoint_interval)."""
    if every is None:
        every = checkpoint_interval(sim, n_steps)
    return Trajectory.apply(sim, x0, v0, w0, laws, n_steps, every)
