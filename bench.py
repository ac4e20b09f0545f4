"""Throughput of the DEM time step on B200: particle-steps/s.

Workload: the mixed-precision configuration -- 1,000,000 polydisperse
superquadrics (equivalent radius lognormal, median 1 mm, sigma 0.25, clipped
to 0.5-2 mm; b/a, c/a ~ U(0.5, 2); n1, n2 ~ U(2, 10)) as a bed in a closed
0.3 x 0.3 x 1.2 m box: a 2.2 mm jittered lattice from the floor up, ~0.12 m
deep, ~6 bounding-sphere candidates per grain.  dt = 1e-6 s, linear
spring-dashpot kn=1e4 N/m, en=0.7, tangential stiffness 0.8 kn with per-pair
tangential history, Coulomb mu=0.5, gravity -z.  One step = one
GrainsCPU::simulate loop iteration (collide + force, gravity, move) over all
particles.  The same grains spread over the whole box (a ~4.7 mm lattice,
~0.01 candidates per grain) are reported as the secondary `dilute` line.

The engine arm runs the tangential-history law (GB_LAW_HOOKE_HISTORY), the
workload's law.  The reference has only its Hooke law, whose relative
velocity takes the absolute contact point as lever arm: in this 1.2 m tall box
a spinning grain's damping force grows with its height, and the packing blows
up within ~100 steps.  The reference CPU path (cpu_baseline, --impl reference)
is timed with that Hooke law on blocks of the same bed, a little less work per
contact.

  python bench.py [--gpus N --steps K --warmup W]          the engine (mixed)
  python bench.py --impl reference [...]                   the reference CPU path

Multi-GPU runs are independent replicas (one seeded packing per rank, no
data-path collective); the device time is the max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from grains3dgpu_b200 import abi, scenes  # noqa: E402

LAW = abi.GB_LAW_HOOKE_HISTORY  # the engine arm's contact law

HBM_FALLBACK_GBS = 6650.0
METRIC = "particle-steps/s"


def measured_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


# Algorithmic bytes for one step (N particles, C cells; S_p = 8, positions are
# FP64 in every mode; S = 4 in the mixed mode, 8 in FP64).  The HBM-rated
# stages, as the hot-path scope defines them:
#   broad phase (hash, sort, cell start): N (3 S_p + 4 + 4 + 8 + 8 + 4) + 8 C
#   integration (the per-particle kernel): N (6 S_p + 30 S), and in the mixed
#     mode the orientation's FP32 remainder read and written, N (2 x 4 S)
# and candidate enumeration (the count kernel and its scan): the sorted key,
# FP64 position + radius, FP32 copy (mixed), id, count and the scan's read and
# write, N (4 + 32 + 16 + 4 + 4 + 8) + 4 C.  The narrow phase is latency-bound
# and is rated in pairs and GJK iterations per second instead.
def stage_bytes(n, c, s):
    return {"broad_phase": n * (3 * 8 + 4 + 4 + 8 + 8 + 4) + 8 * c,
            "integration": n * (6 * 8 + 30 * s + (8 * s if s == 4 else 0)),
            "pair_count": n * (4 + 32 + (16 if s == 4 else 0) + 4 + 4 + 8) + 4 * c}


STAGE_KERNEL = {"broad_phase": "k_hash_count + k_scan_onepass + k_cell_scatter + k_cell_rank",
                "integration": "k_particles"}
STAGE_PHASES = {"broad_phase": ("hash", "sort", "cell_start"), "integration": ("particle",),
                "pair_count": ("pair_count",)}


def stage_report(per_step_ms, n, c, s, hbm):
    out = {}
    for stage, names in STAGE_PHASES.items():
        ms = sum(float(per_step_ms[abi.PHASES.index(k)]) for k in names)
        b = stage_bytes(n, c, s)[stage]
        gbs = b / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
        out[stage] = {"ms": round(ms, 4), "algorithmic_bytes": b, "achieved_gbs": round(gbs, 1),
                      "frac_of_measured_hbm": round(gbs / hbm, 4)}
    return out


def clocks_sampler(out_path):
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    try:
        f = open(out_path, "w")
        return subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                 "-lms", "200"], stdout=f, stderr=subprocess.DEVNULL), f
    except Exception:
        return None, None


def clocks_summary(path, device):
    try:
        rows = [r.split(",") for r in open(path).read().strip().splitlines()]
        rows = [[x.strip() for x in r] for r in rows if len(r) >= 9 and r[0].strip() == str(device)]
    except Exception:
        rows = []
    if not rows:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
    sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
    mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
    reasons = set()
    for r in rows:
        for name, v in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                            "sw_power_cap"], r[5:9]):
            if v.lower().startswith("active"):
                reasons.add(name)
    return {"sm_mhz": float(np.median(sm)) if sm else None,
            "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons)}


def replica_seed(rank):
    """Each rank steps its own seeded packing (replicas; no data exchange)."""
    return 2 + 1000 * rank


BED_PITCH = 2.2e-3  # lattice pitch of the bed


def make_scene(args, rank, workload="bed"):
    if workload == "bed":
        return scenes.polydisperse_bed(seed=replica_seed(rank), n=args.n, pitch=BED_PITCH)
    if workload == "polyhedra":
        return scenes.polyhedra_box(n=args.n, hull_centroid=hull_centroid)
    if workload == "spheres":
        return scenes.sphere_bed(seed=4, n=args.n, box=adjoint_box(args.n))
    return scenes.polydisperse_superquadrics(seed=replica_seed(rank), n=args.n)


def hull_centroid(v):
    """Centroid of the convex hull of v (the engine's host geometry)."""
    from grains3dgpu_b200 import engine
    c, vol = np.zeros(3), abi.C.c_double(0.0)
    assert engine.load().convex_hull_centroid(abi.dptr(np.ascontiguousarray(v)), v.shape[0],
                                              abi.dptr(c), abi.C.byref(vol)) == 0
    return c


def aggregate(world, n_per_rank, steps, t_max):
    """Whole-job particle-steps/s: all ranks' particle-steps over the slowest
    rank's device time."""
    return world * n_per_rank * steps / t_max


def max_over_ranks(value, torch, world, device):
    t = torch.tensor([value], device=device, dtype=torch.float64)
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
def run_engine(args, scene, precision, steps, warmup, torch, rank, world, timing=True, **cfg):
    from grains3dgpu_b200 import engine
    lib = engine.load()
    flags = (abi.GB_FLAG_PHASE_TIMING if timing else 0) | cfg.pop("flags", 0)
    sysm = scenes.System(lib, scene, precision=precision, device=torch.cuda.current_device(),
                         flags=flags, contact_law=LAW, **cfg)
    stream = torch.cuda.current_stream()
    assert lib.set_stream(sysm.ctx, abi.C.c_void_p(stream.cuda_stream)) == 0
    for _ in range(warmup):
        sysm.step(1)
    ms = np.zeros(abi.GB_N_PHASES)
    lib.get_phase_times(sysm.ctx, abi.dptr(ms), None, 1)  # reset accumulators
    launches0 = sysm.stats().kernel_launches
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sysm.step(steps)  # one gb_step call: K steps with no host synchronisation between them
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    elapsed = e0.elapsed_time(e1) / 1e3
    st = sysm.stats()
    launches = st.kernel_launches - launches0
    nsteps = abi.C.c_int64(0)
    if timing:
        lib.get_phase_times(sysm.ctx, abi.dptr(ms), abi.C.byref(nsteps), 0)
    return sysm, elapsed, launches, ms, nsteps.value, st


def e2e_engine(sysm, steps, torch):
    """Same step through the public C ABI with host buffers: every step copies
    the state (transforms and velocities, Grains' host layout) in from pinned
    host memory and reads it back into the same buffers."""
    n = sysm.n
    lib, ctx = sysm.lib, sysm.ctx
    tr = torch.empty((n, 12), dtype=torch.float64, pin_memory=True).numpy()
    kin = torch.empty((n, 6), dtype=torch.float64, pin_memory=True).numpy()
    tr[:] = sysm.transforms()
    kin[:] = sysm.velocities()
    ptr, pkin = abi.dptr(tr), abi.dptr(kin)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(stream)
    for _ in range(steps):
        assert lib.set_transforms(ctx, ptr) == 0 and lib.set_velocities(ctx, pkin) == 0
        assert lib.step(ctx, 1) in (abi.GB_OK, abi.GB_E_OUT_OF_DOMAIN)
        assert lib.get_transforms(ctx, ptr) == 0 and lib.get_velocities(ctx, pkin) == 0
    e1.record(stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    return e0.elapsed_time(e1) / 1e3, wall, n * 18 * 8, n * 18 * 8


def adjoint_box(n, pitch=2.05e-3, margin=1.6e-3, layers=100):
    """A closed box whose lattice holds n sphere-bed sites in about `layers`
    layers, with 30 mm of headroom."""
    m = int(np.ceil(np.sqrt(n / layers)))
    nz = int(np.ceil(n / (m * m)))
    side = 2 * margin + (m - 0.5) * pitch
    return (side, side, 2 * margin + (nz - 0.5) * pitch + 0.03)


def measure_adjoint(torch, n, steps, every):
    """Cost of the adjoint against the forward on the sphere bed in FP64:
    the plain forward (one gb_step call of `steps` steps), the checkpointed
    trajectory's forward (a checkpoint every `every` steps), and its backward
    (each segment replayed from its checkpoint, then the adjoint steps),
    each timed with CUDA events on the engine's stream."""
    from grains3dgpu_b200 import adjoint
    scene = scenes.sphere_bed(seed=4, n=n, box=adjoint_box(n))
    dev = torch.device("cuda", torch.cuda.current_device())
    sim = adjoint.Simulation(scene, precision=abi.GB_FP64, device=dev.index)
    stream = torch.cuda.current_stream()
    ev = lambda: torch.cuda.Event(enable_timing=True)
    state0 = sim.save()
    sim.step(3)
    sim.load(state0)
    torch.cuda.synchronize()
    e0, e1 = ev(), ev()
    e0.record(stream)
    sim.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    t_plain = e0.elapsed_time(e1) / steps
    contacts = sim.sys.stats().contacts
    rng = np.random.default_rng(5)
    wts = [torch.tensor(rng.normal(size=(n, 3)), device=dev) for _ in range(3)]

    def run():
        x0 = torch.tensor(scene.transforms[:, 9:], device=dev, requires_grad=True)
        v0 = torch.tensor(scene.velocities[:, :3], device=dev, requires_grad=True)
        w0 = torch.tensor(scene.velocities[:, 3:], device=dev, requires_grad=True)
        laws = sim.law_tensor().requires_grad_(True)
        torch.cuda.synchronize()
        a, b, c = ev(), ev(), ev()
        a.record(stream)
        out = adjoint.trajectory(sim, x0, v0, w0, laws, steps, every)
        loss = sum((w * s).sum() for w, s in zip(wts, out))
        b.record(stream)
        loss.backward()
        c.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / steps, b.elapsed_time(c) / steps

    run()
    t_fwd, t_bwd = run()
    sim.sys.close()
    return {"workload": f"{n:,} spheres r=1.1 mm on a 2.05 mm lattice (all lattice neighbours "
                        "in contact) settling in a closed box, Hooke law etat=3000 muc=0.05, "
                        "first-order explicit, FP64",
            "n_particles": n, "contacts_per_step": int(contacts), "steps": steps,
            "checkpoint_every": every, "replayed_steps": steps - -(-steps // every),
            "forward_ms_per_step": t_plain,
            "trajectory_forward_ms_per_step": t_fwd, "backward_ms_per_step": t_bwd,
            "adjoint_over_forward": t_bwd / t_plain}


def measure_shapes(args, torch):
    """The same step on the other benchmark shapes, mixed and FP64, on one
    GPU: 200,000 convex polyhedra (hulls of 8-32 points on an ellipsoid, the
    polyhedra packing) and 1,000,000 spheres (the sphere bed, every lattice
    neighbour in contact)."""
    out = {}
    cases = (("polyhedra_200k", lambda: scenes.polyhedra_box(n=200_000,
                                                             hull_centroid=hull_centroid)),
             ("spheres_1M", lambda: scenes.sphere_bed(seed=4, n=1_000_000,
                                                      box=adjoint_box(1_000_000))))
    for name, build in cases:
        scene, res = build(), {}
        for prec, key in ((abi.GB_MIXED, "mixed"), (abi.GB_FP64, "fp64")):
            s, el, _, _, _, st = run_engine(args, scene, prec, args.shape_steps, 3, torch, 0, 1,
                                            timing=False)
            s.close()
            res[key] = {"value": scene.n * args.shape_steps / el,
                        "ms_per_step": el / args.shape_steps * 1e3}
        res["mixed_over_fp64"] = res["mixed"]["value"] / res["fp64"]["value"]
        res["n_particles"] = scene.n
        res["candidate_pairs_last_step"] = int(st.candidate_pairs)
        # the mixed mode's single-step error from the FP64 pose, on (up to)
        # 200,000 of the packing's grains
        res["mixed_vs_fp64_single_step"] = force_error(
            scene.subset(np.arange(min(scene.n, 200_000))), torch)
        out[name] = res
    return out


def full_length(args, torch):
    """Long runs, each in one gb_step call from its generated state, with the
    signed-volume GJK and crust-inclusive bounding tests (with the
    reference's GJK-JH, which misses most contacts of mm grains, grains pass
    into one another and every one of these runs goes non-finite): the 2,000
    superquadrics of the column configuration as a five-layer bed (2.7 mm
    pitch, 60 x 60 x 30 mm; at the stated 2.4 mm pitch randomly oriented
    grains start with intersecting cores) for its 20,000 steps of 2e-6 s
    (FP64 and mixed); the 200,000 polyhedra for their 50,000 steps of 1e-6 s
    (mixed and FP64); the 1,000,000-grain bed for 20,000 of its 100,000
    steps (mixed).  Per run: ms per step, the status, whether the state
    stayed finite, the contacts of the last step and the mean height."""
    from grains3dgpu_b200 import engine
    lib = engine.load()

    def run(scene, prec, steps):
        s = scenes.System(lib, scene, precision=prec, device=torch.cuda.current_device(),
                          contact_law=LAW, gjk_variant=abi.GB_GJK_SV,
                          flags=abi.GB_FLAG_CRUST_BOUNDS)
        stream = torch.cuda.current_stream()
        assert lib.set_stream(s.ctx, abi.C.c_void_p(stream.cuda_stream)) == 0
        # chunks of 1,000 steps, until the steps, a failed step or the cap
        el, status = 0.0, 0
        while s.stats().steps_done < steps and el < args.full_length_cap and status == 0:
            k = int(min(1000, steps - s.stats().steps_done))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            status = lib.step(s.ctx, k)
            e1.record(stream)
            torch.cuda.synchronize()
            el += e0.elapsed_time(e1) / 1e3
            status = 0 if status == abi.GB_E_OUT_OF_DOMAIN else status
        st, tr = s.stats(), s.transforms()
        s.close()
        return {"steps": steps, "status": engine.status_string(status) if status else "ok",
                "steps_done": int(st.steps_done), "ms_per_step": el / max(st.steps_done, 1) * 1e3,
                "finite": bool(np.isfinite(tr).all()), "contacts_last_step": int(st.contacts),
                "wall_contacts_last_step": int(st.obstacle_contacts),
                "mean_height_m": float(np.nanmean(tr[:, 11]))}
    out = {"full_length": True, "law": "tangential-history",
           "gjk": "signed volume, crust-inclusive bounding tests"}
    col = scenes.superquadric_column(n=2000, pitch=2.7e-3, jitter=0.03e-3,
                                     box=(0.060, 0.060, 0.030))
    out["column_2000"] = {"fp64": run(col, abi.GB_FP64, 20_000),
                          "mixed": run(col, abi.GB_MIXED, 20_000)}
    poly = scenes.polyhedra_box(n=200_000, hull_centroid=hull_centroid)
    out["polyhedra_200k"] = {"mixed": run(poly, abi.GB_MIXED, 50_000),
                             "fp64": run(poly, abi.GB_FP64, 50_000)}
    bed = scenes.polydisperse_bed(seed=replica_seed(0), n=1_000_000, pitch=BED_PITCH)
    out["bed_1M"] = {"mixed": run(bed, abi.GB_MIXED, 20_000)}
    return out


def measure_drum(args, torch):
    """The rotating-drum configuration (scenes.rotating_drum): 2,000,000 grains
    (40% spheres, 30% cubes as polyhedra, 30% n = 6 superquadrics) in a drum
    of radius 0.1 m turning at 30 rpm, its length scaled for the grains to
    fill 40% of it, the tangential-history law, grain-wall friction 0.6:
    `drum_steps` steps in one gb_step call, mixed and then FP64 from the same
    initial state, for the ratio.  Two choices of the run keep it finite and
    its contacts real: the signed-volume GJK (the reference's GJK-JH, with its
    absolute determinant threshold, misses most contacts of mm grains) and
    GB_FLAG_CRUST_BOUNDS (the reference's OBB pre-filter lets two cubes reach
    GJK only once they intersect, where the contact normal is 0/0: the state
    turns non-finite at the first cube-cube collision)."""
    scene = scenes.rotating_drum(n=args.drum_n, margin=1.7e-3, v_sigma=0.1)
    cfg = dict(gjk_variant=abi.GB_GJK_SV, flags=abi.GB_FLAG_CRUST_BOUNDS)
    out = {"workload": f"{scene.n:,} grains (40% spheres r=1 mm, 30% cubes 1.6 mm as "
                       "polyhedra, 30% superquadrics n=6 1x1x0.7 mm) in a drum of radius "
                       f"0.1 m turning at 30 rpm, {scene.notes}, wall mu 0.6, dt 1e-6 s; "
                       "initial velocities N(0, 0.1 m/s) per component so that neighbours "
                       "0.13 mm apart on the lattice collide within the run; signed-volume "
                       "GJK, crust-inclusive bounding tests (GB_FLAG_CRUST_BOUNDS)",
           "n_particles": scene.n}
    for prec, key, k in ((abi.GB_MIXED, "mixed", args.drum_steps),
                         (abi.GB_FP64, "fp64", args.drum_steps)):
        s, el, _, _, _, st = run_engine(args, scene, prec, k, 3, torch, 0, 1, timing=False,
                                        **dict(cfg))
        tr = s.transforms()
        out[key] = {"steps": k, "value": scene.n * k / el, "ms_per_step": el / k * 1e3,
                    "contacts_last_step": int(st.contacts),
                    "wall_contacts_last_step": int(st.obstacle_contacts),
                    "finite": bool(np.isfinite(tr).all())}
        s.close()
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def force_error(scene, torch):
    """Single-step error of the mixed mode against the FP64 mode, both given
    the scene's FP64 pose: per contact (metrics.contact_force_errors: the
    force and torque each contact pair puts on its first particle, |x_mixed -
    x_fp64| / |x_fp64|), and per particle (max |F_mixed - F_fp64| over
    particles divided by max |F_fp64|)."""
    from grains3dgpu_b200 import engine, metrics
    lib = engine.load()
    dev = torch.cuda.current_device()
    m = scenes.System(lib, scene, precision=abi.GB_MIXED, device=dev, contact_law=LAW)
    f = scenes.System(lib, scene, precision=abi.GB_FP64, device=dev, contact_law=LAW)
    m.detect()
    f.detect()
    per_contact = metrics.contact_force_errors(m, f)
    a, b = m.torces(), f.torces()
    m.close()
    f.close()
    return {"per_contact": per_contact,
            "per_particle_force": float(np.abs(a[:, :3] - b[:, :3]).max()
                                        / max(np.abs(b[:, :3]).max(), 1e-300)),
            "per_particle_torque": float(np.abs(a[:, 3:] - b[:, 3:]).max()
                                         / max(np.abs(b[:, 3:]).max(), 1e-300))}


# ---------------------------------------------------------------------------
def full_cell_size(scene):
    """Linked-cell size of the whole workload (2 x the largest circumscribed
    radius), computed by the FP64 oracle's rigid-body set-up."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    s = scenes.System(pyoracle.load_oracle(), scene)
    cell = s.stats().cell_size
    s.close()
    return cell


def sample_blocks(scene, m, count):
    """`count` disjoint blocks of about m particles each: s x s lattice columns
    of the bottom h layers (the packing fills the lattice layer by layer), so
    every sampled particle sees the workload's local density."""
    cx, cy, _ = scene.lattice_counts
    k = np.arange(scene.n)
    ix, iy, iz = k % cx, (k // cx) % cy, k // (cx * cy)
    per_row = int(np.ceil(np.sqrt(count)))
    side = max(2, min(cx, cy) // per_row)                 # columns of side x side sites
    layers = max(1, int(np.ceil(m / (side * side))))      # ... and this many layers
    out = []
    for b in range(count):
        bx, by = b % per_row, b // per_row
        sel = ((ix // side) == bx) & ((iy // side) == by) & (iz < layers)
        out.append(np.nonzero(sel)[0])
    return out


def sample_scene(scene, idx, cell):
    """The particles idx as a system of their own, with the workload's cell size."""
    sub = scene.subset(idx)
    probe = scenes.System(_cpu_lib()[0], sub)
    factor = cell / probe.stats().cell_size
    probe.close()
    sub.config["cell_size_factor"] = factor
    return sub


def _cpu_lib():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    if pyoracle.reference_available():
        return pyoracle.load_reference(), "reference"
    return pyoracle.load_oracle(), "port"


class BedSample:
    """One block of the workload stepped by the reference's CPU path.  Every
    timed step starts from the block's initial state (restored before the
    step, outside the timed region): the reference's Hooke law measures the
    relative velocity at the absolute contact point, which drives the bed's
    initially overlapping grains non-finite within ~50 steps, and its
    LinkedCell then writes out of bounds.  So each step is one loop iteration
    over the bed as generated, the state the engine arm starts from."""

    def __init__(self, lib, sub):
        self.sys = scenes.System(lib, sub)
        self.tr0 = np.ascontiguousarray(sub.transforms, np.float64)
        self.kin0 = np.ascontiguousarray(sub.velocities, np.float64)

    def restore(self):
        self.sys.set_transforms(self.tr0)
        self.sys.set_velocities(self.kin0)

    def step(self):
        self.sys.step(1)


def time_reference(scene, m, target_s, max_steps=50, cell=None):
    lib, kind = _cpu_lib()
    cell = cell or full_cell_size(scene)
    blk = BedSample(lib, sample_scene(scene, sample_blocks(scene, m, 1)[0], cell))
    m = blk.sys.n
    blk.restore()
    t0 = time.perf_counter()
    blk.step()
    t1 = time.perf_counter() - t0
    steps = int(max(1, min(max_steps, target_s / max(t1, 1e-6))))
    dt = 0.0
    for _ in range(steps):
        blk.restore()
        t0 = time.perf_counter()
        blk.step()
        dt += time.perf_counter() - t0
    blk.sys.close()
    return {"value": m * steps / dt, "unit": METRIC, "cores": 1, "kind": kind,
            "sample": f"{m} particles (a lattice block of the bed, full-workload cell size) x "
                      f"{steps} steps, each from the block's initial state, {dt:.1f} s, single "
                      f"thread (the reference loop is serial)"}


def reference_arm(args):
    """--impl reference: the reference's own CPU path on every host thread,
    each thread stepping its own disjoint block of the workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    lib, kind = _cpu_lib()
    try:
        nthreads = len(os.sched_getaffinity(0))
    except Exception:
        nthreads = os.cpu_count() or 1
    scene = make_scene(args, 0)
    cell = full_cell_size(scene)
    blocks = [b for b in sample_blocks(scene, args.ref_sample, nthreads) if b.size]
    nthreads = len(blocks)
    samples = [BedSample(lib, sample_scene(scene, b, cell)) for b in blocks]
    m = int(np.mean([b.size for b in blocks]))
    total = int(sum(b.size for b in blocks))

    def run(k):
        dt = 0.0
        for _ in range(k):
            for smp in samples:
                smp.restore()
            ths = [threading.Thread(target=smp.step) for smp in samples]
            t0 = time.perf_counter()
            for t in ths:
                t.start()
            for t in ths:
                t.join()
            dt += time.perf_counter() - t0
        return dt

    run(args.warmup)
    dt = run(args.steps)
    value = total * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": f"sample of {args.n:,} polydisperse superquadrics as a bed "
                               f"(a {BED_PITCH*1e3:.1f} mm jittered lattice from the floor of a "
                               "0.3x0.3x1.2 m box)",
                   "sample_particles_per_thread": m, "threads": nthreads,
                   "steps": "each timed step from the blocks' initial state"},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": nthreads, "kind": kind,
                         "sample": f"{nthreads} threads, each stepping its own lattice block of "
                                   f"~{m} particles of the bed (full-workload cell size), "
                                   f"{args.steps} steps, each from the blocks' initial state"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--n", type=int, default=1_000_000)
    ap.add_argument("--fp64-steps", type=int, default=10)
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--ref-sample", type=int, default=20_000)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--adjoint-n", type=int, default=1_000_000)
    ap.add_argument("--adjoint-steps", type=int, default=100)
    ap.add_argument("--adjoint-every", type=int, default=10,
                    help="checkpoint interval of the adjoint run (its backward replays the rest)")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--shape-steps", type=int, default=10)
    ap.add_argument("--no-shapes", action="store_true")
    ap.add_argument("--no-dilute", action="store_true")
    ap.add_argument("--drum-n", type=int, default=2_000_000)
    ap.add_argument("--drum-steps", type=int, default=5000)
    ap.add_argument("--full-length", action="store_true",
                    help="run the configurations at their full lengths instead (one JSON line)")
    ap.add_argument("--full-length-cap", type=float, default=120.0,
                    help="with --full-length: seconds of device time per run at most")
    ap.add_argument("--timed-only", action="store_true",
                    help="run the headline's warm-up and timed steps only (for profilers)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="with --timed-only: the run mode")
    ap.add_argument("--workload", default="bed",
                    choices=["bed", "dilute", "polyhedra", "spheres"],
                    help="with --timed-only: the packing (polyhedra: --n of the 200,000 "
                         "convex hulls' packing; spheres: the sphere bed)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return reference_arm(args)

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    if args.full_length:
        if rank == 0:
            print(json.dumps(full_length(args, torch)))
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0

    if args.timed_only:
        scene = make_scene(args, rank, args.workload)
        prec = abi.GB_MIXED if args.precision == "mixed" else abi.GB_FP64
        sysm, elapsed, launches, _, _, st = run_engine(args, scene, prec, args.steps,
                                                       args.warmup, torch, rank, world,
                                                       timing=False)
        sysm.close()
        if rank == 0:
            print(json.dumps({"timed_only": True, "workload": args.workload,
                              "precision": args.precision, "n": scene.n,
                              "ms_per_step": elapsed / args.steps * 1e3,
                              "gpu_launches": int(launches),
                              "candidate_pairs": int(st.candidate_pairs),
                              "gjk_pairs": int(st.gjk_calls),
                              "gjk_fp64_pairs": int(st.gjk_fp64_calls),
                              "contacts": int(st.contacts)}))
        if world > 1:
            torch.distributed.destroy_process_group()
        return 0

    scene = make_scene(args, rank)
    fd, clk_path = tempfile.mkstemp(prefix=f"gb_clocks_rank{rank}_", suffix=".csv")
    os.close(fd)
    sampler, fh = clocks_sampler(clk_path)
    # the timed run carries no phase events; the phase split comes from a
    # second, instrumented run of the same workload
    sysm, elapsed, launches, _, _, st = run_engine(
        args, scene, abi.GB_MIXED, args.steps, args.warmup, torch, rank, world, timing=False)
    if sampler:
        sampler.terminate()
        fh.close()
    clocks = clocks_summary(clk_path, torch.cuda.current_device())
    os.unlink(clk_path)
    t_max = max_over_ranks(elapsed, torch, world, "cuda")
    value = aggregate(world, scene.n, args.steps, t_max)

    e2e_dev, e2e_wall, h2d, d2h = e2e_engine(sysm, args.e2e_steps, torch)
    e2e_value = world * scene.n * args.e2e_steps / max(e2e_dev, e2e_wall)
    sysm.close()
    sys_ph, _, _, ms, nsteps, st_ph = run_engine(args, scene, abi.GB_MIXED, min(args.steps, 10),
                                                 3, torch, rank, world, timing=True)
    sys_ph.close()

    # per-stage roofline (phase device time from CUDA events on the launch stream)
    hbm, hbm_kind = measured_hbm()
    per_step = ms / max(nsteps, 1)
    stages = stage_report(per_step, scene.n, st.n_cells, 4, hbm)
    # the roofline of the HBM-bound stages (broad phase and integration): the
    # one with the larger share of the step; the step's largest kernels (the
    # narrow phase, the candidate search) are issue- and latency-bound and are
    # rated in `narrow` and `stages`
    top = max(("broad_phase", "integration"), key=lambda k: stages[k]["ms"])
    dominant = max((k for k in abi.PHASES), key=lambda k: float(per_step[abi.PHASES.index(k)]))
    roofline = {"kernel": STAGE_KERNEL[top], "stage": top, "bound": "hbm",
                "achieved": stages[top]["achieved_gbs"],
                "peak": hbm, "unit": "GB/s", "frac": stages[top]["frac_of_measured_hbm"],
                "traffic": traffic_bytes(top, scene.n), "peak_kind": hbm_kind,
                "limiter": LIMITER.get(top),
                "step_dominant_phase": {"phase": dominant,
                                        "ms": round(float(per_step[abi.PHASES.index(dominant)]), 4),
                                        "limiter": LIMITER.get(dominant)}}
    narrow_ms = float(per_step[abi.PHASES.index("narrow")])
    narrow = {"ms": round(narrow_ms, 4), "candidate_pairs": int(st_ph.candidate_pairs),
              "pairs_per_s": st_ph.candidate_pairs / (narrow_ms * 1e-3) if narrow_ms else None,
              "gjk_iterations_per_step": st_ph.gjk_iterations / max(nsteps, 1),
              "gjk_iterations_per_s": st_ph.gjk_iterations / max(nsteps, 1) / (narrow_ms * 1e-3)
              if narrow_ms else None}

    # the all-FP64 run of the same kernels on the same workload (timed, then
    # instrumented for its phase split)
    s64, el64, _, _, _, _ = run_engine(args, scene, abi.GB_FP64, args.fp64_steps, 3, torch,
                                       rank, world, timing=False)
    s64.close()
    s64, _, _, ms64, n64, _ = run_engine(args, scene, abi.GB_FP64, args.fp64_steps, 3, torch,
                                         rank, world, timing=True)
    s64.close()
    t64 = max_over_ranks(el64, torch, world, "cuda")
    value64 = aggregate(world, scene.n, args.fp64_steps, t64)
    ferr = None
    if rank == 0:
        # both modes from the same FP64 pose: the bottom 200,000 grains of the
        # bed, and 200,000 grains of the spread-out lattice
        ferr = {"bed_200k": force_error(scene.subset(np.arange(min(scene.n, 200_000))), torch),
                "dilute_200k": force_error(make_scene(args, rank, "dilute").subset(
                    np.arange(min(scene.n, 200_000))), torch)}

    dilute = None
    if world == 1 and not args.no_dilute:
        dscene = make_scene(args, rank, "dilute")
        dres = {}
        for prec, key, k in ((abi.GB_MIXED, "mixed", args.steps),
                             (abi.GB_FP64, "fp64", args.fp64_steps)):
            ds, del_, _, _, _, dst = run_engine(args, dscene, prec, k, args.warmup, torch, 0, 1,
                                                timing=False)
            ds.close()
            dres[key] = {"value": dscene.n * k / del_, "ms_per_step": del_ / k * 1e3}
        dres["mixed_over_fp64"] = dres["mixed"]["value"] / dres["fp64"]["value"]
        dres["workload"] = (f"the same {dscene.n:,} grains spread over the whole box "
                            f"({dscene.notes})")
        dres["candidate_pairs_last_step"] = int(dst.candidate_pairs)
        dilute = dres

    shapes = None
    if world == 1 and not args.no_shapes:
        shapes = measure_shapes(args, torch)

    drum = None
    if world == 1 and args.drum_steps > 0:
        drum = measure_drum(args, torch)

    adj = None
    if world == 1 and not args.no_adjoint:
        adj = measure_adjoint(torch, args.adjoint_n, args.adjoint_steps, args.adjoint_every)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = time_reference(scene, args.ref_sample, args.cpu_seconds, cell=st.cell_size)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 (f64 positions, f64 GJK)",
            "data": "synthetic (seeded jittered-lattice packing)",
            "config": {"workload": f"{scene.n:,} polydisperse superquadrics as a bed (a "
                                   f"{BED_PITCH*1e3:.1f} mm jittered lattice from the floor of "
                                   "a 0.3x0.3x1.2 m box), dt=1e-6 s, mixed precision",
                       "n_particles": scene.n, "precision": "mixed",
                       "contact_law": "linear spring-dashpot, kt = 0.8 kn, Coulomb mu = 0.5, "
                                      "per-pair tangential history",
                       "gjk": "GJK with Johnson's sub-algorithm (the reference's)",
                       "n_cells": st.n_cells, "candidate_pairs_last_step": st.candidate_pairs,
                       "candidate_pairs_per_particle": st.candidate_pairs / scene.n,
                       "gjk_pairs_last_step": st.gjk_calls,
                       "gjk_fp64_pairs_last_step": st.gjk_fp64_calls,
                       "contacts_last_step": st.contacts,
                       "l2": "per-step working set > 126 MB L2, no flush",
                       "parallelism": f"replicas x{world}"},
            "roofline": roofline,
            "phases_ms": {k: round(float(v), 4) for k, v in zip(abi.PHASES, per_step)},
            "stages": stages,
            "narrow": narrow,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "steps": args.e2e_steps,
                    "ms_per_step": max(e2e_dev, e2e_wall) / args.e2e_steps * 1e3},
            "fp64": {"value": value64, "ms_per_step": t64 / args.fp64_steps * 1e3,
                     "steps": args.fp64_steps,
                     "phases_ms": {k: round(float(v), 4) for k, v in
                                   zip(abi.PHASES, ms64 / max(n64, 1))},
                     "stages": stage_report(ms64 / max(n64, 1), scene.n, st.n_cells, 8, hbm)},
            "mixed_over_fp64": value / value64,
            "mixed_vs_fp64_single_step": ferr,
            "dilute": dilute,
            "adjoint": adj,
            "other_shapes": shapes,
            "drum": drum,
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        print(json.dumps(line))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


# DRAM bytes (read + write) per particle of the HBM-rated kernels, from ncu
# captures of the bed at 600,000 grains (k_particles with --set full; the
# broad-phase kernels' dram__bytes metrics), whose per-step working set
# exceeds the L2 as the 1,000,000-grain bed's does; the summary is committed
# beside the other profiles.  Their traffic scales with the particle count
# at the bed's density.  Writes that stay in L2 when the kernel ends are not
# counted by the capture.
TRAFFIC_PER_PARTICLE = {"integration": (95.4e6 + 12.2e6) / 600_000,
                        "broad_phase": (14.48e6 + 2.56e6 + 26.54e6 + 0.06e6) / 600_000}


# what bounds each stage or phase, from the same captures and those of the bed
# at 200,000 grains
LIMITER = {"integration": "issue and memory latency: 40% warps active (64 registers, four "
                          "256-thread blocks per SM), 42% issue slots; 159 B per particle "
                          "read from DRAM",
           "broad_phase": "launch and tail latency of short dependent passes (hash 10 us, "
                          "scan, scatter 9 us, rank 20 us at 600k grains); 73 B per particle "
                          "read from DRAM",
           "pair_count": "memory latency of the neighbour walk on the finer grid: 17 "
                         "long-scoreboard stalls per issue at 46% warps active",
           "narrow": "FP32 issue in the cull (42% issue slots, 24 of 32 lanes, 96 registers) "
                     "and FP64 GJK chains at 10-15% warps active (220 registers, 168 in "
                     "its three-block form for long queues)"}


def traffic_bytes(phase, n):
    v = TRAFFIC_PER_PARTICLE.get(phase)
    return None if v is None else v * n

if __name__ == "__main__":
    sys.exit(main())
