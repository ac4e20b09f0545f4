"""Seeded synthetic packings of the benchmark configurations.

Each generator returns a :class:`Scene`: the construction data that
Grains::Construction would read from XML (Grains/Base/src/Grains.cpp:90-300)
as plain arrays -- rigid bodies, per-particle rigid-body ids, transforms,
velocities, obstacles (closed-box walls as Rectangle obstacles, the shape the
reference uses for planar walls) and the contact-model table.

All random draws come from one ``numpy.random.Generator(PCG64(seed))`` in a
fixed order: shapes, centres, jitter, orientations, velocities.
"""
import dataclasses

import os

import numpy as np

from . import abi

# numpy views of the C structs (same field order, natural alignment)
RB_DTYPE = np.dtype([("type", "<i4"), ("n_vertices", "<i4"), ("first_vertex", "<i8"),
                     ("p", "<f8", (5,)), ("crust", "<f8"), ("density", "<f8"),
                     ("material", "<i4"), ("reserved", "<i4")], align=True)
assert RB_DTYPE.itemsize == abi.C.sizeof(abi.RigidBodyDesc)


@dataclasses.dataclass
class Scene:
    name: str
    config: dict
    rbs: np.ndarray          # RB_DTYPE[n_rigid_bodies]
    vertices: np.ndarray     # float64 [n_vertices, 3]
    rb_ids: np.ndarray       # uint32 [N]
    transforms: np.ndarray   # float64 [N, 12]
    velocities: np.ndarray   # float64 [N, 6]
    obstacles: np.ndarray    # RB_DTYPE[n_obstacles]
    obstacle_transforms: np.ndarray  # float64 [n_obstacles, 12]
    contact_models: list     # dicts, l(l+1)/2+s indexed
    notes: str = ""
    lattice_counts: tuple = None  # sites per axis of the jittered lattice (site k = particle k)
    obstacle_velocities: np.ndarray = None  # float64 [n_obstacles, 6] (moving walls) or None

    @property
    def n(self):
        return int(self.rb_ids.shape[0])

    def make_config(self, **overrides):
        kw = dict(self.config)
        kw.update(overrides)
        return abi.make_config(**kw)

    def subset(self, idx):
        """The particles `idx` (and their rigid bodies) as a scene of its own."""
        idx = np.asarray(idx)
        rb_used = np.unique(self.rb_ids[idx])
        remap = np.full(self.rbs.shape[0], -1, np.int64)
        remap[rb_used] = np.arange(rb_used.size)
        rbs = self.rbs[rb_used].copy()
        verts = self.vertices
        if verts.shape[0]:
            chunks, off = [], 0
            for r in rbs:
                if r["type"] == abi.GB_POLYHEDRON:
                    s = int(r["first_vertex"])
                    chunks.append(verts[s:s + int(r["n_vertices"])])
                    r["first_vertex"] = off
                    off += int(r["n_vertices"])
            verts = np.concatenate(chunks) if chunks else np.zeros((0, 3))
        cfg = dict(self.config)
        cfg["n_particles"] = int(idx.size)
        cfg["n_rigid_bodies"] = int(rb_used.size)
        return Scene(self.name + "-subset", cfg, rbs, np.ascontiguousarray(verts),
                     remap[self.rb_ids[idx]].astype(np.uint32),
                     self.transforms[idx].copy(), self.velocities[idx].copy(),
                     self.obstacles, self.obstacle_transforms, self.contact_models,
                     self.notes)


# ---------------------------------------------------------------------------
def random_rotations(rng, n):
    """Uniform random rotation matrices (row-major, 9 each) from unit quaternions."""
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return quat_to_matrix(q)


def quat_to_matrix(q):
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    m = np.empty((q.shape[0], 9))
    m[:, 0] = 1 - 2 * (y * y + z * z)
    m[:, 1] = 2 * (x * y - w * z)
    m[:, 2] = 2 * (x * z + w * y)
    m[:, 3] = 2 * (x * y + w * z)
    m[:, 4] = 1 - 2 * (x * x + z * z)
    m[:, 5] = 2 * (y * z - w * x)
    m[:, 6] = 2 * (x * z - w * y)
    m[:, 7] = 2 * (y * z + w * x)
    m[:, 8] = 1 - 2 * (x * x + y * y)
    return m


def lattice(box, pitch, margin, n, rng, jitter):
    """n jittered cubic-lattice sites filling `box` layer by layer from z=0."""
    counts = [int(np.floor((box[k] - 2 * margin) / pitch)) + 1 for k in range(3)]
    cap = counts[0] * counts[1] * counts[2]
    if cap < n:
        raise ValueError(f"lattice holds {cap} sites < {n}")
    k = np.arange(n)
    ix = k % counts[0]
    iy = (k // counts[0]) % counts[1]
    iz = k // (counts[0] * counts[1])
    pos = np.stack([margin + ix * pitch, margin + iy * pitch, margin + iz * pitch], 1)
    pos += rng.uniform(-jitter, jitter, size=pos.shape)
    return pos, counts


def box_walls(box, material=1):
    """Six Rectangle obstacles (density 0) bounding [0, box]; each normal
    (the rectangle frame's z axis) points into the box."""
    L = box
    descs = np.zeros(6, RB_DTYPE)
    trs = np.zeros((6, 12))
    # (normal axis, side): basis columns chosen so that column 2 = inward normal
    frames = [
        ([[0, 0, 1], [0, 1, 0], [-1, 0, 0]], [0, L[1] / 2, L[2] / 2], (L[2], L[1])),   # x=0, n=+x
        ([[0, 0, -1], [0, 1, 0], [1, 0, 0]], [L[0], L[1] / 2, L[2] / 2], (L[2], L[1])),  # x=L, n=-x
        ([[1, 0, 0], [0, 0, 1], [0, -1, 0]], [L[0] / 2, 0, L[2] / 2], (L[0], L[2])),   # y=0, n=+y
        ([[1, 0, 0], [0, 0, -1], [0, 1, 0]], [L[0] / 2, L[1], L[2] / 2], (L[0], L[2])),  # y=L, n=-y
        ([[1, 0, 0], [0, 1, 0], [0, 0, 1]], [L[0] / 2, L[1] / 2, 0], (L[0], L[1])),    # z=0, n=+z
        ([[1, 0, 0], [0, -1, 0], [0, 0, -1]], [L[0] / 2, L[1] / 2, L[2]], (L[0], L[1])),  # z=L, n=-z
    ]
    for i, (b, o, (lx, ly)) in enumerate(frames):
        descs[i]["type"] = abi.GB_RECTANGLE
        descs[i]["p"][:2] = [lx / 2, ly / 2]
        descs[i]["material"] = material
        trs[i, :9] = np.array(b, float).ravel()
        trs[i, 9:] = o
    return descs, trs


def law(kn=1e4, en=0.7, muc=0.5, etat=0.0, kr=0.0, kt_ratio=0.8):
    return dict(kn=kn, en=en, etat=etat, muc=muc, kr=kr, kt=kt_ratio * kn)


def superquadric_semi_axes(r_eq, ba, ca, n1, n2):
    """Semi-axis a such that the superquadric of axes (a, ba*a, ca*a) and
    exponents (n1, n2) has the volume of a sphere of radius r_eq (volume
    formula of Superquadric::computeVolume, Superquadric.cpp:81-90)."""
    from math import gamma
    e1, e2 = 2.0 / n1, 2.0 / n2
    beta = lambda x, y: gamma(x) * gamma(y) / gamma(x + y)
    unit = 2.0 / 3.0 * e1 * e2 * beta(e1, 0.5 * e1) * beta(0.5 * e2, 0.5 * e2)
    v = 4.0 / 3.0 * np.pi * r_eq ** 3
    return (v / (unit * ba * ca)) ** (1.0 / 3.0)


# ---------------------------------------------------------------------------
def superquadric_column(seed=0, n=2000, box=(0.020, 0.020, 0.080), pitch=2.4e-3, steps=20000,
            shape="superquadric", jitter=0.15e-3, tilt=None):
    """2,000 identical superquadrics a=b=c=1 mm, n1=n2=4, on a 2.4 mm jittered
    lattice (+-0.15 mm) with random orientations, in a closed box.  The box
    is raised from 60 to 80 mm because 2,000 sites at 2.4 mm pitch do not fit
    in 20x20x60 mm; crust = 5% of the semi-axis.  `shape` swaps in 1 mm
    boxes or spheres on the same lattice (parity tests without pow); `tilt`
    (radians) replaces the uniform random orientations by small rotations."""
    rng = np.random.default_rng(seed)
    rbs = np.zeros(1, RB_DTYPE)
    if shape == "superquadric":
        rbs[0]["type"] = abi.GB_SUPERQUADRIC
        rbs[0]["p"] = [1e-3, 1e-3, 1e-3, 4.0, 4.0]
    elif shape == "box":
        rbs[0]["type"] = abi.GB_BOX
        rbs[0]["p"][:3] = [0.8e-3, 0.8e-3, 0.8e-3]
    elif shape == "sphere":
        rbs[0]["type"] = abi.GB_SPHERE
        rbs[0]["p"][0] = 1.1e-3
    else:
        raise ValueError(shape)
    rbs[0]["crust"] = 5e-5
    rbs[0]["density"] = 2500.0
    pos, _ = lattice(box, pitch, 1.6e-3, n, rng, jitter)
    tr = np.zeros((n, 12))
    if tilt is None:
        tr[:, :9] = random_rotations(rng, n)
    else:
        axis = rng.normal(size=(n, 3))
        axis /= np.linalg.norm(axis, axis=1, keepdims=True)
        ang = rng.uniform(0.0, tilt, n)
        q = np.concatenate([np.cos(ang / 2)[:, None], np.sin(ang / 2)[:, None] * axis], 1)
        tr[:, :9] = quat_to_matrix(q)
    tr[:, 9:] = pos
    walls, wtr = box_walls(box)
    cfg = dict(n_particles=n, n_rigid_bodies=1, n_obstacles=6, n_materials=2,
               origin=(0, 0, 0), max_coordinate=box, dt=2e-6, gravity=(0, 0, -9.81))
    return Scene("superquadric_column", cfg, rbs, np.zeros((0, 3)), np.zeros(n, np.uint32), tr,
                 np.zeros((n, 6)), walls, wtr, [law()] * 3,
                 notes=f"box raised to {box[2]*1e3:.0f} mm; {steps} steps nominal")


def ellipsoid_points(rng, axes, k):
    """k points uniform in area on the ellipsoid of semi-axes `axes`
    (rejection on the area-element factor of the sphere-to-ellipsoid map)."""
    a, b, c = axes
    gmax = max(b * c, a * c, a * b)
    out = []
    while len(out) < k:
        u = rng.normal(size=(4 * k, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        g = np.sqrt((b * c * u[:, 0]) ** 2 + (a * c * u[:, 1]) ** 2 + (a * b * u[:, 2]) ** 2)
        keep = rng.uniform(size=u.shape[0]) * gmax < g
        out.extend(list(u[keep] * np.array(axes)))
    return np.array(out[:k])


def polyhedra_box(seed=1, n=200_000, box=(0.100, 0.100, 0.400), pitch=2.6e-3,
            hull_centroid=None):
    """Convex polyhedra: each the hull of 8-32 points uniform on an ellipsoid
    of semi-axes 1 mm x U(0.6,1.4) x U(0.6,1.4) mm, re-centred on the hull
    centroid, on a 2.6 mm jittered lattice (+-0.1 mm) in a closed box."""
    rng = np.random.default_rng(seed)
    nv = rng.integers(8, 33, size=n)
    axes = np.stack([np.full(n, 1e-3), rng.uniform(0.6e-3, 1.4e-3, n),
                     rng.uniform(0.6e-3, 1.4e-3, n)], 1)
    first = np.concatenate([[0], np.cumsum(nv)[:-1]])
    verts = np.zeros((int(nv.sum()), 3))
    for i in range(n):
        verts[first[i]:first[i] + nv[i]] = ellipsoid_points(rng, axes[i], int(nv[i]))
    if hull_centroid is not None:
        for i in range(n):
            sl = slice(first[i], first[i] + nv[i])
            verts[sl] -= hull_centroid(verts[sl])
    rbs = np.zeros(n, RB_DTYPE)
    rbs["type"] = abi.GB_POLYHEDRON
    rbs["n_vertices"] = nv
    rbs["first_vertex"] = first
    rbs["crust"] = 5e-5
    rbs["density"] = 2500.0
    pos, _ = lattice(box, pitch, 1.6e-3, n, rng, 0.1e-3)
    tr = np.zeros((n, 12))
    tr[:, :9] = random_rotations(rng, n)
    tr[:, 9:] = pos
    walls, wtr = box_walls(box)
    cfg = dict(n_particles=n, n_rigid_bodies=n, n_obstacles=6, n_materials=2,
               origin=(0, 0, 0), max_coordinate=box, dt=1e-6, gravity=(0, 0, -9.81))
    return Scene("polyhedra_box", cfg, rbs, verts, np.arange(n, dtype=np.uint32), tr,
                 np.zeros((n, 6)), walls, wtr, [law()] * 3)


def polydisperse_superquadrics(seed=2, n=1_000_000, box=(0.3, 0.3, 1.2), pitch=None):
    """Polydisperse superquadrics: r_eq lognormal (median 1 mm, sigma 0.25)
    clipped to [0.5, 2] mm, b/a and c/a ~ U(0.5, 2), n1, n2 ~ U(2, 10), on the
    densest jittered cubic lattice that holds n sites in the box."""
    rng = np.random.default_rng(seed)
    r_eq = np.clip(1e-3 * np.exp(rng.normal(0.0, 0.25, n)), 0.5e-3, 2e-3)
    ba = rng.uniform(0.5, 2.0, n)
    ca = rng.uniform(0.5, 2.0, n)
    n1 = rng.uniform(2.0, 10.0, n)
    n2 = rng.uniform(2.0, 10.0, n)
    a = np.array([superquadric_semi_axes(r_eq[i], ba[i], ca[i], n1[i], n2[i])
                  for i in range(n)]) if n < 50_000 else _sq_axes_vec(r_eq, ba, ca, n1, n2)
    rbs = np.zeros(n, RB_DTYPE)
    rbs["type"] = abi.GB_SUPERQUADRIC
    rbs["p"] = np.stack([a, ba * a, ca * a, n1, n2], 1)
    rbs["crust"] = 0.05 * np.minimum(a, np.minimum(ba * a, ca * a))
    rbs["density"] = 2500.0
    margin = 2.5e-3
    if pitch is None:
        vol = np.prod([box[k] - 2 * margin for k in range(3)])
        pitch = (vol / n) ** (1 / 3)
        while True:
            cnt = [int(np.floor((box[k] - 2 * margin) / pitch)) + 1 for k in range(3)]
            if cnt[0] * cnt[1] * cnt[2] >= n:
                break
            pitch *= 0.995
    pos, counts = lattice(box, pitch, margin, n, rng, 0.05 * pitch)
    tr = np.zeros((n, 12))
    tr[:, :9] = random_rotations(rng, n)
    tr[:, 9:] = pos
    walls, wtr = box_walls(box)
    cfg = dict(n_particles=n, n_rigid_bodies=n, n_obstacles=6, n_materials=2,
               origin=(0, 0, 0), max_coordinate=box, dt=1e-6, gravity=(0, 0, -9.81))
    return Scene("polydisperse_superquadrics", cfg, rbs, np.zeros((0, 3)), np.arange(n, dtype=np.uint32),
                 tr, np.zeros((n, 6)), walls, wtr, [law()] * 3,
                 notes=f"lattice pitch {pitch*1e3:.3f} mm", lattice_counts=tuple(counts))


def polydisperse_bed(seed=2, n=1_000_000, box=(0.3, 0.3, 1.2), pitch=2.2e-3):
    """The grains of :func:`polydisperse_superquadrics` as a bed: a 2.2 mm
    jittered lattice filling the box from the floor up (about 0.12 m deep for
    1,000,000 grains), a solid fraction of ~0.5 and ~6 bounding-sphere
    candidates per grain -- the contact density of a settled packing, where
    the spread-out lattice has ~0.01."""
    s = polydisperse_superquadrics(seed=seed, n=n, box=box, pitch=pitch)
    s.name = "polydisperse_bed"
    return s


def _sq_axes_vec(r_eq, ba, ca, n1, n2):
    from scipy.special import gamma
    e1, e2 = 2.0 / n1, 2.0 / n2
    beta = lambda x, y: gamma(x) * gamma(y) / gamma(x + y)
    unit = 2.0 / 3.0 * e1 * e2 * beta(e1, 0.5 * e1) * beta(0.5 * e2, 0.5 * e2)
    v = 4.0 / 3.0 * np.pi * r_eq ** 3
    return (v / (unit * ba * ca)) ** (1.0 / 3.0)


def superquadric_column_on_plate(seed=3, n=10_000, column_height=None):
    """Superquadrics with n1, n2 ~ U(2, 8) and semi-axes ~ U(0.8, 1.2) mm in a
    column resting on a plate (its bottom layer within crust range of the
    plate, so contacts exist within the 2,000-step window); initial
    velocities N(0, 0.05 m/s) per component.  The lattice pitch exceeds twice
    the largest bounding-box half-diagonal, so that no two particles overlap
    at the start whatever their orientations (randomly oriented boxy grains
    closer than that start with intersecting cores and blow apart)."""
    rng = np.random.default_rng(seed)
    axes = rng.uniform(0.8e-3, 1.2e-3, size=(n, 3))
    ns = rng.uniform(2.0, 8.0, size=(n, 2))
    rbs = np.zeros(n, RB_DTYPE)
    rbs["type"] = abi.GB_SUPERQUADRIC
    rbs["p"] = np.concatenate([axes, ns], 1)
    rbs["crust"] = 0.05 * axes.min(1)
    rbs["density"] = 2500.0
    side = int(np.ceil(np.sqrt(n / 40)))
    rmax = float(np.linalg.norm(axes, axis=1).max())
    pitch = 2.0 * rmax + 0.05e-3
    margin = rmax + 0.05e-3
    jitter = 0.02e-3
    wide = 2 * margin + (side - 0.5) * pitch
    box = (wide, wide, 0.2 + 40 * pitch)
    pos, counts = lattice(box, pitch, margin, n, rng, jitter)
    tr = np.zeros((n, 12))
    tr[:, :9] = random_rotations(rng, n)
    # the bottom layer lowered onto the plate: its lowest OBB corner 20 um up
    bottom = np.arange(n) < counts[0] * counts[1]
    h = (np.abs(tr[:, 6:9]) * axes).sum(1)  # OBB half-extent along z
    pos[bottom, 2] = h[bottom] + 2e-5
    tr[:, 9:] = pos
    vel = np.zeros((n, 6))
    vel[:, :3] = rng.normal(0.0, 0.05, size=(n, 3))
    walls, wtr = box_walls(box)
    cfg = dict(n_particles=n, n_rigid_bodies=n, n_obstacles=6, n_materials=2,
               origin=(0, 0, 0), max_coordinate=box, dt=2e-6, gravity=(0, 0, -9.81))
    return Scene("superquadric_column_on_plate", cfg, rbs, np.zeros((0, 3)), np.arange(n, dtype=np.uint32),
                 tr, vel, walls, wtr, [law()] * 3)


def sphere_bed(seed=1, n=60, box=(0.009, 0.009, 0.016), pitch=2.05e-3, sink=0.55e-3):
    """Spheres of radius 1.1 mm on a 2.05 mm jittered lattice (every lattice
    neighbour overlaps), lowered by `sink` so that the bottom layer presses on
    the floor, with velocities N(0, 0.05 m/s) - 0.2 m/s downwards, angular
    velocities N(0, 5 rad/s), a viscous tangential coefficient etat = 3000
    and muc = 0.05, so that Coulomb capping occurs: the differentiable
    workload (spheres, Hooke law, walls)."""
    scene = superquadric_column(n=n, pitch=pitch, box=box, shape="sphere")
    rng = np.random.default_rng(seed)
    scene.velocities[:, :3] = rng.normal(size=(n, 3)) * 0.05
    scene.velocities[:, 3:] = rng.normal(size=(n, 3)) * 5.0
    scene.transforms[:, 11] -= sink
    scene.velocities[:, 2] -= 0.2
    scene.contact_models = [dict(m, etat=3000.0, muc=0.05) for m in scene.contact_models]
    scene.name = "sphere_bed"
    scene.notes = f"{n} spheres r=1.1 mm, lattice pitch {pitch*1e3:.2f} mm"
    return scene


def peg_board(seed=7, n=2000, pegs=64, box=(0.03, 0.03, 0.03), pitch=2.05e-3):
    """Spheres of radius 1.1 mm among fixed spherical pegs of the same size
    (obstacles of density 0), all on one 2.05 mm jittered lattice, so that
    every grain next to a peg touches it from the first step; the six box
    walls are obstacles 0-5 and the pegs 6 onwards, past the 32 that the
    per-particle wall mask covers: the obstacles the linked-cell bins serve."""
    rng = np.random.default_rng(seed)
    pos, _ = lattice(box, pitch, 1.2e-3, n + pegs, rng, 0.05e-3)
    pick = rng.permutation(n + pegs)
    peg_pos, grain_pos = pos[pick[:pegs]], pos[pick[pegs:]]
    rbs = np.zeros(1, RB_DTYPE)
    rbs[0]["type"] = abi.GB_SPHERE
    rbs[0]["p"][0] = 1.1e-3
    rbs[0]["crust"] = 5e-5
    rbs[0]["density"] = 2500.0
    walls, wtr = box_walls(box)
    pdesc = np.zeros(pegs, RB_DTYPE)
    pdesc["type"] = abi.GB_SPHERE
    pdesc["p"][:, 0] = 1.1e-3
    pdesc["crust"] = 5e-5
    pdesc["material"] = 1
    ptr = np.zeros((pegs, 12))
    ptr[:, [0, 4, 8]] = 1.0
    ptr[:, 9:] = peg_pos
    tr = np.zeros((n, 12))
    tr[:, :9] = random_rotations(rng, n)
    tr[:, 9:] = grain_pos
    vel = np.zeros((n, 6))
    vel[:, :3] = rng.normal(0.0, 0.05, size=(n, 3))
    cfg = dict(n_particles=n, n_rigid_bodies=1, n_obstacles=6 + pegs, n_materials=2,
               origin=(0, 0, 0), max_coordinate=box, dt=2e-6, gravity=(0, 0, -9.81))
    return Scene("peg_board", cfg, rbs, np.zeros((0, 3)), np.zeros(n, np.uint32), tr, vel,
                 np.concatenate([walls, pdesc]), np.concatenate([wtr, ptr]), [law()] * 3,
                 notes=f"{n} spheres among {pegs} pegs")


def cube_collision(seed=6, speed=0.4, gap=0.1e-3, tilt=0.1, shape="polyhedron"):
    """Two cubes of the drum's kind (edge 1.6 mm, crust 0.04 mm, density 2500;
    convex polyhedra of 8 vertices, or boxes) meeting head on along x at a
    relative speed `speed`, their faces `gap` apart at the start, each turned
    by random angles up to `tilt` rad; no gravity, no walls.  The cube's
    bounding box is the cube, so the reference's OBB pre-filter passes the
    pair only once the cubes intersect (GB_FLAG_CRUST_BOUNDS)."""
    rng = np.random.default_rng(seed)
    rbs = np.zeros(1, RB_DTYPE)
    rbs["density"] = 2500.0
    rbs[0]["crust"] = 0.04e-3
    h = 0.8e-3
    if shape == "polyhedron":
        rbs[0]["type"] = abi.GB_POLYHEDRON
        rbs[0]["n_vertices"] = 8
        verts = np.array([[sx * h, sy * h, sz * h] for sx in (-1, 1) for sy in (-1, 1)
                          for sz in (-1, 1)], float)
    else:
        rbs[0]["type"] = abi.GB_BOX
        rbs[0]["p"][:3] = h
        verts = np.zeros((0, 3))
    q = np.concatenate([np.ones((2, 1)), rng.uniform(-0.5 * tilt, 0.5 * tilt, (2, 3))], 1)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    tr = np.zeros((2, 12))
    tr[:, :9] = quat_to_matrix(q)
    c = np.array([0.01, 0.01, 0.01])
    tr[0, 9:] = c - [h + 0.5 * gap, 0, 0]
    tr[1, 9:] = c + [h + 0.5 * gap, 0, 0]
    vel = np.zeros((2, 6))
    vel[0, 0], vel[1, 0] = 0.5 * speed, -0.5 * speed
    cfg = dict(n_particles=2, n_rigid_bodies=1, n_obstacles=0, n_materials=1,
               origin=(0, 0, 0), max_coordinate=(0.02, 0.02, 0.02), dt=1e-6,
               gravity=(0, 0, 0))
    return Scene("cube_collision", cfg, rbs, verts, np.zeros(2, np.uint32), tr, vel,
                 np.zeros(0, RB_DTYPE), np.zeros((0, 12)), [law()],
                 notes=f"relative speed {speed} m/s, gap {gap * 1e3} mm")


def drum_obstacles(radius, length, centre, material=1):
    """A drum about the world y axis through `centre`: the cylindrical wall
    (GB_DRUM, radius, half-length; frame z = world y) and the two end caps
    (Rectangles at y = centre_y -+ length/2, normals pointing inwards)."""
    descs = np.zeros(3, RB_DTYPE)
    descs["density"] = 0.0
    descs["material"] = material
    descs[0]["type"] = abi.GB_DRUM
    descs[0]["p"][:2] = [radius, 0.5 * length]
    for k in (1, 2):
        descs[k]["type"] = abi.GB_RECTANGLE
        descs[k]["p"][:2] = [radius, radius]
    tr = np.zeros((3, 12))
    # frame axes as columns of the row-major basis: x -> x, y -> -z, z -> y
    tr[0, :9] = [1, 0, 0, 0, 0, 1, 0, -1, 0]
    tr[0, 9:] = centre
    # cap at the low end: normal +y (frame z = y); high end: normal -y
    tr[1, :9] = [1, 0, 0, 0, 0, 1, 0, -1, 0]
    tr[1, 9:] = [centre[0], centre[1] - 0.5 * length, centre[2]]
    tr[2, :9] = [1, 0, 0, 0, 0, -1, 0, 1, 0]
    tr[2, 9:] = [centre[0], centre[1] + 0.5 * length, centre[2]]
    return descs, tr


def rotating_drum(seed=4, n=2_000_000, radius=0.1, rpm=30.0, fill=0.4, pitch=3.3e-3,
                  length=None, wall_mu=0.6, margin=2.0e-3, v_sigma=0.0):
    """The rotating-drum configuration: a seeded mix of 40% spheres (r = 1 mm),
    30% cubes (edge 1.6 mm, as 8-vertex polyhedra) and 30% superquadrics
    (n1 = n2 = 6, semi-axes 1, 1, 0.7 mm), randomly oriented on a jittered
    `pitch` lattice filling the lowest `fill` of a drum of radius 0.1 m whose
    axis is horizontal (world y), turning at 30 rpm (its wall and end caps
    carry that surface velocity), grain-wall friction 0.6.  The drum's length
    is scaled so that the n grains fit: 2,000,000 grains need ~6 m at 40% of
    a 0.1 m cross-section (the nominal 0.05 m holds ~17,000).  The default
    pitch, 3.3 mm with +-2% jitter, keeps every pair of bounding spheres apart
    (2 x 1.58 mm, the superquadric's box half-diagonal, is the largest reach):
    randomly oriented cores that start intersecting meet GJK at a zero
    distance, whose contact normal is 0/0 in the reference's algorithm.
    `v_sigma` > 0 draws initial velocities N(0, v_sigma) per component (last
    in the draw order), so that neighbours meet within a short run."""
    rng = np.random.default_rng(seed)
    kind = rng.choice(3, size=n, p=[0.4, 0.3, 0.3]).astype(np.uint32)
    rbs = np.zeros(3, RB_DTYPE)
    rbs["density"] = 2500.0
    rbs[0]["type"] = abi.GB_SPHERE
    rbs[0]["p"][0] = 1e-3
    rbs[0]["crust"] = 5e-5
    rbs[1]["type"] = abi.GB_POLYHEDRON
    rbs[1]["n_vertices"] = 8
    rbs[1]["first_vertex"] = 0
    rbs[1]["crust"] = 0.04e-3
    rbs[2]["type"] = abi.GB_SUPERQUADRIC
    rbs[2]["p"] = [1e-3, 1e-3, 0.7e-3, 6.0, 6.0]
    rbs[2]["crust"] = 0.035e-3
    h = 0.8e-3
    verts = np.array([[sx * h, sy * h, sz * h] for sx in (-1, 1) for sy in (-1, 1)
                      for sz in (-1, 1)], float)
    # lattice sites of a cross-section below the fill level, `margin` inside the wall
    rin = radius - margin
    # the fill level y0 (from the centre) whose circular segment holds `fill`
    lo, hi = -rin, rin
    for _ in range(60):
        y0 = 0.5 * (lo + hi)
        area = rin * rin * np.arccos(-y0 / rin) + y0 * np.sqrt(rin * rin - y0 * y0)
        lo, hi = (y0, hi) if area < fill * np.pi * rin * rin else (lo, y0)
    g = np.arange(-rin, rin + 1e-12, pitch)
    X, Z = np.meshgrid(g, g, indexing="ij")
    inside = (X * X + Z * Z <= rin * rin) & (Z <= y0)
    sec = np.stack([X[inside], Z[inside]], 1)
    layers = int(np.ceil(n / sec.shape[0]))
    ends = max(margin, 2e-3)  # clearance from the end caps
    if length is None:
        length = 2 * ends + layers * pitch
    ny = int(np.floor((length - 2 * ends) / pitch)) + 1
    if sec.shape[0] * ny < n:
        raise ValueError("the drum holds fewer lattice sites than grains")
    k = np.arange(n)
    c = k % sec.shape[0]
    yl = k // sec.shape[0]
    centre = np.array([radius + 1e-3, 0.5 * length, radius + 1e-3])
    pos = np.stack([centre[0] + sec[c, 0], max(margin, 2e-3) + yl * pitch, centre[2] + sec[c, 1]],
                   1)
    pos += rng.uniform(-0.02 * pitch, 0.02 * pitch, size=pos.shape)
    tr = np.zeros((n, 12))
    tr[:, :9] = random_rotations(rng, n)
    tr[:, 9:] = pos
    walls, wtr = drum_obstacles(radius, length, centre)
    box = (2 * radius + 2e-3, length, 2 * radius + 2e-3)
    cfg = dict(n_particles=n, n_rigid_bodies=3, n_obstacles=3, n_materials=2,
               origin=(0, 0, 0), max_coordinate=box, dt=1e-6, gravity=(0, 0, -9.81))
    laws = [law(), law(muc=wall_mu), law(muc=wall_mu)]
    vel = np.zeros((n, 6))
    if v_sigma > 0.0:
        vel[:, :3] = rng.normal(0.0, v_sigma, size=(n, 3))
    scene = Scene("rotating_drum", cfg, rbs, verts, kind, tr, vel, walls, wtr,
                  laws, notes=f"drum length {length:.3f} m, {sec.shape[0]} sites per layer")
    omega = 2.0 * np.pi * rpm / 60.0
    scene.obstacle_velocities = np.tile([0.0, 0.0, 0.0, 0.0, omega, 0.0], (3, 1))
    return scene


# ---------------------------------------------------------------------------
class System:
    """Applies a Scene to one engine library bound by abi.Bound (gb_, or_ or
    ref_ prefix) and exposes the hot-path calls with numpy in/out."""

    def __init__(self, lib, scene, **config_overrides):
        self.lib = lib
        self.scene = scene
        self.cfg = scene.make_config(**config_overrides)
        st = abi.C.c_int32(0)
        self.ctx = lib.create(abi.C.byref(self.cfg), abi.C.byref(st))
        if not self.ctx:
            raise RuntimeError(f"{lib.prefix}create failed: {st.value}")
        rbs = np.ascontiguousarray(scene.rbs)
        verts = np.ascontiguousarray(scene.vertices, dtype=np.float64)
        self._check(lib.set_rigid_bodies(
            self.ctx, rbs.ctypes.data_as(abi.C.POINTER(abi.RigidBodyDesc)),
            abi.dptr(verts) if verts.size else None, verts.shape[0]), "set_rigid_bodies")
        need = self.cfg.n_materials * (self.cfg.n_materials + 1) // 2
        if len(scene.contact_models) != need:
            raise ValueError(f"{len(scene.contact_models)} contact laws for "
                             f"{self.cfg.n_materials} materials (need {need})")
        cms = abi.contact_model_array(scene.contact_models)
        self._check(lib.set_contact_models(self.ctx, cms), "set_contact_models")
        if self.cfg.n_obstacles:
            ob = np.ascontiguousarray(scene.obstacles)
            self._check(lib.set_obstacles(
                self.ctx, ob.ctypes.data_as(abi.C.POINTER(abi.RigidBodyDesc)),
                abi.dptr(np.ascontiguousarray(scene.obstacle_transforms))), "set_obstacles")
        if scene.obstacle_velocities is not None:
            self._check(lib.set_obstacle_velocities(
                self.ctx, abi.dptr(np.ascontiguousarray(scene.obstacle_velocities, np.float64))),
                "set_obstacle_velocities")
        self._check(lib.set_rigid_body_ids(self.ctx, abi.u32ptr(np.ascontiguousarray(scene.rb_ids))),
                    "set_rigid_body_ids")
        self.set_transforms(scene.transforms)
        self.set_velocities(scene.velocities)

    def _check(self, st, what):
        if st not in (abi.GB_OK, abi.GB_E_OUT_OF_DOMAIN):
            raise RuntimeError(f"{self.lib.prefix}{what} returned {st}")
        return st

    @property
    def n(self):
        return self.cfg.n_particles

    def set_transforms(self, tr):
        self._check(self.lib.set_transforms(self.ctx, abi.dptr(np.ascontiguousarray(tr, np.float64))),
                    "set_transforms")

    def set_velocities(self, kin):
        self._check(self.lib.set_velocities(self.ctx, abi.dptr(np.ascontiguousarray(kin, np.float64))),
                    "set_velocities")

    def transforms(self):
        out = np.zeros((self.n, 12))
        self._check(self.lib.get_transforms(self.ctx, abi.dptr(out)), "get_transforms")
        return out

    def velocities(self):
        out = np.zeros((self.n, 6))
        self._check(self.lib.get_velocities(self.ctx, abi.dptr(out)), "get_velocities")
        return out

    def torces(self):
        out = np.zeros((self.n, 6))
        self._check(self.lib.get_torces(self.ctx, abi.dptr(out)), "get_torces")
        return out

    def set_torces(self, t):
        self._check(self.lib.set_torces(self.ctx, abi.dptr(np.ascontiguousarray(t, np.float64))),
                    "set_torces")

    def rb_props(self, i):
        p = abi.RigidBodyProps()
        self._check(self.lib.get_rigid_body_props(self.ctx, i, abi.C.byref(p)), "get_rigid_body_props")
        return p

    def detect(self, result=None):
        return self._check(self.lib.detect_collision_and_compute_contact_forces(
            self.ctx, abi.i32ptr(result)), "detect")

    def add_external_forces(self):
        return self._check(self.lib.add_external_forces(self.ctx), "add_external_forces")

    def move(self):
        return self._check(self.lib.move_particles(self.ctx), "move_particles")

    def step(self, n=1):
        return self._check(self.lib.step(self.ctx, n), "step")

    def stats(self):
        s = abi.Stats()
        self._check(self.lib.get_stats(self.ctx, abi.C.byref(s)), "get_stats")
        return s

    def dump(self, kind):
        cnt = abi.C.c_int64(0)
        self._check(self.lib.debug_dump(self.ctx, kind, None, 0, abi.C.byref(cnt)), "debug_dump")
        dt = (np.float64 if kind in (abi.GB_DUMP_CONTACT_INFO, abi.GB_DUMP_CONTACT_FORCES)
              else np.uint32)
        out = np.zeros(max(1, cnt.value), dt)
        self._check(self.lib.debug_dump(self.ctx, kind, out.ctypes.data_as(abi.C.c_void_p),
                                        cnt.value, abi.C.byref(cnt)), "debug_dump")
        out = out[:cnt.value]
        if kind in (abi.GB_DUMP_CANDIDATE_PAIRS, abi.GB_DUMP_CONTACT_PAIRS):
            out = out.reshape(-1, 2)
        elif kind == abi.GB_DUMP_CONTACT_INFO:
            out = out.reshape(-1, 7)
        elif kind == abi.GB_DUMP_CONTACT_FORCES:
            out = out.reshape(-1, 6)
        return out

    def rawdata(self, directory, root_name, coordination=False):
        """A RawData post-processing writer on this system (gb_rawdata_open)."""
        return RawDataWriter(self, directory, root_name, coordination)

    def close(self):
        if self.ctx:
            self.lib.destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RawDataWriter:
    """RawDataPostProcessingWriter's start / PostProcessing / end as
    open / write(time) / close (gb_rawdata_open, gb_rawdata_write,
    gb_rawdata_close)."""

    def __init__(self, system, directory, root_name, coordination=False):
        self.system = system
        h = abi.C.c_void_p()
        flags = abi.GB_RAW_COORDINATION_NUMBER if coordination else 0
        system._check(system.lib.rawdata_open(system.ctx, os.fsencode(directory),
                                              os.fsencode(root_name), flags, abi.C.byref(h)),
                      "rawdata_open")
        self.h = h

    def write(self, time):
        return self.system._check(self.system.lib.rawdata_write(self.h, time), "rawdata_write")

    def close(self):
        if self.h:
            h, self.h = self.h, None
            return self.system._check(self.system.lib.rawdata_close(h), "rawdata_close")
