"""Writes a scene as a Grains3D input file (XML) in the vocabulary of the
reference's current XML constructors, with its particle state in insertion
files.

The XML is what ``Grains<T>::initialize`` (Grains/Base/src/Grains.cpp:37-401)
reads: ``<Construction>`` (Origin, LinkedCell, Particles, Obstacles,
ContactForceModels, TemporalSetting), ``<Forces>`` (Gravity) and
``<Simulation>`` (ParticleInsertion, PostProcessing).  Element and attribute
names follow the constructors that read them:

* ``RigidBody(DOMNode*)`` (RigidBody.cpp:62-110): Material, Density and a
  ``<Convex CrustThickness>`` holding one shape element
  (ConvexBuilderFactory.cpp:13-35: Sphere Radius, Box LX LY LZ,
  Superquadric a b c n1 n2, Rectangle LX LY);
* ``Transform3(DOMNode*)`` (Transform3.cpp:44-96): Centre X Y Z and
  AngularPosition (Type="Angles", aX aY aZ in degrees);
* ``ContactForceModelBuilderFactory::create`` (:37-70): ContactForceModel
  Type="Hooke", Material materialA materialB, Parameters kn en etat muc kr;
* ``TimeIntegratorBuilderFactory::create`` (:33-52): FirstOrderExplicit;
* ``Insertion(DOMNode*)`` (Insertion.cpp:141-180): each particle's position,
  orientation angles (radians), velocity and angular velocity from files,
  read with ``operator>>(istream, Vector3)`` (Vector3.cpp:253-258).

Rigid-body materials get the names ``m<k>``.  The reference numbers
materials in the order it first meets them (particles, then obstacles); the
writer checks that this order gives the scene's ids.
"""
import os

import numpy as np

from . import abi


def matrix_to_angles(m):
    """Angles (aX, aY, aZ) of Transform3::setBasis(aX, aY, aZ) (Transform3.cpp:
    151-162: R = Rz(aZ) Ry(aY) Rx(aX)) for the row-major rotation m[9]."""
    m = np.asarray(m, float).reshape(3, 3)
    ay = -np.arcsin(np.clip(m[2, 0], -1.0, 1.0))
    ax = np.arctan2(m[2, 1], m[2, 2])
    az = np.arctan2(m[1, 0], m[0, 0])
    return ax, ay, az


def _fmt(v):
    return repr(float(v))


def _convex_xml(rb, verts=None):
    t, p = int(rb["type"]), rb["p"]
    if t == abi.GB_SUPERQUADRIC:
        shape = (f'<Superquadric a="{_fmt(p[0])}" b="{_fmt(p[1])}" c="{_fmt(p[2])}" '
                 f'n1="{_fmt(p[3])}" n2="{_fmt(p[4])}"/>')
    elif t == abi.GB_SPHERE:
        shape = f'<Sphere Radius="{_fmt(p[0])}"/>'
    elif t == abi.GB_BOX:
        shape = f'<Box LX="{_fmt(2 * p[0])}" LY="{_fmt(2 * p[1])}" LZ="{_fmt(2 * p[2])}"/>'
    elif t == abi.GB_RECTANGLE:
        shape = f'<Rectangle LX="{_fmt(2 * p[0])}" LY="{_fmt(2 * p[1])}"/>'
    else:
        raise ValueError(f"convex type {t} has no Grains3D XML element")
    return f'<Convex CrustThickness="{_fmt(rb["crust"])}">\n          {shape}\n        </Convex>'


def write_grains_xml(scene, directory, name="grains", steps=10, linked_cell_max=None,
                     cell_size_factor=1.0, raw_data_root=None, save_every=None):
    """Writes ``<directory>/<name>.xml`` and the insertion files
    ``<name>_{position,orientation,velocity,angular_velocity}.dat`` for `scene`,
    set up to run `steps` time steps.  ``linked_cell_max`` sets the
    LinkedCell's MX MY MZ (default: the scene's max coordinate).  With
    ``raw_data_root`` a RawData writer saves every `save_every` steps into
    `directory`.  Returns the XML's path."""
    os.makedirs(directory, exist_ok=True)
    cfg = scene.config
    n = scene.n
    dt = float(cfg["dt"])
    # materials, in the order the reference meets them
    seen = []
    for r in scene.rb_ids:
        m = int(scene.rbs[r]["material"])
        if m not in seen:
            seen.append(m)
    for ob in scene.obstacles:
        if int(ob["material"]) not in seen:
            seen.append(int(ob["material"]))
    if seen != list(range(len(seen))):
        raise ValueError(f"materials met in the order {seen}: the reference would renumber them")
    nmat = int(cfg["n_materials"])
    if len(seen) > nmat:
        raise ValueError("more materials than the contact-law table covers")

    # particle types: runs of equal rigid-body ids, one <Particle> each
    runs = []
    for i, r in enumerate(scene.rb_ids):
        if runs and runs[-1][0] == int(r):
            runs[-1][1] += 1
        else:
            runs.append([int(r), 1])
    part_xml = []
    for r, num in runs:
        rb = scene.rbs[r]
        part_xml.append(
            f'      <Particle Number="{num}" Material="m{int(rb["material"])}" '
            f'Density="{_fmt(rb["density"])}">\n        {_convex_xml(rb)}\n'
            f'        <AngularPosition Type="Identity"/>\n      </Particle>')
    obs_xml = []
    for ob, tr in zip(scene.obstacles, scene.obstacle_transforms):
        ax, ay, az = (np.degrees(a) for a in matrix_to_angles(tr[:9]))
        obs_xml.append(
            f'      <Obstacle Material="m{int(ob["material"])}" Density="0">\n'
            f'        {_convex_xml(ob)}\n'
            f'        <Centre X="{_fmt(tr[9])}" Y="{_fmt(tr[10])}" Z="{_fmt(tr[11])}"/>\n'
            f'        <AngularPosition Type="Angles" aX="{_fmt(ax)}" aY="{_fmt(ay)}" '
            f'aZ="{_fmt(az)}"/>\n      </Obstacle>')
    laws = []
    for l in range(nmat):
        for s in range(l + 1):
            m = scene.contact_models[l * (l + 1) // 2 + s]
            laws.append(
                f'      <ContactForceModel Type="Hooke">\n'
                f'        <Material materialA="m{s}" materialB="m{l}"/>\n'
                f'        <Parameters>\n'
                f'          <kn>{_fmt(m["kn"])}</kn>\n          <en>{_fmt(m["en"])}</en>\n'
                f'          <etat>{_fmt(m["etat"])}</etat>\n          <muc>{_fmt(m["muc"])}</muc>\n'
                f'          <kr>{_fmt(m["kr"])}</kr>\n'
                f'        </Parameters>\n      </ContactForceModel>')
    files = {}
    tr = scene.transforms
    angles = np.array([matrix_to_angles(t[:9]) for t in tr]) if n else np.zeros((0, 3))
    for key, data in (("position", tr[:, 9:]), ("orientation", angles),
                      ("velocity", scene.velocities[:, :3]),
                      ("angular_velocity", scene.velocities[:, 3:])):
        path = os.path.join(directory, f"{name}_{key}.dat")
        with open(path, "w") as f:
            for row in data:
                f.write(" ".join(_fmt(v) for v in row) + "\n")
        files[key] = path
    mx = linked_cell_max if linked_cell_max is not None else cfg["max_coordinate"]
    org = cfg["origin"]
    g = cfg["gravity"]
    end = (steps - 0.5) * dt  # the loop runs while t <= End + 1e-15, from t = 0
    # Grains::postProcess reads the front of the save-time queue every step
    # (Grains.cpp:60-73), also once it is empty; the save times therefore run
    # on past the end of the run.
    every = save_every or steps
    writers = ""
    if raw_data_root is not None:
        writers = (f'      <Writers>\n'
                   f'        <RawData Directory="{directory}" RootName="{raw_data_root}"/>\n'
                   f'      </Writers>\n')
    post = (f'    <PostProcessing>\n'
            f'      <TimeSave Start="0" End="{_fmt((2 * steps + every) * dt)}" dt="{_fmt(every * dt)}"/>\n'
            f'{writers}    </PostProcessing>\n')
    xml = f'''<?xml version="1.0" encoding="iso-8859-1"?>
<Grains3D Type="Standard" Precision="Double">
  <Construction>
    <Origin OX="{_fmt(org[0])}" OY="{_fmt(org[1])}" OZ="{_fmt(org[2])}"/>
    <LinkedCell MX="{_fmt(mx[0])}" MY="{_fmt(mx[1])}" MZ="{_fmt(mx[2])}" CellSizeFactor="{_fmt(cell_size_factor)}"/>
    <Particles>
{chr(10).join(part_xml)}
    </Particles>
    <Obstacles>
{chr(10).join(obs_xml)}
    </Obstacles>
    <ContactForceModels>
{chr(10).join(laws)}
    </ContactForceModels>
    <TemporalSetting>
      <TimeInterval Start="0" End="{_fmt(end)}" dt="{_fmt(dt)}"/>
      <TimeIntegration Type="FirstOrderExplicit"/>
    </TemporalSetting>
  </Construction>
  <Forces>
    <Gravity GX="{_fmt(g[0])}" GY="{_fmt(g[1])}" GZ="{_fmt(g[2])}"/>
  </Forces>
  <Simulation>
    <ParticleInsertion>
      <InitialPosition Type="File" Name="{files["position"]}"/>
      <InitialOrientation Type="File" Name="{files["orientation"]}"/>
      <InitialVelocity Type="File" Name="{files["velocity"]}"/>
      <InitialAngularVelocity Type="File" Name="{files["angular_velocity"]}"/>
    </ParticleInsertion>
{post}  </Simulation>
</Grains3D>
'''
    path = os.path.join(directory, f"{name}.xml")
    with open(path, "w") as f:
        f.write(xml)
    return path


def read_state(path):
    """The state file of the XML driver: (transforms [n, 12], velocities [n, 6],
    obstacle transforms [o, 12])."""
    raw = open(path, "rb").read()
    n = int(np.frombuffer(raw[:8], np.int64)[0])
    vals = np.frombuffer(raw[8:], np.float64)
    tr = vals[:12 * n].reshape(n, 12)
    kin = vals[12 * n:18 * n].reshape(n, 6)
    obs = vals[18 * n:].reshape(-1, 12)
    return tr, kin, obs


def with_sentinels(scene, particle_position, obstacle_lift):
    """`scene` with a particle 0 and an obstacle 0 of its own kinds placed
    where they touch nothing: `particle_position` for the particle (a copy of
    particle 0's rigid body, identity orientation, at rest), and a copy of
    the obstacle whose normal points down (the lid), raised by
    `obstacle_lift`.  The reference's XML construction leaves the material id
    of the first rigid body of each material uninitialised
    (RigidBody.cpp:77-90); when those bodies touch nothing, that id is never
    read and the reference's own run from the XML is well defined."""
    import dataclasses
    tr0 = np.zeros((1, 12))
    tr0[0, [0, 4, 8]] = 1.0
    tr0[0, 9:] = particle_position
    lid = int(np.argmin(scene.obstacle_transforms[:, 8]))  # frame z axis most downward
    otr = scene.obstacle_transforms[lid:lid + 1].copy()
    otr[0, 11] += obstacle_lift
    cfg = dict(scene.config)
    cfg["n_particles"] = scene.n + 1
    cfg["n_obstacles"] = int(cfg["n_obstacles"]) + 1
    return dataclasses.replace(
        scene, name=scene.name + "-sentinels", config=cfg,
        rb_ids=np.concatenate([scene.rb_ids[:1], scene.rb_ids]).astype(np.uint32),
        transforms=np.concatenate([tr0, scene.transforms]),
        velocities=np.concatenate([np.zeros((1, 6)), scene.velocities]),
        obstacles=np.concatenate([scene.obstacles[lid:lid + 1], scene.obstacles]),
        obstacle_transforms=np.concatenate([otr, scene.obstacle_transforms]),
        lattice_counts=None)
