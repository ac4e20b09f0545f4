"""The Xerces-free ReaderXML (grains3dgpu_b200/xml/ReaderXML.cpp) and the XML
front end (include/grains_b200_grains.hh), on the CPU.

* The parser: element/text/attribute tree, whitespace text nodes kept (the
  reference's ConvexBuilderFactory takes the second child node of <Convex>),
  comments, processing instructions and the DOCTYPE dropped, entity and
  character references resolved; malformed input rejected.
* Grains3D run from an XML through it: the reference's own GrainsCPU
  (Grains/Base/src/GrainsCPU.cpp) built by Grains<T>::Construction from the
  file equals, bit for bit, the reference path built directly from the same
  data (oracle/_ref's harness).
* The two construction defects GrainsB200 corrects: material ids from the
  material map, and insertion windows that keep their corners.
"""
import os
import subprocess

import numpy as np
import pytest

from grains3dgpu_b200 import grains_xml, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVE = os.path.join(ROOT, "oracle", "_ref", "xml_drive")


@pytest.fixture(scope="module")
def drive():
    if not os.path.exists(DRIVE):
        pytest.skip("oracle/_ref/xml_drive is not built here (needs the reference sources)")
    return DRIVE


def run(*args, check=True):
    r = subprocess.run([DRIVE, *map(str, args)], capture_output=True, text=True, timeout=600)
    if check:
        assert r.returncode == 0, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    return r


TREE_XML = """<?xml version="1.0" encoding="iso-8859-1"?>
<!DOCTYPE Grains3D SYSTEM "x.dtd" [ <!ELEMENT a (b)> ]>
<!-- leading comment -->
<Root Precision='Double' Note="a &amp; b &lt;c&gt; &#65;&#x42;">
  <Convex CrustThickness="5e-5">
    <!-- a comment between the children -->
    <Sphere Radius="0.001"/>
  </Convex>
  <kn>1e4</kn>
  <Text><![CDATA[x < y]]> and &quot;z&quot;</Text>
  <?pi ignored?>
</Root>
"""

TREE_EXPECTED = """<Root Precision=[Double] Note=[a & b <c> AB]>
  #ws
  <Convex CrustThickness=[5e-5]>
    #ws
    <Sphere Radius=[0.001]>
    #ws
  #ws
  <kn>
    #text 1e4
  #ws
  <Text>
    #text x < y and "z"
  #ws
"""


def test_reader_tree(drive, tmp_path):
    p = tmp_path / "t.xml"
    p.write_text(TREE_XML)
    out = run("tree", p).stdout
    assert out == TREE_EXPECTED, out


@pytest.mark.parametrize("text", [
    "<A><B></A></B>",             # mismatched close
    '<A x="1></A>',               # unterminated attribute value
    "<A></A><B/>",                # two document elements
    '<A x="1" x="2"/>',           # attribute given twice
    "<A>&bogus;</A>",             # unknown entity
    "no element",
])
def test_reader_rejects_malformed(drive, tmp_path, text):
    p = tmp_path / "bad.xml"
    p.write_text(text)
    r = run("tree", p, check=False)
    assert r.returncode == 1 and "XML exception" in r.stderr


def column_xml(directory, steps, n=60):
    """The 2,000-superquadric column's grains (n of them on the 2.05 mm lattice)
    as an XML run, with an isolated particle 0 and obstacle 0 (see
    grains_xml.with_sentinels), and the LinkedCell one cell larger than the box
    so that the reference's floored cell counts cover it."""
    sc = scenes.superquadric_column(n=n, pitch=2.05e-3)
    sx = grains_xml.with_sentinels(sc, (0.010, 0.010, 0.075), 0.01)
    cell = 2 * 1.316074013e-3
    lcmax = [sc.config["max_coordinate"][k] + cell for k in range(3)]
    return sx, lcmax, grains_xml.write_grains_xml(sx, str(directory), steps=steps,
                                                  linked_cell_max=lcmax)


def test_xml_run_matches_direct_construction(drive, reference, tmp_path):
    steps = 20
    sx, lcmax, xml = column_xml(tmp_path, steps)
    run("insert", xml, tmp_path / "init.bin")
    tr0, kin0, obs0 = grains_xml.read_state(tmp_path / "init.bin")
    # the XML carries the scene (angles and decimal text round-trip to ~1e-16)
    assert np.abs(tr0 - sx.transforms).max() < 1e-15
    assert np.abs(obs0 - sx.obstacle_transforms).max() < 1e-15
    out = run("run", "cpu", xml, tmp_path / "cpu.bin").stdout
    assert "particles 61" in out
    tr1, kin1, _ = grains_xml.read_state(tmp_path / "cpu.bin")
    import dataclasses
    direct = dataclasses.replace(sx, transforms=tr0, velocities=kin0, obstacle_transforms=obs0)
    direct.config = dict(direct.config, max_coordinate=tuple(lcmax))
    s = scenes.System(reference, direct, pad_grid=0)
    s.step(steps)
    assert np.array_equal(s.transforms(), tr1)
    assert np.array_equal(s.velocities(), kin1)
    assert np.abs(tr1 - tr0).max() > 1e-6  # the grains moved


MATERIALS_XML = """<Grains3D Type="Standard" Precision="Double">
  <Construction>
    <LinkedCell MX="0.02" MY="0.02" MZ="0.02"/>
    <Particles>
      <Particle Number="3" Material="steel" Density="7800">
        <Convex CrustThickness="1e-5">
          <Sphere Radius="0.001"/>
        </Convex>
        <AngularPosition Type="Identity"/>
      </Particle>
      <Particle Number="2" Material="glass" Density="2500">
        <Convex CrustThickness="1e-5">
          <Box LX="0.001" LY="0.001" LZ="0.001"/>
        </Convex>
        <AngularPosition Type="Identity"/>
      </Particle>
    </Particles>
    <Obstacles>
      <Obstacle Material="wall" Density="0">
        <Convex CrustThickness="0">
          <Rectangle LX="0.02" LY="0.02"/>
        </Convex>
        <AngularPosition Type="Identity"/>
      </Obstacle>
      <Obstacle Material="steel" Density="0">
        <Convex CrustThickness="0">
          <Rectangle LX="0.02" LY="0.02"/>
        </Convex>
        <Centre X="0" Y="0" Z="0.02"/>
        <AngularPosition Type="Angles" aX="180" aY="0" aZ="0"/>
      </Obstacle>
    </Obstacles>
  </Construction>
  <Forces><Gravity GX="0" GY="0" GZ="-9.81"/></Forces>
  <Simulation>
    <ParticleInsertion>
      <InitialPosition Type="Random" Seed="Default">
        <Windows>
          <Window Type="Box">
            <MinPoint X="0.002" Y="0.003" Z="0.004"/>
            <MaxPoint X="0.018" Y="0.017" Z="0.016"/>
          </Window>
        </Windows>
      </InitialPosition>
      <InitialOrientation Type="Zero"/>
      <InitialVelocity Type="Constant" X="0" Y="0" Z="-0.1"/>
      <InitialAngularVelocity Type="Zero"/>
    </ParticleInsertion>
  </Simulation>
</Grains3D>
"""


def test_material_ids_from_the_material_map(drive, tmp_path):
    """Materials are numbered in the order they are met (steel 0, glass 1,
    wall 2); every rigid body takes its material's number."""
    p = tmp_path / "m.xml"
    p.write_text(MATERIALS_XML)
    out = run("materials", p).stdout.splitlines()
    assert out[-3] == "particles 0 0 0 1 1"
    assert out[-2] == "obstacles 2 0"
    assert out[-1] == "materials 3"


def test_insertion_window_keeps_its_corners(drive, tmp_path):
    """Random insertion in a Box window: the reference draws inside a window
    collapsed to the origin; with the fix the same draws land inside the
    window's corners, and the constant velocity is inserted either way."""
    p = tmp_path / "m.xml"
    p.write_text(MATERIALS_XML)
    run("insert", p, tmp_path / "ref.bin")
    run("insert", p, tmp_path / "fix.bin", "--fix-insertion")
    run("insert", p, tmp_path / "fix2.bin", "--fix-insertion")
    tr_ref, kin_ref, _ = grains_xml.read_state(tmp_path / "ref.bin")
    tr_fix, kin_fix, _ = grains_xml.read_state(tmp_path / "fix.bin")
    tr_fix2, _, _ = grains_xml.read_state(tmp_path / "fix2.bin")
    assert not tr_ref[:, 9:].any()                     # the collapsed window
    lo, hi = np.array([0.002, 0.003, 0.004]), np.array([0.018, 0.017, 0.016])
    x = tr_fix[:, 9:]
    assert np.all(x >= lo) and np.all(x <= hi)
    assert len(np.unique(x[:, 0])) == x.shape[0]       # distinct draws
    assert np.array_equal(tr_fix, tr_fix2)             # the default seed: deterministic
    assert np.array_equal(tr_fix[:, :9], tr_ref[:, :9])
    assert np.array_equal(kin_fix, kin_ref) and np.allclose(kin_fix[:, 2], -0.1)
