"""Grains3D from an XML input on the B200: GrainsB200 (include/
grains_b200_grains.hh), built by the reference's Grains<T>::Construction
through the Xerces-free ReaderXML, against the reference's own GrainsCPU
built from the same file.  The column of the 2,000-superquadric run (60
grains, FP64-strict): transforms within 1e-12 and velocities within 1e-7 of
the largest, the tolerances of the drop-in check (superquadric supports
differ from the host's pow in the last bits)."""
import os

import numpy as np
import pytest

from grains3dgpu_b200 import grains_xml

from test_xml_cpu import DRIVE, column_xml, run  # noqa: F401

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def drive(gb):
    if not os.path.exists(DRIVE):
        pytest.fail("oracle/_ref/xml_drive is missing: build it here (it travels in-tree)")
    return DRIVE


def test_grains_b200_from_xml_matches_grains_cpu(drive, tmp_path):
    steps = 40
    _, _, xml = column_xml(tmp_path, steps)
    run("run", "cpu", xml, tmp_path / "cpu.bin")
    out = run("run", "b200", xml, tmp_path / "b200.bin").stdout
    tc, kc, oc = grains_xml.read_state(tmp_path / "cpu.bin")
    tg, kg, og = grains_xml.read_state(tmp_path / "b200.bin")
    assert tc.shape == tg.shape == (61, 12)
    assert np.array_equal(oc, og)
    assert np.abs(tg - tc).max() < 1e-12
    assert np.abs(kg - kc).max() <= 1e-7 * np.abs(kc).max()
    assert np.abs(tc - grains_xml.read_state(tmp_path / "cpu.bin")[0]).max() == 0
    contacts = int(out.strip().split()[-1])
    assert contacts > 0  # the column's grains touch during the run


def test_grains_b200_from_xml_with_both_fixes(drive, tmp_path):
    """Spheres and boxes of two materials inserted at random in a box window
    (kept corners), on walls of a third material: the run completes, every
    grain stays inside the window's column, and the material ids of the
    contact laws are the map's."""
    from test_xml_cpu import MATERIALS_XML
    xml = MATERIALS_XML.replace("<Forces>", """<Forces>""").replace(
        "</Construction>",
        """  <TemporalSetting>
      <TimeInterval Start="0" End="1.9e-4" dt="1e-5"/>
      <TimeIntegration Type="FirstOrderExplicit"/>
    </TemporalSetting>
    <ContactForceModels>
      <ContactForceModel Type="Hooke"><Material materialA="steel" materialB="steel"/>
        <Parameters><kn>1e4</kn><en>0.7</en><etat>0</etat><muc>0.5</muc><kr>0</kr></Parameters>
      </ContactForceModel>
      <ContactForceModel Type="Hooke"><Material materialA="steel" materialB="glass"/>
        <Parameters><kn>2e4</kn><en>0.6</en><etat>0</etat><muc>0.4</muc><kr>0</kr></Parameters>
      </ContactForceModel>
      <ContactForceModel Type="Hooke"><Material materialA="glass" materialB="glass"/>
        <Parameters><kn>3e4</kn><en>0.5</en><etat>0</etat><muc>0.3</muc><kr>0</kr></Parameters>
      </ContactForceModel>
      <ContactForceModel Type="Hooke"><Material materialA="wall" materialB="steel"/>
        <Parameters><kn>1e4</kn><en>0.7</en><etat>0</etat><muc>0.5</muc><kr>0</kr></Parameters>
      </ContactForceModel>
      <ContactForceModel Type="Hooke"><Material materialA="wall" materialB="glass"/>
        <Parameters><kn>1e4</kn><en>0.7</en><etat>0</etat><muc>0.5</muc><kr>0</kr></Parameters>
      </ContactForceModel>
      <ContactForceModel Type="Hooke"><Material materialA="wall" materialB="wall"/>
        <Parameters><kn>1e4</kn><en>0.7</en><etat>0</etat><muc>0.5</muc><kr>0</kr></Parameters>
      </ContactForceModel>
    </ContactForceModels>
  </Construction>""")
    p = tmp_path / "fix.xml"
    p.write_text(xml)
    run("run", "b200", p, tmp_path / "b200.bin", "--fix-insertion")
    tr, kin, _ = grains_xml.read_state(tmp_path / "b200.bin")
    assert tr.shape == (5, 12) and np.isfinite(tr).all() and np.isfinite(kin).all()
    x = tr[:, 9:]
    assert np.all(x[:, :2] >= [0.0019, 0.0029]) and np.all(x[:, :2] <= [0.0181, 0.0171])
