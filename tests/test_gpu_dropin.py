"""Drop-in check through the reference's own C++ interface.

oracle/_ref/adapter_drive (built by oracle/Makefile from the reference
sources and oracle/ref/adapter_drive.cpp) steps one packing of 392
superquadrics in a closed box twice -- with the reference's
ComponentManagerCPU and with ComponentManagerB200
(include/grains_b200_component_manager.hh) -- both behind
ComponentManager<double>* and fed the reference's RigidBody, LinkedCell,
HookeContactForceModel and FirstOrderExplicit objects in GrainsCPU::simulate's
call order.  The program checks equal contact counts, transforms within 1e-12
and velocities within 1e-7 of the largest.
"""
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "adapter_drive")


def test_component_manager_b200_matches_reference_cpu(gb):
    if not os.path.exists(EXE):
        pytest.skip("oracle/_ref/adapter_drive not built (needs the reference sources)")
    out = subprocess.run([EXE, "40"], capture_output=True, text=True, timeout=600)
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert out.returncode == 0, line
    assert line["contacts_cpu"] == line["contacts_gpu"] > 0
