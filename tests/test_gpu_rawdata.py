"""RawData post-processing output of the engine (gb_rawdata_*):

* byte for byte against the reference's own RawDataPostProcessingWriter
  (RawDataPostProcessingWriter.cpp:63-231, compiled into oracle/_ref and run
  by the harness on the same state);
* against the format restated here (realToString, GrainsUtils.hh:33-44): per
  component file one line per save, the time then every particle's value
  then every obstacle's (origin, zero velocities), "%.6e" with a zero
  printed as "0"; and the coordination-number option."""
import ctypes as C
import math

import numpy as np
import pytest

from grains3dgpu_b200 import abi, scenes

pytestmark = pytest.mark.gpu

FILES = ["position_x", "position_y", "position_z",
         "translational_velocity_x", "translational_velocity_y", "translational_velocity_z",
         "angular_velocity_x", "angular_velocity_y", "angular_velocity_z"]


def real(v):
    v = float(v)
    if v == 0.0:
        return "-0" if math.copysign(1.0, v) < 0 else "0"
    return "%.6e" % v


def expected_lines(time, tr, kin, obs_tr):
    cols = [tr[:, 9], tr[:, 10], tr[:, 11], kin[:, 0], kin[:, 1], kin[:, 2],
            kin[:, 3], kin[:, 4], kin[:, 5]]
    out = []
    for k, c in enumerate(cols):
        obs = obs_tr[:, 9 + k] if k < 3 else np.zeros(obs_tr.shape[0])
        out.append(" ".join([real(time)] + [real(v) for v in c] + [real(v) for v in obs]))
    return out


@pytest.mark.parametrize("precision", [abi.GB_MIXED, abi.GB_FP64])
@pytest.mark.parametrize("coordination", [False, True])
def test_rawdata_files(gb, tmp_path, precision, coordination):
    scene = scenes.sphere_bed(n=60)  # lattice neighbours overlap from the start
    s = scenes.System(gb, scene, precision=precision)
    w = s.rawdata(str(tmp_path), "run", coordination=coordination)
    want = {f: [] for f in FILES}
    cn_want = []
    dt = scene.config["dt"]
    for k, nsteps in enumerate((0, 30, 30)):
        if nsteps:
            assert s.step(nsteps) in (abi.GB_OK, abi.GB_E_OUT_OF_DOMAIN)
        t = dt * 30 * k
        w.write(t)
        lines = expected_lines(t, s.transforms(), s.velocities(), scene.obstacle_transforms)
        for f, line in zip(FILES, lines):
            want[f].append(line)
        if coordination:
            counts = np.zeros(scene.n, np.int64)
            if nsteps:
                pairs = s.dump(abi.GB_DUMP_CONTACT_PAIRS).astype(np.int64)
                both = set(map(tuple, pairs.tolist()))
                ordered = all((b, a) in both for a, b in both)  # each pair listed both ways
                np.add.at(counts, pairs[:, 0], 1)
                if not ordered:
                    np.add.at(counts, pairs[:, 1], 1)
            cn_want.append(" ".join([real(t)] + [str(int(c)) for c in counts]))
        else:
            cn_want.append("")
    w.close()
    for f in FILES:
        got = (tmp_path / f"run_{f}.dat").read_text().split("\n")
        assert got[-1] == ""
        assert got[:-1] == want[f], f
    got = (tmp_path / "run_coordinationNumber.dat").read_text().split("\n")
    assert got[:-1] == cn_want
    assert (tmp_path / "run_particleType.dat").read_text() == "\n"
    if coordination:
        assert any(int(x) > 0 for x in cn_want[-1].split()[1:])  # the column has contacts
    s.close()


def test_rawdata_files_equal_the_reference_writer(gb, reference, tmp_path):
    """The engine (FP64) and the reference harness hold the same states (the
    harness's, set into the engine before each save); each writes its three
    saves with its own writer; every file is byte-identical."""
    scene = scenes.superquadric_column(n=90, pitch=2.05e-3)
    r = scenes.System(reference, scene)
    g = scenes.System(gb, scene, precision=abi.GB_FP64)
    write = reference.lib.ref_rawdata_write
    write.restype = C.c_int
    write.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_double, C.c_int32]
    close = reference.lib.ref_rawdata_close
    close.restype = C.c_int
    close.argtypes = [C.c_void_p]
    (tmp_path / "ref").mkdir()
    (tmp_path / "gb").mkdir()
    w = g.rawdata(str(tmp_path / "gb"), "run")
    dt = scene.config["dt"]
    for k, nsteps in enumerate((0, 7, 7)):
        if nsteps:
            r.step(nsteps)
        g.set_transforms(r.transforms())
        g.set_velocities(r.velocities())
        t = dt * 7 * k
        assert write(r.ctx, str(tmp_path / "ref").encode(), b"run", t, int(k == 0)) == 0
        w.write(t)
    assert close(r.ctx) == 0
    w.close()
    names = sorted(p.name for p in (tmp_path / "ref").iterdir())
    assert names == sorted(p.name for p in (tmp_path / "gb").iterdir())
    assert len(names) == 11
    for name in names:
        a = (tmp_path / "ref" / name).read_bytes()
        b = (tmp_path / "gb" / name).read_bytes()
        assert a == b, name
    assert len((tmp_path / "ref" / "run_position_z.dat").read_bytes()) > 90 * 3 * 12
    g.close()
    r.close()
