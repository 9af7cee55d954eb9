"""The reference's output files, written from the device state (WrtDat / WrtDatWLL / WrtDat2).

Every row of every file is compared, as text, with the state the solver reports through
mps_get_state / mps_get_mirrors / mps_get_wall_flags formatted with the reference's format
strings (kernel.cu:161-276); pav is checked to be reset after a write (kernel.cu:289), and a
case directory runs end to end with ClcMPS's output cadence.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from mps_cuda_b200 import F32, F64, MPS, SceneDesc, dambreak, dambreak_params, files, select_device
from mps_cuda_b200 import _lib as L

pytestmark = pytest.mark.gpu

DESC = SceneDesc(l0=0.02, tank=(0.4, 0.2, 0.4), block=(8, 6, 10), jitter=0.01, seed=3)


def _solver(prec):
    select_device(0)
    sc = dambreak(DESC)
    rd = np.float64 if prec == F64 else np.float32
    p = dambreak_params(DESC, dt=2e-4, precision=prec)
    return MPS(p, sc["typ"], sc["pos"].astype(rd), sc["vel"].astype(rd), sc["nrm"].astype(rd)), sc


def _lines(path):
    with open(path) as f:
        return f.read().splitlines()


def _fluid_rows(st, fqc, prec):
    rows = []
    for i in np.nonzero(st["typ"] == L.FLD)[0]:
        v = st["vel"][:, i]
        if prec == F64:
            sp = float(np.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]))
            pv = float(st["pav"][i]) / fqc
        else:
            v = v.astype(np.float32)
            sp = float(np.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]))
            pv = float(np.float32(st["pav"][i]) / np.float32(fqc))
        vals = [*st["pos"][:, i], *v, sp, st["prs"][i], pv]
        rows.append(",".join("%f" % float(x) for x in vals))
    return rows


@pytest.mark.parametrize("prec", [F32, F64])
def test_output_files_match_the_state(tmp_path, prec):
    h, sc = _solver(prec)
    try:
        out = files.Output(h, str(tmp_path))
        # wall files at open (WrtDatWLL, file index 0)
        st = h.state()
        se = h.wall_flags()
        walls = np.nonzero(st["typ"] == L.WLL)[0]
        lines = _lines(tmp_path / "outputwall00000.csv")
        assert lines[0] == "Pos.x,Pos.y,Pos.z,Prs,pav,SE"
        assert lines[1:] == ["%f,%f,%f,%f,%f,%d" % (*st["pos"][:, i], 0.0, 0.0, se[i]) for i in walls]
        lines = _lines(tmp_path / "outputWLLvec00000.csv")
        assert lines[0] == "PosM.x,PosM.y,PosM.z,vec.x,vec.y,vec.z"
        rd = h.dtype
        nrm = sc["nrm"].astype(rd)
        assert lines[1:] == ["%f,%f,%f,%f,%f,%f" % (*st["pos"][:, i], *nrm[:, i]) for i in walls]

        h.step(12)
        st = h.state()
        m2 = h.mirrors(2)
        assert st["pav"][st["typ"] == L.FLD].any()
        out.write(1, 12.0)
        h.step(3)  # queued while the writer formats the files
        out.close()
        lines = _lines(tmp_path / "output00001.csv")
        assert lines[0] == "Pos.x,Pos.y,Pos.z,Vel.x,Vel.y,Vel.z,Vel,Prs,pav"
        assert lines[1:] == _fluid_rows(st, 12.0, prec)
        lines = _lines(tmp_path / "outputMRR00001.csv")
        assert lines[0] == "PosM.x,PosM.y,PosM.z,VelM,PrsM"
        assert len(m2["slot"]) > 0 and np.all(np.diff(m2["slot"]) > 0)
        assert lines[1:] == ["%f,%f,%f,%f,%f," % (*m2["pos"][:, k], 0.0, m2["prs"][k])
                             for k in range(len(m2["slot"]))]
    finally:
        h.close()


def test_write_resets_pav_and_restart_file(tmp_path):
    h, _ = _solver(F32)
    try:
        with files.Output(h, str(tmp_path)) as out:
            h.step(5)
            out.write(1, 5.0)
            st = h.state()
            assert not st["pav"].any()  # d_initialize_real_array(d_pav, 0), kernel.cu:289
            h.step(4)
            st = h.state()
            assert st["pav"][st["typ"] == L.FLD].any()
            out.restart()
        fl = np.nonzero(st["typ"] == L.FLD)[0]
        lines = _lines(tmp_path / "seitei.txt")
        assert lines[0] == str(len(fl))
        assert lines[1:] == ["%d %d %f %f %f %f %f %f %f" % (k, L.FLD, *st["pos"][:, i], 0, 0, 0, 0)
                             for k, i in enumerate(fl)]
        # the restart file reads back as an initial.txt of the fluid
        ph = files.physical(min=(0, 0, 0), max=DESC.tank, g=(0, 0, -9.8), fin_tim=1, output_time=1,
                            mach=10, courant=0.2, col_rat=0.2, dst_lmt_rat=0.9, knm_vsc=1e-6,
                            pcl_dst=DESC.l0)
        back = files.read_initial(str(tmp_path / "seitei.txt"), ph)
        assert back["typ"].tolist() == [L.FLD] * len(fl)
        np.testing.assert_allclose(back["pos"], st["pos"][:, fl], atol=1e-6)
    finally:
        h.close()


def test_errors_are_reported(tmp_path):
    h, _ = _solver(F32)
    try:
        o = C.c_void_p()
        rc = L.lib().mps_output_open(h.handle, str(tmp_path / "no" / "such").encode(), C.byref(o))
        assert rc == L.MPS_ERR_ARG and not o.value
        assert "cannot create" in L.lib().mps_last_error().decode()
        with files.Output(h, str(tmp_path)) as out:
            with pytest.raises(L.MPSError):
                out.write(1, 0.0)  # OPT_FQC must be positive
    finally:
        h.close()


def test_run_case_end_to_end(tmp_path):
    select_device(0)
    sc = dambreak(DESC)
    case = tmp_path / "case"
    os.makedirs(case)
    ph = files.physical(min=(0, 0, 0), max=DESC.tank, g=(0, 0, -9.80665), fin_tim=0.02,
                        output_time=0.005, mach=0.1, courant=0.2, col_rat=0.2, dst_lmt_rat=0.9,
                        knm_vsc=1e-6, pcl_dst=DESC.l0)
    files.write_physical(str(case / "MPS_physical.txt"), ph)
    files.write_initial(str(case / "initial.txt"), sc["typ"], sc["pos"], sc["nrm"])
    out = tmp_path / "vtk"
    res = files.run_case(str(case), str(out), F32, dt=2e-4)
    sched = list(files.output_schedule(2e-4, ph.output_time, ph.fin_tim))
    assert res["steps"] == sum(n for n, _ in sched) and res["files"] == len(sched) + 1
    names = sorted(os.listdir(out))
    for k in range(res["files"]):
        assert f"output{k:05d}.csv" in names and f"outputMRR{k:05d}.csv" in names
    assert "seitei.txt" in names and "outputwall00000.csv" in names
    # the fluid fell: the last file's mean z is below the first's
    z0 = np.loadtxt(out / "output00000.csv", delimiter=",", skiprows=1)[:, 2].mean()
    z1 = np.loadtxt(out / f"output{res['files'] - 1:05d}.csv", delimiter=",", skiprows=1)[:, 2].mean()
    assert z1 < z0


def test_output_of_a_two_scene_handle(tmp_path):
    """A batched handle writes the fluid of every scene, scene after scene in id order."""
    from mps_cuda_b200 import MPSBatch
    select_device(0)
    parts = [dambreak(DESC), dambreak(SceneDesc(l0=0.02, tank=(0.4, 0.2, 0.4), block=(6, 6, 6),
                                                 jitter=0.01, seed=9))]
    cat = lambda key: np.concatenate([p[key] for p in parts], axis=-1)
    counts = [p["typ"].shape[0] for p in parts]
    params = [dambreak_params(DESC, dt=2e-4, precision=F32)] * 2
    b = MPSBatch(params, cat("typ"), cat("pos").astype(np.float32), cat("vel").astype(np.float32),
                 cat("nrm").astype(np.float32), counts=counts)
    try:
        with files.Output(b, str(tmp_path)) as out:
            b.step(6)
            st = b.state()
            out.write(1, 6.0)
        lines = _lines(tmp_path / "output00001.csv")
        assert lines[1:] == _fluid_rows(st, 6.0, F32)
        assert len(lines) - 1 == int((st["typ"] == L.FLD).sum()) == 480 + 216
    finally:
        b.close()
