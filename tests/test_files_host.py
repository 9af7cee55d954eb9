"""The reference's input files and parameter derivation (host code, no GPU needed).

MPS_physical.txt and initial.txt are parsed as RdDat parses them (kernel.cu:4-131): every
number as a float, the domain padded by 3.1 l0 with strict bounds, wall normals negated;
SetPara's derived parameters (kernel.cu:396-415) and ClcMPS's output cadence
(kernel.cu:1872-1943) are restated here in numpy and compared.
"""
from __future__ import annotations

import numpy as np
import pytest

from mps_cuda_b200 import F32, F64, SceneDesc, dambreak, files
from mps_cuda_b200 import _lib as L

f32 = np.float32


def _ph(**kw):
    base = dict(min=(0.0, 0.0, 0.0), max=(1.0, 0.2, 0.8), g=(0.0, 0.0, -9.80665), fin_tim=1.5,
                output_time=0.02, mach=10.0, courant=0.2, col_rat=0.2, dst_lmt_rat=0.9,
                knm_vsc=1.0e-6, pcl_dst=0.02)
    base.update(kw)
    return files.physical(**base)


def _fields(ph):
    return [*ph.min, *ph.max, *ph.g, ph.fin_tim, ph.output_time, ph.mach, ph.courant,
            ph.col_rat, ph.dst_lmt_rat, ph.knm_vsc, ph.pcl_dst]


def test_physical_round_trip_reads_floats(tmp_path):
    ph = _ph(knm_vsc=1.234567891e-6, pcl_dst=0.0123456789)
    p = tmp_path / "MPS_physical.txt"
    files.write_physical(str(p), ph)
    back = files.read_physical(str(p))
    assert _fields(back) == [float(f32(v)) for v in _fields(ph)]


def test_physical_reader_is_whitespace_agnostic(tmp_path):
    p = tmp_path / "MPS_physical.txt"
    vals = [-0.1, -0.2, -0.3, 1, 2, 3, 0, -9.8, 0, 2.0, 0.05, 10, 0.2, 0.2, 0.9, 1e-6, 0.01]
    p.write_text(" ".join(str(v) for v in vals[:5]) + "\n\n" + "\t".join(str(v) for v in vals[5:]))
    assert _fields(files.read_physical(str(p))) == [float(f32(v)) for v in vals]


def test_physical_reader_rejects_short_file(tmp_path):
    p = tmp_path / "MPS_physical.txt"
    p.write_text("0 0 0\n1 1 1\n")
    with pytest.raises(L.MPSError) as e:
        files.read_physical(str(p))
    assert e.value.code == L.MPS_ERR_ARG
    with pytest.raises(L.MPSError):
        files.read_physical(str(tmp_path / "missing.txt"))


def _write_rows(path, rows):
    with open(path, "w") as f:
        f.write(f"{len(rows)}\n")
        for k, (t, x, y, z, nx, ny, nz) in enumerate(rows):
            f.write(f"{k} {t} {x} {y} {z} {nx} {ny} {nz} 0\n")


def test_initial_reader_follows_rddat(tmp_path):
    ph = _ph()
    l0 = f32(ph.pcl_dst)
    lo_x = f32(0.0 - 3.1 * float(l0))  # MINc.x = real(MIN.x - 3.1 * PCL_DST) in double, kernel.cu:26
    rows = [
        (L.FLD, 0.5, 0.1, 0.3, 0.7, 0.7, 0.7),      # fluid: normal ignored
        (L.WLL, 0.5, 0.1, 0.0, 0.0, 0.0, -1.0),     # wall: inward normal = -file normal
        (L.OBJ, 0.2, 0.1, 0.4, 1.0, 0.0, 0.0),
        (L.OBJ2, 0.3, 0.1, 0.4, 0.0, 1.0, 0.0),
        (L.FLD, 5.0, 0.1, 0.3, 0, 0, 0),            # outside the padded domain: dropped
        (L.WLL, float(lo_x), 0.1, 0.3, 1, 0, 0),    # on the padded bound: dropped (strict)
        (L.WLL, float(np.nextafter(lo_x, f32(1))), 0.1, 0.3, 1, 0, 0),  # just inside: kept
        (L.FLD, 0.123456789, 0.1, 0.3, 0, 0, 0),    # read as a float
    ]
    p = tmp_path / "initial.txt"
    _write_rows(p, [(t, repr(x) if isinstance(x, float) else x, y, z, nx, ny, nz)
                    for t, x, y, z, nx, ny, nz in rows])
    sc = files.read_initial(str(p), ph)
    keep = [0, 1, 2, 3, 6, 7]
    assert sc["typ"].tolist() == [rows[k][0] for k in keep]
    want_pos = np.array([[float(f32(rows[k][1 + d])) for k in keep] for d in range(3)])
    np.testing.assert_array_equal(sc["pos"], want_pos)
    want_nrm = np.array([[0.0 if rows[k][0] == L.FLD else -float(f32(rows[k][4 + d]))
                          for k in keep] for d in range(3)])
    np.testing.assert_array_equal(sc["nrm"], want_nrm)
    assert sc["pos"].shape == (3, 6) and not sc["vel"].any()


def test_initial_reader_sizes_and_errors(tmp_path):
    ph = _ph()
    p = tmp_path / "initial.txt"
    _write_rows(p, [(L.FLD, 0.1 * k, 0.1, 0.1, 0, 0, 0) for k in range(5)])
    import ctypes as C
    n = C.c_int32(-1)
    rc = L.lib().mps_read_initial(str(p).encode(), C.byref(ph), 0, None, None, None, C.byref(n))
    assert rc == L.MPS_ERR_ARG and n.value == 5  # sizing call
    typ = np.zeros(4, np.int8)
    pos = np.zeros(12)
    nrm = np.zeros(12)
    rc = L.lib().mps_read_initial(str(p).encode(), C.byref(ph), 4, typ.ctypes.data_as(L.c_int8_p),
                                  pos.ctypes.data_as(L.c_double_p), nrm.ctypes.data_as(L.c_double_p),
                                  C.byref(n))
    assert rc == L.MPS_ERR_ARG and n.value == 5  # capacity too small
    # a larger capacity packs the SoA arrays to stride n
    cap = 9
    typ = np.full(cap, 7, np.int8)
    pos = np.full(3 * cap, -1.0)
    nrm = np.full(3 * cap, -1.0)
    rc = L.lib().mps_read_initial(str(p).encode(), C.byref(ph), cap, typ.ctypes.data_as(L.c_int8_p),
                                  pos.ctypes.data_as(L.c_double_p), nrm.ctypes.data_as(L.c_double_p),
                                  C.byref(n))
    assert rc == L.MPS_OK and n.value == 5
    np.testing.assert_array_equal(pos[:15].reshape(3, 5)[0], [float(f32(0.1 * k)) for k in range(5)])
    np.testing.assert_array_equal(pos[:15].reshape(3, 5)[1], [float(f32(0.1))] * 5)
    # a truncated row is an error, not a silent stop
    p.write_text("3\n0 0 0.1 0.1 0.1 0 0 0 0\n1 0 0.2 0.2\n")
    with pytest.raises(L.MPSError):
        files.read_initial(str(p), ph)


def test_initial_round_trip_of_a_dambreak_scene(tmp_path):
    desc = SceneDesc(l0=0.02, tank=(0.3, 0.1, 0.2), block=(5, 3, 4), jitter=0.01, seed=3)
    sc = dambreak(desc)
    ph = _ph(max=(0.3, 0.1, 0.2))
    p = tmp_path / "initial.txt"
    files.write_initial(str(p), sc["typ"], sc["pos"], sc["nrm"])
    back = files.read_initial(str(p), ph)
    assert back["typ"].tolist() == sc["typ"].tolist()
    np.testing.assert_array_equal(back["pos"], sc["pos"].astype(np.float32).astype(np.float64))
    np.testing.assert_array_equal(back["nrm"], sc["nrm"].astype(np.float32).astype(np.float64))


def test_params_from_physical_matches_setpara(tmp_path):
    desc = SceneDesc(l0=0.02, tank=(0.3, 0.1, 0.2), block=(5, 3, 4))
    sc = dambreak(desc)
    for g, ax in (((0.0, 0.0, -9.80665), 2), ((0.0, -9.8, 0.0), 1)):
        ph = _ph(g=g, mach=8.0)
        for prec in (F32, F64):
            p = files.params_from_physical(ph, sc["typ"], sc["pos"], prec)
            fl = sc["typ"] == L.FLD
            H = sc["pos"][ax][fl].max() - sc["pos"][ax][fl].min()
            gg = abs(g[ax])
            umax = np.sqrt(2 * gg * H)
            snd = umax / ph.mach
            assert p.umax == pytest.approx(umax, rel=1e-15)
            assert p.snd == pytest.approx(snd, rel=1e-15)
            assert p.pmax == pytest.approx(1000.0 * gg * H, rel=1e-15)
            assert p.dt == pytest.approx(ph.pcl_dst / (umax + snd), rel=1e-15)
            assert p.rho == 1000.0 and p.precision == prec
            assert list(p.g) == list(ph.g) and p.knm_vsc == ph.knm_vsc
            assert list(p.min) == list(ph.min) and list(p.max) == list(ph.max)
            assert (p.col_rat, p.dst_lmt_rat, p.pcl_dst) == (ph.col_rat, ph.dst_lmt_rat, ph.pcl_dst)


def test_load_case_reads_a_case_directory(tmp_path):
    desc = SceneDesc(l0=0.02, tank=(0.3, 0.1, 0.2), block=(5, 3, 4))
    sc = dambreak(desc)
    ph = _ph(max=(0.3, 0.1, 0.2))
    files.write_physical(str(tmp_path / "MPS_physical.txt"), ph)
    files.write_initial(str(tmp_path / "initial.txt"), sc["typ"], sc["pos"], sc["nrm"])
    p, back, ph2 = files.load_case(str(tmp_path), F64)
    assert back["typ"].shape == sc["typ"].shape and p.precision == F64
    assert p.dt > 0 and p.pmax > 0 and ph2.output_time == pytest.approx(0.02, rel=1e-7)


def _clcmps_schedule(dt, output_time, fin_tim):
    """ClcMPS's loop (kernel.cu:1887-1941) stepped one step at a time in float arithmetic:
    the step count at which each file after the first is written."""
    outtime, tim, step, out = f32(0), f32(0), 0, []
    dt, output_time, fin_tim = f32(dt), f32(output_time), f32(fin_tim)
    while True:
        if outtime >= output_time:
            outtime = f32(outtime - output_time)
            out.append(step)
            if tim >= fin_tim:
                return out
        step += 1
        outtime = f32(outtime + dt)
        tim = f32(tim + dt)


@pytest.mark.parametrize("dt,out_t,fin", [(2e-4, 0.02, 0.1), (1.7e-4, 0.01, 0.05),
                                          (3e-3, 0.005, 0.03)])
def test_output_schedule_matches_clcmps(dt, out_t, fin):
    want = _clcmps_schedule(dt, out_t, fin)
    got = np.cumsum([n for n, _ in files.output_schedule(dt, out_t, fin)]).tolist()
    assert got == want
    flags = [last for _, last in files.output_schedule(dt, out_t, fin)]
    assert flags[-1] and not any(flags[:-1])
    assert len(list(files.output_schedule(dt, out_t, fin, max_files=2))) == min(2, len(want))
    with pytest.raises(ValueError):
        list(files.output_schedule(dt, 0.0, fin))
