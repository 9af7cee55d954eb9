"""Scene generator, parameter helper and the C-ABI surface (no GPU needed)."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from mps_cuda_b200 import F32, F64, SceneDesc, configs, dambreak, dambreak_params, derive
from mps_cuda_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mps_b200.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(mps_\w+)\s*\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", L.library_path()], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (mps_\w+)", out))
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    # and the ctypes binding declares a signature for each
    assert sorted(L.SIGNATURES) == syms
    lib = L.lib()
    for s in syms:
        assert hasattr(lib, s)


def test_binding_constants_equal_the_header_enums():
    """Every MPS_OPT_*, MPS_STAGE_* and MPS_K_* value the Python binding uses is the header's."""
    txt = open(HEADER).read()
    enums = {m[0]: int(m[1]) for m in re.findall(r"\b(MPS_(?:OPT|STAGE|K)_\w+)\s*=\s*(\d+)", txt)}
    assert len(enums) >= 20
    for name, value in enums.items():
        py = name[len("MPS_"):]
        if name == "MPS_K_COUNT":
            assert len(L.KERNEL_GROUPS) == value
        elif hasattr(L, py):
            assert getattr(L, py) == value, name
    for name in ("MPS_OPT_REGISTER_BOUND", "MPS_OPT_CANDIDATE_BATCH", "MPS_OPT_STAGING"):
        assert getattr(L, name[len("MPS_"):]) == enums[name]


def test_status_strings():
    lib = L.lib()
    for code in range(9):
        assert lib.mps_status_string(code)
    assert lib.mps_status_string(99) == b"unknown status"


def test_argument_errors_without_gpu():
    lib = L.lib()
    p = L.mps_params()
    inf = L.mps_info()
    assert lib.mps_derive(C.byref(p), C.byref(inf)) == L.MPS_ERR_ARG  # l0 = 0
    assert b"positive" in lib.mps_last_error()
    d = SceneDesc(0.02, (0.4, 0.2, 0.4), (4, 4, 4)).c()
    typ = np.empty(10, np.int8)
    buf = np.empty(30)
    n = C.c_int32()
    rc = lib.mps_scene_dambreak(C.byref(d), 10, typ.ctypes.data_as(L.c_int8_p),
                                buf.ctypes.data_as(L.c_double_p), buf.ctypes.data_as(L.c_double_p),
                                buf.ctypes.data_as(L.c_double_p), C.byref(n))
    assert rc == L.MPS_ERR_ARG and n.value > 10
    assert lib.mps_step(None, 1) == L.MPS_ERR_ARG
    assert lib.mps_destroy(None) == L.MPS_OK


@pytest.mark.parametrize("prec", [F32, F64])
def test_grid_too_large_for_int32_cells_is_rejected_before_any_device_use(prec):
    """A domain whose bucket grid does not fit int32 fine-cell indices is refused by the host
    arithmetic (64-bit bucket counts), by mps_derive, mps_create and the no-allocation
    bucket build alike, before any device is touched (this runs without a GPU)."""
    lib = L.lib()
    desc = SceneDesc(0.02, (0.4, 0.2, 0.4), (2, 2, 2))
    sc = dambreak(desc)
    for ext in ((2000.0, 2000.0, 2000.0), (1e9, 1.0, 1.0)):
        p = dambreak_params(desc, precision=prec, max=ext)
        inf = L.mps_info()
        assert lib.mps_derive(C.byref(p), C.byref(inf)) == L.MPS_ERR_OVERFLOW
        assert b"bucket" in lib.mps_last_error()
        h = C.c_void_p()
        n = sc["typ"].shape[0]
        rd = np.float64 if prec == F64 else np.float32
        arr = [np.ascontiguousarray(sc[k], rd) for k in ("pos", "vel", "nrm")]
        rc = lib.mps_create(C.byref(p), n, sc["typ"].ctypes.data_as(L.c_int8_p),
                            *(a.ctypes.data_as(C.c_void_p) for a in arr), C.byref(h))
        assert rc == L.MPS_ERR_OVERFLOW and not h.value
        start = np.zeros(4, np.int32)  # host memory: the call must return before using it
        rc = lib.mps_bucket_build_noalloc(C.byref(p), 0, None, None, None, None,
                                          start.ctypes.data_as(C.c_void_p), None)
        assert rc == L.MPS_ERR_OVERFLOW
        assert np.all(start == 0)
    # a grid that fits is still accepted
    p = dambreak_params(desc, precision=prec)
    assert lib.mps_derive(C.byref(p), C.byref(L.mps_info())) == L.MPS_OK


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device status")
def test_create_without_device_reports_nodevice():
    desc = SceneDesc(0.02, (0.4, 0.2, 0.4), (2, 2, 2))
    sc = dambreak(desc)
    p = dambreak_params(desc, precision=F64)
    h = C.c_void_p()
    rc = L.lib().mps_create(C.byref(p), sc["typ"].shape[0], sc["typ"].ctypes.data_as(L.c_int8_p),
                            sc["pos"].ctypes.data_as(C.c_void_p), sc["vel"].ctypes.data_as(C.c_void_p),
                            sc["nrm"].ctypes.data_as(C.c_void_p), C.byref(h))
    assert rc == L.MPS_ERR_NODEVICE and not h.value


def test_dambreak_counts_and_layout():
    desc, _, _ = configs.WORKLOADS["dambreak_l0.02_6k"]
    sc = dambreak(desc)
    typ, pos, nrm = sc["typ"], sc["pos"], sc["nrm"]
    nf = int((typ == 0).sum())
    assert nf == 20 * 10 * 30
    nx, ny, nz = 50, 10, 40
    assert int((typ == 1).sum()) == 2 * ny * nz + 2 * nx * nz + nx * ny
    assert np.all(typ[:nf] == 0) and np.all(typ[nf:] == 1)
    w = typ == 1
    # unit normals pointing into the tank; every wall particle on its face plane
    assert np.allclose(np.linalg.norm(nrm[:, w], axis=0), 1.0)
    assert np.all(nrm[:, ~w] == 0)
    for ax, L_ in enumerate((1.0, 0.2, 0.8)):
        on = w & (np.abs(nrm[ax]) == 1)
        plane = np.where(nrm[ax, on] > 0, 0.0, L_)
        assert np.allclose(pos[ax, on], plane)
    # in-plane positions at half-integer multiples of l0
    frac = (pos[:, w] / 0.02) % 1.0
    onplane = np.abs(nrm[:, w]) == 1
    assert np.allclose(frac[~onplane], 0.5)


def test_dambreak_jitter_is_bounded_and_seeded():
    desc = SceneDesc(0.02, (0.4, 0.2, 0.4), (5, 4, 6), seed=7)
    a, b = dambreak(desc), dambreak(desc)
    assert np.array_equal(a["pos"], b["pos"])
    c = dambreak(SceneDesc(0.02, (0.4, 0.2, 0.4), (5, 4, 6), seed=8))
    assert not np.array_equal(a["pos"], c["pos"])
    nf = 5 * 4 * 6
    base = (np.round(a["pos"][:, :nf] / 0.02 - 0.5) + 0.5) * 0.02
    dev = np.abs(a["pos"][:, :nf] - base)
    assert dev.max() <= 0.01 * 0.02 + 1e-15 and dev.max() > 0.005 * 0.02


def test_initial_velocity_distribution():
    desc, _, _ = configs.WORKLOADS["adjoint_l0.01_48k"]
    sc = dambreak(desc)
    v = sc["vel"][:, sc["typ"] == 0]
    assert v.shape[1] == 48000
    assert abs(v.mean()) < 2e-3 and abs(v.std() - 0.05) < 1e-3


def test_params_dambreak():
    desc = SceneDesc(0.02, (1.0, 0.2, 0.8), (20, 10, 30))
    p = dambreak_params(desc, snd=20.0, dt=2e-4, nu=1e-6, precision=F32)
    H = 29 * 0.02
    assert p.umax == pytest.approx(np.sqrt(2 * 9.81 * H))
    assert p.pmax == pytest.approx(1000 * 9.81 * H)
    assert list(p.g) == [0.0, 0.0, -9.81] and p.rho == 1000.0 and p.snd == 20.0
    inf = derive(p)
    assert inf.prs_coef == pytest.approx(400.0 / inf.n0_grad, rel=1e-6)
    assert inf.rlim2 == pytest.approx((0.9 * 0.02) ** 2, rel=1e-6)
    assert inf.col == pytest.approx(1.2)


def test_batched_scene_draws():
    scenes = configs.batched_scenes()
    assert len(scenes) == 64
    counts = []
    for desc, dt in scenes:
        nf = int(np.prod(desc.block))
        assert 2000 <= nf <= 60000
        assert desc.l0 in (0.01, 0.015, 0.02)
        assert 1.0 <= desc.tank[0] <= 1.6
        assert 0 < dt < 0.25 * desc.l0 / 20.0
        counts.append(nf)
    assert len(set(counts)) > 30  # uneven sizes
    again = configs.batched_scenes()
    assert [d.block for d, _ in again] == [d.block for d, _ in scenes]


def test_cpp_facade_compiles_links_and_runs(tmp_path):
    """include/mps_b200.hpp: a ClcMPS-style loop builds against libmps_b200.so. It writes the
    scene as a case directory and reads it back with RdDat (host only); without a GPU it then
    stops at mps_create with MPS_ERR_NODEVICE, with one it runs 22 steps and writes the
    output files."""
    lib = L.library_path()
    exe = tmp_path / "clcmps_loop"
    src = os.path.join(ROOT, "tests", "cpp", "clcmps_loop.cpp")
    subprocess.run(["/usr/bin/g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), src,
                    "-L", os.path.dirname(lib), "-lmps_b200", "-Wl,-rpath," + os.path.dirname(lib),
                    "-o", str(exe)], check=True, capture_output=True)
    res = subprocess.run([str(exe), str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "case: " in res.stdout
