"""Known-answer tests of the arithmetic the step is built from.

Independent restatements in Python (IEEE double via float, IEEE single via numpy.float32)
of the reference's formulas, compared with the library's derived constants (mps_derive,
host only) and with the oracle: weights (const.cuh:45-46), lattice sums n0 / lmd /
n0_grad (kernel.cu:336-366), bucket index (kernel.cu:521-524), face and corner mirror
reflections (kernel.cu:822-829, 847-886), ChkPcl (kernel.cu:481-513) and the EOS clamps
(kernel.cu:1389-1406).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from mps_cuda_b200 import F32, F64, F32_N64, SceneDesc, dambreak_params, derive
from oracle.oracle import Oracle, params_from


def wei(d, re):
    return (re / d + d / re) - 2.0


def wei_grad(d, re):
    return re / d - d / re


def lattice_sums(l0, T):
    """SetPara's loops (kernel.cu:341-366) in arithmetic type T."""
    l0 = T(l0)
    r, rp = l0 * T(3.1), l0 * T(2.1)
    r2, rp2 = r * r, rp * rp
    n0 = n0g = lmd = lmdg = T(0)
    cnt = 0
    for ix in range(-10, 10):
        for iy in range(-10, 10):
            for iz in range(-10, 10):
                x, y, z = l0 * T(ix), l0 * T(iy), l0 * T(iz)
                d2 = x * x + y * y + z * z
                if d2 == T(0):
                    continue
                d = T(math.sqrt(d2)) if T is float else np.sqrt(d2)
                if d2 < rp2:
                    n0g += (rp / d) - (d / rp)
                    lmdg += d2 * ((rp / d) - (d / rp))
                    cnt += 1
                if d2 < r2:
                    n0 += ((r / d) + (d / r)) - T(2)
                    lmd += d2 * (((r / d) + (d / r)) - T(2))
    return {"n0": n0, "lmd": lmd / n0, "n0_grad": n0g, "lmd_grad": lmdg / n0g, "numn0_grad": cnt,
            "r": r, "rp": rp}


def test_weights():
    re = 0.062
    assert wei(re, re) == 0.0
    assert wei_grad(re, re) == 0.0
    assert wei(0.5 * re, re) == pytest.approx(2.0 + 0.5 - 2.0)
    assert wei_grad(0.5 * re, re) == pytest.approx(2.0 - 0.5)


@pytest.mark.parametrize("l0", [0.02, 0.01, 0.005, 0.0025])
def test_lattice_constants_fp64(l0):
    desc = SceneDesc(l0, (1.0, 0.2, 0.8), (4, 4, 4))
    info = derive(dambreak_params(desc, precision=F64))
    ref = lattice_sums(l0, float)
    for k in ("n0", "lmd", "n0_grad", "lmd_grad", "r", "rp"):
        assert getattr(info, k) == ref[k], k
    assert info.numn0_grad == ref["numn0_grad"] == 32


@pytest.mark.parametrize("l0", [0.02, 0.005])
def test_lattice_constants_fp32(l0):
    desc = SceneDesc(l0, (1.0, 0.2, 0.8), (4, 4, 4))
    info = derive(dambreak_params(desc, precision=F32))
    ref = lattice_sums(l0, np.float32)
    for k in ("n0", "lmd", "n0_grad", "lmd_grad", "r", "rp"):
        assert np.float32(getattr(info, k)) == ref[k], k


@pytest.mark.parametrize("prec", [F32, F64, F32_N64])
def test_derive_equals_oracle(prec):
    desc = SceneDesc(0.02, (1.0, 0.2, 0.8), (20, 10, 30))
    p = dambreak_params(desc, precision=prec)
    info = derive(p)
    dty = np.float64 if prec == F64 else np.float32
    typ = np.array([0], np.int8)
    o = Oracle(params_from(p), typ, np.full((3, 1), 0.1, dty), np.zeros((3, 1), dty),
               np.zeros((3, 1), dty))
    oi = o.info()
    keys = ["n0", "lmd", "n0_grad", "lmd_grad", "r", "rp", "db", "dbinv", "rlim2", "col"]
    if prec != F32_N64:  # the mixed mode reports the double Prs_coef its EOS uses
        keys.append("prs_coef")
    for k in keys:
        assert getattr(info, k) == oi[k], k
    assert (info.nbx, info.nby, info.nbz) == (oi["nbx"], oi["nby"], oi["nbz"]) == (21, 8, 17)
    for d, ax in enumerate("xyz"):
        assert info.minc[d] == oi[f"minc_{ax}"]
        assert info.maxc[d] == oi[f"maxc_{ax}"]


def test_bucket_grid_dimensions():
    # AlcBkt: nB = (int)((MAX - MIN) / DB) + 3 on the padded domain (kernel.cu:317-319)
    for l0, tank, want in ((0.02, (1.0, 0.2, 0.8), (21, 8, 17)),
                           (0.005, (1.6, 0.2, 0.8), (108, 17, 56))):
        info = derive(dambreak_params(SceneDesc(l0, tank, (1, 1, 1)), precision=F32))
        assert (info.nbx, info.nby, info.nbz) == want


def _one_particle_oracle(prec, fluid, walls, normals, l0=0.02, tank=(0.4, 0.4, 0.4)):
    desc = SceneDesc(l0, tank, (1, 1, 1))
    p = params_from(dambreak_params(desc, precision=prec))
    dty = np.float64 if prec == F64 else np.float32
    pos = np.concatenate([np.array(fluid, np.float64).reshape(-1, 3),
                          np.array(walls, np.float64).reshape(-1, 3)]).T.astype(dty)
    nrm = np.concatenate([np.zeros((len(fluid), 3)),
                          np.array(normals, np.float64).reshape(-1, 3)]).T.astype(dty)
    typ = np.array([0] * len(fluid) + [1] * len(walls), np.int8)
    o = Oracle(p, typ, pos, np.zeros_like(pos), nrm)
    return o, typ


@pytest.mark.parametrize("prec", [F32, F64])
def test_bucket_index(prec):
    dt = np.float64 if prec == F64 else np.float32
    desc = SceneDesc(0.02, (0.4, 0.4, 0.4), (1, 1, 1))
    info = derive(dambreak_params(desc, precision=prec))
    pts = np.array([[0.0, 0.0, 0.0], [0.2, 0.1, 0.3], [0.061, 0.062, 0.063], [0.399, 0.001, 0.25]])
    o, _ = _one_particle_oracle(prec, pts, [], [])
    cell = o.diag()["cell"]
    minc = np.array(info.minc, dt)
    dbinv = dt(info.dbinv)
    for k, x in enumerate(pts.astype(dt)):
        ix, iy, iz = (int((x[d] - minc[d]) * dbinv) + 1 for d in range(3))
        assert cell[k] == iz * info.nbx * info.nby + iy * info.nbx + ix


@pytest.mark.parametrize("prec", [F32, F64])
def test_single_wall_face_mirror(prec):
    """A fluid particle above a flat floor gets one mirror, reflected through z = 0."""
    fl = [[0.2, 0.2, 0.013]]
    floor = [[0.2 + dx, 0.2 + dy, 0.0] for dx in (-0.02, 0.0, 0.02) for dy in (-0.02, 0.0, 0.02)]
    o, _ = _one_particle_oracle(prec, fl, floor, [[0, 0, 1]] * len(floor))
    o.phase(2)
    o.phase(3)
    m = o.mirrors()
    assert list(m["slot"]) == [0]
    x = np.array(fl[0])
    np.testing.assert_allclose(m["pos"][:, 0], [x[0], x[1], -x[2]], atol=1e-6)
    o.phase(4)  # the cull keeps a mirror on the far side of the wall
    assert len(o.mirrors()["slot"]) == 1


@pytest.mark.parametrize("prec", [F32, F64])
def test_corner_mirror_two_edges(prec):
    """Near the edge of floor z=0 and wall x=0: two face mirrors and one corner mirror."""
    l0 = 0.02
    fl = [[0.03, 0.2, 0.025]]
    walls, normals = [], []
    for y in (0.19, 0.21):
        for k in range(3):  # wall x=0 rows at z = (k+1/2) l0, floor rows at x = (k+1/2) l0
            walls.append([0.0, y, (k + 0.5) * l0]); normals.append([1, 0, 0])
            walls.append([(k + 0.5) * l0, y, 0.0]); normals.append([0, 0, 1])
    o, typ = _one_particle_oracle(prec, fl, walls, normals)
    w = o.wall_flags()
    edge = w[typ == 1] == 1
    # only the first row of each face (distance l0/sqrt(2) to the other face) is Edge
    assert edge.sum() == 4
    o.phase(2)
    o.phase(3)
    m = o.mirrors()
    assert sorted(m["slot"] % 10) == [0, 1, 2]
    x = np.array(fl[0])
    pts = m["pos"].T.astype(np.float64)
    expect_faces = [[-x[0], x[1], x[2]], [x[0], x[1], -x[2]]]
    for e in expect_faces:
        assert np.abs(pts - e).max(1).min() < 1e-6
    # corner plane: normal (1,0,1)/sqrt2 through the first Edge row (x + z = l0/2)
    n = np.array([1.0, 0.0, 1.0]) / math.sqrt(2)
    d = (x - np.array([0.0, 0.0, 0.5 * l0])) @ n
    corner = x - 2 * d * n
    assert np.abs(pts[m["slot"] % 10 == 2][0] - corner).max() < 1e-6


@pytest.mark.parametrize("prec", [F32, F64])
def test_chkpcl_clamps_speed_and_deletes(prec):
    dt = np.float64 if prec == F64 else np.float32
    fl = [[0.2, 0.2, 0.2], [0.1, 0.1, 0.1]]
    o, typ = _one_particle_oracle(prec, fl, [], [])
    st = o.state()
    umax = math.sqrt(2 * 9.81 * 0.0)  # one-particle block: H = 0 -> umax = 0
    vel = st["vel"].copy()
    vel[:, 0] = [3.0, 4.0, 0.0]
    pos = st["pos"].copy()
    pos[:, 1] = [0.5, 0.1, 0.1]  # outside the tank
    o.set_state(typ=st["typ"], pos=pos, vel=vel, acc=st["acc"], prs=st["prs"], pav=st["pav"])
    o.phase(6)  # UpPcl1: a = 0 -> positions move by v dt, then ChkPcl
    s2 = o.state()
    assert s2["typ"][1] == -1 and np.all(s2["pos"][:, 1] == 0) and s2["prs"][1] == 0
    assert np.linalg.norm(s2["vel"][:, 0].astype(np.float64)) <= umax + 1e-12


def test_eos_clamps():
    """MkPrs: P = max(n - n0, 0) c^2 / n0 rho clamped to [0, Pmax] (kernel.cu:1389-1406)."""
    # dense cluster -> P clamps at Pmax; a lone particle -> n = 0 -> P = -0.0 (kept as zero)
    l0 = 0.02
    fl = [[0.2 + i * 0.3 * l0, 0.2, 0.2] for i in range(6)] + [[0.05, 0.3, 0.3]]
    o, _ = _one_particle_oracle(F64, fl, [], [])
    o.phase(0)
    o.phase(8)
    st = o.state()
    pmax = o.p.pmax
    assert st["prs"][0] == pmax or st["prs"][0] <= pmax
    assert st["prs"][6] == 0.0
    assert np.all(st["prs"] >= 0) and np.all(st["prs"] <= pmax)
