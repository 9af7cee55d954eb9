"""The corrected-matrix pressure gradient (MPS_OPT_GRADIENT = MPS_GRAD_CORRECTED) on the GPU.

The reference ships this PrsGrdTrm behind `#if 0` (kernel.cu:1435-1648). The oracle restates
it and is pinned against the reference's own build of that kernel by the golden vectors
(tests/test_oracle_golden.py); here the sm_100a path is compared with the oracle exactly (==),
method by method and over fused steps, and its two edge cases are checked: a particle with
no neighbour inside rp keeps ChkCol's velocity as its acceleration, and the option leaves the
default path unchanged.
"""
from __future__ import annotations

import numpy as np
import pytest

from mps_cuda_b200 import F32, F32_N64, F64, MPS, MPSError, configs, dambreak, dambreak_params
from mps_cuda_b200 import _lib as L
from oracle.oracle import Oracle, params_from

pytestmark = pytest.mark.gpu

STEP = [0, 2, 3, 4, 5, 6, 0, 7, 0, 8, 2, 3, 4, 9, 10]  # kernel.cu:1904-1935
FIELDS = ("pos", "vel", "acc", "prs", "pav")


def _pair(prec, name="dambreak_l0.02_small", diag=False):
    desc, dt, _ = configs.WORKLOADS[name]
    sc = dambreak(desc)
    p = dambreak_params(desc, dt=dt, precision=prec)
    d = np.float64 if prec == F64 else np.float32
    args = (sc["typ"], sc["pos"].astype(d), sc["vel"].astype(d), sc["nrm"].astype(d))
    g = MPS(p, *args)
    g.set_option(L.OPT_GRADIENT, L.GRAD_CORRECTED)
    if diag:
        g.set_option(L.OPT_DIAG, 1)
    o = Oracle(params_from(p), *args)
    o.set_gradient(1)
    return g, o, p, args


def _same(a, b, where):
    assert np.array_equal(a["typ"], b["typ"]), where
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), (where, f, np.nanmax(np.abs(a[f].astype(float) - b[f])))


@pytest.mark.parametrize("prec", [F32, F64, F32_N64])
def test_every_method_bit_exact(prec):
    g, o, _, _ = _pair(prec, diag=True)
    try:
        for step in range(3):
            for ph in STEP:
                g.phase(ph)
                o.phase(ph)
                _same(g.state(), o.state(), (step, ph))
            dg, do = g.diag(), o.diag()
            for c in ("grd_f", "grd_m"):
                assert np.array_equal(dg[c], do[c]), (step, c)
    finally:
        g.close()


@pytest.mark.parametrize("prec", [F32, F64])
@pytest.mark.parametrize("graph", [0, 1])
def test_fused_steps_bit_exact(prec, graph):
    g, o, _, _ = _pair(prec)
    g.set_option(L.OPT_GRAPH, graph)
    try:
        for chunk in (1, 4, 15):
            g.step(chunk)
            o.step(chunk)
            _same(g.state(), o.state(), chunk)
    finally:
        g.close()


def test_corrected_differs_from_standard_and_switches_back():
    desc, dt, _ = configs.WORKLOADS["dambreak_l0.02_small"]
    sc = dambreak(desc)
    p = dambreak_params(desc, dt=dt, precision=F64)
    hs = [MPS(p, sc["typ"], sc["pos"], sc["vel"], sc["nrm"]) for _ in range(3)]
    try:
        hs[1].set_option(L.OPT_GRADIENT, L.GRAD_CORRECTED)
        hs[2].set_option(L.OPT_GRADIENT, L.GRAD_CORRECTED)
        for h in hs:
            h.step(5)
        hs[2].set_option(L.OPT_GRADIENT, L.GRAD_STANDARD)
        hs[0].step(5)
        hs[2].step(5)
        a, b = hs[0].state(), hs[1].state()
        assert not np.array_equal(a["pos"], b["pos"])  # the variants differ
        # the standard path is what it was, whatever ran before the switch
        o = Oracle(params_from(p), sc["typ"], sc["pos"], sc["vel"], sc["nrm"])
        o.set_gradient(1)
        o.step(5)
        o.set_gradient(0)
        o.step(5)
        _same(hs[2].state(), o.state(), "switch")
        with pytest.raises(MPSError):
            hs[0].set_option(L.OPT_GRADIENT, 2)
    finally:
        for h in hs:
            h.close()


def test_isolated_particle_keeps_chkcol_velocity():
    """A particle with no neighbour inside rp: the reference returns before writing d_Acc
    (kernel.cu:1620), so UpPcl2 applies ChkCol's velocity as the acceleration."""
    desc, dt, _ = configs.WORKLOADS["dambreak_l0.02_small"]
    sc = dambreak(desc)
    p = dambreak_params(desc, dt=dt, precision=F64)
    typ, pos, vel = sc["typ"].copy(), sc["pos"].copy(), sc["vel"].copy()
    fl = np.nonzero(typ == L.FLD)[0]
    k = fl[-1]
    # lift one particle far above the block, inside the domain, moving sideways
    pos[:, k] = [0.5 * desc.tank[0], 0.5 * desc.tank[1], 0.95 * desc.tank[2]]
    vel[:, k] = [0.3, -0.2, 0.0]
    g = MPS(p, typ, pos, vel, sc["nrm"])
    g.set_option(L.OPT_GRADIENT, L.GRAD_CORRECTED)
    o = Oracle(params_from(p), typ, pos, vel, sc["nrm"])
    o.set_gradient(1)
    try:
        g.step(1)
        o.step(1)
        _same(g.state(), o.state(), "isolated")
        st = g.state()
        # VscTrm + UpPcl1 give u* = v + g dt (no neighbours); the kick is then u* (1 + dt)
        u_star = vel[:, k] + np.array(p.g) * p.dt
        want = u_star + u_star * p.dt
        np.testing.assert_allclose(st["vel"][:, k], want, rtol=1e-12)
    finally:
        g.close()


def test_adjoint_refuses_the_corrected_gradient():
    g, _, _, _ = _pair(F64)
    try:
        with pytest.raises(MPSError) as e:
            g.adjoint_record(2, 1)
        assert e.value.code == L.MPS_ERR_UNSUPPORTED
    finally:
        g.close()


def test_batched_scenes_with_the_corrected_gradient():
    """Two scenes in one handle, corrected gradient on: each equals its own oracle."""
    from mps_cuda_b200 import MPSBatch
    descs = []
    for k in range(2):
        d, dt, _ = configs.WORKLOADS["dambreak_l0.02_small"]
        descs.append((type(d)(**{**d.__dict__, "seed": d.seed + 7 * k}), dt))
    parts = [dambreak(d) for d, _ in descs]
    params = [dambreak_params(d, dt=dt, precision=F64) for d, dt in descs]
    cat = lambda key: np.concatenate([p[key] for p in parts], axis=-1)
    counts = [p["typ"].shape[0] for p in parts]
    b = MPSBatch(params, cat("typ"), cat("pos"), cat("vel"), cat("nrm"), counts=counts)
    b.set_option(L.OPT_GRADIENT, L.GRAD_CORRECTED)
    ors = []
    for pp, pt in zip(params, parts):
        o = Oracle(params_from(pp), pt["typ"], pt["pos"], pt["vel"], pt["nrm"])
        o.set_gradient(1)
        ors.append(o)
    try:
        b.step(8)
        for o in ors:
            o.step(8)
        st = b.state()
        off = 0
        for s, (o, n) in enumerate(zip(ors, counts)):
            _same({k: v[..., off:off + n] for k, v in st.items()}, o.state(), s)
            off += n
    finally:
        b.close()
