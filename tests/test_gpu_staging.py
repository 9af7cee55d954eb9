"""VscTrm's candidate walk out of shared memory (MPS_OPT_STAGING) against the oracle.

A block of pass A copies the fine rows its particles' walks reach into shared memory and
walks them there. The candidates and their order are those of the walk through global
memory, so every staging mode must give the oracle's state exactly, with and without the
per-particle diagnostics, in every precision, on a batched handle, and where blocks fall
back to global memory (a tiny staging capacity) or mix both.
"""
from __future__ import annotations

import numpy as np
import pytest

from mps_cuda_b200 import F32, F32_N64, F64, MPS, MPSBatch, configs, dambreak, dambreak_params
from mps_cuda_b200 import _lib as L
from oracle.oracle import Oracle, params_from

pytestmark = pytest.mark.gpu

FIELDS = ("typ", "pos", "vel", "prs", "pav")
MODES = [L.STAGE_POSITIONS, L.STAGE_VELOCITIES]


def _scene(name, prec):
    desc, dt, _ = configs.WORKLOADS[name]
    sc = dambreak(desc)
    p = dambreak_params(desc, dt=dt, precision=prec)
    d = np.float64 if prec == F64 else np.float32
    return p, (sc["typ"], sc["pos"].astype(d), sc["vel"].astype(d), sc["nrm"].astype(d))


def _same(a, b, where):
    for k in FIELDS:
        assert np.array_equal(a[k], b[k]), (where, k)


@pytest.mark.parametrize("prec", [F32, F64, F32_N64])
@pytest.mark.parametrize("mode", MODES)
def test_staged_steps_equal_the_oracle(prec, mode):
    p, args = _scene("dambreak_l0.02_6k", prec)
    g = MPS(p, *args)
    o = Oracle(params_from(p), *args)
    try:
        g.set_option(L.OPT_STAGING, mode)
        g.set_option(L.OPT_GRAPH, 1)
        for k in range(3):
            g.step(2)
            o.step(2)
            _same(g.state(), o.state(), (prec, mode, k))
    finally:
        g.close()
        o.close()


@pytest.mark.parametrize("mode", MODES)
def test_staged_diag_counts_equal_the_oracle(mode):
    p, args = _scene("dambreak_l0.02_6k", F32)
    g = MPS(p, *args)
    o = Oracle(params_from(p), *args)
    try:
        g.set_option(L.OPT_STAGING, mode)
        g.set_option(L.OPT_DIAG, 1)
        g.step(2)
        o.step(2)
        _same(g.state(), o.state(), mode)
        gd, od = g.diag(), o.diag()
        for k in ("vsc_f", "vsc_m"):
            assert np.array_equal(gd[k], od[k]), k
        c = g.counters()
        assert c["stage_blocks"] > 0
    finally:
        g.close()
        o.close()


@pytest.mark.parametrize("cap", [1, 300])
def test_blocks_that_do_not_fit_walk_global_memory(cap):
    """capacity 1: every block falls back; 300: some blocks fit and some do not"""
    p, args = _scene("dambreak_l0.005_384k", F32)
    a, b = MPS(p, *args), MPS(p, *args)
    try:
        b.set_option(L.OPT_STAGING, L.STAGE_POSITIONS)
        b.set_option(L.OPT_STAGE_CAPACITY, cap)
        b.set_option(L.OPT_DIAG, 1)
        a.step(2)
        b.step(2)
        _same(a.state(), b.state(), cap)
        c = b.counters()
        assert c["unstaged_blocks"] > 0
        if cap == 1:
            assert c["stage_blocks"] == 0
    finally:
        a.close()
        b.close()


@pytest.mark.parametrize("mode", MODES)
def test_staged_full_size_equals_global_walk(mode):
    """384 000 particles: staged and global walks give the same state over graph steps. At
    the default capacity most blocks fit a stage of positions; staging velocities too halves
    the capacity, and fewer fit"""
    p, args = _scene("dambreak_l0.005_384k", F32)
    a, b = MPS(p, *args), MPS(p, *args)
    try:
        for h in (a, b):
            h.set_option(L.OPT_GRAPH, 1)
        b.set_option(L.OPT_STAGING, mode)
        a.step(3)
        b.step(3)
        _same(a.state(), b.state(), mode)
        b.set_option(L.OPT_DIAG, 1)
        b.step(1)
        c = b.counters()
        share = c["stage_blocks"] / (c["stage_blocks"] + c["unstaged_blocks"])
        assert share > (0.7 if mode == L.STAGE_POSITIONS else 0.05)
    finally:
        a.close()
        b.close()


def test_staged_batched_scenes_equal_the_oracle():
    names = ["dambreak_l0.02_small", "dambreak_l0.02_6k"]
    parts = [_scene(n, F32) for n in names]
    cat = lambda i: np.concatenate([pa[1][i] for pa in parts], axis=-1)  # noqa: E731
    counts = [pa[1][0].shape[0] for pa in parts]
    b = MPSBatch([pa[0] for pa in parts], cat(0), cat(1), cat(2), cat(3), counts=counts)
    try:
        b.set_option(L.OPT_STAGING, L.STAGE_VELOCITIES)
        b.step(3)
        st = b.state()
        off = 0
        for (p, args), n in zip(parts, counts):
            o = Oracle(params_from(p), *args)
            o.step(3)
            so = o.state()
            for k in FIELDS:
                assert np.array_equal(st[k][..., off:off + n], so[k]), k
            o.close()
            off += n
    finally:
        b.close()
