"""The benchmark workloads at their full size, on the GPU.

Two fused steps of the 384 000-particle dam break (l0 = 0.005) are compared exactly with the
oracle in FP32 and FP64, and two of the 6.1M-particle scene (l0 = 0.0025, FP32, the bench's
headline workload) likewise; the oracle finishes those in seconds on the host's cores. Over
more steps, properties that must hold at any size are checked: the fused step equals the
reference's method-by-method sequence bit for bit, runs are deterministic, particles are
conserved, no counter reports an error, and the bucket lists come out sorted the way the
step requires. Every handle is closed when its test ends, so that full-size device memory
is not held into the next test.
"""
from __future__ import annotations

import contextlib

import numpy as np
import pytest

from mps_cuda_b200 import F32, F64, MPS, configs, dambreak, dambreak_params
from mps_cuda_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _scene(workload, prec):
    desc, dt, _ = configs.WORKLOADS[workload]
    sc = dambreak(desc)
    p = dambreak_params(desc, dt=dt, precision=prec)
    rd = np.float64 if prec == F64 else np.float32
    args = (sc["typ"], sc["pos"].astype(rd), sc["vel"].astype(rd), sc["nrm"].astype(rd))
    return p, args


@pytest.fixture(scope="module")
def big():
    return _scene("dambreak_l0.005_384k", F32)


@contextlib.contextmanager
def handles(p, args, n):
    """n solver handles on the same scene, closed on exit"""
    hs = []
    try:
        for _ in range(n):
            hs.append(MPS(p, *args))
        yield hs
    finally:
        for h in hs:
            h.close()


def _same(a, b):
    for k in ("typ", "pos", "vel", "acc", "prs", "pav"):
        assert np.array_equal(a[k], b[k]), k


def test_fused_step_equals_method_sequence(big):
    p, args = big
    with handles(p, args, 2) as (fused, methods):
        fused.set_option(L.OPT_GRAPH, 1)
        fused.step(2)
        for _ in range(2):
            methods.step_by_methods()
        _same(fused.state(), methods.state())


def test_deterministic_and_conserving(big):
    p, args = big
    with handles(p, args, 2) as (a, b):
        a.step(4)
        b.step(2)
        b.step(2)
        sa, sb = a.state(), b.state()
        c = a.counters()
    _same(sa, sb)
    nf = int((args[0] == 0).sum())
    assert c["n_fluid_alive"] + c["n_deleted"] == nf == 384000
    assert c["err_mirror_slot"] == c["err_mirror_capacity"] == c["err_cell_range"] == c["err_nan"] == 0
    assert 50000 < c["n_mirror_1"] < 200000
    # walls and ids are untouched by the step
    assert np.array_equal(sa["typ"][nf:], args[0][nf:])
    assert np.array_equal(sa["pos"][:, nf:], args[1][:, nf:])


def test_bucket_index_matches_positions(big):
    p, args = big
    with handles(p, args, 1) as (g,):
        g.step(3)
        st, d = g.state(), g.diag()
        inf = g.info()
    x = st["pos"].astype(np.float32)
    minc = np.array(inf.minc, np.float32)
    dbinv = np.float32(inf.dbinv)
    idx = [((x[k] - minc[k]) * dbinv).astype(np.int32) + 1 for k in range(3)]
    cell = idx[2] * inf.nbx * inf.nby + idx[1] * inf.nbx + idx[0]
    live = st["typ"] != -1
    assert np.array_equal(d["cell"][live], cell[live])
    assert np.all(d["cell"][~live] == -1)


def test_skipping_bucket_rows_changes_nothing(big):
    p, args = big
    with handles(p, args, 2) as (a, b):
        b.set_option(L.OPT_CELL_SKIP, 0)
        a.step(2)
        b.step(2)
        _same(a.state(), b.state())


def _steps_equal_oracle(p, args, min_mirrors):
    from oracle.oracle import Oracle, params_from
    o = Oracle(params_from(p), *args)
    try:
        with handles(p, args, 1) as (g,):
            g.set_option(L.OPT_GRAPH, 1)
            g.step(2)
            a = g.state()
            gm = g.mirrors(2)
            c = g.counters()
        o.step(2)
        b = o.state()
        for k in ("typ", "pos", "vel", "prs", "pav"):
            assert np.array_equal(a[k], b[k]), k
        om = o.mirrors()
        assert len(gm["slot"]) > min_mirrors
        assert np.array_equal(gm["slot"], om["slot"]) and np.array_equal(gm["pos"], om["pos"])
        assert np.array_equal(gm["prs"], om["prs"])
        assert c["err_mirror_slot"] == c["err_mirror_capacity"] == c["err_cell_range"] == 0
        assert c["err_nan"] == 0
    finally:
        o.close()


def test_full_size_steps_equal_the_oracle(big):
    """At the 384k workload's own size (384 000 fluid particles, FP32) two fused steps give
    the oracle's state exactly, mirrors included."""
    p, args = big
    _steps_equal_oracle(p, args, 80000)


def test_full_size_f64_steps_equal_the_oracle():
    """The same at 384 000 particles in FP64 (the reference's commented `typedef double
    real`, const.cuh:53)."""
    p, args = _scene("dambreak_l0.005_384k", F64)
    _steps_equal_oracle(p, args, 80000)


def test_largest_scene_steps_equal_the_oracle():
    """The headline workload: 6 144 000 fluid and 614 400 wall particles (l0 = 0.0025, FP32,
    bucket rebuild every step). Two fused steps equal the oracle's exactly, state and the
    second mirror generation."""
    p, args = _scene("dambreak_l0.0025_6.1M", F32)
    assert int((args[0] == 0).sum()) == 6144000
    _steps_equal_oracle(p, args, 300000)
