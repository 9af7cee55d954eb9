"""Size-independent properties at the 384k-particle dam break (l0 = 0.005), on the GPU.

The oracle is too slow at this size for step-by-step comparison, so these tests check what
must hold at any size: the fused step equals the reference's method-by-method sequence
bit for bit, runs are deterministic, particles are conserved, no counter reports an error,
and the bucket lists come out sorted the way the step requires.
"""
from __future__ import annotations

import numpy as np
import pytest

from mps_cuda_b200 import F32, MPS, configs, dambreak, dambreak_params
from mps_cuda_b200 import _lib as L

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big():
    desc, dt, _ = configs.WORKLOADS["dambreak_l0.005_384k"]
    sc = dambreak(desc)
    p = dambreak_params(desc, dt=dt, precision=F32)
    args = (sc["typ"], sc["pos"].astype(np.float32), sc["vel"].astype(np.float32),
            sc["nrm"].astype(np.float32))
    return p, args


def _same(a, b):
    for k in ("typ", "pos", "vel", "acc", "prs", "pav"):
        assert np.array_equal(a[k], b[k]), k


def test_fused_step_equals_method_sequence(big):
    p, args = big
    fused, methods = MPS(p, *args), MPS(p, *args)
    fused.set_option(L.OPT_GRAPH, 1)
    fused.step(2)
    for _ in range(2):
        methods.step_by_methods()
    _same(fused.state(), methods.state())


def test_deterministic_and_conserving(big):
    p, args = big
    a, b = MPS(p, *args), MPS(p, *args)
    a.step(4)
    b.step(2)
    b.step(2)
    sa, sb = a.state(), b.state()
    _same(sa, sb)
    c = a.counters()
    nf = int((args[0] == 0).sum())
    assert c["n_fluid_alive"] + c["n_deleted"] == nf == 384000
    assert c["err_mirror_slot"] == c["err_mirror_capacity"] == c["err_cell_range"] == c["err_nan"] == 0
    assert 50000 < c["n_mirror_1"] < 200000
    # walls and ids are untouched by the step
    assert np.array_equal(sa["typ"][nf:], args[0][nf:])
    assert np.array_equal(sa["pos"][:, nf:], args[1][:, nf:])


def test_bucket_index_matches_positions(big):
    p, args = big
    g = MPS(p, *args)
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
    a, b = MPS(p, *args), MPS(p, *args)
    b.set_option(L.OPT_CELL_SKIP, 0)
    a.step(2)
    b.step(2)
    _same(a.state(), b.state())


def test_full_size_steps_equal_the_oracle(big):
    """At the benchmark's own size (384 000 fluid particles, FP32) two fused steps give the
    oracle's state exactly, mirrors included."""
    from oracle.oracle import Oracle, params_from
    p, args = big
    g = MPS(p, *args)
    o = Oracle(params_from(p), *args)
    try:
        g.step(2)
        o.step(2)
        a, b = g.state(), o.state()
        for k in ("typ", "pos", "vel", "prs", "pav"):
            assert np.array_equal(a[k], b[k]), k
        gm, om = g.mirrors(2), o.mirrors()
        assert len(gm["slot"]) > 80000
        assert np.array_equal(gm["slot"], om["slot"]) and np.array_equal(gm["pos"], om["pos"])
    finally:
        g.close()
