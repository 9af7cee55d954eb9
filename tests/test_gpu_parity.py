"""GPU parity: libmps_b200.so (sm_100a) against the CPU oracle, through the C-ABI.

The GPU kernels and the oracle visit neighbours in the same order and write every
expression in the same rounding form, so the comparisons below are exact (==) for every
array: positions, velocities, accelerations, pressures, mirror sets, bucket indices and
per-particle neighbour counts. The 100-step rollout additionally states the tolerances the
solver is specified to (1e-5 relative for n, P, a in FP64; 0.5 % for the integrals).
"""
from __future__ import annotations

import numpy as np
import pytest

from mps_cuda_b200 import F32, F32_N64, F64, MPS, MPSBatch, MPSError, configs, dambreak, dambreak_params
from mps_cuda_b200 import _lib as L
from oracle.oracle import Oracle, params_from

pytestmark = pytest.mark.gpu

STEP = [0, 2, 3, 4, 5, 6, 0, 7, 0, 8, 2, 3, 4, 9, 10]  # kernel.cu:1904-1935
FIELDS = ("pos", "vel", "acc", "prs", "pav")


def _dt(prec):
    return np.float64 if prec == F64 else np.float32


def _pair(name, prec, diag=True):
    desc, dt, _ = configs.WORKLOADS[name]
    sc = dambreak(desc)
    p = dambreak_params(desc, dt=dt, precision=prec)
    d = _dt(prec)
    args = (sc["typ"], sc["pos"].astype(d), sc["vel"].astype(d), sc["nrm"].astype(d))
    g = MPS(p, *args)
    if diag:
        g.set_option(L.OPT_DIAG, 1)
    return g, Oracle(params_from(p), *args), p, args


def _assert_same_state(a, b, where=""):
    assert np.array_equal(a["typ"], b["typ"]), where
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), (where, f, np.abs(a[f].astype(float) - b[f]).max())


def _assert_same_mirrors(a, b, where=""):
    assert np.array_equal(a["slot"], b["slot"]), where
    assert np.array_equal(a["pos"], b["pos"]), where
    assert np.array_equal(a["prs"], b["prs"]), where


@pytest.mark.parametrize("prec", [F32, F64, F32_N64])
def test_every_method_bit_exact(prec):
    g, o, _, _ = _pair("dambreak_l0.02_small", prec)
    assert np.array_equal(g.wall_flags(), o.wall_flags())
    for step in range(3):
        for ph in STEP:
            g.phase(ph)
            o.phase(ph)
            where = (step, ph)
            _assert_same_state(g.state(), o.state(), where)
            if ph == 3:
                _assert_same_mirrors(g.mirrors(0), o.mirrors(), where)
            if ph == 4:
                _assert_same_mirrors(g.mirrors(1), o.mirrors(), where)
            dg, do = g.diag(), o.diag()
            for c in L.DIAG_COLUMNS:
                assert np.array_equal(dg[c], do[c]), (where, c)
            assert np.array_equal(dg["ndens"], do["ndens"]), where


@pytest.mark.parametrize("prec", [F32, F64, F32_N64])
@pytest.mark.parametrize("graph", [0, 1])
def test_fused_steps_bit_exact(prec, graph):
    g, o, _, _ = _pair("dambreak_l0.02_small", prec, diag=False)
    g.set_option(L.OPT_GRAPH, graph)
    for chunk in (1, 1, 3, 15):
        g.step(chunk)
        o.step(chunk)
        _assert_same_state(g.state(), o.state(), chunk)
    # after a step the reference's mirror arrays hold the step's second generation
    _assert_same_mirrors(g.mirrors(2), o.mirrors())
    c = g.counters()
    assert c["steps"] == 20 and c["err_mirror_slot"] == 0 and c["err_cell_range"] == 0
    assert c["n_fluid_alive"] + c["n_deleted"] == 480


def test_fused_diag_counts_bit_exact():
    g, o, _, _ = _pair("dambreak_l0.02_6k", F32)
    g.step(3)
    o.step(3)
    dg, do = g.diag(), o.diag()
    fl = o.state()["typ"] == 0
    # the fused step records every neighbour count of its last step
    for c in L.DIAG_COLUMNS:
        assert np.array_equal(dg[c][fl], do[c][fl]), c
    assert np.array_equal(dg["ndens"][fl], do["ndens"][fl])
    assert dg["vsc_f"][fl].mean() > 80 and dg["prs_f"][fl].mean() > 20


def test_rollout_100_steps_fp64():
    """cfg 1 (6000 fluid particles, FP64): n, P, a within 1e-5 relative over 100 steps and the
    integrals within 0.5 %; the step is in fact bit-identical to the oracle's."""
    g, o, _, _ = _pair("dambreak_l0.02_6k", F64)
    for k in range(4):
        g.step(25)
        o.step(25)
        a, b = g.state(), o.state()
        fl = b["typ"] == 0
        for f in ("prs", "pos", "vel"):
            x, y = a[f][..., fl], b[f][..., fl]
            assert np.abs(x - y).max() <= 1e-5 * max(np.abs(y).max(), 1e-30), (k, f)
        ia, ib = g.integrals(), o.integrals()
        assert np.all(np.abs(ia - ib) <= 5e-3 * np.abs(ib) + 1e-12), (ia, ib)
        _assert_same_state(a, b, k)
    # accelerations and number density of one more step, method by method
    g.set_option(L.OPT_DIAG, 1)
    for ph in STEP[:-1]:
        g.phase(ph)
        o.phase(ph)
    a, b = g.state(), o.state()
    assert np.array_equal(a["acc"], b["acc"])
    assert np.array_equal(g.diag()["ndens"], o.diag()["ndens"])


@pytest.mark.parametrize("prec", [F32, F32_N64])
def test_batched_scenes_equal_single_scenes(prec):
    """Three scenes in one handle advance exactly like three separate oracles."""
    names = ["dambreak_l0.02_small", "dambreak_l0.02_small", "dambreak_l0.02_6k"]
    descs = []
    for k, n in enumerate(names):
        d, dt, _ = configs.WORKLOADS[n]
        d = type(d)(**{**d.__dict__, "seed": d.seed + k})
        descs.append((d, dt))
    parts = [dambreak(d) for d, _ in descs]
    params = [dambreak_params(d, dt=dt, precision=prec) for d, dt in descs]
    cat = lambda key: np.concatenate([p[key] for p in parts], axis=-1)
    counts = [p["typ"].shape[0] for p in parts]
    b = MPSBatch(params, cat("typ"), cat("pos").astype(np.float32), cat("vel").astype(np.float32),
                 cat("nrm").astype(np.float32), counts=counts)
    ors = [Oracle(params_from(pp), pt["typ"], pt["pos"].astype(np.float32),
                  pt["vel"].astype(np.float32), pt["nrm"].astype(np.float32))
           for pp, pt in zip(params, parts)]
    b.step(10)
    for o in ors:
        o.step(10)
    st = b.state()
    off = 0
    for s, (o, n) in enumerate(zip(ors, counts)):
        sub = {k: v[..., off:off + n] for k, v in st.items()}
        _assert_same_state(sub, o.state(), s)
        ig, io = b.integrals(s), o.integrals()
        assert np.allclose(ig, io, rtol=1e-6, atol=1e-9)
        off += n


def test_state_roundtrip_and_errors():
    g, o, _, args = _pair("dambreak_l0.02_small", F32, diag=False)
    g.step(2)
    st = g.state()
    g.set_state(**st)
    _assert_same_state(g.state(), st)
    # after replacing the state the bucket lists are gone until MkBkt runs
    with pytest.raises(MPSError) as e:
        g.phase(L.PHASE_VSCTRM)
    assert e.value.code == L.MPS_ERR_STATE
    with pytest.raises(MPSError) as e:
        g.phase(99)
    assert e.value.code == L.MPS_ERR_ARG
    # a fused step after set_state rebuilds everything and continues bit-exactly
    o.step(2)
    g.step(3)
    o.step(3)
    _assert_same_state(g.state(), o.state())


@pytest.mark.parametrize("prec", [F32, F64])
def test_autotune_changes_no_result(prec):
    """Tuning tries every candidate of every knob (VscTrm's staging mode, candidate batch and
    block size, the other passes' block sizes and register bounds) on the handle's own state and restores it: the steps after
    it equal the oracle's. Then each knob is forced to every value it can take, and the
    result is still the oracle's; last, each way of using the second stream."""
    g, o, _, _ = _pair("dambreak_l0.02_6k", prec, diag=False)
    g.step(2)
    chosen = g.autotune(2)
    assert chosen["pass_a"] in (64, 128) and chosen["staging"] in (0, 1, 2)
    assert chosen["candidate_batch"] in (2, 4, 8)
    assert 0 <= chosen["register_bound"] <= 7
    for k in ("pass_b", "pass_c", "gen_cull"):
        assert chosen[k] in (32, 64, 96, 128)
    assert g.counters()["steps"] == 2
    g.step(3)
    o.step(5)
    _assert_same_state(g.state(), o.state())
    g.set_option(L.OPT_GRAPH, 1)
    for stage in (L.STAGE_GLOBAL, L.STAGE_POSITIONS, L.STAGE_VELOCITIES):
        for blk in (32, 64, 96, 128):
            g.set_option(L.OPT_STAGING, stage)
            g.set_option(L.OPT_BLOCK, blk)
            g.step(1)
            o.step(1)
            _assert_same_state(g.state(), o.state(), (stage, blk))
    g.set_option(L.OPT_STAGING, L.STAGE_GLOBAL)
    for nb in (2, 8, 4):
        g.set_option(L.OPT_CANDIDATE_BATCH, nb)
        g.step(1)
        o.step(1)
        _assert_same_state(g.state(), o.state(), ("batch", nb))
    for rb in (1, 2, 4, 7, 0):
        g.set_option(L.OPT_REGISTER_BOUND, rb)
        g.step(1)
        o.step(1)
        _assert_same_state(g.state(), o.state(), ("register bound", rb))
    # one stream; the step end on two; the second mirror generation beside pass B; both
    for ov in (0, 1, 2, 3):
        g.set_option(L.OPT_OVERLAP, ov)
        assert g.get_option(L.OPT_OVERLAP) == ov
        g.step(2)
        o.step(2)
        _assert_same_state(g.state(), o.state(), ("overlap", ov))
    g.close()


def test_tuned_shapes_carry_over_to_a_new_handle_of_the_same_class():
    g, _, p, args = _pair("dambreak_l0.02_6k", F32, diag=False)
    chosen = g.autotune(1)
    h = MPS(p, *args)
    assert h.get_option(L.OPT_STAGING) == chosen["staging"]
    assert h.get_option(L.OPT_BLOCK) == chosen["pass_a"]
    assert h.get_option(L.OPT_REGISTER_BOUND) == chosen["register_bound"]
    h.close()
    g.close()


def test_batch_of_64_uneven_scenes_equals_the_oracle():
    """The bench's batched configuration (64 uneven scenes, FP32 state with FP64 number
    density, graph replay): every scene equals its own oracle after four steps."""
    scenes = configs.batched_scenes()
    parts = [dambreak(d) for d, _ in scenes]
    params = [dambreak_params(d, dt=dt, precision=F32_N64) for d, dt in scenes]
    counts = [p["typ"].shape[0] for p in parts]
    cat = lambda k: np.concatenate([p[k] for p in parts], axis=-1).astype(
        np.float32 if k != "typ" else np.int8)
    b = MPSBatch(params, cat("typ"), cat("pos"), cat("vel"), cat("nrm"), counts=counts)
    b.set_option(L.OPT_GRAPH, 1)
    b.step(4)
    st = b.state()
    off = 0
    for s, (pp, pt, n) in enumerate(zip(params, parts, counts)):
        o = Oracle(params_from(pp), pt["typ"], pt["pos"].astype(np.float32),
                   pt["vel"].astype(np.float32), pt["nrm"].astype(np.float32))
        o.step(4)
        sub = {k: v[..., off:off + n] for k, v in st.items()}
        _assert_same_state(sub, o.state(), s)
        o.close()
        off += n


@pytest.mark.parametrize("prec", [F32, F64])
@pytest.mark.parametrize("cap", [1, 8])
def test_list_overflow_path_bit_exact(prec, cap):
    """A particle whose neighbour list would exceed its capacity walks its fine cells again in
    ChkCol/MkPrs and PrsGrdTrm. MPS_OPT_LIST_CAPACITY forces that path on for (nearly) every
    particle: the state, the mirrors and the neighbour counts stay those of the oracle."""
    g, o, _, _ = _pair("dambreak_l0.02_small", prec)
    g.set_option(L.OPT_LIST_CAPACITY, cap)
    g.set_option(L.OPT_GRAPH, 1)
    try:
        for chunk in (1, 4, 15):
            g.step(chunk)
            o.step(chunk)
            _assert_same_state(g.state(), o.state(), (cap, chunk))
        dg, do = g.diag(), o.diag()
        fl = o.state()["typ"] == 0
        for c in ("col_f", "col_w", "col_m", "prs_f", "prs_m", "grd_f", "grd_m"):
            assert np.array_equal(dg[c][fl], do[c][fl]), c
        _assert_same_mirrors(g.mirrors(2), o.mirrors())
        g.set_option(L.OPT_LIST_CAPACITY, 0)  # back to the full lists
        g.step(3)
        o.step(3)
        _assert_same_state(g.state(), o.state(), (cap, "full"))
    finally:
        g.close()


def test_list_capacity_change_voids_a_recorded_rollout():
    g, _, _, _ = _pair("dambreak_l0.02_small", F64, diag=False)
    try:
        g.adjoint_record(4, 2)
        g.set_option(L.OPT_LIST_CAPACITY, 8)
        with pytest.raises(MPSError) as e:
            g.adjoint_backward(np.zeros((3, g.n)), np.zeros((3, g.n)))
        assert e.value.code == L.MPS_ERR_STATE
        with pytest.raises(MPSError):
            g.set_option(L.OPT_LIST_CAPACITY, -1)
    finally:
        g.close()


@pytest.mark.parametrize("graph", [0, 1])
def test_reads_between_steps_change_nothing(graph):
    """A step's end (the next step's mirrors and bucket builds) runs when the next step
    starts or when something needs the sorted state. Reading the state, counters,
    diagnostics or the step's second mirrors in between, or setting the state back to what
    was read, leaves every later result equal to the oracle's."""
    g, o, _, _ = _pair("dambreak_l0.02_6k", F32, diag=False)
    h, _, _, _ = _pair("dambreak_l0.02_6k", F32, diag=False)
    for x in (g, h):
        x.set_option(L.OPT_GRAPH, graph)
    for k in range(4):
        g.step(1)
        o.step(1)
        st = g.state()
        _assert_same_state(st, o.state(), ("state", k))
        c = g.counters()
        assert c["n_fluid_alive"] == int((o.state()["typ"] == L.FLD).sum())
        _assert_same_mirrors(g.mirrors(2), o.mirrors(), ("m2", k))
        if k == 2:
            g.set_state(typ=st["typ"], pos=st["pos"], vel=st["vel"], pav=st["pav"])
    h.step(4)
    _assert_same_state(h.state(), o.state(), "stepped at once")
    _assert_same_mirrors(g.mirrors(1), h.mirrors(1), "m1")
    g.step(2)
    o.step(2)
    _assert_same_state(g.state(), o.state(), "after")
    g.close()
    h.close()


@pytest.mark.parametrize("prec", [F32, F64])
def test_bucket_rows_longer_than_a_block_equal_the_oracle(prec):
    """A tank 287 buckets long: the fluid build's start-table pass walks each bucket row in
    several chunks of 256 buckets, carrying its running starts from chunk to chunk."""
    from mps_cuda_b200 import SceneDesc, derive
    desc = SceneDesc(0.004, (3.5, 0.06, 0.1), (30, 8, 10))
    p = dambreak_params(desc, dt=4e-5, precision=prec)
    assert derive(p).nbx > 256
    sc = dambreak(desc)
    d = _dt(prec)
    args = (sc["typ"], sc["pos"].astype(d), sc["vel"].astype(d), sc["nrm"].astype(d))
    g = MPS(p, *args)
    o = Oracle(params_from(p), *args)
    g.set_option(L.OPT_GRAPH, 1)
    for chunk in (1, 3):
        g.step(chunk)
        o.step(chunk)
        _assert_same_state(g.state(), o.state(), ("long tank", chunk))
    _assert_same_mirrors(g.mirrors(2), o.mirrors())
    g.close()
