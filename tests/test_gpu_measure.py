"""The measurement entry points: the device's work counts and its arithmetic rates.

mps_get_work counts, during steps run with MPS_OPT_DIAG, the fluid candidates each walk
tested and the neighbour-list entries; the neighbour pairs are mps_get_diag's columns. The
counts must bound the pairs (every pair was a tested candidate) and must not depend on where
the walk reads its candidates. mps_measure_arith times the FMA, square-root and division
rates that the bench's compute roofline divides by.
"""
from __future__ import annotations

import numpy as np
import pytest

from mps_cuda_b200 import F32, MPS, configs, dambreak, dambreak_params, measure_arith
from mps_cuda_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _handle():
    desc, dt, _ = configs.WORKLOADS["dambreak_l0.02_6k"]
    sc = dambreak(desc)
    p = dambreak_params(desc, dt=dt, precision=F32)
    return MPS(p, sc["typ"], sc["pos"].astype(np.float32), sc["vel"].astype(np.float32),
               sc["nrm"].astype(np.float32))


def test_work_counts_bound_the_pairs_and_ignore_staging():
    seen = []
    for mode in (L.STAGE_GLOBAL, L.STAGE_POSITIONS):
        g = _handle()
        try:
            g.set_option(L.OPT_STAGING, mode)
            assert g.work() == {"visc_candidates": 0, "list_candidates": 0, "list_entries": 0}
            g.step(1)  # without diagnostics nothing is counted
            assert g.work()["visc_candidates"] == 0
            g.set_option(L.OPT_DIAG, 1)
            g.step(1)
            w, d = g.work(), g.diag()
            fluid = int((g.state()["typ"] == 0).sum())
            # about 100 neighbours inside r per particle at rest density (fewer at the walls
            # and the free surface), about twice as many candidates tested
            assert w["visc_candidates"] >= int(d["vsc_f"].sum()) > 50 * fluid
            assert w["list_candidates"] >= w["list_entries"] >= int(d["prs_f"].sum())
            assert w["list_entries"] >= int(d["col_f"].sum())
            seen.append(w)
        finally:
            g.close()
    assert seen[0] == seen[1]


def test_measured_arithmetic_rates_are_plausible():
    a = measure_arith()
    assert a["sms"] > 0 and a["clock_khz"] > 0
    # a B200 does tens of TFLOP/s of FP32 FMA; FP64 and the IEEE operations are slower
    assert 1e13 < a["fp32_fma_flops"] < 2e15
    assert 1e12 < a["fp64_fma_flops"] <= a["fp32_fma_flops"]
    for k in ("fp32_sqrt_per_s", "fp32_div_per_s", "fp64_sqrt_per_s", "fp64_div_per_s"):
        assert 1e11 < a[k] < a["fp32_fma_flops"], k
    assert a["warp_issue_per_s"] > 0
