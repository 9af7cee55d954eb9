"""Shared test set-up.

Tests marked ``gpu`` need a CUDA device and run the product (libmps_b200.so) against the
CPU oracle; everything else runs on the CPU: the oracle against the golden vectors recorded
from the reference's own kernels, host-side logic, and the C-ABI surface.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a library)")


def golden(prec: str) -> dict:
    return dict(np.load(os.path.join(GOLDEN, f"ref_small_{prec}.npz")))


def golden_params(g: dict):
    from oracle.oracle import oracle_params
    pa = g["params"]
    p = oracle_params()
    p.pcl_dst = pa[0]
    p.min[:] = list(pa[1:4])
    p.max[:] = list(pa[4:7])
    p.g[:] = list(pa[7:10])
    p.knm_vsc, p.col_rat, p.dst_lmt_rat, p.rho = pa[10], pa[11], pa[12], pa[13]
    p.snd, p.dt, p.umax, p.pmax = pa[14], pa[15], pa[16], pa[17]
    p.precision = int(pa[18])
    return p


def golden_state(g: dict, tag: str) -> dict:
    """Full particle state of a recorded snapshot (walls are static and not recorded)."""
    n = g["typ"].shape[0]
    nf = int(g["nf"])
    dt = g["pos"].dtype
    st = {}
    for k in ("pos", "vel", "acc"):
        a = np.zeros((3, n), dt)
        a[:, :nf] = g[f"{tag}_{k}"]
        if k in ("pos", "vel"):
            a[:, nf:] = g[k][:, nf:]
        st[k] = a
    t = g["typ"].copy()
    t[:nf] = g[f"{tag}_typ"]
    st["typ"] = t
    for k in ("prs", "pav"):
        a = np.zeros(n, dt)
        a[:nf] = g[f"{tag}_{k}"]
        st[k] = a
    return st


@pytest.fixture(scope="session")
def small_scene():
    from mps_cuda_b200 import configs, dambreak
    desc, dt, _ = configs.WORKLOADS["dambreak_l0.02_small"]
    return desc, dt, dambreak(desc)
