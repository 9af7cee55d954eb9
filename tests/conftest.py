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


_GOLDEN_CACHE = {}


def golden(prec: str) -> dict:
    """A golden record: "f32", "f64", "corr_f32", "corr_f64" (the small scene, two steps) or
    "6k_f64" (the 6 000-particle dam break, its second step; see golden_6k)."""
    if prec not in _GOLDEN_CACHE:
        if prec == "6k_f64":
            _GOLDEN_CACHE[prec] = golden_6k()
        else:
            _GOLDEN_CACHE[prec] = dict(np.load(os.path.join(GOLDEN, f"ref_small_{prec}.npz")))
    return _GOLDEN_CACHE[prec]


def golden_6k() -> dict:
    """ref_6k_f64.npz expanded to the layout of the small records. The file stores the state
    before the step whole and after each method only what changed; the particles themselves
    are the workload's seeded scene, regenerated here (its checksum is in the file)."""
    from oracle import scenes
    path = os.path.join(GOLDEN, "ref_6k_f64.npz")
    if not os.path.exists(path):
        pytest.skip("ref_6k_f64.npz not recorded (tests/golden/make_golden.py --6k)")
    z = dict(np.load(path))
    scene, _, _ = scenes.WORKLOADS[str(z["workload"])]
    sc = scenes.dambreak(scene)
    nf = int(z["nf"])
    got = np.array([float(sc["pos"].sum()), float(sc["nrm"].sum()), nf])
    assert np.array_equal(got, z["scene_sum"]), "the regenerated scene is not the recorded one"
    g = dict(z)
    g.update(typ=sc["typ"], pos=sc["pos"], vel=sc["vel"], nrm=sc["nrm"])
    keys = ("typ", "pos", "vel", "acc", "prs", "pav", "mslot", "mpos", "mprs", "cell")
    for s in g["record_steps"]:
        for k in range(1, len(g["phases"]) + 1):
            for q in keys:
                if f"s{s}_k{k}_{q}" not in g:
                    g[f"s{s}_k{k}_{q}"] = g[f"s{s}_k{k - 1}_{q}"]
    return g


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
