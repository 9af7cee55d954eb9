"""The dam-break workloads this solver is measured and checked on.

Every scene is a tank with single-layer walls on five faces (open top) and a fluid column
in the x=0 corner; positions are jittered uniformly by +-0.01 l0 from a seed. Physical
constants: rho = 1000, nu = 1e-6, g = -9.81 z, c = 20 m/s, COL_RAT = 0.2, DST_LMT_RAT = 0.9.
"""
from __future__ import annotations

import math

import numpy as np

from ._lib import F32, F64, F32_N64
from .solver import SceneDesc

SND = 20.0
NU = 1e-6
G_Z = -9.81

# name -> (scene, dt, steps)
WORKLOADS = {
    # 20x10x30 = 6000 fluid particles, l0 = 0.02, 1.0 x 0.2 x 0.8 tank
    "dambreak_l0.02_6k": (SceneDesc(0.02, (1.0, 0.2, 0.8), (20, 10, 30), seed=0), 2e-4, 1000),
    # 80x40x120 = 384000 fluid particles, l0 = 0.005, 1.6 x 0.2 x 0.8 tank
    "dambreak_l0.005_384k": (SceneDesc(0.005, (1.6, 0.2, 0.8), (80, 40, 120), seed=0), 5e-5, 2000),
    # 40x20x60 = 48000 fluid particles, l0 = 0.01, initial velocity N(0, 0.05) per component
    "adjoint_l0.01_48k": (SceneDesc(0.01, (1.0, 0.2, 0.8), (40, 20, 60), seed=0, vel_sigma=0.05,
                                    vel_seed=1), 1e-4, 200),
    # 160x160x240 = 6144000 fluid particles, l0 = 0.0025, 1.6 x 0.4 x 0.8 tank
    "dambreak_l0.0025_6.1M": (SceneDesc(0.0025, (1.6, 0.4, 0.8), (160, 160, 240), seed=0), 2.5e-5,
                              500),
    # 125x125x187 = 2921875 fluid particles, l0 = 0.0032: a state larger than L2 that a
    # profiler capture can hold (the 6.1M scene's traffic scaled down)
    "dambreak_l0.0032_2.9M": (SceneDesc(0.0032, (1.6, 0.4, 0.8), (125, 125, 187), seed=0), 3.2e-5,
                              500),
    # small scene for golden vectors and quick checks
    "dambreak_l0.02_small": (SceneDesc(0.02, (0.4, 0.2, 0.4), (8, 6, 10), seed=3), 2e-4, 50),
}


def batched_scenes(n: int = 64, seed: int = 2, nmin: int = 2000, nmax: int = 60000):
    """64 independent dam breaks: column width, depth, height ~ U[0.1, 0.5] m, l0 from
    {0.01, 0.015, 0.02}, tank length ~ U[1.0, 1.6] m, tank width = column depth, tank
    height = column height + 0.3 m. Draws whose fluid count falls outside [nmin, nmax] are
    redrawn. dt per scene from CFL 0.2: dt = 0.2 l0 / (umax + c)."""
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < n:
        w, d, h = rng.uniform(0.1, 0.5, 3)
        l0 = float(rng.choice([0.01, 0.015, 0.02]))
        length = float(rng.uniform(1.0, 1.6))
        bx, by, bz = (max(1, int(round(v / l0))) for v in (w, d, h))
        nf = bx * by * bz
        if not (nmin <= nf <= nmax):
            continue
        tank = (length, by * l0, bz * l0 + 0.3)
        desc = SceneDesc(l0, tank, (bx, by, bz), seed=1000 + len(out))
        umax = math.sqrt(2 * abs(G_Z) * (bz - 1) * l0)
        dt = 0.2 * l0 / (umax + SND)
        out.append((desc, dt))
    return out
