"""Dam-break workloads on the oracle side (TEST INFRASTRUCTURE, not the product).

bench.py's reference arm builds its input with these, so that timing the reference's loops
(the OpenMP oracle, or the reference's own kernels) never loads the product library. The
table restates the product's workload table (``mps_cuda_b200.configs``) and the particles
and parameters come from the oracle's own generator (``oracle_scene.cpp``);
``tests/test_oracle_scene.py`` checks both against the product's, byte for byte.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from .oracle import c_double_p, c_int8_p, lib, oracle_params, oracle_scene_desc

F32, F64, F32_N64 = 0, 1, 2
PRECISIONS = {"f32": F32, "f64": F64, "f32n64": F32_N64}
SND, NU, G_Z = 20.0, 1e-6, -9.81


@dataclass(frozen=True)
class Scene:
    l0: float
    tank: tuple
    block: tuple
    seed: int = 0
    vel_sigma: float = 0.0
    vel_seed: int = 1
    wall_mask: int = 0x1F
    jitter: float = 0.01
    origin: tuple = (0.0, 0.0, 0.0)

    def c(self) -> oracle_scene_desc:
        d = oracle_scene_desc()
        d.l0 = self.l0
        d.tank[:] = list(self.tank)
        d.block[:] = [int(b) for b in self.block]
        d.wall_mask = self.wall_mask
        d.jitter = self.jitter
        d.seed = self.seed
        d.vel_sigma = self.vel_sigma
        d.vel_seed = self.vel_seed
        d.origin[:] = list(self.origin)
        return d


# name -> (scene, dt, steps): tanks with walls on five faces (open top), the fluid column in
# the x = 0 corner
WORKLOADS = {
    "dambreak_l0.02_6k": (Scene(0.02, (1.0, 0.2, 0.8), (20, 10, 30)), 2e-4, 1000),
    "dambreak_l0.005_384k": (Scene(0.005, (1.6, 0.2, 0.8), (80, 40, 120)), 5e-5, 2000),
    "adjoint_l0.01_48k": (Scene(0.01, (1.0, 0.2, 0.8), (40, 20, 60), vel_sigma=0.05, vel_seed=1),
                          1e-4, 200),
    "dambreak_l0.0025_6.1M": (Scene(0.0025, (1.6, 0.4, 0.8), (160, 160, 240)), 2.5e-5, 500),
    "dambreak_l0.0032_2.9M": (Scene(0.0032, (1.6, 0.4, 0.8), (125, 125, 187)), 3.2e-5, 500),
    "dambreak_l0.02_small": (Scene(0.02, (0.4, 0.2, 0.4), (8, 6, 10), seed=3), 2e-4, 50),
}


def dambreak(scene: Scene) -> dict:
    """typ (n,) int8 and pos / vel / nrm (3, n) float64 SoA of a dam-break scene."""
    d = scene.c()
    n = C.c_int32()
    if lib().oracle_scene_dambreak_count(C.byref(d), C.byref(n)) != 0:
        raise ValueError("invalid scene")
    n = n.value
    typ = np.empty(n, np.int8)
    pos, vel, nrm = (np.empty((3, n), np.float64) for _ in range(3))
    rc = lib().oracle_scene_dambreak(C.byref(d), n, typ.ctypes.data_as(c_int8_p),
                                     pos.ctypes.data_as(c_double_p), vel.ctypes.data_as(c_double_p),
                                     nrm.ctypes.data_as(c_double_p))
    if rc != 0:
        raise ValueError("oracle_scene_dambreak failed")
    return {"typ": typ, "pos": pos, "vel": vel, "nrm": nrm}


def dambreak_params(scene: Scene, dt: float, precision: int = F32, snd: float = SND,
                    nu: float = NU, g_z: float = G_Z) -> oracle_params:
    p = oracle_params()
    if lib().oracle_params_dambreak(C.byref(scene.c()), snd, dt, nu, g_z, precision,
                                    C.byref(p)) != 0:
        raise ValueError("invalid scene")
    return p


def workload(name: str, precision: str):
    """(params, typ, pos, vel, nrm) of a named workload, positions in the precision's type."""
    scene, dt, _ = WORKLOADS[name]
    prec = PRECISIONS[precision]
    sc = dambreak(scene)
    p = dambreak_params(scene, dt=dt, precision=prec)
    rd = np.float64 if prec == F64 else np.float32
    return p, sc["typ"], sc["pos"].astype(rd), sc["vel"].astype(rd), sc["nrm"].astype(rd)
