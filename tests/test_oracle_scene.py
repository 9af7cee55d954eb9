"""The oracle's scene generator equals the product's, byte for byte (CPU).

bench.py's reference arm builds its workloads with ``oracle.scenes`` so that it never loads
the product library. Both arms must then time the same input: the same table of workloads,
the same particles (type, position, velocity, normal) and the same parameters.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from mps_cuda_b200 import F32, F32_N64, F64, configs, dambreak, dambreak_params
from mps_cuda_b200.solver import SceneDesc
from oracle import scenes


def _same_desc(a: SceneDesc, b: scenes.Scene):
    assert (a.l0, tuple(a.tank), tuple(a.block), a.wall_mask, a.jitter, a.seed, a.vel_sigma,
            a.vel_seed, tuple(a.origin)) == \
        (b.l0, tuple(b.tank), tuple(b.block), b.wall_mask, b.jitter, b.seed, b.vel_sigma,
         b.vel_seed, tuple(b.origin))


def _same_scene(pd: SceneDesc, od: scenes.Scene, dt: float):
    a, b = dambreak(pd), scenes.dambreak(od)
    for k in ("typ", "pos", "vel", "nrm"):
        assert a[k].dtype == b[k].dtype and a[k].shape == b[k].shape, k
        assert a[k].tobytes() == b[k].tobytes(), k
    for prec in (F32, F64, F32_N64):
        pp = dambreak_params(pd, dt=dt, precision=prec)
        op = scenes.dambreak_params(od, dt=dt, precision=prec)
        assert C.sizeof(pp) == C.sizeof(op)
        assert bytes(pp) == bytes(op), prec


def test_workload_tables_agree():
    assert set(configs.WORKLOADS) == set(scenes.WORKLOADS)
    for name, (pd, dt, steps) in configs.WORKLOADS.items():
        od, odt, osteps = scenes.WORKLOADS[name]
        _same_desc(pd, od)
        assert (dt, steps) == (odt, osteps), name
    assert (scenes.SND, scenes.NU, scenes.G_Z) == (configs.SND, configs.NU, configs.G_Z)


@pytest.mark.parametrize("name", sorted(configs.WORKLOADS))
def test_workload_scenes_identical(name):
    pd, dt, _ = configs.WORKLOADS[name]
    od, _, _ = scenes.WORKLOADS[name]
    _same_scene(pd, od, dt)


def test_other_descriptions_identical():
    """Offsets, partial wall masks, velocities and the batched draws"""
    cases = [SceneDesc(0.015, (0.7, 0.33, 0.5), (9, 7, 5), wall_mask=0x15, seed=11,
                       vel_sigma=0.2, vel_seed=5, origin=(-0.3, 0.1, 2.0), jitter=0.05),
             SceneDesc(0.02, (0.4, 0.2, 0.4), (0, 3, 3), wall_mask=0x3F)]
    cases += [d for d, _ in configs.batched_scenes()[:6]]
    for d in cases:
        od = scenes.Scene(d.l0, tuple(d.tank), tuple(d.block), d.seed, d.vel_sigma, d.vel_seed,
                          d.wall_mask, d.jitter, tuple(d.origin))
        _same_scene(d, od, 1e-4)


def test_workload_helper_types():
    p, typ, pos, vel, nrm = scenes.workload("dambreak_l0.02_small", "f64")
    assert p.precision == F64 and pos.dtype == np.float64 and typ.dtype == np.int8
    p, typ, pos, vel, nrm = scenes.workload("dambreak_l0.02_small", "f32")
    assert p.precision == F32 and pos.dtype == np.float32 and nrm.shape == pos.shape
