"""Moving walls (mps_set_wall_motion): an OBJ plate pushed and turned through a dam break.

The reference declares a rotating wall but never moves one (class.cuh:117-121,
kernel.cu:1879), so the oracle restates the motion defined here. These tests compare the
sm_100a path with the oracle exactly (==) over fused steps, check the walls' places against
the rigid motion computed in numpy, and check that a motion of zero changes nothing.
"""
from __future__ import annotations

import numpy as np
import pytest

from mps_cuda_b200 import F32, F64, MPS, MPSError, SceneDesc, dambreak, dambreak_params
from mps_cuda_b200 import _lib as L
from oracle.oracle import Oracle, params_from

pytestmark = pytest.mark.gpu

DESC = SceneDesc(l0=0.02, tank=(0.4, 0.2, 0.4), block=(8, 6, 10), jitter=0.01, seed=3)
DT = 2e-4
FIELDS = ("pos", "vel", "acc", "prs", "pav")


def _scene():
    """The dam break with a vertical OBJ plate at x = 0.172 m facing the fluid (-x): the
    block's last layer of particles sits at x = 0.15 m, so the plate's mirrors reach it."""
    sc = dambreak(DESC)
    l0 = DESC.l0
    ys = (np.arange(int(DESC.tank[1] / l0)) + 0.5) * l0
    zs = (np.arange(int(0.3 / l0)) + 0.5) * l0
    yy, zz = np.meshgrid(ys, zs, indexing="ij")
    m = yy.size
    plate = np.stack([np.full(m, 0.172), yy.ravel(), zz.ravel()])
    typ = np.concatenate([sc["typ"], np.full(m, L.OBJ, np.int8)])
    pos = np.concatenate([sc["pos"], plate], axis=1)
    vel = np.concatenate([sc["vel"], np.zeros((3, m))], axis=1)
    nrm = np.concatenate([sc["nrm"], np.tile([[-1.0], [0.0], [0.0]], (1, m))], axis=1)
    return typ, pos, vel, nrm


MOTION = dict(center=(0.172, 0.1, 0.15), axis=(0.0, 0.0, 1.0), omega=2.0, velocity=(-0.5, 0.0, 0.0))


def _pair(prec, motion=MOTION):
    typ, pos, vel, nrm = _scene()
    p = dambreak_params(DESC, dt=DT, precision=prec)
    d = np.float64 if prec == F64 else np.float32
    args = (typ, pos.astype(d), vel.astype(d), nrm.astype(d))
    g = MPS(p, *args)
    o = Oracle(params_from(p), *args)
    if motion is not None:
        g.set_wall_motion(L.OBJ, **motion)
        o.set_wall_motion(L.OBJ, **motion)
    return g, o, p, args


def _same(a, b, where):
    assert np.array_equal(a["typ"], b["typ"]), where
    for f in FIELDS:
        assert np.array_equal(a[f], b[f]), (where, f, np.abs(a[f].astype(float) - b[f]).max())


@pytest.mark.parametrize("prec", [F32, F64])
@pytest.mark.parametrize("graph", [0, 1])
def test_moving_plate_bit_exact(prec, graph):
    g, o, _, _ = _pair(prec)
    g.set_option(L.OPT_GRAPH, graph)
    try:
        for chunk in (1, 4, 15):
            g.step(chunk)
            o.step(chunk)
            _same(g.state(), o.state(), chunk)
        assert np.array_equal(g.wall_flags(), o.wall_flags())
        gm, om = g.mirrors(2), o.mirrors()
        assert np.array_equal(gm["slot"], om["slot"]) and np.array_equal(gm["pos"], om["pos"])
    finally:
        g.close()


def test_walls_follow_the_rigid_motion():
    g, _, p, args = _pair(F64)
    typ, pos0 = args[0], args[1]
    plate = np.nonzero(typ == L.OBJ)[0]
    k = 20
    try:
        g.step(k)
        st = g.state()
    finally:
        g.close()
    t = k * p.dt
    th = MOTION["omega"] * t
    c = np.array(MOTION["center"])[:, None]
    rot = np.array([[np.cos(th), -np.sin(th), 0.0], [np.sin(th), np.cos(th), 0.0], [0.0, 0.0, 1.0]])
    want = c + np.array(MOTION["velocity"])[:, None] * t + rot @ (pos0[:, plate] - c)
    np.testing.assert_allclose(st["pos"][:, plate], want, atol=1e-12)
    r = rot @ (pos0[:, plate] - c)
    w = np.array([0.0, 0.0, MOTION["omega"]])
    vwant = np.array(MOTION["velocity"])[:, None] + np.cross(w, r.T).T
    np.testing.assert_allclose(st["vel"][:, plate], vwant, atol=1e-12)
    # the other walls and the distances inside the plate are untouched
    others = np.nonzero((typ != L.OBJ) & (typ != L.FLD))[0]
    assert np.array_equal(st["pos"][:, others], pos0[:, others])
    d0 = np.linalg.norm(pos0[:, plate[0:1]] - pos0[:, plate], axis=0)
    d1 = np.linalg.norm(st["pos"][:, plate[0:1]] - st["pos"][:, plate], axis=0)
    np.testing.assert_allclose(d1, d0, atol=1e-12)


def test_the_plate_pushes_the_fluid():
    still, _, _, _ = _pair(F32, motion=None)
    moving, _, _, _ = _pair(F32)
    try:
        still.step(100)
        moving.step(100)
        a, b = still.state(), moving.state()
    finally:
        still.close()
        moving.close()
    fl = a["typ"] == L.FLD
    # the plate moved 1 cm toward the block's side: the fluid there is pushed back, so the
    # mean x-velocity is lower (by 1.7e-3 m/s in 20 ms, from the layers next to the plate)
    assert b["vel"][0][fl].mean() < a["vel"][0][fl].mean() - 1e-3
    near = fl & (a["pos"][0] > 0.12)
    assert b["vel"][0][near].mean() < a["vel"][0][near].mean() - 2e-3


def test_zero_motion_changes_nothing():
    a, _, _, _ = _pair(F32, motion=None)
    b, _, _, _ = _pair(F32, motion=dict(center=(0, 0, 0), axis=None, omega=0.0,
                                        velocity=(0.0, 0.0, 0.0)))
    c, _, _, args = _pair(F32)
    plate = np.nonzero(args[0] == L.OBJ)[0]
    try:
        for h in (a, b):
            h.step(10)
        _same(a.state(), b.state(), "zero motion")
        c.step(5)
        moved = c.state()["pos"][:, plate]
        assert not np.array_equal(moved, args[1][:, plate])
        c.set_wall_motion(L.OBJ, (0, 0, 0))  # stop: the walls stay where they are
        c.step(10)
        assert np.array_equal(c.state()["pos"][:, plate], moved)
    finally:
        for h in (a, b, c):
            h.close()


def test_errors():
    g, _, _, _ = _pair(F64)
    try:
        with pytest.raises(MPSError) as e:
            g.set_wall_motion(L.WLL, (0, 0, 0), velocity=(1.0, 0, 0))
        assert e.value.code == L.MPS_ERR_ARG
        with pytest.raises(MPSError):
            g.set_wall_motion(L.OBJ, (0, 0, 0), axis=(0, 0, 0), omega=1.0)
        with pytest.raises(MPSError) as e:
            g.adjoint_record(2, 1)
        assert e.value.code == L.MPS_ERR_UNSUPPORTED
    finally:
        g.close()


def test_moving_plate_with_the_corrected_gradient():
    """The two options together: still the oracle's state, exactly."""
    g, o, _, _ = _pair(F64)
    g.set_option(L.OPT_GRADIENT, L.GRAD_CORRECTED)
    o.set_gradient(1)
    try:
        g.step(12)
        o.step(12)
        _same(g.state(), o.state(), "corrected + moving")
    finally:
        g.close()
