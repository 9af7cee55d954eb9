"""The oracle's restatement of the moving walls, on the CPU (no GPU needed).

The oracle is the checker of tests/test_gpu_moving_walls.py, so its own motion is checked
here against the rigid motion computed directly in numpy: walls of the moving type follow
c + v t + R(omega t)(x0 - c) with normals R n0 and velocity v + omega x r, the other walls
stay, and a motion of zero changes nothing.
"""
from __future__ import annotations

import numpy as np

from mps_cuda_b200 import F64, SceneDesc, dambreak, dambreak_params
from mps_cuda_b200 import _lib as L
from oracle.oracle import Oracle, params_from

DESC = SceneDesc(l0=0.02, tank=(0.4, 0.2, 0.4), block=(6, 4, 6), jitter=0.01, seed=5)


def _scene():
    sc = dambreak(DESC)
    ys = (np.arange(10) + 0.5) * DESC.l0
    zs = (np.arange(8) + 0.5) * DESC.l0
    yy, zz = np.meshgrid(ys, zs, indexing="ij")
    m = yy.size
    plate = np.stack([np.full(m, 0.2), yy.ravel(), zz.ravel()])
    typ = np.concatenate([sc["typ"], np.full(m, L.OBJ2, np.int8)])
    pos = np.concatenate([sc["pos"], plate], axis=1)
    vel = np.concatenate([sc["vel"], np.zeros((3, m))], axis=1)
    nrm = np.concatenate([sc["nrm"], np.tile([[-1.0], [0.0], [0.0]], (1, m))], axis=1)
    return typ, pos, vel, nrm


def _rot(axis, th):
    a = np.asarray(axis, float) / np.linalg.norm(axis)
    k = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + np.sin(th) * k + (1 - np.cos(th)) * (k @ k)


def test_oracle_walls_follow_the_rigid_motion():
    typ, pos, vel, nrm = _scene()
    p = dambreak_params(DESC, dt=2e-4, precision=F64)
    o = Oracle(params_from(p), typ, pos, vel, nrm, threads=2)
    c, axis, om, v = (0.2, 0.1, 0.08), (0.3, 0.0, 1.0), 1.5, (-0.2, 0.05, 0.0)
    o.set_wall_motion(L.OBJ2, c, axis, om, v)
    k = 6
    o.step(k)
    st = o.state()
    plate = np.nonzero(typ == L.OBJ2)[0]
    t = k * p.dt
    rot = _rot(axis, om * t)
    cc = np.array(c)[:, None]
    r = rot @ (pos[:, plate] - cc)
    np.testing.assert_allclose(st["pos"][:, plate], cc + np.array(v)[:, None] * t + r, atol=1e-12)
    w = om * np.asarray(axis) / np.linalg.norm(axis)
    np.testing.assert_allclose(st["vel"][:, plate], np.array(v)[:, None] + np.cross(w, r.T).T,
                               atol=1e-12)
    others = np.nonzero((typ != L.OBJ2) & (typ != L.FLD))[0]
    assert np.array_equal(st["pos"][:, others], pos[:, others])
    # a plate of one normal stays a surface: every Edge flag of it is unchanged
    assert not o.wall_flags()[plate].any()


def test_oracle_zero_motion_changes_nothing():
    typ, pos, vel, nrm = _scene()
    p = dambreak_params(DESC, dt=2e-4, precision=F64)
    a = Oracle(params_from(p), typ, pos, vel, nrm, threads=2)
    b = Oracle(params_from(p), typ, pos, vel, nrm, threads=2)
    b.set_wall_motion(L.OBJ2, (0.0, 0.0, 0.0))
    a.step(3)
    b.step(3)
    sa, sb = a.state(), b.state()
    for f in ("typ", "pos", "vel", "prs"):
        assert np.array_equal(sa[f], sb[f]), f
