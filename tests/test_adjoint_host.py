"""Host side of the rollout adjoint: the loss helper and the C-ABI argument checks."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from mps_cuda_b200 import _lib as L
from mps_cuda_b200.adjoint import dambreak_loss


def test_dambreak_loss_numpy_and_torch_agree():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(0)
    pos = rng.uniform(0, 1, (3, 500))
    alive = rng.uniform(0, 1, 500) > 0.1
    target = np.array([0.4, 0.5, 0.6, 0.3])
    a = dambreak_loss(pos, alive, target)
    p = pos[:, alive]
    sel = p[0] > 0.7
    want = np.sum((p.mean(axis=1) - target[:3]) ** 2) + (p[2][sel].mean() - target[3]) ** 2
    assert a == pytest.approx(want, rel=1e-12)
    pt = torch.tensor(pos, requires_grad=True)
    b = dambreak_loss(pt, torch.tensor(alive), torch.tensor(target))
    assert float(b.detach()) == pytest.approx(a, rel=1e-12)
    b.backward()
    g = pt.grad.numpy()
    # d/dx of the centroid term: 2 (c - t) / n_alive on alive particles, zero on deleted ones
    c = p.mean(axis=1)
    assert np.allclose(g[1, alive], 2 * (c[1] - target[1]) / alive.sum())
    assert np.all(g[:, ~alive] == 0)


def test_dambreak_loss_empty_gate_counts_zero():
    pos = np.full((3, 10), 0.2)
    alive = np.ones(10, bool)
    assert dambreak_loss(pos, alive, np.array([0.2, 0.2, 0.2, 0.1])) == pytest.approx(0.01)


def test_adjoint_calls_check_arguments_without_gpu():
    lib = L.lib()
    assert lib.mps_adjoint_record(None, 0, 20) == L.MPS_ERR_ARG
    assert lib.mps_adjoint_record(None, 10, 0) == L.MPS_ERR_ARG
    assert lib.mps_adjoint_record(None, 10, 5) == L.MPS_ERR_ARG  # no handle
    g = C.c_double()
    assert lib.mps_adjoint_backward(None, None, None, None, None, C.byref(g)) == L.MPS_ERR_ARG
