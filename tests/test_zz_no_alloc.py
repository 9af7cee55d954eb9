"""mps_bucket_build_noalloc: the bucket build for callers that cannot allocate device memory.

Such callers -- code inside another framework's memory pool, real-time loops that must not
allocate after start-up, plug-ins that only get input and output buffers -- call this entry
point with their own device buffers; its temporaries live in a fixed array inside the
library. The test checks its output through the C-ABI against the solver's own bucket build
(the bucket index mps_get_diag reports after MkBkt, and the order and start table that index
implies) and against the oracle's MkBkt on the same positions, on two calls in a row, the
second on a moved state while the fixed array still holds the first call's contents. The
comparison is exact: the outputs are integers.

This file is named to be collected last, so that a run stopping at the first failure has
already run every other test.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from mps_cuda_b200 import F32, MPS, configs, dambreak, dambreak_params, derive, select_device
from mps_cuda_b200 import _lib as L
from oracle.oracle import Oracle, params_from

pytestmark = pytest.mark.gpu


def _noalloc(torch, p, typ_d, pos_d, n, nb):
    cell = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    order = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    start = torch.full((nb + 1,), -7, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    rc = L.lib().mps_bucket_build_noalloc(
        C.byref(p), n, C.c_void_p(typ_d.data_ptr()), C.c_void_p(pos_d.data_ptr()),
        C.c_void_p(cell.data_ptr()), C.c_void_p(order.data_ptr()), C.c_void_p(start.data_ptr()),
        C.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    return rc, cell.cpu().numpy(), order.cpu().numpy(), start.cpu().numpy()


def test_noalloc_bucket_build_matches_solver():
    import torch
    torch.cuda.set_device(0)
    select_device(0)
    desc, dt, _ = configs.WORKLOADS["dambreak_l0.02_6k"]
    sc = dambreak(desc)
    p = dambreak_params(desc, dt=dt, precision=F32)
    g = MPS(p, sc["typ"], sc["pos"].astype(np.float32), sc["vel"].astype(np.float32),
            sc["nrm"].astype(np.float32))
    o = Oracle(params_from(p), sc["typ"], sc["pos"].astype(np.float32),
               sc["vel"].astype(np.float32), sc["nrm"].astype(np.float32))
    n = g.n
    nb = derive(p).nbxyz
    for call in range(2):
        st = g.state()
        want = g.diag()["cell"]  # the solver's bucket index of every particle, -1 for GST
        o.set_state(typ=st["typ"], pos=st["pos"])
        o.phase(L.PHASE_MKBKT)  # the oracle's MkBkt (kernel.cu:516-550) on the same positions
        assert np.array_equal(o.diag()["cell"], want), call
        typ_d = torch.from_numpy(st["typ"].copy()).cuda()
        pos_d = torch.from_numpy(np.ascontiguousarray(st["pos"])).cuda()
        rc, cell, order, start = _noalloc(torch, p, typ_d, pos_d, n, nb)
        assert rc == L.MPS_OK, L.lib().mps_last_error()
        assert np.array_equal(cell, want), call
        listed = np.nonzero(want >= 0)[0]
        expect_order = listed[np.lexsort((listed, want[listed]))]
        assert np.array_equal(order[: len(listed)], expect_order), call
        expect_start = np.concatenate([[0], np.cumsum(np.bincount(want[listed], minlength=nb))])
        assert np.array_equal(start, expect_start), call
        g.step(5)  # move the particles before the second call
    g.close()
    o.close()


def test_noalloc_rejects_sizes_beyond_its_array():
    p = dambreak_params(configs.WORKLOADS["dambreak_l0.02_6k"][0], precision=F32)
    one = C.c_void_p(1)  # never dereferenced: the size check comes first
    rc = L.lib().mps_bucket_build_noalloc(C.byref(p), L.NOALLOC_MAX_ITEMS + 1, one, one, one, one,
                                          one, None)
    assert rc == L.MPS_ERR_OVERFLOW
    assert b"MPS_NOALLOC_MAX_ITEMS" in L.lib().mps_last_error()
