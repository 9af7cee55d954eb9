"""ctypes binding of the reference's own kernels (oracle/_ref/libref_mps_*.so).

TEST INFRASTRUCTURE. The libraries are built by ref_build.sh from the reference sources and
run the reference's `class MPS` methods on the GPU. They exist only where that build ran;
callers check :func:`available` first.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
_libs = {}
c_int8_p = C.POINTER(C.c_int8)
c_int32_p = C.POINTER(C.c_int32)

PHASES = ["MkBkt", "Surface_Edge", "ResetMRR", "GenMRR_nonslip", "MkBkt_MRR", "VscTrm", "UpPcl1",
          "ChkCol", "MkPrs", "PrsGrdTrm", "UpPcl2"]
STEP_PHASES = [0, 2, 3, 4, 5, 6, 0, 7, 0, 8, 2, 3, 4, 9, 10]  # kernel.cu:1904-1935


def path(precision: int, corrected: bool = False) -> str:
    """The build of the default kernels, or with ``corrected`` the one whose d_PrsGrdTrm is
    the corrected-matrix variant (kernel.cu:1434-1648)."""
    name = ("corr_" if corrected else "") + ("f64" if precision == 1 else "f32")
    return os.path.join(REF_DIR, f"libref_mps_{name}.so")


def available(precision: int = 0, corrected: bool = False) -> bool:
    return os.path.exists(path(precision, corrected))


def lib(precision: int, corrected: bool = False):
    key = (1 if precision == 1 else 0, bool(corrected))
    if key not in _libs:
        L = C.CDLL(path(*key))
        L.ref_create.restype = C.c_void_p
        L.ref_create.argtypes = [C.c_void_p, C.c_int, c_int8_p, C.c_void_p, C.c_void_p, C.c_void_p]
        for nm in ("ref_phase", "ref_step"):
            getattr(L, nm).restype = C.c_int
            getattr(L, nm).argtypes = [C.c_void_p, C.c_int]
        L.ref_get_state.argtypes = [C.c_void_p, c_int8_p] + [C.c_void_p] * 5
        L.ref_set_state.argtypes = [C.c_void_p, c_int8_p] + [C.c_void_p] * 5
        L.ref_get_wall_flags.argtypes = [C.c_void_p, c_int8_p]
        L.ref_get_mirrors.argtypes = [C.c_void_p, c_int8_p, C.c_void_p, C.c_void_p, c_int32_p]
        L.ref_get_buckets.argtypes = [C.c_void_p, c_int32_p]
        L.ref_get_list_order.argtypes = [C.c_void_p, C.c_int, c_int32_p, c_int32_p]
        L.ref_get_info.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        _libs[key] = L
    return _libs[key]


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Reference:
    """The reference solver on one scene (device memory is never freed by the reference)."""

    def __init__(self, params, typ, pos, vel, nrm, corrected: bool = False):
        self.precision = 1 if params.precision == 1 else 0
        self.dtype = np.float64 if self.precision == 1 else np.float32
        self.L = lib(self.precision, corrected)
        assert self.L.ref_real_size() == np.dtype(self.dtype).itemsize
        typ = np.ascontiguousarray(typ, np.int8)
        self.n = typ.shape[0]
        cv = lambda a: np.ascontiguousarray(np.asarray(a).reshape(3, self.n), self.dtype)
        self._keep = (cv(pos), cv(vel), cv(nrm))
        self.h = self.L.ref_create(C.byref(params), self.n, typ.ctypes.data_as(c_int8_p),
                                   *(_p(a) for a in self._keep))
        if not self.h:
            raise RuntimeError("ref_create failed")

    def phase(self, ph):
        rc = self.L.ref_phase(self.h, ph)
        if rc:
            raise RuntimeError(f"reference phase {ph} failed ({rc})")

    def step(self, n=1):
        rc = self.L.ref_step(self.h, n)
        if rc:
            raise RuntimeError(f"reference step failed ({rc})")

    def state(self):
        n, dt = self.n, self.dtype
        o = {"typ": np.empty(n, np.int8), "pos": np.empty((3, n), dt), "vel": np.empty((3, n), dt),
             "acc": np.empty((3, n), dt), "prs": np.empty(n, dt), "pav": np.empty(n, dt)}
        self.L.ref_get_state(self.h, o["typ"].ctypes.data_as(c_int8_p), _p(o["pos"]), _p(o["vel"]),
                             _p(o["acc"]), _p(o["prs"]), _p(o["pav"]))
        return o

    def wall_flags(self):
        o = np.empty(self.n, np.int8)
        self.L.ref_get_wall_flags(self.h, o.ctypes.data_as(c_int8_p))
        return o

    def mirror_slots(self):
        nm = self.n * 10
        t = np.empty(nm, np.int8)
        p = np.empty((3, nm), self.dtype)
        q = np.empty(nm, self.dtype)
        f = np.empty(nm, np.int32)
        self.L.ref_get_mirrors(self.h, t.ctypes.data_as(c_int8_p), _p(p), _p(q),
                               f.ctypes.data_as(c_int32_p))
        return {"typ": t, "pos": p, "prs": q, "from": f}

    def mirrors(self):
        """Live mirrors (TypM == MRR) sorted by slot."""
        m = self.mirror_slots()
        idx = np.nonzero(m["typ"] == 4)[0]
        return {"slot": idx.astype(np.int32), "pos": m["pos"][:, idx], "prs": m["prs"][idx]}

    def buckets(self):
        o = np.empty(self.n, np.int32)
        self.L.ref_get_buckets(self.h, o.ctypes.data_as(c_int32_p))
        return o

    def list_order(self):
        """Per bucket, the particles in the order of the reference's linked lists:
        (order, start) with bucket b's particles order[start[b]:start[b + 1]]."""
        nb = int(self.info()["nbx"] * self.info()["nby"] * self.info()["nbz"])
        order = np.empty(self.n, np.int32)
        start = np.empty(nb + 1, np.int32)
        self.L.ref_get_list_order(self.h, self.n, order.ctypes.data_as(c_int32_p),
                                  start.ctypes.data_as(c_int32_p))
        return order, start

    def info(self):
        v = (C.c_double * 21)()
        self.L.ref_get_info(self.h, v)
        keys = ["n0", "lmd", "n0_grad", "lmd_grad", "numn0_grad", "r", "rp", "db", "dbinv", "nbx",
                "nby", "nbz", "rlim2", "col", "prs_coef", "minc_x", "minc_y", "minc_z", "maxc_x",
                "maxc_y", "maxc_z"]
        return dict(zip(keys, v[:]))
