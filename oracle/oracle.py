"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs use this module; it checks
the product, it is never part of it. See mps_oracle.cpp for what the oracle restates.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libmps_oracle.so")
_lib = None

c_int8_p = C.POINTER(C.c_int8)
c_int32_p = C.POINTER(C.c_int32)


class oracle_params(C.Structure):
    _fields_ = [("pcl_dst", C.c_double), ("min", C.c_double * 3), ("max", C.c_double * 3),
                ("g", C.c_double * 3), ("knm_vsc", C.c_double), ("col_rat", C.c_double),
                ("dst_lmt_rat", C.c_double), ("rho", C.c_double), ("snd", C.c_double),
                ("dt", C.c_double), ("umax", C.c_double), ("pmax", C.c_double),
                ("precision", C.c_int32), ("reserved", C.c_int32 * 7)]


class oracle_scene_desc(C.Structure):
    _fields_ = [("l0", C.c_double), ("tank", C.c_double * 3), ("block", C.c_int32 * 3),
                ("wall_mask", C.c_int32), ("jitter", C.c_double), ("seed", C.c_uint64),
                ("vel_sigma", C.c_double), ("vel_seed", C.c_uint64), ("origin", C.c_double * 3)]


c_double_p = C.POINTER(C.c_double)

SIGS = {
    "oracle_scene_dambreak_count": (C.c_int, [C.POINTER(oracle_scene_desc), c_int32_p]),
    "oracle_scene_dambreak": (C.c_int, [C.POINTER(oracle_scene_desc), C.c_int32, c_int8_p,
                                        c_double_p, c_double_p, c_double_p]),
    "oracle_params_dambreak": (C.c_int, [C.POINTER(oracle_scene_desc), C.c_double, C.c_double,
                                         C.c_double, C.c_double, C.c_int32,
                                         C.POINTER(oracle_params)]),
    "oracle_create": (C.c_void_p, [C.POINTER(oracle_params), C.c_int32, c_int8_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p]),
    "oracle_destroy": (None, [C.c_void_p]),
    "oracle_set_threads": (C.c_int, [C.c_int32]),
    "oracle_phase": (C.c_int, [C.c_void_p, C.c_int32]),
    "oracle_step": (C.c_int, [C.c_void_p, C.c_int32]),
    "oracle_set_gradient": (C.c_int, [C.c_void_p, C.c_int32]),
    "oracle_set_wall_motion": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_double),
                                         C.POINTER(C.c_double), C.c_double, C.POINTER(C.c_double)]),
    "oracle_get_state": (C.c_int, [C.c_void_p, c_int8_p] + [C.c_void_p] * 5),
    "oracle_set_state": (C.c_int, [C.c_void_p, c_int8_p] + [C.c_void_p] * 5),
    "oracle_get_wall_flags": (C.c_int, [C.c_void_p, c_int8_p]),
    "oracle_set_wall_flags": (C.c_int, [C.c_void_p, c_int8_p]),
    "oracle_get_mirrors": (C.c_int, [C.c_void_p, C.c_int32, c_int32_p, C.c_void_p, C.c_void_p,
                                     c_int32_p]),
    "oracle_set_mirrors": (C.c_int, [C.c_void_p, C.c_int32, c_int32_p, C.c_void_p, C.c_void_p]),
    "oracle_get_diag": (C.c_int, [C.c_void_p, c_int32_p, C.c_void_p]),
    "oracle_get_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "oracle_get_integrals": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
}

INFO_KEYS = ["n0", "lmd", "n0_grad", "lmd_grad", "numn0_grad", "r", "rp", "db", "dbinv", "nbx",
             "nby", "nbz", "rlim2", "col", "prs_coef", "minc_x", "minc_y", "minc_z", "maxc_x",
             "maxc_y", "maxc_z", "err_mirror_slot"]
DIAG_COLUMNS = ["cell", "vsc_f", "vsc_m", "col_f", "col_w", "col_m", "prs_f", "prs_m", "grd_f",
                "grd_m", "gen_w"]


def build():
    srcs = [os.path.join(HERE, f) for f in ("mps_oracle.cpp", "oracle_scene.cpp", "mps_oracle.h")]
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(map(os.path.getmtime, srcs)):
        subprocess.run(["make", "-C", HERE, "libmps_oracle.so"], check=True, capture_output=True)
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        for k, (r, a) in SIGS.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def params_from(p) -> oracle_params:
    """Copy an mps_params (same field order) into an oracle_params."""
    q = oracle_params()
    C.memmove(C.byref(q), C.byref(p), C.sizeof(q))
    return q


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Oracle:
    def __init__(self, params, typ, pos, vel, nrm, threads: int | None = None):
        self.p = params_from(params) if not isinstance(params, oracle_params) else params
        self.precision = self.p.precision
        self.dtype = np.float64 if self.precision == 1 else np.float32
        typ = np.ascontiguousarray(typ, np.int8)
        self.n = typ.shape[0]
        cv = lambda a: np.ascontiguousarray(np.asarray(a).reshape(3, self.n), self.dtype)
        pos, vel, nrm = cv(pos), cv(vel), cv(nrm)
        if threads:
            lib().oracle_set_threads(threads)
        self.h = lib().oracle_create(C.byref(self.p), self.n, typ.ctypes.data_as(c_int8_p),
                                     _ptr(pos), _ptr(vel), _ptr(nrm))
        if not self.h:
            raise RuntimeError("oracle_create failed")

    def close(self):
        if self.h:
            lib().oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def phase(self, ph):
        assert lib().oracle_phase(self.h, ph) == 0

    def step(self, n=1):
        assert lib().oracle_step(self.h, n) == 0

    def set_wall_motion(self, typ: int, center, axis=None, omega: float = 0.0,
                        velocity=(0.0, 0.0, 0.0)):
        c = (C.c_double * 3)(*[float(x) for x in center])
        a = None if axis is None else (C.c_double * 3)(*[float(x) for x in axis])
        v = (C.c_double * 3)(*[float(x) for x in velocity])
        assert lib().oracle_set_wall_motion(self.h, int(typ), c, a, float(omega), v) == 0

    def set_gradient(self, mode: int):
        """PrsGrdTrm variant: 0 as compiled, 1 the corrected-matrix #if 0 variant."""
        assert lib().oracle_set_gradient(self.h, int(mode)) == 0

    def state(self):
        n, dt = self.n, self.dtype
        o = {"typ": np.empty(n, np.int8), "pos": np.empty((3, n), dt), "vel": np.empty((3, n), dt),
             "acc": np.empty((3, n), dt), "prs": np.empty(n, dt), "pav": np.empty(n, dt)}
        lib().oracle_get_state(self.h, o["typ"].ctypes.data_as(c_int8_p), _ptr(o["pos"]),
                               _ptr(o["vel"]), _ptr(o["acc"]), _ptr(o["prs"]), _ptr(o["pav"]))
        return o

    def set_state(self, typ=None, pos=None, vel=None, acc=None, prs=None, pav=None):
        dt, n = self.dtype, self.n
        cv = lambda a, s: None if a is None else np.ascontiguousarray(np.asarray(a).reshape(s), dt)
        typ = None if typ is None else np.ascontiguousarray(typ, np.int8)
        pos, vel, acc, prs, pav = cv(pos, (3, n)), cv(vel, (3, n)), cv(acc, (3, n)), cv(prs, (n,)), cv(pav, (n,))
        lib().oracle_set_state(self.h, None if typ is None else typ.ctypes.data_as(c_int8_p),
                               _ptr(pos), _ptr(vel), _ptr(acc), _ptr(prs), _ptr(pav))

    def wall_flags(self):
        o = np.empty(self.n, np.int8)
        lib().oracle_get_wall_flags(self.h, o.ctypes.data_as(c_int8_p))
        return o

    def set_wall_flags(self, w):
        w = np.ascontiguousarray(w, np.int8)
        lib().oracle_set_wall_flags(self.h, w.ctypes.data_as(c_int8_p))

    def mirrors(self):
        n = C.c_int32()
        lib().oracle_get_mirrors(self.h, 0, None, None, None, C.byref(n))
        cap = max(n.value, 1)
        slot = np.empty(cap, np.int32)
        pos = np.empty((3, cap), self.dtype)
        prs = np.empty(cap, self.dtype)
        lib().oracle_get_mirrors(self.h, cap, slot.ctypes.data_as(c_int32_p), _ptr(pos), _ptr(prs),
                                 C.byref(n))
        m = n.value
        return {"slot": slot[:m], "pos": pos[:, :m], "prs": prs[:m]}

    def set_mirrors(self, slot, pos, prs):
        slot = np.ascontiguousarray(slot, np.int32)
        m = slot.shape[0]
        pos = np.ascontiguousarray(np.asarray(pos).reshape(3, m), self.dtype)
        prs = np.ascontiguousarray(prs, self.dtype)
        assert lib().oracle_set_mirrors(self.h, m, slot.ctypes.data_as(c_int32_p), _ptr(pos),
                                        _ptr(prs)) == 0

    def diag(self):
        tab = np.empty((self.n, len(DIAG_COLUMNS)), np.int32)
        nd = np.empty(self.n, self.dtype)
        lib().oracle_get_diag(self.h, tab.ctypes.data_as(c_int32_p), _ptr(nd))
        out = {k: tab[:, i].copy() for i, k in enumerate(DIAG_COLUMNS)}
        out["ndens"] = nd
        return out

    def info(self):
        v = (C.c_double * 32)()
        lib().oracle_get_info(self.h, v)
        return dict(zip(INFO_KEYS, v[: len(INFO_KEYS)]))

    def integrals(self):
        v = (C.c_double * 6)()
        lib().oracle_get_integrals(self.h, v)
        return np.array(v[:])
