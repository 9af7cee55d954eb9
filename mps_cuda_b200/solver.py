"""Host-side mirror of the reference's solver interface.

The reference's only interface is ``class MPS`` (class.cuh:5-144): argument-less methods
(``MkBkt``, ``Surface_Edge``, ``ResetMRR``, ``GenMRR_nonslip``, ``MkBkt_MRR``, ``VscTrm``,
``UpPcl1``, ``ChkCol``, ``MkPrs``, ``PrsGrdTrm``, ``UpPcl2``, ``DevicetoHost``, ``ClcMPS``)
acting on public members. :class:`MPS` keeps those method names and their meaning on top of
the C-ABI; every call goes to ``libmps_b200.so`` and runs on the GPU. Errors raise
:class:`MPSError` instead of ``exit(1)`` (const.cuh:87-95).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from ._lib import MPSError, check, lib

__all__ = ["MPS", "MPSBatch", "SceneDesc", "dambreak", "dambreak_params", "derive", "select_device", "MPSError",
           "real_dtype", "measure_arith"]


def real_dtype(precision: int):
    return np.float64 if precision == L.F64 else np.float32


@dataclass
class SceneDesc:
    """Dam-break scene (see ``mps_scene_desc`` in include/mps_b200.h)."""
    l0: float
    tank: tuple
    block: tuple
    wall_mask: int = 0x1F
    jitter: float = 0.01
    seed: int = 0
    vel_sigma: float = 0.0
    vel_seed: int = 1
    origin: tuple = (0.0, 0.0, 0.0)

    def c(self) -> L.mps_scene_desc:
        d = L.mps_scene_desc()
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


def dambreak(desc: SceneDesc) -> dict:
    """Particles of a dam-break scene: typ (n,), pos/vel/nrm (3, n) float64 SoA."""
    d = desc.c()
    n = C.c_int32()
    check(lib().mps_scene_dambreak_count(C.byref(d), C.byref(n)), "mps_scene_dambreak_count")
    n = n.value
    typ = np.empty(n, np.int8)
    pos = np.empty((3, n), np.float64)
    vel = np.empty((3, n), np.float64)
    nrm = np.empty((3, n), np.float64)
    out = C.c_int32()
    check(lib().mps_scene_dambreak(C.byref(d), n, typ.ctypes.data_as(L.c_int8_p),
                                   pos.ctypes.data_as(L.c_double_p), vel.ctypes.data_as(L.c_double_p),
                                   nrm.ctypes.data_as(L.c_double_p), C.byref(out)),
          "mps_scene_dambreak")
    return {"typ": typ, "pos": pos, "vel": vel, "nrm": nrm}


def dambreak_params(desc: SceneDesc, snd: float = 20.0, dt: float = 2e-4, nu: float = 1e-6,
                    g_z: float = -9.81, precision: int = L.F32, **over) -> L.mps_params:
    p = L.mps_params()
    check(lib().mps_params_dambreak(C.byref(desc.c()), snd, dt, nu, g_z, precision, C.byref(p)),
          "mps_params_dambreak")
    for k, v in over.items():
        if k in ("min", "max", "g"):
            getattr(p, k)[:] = list(v)
        else:
            setattr(p, k, v)
    return p


def select_device(device: int) -> None:
    """Make `device` current for handles created by this thread (one process per GPU)."""
    check(lib().mps_select_device(int(device)), "mps_select_device")


def measure_arith() -> dict:
    """Arithmetic throughput of the current device (mps_measure_arith): FP32/FP64 fused
    multiply-add flop/s, IEEE square roots and divisions per second, warp issue rate."""
    a = L.mps_arith()
    check(lib().mps_measure_arith(C.byref(a)), "mps_measure_arith")
    return {k: getattr(a, k) for k, _ in L.mps_arith._fields_ if k != "reserved"}


def derive(params: L.mps_params) -> L.mps_info:
    """Derived constants of a scene (host only, no GPU): AlcBkt + SetPara."""
    inf = L.mps_info()
    check(lib().mps_derive(C.byref(params), C.byref(inf)), "mps_derive")
    return inf


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class MPSBatch:
    """A solver handle holding one or more scenes (``mps_create_batch``)."""

    def __init__(self, params, typ, pos, vel, nrm, counts=None):
        if isinstance(params, L.mps_params):
            params = [params]
        self.nscene = len(params)
        self.precision = params[0].precision
        self.dtype = real_dtype(self.precision)
        typ = np.ascontiguousarray(typ, np.int8)
        self.n = typ.shape[0]
        if counts is None:
            counts = [self.n]
        counts = np.ascontiguousarray(counts, np.int32)
        if int(counts.sum()) != self.n:
            raise ValueError("counts do not add up to the particle count")
        pos = np.ascontiguousarray(np.asarray(pos).reshape(3, self.n), self.dtype)
        vel = np.ascontiguousarray(np.asarray(vel).reshape(3, self.n), self.dtype)
        nrm = np.ascontiguousarray(np.asarray(nrm).reshape(3, self.n), self.dtype)
        arr = (L.mps_params * self.nscene)(*params)
        h = C.c_void_p()
        check(lib().mps_create_batch(self.nscene, arr, counts.ctypes.data_as(L.c_int32_p),
                                     typ.ctypes.data_as(L.c_int8_p), _ptr(pos), _ptr(vel), _ptr(nrm),
                                     C.byref(h)), "mps_create")
        self._h = h
        self.counts = counts

    # -- life cycle --------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            for o in list(getattr(self, "_outputs", ())):  # output sets read this handle
                o.close()
            lib().mps_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    # -- options -----------------------------------------------------------------------
    def set_option(self, opt: int, value: int):
        check(lib().mps_set_option(self._h, opt, int(value)), "mps_set_option")

    def set_stream(self, stream_ptr: int):
        check(lib().mps_set_stream(self._h, C.c_void_p(stream_ptr)), "mps_set_stream")

    def get_option(self, opt: int) -> int:
        v = C.c_int32()
        check(lib().mps_get_option(self._h, int(opt), C.byref(v)), "mps_get_option")
        return v.value

    def synchronize(self):
        check(lib().mps_synchronize(self._h), "mps_synchronize")

    def set_wall_motion(self, typ: int, center, axis=None, omega: float = 0.0,
                        velocity=(0.0, 0.0, 0.0)):
        """Prescribed rigid motion of every wall of type `typ` (OBJ or OBJ2): rotation at
        omega rad/s about the line through `center` along `axis`, translation at `velocity`."""
        c = (C.c_double * 3)(*[float(x) for x in center])
        a = None if axis is None else (C.c_double * 3)(*[float(x) for x in axis])
        v = (C.c_double * 3)(*[float(x) for x in velocity])
        check(lib().mps_set_wall_motion(self._h, int(typ), c, a, float(omega), v),
              "mps_set_wall_motion")

    # -- stepping ----------------------------------------------------------------------
    def step(self, n: int = 1):
        check(lib().mps_step(self._h, int(n)), "mps_step")

    def phase(self, ph: int):
        check(lib().mps_phase(self._h, int(ph)), "mps_phase")

    # -- state -------------------------------------------------------------------------
    def info(self, scene: int = 0) -> L.mps_info:
        inf = L.mps_info()
        check(lib().mps_get_info(self._h, scene, C.byref(inf)), "mps_get_info")
        return inf

    def state(self, out: dict | None = None) -> dict:
        """DevicetoHost: the state in id order, into `out` (e.g. pinned buffers) if given;
        arrays missing from `out` are not copied."""
        n, dt = self.n, self.dtype
        if out is None:
            out = {"typ": np.empty(n, np.int8), "pos": np.empty((3, n), dt),
                   "vel": np.empty((3, n), dt), "acc": np.empty((3, n), dt),
                   "prs": np.empty(n, dt), "pav": np.empty(n, dt)}
        t = out.get("typ")
        check(lib().mps_get_state(self._h, None if t is None else t.ctypes.data_as(L.c_int8_p),
                                  _ptr(out.get("pos")), _ptr(out.get("vel")), _ptr(out.get("acc")),
                                  _ptr(out.get("prs")), _ptr(out.get("pav"))), "mps_get_state")
        return out

    def set_state(self, typ=None, pos=None, vel=None, acc=None, prs=None, pav=None):
        dt, n = self.dtype, self.n
        conv = lambda a, shp: None if a is None else np.ascontiguousarray(np.asarray(a).reshape(shp), dt)
        typ = None if typ is None else np.ascontiguousarray(typ, np.int8)
        pos, vel, acc = conv(pos, (3, n)), conv(vel, (3, n)), conv(acc, (3, n))
        prs, pav = conv(prs, (n,)), conv(pav, (n,))
        check(lib().mps_set_state(self._h, None if typ is None else typ.ctypes.data_as(L.c_int8_p),
                                  _ptr(pos), _ptr(vel), _ptr(acc), _ptr(prs), _ptr(pav)),
              "mps_set_state")

    def wall_flags(self) -> np.ndarray:
        out = np.empty(self.n, np.int8)
        check(lib().mps_get_wall_flags(self._h, out.ctypes.data_as(L.c_int8_p)), "mps_get_wall_flags")
        return out

    def mirrors(self, which: int = 1) -> dict:
        """Mirror particles sorted by slot id (i * NumMRR + k)."""
        n = C.c_int32()
        check(lib().mps_get_mirrors(self._h, which, 0, None, None, None, C.byref(n)), "mps_get_mirrors")
        cap = max(n.value, 1)
        slot = np.empty(cap, np.int32)
        pos = np.empty((3, cap), self.dtype)
        prs = np.empty(cap, self.dtype)
        check(lib().mps_get_mirrors(self._h, which, cap, slot.ctypes.data_as(L.c_int32_p), _ptr(pos),
                                    _ptr(prs), C.byref(n)), "mps_get_mirrors")
        m = n.value
        return {"slot": slot[:m], "pos": pos[:, :m], "prs": prs[:m]}

    def diag(self) -> dict:
        tab = np.empty((self.n, len(L.DIAG_COLUMNS)), np.int32)
        nd = np.empty(self.n, self.dtype)
        check(lib().mps_get_diag(self._h, tab.ctypes.data_as(L.c_int32_p), _ptr(nd)), "mps_get_diag")
        out = {k: tab[:, i].copy() for i, k in enumerate(L.DIAG_COLUMNS)}
        out["ndens"] = nd
        return out

    def counters(self) -> dict:
        c = L.mps_counters()
        check(lib().mps_get_counters(self._h, C.byref(c)), "mps_get_counters")
        return {k: getattr(c, k) for k, _ in L.mps_counters._fields_ if not k.startswith("reserved")}

    def work(self) -> dict:
        """Candidates tested and list entries of the steps run with MPS_OPT_DIAG."""
        w = L.mps_work()
        check(lib().mps_get_work(self._h, C.byref(w)), "mps_get_work")
        return {k: getattr(w, k) for k, _ in L.mps_work._fields_ if k != "reserved"}

    def timing(self, reset: bool = False) -> dict:
        """Per kernel group: (total device ms, launches) of the steps timed so far."""
        out = {}
        last = len(L.KERNEL_GROUPS) - 1
        for k, name in enumerate(L.KERNEL_GROUPS):
            ms, n = C.c_double(), C.c_int64()
            rs = 1 if (reset and k == last) else 0  # read every group before clearing
            check(lib().mps_get_timing(self._h, k, C.byref(ms), C.byref(n), rs), "mps_get_timing")
            out[name] = (ms.value, n.value)
        return out

    def autotune(self, trial_steps: int = 3) -> dict:
        """Pick the fastest shapes per kernel group (state restored afterwards): block
        sizes, where VscTrm's walk reads its candidates (key "staging"), its candidates per
        batch, and the register bound of passes B, C and A (key "register_bound", bits 0-2)."""
        out = (C.c_int32 * len(L.KERNEL_GROUPS))()
        check(lib().mps_autotune(self._h, int(trial_steps), out), "mps_autotune")
        d = dict(zip(L.KERNEL_GROUPS, out[:]))
        d["staging"] = self.get_option(L.OPT_STAGING)
        d["candidate_batch"] = self.get_option(L.OPT_CANDIDATE_BATCH)
        d["register_bound"] = self.get_option(L.OPT_REGISTER_BOUND)
        return d

    def integrals(self, scene: int = 0) -> np.ndarray:
        out = (C.c_double * 6)()
        check(lib().mps_get_integrals(self._h, scene, out), "mps_get_integrals")
        return np.array(out[:])

    def adjoint_record(self, nsteps: int, checkpoint_every: int = 20):
        """Advance nsteps steps, keeping the state every checkpoint_every steps."""
        check(lib().mps_adjoint_record(self._h, int(nsteps), int(checkpoint_every)),
              "mps_adjoint_record")

    def adjoint_backward(self, lam_pos=None, lam_vel=None, grad_pos=None, grad_vel=None):
        """Gradients of the recorded rollout's loss given d loss / d (final pos, vel).

        Arrays are (3, n) float64 in particle-id order: numpy arrays, or anything exposing
        a device pointer through ``data_ptr()`` (torch CUDA tensors). Output arrays are
        allocated as numpy when not given. Returns (grad_pos0, grad_vel0, grad_nu).
        """
        def ptr(a):
            if a is None:
                return None
            if hasattr(a, "data_ptr"):
                return C.c_void_p(a.data_ptr())
            assert a.dtype == np.float64 and a.flags.c_contiguous and a.shape == (3, self.n)
            return a.ctypes.data_as(C.c_void_p)
        if grad_pos is None:
            grad_pos = np.empty((3, self.n))
        if grad_vel is None:
            grad_vel = np.empty((3, self.n))
        gnu = C.c_double()
        check(lib().mps_adjoint_backward(self._h, ptr(lam_pos), ptr(lam_vel), ptr(grad_pos),
                                         ptr(grad_vel), C.byref(gnu)), "mps_adjoint_backward")
        return grad_pos, grad_vel, gnu.value


class MPS(MPSBatch):
    """One scene, driven with the reference's method names (class.cuh:8-28).

    ``ClcMPS(n)`` runs n iterations of the loop body of kernel.cu:1904-1941 as one fused,
    stream-ordered sequence; calling the individual methods in the reference's order gives
    the same state.
    """

    def __init__(self, params: L.mps_params, typ, pos, vel, nrm):
        super().__init__([params], typ, pos, vel, nrm)
        self.params = params

    # kernel.cu:532 / 671 / 704 / 896 / 987 / 1122 / 1152 / 1289 / 1414 / 1798 / 1831
    def MkBkt(self): self.phase(L.PHASE_MKBKT)
    def Surface_Edge(self): self.phase(L.PHASE_SURFACE_EDGE)
    def ResetMRR(self): self.phase(L.PHASE_RESETMRR)
    def GenMRR_nonslip(self): self.phase(L.PHASE_GENMRR_NONSLIP)
    def MkBkt_MRR(self): self.phase(L.PHASE_MKBKT_MRR)
    def VscTrm(self): self.phase(L.PHASE_VSCTRM)
    def UpPcl1(self): self.phase(L.PHASE_UPPCL1)
    def ChkCol(self): self.phase(L.PHASE_CHKCOL)
    def MkPrs(self): self.phase(L.PHASE_MKPRS)
    def PrsGrdTrm(self): self.phase(L.PHASE_PRSGRDTRM)
    def UpPcl2(self): self.phase(L.PHASE_UPPCL2)

    def DevicetoHost(self) -> dict:  # kernel.cu:1847-1869
        return self.state()

    def ClcMPS(self, nsteps: int):  # loop body kernel.cu:1904-1941, nsteps times
        self.step(nsteps)

    def step_by_methods(self):
        """One step as the reference's sequence of method calls (kernel.cu:1904-1935)."""
        self.MkBkt()
        self.ResetMRR(); self.GenMRR_nonslip(); self.MkBkt_MRR()
        self.VscTrm()
        self.UpPcl1()
        self.MkBkt()
        self.ChkCol()
        self.MkBkt()
        self.MkPrs()
        self.ResetMRR(); self.GenMRR_nonslip(); self.MkBkt_MRR()
        self.PrsGrdTrm()
        self.UpPcl2()
