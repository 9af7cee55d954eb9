"""The reference's files: MPS_physical.txt / initial.txt in, CSV snapshots and seitei.txt out.

A case directory prepared for frsykzk/MPS_CUDA (``MPS_physical.txt`` + ``initial.txt``, read by
RdDat, kernel.cu:4-143) runs here unchanged: :func:`load_case` reads it and derives the
parameters as SetPara does (kernel.cu:396-415), and :func:`run_case` drives the solver with
ClcMPS's output cadence (kernel.cu:1872-1943), writing the reference's files
(output%05d.csv, outputMRR%05d.csv, outputwall00000.csv, outputWLLvec00000.csv, seitei.txt)
through :class:`Output`. The parsing and formatting are native (``mps_io.cpp``,
``mps_output.cu``); the CSV files are formatted on a writer thread while the GPU steps on.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref

import numpy as np

from . import _lib as L
from ._lib import check, lib
from .solver import MPS


def _p(a):
    return a.ctypes.data_as(L.c_double_p)


def read_physical(path: str) -> L.mps_physical:
    """MPS_physical.txt (kernel.cu:12-22): 17 numbers, each read as a float."""
    ph = L.mps_physical()
    check(lib().mps_read_physical(os.fsencode(path), C.byref(ph)), "mps_read_physical")
    return ph


def write_physical(path: str, ph: L.mps_physical) -> None:
    check(lib().mps_write_physical(os.fsencode(path), C.byref(ph)), "mps_write_physical")


def physical(*, min, max, g, fin_tim, output_time, mach, courant, col_rat, dst_lmt_rat,
             knm_vsc, pcl_dst) -> L.mps_physical:
    """An mps_physical from keyword values (the 17 numbers of MPS_physical.txt)."""
    ph = L.mps_physical()
    for d in range(3):
        ph.min[d], ph.max[d], ph.g[d] = min[d], max[d], g[d]
    ph.fin_tim, ph.output_time, ph.mach, ph.courant = fin_tim, output_time, mach, courant
    ph.col_rat, ph.dst_lmt_rat, ph.knm_vsc, ph.pcl_dst = col_rat, dst_lmt_rat, knm_vsc, pcl_dst
    return ph


def read_initial(path: str, ph: L.mps_physical) -> dict:
    """initial.txt (kernel.cu:59-131): typ (n,), pos and inward nrm (3, n) as doubles, vel = 0.
    Particles outside the padded domain of ``ph`` are dropped, as RdDat drops them."""
    n = C.c_int32(0)
    rc = lib().mps_read_initial(os.fsencode(path), C.byref(ph), 0, None, None, None, C.byref(n))
    if rc != L.MPS_OK and n.value == 0:
        check(rc, "mps_read_initial")
    cap = max(n.value, 1)
    typ = np.zeros(cap, np.int8)
    pos = np.zeros(3 * cap)
    nrm = np.zeros(3 * cap)
    check(lib().mps_read_initial(os.fsencode(path), C.byref(ph), cap,
                                 typ.ctypes.data_as(L.c_int8_p), _p(pos), _p(nrm), C.byref(n)),
          "mps_read_initial")
    k = n.value
    return {"typ": typ[:k].copy(), "pos": pos[:3 * k].reshape(3, k).copy(),
            "nrm": nrm[:3 * k].reshape(3, k).copy(), "vel": np.zeros((3, k))}


def write_initial(path: str, typ, pos, nrm) -> None:
    """initial.txt from id-ordered arrays; the inward normals are written outward, as the
    file holds them."""
    typ = np.ascontiguousarray(typ, np.int8)
    n = typ.shape[0]
    pos = np.ascontiguousarray(np.asarray(pos, np.float64).reshape(3, n))
    nrm = np.ascontiguousarray(np.asarray(nrm, np.float64).reshape(3, n))
    check(lib().mps_write_initial(os.fsencode(path), n, typ.ctypes.data_as(L.c_int8_p), _p(pos),
                                  _p(nrm)), "mps_write_initial")


def params_from_physical(ph: L.mps_physical, typ, pos, precision: int = L.F32) -> L.mps_params:
    """SetPara's parameters (kernel.cu:396-415) for this scene."""
    typ = np.ascontiguousarray(typ, np.int8)
    n = typ.shape[0]
    pos = np.ascontiguousarray(np.asarray(pos, np.float64).reshape(3, n))
    p = L.mps_params()
    check(lib().mps_params_from_physical(C.byref(ph), n, typ.ctypes.data_as(L.c_int8_p), _p(pos),
                                         precision, C.byref(p)), "mps_params_from_physical")
    return p


def load_case(case_dir: str, precision: int = L.F32):
    """(params, scene, physical) of a reference case directory: RdDat + SetPara."""
    ph = read_physical(os.path.join(case_dir, "MPS_physical.txt"))
    sc = read_initial(os.path.join(case_dir, "initial.txt"), ph)
    return params_from_physical(ph, sc["typ"], sc["pos"], precision), sc, ph


class Output:
    """The reference's output files of one solver handle (WrtDat / WrtDatWLL / WrtDat2).

    Opening writes the wall files; :meth:`write` snapshots the state on the device and
    returns while a writer thread formats the CSV files; :meth:`close` waits for them."""

    def __init__(self, solver, directory: str):
        os.makedirs(directory, exist_ok=True)
        self.dir = directory
        self._o = None
        o = C.c_void_p()
        check(lib().mps_output_open(solver.handle, os.fsencode(directory), C.byref(o)),
              "mps_output_open")
        self._o = o
        # closing the solver closes its output sets first
        self._solver = weakref.ref(solver)
        if not hasattr(solver, "_outputs"):
            solver._outputs = weakref.WeakSet()
        solver._outputs.add(self)

    def write(self, index: int, opt_fqc: float) -> None:
        """output%05d.csv and outputMRR%05d.csv of the current state; then pav = 0."""
        check(lib().mps_output_write(self._o, int(index), float(opt_fqc)), "mps_output_write")

    def restart(self) -> None:
        """seitei.txt of the current state."""
        check(lib().mps_output_restart(self._o), "mps_output_restart")

    def close(self) -> None:
        if getattr(self, "_o", None) is not None:
            o, self._o = self._o, None
            s = self._solver()
            if s is not None and hasattr(s, "_outputs"):
                s._outputs.discard(self)
            check(lib().mps_output_close(o), "mps_output_close")

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def output_schedule(dt: float, output_time: float, fin_tim: float, max_files: int | None = None):
    """Steps between the output files of ClcMPS (kernel.cu:1872-1943), in the reference's
    float arithmetic: a file is written when outtime >= output_time at the top of the loop,
    outtime and TIM advance by dt after each step, and the run ends at the first file with
    TIM >= FIN_TIM. Yields the number of steps before each file after the first."""
    f32 = np.float32
    dt_, out_t, fin = f32(dt), f32(output_time), f32(fin_tim)
    if not (dt_ > 0 and out_t > 0):
        raise ValueError("dt and output_time must be positive")
    outtime, tim = f32(0.0), f32(0.0)
    files = 0
    while max_files is None or files < max_files:
        n = 0
        while not outtime >= out_t:
            outtime = f32(outtime + dt_)
            tim = f32(tim + dt_)
            n += 1
        outtime = f32(outtime - out_t)
        files += 1
        yield n, bool(tim >= fin)
        if tim >= fin:
            return


def run_case(case_dir: str, out_dir: str, precision: int = L.F32, max_files: int | None = None,
             dt: float | None = None) -> dict:
    """ClcMPS for a case directory: the initial files, then one output%05d.csv per
    output_time and seitei.txt at FIN_TIM (or after ``max_files`` further files). ``dt``
    overrides SetPara's step. Returns the steps run and the files written."""
    params, sc, ph = load_case(case_dir, precision)
    if dt is not None:
        params.dt = dt
    rd = np.float64 if precision == L.F64 else np.float32
    h = MPS(params, sc["typ"], sc["pos"].astype(rd), sc["vel"].astype(rd), sc["nrm"].astype(rd))
    steps = 0
    index = 0
    try:
        with Output(h, out_dir) as out:
            out.write(index, 1.0)  # WrtDat at OPT_FQC = 1 (kernel.cu:1876-1882)
            index += 1
            for n, _last in output_schedule(params.dt, ph.output_time, ph.fin_tim, max_files):
                h.step(n)
                steps += n
                out.write(index, float(np.float32(n)))  # OPT_FQC counts the interval's steps
                index += 1
            out.restart()  # WrtDat2 (kernel.cu:1897-1899)
    finally:
        h.close()
    return {"steps": steps, "files": index, "dt": params.dt}
