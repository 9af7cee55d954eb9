"""ctypes binding of ``libmps_b200.so`` (the C-ABI in ``include/mps_b200.h``).

The library is loaded from this package directory. If it is missing or older than its
sources it is rebuilt with nvcc; if that is impossible the import fails loudly -- there is no
CPU fallback behind this package.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from . import build as _build

_lock = threading.Lock()
_lib = None

c_int8_p = C.POINTER(C.c_int8)
c_int32_p = C.POINTER(C.c_int32)
c_double_p = C.POINTER(C.c_double)

# status codes / enums (mirror include/mps_b200.h)
MPS_OK, MPS_ERR_ARG, MPS_ERR_CUDA, MPS_ERR_NOMEM, MPS_ERR_STATE = 0, 1, 2, 3, 4
MPS_ERR_OVERFLOW, MPS_ERR_TIMEOUT, MPS_ERR_UNSUPPORTED, MPS_ERR_NODEVICE = 5, 6, 7, 8
GST, FLD, WLL, OBJ, OBJ2, MRR = -1, 0, 1, 2, 3, 4
SURFACE, EDGE = 0, 1
NUM_MRR = 10
NOALLOC_MAX_ITEMS = 1 << 20
NOALLOC_MAX_BUCKETS = 1 << 20
F32, F64, F32_N64 = 0, 1, 2
(PHASE_MKBKT, PHASE_SURFACE_EDGE, PHASE_RESETMRR, PHASE_GENMRR_NONSLIP, PHASE_MKBKT_MRR,
 PHASE_VSCTRM, PHASE_UPPCL1, PHASE_CHKCOL, PHASE_MKPRS, PHASE_PRSGRDTRM, PHASE_UPPCL2) = range(11)
OPT_DIAG, OPT_GRAPH, OPT_BLOCK, OPT_CELL_SKIP, OPT_TIMING, OPT_GRADIENT = 0, 1, 2, 3, 4, 5
OPT_LIST_CAPACITY = 6
OPT_STAGING, OPT_STAGE_CAPACITY, OPT_CANDIDATE_BATCH = 7, 8, 9
OPT_REGISTER_BOUND = 10
OPT_OVERLAP = 11
STAGE_GLOBAL, STAGE_POSITIONS, STAGE_VELOCITIES = 0, 1, 2
GRAD_STANDARD, GRAD_CORRECTED = 0, 1
KERNEL_GROUPS = ["pass_a", "pass_b", "pass_c", "gen_cull", "bin_fluid", "bin_mirror"]
DIAG_COLUMNS = ["cell", "vsc_f", "vsc_m", "col_f", "col_w", "col_m", "prs_f", "prs_m",
                "grd_f", "grd_m", "gen_w"]


class mps_params(C.Structure):
    _fields_ = [("pcl_dst", C.c_double), ("min", C.c_double * 3), ("max", C.c_double * 3),
                ("g", C.c_double * 3), ("knm_vsc", C.c_double), ("col_rat", C.c_double),
                ("dst_lmt_rat", C.c_double), ("rho", C.c_double), ("snd", C.c_double),
                ("dt", C.c_double), ("umax", C.c_double), ("pmax", C.c_double),
                ("precision", C.c_int32), ("reserved", C.c_int32 * 7)]


class mps_info(C.Structure):
    _fields_ = [("n_particles", C.c_int32), ("n_fluid", C.c_int32), ("n_wall", C.c_int32),
                ("nbx", C.c_int32), ("nby", C.c_int32), ("nbz", C.c_int32), ("nbxyz", C.c_int32),
                ("r", C.c_double), ("rp", C.c_double), ("db", C.c_double), ("dbinv", C.c_double),
                ("n0", C.c_double), ("lmd", C.c_double), ("n0_grad", C.c_double),
                ("lmd_grad", C.c_double), ("numn0_grad", C.c_int32), ("pad0", C.c_int32),
                ("rlim2", C.c_double), ("col", C.c_double), ("prs_coef", C.c_double),
                ("pmax", C.c_double), ("umax", C.c_double), ("dt", C.c_double),
                ("snd", C.c_double), ("minc", C.c_double * 3), ("maxc", C.c_double * 3)]


class mps_counters(C.Structure):
    _fields_ = [("steps", C.c_int64), ("n_fluid_alive", C.c_int32), ("n_deleted", C.c_int32),
                ("n_mirror_1", C.c_int32), ("n_mirror_2", C.c_int32),
                ("err_mirror_slot", C.c_int32), ("err_mirror_capacity", C.c_int32),
                ("err_cell_range", C.c_int32), ("err_nan", C.c_int32),
                ("reserved0", C.c_int32), ("kernel_launches", C.c_int64),
                ("stage_blocks", C.c_int32), ("unstaged_blocks", C.c_int32)]


class mps_work(C.Structure):
    _fields_ = [("visc_candidates", C.c_int64), ("list_candidates", C.c_int64),
                ("list_entries", C.c_int64), ("reserved", C.c_int64 * 5)]


class mps_arith(C.Structure):
    _fields_ = [("fp32_fma_flops", C.c_double), ("fp64_fma_flops", C.c_double),
                ("fp32_sqrt_per_s", C.c_double), ("fp32_div_per_s", C.c_double),
                ("fp64_sqrt_per_s", C.c_double), ("fp64_div_per_s", C.c_double),
                ("warp_issue_per_s", C.c_double), ("sms", C.c_int32), ("clock_khz", C.c_int32),
                ("reserved", C.c_double * 4)]


class mps_physical(C.Structure):
    _fields_ = [("min", C.c_double * 3), ("max", C.c_double * 3), ("g", C.c_double * 3),
                ("fin_tim", C.c_double), ("output_time", C.c_double), ("mach", C.c_double),
                ("courant", C.c_double), ("col_rat", C.c_double), ("dst_lmt_rat", C.c_double),
                ("knm_vsc", C.c_double), ("pcl_dst", C.c_double)]


class mps_scene_desc(C.Structure):
    _fields_ = [("l0", C.c_double), ("tank", C.c_double * 3), ("block", C.c_int32 * 3),
                ("wall_mask", C.c_int32), ("jitter", C.c_double), ("seed", C.c_uint64),
                ("vel_sigma", C.c_double), ("vel_seed", C.c_uint64), ("origin", C.c_double * 3)]


# symbol -> (restype, argtypes); every symbol include/mps_b200.h declares
SIGNATURES = {
    "mps_scene_dambreak_count": (C.c_int, [C.POINTER(mps_scene_desc), c_int32_p]),
    "mps_scene_dambreak": (C.c_int, [C.POINTER(mps_scene_desc), C.c_int32, c_int8_p, c_double_p,
                                     c_double_p, c_double_p, c_int32_p]),
    "mps_params_dambreak": (C.c_int, [C.POINTER(mps_scene_desc), C.c_double, C.c_double,
                                      C.c_double, C.c_double, C.c_int32, C.POINTER(mps_params)]),
    "mps_select_device": (C.c_int, [C.c_int32]),
    "mps_derive": (C.c_int, [C.POINTER(mps_params), C.POINTER(mps_info)]),
    "mps_create": (C.c_int, [C.POINTER(mps_params), C.c_int32, c_int8_p, C.c_void_p, C.c_void_p,
                             C.c_void_p, C.POINTER(C.c_void_p)]),
    "mps_create_batch": (C.c_int, [C.c_int32, C.POINTER(mps_params), c_int32_p, c_int8_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]),
    "mps_destroy": (C.c_int, [C.c_void_p]),
    "mps_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "mps_set_option": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "mps_synchronize": (C.c_int, [C.c_void_p]),
    "mps_step": (C.c_int, [C.c_void_p, C.c_int32]),
    "mps_phase": (C.c_int, [C.c_void_p, C.c_int32]),
    "mps_get_info": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(mps_info)]),
    "mps_get_state": (C.c_int, [C.c_void_p, c_int8_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.c_void_p]),
    "mps_set_state": (C.c_int, [C.c_void_p, c_int8_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.c_void_p]),
    "mps_get_wall_flags": (C.c_int, [C.c_void_p, c_int8_p]),
    "mps_get_mirrors": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, c_int32_p, C.c_void_p,
                                  C.c_void_p, c_int32_p]),
    "mps_get_diag": (C.c_int, [C.c_void_p, c_int32_p, C.c_void_p]),
    "mps_get_counters": (C.c_int, [C.c_void_p, C.POINTER(mps_counters)]),
    "mps_get_work": (C.c_int, [C.c_void_p, C.POINTER(mps_work)]),
    "mps_get_option": (C.c_int, [C.c_void_p, C.c_int32, c_int32_p]),
    "mps_measure_arith": (C.c_int, [C.POINTER(mps_arith)]),
    "mps_get_timing": (C.c_int, [C.c_void_p, C.c_int32, c_double_p, C.POINTER(C.c_int64),
                                 C.c_int32]),
    "mps_autotune": (C.c_int, [C.c_void_p, C.c_int32, c_int32_p]),
    "mps_get_integrals": (C.c_int, [C.c_void_p, C.c_int32, c_double_p]),
    "mps_adjoint_record": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32]),
    "mps_adjoint_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p, c_double_p]),
    "mps_bucket_build_noalloc": (C.c_int, [C.POINTER(mps_params), C.c_int32, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p]),
    "mps_read_physical": (C.c_int, [C.c_char_p, C.POINTER(mps_physical)]),
    "mps_write_physical": (C.c_int, [C.c_char_p, C.POINTER(mps_physical)]),
    "mps_read_initial": (C.c_int, [C.c_char_p, C.POINTER(mps_physical), C.c_int32, c_int8_p,
                                   c_double_p, c_double_p, c_int32_p]),
    "mps_write_initial": (C.c_int, [C.c_char_p, C.c_int32, c_int8_p, c_double_p, c_double_p]),
    "mps_params_from_physical": (C.c_int, [C.POINTER(mps_physical), C.c_int32, c_int8_p,
                                           c_double_p, C.c_int32, C.POINTER(mps_params)]),
    "mps_output_open": (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(C.c_void_p)]),
    "mps_output_write": (C.c_int, [C.c_void_p, C.c_int32, C.c_double]),
    "mps_output_restart": (C.c_int, [C.c_void_p]),
    "mps_output_close": (C.c_int, [C.c_void_p]),
    "mps_set_wall_motion": (C.c_int, [C.c_void_p, C.c_int32, c_double_p, c_double_p, C.c_double,
                                      c_double_p]),
    "mps_status_string": (C.c_char_p, [C.c_int32]),
    "mps_last_error": (C.c_char_p, []),
}


class MPSError(RuntimeError):
    def __init__(self, code: int, where: str, detail: str):
        super().__init__(f"{where}: status {code} ({detail})")
        self.code = code


def lib():
    """Load (building if needed) the native library."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = _build.LIB
        if not _build.up_to_date(path):
            _build.build()
        L = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
        return _lib


def check(rc: int, where: str) -> None:
    if rc != MPS_OK:
        L = lib()
        msg = (L.mps_last_error() or b"").decode(errors="replace")
        raise MPSError(rc, where, msg or L.mps_status_string(rc).decode())


def library_path() -> str:
    return os.path.abspath(_build.LIB)
