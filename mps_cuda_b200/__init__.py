"""mps_cuda_b200 -- B200-native explicit MPS solver (drop-in for frsykzk/MPS_CUDA's step).

The solver itself is ``libmps_b200.so`` (hand-written sm_100a kernels behind the C-ABI of
``include/mps_b200.h``); this package binds it with ctypes and mirrors the reference's
``class MPS`` method names. Importing the package does not touch the GPU.
"""
from ._lib import (F32, F32_N64, F64, FLD, GST, MRR, OBJ, OBJ2, WLL, MPSError, lib,
                   library_path)
from .solver import (MPS, MPSBatch, SceneDesc, dambreak, dambreak_params, derive,
                     measure_arith, real_dtype, select_device)

__all__ = ["MPS", "MPSBatch", "SceneDesc", "dambreak", "dambreak_params", "derive", "measure_arith",
           "select_device", "MPSError", "lib",
           "library_path", "real_dtype", "F32", "F64", "F32_N64", "GST", "FLD", "WLL", "OBJ",
           "OBJ2", "MRR"]
