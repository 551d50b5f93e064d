"""Loader for librmetis_gpu.so (the in-tree CUDA build). There is no CPU
fallback: if the library is missing, importing the bindings raises."""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librmetis_gpu.so")

I32P = ctypes.POINTER(ctypes.c_int32)
I64P = ctypes.POINTER(ctypes.c_int64)
F32P = ctypes.POINTER(ctypes.c_float)
F64P = ctypes.POINTER(ctypes.c_double)
VP = ctypes.c_void_p

# Every symbol declared in include/rmetis.h with its ctypes signature.
SIGNATURES = {
    "RMETIS_SetDefaultOptions": [I32P],
    "RMETIS_PartGraphKway": [I32P, I32P, I32P, I32P, I32P, I32P, I32P, I32P, F32P, F32P, I32P, I32P, I32P],
    "RMETIS_PartGraphRecursive": [I32P, I32P, I32P, I32P, I32P, I32P, I32P, I32P, F32P, F32P, I32P, I32P, I32P],
    "RMETIS_NodeND": [I32P, I32P, I32P, I32P, I32P, I32P, I32P],
    "RMETIS_GPU_PartGraphKwayDevice": [I32P, I32P, VP, VP, VP, VP, I32P, F32P, F32P, I32P, I32P, VP],
    "RMETIS_GPU_SetStream": [VP],
    "RMETIS_GPU_SetTuning": [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int],
    "RMETIS_GPU_SetPoolTuning": [ctypes.c_int, ctypes.c_int],
    "RMETIS_GPU_SetRefineMode": [ctypes.c_int],
    "RMETIS_GPU_SetKernelShapes": [ctypes.c_int, ctypes.c_int],
    "RMETIS_GPU_SetProfiling": [ctypes.c_int],
    "RMETIS_GPU_GetProfile": [I64P, F64P, F64P, ctypes.c_int],
    "RMETIS_GPU_PartGraphKwayTrace": [I32P, I32P, I32P, I32P, I32P, I32P, I32P, F32P, F32P, I32P, I32P, I32P,
                                      I32P, ctypes.c_int64, I64P, ctypes.c_int64, I64P, I32P, I64P],
    "RMETIS_GPU_EdgeCut": [ctypes.c_int32, I32P, I32P, I32P, I32P, I32P],
    "RMETIS_GPU_PartitionWeights": [ctypes.c_int32, ctypes.c_int32, I32P, I32P, ctypes.c_int32, I32P],
    "RMETIS_GPU_BuildCoarseGraph": [ctypes.c_int32, ctypes.c_int32, I32P, I32P, I32P, I32P, I32P, I32P, I32P,
                                    I32P, I32P, I32P, I32P],
    "RMETIS_GPU_Project": [ctypes.c_int32, I32P, ctypes.c_int32, I32P, I32P],
    "RMETIS_GPU_GainTable": [ctypes.c_int32, I32P, I32P, I32P, I32P, ctypes.c_int32, I32P, I32P, I32P, I32P, I32P],
    "RMETIS_GPU_Match": [ctypes.c_int32, I32P, I32P, I32P, ctypes.c_int, ctypes.c_uint64, ctypes.c_int, I32P],
    "RMETIS_GPU_GrowPartition": [ctypes.c_int32, ctypes.c_int32, I32P, I32P, I32P, I32P, ctypes.c_int32, F64P,
                                 ctypes.c_int32, I32P, I32P, I64P],
    "RMETIS_GPU_GreedyRefine": [ctypes.c_int32, ctypes.c_int32, I32P, I32P, I32P, I32P, I32P, ctypes.c_int32, F64P,
                                F64P, ctypes.c_int32, I32P, I64P],
    "RMETIS_GPU_FmRefine": [ctypes.c_int32, ctypes.c_int32, I32P, I32P, I32P, I32P, I32P, ctypes.c_int32, F64P,
                            F64P, ctypes.c_int32, I32P, I64P],
    "RMETIS_GPU_Fm2Refine": [ctypes.c_int32, ctypes.c_int32, I32P, I32P, I32P, I32P, I32P, F64P, F64P,
                             ctypes.c_int32, I32P, I64P],
    "RMETIS_GPU_EdgeCutWeightsNoAlloc": [ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, VP, VP, VP, VP, VP,
                                         ctypes.c_int32, VP, VP, VP],
    "RMETIS_GPU_SetFmFusedMax": [ctypes.c_int32],
    "RMETIS_GPU_SetFusedEdgeFactor": [ctypes.c_int32],
    "RMETIS_GPU_SetCoopMatching": [ctypes.c_int32],
    "RMETIS_GPU_SetBatchMode": [ctypes.c_int32, ctypes.c_int32],
    "RMETIS_GPU_PartGraphKwayBatch": [ctypes.c_int32, ctypes.c_int32, I64P, I64P, I32P, I32P, I32P, I32P, I32P,
                                      F32P, I32P, I32P, I32P, I32P],
    "RMETIS_GPU_SubmitKway": [I32P, I32P, I32P, I32P, I32P, I32P, I32P, F32P, F32P, I32P, I32P, I32P],
    "RMETIS_GPU_PollKway": [ctypes.c_int64],
    "RMETIS_GPU_WaitKway": [ctypes.c_int64],
}

# Return types other than int.
RESTYPES = {"RMETIS_GPU_SubmitKway": ctypes.c_int64}

_lib = None


def load() -> ctypes.CDLL:
    """Load the CUDA library, raising if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m rmetis_b200.build` "
                "(there is no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = RESTYPES.get(name, ctypes.c_int)
        _lib = lib
    return _lib
