"""ctypes binding of libgvizcuda's C ABI (include/gvizcuda.h).

The shared library is built in-tree (grapher_b200/lib/libgvizcuda.so) by
grapher_b200.build. There is no fallback: if the library is missing or a
CUDA device is absent, calls fail with an explicit error.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libgvizcuda.so")

MODEL_FR = 0
MODEL_LINLOG = 1
FP32 = 0
FP64 = 1

ERRORS = {
    0: "ok", -1: "allocation failed", -2: "only 2-D layouts are supported",
    -3: "invalid argument", -4: "CUDA runtime error", -5: "Begin has not been called",
    -6: "a vertex position is NaN or infinite",
    -7: "more than 4096 distinct points share one depth-32 quadtree cell",
    -8: "no usable CUDA device", -9: "size beyond a supported limit",
}


class GvizCudaError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        super().__init__(f"{what}: {ERRORS.get(code, 'unknown error')} ({code})")


class ForceParams(C.Structure):
    """gvizCudaForceParams: the embedder's configuration
    (include/embedders/gvizForceEmbedder.h:52-125) plus the GPU options."""

    _fields_ = [
        ("edgeLength", C.c_double),
        ("theta", C.c_double),
        ("nodesPerCell", C.c_uint32),
        ("barnesHutEnabled", C.c_int32),
        ("gravityK", C.c_double),
        ("radiusBase", C.c_double),
        ("radiusPerDegree", C.c_double),
        ("overlapConstant", C.c_double),
        ("preventOverlap", C.c_int32),
        ("precision", C.c_int32),
        ("jitterTolerance", C.c_double),
        ("strictReductions", C.c_int32),
        ("farField", C.c_int32),
        ("farGroupSpread", C.c_double),
        ("farCellGroups", C.c_int32),
        ("farHubTargets", C.c_int32),
        ("farHubTheta", C.c_double),
    ]


class GraphDesc(C.Structure):
    _fields_ = [
        ("vertexCount", C.c_size_t),
        ("rowOffsets", C.POINTER(C.c_uint64)),
        ("neighbors", C.POINTER(C.c_uint32)),
        ("degree", C.POINTER(C.c_uint64)),
        ("graphCount", C.c_size_t),
        ("graphOffsets", C.POINTER(C.c_uint64)),
        ("model", C.c_int32),
        ("device", C.c_int32),
    ]


class Csr(C.Structure):
    _fields_ = [
        ("vertexCount", C.c_size_t),
        ("entryCount", C.c_size_t),
        ("rowOffsets", C.POINTER(C.c_uint64)),
        ("neighbors", C.POINTER(C.c_uint32)),
        ("externalIds", C.POINTER(C.c_int64)),
        ("directed", C.c_int32),
    ]


class StepStats(C.Structure):
    _fields_ = [
        ("maxDisp", C.c_double),
        ("speed", C.c_double),
        ("meanAttractive", C.c_double),
        ("meanRepulsive", C.c_double),
        ("meanGravity", C.c_double),
    ]


_lib = None

P = C.c_void_p
D = C.c_double
DP = C.POINTER(C.c_double)
U32P = C.POINTER(C.c_uint32)
U64P = C.POINTER(C.c_uint64)
I32P = C.POINTER(C.c_int32)
SZ = C.c_size_t

class GripRoundStats(C.Structure):
    _fields_ = [
        ("maxDisplacement", C.c_double),
        ("meanDisplacement", C.c_double),
        ("meanForce", C.c_double),
        ("meanHeat", C.c_double),
    ]


_SIGS = {
    "gvizCudaGripCreate": (C.c_int, [C.POINTER(P), SZ, U64P, U32P, C.c_int32]),
    "gvizCudaGripDestroy": (None, [P]),
    "gvizCudaGripSetPositions": (C.c_int, [P, DP]),
    "gvizCudaGripGetPositions": (C.c_int, [P, DP]),
    "gvizCudaGripSetLayer": (C.c_int, [P, SZ, U32P, SZ, U64P, U32P, U32P]),
    "gvizCudaGripRefineRound": (C.c_int, [P, C.POINTER(GripRoundStats)]),
    "gvizCudaGripSetStrictReductions": (C.c_int, [P, C.c_int32]),
    "gvizCudaGripGetDecorators": (C.c_int, [P, DP, DP, DP]),
    "gvizCudaGripTimeRounds": (C.c_int, [P, C.c_uint32, C.POINTER(C.c_float),
                                         C.POINTER(C.c_float)]),
    "gvizCudaGripKNearest": (C.c_int64, [SZ, U64P, U32P, U32P, SZ, C.POINTER(C.c_uint8),
                                         C.c_uint32, U64P, U32P, U32P]),
    "gvizCudaForceDefaultParams": (None, [C.POINTER(ForceParams)]),
    "gvizCudaForceCreate": (C.c_int, [C.POINTER(P), C.POINTER(GraphDesc)]),
    "gvizCudaForceDestroy": (None, [P]),
    "gvizCudaForceSetParams": (C.c_int, [P, C.POINTER(ForceParams)]),
    "gvizCudaForceGetParams": (C.c_int, [P, C.POINTER(ForceParams)]),
    "gvizCudaForceSetPositions": (C.c_int, [P, DP]),
    "gvizCudaForceGetPositions": (C.c_int, [P, DP]),
    "gvizCudaForceBegin": (C.c_int, [P]),
    "gvizCudaForceSetFa2State": (C.c_int, [P, DP, DP, DP]),
    "gvizCudaForceGetFa2State": (C.c_int, [P, DP, DP, DP]),
    "gvizCudaForceStep": (D, [P, C.POINTER(StepStats)]),
    "gvizCudaForceStepHost": (D, [P, DP, C.POINTER(StepStats)]),
    "gvizCudaForceRunHost": (D, [P, DP, C.c_uint32, C.POINTER(StepStats)]),
    "gvizCudaForceEnqueueSteps": (C.c_int, [P, C.c_uint32]),
    "gvizCudaForceSynchronize": (C.c_int, [P]),
    "gvizCudaForceRun": (C.c_int, [P, SZ, D, U64P]),
    "gvizCudaForceStatHistory": (C.c_int64, [P, C.c_uint32, DP, SZ]),
    "gvizCudaForceGetForces": (C.c_int, [P, DP, DP, DP, DP, DP, DP, DP]),
    "gvizCudaForceTreeLeaves": (C.c_int, [P, I32P, U64P, U64P, U64P]),
    "gvizCudaForceTreeNodes": (C.c_int64, [P, SZ, I32P, U64P, U64P, DP, DP, DP, U64P]),
    "gvizCudaForceExactRepulsion": (C.c_int, [P, U32P, SZ, DP]),
    "gvizCudaForceRepulsion": (C.c_int, [P, DP]),
    "gvizCudaForceCountInteractions": (C.c_int, [P, U64P, U64P]),
    "gvizCudaForceCountFarRows": (C.c_int, [P, U64P, U64P, U64P]),
    "gvizCudaForceFarGroups": (C.c_int, [P, U32P, U64P]),
    "gvizCudaForceProfileStep": (C.c_int, [P, SZ, C.POINTER(C.c_char_p), DP]),
    "gvizCudaForceTimeSteps": (C.c_int, [P, C.c_uint32, C.POINTER(C.c_float)]),
    "gvizCudaForceStepKernelCount": (C.c_int, [P]),
    "gvizCudaForceLastError": (C.c_int, [P]),
    "gvizCudaErrorString": (C.c_char_p, [C.c_int]),
    "gvizCudaForceSetStream": (C.c_int, [P, P]),
    "gvizCudaFa2SpeedUpdateNoAlloc": (C.c_int, [P, P, P, SZ, D, P, P, P]),
    "gvizCudaMlpCreate": (C.c_int, [C.POINTER(P), C.c_int, C.c_uint64]),
    "gvizCudaMlpDestroy": (None, [P]),
    "gvizCudaMlpParamCount": (C.c_int, []),
    "gvizCudaMlpSetTrainingKernels": (C.c_int, [P, C.c_int]),
    "gvizCudaMlpSetWeights": (C.c_int, [P, C.POINTER(C.c_float)]),
    "gvizCudaMlpGetWeights": (C.c_int, [P, C.POINTER(C.c_float)]),
    "gvizCudaMlpGradient": (C.c_int, [P, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                      C.POINTER(C.c_float), SZ, C.POINTER(C.c_float),
                                      C.POINTER(C.c_float)]),
    "gvizCudaMlpTrain": (C.c_int, [P, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                   C.POINTER(C.c_float), SZ, C.c_uint32, C.c_uint32,
                                   C.c_float, C.c_uint64, C.POINTER(C.c_float)]),
    "gvizCudaMlpInfer": (C.c_int, [P, C.POINTER(C.c_float), SZ, C.POINTER(C.c_float)]),
    "gvizCudaForceSetFarFieldModel": (C.c_int, [P, P]),
    "gvizCudaForceHarvestFarField": (C.c_int64, [P, U32P, SZ, D, C.POINTER(C.c_float),
                                                 C.POINTER(C.c_float), C.POINTER(C.c_float),
                                                 U32P, SZ]),
    "gvizCudaEdgesToCsr": (C.c_int, [SZ, U32P, U32P, SZ, U64P, U32P]),
    "gvizCudaForceAutotune": (C.c_int, [P, U32P, I32P, C.POINTER(C.c_float)]),
    "gvizCudaForceSetWalkShape": (C.c_int, [P, C.c_uint32, C.c_int32]),
    "gvizCudaForceGetWalkShape": (C.c_int, [P, U32P, I32P, U32P]),
    "gvizCudaForceSetWalkStackCap": (C.c_int, [P, C.c_uint32]),
    "gvizCudaForceSetFarJudge": (C.c_int, [P, C.c_uint32, C.c_uint32, D, D, C.c_uint64]),
    "gvizCudaForceJudgeFarField": (C.c_int, [P, DP, DP, I32P]),
    "gvizCudaForceFarJudgeStatus": (C.c_int, [P, U64P, DP, DP, I32P]),
    "gvizCudaForceSaveCheckpoint": (C.c_int, [P, C.c_char_p, C.c_char_p]),
    "gvizCudaForceLoadCheckpoint": (C.c_int, [P, C.c_char_p, C.c_int, C.c_char_p, SZ]),
    "gvizCudaForceSaveEmbeddingText": (C.c_int, [P, C.c_char_p, C.c_char_p]),
    "gvizCudaLoadEdgesFile": (C.c_int, [C.c_char_p, C.c_int, C.c_int, C.POINTER(Csr)]),
    "gvizCudaLoadObjFile": (C.c_int, [C.c_char_p, C.POINTER(Csr)]),
    "gvizCudaLoadGexfFile": (C.c_int, [C.c_char_p, C.POINTER(Csr)]),
    "gvizCudaCsrFree": (None, [C.POINTER(Csr)]),
    "gvizCudaRandomizePositions": (None, [DP, SZ, D, C.c_uint]),
}

# entry points present only once their features are built; bound if exported
OPTIONAL = set()


def lib() -> C.CDLL:
    """Loads libgvizcuda.so; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m grapher_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            if name in OPTIONAL and not hasattr(L, name):
                continue
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


# libgvizworkloads.so (include/gvizworkloads.h): synthetic graphs, host only
WORKLOADS_PATH = os.path.join(HERE, "lib", "libgvizworkloads.so")
_WSIGS = {
    "gvizGenGrid": (SZ, [SZ, SZ, U32P, U32P]),
    "gvizGenRandomConnected": (SZ, [SZ, D, C.c_uint, U32P, U32P]),
    "gvizGenBarabasiAlbert": (SZ, [SZ, C.c_uint32, C.c_uint64, U32P, U32P]),
    "gvizGenErdosRenyi": (SZ, [SZ, SZ, C.c_uint64, U32P, U32P]),
    "gvizGenRmat": (SZ, [C.c_uint32, SZ, D, D, D, C.c_uint64, U32P, U32P]),
}
_wlib = None


def workloads_lib() -> C.CDLL:
    """Loads libgvizworkloads.so (it does not load libgvizcuda)."""
    global _wlib
    if _wlib is None:
        if not os.path.exists(WORKLOADS_PATH):
            raise RuntimeError(
                f"{WORKLOADS_PATH} is missing: build it with `python -m grapher_b200.build`")
        L = C.CDLL(WORKLOADS_PATH)
        for name, (res, args) in _WSIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _wlib = L
    return _wlib


def check(code: int, what: str = "") -> int:
    if code < 0:
        raise GvizCudaError(int(code), what)
    return code


def ptr(a, ctype):
    """ctypes pointer to a contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))
