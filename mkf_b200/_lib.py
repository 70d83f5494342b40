"""ctypes declarations of libMKF.so (the C ABI declared in include/*.h).

The library is the product: CUDA kernels for sm_100a behind plain C entry points. This module
only declares the entry points and the ABI structs so Python (tests, bench) can call them. It
never falls back to anything else: if the library is missing it raises.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libMKF.so")

ENC_F32 = 0xF4
ENC_F64 = 0xF8
BMC_LT, BMC_EQ, BMC_GT, BMC_AL = 0x1, 0x2, 0x4, 0x7
MKF_OK = 0
MKF_F_ACCUMULATE = 0x1
MKF_MAX_THRESH = 32
MKFCU_PROFILE_FAST = 3
MKFCU_PROFILE_FLEX = 2

ERRORS = {
    -1: "MKF_ERR_ARG", -2: "MKF_ERR_CUDA", -3: "MKF_ERR_NOMEM", -4: "MKF_ERR_TIMEOUT",
    -5: "MKF_ERR_UNSUPPORTED", -6: "MKF_ERR_BUSY", -7: "MKF_ERR_NOTFOUND",
}


class BinMapF64(C.Structure):
    _fields_ = [("t", C.c_double * 1), ("m", C.c_uint32)]


class BMOrg(C.Structure):
    _fields_ = [("rowElem", C.c_uint32), ("rowPairs", C.c_uint32), ("planePairs", C.c_uint32),
                ("rowWS", C.c_uint32), ("planeWS", C.c_uint32)]


class ConstFieldPtr(C.Union):
    _fields_ = [("p", C.c_void_p), ("w", C.c_size_t)]


class BMFieldInfo(C.Structure):
    _fields_ = [("fieldTableMask", C.c_uint32), ("elemID", C.c_uint8), ("oprID", C.c_uint8),
                ("profID", C.c_uint8), ("flags", C.c_uint8), ("pD", C.POINTER(C.c_int)),
                ("pS", C.POINTER(C.c_long)), ("pFieldDevPtrTable", C.POINTER(ConstFieldPtr))]


class KernInfo(C.Structure):
    _fields_ = [("dtms", C.c_float * 2)]


class Context(C.Structure):
    _fields_ = [("nField", C.c_int), ("nElem", C.c_int), ("enc", C.c_uint8), ("bytesElem", C.c_uint8),
                ("pad", C.c_uint8 * 2), ("bytesF", C.c_long), ("nU", C.c_long), ("bytesU", C.c_long),
                ("nZ", C.c_long), ("bytesZ", C.c_long), ("pDF", C.c_void_p), ("pHF", C.c_void_p),
                ("pDU", C.c_void_p), ("pHU", C.c_void_p), ("pDZ", C.c_void_p), ("pHZ", C.c_void_p),
                ("bmo", BMOrg), ("ki", KernInfo)]


class MKFFieldDesc(C.Structure):
    _fields_ = [("p", C.c_void_p), ("enc", C.c_uint8), ("pad_", C.c_uint8 * 3),
                ("def_", C.c_int32 * 3), ("stride", C.c_int64 * 3)]


class MKFThreshSet(C.Structure):
    _fields_ = [("nT", C.c_int32), ("mAll", C.c_uint32), ("t", C.POINTER(C.c_double)),
                ("m", C.POINTER(C.c_uint32))]


# (name, restype, argtypes) of every exported C entry point
_P = C.c_void_p
MKF_REQ_HOST_FIELD = 0x1


class MKFServerConfig(C.Structure):
    _fields_ = [("hbmBudget", C.c_uint64), ("maxFieldsPerLaunch", C.c_int32), ("device", C.c_int32)]


class MKFRequest(C.Structure):
    _fields_ = [("field", MKFFieldDesc), ("thresh", MKFThreshSet), ("flags", C.c_uint32), ("pad_", C.c_uint32),
                ("hostOut", C.c_void_p)]


class MKFServerStats(C.Structure):
    _fields_ = [("completed", C.c_uint64), ("failed", C.c_uint64), ("launches", C.c_uint64),
                ("maxFieldsInLaunch", C.c_uint32), ("pad_", C.c_uint32), ("meanFieldsInLaunch", C.c_double),
                ("p50", C.c_double), ("p99", C.c_double), ("mean", C.c_double), ("max", C.c_double),
                ("deviceBytesInUse", C.c_uint64), ("launchDeviceSec", C.c_double), ("planHostSec", C.c_double)]


_SIG = [
    ("binMapCUDA", _P, [C.POINTER(KernInfo), _P, C.POINTER(BMOrg), C.POINTER(BMFieldInfo), C.POINTER(BinMapF64)]),
    ("binMapCUDACleanup", None, []),
    ("mkfCUDAGetBPFD", _P, [C.POINTER(KernInfo), _P, C.POINTER(BMOrg), _P, C.c_int]),
    ("mkfCUDAGetBPFDH", _P, [C.POINTER(KernInfo), _P, C.POINTER(BMOrg), _P, C.c_int]),
    ("mkfCUDAGetBPFDautoCtx", C.c_int, [C.POINTER(Context), C.POINTER(C.c_int), C.POINTER(BinMapF64), C.c_int]),
    ("mkfCUDACleanup", None, [C.c_int]),
    ("setBinMapF64", C.POINTER(BinMapF64), [C.POINTER(BinMapF64), C.c_char_p, C.c_float]),
    ("setBMO", C.c_size_t, [C.POINTER(BMOrg), C.POINTER(C.c_int), C.c_char]),
    ("copyNonZeroDef", C.c_int, [C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int]),
    ("copyValidPtrByMask", C.c_int, [C.POINTER(ConstFieldPtr), C.c_int, C.POINTER(ConstFieldPtr), C.c_uint32]),
    ("countValidPtrByMask", C.c_int, [C.POINTER(ConstFieldPtr), C.c_uint32]),
    ("genStride", C.c_int, [C.POINTER(C.c_long), C.c_int, C.c_int, C.POINTER(C.c_int), C.c_long]),
    ("copyOrGenStride", C.c_int, [C.POINTER(C.c_long), C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_long)]),
    ("asFieldTab", C.POINTER(ConstFieldPtr), [C.POINTER(C.c_void_p), C.c_uint8]),
    ("setupFields", C.POINTER(BMFieldInfo), [C.POINTER(BMFieldInfo), C.POINTER(C.c_void_p), C.c_int,
                                             C.POINTER(C.c_int), C.c_int, C.c_int]),
    ("autoFieldPtr", C.POINTER(C.c_void_p), [C.POINTER(ConstFieldPtr), C.POINTER(Context)]),
    ("encSizeN", C.c_size_t, [C.POINTER(C.c_int), C.c_size_t, C.c_uint8]),
    ("encAlignment", C.c_int, [C.c_uint8]),
    ("c8sGetMap", C.c_int, [C.POINTER(C.c_uint8)]),
    ("volFrac", C.c_float, [_P]),
    ("mkfRefMeasureBPFD", None, [C.POINTER(C.c_float), _P, C.c_float]),
    ("mkfSelectMeasuresBPFD", C.c_int, [C.POINTER(C.c_float), C.c_char_p, _P, C.c_float, C.c_int]),
    ("ctuInfo", C.c_int, []),
    ("cuBuffAlloc", C.c_int, [C.POINTER(Context), C.c_uint]),
    ("cuBuffRelease", C.c_int, [C.POINTER(Context)]),
    ("sumNZ", C.c_size_t, [_P, C.c_size_t]),
    ("prodNI", C.c_int, [C.POINTER(C.c_int), C.c_int]),
    ("sumNI", C.c_int, [C.POINTER(C.c_int), C.c_int]),
    ("mkfLastError", C.c_char_p, []),
    ("mkfFieldBPFD", C.c_int, [_P, C.POINTER(MKFFieldDesc), C.POINTER(MKFThreshSet), C.c_int, _P]),
    ("mkfFieldBPFDMoments", C.c_int, [_P, _P, C.POINTER(MKFFieldDesc), C.POINTER(MKFThreshSet), C.c_int, _P]),
    ("mkfFieldBPFDHost", C.c_int, [_P, C.POINTER(MKFFieldDesc), C.POINTER(MKFThreshSet)]),
    ("mkfFieldBPFDHostNoAlloc", C.c_int, [_P, C.POINTER(MKFFieldDesc), C.POINTER(MKFThreshSet), _P]),
    ("mkfBatchPlanCreate", C.c_int, [C.POINTER(C.c_void_p), _P, C.POINTER(MKFFieldDesc), C.POINTER(MKFThreshSet), C.c_int]),
    ("mkfBatchPlanLaunch", C.c_int, [_P, _P]),
    ("mkfBatchPlanLaunchGraph", C.c_int, [_P, _P]),
    ("mkfBatchPlanDestroy", C.c_int, [_P]),
    ("mkfBatchBPFD", C.c_int, [_P, C.POINTER(MKFFieldDesc), C.POINTER(MKFThreshSet), C.c_int, C.c_int, _P]),
    ("mkfTune", C.c_int, [C.POINTER(MKFFieldDesc), C.POINTER(MKFThreshSet), _P]),
    ("mkfSetTuning", C.c_int, [C.c_int]),
    ("mkfKernelFaults", C.c_int, [C.c_int]),
    ("mkfTuneSet", C.c_int, [C.POINTER(MKFFieldDesc), C.POINTER(MKFThreshSet), C.c_int, C.c_int, _P]),
    ("mkfTuneQuery", C.c_int, [C.POINTER(MKFFieldDesc), C.POINTER(MKFThreshSet), C.POINTER(C.c_int), C.POINTER(C.c_int), _P]),
    ("mkfServerCreate", C.c_int, [C.POINTER(C.c_void_p), C.POINTER(MKFServerConfig)]),
    ("mkfServerSubmit", C.c_int, [_P, C.POINTER(MKFRequest), C.POINTER(C.c_uint64)]),
    ("mkfServerWait", C.c_int, [_P, C.c_uint64, C.c_double, C.POINTER(C.c_void_p), C.POINTER(C.c_double)]),
    ("mkfServerCopyCounts", C.c_int, [_P, C.c_uint64, _P, _P]),
    ("mkfServerRelease", C.c_int, [_P, C.c_uint64]),
    ("mkfServerStats", C.c_int, [_P, C.POINTER(MKFServerStats), C.c_int]),
    ("mkfServerDestroy", C.c_int, [_P]),
    ("mkfMeasuresF64", C.c_int, [_P, _P, C.c_int]),
    ("mkfMeasuresF64Dev", C.c_int, [_P, _P, C.c_int, _P]),
]

_lib = None


class MKFError(RuntimeError):
    pass


def lib() -> C.CDLL:
    """The loaded libMKF.so. Raises if it has not been built: there is no other implementation."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise MKFError(f"libMKF.so not found at {LIB_PATH}; build it with __graft_entry__.build() "
                           "(make -C mkf_b200/csrc)")
        L = C.CDLL(LIB_PATH)
        for name, res, args in _SIG:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int, what: str) -> None:
    if rc != MKF_OK:
        msg = lib().mkfLastError()
        raise MKFError(f"{what} failed: {ERRORS.get(rc, rc)}: {msg.decode() if msg else ''}")


def exported_symbols():
    return [name for name, _, _ in _SIG] + ["ctuErr"]
