"""ctypes access to the CPU oracles. TEST INFRASTRUCTURE ONLY.

Only the tests, ``__graft_entry__.smoke()``, and the CPU-baseline leg and the reference arm
(``--impl reference``) of ``bench.py`` may import this module; the product library never does.

* :class:`Oracle` wraps ``liboracle.so``, the project's CPU restatement of the MKF path
  (``mkf_oracle.c``).
* :class:`RefOracle` wraps ``_ref/libmkfref.so``, the reference MKF C path compiled from its own
  sources (``Makefile``). It exists only where it was built.
* :class:`RefCuda` wraps ``_ref/libmkfrefcuda.so``, the reference MKF CUDA path
  (``binMapCUDA`` + ``mkfCUDAGetBPFD``) compiled unmodified for sm_100a: a GPU cross-check and
  the recompiled-reference timing point. It exists only where it was built.
* :func:`bpfd_numpy` is a third, vectorised formulation used to cross-check the other two.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ENC_F32 = 0xF4
ENC_F64 = 0xF8
BMC_LT, BMC_EQ, BMC_GT = 1, 2, 4

_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build() -> None:
    """Build the oracle libraries with oracle/Makefile (the reference part only where its
    sources exist)."""
    import subprocess

    subprocess.run(["make", "-s", "-C", HERE], check=True)


def layout(def3):
    """(rowWS, planeWS) of the full packed map, setBMO profID 0 (binMapUtil.c:60-87)."""
    row = (int(def3[0]) + 31) >> 5
    return row, row * int(def3[1])


def _def(def3):
    return (C.c_int * 3)(*[int(v) for v in def3])


def _stride(stride):
    if stride is None:
        return None
    return (C.c_long * 3)(*[int(v) for v in stride])


def _enc(a: np.ndarray) -> int:
    if a.dtype == np.float32:
        return ENC_F32
    if a.dtype == np.float64:
        return ENC_F64
    raise TypeError(a.dtype)


class Oracle:
    """The project's CPU restatement (mkf_oracle.c)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_map_value.restype = C.c_uint
        L.orc_map_value.argtypes = [C.c_double, C.c_double, C.c_uint]
        L.orc_pack.restype = None
        L.orc_pack.argtypes = [_u32p, C.POINTER(C.c_void_p), C.c_int, C.c_int, C.POINTER(C.c_int),
                               C.POINTER(C.c_long), C.c_double, C.c_uint, C.c_uint32, C.c_uint32]
        L.orc_bpfd_pbm.restype = None
        L.orc_bpfd_pbm.argtypes = [_u64p, _u32p, C.c_int, C.c_int, C.c_int, C.c_uint32, C.c_uint32]
        L.orc_bpfd_field.restype = None
        L.orc_bpfd_field.argtypes = [_u64p, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_long),
                                     C.c_int, _f64p, _u32p]
        L.orc_group_map.argtypes = [np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")]
        L.orc_weights.argtypes = [np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS"), _f64p, _f64p]
        L.orc_group_counts.argtypes = [_u64p, _u64p]
        L.orc_measures.argtypes = [_f64p, _u64p]
        L.orc_select_measures.restype = C.c_int
        L.orc_select_measures.argtypes = [np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS"),
                                          C.c_char_p, _u64p, C.c_float]
        self.L = L

    def map_value(self, f: float, t: float, m: int) -> int:
        return int(self.L.orc_map_value(f, t, m))

    def pack(self, fields, def3, t: float, m: int, stride=None) -> np.ndarray:
        """Packed map (uint32[Z*planeWS]) of the element-wise sum of `fields` (same dtype)."""
        if isinstance(fields, np.ndarray):
            fields = [fields]
        enc = _enc(fields[0])
        row, plane = layout(def3)
        out = np.zeros(plane * int(def3[2]), np.uint32)
        ptrs = (C.c_void_p * len(fields))(*[f.ctypes.data for f in fields])
        self.L.orc_pack(out, ptrs, len(fields), enc, _def(def3), _stride(stride), float(t), int(m), row, plane)
        return out

    def bpfd_pbm(self, pbm: np.ndarray, def3, rowWS=None, planeWS=None) -> np.ndarray:
        r, p = layout(def3)
        h = np.zeros(256, np.uint64)
        self.L.orc_bpfd_pbm(h, np.ascontiguousarray(pbm, np.uint32), int(def3[0]), int(def3[1]), int(def3[2]),
                            rowWS or r, planeWS or p)
        return h

    def bpfd_field(self, f: np.ndarray, def3, t, m, stride=None) -> np.ndarray:
        """uint64[K,256] pattern counts of field f for thresholds t (compared exactly in double)."""
        t = np.atleast_1d(np.asarray(t, np.float64)).copy()
        m = np.broadcast_to(np.asarray(m, np.uint32), t.shape).copy()
        h = np.zeros((t.size, 256), np.uint64)
        self.L.orc_bpfd_field(h, f.ctypes.data, _enc(f), _def(def3), _stride(stride), t.size, t, m)
        return h

    def group_map(self) -> np.ndarray:
        g = np.zeros(256, np.uint8)
        self.L.orc_group_map(g)
        return g

    def weights(self):
        wk = np.zeros(22, np.int32)
        ws = np.zeros(22, np.float64)
        wm = np.zeros(22, np.float64)
        self.L.orc_weights(wk, ws, wm)
        return wk, ws, wm

    def measures(self, h: np.ndarray) -> np.ndarray:
        """[V, S, M, chi] in double for one uint64[256] distribution."""
        r = np.zeros(4, np.float64)
        self.L.orc_measures(r, np.ascontiguousarray(h, np.uint64))
        return r

    def select_measures(self, h: np.ndarray, s: float):
        m = np.zeros(4, np.float32)
        sym = C.create_string_buffer(16)
        rv = self.L.orc_select_measures(m, sym, np.ascontiguousarray(h, np.uint64), s)
        return rv, m, sym.raw[:12]


class RefOracle:
    """The reference MKF C path (compiled from the reference's sources by oracle/Makefile)."""

    PATH = os.path.join(HERE, "_ref", "libmkfref.so")

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls.PATH)

    def __init__(self):
        L = C.CDLL(self.PATH)
        L.refh_bpfd_simple.restype = C.c_int
        L.refh_bpfd_simple.argtypes = [_u64p, _f64p, C.POINTER(C.c_int), C.c_double, C.c_uint]
        L.refh_pack.restype = None
        L.refh_pack.argtypes = [_u32p, _f64p, C.POINTER(C.c_int), C.c_double, C.c_uint]
        L.refh_bpfd_pbm.restype = None
        L.refh_bpfd_pbm.argtypes = [_u64p, _u32p, C.POINTER(C.c_int)]
        L.refh_bpfd_mt.restype = C.c_int
        L.refh_bpfd_mt.argtypes = [_u64p, C.c_void_p, C.POINTER(C.c_int), C.c_double, C.c_uint, C.c_int]
        L.c8sGetMap.restype = C.c_int
        L.c8sGetMap.argtypes = [np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")]
        L.mkfSelectMeasuresBPFD.restype = C.c_int
        L.mkfSelectMeasuresBPFD.argtypes = [np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS"),
                                            C.c_char_p, _u64p, C.c_float, C.c_int]
        L.volFrac.restype = C.c_float
        L.volFrac.argtypes = [_u64p]
        self.L = L

    @staticmethod
    def padded(f: np.ndarray) -> np.ndarray:
        """FP64 copy with 64 elements of slack: the reference CPU map reads up to 31 elements past
        each row when X % 32 != 0 (binMapACC.c:86-90)."""
        flat = np.zeros(f.size + 64, np.float64)
        flat[: f.size] = np.asarray(f, np.float64).ravel()
        return flat

    def bpfd_simple(self, f: np.ndarray, def3, t: float, m: int) -> np.ndarray:
        h = np.zeros(256, np.uint64)
        ok = self.L.refh_bpfd_simple(h, self.padded(f), _def(def3), float(t), int(m))
        assert ok
        return h

    def pack(self, f: np.ndarray, def3, t: float, m: int) -> np.ndarray:
        row, plane = layout(def3)
        out = np.zeros(plane * int(def3[2]) + 1, np.uint32)
        self.L.refh_pack(out, self.padded(f), _def(def3), float(t), int(m))
        return out[:-1]

    def bpfd_pbm(self, pbm: np.ndarray, def3) -> np.ndarray:
        h = np.zeros(256, np.uint64)
        self.L.refh_bpfd_pbm(h, np.ascontiguousarray(pbm, np.uint32), _def(def3))
        return h

    def bpfd_mt(self, f_padded: np.ndarray, def3, t: float, m: int, threads: int) -> np.ndarray:
        """Multi-threaded reference path; f_padded must be FP64 with >= 32 elements of slack."""
        h = np.zeros(256, np.uint64)
        ok = self.L.refh_bpfd_mt(h, f_padded.ctypes.data, _def(def3), float(t), int(m), int(threads))
        assert ok
        return h

    def c8s_map(self) -> np.ndarray:
        g = np.zeros(256, np.uint8)
        n = self.L.c8sGetMap(g)
        assert n == 22
        return g

    def select_measures(self, h: np.ndarray, s: float, pid: int = 5):
        m = np.zeros(4, np.float32)
        sym = C.create_string_buffer(16)
        rv = self.L.mkfSelectMeasuresBPFD(m, sym, np.ascontiguousarray(h, np.uint64), s, pid)
        return rv, m, sym.raw[:12]


class RefCuda:
    """The reference MKF CUDA path, compiled unmodified from its .cu/.c sources for sm_100a
    (oracle/Makefile, ref_cuda_harness.cu). All pointers are device addresses (ints)."""

    PATH = os.path.join(HERE, "_ref", "libmkfrefcuda.so")

    @classmethod
    def available(cls) -> bool:
        return os.path.exists(cls.PATH)

    def __init__(self):
        L = C.CDLL(self.PATH)
        L.refcu_pbm_words.restype = C.c_size_t
        L.refcu_pbm_words.argtypes = [C.POINTER(C.c_int)]
        L.refcu_bpfd.restype = C.c_int
        L.refcu_bpfd.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                 np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS"), C.c_int, C.c_char_p,
                                 C.POINTER(C.c_float), C.POINTER(C.c_float)]
        self.L = L

    def pbm_words(self, def3) -> int:
        """Words of the packed map binMapCUDA writes for def3 (setBMO, binMapUtil.c:60-87)."""
        return int(self.L.refcu_pbm_words(_def(def3)))

    def bpfd(self, counts_ptr: int, pbm_ptr: int, field_ptr: int, elem_bytes: int, def3, thresholds,
             rel: str = ">"):
        """One binMapCUDA + mkfCUDAGetBPFD call pair per threshold into counts_ptr + 256 k (u64,
        zeroed by the caller). Thresholds pass through the reference's float parameter. Returns
        the reference's own summed stage timings (map ms, BPFD ms)."""
        t = np.ascontiguousarray(np.asarray(thresholds, np.float64).ravel())
        ms_map, ms_bpfd = C.c_float(0), C.c_float(0)
        ok = self.L.refcu_bpfd(C.c_void_p(counts_ptr), C.c_void_p(pbm_ptr), C.c_void_p(field_ptr),
                               int(elem_bytes), _def(def3), t, int(t.size), rel.encode(),
                               C.byref(ms_map), C.byref(ms_bpfd))
        if not ok:
            raise RuntimeError("reference CUDA path rejected the input or failed")
        return ms_map.value, ms_bpfd.value

    def bpfd_torch(self, field, thresholds, rel: str = ">"):
        """Counts u64[K][256] (as a host numpy array) of a contiguous (Z, Y, X) FP32/FP64 CUDA
        tensor by the reference CUDA path; X must be a multiple of 32."""
        import torch

        Z, Y, X = field.shape
        d = (X, Y, Z)
        pbm = torch.empty(self.pbm_words(d), dtype=torch.int32, device=field.device)
        k = int(np.asarray(thresholds).size)
        counts = torch.zeros((k, 256), dtype=torch.int64, device=field.device)
        self.bpfd(counts.data_ptr(), pbm.data_ptr(), field.data_ptr(), field.element_size(), d, thresholds, rel)
        torch.cuda.synchronize(field.device)
        return counts.cpu().numpy().view(np.uint64)


def bits_numpy(f: np.ndarray, t: float, m: int) -> np.ndarray:
    """Map of every element, vectorised: bit (m >> (1 - (f<t) + (f>t))) & 1, compared in double."""
    v = np.asarray(f, np.float64)
    rel = 1 - (v < t).astype(np.int64) + (v > t).astype(np.int64)
    return ((int(m) >> rel) & 1).astype(np.uint8)


def bpfd_numpy(f: np.ndarray, t: float, m: int) -> np.ndarray:
    """uint64[256] pattern counts of a (Z,Y,X) field by array slicing: an independent
    formulation of the 2x2x2 cell code (bit i = corner (i&1, (i>>1)&1, (i>>2)&1) in (x,y,z))."""
    b = bits_numpy(f, t, m)
    Z, Y, X = b.shape
    if min(X, Y, Z) < 2:
        return np.zeros(256, np.uint64)
    c = np.zeros((Z - 1, Y - 1, X - 1), np.uint16)
    for i in range(8):
        dx, dy, dz = i & 1, (i >> 1) & 1, (i >> 2) & 1
        c |= b[dz:Z - 1 + dz, dy:Y - 1 + dy, dx:X - 1 + dx].astype(np.uint16) << i
    return np.bincount(c.ravel(), minlength=256).astype(np.uint64)
