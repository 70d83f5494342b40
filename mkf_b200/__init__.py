"""MKF on B200: Minkowski functionals of thresholded 3D scalar fields.

The product is the C library ``libMKF.so`` (``mkf_b200/csrc``, sm_100a CUDA kernels behind the
C ABI declared in ``include/``). This package is its Python face: thin wrappers that pass torch
CUDA tensors (device memory) or numpy arrays (host memory) to the C entry points. Names follow
the original MKF interface (``binMapCUDA``, ``mkfCUDAGetBPFD``, ...); the B200 additions take
several thresholds per call.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import _lib
from ._lib import (BMC_AL, BMC_EQ, BMC_GT, BMC_LT, ENC_F32, ENC_F64, MKF_F_ACCUMULATE, MKF_REQ_HOST_FIELD, BinMapF64,
                   BMFieldInfo, BMOrg, ConstFieldPtr, KernInfo, MKFError, MKFFieldDesc, MKFRequest, MKFServerConfig,
                   MKFServerStats, MKFThreshSet, check, lib)

__all__ = [
    "build", "lib", "MKFError", "BatchPlan", "Server", "relation_mask", "field_bpfd", "field_bpfd_moments", "field_bpfd_host", "tune", "tuned", "set_batch_tuning", "batch_bpfd",
    "bin_map_cuda", "get_bpfd", "get_bpfd_host", "measures", "measures_dev", "select_measures",
    "ENC_F32", "ENC_F64", "BMC_LT", "BMC_EQ", "BMC_GT", "BMC_AL",
]


def build(jobs: int = 4) -> str:
    """Compile libMKF.so for sm_100a in-tree (make -C mkf_b200/csrc). Returns the library path."""
    csrc = os.path.join(_lib.PKG, "csrc")
    subprocess.run(["make", "-s", "-j", str(jobs), "-C", csrc], check=True)
    return _lib.LIB_PATH


def relation_mask(rel: str) -> int:
    """Relation string -> mask bits, as setBinMapF64 parses it ('<', '=', '>', leading '!')."""
    bm = BinMapF64()
    lib().setBinMapF64(C.byref(bm), rel.encode(), 0.0)
    return int(bm.m)


def _torch():
    import torch

    return torch


def _enc_of(t) -> int:
    torch = _torch()
    if t.dtype == torch.float32:
        return ENC_F32
    if t.dtype == torch.float64:
        return ENC_F64
    raise TypeError(f"unsupported dtype {t.dtype}")


def _field_desc(ptr: int, enc: int, shape_zyx, strides_zyx=None) -> MKFFieldDesc:
    """Descriptor of a (Z, Y, X) field; strides in elements (None = planar)."""
    d = MKFFieldDesc()
    d.p = ptr
    d.enc = enc
    z, y, x = (int(v) for v in shape_zyx)
    d.def_[0], d.def_[1], d.def_[2] = x, y, z
    if strides_zyx is not None:
        sz, sy, sx = (int(v) for v in strides_zyx)
        d.stride[0], d.stride[1], d.stride[2] = sx, sy, sz
    return d


class _Thresholds:
    """Keeps the ctypes arrays of a threshold set alive while a call uses them."""

    def __init__(self, t, m):
        t = np.atleast_1d(np.asarray(t, np.float64))
        self.t = (C.c_double * t.size)(*t.tolist())
        ts = MKFThreshSet()
        ts.nT = t.size
        if np.ndim(m) == 0:
            ts.mAll = int(m)
            ts.m = None
            self.m = None
        else:
            mm = np.broadcast_to(np.asarray(m, np.uint32), t.shape)
            self.m = (C.c_uint32 * t.size)(*mm.tolist())
            ts.m = C.cast(self.m, C.POINTER(C.c_uint32))
        ts.t = C.cast(self.t, C.POINTER(C.c_double))
        self.ts = ts
        self.n = t.size


def _stream_ptr(stream) -> int | None:
    if stream is None:
        torch = _torch()
        return torch.cuda.current_stream().cuda_stream
    return int(stream.cuda_stream) if hasattr(stream, "cuda_stream") else int(stream)


def field_bpfd(field, thresholds, mask=BMC_GT, out=None, accumulate=False, stream=None):
    """Pattern counts of a CUDA field tensor (Z, Y, X), FP32/FP64, for K thresholds in one read.

    Returns (or fills) a uint64-valued int64 CUDA tensor of shape (K, 256)."""
    torch = _torch()
    th = _Thresholds(thresholds, mask)
    if out is None:
        out = torch.zeros((th.n, 256), dtype=torch.int64, device=field.device)
    strides = None if field.is_contiguous() else field.stride()
    d = _field_desc(field.data_ptr(), _enc_of(field), field.shape, strides)
    rc = lib().mkfFieldBPFD(out.data_ptr(), C.byref(d), C.byref(th.ts),
                            MKF_F_ACCUMULATE if accumulate else 0, _stream_ptr(stream))
    check(rc, "mkfFieldBPFD")
    return out


def field_bpfd_moments(field, thresholds, mask=BMC_GT, stream=None):
    """Pattern counts of a CUDA field for one or two thresholds together with, from the same read,
    per threshold and map value the sum of f and of f^2 (FP64). Returns (counts (K, 256) int64,
    moments (K, 2, 2) float64), both CUDA tensors."""
    torch = _torch()
    th = _Thresholds(thresholds, mask)
    out = torch.zeros((th.n, 256), dtype=torch.int64, device=field.device)
    mom = torch.zeros((th.n, 2, 2), dtype=torch.float64, device=field.device)
    strides = None if field.is_contiguous() else field.stride()
    d = _field_desc(field.data_ptr(), _enc_of(field), field.shape, strides)
    check(lib().mkfFieldBPFDMoments(out.data_ptr(), mom.data_ptr(), C.byref(d), C.byref(th.ts), 0, _stream_ptr(stream)),
          "mkfFieldBPFDMoments")
    return out, mom


def tune(field, thresholds, mask=BMC_GT, stream=None, depth=None, variant=0) -> None:
    """mkfTune: time the candidate slab depths (and kernel variants) on this CUDA field and keep the
    fastest for fields of the same kind (synchronous; the counts of later calls do not change, only
    their speed). With `depth`, mkfTuneSet: record that depth and `variant` for such fields instead
    (depth 0 forgets the entry)."""
    th = _Thresholds(thresholds, mask)
    strides = None if field.is_contiguous() else field.stride()
    d = _field_desc(field.data_ptr(), _enc_of(field), field.shape, strides)
    if depth is not None:
        check(lib().mkfTuneSet(C.byref(d), C.byref(th.ts), int(depth), int(variant), _stream_ptr(stream)), "mkfTuneSet")
        return
    check(lib().mkfTune(C.byref(d), C.byref(th.ts), _stream_ptr(stream)), "mkfTune")


def tuned(field, thresholds, mask=BMC_GT, stream=None):
    """mkfTuneQuery: (depth, variant) recorded for this field's kind, (0, 0) when none is."""
    th = _Thresholds(thresholds, mask)
    strides = None if field.is_contiguous() else field.stride()
    d = _field_desc(field.data_ptr(), _enc_of(field), field.shape, strides)
    dep, var = C.c_int(), C.c_int()
    check(lib().mkfTuneQuery(C.byref(d), C.byref(th.ts), C.byref(dep), C.byref(var), _stream_ptr(stream)), "mkfTuneQuery")
    return dep.value, var.value


def set_batch_tuning(on: bool) -> bool:
    """Switch the tuning of new batch plans on or off; returns the previous setting."""
    return bool(lib().mkfSetTuning(int(bool(on))))


def field_bpfd_host(field: np.ndarray, thresholds, mask=BMC_GT) -> np.ndarray:
    """Pattern counts of a HOST (Z, Y, X) array: copied to the GPU in slabs overlapped with the
    counting kernel. Returns uint64 (K, 256)."""
    th = _Thresholds(thresholds, mask)
    if field.dtype == np.float32:
        enc = ENC_F32
    elif field.dtype == np.float64:
        enc = ENC_F64
    else:
        raise TypeError(field.dtype)
    if not field.flags["C_CONTIGUOUS"]:
        raise ValueError("host fields must be C-contiguous")
    out = np.zeros((th.n, 256), np.uint64)
    d = _field_desc(field.ctypes.data, enc, field.shape)
    rc = lib().mkfFieldBPFDHost(out.ctypes.data, C.byref(d), C.byref(th.ts))
    check(rc, "mkfFieldBPFDHost")
    return out


def batch_bpfd(fields, thresholds_list, masks=None, out=None, stream=None):
    """Pattern counts of several CUDA fields (each with its own thresholds) in one call."""
    torch = _torch()
    n = len(fields)
    masks = masks if masks is not None else [BMC_GT] * n
    ths = [_Thresholds(t, m) for t, m in zip(thresholds_list, masks)]
    total = sum(t.n for t in ths)
    if out is None:
        out = torch.zeros((total, 256), dtype=torch.int64, device=fields[0].device)
    descs = (MKFFieldDesc * n)()
    sets = (MKFThreshSet * n)()
    for i, f in enumerate(fields):
        strides = None if f.is_contiguous() else f.stride()
        descs[i] = _field_desc(f.data_ptr(), _enc_of(f), f.shape, strides)
        sets[i] = ths[i].ts
    rc = lib().mkfBatchBPFD(out.data_ptr(), descs, sets, n, 0, _stream_ptr(stream))
    check(rc, "mkfBatchBPFD")
    return out


class BatchPlan:
    """A reusable batch (mkfBatchPlanCreate): the work list stays on the device, so the same fields
    (same buffers, new contents) can be counted again with launch() or as a CUDA graph with
    launch_graph()."""

    def __init__(self, fields, thresholds_list, masks=None, out=None):
        torch = _torch()
        n = len(fields)
        masks = masks if masks is not None else [BMC_GT] * n
        self._ths = [_Thresholds(t, m) for t, m in zip(thresholds_list, masks)]
        total = sum(t.n for t in self._ths)
        self.out = out if out is not None else torch.zeros((total, 256), dtype=torch.int64, device=fields[0].device)
        self._fields = list(fields)
        descs = (MKFFieldDesc * n)()
        sets = (MKFThreshSet * n)()
        for i, f in enumerate(fields):
            strides = None if f.is_contiguous() else f.stride()
            descs[i] = _field_desc(f.data_ptr(), _enc_of(f), f.shape, strides)
            sets[i] = self._ths[i].ts
        h = C.c_void_p()
        check(lib().mkfBatchPlanCreate(C.byref(h), self.out.data_ptr(), descs, sets, n), "mkfBatchPlanCreate")
        self._h = h

    def launch(self, stream=None):
        check(lib().mkfBatchPlanLaunch(self._h, _stream_ptr(stream)), "mkfBatchPlanLaunch")
        return self.out

    def launch_graph(self, stream=None):
        check(lib().mkfBatchPlanLaunchGraph(self._h, _stream_ptr(stream)), "mkfBatchPlanLaunchGraph")
        return self.out

    def close(self):
        if self._h:
            _torch().cuda.synchronize()
            lib().mkfBatchPlanDestroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """The request loop (mkfServerCreate): submit() fields as CUDA tensors (device-resident) or
    pinned host tensors / arrays (staged by the server), wait() for their counts. Requests submitted
    while others run are admitted into the next launch as the device-memory budget allows."""

    def __init__(self, hbm_budget: int = 0, max_fields_per_launch: int = 0, device: int = 0):
        cfg = MKFServerConfig(hbm_budget, max_fields_per_launch, device)
        h = C.c_void_p()
        check(lib().mkfServerCreate(C.byref(h), C.byref(cfg)), "mkfServerCreate")
        self._h = h
        self._keep = {}  # ticket -> objects the request points to

    def submit(self, field, thresholds, mask=BMC_GT, host_out: bool = False) -> int:
        """Queue one field (CUDA tensor, or a pinned CPU tensor / numpy array viewing pinned memory).
        With host_out the counts come back as a numpy array from wait(); otherwise they stay on the
        device until release()."""
        th = _Thresholds(thresholds, mask)
        req = MKFRequest()
        if isinstance(field, np.ndarray):
            enc = ENC_F32 if field.dtype == np.float32 else ENC_F64 if field.dtype == np.float64 else None
            if enc is None or not field.flags["C_CONTIGUOUS"]:
                raise TypeError("host fields must be C-contiguous float32/float64")
            req.field = _field_desc(field.ctypes.data, enc, field.shape)
            req.flags = MKF_REQ_HOST_FIELD
        elif field.device.type == "cpu":
            if not field.is_contiguous():
                raise ValueError("host fields must be contiguous")
            req.field = _field_desc(field.data_ptr(), _enc_of(field), field.shape)
            req.flags = MKF_REQ_HOST_FIELD
        else:
            strides = None if field.is_contiguous() else field.stride()
            req.field = _field_desc(field.data_ptr(), _enc_of(field), field.shape, strides)
        req.thresh = th.ts
        out = np.zeros((th.n, 256), np.uint64) if host_out else None
        req.hostOut = out.ctypes.data if host_out else None
        tk = C.c_uint64()
        check(lib().mkfServerSubmit(self._h, C.byref(req), C.byref(tk)), "mkfServerSubmit")
        self._keep[tk.value] = (field, out, th.n)
        return tk.value

    def wait(self, ticket: int, timeout: float = 60.0):
        """Block until the ticket is done. Returns (counts, latency_s): a numpy (K, 256) uint64 array
        for host_out requests (the ticket is then released), else the device address of the counts."""
        dev = C.c_void_p()
        lat = C.c_double()
        check(lib().mkfServerWait(self._h, ticket, timeout, C.byref(dev), C.byref(lat)), "mkfServerWait")
        field, out, n = self._keep[ticket]
        if out is not None:
            self.release(ticket)
            return out, lat.value
        return dev.value, lat.value

    def counts(self, ticket: int) -> np.ndarray:
        """Host copy of a finished ticket's device-resident counts."""
        n = self._keep[ticket][2]
        out = np.zeros((n, 256), np.uint64)
        check(lib().mkfServerCopyCounts(self._h, ticket, out.ctypes.data, None), "mkfServerCopyCounts")
        return out

    def release(self, ticket: int) -> None:
        check(lib().mkfServerRelease(self._h, ticket), "mkfServerRelease")
        self._keep.pop(ticket, None)

    def stats(self, reset: bool = False) -> dict:
        st = MKFServerStats()
        check(lib().mkfServerStats(self._h, C.byref(st), int(reset)), "mkfServerStats")
        return {f: getattr(st, f) for f, _ in MKFServerStats._fields_ if f != "pad_"}

    def close(self):
        if self._h:
            lib().mkfServerDestroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bin_map_cuda(fields, rel: str, t: float, prof_id: int = 0, out=None, strides_zyx=None):
    """binMapCUDA: threshold one or more (summed) CUDA fields into a packed binary map.

    Returns (map tensor int32 on the device, BMOrg, KernInfo)."""
    torch = _torch()
    if not isinstance(fields, (list, tuple)):
        fields = [fields]
    f0 = fields[0]
    z, y, x = f0.shape
    defs = (C.c_int * 3)(x, y, z)
    table = (ConstFieldPtr * 4)()
    for i, f in enumerate(fields):
        table[i].p = f.data_ptr()
    fi = BMFieldInfo()
    fi.fieldTableMask = (1 << len(fields)) - 1
    fi.elemID = _enc_of(f0)
    fi.profID = prof_id
    fi.pD = defs
    st = None
    if strides_zyx is not None:
        st = (C.c_long * 3)(int(strides_zyx[2]), int(strides_zyx[1]), int(strides_zyx[0]))
        fi.pS = st
    fi.pFieldDevPtrTable = table
    bm = BinMapF64()
    lib().setBinMapF64(C.byref(bm), rel.encode(), float(t))
    org = BMOrg()
    cd = (C.c_int * 3)()
    lib().copyNonZeroDef(cd, (C.c_int * 3)(x, y, z), 3)
    words = max(lib().setBMO(None, (C.c_int * 3)(x, y, z), bytes([prof_id & 0xFF])),
                lib().setBMO(None, cd, bytes([prof_id & 0xFF])))
    if out is None:
        out = torch.zeros(max(int(words), 1), dtype=torch.int32, device=f0.device)
    ki = KernInfo()
    torch.cuda.synchronize()
    p = lib().binMapCUDA(C.byref(ki), out.data_ptr(), C.byref(org), C.byref(fi), C.byref(bm))
    if not p:
        raise MKFError("binMapCUDA returned NULL")
    return out, org, ki


def get_bpfd(pbm, org: BMOrg, out=None, profile: int = _lib.MKFCU_PROFILE_FAST):
    """mkfCUDAGetBPFD: add the 256 pattern counts of a device map to `out` (int64 CUDA tensor)."""
    torch = _torch()
    if out is None:
        out = torch.zeros(256, dtype=torch.int64, device=pbm.device)
    ki = KernInfo()
    torch.cuda.synchronize()
    p = lib().mkfCUDAGetBPFD(C.byref(ki), out.data_ptr(), C.byref(org), pbm.data_ptr(), profile)
    if not p:
        raise MKFError("mkfCUDAGetBPFD returned NULL")
    return out


def get_bpfd_host(pbm, org: BMOrg, profile: int = _lib.MKFCU_PROFILE_FAST) -> np.ndarray:
    """mkfCUDAGetBPFDH: pattern counts of a device map, returned in a host array."""
    out = np.zeros(256, np.uint64)
    ki = KernInfo()
    _torch().cuda.synchronize()
    p = lib().mkfCUDAGetBPFDH(C.byref(ki), out.ctypes.data, C.byref(org), pbm.data_ptr(), profile)
    if not p:
        raise MKFError("mkfCUDAGetBPFDH returned NULL")
    return out


def measures(bpfd) -> np.ndarray:
    """[V, S, M, chi] in double for each distribution of a (K, 256) host array."""
    h = np.ascontiguousarray(np.atleast_2d(np.asarray(bpfd)).astype(np.uint64))
    r = np.zeros((h.shape[0], 4), np.float64)
    check(lib().mkfMeasuresF64(r.ctypes.data, h.ctypes.data, h.shape[0]), "mkfMeasuresF64")
    return r


def measures_dev(bpfd, stream=None):
    """[V, S, M, chi] computed on the GPU from a (K, 256) CUDA tensor; returns a CUDA tensor."""
    torch = _torch()
    h = bpfd.reshape(-1, 256).contiguous()
    r = torch.empty((h.shape[0], 4), dtype=torch.float64, device=h.device)
    check(lib().mkfMeasuresF64Dev(r.data_ptr(), h.data_ptr(), h.shape[0], _stream_ptr(stream)), "mkfMeasuresF64Dev")
    return r


def select_measures(bpfd, s: float, prof_id: int = 5):
    """mkfSelectMeasuresBPFD: the original single-precision (Kv, -1, -1, Vv) selection."""
    h = np.ascontiguousarray(np.asarray(bpfd, np.uint64))
    m = (C.c_float * 4)()
    sym = C.create_string_buffer(16)
    rv = lib().mkfSelectMeasuresBPFD(m, sym, h.ctypes.data, s, prof_id)
    return rv, np.array(m[:], np.float32), sym.raw[:12]
