"""mkfFieldBPFDHostNoAlloc: the host-field entry point for callers that cannot let a library
allocate device memory (for example an analysis running inside a simulation that owns all device
memory through its own pool). Its scratch is a fixed 32 MiB staging area and 32 x 256 counts in
the library's own device arrays.

Checked through the C ABI against the allocating entry point mkfFieldBPFDHost, exactly (the
counts are integers), on two calls in a row, since every call reuses the same scratch. This file
is collected last so that a run stopping at its first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(mkf, fn, field, t, m):
    L = mkf.lib()
    th = mkf._Thresholds(t, m)
    enc = mkf.ENC_F32 if field.dtype == np.float32 else mkf.ENC_F64
    d = mkf._field_desc(field.ctypes.data, enc, field.shape)
    out = np.zeros((th.n, 256), np.uint64)
    if fn == "noalloc":
        rc = L.mkfFieldBPFDHostNoAlloc(out.ctypes.data, C.byref(d), C.byref(th.ts), None)
    else:
        rc = L.mkfFieldBPFDHost(out.ctypes.data, C.byref(d), C.byref(th.ts))
    return rc, out


def test_no_alloc_matches_allocating_entry_point(mkf, cuda):
    rng = np.random.default_rng(41)
    # 8 MiB planes: the 32 MiB staging area takes 3 plane pairs per slab, so 19 pairs need 7 slabs
    f64 = rng.standard_normal((20, 1024, 1024))
    t16 = np.linspace(-2.0, 2.0, 16)
    rc, want = _call(mkf, "host", f64, t16, mkf.BMC_GT)
    assert rc == 0
    assert (want.sum(axis=1) == 19 * 1023 * 1023).all()
    for _ in range(2):
        rc, got = _call(mkf, "noalloc", f64, t16, mkf.BMC_GT)
        assert rc == 0, mkf.lib().mkfLastError()
        assert (got == want).all()
    # FP32 field, mixed relations (general path) and constant maps, uneven row length
    f32 = (rng.standard_normal((33, 70, 45)) * 2).astype(np.float32)
    t = [0.5, -1.0, 0.0, 1.5, float("nan"), 0.25]
    m = [mkf.BMC_GT, mkf.BMC_LT | mkf.BMC_EQ, mkf.BMC_EQ, mkf.BMC_AL, mkf.BMC_EQ, mkf.BMC_GT | mkf.BMC_LT]
    rc, want = _call(mkf, "host", f32, t, m)
    assert rc == 0
    for _ in range(2):
        rc, got = _call(mkf, "noalloc", f32, t, m)
        assert rc == 0, mkf.lib().mkfLastError()
        assert (got == want).all()


_CASES = {
    # FP32, 8 thresholds of '<=' (rank table, rank counts thresholds below or at the value)
    "f32_le_k8": ((40, 60, 90), np.float32, list(np.linspace(-1.5, 1.5, 8)), 3),
    # one and two thresholds of '>=' (the word-parallel kernel, as in mkfFieldBPFD)
    "f32_ge_k1": ((50, 64, 100), np.float32, [0.1], 6),
    "f64_ge_k2": ((30, 40, 70), np.float64, [-0.4, 0.3], 6),
    # FP64, 16 thresholds of '<' (rank table, complemented codes)
    "f64_lt_k16": ((25, 33, 47), np.float64, list(np.linspace(-2, 2, 16)), 1),
    # a field smaller than one work item, and one of a single plane (no cells)
    "f64_small": ((3, 7, 5), np.float64, [-0.5, 0.0, 0.5], 4),
    "f32_one_plane": ((1, 30, 40), np.float32, [0.0, 0.2, 0.4], 4),
    # every threshold a constant map: nothing is copied
    "f32_constant": ((6, 9, 11), np.float32, [0.0, float("nan"), 1.0], [7, 2, 0]),
}


@pytest.mark.parametrize("case", sorted(_CASES))
def test_no_alloc_matches_allocating_entry_point_per_kernel(mkf, cuda, case):
    """Each kernel route of the no-allocation path (word kernel, rank table for every relation,
    tiny fields, constant maps) equals mkfFieldBPFDHost exactly, twice in a row."""
    shape, dtype, t, m = _CASES[case]
    rng = np.random.default_rng(sum(case.encode()))
    f = rng.standard_normal(shape).astype(dtype)
    rc, want = _call(mkf, "host", f, t, m)
    assert rc == 0, mkf.lib().mkfLastError()
    for _ in range(2):
        rc, got = _call(mkf, "noalloc", f, t, m)
        assert rc == 0, mkf.lib().mkfLastError()
        assert (got == want).all(), case


def test_no_alloc_rejects_planes_beyond_the_staging_area(mkf, cuda):
    # 2048 x 2048 FP64 planes are 32 MiB: two of them do not fit the 32 MiB staging area. The
    # check happens before any device work, so a descriptor of the right size is enough.
    big = np.zeros(8, np.float64)
    th = mkf._Thresholds([0.0], mkf.BMC_GT)
    d = mkf._field_desc(big.ctypes.data, mkf.ENC_F64, (3, 2048, 2048))
    out = np.zeros((1, 256), np.uint64)
    rc = mkf.lib().mkfFieldBPFDHostNoAlloc(out.ctypes.data, C.byref(d), C.byref(th.ts), None)
    assert rc == -3
    assert b"staging area" in mkf.lib().mkfLastError()
