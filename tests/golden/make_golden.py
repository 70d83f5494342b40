"""Generate the golden fixtures of tests/golden from the REFERENCE MKF implementation.

Run in a container that has the reference sources (default /root/reference):

    python tests/golden/make_golden.py [--ref /root/reference]

It builds oracle/_ref/libmkfref.so (the reference C path compiled from its own sources, see
oracle/Makefile) and records, for seeded inputs:

* ref_cases.npz   fields, thresholds, relation masks and the reference's pattern counts
                  (mkfAccGetBPFDSimple, one call per threshold), its packed maps, its float
                  measures (mkfSelectMeasuresBPFD) and its group map (c8sGetMap);
* ref_host.json   results of the reference's host helpers (setBMO, setBinMapF64, copyNonZeroDef,
                  genStride, copyOrGenStride, encSizeN, encAlignment, volFrac, ...);
* abi_layout.json sizes and member offsets of the ABI structs under the reference headers.

The reference CPU path double-counts rows shorter than 32 elements (mkfACC.c:137-150); cases
with X < 32 store that output under "ref_short_*" only to document the difference.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))


def sphere(n, r, amp, rng, dtype):
    c = (n - 1) / 2.0
    z, y, x = np.meshgrid(*(np.arange(n, dtype=np.float64),) * 3, indexing="ij")
    f = r - np.sqrt((x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2) + amp * (rng.random((n, n, n)) - 0.5)
    return f.astype(dtype)


def grf(shape, sigma, rng):
    w = rng.standard_normal(shape)
    k = [np.fft.fftfreq(s) * 2 * np.pi for s in shape]
    kz, ky, kx = np.meshgrid(*k, indexing="ij")
    f = np.real(np.fft.ifftn(np.fft.fftn(w) * np.exp(-0.5 * sigma * sigma * (kx ** 2 + ky ** 2 + kz ** 2))))
    return (f - f.mean()) / f.std()


def build_cases(rng):
    cases = []
    # sphere + noise, FP32, '>' 0 (the plain single-field configuration, scaled down)
    cases.append(dict(name="sphere64_f32", f=sphere(64, 24.0, 1.0, rng, np.float32), t=[0.0], m=[4]))
    # Gaussian random field, FP64, 16 thresholds in [-2, 2] (the multi-threshold configuration, scaled down)
    cases.append(dict(name="grf_f64_k16", f=grf((36, 48, 40), 2.0, rng),
                      t=np.linspace(-2, 2, 16).astype(np.float32).astype(np.float64).tolist(), m=[4] * 16))
    # uneven row lengths with every relation, on integer-valued data so equality occurs
    for shape in [(9, 17, 33), (7, 5, 65), (4, 3, 100), (2, 2, 32), (5, 6, 63), (3, 4, 64)]:
        f = rng.integers(-2, 3, size=shape).astype(np.float64)
        ms = [1, 2, 3, 4, 5, 6, 7, 0]
        cases.append(dict(name="int_%dx%dx%d" % shape[::-1], f=f, t=[0.0] * len(ms), m=ms))
    # special values: NaN, +-inf, +-0 against thresholds 0 and inf
    f = rng.standard_normal((6, 7, 40))
    flat = f.ravel()
    idx = rng.choice(flat.size, 60, replace=False)
    flat[idx[:15]] = np.nan
    flat[idx[15:30]] = np.inf
    flat[idx[30:45]] = -np.inf
    flat[idx[45:52]] = 0.0
    flat[idx[52:60]] = -0.0
    cases.append(dict(name="special_f64", f=f, t=[0.0, 0.0, 0.0, float("inf"), float("-inf")], m=[4, 2, 3, 6, 4]))
    return cases


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    args = ap.parse_args()
    subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), f"REF={args.ref}"], check=True)
    from oracle import RefOracle, layout

    ref = RefOracle()
    L = ref.L
    rng = np.random.default_rng(20261203)
    out = {}
    names = []
    for c in build_cases(rng):
        f = c["f"]
        Z, Y, X = f.shape
        d = (X, Y, Z)
        hs, maps = [], []
        for t, m in zip(c["t"], c["m"]):
            hs.append(ref.bpfd_simple(f, d, t, m))
            maps.append(ref.pack(f, d, t, m))
        key = c["name"]
        names.append(key)
        out[key + "/field"] = f
        out[key + "/t"] = np.asarray(c["t"], np.float64)
        out[key + "/m"] = np.asarray(c["m"], np.uint32)
        out[key + "/bpfd"] = np.stack(hs)
        out[key + "/pbm"] = np.stack(maps)
        sel = [ref.select_measures(h, 3.0 / (X + Y + Z)) for h in hs]
        out[key + "/sel_m"] = np.stack([s[1] for s in sel])
    # rows shorter than 32: the reference output, kept only to document the difference
    for shape in [(5, 6, 17), (3, 4, 31), (4, 4, 1)]:
        f = rng.standard_normal(shape)
        Z, Y, X = shape
        key = "short_%dx%dx%d" % (X, Y, Z)
        out[key + "/field"] = f
        out[key + "/ref_short_bpfd"] = ref.bpfd_simple(f, (X, Y, Z), 0.0, 4)
        names.append(key)
    out["c8s_map"] = ref.c8s_map()
    out["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "ref_cases.npz"), **out)

    # ---- host helpers
    host = {}
    L.setBMO.restype = C.c_size_t
    L.setBMO.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.c_char]
    rows = []
    for dd in [(256, 256, 256), (33, 17, 9), (1, 5, 7), (100, 1, 1), (31, 2, 3), (64, 64, 2)]:
        for prof in (0, 1, 3, 0x10, 0x22):
            o = (C.c_uint32 * 5)()
            n = L.setBMO(o, (C.c_int * 3)(*dd), bytes([prof]))
            rows.append(dict(def_=dd, prof=prof, ret=int(n), org=list(o)))
    host["setBMO"] = rows

    class BM(C.Structure):
        _fields_ = [("t", C.c_double), ("m", C.c_uint32)]

    L.setBinMapF64.argtypes = [C.POINTER(BM), C.c_char_p, C.c_float]
    rows = []
    for rel in ["<", "=", ">", "<=", ">=", "!=", "!<", "!>", "!", "<>", "=<>", "x>", "!=>", ">!", "", "<=>"]:
        for t in (0.0, 0.1, -2.5, 1e30):
            bm = BM()
            L.setBinMapF64(C.byref(bm), rel.encode(), t)
            rows.append(dict(rel=rel, t_in=t, t=bm.t, m=bm.m))
    host["setBinMapF64"] = rows

    L.copyNonZeroDef.argtypes = [C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int]
    rows = []
    for dd in [(1, 64, 64), (64, 1, 64), (64, 64, 1), (1, 1, 1), (0, 5, 1), (7, 8, 9), (2, 1, 3)]:
        r = (C.c_int * 3)()
        n = L.copyNonZeroDef(r, (C.c_int * 3)(*dd), 3)
        rows.append(dict(def_=dd, ret=n, out=list(r)))
    host["copyNonZeroDef"] = rows

    L.genStride.argtypes = [C.POINTER(C.c_long), C.c_int, C.c_int, C.POINTER(C.c_int), C.c_long]
    L.copyOrGenStride.argtypes = [C.POINTER(C.c_long), C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_long)]
    rows = []
    for dd in [(5, 7, 11), (32, 16, 8)]:
        for n, start, st in [(3, 0, 1), (1, 2, 1), (1, 1, 1), (2, 1, 3), (3, 0, 0)]:
            fs = (C.c_long * 3)()
            r = L.genStride(fs, n, start, (C.c_int * 3)(*dd), st)
            fs2 = (C.c_long * 3)()
            r2 = L.copyOrGenStride(fs2, n, start, (C.c_int * 3)(*dd), None)
            rows.append(dict(def_=dd, n=n, start=start, stride=st, ret=r, out=list(fs)[:max(r, 0)],
                             ret_cog=r2, out_cog=list(fs2)[:max(r2, 0)]))
    host["genStride"] = rows

    L.encSizeN.restype = C.c_size_t
    L.encSizeN.argtypes = [C.POINTER(C.c_int), C.c_size_t, C.c_uint8]
    L.encAlignment.argtypes = [C.c_uint8]
    rows = []
    for e in (0xF4, 0xF8, 0x08, 0x01, 0xE4, 0xE2):
        b = C.c_int()
        n = L.encSizeN(C.byref(b), 1000, e)
        rows.append(dict(enc=e, size=int(n), bits=b.value, align=L.encAlignment(e)))
    host["encoding"] = rows

    class CFP(C.Union):
        _fields_ = [("p", C.c_void_p)]

    L.countValidPtrByMask.argtypes = [C.POINTER(CFP), C.c_uint32]
    L.copyValidPtrByMask.argtypes = [C.POINTER(CFP), C.c_int, C.POINTER(CFP), C.c_uint32]
    tab = (CFP * 8)()
    for i, p in enumerate([0x1000, 0, 0x3000, 0x4000, 0, 0x6000, 0x7000, 0x8000]):
        tab[i].p = p or None
    rows = []
    for mask in (0x1, 0x2, 0x3, 0x5, 0xF, 0xFF, 0x12, 0x80, 0):
        for mx in (1, 2, 4):
            r = (CFP * 8)()
            n = L.copyValidPtrByMask(r, mx, tab, mask)
            rows.append(dict(mask=mask, max=mx, count=L.countValidPtrByMask(tab, mask), n=n,
                             out=[r[i].p or 0 for i in range(n)]))
    host["ptrByMask"] = dict(table=[0x1000, 0, 0x3000, 0x4000, 0, 0x6000, 0x7000, 0x8000], rows=rows)
    with open(os.path.join(HERE, "ref_host.json"), "w") as fh:
        json.dump(host, fh, indent=1)

    # ---- ABI layout under the reference headers
    with tempfile.TemporaryDirectory() as td:
        exe = os.path.join(td, "probe")
        subprocess.run(["gcc", "-std=gnu11", "-I" + os.path.join(args.ref, "src"), "-I" + os.path.join(REPO, "oracle", "shim"),
                        "-o", exe, os.path.join(HERE, "abi_probe.c")], check=True)
        lay = json.loads(subprocess.run([exe], check=True, capture_output=True, text=True).stdout)
    with open(os.path.join(HERE, "abi_layout.json"), "w") as fh:
        json.dump(lay, fh, indent=1)
    print("wrote", len(names), "cases")


if __name__ == "__main__":
    main()
