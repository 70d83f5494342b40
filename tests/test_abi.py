"""The C ABI of libMKF.so: symbols, struct layout and host-side helpers, checked against the
reference (golden values recorded from the reference build). CPU only: nothing here launches a
kernel or touches a GPU."""
import ctypes as C
import json
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, REPO

INCLUDE = os.path.join(REPO, "include")


def header_functions():
    """Names of the functions declared in include/*.h."""
    names = set()
    decl = re.compile(r"^\s*(?:extern\s+)?(?:const\s+)?[A-Za-z_][\w\s\*]*?[\s\*]([A-Za-z_]\w*)\s*\(")
    for fn in os.listdir(INCLUDE):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(INCLUDE, fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//[^\n]*", "", src)
        for line in src.splitlines():
            if line.lstrip().startswith("#") or "typedef" in line:
                continue
            m = decl.match(line)
            if m and m.group(1) not in ("if", "while", "for", "return", "sizeof"):
                names.add(m.group(1))
    return names


def exported(lib_path):
    out = subprocess.run(["nm", "-D", "--defined-only", lib_path], check=True, capture_output=True, text=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if " T " in ln}


def test_library_exports_every_declared_function(mkf):
    from mkf_b200 import _lib

    declared = header_functions()
    assert {"binMapCUDA", "mkfCUDAGetBPFD", "mkfCUDAGetBPFDH", "mkfFieldBPFD", "setBMO"} <= declared
    syms = exported(_lib.LIB_PATH)
    missing = {n for n in declared if n != "ctuErr" and n not in syms}
    assert not missing, missing
    assert "_Z6ctuErrP9cudaErrorPKc" in syms  # C++ linkage, as the original declares it
    for name in _lib.exported_symbols():
        if name != "ctuErr":
            assert name in syms, name


def test_struct_layout_matches_reference(tmp_path):
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=gnu11", "-I" + INCLUDE, "-o", str(exe), os.path.join(GOLDEN, "abi_probe.c")], check=True)
    ours = json.loads(subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout)
    ref = json.load(open(os.path.join(GOLDEN, "abi_layout.json")))
    assert ours == ref


def test_ctypes_mirror_layout():
    from mkf_b200 import _lib

    ref = json.load(open(os.path.join(GOLDEN, "abi_layout.json")))
    for name, cls in [("BinMapF64", _lib.BinMapF64), ("BMOrg", _lib.BMOrg), ("BMFieldInfo", _lib.BMFieldInfo),
                      ("KernInfo", _lib.KernInfo), ("Context", _lib.Context)]:
        assert C.sizeof(cls) == ref[name]["size"], name
        for f, off in ref[name].items():
            if f != "size":
                assert getattr(cls, f).offset == off, (name, f)


@pytest.fixture(scope="module")
def host_golden():
    return json.load(open(os.path.join(GOLDEN, "ref_host.json")))


def test_setBMO(mkf, host_golden):
    L = mkf.lib()
    for row in host_golden["setBMO"]:
        o = mkf.BMOrg()
        n = L.setBMO(C.byref(o), (C.c_int * 3)(*row["def_"]), bytes([row["prof"]]))
        assert n == row["ret"]
        assert [o.rowElem, o.rowPairs, o.planePairs, o.rowWS, o.planeWS] == row["org"], row


def test_setBinMapF64(mkf, host_golden):
    L = mkf.lib()
    for row in host_golden["setBinMapF64"]:
        bm = mkf.BinMapF64()
        L.setBinMapF64(C.byref(bm), row["rel"].encode(), row["t_in"])
        assert bm.m == row["m"], row
        assert bm.t[0] == row["t"], row


def test_copyNonZeroDef(mkf, host_golden):
    L = mkf.lib()
    for row in host_golden["copyNonZeroDef"]:
        r = (C.c_int * 3)()
        n = L.copyNonZeroDef(r, (C.c_int * 3)(*row["def_"]), 3)
        assert n == row["ret"] and list(r) == row["out"], row


def test_genStride(mkf, host_golden):
    L = mkf.lib()
    for row in host_golden["genStride"]:
        fs = (C.c_long * 3)()
        r = L.genStride(fs, row["n"], row["start"], (C.c_int * 3)(*row["def_"]), row["stride"])
        assert r == row["ret"] and list(fs)[:max(r, 0)] == row["out"], row
        fs2 = (C.c_long * 3)()
        r2 = L.copyOrGenStride(fs2, row["n"], row["start"], (C.c_int * 3)(*row["def_"]), None)
        assert r2 == row["ret_cog"] and list(fs2)[:max(r2, 0)] == row["out_cog"], row


def test_encoding(mkf, host_golden):
    L = mkf.lib()
    for row in host_golden["encoding"]:
        b = C.c_int()
        assert L.encSizeN(C.byref(b), 1000, row["enc"]) == row["size"]
        assert b.value == row["bits"]
        assert L.encAlignment(row["enc"]) == row["align"]


def test_pointer_table_helpers(mkf, host_golden):
    L = mkf.lib()
    g = host_golden["ptrByMask"]
    tab = (mkf.ConstFieldPtr * 8)()
    for i, p in enumerate(g["table"]):
        tab[i].p = p or None
    for row in g["rows"]:
        assert L.countValidPtrByMask(tab, row["mask"]) == row["count"], row
        r = (mkf.ConstFieldPtr * 8)()
        n = L.copyValidPtrByMask(r, row["max"], tab, row["mask"])
        assert n == row["n"] and [r[i].p or 0 for i in range(n)] == row["out"], row


def test_group_map_and_float_measures(mkf, golden):
    L = mkf.lib()
    g = (C.c_uint8 * 256)()
    assert L.c8sGetMap(g) == 22
    assert bytes(g) == golden["c8s_map"].tobytes()
    for key in [str(n) for n in golden["names"] if not str(n).startswith("short_")]:
        f = golden[key + "/field"]
        Z, Y, X = f.shape
        for k, h in enumerate(golden[key + "/bpfd"]):
            rv, m, sym = mkf.select_measures(h, 3.0 / (X + Y + Z))
            assert rv == 2 and sym == b"Kv       Vv\x00"
            assert m.tobytes() == golden[key + "/sel_m"][k].tobytes(), key
            hh = np.ascontiguousarray(h, np.uint64)
            vf = L.volFrac(hh.ctypes.data)
            assert np.float32(vf) == golden[key + "/sel_m"][k][3]
    m = (C.c_float * 4)()
    L.mkfRefMeasureBPFD(m, golden["sphere64_f32/bpfd"][0].ctypes.data, 1.0)
    assert list(m) == [-1, -1, -1, -1]


def test_f64_measures_equal_oracle(mkf, oracle, golden):
    for key in [str(n) for n in golden["names"] if not str(n).startswith("short_")]:
        hs = golden[key + "/bpfd"]
        r = mkf.measures(hs)
        for k in range(hs.shape[0]):
            assert (r[k] == oracle.measures(hs[k])).all(), key


def test_argument_errors_need_no_gpu(mkf):
    L = mkf.lib()
    d = mkf.MKFFieldDesc()
    ts = mkf.MKFThreshSet()
    assert L.mkfFieldBPFD(None, C.byref(d), C.byref(ts), 0, None) == -1
    d.p = 16
    d.enc = mkf.ENC_F32
    ts.nT = 0
    assert L.mkfFieldBPFD(16, C.byref(d), C.byref(ts), 0, None) == -1
    assert b"nT" in L.mkfLastError()
    ts.nT = 33
    assert L.mkfFieldBPFD(16, C.byref(d), C.byref(ts), 0, None) == -1
    assert L.mkfMeasuresF64(None, None, 1) == -1
    assert L.mkfCUDAGetBPFD(None, None, None, None, 3) is None
