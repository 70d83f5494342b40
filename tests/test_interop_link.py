"""The original OpenACC interop caller, built against this library's headers and linked to libMKF.so.

`mkfAccCUDAGetBPFD` (MKF src/mkfACC.c:248-318) hands OpenACC device pointers of a field to
`binMapCUDA` and `mkfCUDAGetBPFDH`. Its source, with the original CPU map it shares a file set with
(src/binMapACC.c), is compiled unchanged here with MKF_ACC_CUDA_INTEROP against `include/` (the
original's util.h comes from the oracle's stand-in), then linked into a shared object with
`--no-undefined` against libMKF.so and libgomp: every symbol it needs from the MKF library must
resolve in libMKF.so. CPU only, and nothing is run: gcc's OpenACC has no device offload here, so
its host fallback would hand host pointers to the CUDA entry points.

Needs the original sources (MKF_REFERENCE, default the reference checkout); skipped without them.
"""
import os
import shutil
import subprocess

import pytest

from conftest import REPO

REF_SRC = os.path.join(os.environ.get("MKF_REFERENCE", "/root/reference"), "src")
ACC_FILES = ["mkfACC.c", "mkfACC.h", "binMapACC.c", "binMapACC.h", "mkfTest.h"]


def _have_openacc() -> bool:
    r = subprocess.run(["gcc", "-E", "-x", "c", "-", "-o", os.devnull], input="#include <openacc.h>\n",
                       capture_output=True, text=True)
    return r.returncode == 0


def _exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], check=True, capture_output=True, text=True).stdout
    return {ln.split()[-1].split("@")[0] for ln in out.splitlines() if ln.strip()}


def _undefined(obj):
    out = subprocess.run(["nm", "-u", obj], check=True, capture_output=True, text=True).stdout
    return {ln.split()[-1].split("@")[0] for ln in out.splitlines() if ln.strip()}


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_SRC, "mkfACC.c")), reason="original MKF sources not present")
@pytest.mark.skipif(not _have_openacc(), reason="gcc's openacc.h (libgomp) not installed")
def test_openacc_interop_caller_links_against_libmkf(tmp_path, mkf):
    from mkf_b200 import _lib

    # the caller's own files in a directory of their own, so that its quoted includes of the
    # headers this library replaces (mkfCUDA.h, binMapUtil.h, mkfUtil.h, ...) find include/
    for fn in ACC_FILES:
        shutil.copy(os.path.join(REF_SRC, fn), tmp_path / fn)
    inc = ["-I" + str(tmp_path), "-I" + os.path.join(REPO, "include"), "-I" + os.path.join(REPO, "oracle", "shim")]
    cc = ["gcc", "-std=gnu11", "-fPIC", "-w", "-c"]
    acc_o, map_o = str(tmp_path / "mkfACC.o"), str(tmp_path / "binMapACC.o")
    # openacc.h is included by the caller only under PGI; gcc's declares the same acc_* API
    subprocess.run(cc + ["-DMKF_ACC_CUDA_INTEROP", "-include", "openacc.h"] + inc +
                   [str(tmp_path / "mkfACC.c"), "-o", acc_o], check=True)
    subprocess.run(cc + inc + [str(tmp_path / "binMapACC.c"), "-o", map_o], check=True)

    lib_dir, lib_name = os.path.split(_lib.LIB_PATH)
    so = str(tmp_path / "libaccinterop.so")
    r = subprocess.run(["gcc", "-shared", "-Wl,--no-undefined", "-o", so, acc_o, map_o, "-L" + lib_dir,
                        "-l:" + lib_name, "-Wl,-rpath," + lib_dir, "-lgomp", "-lm"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

    assert "mkfAccCUDAGetBPFD" in _exported(so)
    ours = _exported(_lib.LIB_PATH)
    from_mkf = _undefined(acc_o) - _exported(so) - {"acc_get_device_type", "acc_set_device_type", "GOACC_data_start",
                                                    "GOACC_data_end", "memset", "__stack_chk_fail"}
    # the MKF entry points the interop path calls all come from libMKF.so
    assert {"binMapCUDA", "mkfCUDAGetBPFDH", "setBMO", "prodNI"} <= from_mkf
    assert from_mkf <= ours, from_mkf - ours
