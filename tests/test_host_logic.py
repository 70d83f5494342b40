"""Host-side logic that needs no GPU: the request loop's device-memory sub-allocator, compiled
from the library's own header with the host compiler and checked against a model."""
import os
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_arena_allocator(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    exe = tmp_path / "arena_check"
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", os.path.join(REPO, "mkf_b200", "csrc"),
                    os.path.join(REPO, "tests", "arena_check.cpp"), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "arena check ok" in r.stdout
