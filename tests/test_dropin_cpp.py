"""The C++ drop-in headers (include/gwn/*.cuh) compile with a plain C++20 host compiler and, on a
GPU, a program written against smallgwn's API runs its unit-test cases through libgwnb.so.
"""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import pytest

from smallgwn_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "cpp" / "dropin_test.cpp"


def cuda_root() -> Path:
    nvcc = shutil.which("nvcc")
    if nvcc:
        return Path(nvcc).resolve().parents[1]
    return Path("/usr/local/cuda")


def compile_program(out: Path) -> Path:
    _lib.load()  # make sure the library is built
    cr = cuda_root()
    libdir = _lib.library_path().parent
    cmd = ["g++", "-std=c++20", "-O1", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"), "-I", str(cr / "include"), str(SRC),
           "-L", str(libdir), "-lgwnb", "-L", str(cr / "lib64"), "-lcudart", f"-Wl,-rpath,{libdir}",
           f"-Wl,-rpath,{cr / 'lib64'}", "-o", str(out)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return out


def test_dropin_headers_compile_with_host_compiler(tmp_path):
    exe = compile_program(tmp_path / "dropin_test")
    assert subprocess.run([str(exe), "--compile-only"]).returncode == 0


def test_dropin_host_checks(tmp_path):
    """Cases that need no GPU: the matrix upload's refusals and PLY round trips."""
    exe = compile_program(tmp_path / "dropin_test")
    res = subprocess.run([str(exe), "--host-checks"], capture_output=True, text=True, timeout=120)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "host checks passed" in res.stdout


@pytest.mark.gpu
def test_dropin_program_passes_reference_unit_cases(tmp_path):
    exe = compile_program(tmp_path / "dropin_test")
    res = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "all checks passed" in res.stdout
