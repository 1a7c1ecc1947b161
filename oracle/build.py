"""Build the oracle libraries (test infrastructure).

    python oracle/build.py

1. oracle/_build/liboracle.so -- gcc build of gwn_oracle.c, the CPU restatement of smallgwn's
   algorithms (OpenMP, -ffp-contract=off).
2. oracle/_ref/libgwnref.so -- smallgwn's own CUDA kernels, compiled for sm_100a from the
   project's headers where they lie through the thin extern "C" shim oracle/ref_shim.cu. Built
   only when those headers exist; the built library travels with the repository to GPU machines,
   the headers do not.
The reference project's location is this recipe's one input: GWN_REFERENCE_ROOT when set, else the
read-only mount the reference is provided at in the build container.
3. oracle/_ref/libgwnrefcpu.so -- smallgwn's own CPU reference code compiled with g++ from where it
   lies: the exact brute force of tests/reference_cpu.cuh and the vendored SideFX HDK Taylor tree
   (tests/reference_hdk/UT_SolidAngle.cpp, UT_Array.cpp) behind oracle/ref_cpu.cpp, with the small
   Eigen / oneTBB stand-ins of oracle/shims/ in place of those libraries (not installed here).
   Built only when the reference sources exist; portable x86-64 flags (SSE4.2, which the HDK's
   SIMD code needs), so the library also runs on the GPU machines.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load these libraries.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
REF = HERE / "_ref"
ORACLE_SO = BUILD / "liboracle.so"
REF_SO = REF / "libgwnref.so"
REF_CPU_SO = REF / "libgwnrefcpu.so"
REFERENCE_ROOT = Path(os.environ.get("GWN_REFERENCE_ROOT", "/root/reference"))
REFERENCE_INCLUDE = REFERENCE_ROOT / "include"


def _newer(target: Path, *deps: Path) -> bool:
    return not target.exists() or any(d.stat().st_mtime > target.stat().st_mtime for d in deps if d.exists())


def build_oracle(force: bool = False) -> Path:
    src = HERE / "gwn_oracle.c"
    if force or _newer(ORACLE_SO, src, Path(__file__)):
        BUILD.mkdir(exist_ok=True)
        cmd = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
               "-fno-fast-math", "-Wall", "-Wno-unused-function", str(src), "-o", str(ORACLE_SO), "-lm"]
        subprocess.run(cmd, check=True)
    return ORACLE_SO


def build_reference(force: bool = False) -> Path | None:
    """Compile smallgwn's kernels into oracle/_ref when its headers are present; else skip."""
    shim = HERE / "ref_shim.cu"
    if not (REFERENCE_INCLUDE / "gwn" / "gwn.cuh").exists():
        return REF_SO if REF_SO.exists() else None
    if force or _newer(REF_SO, shim, Path(__file__)):
        REF.mkdir(exist_ok=True)
        nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
        cmd = [nvcc, "-std=c++20", "--expt-relaxed-constexpr", "-O3", "-DNDEBUG",
               "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC", "-shared",
               "-I", str(REFERENCE_INCLUDE), str(shim), "-o", str(REF_SO)]
        subprocess.run(cmd, check=True)
    return REF_SO


def build_reference_cpu(force: bool = False) -> Path | None:
    """Compile smallgwn's CPU reference code into oracle/_ref when its sources are present; else skip."""
    shim = HERE / "ref_cpu.cpp"
    tests = REFERENCE_ROOT / "tests"
    hdk = tests / "reference_hdk"
    sources = [shim, hdk / "UT_SolidAngle.cpp", hdk / "UT_Array.cpp"]
    if not (tests / "reference_cpu.cuh").exists() or not all(p.exists() for p in sources[1:]):
        return REF_CPU_SO if REF_CPU_SO.exists() else None
    shims = HERE / "shims"
    deps = [*sources, Path(__file__), *shims.rglob("*")]
    if force or _newer(REF_CPU_SO, *deps):
        REF.mkdir(exist_ok=True)
        cuda_include = Path(shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc").resolve().parents[1] / "include"
        cmd = ["g++", "-std=c++20", "-O3", "-msse4.2", "-fPIC", "-shared", "-pthread", "-I", str(shims),
               "-I", str(REFERENCE_INCLUDE), "-I", str(tests), "-I", str(hdk), "-I", str(cuda_include),
               *map(str, sources), "-o", str(REF_CPU_SO)]
        subprocess.run(cmd, check=True)
    return REF_CPU_SO


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build_oracle(force))
    print(build_reference(force))
    print(build_reference_cpu(force))
