"""Builds libkerrtrace.so in-tree (sm_100a) with nvcc and g++.

The kernels translation unit is compiled with -use_fast_math, the flag set the reference
builds kernel.cu with (config.yaml `cuda.use_fast_math: true`, src/renderer/init.rs:112-118).
The host translation unit restates the reference's Rust host arithmetic and is compiled with
-ffp-contract=off so that only the fused multiply-adds the Rust code spells out (mul_add) are
fused.  cudart is linked statically so the library loads without any runtime search path.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libkerrtrace.so"
BUILD = ROOT / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found")
    return cand


def _run(cmd: list[str]) -> str:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"command failed ({proc.returncode}): {' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")
    return proc.stdout + proc.stderr


def sources() -> list[Path]:
    return sorted(p for p in CSRC.iterdir() if p.suffix in (".cu", ".cuh", ".cpp", ".h")) + [ROOT / "include" / "kerrtrace.h"]


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in sources())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    BUILD.mkdir(exist_ok=True)
    nvcc = _nvcc()
    cuda_home = Path(nvcc).resolve().parent.parent
    inc = ["-I", str(ROOT / "include"), "-I", str(CSRC)]
    k_obj = BUILD / "kt_kernels.o"
    h_obj = BUILD / "kt_host.o"
    log = _run([nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-use_fast_math", "-Xptxas", "-v",
                "-Xcompiler", "-fPIC", *inc, "-c", str(CSRC / "kt_kernels.cu"), "-o", str(k_obj)])
    (BUILD / "ptxas_kt_kernels.txt").write_text(log)
    if verbose:
        print(log)
    n_obj = BUILD / "kt_noalloc.o"
    log = _run([nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-use_fast_math", "-Xptxas", "-v",
                "-Xcompiler", "-fPIC", *inc, "-c", str(CSRC / "kt_noalloc.cu"), "-o", str(n_obj)])
    (BUILD / "ptxas_kt_noalloc.txt").write_text(log)
    l_obj = BUILD / "kt_luts.o"  # accurate libm: no fast math
    log = _run([nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xptxas", "-v",
                "-Xcompiler", "-fPIC", *inc, "-c", str(CSRC / "kt_luts.cu"), "-o", str(l_obj)])
    (BUILD / "ptxas_kt_luts.txt").write_text(log)
    d_obj = BUILD / "kt_diff.o"
    log = _run([nvcc, *ARCH, "-lineinfo", "-O3", "-std=c++17", "-use_fast_math", "-Xptxas", "-v",
                "-Xcompiler", "-fPIC", *inc, "-c", str(CSRC / "kt_diff.cu"), "-o", str(d_obj)])
    (BUILD / "ptxas_kt_diff.txt").write_text(log)
    gxx = shutil.which("g++") or "g++"
    _run([gxx, "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", *inc,
          "-I", str(cuda_home / "include"), "-c", str(CSRC / "kt_host.cpp"), "-o", str(h_obj)])
    dh_obj = BUILD / "kt_diff_host.o"
    _run([gxx, "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", *inc,
          "-I", str(cuda_home / "include"), "-c", str(CSRC / "kt_diff_host.cpp"), "-o", str(dh_obj)])
    t_obj = BUILD / "kt_tune.o"
    _run([gxx, "-std=c++17", "-O2", "-fPIC", *inc, "-I", str(cuda_home / "include"), "-c", str(CSRC / "kt_tune.cpp"),
          "-o", str(t_obj)])
    a_obj = BUILD / "kt_app.o"
    _run([gxx, "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", *inc,
          "-I", str(cuda_home / "include"), "-c", str(CSRC / "kt_app.cpp"), "-o", str(a_obj)])
    tmp = LIB.with_suffix(".so.tmp")
    _run([nvcc, *ARCH, "-shared", "-cudart", "static", str(k_obj), str(n_obj), str(d_obj), str(h_obj), str(dh_obj),
          str(a_obj), str(l_obj), str(t_obj), "-o", str(tmp)])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
