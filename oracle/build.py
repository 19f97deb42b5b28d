"""Build recipe of the checker (TEST INFRASTRUCTURE ONLY).

1. oracle/libkt_oracle.so  — the CPU restatement (kt_oracle.cpp), g++ with OpenMP.
2. oracle/_ref/libktref_<scene>.so — the reference's own cuda/kernel.cu compiled from its
   source tree for sm_100a, once per scene whose `#define` set differs (the reference bakes
   its integrator knobs into the source, src/renderer/utils.rs:121-163).  Only built when the
   reference tree is present (the build container); the .so files travel with the repository
   snapshot to the GPU machine.

The `#define` text is produced here independently of the product library, with Rust's
`{:.10}` formatting of the f32 value (Python's exact decimal formatting of the same binary
value); the scene values it formats come from the oracle's host restatement.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
# The reference source tree (read only); KT_REFERENCE_DIR overrides the default location.
REF_DIR = Path(os.environ.get("KT_REFERENCE_DIR", "/root/reference"))
REF_OUT = HERE / "_ref"
ORACLE_LIB = HERE / "libkt_oracle.so"
REF_SCENES = ("c1", "c2", "t1", "t2")


def _run(cmd: list[str]) -> None:
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{proc.stdout}\n{proc.stderr}")


def build_oracle(force: bool = False) -> Path:
    src = HERE / "kt_oracle.cpp"
    if not force and ORACLE_LIB.exists() and ORACLE_LIB.stat().st_mtime >= src.stat().st_mtime:
        return ORACLE_LIB
    tmp = ORACLE_LIB.with_suffix(".so.tmp")
    _run([shutil.which("g++") or "g++", "-std=c++17", "-O2", "-fopenmp", "-fPIC", "-shared",
          "-ffp-contract=off", "-fno-fast-math", str(src), "-o", str(tmp)])
    os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


def f32(x: float) -> float:
    import numpy as np
    return float(np.float32(x))


def defines_text(cfg) -> str:
    """The header the reference's build_cuda_defines would emit for this config."""
    ints = [("CONFIG_SPP", cfg.spp), ("CONFIG_SKY_GRID_DIVISIONS", cfg.sky_grid_divisions),
            ("CONFIG_INTEGRATOR_MAX_STEPS", cfg.max_steps), ("CONFIG_INTEGRATOR_MAX_ATTEMPTS", cfg.max_attempts)]
    floats = [("CONFIG_EXPOSURE_SCALE", cfg.exposure_scale), ("CONFIG_SKY_LINE_THICKNESS", cfg.sky_line_thickness),
              ("CONFIG_SKY_INTENSITY", cfg.sky_intensity), ("CONFIG_DISK_OUTER_RADIUS", cfg.disk_outer_radius),
              ("CONFIG_DISK_TEMPERATURE_SCALE", cfg.disk_temperature_scale),
              ("CONFIG_INTEGRATOR_INITIAL_STEP", cfg.initial_step), ("CONFIG_INTEGRATOR_TOLERANCE", cfg.tolerance),
              ("CONFIG_TRANSMITTANCE_CUTOFF", cfg.transmittance_cutoff),
              ("CONFIG_HORIZON_EPSILON", cfg.horizon_epsilon), ("CONFIG_ESCAPE_RADIUS", cfg.escape_radius),
              ("CONFIG_BLACKBODY_WAVELENGTH_STEP", cfg.wavelength_step)]
    lines = [f"#define {k} {int(v)}" for k, v in ints] + [f"#define {k} {f32(v):.10f}" for k, v in floats]
    return "\n".join(lines) + "\n"


def build_reference(force: bool = False) -> list[Path]:
    if not (REF_DIR / "cuda" / "kernel.cu").exists():
        return []
    sys.path.insert(0, str(ROOT))
    import oracle
    from kerrtrace_b200 import workloads
    host = oracle.Host()  # scene values from the oracle's host restatement, not the product
    REF_OUT.mkdir(exist_ok=True)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    built = []
    for name in REF_SCENES:
        cfg, _ = workloads.scene(name, host=host)
        hdr = REF_OUT / f"defines_{name}.h"
        text = defines_text(cfg)
        lib = REF_OUT / f"libktref_{name}.so"
        harness = HERE / "ref_harness.cu"
        stale = (not lib.exists() or not hdr.exists() or hdr.read_text() != text
                 or lib.stat().st_mtime < harness.stat().st_mtime)
        if force or stale:
            hdr.write_text(text)
            tmp = lib.with_suffix(".so.tmp")
            _run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-use_fast_math", "-shared",
                  "-Xcompiler", "-fPIC", "-cudart", "static", "-include", str(hdr), "-I", str(REF_DIR / "cuda"),
                  str(harness), "-o", str(tmp)])
            os.replace(tmp, lib)
        built.append(lib)
    return built


def build(force: bool = False) -> None:
    build_oracle(force)
    build_reference(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print(ORACLE_LIB)
    for p in sorted(REF_OUT.glob("*.so")):
        print(p)
