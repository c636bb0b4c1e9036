"""Build libps2cuda.so in-tree with nvcc for sm_100a (no GPU needed)."""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
SOURCES = [CSRC / "ps2_kernels.cu", CSRC / "ps2_api.cu"]
HEADERS = [CSRC / "ps2_kernels.cuh", CSRC / "ps2_device.cuh", CSRC / "interp10_taps.h", CSRC / "trial_interp_taps.h", CSRC / "sincos_poly.h", CSRC / "atan_poly.h",
           HERE.parent / "include" / "ps2cuda.h"]
TARGET = HERE / "libps2cuda.so"

NVCC_FLAGS = [
    "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def needs_build() -> bool:
    if not TARGET.exists():
        return True
    t = TARGET.stat().st_mtime
    return any(p.stat().st_mtime > t for p in SOURCES + HEADERS)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return TARGET
    cmd = [nvcc(), *NVCC_FLAGS, "-o", str(TARGET), *map(str, SOURCES)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True, cwd=str(HERE))
    return TARGET


if __name__ == "__main__":
    build(force=True, verbose=True)
    print(TARGET)
