"""In-tree build of the CUDA library and the drop-in driver.

    python -m mixedprecisionfaracoustic_b200.build        # or build() from Python

Produces, next to this file:
    lib/libbiot_b200.so       the C-ABI library (include/biot.h), sm_100a only
    bin/biot_reference_run    the reference program's drop-in (C++ host driver)

nvcc cross-compiles for sm_100a without a GPU.  Objects are compiled in
parallel into _build/ and relinked only when a source is newer.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "lib" / "libbiot_b200.so"
BIN = PKG / "bin" / "biot_reference_run"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
LIB_SOURCES = ["step.cu", "step_inter.cu", "step_fused.cu", "step_staged.cu", "step_march.cu", "precompute.cu", "medium_index.cu", "reduce.cu", "codec.cu", "shot.cu", "sim.cu", "batch.cu", "server.cu", "noalloc.cu",
               "medium.cpp"]
DRIVER = "driver_main.cpp"


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx() -> list[str]:
    # the system g++ (a wrapper earlier on PATH may lack parts of the toolchain)
    return ["-ccbin", "/usr/bin/g++"] if Path("/usr/bin/g++").exists() else []


def _headers() -> list[Path]:
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [INCLUDE / "biot.h"]


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, verbose: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    if not _stale(obj, [src] + _headers()):
        return obj
    cmd = [_nvcc(), *_host_cxx(), "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC",
           "-Xcompiler", "-Wall", "-diag-suppress", "177", "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIB.parent.mkdir(exist_ok=True)
    BIN.parent.mkdir(exist_ok=True)
    srcs = [CSRC / s for s in LIB_SOURCES]
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if _stale(LIB, objs):
        cmd = [_nvcc(), *_host_cxx(), "-shared", *ARCH, "-o", str(LIB), *map(str, objs), "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    drv = CSRC / DRIVER
    if _stale(BIN, [drv, LIB, INCLUDE / "biot.h"]):
        cmd = [_nvcc(), *_host_cxx(), "-std=c++17", "-O2", *ARCH, "-I", str(INCLUDE), str(drv), "-o", str(BIN),
               "-L", str(LIB.parent), "-lbiot_b200", "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN/../lib"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"driver build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
