"""Build libfwi2d.so and the modeling / migration / inversion executables in-tree.

Device code is compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``);
host code with g++ and ``-ffp-contract=off`` so every float expression rounds as
written.  ``k_rbc.cu`` is compiled with ``-fmad=false`` so the random boundary
is bit-identical to a host evaluation.  Objects are rebuilt when a source or
header is newer than the object.

    python -m fwi2d_b200.build          # or: python fwi2d_b200/build.py
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
BIN = PKG / "bin"
LIB = PKG / "libfwi2d.so"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA / "bin" / "nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-ffp-contract=off"] + ARCH
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fopenmp", "-Wall", "-Wno-unused-function",
             f"-I{CUDA / 'include'}"]

CU_SOURCES = {
    "k_stencil.cu": [],
    "k_fwd_tma.cu": [],
    "k_fwd_loop.cu": [],
    "k_fwd_res.cu": [],
    "k_bwd_loop.cu": [],
    "k_prep.cu": ["-fmad=false"],
    "k_nn.cu": [],
    "k_nn_tma.cu": [],
    "k_util.cu": [],
    "k_rbc.cu": ["-fmad=false"],
    "k_noalloc.cu": [],
}
CXX_SOURCES = ["host.cpp", "engine.cpp", "capi.cpp", "capi_nn.cpp"]
APPS = ["modeling", "migration", "inversion"]


def _headers() -> list[Path]:
    return (list(CSRC.glob("*.h")) + list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh"))
            + [ROOT / "include" / "fwi2d.h"])


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(verbose: bool = False, jobs: int | None = None) -> Path:
    OBJ.mkdir(exist_ok=True)
    BIN.mkdir(exist_ok=True)
    hdrs = _headers()
    steps = []
    objs = []
    for src, extra in CU_SOURCES.items():
        o = OBJ / (src + ".o")
        objs.append(o)
        if _stale(o, [CSRC / src] + hdrs):
            steps.append([NVCC, *NVCC_FLAGS, *extra, "-c", str(CSRC / src), "-o", str(o)])
    for src in CXX_SOURCES:
        o = OBJ / (src + ".o")
        objs.append(o)
        if _stale(o, [CSRC / src] + hdrs):
            steps.append(["g++", *CXX_FLAGS, "-c", str(CSRC / src), "-o", str(o)])
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for cmd, fut in [(c, ex.submit(_run, c)) for c in steps]:
            if verbose:
                print(" ".join(cmd))
            fut.result()
    if steps or not LIB.exists() or _stale(LIB, objs):
        _run([NVCC, "-shared", *ARCH, "-cudart", "static", "-o", str(LIB), *map(str, objs),
              "-Xcompiler", "-fopenmp", "-lgomp", "-lpthread", "-ldl", "-lrt"])
    for app in APPS:
        exe = BIN / app
        src = CSRC / "apps" / f"{app}_main.cpp"
        if _stale(exe, [src, LIB, CSRC / "apps" / "app_common.hpp"]):
            _run(["g++", "-O2", "-std=c++17", "-pthread", "-o", str(exe), str(src), f"-L{PKG}", "-lfwi2d",
                  "-Wl,-rpath,$ORIGIN/.."])
    return LIB


def clean() -> None:
    shutil.rmtree(OBJ, ignore_errors=True)
    shutil.rmtree(BIN, ignore_errors=True)
    if LIB.exists():
        LIB.unlink()


if __name__ == "__main__":
    if "--clean" in sys.argv:
        clean()
    print(build(verbose="-v" in sys.argv))
