"""Build the in-tree CUDA library ``lib/libhicma_tlr.so`` (sm_100a), its
bounds-checked variant ``lib/libhicma_tlr_checked.so`` (host sources compiled
with TLR_BOUNDS_CHECK, same kernels) and the ``testing_dpotrf_tlr``
command-line driver.

Usage: ``python -m hicma_parsec_b200.build [--force]`` (also called by
``__graft_entry__.build()``).  nvcc cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libhicma_tlr.so")
LIB_CHECKED = os.path.join(LIBDIR, "libhicma_tlr_checked.so")
OBJ_CHECKED = os.path.join(OBJ, "checked")
# sources whose host code carries the launch checks of the checked build
CHECKED_SOURCES = ["tlr_engine.cu", "serve.cu", "k_potrf.cu"]
CLI_SRC = os.path.join(HERE, "cli", "testing_dpotrf_tlr.c")
CLI = os.path.join(LIBDIR, "testing_dpotrf_tlr")
SOURCES = ["k_gemm.cu", "k_tile.cu", "k_potrf.cu", "k_potrf_tile.cu", "k_qr.cu", "k_rcholqr.cu", "k_proj.cu", "k_svd.cu",
           "tlr_engine.cu", "serve.cu"]
HEADERS = ["tlr_internal.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
              "-Xptxas", "-v"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _compile(nvcc: str, src: str, force: bool, checked: bool = False) -> tuple[str, str]:
    out = os.path.join(OBJ_CHECKED if checked else OBJ, os.path.basename(src).replace(".cu", ".o"))
    deps = [src] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "hicma_tlr.h")]
    if not force and _newer(out, deps):
        return out, ""
    cmd = [nvcc, *ARCH, *NVCC_FLAGS, *(["-DTLR_BOUNDS_CHECK"] if checked else []), "-c", src, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return out, r.stderr


def _link(nvcc: str, out: str, objs: list[str], force: bool) -> None:
    if force or not _newer(out, objs):
        cmd = [nvcc, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", out, *objs, "-lpthread", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ_CHECKED, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    nvcc = _nvcc()
    jobs = [(s, False) for s in SOURCES] + [(s, True) for s in CHECKED_SOURCES]
    with cf.ThreadPoolExecutor(max_workers=len(jobs)) as ex:
        results = list(ex.map(lambda j: _compile(nvcc, os.path.join(CSRC, j[0]), force, j[1]), jobs))
    objs = [o for (o, _), (_, chk) in zip(results, jobs) if not chk]
    checked = {os.path.basename(o): o for (o, _), (_, chk) in zip(results, jobs) if chk}
    if verbose:
        for _, log in results:
            if log:
                sys.stderr.write(log)
    _link(nvcc, LIB, objs, force)
    _link(nvcc, LIB_CHECKED, [checked.get(os.path.basename(o), o) for o in objs], force)
    if os.path.exists(CLI_SRC) and (force or not _newer(CLI, [CLI_SRC, LIB])):
        cmd = ["gcc", "-O2", "-std=c11", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"),
               CLI_SRC, "-o", CLI, "-L", LIBDIR, "-lhicma_tlr", f"-Wl,-rpath,$ORIGIN", "-lm"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"CLI build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
