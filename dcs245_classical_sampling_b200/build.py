"""Build the in-tree CUDA library ``libdcs245.so`` for sm_100a with nvcc.

The library is loaded by ``dcs245_classical_sampling_b200._lib`` through ctypes; it exports
the C ABI declared in ``include/dcs245.h``.  Run ``python -m dcs245_classical_sampling_b200.build``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = REPO / "include"
LIB = PKG / "libdcs245.so"
SOURCES = ["abi.cu", "step.cu", "fused.cu", "runs.cu", "runs_r4.cu", "runs_packed.cu", "jit.cu", "block.cu",
           "draw.cu", "serve.cu", "planner.cu", "gather.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def build(verbose=False, ptxas_info=False, force=False):
    """Compile every stale source to an object (in parallel: the register-run kernels take
    minutes) and link the shared library.  An object is stale when its source or any header is
    newer; force=True recompiles everything."""
    from concurrent.futures import ThreadPoolExecutor
    srcs = [CSRC / s for s in SOURCES if (CSRC / s).exists()]
    deps = srcs + list(CSRC.glob("*.cuh")) + [INCLUDE / "dcs245.h"]
    if not force and LIB.exists() and all(LIB.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return LIB
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    flags = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
             "--expt-relaxed-constexpr", f"-I{INCLUDE}", f"-I{CSRC}"]
    if ptxas_info:
        flags.append("-Xptxas=-v")

    headers = list(CSRC.glob("*.cuh")) + [INCLUDE / "dcs245.h"]
    newest_header = max(h.stat().st_mtime for h in headers)

    def compile_one(src):
        obj = objdir / (src.stem + ".o")
        if (not force and obj.exists() and obj.stat().st_mtime >= src.stat().st_mtime
                and obj.stat().st_mtime >= newest_header):
            return obj, subprocess.CompletedProcess([], 0, "", "")  # object is current
        cmd = [nvcc_path(), *flags, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        return obj, subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=len(srcs)) as ex:
        results = list(ex.map(compile_one, srcs))
    for obj, r in results:
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {obj.stem}.cu:\n" + r.stdout + r.stderr)
        if verbose or ptxas_info:
            print(r.stdout + r.stderr)
    cmd = [nvcc_path(), *ARCH, "-shared", "-o", str(LIB) + ".tmp", *[str(o) for o, _ in results], "-lnvrtc"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv, force=True)
