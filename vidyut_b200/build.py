"""Build the sm_100a shared library libvidyut_b200.so in-tree.

    python -m vidyut_b200.build            # builds vidyut_b200/libvidyut_b200.so

nvcc cross-compiles for sm_100a without a GPU.  The library is linked with the
static CUDA runtime so it does not depend on the runtime that PyTorch bundles.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libvidyut_b200.so"
BUILD = PKG / "_build"

SOURCES = ["vd_kernels.cu", "vd_batch_kernels.cu", "vd_abi.cu", "vd_spec.cpp", "vd_batch.cu", "vd_server.cu",
           "vd_poisson.cu", "vd_diffusion.cu", "vd_plotfile.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC,-O3", "-Xptxas", "-O3"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False, force: bool = False) -> Path:
    from concurrent.futures import ThreadPoolExecutor
    BUILD.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [PKG.parent / "include" / "vidyut_b200.h"]
    objs, jobs = [], []
    for src in SOURCES:
        s = CSRC / src
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", str(s), "-o", str(o)]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            jobs.append((src, cmd))

    def run(job):
        src, cmd = job
        if verbose:
            print(" ".join(cmd), flush=True)
        return src, subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=max(1, len(jobs))) as ex:
        results = list(ex.map(run, jobs))
    for src, r in results:
        if r.returncode != 0 or verbose or ptxas_info:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}")
    if force or _stale(LIB, objs):
        cuda_lib = Path(nvcc()).resolve().parent.parent / "lib64"
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-cudart", "static",
               f"-L{cuda_lib}", "-lnvrtc", "-Xlinker", f"-rpath,{cuda_lib}"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv, force="-f" in sys.argv)
    print(LIB)
