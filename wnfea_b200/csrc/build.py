"""Build libwnfea_cuda.so in-tree for sm_100a with nvcc (no JIT, no torch extension).

Usage: python -m wnfea_b200.csrc.build  [--force]
Each .cu / .cpp in this directory is compiled to an object under _build/ (rebuilt when its
source or any header changed) and linked into wnfea_b200/libwnfea_cuda.so.
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
PKG = HERE.parent
ROOT = PKG.parent
OUT = PKG / "libwnfea_cuda.so"
BUILD = HERE / "_build"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# host code (the AMG setup) for x86-64-v3: AVX2 + FMA, present on every current server CPU
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3,-march=x86-64-v3", "--expt-relaxed-constexpr",
              "-Xptxas", "-O3", f"-I{ROOT / 'include'}"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libwnfea_cuda.so")
    return cand


def _headers_mtime() -> float:
    hs = list(HERE.glob("*.h")) + list(HERE.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _compile(src: Path, force: bool, verbose_ptxas: bool) -> Path:
    obj = BUILD / (src.name + ".o")
    if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, _headers_mtime()):
        return obj
    cmd = [_nvcc(), *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
    if verbose_ptxas and src.suffix == ".cu":
        cmd += ["-Xptxas", "-v"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stdout}\n{res.stderr}")
    if verbose_ptxas:
        sys.stderr.write(res.stderr)
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(HERE.glob("*.cu")) + sorted(HERE.glob("*.cpp"))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose_ptxas), srcs))
    if force or not OUT.exists() or OUT.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [_nvcc(), *ARCH, "-shared", "-o", str(OUT), *map(str, objs), "-lpthread"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv))
