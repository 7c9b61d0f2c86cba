"""ORACLE (test infrastructure only) -- build the reference's own CPU kernels from source.

Compiles the reference's wnfea/solver/native/kernels.cpp (co-rotational beam and C3D10
internal forces, kernels.cpp:19-376) with g++ into oracle/_ref/libwnfea_ref_kernels.so.
The reference only ships this code as a Windows .dll; that binary is never used.  Nothing
is copied: the source is compiled where it lies.

    python oracle/build_ref.py [/path/to/reference]
"""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref" / "libwnfea_ref_kernels.so"


def build(ref: str = "/root/reference") -> Path | None:
    src = Path(ref) / "wnfea" / "solver" / "native" / "kernels.cpp"
    if not src.exists():
        return OUT if OUT.exists() else None
    OUT.parent.mkdir(exist_ok=True)
    if OUT.exists() and OUT.stat().st_mtime >= src.stat().st_mtime:
        return OUT
    # x86-64-v3 (AVX2/FMA) rather than -march=native: the library also runs on other hosts
    cmd = ["g++", "-O3", "-march=x86-64-v3", "-shared", "-fPIC", str(src), "-o", str(OUT)]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else "/root/reference"))
