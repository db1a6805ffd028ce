"""In-tree build of libmtl4_b200.so for sm_100a (nvcc, no JIT cache)."""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
SRC = PKG / "csrc"
OUT = PKG / "libmtl4_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
         "-Xcompiler", "-fPIC", "-shared"]


def sources():
    return sorted(SRC.glob("*.cu")) + sorted(SRC.glob("*.cuh")) + [PKG.parent / "include" / "mtl4_b200" / "mtlg.h"]


def needs_build() -> bool:
    if not OUT.exists():
        return True
    t = OUT.stat().st_mtime
    return any(p.stat().st_mtime > t for p in sources())


def build_library(force: bool = False, verbose: bool = False) -> Path:
    if force or needs_build():
        cmd = [NVCC, *FLAGS, str(SRC / "mtlg.cu"), str(SRC / "noalloc.cu"), "-o", str(OUT)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build_library(force=True, verbose=True)
