"""Build the sm_100a CUDA library libgofish_b200.so in-tree (no JIT cache, no pip install).

    python -m parallelpopgen_b200.build          # incremental
    python -m parallelpopgen_b200.build --force  # rebuild everything

Every .cu file under csrc/ is compiled with nvcc for sm_100a only and linked into one shared
library next to this file.  --use_fast_math matches the flags the reference builds its kernels with
(examples/*/makefile: `-O3 --use_fast_math`), which the bit-exact parity contract depends on.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libgofish_b200.so"
INCLUDE = PKG.parent / "include"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CFLAGS = ["-O3", "--use_fast_math", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
          "-I", str(INCLUDE), "-I", str(CSRC)]


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _run(cmd: list[str]) -> None:
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose_ptxas: bool = False, defines: list[str] | None = None,
          out: Path | None = None, build_dir: Path | None = None) -> Path:
    """Compile csrc/*.cu into one shared library (default: libgofish_b200.so next to this file).
    `defines` (e.g. ["GF_DRIFT_MIN_BLOCKS=6"]) and `out`/`build_dir` build a variant elsewhere."""
    bdir = build_dir or BUILD
    lib = out or LIB
    dflags = [f"-D{d}" for d in (defines or [])]
    bdir.mkdir(parents=True, exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    hdr_mtime = max((h.stat().st_mtime for h in _headers()), default=0.0)
    objects = []
    rebuilt = False
    for src in sources:
        obj = bdir / (src.stem + ".o")
        objects.append(obj)
        if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr_mtime):
            extra = ["-Xptxas", "-v"] if verbose_ptxas else []
            _run([NVCC, *ARCH, *CFLAGS, *dflags, *extra, "-c", str(src), "-o", str(obj)])
            rebuilt = True
    if force or rebuilt or not lib.exists():
        _run([NVCC, *ARCH, "-shared", "-o", str(lib), *map(str, objects), "-lcudart"])
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="--ptxas-v" in sys.argv)
