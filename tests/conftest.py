import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the sm_100a kernels")


def has_gpu() -> bool:
    try:
        import ctypes
        cudart = None
        for name in ("libcudart.so.12", "libcudart.so"):
            try:
                cudart = ctypes.CDLL(name)
                break
            except OSError:
                continue
        if cudart is None:
            return False
        n = ctypes.c_int(0)
        return cudart.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def gofish_driver() -> Path:
    """The drop-in C++ driver (tests/cpp/gofish_driver.cpp) built with g++ against include/3P."""
    out = ROOT / "tests" / "_build" / "gofish_driver"
    src = ROOT / "tests" / "cpp" / "gofish_driver.cpp"
    deps = [src, ROOT / "tests" / "cpp" / "scenarios.h", *(ROOT / "include" / "3P").glob("*"),
            ROOT / "include" / "gofish_b200.h", ROOT / "parallelpopgen_b200" / "libgofish_b200.so"]
    if not out.exists() or out.stat().st_mtime < max(d.stat().st_mtime for d in deps):
        out.parent.mkdir(exist_ok=True)
        subprocess.run(["g++", "-O2", "-std=c++17", "-I", str(ROOT / "include" / "3P"), "-I", str(src.parent),
                        str(src), "-o", str(out), "-L", str(ROOT / "parallelpopgen_b200"), "-lgofish_b200",
                        "-Wl,-rpath," + str(ROOT / "parallelpopgen_b200")], check=True)
    return out


@pytest.fixture(scope="session")
def gofish_driver_nvcc() -> Path:
    """The same drop-in driver compiled by nvcc (as a CUDA translation unit, with the reference's
    -O3 --use_fast_math), so that selection functors without exact affine coefficients take the
    device-evaluated path of include/3P/go_fish.cuh."""
    out = ROOT / "tests" / "_build" / "gofish_driver_nvcc"
    src = ROOT / "tests" / "cpp" / "gofish_driver.cpp"
    deps = [src, ROOT / "tests" / "cpp" / "scenarios.h", *(ROOT / "include" / "3P").glob("*"),
            ROOT / "include" / "gofish_b200.h", ROOT / "parallelpopgen_b200" / "libgofish_b200.so"]
    if not out.exists() or out.stat().st_mtime < max(d.stat().st_mtime for d in deps):
        out.parent.mkdir(exist_ok=True)
        subprocess.run(["/usr/local/cuda/bin/nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3",
                        "--use_fast_math", "-std=c++17", "-x", "cu", "-I", str(ROOT / "include" / "3P"),
                        "-I", str(src.parent), str(src), "-o", str(out), "-L", str(ROOT / "parallelpopgen_b200"),
                        "-lgofish_b200", "-Xlinker", "-rpath," + str(ROOT / "parallelpopgen_b200")], check=True)
    return out


@pytest.fixture(scope="session")
def ref_driver() -> Path:
    """The reference built from its own sources (oracle/build_ref.sh); skip when absent."""
    p = ROOT / "oracle" / "_ref" / "ref_driver"
    if not p.exists():
        pytest.skip("oracle/_ref/ref_driver not built (the reference sources were not available at build time)")
    return p
