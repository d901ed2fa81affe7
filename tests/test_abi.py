"""The C ABI library: loads without a GPU, exports every entry point include/gofish_b200.h declares,
and its host-only entry point reproduces the reference's host RNG exactly.  No GPU needed."""
from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import parallelpopgen_b200 as pb
from parallelpopgen_b200 import _capi

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "gofish_b200.h"
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions() -> list[str]:
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(gf_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = _capi.load()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes table binds all of them
    assert set(names) <= set(_capi.SIGNATURES), set(names) - set(_capi.SIGNATURES)
    out = subprocess.run(["nm", "-D", "--defined-only", str(_capi.LIB_PATH)], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(rf"\bT {n}$", out, flags=re.M), n


def test_library_is_built_for_sm100a_only():
    """Every object of the library is compiled for sm_100a and nothing else (the build's only
    -gencode pair; no PTX for other architectures is embedded)."""
    from parallelpopgen_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert "--use_fast_math" in build.CFLAGS


def test_struct_layouts_match_the_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(f'''#include "{HEADER}"
#include <stdio.h>
#include <stddef.h>
int main(void) {{
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(gf_generation), sizeof(gf_population_params),
         sizeof(gf_mse_population), sizeof(gf_sim_config), offsetof(gf_generation, migration),
         sizeof(gf_sim_stats), sizeof(gf_kernel_times), sizeof(gf_batch_stats), sizeof(gf_tuning),
         sizeof(gf_replicate));
  return 0;
}}''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", str(src), "-o", str(exe)], check=True)
    sizes = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert sizes[0] == _capi.GEN_DTYPE.itemsize
    assert sizes[1] == _capi.POP_DTYPE.itemsize
    assert sizes[2] == _capi.MSE_DTYPE.itemsize
    assert sizes[3] == ctypes.sizeof(_capi.SimConfig)
    assert sizes[4] == _capi.GEN_DTYPE.fields["migration"][1]
    assert sizes[5] == ctypes.sizeof(_capi.SimStats)
    assert sizes[6] == ctypes.sizeof(_capi.KernelTimes)
    assert sizes[7] == ctypes.sizeof(_capi.BatchStats)
    assert sizes[8] == ctypes.sizeof(_capi.Tuning)
    assert sizes[9] == ctypes.sizeof(_capi.Replicate)


def test_status_strings_and_version():
    lib = _capi.load()
    assert lib.gf_version() == b"0.1.0"
    for code in range(8):
        assert lib.gf_status_string(code) not in (b"", b"unknown status")


def test_engine_without_gpu_reports_no_device():
    from conftest import has_gpu
    if has_gpu():
        pytest.skip("a GPU is present")
    h = ctypes.c_void_p()
    assert _capi.load().gf_engine_create(0, None, ctypes.byref(h)) == 7  # GF_ERR_NO_DEVICE
    with pytest.raises(pb.GoFishError):
        pb.Engine()


def test_host_new_mutation_count_matches_reference_host_code():
    """gf_new_mutation_count is the product's host-side draw of the per-generation new-mutation count;
    the golden vectors were drawn by the reference's RNG::ApproxRandPois1 on the host."""
    b = np.fromfile(ROOT / "tests" / "golden" / "ref_hostrng.bin", dtype=np.int32)
    nph = int(b[0])
    po = b[2 + nph * 10:].reshape(-1, 6)
    lib = _capi.load()
    n = 0
    for r in po:
        mean = float(np.int32(r[2]).view(np.float32))
        # mean = mu * Nc * L with Nc * L = 1e12: pick mu so that the product is exactly `mean`
        mu = np.float32(mean / 1e12)
        if float(mu * np.float32(1e6) * np.float32(1e6)) != mean:
            continue
        got = lib.gf_new_mutation_count(int(r[0]), int(r[1]), float(mu), 1000000, 1e6, int(r[3]), int(r[4]))
        assert got == r[5], (mean, int(r[3]), int(r[4]))
        n += 1
    assert n > 500
