"""gf_site_frequency_spectrum_noalloc: the SFS entry point for callers that cannot allocate device
memory (a framework that owns the GPU memory budget, or a latency-critical path where cudaMalloc would
synchronize the device).  Called through the C ABI, it must give the same SFS as the engine-based
entry point gf_site_frequency_spectrum_device (within the SFS tolerance of the other tests: 1e-5
relative) on calls in a row -- the calls share one scratch array, so the later calls also check that
nothing of an earlier call leaks into them: the third call takes the histogram path again with a
smaller population than the first, so stale counts above its own range, or counts the first call left
in its range, would show in its spectrum -- and the calls after the first must not change the device's
free memory.  This file is collected last on purpose."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_sfs_matches_engine_sfs_on_calls_in_a_row():
    import torch

    from parallelpopgen_b200 import Engine, _capi

    lib = _capi.load()
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    rng = np.random.default_rng(12)
    Nc, L = 400000, 2.5e8
    # call 1: engine frequencies on the 1/Nc grid (histogram projection), n = 1000
    j = np.minimum(rng.geometric(2e-5, size=2_000_000), Nc)
    j[rng.random(j.size) < 0.05] = 0
    grid = (j.astype(np.float32) / np.float32(Nc)).astype(np.float32)
    # call 2: frequencies off the grid (direct projection), smaller population and sample
    off = rng.random(300_000).astype(np.float32)
    # call 3: the histogram path again, a smaller population than call 1 (its counts must start at zero)
    Nc3 = 30000
    j3 = np.minimum(rng.geometric(3e-4, size=500_000), Nc3)
    grid3 = (j3.astype(np.float32) / np.float32(Nc3)).astype(np.float32)
    cases = [(grid, Nc, 1000), (off, 50000, 100), (grid3, Nc3, 500)]
    with Engine(device=0, stream=stream.cuda_stream) as eng:
        for k, (x, nc, n) in enumerate(cases):
            d_x = torch.from_numpy(x).cuda()
            want = torch.empty(n, dtype=torch.float32, device="cuda")
            eng.site_frequency_spectrum_device(d_x.data_ptr(), len(x), nc, n, L, want.data_ptr())
            eng.synchronize()
            got = torch.full((n,), float("nan"), dtype=torch.float32, device="cuda")
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            st = lib.gf_site_frequency_spectrum_noalloc(ctypes.c_void_p(d_x.data_ptr()), len(x), nc, n, L,
                                                        ctypes.c_void_p(got.data_ptr()),
                                                        ctypes.c_void_p(stream.cuda_stream))
            assert st == 0, _capi.STATUS_NAMES.get(st, st)
            stream.synchronize()
            free_after = torch.cuda.mem_get_info()[0]
            # the first call on the device may load the module that holds the scratch array (lazy
            # module loading), which is when the array takes its memory: exempt from the check
            if k > 0:
                assert free_after == free_before, f"call {k + 1} changed free device memory"
            np.testing.assert_allclose(got.cpu().numpy().astype(np.float64), want.cpu().numpy().astype(np.float64),
                                       rtol=1e-5, atol=1e-3)


def test_noalloc_sfs_rejects_sizes_beyond_its_scratch():
    import torch

    from parallelpopgen_b200 import _capi

    lib = _capi.load()
    d_x = torch.zeros(16, dtype=torch.float32, device="cuda")
    d_out = torch.zeros(2048, dtype=torch.float32, device="cuda")
    big_nc = (1 << 20) + 1
    assert lib.gf_site_frequency_spectrum_noalloc(ctypes.c_void_p(d_x.data_ptr()), 16, big_nc, 10, 1e6,
                                                  ctypes.c_void_p(d_out.data_ptr()), None) == 4  # GF_ERR_CAPACITY
    assert lib.gf_site_frequency_spectrum_noalloc(ctypes.c_void_p(d_x.data_ptr()), 16, 100000, 1024, 1e6,
                                                  ctypes.c_void_p(d_out.data_ptr()), None) == 4
    assert lib.gf_site_frequency_spectrum_noalloc(ctypes.c_void_p(d_x.data_ptr()), 16, 100, 100, 1e6,
                                                  ctypes.c_void_p(d_out.data_ptr()), None) == 1  # n >= Nc
