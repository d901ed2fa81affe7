"""Engines are independent: two simulations run at the same time from two host threads, each on its
own engine and stream, end in exactly the states they reach when run one after the other."""
from __future__ import annotations

import threading

import numpy as np
import pytest
import torch

from parallelpopgen_b200 import ConstantModel, Engine, constant_generations

pytestmark = pytest.mark.gpu


def _run(eng, model, seeds, gens):
    eng.begin_mse(model.mse_pops(), seed1=seeds[0], seed2=seeds[1], num_sites=2e7, compact_interval=25)
    eng.run(gens)
    return eng.read_state()


def test_concurrent_engines_match_sequential_runs():
    models = [ConstantModel(N=20000, mu=1e-9),
              ConstantModel(N=15000, mu=1e-9, h=0.3, s=ConstantModel.s_from_gamma(-10.0, 15000, 0.0))]
    seeds = [(11, 12), (13, 14)]
    gens = [constant_generations(m, 1, 600, 25) for m in models]
    with Engine() as e:
        want = [_run(e, models[k], seeds[k], gens[k]) for k in range(2)]
    streams = [torch.cuda.Stream() for _ in range(2)]
    engines = [Engine(stream=s.cuda_stream) for s in streams]
    got = [None, None]
    try:
        for _ in range(2):     # twice: the second pass reuses each engine's buffers
            def work(k):
                got[k] = _run(engines[k], models[k], seeds[k], gens[k])
            threads = [threading.Thread(target=work, args=(k,)) for k in range(2)]
            for t in threads:
                t.start()
            for t in threads:
                t.join()
            for k in range(2):
                (fw, iw), (fg, ig) = want[k], got[k]
                assert np.array_equal(fw.view(np.uint32), fg.view(np.uint32)), k
                assert np.array_equal(iw, ig), k
    finally:
        for e in engines:
            e.close()
