"""Autotuner: every launch candidate gives the same state bit for bit, and the tuned engine
reproduces the untuned run."""
from __future__ import annotations

import numpy as np
import pytest

from parallelpopgen_b200 import ConstantModel, Engine, constant_generations
from parallelpopgen_b200.autotune import LAUNCH_CANDIDATES, tune_batch_cadence, tune_launch

pytestmark = pytest.mark.gpu


def _run(e, model, gens, L):
    e.begin_mse(model.mse_pops(), seed1=7, seed2=9, num_sites=L, compact_interval=25)
    e.run(gens)
    return e.read_state()


def test_launch_candidates_agree(tmp_path, monkeypatch):
    monkeypatch.setenv("PARALLELPOPGEN_B200_CACHE", str(tmp_path / "c.json"))
    model = ConstantModel(N=20000, mu=1e-8, s=ConstantModel.s_from_gamma(-5.0, 20000, 0.1), h=0.3, F=0.1)
    L = 2e6
    gens = constant_generations(model, 1, 300, 25)
    with Engine() as e:
        ref_f, ref_ids = _run(e, model, gens, L)
        for cand in LAUNCH_CANDIDATES:
            e.set_tuning(**cand)
            f, ids = _run(e, model, gens, L)
            assert np.array_equal(f.view(np.uint32), ref_f.view(np.uint32)), cand
            assert np.array_equal(ids, ref_ids), cand
        e.set_tuning(0, 0, 1)
        res = tune_launch(e, model, L, generations=60)
        assert res["tuning"] in LAUNCH_CANDIDATES and len(res["trials"]) == len(LAUNCH_CANDIDATES)
        f, ids = _run(e, model, gens, L)
        assert np.array_equal(f.view(np.uint32), ref_f.view(np.uint32))
        again = tune_launch(e, model, L, generations=60)      # served from the cache
        assert again["tuning"] == res["tuning"]


def test_batch_cadence_choice(tmp_path, monkeypatch):
    monkeypatch.setenv("PARALLELPOPGEN_B200_CACHE", str(tmp_path / "c.json"))
    from parallelpopgen_b200 import replicate
    reps = [replicate(seed1=1 + r, seed2=2 + r, num_sites=1e6, mu=1e-8, F=0.0, h=0.5, s=0.0, N0=500 + 10 * r,
                      num_generations=200) for r in range(16)]
    with Engine() as e:
        res = tune_batch_cadence(e, reps, sample=8, max_generations=100, cadences=(10, 25))
    assert res["compact_interval"] in (10, 25) and len(res["trials"]) == 2
    assert all(r.num_generations == 200 for r in reps)      # the caller's replicates are untouched
