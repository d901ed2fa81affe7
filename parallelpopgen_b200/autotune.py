"""Autotuner for the engine's launch choices and the batched engine's compaction cadence.

Launch choices (`gf_tuning`: per-thread draws in lane order, warp-pooled draws or per-thread draws
grouped by sampler branch, or the normal approximation of a quad's four lanes first; resident drift
blocks per SM; window launches on/off) never change results; the tuner times a short calibration run per candidate
and keeps the fastest.  The compaction cadence of batched replicates does change results (the
Philox counter of a mutation is its slot, and compaction moves slots), so it is tuned only when the
caller asks for it -- batched statistics, where any cadence gives a valid, differently-seeded
sample -- and the chosen cadence is returned so the equivalent plain run can use it.

Results are cached per (device name, workload bucket) in a JSON file
(`$PARALLELPOPGEN_B200_CACHE`, default `~/.cache/parallelpopgen_b200/autotune.json`).
"""
from __future__ import annotations

import json
import math
import os
import time
from pathlib import Path

import numpy as np

from .engine import ConstantModel, Engine, constant_generations

LAUNCH_CANDIDATES = [
    {"draw_strategy": 0, "blocks_per_sm": 0, "windows": 1},
    {"draw_strategy": 0, "blocks_per_sm": 4, "windows": 1},
    {"draw_strategy": 1, "blocks_per_sm": 0, "windows": 1},
    {"draw_strategy": 2, "blocks_per_sm": 0, "windows": 1},
    {"draw_strategy": 3, "blocks_per_sm": 0, "windows": 1},
    {"draw_strategy": 4, "blocks_per_sm": 0, "windows": 1},
    {"draw_strategy": 0, "blocks_per_sm": 0, "windows": 0},
    {"draw_strategy": 2, "blocks_per_sm": 0, "windows": 0},
]
CADENCE_CANDIDATES = (10, 25, 50, 100)


def clone_replicate(rep):
    from ._capi import Replicate
    return Replicate(*[getattr(rep, f) for f, _ in Replicate._fields_])


def cache_path() -> Path:
    p = os.environ.get("PARALLELPOPGEN_B200_CACHE")
    return Path(p) if p else Path.home() / ".cache" / "parallelpopgen_b200" / "autotune.json"


def _load_cache() -> dict:
    try:
        return json.loads(cache_path().read_text())
    except Exception:
        return {}


def _store_cache(c: dict) -> None:
    try:
        cache_path().parent.mkdir(parents=True, exist_ok=True)
        cache_path().write_text(json.dumps(c, indent=1, sort_keys=True))
    except OSError:
        pass


def _device_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name()
    except Exception:
        return "cuda"


def bucket(num_mutations: float, populations: int = 1) -> str:
    """Workload bucket: mutation count rounded to a power of two, population count."""
    return f"M2^{int(round(math.log2(max(num_mutations, 1))))}:P{populations}"


def tune_launch(engine: Engine, model: ConstantModel, num_sites: float, generations: int = 100,
                compact_interval: int = 25, seeds=(1, 2), use_cache: bool = True) -> dict:
    """Pick the fastest launch choices for a single-population workload and apply them to `engine`.
    Returns {"tuning": ..., "mutation_generations_per_s": ..., "trials": [...]}."""
    gens = constant_generations(model, 1, generations, compact_interval)
    engine.begin_mse(model.mse_pops(), seed1=seeds[0], seed2=seeds[1], num_sites=num_sites,
                     compact_interval=compact_interval)
    key = f"{_device_name()}|launch|{bucket(engine.num_mutations(), model.P)}"
    cache = _load_cache()
    if use_cache and key in cache:
        engine.set_tuning(**cache[key]["tuning"])
        return cache[key]
    trials = []
    for cand in LAUNCH_CANDIDATES:
        engine.set_tuning(**cand)
        best = 0.0
        for _ in range(2):
            engine.begin_mse(model.mse_pops(), seed1=seeds[0], seed2=seeds[1], num_sites=num_sites,
                             compact_interval=compact_interval)
            engine.synchronize()
            t0 = time.perf_counter()
            engine.run(gens)
            engine.synchronize()
            dt = time.perf_counter() - t0
            best = max(best, engine.stats()["mutation_generations"] / dt)
        trials.append({"tuning": cand, "mutation_generations_per_s": best})
    win = max(trials, key=lambda t: t["mutation_generations_per_s"])
    engine.set_tuning(**win["tuning"])
    res = {"tuning": win["tuning"], "mutation_generations_per_s": win["mutation_generations_per_s"], "trials": trials}
    cache[key] = res
    _store_cache(cache)
    return res


def tune_batch_cadence(engine: Engine, reps: list, sample: int = 256, max_generations: int = 2000,
                       cadences=CADENCE_CANDIDATES, repeats: int = 2, use_cache: bool = True) -> dict:
    """Pick the compaction cadence that simulates a sample of batched replicates (each cut to at most
    `max_generations` generations) in the least time.  Mutation-generations are not the criterion:
    a slower cadence keeps lost and fixed slots longer, which inflates that count without simulating
    more.  Returns {"compact_interval": c, "trials": [...]}; the caller applies it to its replicates."""
    rng = np.random.default_rng(0)
    idx = rng.choice(len(reps), size=min(sample, len(reps)), replace=False)
    base = [clone_replicate(reps[i]) for i in idx]
    for r in base:
        r.num_generations = min(r.num_generations, max_generations)
    mean_n = float(np.mean([r.N0 for r in base]))
    key = f"{_device_name()}|cadence|N{int(round(math.log2(mean_n)))}|R{len(base)}|G{max_generations}"
    cache = _load_cache()
    if use_cache and key in cache:
        return cache[key]
    trials = []
    for c in cadences:
        for r in base:
            r.compact_interval = int(c)
        best = math.inf
        for _ in range(repeats):
            engine.batch_begin(base)
            engine.synchronize()
            t0 = time.perf_counter()
            engine.batch_run()
            engine.synchronize()
            best = min(best, time.perf_counter() - t0)
        trials.append({"compact_interval": int(c), "seconds": best,
                       "generations_per_s": sum(r.num_generations for r in base) / best})
    win = min(trials, key=lambda t: t["seconds"])
    res = {"compact_interval": win["compact_interval"], "trials": trials}
    cache[key] = res
    _store_cache(cache)
    return res
