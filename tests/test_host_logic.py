"""Host-side logic without a GPU: the per-generation records the engine receives, the compaction
schedule of run_sim, the float semantics of model parameters, and the benchmark's replica plumbing
across two processes (gloo)."""
from __future__ import annotations

import os
import socket
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

from parallelpopgen_b200 import ConstantModel, constant_generations
from parallelpopgen_b200._capi import GEN_DTYPE, MAX_POPULATIONS


def reference_schedule(start: int, final: int, ci: int) -> list[int]:
    """Compaction generations of the run_sim loop (go_fish_impl.cuh:643-706) without preserve/sample."""
    out, nxt = [], start + ci
    for g in range(start + 1, final + 1):
        if (g == nxt or g == final) and ci > 0:
            out.append(g)
            nxt = g + ci
    return out


@pytest.mark.parametrize("start,count,ci", [(0, 1000, 35), (0, 10000, 25), (20000, 1000, 100), (0, 7, 0), (5, 3, 1)])
def test_compaction_schedule_matches_run_sim(start, count, ci):
    g = constant_generations(ConstantModel(N=1000), start + 1, count, ci)
    got = list(g["generation"][g["compact"] == 1])
    assert got == reference_schedule(start, start + count, ci)
    assert list(g["generation"]) == list(range(start + 1, start + count + 1))


def test_generation_records_carry_the_model():
    m = ConstantModel(N=1234, F=0.25, h=0.3, s=-0.001, mu=2e-9, P=3, m=0.01)
    g = constant_generations(m, 1, 4, 2)
    assert g.dtype == GEN_DTYPE
    pops = g["pop"]
    assert (pops["Nchrom_e"][:, :3] == m.Nchrom_e).all() and (pops["Nchrom_e"][:, 3:] == 0).all()
    assert (pops["drift"][:, :3] == 1).all() and (pops["alive"][:, :3] == 1).all()
    assert np.allclose(pops["sel_intercept"][:, :3], -0.001)
    mig = g["migration"][0].reshape(MAX_POPULATIONS, MAX_POPULATIONS)
    assert mig[0, 0] == np.float32(1) - np.float32(2) * np.float32(0.01)
    assert mig[0, 1] == np.float32(0.01) and mig[3, 3] == 0


def test_effective_chromosomes_and_gamma_use_float_arithmetic():
    # 2 * N / (1 + F) in float, truncated (go_fish_impl.cuh:659)
    assert ConstantModel(N=200000).Nchrom_e == 400000
    assert ConstantModel(N=1000, F=1.0).Nchrom_e == 1000
    assert ConstantModel(N=10000, F=0.1).Nchrom_e == int(np.float32(20000) / np.float32(1.1))
    s = ConstantModel.s_from_gamma(-10.0, 200000, 0.0)
    assert s == float(np.float32(-10.0) / np.float32(400000.0))


def _free_port() -> int:
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _replica_worker(rank, world, port, out):
    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mx, sm = bench.reduce_over_ranks([10.0 + rank, 5.0 * rank], [1e9 * (rank + 1), 7.0], world)
        seeds = [(h["seed1"], h["seed2"]) for h in bench.build_halves(rank, 3)]
        out[rank] = (mx, sm, seeds)
    finally:
        dist.destroy_process_group()


def test_bench_replicas_reduce_over_two_gloo_ranks():
    world = 2
    port = _free_port()
    out = mp.Manager().dict()
    mp.spawn(_replica_worker, args=(world, port, out), nprocs=world, join=True)
    for r in range(world):
        mx, sm, _ = out[r]
        assert mx == [11.0, 5.0]          # max over ranks of the timings
        assert sm == [3e9, 14.0]          # total work of all replicas
    # every rank simulates its own replicas: no seed pair repeats across ranks or halves
    seeds = [s for r in range(world) for s in out[r][2]]
    assert len(set(seeds)) == len(seeds) == 4


def test_autotune_helpers(tmp_path, monkeypatch):
    """Cache location, workload buckets and replicate cloning of the autotuner (no GPU)."""
    from parallelpopgen_b200 import replicate
    from parallelpopgen_b200.autotune import bucket, cache_path, clone_replicate
    monkeypatch.setenv("PARALLELPOPGEN_B200_CACHE", str(tmp_path / "x.json"))
    assert cache_path() == tmp_path / "x.json"
    assert bucket(1 << 20) == "M2^20:P1" and bucket(0, 3) == "M2^0:P3"
    r = replicate(seed1=-5, seed2=6, num_sites=1e7, mu=1e-9, F=0.2, h=0.1, s=-1e-3, N0=1234, num_generations=99)
    c = clone_replicate(r)
    c.num_generations = 7
    assert r.num_generations == 99 and c.N0 == 1234 and c.seed1 == -5


def test_batched_bench_workload_draws():
    """The batched benchmark's parameter draws stay inside their stated ranges."""
    import bench
    reps = bench.batched_replicates(256, 1e4)
    N0 = np.array([r.N0 for r in reps])
    assert N0.min() >= 1000 and N0.max() <= 10000
    assert all(r.num_generations == 4 * r.N0 for r in reps)
    assert all(r.N_min == r.N0 // 10 and r.N_max == 10 * r.N0 for r in reps)
    assert all(0.0 <= r.F <= 0.5 and 0.0 <= r.h <= 1.0 for r in reps)


def test_multipop_bench_schedule():
    """The three-population benchmark's records: founding generations copy the parent, migration columns
    of existing populations sum to 1, segmented tables reproduce the continuous compaction schedule."""
    import bench
    from parallelpopgen_b200._capi import MAX_POPULATIONS as MP
    whole = bench.multipop_generations(1, 3000, last_generation=3000)
    parts = np.concatenate([bench.multipop_generations(a, min(a + 499, 3000), last_generation=3000)
                            for a in range(1, 3001, 500)])
    assert np.array_equal(whole["compact"], parts["compact"]) and np.array_equal(whole["preserve"], parts["preserve"])
    assert whole["preserve"][499] == 1 and whole["compact"][2999] == 1
    g1, g2000 = whole[0], whole[1999]
    assert g1["migration"][0 * MP + 1] == 1.0 and g2000["migration"][1 * MP + 2] == 1.0
    for G in (whole[10], whole[2500]):
        for to in range(3):
            if G["pop"]["drift"][to]:
                col = sum(float(G["migration"][f * MP + to]) for f in range(3))
                assert abs(col - 1.0) < 1e-6
    assert whole[0]["pop"]["drift"][2] == 0 and whole[2500]["pop"]["drift"][2] == 1
    assert whole[2500]["pop"]["F"][2] == np.float32(0.1)


def test_reference_arm_prints_the_contract_line():
    """`bench.py --impl reference` (the CPU restatement timed on the host cores) prints one JSON line
    with the metric, the `impl` tag, a `cpu_baseline` describing the run and an `e2e` with no copies."""
    import json
    import subprocess
    import sys
    root = Path(__file__).resolve().parents[1]
    out = subprocess.run([sys.executable, str(root / "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0"], capture_output=True, text=True, timeout=600, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == "mutation-generations/s"
    assert line["value"] > 0 and line["higher_is_better"] is True and line["steps"] == 1
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
