#!/usr/bin/env python
"""Headline benchmark: GO_Fish plain engine, mutation-generations/s on B200.

Workload (one "step"): the large single-population configuration -- N = 200,000 diploids
(Nchrom_e = 400,000), mu = 1e-9, h = 0.5, F = 0, L = 5e8 sites with purifying selection
gamma = 2Ns = -10 on half of the sites and the other half neutral, mutation-selection-equilibrium
start, 10,000 generations with compaction every 25, then the site frequency spectrum of a sample of
n = 1,000.  Selection acts per (population, generation, frequency) in GO_Fish, so "gamma on 50% of
new mutations" is run exactly as two independent simulations of L = 2.5e8 sites each (neutral and
gamma = -10), which is the same model under the Poisson-random-field independence of sites.  The two
simulations run concurrently, each on its own engine, stream and host thread.

Metric: mutation-generations/s = sum over generations of the mutation slots the drift pass updated,
divided by device time.  `value` times the whole step on the device (MSE initialization, every
generation, compactions, SFS) with the engine's inputs built on the host beforehand; `e2e` repeats the
step through the C ABI with host buffers, reading the final frequencies, mutation IDs and the SFS back
to host memory inside the timed region.  Synthetic inputs: the simulation draws its own state.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

--impl reference times the CPU restatement of the same per-generation update (oracle/, all host
threads) on a bounded sample of the same workload; the reference ships no CPU path of its own.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_IND = 200_000
MU = 1e-9
L_HALF = 2.5e8
GENS = 10_000
COMPACT = 25
SFS_N = 1000
GAMMA_SEL = -10.0
H = 0.5
SEED1, SEED2 = 0xBEEF, 0xDECAF
ALG_BYTES_PER_MUTGEN = 8  # P = 1: read one fp32 frequency, write one fp32 frequency
# Thread instructions per mutation-generation of the window kernel on this workload (ncu
# smsp__thread_inst_executed / mutation-generations of one launch: 73, neutral half),
# the figure behind the instruction-issue ceiling reported beside the HBM roofline.
THREAD_INSTR_PER_MUTGEN = 73
B200_SMS, SCHEDULERS_PER_SM = 148, 4


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                f = [x.strip() for x in out.stdout.strip().split(",")]
                if len(f) >= 7:
                    self.samples.append(f)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=6)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def reduce_over_ranks(max_values, sum_values, world: int, device=None):
    """Max over ranks of the timing values and sum over ranks of the work values (replicas: the only
    cross-rank exchange of this benchmark; the simulations themselves share nothing)."""
    if world <= 1:
        return [float(x) for x in max_values], [float(x) for x in sum_values]
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(max_values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    w = torch.tensor(list(sum_values), dtype=torch.float64, device=device)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return t.tolist(), w.tolist()


# ------------------------------------------------------------------------------------------------
# B200 arm
# ------------------------------------------------------------------------------------------------
def build_halves(rank: int, gens_per_sim: int = GENS):
    from parallelpopgen_b200 import ConstantModel, constant_generations
    halves = []
    for k, gamma in enumerate((0.0, GAMMA_SEL)):
        s = ConstantModel.s_from_gamma(gamma, N_IND, 0.0) if gamma else 0.0
        model = ConstantModel(N=N_IND, F=0.0, h=H, s=s, mu=MU)
        gens = constant_generations(model, 1, gens_per_sim, COMPACT)
        halves.append({"model": model, "gens": gens, "seed1": SEED1 + 2 * (2 * rank + k), "seed2": SEED2 - 2 * (2 * rank + k)})
    return halves


def run_b200(args, rank, local_rank, world):
    """The headline step: the two halves are independent simulations, run concurrently on two engines
    (one stream and one host thread each), so one simulation's compaction kernels and launch tails
    overlap the other's window kernels.  Time = CUDA events on a third stream that waits for both."""
    import threading

    import torch
    from parallelpopgen_b200 import Engine

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    main = torch.cuda.Stream(device=dev)
    streams = [torch.cuda.Stream(device=dev) for _ in range(2)]
    engines = [Engine(device=local_rank, stream=st.cuda_stream) for st in streams]
    halves = build_halves(rank, args.gens)
    Nc = halves[0]["model"].Nchrom_e
    d_sfs = [torch.empty(SFS_N, dtype=torch.float32, device=dev) for _ in range(2)]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # 256 MB > 126 MB L2
    reserve = 12_000_000

    def device_half(k, eng):
        """One half on device-resident state; returns its mutation-generations."""
        hv = halves[k]
        eng.begin_mse(hv["model"].mse_pops(), seed1=hv["seed1"], seed2=hv["seed2"], num_sites=L_HALF,
                      compact_interval=COMPACT, reserve=reserve)
        eng.run(hv["gens"])
        d_freq, stride, M = eng.device_state()
        eng.site_frequency_spectrum_device(d_freq, M, Nc, SFS_N, L_HALF, d_sfs[k].data_ptr())
        return eng.stats()["mutation_generations"]

    # page-locked host buffers for the e2e step's outputs (allocated once, outside the timed region)
    h_freq = [torch.empty(reserve, dtype=torch.float32, pin_memory=True).numpy() for _ in range(2)]
    h_ids = [torch.empty((reserve, 4), dtype=torch.int32, pin_memory=True).numpy() for _ in range(2)]

    def e2e_half(k, eng):
        """One half through the C ABI with host buffers: final frequencies, IDs and SFS to host."""
        hv = halves[k]
        eng.begin_mse(hv["model"].mse_pops(), seed1=hv["seed1"], seed2=hv["seed2"], num_sites=L_HALF,
                      compact_interval=COMPACT, reserve=reserve)
        eng.run(hv["gens"])
        M = eng.read_state_into(h_freq[k], h_ids[k])
        sfs = eng.site_frequency_spectrum(h_freq[k][:M], Nc, SFS_N, L_HALF)
        return (eng.stats()["mutation_generations"], hv["gens"].nbytes + 4 * M, 4 * M + 16 * M + sfs.nbytes)

    def concurrent(fn):
        """Both halves at once; returns (their results, elapsed ms by CUDA events)."""
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(main)
        for st in streams:
            st.wait_event(ev0)
        out = [None, None]

        def work(k):
            out[k] = fn(k, engines[k])

        threads = [threading.Thread(target=work, args=(k,)) for k in range(2)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        for st in streams:
            e = torch.cuda.Event()
            e.record(st)
            main.wait_event(e)
        ev1.record(main)
        ev1.synchronize()
        if any(o is None for o in out):
            raise RuntimeError("a half failed")
        return out, ev0.elapsed_time(ev1)

    def flush_l2():
        with torch.cuda.stream(main):
            flush.fill_(1.0)
        main.synchronize()

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        concurrent(device_half)
        concurrent(e2e_half)
    barrier()

    # ---- value: device time of the whole step ----
    launches0 = sum(e.stats()["kernel_launches"] for e in engines)
    times = []
    mg_total = 0.0
    with ClockSampler(local_rank) as clk:
        for _ in range(args.steps):
            flush_l2()
            out, ms = concurrent(device_half)
            times.append(ms)
            mg_total += sum(out)
    launches = (sum(e.stats()["kernel_launches"] for e in engines) - launches0) // max(args.steps, 1) * args.steps
    barrier()
    ms_total = float(sum(times))

    # ---- roofline: one more step, the halves one after the other on one engine, with every drift
    # launch bracketed by CUDA events (uncontended kernel times) ----
    flush_l2()
    eng = engines[0]
    eng.set_profiling(True)
    eng.read_profile()
    prof_mg = device_half(0, eng) + device_half(1, eng)
    prof = eng.read_profile()
    eng.set_profiling(False)
    barrier()

    # ---- e2e: host buffers, copies inside the timed region ----
    e2e_times, e2e_mg, h2d_b, d2h_b = [], 0.0, 0, 0
    for _ in range(args.steps):
        flush_l2()
        out, ms = concurrent(e2e_half)
        e2e_times.append(ms)
        e2e_mg += sum(o[0] for o in out)
        h2d_b, d2h_b = sum(o[1] for o in out), sum(o[2] for o in out)
    barrier()

    # max time over ranks, total work over ranks
    (ms_total, e2e_ms), (mg_all, e2e_mg_all) = reduce_over_ranks([ms_total, float(sum(e2e_times))],
                                                                 [mg_total, e2e_mg], world, device=dev)

    if rank != 0:
        return
    peak, peak_kind = measured_peaks()
    drift_bytes = ALG_BYTES_PER_MUTGEN * prof_mg  # the profiled step's drift launches
    achieved = drift_bytes / (prof["drift_ms"] * 1e-3) / 1e9 if prof["drift_ms"] > 0 else None
    traffic = None
    tfile = ROOT / "profiles" / "drift_traffic.json"
    if tfile.exists():
        try:
            traffic = json.loads(tfile.read_text()).get("dram_bytes_per_mutation_generation")
            if traffic is not None:
                traffic = traffic * prof_mg / max(prof["drift_launches"], 1)
        except Exception:
            traffic = None
    cpu = cpu_baseline_sample(threads=os.cpu_count() or 1) if not args.skip_cpu_baseline else None
    value = mg_all / (ms_total * 1e-3)
    line = {
        "metric": "mutation-generations/s",
        "value": value,
        "unit": "mutation-generations/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_total / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (the simulation draws its own mutation-selection-equilibrium start)",
        "config": {
            "workload": "GO_Fish single population N=200,000 (Nchrom_e 400,000), mu 1e-9, L=5e8 as 2 x 2.5e8 "
                        "(neutral + gamma=-10, h=0.5), MSE start, 10,000 generations, compact every 25, SFS n=1000",
            "generations_per_step": 2 * args.gens,
            "mutation_generations_per_step": mg_total / args.steps,
            "l2": "256 MB buffer written between steps (L2 is 126 MB); the 10-40 MB working set of one "
                  "simulation is L2-resident inside a step",
            "parallelism": f"replicas x{world} (independent seeds per rank, no collective); the two halves "
                           "run concurrently on two engines and streams",
        },
        "e2e": {
            "value": e2e_mg_all / (e2e_ms * 1e-3),
            "unit": "mutation-generations/s",
            "h2d_bytes_per_step": int(h2d_b),
            "d2h_bytes_per_step": int(d2h_b),
            "ms_per_step": e2e_ms / args.steps,
        },
        "gpu_launches": int(launches),
        "roofline": {
            "bound": "hbm",
            "kernel": "window_kernel (every generation of a compaction window per launch: selection, drift, "
                      "births, compaction flags); its segmented scan and scatter are compact_ms_per_step",
            "achieved": achieved,
            "peak": peak,
            "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None,
            "peak_source": peak_kind,
            "traffic": traffic,
            "drift_ms_per_step": prof["drift_ms"],
            "drift_launches_per_step": prof["drift_launches"],
            "drift_us_per_launch": 1e3 * prof["drift_ms"] / max(prof["drift_launches"], 1),
            "compact_ms_per_step": prof["compact_ms"],
            "bytes_per_mutation_generation": ALG_BYTES_PER_MUTGEN,
        },
        "cpu_baseline": cpu,
        "clocks": clk.summary(),
    }
    # over the whole timed step (MSE start, windows, compactions, SFS, both halves at once)
    line["roofline"]["step"] = {"achieved": ALG_BYTES_PER_MUTGEN * value / 1e9, "unit": "GB/s",
                                "frac": ALG_BYTES_PER_MUTGEN * value / 1e9 / peak}
    # the kernel is issue-bound: its rate against the instruction-issue ceiling at full warps
    mhz = line["clocks"].get("sm_mhz") or 1965.0
    issue_ceiling = B200_SMS * SCHEDULERS_PER_SM * mhz * 1e6 * 32 / THREAD_INSTR_PER_MUTGEN
    if achieved:
        line["roofline"]["issue"] = {
            "thread_instructions_per_mutation_generation": THREAD_INSTR_PER_MUTGEN,
            "ceiling": issue_ceiling, "unit": "mutation-generations/s",
            "frac": achieved * 1e9 / ALG_BYTES_PER_MUTGEN / issue_ceiling,
        }
    if world == 1 and not args.no_workloads:
        for e in engines:
            e.close()
        del flush
        torch.cuda.empty_cache()
        line["workloads"] = extra_workloads()
    print(json.dumps(line), flush=True)


def extra_workloads() -> dict:
    """The other measured configurations, each with its own fixed step counts (independent of --steps):
    batched ragged replicates over the full N0 range with the looped plain engine beside them, the
    three-population model, and surrogate inference."""
    out = {}
    t0 = time.perf_counter()
    b = measure_batched(4096, 1e5, plain_sample=8, steps=1, warmup=1, profile=False)
    b["wall_s"] = time.perf_counter() - t0
    out["batched"] = b
    t0 = time.perf_counter()
    m = measure_multipop(MP_GENS, steps=2, warmup=1)
    m["wall_s"] = time.perf_counter() - t0
    out["multipop"] = m
    out["surrogate_forward"] = measure_surrogate_forward(steps=50, warmup=10)
    return out


# ------------------------------------------------------------------------------------------------
# CPU restatement (oracle) -- the reference arm and the cpu_baseline
# ------------------------------------------------------------------------------------------------
def equilibrium_state(rng, Nc, L, mu):
    i = np.arange(1, Nc)
    counts = rng.poisson(2 * mu * L / (i / Nc))
    return np.repeat((i.astype(np.float32) / np.float32(Nc)).astype(np.float32), counts)


def cpu_sample(threads: int, gens: int, seed: int = 1):
    """`gens` generations of each half (neutral, then gamma = -10 with h = 0.5) of the headline workload
    from a synthetic neutral-equilibrium state of ~2.7 M mutations; returns (mutation-generations, s)."""
    import oracle.oracle as orc  # CPU restatement: the timed baseline, never the product
    from parallelpopgen_b200 import ConstantModel
    Nc = 2 * N_IND
    x = equilibrium_state(np.random.default_rng(seed), Nc, L_HALF, MU)
    mg_all, dt_all = 0.0, 0.0
    for sel in (0.0, ConstantModel.s_from_gamma(GAMMA_SEL, N_IND, 0.0)):
        t0 = time.perf_counter()
        _, _, mg = orc.run_single(x, first_gen=0, num_gens=gens, Nc=Nc, F=0.0, h=H, s=sel, mu=MU,
                                  num_sites=L_HALF, seed1=SEED1, seed2=SEED2, compact_interval=COMPACT,
                                  capacity=2 * len(x) + 4_000_000, threads=threads)
        dt_all += time.perf_counter() - t0
        mg_all += mg
    return mg_all, dt_all


def cpu_baseline_sample(threads: int, gens: int = 40, serial_gens: int = 4):
    """The CPU restatement on all host threads (the baseline) and, on a shorter sample, on one thread
    (about 20 core-seconds of work in all)."""
    mg, dt = cpu_sample(threads, gens)
    smg, sdt = cpu_sample(1, serial_gens)
    return {"value": mg / dt, "unit": "mutation-generations/s", "cores": threads, "kind": "port",
            "sample": f"{gens} generations of each half (neutral, and gamma = -10 with h = 0.5; Nchrom_e 400,000, "
                      f"L 2.5e8, ~2.7M mutations) from a synthetic equilibrium state; {dt:.1f} s wall on "
                      f"{threads} threads",
            "serial": {"value": smg / sdt, "cores": 1,
                       "sample": f"{serial_gens} generations of each half on one thread; {sdt:.1f} s"}}


def run_reference(args, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    gens = 10
    for _ in range(args.warmup):
        cpu_sample(threads, 1)
    total_mg, total_s = 0.0, 0.0
    for k in range(args.steps):
        mg, dt = cpu_sample(threads, gens, seed=k + 1)
        total_mg += mg
        total_s += dt
    v = total_mg / total_s
    print(json.dumps({
        "metric": "mutation-generations/s", "value": v, "unit": "mutation-generations/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_s * 1e3 / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic", "impl": "reference",
        "config": {"workload": "GO_Fish single population N=200,000 (Nchrom_e 400,000), mu 1e-9, L=5e8 as 2 x 2.5e8 "
                               "(neutral + gamma=-10, h=0.5), MSE start, 10,000 generations, compact every 25, "
                               "SFS n=1000", "parallelism": "CPU threads"},
        "cpu_baseline": {"value": v, "unit": "mutation-generations/s", "cores": threads, "kind": "port",
                         "sample": f"{gens} generations of each half (neutral, gamma = -10) per step from a "
                                   "~2.7M-mutation equilibrium state, CPU restatement of the reference's "
                                   "per-generation update (the reference ships no CPU implementation of this path)"},
        "e2e": {"value": v, "unit": "mutation-generations/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ------------------------------------------------------------------------------------------------
# batched replicates: simulations/s of one batched launch sequence vs the same replicates looped
# through the plain engine
# ------------------------------------------------------------------------------------------------
def batched_replicates(R: int, n_max: float, seed: int = 2024):
    """Seeded parameter draws of the batched workload: N0 log-uniform in [1e3, n_max], gamma uniform in
    [-100, 10], h in [0, 1], F in [0, 0.5], exponential growth r in [-0.001, 0.01] clamped to
    [N0/10, 10 N0], mu 1e-9, L 1e7, 4 N0 generations, seeds (0xbeef + 2r, 0xdecaf - 2r)."""
    from parallelpopgen_b200 import ConstantModel, replicate
    rng = np.random.default_rng(seed)
    reps = []
    for r in range(R):
        N0 = int(round(np.exp(rng.uniform(np.log(1e3), np.log(n_max)))))
        gamma = float(rng.uniform(-100.0, 10.0))
        h = float(rng.uniform(0.0, 1.0))
        F = float(rng.uniform(0.0, 0.5))
        rate = float(rng.uniform(-0.001, 0.01))
        reps.append(replicate(seed1=0xBEEF + 2 * r, seed2=0xDECAF - 2 * r, num_sites=1e7, mu=1e-9, F=F, h=h,
                              s=ConstantModel.s_from_gamma(gamma, N0, F), N0=N0, growth_rate=rate,
                              N_min=max(N0 // 10, 1), N_max=10 * N0, num_generations=4 * N0,
                              compact_interval=25))
    return reps


def run_batched(args):
    print(json.dumps(measure_batched(args.replicates, args.n_max, args.plain_sample, args.steps, args.warmup)),
          flush=True)


def measure_batched(replicates: int, n_max: float, plain_sample: int, steps: int, warmup: int,
                    profile: bool = True) -> dict:
    import torch
    from parallelpopgen_b200 import Engine, replicate_mse_pops, replicate_plain_generations, replicate_population
    from parallelpopgen_b200.autotune import tune_batch_cadence

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    eng = Engine(device=0, stream=stream.cuda_stream)
    reps = batched_replicates(replicates, n_max)
    tuned = tune_batch_cadence(eng, reps, use_cache=False)
    for r in reps:
        r.compact_interval = tuned["compact_interval"]
    n = 100

    def batch_step():
        eng.batch_begin(reps)
        eng.batch_run()
        sfs = eng.batch_sfs(n, len(reps))
        return eng.batch_stats(), sfs

    for _ in range(warmup):
        batch_step()
    times, st = [], None
    with ClockSampler(0) as clk:
        for _ in range(steps):
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            st, sfs = batch_step()
            ev1.record(stream)
            ev1.synchronize()
            times.append(ev0.elapsed_time(ev1) * 1e-3)
    batch_s = float(np.mean(times))
    phases, prof = None, {"drift_ms": None, "drift_launches": None}
    if profile:
        # one more batch with the window launches bracketed by CUDA events (device time of the drift
        # work) and host wall-clock phases, the device synchronised between them
        eng.set_profiling(True)
        eng.read_profile()
        ph0 = time.perf_counter()
        eng.batch_begin(reps)
        eng.synchronize()
        ph1 = time.perf_counter()
        eng.batch_run()                      # returns after reading the counts back
        ph2 = time.perf_counter()
        eng.batch_sfs(n, len(reps))
        ph3 = time.perf_counter()
        phases = {"begin": 1e3 * (ph1 - ph0), "run": 1e3 * (ph2 - ph1), "sfs": 1e3 * (ph3 - ph2)}
        prof = eng.read_profile()
        eng.set_profiling(False)
    # the same replicates, one plain engine run each (a random sample, timed engine calls only)
    rng = np.random.default_rng(7)
    sample = rng.choice(len(reps), size=min(plain_sample, len(reps)), replace=False)
    prepared = [(reps[i], replicate_mse_pops(reps[i]), replicate_plain_generations(reps[i])) for i in sample]
    d_sfs = torch.empty(n, dtype=torch.float32, device="cuda")
    eng = Engine(device=0, stream=stream.cuda_stream)     # a fresh engine: no batch state alongside
    plain_s = 0.0
    for rep, pops, gens in prepared:
        Nc = int(np.float32(2 * replicate_population(rep, rep.num_generations)) /
                 np.float32(np.float32(1) + np.float32(rep.F)))
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        eng.begin_mse(pops, seed1=rep.seed1, seed2=rep.seed2, num_sites=rep.num_sites,
                      compact_interval=rep.compact_interval)
        eng.run(gens)
        d_freq, _, M = eng.device_state()
        eng.site_frequency_spectrum_device(d_freq, M, Nc, n, rep.num_sites, d_sfs.data_ptr())
        ev1.record(stream)
        ev1.synchronize()
        plain_s += ev0.elapsed_time(ev1) * 1e-3
    plain_rate = len(prepared) / plain_s
    value = len(reps) / batch_s
    return {
        "metric": "simulations/s (batched ragged replicates)", "value": value, "unit": "simulations/s",
        "n_gpus": 1, "steps": steps, "warmup": warmup, "ms_per_step": batch_s * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{len(reps)} single-population replicates: N0 log-uniform [1e3, {n_max:g}], "
                               "gamma U[-100, 10], h U[0, 1], F U[0, 0.5], growth r U[-0.001, 0.01] clamped to "
                               "[N0/10, 10 N0], mu 1e-9, L 1e7, 4 N0 generations, MSE start, SFS n=100",
                   "compact_interval": tuned["compact_interval"], "cadence_trials": tuned["trials"],
                   "host_threads": os.cpu_count()},
        "mutation_generations_per_step": st["mutation_generations"],
        "mutation_generations_per_s": st["mutation_generations"] / batch_s,
        "super_steps": st["super_steps"],
        "record_wait_ms_per_batch": st["record_wait_ms"], "record_producers": st["record_producers"],
        "phases_ms_profiled_batch": phases,
        "window_ms_per_step": prof["drift_ms"], "window_launches_per_step": prof["drift_launches"],
        "looped_plain": {"value": plain_rate, "unit": "simulations/s", "sample": len(prepared),
                         "speedup_batched_over_looped": value / plain_rate},
        "clocks": clk.summary(),
    }


# ------------------------------------------------------------------------------------------------
# surrogate: train on batched-simulator spectra, evaluate against held-out simulator means, and compare
# SFS queries/s with the simulator at matched error
# ------------------------------------------------------------------------------------------------
def run_surrogate(args):
    import torch
    from parallelpopgen_b200 import Engine
    from parallelpopgen_b200 import surrogate as sg

    torch.cuda.set_device(0)
    if args.infer_only:
        return surrogate_inference_only(args)
    eng = Engine(device=0)
    cached = None
    if args.data_cache and os.path.exists(args.data_cache):
        cached = np.load(args.data_cache)
        if (len(cached["ptrain"]) != args.train_draws or len(cached["peval"]) != args.eval_draws
                or "ref_var" not in cached):
            cached = None
    if cached is not None:
        ptrain, train_sfs, peval, ref = cached["ptrain"], cached["train_sfs"], cached["peval"], cached["ref"]
        ref_var = cached["ref_var"]
        t_data = float(cached["t_data"]) if "t_data" in cached else None
    else:
        t0 = time.perf_counter()
        ptrain = sg.draw_parameters(args.train_draws, seed=101)
        train_sfs = sg.simulate_spectra(eng, ptrain, reps=16, seed=1 << 20)
        eng.synchronize()
        t_data = time.perf_counter() - t0
        peval = sg.draw_parameters(args.eval_draws, seed=202)
        # reference spectra: 64-replicate means, with their per-bin variance
        ref, ref_var = sg.simulate_spectra(eng, peval, reps=64, seed=1 << 28, with_variance=True)
        if args.data_cache:
            np.savez(args.data_cache, ptrain=ptrain, train_sfs=train_sfs.astype(np.float32), peval=peval,
                     ref=ref, ref_var=ref_var, t_data=t_data)
    # simulator throughput on the training distribution: 512 draws x 16 replicates, timed on its own
    # (after one untimed run, which sizes the engine's buffers)
    sg.simulate_spectra(eng, ptrain[:512], reps=16, seed=(1 << 29) + 3)
    eng.synchronize()
    t0 = time.perf_counter()
    sg.simulate_spectra(eng, ptrain[:512], reps=16, seed=(1 << 29) + 7)
    eng.synchronize()
    sims_per_s = 512 * 16 / (time.perf_counter() - t0)
    indep = sg.simulate_spectra(eng, peval, reps=16, seed=(1 << 28) + (1 << 26))   # independent replicates

    X = torch.from_numpy(sg.encode(ptrain)).cuda()
    t_raw = sg.spectra_to_targets(train_sfs)
    scale = sg.TargetScale.fit(t_raw)
    T = torch.from_numpy(scale.apply(t_raw)).cuda()
    mlp = sg.Mlp(capacity=max(32768, args.batch), lr=args.lr, weight_decay=args.weight_decay)
    mlp.set_params(sg.init_params(0))
    tr = sg.train(mlp, X, T, steps=args.train_steps, batch=args.batch, lr=args.lr, log_every=5000)

    surr = sg.Surrogate(mlp, eng, scale=scale)
    pred = surr.predict(peval)
    err, used = sg.median_relative_error(pred, ref)
    report = sg.error_report(pred, ref, ref_var, reps=64)
    # queries from the batched workload's distribution (N0 up to 1e5): the share the network answers
    queries = sg.draw_query_parameters(65536, seed=505)
    coverage = float(sg.in_support(queries).mean())
    # the simulator's own error with k replicates per query (k = 16 from independent seeds; fewer from
    # subsets of them are not available without rerunning, so k < 16 are simulated separately)
    sim_err = {16: sg.median_relative_error(indep / indep.sum(axis=1, keepdims=True), ref)[0]}
    for k in (1, 4):
        sk = sg.simulate_spectra(eng, peval, reps=k, seed=(1 << 28) + (1 << 27) + k)
        sim_err[k] = sg.median_relative_error(sk / sk.sum(axis=1, keepdims=True), ref)[0]
    # replicates the simulator needs for the surrogate's error: the simulator's error is sampling noise,
    # falling as 1/sqrt(k), so interpolate from the measured point nearest below the surrogate's error
    # (never fewer than one replicate per query)
    ks = sorted(sim_err)
    below = [k for k in ks if sim_err[k] >= err]
    k0 = below[-1] if below else ks[0]
    k_match = max(1.0, k0 * (sim_err[k0] / err) ** 2)
    sim_queries_per_s = sims_per_s / k_match

    # inference throughput: device-resident batches of B queries
    def time_forward(B, iters):
        xq = torch.from_numpy(sg.encode(sg.draw_parameters(B, seed=303))).cuda()
        yq = torch.empty((B, 99), dtype=torch.float32, device="cuda")
        for _ in range(10):
            mlp.forward_ptr(xq.data_ptr(), B, yq.data_ptr())
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(iters):
            mlp.forward_ptr(xq.data_ptr(), B, yq.data_ptr())
        ev1.record()
        ev1.synchronize()
        return ev0.elapsed_time(ev1) * 1e-3 / iters

    fwd_small = time_forward(4096, 200)
    B = 32768
    fwd_s = time_forward(B, 100)
    q_per_s = B / fwd_s
    flops = 2.0 * B * (6 * 512 + 3 * 512 * 512 + 512 * 99)
    # end to end through the query API (host parameters in, host spectra out)
    hostq = sg.draw_parameters(4096, seed=404)
    surr.query(hostq)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for _ in range(5):
        surr.query(hostq)
    e2e_q_per_s = 5 * len(hostq) / (time.perf_counter() - t1)
    peak, peak_kind = tensor_peak()
    tf = flops / fwd_s / 1e12
    print(json.dumps({
        "metric": "SFS queries/s (surrogate)", "value": q_per_s, "unit": "queries/s", "n_gpus": 1,
        "higher_is_better": True, "dtype": "bf16 (fp32 accumulate)", "data": "synthetic (batched simulator)",
        "config": {"workload": "6->512x4->99 GELU MLP, per-bin standardised log-spectrum targets; train " f"{args.train_draws} draws x 16 replicates, "
                               f"eval {args.eval_draws} draws x 64 replicates; support: logN [log 1e3, log 1e4], "
                               "gamma [-100, 10], h [0, 1], F [0, 0.5], r [-0.001, 0.01], T [0.05, 1]; "
                               f"theta {sg.THETA:g}, L {sg.NUM_SITES:g}, n 100",
                   "train_steps": args.train_steps, "batch": args.batch, "lr": args.lr,
                   "weight_decay": args.weight_decay, "inference_batch": B},
        "median_rel_error": err, "bins_used": used, "error": report,
        "queries_in_support": coverage,
        "queries_routed_to_simulator": 1.0 - coverage,
        "query_distribution": "log N0 U[log 1e3, log 1e5], the other parameters over the support",
        "simulator_median_rel_error": {str(k): v for k, v in sim_err.items()},
        "matched_replicates": k_match,
        "simulator_sims_per_s": sims_per_s,
        "simulator_queries_per_s_at_matched_error": sim_queries_per_s,
        "speedup_at_matched_error": q_per_s / sim_queries_per_s,
        "e2e": {"value": e2e_q_per_s, "unit": "queries/s", "path": "Surrogate.query (host in, host out)"},
        "train": {"seconds": tr.seconds, "steps": tr.steps, "ms_per_step": tr.seconds / tr.steps * 1e3,
                  "losses": tr.losses, "data_seconds": t_data},
        "roofline": {"bound": "tensor", "achieved": tf, "peak": peak, "peak_kind": peak_kind,
                     "unit": "TFLOP/s", "frac": tf / peak, "forward_us": fwd_s * 1e6,
                     "forward_us_4096": fwd_small * 1e6, "queries_per_s_4096": 4096 / fwd_small},
    }), flush=True)


def surrogate_inference_only(args):
    """Forward passes of the surrogate network with initial weights (throughput does not depend on them):
    the tensor-core kernels alone, for profiling."""
    print(json.dumps(measure_surrogate_forward(args.steps, args.warmup)), flush=True)


def measure_surrogate_forward(steps: int, warmup: int, B: int = 32768) -> dict:
    import torch
    from parallelpopgen_b200 import surrogate as sg
    mlp = sg.Mlp(capacity=B)
    mlp.set_params(sg.init_params(0))
    xq = torch.from_numpy(sg.encode(sg.draw_parameters(B, seed=303))).cuda()
    yq = torch.empty((B, 99), dtype=torch.float32, device="cuda")
    def timed(fused: int) -> float:
        assert mlp.lib.gf_mlp_set_fused_inference(mlp.h, fused) == 0
        for _ in range(warmup):
            mlp.forward_ptr(xq.data_ptr(), B, yq.data_ptr())
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(steps):
            mlp.forward_ptr(xq.data_ptr(), B, yq.data_ptr())
        ev1.record()
        ev1.synchronize()
        mlp.check()
        return ev0.elapsed_time(ev1) * 1e-3 / steps

    layered_s = timed(0)   # one tensor-core GEMM per layer, for comparison
    fwd_s = timed(1)       # the fused five-layer kernel (the default inference path)
    flop_per_query = 2.0 * (6 * 512 + 3 * 512 * 512 + 512 * 99)
    flops = flop_per_query * B
    peak, kind = tensor_peak()
    tf = flops / fwd_s / 1e12
    # the same kernel on a batch of exactly two 128-row tiles per SM: at 32,768 queries (256 tiles on
    # 148 SMs) 108 CTAs run two tiles and 40 run one, so the pass lasts as long as two tiles
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    B2 = 2 * 128 * sms
    mlp2 = sg.Mlp(capacity=B2)
    mlp2.set_params(sg.init_params(0))
    x2 = torch.from_numpy(sg.encode(sg.draw_parameters(B2, seed=305))).cuda()
    y2 = torch.empty((B2, 99), dtype=torch.float32, device="cuda")
    for _ in range(warmup):
        mlp2.forward_ptr(x2.data_ptr(), B2, y2.data_ptr())
    b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b0.record()
    for _ in range(steps):
        mlp2.forward_ptr(x2.data_ptr(), B2, y2.data_ptr())
    b1.record()
    b1.synchronize()
    mlp2.check()
    full_s = b0.elapsed_time(b1) * 1e-3 / steps
    full_tf = flop_per_query * B2 / full_s / 1e12
    # end to end: host parameters in, host spectra out, through the network's pointer API
    hx = torch.from_numpy(sg.encode(sg.draw_parameters(B, seed=304))).pin_memory()
    hy = torch.empty((B, 99), dtype=torch.float32).pin_memory()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        xq.copy_(hx, non_blocking=True)
        mlp.forward_ptr(xq.data_ptr(), B, yq.data_ptr())
        hy.copy_(yq, non_blocking=True)
    e1.record()
    e1.synchronize()
    e2e_s = e0.elapsed_time(e1) * 1e-3 / steps
    return {"metric": "SFS queries/s (surrogate forward)", "value": B / fwd_s, "unit": "queries/s",
            "n_gpus": 1, "steps": steps, "warmup": warmup, "batch": B, "dtype": "bf16 (fp32 accumulate)",
            "e2e": {"value": B / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": int(hx.numel() * 4),
                    "d2h_bytes_per_step": int(hy.numel() * 4)},
            "roofline": {"bound": "tensor", "achieved": tf, "peak": peak, "peak_kind": kind,
                         "unit": "TFLOP/s", "frac": tf / peak, "forward_us": fwd_s * 1e6,
                         "kernel": "fused_forward_kernel (five layers per 128-row tile, activations on chip)",
                         "layered_forward_us": layered_s * 1e6,
                         "two_tiles_per_sm": {"batch": B2, "forward_us": full_s * 1e6, "queries_per_s": B2 / full_s,
                                              "achieved": full_tf, "frac": full_tf / peak}}}


# ------------------------------------------------------------------------------------------------
# multi-population demography (multi-population window kernel, P = 3)
# ------------------------------------------------------------------------------------------------
MP_GENS, MP_L, MP_MU, MP_M, MP_H = 5000, 2e8, 1e-9, 1e-4, 0.3
MP_N0, MP_R, MP_CAPS, MP_FOUND = 10_000, 0.005, (100_000, 250_000, 500_000), (0, 1, 2000)
MP_SHIFT, MP_GAMMA = 3000, (-5.0, 2.0)


def multipop_size(pop: int, g: int) -> int:
    """Population `pop` exists from generation MP_FOUND[pop] (the ancestral population 0 from the start),
    starts at N = 1e4 and grows exponentially at r = 0.005 to its cap (1e5, 2.5e5, 5e5)."""
    f = MP_FOUND[pop]
    if pop > 0 and g < max(f, 1):
        return 0
    t = g - f
    return int(min(MP_CAPS[pop], round(MP_N0 * np.exp(MP_R * t))))


def multipop_generations(first: int, last: int, sample_every: int = 500, compact_interval: int = 35,
                         last_generation: int = MP_GENS):
    """gf_generation records of generations first..last, packed the way GO_Fish::run_sim packs them:
    population 1 founded from population 0 at generation 1, population 2 from population 1 at 2000
    (migration proportion 1 from the parent in the founding generation), symmetric migration 1e-4 among
    existing populations otherwise, selection gamma -5 then +2 from generation 3000 (s = gamma / 2e4,
    selection_constant of the ancestral size), h 0.3, inbreeding F 0.1 in population 2, mu 1e-9, L 2e8,
    a time sample (preserve + compaction) every 500 generations."""
    from parallelpopgen_b200._capi import GEN_DTYPE, MAX_POPULATIONS as MP
    gens = np.zeros(last - first + 1, dtype=GEN_DTYPE)
    # the reference's schedule: every compact_interval generations from the start, restarted at each
    # compaction, plus the final generation and every time sample
    next_compact = compact_interval
    for g in range(1, first):
        if g == next_compact or g % sample_every == 0:
            next_compact = g + compact_interval
    for i, g in enumerate(range(first, last + 1)):
        G = gens[i]
        G["generation"] = g
        exists = [multipop_size(p, g) > 0 for p in range(3)]
        gamma = MP_GAMMA[0] if g < MP_SHIFT else MP_GAMMA[1]
        for p in range(3):
            N = multipop_size(p, g)
            F = 0.1 if p == 2 else 0.0
            pp = G["pop"][p]
            pp["drift"] = 1 if N > 0 else 0
            pp["Nchrom_e"] = int(np.float32(2 * N) / np.float32(1 + np.float32(F))) if N > 0 else 0
            pp["alive"] = pp["mutate"] = 1 if N > 0 else 0
            pp["mu"], pp["F"], pp["h"] = MP_MU, F, MP_H
            pp["sel_slope"], pp["sel_intercept"] = 0.0, np.float32(gamma) / np.float32(2 * MP_N0)
        mig = G["migration"]
        n_exist = sum(exists)
        for to in range(3):
            if not exists[to]:
                continue
            founder = {1: 0, 2: 1}.get(to)
            if to > 0 and g == max(MP_FOUND[to], 1):
                mig[founder * MP + to] = 1.0               # the founding generation copies the parent
                continue
            for frm in range(3):
                if exists[frm]:
                    mig[frm * MP + to] = (1.0 - (n_exist - 1) * MP_M) if frm == to else MP_M
        preserve = g % sample_every == 0
        compact = g == next_compact or g == last_generation or preserve
        G["compact"] = 1 if compact else 0
        G["preserve"] = 1 if (compact and preserve) else 0
        if compact:
            next_compact = g + compact_interval
    return gens


def run_multipop(args):
    print(json.dumps(measure_multipop(args.mp_gens, args.steps, args.warmup)), flush=True)


def measure_multipop(total: int, steps: int, warmup: int) -> dict:
    import torch
    from parallelpopgen_b200 import Engine
    from parallelpopgen_b200._capi import MSE_DTYPE
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    eng = Engine(device=0, stream=stream.cuda_stream)
    segments = [multipop_generations(a, min(a + 499, total), last_generation=total) for a in range(1, total + 1, 500)]
    pops = np.zeros(3, dtype=MSE_DTYPE)
    pops[0] = (MP_N0, 2 * MP_N0, MP_MU, 0.0, MP_H, 0.0, np.float32(MP_GAMMA[0]) / np.float32(2 * MP_N0))
    reserve = 48_000_000     # time samples preserve their survivors: the state grows past 25 M slots
    # two page-locked sample buffers, used in turn: a sample's copy runs while the next segment does
    bufs = [(torch.empty(3 * reserve, dtype=torch.float32, pin_memory=True).numpy(),
             torch.empty((reserve, 4), dtype=torch.int32, pin_memory=True).numpy()) for _ in range(2)]
    n = 200

    def step(samples: bool):
        eng.begin_mse(pops, seed1=SEED1, seed2=SEED2, num_sites=MP_L, compact_interval=35, reserve=reserve)
        d2h, M, last = 0, 0, None
        for k, seg in enumerate(segments):
            eng.run(seg)
            if samples:     # the time sample taken at the segment's last generation (rows packed [3][M])
                if last is not None:
                    M, nbytes = eng.sample_wait(with_bytes=True)
                    d2h += nbytes
                last = bufs[k % 2]
                eng.sample_begin(*last)
        if samples:
            M, nbytes = eng.sample_wait(with_bytes=True)
            d2h += nbytes
        return eng.stats()["mutation_generations"], d2h, M, (last[0] if last is not None else None)

    for _ in range(warmup):
        step(False)
    step(True)   # untimed: the first time sample sets up the engine's sample scratch and copy stream
    times, mg = [], 0.0
    with ClockSampler(0) as clk:
        for _ in range(steps):
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            m, _, _, _ = step(False)
            ev1.record(stream)
            ev1.synchronize()
            times.append(ev0.elapsed_time(ev1))
            mg += m
    e2e_t, e2e_mg, d2h = [], 0.0, 0
    for _ in range(steps):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        m, d2h, M, h_freq = step(True)
        # the final sample's SFS of a sample of 200 in each population
        for p in range(3):
            Nc = int(np.float32(2 * multipop_size(p, total)) / np.float32(1 + np.float32(0.1 if p == 2 else 0.0)))
            if Nc > n:          # populations founded later than a shortened run's end are skipped
                eng.site_frequency_spectrum(h_freq[p * M:(p + 1) * M], Nc, n, MP_L)
        ev1.record(stream)
        ev1.synchronize()
        e2e_t.append(ev0.elapsed_time(ev1))
        e2e_mg += m
    value = mg / (sum(times) * 1e-3)
    return {
        "metric": "mutation-generations/s (multi-population)", "value": value, "unit": "mutation-generations/s",
        "n_gpus": 1, "steps": steps, "warmup": warmup, "ms_per_step": sum(times) / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "3 populations: ancestral N=1e4 (MSE start), population 1 founded at generation 1, "
                               "population 2 at 2000, exponential growth r=0.005 to 1e5 / 2.5e5 / 5e5, symmetric "
                               "migration 1e-4, gamma -5 -> +2 at 3000, h 0.3, F 0.1 in population 2, mu 1e-9, "
                               "L 2e8, 5000 generations, compaction every 35 and at every time sample (500)",
                   "kernel": "window_mp_kernel (P = 3: all generations of a compaction window per launch)"},
        "mutation_generations_per_step": mg / steps,
        "e2e": {"value": e2e_mg / (sum(e2e_t) * 1e-3), "unit": "mutation-generations/s",
                "path": "10 time samples copied into page-locked buffers while the next segment runs "
                        "(gf_sim_sample_begin / _wait), SFS n=200 of each population",
                "h2d_bytes_per_step": int(sum(seg.nbytes for seg in segments)), "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "bytes_per_mutation_generation": 48,
                     "achieved": 48 * value / 1e9, "unit": "GB/s", "peak": measured_peaks()[0],
                     "frac": 48 * value / 1e9 / measured_peaks()[0]},
        "clocks": clk.summary(),
    }


def tensor_peak():
    """(bf16 dense TFLOP/s, "measured" | "fallback") for a kernel timed on its own (burst figure)."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        if "bf16_tflops" in d:
            return float(d["bf16_tflops"]), "measured"
    return 1590.0, "fallback"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--skip-cpu-baseline", action="store_true")
    ap.add_argument("--no-workloads", action="store_true",
                    help="plain workload only: leave out the batched, multi-population and surrogate sub-objects")
    ap.add_argument("--workload", default="plain", choices=["plain", "batched", "surrogate", "multipop"],
                    help="plain: the headline single-population workload; batched: batched ragged replicates; "
                         "surrogate: the SFS surrogate network against the simulator")
    ap.add_argument("--mp-gens", type=int, default=MP_GENS, help="multipop workload: generations per run")
    ap.add_argument("--train-draws", type=int, default=65536)
    ap.add_argument("--eval-draws", type=int, default=4096)
    ap.add_argument("--train-steps", type=int, default=120000)
    ap.add_argument("--infer-only", action="store_true",
                    help="surrogate workload: time forward passes of batches of 32768 queries only")
    ap.add_argument("--weight-decay", type=float, default=0.1)
    ap.add_argument("--data-cache", default="",
                    help="npz file holding (or receiving) the simulated training / evaluation spectra")
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--replicates", type=int, default=4096)
    ap.add_argument("--n-max", type=float, default=1e4)
    ap.add_argument("--plain-sample", type=int, default=32)
    ap.add_argument("--gens", type=int, default=GENS,
                    help="generations per simulation (profiling captures use a shorter run)")
    args = ap.parse_args()
    rank, local_rank, world = dist_env()
    if args.workload == "batched":
        if rank == 0:
            run_batched(args)
        return
    if args.workload == "surrogate":
        if rank == 0:
            run_surrogate(args)
        return
    if args.workload == "multipop":
        if rank == 0:
            run_multipop(args)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import torch
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local_rank))
    try:
        run_b200(args, rank, local_rank, world)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
