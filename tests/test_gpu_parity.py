"""GPU parity of the sm_100a engine against the reference run on the same GPU (oracle/_ref) and the CPU
oracle (oracle/).

Bar: bit-exact against the reference for every integer allele count, frequency, mutation ID and
histogram bin; the projected SFS within 2e-4 relative per bin of the reference (whose float atomics
are order-dependent) and within 1e-5 of the oracle's double-precision projection.  Against the CPU
oracle, drawn counts agree except for draws near a rounding boundary: CUDA's fast-math normcdfinv
carries a few 1e-5 of relative error, which the oracle's double-precision inverse does not, so a
normal-branch draw with standard deviation sd lands one count apart with probability ~1e-5 * sd.
The tolerance is: every difference is one count, and at most 1% of draws differ.
"""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from gfdump import Dump
from parallelpopgen_b200 import ConstantModel, Engine, constant_generations

import oracle.oracle as orc  # noqa: E402  (checker)

pytestmark = pytest.mark.gpu

SEED1, SEED2 = 0xBEEF, 0xDECAF


def run_engine_one_generation(freq: np.ndarray, *, N: int, F=0.0, h=0.5, s=0.0, slope=0.0, gen=1,
                              seed1=SEED1, seed2=SEED2) -> np.ndarray:
    with Engine() as e:
        e.begin_from_state(freq, None, seed1=seed1, seed2=seed2, num_sites=1e6, compact_interval=0)
        model = ConstantModel(N=1, F=F, h=h, s=s)
        g = constant_generations(model, gen, 1, compact_interval=0, mutate=False)
        g["pop"]["Nchrom_e"][:, 0] = N
        g["pop"]["sel_slope"][:, 0] = slope
        e.run(g)
        out, _ = e.read_state(with_ids=False)
    return out[0]


def freq_grid(N: int, M: int, rng: np.random.Generator) -> np.ndarray:
    """Frequencies j/N (engine values) covering lost, fixed, rare, common and near-fixed classes."""
    j = np.concatenate([
        np.array([0, 1, 2, 3, N - 3, N - 2, N - 1, N, N // 2]),
        rng.integers(0, N + 1, size=M - 9),
        rng.integers(0, min(N, 12) + 1, size=0),
    ])[:M]
    return (j.astype(np.float32) / np.float32(N)).astype(np.float32)


DRIFT_CASES = [
    # N, F, h, s, slope, M
    (20000, 0.0, 0.5, 0.0, 0.0, 200003),
    (20000, 0.0, 0.5, -0.00025, 0.0, 100001),
    (400000, 0.0, 0.5, -0.0000125, 0.0, 200002),
    (1000, 1.0, 0.0, -0.001, 0.0, 50001),
    (1000, 0.1, 0.3, 0.002, 0.0, 50000),
    (99, 0.0, 0.5, 0.0, 0.0, 20003),
    (50, 0.0, 0.2, -0.05, 0.0, 20001),
    (100, 0.0, 0.5, 0.01, 0.0, 20002),
    (2000, 0.0, 0.5, -0.001, 0.004, 40001),
]


@pytest.mark.parametrize("N,F,h,s,slope,M", DRIFT_CASES)
def test_one_generation_matches_reference_kernel(ref_driver, tmp_path, N, F, h, s, slope, M):
    """Same input row through the reference's migration_selection_drift and the fused kernel."""
    rng = np.random.default_rng(N * 7 + M)
    x = freq_grid(N, M, rng)
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        f.write(np.int32(M).tobytes())
        f.write(x.tobytes())
    out = tmp_path / "out.bin"
    args = [f"N={N}", f"F={F}", f"h={h}", f"s={s}", f"slope={slope}", "gen=7", f"seed1={SEED1}", f"seed2={SEED2}"]
    subprocess.run([str(ref_driver), "drift1", str(inp), str(out), *args], check=True)
    ref = np.fromfile(out, dtype=np.float32)
    mine = run_engine_one_generation(x, N=N, F=F, h=h, s=s, slope=slope, gen=7)
    bad = np.flatnonzero(ref.view(np.uint32) != mine.view(np.uint32))
    assert bad.size == 0, f"{bad.size} of {M} slots differ; first {bad[:5]}: ref {ref[bad[:5]]} mine {mine[bad[:5]]}"


@pytest.mark.parametrize("N,F,h,s,slope,M", DRIFT_CASES[:6])
def test_one_generation_matches_oracle(N, F, h, s, slope, M):
    rng = np.random.default_rng(N * 11 + M)
    x = freq_grid(N, M, rng)
    mine = run_engine_one_generation(x, N=N, F=F, h=h, s=s, slope=slope, gen=3)
    ref = orc.drift(x, generation=3, seed1=SEED1, seed2=SEED2, Nc=N, F=F, h=h, sel_intercept=s, sel_slope=slope)[0]
    cm = np.rint(mine.astype(np.float64) * N)
    cr = np.rint(ref.astype(np.float64) * N)
    diff = np.abs(cm - cr)
    assert diff.max() <= 1, f"max count difference {diff.max()}"
    assert (diff > 0).mean() <= 1e-2, f"{(diff > 0).sum()} of {M} draws differ"


def run_driver(driver: Path, scenario: str, out: Path, args: list[str]) -> Dump:
    r = subprocess.run([str(driver), scenario, str(out), *args], check=True, capture_output=True, text=True)
    return Dump(out)


def assert_dumps_equal(a: Dump, b: Dump, sfs_rtol=2e-4):
    """Bit-exact comparison of two dumps.  Rows of populations that do not exist at a sample
    (Nchrom_e == 0) are skipped: the reference never writes them, so they hold whatever its device
    allocation held (go_fish_impl.cuh:651-656 skips the population; its buffers are fresh cudaMalloc
    memory after every compaction, :428), while this engine keeps them at zero."""
    assert a.P == b.P
    assert len(a.samples) == len(b.samples)
    for sa, sb in zip(a.samples, b.samples):
        assert sa["generation"] == sb["generation"]
        assert sa["M"] == sb["M"], f"generation {sa['generation']}: {sa['M']} vs {sb['M']} mutations"
        assert np.array_equal(sa["Nc"], sb["Nc"]) and np.array_equal(sa["extinct"], sb["extinct"])
        for p in range(a.P):
            if sa["Nc"][p] <= 0:
                continue
            bad = np.flatnonzero(sa["freq"][p].view(np.uint32) != sb["freq"][p].view(np.uint32))
            assert bad.size == 0, f"generation {sa['generation']} population {p}: {bad.size} frequencies differ"
    assert np.array_equal(a.ids, b.ids)
    assert a.spectra.keys() == b.spectra.keys()
    for k in a.spectra:
        x, y = a.spectra[k].astype(np.float64), b.spectra[k].astype(np.float64)
        if k[2] == "hist":
            assert np.array_equal(x, y), k
        else:
            np.testing.assert_allclose(x, y, rtol=sfs_rtol, atol=1e-3, err_msg=str(k))


WF_CFG1 = ["N=10000", "L=2e7", "gens=1000", "compact=35", "mse=1", "sfs_n=100", "hist=1", "sample_every=250"]


def test_cfg1_neutral_matches_reference(gofish_driver, ref_driver, tmp_path):
    """1 pop, N=1e4, L=2e7, neutral, MSE start, 1000 generations (the CPU-runnable configuration)."""
    mine = run_driver(gofish_driver, "wf", tmp_path / "mine.bin", WF_CFG1)
    subprocess.run([str(ref_driver), "sim", "wf", str(tmp_path / "ref.bin"), *WF_CFG1], check=True, capture_output=True)
    ref = Dump(tmp_path / "ref.bin")
    assert mine.samples[-1]["M"] > 1000
    assert_dumps_equal(mine, ref)


@pytest.mark.parametrize("extra", [
    ["gamma=-10", "h=0.5", "mse=0", "gens=3000", "compact=25"],
    ["gamma=5", "h=0.3", "F=0.1", "mse=0", "gens=2000", "compact=10"],
    ["N=40", "mse=0", "gens=3000", "L=2e8"],
    ["pops=2", "m=0.01", "mse=1", "gens=500"],
    # seasonal selection: the sine is evaluated on the device, as the reference's kernel evaluates it
    ["sine_A=20", "sine_pi=0.05", "sine_rho=0.3", "gamma=-2", "mse=0", "gens=2000", "compact=25"],
    # ... in one of two populations exchanging migrants (selection_population_specific around it)
    ["sine_A=-30", "sine_pi=0.02", "gamma=1", "sine_pop=1", "pops=2", "m=0.005", "mse=0", "gens=1500",
     "compact=30"],
])
def test_wf_variants_match_reference(gofish_driver, ref_driver, tmp_path, extra):
    args = ["N=5000", "L=1e7", "sfs_n=50", "hist=1", "sample_every=0", *extra]
    mine = run_driver(gofish_driver, "wf", tmp_path / "mine.bin", args)
    subprocess.run([str(ref_driver), "sim", "wf", str(tmp_path / "ref.bin"), *args], check=True, capture_output=True)
    assert_dumps_equal(mine, Dump(tmp_path / "ref.bin"))


def random_wf_cases(count: int, seed: int = 2026):
    """Seeded draws over the single- and multi-population model space: population size (log-uniform
    50 to 20,000), one to three populations with symmetric migration, selection, dominance, inbreeding,
    mutation rate, sites, run length, compaction cadence and sampling.  Selected runs start blank: the
    reference's selected equilibrium start is not deterministic (its float scan), so only neutral runs
    start at equilibrium."""
    rng = np.random.default_rng(seed)
    cases = []
    for _ in range(count):
        pops = int(rng.choice([1, 1, 2, 3]))
        gamma = 0.0 if rng.random() < 0.3 else float(np.round(rng.uniform(-50, 10), 2))
        case = [f"seed1={int(rng.integers(1, 2**31 - 1))}", f"seed2={int(rng.integers(1, 2**31 - 1))}",
                f"N={int(np.exp(rng.uniform(np.log(50), np.log(20000))))}", f"pops={pops}",
                f"gamma={gamma}", f"h={float(np.round(rng.uniform(0, 1), 3))}",
                f"F={0.0 if rng.random() < 0.5 else float(np.round(rng.uniform(0, 0.5), 3))}",
                f"mu={float(rng.choice([1e-9, 1e-8]))}", f"L={float(np.round(np.exp(rng.uniform(np.log(1e6), np.log(5e7))), -3))}",
                f"gens={int(rng.integers(200, 1500))}", f"compact={int(rng.integers(5, 50))}",
                f"sample_every={int(rng.choice([0, 100, 250]))}", f"mse={1 if gamma == 0.0 else 0}"]
        if pops > 1:
            case.append(f"m={float(np.round(np.exp(rng.uniform(np.log(1e-4), np.log(0.02))), 6))}")
        cases.append(case)
    return cases


@pytest.mark.parametrize("case", random_wf_cases(12), ids=lambda c: "-".join(x.split("=")[1] for x in c[2:5]))
def test_random_wf_scenarios_match_reference(gofish_driver, ref_driver, tmp_path, case):
    """Seeded random scenarios over the model space the reference's run_sim covers, each bit-exact
    against the reference built and run on the same GPU (frequencies, IDs, histograms; SFS within the
    tolerance)."""
    args = ["sfs_n=50", "hist=1", *case]
    mine = run_driver(gofish_driver, "wf", tmp_path / "mine.bin", args)
    subprocess.run([str(ref_driver), "sim", "wf", str(tmp_path / "ref.bin"), *args], check=True, capture_output=True)
    assert_dumps_equal(mine, Dump(tmp_path / "ref.bin"))


@pytest.mark.parametrize("extra", [
    ["quad_a=-40", "gamma=2", "gens=2000", "compact=25"],
    ["quad_a=30", "gamma=-3", "pops=2", "m=0.01", "gens=1500", "compact=20"],
])
def test_user_device_selection_functor_matches_reference(gofish_driver_nvcc, ref_driver, tmp_path, extra):
    """A user selection functor that is not affine in frequency (s = a x^2 + b, a __device__ call
    operator as the reference's functor contract asks): in a translation unit compiled by nvcc the
    front-end instantiates its selection kernel for the functor and the engine reads the per-mutation
    coefficients it writes, so the run is bit-exact against the reference, with and without migration."""
    args = ["N=5000", "L=1e7", "sfs_n=50", "hist=1", "sample_every=0", "mse=0", *extra]
    mine = run_driver(gofish_driver_nvcc, "wf", tmp_path / "mine.bin", args)
    subprocess.run([str(ref_driver), "sim", "wf", str(tmp_path / "ref.bin"), *args], check=True, capture_output=True)
    ref = Dump(tmp_path / "ref.bin")
    assert ref.samples[-1]["M"] > 1000
    assert_dumps_equal(mine, ref)


def test_user_device_selection_functor_three_populations(gofish_driver_nvcc, ref_driver, tmp_path):
    """The device-evaluated user functor with three populations exchanging migrants (the benchmark's
    three-population model after its last founding, continued from one stored state for 300
    generations): x_mig mixes three rows before the functor sees it."""
    start = tmp_path / "start.bin"
    run_driver(gofish_driver_nvcc, "multipop", tmp_path / "stage1.bin", ["gens=2100", "sample_every=0", "L=5e7",
                                                                         f"state_out={start}"])
    args = ["gens=300", "sample_every=0", "L=5e7", "quad_a=-60", "sfs_n=100", "hist=1", f"state_in={start}"]
    mine = run_driver(gofish_driver_nvcc, "multipop", tmp_path / "mine.bin", args)
    subprocess.run([str(ref_driver), "sim", "multipop", str(tmp_path / "ref.bin"), *args], check=True,
                   capture_output=True)
    ref = Dump(tmp_path / "ref.bin")
    assert ref.samples[-1]["generation"] == 2400 and ref.samples[-1]["M"] > 100_000
    assert_dumps_equal(mine, ref)


def test_user_selection_functor_limits(gofish_driver, gofish_driver_nvcc, tmp_path):
    """Where the device path is not available the front-end says so: a plain C++ translation unit can
    only use selection models that are affine in frequency, and the equilibrium start integrates an
    affine model at generation 0."""
    args = ["N=2000", "L=1e6", "gens=10", "quad_a=-40", "gamma=2"]
    r = subprocess.run([str(gofish_driver), "wf", str(tmp_path / "a.bin"), *args, "mse=0"], capture_output=True,
                       text=True)
    assert r.returncode == 1 and "not affine in frequency" in r.stderr
    r = subprocess.run([str(gofish_driver_nvcc), "wf", str(tmp_path / "b.bin"), *args, "mse=1"], capture_output=True,
                       text=True)
    assert r.returncode == 1 and "affine in frequency at generation 0" in r.stderr


def test_resume_and_preserve_match_reference(gofish_driver, ref_driver, tmp_path):
    """Two inbred populations: blank start, burn-in, resume from the burn-in sample, sampling the start.
    The text dump of operator<< (inline_go_fish_data_struct.hpp:208-267) must be byte-identical too."""
    args = ["gens1=3000", "gens2=500", "L=2e7", "sfs_n=20", "hist=1"]
    mine = run_driver(gofish_driver, "compilation", tmp_path / "mine.bin", [*args, f"text={tmp_path / 'mine.txt'}"])
    subprocess.run([str(ref_driver), "sim", "compilation", str(tmp_path / "ref.bin"), *args,
                    f"text={tmp_path / 'ref.txt'}"], check=True, capture_output=True)
    assert_dumps_equal(mine, Dump(tmp_path / "ref.bin"))
    ref_text = (tmp_path / "ref.txt").read_bytes()
    assert ref_text.count(b"\n") > 100
    assert (tmp_path / "mine.txt").read_bytes() == ref_text


# The benchmarked single-population workload: one half of N = 2e5 diploids (Nchrom_e 4e5), L = 2.5e8,
# compaction every 25 generations, SFS of a sample of 1000 and the full population histogram.  About
# 2.7 M segregating mutations at the start and 2e5 new ones every generation, so the quad/tail split,
# capacity growth and the mix of Poisson and normal draws are the ones the benchmark exercises.
CFG2_HALF = ["N=200000", "L=2.5e8", "gens=300", "compact=25", "sfs_n=1000", "hist=1", "sample_every=0"]


def test_cfg2_neutral_half_matches_reference(gofish_driver, ref_driver, tmp_path):
    """The neutral half of the benchmark from its mutation-selection-equilibrium start (deterministic in
    the reference when s = 0), 300 generations."""
    args = [*CFG2_HALF, "mse=1"]
    mine = run_driver(gofish_driver, "wf", tmp_path / "mine.bin", args)
    subprocess.run([str(ref_driver), "sim", "wf", str(tmp_path / "ref.bin"), *args], check=True, capture_output=True)
    ref = Dump(tmp_path / "ref.bin")
    assert ref.samples[-1]["M"] > 2_000_000
    assert_dumps_equal(mine, ref)


def test_cfg2_selected_half_matches_reference(gofish_driver, ref_driver, tmp_path):
    """The gamma = -10, h = 0.5 half of the benchmark.  The reference's equilibrium start with selection
    sums floats in a nondeterministic order (a CUB scan, go_fish_impl.cu:13-32), so both programs
    continue from one stored reference state: the reference's own equilibrium start run for 25
    generations, then 300 generations in each program from that state (prev_sim, init_mse = false)."""
    start = tmp_path / "start.bin"
    subprocess.run([str(ref_driver), "sim", "wf", str(tmp_path / "stage1.bin"), *CFG2_HALF, "gens=25", "mse=1",
                    "gamma=-10", "h=0.5", f"state_out={start}"], check=True, capture_output=True)
    args = [*CFG2_HALF, "gamma=-10", "h=0.5", f"state_in={start}"]
    mine = run_driver(gofish_driver, "wf", tmp_path / "mine.bin", args)
    subprocess.run([str(ref_driver), "sim", "wf", str(tmp_path / "ref.bin"), *args], check=True, capture_output=True)
    ref = Dump(tmp_path / "ref.bin")
    assert ref.samples[-1]["generation"] == 325 and ref.samples[-1]["M"] > 1_000_000
    assert_dumps_equal(mine, ref)


def test_multipop_after_the_split_matches_reference(gofish_driver, ref_driver, tmp_path):
    """The benchmarked three-population model (scenario multipop): growth to the caps, migration 1e-4,
    F = 0.1 in population 2, L = 2e8, a time sample every 500 generations, through the switch from
    gamma -5 to +2 at generation 3000.  Before population 2 is founded (generation 2000) the reference
    never writes its rows, which then hold whatever its fresh device allocations held, and its migration
    sum multiplies them by a zero rate (go_fish_impl.cuh:98-102, 651-656), so the reference is only well
    defined once every population exists.  Both programs therefore continue from one stored state at
    generation 2100, written by this library, for 1000 generations."""
    start = tmp_path / "start.bin"
    run_driver(gofish_driver, "multipop", tmp_path / "stage1.bin", ["gens=2100", "sample_every=0",
                                                                    f"state_out={start}"])
    args = ["gens=1000", "sample_every=500", "sfs_n=200", "hist=1", f"state_in={start}"]
    mine = run_driver(gofish_driver, "multipop", tmp_path / "mine.bin", args)
    subprocess.run([str(ref_driver), "sim", "multipop", str(tmp_path / "ref.bin"), *args], check=True,
                   capture_output=True)
    ref = Dump(tmp_path / "ref.bin")
    assert [s["generation"] for s in ref.samples] == [2500, 3000, 3100]
    assert ref.samples[-1]["M"] > 1_000_000 and (ref.samples[-1]["Nc"] > 0).all()
    assert_dumps_equal(mine, ref)


def test_split3_matches_reference(gofish_driver, ref_driver, tmp_path):
    """Three populations founded from an ancestor, logistic growth, founding and symmetric migration,
    piecewise selection, inbreeding in one population, time samples with preservation.

    Both daughter populations are founded at generation 1.  While a population does not exist yet,
    the reference never writes its rows, which then hold recycled device memory (freed flag words or
    preserved IDs read as floats can be NaN), and its migration sum multiplies them by a zero rate:
    0 * NaN corrupts live populations, so the reference's result depends on allocator history.  This
    engine keeps such rows at zero; the bit-exact comparison uses a schedule on which the reference is
    well defined."""
    args = ["L=2e6", "gens=900", "split1=1", "split2=1", "switch_gen=500", "sample_every=200", "K0=20000",
            "K1=30000", "K2=40000", "N0=5000", "mse=1", "sfs_n=30", "hist=1"]
    mine = run_driver(gofish_driver, "split3", tmp_path / "mine.bin", args)
    subprocess.run([str(ref_driver), "sim", "split3", str(tmp_path / "ref.bin"), *args], check=True,
                   capture_output=True)
    assert_dumps_equal(mine, Dump(tmp_path / "ref.bin"))


def test_compaction_matches_oracle():
    """Stable compaction: the engine's compacted state equals the oracle's compaction of the same
    generation's uncompacted state (lost, fixed and preserved slots, two populations)."""
    rng = np.random.default_rng(5)
    P, M, N = 2, 30001, 1000
    j = rng.integers(0, N + 1, size=(P, M))
    j[:, rng.random(M) < 0.3] = 0
    j[:, rng.random(M) < 0.1] = N
    freq = (j.astype(np.float32) / np.float32(N)).astype(np.float32)
    ids = np.zeros((M, 4), dtype=np.int32)
    ids[:, 0] = rng.integers(0, 5000, size=M)
    ids[:, 1] = rng.integers(0, P, size=M)
    ids[:, 2] = np.arange(1, M + 1)
    ids[rng.random(M) < 0.05, 2] *= -1
    model = ConstantModel(N=N // 2, P=P, m=0.0)
    states = []
    for compact in (0, 1):
        with Engine() as e:
            e.begin_from_state(freq, ids, seed1=1, seed2=2, num_sites=1e7, compact_interval=compact)
            g = constant_generations(model, 1, 1, compact_interval=compact, mutate=True)
            g["pop"]["mu"][:, :P] = 1e-7  # a few new mutations join the compaction
            e.run(g)
            states.append(e.read_state())
    (f0, i0), (f1, i1) = states
    assert f0.shape[1] >= M
    want_f, want_ids = orc.compact(f0, i0, alive=[1, 1])
    assert 0 < want_f.shape[1] < f0.shape[1]
    assert np.array_equal(i1, want_ids)
    assert np.array_equal(f1.view(np.uint32), want_f.view(np.uint32))
    # and with the preserve mark
    with Engine() as e:
        e.begin_from_state(freq, ids, seed1=1, seed2=2, num_sites=1e7, compact_interval=1)
        g = constant_generations(model, 1, 1, compact_interval=1, mutate=True)
        g["pop"]["mu"][:, :P] = 1e-7
        g["preserve"] = 1
        e.run(g)
        fp, ip = e.read_state()
    want_f, want_ids = orc.compact(f0, i0, alive=[1, 1], preserve=True)
    assert np.array_equal(ip, want_ids) and (ip[:, 2] < 0).all()
    assert np.array_equal(fp.view(np.uint32), want_f.view(np.uint32))


def test_histogram_and_sfs_match_oracle():
    rng = np.random.default_rng(9)
    Nc, M, L = 20000, 300000, 2e7
    j = np.minimum(rng.geometric(0.0005, size=M), Nc)
    j[rng.random(M) < 0.02] = 0
    x = (j.astype(np.float32) / np.float32(Nc)).astype(np.float32)
    with Engine() as e:
        h = e.population_histogram(x, Nc, L)
        np.testing.assert_array_equal(h, orc.histogram(x, Nc, L))
        for n in (2, 100, 1000):
            got = e.site_frequency_spectrum(x, Nc, n, L).astype(np.float64)
            want = orc.sfs(x, n, L)
            np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-4)
        # frequencies off the 1/Nc grid take the direct projection
        y = rng.random(5000).astype(np.float32)
        got = e.site_frequency_spectrum(y, Nc, 64, L).astype(np.float64)
        np.testing.assert_allclose(got, orc.sfs(y, 64, L), rtol=1e-5, atol=1e-4)


@pytest.mark.parametrize("gamma,ci,mse", [(0.0, 25, True), (-10.0, 25, True), (4.0, 7, False), (0.0, 0, True)])
def test_window_path_equals_per_generation_path(gamma, ci, mse):
    """Single-population generations run as window launches by default; the per-generation kernel
    must give the same state bit for bit (including compactions, births and IDs)."""
    N = 3000
    s = ConstantModel.s_from_gamma(gamma, N, 0.0) if gamma else 0.0
    model = ConstantModel(N=N, s=s, mu=2e-8, h=0.3)
    gens = constant_generations(model, 1, 300, ci)
    out = []
    for windows in (1, 0):
        with Engine() as e:
            e.set_tuning(windows=windows)
            if mse:
                e.begin_mse(model.mse_pops(), seed1=7, seed2=9, num_sites=2e6, compact_interval=ci)
            else:
                e.begin_blank(seed1=7, seed2=9, num_sites=2e6, compact_interval=ci)
            e.run(gens)
            out.append(e.read_state() + (e.stats()["mutation_generations"],))
    (f1, i1, m1), (f0, i0, m0) = out
    assert f1.shape == f0.shape and f1.shape[1] > 100
    assert np.array_equal(f1.view(np.uint32), f0.view(np.uint32))
    assert np.array_equal(i1, i0)
    assert m1 == m0


@pytest.mark.parametrize("pops", [1, 3])
def test_draw_strategies_agree(pops):
    """The five draw schedules (lane order, warp-pooled, grouped by sampler branch, normal
    approximation of all lanes first, normal approximation per thread with the search draws pooled
    per warp) call the same sampler on the same inputs, so window and per-generation runs, single- and multi-population,
    give the same state bit for bit under every one of them."""
    N = 4000
    if pops == 1:
        model = ConstantModel(N=N, s=ConstantModel.s_from_gamma(-4.0, N, 0.0), mu=2e-8, h=0.3)
    else:
        model = ConstantModel(N=N, s=ConstantModel.s_from_gamma(-4.0, N, 0.0), mu=2e-8, h=0.3, P=3, m=0.01)
    gens = constant_generations(model, 1, 200, 25)
    out = []
    for strategy in (0, 1, 2, 3, 4):
        for windows in ((1, 0) if pops == 1 else (1,)):
            with Engine() as e:
                e.set_tuning(draw_strategy=strategy, windows=windows)
                e.begin_mse(model.mse_pops(), seed1=11, seed2=13, num_sites=4e6, compact_interval=25)
                e.run(gens)
                out.append(((strategy, windows),) + e.read_state())
    (_, f0, i0) = out[0]
    assert f0.shape[1] > 1000
    for key, f, ids in out[1:]:
        assert np.array_equal(f.view(np.uint32), f0.view(np.uint32)), key
        assert np.array_equal(ids, i0), key
