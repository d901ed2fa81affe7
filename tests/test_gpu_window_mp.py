"""Multi-population window kernel: runs of 2 to 4 populations whose compaction windows are single
launches give the same state, IDs and work count bit for bit as one launch per generation, through
founding, migration, mixed neutral and selected populations, inbreeding, births, compactions on and off
the window grid, preserved time samples, an extinction (after which every generation runs alone) and
a resumed state whose not-yet-founded population row is nonzero (which no window may hold)."""
from __future__ import annotations

import numpy as np
import pytest

from parallelpopgen_b200 import Engine
from parallelpopgen_b200._capi import GEN_DTYPE, MAX_POPULATIONS, MSE_DTYPE

pytestmark = pytest.mark.gpu


def schedule(P: int, first: int, last: int, *, found=(0, 1, 40), sizes=(3000, 2500, 2000), m=0.01,
             gammas=(-4.0, 0.0, 3.0), shift=60, F=(0.0, 0.0, 0.2, 0.1), h=(0.5, 0.3, 0.5, 0.8),
             compact_interval=25, sample_every=50, extinct_at=None, mu=2e-8):
    """Generation records: population p exists from generation found[p] (founded from p - 1 with
    migration proportion 1 in its founding generation), constant size, symmetric migration m among the
    existing populations otherwise; selection gamma_p switches sign at `shift`; a preserved time sample
    every `sample_every`; population P - 1 goes extinct at `extinct_at`."""
    found = tuple(found) + (found[-1] + 15,) * (P - len(found))
    sizes = tuple(sizes) + (1800,) * (P - len(sizes))
    gammas = tuple(gammas) + (1.0,) * (P - len(gammas))
    gens = np.zeros(last - first + 1, dtype=GEN_DTYPE)
    next_compact = compact_interval
    for g in range(1, first):
        if g == next_compact or g % sample_every == 0:
            next_compact = g + compact_interval
    for i, g in enumerate(range(first, last + 1)):
        G = gens[i]
        G["generation"] = g
        exists = [g >= max(found[p], 1) if p > 0 else True for p in range(P)]
        if extinct_at is not None and g >= extinct_at:
            exists[P - 1] = False
        for p in range(P):
            pp = G["pop"][p]
            N = sizes[p]
            if extinct_at is not None and p == P - 1 and g >= extinct_at:
                # the extinction generation drifts with N = 0 (clearing the row); later ones do not run
                pp["drift"] = 1 if g == extinct_at else 0
                pp["Nchrom_e"] = 0
                continue
            if not exists[p]:
                continue
            pp["drift"] = pp["alive"] = pp["mutate"] = 1
            pp["Nchrom_e"] = int(np.float32(2 * N) / np.float32(1 + np.float32(F[p])))
            pp["mu"], pp["F"], pp["h"] = mu, F[p], h[p]
            gamma = gammas[p] if g < shift else -gammas[p]
            pp["sel_intercept"] = np.float32(gamma) / np.float32(2 * sizes[0])
        mig = G["migration"]
        n_exist = sum(exists)
        for to in range(P):
            if not exists[to]:
                continue
            if to > 0 and g == max(found[to], 1):
                mig[(to - 1) * MAX_POPULATIONS + to] = 1.0
                continue
            for frm in range(P):
                if exists[frm]:
                    mig[frm * MAX_POPULATIONS + to] = (1.0 - (n_exist - 1) * m) if frm == to else m
        preserve = g % sample_every == 0
        compact = g == next_compact or g == last or preserve
        G["compact"] = 1 if compact else 0
        G["preserve"] = 1 if (compact and preserve) else 0
        if compact:
            next_compact = g + compact_interval
    return gens


def mse_start(P: int, N0: int = 3000):
    pops = np.zeros(P, dtype=MSE_DTYPE)
    pops[0] = (N0, 2 * N0, 2e-8, 0.0, 0.5, 0.0, np.float32(-4.0) / np.float32(2 * N0))
    return pops


def run_both(setup, segments):
    out = []
    for windows in (1, 0):
        with Engine() as e:
            e.set_tuning(windows=windows)
            setup(e)
            launches0 = e.stats()["kernel_launches"]
            for seg in segments:
                e.run(seg)
            f, ids = e.read_state()
            st = e.stats()
            out.append((f, ids, st["mutation_generations"], st["kernel_launches"] - launches0))
    return out


def assert_same(out, min_slots=1000):
    (f1, i1, m1, l1), (f0, i0, m0, l0) = out
    assert f1.shape == f0.shape and f1.shape[1] > min_slots, (f1.shape, f0.shape)
    bad = np.flatnonzero((f1.view(np.uint32) != f0.view(np.uint32)).any(axis=0))
    assert bad.size == 0, f"{bad.size} slots differ, first {bad[:5]}"
    assert np.array_equal(i1, i0)
    assert m1 == m0
    return l1, l0


@pytest.mark.parametrize("P", [2, 3, 4])
def test_windows_equal_per_generation_launches(P):
    gens = schedule(P, 1, 200)
    segments = [gens[:73], gens[73:150], gens[150:]]   # run() calls that split windows
    out = run_both(lambda e: e.begin_mse(mse_start(P), seed1=21, seed2=22, num_sites=2e6, compact_interval=25),
                   segments)
    l1, l0 = assert_same(out)
    assert l1 < l0 / 3, (l1, l0)   # the windows replaced most per-generation launches


def test_compaction_off_the_window_grid_and_blank_start():
    gens = schedule(3, 1, 180, found=(0, 3, 17), compact_interval=7, sample_every=45, m=0.05)
    out = run_both(lambda e: e.begin_blank(seed1=5, seed2=6, num_sites=4e6, P=3, compact_interval=7), [gens])
    assert_same(out, min_slots=200)


def test_no_compaction_windows_reach_their_length_limit():
    gens = schedule(2, 1, 300, compact_interval=0, sample_every=10**6)
    gens["compact"] = 0
    gens["preserve"] = 0
    out = run_both(lambda e: e.begin_mse(mse_start(2), seed1=3, seed2=4, num_sites=1e6, compact_interval=0),
                   [gens])
    assert_same(out)


def test_extinction_then_per_generation_launches():
    gens = schedule(3, 1, 160, extinct_at=90)
    out = run_both(lambda e: e.begin_mse(mse_start(3), seed1=8, seed2=9, num_sites=2e6, compact_interval=25),
                   [gens])
    l1, l0 = assert_same(out)
    assert l1 < l0


def test_resumed_nonzero_row_of_an_unfounded_population():
    """A resumed state may hold values in the row of a population the schedule has not founded yet;
    the per-generation kernel leaves that row to the ping-pong buffers, so no window may hold it."""
    rng = np.random.default_rng(3)
    M = 20000
    N = 4000
    freq = np.zeros((3, M), dtype=np.float32)
    freq[0] = rng.integers(1, N, size=M).astype(np.float32) / np.float32(N)
    freq[2, ::7] = np.float32(0.25)                    # population 2 is not founded until generation 40
    ids = np.zeros((M, 4), dtype=np.int32)
    ids[:, 2] = np.arange(1, M + 1)
    gens = schedule(3, 1, 120, found=(0, 1, 40), sizes=(2000, 2000, 2000))
    out = run_both(lambda e: e.begin_from_state(freq, ids, seed1=1, seed2=2, num_sites=2e6, compact_interval=25),
                   [gens])
    assert_same(out)


@pytest.mark.parametrize("P", [1, 3])
def test_async_time_samples_equal_synchronous_reads(P):
    """Time samples copied while the next generations run (gf_sim_sample_begin / _wait, two page-locked
    buffer sets used in turn) equal, bit for bit, the synchronous reads of an identical run at the same
    generations: rows packed [P][M] and the mutation IDs."""
    import torch
    gens = schedule(P, 1, 300, sample_every=60)
    segments = [gens[a:a + 60] for a in range(0, 300, 60)]
    setup = (lambda e: e.begin_mse(mse_start(P), seed1=31, seed2=32, num_sites=4e6, compact_interval=25))
    want = []
    with Engine() as e:
        setup(e)
        for seg in segments:
            e.run(seg)
            want.append(e.read_state())
    cap = 200_000
    bufs = [(torch.empty(P * cap, dtype=torch.float32).pin_memory().numpy(),
             torch.empty((cap, 4), dtype=torch.int32).pin_memory().numpy()) for _ in range(2)]
    got = []
    with Engine() as e:
        setup(e)
        pending = None
        for k, seg in enumerate(segments):
            e.run(seg)
            if pending is not None:           # the previous sample's copy overlapped this segment
                M = e.sample_wait()
                f, ids = pending
                got.append((f[:P * M].reshape(P, M).copy(), ids[:M].copy()))
            f, ids = bufs[k % 2]
            e.sample_begin(f, ids)
            pending = (f, ids)
        M = e.sample_wait()
        f, ids = pending
        got.append((f[:P * M].reshape(P, M).copy(), ids[:M].copy()))
    assert len(got) == len(want)
    for (fa, ia), (fb, ib) in zip(got, want):
        assert fa.shape == fb.shape and fa.shape[1] > 100, (fa.shape, fb.shape)
        assert np.array_equal(fa.view(np.uint32), fb.view(np.uint32))
        assert np.array_equal(ia, ib)


def test_async_time_sample_misuse_is_reported():
    """A wait with no sample in flight, a second begin while one is in flight, and caller arrays too small
    for the state come back as status codes; the engine stays usable."""
    import torch
    from parallelpopgen_b200._capi import GoFishError
    gens = schedule(2, 1, 60, sample_every=60)
    with Engine() as e:
        e.begin_mse(mse_start(2), seed1=41, seed2=42, num_sites=4e6, compact_interval=25)
        e.run(gens)
        with pytest.raises(GoFishError, match="no time sample in flight"):
            e.sample_wait()
        tiny = torch.empty(2 * 10, dtype=torch.float32).pin_memory().numpy()
        with pytest.raises(GoFishError, match="GF_ERR_CAPACITY"):
            e.sample_begin(tiny)
        f = torch.empty(2 * 200_000, dtype=torch.float32).pin_memory().numpy()
        e.sample_begin(f)
        with pytest.raises(GoFishError, match="already in flight"):
            e.sample_begin(f)
        M = e.sample_wait()
        want, _ = e.read_state()
        assert want.shape[1] == M
        assert np.array_equal(f[:2 * M].reshape(2, M).view(np.uint32), want.view(np.uint32))
