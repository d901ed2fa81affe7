"""Batched ragged replicates: every replicate of a batch must equal, bit for bit, the plain engine
run with the same seeds, model and compaction schedule (final frequencies and mutation IDs), and its
SFS must match the plain engine's SFS of that state (1e-5 relative)."""
from __future__ import annotations

import numpy as np
import pytest

from parallelpopgen_b200 import (ConstantModel, Engine, replicate, replicate_mse_pops, replicate_plain_generations,
                                 replicate_population)

pytestmark = pytest.mark.gpu


def make_replicates(count: int, seed: int, max_gens: int):
    rng = np.random.default_rng(seed)
    reps = []
    for r in range(count):
        N0 = int(np.exp(rng.uniform(np.log(300), np.log(4000))))
        gamma = float(rng.uniform(-40, 8)) if r % 3 else 0.0
        F = float(rng.uniform(0, 0.5))
        s = ConstantModel.s_from_gamma(gamma, N0, F) if gamma else 0.0
        rate = float(rng.uniform(-0.001, 0.01))
        reps.append(replicate(seed1=0xBEEF + 2 * r, seed2=0xDECAF - 2 * r, num_sites=float(rng.choice([2e6, 1e7])),
                              mu=1e-8, F=F, h=float(rng.uniform(0, 1)), s=s, N0=N0, growth_rate=rate,
                              N_min=max(N0 // 4, 50), N_max=4 * N0, num_generations=int(min(4 * N0, max_gens)),
                              compact_interval=int(rng.integers(5, 40))))
    return reps


def plain_run(rep):
    with Engine() as e:
        e.begin_mse(replicate_mse_pops(rep), seed1=rep.seed1, seed2=rep.seed2, num_sites=rep.num_sites,
                    compact_interval=rep.compact_interval)
        e.run(replicate_plain_generations(rep))
        f, ids = e.read_state()
        return f[0], ids


def test_batched_replicates_equal_plain_runs():
    reps = make_replicates(12, seed=3, max_gens=1500)
    with Engine() as e:
        e.batch_begin(reps)
        assert e.batch_run() == 0
        states = [e.batch_read_state(r) for r in range(len(reps))]
        st = e.batch_stats()
        sfs = e.batch_sfs(40, len(reps))
    assert st["active"] == 0 and st["generations"] == sum(r.num_generations for r in reps)
    with Engine() as plain:
        for r, rep in enumerate(reps):
            f_b, ids_b, gen = states[r]
            assert gen == rep.num_generations
            f_p, ids_p = plain_run(rep)
            assert f_b.shape == f_p.shape, (r, f_b.shape, f_p.shape)
            assert np.array_equal(f_b.view(np.uint32), f_p.view(np.uint32)), r
            assert np.array_equal(ids_b, ids_p), r
            Nc = int(np.float32(2 * replicate_population(rep, rep.num_generations)) /
                     np.float32(np.float32(1) + np.float32(rep.F)))
            want = plain.site_frequency_spectrum(f_p, Nc, 40, rep.num_sites)
            np.testing.assert_allclose(sfs[r].astype(np.float64), want.astype(np.float64), rtol=1e-5, atol=1e-3)


def test_batched_super_steps_are_resumable():
    """Running a batch in chunks of super-steps gives the same states as running it to completion."""
    reps = make_replicates(5, seed=11, max_gens=600)
    out = []
    for chunk in (0, 7):
        with Engine() as e:
            e.batch_begin(reps)
            if chunk:
                while e.batch_run(chunk) > 0:
                    pass
            else:
                e.batch_run()
            out.append([e.batch_read_state(r)[0] for r in range(len(reps))])
    for a, b in zip(*out):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_slab_graphs_equal_single_steps():
    """A record slab's super-steps replayed as one CUDA graph give the same states, counts and statistics
    as the same super-steps launched one at a time (profiling mode launches them one at a time), whether
    the batch runs to completion or in chunks that start slabs at both buffer parities; the batch is long
    enough for many slabs (the graphs are used from the second one on)."""
    reps = make_replicates(24, seed=21, max_gens=3000)
    runs = []
    for profiling, chunk in ((True, 0), (False, 0), (False, 53)):
        with Engine() as e:
            e.set_profiling(profiling)
            e.batch_begin(reps)
            if chunk:
                while e.batch_run(chunk) > 0:
                    pass
            else:
                assert e.batch_run() == 0
            st = e.batch_stats()
            runs.append(([e.batch_read_state(r) for r in range(len(reps))], st["generations"], st["super_steps"],
                         st["mutation_generations"]))
    (ref, gens, steps, mg) = runs[0]
    assert steps >= 100   # slabs of 512 / (largest cadence) super-steps: many of them
    for states, g, k, m in runs[1:]:
        assert g == gens and k == steps and m == mg
        for (fa, ia, ga), (fb, ib, gb) in zip(ref, states):
            assert ga == gb
            assert np.array_equal(fa.view(np.uint32), fb.view(np.uint32))
            assert np.array_equal(ia, ib)


def test_beneficial_growing_replicate_fits_its_segment():
    """Positive selection raises the equilibrium count of segregating sites above the neutral one, and a
    growing population carries that excess to its larger size.  This replicate (gamma = +10 at N0, h =
    0.875, tenfold growth, cadence 5; one of the benchmark's full-range draws) overflowed a segment sized
    from the neutral count (20,546 slots against 20,480); sized from its own equilibrium start it runs
    and equals the plain run."""
    rep = replicate(seed1=52533, seed2=908905, num_sites=1e7, mu=1e-9, F=0.14773035049438477,
                    h=0.8749696016311646, s=0.0025522892829030752, N0=2246, growth_rate=0.0009652790613472462,
                    N_min=224, N_max=22460, num_generations=8984, compact_interval=5)
    with Engine() as e:
        e.batch_begin([rep])
        assert e.batch_run() == 0
        f_b, ids_b, gen = e.batch_read_state(0)
    assert gen == rep.num_generations
    f_p, ids_p = plain_run(rep)
    assert np.array_equal(f_b.view(np.uint32), f_p.view(np.uint32))
    assert np.array_equal(ids_b, ids_p)


def test_streamed_records_agree():
    """Generation records are drawn by host threads region by region while the super-steps run: all
    regions resident (a large budget), a ring of a few regions (a budget of a few regions), a ring of
    two (a tiny budget) and the per-super-step path (budget 0) must give the same states, also when
    the batch runs in chunks of super-steps."""
    reps = make_replicates(64, seed=29, max_gens=4000)
    total = sum(r.num_generations for r in reps)
    assert total >= 1 << 17, total
    out = []
    for budget, steps in ((1 << 26, 0), (1 << 26, 9), (100_000, 0), (600, 7), (0, 0)):
        with Engine() as e:
            e.batch_set_record_budget(budget)
            e.batch_begin(reps)
            if steps:
                while e.batch_run(steps) > 0:
                    pass
            else:
                assert e.batch_run() == 0
            out.append([e.batch_read_state(r) for r in range(len(reps))])
            assert e.batch_stats()["generations"] == total
    for other in out[1:]:
        for (fa, ia, ga), (fb, ib, gb) in zip(out[0], other):
            assert ga == gb
            assert np.array_equal(fa.view(np.uint32), fb.view(np.uint32))
            assert np.array_equal(ia, ib)


def test_record_paths_agree():
    """All records resident, records cycling through a ring of regions (a budget far below the batch's
    total), and records built per super-step with a count read-back (budget 0) must give the same
    states, also when the batch runs in chunks of super-steps."""
    reps = make_replicates(6, seed=17, max_gens=700)
    out = []
    for budget in (1 << 26, 600, 0):
        with Engine() as e:
            e.batch_set_record_budget(budget)
            e.batch_begin(reps)
            while e.batch_run(5) > 0:
                pass
            out.append([e.batch_read_state(r) for r in range(len(reps))])
            st = e.batch_stats()
            assert st["active"] == 0 and st["generations"] == sum(r.num_generations for r in reps)
    for other in out[1:]:
        for (fa, ia, ga), (fb, ib, gb) in zip(out[0], other):
            assert ga == gb
            assert np.array_equal(fa.view(np.uint32), fb.view(np.uint32))
            assert np.array_equal(ia, ib)
