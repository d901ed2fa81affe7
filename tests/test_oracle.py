"""CPU oracle pinned against the reference's own host code (golden vectors in tests/golden/, made by
tests/golden/make_golden.py) and against independent formulas.  No GPU needed."""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np
import pytest
from scipy import special, stats

import oracle.oracle as orc

GOLDEN = Path(__file__).resolve().parent / "golden"


def hostrng():
    b = np.fromfile(GOLDEN / "ref_hostrng.bin", dtype=np.int32)
    nph, npo = int(b[0]), int(b[1])
    ph = b[2:2 + nph * 10].reshape(-1, 10)
    po = b[2 + nph * 10:].reshape(-1, 6)
    assert len(po) == npo
    return ph, po


def test_philox_matches_reference_host_vectors():
    ph, _ = hostrng()
    assert len(ph) == 216
    for r in ph:
        got = orc.philox(int(r[0]), int(r[1]), int(r[2]), int(r[3]), int(r[4]), int(r[5]))
        assert np.array_equal(got, r[6:10].view(np.uint32)), r[:6]


def test_poisson_draw_matches_reference_host_vectors():
    """The new-mutation count path: ApproxRandPois1 with counter (1, generation, pop, 0), drawn on the
    host.  Covers the sequential-search branch (mean <= 6) and the normal branch."""
    _, po = hostrng()
    for r in po:
        mean = float(np.int32(r[2]).view(np.float32))
        got = orc.lib().or_pois_draw(mean, mean, 1e12, int(r[0]), int(r[1]), 1, int(r[3]), int(r[4]))
        assert got == r[5], (mean, int(r[3]), int(r[4]))


def test_normcdfinv_is_accurate():
    p = np.concatenate([np.linspace(1e-9, 1 - 1e-9, 2001), [2 ** -33, 1e-6, 0.02425, 0.5, 0.97575, 1 - 2 ** -24]])
    got = np.array([orc.lib().or_normcdfinv(float(x)) for x in p])
    want = special.ndtri(p)
    assert np.max(np.abs(got - want) / np.maximum(1.0, np.abs(want))) < 1e-9  # float inputs need 1e-7
    assert orc.lib().or_normcdfinv(1.0) == math.inf and orc.lib().or_normcdfinv(0.0) == -math.inf


def test_uniform_mapping_is_open_closed():
    assert orc.lib().or_u01(0) == np.float32(2.0 ** -33)
    assert orc.lib().or_u01(0xFFFFFFFF) == 1.0  # rounds up to 1: the reference's u lies in (0, 1]
    assert orc.lib().or_u01(1 << 31) == np.float32(0.5) + np.float32(2.0 ** -33)


@pytest.mark.parametrize("mean,cap", [(0.5, 11), (1.0, 11), (1.5, 14), (2.0, 14), (3.0, 17), (4.0, 20), (5.0, 22),
                                      (6.0, 24)])
def test_poisson_search_caps(mean, cap):
    """poiscdfinv stops at a mean-dependent cap even when the float CDF has not reached u
    (shared.cuh:188-248): no draw exceeds the cap, and the largest u reaches it or the point where
    the float CDF rounds to 1."""
    u = np.concatenate([np.linspace(0.0, 1.0, 4001, dtype=np.float32), [np.float32(1.0)]])
    got = np.array([orc.lib().or_pois_search(float(x), mean) for x in u])
    assert got.max() <= cap
    assert orc.lib().or_pois_search(np.float32(1e-30), mean) == 0


def test_poisson_search_is_the_inverse_cdf():
    rng = np.random.default_rng(3)
    for mean in (0.2, 1.0, 3.3, 5.9):
        u = rng.random(2000).astype(np.float32)
        got = np.array([orc.lib().or_pois_search(float(x), mean) for x in u])
        want = stats.poisson.ppf(u.astype(np.float64), mean)
        assert np.mean(got == want) > 0.995


def test_binomial_search_for_small_populations():
    rng = np.random.default_rng(4)
    n = 40.0
    for mean in (0.5, 2.0, 5.5):
        u = rng.random(2000).astype(np.float32)
        got = np.array([orc.lib().or_binom_search(float(x), mean, mean / n, n) for x in u])
        want = stats.binom.ppf(u.astype(np.float64), int(n), mean / n)
        assert np.mean(got == want) > 0.99


def test_binomial_draw_branches():
    """Branch structure of ApproxRandBinomHelper (shared.cu:10-18)."""
    L = orc.lib()
    bits = 0x80000000
    assert L.or_binom_draw(bits, 0.0, 0.0, 1000.0) == 0                 # lost stays lost
    assert L.or_binom_draw(bits, 1000.0, 0.0, 1000.0) == 1000           # fixed stays fixed
    assert L.or_binom_draw(bits, 500.0, 250.0, 1000.0) == 500           # u = 0.5: z = 0
    assert L.or_binom_draw(0xFFFFFFFF, 500.0, 250.0, 1000.0) == 2147483647  # u = 1: +inf, saturates


def test_drift_counter_layout_quad_and_tail():
    """Slots in whole quads use Philox(k = i/4 + 2) lane i%4; the scalar tail uses Philox(k = i + 2) lane x."""
    N, M = 20000, 11
    x = np.full(M, 0.5, dtype=np.float32)
    out = orc.drift(x, generation=5, seed1=1, seed2=2, Nc=N)[0]
    for i in range(M):
        if i < 8:
            bits = orc.philox(1, 2, i // 4 + 2, 5, 0)[i % 4]
        else:
            bits = orc.philox(1, 2, i + 2, 5, 0)[0]
        u = orc.lib().or_u01(int(bits))
        z = orc.lib().or_normcdfinv(float(u))
        j = int(np.round(np.float32(z) * np.sqrt(np.float32(5000.0)) + np.float32(10000.0)))
        assert abs(round(float(out[i]) * N) - j) <= 1


def test_compaction_is_stable_and_honours_preserve():
    freq = np.array([[0.0, 0.5, 1.0, 0.25, 0.0, 0.75]], dtype=np.float32)
    ids = np.zeros((6, 4), dtype=np.int32)
    ids[:, 2] = np.arange(1, 7)
    ids[4, 2] = -5  # preserved although lost
    f, i = orc.compact(freq, ids, alive=[1])
    assert list(i[:, 2]) == [2, 4, -5, 6]
    assert list(f[0]) == [0.5, 0.25, 0.0, 0.75]
    f, i = orc.compact(freq, ids, alive=[1], preserve=True)
    assert (i[:, 2] < 0).all()
    # a mutation lost in one population and segregating in another stays
    two = np.array([[0.0, 1.0], [0.5, 1.0]], dtype=np.float32)
    f, i = orc.compact(two, ids[:2], alive=[1, 1])
    assert list(i[:, 2]) == [1]
    f, i = orc.compact(two, ids[:2], alive=[1, 0])  # population 1 not alive: only population 0 counts
    assert len(i) == 0


def test_histogram_and_sfs_definitions():
    Nc, L = 100, 1000.0
    f = (np.array([0, 1, 1, 50, 99, 100]) / np.float32(Nc)).astype(np.float32)
    h = orc.histogram(f, Nc, L)
    assert h[1] == 2 and h[50] == 1 and h[99] == 1
    assert h[0] == 2 + (L - len(f))  # lost + fixed + monomorphic sites
    n = 10
    sfs = orc.sfs(f, n, L)
    want = np.zeros(n + 1)
    for p in f:
        if 0 < p < 1:
            want += stats.binom.pmf(np.arange(n + 1), n, float(p))
    np.testing.assert_allclose(sfs[1:], want[1:n], rtol=1e-12)
    assert abs(sfs[0] - (want[0] + want[n] + 2 + (L - len(f)))) < 1e-9
    assert abs(sfs.sum() - L) < 1e-6  # every site lands in exactly one bin


def test_single_population_run_is_neutral_equilibrium_like():
    """Oracle sanity: a neutral population started at equilibrium keeps theta * H_{2N-1} mutations."""
    Nc, L, mu = 2000, 1e6, 1e-8
    rng = np.random.default_rng(1)
    i = np.arange(1, Nc)
    x = np.repeat((i / Nc).astype(np.float32), rng.poisson(2 * mu * L / (i / Nc)))
    f, ids, mg = orc.run_single(x, first_gen=0, num_gens=200, Nc=Nc, F=0.0, h=0.5, s=0.0, mu=mu, num_sites=L,
                                seed1=1, seed2=2, compact_interval=25, capacity=4 * len(x) + 10000)
    expected = 2 * mu * L * Nc * np.sum(1.0 / i)
    assert abs(len(f) - expected) < 5 * math.sqrt(expected) + 0.05 * expected
    assert mg > 200 * 0.8 * expected


def test_joint_oracle_matches_brute_force():
    """The joint-SFS restatement against an explicit loop over mutations and sample counts."""
    import math
    from oracle.joint_oracle import joint_sfs
    rng = np.random.default_rng(8)
    Nc = 50
    fa = (rng.integers(0, Nc + 1, 40) / Nc).astype(np.float32)
    fb = (rng.integers(0, Nc + 1, 40) / Nc).astype(np.float32)
    na, nb, L = 5, 4, 1000.0
    want = np.zeros((na + 1, nb + 1))
    want[0, 0] = L - 40
    for pa, pb in zip(fa.astype(np.float64), fb.astype(np.float64)):
        for i in range(na + 1):
            for j in range(nb + 1):
                want[i, j] += (math.comb(na, i) * pa ** i * (1 - pa) ** (na - i) *
                               math.comb(nb, j) * pb ** j * (1 - pb) ** (nb - j))
    got = joint_sfs(fa, fb, na, nb, L)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)
    assert abs(got.sum() - L) < 1e-9


def test_joint3_oracle_matches_brute_force():
    """The three-population joint-SFS restatement against an explicit loop."""
    import math
    from oracle.joint_oracle import joint3_sfs
    rng = np.random.default_rng(9)
    Nc = 40
    f = [(rng.integers(0, Nc + 1, 25) / Nc).astype(np.float32) for _ in range(3)]
    n, L = (3, 4, 2), 500.0
    want = np.zeros((n[0] + 1, n[1] + 1, n[2] + 1))
    want[0, 0, 0] = L - 25

    def pmf(p, n_, k):
        return math.comb(n_, k) * p ** k * (1 - p) ** (n_ - k)

    for pa, pb, pc in zip(*(x.astype(np.float64) for x in f)):
        for i in range(n[0] + 1):
            for j in range(n[1] + 1):
                for k in range(n[2] + 1):
                    want[i, j, k] += pmf(pa, n[0], i) * pmf(pb, n[1], j) * pmf(pc, n[2], k)
    got = joint3_sfs(*f, *n, L)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)
    assert abs(got.sum() - L) < 1e-9
