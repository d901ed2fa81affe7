"""Joint (two- and three-population) SFS on the GPU: against the CPU restatement, its marginals against
the engine's SFS and the pairwise joint SFS, total mass, and on simulated multi-population states."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.joint_oracle import joint3_sfs, joint_sfs
from parallelpopgen_b200 import ConstantModel, Engine, constant_generations

pytestmark = pytest.mark.gpu


def _rows(rng, M, Nc):
    fa = (rng.integers(0, Nc + 1, M) / Nc).astype(np.float32)
    fb = (rng.integers(0, Nc + 1, M) / Nc).astype(np.float32)
    return fa, fb


@pytest.mark.parametrize("M,na,nb", [(3000, 20, 30), (517, 150, 140), (1, 1, 1), (20000, 100, 100)])
def test_joint_matches_oracle(M, na, nb):
    rng = np.random.default_rng(M + na)
    fa, fb = _rows(rng, M, 400)
    L = 1e7
    with Engine() as e:
        got = e.joint_site_frequency_spectrum(fa, fb, na, nb, L).astype(np.float64)
    want = joint_sfs(fa, fb, na, nb, L)
    # double accumulation on both sides; the output is fp32
    np.testing.assert_allclose(got, want, rtol=2e-7, atol=1e-6 * M / (na * nb) + 1e-30)
    assert abs(got.sum() - L) <= 1e-6 * L


def test_joint_without_mutations():
    with Engine() as e:
        got = e.joint_site_frequency_spectrum(np.zeros(0, np.float32), np.zeros(0, np.float32), 3, 2, 500.0)
    want = np.zeros((4, 3), np.float32)
    want[0, 0] = 500.0
    assert np.array_equal(got, want)


def test_joint_on_simulated_two_population_state():
    """Two populations with migration: the joint spectrum's marginals equal each population's SFS (bins
    1 .. n-1), and its total is the number of sites."""
    model = ConstantModel(N=2000, mu=1e-8, P=2, m=1e-3)
    L = 2e6
    with Engine() as e:
        e.begin_mse(model.mse_pops(), seed1=3, seed2=4, num_sites=L, compact_interval=20)
        e.run(constant_generations(model, 1, 300, 20))
        f, _ = e.read_state(with_ids=False)
        n_a, n_b = 60, 50
        J = e.joint_site_frequency_spectrum(f[0], f[1], n_a, n_b, L).astype(np.float64)
        sa = e.site_frequency_spectrum(f[0], model.Nchrom_e, n_a, L).astype(np.float64)
        sb = e.site_frequency_spectrum(f[1], model.Nchrom_e, n_b, L).astype(np.float64)
    assert f.shape[0] == 2 and f.shape[1] > 100
    np.testing.assert_allclose(J.sum(axis=1)[1:n_a], sa[1:n_a], rtol=1e-5)
    np.testing.assert_allclose(J.sum(axis=0)[1:n_b], sb[1:n_b], rtol=1e-5)
    assert abs(J.sum() - L) <= 1e-5 * L
    # populations exchange migrants: shared variants exist off the axes
    assert J[1:n_a, 1:n_b].sum() > 0


@pytest.mark.parametrize("M,n", [(4000, (12, 9, 7)), (300, (40, 30, 20)), (1, (1, 1, 1)), (20000, (150, 3, 129))])
def test_joint3_matches_oracle(M, n):
    rng = np.random.default_rng(M + sum(n))
    fa, fb = _rows(rng, M, 300)
    fc = (rng.integers(0, 301, M) / 300).astype(np.float32)
    L = 1e7
    with Engine() as e:
        got = e.joint3_site_frequency_spectrum(fa, fb, fc, *n, L).astype(np.float64)
    want = joint3_sfs(fa, fb, fc, *n, L)
    np.testing.assert_allclose(got, want, rtol=2e-7, atol=1e-6 * M / (n[0] * n[1] * n[2]) + 1e-30)
    assert abs(got.sum() - L) <= 1e-6 * L


def test_joint3_limits_and_empty_state():
    with Engine() as e:
        got = e.joint3_site_frequency_spectrum(*(np.zeros(0, np.float32),) * 3, 2, 3, 1, 100.0)
        want = np.zeros((3, 4, 2), np.float32)
        want[0, 0, 0] = 100.0
        assert np.array_equal(got, want)
        from parallelpopgen_b200._capi import GoFishError
        with pytest.raises(GoFishError):   # 257^3 bins: beyond the three-population limit
            e.joint3_site_frequency_spectrum(*(np.full(4, 0.5, np.float32),) * 3, 256, 256, 256, 100.0)


def test_joint3_on_simulated_three_population_state():
    """Three populations with migration: summed over one population the joint spectrum equals the
    pairwise joint spectrum of the other two, and its total is the number of sites."""
    model = ConstantModel(N=1500, mu=1e-8, P=3, m=2e-3)
    L = 2e6
    with Engine() as e:
        e.begin_mse(model.mse_pops(), seed1=5, seed2=6, num_sites=L, compact_interval=20)
        e.run(constant_generations(model, 1, 300, 20))
        f, _ = e.read_state(with_ids=False)
        n = (30, 24, 18)
        J3 = e.joint3_site_frequency_spectrum(f[0], f[1], f[2], *n, L).astype(np.float64)
        J01 = e.joint_site_frequency_spectrum(f[0], f[1], n[0], n[1], L).astype(np.float64)
        J02 = e.joint_site_frequency_spectrum(f[0], f[2], n[0], n[2], L).astype(np.float64)
    assert f.shape[0] == 3 and f.shape[1] > 100
    np.testing.assert_allclose(J3.sum(axis=2), J01, rtol=1e-5, atol=1e-3)
    np.testing.assert_allclose(J3.sum(axis=1), J02, rtol=1e-5, atol=1e-3)
    assert abs(J3.sum() - L) <= 1e-5 * L
    assert J3[1:, 1:, 1:].sum() > 0     # variants shared by all three populations
