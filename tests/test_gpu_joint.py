"""Joint (two-population) SFS on the GPU: against the CPU restatement, its single-population marginals
against the engine's SFS, total mass, and on a simulated two-population state."""
from __future__ import annotations

import numpy as np
import pytest

from oracle.joint_oracle import joint_sfs
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
