"""Statistical oracle: the neutral constant-size mean SFS over 256 seeded replicates against the
Poisson-random-field expectation E[xi_i] = theta / i, theta = 2 mu Nchrom_e L (here 800).

Single-population runs at N = 1e4 (Nchrom_e = 2e4), mu = 1e-9, L = 2e7, MSE start, 1000 generations,
compaction every 35, sample SFS n = 100 -- run as one batch of replicates (each replicate equals the
plain engine run of its seeds bit for bit).  Per bin: |z| < 4.5 against the replicate standard error
(99 bins); where that error resolves 1 % (SE < 0.25 % of the expectation) the mean must be within 1 %;
the total number of segregating sites in the sample must be within 1 % of theta * H_99."""
from __future__ import annotations

import numpy as np
import pytest

from parallelpopgen_b200 import Engine, replicate

pytestmark = pytest.mark.gpu


def test_neutral_mean_sfs_matches_theta_over_i():
    R, N, mu, L, n = 256, 10_000, 1e-9, 2e7, 100
    reps = [replicate(seed1=0xBEEF + 7 * r, seed2=0xDECAF + 13 * r, num_sites=L, mu=mu, F=0.0, h=0.5, s=0.0, N0=N,
                      num_generations=1000, compact_interval=35) for r in range(R)]
    with Engine() as e:
        e.batch_begin(reps)
        assert e.batch_run() == 0
        sfs = e.batch_sfs(n, R).astype(np.float64)[:, 1:n]     # bins 1..99
    theta = 2 * mu * (2 * N) * L
    i = np.arange(1, n)
    expect = theta / i
    mean = sfs.mean(axis=0)
    se = sfs.std(axis=0, ddof=1) / np.sqrt(R)
    z = (mean - expect) / se
    assert np.all(np.abs(z) < 4.5), (np.argmax(np.abs(z)) + 1, z[np.argmax(np.abs(z))])
    resolvable = se < 0.0025 * expect
    assert resolvable.sum() >= 5
    assert np.all(np.abs(mean[resolvable] / expect[resolvable] - 1) < 0.01), mean[resolvable] / expect[resolvable]
    total = mean.sum()
    print(f"neutral SFS: max |z| {np.abs(z).max():.2f} (bin {np.argmax(np.abs(z)) + 1}), {resolvable.sum()} bins "
          f"resolve 1 %, their largest deviation {np.abs(mean[resolvable] / expect[resolvable] - 1).max():.4f}, "
          f"total / (theta H_99) = {total / (theta * np.sum(1.0 / i)):.5f}")
    assert abs(total / (theta * np.sum(1.0 / i)) - 1) < 0.01, total / (theta * np.sum(1.0 / i))
