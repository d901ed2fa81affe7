"""CPU restatement of the joint (two- and three-population) SFS projection.  TEST INFRASTRUCTURE ONLY:
imported by tests/ to check the GPU path, never by the product.

The reference projects one population's frequency p onto a sample of n as C(n,k) p^k (1-p)^(n-k)
(spectrum.cu:90-139, binom_coeff and binom); the joint form multiplies the two populations'
projections of each mutation and sums over mutations, with the num_sites - M monomorphic sites at
(0, 0).  No reference file computes it (the reference's Spectrum API has single-population marginals
only), so this restatement is pinned by its own definition: a brute-force loop in the CPU tests, and
the single-population marginal property on the GPU.
"""
from __future__ import annotations

import numpy as np
from scipy.special import gammaln


def sample_pmf(p: np.ndarray, n: int) -> np.ndarray:
    """[len(p)][n + 1] binomial pmfs in float64 (point masses at p <= 0 and p >= 1)."""
    p = np.asarray(p, dtype=np.float64)
    k = np.arange(n + 1)
    lgc = gammaln(n + 1.0) - gammaln(k + 1.0) - gammaln(n - k + 1.0)
    inner = (p > 0) & (p < 1)
    out = np.zeros((len(p), n + 1))
    pi = p[inner]
    out[inner] = np.exp(lgc[None, :] + k[None, :] * np.log(pi)[:, None] + (n - k)[None, :] * np.log1p(-pi)[:, None])
    out[p <= 0, 0] = 1.0
    out[p >= 1, n] = 1.0
    return out


def joint_sfs(freq_a: np.ndarray, freq_b: np.ndarray, n_a: int, n_b: int, num_sites: float) -> np.ndarray:
    """[n_a + 1][n_b + 1] expected joint SFS (float64)."""
    A = sample_pmf(np.asarray(freq_a, dtype=np.float32), n_a)
    B = sample_pmf(np.asarray(freq_b, dtype=np.float32), n_b)
    out = A.T @ B
    out[0, 0] += float(np.float32(num_sites)) - len(freq_a)
    return out


def joint3_sfs(freq_a: np.ndarray, freq_b: np.ndarray, freq_c: np.ndarray, n_a: int, n_b: int, n_c: int,
               num_sites: float) -> np.ndarray:
    """[n_a + 1][n_b + 1][n_c + 1] expected joint SFS of three populations (float64): every mutation
    contributes the product of its three projections; the num_sites - M monomorphic sites go to (0, 0, 0)."""
    A = sample_pmf(np.asarray(freq_a, dtype=np.float32), n_a)
    B = sample_pmf(np.asarray(freq_b, dtype=np.float32), n_b)
    C = sample_pmf(np.asarray(freq_c, dtype=np.float32), n_c)
    out = np.einsum("mi,mj,mk->ijk", A, B, C, optimize=True)
    out[0, 0, 0] += float(np.float32(num_sites)) - len(freq_a)
    return out
