"""Edge cases of the engine on the GPU: the largest population count (16) with migration against the
CPU restatement, an extinction that empties the state, and the status codes of invalid calls (no call
here may fault the GPU: every rejection happens on the host)."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import oracle.oracle as orc
from parallelpopgen_b200 import ConstantModel, Engine, GoFishError, constant_generations
from parallelpopgen_b200._capi import GEN_DTYPE, MAX_POPULATIONS, MSE_DTYPE

pytestmark = pytest.mark.gpu
SEED1, SEED2 = 0xBEEF, 0xDECAF


def test_sixteen_populations_with_migration_match_oracle():
    P, M, Nc = MAX_POPULATIONS, 20003, 4000
    rng = np.random.default_rng(16)
    x = (rng.integers(0, Nc + 1, size=(P, M)) / Nc).astype(np.float32)
    mig = rng.uniform(0.0, 0.02, size=(P, P)).astype(np.float32)
    np.fill_diagonal(mig, 0.0)
    for to in range(P):                                  # proportions into each population sum to 1
        mig[to, to] = np.float32(1.0) - mig[:, to].sum(dtype=np.float32)
    g = np.zeros(1, dtype=GEN_DTYPE)
    g["generation"] = 5
    pops = g["pop"][0]
    pops["Nchrom_e"][:P] = Nc
    pops["drift"][:P] = pops["alive"][:P] = 1
    pops["mu"][:P], pops["F"][:P], pops["h"][:P] = 1e-9, 0.0, 0.5
    for f in range(P):
        for t in range(P):
            g["migration"][0][f * MAX_POPULATIONS + t] = mig[f, t]
    with Engine() as e:
        e.begin_from_state(x, None, seed1=SEED1, seed2=SEED2, num_sites=1e6, compact_interval=0)
        e.run(g)
        mine, _ = e.read_state(with_ids=False)
    ref = orc.drift(x, generation=5, seed1=SEED1, seed2=SEED2, Nc=Nc, mig=mig)
    cm = np.rint(mine.astype(np.float64) * Nc)
    cr = np.rint(ref.astype(np.float64) * Nc)
    diff = np.abs(cm - cr)
    assert mine.shape == (P, M)
    assert diff.max() <= 1 and (diff > 0).mean() <= 1e-2, (diff.max(), (diff > 0).mean())


def test_seventeen_populations_are_rejected():
    pops = np.zeros(MAX_POPULATIONS + 1, dtype=MSE_DTYPE)
    pops["N_ind"], pops["Nchrom_e"], pops["mu"], pops["h"] = 100, 200, 1e-9, 0.5
    with Engine() as e:
        with pytest.raises(GoFishError) as err:
            e.begin_mse(pops, seed1=1, seed2=2, num_sites=1e5)
        assert "INVALID_ARGUMENT" in str(err.value)


def test_extinction_empties_the_state():
    """The population dies at generation 40: every mutation is lost, the next compaction leaves no slot,
    and reading and histogramming the empty state work."""
    model = ConstantModel(N=2000, mu=1e-8)
    gens = constant_generations(model, 1, 80, 10)
    pop = gens["pop"][:, 0]
    pop["Nchrom_e"][39:] = 0
    pop["alive"][39:] = 0
    pop["mutate"][39:] = 0
    pop["drift"][40:] = 0                             # extinct after the extinction generation
    with Engine() as e:
        e.begin_mse(model.mse_pops(), seed1=3, seed2=4, num_sites=1e6, compact_interval=10)
        e.run(gens[:30])
        assert e.num_mutations() > 0
        e.run(gens[30:])
        f, ids = e.read_state()
        assert f.shape == (1, 0) and ids.shape == (0, 4)
        h = e.population_histogram(np.zeros(0, np.float32), 100, 1e6)
    assert h[0] == 1e6 and not h[1:].any()


def test_invalid_calls_return_status_codes():
    with Engine() as e:
        lib, h = e.lib, e.h
        g = np.zeros(1, dtype=GEN_DTYPE)
        assert lib.gf_sim_run(h, g.ctypes.data, 1) == 5                       # GF_ERR_STATE: no simulation
        model = ConstantModel(N=500, mu=1e-8)
        e.begin_mse(model.mse_pops(), seed1=1, seed2=2, num_sites=1e6, compact_interval=10)
        e.run(constant_generations(model, 1, 20, 10))
        M = e.num_mutations()
        assert M > 2
        buf = np.zeros(2, np.float32)
        got = ctypes.c_int32()
        assert lib.gf_sim_read_state(h, buf.ctypes.data, None, 2, ctypes.byref(got)) == 4   # GF_ERR_CAPACITY
        assert got.value == M
        f, _ = e.read_state(with_ids=False)
        with pytest.raises(GoFishError):                                      # sample size >= Nchrom_e
            e.site_frequency_spectrum(f[0], model.Nchrom_e, model.Nchrom_e, 1e6)
        with pytest.raises(GoFishError):
            e.joint_site_frequency_spectrum(f[0], f[0], 0, 10, 1e6)
        # the engine is still usable after every rejection
        e.run(constant_generations(model, 21, 5, 10, next_compact=30))
        assert e.num_mutations() > 0
