"""Python handle on the C ABI: one gf_engine, its simulation and its Spectrum calls.

This is plumbing for tests and benchmarks; the drop-in API for reference users is the C++ front-end
in include/3P/ (GO_Fish::run_sim, Sim_Model, Spectrum).  `constant_generations` builds the same
per-generation records that GO_Fish::run_sim packs for a constant model (go_fish_impl.cuh:645-714).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _capi
from ._capi import GEN_DTYPE, MAX_POPULATIONS, MSE_DTYPE, GoFishError, SimConfig, ptr


class Engine:
    """One gf_engine: a device, a stream and the buffers of one simulation."""

    def __init__(self, device: int = -1, stream: int | None = None):
        self.lib = _capi.load()
        h = ctypes.c_void_p()
        st = self.lib.gf_engine_create(device, ctypes.c_void_p(stream) if stream else None, ctypes.byref(h))
        if st != _capi.GF_OK:
            raise GoFishError(st, "gf_engine_create failed")
        self.h = h
        self.P = 1
        self.num_sites = 0.0

    def close(self) -> None:
        if self.h:
            self.lib.gf_engine_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        if st != _capi.GF_OK:
            raise GoFishError(st, self.lib.gf_engine_last_error(self.h).decode())

    @property
    def device(self) -> int:
        return self.lib.gf_engine_device(self.h)

    # ---- simulation lifecycle ----
    def _config(self, seed1, seed2, num_sites, P, compact_interval, reserve):
        self.P = P
        self.num_sites = float(num_sites)
        return SimConfig(int(np.int32(np.uint32(seed1 & 0xFFFFFFFF))), int(np.int32(np.uint32(seed2 & 0xFFFFFFFF))),
                         float(num_sites), int(P), int(compact_interval), int(reserve))

    def begin_blank(self, *, seed1, seed2, num_sites, P=1, compact_interval=35, reserve=0, start_generation=0):
        cfg = self._config(seed1, seed2, num_sites, P, compact_interval, reserve)
        self._check(self.lib.gf_sim_begin_blank(self.h, ctypes.byref(cfg), start_generation))

    def begin_from_state(self, freq: np.ndarray, ids: np.ndarray | None, *, seed1, seed2, num_sites,
                         compact_interval=35, preserve=False, reserve=0, start_generation=0,
                         extinct: np.ndarray | None = None):
        freq = np.ascontiguousarray(freq, dtype=np.float32)
        if freq.ndim == 1:
            freq = freq[None, :]
        P, M = freq.shape
        if ids is None:
            ids = np.zeros((M, 4), dtype=np.int32)
            ids[:, 2] = np.arange(1, M + 1)
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        ext = None if extinct is None else np.ascontiguousarray(extinct, dtype=np.uint8)
        cfg = self._config(seed1, seed2, num_sites, P, compact_interval, reserve)
        self._check(self.lib.gf_sim_begin_from_state(self.h, ctypes.byref(cfg), start_generation, ptr(freq), ptr(ids),
                                                     M, ptr(ext), int(preserve)))

    def begin_mse(self, pops: np.ndarray, *, seed1, seed2, num_sites, compact_interval=35, preserve=False,
                  reserve=0):
        pops = np.ascontiguousarray(pops, dtype=MSE_DTYPE)
        cfg = self._config(seed1, seed2, num_sites, len(pops), compact_interval, reserve)
        self._check(self.lib.gf_sim_begin_mse(self.h, ctypes.byref(cfg), ptr(pops), int(preserve)))

    def run(self, gens: np.ndarray) -> None:
        gens = np.ascontiguousarray(gens, dtype=GEN_DTYPE)
        self._check(self.lib.gf_sim_run(self.h, ptr(gens), len(gens)))

    def num_mutations(self) -> int:
        m = ctypes.c_int32()
        self._check(self.lib.gf_sim_num_mutations(self.h, ctypes.byref(m)))
        return m.value

    def read_state(self, with_ids: bool = True):
        M = self.num_mutations()
        freq = np.empty((self.P, max(M, 1)), dtype=np.float32)
        ids = np.empty((max(M, 1), 4), dtype=np.int32) if with_ids else None
        got = ctypes.c_int32()
        self._check(self.lib.gf_sim_read_state(self.h, ptr(freq), ptr(ids), max(M, 1), ctypes.byref(got)))
        M = got.value
        return freq[:, :M], (ids[:M] if with_ids else None)

    def read_state_into(self, freq_out: np.ndarray, ids_out: np.ndarray | None = None) -> int:
        """Copy the current state into caller-owned arrays and return M: `freq_out` (fp32, at least
        P * capacity values) receives the rows packed as [P][M], `ids_out` ([>= M][4] int32) the
        reference's mutation IDs.  Page-locked arrays make both copies direct DMA transfers."""
        got = ctypes.c_int32()
        cap = freq_out.size // max(self.P, 1)
        if ids_out is not None and ids_out.shape[0] < cap:
            cap = ids_out.shape[0]
        self._check(self.lib.gf_sim_read_state(self.h, ptr(freq_out), ptr(ids_out), int(cap), ctypes.byref(got)))
        return got.value

    def sample_begin(self, freq_out: np.ndarray, ids_out: np.ndarray | None = None) -> None:
        """Start copying the current state into caller-owned arrays while later generations run
        (gf_sim_sample_begin): the rows arrive packed as [P][M] at the front of `freq_out`, the IDs in the
        first M rows of `ids_out`.  Page-locked arrays keep the copies asynchronous; leave them untouched
        until sample_wait, which returns M."""
        cap = freq_out.size // max(self.P, 1)
        if ids_out is not None and ids_out.shape[0] < cap:
            cap = ids_out.shape[0]
        self._check(self.lib.gf_sim_sample_begin(self.h, ptr(freq_out), ptr(ids_out), int(cap)))

    def sample_wait(self, with_bytes: bool = False):
        """M of the sample in flight (and, with_bytes, the bytes its copies moved)."""
        got = ctypes.c_int32()
        nbytes = ctypes.c_int64()
        self._check(self.lib.gf_sim_sample_wait(self.h, ctypes.byref(got), ctypes.byref(nbytes)))
        return (got.value, nbytes.value) if with_bytes else got.value

    def device_state(self):
        p = ctypes.c_void_p()
        stride = ctypes.c_int32()
        m = ctypes.c_int32()
        self._check(self.lib.gf_sim_device_state(self.h, ctypes.byref(p), ctypes.byref(stride), ctypes.byref(m)))
        return p.value, stride.value, m.value

    def stats(self) -> dict:
        st = _capi.SimStats()
        self._check(self.lib.gf_sim_stats_read(self.h, ctypes.byref(st)))
        return {"mutation_generations": st.mutation_generations, "generations": st.generations,
                "compactions": st.compactions, "kernel_launches": st.kernel_launches}

    def set_tuning(self, draw_strategy: int = 0, blocks_per_sm: int = 0, windows: int = 1) -> None:
        """Launch choices that never change results (gf_engine_set_tuning): draw_strategy 0 = each thread
        draws its lanes in order, 1 = warp-pooled draws, 2 = a thread's lanes grouped by sampler branch,
        3 = the normal approximation of a quad's lanes first, 4 = the normal approximation per thread
        and the warp's search draws pooled; blocks_per_sm caps the resident drift
        blocks (0 = occupancy maximum); windows = 0 runs one launch per generation."""
        t = _capi.Tuning(int(draw_strategy), int(blocks_per_sm), int(windows))
        self._check(self.lib.gf_engine_set_tuning(self.h, ctypes.byref(t)))

    def get_tuning(self) -> dict:
        t = _capi.Tuning()
        self._check(self.lib.gf_engine_get_tuning(self.h, ctypes.byref(t)))
        return {"draw_strategy": t.draw_strategy, "blocks_per_sm": t.blocks_per_sm, "windows": t.windows}

    def set_profiling(self, enable: bool) -> None:
        self._check(self.lib.gf_engine_set_profiling(self.h, int(enable)))

    def read_profile(self) -> dict:
        kt = _capi.KernelTimes()
        self._check(self.lib.gf_engine_read_profile(self.h, ctypes.byref(kt)))
        return {"drift_ms": kt.drift_ms, "drift_launches": kt.drift_launches, "compact_ms": kt.compact_ms,
                "compactions": kt.compactions}

    # ---- batched replicates ----
    def batch_begin(self, reps) -> None:
        arr = (_capi.Replicate * len(reps))(*reps)
        self._batch = arr
        self._check(self.lib.gf_batch_begin(self.h, ctypes.cast(arr, ctypes.c_void_p), len(reps)))

    def batch_set_record_budget(self, records: int) -> None:
        self._check(self.lib.gf_batch_set_record_budget(self.h, int(records)))

    def batch_run(self, max_super_steps: int = 0) -> int:
        active = ctypes.c_int32()
        self._check(self.lib.gf_batch_run(self.h, int(max_super_steps), ctypes.byref(active)))
        return active.value

    def batch_read_state(self, r: int, with_ids: bool = True):
        """(frequencies, IDs, generation) of replicate r."""
        M = ctypes.c_int32()
        gen = ctypes.c_int32()
        self.lib.gf_batch_read_state(self.h, r, None, None, 0, ctypes.byref(M), ctypes.byref(gen))  # size query
        n = M.value
        freq = np.empty(max(n, 1), dtype=np.float32)
        ids = np.empty((max(n, 1), 4), dtype=np.int32) if with_ids else None
        self._check(self.lib.gf_batch_read_state(self.h, r, ptr(freq), ptr(ids), max(n, 1), ctypes.byref(M),
                                                 ctypes.byref(gen)))
        return freq[:n], (ids[:n] if with_ids else None), gen.value

    def batch_sfs(self, n: int, R: int) -> np.ndarray:
        out = np.empty((R, n), dtype=np.float32)
        self._check(self.lib.gf_batch_sfs(self.h, int(n), ptr(out)))
        return out

    def batch_stats(self) -> dict:
        st = _capi.BatchStats()
        self._check(self.lib.gf_batch_stats_read(self.h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in _capi.BatchStats._fields_}

    def synchronize(self) -> None:
        self._check(self.lib.gf_engine_synchronize(self.h))

    # ---- Spectrum ----
    def population_histogram(self, freq: np.ndarray, Nc: int, num_sites: float) -> np.ndarray:
        freq = np.ascontiguousarray(freq, dtype=np.float32)
        out = np.empty(Nc, dtype=np.float32)
        self._check(self.lib.gf_population_histogram(self.h, ptr(freq), len(freq), Nc, float(num_sites), ptr(out)))
        return out

    def site_frequency_spectrum(self, freq: np.ndarray, Nc: int, n: int, num_sites: float) -> np.ndarray:
        freq = np.ascontiguousarray(freq, dtype=np.float32)
        out = np.empty(n, dtype=np.float32)
        self._check(self.lib.gf_site_frequency_spectrum(self.h, ptr(freq), len(freq), Nc, n, float(num_sites),
                                                        ptr(out)))
        return out

    def joint_site_frequency_spectrum(self, freq_a: np.ndarray, freq_b: np.ndarray, n_a: int, n_b: int,
                                      num_sites: float) -> np.ndarray:
        """Expected joint SFS [n_a + 1][n_b + 1] of two populations' rows of the same mutations."""
        fa = np.ascontiguousarray(freq_a, dtype=np.float32)
        fb = np.ascontiguousarray(freq_b, dtype=np.float32)
        if fa.shape != fb.shape:
            raise ValueError("the two rows must hold the same mutations")
        out = np.empty((n_a + 1, n_b + 1), dtype=np.float32)
        self._check(self.lib.gf_joint_site_frequency_spectrum(self.h, ptr(fa), ptr(fb), len(fa), int(n_a), int(n_b),
                                                              float(num_sites), ptr(out)))
        return out

    def joint3_site_frequency_spectrum(self, freq_a: np.ndarray, freq_b: np.ndarray, freq_c: np.ndarray, n_a: int,
                                       n_b: int, n_c: int, num_sites: float) -> np.ndarray:
        """Expected joint SFS [n_a + 1][n_b + 1][n_c + 1] of three populations' rows of the same mutations."""
        fa = np.ascontiguousarray(freq_a, dtype=np.float32)
        fb = np.ascontiguousarray(freq_b, dtype=np.float32)
        fc = np.ascontiguousarray(freq_c, dtype=np.float32)
        if fa.shape != fb.shape or fa.shape != fc.shape:
            raise ValueError("the three rows must hold the same mutations")
        out = np.empty((n_a + 1, n_b + 1, n_c + 1), dtype=np.float32)
        self._check(self.lib.gf_joint3_site_frequency_spectrum(self.h, ptr(fa), ptr(fb), ptr(fc), len(fa), int(n_a),
                                                               int(n_b), int(n_c), float(num_sites), ptr(out)))
        return out

    def joint_site_frequency_spectrum_device(self, d_freq_a: int, d_freq_b: int, M: int, n_a: int, n_b: int,
                                             num_sites: float, d_out: int) -> None:
        self._check(self.lib.gf_joint_site_frequency_spectrum_device(
            self.h, ctypes.c_void_p(d_freq_a), ctypes.c_void_p(d_freq_b), int(M), int(n_a), int(n_b),
            float(num_sites), ctypes.c_void_p(d_out)))

    def site_frequency_spectrum_device(self, d_freq: int, M: int, Nc: int, n: int, num_sites: float,
                                       d_out: int) -> None:
        self._check(self.lib.gf_site_frequency_spectrum_device(self.h, ctypes.c_void_p(d_freq), M, Nc, n,
                                                               float(num_sites), ctypes.c_void_p(d_out)))


def replicate(*, seed1, seed2, num_sites, mu, F, h, s, N0, growth_rate=0.0, N_min=1, N_max=None,
              num_generations, compact_interval=25, sel_slope=0.0):
    """A gf_replicate record (batched engine)."""
    return _capi.Replicate(int(np.int32(np.uint32(seed1 & 0xFFFFFFFF))), int(np.int32(np.uint32(seed2 & 0xFFFFFFFF))),
                           float(num_sites), float(mu), float(F), float(h), float(sel_slope), float(s), int(N0),
                           float(growth_rate), int(N_min), int(N_max if N_max is not None else N0),
                           int(num_generations), int(compact_interval))


def replicate_population(rep, generation: int) -> int:
    return _capi.load().gf_replicate_population(ctypes.byref(rep), int(generation))


def replicate_plain_generations(rep, first: int = 1) -> np.ndarray:
    """Per-generation records of the plain engine run equivalent to a batched replicate."""
    G = rep.num_generations
    gens = np.zeros(G, dtype=GEN_DTYPE)
    g = np.arange(first, first + G)
    gens["generation"] = g
    ci = rep.compact_interval
    gens["compact"] = (((g % ci) == 0) | (g == first + G - 1)).astype(np.int32)
    N = np.empty(G, dtype=np.int32)
    _capi.load().gf_replicate_population_table(ctypes.byref(rep), int(first), int(G), N.ctypes.data)
    N = N.astype(np.int64)
    Nc = (np.float32(2) * N.astype(np.float32) / np.float32(np.float32(1) + np.float32(rep.F))).astype(np.int32)
    pops = gens["pop"]
    pops["Nchrom_e"][:, 0] = Nc
    pops["drift"][:, 0] = 1
    pops["alive"][:, 0] = (N > 0).astype(np.int32)
    pops["mutate"][:, 0] = 1
    pops["mu"][:, 0] = rep.mu
    pops["F"][:, 0] = rep.F
    pops["h"][:, 0] = rep.h
    pops["sel_slope"][:, 0] = rep.sel_slope
    pops["sel_intercept"][:, 0] = rep.sel_intercept
    gens["migration"][:, 0] = 1.0
    return gens


def replicate_mse_pops(rep) -> np.ndarray:
    pops = np.zeros(1, dtype=MSE_DTYPE)
    N0 = replicate_population(rep, 0)
    pops["N_ind"] = N0
    pops["Nchrom_e"] = int(np.float32(2 * N0) / np.float32(np.float32(1) + np.float32(rep.F)))
    pops["mu"] = rep.mu
    pops["F"] = rep.F
    pops["h"] = rep.h
    pops["sel_slope"] = rep.sel_slope
    pops["sel_intercept"] = rep.sel_intercept
    return pops


def new_mutation_count(seed1, seed2, mu, Nchrom_e, num_sites, generation, pop) -> int:
    lib = _capi.load()
    return lib.gf_new_mutation_count(int(np.int32(np.uint32(seed1 & 0xFFFFFFFF))),
                                     int(np.int32(np.uint32(seed2 & 0xFFFFFFFF))), float(mu), int(Nchrom_e),
                                     float(num_sites), int(generation), int(pop))


@dataclass
class ConstantModel:
    """A constant single-population model (demography_constant, F/mu/h constant, selection_constant)."""
    N: int                 # individuals
    F: float = 0.0
    h: float = 0.5
    s: float = 0.0         # selection coefficient (use from_gamma for effective selection)
    mu: float = 1e-9
    P: int = 1
    m: float = 0.0         # migration_constant_equal rate

    @property
    def Nchrom_e(self) -> int:
        # 2 * N / (1 + F) in float, truncated, as the reference evaluates it (go_fish_impl.cuh:659)
        return int(np.float32(2 * self.N) / np.float32(np.float32(1) + np.float32(self.F)))

    @staticmethod
    def s_from_gamma(gamma: float, N: int, F: float) -> float:
        # selection_constant(gamma, demography, F) (template_inline_simulation_functors.cuh:52)
        denom = np.float32(2 * N) / np.float32(np.float32(1) + np.float32(F))
        return float(np.float32(gamma) / np.float32(denom))

    def mse_pops(self) -> np.ndarray:
        pops = np.zeros(self.P, dtype=MSE_DTYPE)
        pops["N_ind"] = self.N
        pops["Nchrom_e"] = self.Nchrom_e
        pops["mu"] = self.mu
        pops["F"] = self.F
        pops["h"] = self.h
        pops["sel_slope"] = 0.0
        pops["sel_intercept"] = self.s
        return pops

    def migration_rate(self, frm: int, to: int) -> float:
        if frm == to:
            return float(np.float32(1) - np.float32(self.P - 1) * np.float32(self.m))
        return float(np.float32(self.m)) if self.P > 1 else 0.0


def constant_generations(model: ConstantModel, first: int, count: int, compact_interval: int,
                         final_generation: int | None = None, next_compact: int | None = None,
                         mutate: bool = True) -> np.ndarray:
    """Per-generation records for generations first .. first+count-1 of a constant model, with the
    reference's compaction schedule (every compact_interval generations and at the final one)."""
    gens = np.zeros(count, dtype=GEN_DTYPE)
    P = model.P
    final = final_generation if final_generation is not None else first + count - 1
    nc = next_compact if next_compact is not None else (first - 1) + compact_interval
    mig = np.zeros(MAX_POPULATIONS * MAX_POPULATIONS, dtype=np.float32)
    for f in range(P):
        for t in range(P):
            mig[f * MAX_POPULATIONS + t] = model.migration_rate(f, t)
    g = np.arange(first, first + count, dtype=np.int64)
    gens["generation"] = g
    compact = np.zeros(count, dtype=bool)
    if compact_interval > 0:
        # compaction at nc, nc + ci, ... and at the final generation
        on_schedule = (g >= nc) & (((g - nc) % compact_interval) == 0)
        compact = on_schedule | (g == final)
    gens["compact"] = compact.astype(np.int32)
    pops = gens["pop"]
    pops["Nchrom_e"][:, :P] = model.Nchrom_e
    pops["drift"][:, :P] = 1
    pops["alive"][:, :P] = 1
    pops["mutate"][:, :P] = int(mutate)
    pops["mu"][:, :P] = model.mu
    pops["F"][:, :P] = model.F
    pops["h"][:, :P] = model.h
    pops["sel_slope"][:, :P] = 0.0
    pops["sel_intercept"][:, :P] = model.s
    gens["migration"][:] = mig
    return gens
