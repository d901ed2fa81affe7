"""ctypes wrapper of the CPU oracle (oracle/_build/liboracle.so).  TEST INFRASTRUCTURE ONLY: imported by
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arms, never by the product.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
REF_DRIVER = HERE / "_ref" / "ref_driver"
MAXP = 16

_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = ctypes.CDLL(str(LIB))
        P, I, F, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double
        U = ctypes.c_uint32
        L.or_philox.argtypes = [U, U, P, P]
        L.or_philox.restype = None
        L.or_u01.argtypes = [U]
        L.or_u01.restype = F
        L.or_normcdfinv.argtypes = [D]
        L.or_normcdfinv.restype = D
        L.or_pois_search.argtypes = [F, F]
        L.or_pois_search.restype = I
        L.or_binom_search.argtypes = [F, F, F, F]
        L.or_binom_search.restype = I
        L.or_binom_draw.argtypes = [U, F, F, F]
        L.or_binom_draw.restype = I
        L.or_pois_draw.argtypes = [F, F, F, I, I, I, I, I]
        L.or_pois_draw.restype = I
        L.or_new_mutation_count.argtypes = [I, I, F, I, F, I, I]
        L.or_new_mutation_count.restype = I
        L.or_drift.argtypes = [P, P, ctypes.c_long, I, P, I]
        L.or_drift.restype = None
        L.or_add_new.argtypes = [P, ctypes.c_long, I, P, I, I, F, I, I]
        L.or_add_new.restype = None
        L.or_compact.argtypes = [P, ctypes.c_long, I, P, I, P, I]
        L.or_compact.restype = I
        L.or_histogram.argtypes = [P, I, I, F, P]
        L.or_histogram.restype = None
        L.or_sfs.argtypes = [P, I, I, F, P]
        L.or_sfs.restype = None
        L.or_run_single.argtypes = [P, P, P, I, I, I, I, I, F, F, F, F, F, F, I, I, I, I, ctypes.POINTER(D)]
        L.or_run_single.restype = I
        L.or_max_threads.argtypes = []
        L.or_max_threads.restype = I
        _lib = L
    return _lib


class Gen(ctypes.Structure):
    _fields_ = [
        ("generation", ctypes.c_int), ("P", ctypes.c_int), ("seed1", ctypes.c_int), ("seed2", ctypes.c_int),
        ("drift", ctypes.c_int * MAXP), ("Nc", ctypes.c_int * MAXP), ("F", ctypes.c_float * MAXP),
        ("h", ctypes.c_float * MAXP), ("sel_slope", ctypes.c_float * MAXP), ("sel_intercept", ctypes.c_float * MAXP),
        ("mig", ctypes.c_float * (MAXP * MAXP)),
    ]


def i32(v: int) -> int:
    return int(np.int32(np.uint32(v & 0xFFFFFFFF)))


def philox(seed1, seed2, k, step, pop, rnd=0) -> np.ndarray:
    out = np.zeros(4, dtype=np.uint32)
    ctr = np.array([k, step, pop, rnd], dtype=np.uint64).astype(np.uint32)
    lib().or_philox(seed1 & 0xFFFFFFFF, seed2 & 0xFFFFFFFF, ctr.ctypes.data, out.ctypes.data)
    return out


def drift(prev: np.ndarray, *, generation, seed1, seed2, Nc, F=0.0, h=0.5, sel_slope=0.0, sel_intercept=0.0,
          mig=None, drift_mask=None, threads=1) -> np.ndarray:
    """One generation of migration/selection/drift for [P][M] rows (per-population parameter lists)."""
    prev = np.ascontiguousarray(prev, dtype=np.float32)
    if prev.ndim == 1:
        prev = prev[None, :]
    P, M = prev.shape
    g = Gen()
    g.generation, g.P, g.seed1, g.seed2 = generation, P, i32(seed1), i32(seed2)

    def per_pop(v):
        return list(v) if np.ndim(v) else [v] * P

    for p, (n, f, hh, a, b) in enumerate(zip(per_pop(Nc), per_pop(F), per_pop(h), per_pop(sel_slope),
                                            per_pop(sel_intercept))):
        g.drift[p] = 1 if drift_mask is None else int(drift_mask[p])
        g.Nc[p], g.F[p], g.h[p], g.sel_slope[p], g.sel_intercept[p] = int(n), f, hh, a, b
    m = np.eye(P, dtype=np.float32) if mig is None else np.asarray(mig, dtype=np.float32)
    for fr in range(P):
        for to in range(P):
            g.mig[fr * P + to] = m[fr, to]
    nxt = prev.copy()
    lib().or_drift(prev.ctypes.data, nxt.ctypes.data, M, M, ctypes.byref(g), threads)
    return nxt


def compact(freq: np.ndarray, ids: np.ndarray, alive, preserve=False):
    freq = np.ascontiguousarray(freq, dtype=np.float32).copy()
    if freq.ndim == 1:
        freq = freq[None, :]
    ids = np.ascontiguousarray(ids, dtype=np.int32).copy()
    P, M = freq.shape
    al = np.asarray(alive, dtype=np.int32)
    n = lib().or_compact(freq.ctypes.data, M, P, ids.ctypes.data, M, al.ctypes.data, int(preserve))
    return freq[:, :n], ids[:n]


def histogram(freq: np.ndarray, Nc: int, num_sites: float) -> np.ndarray:
    freq = np.ascontiguousarray(freq, dtype=np.float32)
    out = np.zeros(Nc, dtype=np.float32)
    lib().or_histogram(freq.ctypes.data, len(freq), Nc, num_sites, out.ctypes.data)
    return out


def sfs(freq: np.ndarray, n: int, num_sites: float) -> np.ndarray:
    freq = np.ascontiguousarray(freq, dtype=np.float32)
    out = np.zeros(n, dtype=np.float64)
    lib().or_sfs(freq.ctypes.data, len(freq), n, num_sites, out.ctypes.data)
    return out


def new_mutation_count(seed1, seed2, mu, Nc, num_sites, generation, pop) -> int:
    return lib().or_new_mutation_count(i32(seed1), i32(seed2), mu, Nc, num_sites, generation, pop)


def run_single(freq0: np.ndarray, *, first_gen, num_gens, Nc, F, h, s, mu, num_sites, seed1, seed2,
               compact_interval, capacity, threads=1):
    """Whole single-population run on the CPU; returns (final freq, ids, mutation-generations)."""
    cap = int(capacity)
    M = len(freq0)
    freq = np.zeros(cap, dtype=np.float32)
    freq[:M] = freq0
    scratch = np.zeros(cap, dtype=np.float32)
    ids = np.zeros((cap, 4), dtype=np.int32)
    ids[:M, 2] = np.arange(1, M + 1)
    mg = ctypes.c_double()
    n = lib().or_run_single(freq.ctypes.data, scratch.ctypes.data, ids.ctypes.data, M, cap, first_gen, num_gens, Nc,
                            F, h, 0.0, s, mu, num_sites, i32(seed1), i32(seed2), compact_interval, threads,
                            ctypes.byref(mg))
    if n < 0:
        raise RuntimeError("oracle capacity exceeded")
    return freq[:n], ids[:n], mg.value


def max_threads() -> int:
    return lib().or_max_threads()
