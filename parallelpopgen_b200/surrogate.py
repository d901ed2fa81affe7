"""SFS surrogate: a 6 -> 512 x 4 -> 99 GELU network (bf16 tensor-core GEMMs, fp32 accumulation, Adam)
that maps model parameters to the log of the normalised expected SFS of a sample of 100, trained only on
spectra the batched simulator produces, with the simulator as the fallback outside its support.

The reference answers every SFS query by simulation: GO_Fish::run_sim (go_fish.cuh:280) followed by
Spectrum::site_frequency_spectrum (spectrum.h:90).  `Surrogate.query` is the drop-in for that pair of
calls on the parameter family below; `simulate_spectra` is the simulator side (the batched engine,
whose replicates equal plain GO_Fish runs bit for bit).

Parameter family (one population, MSE start at N0, then exponential growth for T*2*N0 generations):
    log N0 in [log 1e3, log 1e4]      gamma = 2 N s (selection_constant semantics) in [-100, 10]
    h in [0, 1]                        F in [0, 0.5]
    r in [-0.001, 0.01] per generation, N clamped to [N0/10, 10 N0]      T in [0.05, 1]
theta = 4 N0 mu L is held at THETA (mu = THETA / (4 N0 L)), so spectra differ only through the shape.
Queries with N0 in (1e4, 1e5] (the upper half of the batched-replicate workload's range) are outside
the support and go to the simulator.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass

import numpy as np

from . import _capi
from ._capi import GoFishError, MlpConfig
from .engine import ConstantModel, Engine, replicate

N_SAMPLE = 100
OUTPUTS = 99
THETA = 2000.0
NUM_SITES = 1e7
LOG_FLOOR = 1e-4          # targets are log(max(p, LOG_FLOOR)): bins below hold well under one site
GAMMA_SCALE = 5.0         # gamma enters the network as asinh(gamma / GAMMA_SCALE), rescaled to [-1, 1]

# name, low, high (inputs are scaled to [-1, 1] over these ranges)
SUPPORT = (
    ("logN", math.log(1e3), math.log(1e4)),
    ("gamma", -100.0, 10.0),
    ("h", 0.0, 1.0),
    ("F", 0.0, 0.5),
    ("r", -0.001, 0.01),
    ("T", 0.05, 1.0),
)
LOW = np.array([s[1] for s in SUPPORT])
HIGH = np.array([s[2] for s in SUPPORT])


def param_count() -> int:
    return int(_capi.load().gf_mlp_param_count())


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform hidden layers, a small output layer, zero biases (flat, in the C layout)."""
    rng = np.random.default_rng(seed)
    shapes = [(512, 6), (512, 512), (512, 512), (512, 512), (99, 512)]
    parts = []
    for i, (r, c) in enumerate(shapes):
        bound = math.sqrt(6.0 / c) if i < 4 else math.sqrt(1.0 / c)
        parts.append(rng.uniform(-bound, bound, r * c).astype(np.float32))
        parts.append(np.zeros(r, np.float32))
    return np.concatenate(parts)


class Mlp:
    """The network's device state (C ABI: include/gf_surrogate.h).  Inputs and outputs are CUDA
    float32 tensors (torch) or raw device pointers."""

    def __init__(self, capacity: int = 4096, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999,
                 eps: float = 1e-8, weight_decay: float = 0.0, device: int = 0, stream=None):
        self.lib = _capi.load()
        self.capacity = capacity
        cfg = MlpConfig(int(capacity), float(lr), float(beta1), float(beta2), float(eps), float(weight_decay))
        h = ctypes.c_void_p()
        st = self.lib.gf_mlp_create(int(device), stream, ctypes.byref(cfg), ctypes.byref(h))
        if st != 0:
            raise GoFishError(st, "gf_mlp_create failed")
        self.h = h

    def close(self):
        if self.h:
            self.lib.gf_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != 0:
            raise GoFishError(st, self.lib.gf_mlp_last_error(self.h).decode())

    def set_params(self, vec: np.ndarray):
        v = np.ascontiguousarray(vec, dtype=np.float32)
        self._check(self.lib.gf_mlp_set_params(self.h, v.ctypes.data, len(v)))

    def get_params(self) -> np.ndarray:
        v = np.empty(param_count(), np.float32)
        self._check(self.lib.gf_mlp_get_params(self.h, v.ctypes.data, len(v)))
        return v

    def set_learning_rate(self, lr: float):
        self._check(self.lib.gf_mlp_set_learning_rate(self.h, float(lr)))

    def forward_ptr(self, d_x: int, batch: int, d_y: int):
        self._check(self.lib.gf_mlp_forward(self.h, d_x, int(batch), d_y))

    def forward(self, x):
        import torch
        y = torch.empty((x.shape[0], OUTPUTS), dtype=torch.float32, device=x.device)
        self.forward_ptr(x.data_ptr(), x.shape[0], y.data_ptr())
        return y

    def gradients(self, x, t):
        g = np.empty(param_count(), np.float32)
        loss = ctypes.c_float()
        self._check(self.lib.gf_mlp_gradients(self.h, x.data_ptr(), t.data_ptr(), x.shape[0], g.ctypes.data,
                                              ctypes.byref(loss)))
        return g, loss.value

    def train_step(self, x, t, d_loss: int | None = None):
        self._check(self.lib.gf_mlp_train_step(self.h, x.data_ptr(), t.data_ptr(), x.shape[0], d_loss))

    def check(self):
        self._check(self.lib.gf_mlp_check(self.h))


def bf16_gemm(a, b):
    """C = A B^T on the tensor cores (torch bf16 CUDA tensors, K-contiguous) -> fp32 tensor."""
    import torch
    M, K = a.shape
    N = b.shape[0]
    c = torch.empty((M, N), dtype=torch.float32, device=a.device)
    st = _capi.load().gf_bf16_gemm(a.data_ptr(), b.data_ptr(), M, N, K, c.data_ptr(),
                                   torch.cuda.current_stream().cuda_stream)
    if st != 0:
        raise GoFishError(st, "gf_bf16_gemm failed")
    return c


# ------------------------------------------------------------------------------------------------
# parameters <-> features, simulator side
# ------------------------------------------------------------------------------------------------
def draw_parameters(count: int, seed: int) -> np.ndarray:
    """Uniform draws over the support box: [count][6] (logN, gamma, h, F, r, T)."""
    rng = np.random.default_rng(seed)
    return LOW + (HIGH - LOW) * rng.uniform(size=(count, len(SUPPORT)))


def in_support(params: np.ndarray) -> np.ndarray:
    return np.all((params >= LOW) & (params <= HIGH), axis=1)


def draw_query_parameters(count: int, seed: int) -> np.ndarray:
    """Queries from the batched-replicate workload's distribution: log N0 uniform in [log 1e3, log 1e5],
    gamma, h, F, r as the support, T uniform over the support's range.  About half fall in the support
    (N0 <= 1e4)."""
    p = draw_parameters(count, seed)
    rng = np.random.default_rng(seed + 0x9E3779B9)
    p[:, 0] = rng.uniform(math.log(1e3), math.log(1e5), size=count)
    return p


def encode(params: np.ndarray) -> np.ndarray:
    """Network inputs: every parameter scaled linearly to [-1, 1] over the support, except gamma, which
    is scaled through asinh(gamma / 5) (the spectrum's dependence on strong selection is close to
    logarithmic in |gamma|)."""
    params = np.asarray(params, dtype=np.float64)
    x = 2.0 * (params - LOW) / (HIGH - LOW) - 1.0
    g_lo, g_hi = np.arcsinh(LOW[1] / GAMMA_SCALE), np.arcsinh(HIGH[1] / GAMMA_SCALE)
    x[:, 1] = 2.0 * (np.arcsinh(params[:, 1] / GAMMA_SCALE) - g_lo) / (g_hi - g_lo) - 1.0
    return x.astype(np.float32)


def replicate_for(p: np.ndarray, seed1: int, seed2: int, compact_interval: int = 25):
    logN, gamma, h, F, r, T = (float(v) for v in p)
    N0 = int(round(math.exp(logN)))
    mu = THETA / (4.0 * N0 * NUM_SITES)
    return replicate(seed1=seed1, seed2=seed2, num_sites=NUM_SITES, mu=mu, F=F, h=h,
                     s=ConstantModel.s_from_gamma(gamma, N0, F), N0=N0, growth_rate=r, N_min=max(N0 // 10, 1),
                     N_max=10 * N0, num_generations=max(1, int(round(T * 2 * N0))),
                     compact_interval=compact_interval)


def simulate_spectra(engine: Engine, params: np.ndarray, reps: int, seed: int, chunk: int = 8192,
                     compact_interval: int = 25, with_variance: bool = False):
    """Mean SFS (bins 1..99, expected site counts) over `reps` replicates per parameter row, from the
    batched engine.  Replicate k of row i uses seeds (seed + 2(i reps + k), seed + 2(i reps + k) + 1).
    Replicates are grouped into batches of similar length (generations), so that a batch does not wait
    on a few long replicates; the result does not depend on the grouping.  with_variance: also return
    the per-bin variance over the replicates (ddof = 1)."""
    out = np.zeros((len(params), OUTPUTS), np.float64)
    sq = np.zeros((len(params), OUTPUTS), np.float64)
    gens = np.exp(params[:, 0]) * params[:, 5]
    order = np.argsort(gens, kind="stable")
    jobs = [(int(i), k) for i in order for k in range(reps)]
    for c0 in range(0, len(jobs), chunk):
        part = jobs[c0:c0 + chunk]
        recs = []
        for i, k in part:
            base = seed + 2 * (i * reps + k)
            recs.append(replicate_for(params[i], base & 0x7FFFFFFF, (base + 1) & 0x7FFFFFFF, compact_interval))
        engine.batch_begin(recs)
        engine.batch_run()
        sfs = engine.batch_sfs(N_SAMPLE, len(recs))
        for (i, _), row in zip(part, sfs):
            v = row[1:N_SAMPLE].astype(np.float64)
            out[i] += v
            sq[i] += v * v
    mean = out / reps
    if not with_variance:
        return mean
    var = np.maximum(sq - reps * mean * mean, 0.0) / max(reps - 1, 1)
    return mean, var


def spectra_to_targets(mean_sfs: np.ndarray) -> np.ndarray:
    p = mean_sfs / np.maximum(mean_sfs.sum(axis=1, keepdims=True), 1e-30)
    return np.log(np.maximum(p, LOG_FLOOR)).astype(np.float32)


@dataclass
class TargetScale:
    """Per-bin standardisation of the log-spectrum targets: the network learns (t - mean) / std, so its
    outputs are O(1) and the bf16 rounding of its activations and weights costs a fraction of a
    standard deviation instead of a fixed fraction of |log p| (up to ~9)."""
    mean: np.ndarray
    std: np.ndarray

    @staticmethod
    def fit(targets: np.ndarray) -> "TargetScale":
        t = np.asarray(targets, dtype=np.float64)
        return TargetScale(t.mean(axis=0), np.maximum(t.std(axis=0), 1e-3))

    def apply(self, targets: np.ndarray) -> np.ndarray:
        return ((np.asarray(targets, dtype=np.float64) - self.mean) / self.std).astype(np.float32)

    def invert(self, outputs: np.ndarray) -> np.ndarray:
        return np.asarray(outputs, dtype=np.float64) * self.std + self.mean


def median_relative_error(pred_p: np.ndarray, sim_mean: np.ndarray, min_count: float = 1.0):
    """Median over (query, bin) of |pred - sim| / sim on normalised spectra, over bins whose simulated
    mean count is at least `min_count` sites per replicate.  Returns (median, fraction of bins used)."""
    sim_p = sim_mean / sim_mean.sum(axis=1, keepdims=True)
    mask = sim_mean >= min_count
    rel = np.abs(pred_p - sim_p)[mask] / sim_p[mask]
    return float(np.median(rel)), float(mask.mean())


def error_report(pred_p: np.ndarray, sim_mean: np.ndarray, sim_var: np.ndarray, reps: int,
                 max_rel_se: float = 0.10) -> dict:
    """Median per-bin relative error |pred - sim| / sim on normalised spectra:
    * over every bin whose simulated mean is nonzero ("all"),
    * over the bins the simulator's own mean resolves: standard error of the `reps`-replicate mean below
      `max_rel_se` of the mean ("resolved"), with the fraction of bins that criterion keeps.
    Bins with a zero simulated mean have no relative error and are counted separately."""
    sim_p = sim_mean / sim_mean.sum(axis=1, keepdims=True)
    nz = sim_mean > 0
    rel = np.full(sim_mean.shape, np.nan)
    rel[nz] = np.abs(pred_p[nz] - sim_p[nz]) / sim_p[nz]
    se = np.sqrt(sim_var / reps)
    resolved = nz & (se < max_rel_se * sim_mean)
    return {"median_all": float(np.median(rel[nz])), "bins_nonzero": float(nz.mean()),
            "median_resolved": float(np.median(rel[resolved])) if resolved.any() else None,
            "bins_resolved": float(resolved.mean()), "resolved_criterion": f"SE of the {reps}-replicate mean "
                                                                            f"< {max_rel_se:g} x mean"}


# ------------------------------------------------------------------------------------------------
# training and queries
# ------------------------------------------------------------------------------------------------
@dataclass
class TrainResult:
    steps: int
    seconds: float
    final_loss: float
    losses: list


def train(mlp: Mlp, x, t, steps: int, batch: int = 1024, lr: float = 1e-3, lr_min: float = 1e-5,
          seed: int = 0, log_every: int = 500) -> TrainResult:
    """Adam on minibatches drawn with replacement, cosine learning-rate decay; x, t are CUDA tensors."""
    import torch
    gen = torch.Generator(device=x.device)
    gen.manual_seed(seed)
    d_loss = torch.zeros(1, dtype=torch.float32, device=x.device)
    xb = torch.empty((batch, x.shape[1]), dtype=torch.float32, device=x.device)
    tb = torch.empty((batch, t.shape[1]), dtype=torch.float32, device=x.device)
    losses = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s in range(steps):
        mlp.set_learning_rate(lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * s / steps)))
        idx = torch.randint(0, x.shape[0], (batch,), device=x.device, generator=gen)
        torch.index_select(x, 0, idx, out=xb)
        torch.index_select(t, 0, idx, out=tb)
        mlp.train_step(xb, tb, d_loss.data_ptr())
        if log_every and (s % log_every == 0 or s == steps - 1):
            losses.append((s, float(d_loss.item())))
    torch.cuda.synchronize()
    mlp.check()
    return TrainResult(steps, time.perf_counter() - t0, losses[-1][1] if losses else float("nan"), losses)


class Surrogate:
    """SFS queries answered by the network inside its support and by the simulator outside it."""

    def __init__(self, mlp: Mlp, engine: Engine, fallback_reps: int = 64, seed: int = 0x5EED,
                 scale: TargetScale | None = None):
        self.mlp = mlp
        self.scale = scale
        self.engine = engine
        self.fallback_reps = fallback_reps
        self.seed = seed

    def predict(self, params: np.ndarray) -> np.ndarray:
        """Normalised expected SFS (bins 1..99) of in-support rows, from the network."""
        import torch
        B = len(params)
        Bp = ((B + 127) // 128) * 128
        x = np.zeros((Bp, 6), np.float32)
        x[:B] = encode(params)
        out = np.empty((B, OUTPUTS), np.float32)
        for c0 in range(0, Bp, self.mlp.capacity):
            xs = torch.from_numpy(x[c0:c0 + self.mlp.capacity]).cuda()
            y = self.mlp.forward(xs).cpu().numpy()
            n = min(len(y), B - c0)
            if n > 0:
                out[c0:c0 + n] = y[:n]
        logp = self.scale.invert(out) if self.scale is not None else out.astype(np.float64)
        p = np.exp(logp)
        return p / p.sum(axis=1, keepdims=True)

    def query(self, params: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        """(normalised SFS per row, routed_to_simulator mask)."""
        params = np.atleast_2d(np.asarray(params, dtype=np.float64))
        ok = in_support(params)
        res = np.zeros((len(params), OUTPUTS))
        if ok.any():
            res[ok] = self.predict(params[ok])
        if (~ok).any():
            sims = simulate_spectra(self.engine, params[~ok], self.fallback_reps, self.seed)
            res[~ok] = sims / sims.sum(axis=1, keepdims=True)
        return res, ~ok
