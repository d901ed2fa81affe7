"""CPU restatement of the SFS surrogate network (forward pass, loss, gradients, Adam).  TEST
INFRASTRUCTURE ONLY: imported by tests/ and bench.py to check the tensor-core path, never by the
product.

The reference has no such network (3P answers every SFS query by simulation: GO_Fish::run_sim,
go_fish.cuh:280, then Spectrum::site_frequency_spectrum, spectrum.h:90), so there is no reference file
to follow; this module states the network the surrogate is defined as:

    a_0 = x                                   x: 6 scaled parameters
    z_l = a_{l-1} W_l^T + b_l,  a_l = GELU(z_l)   l = 1..4, width 512,
                                               GELU(z) = z/2 (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))
    out = a_4 W_5^T + b_5                      99 outputs
    loss = mean over rows and outputs of (out - target)^2

`emulate_bf16=True` rounds to bf16 (round to nearest even) exactly where the GPU path stores bf16:
the inputs, the weights, the hidden activations a_l, and the gradients dOut / dz_l that feed the
tensor-core GEMMs; everything else (accumulation, pre-activations z_l, bias gradients, Adam) is fp32.
With `emulate_bf16=False` and dtype float64 it is the exact network; its gradients are pinned against
central finite differences and against torch autograd in the CPU tests.
"""
from __future__ import annotations

import numpy as np

INPUTS, HIDDEN, OUTPUTS, LAYERS = 6, 512, 99, 5
SHAPES = [(HIDDEN, INPUTS), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (OUTPUTS, HIDDEN)]


def param_count() -> int:
    return sum(r * c + r for r, c in SHAPES)


def split(vec: np.ndarray) -> list[tuple[np.ndarray, np.ndarray]]:
    """Flat parameter vector (W1, b1, ..., W5, b5; row-major out x in) -> [(W, b)]."""
    out, o = [], 0
    for r, c in SHAPES:
        W = vec[o:o + r * c].reshape(r, c)
        o += r * c
        b = vec[o:o + r]
        o += r
        out.append((W, b))
    assert o == len(vec)
    return out


def join(params: list[tuple[np.ndarray, np.ndarray]]) -> np.ndarray:
    return np.concatenate([np.concatenate([W.ravel(), b.ravel()]) for W, b in params])


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest bf16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = ((u >> 16) & 1) + np.uint32(0x7FFF)
    return ((u + r) & np.uint32(0xFFFF0000)).view(np.float32)


GELU_C = np.sqrt(2.0 / np.pi)
GELU_A = 0.044715


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(GELU_C * (z + GELU_A * z ** 3)))


def gelu_grad(z):
    t = np.tanh(GELU_C * (z + GELU_A * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_C * (1.0 + 3.0 * GELU_A * z * z)


def forward(vec: np.ndarray, x: np.ndarray, emulate_bf16: bool = True, dtype=np.float32):
    q = bf16 if emulate_bf16 else (lambda a: a)
    params = split(vec.astype(dtype))
    a = q(x.astype(dtype)).astype(dtype)
    zs, acts = [], [a]
    for W, b in params[:4]:
        z = (a @ q(W).astype(dtype).T + b).astype(dtype)
        zs.append(z)
        a = q(gelu(z).astype(dtype)).astype(dtype)
        acts.append(a)
    W, b = params[4]
    out = (a @ q(W).astype(dtype).T + b).astype(dtype)
    return out, zs, acts


def gradients(vec: np.ndarray, x: np.ndarray, target: np.ndarray, emulate_bf16: bool = True, dtype=np.float32):
    """(flat gradient, loss) of the mean squared error."""
    q = bf16 if emulate_bf16 else (lambda a: a)
    params = split(vec.astype(dtype))
    out, zs, acts = forward(vec, x, emulate_bf16, dtype)
    B = x.shape[0]
    d = (out - target.astype(dtype)).astype(dtype)
    loss = float(np.mean(d.astype(np.float64) ** 2))
    g_full = (dtype(2.0) / dtype(B * OUTPUTS) * d).astype(dtype)
    grads = [None] * LAYERS
    g = q(g_full).astype(dtype)
    grads[4] = (g.T @ acts[4], g_full.sum(axis=0))
    dy = g @ q(params[4][0]).astype(dtype)
    for l in range(3, -1, -1):
        dz_full = (dy * gelu_grad(zs[l])).astype(dtype)
        dz = q(dz_full).astype(dtype)
        grads[l] = (dz.T @ acts[l], dz_full.sum(axis=0))
        if l > 0:
            dy = dz @ q(params[l][0]).astype(dtype)
    return join(grads).astype(dtype), loss


def adam(vec, grad, m, v, step, lr, beta1=0.9, beta2=0.999, eps=1e-8, decay=0.0):
    """One Adam step (decoupled weight decay as a fraction of lr), fp32, in place; returns vec."""
    m *= beta1
    m += (1 - beta1) * grad
    v *= beta2
    v += (1 - beta2) * grad * grad
    bc1 = np.float32(1.0 - beta1 ** step)
    bc2 = np.float32(1.0 - beta2 ** step)
    vec -= np.float32(lr * decay) * vec
    vec -= np.float32(lr) * (m / bc1) / (np.sqrt(v / bc2) + np.float32(eps))
    return vec
