"""Surrogate network, CPU side: the oracle's gradients against finite differences and torch autograd,
its bf16 rounding and Adam step against torch, the host-side parameter mapping, and the library's
parameter count.  No GPU."""
from __future__ import annotations

import math

import numpy as np
import torch

from oracle import mlp_oracle as mo


def _case(seed=0, B=8):
    rng = np.random.default_rng(seed)
    vec = rng.normal(0, 0.05, mo.param_count())
    x = rng.uniform(-1, 1, (B, mo.INPUTS))
    t = rng.normal(0, 1, (B, mo.OUTPUTS))
    return vec, x, t


def test_oracle_gradients_match_finite_differences():
    vec, x, t = _case()
    g, _ = mo.gradients(vec, x, t, emulate_bf16=False, dtype=np.float64)
    rng = np.random.default_rng(1)
    # a few coordinates of every layer's weights and biases
    starts = np.cumsum([0] + [r * c + r for r, c in mo.SHAPES])
    idx = np.concatenate([rng.integers(starts[i], starts[i + 1], 4) for i in range(mo.LAYERS)])
    for i in idx:
        h = 1e-6
        vp, vm = vec.copy(), vec.copy()
        vp[i] += h
        vm[i] -= h
        lp = np.mean((mo.forward(vp, x, False, np.float64)[0] - t) ** 2)
        lm = np.mean((mo.forward(vm, x, False, np.float64)[0] - t) ** 2)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (i, g[i], fd)


def test_oracle_gradients_match_torch_autograd():
    vec, x, t = _case(seed=3, B=16)
    g, loss = mo.gradients(vec, x, t, emulate_bf16=False, dtype=np.float64)
    ps = [(torch.tensor(W, requires_grad=True), torch.tensor(b, requires_grad=True)) for W, b in mo.split(vec)]
    a = torch.tensor(x)
    for W, b in ps[:4]:
        a = torch.nn.functional.gelu(a @ W.T + b, approximate="tanh")
    out = a @ ps[4][0].T + ps[4][1]
    L = torch.mean((out - torch.tensor(t)) ** 2)
    L.backward()
    want = np.concatenate([np.concatenate([W.grad.numpy().ravel(), b.grad.numpy()]) for W, b in ps])
    assert abs(L.item() - loss) < 1e-12
    np.testing.assert_allclose(g, want, rtol=1e-9, atol=1e-14)


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(5)
    x = np.concatenate([rng.normal(0, 1, 10000), rng.normal(0, 1e-30, 100), [0.0, -0.0, 1.0, 65504.0]])
    x = x.astype(np.float32)
    want = torch.tensor(x).to(torch.bfloat16).float().numpy()
    assert np.array_equal(mo.bf16(x).view(np.uint32), want.view(np.uint32))


def test_adam_step_matches_torch():
    rng = np.random.default_rng(7)
    w0 = rng.normal(0, 1, 1000).astype(np.float32)
    grads = [rng.normal(0, 1, 1000).astype(np.float32) for _ in range(3)]
    w = w0.copy()
    m = np.zeros_like(w)
    v = np.zeros_like(w)
    p = torch.tensor(w0.copy(), requires_grad=True)
    opt = torch.optim.Adam([p], lr=1e-3, betas=(0.9, 0.999), eps=1e-8)
    for step, g in enumerate(grads, 1):
        mo.adam(w, g, m, v, step, 1e-3)
        p.grad = torch.tensor(g)
        opt.step()
    np.testing.assert_allclose(w, p.detach().numpy(), rtol=1e-6, atol=1e-7)


def test_library_parameter_count():
    from parallelpopgen_b200 import _capi
    assert _capi.load().gf_mlp_param_count() == mo.param_count() == 842339


def test_parameter_mapping():
    from parallelpopgen_b200 import surrogate as sg
    p = sg.draw_parameters(1000, seed=1)
    assert sg.in_support(p).all()
    x = sg.encode(p)
    assert x.min() >= -1 and x.max() <= 1 and x.dtype == np.float32
    q = p[:3].copy()
    q[0, 1] = 20.0        # gamma above the support
    q[1, 0] = math.log(100.0)
    assert list(sg.in_support(q)) == [False, False, True]
    rep = sg.replicate_for(np.array([math.log(1000.0), -10.0, 0.3, 0.2, 0.001, 0.5]), 11, 12)
    assert rep.N0 == 1000 and rep.num_generations == 1000 and rep.N_min == 100 and rep.N_max == 10000
    assert abs(rep.mu * 4 * 1000 * sg.NUM_SITES - sg.THETA) < 1e-3 * sg.THETA
    t = sg.spectra_to_targets(np.array([[1.0] * 98 + [0.0]]))
    assert t.shape == (1, 99) and abs(t[0, 0] - math.log(1 / 98)) < 1e-6 and abs(t[0, -1] - math.log(sg.LOG_FLOOR)) < 1e-5


def test_target_scale_round_trip():
    from parallelpopgen_b200 import surrogate as sg
    rng = np.random.default_rng(2)
    t = rng.normal(-5, 2, (300, 99)).astype(np.float32)
    t[:, 7] = -9.2      # a constant bin keeps a floor on its scale
    sc = sg.TargetScale.fit(t)
    z = sc.apply(t)
    assert abs(z[:, :7].mean()) < 1e-5 and abs(z[:, :7].std() - 1) < 1e-3
    assert np.all(np.isfinite(z)) and np.allclose(z[:, 7], 0.0)
    np.testing.assert_allclose(sc.invert(z), t, rtol=1e-5, atol=1e-5)
