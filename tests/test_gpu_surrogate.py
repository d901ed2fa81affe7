"""Surrogate network on the tensor cores: the tcgen05 GEMM against a torch fp32 product of the same
bf16 operands, the forward pass and the gradients against the CPU oracle (bf16 rounding emulated at
the same points, and plain fp32), the Adam update against the oracle's Adam applied to the GPU's own
gradients, and training on simulator spectra."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 64, 64), (128, 128, 64), (256, 512, 512), (512, 128, 1024),
                                   (1024, 512, 4096), (384, 64, 192)])
def test_bf16_gemm_matches_fp32_product(M, N, K):
    from parallelpopgen_b200.surrogate import bf16_gemm
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N + K)
    a = torch.randn((M, K), device="cuda", generator=g).to(torch.bfloat16)
    b = torch.randn((N, K), device="cuda", generator=g).to(torch.bfloat16)
    c = bf16_gemm(a, b)
    torch.cuda.synchronize()
    want = a.double() @ b.double().T
    # fp32 accumulation of exact bf16 products: error ~ K * 2^-24 * |a||b|
    tol = 4 * K * 2.0 ** -24 * (a.double().abs() @ b.double().abs().T)
    assert torch.all((c.double() - want).abs() <= tol + 1e-6), float((c.double() - want).abs().max())


def _net(seed, B):
    from parallelpopgen_b200.surrogate import Mlp, init_params
    rng = np.random.default_rng(seed)
    vec = init_params(seed)
    vec[-99:] = rng.normal(0, 0.1, 99).astype(np.float32)          # nonzero output bias
    x = rng.uniform(-1, 1, (B, 6)).astype(np.float32)
    t = rng.normal(-4, 1, (B, 99)).astype(np.float32)
    mlp = Mlp(capacity=max(B, 512), lr=1e-3)
    mlp.set_params(vec)
    return mlp, vec, x, t


def _rel(a, b):
    return float(np.linalg.norm(a.astype(np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def test_params_round_trip():
    mlp, vec, _, _ = _net(1, 128)
    assert np.array_equal(mlp.get_params(), vec)


def test_forward_matches_oracle():
    mlp, vec, x, _ = _net(2, 512)
    y = mlp.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    want, _, _ = mo.forward(vec, x, emulate_bf16=True)
    exact, _, _ = mo.forward(vec.astype(np.float64), x.astype(np.float64), emulate_bf16=False, dtype=np.float64)
    # same bf16 rounding points: only the fp32 accumulation order differs (and the rare bf16 tie it flips)
    assert _rel(y, want) < 2e-3, _rel(y, want)
    # against the exact network: bf16 weights and activations (unit roundoff 2^-9) through 5 layers
    assert _rel(y, exact) < 3e-2, _rel(y, exact)


@pytest.mark.parametrize("B", [128, 512, 4096, 148 * 128 + 256, 2 * 148 * 128 + 128])
def test_fused_forward_equals_layered_forward(B):
    """The fused five-layer inference kernel issues each layer's MMAs in the layered GEMMs' order and
    rounds the activations at the same points, so its outputs equal the one-GEMM-per-layer path bit for
    bit (one tile; one tile per CTA; more tiles than SMs; three tiles on some CTAs, two on the rest)."""
    from parallelpopgen_b200 import _capi
    mlp, vec, x, _ = _net(7, B)
    xs = torch.from_numpy(x).cuda()
    fused = mlp.forward(xs).cpu().numpy()
    mlp.check()
    lib = _capi.load()
    assert lib.gf_mlp_set_fused_inference(mlp.h, 0) == 0
    layered = mlp.forward(xs).cpu().numpy()
    mlp.check()
    assert lib.gf_mlp_set_fused_inference(mlp.h, 1) == 0
    assert np.isfinite(fused).all()
    assert np.array_equal(fused.view(np.uint32), layered.view(np.uint32))


def test_gradients_match_oracle():
    mlp, vec, x, t = _net(3, 512)
    g, loss = mlp.gradients(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda())
    want, want_loss = mo.gradients(vec, x, t, emulate_bf16=True)
    exact, exact_loss = mo.gradients(vec.astype(np.float64), x.astype(np.float64), t.astype(np.float64),
                                     emulate_bf16=False, dtype=np.float64)
    assert abs(loss - want_loss) <= 1e-4 * want_loss
    starts = np.cumsum([0] + [r * c + r for r, c in mo.SHAPES])
    for l in range(mo.LAYERS):
        sl = slice(starts[l], starts[l + 1])
        assert _rel(g[sl], want[sl]) < 1e-2, (l, _rel(g[sl], want[sl]))
        assert _rel(g[sl], exact[sl]) < 5e-2, (l, _rel(g[sl], exact[sl]))


def test_adam_update_matches_oracle():
    mlp, vec, x, t = _net(4, 256)
    xs, ts = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    w = vec.copy()
    m = np.zeros_like(w)
    v = np.zeros_like(w)
    for step in (1, 2, 3):
        g, _ = mlp.gradients(xs, ts)                 # gradients at the current GPU parameters
        mlp.train_step(xs, ts)
        mo.adam(w, g, m, v, step, 1e-3)
        got = mlp.get_params()
        # same gradient, same formula: fp32 rounding only (sqrt / division order)
        np.testing.assert_allclose(got, w, rtol=1e-5, atol=1e-7)
        w = got.copy()                               # follow the GPU trajectory


def test_training_reduces_loss():
    from parallelpopgen_b200.surrogate import train
    mlp, vec, x, _ = _net(5, 4096)
    # a smooth target function of the six inputs
    xs = np.random.default_rng(9).uniform(-1, 1, (4096, 6)).astype(np.float32)
    freq = np.arange(1, 100) / 100.0
    t = (-np.log(np.arange(1, 100))[None, :] + np.sin(xs[:, :1] * 2 + freq[None, :] * 3) * xs[:, 1:2]
         + 0.5 * xs[:, 2:3] * freq[None, :]).astype(np.float32)
    X, T = torch.from_numpy(xs).cuda(), torch.from_numpy(t).cuda()
    res = train(mlp, X, T, steps=600, batch=512, lr=1e-3, log_every=100)
    first, last = res.losses[0][1], res.final_loss
    assert last < first / 20, res.losses


def test_surrogate_on_simulator_spectra():
    """A small end-to-end run: train on batched-simulator spectra, compare with held-out simulator means,
    and route an out-of-support query to the simulator."""
    from parallelpopgen_b200 import Engine
    from parallelpopgen_b200 import surrogate as sg
    with Engine() as e:
        ptrain = sg.draw_parameters(1024, seed=21)
        ptrain[:, 0] = sg.LOW[0] + (ptrain[:, 0] - sg.LOW[0]) * 0.1         # small N: quick
        sims = sg.simulate_spectra(e, ptrain, reps=4, seed=1000)
        assert np.all(sims.sum(axis=1) > 0)
        X = torch.from_numpy(sg.encode(ptrain)).cuda()
        T = torch.from_numpy(sg.spectra_to_targets(sims)).cuda()
        mlp = sg.Mlp(capacity=1024, lr=1e-3)
        mlp.set_params(sg.init_params(0))
        res = sg.train(mlp, X, T, steps=1500, batch=512, lr=1e-3, log_every=500)
        assert res.final_loss < res.losses[0][1] / 5
        s = sg.Surrogate(mlp, e, fallback_reps=4)
        q = ptrain[:3].copy()
        q[2, 1] = 50.0                                     # gamma outside the support
        p, routed = s.query(q)
        assert list(routed) == [False, False, True]
        assert np.allclose(p.sum(axis=1), 1.0)
        mlp.check()


def test_trained_network_beats_answers_without_it():
    """What the network adds over answering from the same simulated data without it: on held-out
    parameter draws, its median per-bin relative error against 16-replicate simulator means must be
    well below that of the training set's mean spectrum (one answer for every query) and that of the
    nearest training draw's spectrum (a table lookup over the same simulations).  Measured on B200 with
    N in [500, 660]: 2.8 % against 84 % and 17 %."""
    from parallelpopgen_b200 import Engine
    from parallelpopgen_b200 import surrogate as sg

    def small_n(p):
        p[:, 0] = sg.LOW[0] + (p[:, 0] - sg.LOW[0]) * 0.1          # N in [1000, ~1260]: quick runs
        return p

    with Engine() as e:
        ptrain = small_n(sg.draw_parameters(2048, seed=31))
        ptest = small_n(sg.draw_parameters(128, seed=32))
        train_sims = sg.simulate_spectra(e, ptrain, reps=4, seed=2000)
        truth = sg.simulate_spectra(e, ptest, reps=16, seed=9000)
        targets = sg.spectra_to_targets(train_sims)
        scale = sg.TargetScale.fit(targets)
        X = torch.from_numpy(sg.encode(ptrain)).cuda()
        T = torch.from_numpy(scale.apply(targets)).cuda()
        mlp = sg.Mlp(capacity=2048, lr=1e-3)
        mlp.set_params(sg.init_params(0))
        sg.train(mlp, X, T, steps=3000, batch=512, lr=1e-3, log_every=1000)
        net = sg.Surrogate(mlp, e, scale=scale).predict(ptest)
        mlp.check()
    train_p = train_sims / train_sims.sum(axis=1, keepdims=True)
    constant = np.repeat(train_p.mean(axis=0, keepdims=True), len(ptest), axis=0)
    xtr, xte = sg.encode(ptrain), sg.encode(ptest)
    nearest = train_p[np.argmin(((xte[:, None, :] - xtr[None, :, :]) ** 2).sum(axis=2), axis=1)]
    err_net = sg.median_relative_error(net, truth)[0]
    err_const = sg.median_relative_error(constant, truth)[0]
    err_nn = sg.median_relative_error(nearest, truth)[0]
    print(f"median per-bin relative error: network {err_net:.4f}, training mean {err_const:.4f}, "
          f"nearest training draw {err_nn:.4f}")
    assert err_net < 0.5 * err_const, (err_net, err_const)
    assert err_net < 0.5 * err_nn, (err_net, err_nn)


def test_bounded_wait_reports_and_recovers():
    """Failure path without a GPU fault: an injected missing accumulator hand-off makes the GEMM's
    bounded wait run out; the kernel ends, the fault word reports it once, and the next pass is exact."""
    from parallelpopgen_b200 import _capi
    mlp, vec, x, _ = _net(6, 512)
    xs = torch.from_numpy(x).cuda()
    want = mlp.forward(xs).cpu().numpy()
    mlp.check()
    lib = _capi.load()
    assert lib.gf_mlp_inject_fault(mlp.h, 1) == 0
    mlp.forward(xs)
    assert lib.gf_mlp_check(mlp.h) == 6            # GF_ERR_DEVICE
    assert b"ran out" in lib.gf_mlp_last_error(mlp.h)
    assert lib.gf_mlp_check(mlp.h) == 0            # reported once, cleared
    again = mlp.forward(xs).cpu().numpy()
    mlp.check()
    assert np.array_equal(again.view(np.uint32), want.view(np.uint32))
