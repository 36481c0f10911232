"""GPU tests of the recurrent surrogate (tensor-core GEMMs + rno kernels).

* gradients of one TBPTT window against the float64 oracle with the device's bf16 rounding
  points (relative L2 error < 2e-2 per tensor) and against torch autograd in float32 on the
  same bf16 weights (relative L2 error < 5e-2);
* training on viscoplastic material-point paths lowers the loss and the trained network's
  stress error beats the same network's error before training and the elastic predictor.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import concrete_impact_b200 as cib
from concrete_impact_b200 import batched
from concrete_impact_b200.rno import IN_PAD, OUT_PAD, RNOConfig, RNODataset, RNOScales, RNOSurrogate
from concrete_impact_b200.rve_builders import random_strain_path
from oracle import j2vp as oj
from oracle.rno import window_forward_backward

pytestmark = pytest.mark.gpu


def _window(T, B, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    r = lambda *s: torch.randn(s, generator=g, device="cuda")  # noqa: E731
    return r(T, B, 6), r(T, B, 6), r(T, B, 6), torch.rand((T, B), generator=g, device="cuda") * 0.3, r(B, 6) * 0.1


def _rel(a, b) -> float:
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("fused", [True, False])
def test_window_gradients_match_oracle_and_autograd(fused: bool) -> None:
    T, B = 6, 256
    model = RNOSurrogate(RNOConfig(seed=3))
    model.fused = fused
    strain, rate, target, coef, z0 = _window(T, B, 1)
    model.load_window(strain, rate, target, coef, z0)
    model.window_gradients(T, B)
    torch.cuda.synchronize()
    assert int(model.err.item()) == 0
    loss = model.window_loss()
    grads = [(gw.cpu().numpy(), gb.cpu().numpy()) for gw, gb in model.gradients()]
    params = [(L.w.cpu().numpy(), L.b.cpu().numpy()) for L in model.layers]
    np_in = [x.cpu().numpy().astype(np.float64) for x in (strain, rate, target, coef, z0)]
    oloss, ograds, _, _ = window_forward_backward(params, *np_in, bf16=True)
    assert loss == pytest.approx(oloss, rel=1e-3)
    for (gw, gb), (ow, ob) in zip(grads, ograds):
        assert _rel(gw, ow) < 2e-2 and _rel(gb, ob) < 2e-2
    # torch autograd, float32, same bf16 weights and inputs
    Ws = [L.wb.float().clone().requires_grad_(True) for L in model.layers]
    bs = [L.b.clone().requires_grad_(True) for L in model.layers]
    z = z0.clone()
    total = 0.0
    for t in range(T):
        x = torch.zeros((B, IN_PAD), device="cuda")
        x[:, 0:6], x[:, 6:12], x[:, 12:18] = strain[t], rate[t], z
        a = x.to(torch.bfloat16).float()
        for i in range(3):
            a = torch.nn.functional.gelu(a @ Ws[i].T + bs[i]).to(torch.bfloat16).float()
        y = a @ Ws[3].T + bs[3]
        total = total + ((y[:, :6] - target[t]) ** 2).sum()
        z = z + coef[t][:, None] * y[:, 6:12]
    total = total / (T * B * 6)
    total.backward()
    for (gw, gb), W, b in zip(grads, Ws, bs):
        assert _rel(gw, W.grad.cpu().numpy()) < 5e-2 and _rel(gb, b.grad.cpu().numpy()) < 5e-2


def test_fused_window_matches_unfused_kernels() -> None:
    """The fused recurrent kernels and the per-step GEMM path compute the same window
    (ragged batch: 300 paths = 2 full CTAs + 44 rows)."""
    T, B = 7, 300
    fused, plain = RNOSurrogate(RNOConfig(seed=4)), RNOSurrogate(RNOConfig(seed=4))
    plain.fused = False
    window = _window(T, B, 2)
    for m in (fused, plain):
        m.load_window(*window)
        m.window_gradients(T, B)
    torch.cuda.synchronize()
    assert int(fused.err.item()) == 0 and int(plain.err.item()) == 0
    assert fused.window_loss() == pytest.approx(plain.window_loss(), rel=1e-5)
    wf, wp = fused._window, plain._window
    assert _rel(wf["z"].cpu(), wp["z"].cpu()) < 1e-5
    for i in range(3):
        assert _rel(wf["Z"][i].cpu(), wp["Z"][i].cpu()) < 1e-5
        assert _rel(wf["Ht"][i].float().cpu(), wp["Ht"][i].float().cpu()) < 1e-3
        assert _rel(wf["dZt"][i].float().cpu(), wp["dZt"][i].float().cpu()) < 1e-2
    for (gf, bf), (gp, bp) in zip(fused.gradients(), plain.gradients()):
        assert _rel(gf.cpu(), gp.cpu()) < 1e-2 and _rel(bf.cpu(), bp.cpu()) < 1e-2


def test_fused_skip_gradients_match_oracle() -> None:
    T, B = 5, 200
    model = RNOSurrogate(RNOConfig(seed=6), RNOScales(1.0, 1.0, 1.0))
    g = np.random.default_rng(3)
    K = g.normal(size=(6, 6)) * 0.3
    model.set_elastic_skip(K)  # unit scales: the normalised skip is K itself
    window = _window(T, B, 5)
    model.load_window(*window)
    model.window_gradients(T, B)
    torch.cuda.synchronize()
    assert int(model.err.item()) == 0
    grads = [(gw.cpu().numpy(), gb.cpu().numpy()) for gw, gb in model.gradients()]
    params = [(L.w.cpu().numpy(), L.b.cpu().numpy()) for L in model.layers]
    np_in = [x.cpu().numpy().astype(np.float64) for x in window]
    skip32 = model.skip.cpu().numpy().astype(np.float64)
    oloss, ograds, oz, _ = window_forward_backward(params, *np_in, bf16=True, skip=skip32)
    assert model.window_loss() == pytest.approx(oloss, rel=1e-3)
    assert _rel(model._window["z"][T].cpu().numpy(), oz) < 1e-3
    for (gw, gb), (ow, ob) in zip(grads, ograds):
        assert _rel(gw, ow) < 2e-2 and _rel(gb, ob) < 2e-2


def test_fused_predict_and_rollout_match_unfused() -> None:
    data = _material_point_dataset(P=130, T=12, seed=11)
    rates = data.rates()
    scales = RNOScales.from_data(data.strain[:, 1:], rates, data.stress[:, 1:])
    fused, plain = RNOSurrogate(RNOConfig(seed=2), scales), RNOSurrogate(RNOConfig(seed=2), scales)
    plain.fused = False
    z = torch.randn((130, 6), device="cuda") * 0.1
    coef = torch.rand(130, device="cuda") * 0.2
    sf, zf, _ = fused.predict(data.strain[:, 3], rates[:, 2], z, coef)
    sp, zp, _ = plain.predict(data.strain[:, 3], rates[:, 2], z, coef)
    assert _rel(sf.cpu(), sp.cpu()) < 1e-5 and _rel(zf.cpu(), zp.cpu()) < 1e-5
    rf, rp = fused.rollout(data), plain.rollout(data)
    assert _rel(rf.cpu(), rp.cpu()) < 1e-4


def test_persistent_forward_runs_more_tiles_than_ctas() -> None:
    """The forward window kernel runs one CTA per SM over 128-path tiles: a ragged batch of
    313 tiles (more than one per CTA) gives the per-step GEMM path's latents and per-tile
    window loss, and the inference kernel (two tiles in flight per CTA) its stresses and
    latents."""
    T, B = 2, 40_000
    fused, plain = RNOSurrogate(RNOConfig(seed=8)), RNOSurrogate(RNOConfig(seed=8))
    plain.fused = False
    window = _window(T, B, 9)
    for m in (fused, plain):
        m.load_window(*window)
        m.window_step(T, B, train=False)
    torch.cuda.synchronize()
    assert int(fused.err.item()) == 0 and int(plain.err.item()) == 0
    assert fused.window_loss() == pytest.approx(plain.window_loss(), rel=1e-5)
    assert _rel(fused._window["z"].cpu(), plain._window["z"].cpu()) < 1e-5
    # an inference step over more than two tiles per SM runs the two-tiles-per-CTA kernel
    strain, rate, target, coef, z0 = window
    sf, zf, _ = fused.predict(strain[0], rate[0], z0, coef[0])
    sp, zp, _ = plain.predict(strain[0], rate[0], z0, coef[0])
    assert _rel(sf.cpu(), sp.cpu()) < 1e-5 and _rel(zf.cpu(), zp.cpu()) < 1e-5
    # ... with the arithmetic of the training forward kernel: the same latent bit for bit
    fused.load_window(strain[:1], rate[:1], target[:1], coef[:1], z0)
    fused.window_step(1, B, train=False)
    torch.cuda.synchronize()
    assert int(fused.err.item()) == 0
    assert torch.equal(fused._window["z"][1], zf)


def test_training_divergence_guard_restores_finite_weights() -> None:
    data = _material_point_dataset(P=128, T=50, seed=13)
    scales = RNOScales.from_data(data.strain[:, 1:], data.rates(), data.stress[:, 1:])
    model = RNOSurrogate(RNOConfig(batch_paths=128, tbptt_steps=50, learning_rate=1.0e30, seed=2), scales)
    before = [L.w.clone() for L in model.layers]
    history = model.fit(data, epochs=2)
    # epoch 1 evaluates the initial weights (finite) and then steps them to ~1e30; epoch 2's
    # loss overflows, so the guard restores the start of epoch 1
    assert model.divergences == 1 and np.isfinite(history[0]) and not np.isfinite(history[1])
    for L, w0 in zip(model.layers, before):
        assert torch.equal(L.w, w0) and bool(torch.isfinite(L.wb.float()).all())


def test_checkpoint_resume_continues_training_exactly() -> None:
    data = _material_point_dataset(P=256, T=50, seed=17)
    scales = RNOScales.from_data(data.strain[:, 1:], data.rates(), data.stress[:, 1:])
    cfg = RNOConfig(batch_paths=128, tbptt_steps=50, seed=3)
    a = RNOSurrogate(cfg, scales)
    a.fit(data, epochs=2)
    ck = a.checkpoint()
    b = RNOSurrogate(cfg, RNOScales(1.0, 1.0, 1.0))
    b.load_checkpoint(ck)
    ha, hb = a.fit(data, epochs=1), b.fit(data, epochs=1)
    assert ha == hb
    for La, Lb in zip(a.layers, b.layers):
        assert torch.equal(La.w, Lb.w) and torch.equal(La.mw, Lb.mw)
    assert int(a.step.item()) == int(b.step.item()) == 3 * 2


def _material_point_dataset(P: int, T: int, seed: int, dt: float = 2.0e-6) -> RNODataset:
    """Macro stress paths of one viscoplastic mortar point (GPU return map) under random
    piecewise-linear strain paths (|strain| <= 2e-3) with a common time step."""
    mat = cib.J2ViscoplasticMaterial("mortar", 2200.0, 25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0)
    settings = cib.MaterialUpdateSettings(50, 1e-10, 1e-12, 1e-10)
    eps = torch.as_tensor(np.asarray([random_strain_path(seed + p, steps=T, max_abs=2e-3)[1] for p in range(P)]),
                          device="cuda")  # (P, T+1, 6)  # fmt: skip
    stress = torch.zeros_like(eps)
    state = batched.SoAState(torch.zeros((6, P), dtype=torch.float64, device="cuda"),
                             torch.zeros((6, P), dtype=torch.float64, device="cuda"),
                             torch.zeros(P, dtype=torch.float64, device="cuda"))  # fmt: skip
    for t in range(T):
        de = (eps[:, t + 1] - eps[:, t]).T.contiguous()
        state, _ = batched.j2vp_update_soa(mat, settings, dt, de, state, with_tangent=False)
        stress[:, t + 1] = state.stress.T
    return RNODataset(eps, stress, torch.full((P, T), dt, dtype=torch.float64, device="cuda"))


def test_training_reduces_error_below_untrained_and_elastic_predictors() -> None:
    data = _material_point_dataset(P=256, T=100, seed=7)
    rates = data.rates()
    scales = RNOScales.from_data(data.strain[:, 1:], rates, data.stress[:, 1:])
    model = RNOSurrogate(RNOConfig(batch_paths=256, tbptt_steps=50, learning_rate=2e-3, seed=1), scales)
    target = data.stress[:, 1:].float()

    def err(pred):
        return float(((pred - target) ** 2).sum().sqrt() / (target**2).sum().sqrt())

    before = err(model.rollout(data))
    history = model.fit(data, epochs=150)
    after = err(model.rollout(data))
    c = torch.as_tensor(oj.elasticity_matrix(25.0e9, 0.2), device="cuda")
    elastic = err((data.strain[:, 1:] @ c.T).float())
    assert history[-1] < 0.1 * history[0]
    assert after < 0.25 * before
    assert after < 0.5 * elastic, (after, elastic)
