"""GPU tests of the energy-based RVE-RNO kernel (concrete_impact_b200.energy_rno) on the
reference's trained model: anchors, every step of a 12-step rollout of 128 points with the
reference's inputs, the other integrator, a chained rollout on the kernel's own latent
states, a partial tile, the material-point adapter and the artifact loader."""

from __future__ import annotations

import json

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from conftest import load_case  # noqa: E402
from concrete_impact_b200.energy_rno import (EnergyDissipationRVERNO, RVERNOMaterialAdapter,  # noqa: E402
                                             RVERNOModelConfig, SurrogateCapabilityError, load_rve_rno_state_dict)
from concrete_impact_b200.materials import MaterialPointRequest, MaterialResponseRequirements, MaterialUpdateSettings  # noqa: E402

KEYS = ("stress", "latent_state", "state_rate", "dimensionless_state_rate", "dissipation", "free_energy",
        "nonequilibrium_energy_increment")  # fmt: skip
# relative to each field's maximum; both sides are FP32 with different summation orders
TOL = {"stress": 2e-4, "latent_state": 1e-5, "state_rate": 5e-5, "dimensionless_state_rate": 5e-5,
       "dissipation": 5e-5, "free_energy": 1e-3, "nonequilibrium_energy_increment": 1e-3}  # fmt: skip


def _model(integrator=None):
    g, meta = load_case("rno_energy_c48")
    spec = {k: v for k, v in meta["model"].items() if k != "device"}
    if integrator:
        spec["integrator"] = integrator
    model = EnergyDissipationRVERNO(RVERNOModelConfig(**spec))
    model.load_state_dict({k[3:]: g[k] for k in g if k.startswith("w__")})
    return model, g, meta


def _check(res, g, prefix, step, tol_scale=1.0):
    for key in KEYS:
        ref = g[f"{prefix}__{key}"]
        np.testing.assert_allclose(getattr(res, key).cpu().numpy(), ref[step], rtol=0,
                                   atol=tol_scale * TOL[key] * np.abs(ref).max(), err_msg=key)  # fmt: skip


def test_anchors_and_every_rollout_step_match_reference() -> None:
    model, g, meta = _model()
    anchors = model.prepare_energy_anchors()
    a = anchors.packed.cpu().numpy()
    assert a[0] == pytest.approx(float(g["anchor_equilibrium_value"]), rel=1e-5)
    np.testing.assert_allclose(a[1:7], g["anchor_equilibrium_gradient"], rtol=0,
                               atol=1e-5 * np.abs(g["anchor_equilibrium_gradient"]).max())  # fmt: skip
    assert a[7] == pytest.approx(float(g["anchor_nonequilibrium_value"]), rel=1e-4, abs=1e-4)
    np.testing.assert_allclose(a[8:14], g["anchor_nonequilibrium_gradient"], rtol=0,
                               atol=1e-5 * np.abs(g["anchor_nonequilibrium_gradient"]).max())  # fmt: skip
    for step in range(meta["steps"]):
        res = model.update_batch(g["strain"][step], g["latent_in"][step], g["time_step"], anchors)
        _check(res, g, "out", step)


def test_semi_implicit_integrator_and_chained_rollout() -> None:
    model, g, meta = _model("cs_semi_implicit_forward_euler")
    last = meta["steps"] - 1
    res = model.update_batch(g["strain"][last], g["latent_in"][last], g["time_step"])
    _check(res, g, "semi", 0)
    model, g, meta = _model()
    latent = torch.zeros((g["strain"].shape[1], 6), dtype=torch.float32, device="cuda")
    anchors = model.prepare_energy_anchors()
    for step in range(meta["steps"]):
        res = model.update_batch(g["strain"][step], latent, g["time_step"], anchors)
        latent = res.latent_state
        _check(res, g, "out", step, tol_scale=2.0)


def test_partial_tile_equals_full_batch_rows() -> None:
    model, g, meta = _model()
    anchors = model.prepare_energy_anchors()
    full = model.update_batch(g["strain"][5], g["latent_in"][5], g["time_step"], anchors)
    part = model.update_batch(g["strain"][5][:77], g["latent_in"][5][:77], g["time_step"][:77], anchors)
    for key in KEYS:
        assert torch.equal(getattr(part, key), getattr(full, key)[:77]), key
    assert full.tangent is None


def test_material_adapter_and_artifact_loader(tmp_path) -> None:
    model, g, meta = _model()
    adapter = RVERNOMaterialAdapter(model, "rve_rno", 2400.0, 4000.0)
    state = adapter.initialize_state(g["strain"].shape[1])
    dt = float(g["time_step"][0])
    request = MaterialPointRequest(g["strain"][0].astype(np.float64), None, dt, "three_dimensional",
                                   MaterialUpdateSettings(50, 1e-10, 1e-12, 1e-10))  # fmt: skip
    resp = adapter.update(request, state, MaterialResponseRequirements(tangent=False, free_energy=True, dissipation=True))
    ref = model.update_batch(g["strain"][0], np.zeros((g["strain"].shape[1], 6)), np.full(g["strain"].shape[1], dt))
    assert isinstance(resp.stresses, np.ndarray) and resp.stresses.dtype == np.float64
    np.testing.assert_array_equal(resp.stresses, ref.stress.double().cpu().numpy())
    np.testing.assert_array_equal(resp.state.variables["latent_state"], ref.latent_state.double().cpu().numpy())
    with_tangent = adapter.update(request, state, MaterialResponseRequirements(tangent=True))
    np.testing.assert_array_equal(with_tangent.stresses, resp.stresses)
    assert with_tangent.tangents.shape == (g["strain"].shape[1], 6, 6) and with_tangent.tangents.dtype == np.float64
    spec = {k: v for k, v in meta["model"].items() if k != "device"}
    weights = {k[3:]: torch.as_tensor(g[k]) for k in g if k.startswith("w__")}
    torch.save({"epoch": 0, "model_state_dict": weights}, tmp_path / "best_model.pt")
    metadata = {"model_family": spec["family"], "deployment_integrator": "explicit_only",
                **{k: spec[k] for k in ("integrator", "evolution", "reference_time_scale", "latent_dimension",
                                        "hidden_size", "hidden_layers", "activation", "dtype")}}  # fmt: skip
    (tmp_path / "meta.json").write_text(json.dumps(metadata))
    loaded = load_rve_rno_state_dict(RVERNOModelConfig(**spec), tmp_path / "best_model.pt", tmp_path / "meta.json")
    assert torch.equal(loaded.params, model.params)
    with pytest.raises(ValueError, match="does not match"):
        load_rve_rno_state_dict(RVERNOModelConfig(**dict(spec, hidden_layers=3)), tmp_path / "best_model.pt",
                                tmp_path / "meta.json")  # fmt: skip


def test_algorithmic_tangent_matches_reference_autograd_tangent() -> None:
    """cib_energy_rno_tangent (forward-over-reverse second derivatives of the three networks,
    through the candidate latent state of the current-state integrator) against the
    reference's FP32 autograd tangent of 16 points at the last rollout step, and against
    central differences of the GPU stress for both integrators."""
    model, g, meta = _model()
    last = meta["steps"] - 1
    anchors = model.prepare_energy_anchors()
    res = model.update_batch(g["strain"][last][:16], g["latent_in"][last][:16], g["time_step"][:16], anchors,
                             compute_tangent=True)  # fmt: skip
    ref = g["tangent_last16"]
    got = res.tangent.double().cpu().numpy()
    np.testing.assert_allclose(got, ref, rtol=0, atol=2e-4 * np.abs(ref).max())
    for integrator in ("current_state_stress_forward_euler", "cs_semi_implicit_forward_euler"):
        model, g, meta = _model(integrator)
        anchors = model.prepare_energy_anchors()
        eps = torch.as_tensor(g["strain"][last][:32], dtype=torch.float64)
        z, dt = g["latent_in"][last][:32], g["time_step"][:32]
        tan = model.update_batch(eps, z, dt, anchors, compute_tangent=True).tangent.double().cpu().numpy()
        h = 1e-3 * float(eps.abs().max())
        fd = np.zeros_like(tan)
        for j in range(6):
            plus, minus = eps.clone(), eps.clone()
            plus[:, j] += h
            minus[:, j] -= h
            sp = model.update_batch(plus, z, dt, anchors).stress.double().cpu().numpy()
            sm = model.update_batch(minus, z, dt, anchors).stress.double().cpu().numpy()
            fd[:, :, j] = (sp - sm) / (2.0 * h)
        np.testing.assert_allclose(tan, fd, rtol=0, atol=2e-2 * np.abs(tan).max(), err_msg=integrator)
