"""CPU tests of the energy-based RVE-RNO oracle and of the GPU path's parameter layout.

Pinned to the reference's trained model (artifacts/rve_rno/c48_v2_liu_direct, run by
tests/golden/make_golden.py through its own EnergyDissipationRVERNO.update_batch in FP32):
the float64 oracle reproduces the anchors and a 12-step rollout of 128 points within the
FP32 rounding of the reference (cancellation against the zero-state anchors dominates).
The packed parameter array of concrete_impact_b200.energy_rno is checked against the
offsets the kernel uses (cib_energy_rno_param_count and the per-layer W, W^T, bias order).
"""

from __future__ import annotations

import numpy as np
import pytest

from concrete_impact_b200 import _native
from concrete_impact_b200.energy_rno import RVERNOModelConfig, pack_state_dict
from conftest import load_case
from oracle import rno_energy as oe

KEYS = ("stress", "latent_state", "state_rate", "dimensionless_state_rate", "dissipation", "free_energy",
        "nonequilibrium_energy_increment")  # fmt: skip
# tolerances relative to each field's maximum: the reference runs in FP32
TOL = {"stress": 5e-5, "latent_state": 1e-6, "state_rate": 1e-5, "dimensionless_state_rate": 1e-5,
       "dissipation": 1e-5, "free_energy": 3e-4, "nonequilibrium_energy_increment": 2e-4}  # fmt: skip


def _case():
    g, meta = load_case("rno_energy_c48")
    sd = {k[3:]: g[k] for k in g if k.startswith("w__")}
    return g, meta, sd


def test_oracle_matches_reference_rollout() -> None:
    g, meta, sd = _case()
    tau = meta["model"]["reference_time_scale"]
    a = oe.anchors(sd, 6)
    assert a["eq_value"] == pytest.approx(float(g["anchor_equilibrium_value"]), rel=1e-6)
    np.testing.assert_allclose(a["eq_grad"], g["anchor_equilibrium_gradient"], rtol=0,
                               atol=2e-6 * np.abs(g["anchor_equilibrium_gradient"]).max())  # fmt: skip
    np.testing.assert_allclose(a["neq_grad"], g["anchor_nonequilibrium_gradient"], rtol=0,
                               atol=2e-6 * np.abs(g["anchor_nonequilibrium_gradient"]).max())  # fmt: skip
    for step in range(meta["steps"]):
        out = oe.update(sd, g["strain"][step], g["latent_in"][step], g["time_step"], tau, meta["model"]["integrator"])
        for key in KEYS:
            ref = g[f"out__{key}"]
            np.testing.assert_allclose(out[key], ref[step], rtol=0, atol=TOL[key] * np.abs(ref).max(), err_msg=key)
    last = meta["steps"] - 1
    out = oe.update(sd, g["strain"][last], g["latent_in"][last], g["time_step"], tau, "cs_semi_implicit_forward_euler")
    for key in ("stress", "latent_state", "free_energy"):
        ref = g[f"semi__{key}"][0]
        np.testing.assert_allclose(out[key], ref, rtol=0, atol=TOL[key] * np.abs(ref).max(), err_msg=key)


def test_packed_parameters_follow_the_kernel_layout() -> None:
    g, meta, sd = _case()
    cfg = RVERNOModelConfig(**{k: v for k, v in meta["model"].items() if k != "device"})
    packed = pack_state_dict(cfg, sd).astype(np.float64)
    lib = _native.load_library()
    assert packed.size == lib.cib_energy_rno_param_count(cfg.hidden_size, cfg.hidden_layers, cfg.latent_dimension)
    H, NL, L = cfg.hidden_size, cfg.hidden_layers, cfg.latent_dimension
    offset = 0
    for prefix, n_in, n_out, bias in (("equilibrium_energy.network.network", 6, 1, False),
                                      ("nonequilibrium_energy.network.network", 6 + L, 1, False),
                                      ("state_evolution.network", 6 + L, L, True)):  # fmt: skip
        for layer in range(NL):
            n_l = n_in if layer == 0 else H
            w = packed[offset:offset + H * n_l].reshape(H, n_l)
            wt = packed[offset + H * n_l:offset + 2 * H * n_l].reshape(n_l, H)
            b = packed[offset + 2 * H * n_l:offset + 2 * H * n_l + H]
            np.testing.assert_array_equal(w, sd[f"{prefix}.{2 * layer}.weight"])
            np.testing.assert_array_equal(wt, w.T)
            np.testing.assert_array_equal(b, sd[f"{prefix}.{2 * layer}.bias"])
            offset += 2 * H * n_l + H
        np.testing.assert_array_equal(packed[offset:offset + n_out * H].reshape(n_out, H), sd[f"{prefix}.{2 * NL}.weight"])
        ref_b = sd[f"{prefix}.{2 * NL}.bias"] if bias else np.zeros(n_out)
        np.testing.assert_array_equal(packed[offset + n_out * H:offset + n_out * H + n_out], ref_b)
        offset += n_out * H + n_out
    assert offset == packed.size
    with pytest.raises(KeyError):
        pack_state_dict(cfg, dict(sd, extra=np.zeros(1)))
    with pytest.raises(ValueError):
        RVERNOModelConfig(**dict({k: v for k, v in meta["model"].items() if k != "device"}, strain_input_scale=(1.0,)))


def test_loader_rejects_mismatched_artifact_metadata(tmp_path) -> None:
    """The architecture contract is checked before any device work (deployment.py:36-57)."""
    import json

    from concrete_impact_b200.energy_rno import load_rve_rno_state_dict

    _, meta, _ = _case()
    spec = {k: v for k, v in meta["model"].items() if k != "device"}
    metadata = {"model_family": spec["family"], "deployment_integrator": "explicit_only",
                **{k: spec[k] for k in ("integrator", "evolution", "reference_time_scale", "latent_dimension",
                                        "hidden_size", "hidden_layers", "activation", "dtype")}}  # fmt: skip
    metadata["hidden_size"] = 64
    (tmp_path / "meta.json").write_text(json.dumps(metadata))
    with pytest.raises(ValueError, match="does not match"):
        load_rve_rno_state_dict(RVERNOModelConfig(**spec), tmp_path / "missing.pt", tmp_path / "meta.json")
    with pytest.raises(ValueError):
        RVERNOModelConfig(**dict(spec, integrator="backward_euler"))
    with pytest.raises(ValueError):
        RVERNOModelConfig(**dict(spec, reference_time_scale=0.0))


def test_oracle_tangent_matches_reference_autograd_tangent() -> None:
    """Central differences of the float64 update against the reference's FP32 autograd
    tangent of 16 points at the last rollout step (the GPU path does not provide it yet)."""
    g, meta, sd = _case()
    last = meta["steps"] - 1
    ref = g["tangent_last16"]
    tan = oe.tangent_fd(sd, g["strain"][last][:16], g["latent_in"][last][:16], g["time_step"][:16],
                        meta["model"]["reference_time_scale"], meta["model"]["integrator"])  # fmt: skip
    np.testing.assert_allclose(tan, ref, rtol=0, atol=1e-4 * np.abs(ref).max())
