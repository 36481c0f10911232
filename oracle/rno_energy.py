"""NumPy oracle of the reference's energy-based RVE-RNO update -- test infrastructure only.

Float64 restatement of
  ScalarMLP.value_and_input_gradient   src/concrete_impact/nn/models/rve_rno.py:110-129
  MultilayerPerceptron (SiLU)          :63-93
  prepare_energy_anchors               :227-247
  _constitutive_tensors                :334-418 (direct_rate evolution, both integrators)
on a state dict with the reference's key names.
"""

from __future__ import annotations

import numpy as np


def _silu(z):
    return z / (1.0 + np.exp(-z))


def _silu_prime(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def _layers(sd: dict, prefix: str):
    ws, bs = [], []
    i = 0
    while f"{prefix}.{i}.weight" in sd:
        ws.append(np.asarray(sd[f"{prefix}.{i}.weight"], dtype=np.float64))
        b = sd.get(f"{prefix}.{i}.bias")
        bs.append(None if b is None else np.asarray(b, dtype=np.float64))
        i += 2
    return ws, bs


def mlp(sd: dict, prefix: str, x: np.ndarray) -> np.ndarray:
    ws, bs = _layers(sd, prefix)
    h = x
    for w, b in zip(ws[:-1], bs[:-1]):
        h = _silu(h @ w.T + b)
    out = h @ ws[-1].T
    return out if bs[-1] is None else out + bs[-1]


def value_and_gradient(sd: dict, prefix: str, x: np.ndarray):
    """Scalar potential and its input gradient (hand-written backward, as the reference)."""
    ws, bs = _layers(sd, prefix)
    h, zs = x, []
    for w, b in zip(ws[:-1], bs[:-1]):
        z = h @ w.T + b
        zs.append(z)
        h = _silu(z)
    value = (h @ ws[-1].T)[..., 0]
    g = np.broadcast_to(ws[-1][0], h.shape)
    for w, z in zip(reversed(ws[:-1]), reversed(zs)):
        g = (g * _silu_prime(z)) @ w
    return value, g


def anchors(sd: dict, latent: int) -> dict:
    ve, ge = value_and_gradient(sd, "equilibrium_energy.network.network", np.zeros((1, 6)))
    vn, gn = value_and_gradient(sd, "nonequilibrium_energy.network.network", np.zeros((1, 6 + latent)))
    return {"eq_value": ve[0], "eq_grad": ge[0], "neq_value": vn[0], "neq_grad": gn[0, :6]}


def update(sd: dict, strain, latent, time_step, reference_time_scale: float, integrator: str,
           strain_scale=None, anchor: dict | None = None) -> dict:  # fmt: skip
    """One update of every point (direct_rate evolution)."""
    strain = np.asarray(strain, dtype=np.float64)
    latent = np.asarray(latent, dtype=np.float64)
    scale = np.ones(6) if strain_scale is None else np.asarray(strain_scale, dtype=np.float64)
    a = anchor or anchors(sd, latent.shape[1])
    x = strain / scale
    ve, ge = value_and_gradient(sd, "equilibrium_energy.network.network", x)
    equilibrium = ve - a["eq_value"] - (x * a["eq_grad"]).sum(-1)
    eq_stress = (ge - a["eq_grad"]) / scale
    prev_state = np.concatenate([x, latent], axis=-1)
    vp, gp = value_and_gradient(sd, "nonequilibrium_energy.network.network", prev_state)
    prev_neq = vp - a["neq_value"] - (x * a["neq_grad"]).sum(-1)
    beta = gp[:, 6:]
    rate_dimless = mlp(sd, "state_evolution.network", prev_state)
    rate = rate_dimless / reference_time_scale
    dissipation = -(beta * rate).sum(-1)
    candidate = latent + (np.asarray(time_step, dtype=np.float64) / reference_time_scale)[:, None] * rate_dimless
    vc, gc = value_and_gradient(sd, "nonequilibrium_energy.network.network", np.concatenate([x, candidate], axis=-1))
    cand_neq = vc - a["neq_value"] - (x * a["neq_grad"]).sum(-1)
    if integrator == "current_state_stress_forward_euler":
        resp_neq, resp_stress = cand_neq, (gc[:, :6] - a["neq_grad"]) / scale
    else:
        resp_neq, resp_stress = prev_neq, (gp[:, :6] - a["neq_grad"]) / scale
    return {"stress": eq_stress + resp_stress, "latent_state": candidate, "state_rate": rate,
            "dimensionless_state_rate": rate_dimless, "dissipation": dissipation,
            "free_energy": equilibrium + resp_neq, "thermodynamic_violation": np.maximum(-dissipation, 0.0),
            "nonequilibrium_energy_increment": cand_neq - prev_neq}  # fmt: skip


def tangent_fd(sd: dict, strain, latent, time_step, reference_time_scale: float, integrator: str,
               strain_scale=None, anchor: dict | None = None, relative_step: float = 1.0e-6) -> np.ndarray:
    """d stress / d strain (B, 6, 6) by central differences of ``update`` in float64 -- the
    quantity the reference obtains by automatic differentiation (rve_rno.py:280-293), with
    the candidate latent state following the strain through the forward-Euler step."""
    strain = np.asarray(strain, dtype=np.float64)
    a = anchor or anchors(sd, np.asarray(latent).shape[1])
    h = relative_step * max(float(np.abs(strain).max()), 1.0e-3)
    out = np.zeros((strain.shape[0], 6, 6))
    for c in range(6):
        e = np.zeros(6)
        e[c] = h
        plus = update(sd, strain + e, latent, time_step, reference_time_scale, integrator, strain_scale, a)["stress"]
        minus = update(sd, strain - e, latent, time_step, reference_time_scale, integrator, strain_scale, a)["stress"]
        out[:, :, c] = (plus - minus) / (2.0 * h)
    return out
