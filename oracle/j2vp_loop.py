"""Per-point oracle of the J2 Perzyna update -- test infrastructure only.

Restates the reference's own execution shape: a Python loop over points
(src/fem/materials/plasticity.py:364-420) in which each point builds the trial stress
with a 6x6 matrix-vector product, solves the multiplier, assembles the 6x6 consistent
tangent from the projection matrices (:929-963), and fills a per-point diagnostics record
that is scattered into batch arrays (:1662-1694), plus the increment diagnostics
(:684-708).  The reference itself cannot travel to a machine without its checkout, so
this port stands in for it when timing the reference's CPU cost; the vectorised oracle
(oracle.j2vp) is the one used for checking.
"""

from __future__ import annotations

import math

import numpy as np

from .j2vp import ENGINEERING, J2Params, elasticity_matrix

IDENTITY = np.asarray([1.0, 1.0, 1.0, 0.0, 0.0, 0.0])
WEIGHTS = np.asarray([1.0, 1.0, 1.0, 2.0, 2.0, 2.0])
E2T = np.diag([1.0, 1.0, 1.0, 0.5, 0.5, 0.5])
P_VOL = np.outer(IDENTITY, IDENTITY) / 3.0
P_DEV = np.eye(6) - P_VOL


def _q(dev: np.ndarray) -> float:
    radicand = 1.5 * float(np.sum(WEIGHTS * dev * dev))
    if not math.isfinite(radicand) or radicand < 0.0:
        raise FloatingPointError("invalid J2 invariant")
    return math.sqrt(radicand)


def _dev(s: np.ndarray) -> np.ndarray:
    return s - (float(np.sum(s[:3])) / 3.0) * IDENTITY


def _point(p: J2Params, c_el, g, k, strain, ep, q0, dt):
    trial = c_el @ (strain - ep)
    dev = _dev(trial)
    q = _q(dev)
    ftr = q - (p.yield_stress + p.hardening_modulus * q0)
    scale = max(p.yield_stress, p.reference_stress, q)
    thr = p.yield_relative_tolerance * scale
    diag = {"trial_yield_value": ftr, "yield_scale": scale, "yield_activation_threshold": thr,
            "yield_activation_margin": (ftr - thr) / scale, "time_step": dt}  # fmt: skip
    if ftr <= thr:
        eel = strain - ep
        diag.update(plastic_multiplier=0.0, viscoplastic_active=0.0, equivalent_plastic_strain=q0, yield_value=ftr,
                    equivalent_stress=q, plastic_work=0.0, active_surface=0.0)  # fmt: skip
        return trial, ep.copy(), q0, c_el, 0.5 * float((c_el @ eel) @ eel) + 0.5 * p.hardening_modulus * q0**2, 0.0, diag
    n = 1.5 * dev / q
    slope = 3.0 * g + p.hardening_modulus
    tau_sref = p.time_scale * p.reference_stress
    if p.rate_exponent == 1.0:
        dg = ftr / (tau_sref / dt + slope)
        hv = tau_sref / dt + slope
    else:
        upper = ftr / slope
        tol = max(p.residual_absolute_tolerance, p.residual_relative_tolerance * upper)
        dg = 0.5 * upper
        for _ in range(p.max_iterations):
            nov = (ftr - slope * dg) / p.reference_stress
            res = dg - dt * nov**p.rate_exponent / p.time_scale
            if abs(res) <= tol:
                break
            der = 1.0 + dt * p.rate_exponent * slope * nov ** (p.rate_exponent - 1.0) / tau_sref
            dg -= res / der
        fy = q - 3.0 * g * dg - (p.yield_stress + p.hardening_modulus * (q0 + dg))
        hv = 1.0 / (dt * p.rate_exponent * (fy / p.reference_stress) ** (p.rate_exponent - 1.0) / tau_sref) + slope
    stress = trial - 2.0 * g * dg * n
    inc = dg * (np.diag(ENGINEERING) @ n)
    ep1 = ep + inc
    q1 = q0 + dg
    tangent = (3.0 * k * E2T @ P_VOL + (2.0 * g - 6.0 * g * g * dg / q) * E2T @ P_DEV
               + 4.0 * g * g * (dg / q - 1.0 / hv) * np.outer(n, n))  # fmt: skip
    qf = _q(_dev(stress))
    pw = float(stress @ inc)
    eel = strain - ep1
    psi = 0.5 * float((c_el @ eel) @ eel) + 0.5 * p.hardening_modulus * q1**2
    diss = pw / dt - p.hardening_modulus * q1 * dg / dt
    diag.update(plastic_multiplier=dg, viscoplastic_active=1.0, equivalent_plastic_strain=q1,
                yield_value=qf - (p.yield_stress + p.hardening_modulus * q1), equivalent_stress=qf, plastic_work=pw,
                active_surface=4.0, viscoplastic_hv=hv)  # fmt: skip
    return stress, ep1, q1, tangent, psi, diss, diag


def update_points_loop(p: J2Params, strains, plastic_strain, eqps, dt, strain_rates=None) -> dict:
    """Reference-shaped per-point batch update of (n,6) arrays; returns the batch outputs."""
    c_el = elasticity_matrix(p.young_modulus, p.poisson_ratio)
    g, k = p.shear_modulus, p.bulk_modulus
    n = strains.shape[0]
    stresses = np.zeros((n, 6))
    tangents = np.zeros((n, 6, 6))
    ep_out = np.array(plastic_strain, copy=True)
    q_out = np.array(eqps, copy=True)
    psi = np.zeros(n)
    diss = np.zeros(n)
    diagnostics: dict[str, np.ndarray] = {}
    for i in range(n):
        s, ep1, q1, tan, e, d, diag = _point(p, c_el, g, k, strains[i], plastic_strain[i], float(eqps[i]), dt)
        if strain_rates is not None:
            de = dt * strain_rates[i]
            sprev = c_el @ ((strains[i] - de) - plastic_strain[i])
            diag["incremental_work_density"] = 0.5 * float((sprev + s) @ de)
            diag["equivalent_stress_increment"] = _q(_dev(s)) - _q(_dev(sprev))
        stresses[i] = s
        tangents[i] = tan
        ep_out[i] = ep1
        q_out[i] = q1
        psi[i] = e
        diss[i] = d
        for name, value in diag.items():
            if name not in diagnostics:
                diagnostics[name] = np.zeros(n)
            diagnostics[name][i] = value
    return {"stresses": stresses, "tangents": tangents, "plastic_strain": ep_out, "equivalent_plastic_strain": q_out,
            "free_energy": psi, "dissipation": diss, "diagnostics": diagnostics}  # fmt: skip
