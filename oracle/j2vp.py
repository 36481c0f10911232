"""NumPy oracle of the J2 Perzyna return map -- test infrastructure only.

Vectorised restatement of the reference's
  _update_points                         src/fem/materials/plasticity.py:343-431
  _update_j2_viscoplastic_point          src/fem/materials/plasticity.py:526-681
  _append_j2_increment_diagnostics       src/fem/materials/plasticity.py:684-708
  _solve_j2_viscoplastic_multiplier      src/fem/materials/plasticity.py:711-854
  _compute_j2_viscoplastic_hv            src/fem/materials/plasticity.py:907-926
  _j2_viscoplastic_consistent_tangent    src/fem/materials/plasticity.py:929-963
  _elasticity_matrix / _compute_j2_equivalent_stress   :1408-1465
evaluated for all points at once in float64 (or float32 to model the FP32 kernels).
Failures are reported as per-point status codes with the numbering of include/cib200.h.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

OK = 0
NON_FINITE_J2_INVARIANT = 1
NEGATIVE_J2_INVARIANT = 2
INVALID_YIELD_ACTIVATION_TOLERANCE = 3
NON_FINITE_CLOSED_FORM = 4
CLOSED_FORM_SOLUTION_OUT_OF_BOUNDS = 5
INVALID_ITERATION_LIMIT = 6
NON_FINITE_PROBLEM_SCALE = 7
INVALID_CORRECTED_OVERSTRESS = 8
NON_FINITE_ITERATION_VALUE = 9
NON_POSITIVE_DERIVATIVE = 10
CONVERGED_SOLUTION_OUT_OF_BOUNDS = 11
NON_FINITE_NEWTON_CANDIDATE = 12
NEWTON_CANDIDATE_OUT_OF_BOUNDS = 13
MAXIMUM_ITERATIONS_EXCEEDED = 14
NON_POSITIVE_TANGENT_OVERSTRESS = 15

REASONS = [
    "ok", "non_finite_j2_invariant", "negative_j2_invariant", "invalid_yield_activation_tolerance",
    "non_finite_closed_form", "closed_form_solution_out_of_bounds", "invalid_iteration_limit",
    "non_finite_problem_scale", "invalid_corrected_overstress", "non_finite_iteration_value",
    "non_positive_derivative", "converged_solution_out_of_bounds", "non_finite_newton_candidate",
    "newton_candidate_out_of_bounds", "maximum_iterations_exceeded", "non_positive_tangent_overstress",
]  # fmt: skip

DIAGNOSTIC_NAMES = [
    "yield_value", "plastic_work", "local_iterations", "active_surface", "plastic_multiplier",
    "viscoplastic_multiplier", "equivalent_stress", "trial_yield_value", "yield_scale",
    "yield_activation_threshold", "yield_activation_margin", "viscoplastic_active", "time_step",
    "equivalent_plastic_strain", "viscoplastic_hv", "plastic_power", "hardening_storage_rate",
    "local_residual", "root_lower_bound", "root_upper_bound", "incremental_work_density",
    "equivalent_stress_increment",
]  # fmt: skip

STRESS_WEIGHTS = np.asarray([1.0, 1.0, 1.0, 2.0, 2.0, 2.0])
ENGINEERING = np.asarray([1.0, 1.0, 1.0, 2.0, 2.0, 2.0])


@dataclass(frozen=True)
class J2Params:
    """J2ViscoplasticMaterial parameters plus MaterialUpdateSettings."""

    young_modulus: float
    poisson_ratio: float
    yield_stress: float
    hardening_modulus: float
    time_scale: float
    reference_stress: float
    rate_exponent: float
    max_iterations: int = 50
    yield_relative_tolerance: float = 1.0e-10
    residual_absolute_tolerance: float = 1.0e-12
    residual_relative_tolerance: float = 1.0e-10

    @property
    def shear_modulus(self) -> float:
        return self.young_modulus / (2.0 * (1.0 + self.poisson_ratio))

    @property
    def bulk_modulus(self) -> float:
        return self.young_modulus / (3.0 * (1.0 - 2.0 * self.poisson_ratio))

    @property
    def lame_lambda(self) -> float:
        e, nu = self.young_modulus, self.poisson_ratio
        return e * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))


def elasticity_matrix(young_modulus: float, poisson_ratio: float) -> np.ndarray:
    """Isotropic 6x6 stiffness for engineering shear strains (plasticity.py:1408-1423)."""
    g = young_modulus / (2.0 * (1.0 + poisson_ratio))
    lam = young_modulus * poisson_ratio / ((1.0 + poisson_ratio) * (1.0 - 2.0 * poisson_ratio))
    c = np.zeros((6, 6))
    c[:3, :3] = lam
    c[[0, 1, 2], [0, 1, 2]] += 2.0 * g
    c[[3, 4, 5], [3, 4, 5]] = g
    return c


def deviatoric(stress: np.ndarray) -> np.ndarray:
    """Rows minus their mean normal stress on the normal components (plasticity.py:1473-1475)."""
    dev = stress.copy()
    dev[..., :3] -= (np.sum(stress[..., :3], axis=-1) / 3.0)[..., None]
    return dev


def j2_radicand(dev: np.ndarray) -> np.ndarray:
    """1.5 * sum(w_i s_i^2) (plasticity.py:1441-1465)."""
    return 1.5 * np.sum(STRESS_WEIGHTS * dev * dev, axis=-1)


def _solve_multiplier(p: J2Params, ftr, dt, dtype):
    """Vectorised _solve_j2_viscoplastic_multiplier; returns (dgamma, iterations, residual, status)."""
    one = dtype(1.0)
    g = dtype(p.shear_modulus)
    slope = dtype(3.0 * p.shear_modulus + p.hardening_modulus)
    upper = ftr / slope
    tol = np.where(dtype(p.residual_relative_tolerance) * upper > dtype(p.residual_absolute_tolerance),
                   dtype(p.residual_relative_tolerance) * upper, dtype(p.residual_absolute_tolerance))  # fmt: skip
    n = ftr.shape[0]
    status = np.zeros(n, dtype=np.int32)
    dgamma = np.zeros(n, dtype=dtype)
    iters = np.zeros(n, dtype=np.int32)
    residual = np.zeros(n, dtype=dtype)
    tau_sref = dtype(p.time_scale * p.reference_stress)
    if p.rate_exponent == 1.0:
        with np.errstate(all="ignore"):
            denom = tau_sref / dtype(dt) + slope
            x = ftr / denom
            corr = ftr - slope * x
            res = x - dtype(dt) * corr / tau_sref
            der = one + dtype(dt) * slope / tau_sref
        finite = np.isfinite(denom) & np.isfinite(x) & np.isfinite(corr) & np.isfinite(res) & np.isfinite(der)
        status[~finite] = NON_FINITE_CLOSED_FORM
        bad = finite & (~((x > 0) & (x < upper)) | (corr <= 0))
        status[bad] = CLOSED_FORM_SOLUTION_OUT_OF_BOUNDS
        return x, iters, res, status
    if p.max_iterations <= 0:
        status[:] = INVALID_ITERATION_LIMIT
        return dgamma, iters, residual, status
    scale_ok = np.isfinite(upper) & np.isfinite(tol)
    status[~scale_ok] = NON_FINITE_PROBLEM_SCALE
    x = dtype(0.5) * upper
    live = scale_ok.copy()
    m = dtype(p.rate_exponent)
    sref = dtype(p.reference_stress)
    tau = dtype(p.time_scale)
    del g
    for it in range(1, p.max_iterations + 1):
        if not live.any():
            break
        with np.errstate(all="ignore"):
            over = ftr - slope * x
            nov = over / sref
            bad = live & (~np.isfinite(nov) | (nov <= 0))
            status[bad] = INVALID_CORRECTED_OVERSTRESS
            live &= ~bad
            rate = np.power(nov, m) / tau
            res = x - dtype(dt) * rate
            der = one + dtype(dt) * m * slope * np.power(nov, m - one) / (tau * sref)
        bad = live & ~(np.isfinite(rate) & np.isfinite(res) & np.isfinite(der))
        status[bad] = NON_FINITE_ITERATION_VALUE
        live &= ~bad
        bad = live & (der <= 0)
        status[bad] = NON_POSITIVE_DERIVATIVE
        live &= ~bad
        conv = live & (np.abs(res) <= tol)
        oob = conv & (~((x > 0) & (x < upper)) | (over <= 0))
        status[oob] = CONVERGED_SOLUTION_OUT_OF_BOUNDS
        ok = conv & ~oob
        dgamma[ok] = x[ok]
        iters[ok] = it
        residual[ok] = res[ok]
        live &= ~conv
        with np.errstate(all="ignore"):
            cand = x - res / der
        bad = live & ~np.isfinite(cand)
        status[bad] = NON_FINITE_NEWTON_CANDIDATE
        live &= ~bad
        bad = live & ~((cand > 0) & (cand < upper))
        status[bad] = NEWTON_CANDIDATE_OUT_OF_BOUNDS
        live &= ~bad
        if it == p.max_iterations:
            status[live] = MAXIMUM_ITERATIONS_EXCEEDED
            live[:] = False
        x = np.where(live, cand, x)
    return dgamma, iters, residual, status


def return_map(p: J2Params, trial_stress: np.ndarray, eqps_n: np.ndarray, dt: float, dtype=np.float64) -> dict:
    """Return map from trial stresses (n,6) and committed equivalent plastic strain (n,).

    Returns a dict with stress, flow direction n, dgamma, q_tr, f_tr, yield_scale,
    threshold, hv, tan_f, tan_c, local_residual, iterations, active and status.
    """
    sig = np.asarray(trial_stress, dtype=dtype)
    nrm = sig.shape[0]
    dev = deviatoric(sig)
    with np.errstate(all="ignore"):
        rad = j2_radicand(dev).astype(dtype)
    status = np.zeros(nrm, dtype=np.int32)
    status[~np.isfinite(rad)] = NON_FINITE_J2_INVARIANT
    status[np.isfinite(rad) & (rad < 0)] = NEGATIVE_J2_INVARIANT
    with np.errstate(all="ignore"):
        q = np.sqrt(np.where(status == OK, rad, 0)).astype(dtype)
        radius = dtype(p.yield_stress) + dtype(p.hardening_modulus) * np.asarray(eqps_n).astype(dtype)
        ftr = q - radius
    ys = np.maximum(np.maximum(dtype(p.yield_stress), dtype(p.reference_stress)), q).astype(dtype)
    thr = dtype(p.yield_relative_tolerance) * ys
    tol_bad = (not np.isfinite(p.yield_relative_tolerance)) or p.yield_relative_tolerance < 0.0
    status[(status == OK) & (tol_bad | ~np.isfinite(thr))] = INVALID_YIELD_ACTIVATION_TOLERANCE
    active = (status == OK) & (ftr > thr)
    g = dtype(p.shear_modulus)
    nvec = np.zeros_like(sig)
    with np.errstate(all="ignore"):
        nvec[active] = dtype(1.5) * dev[active] / q[active, None]
    dgamma = np.zeros(nrm, dtype=dtype)
    iters = np.zeros(nrm, dtype=np.int32)
    local_res = np.zeros(nrm, dtype=dtype)
    if active.any():
        dg, it, res, st = _solve_multiplier(p, ftr[active], dt, dtype)
        dgamma[active] = dg
        iters[active] = it
        local_res[active] = res
        status[active] = st
    active &= status == OK
    stress = sig - (dtype(2.0) * g * dgamma)[:, None] * nvec
    slope = dtype(3.0 * p.shear_modulus + p.hardening_modulus)
    hv = np.zeros(nrm, dtype=dtype)
    if p.rate_exponent == 1.0:
        hv[active] = dtype(p.time_scale * p.reference_stress) / dtype(dt) + slope
    elif active.any():
        qf = np.sqrt(j2_radicand(deviatoric(stress[active]))).astype(dtype)
        fy = qf - (dtype(p.yield_stress) + dtype(p.hardening_modulus) * (eqps_n[active] + dgamma[active]).astype(dtype))
        idx = np.flatnonzero(active)
        badt = fy <= 0
        status[idx[badt]] = NON_POSITIVE_TANGENT_OVERSTRESS
        with np.errstate(all="ignore"):
            m = dtype(p.rate_exponent)
            flow = m * np.power(fy / dtype(p.reference_stress), m - 1) / dtype(p.time_scale * p.reference_stress)
            hv[active] = dtype(1.0) / (dtype(dt) * flow) + slope
        active &= status == OK
    tan_f = np.full(nrm, dtype(2.0) * g, dtype=dtype)
    tan_c = np.zeros(nrm, dtype=dtype)
    with np.errstate(all="ignore"):
        tan_f[active] = dtype(2.0) * g - dtype(6.0) * g * g * dgamma[active] / q[active]
        tan_c[active] = dtype(4.0) * g * g * (dgamma[active] / q[active] - dtype(1.0) / hv[active])
    return {
        "stress": stress, "n": nvec, "dgamma": dgamma, "q_tr": q, "f_tr": ftr, "yield_scale": ys,
        "threshold": thr, "hv": hv, "tan_f": tan_f, "tan_c": tan_c, "local_residual": local_res,
        "iterations": iters, "active": active, "status": status,
    }  # fmt: skip


def consistent_tangent(p: J2Params, rm: dict, dtype=np.float64) -> np.ndarray:
    """6x6 tangents (n,6,6): elasticity for elastic points, plasticity.py:929-963 otherwise."""
    nrm = rm["stress"].shape[0]
    c_el = elasticity_matrix(p.young_modulus, p.poisson_ratio).astype(dtype)
    tan = np.repeat(c_el[None], nrm, axis=0)
    act = rm["active"]
    if act.any():
        vol = np.zeros((6, 6), dtype=dtype)
        vol[:3, :3] = dtype(p.bulk_modulus)
        dev = np.zeros((6, 6), dtype=dtype)
        dev[:3, :3] = -dtype(1.0 / 3.0)
        dev[[0, 1, 2], [0, 1, 2]] += dtype(1.0)
        dev[[3, 4, 5], [3, 4, 5]] = dtype(0.5)
        n = rm["n"][act]
        tan[act] = (vol[None] + rm["tan_f"][act, None, None] * dev[None]
                    + rm["tan_c"][act, None, None] * (n[:, :, None] * n[:, None, :]))  # fmt: skip
    return tan


def update_reference_form(
    p: J2Params,
    strains: np.ndarray,
    plastic_strain: np.ndarray,
    eqps: np.ndarray,
    vpm: np.ndarray,
    dt: float,
    strain_rates: np.ndarray | None = None,
) -> dict:
    """J2ViscoplasticMaterial.update with all outputs (float64).

    Returns stresses, tangents, free_energy, dissipation, the state arrays and the
    diagnostics dict with the reference's keys, plus per-point ``status``.
    """
    strains = np.asarray(strains, dtype=np.float64)
    c_el = elasticity_matrix(p.young_modulus, p.poisson_ratio)
    trial = (strains - plastic_strain) @ c_el.T
    rm = return_map(p, trial, eqps, dt)
    act = rm["active"]
    dg = rm["dgamma"]
    inc = dg[:, None] * ENGINEERING[None, :] * rm["n"]
    ep1 = plastic_strain + inc
    q1 = eqps + dg
    vpm1 = vpm + dg
    stress = rm["stress"]
    status = rm["status"].copy()
    qf = np.where(act, np.sqrt(np.maximum(j2_radicand(deviatoric(stress)), 0.0)), rm["q_tr"])
    fy = np.where(act, qf - (p.yield_stress + p.hardening_modulus * q1), rm["f_tr"])
    pw = np.where(act, np.sum(stress * inc, axis=1), 0.0)
    eel = strains - ep1
    psi = 0.5 * np.sum((eel @ c_el.T) * eel, axis=1) + 0.5 * p.hardening_modulus * q1**2
    hard = np.where(act, p.hardening_modulus * q1 * dg / dt, 0.0)
    diss = np.where(act, pw / dt - hard, 0.0)
    slope = 3.0 * p.shear_modulus + p.hardening_modulus
    diag = {
        "yield_value": fy,
        "plastic_work": pw,
        "local_iterations": rm["iterations"].astype(np.float64),
        "active_surface": np.where(act, 4.0, 0.0),
        "plastic_multiplier": dg,
        "viscoplastic_multiplier": dg,
        "equivalent_stress": qf,
        "trial_yield_value": rm["f_tr"],
        "yield_scale": rm["yield_scale"],
        "yield_activation_threshold": rm["threshold"],
        "yield_activation_margin": (rm["f_tr"] - rm["threshold"]) / rm["yield_scale"],
        "viscoplastic_active": np.where(act, 1.0, 0.0),
        "time_step": np.full(strains.shape[0], float(dt)),
        "equivalent_plastic_strain": q1,
        "plastic_power": np.where(act, pw / dt, 0.0),
        "hardening_storage_rate": hard,
        "local_residual": np.where(act, rm["local_residual"], 0.0),
        "root_lower_bound": np.zeros(strains.shape[0]),
        "root_upper_bound": np.where(act, rm["f_tr"] / slope, 0.0),
    }
    if act.any():
        diag["viscoplastic_hv"] = np.where(act, rm["hv"], 0.0)
    if strain_rates is not None:
        de = dt * np.asarray(strain_rates, dtype=np.float64)
        sprev = ((strains - de) - plastic_strain) @ c_el.T
        with np.errstate(all="ignore"):
            rp = j2_radicand(deviatoric(sprev))
            rc = j2_radicand(deviatoric(stress))
        bad = (status == OK) & ~(np.isfinite(rp) & np.isfinite(rc))
        status[bad] = NON_FINITE_J2_INVARIANT
        diag["incremental_work_density"] = 0.5 * np.sum((sprev + stress) * de, axis=1)
        with np.errstate(all="ignore"):
            diag["equivalent_stress_increment"] = np.sqrt(rc) - np.sqrt(rp)
    return {
        "stresses": stress,
        "tangents": consistent_tangent(p, rm),
        "free_energy": psi,
        "dissipation": diss,
        "plastic_strain": ep1,
        "equivalent_plastic_strain": q1,
        "viscoplastic_multiplier": vpm1,
        "diagnostics": diag,
        "status": status,
    }


def update_incremental(
    p: J2Params,
    dstrain: np.ndarray,
    stress_n: np.ndarray,
    plastic_strain_n: np.ndarray,
    eqps_n: np.ndarray,
    dt: float,
    dtype=np.float64,
) -> dict:
    """Batched incremental form with stress-carried state, points as rows (n,6).

    Trial stress = stress_n + C dstrain (the reference's C(strain - plastic_strain) with
    strain = C^-1 stress_n + plastic_strain_n + dstrain).  ``dtype`` float32 models the
    FP32 kernels (equivalent plastic strain history stays float64).
    """
    c_el = elasticity_matrix(p.young_modulus, p.poisson_ratio).astype(dtype)
    trial = np.asarray(stress_n, dtype=dtype) + np.asarray(dstrain, dtype=dtype) @ c_el.T
    rm = return_map(p, trial, np.asarray(eqps_n, dtype=np.float64), dt, dtype=dtype)
    dg = rm["dgamma"]
    ep1 = np.asarray(plastic_strain_n, dtype=dtype) + dg[:, None] * ENGINEERING.astype(dtype)[None, :] * rm["n"]
    return {
        "stress": rm["stress"],
        "plastic_strain": ep1,
        "eqps": np.asarray(eqps_n, dtype=np.float64) + dg.astype(np.float64),
        "tangent": consistent_tangent(p, rm, dtype=dtype),
        "active": rm["active"],
        "status": rm["status"],
    }


def config1_inputs(n: int, seed: int = 1234, dtype=np.float64) -> dict:
    """Seeded synthetic batch of the isolated return-map workload, points as rows.

    Strain increments N(0, 2e-4^2) per component; equivalent plastic strain U[0, 0.01];
    plastic strain zero; stress = random deviatoric direction scaled to q = U[0.8, 1.0]
    times the current yield radius (mortar: E 25 GPa, nu 0.2, sigma_y 20 MPa, H 2 GPa).
    """
    rng = np.random.default_rng(seed)
    p = mortar_params()
    eqps = rng.uniform(0.0, 0.01, size=n)
    direction = rng.standard_normal((n, 6))
    direction = deviatoric(direction)
    qdir = np.sqrt(j2_radicand(direction))
    radius = p.yield_stress + p.hardening_modulus * eqps
    stress = direction * (rng.uniform(0.8, 1.0, size=n) * radius / qdir)[:, None]
    dstrain = rng.normal(0.0, 2.0e-4, size=(n, 6))
    return {
        "dstrain": dstrain.astype(dtype),
        "stress": stress.astype(dtype),
        "plastic_strain": np.zeros((n, 6), dtype=dtype),
        "eqps": eqps,
        "dt": 1.0e-5,
    }


def mortar_params() -> J2Params:
    """Mortar phase of the two-phase RVE: J2 Perzyna, m = 1, eta = 1e-3 s."""
    return J2Params(
        young_modulus=25.0e9,
        poisson_ratio=0.2,
        yield_stress=20.0e6,
        hardening_modulus=2.0e9,
        time_scale=1.0e-3,
        reference_stress=20.0e6,
        rate_exponent=1.0,
    )
