"""NumPy/SciPy oracle of implicit Newmark material dynamics -- test infrastructure only.

Restates, with direct sparse solves on structured Hex8 bars, the reference's
  solve_material_implicit_newmark      src/fem/dynamics/material.py:300-443
  _solve_implicit_step                 src/fem/dynamics/material.py:446-662
  _evaluate_implicit_trial             src/fem/dynamics/material.py:665-701
  assemble_consistent_mass_matrix      src/fem/assembly/elasticity.py:50-70, 109-140
  cut_back_time_step / grow_time_step  src/fem/solvers/time_step.py:12-31
  perform_armijo_search                src/fem/solvers/line_search.py:40-67
  energy histories                     src/fem/dynamics/material.py:781-927
with a pointwise macro material: the J2 Perzyna oracle (``PointJ2``) or one periodic RVE
oracle solve per macro point (``PointRVE``, the FE2 case of RVEHomogenizedMaterial).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
from scipy.sparse import coo_matrix
from scipy.sparse.linalg import spsolve

from . import j2vp as oj
from .fe2 import _shape_values
from .rve import RVEOracle, b_matrices


class RecoverableStepError(RuntimeError):
    """A step failure that the adaptive controller may retry with a smaller step."""

    def __init__(self, reason: str) -> None:
        super().__init__(reason)
        self.reason = reason


def consistent_mass(nodes, elements, density: float):
    """rho * sum_q N^T N detJ over 2x2x2 Gauss points (CSR, DOF 3 n + c)."""
    g = 1.0 / math.sqrt(3.0)
    pts = np.asarray([(a, b, c) for a in (-g, g) for b in (-g, g) for c in (-g, g)])
    nq = _shape_values(pts)  # (q, 8)
    _, det = b_matrices(nodes, elements)
    me = density * np.einsum("qa,qb,eq->eab", nq, nq, det)  # (E, 8, 8)
    ne = elements.shape[0]
    rows, cols, vals = [], [], []
    for c in range(3):
        dof = 3 * elements + c
        rows.append(np.repeat(dof, 8, axis=1).ravel())
        cols.append(np.tile(dof, (1, 8)).ravel())
        vals.append(me.reshape(ne, 64).ravel())
    n3 = 3 * nodes.shape[0]
    return coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n3, n3)).tocsr()


class PointJ2:
    """J2ViscoplasticMaterial at every macro point (oracle.j2vp, reference form)."""

    def __init__(self, params: oj.J2Params) -> None:
        self.params = params

    def initial_state(self, n: int) -> dict:
        return {"plastic_strain": np.zeros((n, 6)), "eqps": np.zeros(n), "vpm": np.zeros(n)}

    def update(self, strains, rates, dt, state, need_tangent=True) -> dict:
        out = oj.update_reference_form(self.params, strains, state["plastic_strain"], state["eqps"], state["vpm"], dt,
                                       rates)  # fmt: skip
        if np.any(out["status"] != 0):
            raise FloatingPointError("material point failure")
        return {"stress": out["stresses"], "tangent": out["tangents"], "psi": out["free_energy"],
                "diss": out["dissipation"], "eqps": out["equivalent_plastic_strain"],
                "state": {"plastic_strain": out["plastic_strain"], "eqps": out["equivalent_plastic_strain"],
                          "vpm": out["viscoplastic_multiplier"]}}  # fmt: skip


class PointRVE:
    """One periodic RVE oracle solve per macro point (RVEHomogenizedMaterial)."""

    def __init__(self, rve: RVEOracle) -> None:
        self.rve = rve

    def initial_state(self, n: int) -> dict:
        return {"points": [self.rve.initial_state() for _ in range(n)]}

    def update(self, strains, rates, dt, state, need_tangent=True) -> dict:
        n = strains.shape[0]
        out = {"stress": np.zeros((n, 6)), "tangent": np.zeros((n, 6, 6)), "psi": np.zeros(n), "diss": np.zeros(n),
               "eqps": np.zeros(n), "state": {"points": []}}  # fmt: skip
        for i in range(n):
            r = self.rve.solve(np.asarray(strains[i]), dt, state["points"][i], need_tangent)
            out["stress"][i] = r["macro_stress"]
            if need_tangent:
                out["tangent"][i] = r["effective_tangent"]
            out["psi"][i] = r["free_energy_density"]
            out["diss"][i] = r["dissipation_density"]
            out["state"]["points"].append(r["state"])
        return out


@dataclass(frozen=True)
class Adaptive:
    enabled: bool = False
    minimum_factor: float = 1.0 / 16.0
    maximum_factor: float = 2.0
    cutback_factor: float = 0.5
    growth_factor: float = 2.0
    easy_iteration_limit: int = 4
    easy_step_count: int = 3


class Bar:
    """Mesh operators of one structured Hex8 mesh for the macro solve."""

    def __init__(self, nodes, elements, density: float) -> None:
        self.nodes, self.elements = nodes, elements
        self.b, self.jw = b_matrices(nodes, elements)
        self.weights = self.jw.reshape(-1)
        self.dofs = (3 * elements[:, :, None] + np.arange(3)).reshape(-1, 24)
        self.rows = np.repeat(self.dofs, 24, axis=1).ravel()
        self.cols = np.tile(self.dofs, (1, 24)).ravel()
        self.mass = consistent_mass(nodes, elements, density)
        self.n_dof = 3 * nodes.shape[0]

    def assemble(self, material, state, u, u_prev, dt, need_tangent=True) -> dict:
        ue, up = u[self.dofs], u_prev[self.dofs]
        eps = np.einsum("eqij,ej->eqi", self.b, ue).reshape(-1, 6)
        rate = (np.einsum("eqij,ej->eqi", self.b, ue - up) / dt).reshape(-1, 6)
        resp = material.update(eps, rate, dt, state, need_tangent)
        ne = self.elements.shape[0]
        fe = np.einsum("eqij,eqi,eq->ej", self.b, resp["stress"].reshape(ne, 8, 6), self.jw)
        f = np.zeros(self.n_dof)
        np.add.at(f, self.dofs.ravel(), fe.ravel())
        k = None
        if need_tangent:
            ke = np.einsum("eqki,eqkl,eqlj,eq->eij", self.b, resp["tangent"].reshape(ne, 8, 6, 6), self.b, self.jw)
            k = coo_matrix((ke.ravel(), (self.rows, self.cols)), shape=(self.n_dof, self.n_dof)).tocsr()
        return {"f": f, "K": k, **resp}


def implicit_newmark(bar: Bar, material, fixed, load, dt0: float, num_steps: int, beta: float, gamma: float,
                     newton: dict, adaptive: Adaptive = Adaptive()) -> dict:  # fmt: skip
    """Histories of solve_material_implicit_newmark from rest (zero initial fields).

    ``newton``: max_iterations, residual_absolute/relative_tolerance,
    increment_absolute/relative_tolerance, armijo (dict of sufficient_decrease,
    reduction_factor, max_backtracks, or None).
    """
    n = bar.n_dof
    free = np.setdiff1d(np.arange(n), fixed)
    mass = bar.mass
    m_ff = mass[free][:, free].tocsc()
    final_time = dt0 * num_steps
    u = np.zeros(n)
    v = np.zeros(n)
    asm = bar.assemble(material, material.initial_state(bar.weights.size), u, u, dt0)
    a = np.zeros(n)
    a[free] = spsolve(m_ff, (load(0.0) - asm["f"])[free])
    cur = {"t": 0.0, "u": u, "v": v, "a": a, "state": asm["state"], "asm": asm}
    states, intervals, rejected, reasons, pending = [cur], [], [0], [()], []
    dt = dt0
    min_dt = dt0 * adaptive.minimum_factor
    easy = 0
    while cur["t"] < final_time:
        trial = min(dt, final_time - cur["t"])
        try:
            interval = _step(bar, material, cur, trial, free, load, newton, beta, gamma)
        except RecoverableStepError as error:
            if not adaptive.enabled:
                raise
            pending.append(error.reason)
            if trial <= min_dt:
                raise
            dt = max(min_dt, trial * adaptive.cutback_factor)
            easy = 0
            continue
        cur = interval["state"]
        states.append(cur)
        intervals.append(interval)
        rejected.append(len(pending))
        reasons.append(tuple(pending))
        easy_step = not pending and interval["backtracks"] == 0 and interval["iterations"] <= adaptive.easy_iteration_limit
        easy = easy + 1 if easy_step else 0
        pending = []
        if adaptive.enabled and easy >= adaptive.easy_step_count:
            dt = min(dt0 * adaptive.maximum_factor, trial * adaptive.growth_factor)
            easy = 0
        else:
            dt = trial
    steps = len(states)
    out = {"times": np.asarray([s["t"] for s in states]), "displacement": np.stack([s["u"] for s in states]),
           "velocity": np.stack([s["v"] for s in states]), "acceleration": np.stack([s["a"] for s in states]),
           "stresses": np.stack([s["asm"]["stress"] for s in states]),
           "equivalent_plastic_strain": np.stack([s["asm"]["eqps"] for s in states]),
           "kinetic_energy": np.asarray([0.5 * s["v"] @ (mass @ s["v"]) for s in states]),
           "free_energy": np.asarray([float(s["asm"]["psi"] @ bar.weights) for s in states]),
           "newton_iterations": np.zeros(steps, dtype=np.int64), "armijo_backtracks": np.zeros(steps, dtype=np.int64),
           "dissipated_energy": np.zeros(steps), "external_work": np.zeros(steps),
           "rejected_step_counts": np.asarray(rejected, dtype=np.int64), "rejected_reasons": reasons}  # fmt: skip
    for i, iv in enumerate(intervals, start=1):
        out["dissipated_energy"][i] = out["dissipated_energy"][i - 1] + iv["dissipation"]
        out["external_work"][i] = out["external_work"][i - 1] + iv["work"]
        out["newton_iterations"][i] = iv["iterations"]
        out["armijo_backtracks"][i] = iv["backtracks"]
    e0 = out["kinetic_energy"][0] + out["free_energy"][0]
    out["energy_residual"] = out["kinetic_energy"] + out["free_energy"] + out["dissipated_energy"] - out["external_work"] - e0
    out["accepted_time_steps"] = np.concatenate([[0.0], np.diff(out["times"])])
    return out


def _step(bar: Bar, material, start, dt, free, load, newton, beta, gamma) -> dict:
    """One implicit Newmark step from a committed state (full Newton, optional Armijo)."""
    target = start["t"] + dt
    u_pred = start["u"] + dt * start["v"] + dt**2 * (0.5 - beta) * start["a"]
    v_pred = start["v"] + dt * (1.0 - gamma) * start["a"]
    u = u_pred.copy()
    u[np.setdiff1d(np.arange(u.size), free)] = 0.0
    ext = load(target)
    mass = bar.mass
    init = None
    last_inc = math.inf
    backtracks = 0

    def trial(x, need_tangent=True):
        acc = (x - u_pred) / (beta * dt**2)
        vel = v_pred + gamma * dt * acc
        asm = bar.assemble(material, start["state"], x, start["u"], dt, need_tangent)
        return acc, vel, asm, mass @ acc + asm["f"] - ext

    def accept(x, acc, vel, asm, it):
        return {"state": {"t": target, "u": x, "v": vel, "a": acc, "state": asm["state"], "asm": asm},
                "dissipation": float(dt * (asm["diss"] @ bar.weights)),
                "work": float(0.5 * (load(start["t"]) + ext) @ (x - start["u"])), "iterations": it,
                "backtracks": backtracks}  # fmt: skip

    for it in range(newton["max_iterations"] + 1):
        acc, vel, asm, r = trial(u)
        rn = float(np.linalg.norm(r[free]))
        init = rn if init is None else init
        tol = max(newton["residual_absolute_tolerance"], newton["residual_relative_tolerance"] * init)
        itol = max(newton["increment_absolute_tolerance"],
                   newton["increment_relative_tolerance"] * max(float(np.linalg.norm(u[free])), 1.0))  # fmt: skip
        if rn <= tol and (it == 0 or last_inc <= itol):
            return accept(u, acc, vel, asm, it)
        if it == newton["max_iterations"]:
            break
        k_eff = (asm["K"] + mass / (beta * dt**2)).tocsr()
        inc = np.asarray(spsolve(k_eff[free][:, free].tocsc(), -r[free]))
        if not np.all(np.isfinite(inc)):
            raise FloatingPointError("non_finite_increment")
        inc_n = float(np.linalg.norm(inc))
        if rn <= tol and inc_n <= itol:
            return accept(u, acc, vel, asm, it)
        step = 1.0
        arm = newton.get("armijo")
        if arm:
            for bt in range(arm["max_backtracks"] + 1):
                step = arm["reduction_factor"] ** bt
                cand = u.copy()
                cand[free] += step * inc
                cn = float(np.linalg.norm(trial(cand, False)[3][free]))
                if 0.5 * cn**2 <= 0.5 * rn**2 - arm["sufficient_decrease"] * step * rn**2:
                    backtracks += bt
                    break
            else:
                raise RecoverableStepError("armijo_exhausted")
        u = u.copy()
        u[free] += step * inc
        last_inc = float(np.linalg.norm(step * inc))
    raise RecoverableStepError("maximum_iterations_exceeded")
