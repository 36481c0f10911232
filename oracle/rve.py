"""NumPy/SciPy oracle of the periodic Hex8 RVE solve -- test infrastructure only.

Vectorised restatement of the reference's
  _build_hex8_quadrature_geometry        src/fem/assembly/nonlinear_solid.py:391-425
  _compute_hex8_strain_fields            src/fem/assembly/nonlinear_solid.py:428-454
  PhasedMaterialModel.update             src/fem/materials/phased.py:67-143
  _assemble_force_and_tangent            src/fem/assembly/nonlinear_solid.py:457-493
  solve_rve_microequilibrium             src/fem/rve/solver.py:62-227 (direct solves)
  perform_armijo_search                  src/fem/solvers/line_search.py:40-67
  _build_rve_response (stress, energies, work, Hill-Mandel)   src/fem/rve/solver.py:253-364
  _compute_effective_tangent             src/fem/rve/solver.py:438-461
for structured periodic boxes with J2 viscoplastic and linear elastic phases.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.sparse import coo_matrix
from scipy.sparse.linalg import spsolve

from . import j2vp as oj


@dataclass
class OraclePhase:
    kind: str  # "j2" or "elastic"
    params: oj.J2Params | None = None
    young_modulus: float = 0.0
    poisson_ratio: float = 0.0


@dataclass
class OracleRVE:
    divisions: tuple[int, int, int]
    lengths: tuple[float, float, float]
    phases: list[OraclePhase]
    element_phase: np.ndarray
    newton: dict  # max_iterations, residual_absolute/relative, increment_absolute/relative, armijo (dict|None)


def box_mesh(lengths, divisions):
    nx, ny, nz = divisions
    xs, ys, zs = (np.linspace(0.0, lengths[a], divisions[a] + 1) for a in range(3))
    zz, yy, xx = np.meshgrid(zs, ys, xs, indexing="ij")
    nodes = np.column_stack([xx.ravel(), yy.ravel(), zz.ravel()])
    k, j, i = (a.ravel() for a in np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij"))
    nid = lambda a, b, c: a + (nx + 1) * (b + (ny + 1) * c)  # noqa: E731
    elements = np.column_stack([nid(i, j, k), nid(i + 1, j, k), nid(i, j + 1, k), nid(i + 1, j + 1, k),
                                nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i, j + 1, k + 1), nid(i + 1, j + 1, k + 1)])  # fmt: skip
    return nodes, elements


def periodic_operators(nodes, divisions):
    """Transformation T (class 0 eliminated), affine map A, class ids (periodic.py:20-169)."""
    nx, ny, nz = divisions
    kk, jj, ii = (a.ravel() for a in np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij"))
    cls = (ii % nx) + nx * ((jj % ny) + ny * (kk % nz))
    n = nodes.shape[0]
    ids = np.flatnonzero(cls != 0)
    rows = (3 * ids[:, None] + np.arange(3)).ravel()
    cols = (3 * (cls[ids] - 1)[:, None] + np.arange(3)).ravel()
    t = coo_matrix((np.ones(rows.size), (rows, cols)), shape=(3 * n, 3 * (nx * ny * nz - 1))).tocsr()
    rel = nodes - nodes.min(axis=0)
    a = np.zeros((3 * n, 6))
    a[0::3, 0], a[0::3, 4], a[0::3, 5] = rel[:, 0], 0.5 * rel[:, 2], 0.5 * rel[:, 1]
    a[1::3, 1], a[1::3, 3], a[1::3, 5] = rel[:, 1], 0.5 * rel[:, 2], 0.5 * rel[:, 0]
    a[2::3, 2], a[2::3, 3], a[2::3, 4] = rel[:, 2], 0.5 * rel[:, 1], 0.5 * rel[:, 0]
    return t, a, cls


def b_matrices(nodes, elements):
    """(E, 8, 6, 24) strain-displacement matrices and (E, 8) J*w weights."""
    g = 1.0 / np.sqrt(3.0)
    pts = np.asarray([(a, b, c) for a in (-g, g) for b in (-g, g) for c in (-g, g)])
    signs = np.asarray([[(-1, 1)[(a >> d) & 1] for d in range(3)] for a in range(8)], dtype=np.float64)
    f = 1.0 + pts[:, None, :] * signs[None, :, :]
    dref = np.zeros((8, 8, 3))
    dref[:, :, 0] = 0.125 * signs[None, :, 0] * f[:, :, 1] * f[:, :, 2]
    dref[:, :, 1] = 0.125 * signs[None, :, 1] * f[:, :, 0] * f[:, :, 2]
    dref[:, :, 2] = 0.125 * signs[None, :, 2] * f[:, :, 0] * f[:, :, 1]
    xe = nodes[elements]  # (E, 8, 3)
    jac = np.einsum("eai,qaj->eqij", xe, dref)
    det = np.linalg.det(jac)
    dphys = np.einsum("qaj,eqji->eqai", dref, np.linalg.inv(jac))
    E = elements.shape[0]
    b = np.zeros((E, 8, 6, 24))
    gx, gy, gz = dphys[..., 0], dphys[..., 1], dphys[..., 2]
    for a in range(8):
        b[:, :, 0, 3 * a] = gx[:, :, a]
        b[:, :, 1, 3 * a + 1] = gy[:, :, a]
        b[:, :, 2, 3 * a + 2] = gz[:, :, a]
        b[:, :, 3, 3 * a + 1] = gz[:, :, a]
        b[:, :, 3, 3 * a + 2] = gy[:, :, a]
        b[:, :, 4, 3 * a] = gz[:, :, a]
        b[:, :, 4, 3 * a + 2] = gx[:, :, a]
        b[:, :, 5, 3 * a] = gy[:, :, a]
        b[:, :, 5, 3 * a + 1] = gx[:, :, a]
    return b, det  # weights are 1 for the 2x2x2 rule


class RVEOracle:
    """Direct-solve periodic RVE, one instance per geometry."""

    def __init__(self, rve: OracleRVE) -> None:
        self.rve = rve
        self.nodes, self.elements = box_mesh(rve.lengths, rve.divisions)
        self.t, self.a, self.cls = periodic_operators(self.nodes, rve.divisions)
        self.b, self.jw = b_matrices(self.nodes, self.elements)
        self.weights = self.jw.reshape(-1)
        self.volume = float(self.weights.sum())
        self.dofs = (3 * self.elements[:, :, None] + np.arange(3)).reshape(-1, 24)
        self.point_phase = np.repeat(np.asarray(rve.element_phase), 8)
        E = self.elements.shape[0]
        self.rows = np.repeat(self.dofs, 24, axis=1).ravel()
        self.cols = np.tile(self.dofs, (1, 24)).ravel()
        self.n_gp = 8 * E

    def initial_state(self):
        return {"plastic_strain": np.zeros((self.n_gp, 6)), "eqps": np.zeros(self.n_gp), "vpm": np.zeros(self.n_gp),
                "macro": np.zeros(6), "w": np.zeros(self.t.shape[1])}  # fmt: skip

    def assemble(self, u, u_prev, dt, state):
        ue = u[self.dofs]
        up = u_prev[self.dofs]
        eps = np.matmul(self.b, ue[:, None, :, None])[..., 0].reshape(-1, 6)
        rate = (np.matmul(self.b, (ue - up)[:, None, :, None])[..., 0] / dt).reshape(-1, 6)
        n = self.n_gp
        stress, tangent = np.zeros((n, 6)), np.zeros((n, 6, 6))
        psi, diss = np.zeros(n), np.zeros(n)
        iwd, active, margin = np.zeros(n), np.zeros(n), np.full(n, np.nan)
        new = {k: v.copy() for k, v in state.items() if k in ("plastic_strain", "eqps", "vpm")}
        status = np.zeros(n, dtype=np.int32)
        for pid, ph in enumerate(self.rve.phases):
            ids = np.flatnonzero(self.point_phase == pid)
            if ph.kind == "j2":
                out = oj.update_reference_form(ph.params, eps[ids], state["plastic_strain"][ids], state["eqps"][ids],
                                               state["vpm"][ids], dt, rate[ids])  # fmt: skip
                stress[ids], tangent[ids] = out["stresses"], out["tangents"]
                psi[ids], diss[ids] = out["free_energy"], out["dissipation"]
                new["plastic_strain"][ids] = out["plastic_strain"]
                new["eqps"][ids] = out["equivalent_plastic_strain"]
                new["vpm"][ids] = out["viscoplastic_multiplier"]
                iwd[ids] = out["diagnostics"]["incremental_work_density"]
                active[ids] = out["diagnostics"]["viscoplastic_active"]
                margin[ids] = out["diagnostics"]["yield_activation_margin"]
                status[ids] = out["status"]
            else:
                c = oj.elasticity_matrix(ph.young_modulus, ph.poisson_ratio)
                stress[ids] = eps[ids] @ c.T
                tangent[ids] = c
                psi[ids] = 0.5 * np.einsum("qi,qi->q", eps[ids], stress[ids])
                de = dt * rate[ids]
                prev = stress[ids] - de @ c.T
                iwd[ids] = 0.5 * np.einsum("qi,qi->q", prev + stress[ids], de)
        if np.any(status != 0):
            raise FloatingPointError(f"material failure at point {int(np.flatnonzero(status)[0])}")
        E = self.elements.shape[0]
        s4 = stress.reshape(E, 8, 6)
        t4 = tangent.reshape(E, 8, 6, 6)
        fe = np.einsum("eqij,eqi,eq->ej", self.b, s4, self.jw, optimize=True)
        f = np.zeros(u.size)
        np.add.at(f, self.dofs.ravel(), fe.ravel())
        # K_e = sum_q w B^T C B: batched products (the same sum as the reference's per-element
        # loop, in a different floating-point order)
        cb = np.matmul(t4, self.b)  # (E, 8, 6, 24)
        ke = np.einsum("eqki,eqkj,eq->eij", self.b, cb, self.jw, optimize=True)
        k = coo_matrix((ke.ravel(), (self.rows, self.cols)), shape=(u.size, u.size)).tocsr()
        return {"f": f, "K": k, "eps": eps, "rate": rate, "stress": stress, "psi": psi, "diss": diss, "state": new,
                "iwd": iwd, "active": active, "margin": margin}  # fmt: skip

    def solve(self, macro, dt, state, need_tangent=True):
        """One solve_rve_microequilibrium step; returns a dict of responses and the next state."""
        ns = self.rve.newton
        t, a = self.t, self.a
        u_prev = t @ state["w"] + a @ state["macro"]
        w = state["w"].copy()
        init = None
        last_inc = np.inf
        backtracks = 0
        for it in range(ns["max_iterations"] + 1):
            u = t @ w + a @ macro
            asm = self.assemble(u, u_prev, dt, state)
            r = t.T @ asm["f"]
            rn = float(np.linalg.norm(r))
            init = rn if init is None else init
            tol = max(ns["residual_absolute_tolerance"], ns["residual_relative_tolerance"] * init)
            inc_tol = max(ns["increment_absolute_tolerance"], ns["increment_relative_tolerance"] * max(float(np.linalg.norm(w)), 1.0))
            if rn <= tol and (it == 0 or last_inc <= inc_tol):
                return self._response(macro, dt, state, w, u, asm, it, backtracks, rn, tol, need_tangent)
            if it == ns["max_iterations"]:
                raise RuntimeError("maximum_iterations_exceeded")
            kr = (t.T @ asm["K"] @ t).tocsr()
            dw = np.asarray(spsolve(kr, -r))
            inc = float(np.linalg.norm(dw))
            if rn <= tol and inc <= inc_tol:
                return self._response(macro, dt, state, w, u, asm, it, backtracks, rn, tol, need_tangent)
            step = 1.0
            arm = ns.get("armijo")
            if arm:
                merit = 0.5 * rn**2
                for bt in range(arm["max_backtracks"] + 1):
                    step = arm["reduction_factor"] ** bt
                    cand = self.assemble(t @ (w + step * dw) + a @ macro, u_prev, dt, state)
                    cn = float(np.linalg.norm(t.T @ cand["f"]))
                    if 0.5 * cn**2 <= merit - arm["sufficient_decrease"] * step * rn**2:
                        backtracks += bt
                        break
                else:
                    raise RuntimeError("armijo_exhausted")
            w = w + step * dw
            last_inc = float(np.linalg.norm(step * dw))
        raise AssertionError("unreachable")

    def _response(self, macro, dt, state, w, u, asm, it, bts, rn, tol, need_tangent):
        wts = self.weights
        vol = self.volume
        sigma = (asm["stress"] * wts[:, None]).sum(0) / vol
        ceff = None
        if need_tangent:
            k = asm["K"]
            kea = np.asarray(k @ self.a)
            kee = self.a.T @ kea
            kww = (self.t.T @ k @ self.t).tocsc()
            kwe = np.asarray(self.t.T @ kea)
            sens = np.asarray(spsolve(kww, kwe))
            ceff = (kee - kwe.T @ sens) / vol
        prev = asm["eps"] - dt * asm["rate"]
        micro_work = float(np.sum(np.einsum("ij,ij->i", asm["stress"], asm["eps"] - prev) * wts) / vol)
        macro_work = float(sigma @ (macro - state["macro"]))
        nxt = dict(asm["state"])
        nxt["macro"] = macro.copy()
        nxt["w"] = w.copy()
        return {
            "macro_stress": sigma, "effective_tangent": ceff, "state": nxt, "displacement": u,
            "newton_iterations": it, "armijo_backtracks": bts, "residual_norm": rn, "residual_tolerance": tol,
            "free_energy_density": float((asm["psi"] * wts).sum() / vol),
            "dissipation_density": float((asm["diss"] * wts).sum() / vol),
            "micro_work": micro_work, "macro_work": macro_work,
            "active_fraction": float(wts[asm["active"] > 0.5].sum() / vol),
            "positive_work": float((np.maximum(asm["iwd"], 0) * wts).sum() / vol),
            "negative_work": float((np.minimum(asm["iwd"], 0) * wts).sum() / vol),
            "micro_stresses": asm["stress"], "micro_strains": asm["eps"],
        }  # fmt: skip
