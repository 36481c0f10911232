"""NumPy oracle of the explicit macro dynamics -- test infrastructure only.

Restates, for a structured Hex8 bar and a linear elastic material (internal force K u) or
a J2 Perzyna material (internal force sum B^T sigma w from the J2 oracle):
  assemble_lumped_mass_vector (row sum of the consistent mass)   src/fem/assembly/elasticity.py:73-77
  assemble_uniform_boundary_pressure (traction -p n on a face)   src/fem/assembly/load.py:40-77
  solve_material_explicit velocity-Verlet step and histories     src/fem/dynamics/material.py:89-297
"""

from __future__ import annotations

import numpy as np
from scipy.sparse import coo_matrix

from . import j2vp as oj
from .j2vp import elasticity_matrix
from .rve import b_matrices, box_mesh


def _shape_values(pts: np.ndarray) -> np.ndarray:
    signs = np.asarray([[(-1, 1)[(a >> d) & 1] for d in range(3)] for a in range(8)], dtype=np.float64)
    return 0.125 * np.prod(1.0 + pts[:, None, :] * signs[None, :, :], axis=2)  # (q, 8)


def lumped_mass(nodes: np.ndarray, elements: np.ndarray, density: float) -> np.ndarray:
    """Row sums of rho * int N_a N_b dV over 2x2x2 Gauss points, per DOF (3N,)."""
    g = 1.0 / np.sqrt(3.0)
    pts = np.asarray([(a, b, c) for a in (-g, g) for b in (-g, g) for c in (-g, g)])
    nq = _shape_values(pts)
    _, det = b_matrices(nodes, elements)
    # row sum of N_a N_b over b is N_a (partition of unity)
    me = density * np.einsum("qa,eq->ea", nq, det)
    m = np.zeros(nodes.shape[0])
    np.add.at(m, elements.reshape(-1), me.reshape(-1))
    return np.repeat(m, 3)


def face_pressure_force(nodes: np.ndarray, lengths, divisions) -> np.ndarray:
    """Nodal force of a unit pressure on the x = L face (outward normal +x), 2x2 quadrature."""
    nx, ny, nz = divisions
    hy, hz = lengths[1] / ny, lengths[2] / nz
    f = np.zeros(3 * nodes.shape[0])
    g = 1.0 / np.sqrt(3.0)
    nid = lambda i, j, k: i + (nx + 1) * (j + (ny + 1) * k)  # noqa: E731
    for k in range(nz):
        for j in range(ny):
            quad = [nid(nx, j, k), nid(nx, j + 1, k), nid(nx, j, k + 1), nid(nx, j + 1, k + 1)]
            for s in (-g, g):
                for t in (-g, g):
                    n = 0.25 * np.asarray([(1 - s) * (1 - t), (1 + s) * (1 - t), (1 - s) * (1 + t), (1 + s) * (1 + t)])
                    jw = 0.25 * hy * hz
                    for a, node in enumerate(quad):
                        f[3 * node] += -1.0 * n[a] * jw
    return f


def elastic_stiffness(nodes, elements, young_modulus: float, poisson_ratio: float):
    """K = sum_e sum_q B^T C B detJ (CSR)."""
    b, det = b_matrices(nodes, elements)
    c = elasticity_matrix(young_modulus, poisson_ratio)
    ke = np.einsum("eqia,ij,eqjb,eq->eab", b, c, b, det)
    dof = (3 * elements[:, :, None] + np.arange(3)).reshape(elements.shape[0], 24)
    rows = np.repeat(dof, 24, axis=1).ravel()
    cols = np.tile(dof, (1, 24)).ravel()
    n3 = 3 * nodes.shape[0]
    return coo_matrix((ke.ravel(), (rows, cols)), shape=(n3, n3)).tocsr()


def explicit_elastic_bar(divisions, lengths, density, young_modulus, poisson_ratio, dt, steps, pressure):
    """Velocity Verlet on the bar (x = 0 face fixed); returns (u, v, a) after ``steps``."""
    nodes, elements = box_mesh(lengths, divisions)
    m = lumped_mass(nodes, elements, density)
    f_unit = face_pressure_force(nodes, lengths, divisions)
    k = elastic_stiffness(nodes, elements, young_modulus, poisson_ratio)
    fixed = np.repeat(np.isclose(nodes[:, 0], 0.0), 3)
    n3 = 3 * nodes.shape[0]
    u, v, a = np.zeros(n3), np.zeros(n3), np.zeros(n3)
    for step in range(steps):
        t1 = (step + 1) * dt
        un = u + dt * v + 0.5 * dt * dt * a
        un[fixed] = 0.0
        an = (pressure(t1) * f_unit - k @ un) / m
        an[fixed] = 0.0
        vn = v + 0.5 * dt * (a + an)
        vn[fixed] = 0.0
        u, v, a = un, vn, an
    return u, v, a


def explicit_j2_bar(divisions, lengths, params: oj.J2Params, density: float, dt: float, steps: int, load, fixed_dofs):
    """solve_material_explicit on a J2 Perzyna bar: ``load(t)`` is the external force
    vector, ``fixed_dofs`` the homogeneous Dirichlet DOFs.  Returns the histories
    (times, u, v, a, stresses, eqps, kinetic, dissipated energy, external work)."""
    nodes, elements = box_mesh(lengths, divisions)
    b, jw = b_matrices(nodes, elements)
    dofs = (3 * elements[:, :, None] + np.arange(3)).reshape(-1, 24)
    m = lumped_mass(nodes, elements, density)
    n3, npts = 3 * nodes.shape[0], 8 * elements.shape[0]
    fixed = np.zeros(n3, dtype=bool)
    fixed[np.asarray(fixed_dofs)] = True
    state = {"ep": np.zeros((npts, 6)), "q": np.zeros(npts), "vpm": np.zeros(npts)}
    weights = jw.reshape(-1)

    def assemble(u, u_prev, st):
        eps = np.einsum("eqij,ej->eqi", b, u[dofs]).reshape(-1, 6)
        rate = (np.einsum("eqij,ej->eqi", b, (u - u_prev)[dofs]) / dt).reshape(-1, 6)
        out = oj.update_reference_form(params, eps, st["ep"], st["q"], st["vpm"], dt, rate)
        if np.any(out["status"] != 0):
            raise FloatingPointError("J2 point failure")
        f = np.zeros(n3)
        np.add.at(f, dofs.ravel(), np.einsum("eqij,eqi,eq->ej", b, out["stresses"].reshape(-1, 8, 6), jw).ravel())
        new = {"ep": out["plastic_strain"], "q": out["equivalent_plastic_strain"], "vpm": out["viscoplastic_multiplier"]}
        return f, out, new

    u, v = np.zeros(n3), np.zeros(n3)
    f_int, out, state = assemble(u, u, state)
    external = load(0.0)
    a = (external - f_int) / m
    a[fixed] = 0.0
    hist = {"times": [0.0], "u": [u], "v": [v], "a": [a], "stresses": [out["stresses"]],
            "eqps": [out["equivalent_plastic_strain"]], "kinetic": [0.5 * np.sum(m * v * v)], "dissipated": [0.0],
            "work": [0.0]}  # fmt: skip
    for step in range(steps):
        t1 = (step + 1) * dt
        un = u + dt * v + 0.5 * dt**2 * a
        un[fixed] = 0.0
        f_int, out, state = assemble(un, u, state)
        external1 = load(t1)
        an = (external1 - f_int) / m
        an[fixed] = 0.0
        vn = v + 0.5 * dt * (a + an)
        vn[fixed] = 0.0
        hist["dissipated"].append(hist["dissipated"][-1] + dt * float(np.dot(out["dissipation"], weights)))
        hist["work"].append(hist["work"][-1] + 0.5 * float((external + external1) @ (un - u)))
        u, v, a, external = un, vn, an, external1
        for key, value in (("times", t1), ("u", u), ("v", v), ("a", a), ("stresses", out["stresses"]),
                           ("eqps", out["equivalent_plastic_strain"]), ("kinetic", 0.5 * np.sum(m * v * v))):
            hist[key].append(value)
    return {k: np.asarray(val) for k, val in hist.items()}
