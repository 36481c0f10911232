"""GPU tests of implicit Newmark material dynamics (concrete_impact_b200.dynamics) and the
kernels of csrc/newmark.cu.

* the consistent mass in the tangent's CSR pattern against the oracle (distorted mesh);
* the Jacobi-PCG solve of the effective tangent against a direct solve: accuracy, zero
  fixed DOFs, bitwise repeatability, the iteration-limit status and a zero right side;
* the Newmark kinematics and residual kernels against their formulas;
* whole runs against the reference's own solve_material_implicit_newmark (golden histories
  from tests/golden/make_golden.py): J2 Perzyna bar with fixed steps, the adaptive run with
  Armijo and forced cutbacks (same accepted times, rejections and reasons), and implicit
  FE2 with a two-phase 4^3 RVE at every macro point (RVEHomogenizedMaterial, effective
  tangents from the device RVE batch);
* the reference's bundle layout (mesh_info + material) as the mesh argument, and a run
  that keeps only the final fields.
"""

from __future__ import annotations

import math
from types import SimpleNamespace

import numpy as np
import pytest
import torch
from scipy.sparse import csr_matrix
from scipy.sparse.linalg import spsolve

pytestmark = pytest.mark.gpu

from conftest import load_case  # noqa: E402
from concrete_impact_b200.dynamics import (  # noqa: E402
    AdaptiveTimeStepSettings,
    DirichletDofSet,
    MacroLinearSolverOptions,
    MacroOperators,
    TimeIntegrationSettings,
    solve_material_implicit_newmark,
)
from concrete_impact_b200.materials import J2ViscoplasticMaterial, LinearElasticMaterial, MaterialUpdateSettings  # noqa: E402
from concrete_impact_b200.rve import ArmijoSettings, NonlinearNewtonSettings  # noqa: E402
from concrete_impact_b200.rve_builders import build_two_phase_sphere_rve  # noqa: E402
from concrete_impact_b200.rve_material import RVEHomogenizedMaterial  # noqa: E402
from oracle import fe2 as of  # noqa: E402
from oracle import newmark as on  # noqa: E402
from oracle.rve import box_mesh  # noqa: E402


def _left_fixed(nodes):
    left = np.flatnonzero(np.isclose(nodes[:, 0], 0.0))
    return (3 * left[:, None] + np.arange(3)).ravel()


def _pattern_values(ops: MacroOperators, matrix) -> np.ndarray:
    """Entries of a SciPy matrix at the operators' CSR pattern."""
    rows = np.repeat(np.arange(ops.n), np.diff(ops.cache.csr_indptr))
    return np.asarray(matrix.tocsr()[rows, ops.cache.csr_indices]).ravel()


def test_consistent_mass_csr_matches_oracle() -> None:
    rng = np.random.default_rng(3)
    nodes, elements = box_mesh((0.3, 0.2, 0.1), (3, 2, 2))
    nodes = nodes + rng.uniform(-0.01, 0.01, nodes.shape)
    ops = MacroOperators(nodes, elements, 2400.0, np.zeros(0, dtype=np.int64))
    ref = on.consistent_mass(nodes, elements, 2400.0)
    got = csr_matrix((ops.mass.cpu().numpy(), ops.cache.csr_indices, ops.cache.csr_indptr), shape=ref.shape)
    assert abs(got - ref).max() <= 1e-13 * abs(ref).max()


def _elastic_bar_system():
    nodes, elements = box_mesh((0.4, 0.1, 0.1), (8, 2, 2))
    fixed = _left_fixed(nodes)
    ops = MacroOperators(nodes, elements, 2400.0, fixed)
    k = of.elastic_stiffness(nodes, elements, 25.0e9, 0.2)
    kv = torch.as_tensor(_pattern_values(ops, k), device="cuda")
    return ops, k, kv, fixed


def test_csr_pcg_matches_direct_solve_and_repeats_bitwise() -> None:
    ops, k, kv, fixed = _elastic_bar_system()
    beta_dt2 = 0.25 * (2.0e-6) ** 2
    g = torch.Generator(device="cuda").manual_seed(5)
    rhs = torch.randn(ops.n, generator=g, device="cuda", dtype=torch.float64)
    x1, status, iterations, rel = ops.solve(kv, beta_dt2, rhs)
    assert status == 0 and 0 < iterations < 1000 and rel <= 1e-12
    free = np.setdiff1d(np.arange(ops.n), fixed)
    m = on.consistent_mass(ops.nodes, ops.elements, 2400.0)
    a = (k + m / beta_dt2).tocsr()[free][:, free]
    xd = spsolve(a.tocsc(), rhs.cpu().numpy()[free])
    x = x1.cpu().numpy()
    assert np.all(x[fixed] == 0.0)
    np.testing.assert_allclose(x[free], xd, rtol=0, atol=1e-9 * np.abs(xd).max())
    x2 = ops.solve(kv, beta_dt2, rhs)[0]
    assert torch.equal(x1, x2)


def test_csr_pcg_iteration_limit_and_zero_rhs() -> None:
    ops, _, kv, _ = _elastic_bar_system()
    ops.linear = MacroLinearSolverOptions(max_iterations=2, check_every=1)
    rhs = torch.ones(ops.n, dtype=torch.float64, device="cuda")
    _, status, iterations, rel = ops.solve(kv, 1.0e30, rhs)  # stiffness only: not solved in 2 iterations
    assert status == 1 and iterations == 2 and rel > 1e-12
    ops.linear = MacroLinearSolverOptions()
    x, status, iterations, rel = ops.solve(kv, 1.0e30, torch.zeros_like(rhs))
    assert status == 0 and iterations == 0 and rel == 0.0 and not bool(x.any())


def test_newmark_kinematics_and_residual_kernels() -> None:
    ops, _, _, fixed = _elastic_bar_system()
    g = torch.Generator(device="cuda").manual_seed(9)
    u, up, vp, fi, fe = (torch.randn(ops.n, generator=g, device="cuda", dtype=torch.float64) for _ in range(5))
    beta_dt2, gamma_dt = 0.25 * 3.0e-6**2, 0.5 * 3.0e-6
    a, v = ops.kinematics(u, up, vp, beta_dt2, gamma_dt)
    torch.testing.assert_close(a, (u - up) / beta_dt2, rtol=1e-15, atol=0.0)  # torch scales by 1 / beta_dt2
    torch.testing.assert_close(v, vp + gamma_dt * a, rtol=1e-15, atol=1e-300)
    r = ops.residual(a, fi, fe).cpu().numpy()
    m = on.consistent_mass(ops.nodes, ops.elements, 2400.0)
    ref = m @ a.cpu().numpy() + fi.cpu().numpy() - fe.cpu().numpy()
    ref[fixed] = 0.0
    np.testing.assert_allclose(r, ref, rtol=0, atol=1e-13 * np.abs(ref).max())


# --------------------------------------------------------------------------------------
# Whole runs against the reference's golden histories.

FIELDS = {"displacement": 1e-7, "velocity": 1e-7, "acceleration": 1e-6, "stresses": 1e-7, "kinetic_energy": 1e-7,
          "free_energy": 1e-7, "dissipated_energy": 1e-7, "external_work": 1e-7}  # fmt: skip


def _run(name: str, material, mesh_kind: str = "plain", record_fields: bool = True):
    g, meta = load_case(name)
    nodes, elements = box_mesh(meta["bar"]["lengths"], meta["bar"]["divisions"])
    if mesh_kind == "bundle":
        mesh = SimpleNamespace(mesh_info=SimpleNamespace(nodes=nodes, elements=elements, dimension=3), material=material)
    else:
        mesh = SimpleNamespace(nodes=nodes, elements=elements, material=material)
    unit = torch.as_tensor(g["unit_force"], device="cuda")
    amp, dur = meta["amplitude"], meta["duration"]

    def load(t):
        return (amp * math.sin(math.pi * t / dur) if 0.0 <= t <= dur else 0.0) * unit

    ts = TimeIntegrationSettings("newmark", meta["time_step"], meta["num_steps"], meta["beta"], meta["gamma"], 1.0,
                                 AdaptiveTimeStepSettings(enabled=meta["adaptive"]))  # fmt: skip
    newton = NonlinearNewtonSettings(*meta["newton"][:5], ArmijoSettings(enabled=meta["newton"][5]))
    n = 3 * nodes.shape[0]
    sol = solve_material_implicit_newmark(mesh, ts, np.zeros(n), np.zeros(n),
                                          DirichletDofSet(g["fixed_dofs"], np.zeros(g["fixed_dofs"].size)), load,
                                          "three_dimensional", MaterialUpdateSettings(*meta["update_settings"]), newton,
                                          record_fields=record_fields)  # fmt: skip
    return sol, g, meta


def _mortar(meta) -> J2ViscoplasticMaterial:
    p = meta["material"]["params"]
    return J2ViscoplasticMaterial("mortar", meta["material"]["density"], p["young_modulus"], p["poisson_ratio"],
                                  p["yield_stress"], p["hardening_modulus"], p["time_scale"], p["reference_stress"],
                                  p["rate_exponent"])  # fmt: skip


def _check_histories(sol, g, tolerances=FIELDS, exact_newton=True) -> None:
    np.testing.assert_array_equal(sol.times, g["times"])
    np.testing.assert_array_equal(sol.rejected_step_counts, g["rejected_step_counts"])
    if exact_newton:
        np.testing.assert_array_equal(sol.newton_iterations, g["newton_iterations"])
        np.testing.assert_array_equal(sol.armijo_backtracks, g["armijo_backtracks"])
    else:
        assert np.abs(sol.newton_iterations - g["newton_iterations"]).max() <= 1
    for key, tol in tolerances.items():
        ref = g[key]
        np.testing.assert_allclose(getattr(sol, key), ref, rtol=0, atol=tol * np.abs(ref).max(), err_msg=key)


@pytest.mark.parametrize("name", ["newmark_j2_bar_fixed", "newmark_j2_bar_adaptive"])
def test_implicit_newmark_j2_matches_reference(name) -> None:
    _, meta = load_case(name)
    sol, g, meta = _run(name, _mortar(meta))
    _check_histories(sol, g)
    assert [list(r) for r in sol.rejected_reasons] == meta["rejected_reasons"]
    np.testing.assert_allclose(sol.equivalent_plastic_strain, g["equivalent_plastic_strain"], rtol=0,
                               atol=1e-7 * np.abs(g["equivalent_plastic_strain"]).max())  # fmt: skip
    assert sol.equivalent_plastic_strain.max() > 1e-3  # the pulse drives the bar plastic


def test_implicit_newmark_accepts_reference_bundle_and_final_fields_only() -> None:
    _, meta = load_case("newmark_j2_bar_fixed")
    full, g, _ = _run("newmark_j2_bar_fixed", _mortar(meta))
    last, _, _ = _run("newmark_j2_bar_fixed", _mortar(meta), mesh_kind="bundle", record_fields=False)
    np.testing.assert_array_equal(last.times, full.times)
    np.testing.assert_array_equal(last.kinetic_energy, full.kinetic_energy)
    assert last.displacement.shape == (1, full.displacement.shape[1])
    np.testing.assert_array_equal(last.displacement[0], full.displacement[-1])
    np.testing.assert_array_equal(last.stresses[0], full.stresses[-1])


def test_implicit_fe2_with_rve_points_matches_reference() -> None:
    _, meta = load_case("newmark_fe2_bar")
    r = meta["rve"]
    mortar = J2ViscoplasticMaterial("mortar", 2200.0, 25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0)
    aggregate = LinearElasticMaterial("aggregate", 2600.0, 50.0e9, 0.2)
    newton = NonlinearNewtonSettings(*r["newton"][:5], ArmijoSettings(enabled=r["newton"][5]))
    model = build_two_phase_sphere_rve(tuple(r["divisions"]), mortar, aggregate, newton, seed=r["seed"])
    g, _ = load_case("newmark_fe2_bar")
    np.testing.assert_array_equal(model.element_phase_ids, g["element_phase"])
    assert model.material.density == pytest.approx(r["density"], rel=1e-15)
    material = RVEHomogenizedMaterial(model, "two_phase_rve")
    try:
        sol, g, _ = _run("newmark_fe2_bar", material)
    finally:
        material.close()
    tolerances = {key: 1e-6 for key in FIELDS}
    _check_histories(sol, g, tolerances, exact_newton=False)
    assert sol.dissipated_energy[-1] > 0.0  # the mortar phase yields inside the RVEs
