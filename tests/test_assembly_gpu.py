"""GPU tests of the general Hex8 assembly (cib_hex8_* through the C ABI).

Reference unit tests of src/fem/assembly/nonlinear_solid.py re-run on the GPU path, plus
force and CSR tangent on a distorted two-phase mesh against the oracle's dense assembly
(float64, rtol 1e-11).
"""

from __future__ import annotations

import numpy as np
import pytest

import concrete_impact_b200 as cib
from concrete_impact_b200 import assembly as A
from concrete_impact_b200.rve import build_structured_hex8_box
from oracle import j2vp as oj
from oracle.rve import b_matrices

pytestmark = pytest.mark.gpu

SETTINGS = cib.MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)


def test_uniform_elastic_reaction_and_state_untouched() -> None:
    """Reference tests/unit/fem/test_nonlinear_solid.py:29."""
    material = cib.J2ViscoplasticMaterial("assembly_test", 1.0, 1000.0, 0.25, 1.0e6, 80.0, 30.0, 10.0, 1.0)
    nodes, elements = build_structured_hex8_box((1.0, 1.0, 1.0), (1, 1, 1))
    state = A.initialize_hex8_material_state(material, elements.shape[0])
    snapshot = {k: v.copy() for k, v in state.variables.items()}
    u = np.zeros(3 * nodes.shape[0])
    u[0::3] = 1.0e-3 * nodes[:, 0]
    result = A.assemble_hex8_material_response(nodes, elements, material, state, u, np.zeros_like(u), 1.0, SETTINGS,
                                               need_tangent=True)  # fmt: skip
    right = np.flatnonzero(np.isclose(nodes[:, 0], 1.0))
    reaction = float(np.sum(result.internal_force[3 * right]))
    g = 1000.0 / (2.0 * 1.25)
    lam = 1000.0 * 0.25 / (1.25 * 0.5)
    assert reaction == pytest.approx((lam + 2.0 * g) * 1.0e-3, rel=1.0e-12, abs=1.0e-12)
    for k, v in state.variables.items():
        assert np.array_equal(v, snapshot[k])


def test_material_failure_reports_element_and_quadrature_context() -> None:
    """Reference tests/unit/fem/test_nonlinear_solid.py:110."""
    material = cib.J2ViscoplasticMaterial("assembly_failure_test", 1.0, 1000.0, 0.25, 1.0, 10.0, 0.02, 1.0, 2.0)
    nodes, elements = build_structured_hex8_box((1.0, 1.0, 1.0), (1, 1, 1))
    state = A.initialize_hex8_material_state(material, 1)
    snapshot = {k: v.copy() for k, v in state.variables.items()}
    u = np.zeros(3 * nodes.shape[0])
    u[0::3] = 0.02 * nodes[:, 0]
    with pytest.raises(cib.MaterialPointConvergenceError) as info:
        A.assemble_hex8_material_response(nodes, elements, material, state, u, np.zeros_like(u), 1.0e-3,
                                          cib.MaterialUpdateSettings(1, 1.0e-10, 1.0e-30, 1.0e-30))  # fmt: skip
    d = info.value.diagnostics
    assert d["point_id"] == 0 and d["element_id"] == 0 and d["quadrature_id"] == 0
    for k, v in state.variables.items():
        assert np.array_equal(v, snapshot[k])


def test_distorted_two_phase_mesh_force_and_tangent_match_dense_oracle() -> None:
    rng = np.random.default_rng(4)
    nodes, elements = build_structured_hex8_box((1.0, 0.8, 1.2), (3, 2, 4))
    nodes = nodes + rng.uniform(-0.04, 0.04, size=nodes.shape)
    ne, nn = elements.shape[0], nodes.shape[0]
    mortar = cib.J2ViscoplasticMaterial("mortar", 2200.0, 25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0)
    aggregate = cib.LinearElasticMaterial("aggregate", 2600.0, 50.0e9, 0.2)
    phase = rng.integers(0, 2, size=ne)
    model = cib.PhasedMaterialModel("m", (cib.RVEPhase("matrix", mortar), cib.RVEPhase("inclusion", aggregate)),
                                    np.repeat(phase, 8), 2400.0)  # fmt: skip
    state = model.initialize_state(8 * ne)
    u = rng.normal(0.0, 1.5e-3, size=3 * nn)
    up = u - rng.normal(0.0, 2e-4, size=3 * nn)
    dt = 1.0e-5
    cache = A.build_hex8_material_assembly_cache(nodes, elements)
    res = A.assemble_hex8_material_response_cached(nodes, elements, model, state, u, up, dt, SETTINGS, cache)
    b, jw = b_matrices(nodes, elements)
    np.testing.assert_allclose(cache.jacobian_weights, jw, rtol=1e-13)
    np.testing.assert_allclose(cache.b_matrices, b, rtol=1e-12, atol=1e-12)
    dofs = (3 * elements[:, :, None] + np.arange(3)).reshape(ne, 24)
    eps = np.einsum("eqij,ej->eqi", b, u[dofs]).reshape(-1, 6)
    np.testing.assert_allclose(res.strains, eps, rtol=1e-12, atol=1e-16)
    # material response on the CPU oracle, then dense assembly
    pts = np.repeat(phase, 8)
    stress = np.zeros((8 * ne, 6))
    tang = np.zeros((8 * ne, 6, 6))
    j2 = pts == 0
    out = oj.update_reference_form(oj.mortar_params(), eps[j2], np.zeros((j2.sum(), 6)), np.zeros(j2.sum()),
                                   np.zeros(j2.sum()), dt)  # fmt: skip
    stress[j2], tang[j2] = out["stresses"], out["tangents"]
    c = oj.elasticity_matrix(50.0e9, 0.2)
    stress[~j2] = eps[~j2] @ c.T
    tang[~j2] = c
    f = np.zeros(3 * nn)
    np.add.at(f, dofs.ravel(), np.einsum("eqij,eqi,eq->ej", b, stress.reshape(ne, 8, 6), jw).ravel())
    k = np.zeros((3 * nn, 3 * nn))
    ke = np.einsum("eqki,eqkl,eqlj,eq->eij", b, tang.reshape(ne, 8, 6, 6), b, jw)
    for e in range(ne):
        k[np.ix_(dofs[e], dofs[e])] += ke[e]
    np.testing.assert_allclose(res.internal_force, f, rtol=1e-10, atol=1e-10 * np.abs(f).max())
    kd = res.tangent.toarray()
    np.testing.assert_allclose(kd, k, rtol=1e-10, atol=1e-11 * np.abs(k).max())
    assert res.tangent.has_sorted_indices
