"""GPU tests of the FE^2 macro adapter RVEHomogenizedMaterial (one RVE per macro point in
one device batch), after the reference's adapter test
(tests/unit/fem/test_rve_dynamics.py:61-107): independent per-point states and
diagnostics, the wave speed of the stiffest phase, and agreement with the single-RVE
solve of each point; the committed state is never written."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import concrete_impact_b200 as cib
from concrete_impact_b200 import rve as R
from concrete_impact_b200.rve_builders import build_two_phase_sphere_rve
from concrete_impact_b200.rve_material import RVEHomogenizedMaterial

pytestmark = pytest.mark.gpu

SETTINGS = cib.MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)


def _model():
    matrix = cib.J2ViscoplasticMaterial("matrix", 2400.0, 1000.0, 0.2, 10.0, 20.0, 0.02, 10.0, 2.0)
    inclusion = cib.LinearElasticMaterial("inclusion", 7850.0, 6666.666666666667, 0.3)
    newton = R.NonlinearNewtonSettings(20, 1.0e-10, 1.0e-10, 1.0e-12, 1.0e-10, R.ArmijoSettings(enabled=True))
    return build_two_phase_sphere_rve((4, 4, 4), matrix, inclusion, newton, seed=3), inclusion


def _request(strains, rates):
    return cib.MaterialPointRequest(np.asarray(strains), np.asarray(rates), 1.0e-3, "three_dimensional", SETTINGS)


def test_adapter_keeps_independent_macro_point_states() -> None:
    model, inclusion = _model()
    adapter = RVEHomogenizedMaterial(model, "two_phase")
    state = adapter.initialize_state(2)
    before = {k: np.array(v, copy=True) for k, v in state.variables.items()}
    req = _request([[0, 0, 0, 0, 0, 0.03], [0, 0, 0, 0, 0, 0.002]], [[0, 0, 0, 0, 0, 30.0], [0, 0, 0, 0, 0, 2.0]])
    resp = adapter.update(req, state, cib.MaterialResponseRequirements(tangent=True, free_energy=True, dissipation=True))
    assert adapter.maximum_wave_speed == inclusion.maximum_wave_speed
    phase_q = np.asarray(resp.diagnostics["phase_matrix__equivalent_plastic_strain"])
    assert phase_q[0] > phase_q[1]
    ms = resp.state.variables["rve_macro_strain"]
    assert not np.shares_memory(ms[0], ms[1])
    for k, v in state.variables.items():  # the committed state is untouched
        assert np.array_equal(v, before[k]), k
    assert resp.tangents.shape == (2, 6, 6) and resp.free_energy.shape == (2,) and resp.dissipation.shape == (2,)


def test_adapter_matches_single_rve_solves() -> None:
    model, _ = _model()
    adapter = RVEHomogenizedMaterial(model, "two_phase")
    strains = np.random.default_rng(0).normal(0.0, 4e-3, size=(3, 6))
    rates = strains / 1.0e-3
    resp = adapter.update(_request(strains, rates), adapter.initialize_state(3),
                          cib.MaterialResponseRequirements(tangent=True))  # fmt: skip
    cache = R.build_rve_operator_cache(model)
    for i in range(3):
        single = R.solve_rve_microequilibrium(
            model, R.RVERequest(strains[i], 1.0e-3, SETTINGS, cib.MaterialResponseRequirements(tangent=True)),
            R.initialize_rve_state(model), cache)  # fmt: skip
        ref = np.asarray(single.macro_stress)
        np.testing.assert_allclose(np.asarray(resp.stresses[i]), ref, rtol=0, atol=1e-9 * np.abs(ref).max())
        tref = np.asarray(single.effective_tangent)
        np.testing.assert_allclose(np.asarray(resp.tangents[i]), tref, rtol=0, atol=1e-8 * np.abs(tref).max())


def test_effective_tangent_with_cluster_pcg_matches_one_cta() -> None:
    model, _ = _model()
    strain = np.array([2e-3, -1e-3, 5e-4, 1e-3, 0.0, 2e-3])
    out = {}
    for cluster in (1, 4):
        cache = R.build_rve_operator_cache(model, linear_solver=R.LinearSolverOptions(cluster=cluster))
        out[cluster] = R.solve_rve_microequilibrium(
            model, R.RVERequest(strain, 1.0e-3, SETTINGS, cib.MaterialResponseRequirements(tangent=True)),
            R.initialize_rve_state(model), cache)  # fmt: skip
    t1, t4 = np.asarray(out[1].effective_tangent), np.asarray(out[4].effective_tangent)
    np.testing.assert_allclose(t4, t1, rtol=0, atol=1e-8 * np.abs(t1).max())
    s1, s4 = np.asarray(out[1].macro_stress), np.asarray(out[4].macro_stress)
    np.testing.assert_allclose(s4, s1, rtol=0, atol=1e-9 * np.abs(s1).max())
