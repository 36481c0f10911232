"""GPU tests of the explicit velocity-Verlet material dynamics drop-in
(concrete_impact_b200.dynamics.solve_material_explicit, check_explicit_stability) against
the reference's own solve_material_explicit (golden histories from
tests/golden/make_golden.py, group "explicit"):

* a J2 Perzyna bar (8x1x1 elements, 40 MPa half-sine on the free end, 60 steps): every
  history within 1e-9 of its maximum (the update sequence is the reference's, in FP64);
* explicit FE2 with a two-phase 4^3 RVE at each of the 24 macro points of a 3x1x1 bar
  (RVEHomogenizedMaterial, one device batch of RVE solves per step): within 1e-6 (the RVE
  solves converge to the reference's Newton tolerances, not to its direct-solve iterates);
* the CFL bound and the reference's refusal message for a step above it.
"""

from __future__ import annotations

import math
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from conftest import load_case
from concrete_impact_b200.dynamics import (
    DirichletDofSet,
    TimeIntegrationSettings,
    check_explicit_stability,
    solve_material_explicit,
)
from concrete_impact_b200.materials import J2ViscoplasticMaterial, LinearElasticMaterial, MaterialUpdateSettings
from concrete_impact_b200.rve import ArmijoSettings, NonlinearNewtonSettings
from concrete_impact_b200.rve_builders import build_two_phase_sphere_rve
from concrete_impact_b200.rve_material import RVEHomogenizedMaterial
from oracle.rve import box_mesh

pytestmark = pytest.mark.gpu

HISTORIES = ("displacement", "velocity", "acceleration", "internal_force", "external_force", "stresses",
             "equivalent_plastic_strain", "kinetic_energy", "free_energy", "dissipated_energy", "external_work",
             "energy_residual", "positive_incremental_work", "negative_incremental_work",
             "viscoplastic_active_volume_fraction")  # fmt: skip


def _mortar() -> J2ViscoplasticMaterial:
    return J2ViscoplasticMaterial("mortar", 2200.0, 25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0)


def _mesh(meta, material, bundle: bool = False):
    nodes, elements = box_mesh(meta["bar"]["lengths"], meta["bar"]["divisions"])
    if bundle:
        return SimpleNamespace(mesh_info=SimpleNamespace(nodes=nodes, elements=elements, dimension=3),
                               material=material), nodes  # fmt: skip
    return SimpleNamespace(nodes=nodes, elements=elements, material=material), nodes


def _run(name: str, material, bundle: bool = False, record_fields: bool = True):
    g, meta = load_case(name)
    mesh, nodes = _mesh(meta, material, bundle)
    unit = torch.as_tensor(g["unit_force"], device="cuda")
    amp, dur = meta["amplitude"], meta["duration"]

    def load(t):
        return (amp * math.sin(math.pi * t / dur) if 0.0 <= t <= dur else 0.0) * unit

    ts = TimeIntegrationSettings("explicit", meta["time_step"], meta["num_steps"], 0.0, 0.5, meta["cfl_safety_factor"])
    n = 3 * nodes.shape[0]
    sol = solve_material_explicit(mesh, ts, np.zeros(n), np.zeros(n),
                                  DirichletDofSet(g["fixed_dofs"], np.zeros(g["fixed_dofs"].size)), load,
                                  "three_dimensional", MaterialUpdateSettings(*meta["update_settings"]),
                                  record_fields=record_fields)  # fmt: skip
    return sol, g, meta


def _check(sol, g, tol: float) -> None:
    np.testing.assert_allclose(sol.times, g["times"], rtol=1e-15)
    np.testing.assert_allclose(sol.accepted_time_steps, g["accepted_time_steps"], rtol=1e-12)
    for key in HISTORIES:
        ref = g[key]
        scale = max(np.abs(ref).max(), 1e-300)
        np.testing.assert_allclose(getattr(sol, key), ref, rtol=0, atol=tol * scale, err_msg=key)


def test_explicit_j2_bar_matches_reference() -> None:
    sol, g, meta = _run("explicit_j2_bar", _mortar())
    _check(sol, g, 1e-9)
    assert sol.equivalent_plastic_strain.max() > 1e-4  # the pulse drives the loaded end plastic
    assert np.all(sol.newton_iterations == 0) and sol.integrator_diagnostics == {}


def test_explicit_accepts_reference_bundle_and_final_fields_only() -> None:
    full, _, _ = _run("explicit_j2_bar", _mortar())
    last, _, _ = _run("explicit_j2_bar", _mortar(), bundle=True, record_fields=False)
    np.testing.assert_array_equal(last.kinetic_energy, full.kinetic_energy)
    assert last.displacement.shape == (1, full.displacement.shape[1])
    np.testing.assert_array_equal(last.displacement[0], full.displacement[-1])


def test_cfl_bound_and_refusal_match_reference() -> None:
    _, meta = load_case("explicit_j2_bar")
    mesh, _ = _mesh(meta, _mortar())
    report = check_explicit_stability(mesh, TimeIntegrationSettings("explicit", 1.0e-6, 1, 0.0, 0.5, 0.9))
    assert report.stable_time_step == pytest.approx(meta["stable_time_step"], rel=1e-14)
    assert report.minimum_length == pytest.approx(meta["minimum_length"], rel=1e-14)
    assert report.maximum_wave_speed == pytest.approx(meta["maximum_wave_speed"], rel=1e-14)
    bad = meta["cfl_violation"]
    with pytest.raises(ValueError) as info:
        check_explicit_stability(mesh, TimeIntegrationSettings("explicit", bad["time_step"], 1, 0.0, 0.5, 0.9))
    assert str(info.value) == bad["message"]


def test_explicit_fe2_with_rve_points_matches_reference() -> None:
    g, meta = load_case("explicit_fe2_bar")
    r = meta["rve"]
    aggregate = LinearElasticMaterial("aggregate", 2600.0, 50.0e9, 0.2)
    newton = NonlinearNewtonSettings(*r["newton"][:5], ArmijoSettings(enabled=r["newton"][5]))
    model = build_two_phase_sphere_rve(tuple(r["divisions"]), _mortar(), aggregate, newton, seed=r["seed"])
    np.testing.assert_array_equal(model.element_phase_ids, g["element_phase"])
    material = RVEHomogenizedMaterial(model, "two_phase_rve")
    try:
        sol, g, _ = _run("explicit_fe2_bar", material)
    finally:
        material.close()
    _check(sol, g, 1e-6)
    assert np.abs(sol.stresses).max() > 1e6
