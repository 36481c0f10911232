"""GPU tests of the general-mesh RVE path (concrete_impact_b200.rve_general).

* the reference's cylindrical O-grid RVE (golden solves of its own
  solve_rve_microequilibrium) through the public API: homogenised stress, effective
  tangent, fluctuation and displacement, Newton iterations, the consistency diagnostics;
* the same path through solve_prescribed_rve_path (dispatch from the operator cache);
* a structured box RVE solved by the general path against the batched box path (two
  independent device implementations of the same solve);
* the FE2 macro adapter (RVEHomogenizedMaterial) with O-grid RVEs at its points against
  single solves, with the reference's macro diagnostics.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from conftest import load_case  # noqa: E402
from concrete_impact_b200.materials import (J2ViscoplasticMaterial, LinearElasticMaterial,  # noqa: E402
                                            MaterialPointRequest, MaterialResponseRequirements, MaterialUpdateSettings)
from concrete_impact_b200.rve import (NonlinearNewtonSettings, RVERequest, build_rve_operator_cache,  # noqa: E402
                                      initialize_rve_state, solve_prescribed_rve_path, solve_rve_microequilibrium)
from concrete_impact_b200.rve_builders import (build_cylindrical_ogrid_hex8, build_cylindrical_two_phase_rve,  # noqa: E402
                                               build_two_phase_sphere_rve)
from concrete_impact_b200.rve_general import GeneralRVEOperators, solve_general_rve_microequilibrium  # noqa: E402

UPDATE = MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)


def _materials():
    return (J2ViscoplasticMaterial("mortar", 2200.0, 25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0),
            LinearElasticMaterial("aggregate", 2600.0, 50.0e9, 0.2))  # fmt: skip


def _ogrid_model(meta):
    s = meta["mesh"]
    mesh = build_cylindrical_ogrid_hex8(s["lengths"], s["inclusion_volume_fraction"], s["circumferential_divisions"],
                                        s["matrix_radial_divisions"], s["axial_divisions"])  # fmt: skip
    return build_cylindrical_two_phase_rve(mesh, *_materials(), NonlinearNewtonSettings(*meta["newton"][:5]), 1.0)


def _close(actual, ref, tol, what):
    np.testing.assert_allclose(np.asarray(actual), ref, rtol=0, atol=tol * np.abs(ref).max(), err_msg=what)


def test_ogrid_rve_matches_reference_solves() -> None:
    g, meta = load_case("rve_ogrid_cylinder")
    model = _ogrid_model(meta)
    cache = build_rve_operator_cache(model)
    assert isinstance(cache.batch, GeneralRVEOperators)
    state = initialize_rve_state(model)
    for step in range(meta["steps"]):
        request = RVERequest(g[f"s{step}__macro_strain"], meta["time_step"], UPDATE, MaterialResponseRequirements(tangent=True))
        out = solve_rve_microequilibrium(model, request, state, cache)
        state = out.state
        ref = meta["scalars"][step]
        assert out.diagnostics["newton_iterations"] == ref["newton_iterations"]
        _close(out.macro_stress, g[f"s{step}__macro_stress"], 1e-9, "macro_stress")
        _close(out.effective_tangent, g[f"s{step}__effective_tangent"], 1e-8, "effective_tangent")
        _close(out.state.fluctuation_dofs, g[f"s{step}__fluctuation"], 1e-8, "fluctuation")
        _close(out.displacement, g[f"s{step}__displacement"], 1e-9, "displacement")
        _close(out.micro_stresses, g[f"s{step}__micro_stresses"], 1e-8, "micro_stresses")
        for key in ("viscoplastic_active_volume_fraction", "unloading_volume_fraction"):
            assert out.diagnostics[key] == pytest.approx(ref[key], abs=1e-12), key
        for key in ("positive_work_density", "macro_work_increment", "micro_work_increment"):
            assert out.diagnostics[key] == pytest.approx(ref[key], rel=1e-7, abs=1e-6), key
        assert out.free_energy_density == pytest.approx(ref["free_energy_density"], rel=1e-8)
        assert out.diagnostics["virtual_work_stress_error"] <= 1e-10 * np.abs(g[f"s{step}__macro_stress"]).max()
        assert out.diagnostics["hill_mandel_error"] <= 1e-9 and out.diagnostics["periodic_fluctuation_error"] <= 1e-15
        assert set(out.phase_diagnostics) == {"matrix", "inclusion"}
    assert float(np.asarray(out.state.material_state.variables["phase_matrix__equivalent_plastic_strain"]).max()) > 0.0


def test_ogrid_rve_through_path_driver() -> None:
    g, meta = load_case("rve_ogrid_cylinder")
    model = _ogrid_model(meta)
    steps = meta["steps"]
    times = meta["time_step"] * np.arange(steps + 1)
    strains = np.vstack([np.zeros(6)] + [g[f"s{k}__macro_strain"] for k in range(steps)])
    result = solve_prescribed_rve_path(model, times, strains, UPDATE)
    assert len(result.responses) == steps
    _close(result.responses[-1].macro_stress, g[f"s{steps - 1}__macro_stress"], 1e-9, "macro_stress")


def test_general_path_matches_box_path_on_a_box_rve() -> None:
    mortar, aggregate = _materials()
    newton = NonlinearNewtonSettings(25, 1.0e-6, 1.0e-8, 1.0e-14, 1.0e-10)
    model = build_two_phase_sphere_rve((4, 4, 4), mortar, aggregate, newton, seed=7)
    ops = GeneralRVEOperators(model)
    box_cache = build_rve_operator_cache(model)
    s_box = s_gen = initialize_rve_state(model)
    direction = np.asarray([-1.0, 0.22, 0.22, 0.05, -0.03, 0.08])
    for amp in (0.6e-3, 1.4e-3):
        request = RVERequest(amp * direction, 5.0e-6, UPDATE, MaterialResponseRequirements(tangent=True))
        box = solve_rve_microequilibrium(model, request, s_box, box_cache)
        gen = solve_general_rve_microequilibrium(model, request, s_gen, ops)
        s_box, s_gen = box.state, gen.state
        _close(gen.macro_stress, np.asarray(box.macro_stress), 1e-9, "macro_stress")
        _close(gen.effective_tangent, np.asarray(box.effective_tangent), 1e-8, "effective_tangent")
        _close(gen.state.fluctuation_dofs, np.asarray(box.state.fluctuation_dofs), 1e-8, "fluctuation")
        assert abs(gen.diagnostics["newton_iterations"] - box.diagnostics["newton_iterations"]) <= 1


def test_fe2_adapter_with_ogrid_rves_matches_single_solves() -> None:
    from concrete_impact_b200.rve_material import RVEHomogenizedMaterial

    g, meta = load_case("rve_ogrid_cylinder")
    model = _ogrid_model(meta)
    adapter = RVEHomogenizedMaterial(model, "ogrid_rve")
    strains = np.stack([g[f"s{k}__macro_strain"] for k in range(3)])
    request = MaterialPointRequest(strains, strains / meta["time_step"], meta["time_step"], "three_dimensional", UPDATE)
    state = adapter.initialize_state(3)
    resp = adapter.update(request, state, MaterialResponseRequirements(tangent=True, free_energy=True, dissipation=True))
    cache = build_rve_operator_cache(model)
    for i in range(3):
        single = solve_rve_microequilibrium(model, RVERequest(strains[i], meta["time_step"], UPDATE,
                                                              MaterialResponseRequirements(tangent=True)),
                                            initialize_rve_state(model), cache)  # fmt: skip
        np.testing.assert_allclose(resp.stresses[i], single.macro_stress, rtol=0, atol=1e-12 * np.abs(single.macro_stress).max())
        np.testing.assert_allclose(resp.tangents[i], single.effective_tangent, rtol=0,
                                   atol=1e-12 * np.abs(single.effective_tangent).max())  # fmt: skip
        np.testing.assert_allclose(resp.state.variables["rve_fluctuation_dofs"][i], single.state.fluctuation_dofs,
                                   rtol=0, atol=1e-12 * max(np.abs(single.state.fluctuation_dofs).max(), 1e-30))  # fmt: skip
    assert np.all(state.variables["rve_macro_strain"] == 0.0)  # the committed state is untouched
    np.testing.assert_array_equal(resp.state.variables["rve_macro_strain"], strains)
    for key in ("incremental_work_density", "viscoplastic_active", "hill_mandel_error", "micro_newton_iterations",
                "phase_matrix__volume_fraction", "phase_inclusion__stress_xx", "phase_matrix__equivalent_plastic_strain"):
        assert resp.diagnostics[key].shape == (3,), key
    assert resp.diagnostics["phase_matrix__equivalent_plastic_strain"][2] > 0.0
