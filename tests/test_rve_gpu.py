"""GPU parity tests of the periodic RVE solve (cib_rve_* through the C ABI).

Golden vectors come from the reference's own solve_rve_microequilibrium (tests/golden).
Tolerances: float64 element kernels within 1e-6 relative of the reference's homogenised
stress and tangent (measured ~1e-10); float32 element kernels within 1e-4.  The reference's
homogeneous-RVE unit test (RVE == material point) is re-run on the GPU path.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import concrete_impact_b200 as cib
from concrete_impact_b200 import rve as R
from concrete_impact_b200.rve_builders import build_structured_rve, build_two_phase_sphere_rve, config0_materials
from tests.conftest import load_case

pytestmark = pytest.mark.gpu

UPDATE = cib.MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)


def _newton(meta) -> R.NonlinearNewtonSettings:
    mi, ra, rr, ia, ir, armijo = meta["newton"]
    return R.NonlinearNewtonSettings(mi, ra, rr, ia, ir, R.ArmijoSettings(enabled=bool(armijo)))


def _homogeneous_model(meta) -> R.StructuredHex8RVE:
    p = meta["material"]["params"]
    material = cib.J2ViscoplasticMaterial("single_phase_rve_j2", 1.0, **p)
    return build_structured_rve(tuple(meta["divisions"]), material, _newton(meta), hill_mandel_power_scale=10.0)


def _two_phase_model(arrays, meta, newton=None) -> R.StructuredHex8RVE:
    mortar, aggregate = config0_materials()
    div = tuple(meta["divisions"])
    model = build_two_phase_sphere_rve(div, mortar, aggregate, newton or _newton(meta), seed=meta["seed"])
    assert np.array_equal(model.element_phase_ids, arrays["element_phase"])
    return model


def _rel(got, ref) -> float:
    got, ref = np.asarray(got, dtype=np.float64), np.asarray(ref, dtype=np.float64)
    return float(np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-300))


@pytest.mark.parametrize("n", [1, 2])
def test_homogeneous_rve_recovers_material_point(n: int) -> None:
    """Reference tests/unit/fem/test_rve.py:66 on the GPU, plus the reference's own outputs."""
    arrays, meta = load_case(f"rve_homogeneous_{n}")
    model = _homogeneous_model(meta)
    material = model.material
    cache = R.build_rve_operator_cache(model)
    rve_state = R.initialize_rve_state(model)
    point_state = material.initialize_state(1)
    previous = np.zeros(6)
    for step in range(meta["steps"]):
        p = f"s{step}__"
        macro = arrays[p + "macro_strain"]
        response = R.solve_rve_microequilibrium(model, R.RVERequest(macro, 1.0e-3, UPDATE), rve_state, cache)
        point = material.update(
            cib.MaterialPointRequest(macro.reshape(1, 6), ((macro - previous) / 1.0e-3).reshape(1, 6), 1.0e-3,
                                     "three_dimensional", UPDATE),
            point_state, cib.MaterialResponseRequirements(tangent=True, free_energy=True, dissipation=True))  # fmt: skip
        assert np.allclose(response.macro_stress, point.stresses[0], atol=1.0e-10)
        assert np.allclose(response.effective_tangent, point.tangents[0], rtol=1.0e-10, atol=1.0e-9)
        assert response.diagnostics["periodic_fluctuation_error"] <= 1.0e-14
        assert response.diagnostics["hill_mandel_error"] <= 1.0e-12
        assert response.diagnostics["virtual_work_stress_error"] <= 1.0e-10
        for name, values in point.state.variables.items():
            got = response.state.material_state.variables[name]
            assert np.allclose(got, np.repeat(values, got.shape[0], axis=0), atol=1.0e-12)
        # and the reference's own RVE outputs
        np.testing.assert_allclose(response.macro_stress, arrays[p + "macro_stress"], atol=1e-10)
        np.testing.assert_allclose(response.effective_tangent, arrays[p + "effective_tangent"], rtol=1e-10, atol=1e-9)
        assert response.diagnostics["newton_iterations"] == meta["scalars"][step]["newton_iterations"]
        rve_state, point_state, previous = response.state, point.state, macro


@pytest.mark.parametrize("n", [4, 8])
def test_two_phase_rve_matches_reference_fp64(n: int) -> None:
    arrays, meta = load_case(f"rve_two_phase_{n}")
    model = _two_phase_model(arrays, meta)
    cache = R.build_rve_operator_cache(model)
    state = R.initialize_rve_state(model)
    for step in range(meta["steps"]):
        p = f"s{step}__"
        request = R.RVERequest(arrays[p + "macro_strain"], meta["time_step"], UPDATE)
        response = R.solve_rve_microequilibrium(model, request, state, cache)
        sc = meta["scalars"][step]
        assert _rel(response.macro_stress, arrays[p + "macro_stress"]) < 1e-6
        assert _rel(response.effective_tangent, arrays[p + "effective_tangent"]) < 1e-6
        assert _rel(response.micro_stresses, arrays[p + "micro_stresses"]) < 1e-6
        assert _rel(response.micro_strains, arrays[p + "micro_strains"]) < 1e-6
        eq_key = "phase_matrix__equivalent_plastic_strain"
        np.testing.assert_allclose(response.state.material_state.variables[eq_key], arrays[p + "state__" + eq_key],
                                   rtol=1e-6, atol=1e-9 * max(np.abs(arrays[p + "state__" + eq_key]).max(), 1e-30))  # fmt: skip
        np.testing.assert_allclose(response.state.fluctuation_dofs, arrays[p + "fluctuation"], rtol=1e-6,
                                   atol=1e-6 * np.abs(arrays[p + "fluctuation"]).max())  # fmt: skip
        assert response.diagnostics["newton_iterations"] == sc["newton_iterations"]
        for key in ("viscoplastic_active_volume_fraction", "unloading_volume_fraction"):
            assert response.diagnostics[key] == pytest.approx(sc[key], abs=1e-12)
        for key in ("free_energy_density", "dissipation_density", "positive_work_density", "negative_work_density",
                    "macro_work_increment", "micro_work_increment", "minimum_yield_activation_margin",
                    "maximum_yield_activation_margin"):  # fmt: skip
            got = response.free_energy_density if key == "free_energy_density" else (
                response.dissipation_density if key == "dissipation_density" else response.diagnostics[key])
            assert got == pytest.approx(sc[key], rel=1e-6, abs=1e-9 * max(abs(sc[key]), 1.0)), key
        for key in ("hill_mandel_error", "periodic_fluctuation_error", "virtual_work_stress_error",
                    "periodic_class_reaction_error", "reaction_antiperiodicity_error"):  # fmt: skip
            assert response.diagnostics[key] <= max(10 * sc[key], 1e-10), key
        mdiag = {k.removeprefix(p + "mdiag__"): v for k, v in arrays.items() if k.startswith(p + "mdiag__")}
        assert set(response.micro_diagnostics) == set(mdiag)
        for key, ref in mdiag.items():
            got = response.micro_diagnostics[key]
            both_nan = np.isnan(ref) & np.isnan(got)
            assert np.array_equal(np.isnan(ref), np.isnan(got)), key
            if key == "local_residual":
                continue
            scale = max(np.nanmax(np.abs(ref)) if np.any(~both_nan) else 0.0, 1e-30)
            np.testing.assert_allclose(got[~both_nan], ref[~both_nan], rtol=1e-6, atol=1e-7 * scale, err_msg=key)
        state = response.state


def test_two_phase_rve_fp32_within_tolerance() -> None:
    """float32 element kernels with float64 reductions and history: homogenised stress and
    tangent within 1e-4 of the reference's float64 solve."""
    arrays, meta = load_case("rve_two_phase_8")
    newton = R.NonlinearNewtonSettings(25, 1.0e-6, 1.0e-6, 1.0e-14, 1.0e-6)
    model = _two_phase_model(arrays, meta, newton)
    cache = R.build_rve_operator_cache(model, precision=32)
    state = R.initialize_rve_state(model)
    for step in range(meta["steps"]):
        p = f"s{step}__"
        response = R.solve_rve_microequilibrium(model, R.RVERequest(arrays[p + "macro_strain"], meta["time_step"], UPDATE),
                                                state, cache)  # fmt: skip
        assert _rel(response.macro_stress, arrays[p + "macro_stress"]) < 1e-4
        assert _rel(response.effective_tangent, arrays[p + "effective_tangent"]) < 1e-4
        state = response.state


def test_batched_rves_equal_single_solves_bitwise() -> None:
    """A batch of RVEs of different sizes, strains and time steps gives, RVE by RVE, the
    bitwise result of solving each alone (one CTA per RVE; fixed reduction order)."""
    mortar, aggregate = config0_materials()
    newton = R.NonlinearNewtonSettings(25, 1.0e-6, 1.0e-8, 1.0e-14, 1.0e-10)
    models = [build_two_phase_sphere_rve((n, n, n), mortar, aggregate, newton, seed=s) for n, s in ((4, 1), (6, 2), (2, 3))]
    strains = np.asarray([[-1.5e-3, 3e-4, 3e-4, 0, 0, 1e-4], [1e-3, -2e-4, -2e-4, 5e-4, 0, 0], [-2e-3, 0, 0, 0, 1e-3, 0]])
    dts = np.asarray([5e-6, 1e-5, 2e-6])
    batch = R.RVEBatch(models)
    batch.macro.copy_(torch.as_tensor(strains, device=batch.device))
    batch.dt.copy_(torch.as_tensor(dts, device=batch.device))
    R.solve_batch_step(batch, newton, UPDATE, False)
    batch.response(batch.batch_struct(UPDATE), batch.w, None, None)
    sums = batch.sums.cpu().numpy().copy()
    tangent = batch.effective_tangent(batch.batch_struct(UPDATE)).cpu().numpy().copy()
    for i, model in enumerate(models):
        single = R.RVEBatch([model])
        single.macro.copy_(torch.as_tensor(strains[i : i + 1], device=single.device))
        single.dt.fill_(float(dts[i]))
        R.solve_batch_step(single, newton, UPDATE, False)
        single.response(single.batch_struct(UPDATE), single.w, None, None)
        assert np.array_equal(single.sums.cpu().numpy()[0], sums[i])
        assert np.array_equal(single.effective_tangent(single.batch_struct(UPDATE)).cpu().numpy()[0], tangent[i])


def test_rve_solve_is_deterministic() -> None:
    arrays, meta = load_case("rve_two_phase_4")
    model = _two_phase_model(arrays, meta)
    cache = R.build_rve_operator_cache(model)
    state = R.initialize_rve_state(model)
    request = R.RVERequest(arrays["s1__macro_strain"], meta["time_step"], UPDATE)
    a = R.solve_rve_microequilibrium(model, request, state, cache)
    b = R.solve_rve_microequilibrium(model, request, state, cache)
    assert np.array_equal(a.macro_stress, b.macro_stress)
    assert np.array_equal(a.effective_tangent, b.effective_tangent)
    assert np.array_equal(a.micro_stresses, b.micro_stresses)


def test_rve_newton_iteration_limit_raises_equilibrium_error() -> None:
    arrays, meta = load_case("rve_two_phase_4")
    newton = R.NonlinearNewtonSettings(0, 1.0e-6, 1.0e-8, 1.0e-14, 1.0e-10)
    model = _two_phase_model(arrays, meta, newton)
    with pytest.raises(R.RVEEquilibriumError) as info:
        R.solve_rve_microequilibrium(model, R.RVERequest(arrays["s1__macro_strain"], meta["time_step"], UPDATE),
                                     R.initialize_rve_state(model))  # fmt: skip
    assert info.value.reason == "maximum_iterations_exceeded"
    assert info.value.diagnostics["iteration"] == 0


def test_rve_material_failure_carries_point_context() -> None:
    material = cib.J2ViscoplasticMaterial("assembly_failure_test", 1.0, 1000.0, 0.25, 1.0, 10.0, 0.02, 1.0, 2.0)
    newton = R.NonlinearNewtonSettings(5, 1e-10, 1e-10, 1e-12, 1e-10)
    model = build_structured_rve((1, 1, 1), material, newton)
    settings = cib.MaterialUpdateSettings(1, 1.0e-10, 1.0e-30, 1.0e-30)
    state = R.initialize_rve_state(model)
    with pytest.raises(cib.MaterialPointConvergenceError) as info:
        R.solve_rve_microequilibrium(model, R.RVERequest(np.asarray([0.02, 0, 0, 0, 0, 0]), 1.0e-3, settings), state)
    err = info.value
    assert err.reason == "maximum_iterations_exceeded"
    assert err.diagnostics["point_id"] == 0
    assert err.diagnostics["element_id"] == 0 and err.diagnostics["quadrature_id"] == 0
    assert np.all(state.material_state.variables["equivalent_plastic_strain"] == 0.0)


def test_prescribed_path_reports_only_accepted_steps() -> None:
    arrays, meta = load_case("rve_homogeneous_1")
    model = _homogeneous_model(meta)
    events = []
    times = np.asarray([0.0, 1.0e-3, 2.0e-3])
    strains = np.zeros((3, 6))
    strains[1:, 5] = [0.01, 0.02]
    result = R.solve_prescribed_rve_path(model, times, strains, UPDATE, events.append)
    assert len(result.responses) == 2
    assert [e.accepted_step for e in events] == [1, 2]
    assert [e.physical_time for e in events] == [1.0e-3, 2.0e-3]
