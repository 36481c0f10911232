"""GPU parity tests of the J2 Perzyna return map (cib_j2vp_* through the C ABI).

Tolerances: float64 kernels within rtol 1e-9 of the reference / oracle (the bar is 1e-6);
float32 kernels within 1e-4 relative to the largest magnitude of each output.
The reference's own unit tests of the J2 viscoplastic model are re-run on the GPU path.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import concrete_impact_b200 as cib
from concrete_impact_b200 import batched
from oracle import j2vp as oj
from oracle.native import j2vp_incremental_c
from tests.conftest import golden_names, load_case, load_failures

pytestmark = pytest.mark.gpu

FULL = cib.MaterialResponseRequirements(tangent=True, free_energy=True, dissipation=True)
SETTINGS = cib.MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)


def _material(params: dict, name: str = "m", density: float = 1.0) -> cib.J2ViscoplasticMaterial:
    return cib.J2ViscoplasticMaterial(name=name, density=density, **params)


def _test_material(m: float, tau: float, sref: float = 10.0) -> cib.J2ViscoplasticMaterial:
    return cib.J2ViscoplasticMaterial("j2_vp_test", 1.0, 3339.9160679991464, 0.36994096308414537, 10.0, 80.0, tau,
                                      sref, m)  # fmt: skip


def _request(strain, time_step=1.0, rates=None, settings=SETTINGS):
    strain = np.asarray(strain, dtype=np.float64).reshape(-1, 6)
    return cib.MaterialPointRequest(strain, rates, time_step, "three_dimensional", settings)


def _close(got, ref, rtol=1e-9, rel_atol=1e-12, what=""):
    got = np.asarray(got)
    ref = np.asarray(ref)
    scale = max(float(np.max(np.abs(ref))) if ref.size else 0.0, 1e-300)
    np.testing.assert_allclose(got, ref, rtol=rtol, atol=rel_atol * scale, err_msg=what)


@pytest.mark.parametrize("name", [n for n in golden_names("j2_") if "incremental" not in n])
def test_reference_form_matches_reference_outputs(name: str) -> None:
    arrays, meta = load_case(name)
    material = _material(meta["material"]["params"], meta["material"]["name"])
    state = cib.MaterialState({"plastic_strain": arrays["plastic_strain_n"].copy(),
                               "equivalent_plastic_strain": arrays["eqps_n"].copy(),
                               "viscoplastic_multiplier": arrays["vpm_n"].copy()})  # fmt: skip
    response = material.update(_request(arrays["strain"], meta["time_step"], arrays.get("strain_rates")), state, FULL)
    _close(response.stresses, arrays["stresses"], what="stresses")
    _close(response.tangents, arrays["tangents"], what="tangents")
    _close(response.free_energy, arrays["free_energy"], what="free_energy")
    _close(response.dissipation, arrays["dissipation"], what="dissipation")
    for key in ("plastic_strain", "equivalent_plastic_strain", "viscoplastic_multiplier"):
        _close(response.state.variables[key], arrays[key], what=key)
    ref_diag = {k.removeprefix("diag__"): v for k, v in arrays.items() if k.startswith("diag__")}
    assert set(response.diagnostics) == set(ref_diag)
    for key, ref in ref_diag.items():
        if key == "local_residual":  # roundoff-level: compare on the multiplier's scale
            np.testing.assert_allclose(response.diagnostics[key], ref,
                                       atol=1e-12 * np.max(np.abs(ref_diag["plastic_multiplier"])))  # fmt: skip
        else:
            _close(response.diagnostics[key], ref, what=key)


def test_failures_raise_the_reference_exception() -> None:
    for key, case in load_failures().items():
        max_it, yrel, rabs, rrel = case["settings"]
        material = cib.J2ViscoplasticMaterial(name=f"fail_{key}", density=1.0, **case["params"])
        settings = cib.MaterialUpdateSettings(int(max_it), yrel, rabs, rrel)
        state = material.initialize_state(3)
        snapshot = {k: v.copy() for k, v in state.variables.items()}
        with pytest.raises(cib.MaterialPointConvergenceError) as info:
            material.update(_request(case["strain"], case["time_step"], settings=settings), state)
        error, ref = info.value, case["diagnostics"]
        assert error.reason == case["reason"], key
        assert str(error) == case["message"], key
        assert error.diagnostics["point_id"] == ref["point_id"], key
        assert error.diagnostics["algorithm"] == ref["algorithm"], key
        for field in ("iteration", "max_iterations", "residual", "newton_candidate", "physical_upper_bound",
                      "plastic_multiplier", "corrected_overstress", "trial_equivalent_stress", "radicand"):  # fmt: skip
            if field in ref:
                got, want = error.diagnostics[field], ref[field]
                if isinstance(want, float):
                    assert got == pytest.approx(want, rel=1e-9), (key, field)
                else:
                    assert got == want, (key, field)
        assert set(ref) <= set(error.diagnostics) | {"strain"}, (key, set(ref) - set(error.diagnostics))
        for k, v in state.variables.items():
            assert np.array_equal(v, snapshot[k])


def test_committed_state_is_not_mutated_and_repeatable() -> None:
    material = _test_material(2.0, 0.02)
    state = material.initialize_state(1)
    snapshot = {k: v.copy() for k, v in state.variables.items()}
    strain = [0.0, 0.0, 0.0, 0.0, 0.0, 6.0e-3]
    first = material.update(_request(strain, 1e-3), state)
    second = material.update(_request(strain, 1e-3), state)
    for k, v in state.variables.items():
        assert np.array_equal(v, snapshot[k])
    assert np.array_equal(first.stresses, second.stresses)
    assert first.state.variables["equivalent_plastic_strain"][0] > 0.0


def test_device_tensors_stay_on_the_device() -> None:
    material = _test_material(1.0, 30.0)
    state = material.initialize_state(4)
    dev_state = cib.MaterialState({k: torch.as_tensor(v, device="cuda") for k, v in state.variables.items()})
    strain = torch.zeros((4, 6), dtype=torch.float64, device="cuda")
    strain[:, 5] = torch.linspace(0.0, 0.02, 4, device="cuda", dtype=torch.float64)
    response = material.update(cib.MaterialPointRequest(strain, None, 2.0, "three_dimensional", SETTINGS), dev_state, FULL)
    assert response.stresses.is_cuda and response.tangents.is_cuda
    host = material.update(_request(strain.cpu().numpy(), 2.0), state, FULL)
    np.testing.assert_array_equal(response.stresses.cpu().numpy(), host.stresses)


def test_empty_batch() -> None:
    material = _test_material(1.0, 30.0)
    response = material.update(_request(np.zeros((0, 6))), material.initialize_state(0), FULL)
    assert response.stresses.shape == (0, 6) and response.tangents.shape == (0, 6, 6)
    assert response.diagnostics == {}


@pytest.mark.parametrize("m,tau,dt", [(1.0, 30.0, 2.0), (2.0, 0.02, 1.0e-3)])
def test_consistent_tangent_matches_central_difference(m: float, tau: float, dt: float) -> None:
    """Reference tests plasticity.py test file :179 and :210 on the GPU path."""
    material = _test_material(m, tau)
    strain = np.asarray([0.004, -0.0015, -0.001, 0.002, -0.003, 0.02])
    state = material.initialize_state(1)
    base = material.update(_request(strain, dt), state, FULL)
    assert base.diagnostics["active_surface"][0] == pytest.approx(4.0)
    perturbed = []
    for j in range(6):
        h = 1e-7 * max(1.0, abs(strain[j]))
        for sign in (1.0, -1.0):
            e = strain.copy()
            e[j] += sign * h
            perturbed.append(e)
    batch = material.update(_request(np.asarray(perturbed), dt), material.initialize_state(12))
    fd = np.zeros((6, 6))
    for j in range(6):
        h = 1e-7 * max(1.0, abs(strain[j]))
        fd[:, j] = (batch.stresses[2 * j] - batch.stresses[2 * j + 1]) / (2 * h)
    np.testing.assert_allclose(base.tangents[0], fd, rtol=1e-5, atol=1e-6)
    if m == 2.0:
        q = base.state.variables["equivalent_plastic_strain"][0]
        eel = strain - base.state.variables["plastic_strain"][0]
        assert base.free_energy[0] == pytest.approx(0.5 * base.stresses[0] @ eel + 0.5 * 80.0 * q**2, rel=1e-12)
        assert base.dissipation[0] == pytest.approx(
            base.diagnostics["plastic_power"][0] - base.diagnostics["hardening_storage_rate"][0], rel=1e-12, abs=1e-12)
        assert abs(base.diagnostics["local_residual"][0]) <= 1e-12


def test_multiplier_depends_on_physical_time_step() -> None:
    material = _test_material(1.0, 30.0)
    strain = [0.0, 0.0, 0.0, 0.0, 0.0, 0.02]
    small = material.update(_request(strain, 0.5), material.initialize_state(1))
    large = material.update(_request(strain, 5.0), material.initialize_state(1))
    assert large.diagnostics["viscoplastic_multiplier"][0] > small.diagnostics["viscoplastic_multiplier"][0]
    assert large.stresses[0, 5] < small.stresses[0, 5]


def test_yield_activation_uses_relative_stress_scale() -> None:
    material = _test_material(2.0, 0.02)
    g = material.shear_modulus
    settings = cib.MaterialUpdateSettings(50, 1.0e-3, 1.0e-12, 1.0e-10)
    strains = np.zeros((2, 6))
    strains[:, 5] = [(10.0 + over) / (np.sqrt(3.0) * g) for over in (5.0e-3, 2.0e-2)]
    r = material.update(_request(strains, 1.0e-3, settings=settings), material.initialize_state(2))
    d = r.diagnostics
    assert 0.0 < d["trial_yield_value"][0] < d["yield_activation_threshold"][0]
    assert d["plastic_multiplier"][0] == 0.0 and d["yield_activation_margin"][0] < 0.0 and d["viscoplastic_active"][0] == 0.0
    assert d["trial_yield_value"][1] > d["yield_activation_threshold"][1]
    assert d["plastic_multiplier"][1] > 0.0 and d["yield_activation_margin"][1] > 0.0 and d["viscoplastic_active"][1] == 1.0


def test_loading_diagnostics_separate_work_stress_and_flow() -> None:
    material = _test_material(2.0, 0.02)
    loaded_strain = np.zeros(6)
    loaded_strain[5] = 0.02
    rate = (loaded_strain / 1e-3).reshape(1, 6)  # step-average rate from a zero previous strain
    loaded = material.update(_request(loaded_strain, 1e-3, rate), material.initialize_state(1), FULL)
    assert loaded.diagnostics["incremental_work_density"][0] > 0.0
    assert loaded.diagnostics["equivalent_stress_increment"][0] > 0.0
    assert loaded.diagnostics["viscoplastic_active"][0] == 1.0
    relaxed = material.update(_request(loaded_strain, 1e-3, np.zeros((1, 6))), loaded.state, FULL)
    assert relaxed.diagnostics["incremental_work_density"][0] == pytest.approx(0.0)
    assert relaxed.diagnostics["equivalent_stress_increment"][0] < 0.0
    assert relaxed.diagnostics["viscoplastic_active"][0] == 1.0


# ---------------------------------------------------------------------------------------
# SoA streaming kernel.


def _soa_inputs(n: int, seed: int, dtype: torch.dtype):
    inp = oj.config1_inputs(n, seed=seed)
    dev = torch.device("cuda")
    de = torch.as_tensor(inp["dstrain"].T.copy(), device=dev).to(dtype)
    st = batched.SoAState(torch.as_tensor(inp["stress"].T.copy(), device=dev).to(dtype),
                          torch.as_tensor(inp["plastic_strain"].T.copy(), device=dev).to(dtype),
                          torch.as_tensor(inp["eqps"], device=dev))  # fmt: skip
    return inp, de, st


def _mortar() -> cib.J2ViscoplasticMaterial:
    p = oj.mortar_params()
    return cib.J2ViscoplasticMaterial("mortar", 2200.0, p.young_modulus, p.poisson_ratio, p.yield_stress,
                                      p.hardening_modulus, p.time_scale, p.reference_stress, p.rate_exponent)  # fmt: skip


@pytest.mark.parametrize("n", [1, 3, 4, 1000, (1 << 18) + 3])
def test_soa_f64_matches_c_oracle(n: int) -> None:
    inp, de, st = _soa_inputs(n, 11, torch.float64)
    new, tan = batched.j2vp_update_soa(_mortar(), SETTINGS, inp["dt"], de, st)
    ref = j2vp_incremental_c(oj.mortar_params(), inp["dt"], inp["dstrain"].T, inp["stress"].T, inp["plastic_strain"].T,
                             inp["eqps"])  # fmt: skip
    _close(new.stress.cpu().numpy(), ref["stress"], rtol=1e-12, what="stress")
    _close(new.plastic_strain.cpu().numpy(), ref["plastic_strain"], rtol=1e-12, rel_atol=1e-12, what="plastic strain")
    _close(new.eqps.cpu().numpy(), ref["eqps"], rtol=1e-13, what="eqps")
    _close(tan.cpu().numpy(), ref["tangent"], rtol=1e-11, what="tangent")


def test_soa_matches_golden_reference_case_f64_and_f32() -> None:
    arrays, meta = load_case("j2_incremental_config1")
    material = _mortar()
    for dtype, rtol, rel_atol in ((torch.float64, 1e-9, 1e-10), (torch.float32, 1e-4, 1e-4)):
        dev = torch.device("cuda")
        de = torch.as_tensor(arrays["dstrain"].T.copy(), device=dev).to(dtype)
        st = batched.SoAState(torch.as_tensor(arrays["stress_n"].T.copy(), device=dev).to(dtype),
                              torch.as_tensor(arrays["plastic_strain_n"].T.copy(), device=dev).to(dtype),
                              torch.as_tensor(arrays["eqps_n"], device=dev))  # fmt: skip
        new, tan = batched.j2vp_update_soa(material, SETTINGS, meta["time_step"], de, st)
        s = new.stress.double().cpu().numpy().T
        _close(s, arrays["stresses"], rtol=rtol, rel_atol=rel_atol, what=f"stress {dtype}")
        t = tan.double().cpu().numpy().T.reshape(-1, 6, 6)
        _close(t, arrays["tangents"], rtol=rtol, rel_atol=rel_atol, what=f"tangent {dtype}")
        _close(new.eqps.cpu().numpy(), arrays["equivalent_plastic_strain"], rtol=1e-6 if dtype == torch.float32 else 1e-12,
               rel_atol=1e-6, what=f"eqps {dtype}")  # fmt: skip


def test_soa_f32_within_fp32_tolerance_of_f64_oracle() -> None:
    n = 1 << 20
    inp, de, st = _soa_inputs(n, 21, torch.float32)
    new, tan = batched.j2vp_update_soa(_mortar(), SETTINGS, inp["dt"], de, st)
    ref = oj.update_incremental(oj.mortar_params(), inp["dstrain"], inp["stress"], inp["plastic_strain"], inp["eqps"], inp["dt"])
    s = new.stress.double().cpu().numpy().T
    assert np.max(np.abs(s - ref["stress"])) / np.max(np.abs(ref["stress"])) < 1e-4
    t = tan.double().cpu().numpy().T.reshape(-1, 6, 6)
    assert np.max(np.abs(t - ref["tangent"])) / np.max(np.abs(ref["tangent"])) < 1e-4


def test_soa_full_size_against_oracle_and_consistency() -> None:
    """16,777,216 points in float64: all stresses/state against the C oracle, tangents on a
    strided sample, plus the size-independent consistency condition of active points
    (final overstress = tau sigma_ref dgamma / dt for m = 1)."""
    n = 16_777_216
    inp, de, st = _soa_inputs(n, 1234, torch.float64)
    new, tan = batched.j2vp_update_soa(_mortar(), SETTINGS, inp["dt"], de, st)
    ref = j2vp_incremental_c(oj.mortar_params(), inp["dt"], inp["dstrain"].T, inp["stress"].T, inp["plastic_strain"].T,
                             inp["eqps"], with_tangent=False)  # fmt: skip
    s = new.stress.cpu().numpy()
    _close(s, ref["stress"], rtol=1e-12, what="stress")
    q1 = new.eqps.cpu().numpy()
    _close(q1, ref["eqps"], rtol=1e-13, what="eqps")
    sample = slice(0, n, 4099)
    t_sub = tan[:, sample].cpu().numpy()
    sub = oj.update_incremental(oj.mortar_params(), inp["dstrain"][sample], inp["stress"][sample],
                                inp["plastic_strain"][sample], inp["eqps"][sample], inp["dt"])  # fmt: skip
    _close(t_sub.T.reshape(-1, 6, 6), sub["tangent"], rtol=1e-12, what="tangent sample")
    p = oj.mortar_params()
    dg = q1 - inp["eqps"]
    act = dg > 0
    assert 0.2 < act.mean() < 0.6
    qf = np.sqrt(oj.j2_radicand(oj.deviatoric(s[:, act].T)))
    over = qf - (p.yield_stress + p.hardening_modulus * q1[act])
    # absolute floor: q_final - radius cancels two ~2e7 Pa numbers (float64 roundoff ~1e-8 Pa)
    np.testing.assert_allclose(over, p.time_scale * p.reference_stress * dg[act] / inp["dt"], rtol=1e-8,
                               atol=1e-15 * p.yield_stress * 10)


def test_soa_is_deterministic() -> None:
    inp, de, st = _soa_inputs(100_003, 3, torch.float64)
    a, ta = batched.j2vp_update_soa(_mortar(), SETTINGS, inp["dt"], de, st)
    b, tb = batched.j2vp_update_soa(_mortar(), SETTINGS, inp["dt"], de, st)
    assert torch.equal(a.stress, b.stress) and torch.equal(ta, tb) and torch.equal(a.eqps, b.eqps)


def test_soa_failure_reports_point_and_reason() -> None:
    material = cib.J2ViscoplasticMaterial("vp", 1.0, 3339.9160679991464, 0.36994096308414537, 10.0, 80.0, 0.02,
                                          1.0e-300, 2.0)  # fmt: skip
    n = 64
    de = torch.zeros((6, n), dtype=torch.float64, device="cuda")
    de[5, 37] = 0.02
    st = batched.SoAState(torch.zeros((6, n), dtype=torch.float64, device="cuda"),
                          torch.zeros((6, n), dtype=torch.float64, device="cuda"),
                          torch.zeros(n, dtype=torch.float64, device="cuda"))  # fmt: skip
    with pytest.raises(cib.MaterialPointConvergenceError) as info:
        batched.j2vp_update_soa(material, SETTINGS, 1e-3, de, st)
    assert info.value.reason == "non_finite_iteration_value"
    assert info.value.diagnostics["point_id"] == 37


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_host_pipeline_equals_device_path(dtype: torch.dtype) -> None:
    n = 300_007
    inp, de, st = _soa_inputs(n, 8, dtype)
    dev_new, dev_tan = batched.j2vp_update_soa(_mortar(), SETTINGS, inp["dt"], de, st)
    pipe = batched.J2HostPipeline(_mortar(), SETTINGS, dtype, chunk=1 << 16)
    de_h = de.cpu().pin_memory()
    st_h = batched.SoAState(st.stress.cpu().pin_memory(), st.plastic_strain.cpu().pin_memory(), st.eqps.cpu().pin_memory())
    out = batched.SoAState(torch.empty((6, n), dtype=dtype).pin_memory(), torch.empty((6, n), dtype=dtype).pin_memory(),
                           torch.empty(n, dtype=torch.float64).pin_memory())  # fmt: skip
    tan = torch.empty((36, n), dtype=dtype).pin_memory()
    assert pipe.run(inp["dt"], de_h, st_h, out, tan) == -1
    assert torch.equal(out.stress, dev_new.stress.cpu())
    assert torch.equal(out.plastic_strain, dev_new.plastic_strain.cpu())
    assert torch.equal(out.eqps, dev_new.eqps.cpu())
    assert torch.equal(tan, dev_tan.cpu())


@pytest.mark.parametrize("dtype,rtol", [(torch.float64, 1e-12), (torch.float32, 2e-6)])
@pytest.mark.parametrize("n", [5, 100_003])
def test_compact_tangent_expands_to_the_full_tangent(dtype: torch.dtype, rtol: float, n: int) -> None:
    """cib_j2vp_update_soa_compact_*: the same state as the full-tangent entry, and its 8
    rows (n, f, c) give the full consistent tangent C = K 1(x)1 + f P + c n(x)n."""
    inp, de, st = _soa_inputs(n, 21, dtype)
    new, tan = batched.j2vp_update_soa(_mortar(), SETTINGS, inp["dt"], de, st)
    flags = torch.full((1,), -1, dtype=torch.int64, device=de.device)
    out = batched.SoAState.empty(n, dtype, de.device)
    compact = torch.empty((8, n), dtype=dtype, device=de.device)
    batched.launch_j2vp_soa(_mortar(), SETTINGS, inp["dt"], de, st, out, compact, flags)
    torch.cuda.synchronize()
    assert int(flags[0]) == -1
    assert torch.equal(out.stress, new.stress) and torch.equal(out.eqps, new.eqps)
    full = batched.expand_compact_tangent(compact.double(), _mortar()).cpu().numpy()
    ref = tan.double().cpu().numpy()
    assert np.abs(full - ref).max() <= rtol * np.abs(ref).max()
    plastic = compact[7].cpu().numpy() != 0.0
    assert 0.1 < plastic.mean() < 0.9  # both branches occur


def test_host_pipeline_compact_tangent() -> None:
    n = 70_001
    inp, de, st = _soa_inputs(n, 9, torch.float64)
    flags = torch.full((1,), -1, dtype=torch.int64, device=de.device)
    dev_out = batched.SoAState.empty(n, torch.float64, de.device)
    dev_c = torch.empty((8, n), dtype=torch.float64, device=de.device)
    batched.launch_j2vp_soa(_mortar(), SETTINGS, inp["dt"], de, st, dev_out, dev_c, flags)
    pipe = batched.J2HostPipeline(_mortar(), SETTINGS, torch.float64, chunk=1 << 15, compact_tangent=True)
    de_h = de.cpu().pin_memory()
    st_h = batched.SoAState(st.stress.cpu().pin_memory(), st.plastic_strain.cpu().pin_memory(), st.eqps.cpu().pin_memory())
    out = batched.SoAState(torch.empty((6, n), dtype=torch.float64).pin_memory(),
                           torch.empty((6, n), dtype=torch.float64).pin_memory(),
                           torch.empty(n, dtype=torch.float64).pin_memory())  # fmt: skip
    tan = torch.empty((8, n), dtype=torch.float64).pin_memory()
    assert pipe.run(inp["dt"], de_h, st_h, out, tan) == -1
    assert torch.equal(out.stress, dev_out.stress.cpu()) and torch.equal(tan, dev_c.cpu())
    assert batched.J2HostPipeline.bytes_per_point(torch.float64, True, True) == (152, 168)
