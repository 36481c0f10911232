"""CPU tests: the NumPy oracle against golden vectors from the reference implementation.

These pin the oracle before any GPU result is compared with it.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import j2vp as oj
from tests.conftest import golden_names, load_case, load_failures


def _params(meta, settings=None) -> oj.J2Params:
    p = meta["material"]["params"]
    return oj.J2Params(**p) if settings is None else oj.J2Params(**p, **settings)


@pytest.mark.parametrize("name", [n for n in golden_names("j2_") if "incremental" not in n])
def test_oracle_reference_form_matches_reference(name: str) -> None:
    """Every output of J2ViscoplasticMaterial.update, point by point (rel 1e-12)."""
    arrays, meta = load_case(name)
    p = _params(meta)
    out = oj.update_reference_form(
        p, arrays["strain"], arrays["plastic_strain_n"], arrays["eqps_n"], arrays["vpm_n"], meta["time_step"],
        arrays.get("strain_rates"),
    )  # fmt: skip
    assert np.all(out["status"] == oj.OK)
    scale = np.max(np.abs(arrays["stresses"]))
    np.testing.assert_allclose(out["stresses"], arrays["stresses"], rtol=1e-12, atol=1e-12 * scale)
    tscale = np.max(np.abs(arrays["tangents"]))
    np.testing.assert_allclose(out["tangents"], arrays["tangents"], rtol=1e-10, atol=1e-12 * tscale)
    for key in ("plastic_strain", "equivalent_plastic_strain", "viscoplastic_multiplier"):
        np.testing.assert_allclose(out[key], arrays[key], rtol=1e-12, atol=1e-18)
    for key in ("free_energy", "dissipation"):
        ref = arrays[key]
        np.testing.assert_allclose(out[key], ref, rtol=1e-10, atol=1e-12 * max(np.max(np.abs(ref)), 1e-300))
    ref_diag = {k.removeprefix("diag__"): v for k, v in arrays.items() if k.startswith("diag__")}
    assert set(ref_diag) == set(out["diagnostics"])
    for key, ref in ref_diag.items():
        got = out["diagnostics"][key]
        # local_residual is a roundoff-level quantity: compare it on the multiplier's scale.
        scale_key = "plastic_multiplier" if key == "local_residual" else key
        atol = 1e-12 * max(np.max(np.abs(ref_diag[scale_key])), 1e-30)
        np.testing.assert_allclose(got, ref, rtol=1e-9, atol=atol, err_msg=key)


def test_oracle_incremental_form_matches_reference_total_strain_call() -> None:
    """Stress-carried incremental form == reference call with strain = C^-1 s_n + ep_n + de."""
    arrays, meta = load_case("j2_incremental_config1")
    p = _params(meta)
    out = oj.update_incremental(
        p, arrays["dstrain"], arrays["stress_n"], arrays["plastic_strain_n"], arrays["eqps_n"], meta["time_step"]
    )
    assert np.all(out["status"] == oj.OK)
    scale = np.max(np.abs(arrays["stresses"]))
    np.testing.assert_allclose(out["stress"], arrays["stresses"], rtol=1e-9, atol=1e-10 * scale)
    np.testing.assert_allclose(out["tangent"], arrays["tangents"], rtol=1e-9, atol=1e-10 * np.max(np.abs(arrays["tangents"])))
    np.testing.assert_allclose(out["eqps"], arrays["equivalent_plastic_strain"], rtol=1e-12, atol=1e-18)
    np.testing.assert_array_equal(out["active"], arrays["viscoplastic_active"] > 0.5)
    assert 0.2 < out["active"].mean() < 0.6


def test_oracle_failure_reasons_match_reference() -> None:
    """Reason codes of the reference's failing points (point 1 of 3 fails)."""
    for key, case in load_failures().items():
        params = dict(case["params"])
        max_it, yrel, rabs, rrel = case["settings"]
        p = oj.J2Params(**params, max_iterations=int(max_it), yield_relative_tolerance=yrel,
                        residual_absolute_tolerance=rabs, residual_relative_tolerance=rrel)  # fmt: skip
        strain = np.asarray(case["strain"], dtype=np.float64)
        out = oj.update_reference_form(p, strain, np.zeros((3, 6)), np.zeros(3), np.zeros(3), case["time_step"])
        failing = np.flatnonzero(out["status"] != oj.OK)
        if key == "activation_tolerance":
            # A negative tolerance invalidates every point; the reference stops at the first one.
            assert failing[0] == 0
        else:
            assert list(failing) == [1], key
        assert oj.REASONS[out["status"][failing[0]]] == case["reason"], key


def test_oracle_tangent_matches_central_difference() -> None:
    """Analytic consistent tangent vs a central difference of the stress (m = 1 and m = 2)."""
    strain = np.asarray([[0.004, -0.0015, -0.001, 0.002, -0.003, 0.02]])
    for m, tau, dt in ((1.0, 30.0, 2.0), (2.0, 0.02, 1.0e-3)):
        p = oj.J2Params(3339.9160679991464, 0.36994096308414537, 10.0, 80.0, tau, 10.0, m)
        zero6, zero1 = np.zeros((1, 6)), np.zeros(1)
        base = oj.update_reference_form(p, strain, zero6, zero1, zero1, dt)
        assert base["diagnostics"]["active_surface"][0] == 4.0
        fd = np.zeros((6, 6))
        for j in range(6):
            h = 1e-7 * max(1.0, abs(strain[0, j]))
            plus, minus = strain.copy(), strain.copy()
            plus[0, j] += h
            minus[0, j] -= h
            sp = oj.update_reference_form(p, plus, zero6, zero1, zero1, dt)["stresses"][0]
            sm = oj.update_reference_form(p, minus, zero6, zero1, zero1, dt)["stresses"][0]
            fd[:, j] = (sp - sm) / (2 * h)
        np.testing.assert_allclose(base["tangents"][0], fd, rtol=1e-5, atol=1e-6)


def test_oracle_float32_model_within_fp32_tolerance() -> None:
    """The float32 model of the FP32 kernels stays within 1e-4 of the float64 oracle."""
    inputs = oj.config1_inputs(4096, seed=7)
    p = oj.mortar_params()
    ref = oj.update_incremental(p, inputs["dstrain"], inputs["stress"], inputs["plastic_strain"], inputs["eqps"], inputs["dt"])
    f32 = oj.update_incremental(
        p, inputs["dstrain"], inputs["stress"], inputs["plastic_strain"], inputs["eqps"], inputs["dt"], dtype=np.float32
    )
    scale = np.max(np.abs(ref["stress"]))
    assert np.max(np.abs(f32["stress"] - ref["stress"])) / scale < 1e-4
