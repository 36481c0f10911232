"""Generate golden vectors by running the reference implementation itself.

Run in a container that holds the reference checkout (read-only) at REFERENCE_SRC:

    python tests/golden/make_golden.py [--reference /root/reference/src]

The reference imports gmsh, meshio and h5py at module level in files that the material
and RVE paths never execute; empty stand-in modules are put on sys.path for them.  The
outputs are small compressed .npz files in this directory; the GPU box never needs the
reference.
"""

from __future__ import annotations

import argparse
import json
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def _import_reference(src: str) -> None:
    stubs = Path(tempfile.mkdtemp(prefix="ref_stubs_"))
    for name in ("gmsh", "meshio", "h5py"):
        (stubs / f"{name}.py").write_text("")
    sys.path[:0] = [str(stubs), src]


def _settings(mod, max_iterations=50, yrel=1.0e-10, rabs=1.0e-12, rrel=1.0e-10):
    return mod.MaterialUpdateSettings(max_iterations, yrel, rabs, rrel)


def _j2_material(plasticity, spec):
    return plasticity.J2ViscoplasticMaterial(name=spec["name"], density=spec["density"], **spec["params"])


MATERIALS = {
    # Mortar of the two-phase RVE (SI units): m = 1 closed form.
    "mortar": {"name": "mortar", "density": 2200.0, "params": dict(
        young_modulus=25.0e9, poisson_ratio=0.2, yield_stress=20.0e6, hardening_modulus=2.0e9,
        time_scale=1.0e-3, reference_stress=20.0e6, rate_exponent=1.0)},
    # The reference unit-test material with m = 2 (local Newton).
    "test_m2": {"name": "j2_vp_quadratic_test", "density": 1.0, "params": dict(
        young_modulus=3339.9160679991464, poisson_ratio=0.36994096308414537, yield_stress=10.0,
        hardening_modulus=80.0, time_scale=0.02, reference_stress=10.0, rate_exponent=2.0)},
    # The reference unit-test material with m = 1 and a long time scale.
    "test_m1": {"name": "j2_vp_tangent_test", "density": 1.0, "params": dict(
        young_modulus=3339.9160679991464, poisson_ratio=0.36994096308414537, yield_stress=10.0,
        hardening_modulus=80.0, time_scale=30.0, reference_stress=10.0, rate_exponent=1.0)},
}  # fmt: skip


def _random_points(rng, n, scale, eqps_max):
    strain = rng.normal(0.0, scale, size=(n, 6))
    plastic = rng.normal(0.0, 0.2 * scale, size=(n, 6))
    plastic[:, :3] -= plastic[:, :3].mean(axis=1, keepdims=True)
    eqps = rng.uniform(0.0, eqps_max, size=n)
    vpm = rng.uniform(0.0, eqps_max, size=n)
    rates = rng.normal(0.0, scale, size=(n, 6)) * 50.0
    return strain, plastic, eqps, vpm, rates


def make_j2_cases(data_mod, plasticity):
    cases = {}
    rng = np.random.default_rng(20260701)
    plan = [
        ("mortar", 512, 5.0e-4, 0.01, 1.0e-5),
        ("test_m2", 256, 3.0e-3, 0.02, 1.0e-3),
        ("test_m1", 256, 3.0e-3, 0.02, 2.0),
    ]
    for key, n, scale, eqps_max, dt in plan:
        spec = MATERIALS[key]
        material = _j2_material(plasticity, spec)
        strain, plastic, eqps, vpm, rates = _random_points(rng, n, scale, eqps_max)
        state = data_mod.MaterialState({
            "plastic_strain": plastic.copy(), "equivalent_plastic_strain": eqps.copy(),
            "viscoplastic_multiplier": vpm.copy()})  # fmt: skip
        for with_rates in (True, False):
            request = data_mod.MaterialPointRequest(
                strains=strain, strain_rates=rates if with_rates else None, time_step=dt,
                kinematics="three_dimensional", update_settings=_settings(data_mod))  # fmt: skip
            response = material.update(
                request, state, data_mod.MaterialResponseRequirements(tangent=True, free_energy=True, dissipation=True))
            arrays = {
                "strain": strain, "plastic_strain_n": plastic, "eqps_n": eqps, "vpm_n": vpm,
                "stresses": response.stresses, "tangents": response.tangents,
                "free_energy": response.free_energy, "dissipation": response.dissipation,
                "plastic_strain": response.state.variables["plastic_strain"],
                "equivalent_plastic_strain": response.state.variables["equivalent_plastic_strain"],
                "viscoplastic_multiplier": response.state.variables["viscoplastic_multiplier"],
            }  # fmt: skip
            if with_rates:
                arrays["strain_rates"] = rates
            for name, values in response.diagnostics.items():
                arrays[f"diag__{name}"] = values
            meta = {"material": spec, "time_step": dt, "with_rates": with_rates,
                    "active_fraction": float(np.mean(response.diagnostics["viscoplastic_active"]))}  # fmt: skip
            cases[f"j2_{key}_{'rates' if with_rates else 'norates'}"] = (arrays, meta)
    return cases


def make_incremental_case(data_mod, plasticity):
    """The isolated-return-map workload (seeded) through the reference's total-strain API."""
    sys.path.insert(0, str(REPO))
    from oracle.j2vp import config1_inputs, elasticity_matrix

    n = 2048
    inputs = config1_inputs(n, seed=1234)
    spec = MATERIALS["mortar"]
    material = _j2_material(plasticity, spec)
    c = elasticity_matrix(spec["params"]["young_modulus"], spec["params"]["poisson_ratio"])
    strain = inputs["stress"] @ np.linalg.inv(c).T + inputs["plastic_strain"] + inputs["dstrain"]
    state = data_mod.MaterialState({
        "plastic_strain": inputs["plastic_strain"].copy(), "equivalent_plastic_strain": inputs["eqps"].copy(),
        "viscoplastic_multiplier": np.zeros(n)})  # fmt: skip
    request = data_mod.MaterialPointRequest(strain, None, inputs["dt"], "three_dimensional", _settings(data_mod))
    response = material.update(request, state, data_mod.MaterialResponseRequirements(tangent=True))
    arrays = {
        "dstrain": inputs["dstrain"], "stress_n": inputs["stress"], "plastic_strain_n": inputs["plastic_strain"],
        "eqps_n": inputs["eqps"], "stresses": response.stresses, "tangents": response.tangents,
        "plastic_strain": response.state.variables["plastic_strain"],
        "equivalent_plastic_strain": response.state.variables["equivalent_plastic_strain"],
        "viscoplastic_active": response.diagnostics["viscoplastic_active"],
    }  # fmt: skip
    meta = {"material": spec, "time_step": inputs["dt"], "seed": 1234, "n": n,
            "active_fraction": float(np.mean(response.diagnostics["viscoplastic_active"]))}  # fmt: skip
    return {"j2_incremental_config1": (arrays, meta)}


def make_failure_cases(data_mod, plasticity, errors):
    """Failing points: reason strings and diagnostics of MaterialPointConvergenceError."""
    out = {}
    strain = np.asarray([0.004, -0.0015, -0.001, 0.002, -0.003, 0.02])
    base = MATERIALS["test_m2"]
    scenarios = {
        "max_iterations": (dict(base["params"]), _settings(data_mod, 1, 1.0e-10, 1.0e-30, 1.0e-30), strain, 1.0e-3),
        "non_finite_iteration": (dict(base["params"], reference_stress=1.0e-300), _settings(data_mod), strain, 1.0e-3),
        "non_finite_invariant": (dict(base["params"]), _settings(data_mod),
                                 np.asarray([0.0, 0.0, 0.0, 0.0, 0.0, np.nan]), 1.0e-3),
        "activation_tolerance": (dict(base["params"]), _settings(data_mod, 50, -1.0), strain, 1.0e-3),
    }  # fmt: skip
    for key, (params, settings, eps, dt) in scenarios.items():
        material = plasticity.J2ViscoplasticMaterial(name=f"fail_{key}", density=1.0, **params)
        points = np.zeros((3, 6))
        points[1] = eps  # point 1 fails; points 0 and 2 are at rest
        request = data_mod.MaterialPointRequest(points, None, dt, "three_dimensional", settings)
        try:
            material.update(request, material.initialize_state(3))
        except errors.MaterialPointConvergenceError as error:
            out[key] = {"params": params, "settings": list(settings.__dict__.values()), "strain": points.tolist(),
                        "time_step": dt, "reason": error.reason, "message": str(error),
                        "diagnostics": error.diagnostics}  # fmt: skip
        else:
            raise AssertionError(f"scenario {key} did not fail")
    return out


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--reference", default="/root/reference/src")
    args = parser.parse_args()
    _import_reference(args.reference)
    from fem.materials import data as data_mod
    from fem.materials import errors, plasticity

    cases = {}
    cases.update(make_j2_cases(data_mod, plasticity))
    cases.update(make_incremental_case(data_mod, plasticity))
    manifest = {}
    for name, (arrays, meta) in cases.items():
        np.savez_compressed(HERE / f"{name}.npz", **arrays)
        manifest[name] = meta
    failures = make_failure_cases(data_mod, plasticity, errors)
    (HERE / "j2_failures.json").write_text(json.dumps(failures, indent=1, sort_keys=True))
    (HERE / "manifest.json").write_text(json.dumps(manifest, indent=1, sort_keys=True))
    print("wrote", sorted(manifest), "and j2_failures.json")


if __name__ == "__main__":
    main()
