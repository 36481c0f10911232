"""Generate golden vectors by running the reference implementation itself.

Run in a container that holds the reference checkout (read-only); pass its ``src``
directory, or set the environment variable CIB_REFERENCE_SRC:

    python tests/golden/make_golden.py --reference <checkout>/src

The reference imports gmsh, meshio and h5py at module level in files that the material
and RVE paths never execute; empty stand-in modules are put on sys.path for them.  The
outputs are small compressed .npz files in this directory; the GPU box never needs the
reference.
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile
import time
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


def _rve_arrays(prefix: str, response, macro) -> dict:
    out = {f"{prefix}macro_strain": macro, f"{prefix}macro_stress": response.macro_stress,
           f"{prefix}fluctuation": response.state.fluctuation_dofs,
           f"{prefix}micro_stresses": response.micro_stresses,
           f"{prefix}micro_strains": response.micro_strains}  # fmt: skip
    if response.effective_tangent is not None:
        out[f"{prefix}effective_tangent"] = response.effective_tangent
    for name, values in response.state.material_state.variables.items():
        out[f"{prefix}state__{name}"] = values
    for name, values in response.micro_diagnostics.items():
        out[f"{prefix}mdiag__{name}"] = values
    scalars = {k: v for k, v in response.diagnostics.items() if isinstance(v, (int, float))}
    scalars["free_energy_density"] = response.free_energy_density
    scalars["dissipation_density"] = response.dissipation_density
    return out, scalars


# Uneven RVE batch of the 256-RVE workload: per RVE i, edge drawn from EDGES with seed
# 1000 + i, sphere layout seed i, random 4-segment macro path seed 5000 + i (200 steps).
# The golden RVEs are the first workload RVE of each edge, advanced over coarse steps of
# their own paths (time indices 0, 10, 20, 30) so that the mortar yields.
RVE_BATCH_EDGES = (8, 12, 16, 20, 24)
RVE_BATCH_TIME_INDICES = (0, 10, 20, 30)


def rve_batch_golden_members() -> list[tuple[int, int]]:
    """(workload RVE index, edge) of the first RVE of each edge of the 256-RVE workload."""
    found = {}
    for i in range(256):
        edge = int(np.random.default_rng(1000 + i).choice(RVE_BATCH_EDGES))
        found.setdefault(edge, i)
    return [(found[e], e) for e in RVE_BATCH_EDGES]


def make_rve_batch_cases():
    """The reference's solve_rve_microequilibrium (FP64, direct solves) on one RVE of each
    edge of the uneven 256-RVE workload, along its own macro path; homogenised stress and
    Newton iterations per step."""
    from fem.materials.linear_elastic import LinearElasticMaterial
    from fem.materials.phased import PhasedMaterialModel, RVEPhase
    from fem.materials.plasticity import J2ViscoplasticMaterial
    from fem.mesh.structured import build_structured_hex8_box
    from fem.rve import (RVERequest, StructuredHex8RVE, build_structured_hex8_periodic_constraint,
                         initialize_rve_state, solve_rve_microequilibrium)  # fmt: skip
    from fem.solvers.data import ArmijoSettings, NonlinearNewtonSettings
    from fem.materials.data import MaterialUpdateSettings

    sys.path.insert(0, str(REPO))
    from concrete_impact_b200.rve_builders import draw_spheres, random_strain_path, sphere_phase_map

    update = MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)
    mortar = J2ViscoplasticMaterial("mortar", 2200.0, 25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0)
    aggregate = LinearElasticMaterial("aggregate", 2600.0, 50.0e9, 0.2)
    newton = NonlinearNewtonSettings(25, 1.0e-6, 1.0e-8, 1.0e-14, 1.0e-10, ArmijoSettings(enabled=False))
    cases = {}
    for index, edge in rve_batch_golden_members():
        div = (edge, edge, edge)
        nodes, elements = build_structured_hex8_box((1.0, 1.0, 1.0), div)
        phase = sphere_phase_map(div, draw_spheres(index))
        phased = PhasedMaterialModel("mortar__aggregate", (RVEPhase("matrix", mortar), RVEPhase("inclusion", aggregate)),
                                     np.repeat(phase, 8), 2360.0)  # fmt: skip
        model = StructuredHex8RVE(nodes, elements, div, phased, build_structured_hex8_periodic_constraint(nodes, div),
                                  newton, element_phase_ids=phase, phase_names=("matrix", "inclusion"))  # fmt: skip
        times, strains = random_strain_path(5000 + index, 200, 4, 1.0e-2, (1.0, 1000.0))
        ti = np.asarray(RVE_BATCH_TIME_INDICES)
        state = initialize_rve_state(model)
        stress, newton_its, active, eqps = [], [], [], []
        t0 = time.perf_counter()
        for a, b in zip(ti[:-1], ti[1:]):
            response = solve_rve_microequilibrium(model, RVERequest(strains[b], float(times[b] - times[a]), update),
                                                  state)  # fmt: skip
            stress.append(response.macro_stress)
            newton_its.append(int(response.diagnostics["newton_iterations"]))
            active.append(float(response.diagnostics.get("viscoplastic_active_volume_fraction", np.nan)))
            eqps.append(float(np.mean(response.state.material_state.variables["phase_matrix__equivalent_plastic_strain"])))
            state = response.state
        seconds = time.perf_counter() - t0
        print(f"rve_batch edge {edge} (RVE {index}): {seconds:.1f} s", flush=True)
        arrays = {"element_phase": phase.astype(np.uint8), "macro_strain": strains[ti[1:]],
                  "time_step": np.diff(times[ti]), "macro_stress": np.asarray(stress)}  # fmt: skip
        meta = {"kind": "rve_batch_member", "workload_index": index, "edge": edge, "layout_seed": index,
                "path_seed": 5000 + index, "time_indices": list(RVE_BATCH_TIME_INDICES),
                "newton_iterations": newton_its, "mean_matrix_eqps": eqps, "active_fraction": active,
                "newton": [25, 1.0e-6, 1.0e-8, 1.0e-14, 1.0e-10, False], "reference_seconds": seconds}  # fmt: skip
        cases[f"rve_batch_edge{edge}"] = (arrays, meta)
    return cases


def make_rve_path_cases(steps: int = 30):
    """The mixed-control uniaxial compression path of the 8^3 concrete RVE (seed 0): xx
    strain ramped to -0.5 % in 100 steps at 10 /s, the other components free at zero
    macro stress.  The outer iteration is this package's harness loop
    (rve_builders.solve_mixed_control_step, which corrects the free components with the
    effective tangent); every RVE solve inside it is the reference's
    solve_rve_microequilibrium with its effective tangent.  First ``steps`` steps."""
    from fem.materials.data import MaterialResponseRequirements, MaterialUpdateSettings
    from fem.materials.linear_elastic import LinearElasticMaterial
    from fem.materials.phased import PhasedMaterialModel, RVEPhase
    from fem.materials.plasticity import J2ViscoplasticMaterial
    from fem.mesh.structured import build_structured_hex8_box
    from fem.rve import (RVERequest, StructuredHex8RVE, build_structured_hex8_periodic_constraint,
                         initialize_rve_state, solve_rve_microequilibrium)  # fmt: skip
    from fem.solvers.data import ArmijoSettings, NonlinearNewtonSettings

    sys.path.insert(0, str(REPO))
    from concrete_impact_b200.rve_builders import draw_spheres, solve_mixed_control_step, sphere_phase_map, uniaxial_path

    update = MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)
    mortar = J2ViscoplasticMaterial("mortar", 2200.0, 25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0)
    aggregate = LinearElasticMaterial("aggregate", 2600.0, 50.0e9, 0.2)
    newton = NonlinearNewtonSettings(25, 1.0e-6, 1.0e-8, 1.0e-14, 1.0e-10, ArmijoSettings(enabled=False))
    div = (8, 8, 8)
    nodes, elements = build_structured_hex8_box((1.0, 1.0, 1.0), div)
    phase = sphere_phase_map(div, draw_spheres(0))
    phased = PhasedMaterialModel("mortar__aggregate", (RVEPhase("matrix", mortar), RVEPhase("inclusion", aggregate)),
                                 np.repeat(phase, 8), 2360.0)  # fmt: skip
    model = StructuredHex8RVE(nodes, elements, div, phased, build_structured_hex8_periodic_constraint(nodes, div),
                              newton, element_phase_ids=phase, phase_names=("matrix", "inclusion"))  # fmt: skip

    def solve(request, state):
        return solve_rve_microequilibrium(model, RVERequest(np.asarray(request.macro_strain), request.time_step, update,
                                                            MaterialResponseRequirements(tangent=True)), state)  # fmt: skip

    times, exx = uniaxial_path(100)
    state = initialize_rve_state(model)
    guess = np.zeros(6)
    strain, stress, outer = [], [], []
    for step in range(1, steps + 1):
        res = solve_mixed_control_step(solve, state, {0: float(exx[step])}, guess, float(times[step] - times[step - 1]),
                                       update, stress_tolerance=1.0e-6 * 20.0e6)  # fmt: skip
        state = res.response.state
        guess = res.macro_strain
        strain.append(res.macro_strain.copy())
        stress.append(np.asarray(res.response.macro_stress))
        outer.append(int(res.outer_iterations))
    arrays = {"element_phase": phase.astype(np.uint8), "times": times[: steps + 1], "macro_strain": np.asarray(strain),
              "macro_stress": np.asarray(stress)}  # fmt: skip
    meta = {"kind": "mixed_control_path", "divisions": div, "layout_seed": 0, "steps": steps,
            "outer_iterations": outer, "stress_tolerance": 1.0e-6 * 20.0e6,
            "newton": [25, 1.0e-6, 1.0e-8, 1.0e-14, 1.0e-10, False]}  # fmt: skip
    return {"rve_path_uniaxial_8": (arrays, meta)}


def make_rve_cases():
    """RVE solves of the reference on structured periodic boxes (homogeneous and two-phase)."""
    from fem.materials.data import MaterialResponseRequirements
    from fem.materials.linear_elastic import LinearElasticMaterial
    from fem.materials.phased import PhasedMaterialModel, RVEPhase
    from fem.materials.plasticity import J2ViscoplasticMaterial
    from fem.mesh.structured import build_structured_hex8_box
    from fem.rve import (RVERequest, StructuredHex8RVE, build_structured_hex8_periodic_constraint,
                         initialize_rve_state, solve_rve_microequilibrium)  # fmt: skip
    from fem.solvers.data import ArmijoSettings, NonlinearNewtonSettings
    from fem.materials.data import MaterialUpdateSettings

    sys.path.insert(0, str(REPO))
    from concrete_impact_b200.rve_builders import draw_spheres, sphere_phase_map

    cases = {}
    update = MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)
    # (1) homogeneous RVE of the reference unit test (m = 2, Armijo), 4-step path
    mat = J2ViscoplasticMaterial("single_phase_rve_j2", 1.0, 3339.9160679991464, 0.36994096308414537, 10.0, 80.0,
                                 0.02, 10.0, 2.0)  # fmt: skip
    path = [np.asarray([0.002, -0.0005, -0.0005, 0.0, 0.0, 0.01]),
            np.asarray([0.004, -0.0010, -0.0010, 0.002, -0.003, 0.02]),
            np.asarray([0.003, -0.0008, -0.0008, 0.001, -0.002, 0.012]),
            np.asarray([0.0045, -0.0012, -0.0012, -0.001, 0.002, -0.01])]  # fmt: skip
    newton_h = NonlinearNewtonSettings(20, 1.0e-10, 1.0e-10, 1.0e-12, 1.0e-10, ArmijoSettings(enabled=True))
    for div in ((1, 1, 1), (2, 2, 2)):
        nodes, elements = build_structured_hex8_box((1.0, 1.0, 1.0), div)
        model = StructuredHex8RVE(nodes, elements, div, mat, build_structured_hex8_periodic_constraint(nodes, div),
                                  newton_h, hill_mandel_power_scale=10.0)  # fmt: skip
        state = initialize_rve_state(model)
        arrays, meta_steps = {}, []
        for step, macro in enumerate(path):
            response = solve_rve_microequilibrium(model, RVERequest(macro, 1.0e-3, update), state)
            a, sc = _rve_arrays(f"s{step}__", response, macro)
            arrays.update(a)
            meta_steps.append(sc)
            state = response.state
        meta = {"kind": "homogeneous", "divisions": div, "time_step": 1.0e-3, "steps": len(path), "scalars": meta_steps,
                "material": {"params": dict(young_modulus=mat.young_modulus, poisson_ratio=mat.poisson_ratio,
                             yield_stress=mat.yield_stress, hardening_modulus=mat.hardening_modulus,
                             time_scale=mat.time_scale, reference_stress=mat.reference_stress,
                             rate_exponent=mat.rate_exponent)},
                "newton": [20, 1.0e-10, 1.0e-10, 1.0e-12, 1.0e-10, True], "hill_mandel_power_scale": 10.0}  # fmt: skip
        cases[f"rve_homogeneous_{div[0]}"] = (arrays, meta)
    # (2) two-phase concrete RVEs: mortar J2 Perzyna + elastic aggregate, sphere layouts
    mortar = J2ViscoplasticMaterial("mortar", 2200.0, 25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0)
    aggregate = LinearElasticMaterial("aggregate", 2600.0, 50.0e9, 0.2)
    newton_c = NonlinearNewtonSettings(25, 1.0e-6, 1.0e-8, 1.0e-14, 1.0e-10, ArmijoSettings(enabled=False))
    direction = np.asarray([-1.0, 0.22, 0.22, 0.05, -0.03, 0.08])
    for n, seed, amplitudes in ((4, 7, (0.4e-3, 1.2e-3, 2.0e-3)), (8, 0, (0.6e-3, 1.4e-3, 2.2e-3))):
        div = (n, n, n)
        nodes, elements = build_structured_hex8_box((1.0, 1.0, 1.0), div)
        phase = sphere_phase_map(div, draw_spheres(seed))
        phased = PhasedMaterialModel("mortar__aggregate", (RVEPhase("matrix", mortar), RVEPhase("inclusion", aggregate)),
                                     np.repeat(phase, 8), 2360.0)  # fmt: skip
        model = StructuredHex8RVE(nodes, elements, div, phased, build_structured_hex8_periodic_constraint(nodes, div),
                                  newton_c, element_phase_ids=phase, phase_names=("matrix", "inclusion"))  # fmt: skip
        state = initialize_rve_state(model)
        arrays, meta_steps = {"element_phase": phase}, []
        for step, amp in enumerate(amplitudes):
            macro = amp * direction
            response = solve_rve_microequilibrium(
                model, RVERequest(macro, 5.0e-6, update, MaterialResponseRequirements(tangent=True)), state)
            a, sc = _rve_arrays(f"s{step}__", response, macro)
            arrays.update(a)
            meta_steps.append(sc)
            state = response.state
        meta = {"kind": "two_phase", "divisions": div, "seed": seed, "time_step": 5.0e-6, "steps": len(amplitudes),
                "scalars": meta_steps, "newton": [25, 1.0e-6, 1.0e-8, 1.0e-14, 1.0e-10, False],
                "hill_mandel_power_scale": 1.0}  # fmt: skip
        cases[f"rve_two_phase_{n}"] = (arrays, meta)
    return cases


def _newmark_bar(divisions, lengths, material):
    """Duck-typed preprocess bundle of a structured bar: the fields the reference's
    material-dynamics solver reads (mesh_info, shape_function_cache, material)."""
    from types import SimpleNamespace

    import fem.preprocess  # noqa: F401  (import order: fem.quadrature.cache imports fem.preprocess)
    from fem.mesh.structured import build_structured_hex8_box
    from fem.quadrature.cache import precompute_shape_functions

    nodes, elements = build_structured_hex8_box(tuple(lengths), tuple(divisions))
    nn = nodes.shape[0]
    mesh_info = SimpleNamespace(nodes=nodes, elements=elements, element_type="hex8", dimension=3,
                                dof_map=np.arange(3 * nn, dtype=np.int64).reshape(nn, 3))  # fmt: skip
    cache = precompute_shape_functions(mesh_info, SimpleNamespace(quadrature={"order": 2}))
    left = np.flatnonzero(np.isclose(nodes[:, 0], 0.0))
    right = np.flatnonzero(np.isclose(nodes[:, 0], lengths[0]))
    fixed = (3 * left[:, None] + np.arange(3)).ravel()
    # consistent nodal force of a unit pressure on the x = L face (bilinear face, uniform)
    unit = np.zeros(3 * nn)
    ny, nz = divisions[1], divisions[2]
    face = lengths[1] * lengths[2] / (ny * nz)
    for k in range(nz):
        for j in range(ny):
            for dj, dk in ((0, 0), (1, 0), (0, 1), (1, 1)):
                node = divisions[0] + (divisions[0] + 1) * ((j + dj) + (ny + 1) * (k + dk))
                unit[3 * node] -= face / 4.0
    bundle = SimpleNamespace(mesh_info=mesh_info, shape_function_cache=cache, material=material)
    return bundle, nodes, elements, fixed, unit, right


def _newmark_run(bundle, nodes, fixed, unit, amplitude, duration, dt, steps, adaptive, newton_args, armijo):
    import math

    from fem.dynamics.material import solve_material_implicit_newmark
    from fem.materials.data import MaterialUpdateSettings
    from fem.solvers.data import (AdaptiveTimeStepSettings, ArmijoSettings, DirichletDofSet, NonlinearNewtonSettings,
                                  TimeIntegrationSettings)  # fmt: skip

    def load(t):
        return (amplitude * math.sin(math.pi * t / duration) if 0.0 <= t <= duration else 0.0) * unit

    n_dof = 3 * nodes.shape[0]
    sol = solve_material_implicit_newmark(
        bundle, TimeIntegrationSettings("newmark", dt, steps, 0.25, 0.5, 1.0, AdaptiveTimeStepSettings(enabled=adaptive)),
        np.zeros(n_dof), np.zeros(n_dof), DirichletDofSet(fixed, np.zeros(fixed.size)), load, "three_dimensional",
        MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10),
        NonlinearNewtonSettings(*newton_args, ArmijoSettings(enabled=armijo)))  # fmt: skip
    arrays = {name: np.asarray(getattr(sol, name)) for name in (
        "times", "displacement", "velocity", "acceleration", "stresses", "equivalent_plastic_strain",
        "kinetic_energy", "free_energy", "dissipated_energy", "external_work", "energy_residual",
        "newton_iterations", "armijo_backtracks", "accepted_time_steps", "rejected_step_counts")}  # fmt: skip
    arrays["fixed_dofs"] = fixed
    arrays["unit_force"] = unit
    meta = {"amplitude": amplitude, "duration": duration, "time_step": dt, "num_steps": steps, "beta": 0.25,
            "gamma": 0.5, "adaptive": adaptive, "newton": list(newton_args) + [armijo],
            "update_settings": [50, 1.0e-10, 1.0e-12, 1.0e-10], "accepted_steps": int(arrays["times"].size - 1),
            "rejected": int(arrays["rejected_step_counts"].sum()),
            "rejected_reasons": [list(r) for r in sol.rejected_reasons]}  # fmt: skip
    return arrays, meta


def _explicit_run(bundle, nodes, fixed, unit, amplitude, duration, dt, steps):
    import math

    from fem.dynamics.material import solve_material_explicit
    from fem.materials.data import MaterialUpdateSettings
    from fem.solvers.data import DirichletDofSet, TimeIntegrationSettings

    def load(t):
        return (amplitude * math.sin(math.pi * t / duration) if 0.0 <= t <= duration else 0.0) * unit

    n_dof = 3 * nodes.shape[0]
    sol = solve_material_explicit(
        bundle, TimeIntegrationSettings("explicit", dt, steps, 0.0, 0.5, 0.9), np.zeros(n_dof), np.zeros(n_dof),
        DirichletDofSet(fixed, np.zeros(fixed.size)), load, "three_dimensional",
        MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10))  # fmt: skip
    arrays = {name: np.asarray(getattr(sol, name)) for name in (
        "times", "displacement", "velocity", "acceleration", "internal_force", "external_force", "stresses",
        "equivalent_plastic_strain", "kinetic_energy", "free_energy", "dissipated_energy", "external_work",
        "energy_residual", "positive_incremental_work", "negative_incremental_work", "unloading_volume_fraction",
        "viscoplastic_active_volume_fraction", "accepted_time_steps")}  # fmt: skip
    arrays["fixed_dofs"] = fixed
    arrays["unit_force"] = unit
    meta = {"amplitude": amplitude, "duration": duration, "time_step": dt, "num_steps": steps,
            "cfl_safety_factor": 0.9, "update_settings": [50, 1.0e-10, 1.0e-12, 1.0e-10]}  # fmt: skip
    return arrays, meta


def make_explicit_cases():
    """Explicit velocity-Verlet material dynamics of the reference (solve_material_explicit,
    src/fem/dynamics/material.py:89-297) on pressure-pulse bars: J2 Perzyna at the macro
    points (8x1x1 bar, 40 MPa half-sine), and explicit FE2 with a two-phase 4^3 RVE
    (RVEHomogenizedMaterial) at each of the 24 points of a 3x1x1 bar; plus the reference's
    CFL refusal (check_explicit_stability, src/fem/dynamics/stability.py:34-48)."""
    from fem.dynamics.stability import check_explicit_stability
    from fem.materials.linear_elastic import LinearElasticMaterial
    from fem.materials.phased import PhasedMaterialModel, RVEPhase
    from fem.materials.plasticity import J2ViscoplasticMaterial
    from fem.mesh.structured import build_structured_hex8_box
    from fem.rve import StructuredHex8RVE, build_structured_hex8_periodic_constraint
    from fem.rve.material import RVEHomogenizedMaterial
    from fem.solvers.data import ArmijoSettings, NonlinearNewtonSettings, TimeIntegrationSettings

    sys.path.insert(0, str(REPO))
    from concrete_impact_b200.rve_builders import draw_spheres, sphere_phase_map

    cases = {}
    mortar = J2ViscoplasticMaterial("mortar", 2200.0, 25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0)
    bar = {"divisions": (8, 1, 1), "lengths": (0.08, 0.01, 0.01)}
    bundle, nodes, elements, fixed, unit, _ = _newmark_bar(bar["divisions"], bar["lengths"], mortar)
    report = check_explicit_stability(bundle, TimeIntegrationSettings("explicit", 1.0e-6, 1, 0.0, 0.5, 0.9))
    arrays, meta = _explicit_run(bundle, nodes, fixed, unit, 40.0e6, 20.0e-6, 1.0e-6, 60)
    meta.update(bar=bar, material=MATERIALS["mortar"], stable_time_step=report.stable_time_step,
                minimum_length=report.minimum_length, maximum_wave_speed=report.maximum_wave_speed)  # fmt: skip
    try:
        check_explicit_stability(bundle, TimeIntegrationSettings("explicit", 1.0e-5, 1, 0.0, 0.5, 0.9))
        raise AssertionError("the reference accepted a step above its CFL bound")
    except ValueError as error:
        meta["cfl_violation"] = {"time_step": 1.0e-5, "message": str(error)}
    cases["explicit_j2_bar"] = (arrays, meta)
    aggregate = LinearElasticMaterial("aggregate", 2600.0, 50.0e9, 0.2)
    div = (4, 4, 4)
    rnodes, relements = build_structured_hex8_box((1.0, 1.0, 1.0), div)
    phase = sphere_phase_map(div, draw_spheres(7))
    frac = float(phase.mean())
    density = 2200.0 * (1.0 - frac) + 2600.0 * frac
    phased = PhasedMaterialModel("mortar__aggregate", (RVEPhase("matrix", mortar), RVEPhase("inclusion", aggregate)),
                                 np.repeat(phase, 8), density)  # fmt: skip
    rve_newton = NonlinearNewtonSettings(25, 1.0e-6, 1.0e-8, 1.0e-14, 1.0e-10, ArmijoSettings(enabled=False))
    model = StructuredHex8RVE(rnodes, relements, div, phased, build_structured_hex8_periodic_constraint(rnodes, div),
                              rve_newton, element_phase_ids=phase, phase_names=("matrix", "inclusion"))  # fmt: skip
    fe2_bar = {"divisions": (3, 1, 1), "lengths": (0.03, 0.01, 0.01)}
    material = RVEHomogenizedMaterial(model, "two_phase_rve")
    bundle, nodes, elements, fixed, unit, _ = _newmark_bar(fe2_bar["divisions"], fe2_bar["lengths"], material)
    report = check_explicit_stability(bundle, TimeIntegrationSettings("explicit", 1.0e-6, 1, 0.0, 0.5, 0.9))
    arrays, meta = _explicit_run(bundle, nodes, fixed, unit, 40.0e6, 10.0e-6, 1.0e-6, 12)
    arrays["element_phase"] = phase
    meta.update(bar=fe2_bar, stable_time_step=report.stable_time_step,
                rve={"divisions": div, "seed": 7, "density": density,
                     "newton": [25, 1.0e-6, 1.0e-8, 1.0e-14, 1.0e-10, False]})  # fmt: skip
    cases["explicit_fe2_bar"] = (arrays, meta)
    return cases


def make_newmark_cases():
    """Implicit Newmark material dynamics of the reference (solve_material_implicit_newmark)
    on small pressure-pulse bars: J2 Perzyna at the macro points (fixed steps; adaptive
    steps with Armijo and a two-iteration Newton budget that forces cutbacks), and FE2 with
    a two-phase 4^3 RVE (RVEHomogenizedMaterial) at every macro point."""
    from fem.materials.linear_elastic import LinearElasticMaterial
    from fem.materials.phased import PhasedMaterialModel, RVEPhase
    from fem.materials.plasticity import J2ViscoplasticMaterial
    from fem.mesh.structured import build_structured_hex8_box
    from fem.rve import StructuredHex8RVE, build_structured_hex8_periodic_constraint
    from fem.rve.material import RVEHomogenizedMaterial
    from fem.solvers.data import ArmijoSettings, NonlinearNewtonSettings

    sys.path.insert(0, str(REPO))
    from concrete_impact_b200.rve_builders import draw_spheres, sphere_phase_map

    cases = {}
    mortar = J2ViscoplasticMaterial("mortar", 2200.0, 25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0)
    bar = {"divisions": (6, 1, 1), "lengths": (0.06, 0.01, 0.01)}
    bundle, nodes, elements, fixed, unit, _ = _newmark_bar(bar["divisions"], bar["lengths"], mortar)
    runs = {
        "newmark_j2_bar_fixed": dict(dt=2.0e-6, steps=20, adaptive=False, newton=(20, 1.0e-6, 1.0e-10, 1.0e-14, 1.0e-10),
                                     armijo=False),
        "newmark_j2_bar_adaptive": dict(dt=4.0e-6, steps=10, adaptive=True, newton=(2, 1.0e-6, 1.0e-10, 1.0e-14, 1.0e-10),
                                        armijo=True),
    }  # fmt: skip
    for name, run in runs.items():
        arrays, meta = _newmark_run(bundle, nodes, fixed, unit, 40.0e6, 20.0e-6, run["dt"], run["steps"],
                                    run["adaptive"], run["newton"], run["armijo"])  # fmt: skip
        meta.update(bar=bar, material=MATERIALS["mortar"])
        cases[name] = (arrays, meta)
    # FE2: the same bar geometry in 3 elements, a two-phase 4^3 RVE at each of the 24 points
    aggregate = LinearElasticMaterial("aggregate", 2600.0, 50.0e9, 0.2)
    div = (4, 4, 4)
    rnodes, relements = build_structured_hex8_box((1.0, 1.0, 1.0), div)
    phase = sphere_phase_map(div, draw_spheres(7))
    frac = float(phase.mean())
    density = 2200.0 * (1.0 - frac) + 2600.0 * frac
    phased = PhasedMaterialModel("mortar__aggregate", (RVEPhase("matrix", mortar), RVEPhase("inclusion", aggregate)),
                                 np.repeat(phase, 8), density)  # fmt: skip
    rve_newton = NonlinearNewtonSettings(25, 1.0e-6, 1.0e-8, 1.0e-14, 1.0e-10, ArmijoSettings(enabled=False))
    model = StructuredHex8RVE(rnodes, relements, div, phased, build_structured_hex8_periodic_constraint(rnodes, div),
                              rve_newton, element_phase_ids=phase, phase_names=("matrix", "inclusion"))  # fmt: skip
    fe2_bar = {"divisions": (3, 1, 1), "lengths": (0.03, 0.01, 0.01)}
    material = RVEHomogenizedMaterial(model, "two_phase_rve")
    bundle, nodes, elements, fixed, unit, _ = _newmark_bar(fe2_bar["divisions"], fe2_bar["lengths"], material)
    arrays, meta = _newmark_run(bundle, nodes, fixed, unit, 40.0e6, 10.0e-6, 2.0e-6, 8, False,
                                (20, 1.0e-6, 1.0e-10, 1.0e-14, 1.0e-10), False)  # fmt: skip
    arrays["element_phase"] = phase
    meta.update(bar=fe2_bar, rve={"divisions": div, "seed": 7, "density": density,
                                  "newton": [25, 1.0e-6, 1.0e-8, 1.0e-14, 1.0e-10, False]})  # fmt: skip
    cases["newmark_fe2_bar"] = (arrays, meta)
    return cases


def make_ogrid_cases():
    """The reference's cylindrical O-grid RVE (build_cylindrical_ogrid_hex8,
    build_cylindrical_two_phase_rve): the mesh and its periodic topology, and three RVE
    solves along a compression path with effective tangents (mortar J2 matrix, elastic
    cylindrical inclusion)."""
    from fem.materials.data import MaterialResponseRequirements, MaterialUpdateSettings
    from fem.materials.linear_elastic import LinearElasticMaterial
    from fem.materials.plasticity import J2ViscoplasticMaterial
    from fem.mesh.structured import build_cylindrical_ogrid_hex8
    from fem.rve import RVERequest, initialize_rve_state, solve_rve_microequilibrium
    from fem.rve.builders import build_cylindrical_two_phase_rve
    from fem.solvers.data import ArmijoSettings, NonlinearNewtonSettings

    spec = {"lengths": (1.0, 1.0, 0.5), "inclusion_volume_fraction": 0.3, "circumferential_divisions": 8,
            "matrix_radial_divisions": 2, "axial_divisions": 2}  # fmt: skip
    mesh = build_cylindrical_ogrid_hex8(spec["lengths"], spec["inclusion_volume_fraction"],
                                       spec["circumferential_divisions"], spec["matrix_radial_divisions"],
                                       spec["axial_divisions"])  # fmt: skip
    arrays = {"nodes": mesh.nodes, "elements": mesh.elements, "element_phase_ids": mesh.element_phase_ids,
              "periodic_class_ids": mesh.periodic_class_ids}  # fmt: skip
    for axis, (minus, plus) in zip("xyz", mesh.opposite_face_nodes):
        arrays[f"face_{axis}_minus"] = np.asarray(minus)
        arrays[f"face_{axis}_plus"] = np.asarray(plus)
    mortar = J2ViscoplasticMaterial("mortar", 2200.0, 25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0)
    aggregate = LinearElasticMaterial("aggregate", 2600.0, 50.0e9, 0.2)
    newton = NonlinearNewtonSettings(25, 1.0e-6, 1.0e-8, 1.0e-14, 1.0e-10, ArmijoSettings(enabled=False))
    model = build_cylindrical_two_phase_rve(mesh, mortar, aggregate, newton, 1.0)
    update = MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)
    state = initialize_rve_state(model)
    direction = np.asarray([-1.0, 0.22, 0.22, 0.05, -0.03, 0.08])
    amplitudes = (0.6e-3, 1.4e-3, 2.2e-3)
    scalars = []
    for step, amp in enumerate(amplitudes):
        macro = amp * direction
        response = solve_rve_microequilibrium(
            model, RVERequest(macro, 5.0e-6, update, MaterialResponseRequirements(tangent=True)), state)
        a, sc = _rve_arrays(f"s{step}__", response, macro)
        a[f"s{step}__displacement"] = response.displacement
        arrays.update(a)
        scalars.append(sc)
        state = response.state
    meta = {"mesh": spec, "analytic_inclusion_area": mesh.analytic_inclusion_area,
            "discrete_inclusion_area": mesh.discrete_inclusion_area, "time_step": 5.0e-6, "steps": len(amplitudes),
            "amplitudes": list(amplitudes), "direction": direction.tolist(), "scalars": scalars,
            "newton": [25, 1.0e-6, 1.0e-8, 1.0e-14, 1.0e-10, False], "hill_mandel_power_scale": 1.0,
            "effective_density": float(model.material.density)}  # fmt: skip
    return {"rve_ogrid_cylinder": (arrays, meta)}


def make_rno_energy_cases(src: str):
    """The reference's trained energy-based RVE-RNO (artifacts/rve_rno/c48_v2_liu_direct):
    its weights, energy anchors and a 12-step rollout of update_batch (FP32, CPU) for 128
    points along seeded linear strain ramps, with the trained integrator
    (current_state_stress_forward_euler) and, on the last step's inputs, the
    cs_semi_implicit_forward_euler branch."""
    import torch

    from concrete_impact.nn.config import RVERNOModelConfig
    from concrete_impact.nn.models.rve_rno import EnergyDissipationRVERNO

    artifact = Path(src).parent / "artifacts" / "rve_rno" / "c48_v2_liu_direct"
    metadata = json.loads((artifact / "artifact_metadata.json").read_text())
    fields = ("integrator", "evolution", "reference_time_scale", "latent_dimension", "hidden_size", "hidden_layers",
              "activation", "time_representation", "dtype")  # fmt: skip
    spec = {k: metadata[k] for k in fields}
    spec.update(family=metadata["model_family"], device="cpu")
    state_dict = torch.load(artifact / "best_model.pt", map_location="cpu", weights_only=True)["model_state_dict"]
    models = {}
    for integrator in ("current_state_stress_forward_euler", "cs_semi_implicit_forward_euler"):
        model = EnergyDissipationRVERNO(RVERNOModelConfig(**dict(spec, integrator=integrator)))
        model.load_state_dict(state_dict, strict=True)
        model.eval()
        models[integrator] = model
    rng = np.random.default_rng(91000)
    n, steps = 128, 12
    norm = metadata["normalization"]["macro_strain"]
    target = np.asarray(norm["mean"]) + np.asarray(norm["rms_scale"]) * rng.standard_normal((n, 6))
    dt = np.exp(rng.uniform(np.log(1.0e-4), np.log(2.0e-3), size=n))
    arrays = {f"w__{k}": v.numpy() for k, v in state_dict.items()}
    main = models["current_state_stress_forward_euler"]
    anchors = main.prepare_energy_anchors()
    arrays.update(anchor_equilibrium_value=anchors.equilibrium_value.detach().numpy(),
                  anchor_equilibrium_gradient=anchors.equilibrium_strain_gradient.detach().numpy(),
                  anchor_nonequilibrium_value=anchors.nonequilibrium_value.detach().numpy(),
                  anchor_nonequilibrium_gradient=anchors.nonequilibrium_strain_gradient.detach().numpy())  # fmt: skip
    latent = torch.zeros((n, 6), dtype=torch.float32)
    keys = ("stress", "latent_state", "state_rate", "dimensionless_state_rate", "dissipation", "free_energy",
            "thermodynamic_violation", "nonequilibrium_energy_increment")  # fmt: skip
    out = {k: [] for k in keys}
    strains, latents_in, semi = [], [], {k: [] for k in keys}
    with torch.no_grad():
        for step in range(1, steps + 1):
            strain = torch.as_tensor(target * step / steps, dtype=torch.float32)
            time_step = torch.as_tensor(dt, dtype=torch.float32)
            strains.append(strain.numpy())
            latents_in.append(latent.numpy())
            res = main.update_batch(strain, latent, time_step, anchors)
            for k in keys:
                out[k].append(getattr(res, k).numpy())
            if step == steps:  # the other integrator on the last step's inputs
                other = models["cs_semi_implicit_forward_euler"].update_batch(strain, latent, time_step, anchors)
                for k in keys:
                    semi[k].append(getattr(other, k).numpy())
                with torch.enable_grad():  # the algorithmic tangent (autograd) of 16 points
                    tan = main.update_batch(strain[:16], latent[:16], time_step[:16], anchors, compute_tangent=True)
                    arrays["tangent_last16"] = tan.tangent.detach().numpy()
            latent = res.latent_state
    arrays.update(strain=np.stack(strains), latent_in=np.stack(latents_in), time_step=dt.astype(np.float32))
    arrays.update({f"out__{k}": np.stack(v) for k, v in out.items()})
    arrays.update({f"semi__{k}": np.stack(v) for k, v in semi.items()})
    meta = {"model": spec, "points": n, "steps": steps, "seed": 91000, "artifact": "artifacts/rve_rno/c48_v2_liu_direct",
            "accepted_time_step_range": metadata["accepted_time_step_range"]}  # fmt: skip
    return {"rno_energy_c48": (arrays, meta)}


GROUPS = ("j2", "rve", "newmark", "ogrid", "rno_energy", "rve_batch", "rve_path", "explicit")


def main() -> None:
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--reference", default=os.environ.get("CIB_REFERENCE_SRC"),
                        help="the reference checkout's src directory (default: $CIB_REFERENCE_SRC)")
    parser.add_argument("--only", choices=GROUPS, action="append",
                        help="regenerate only these groups (default: all); the manifest keeps the other entries")
    args = parser.parse_args()
    if not args.reference:
        parser.error("give --reference <checkout>/src or set CIB_REFERENCE_SRC")
    groups = set(args.only or GROUPS)
    _import_reference(args.reference)
    from fem.materials import data as data_mod
    from fem.materials import errors, plasticity

    cases = {}
    if "j2" in groups:
        cases.update(make_j2_cases(data_mod, plasticity))
        cases.update(make_incremental_case(data_mod, plasticity))
    if "rve" in groups:
        cases.update(make_rve_cases())
    if "newmark" in groups:
        cases.update(make_newmark_cases())
    if "ogrid" in groups:
        cases.update(make_ogrid_cases())
    if "rno_energy" in groups:
        cases.update(make_rno_energy_cases(args.reference))
    if "rve_batch" in groups:
        cases.update(make_rve_batch_cases())
    if "rve_path" in groups:
        cases.update(make_rve_path_cases())
    if "explicit" in groups:
        cases.update(make_explicit_cases())
    path = HERE / "manifest.json"
    manifest = json.loads(path.read_text()) if path.exists() and args.only else {}
    for name, (arrays, meta) in cases.items():
        np.savez_compressed(HERE / f"{name}.npz", **arrays)
        manifest[name] = json.loads(json.dumps(meta, default=lambda o: o.tolist() if hasattr(o, "tolist") else str(o)))
    if "j2" in groups:
        failures = make_failure_cases(data_mod, plasticity, errors)
        (HERE / "j2_failures.json").write_text(json.dumps(failures, indent=1, sort_keys=True))
    path.write_text(json.dumps(manifest, indent=1, sort_keys=True))
    print("wrote", sorted(cases))


if __name__ == "__main__":
    main()
