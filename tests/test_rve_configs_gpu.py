"""GPU parity at the benchmarked RVE configurations, against the reference's own runs.

Golden vectors (tests/golden, made by tests/golden/make_golden.py, groups rve_batch and
rve_path) come from the reference's solve_rve_microequilibrium (FP64, direct solves):

* Uneven RVE batch (the 256-RVE workload): the first RVE of each edge 8, 12, 16, 20, 24
  -- its sphere layout (seed = workload index) and its own random macro path (seed
  5000 + index), advanced over time indices 0, 10, 20, 30.  Here the five RVEs are solved
  together in ONE device batch: FP64 element kernels with exact PCG solves within 1e-6
  relative of the reference's homogenised stress, and FP32 element kernels with the
  workload's settings (FP32 Newton tolerances, Eisenstat-Walker inexact PCG solves,
  cluster PCG) within 1e-4.
* Mixed-control uniaxial path of the 8^3 RVE (xx strain to -0.5 % in 100 steps at 10 /s,
  other components at zero macro stress), its first 30 steps (into the viscoplastic
  range), through solve_rve_microequilibrium inside the same outer loop: converged macro
  strains and stresses within 1e-6.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import concrete_impact_b200 as cib
from concrete_impact_b200 import rve as R
from concrete_impact_b200.benchmarks import concrete_rve
from concrete_impact_b200.rve_builders import random_strain_path, solve_mixed_control_step, uniaxial_path
from tests.conftest import golden_names, load_case

pytestmark = pytest.mark.gpu

UPDATE = cib.MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)


def _members():
    cases = [load_case(name) for name in golden_names("rve_batch_edge")]
    return sorted(cases, key=lambda c: c[1]["edge"])


def _batch_stresses(precision: int, linear: R.LinearSolverOptions) -> tuple[np.ndarray, list]:
    """Homogenised stress (steps, R, 6) of the golden members solved as one device batch."""
    cases = _members()
    models = []
    for arrays, meta in cases:
        model = concrete_rve(meta["edge"], meta["layout_seed"], precision)
        assert np.array_equal(model.element_phase_ids, arrays["element_phase"])
        # the golden's inputs are the workload's own path
        times, strains = random_strain_path(meta["path_seed"], 200, 4, 1.0e-2, (1.0, 1000.0))
        ti = np.asarray(meta["time_indices"])
        np.testing.assert_array_equal(strains[ti[1:]], arrays["macro_strain"])
        np.testing.assert_allclose(np.diff(times[ti]), arrays["time_step"], rtol=1e-15)
        models.append(model)
    batch = R.RVEBatch(models, precision=precision, linear_solver=linear)
    newton = models[0].newton_settings
    vol = torch.as_tensor(batch.volumes, device=batch.device)[:, None]
    out, iterations = [], []
    for step in range(cases[0][0]["macro_strain"].shape[0]):
        batch.macro.copy_(torch.as_tensor(np.stack([a["macro_strain"][step] for a, _ in cases]), device=batch.device))
        batch.dt.copy_(torch.as_tensor([a["time_step"][step] for a, _ in cases], device=batch.device))
        res = R.solve_batch_step(batch, newton, UPDATE, False)
        batch.response(batch.batch_struct(UPDATE), batch.w, None, None)
        out.append((batch.sums[:, R.RS_SIGMA : R.RS_SIGMA + 6] / vol).cpu().numpy())
        iterations.append(res.newton_iterations.copy())
        batch.commit()
    return np.asarray(out), iterations


def _max_rel(got: np.ndarray, cases) -> np.ndarray:
    """Per step and RVE: max |error| over the 6 components / max |reference stress|."""
    ref = np.stack([a["macro_stress"] for a, _ in cases], axis=1)  # (steps, R, 6)
    return np.abs(got - ref).max(axis=2) / np.abs(ref).max(axis=2)


def test_uneven_batch_fp64_matches_reference() -> None:
    cases = _members()
    assert [m["edge"] for _, m in cases] == [8, 12, 16, 20, 24]
    got, iterations = _batch_stresses(64, R.LinearSolverOptions(cluster="auto"))
    err = _max_rel(got, cases)
    assert err.max() < 1.0e-6, err
    # the path reaches the viscoplastic regime (the reference's own diagnostics)
    assert max(max(m["active_fraction"]) for _, m in cases) > 0.05
    # Newton iteration counts as the reference's (the PCG solves to 1e-11 relative)
    ref_its = np.asarray([m["newton_iterations"] for _, m in cases]).T
    assert np.abs(np.asarray(iterations) - ref_its).max() <= 1, (iterations, ref_its)


def test_uneven_batch_fp32_workload_settings_match_reference() -> None:
    cases = _members()
    linear = R.LinearSolverOptions(cluster="auto", forcing="eisenstat_walker")
    got, _ = _batch_stresses(32, linear)
    err = _max_rel(got, cases)
    assert err.max() < 1.0e-4, err


def test_mixed_control_path_matches_reference() -> None:
    arrays, meta = load_case("rve_path_uniaxial_8")
    model = concrete_rve(8, 0, 64)
    assert np.array_equal(model.element_phase_ids, arrays["element_phase"])
    cache = R.build_rve_operator_cache(model, linear_solver=R.LinearSolverOptions(cluster=8))

    def solve(request, state):
        return R.solve_rve_microequilibrium(model, request, state, cache)

    times, exx = uniaxial_path(100)
    np.testing.assert_array_equal(times[: meta["steps"] + 1], arrays["times"])
    state = R.initialize_rve_state(model)
    guess = np.zeros(6)
    for step in range(1, meta["steps"] + 1):
        res = solve_mixed_control_step(solve, state, {0: float(exx[step])}, guess, float(times[step] - times[step - 1]),
                                       UPDATE, stress_tolerance=meta["stress_tolerance"])  # fmt: skip
        state, guess = res.response.state, res.macro_strain
        ref_strain, ref_stress = arrays["macro_strain"][step - 1], arrays["macro_stress"][step - 1]
        assert np.abs(res.macro_strain - ref_strain).max() <= 1e-6 * np.abs(ref_strain).max()
        # the free components are zero to the outer tolerance on both sides: compare against
        # the prescribed-component stress scale
        assert np.abs(res.response.macro_stress - ref_stress).max() <= 1e-6 * np.abs(ref_stress).max()
        assert res.outer_iterations == meta["outer_iterations"][step - 1]
