"""GPU: the device-controlled batched Newton solve (one CUDA graph per step, decisions on
the device) against the host-driven Newton loop of rve.solve_batch_step.

Both run the same kernels on the same inputs and take the same decisions, so the Newton
and PCG iteration counts are equal and the converged states agree to rounding (1e-12
relative on the homogenised stress and the fluctuation; they are normally bitwise equal).
Covered: an uneven FP64 batch with exact PCG solves, an uneven FP32 batch with the
Eisenstat-Walker inexact solves, a live mask, and the maximum-iterations error.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import concrete_impact_b200 as cib
from concrete_impact_b200 import rve as R
from concrete_impact_b200.benchmarks import concrete_rve
from concrete_impact_b200.rve_builders import random_strain_path

pytestmark = pytest.mark.gpu

UPDATE = cib.MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)
EDGES = (8, 4, 12, 6, 8)


def _run(precision: int, device_control: bool, forcing=None, steps=(0, 8, 16, 24), live=None, newton=None):
    models = [concrete_rve(e, 30 + i, precision) for i, e in enumerate(EDGES)]
    batch = R.RVEBatch(models, precision=precision, linear_solver=R.LinearSolverOptions(cluster="auto", forcing=forcing),
                       device_control=device_control)  # fmt: skip
    newton = newton or models[0].newton_settings
    paths = [random_strain_path(7000 + i, 40, 3, 8.0e-3, (10.0, 100.0)) for i in range(len(models))]
    vol = torch.as_tensor(batch.volumes, device=batch.device)[:, None]
    out = []
    for a, b in zip(steps[:-1], steps[1:]):
        batch.macro.copy_(torch.as_tensor(np.stack([p[1][b] for p in paths]), device=batch.device))
        batch.dt.copy_(torch.as_tensor([p[0][b] - p[0][a] for p in paths], device=batch.device))
        res = R.solve_batch_step(batch, newton, UPDATE, False, live_mask=live)
        batch.response(batch.batch_struct(UPDATE), batch.w, None, None)
        out.append({"its": res.newton_iterations.copy(), "pcg": res.pcg_iterations.copy(),
                    "res": res.residual_norm.copy(), "tol": res.residual_tolerance.copy(),
                    "sigma": (batch.sums[:, R.RS_SIGMA : R.RS_SIGMA + 6] / vol).cpu().numpy(),
                    "w": batch.w.cpu().numpy(), "active": batch.active.cpu().numpy()})  # fmt: skip
        batch.commit()
    return out


def _compare(host, dev) -> None:
    for h, d in zip(host, dev):
        np.testing.assert_array_equal(d["its"], h["its"])
        np.testing.assert_array_equal(d["pcg"], h["pcg"])
        np.testing.assert_array_equal(d["active"], h["active"])
        np.testing.assert_allclose(d["sigma"], h["sigma"], rtol=1e-12, atol=1e-12 * np.abs(h["sigma"]).max())
        np.testing.assert_allclose(d["w"], h["w"], rtol=1e-12, atol=1e-12 * np.abs(h["w"]).max())
        np.testing.assert_allclose(d["res"], h["res"], rtol=1e-10, atol=1e-12 * max(np.abs(h["res"]).max(), 1e-300))
        np.testing.assert_allclose(d["tol"], h["tol"], rtol=1e-12)


def test_graph_newton_matches_host_loop_fp64() -> None:
    host, dev = _run(64, False), _run(64, True)
    assert max(int(h["its"].max()) for h in host) >= 2  # the steps are nonlinear
    _compare(host, dev)


def test_graph_newton_matches_host_loop_fp32_inexact() -> None:
    _compare(_run(32, False, "eisenstat_walker"), _run(32, True, "eisenstat_walker"))


def test_graph_newton_respects_the_live_mask() -> None:
    live = np.array([True, False, True, True, False])
    host, dev = _run(64, False, live=live, steps=(0, 10, 20)), _run(64, True, live=live, steps=(0, 10, 20))
    _compare(host, dev)
    assert np.all(dev[-1]["its"][~live] == 0)


def test_graph_newton_raises_the_host_loops_maximum_iterations_error() -> None:
    tight = R.NonlinearNewtonSettings(1, 1.0e-6, 1.0e-14, 1.0e-20, 1.0e-16, R.ArmijoSettings(enabled=False))
    errors = []
    for device_control in (False, True):
        with pytest.raises(R.RVEEquilibriumError) as info:
            _run(64, device_control, steps=(0, 16), newton=tight)
        errors.append(info.value)
    assert errors[0].reason == errors[1].reason == "maximum_iterations_exceeded"
    assert errors[0].diagnostics["rve_index"] == errors[1].diagnostics["rve_index"]
    assert errors[0].diagnostics["iteration"] == errors[1].diagnostics["iteration"]


@pytest.mark.parametrize("device_control", [False, True])
def test_live_prefix_view_equals_a_batch_of_those_rves(device_control: bool) -> None:
    """A live mask that covers the first RVEs launches the kernels over that prefix of the
    batch; the states of those RVEs must be those of a batch holding only them (the
    Gauss-point arrays keep the whole batch's stride)."""
    models = [concrete_rve(e, 30 + i, 64) for i, e in enumerate(EDGES)]
    paths = [random_strain_path(7000 + i, 40, 3, 8.0e-3, (10.0, 100.0)) for i in range(len(models))]
    live = np.array([True, True, True, False, False])
    results = []
    for subset, mask in ((models[:3], None), (models, live)):
        batch = R.RVEBatch(subset, precision=64, linear_solver=R.LinearSolverOptions(cluster=4),
                           device_control=device_control)  # fmt: skip
        n = len(subset)
        vol = torch.as_tensor(batch.volumes, device=batch.device)[:, None]
        out = []
        for a, b in ((0, 8), (8, 16)):
            batch.macro.copy_(torch.as_tensor(np.stack([p[1][b] for p in paths[:n]]), device=batch.device))
            batch.dt.copy_(torch.as_tensor([p[0][b] - p[0][a] for p in paths[:n]], device=batch.device))
            R.solve_batch_step(batch, batch.models[0].newton_settings, UPDATE, False, live_mask=mask)
            batch.response(batch.batch_struct(UPDATE), batch.w, None, None)
            out.append((batch.sums[:3, R.RS_SIGMA : R.RS_SIGMA + 6] / vol[:3]).cpu().numpy())
            batch.commit()
        results.append(np.asarray(out))
    np.testing.assert_allclose(results[1], results[0], rtol=1e-12, atol=1e-12 * np.abs(results[0]).max())
