"""GPU tests of the cluster PCG (cib_rve_pcg_cluster): 2, 4 or 8 CTAs of one thread-block
cluster share each RVE's reduced system; the solution must equal the one-CTA solve up to
the reordering of its dot products, for uneven batches in both element precisions."""

from __future__ import annotations

import numpy as np
import pytest
import torch

import concrete_impact_b200 as cib
from concrete_impact_b200 import rve as R
from concrete_impact_b200.rve_builders import build_two_phase_sphere_rve, config0_materials, default_newton, fp32_newton

pytestmark = pytest.mark.gpu

UPDATE = cib.MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)


def _models(edges, precision):
    mortar, aggregate = config0_materials()
    newton = default_newton() if precision == 64 else fp32_newton()
    return [build_two_phase_sphere_rve((e, e, e), mortar, aggregate, newton, seed=i) for i, e in enumerate(edges)]


def _solve(models, precision, cluster, strains, dt=5.0e-6):
    batch = R.RVEBatch(models, precision=precision, linear_solver=R.LinearSolverOptions(cluster=cluster))
    batch.macro.copy_(torch.as_tensor(strains, device=batch.device))
    batch.dt.fill_(dt)
    res = R.solve_batch_step(batch, models[0].newton_settings, UPDATE, False)
    batch.response(batch.batch_struct(UPDATE), batch.w, None, None)
    stress = (batch.sums[:, R.RS_SIGMA : R.RS_SIGMA + 6] / torch.as_tensor(batch.volumes, device=batch.device)[:, None])
    return stress.cpu().numpy(), res, batch


@pytest.mark.parametrize("precision,tol", [(64, 1e-9), (32, 2e-5)])
def test_cluster_pcg_matches_one_cta(precision: int, tol: float) -> None:
    edges = [8, 12, 16, 8, 9]
    models = _models(edges, precision)
    strains = np.random.default_rng(3).normal(0.0, 1.5e-3, size=(len(edges), 6))
    ref, res_ref, _ = _solve(models, precision, 1, strains)
    for cluster in (2, 4, 8):
        got, res, batch = _solve(models, precision, cluster, strains)
        assert batch.cluster == cluster
        scale = np.abs(ref).max(axis=1, keepdims=True)
        assert np.all(np.abs(got - ref) <= tol * scale), (cluster, np.abs(got - ref).max())
        assert np.all(np.abs(res.newton_iterations - res_ref.newton_iterations) <= 1)
        # PCG iteration counts only move by the roundoff of the reordered dot products (in
        # FP32 the solve ends near the operator's roundoff floor, where the count of a single
        # system is sensitive to the last bits; the total over the batch stays close)
        got_its, ref_its = res.pcg_iterations, res_ref.pcg_iterations
        slack = 2 + 0.02 * ref_its if precision == 64 else 10 + 0.5 * ref_its
        assert np.all(np.abs(got_its - ref_its) <= slack), (cluster, got_its.tolist(), ref_its.tolist())
        if precision == 32:
            assert abs(int(got_its.sum()) - int(ref_its.sum())) <= 0.15 * int(ref_its.sum()), (cluster, got_its, ref_its)


def test_cluster_pcg_is_deterministic_and_rejects_thin_rves() -> None:
    models = _models([8, 12], 64)
    strains = np.random.default_rng(4).normal(0.0, 1.0e-3, size=(2, 6))
    a, _, _ = _solve(models, 64, 8, strains)
    b, _, _ = _solve(models, 64, 8, strains)
    assert np.array_equal(a, b)
    with pytest.raises(ValueError, match="element layers"):
        R.RVEBatch(_models([4], 64), precision=64, linear_solver=R.LinearSolverOptions(cluster=8))


def test_auto_and_tuned_cluster_choice() -> None:
    models = _models([8, 24], 32)
    batch = R.RVEBatch(models, precision=32, linear_solver=R.LinearSolverOptions(cluster="auto"))
    assert batch.cluster == 8  # 24^3 = 13,824 elements, smallest nz 8
    small = R.RVEBatch(_models([8, 8], 32), precision=32, linear_solver=R.LinearSolverOptions(cluster="auto"))
    assert small.cluster == 1
    batch.macro.copy_(torch.full((2, 6), 1.0e-3, dtype=torch.float64, device=batch.device))
    batch.dt.fill_(5.0e-6)
    out = R.tune_pcg_cluster(batch, UPDATE, persist=False)
    expected = {"1/0"} | {f"{c}/{s}" for c in (2, 4, 8) for s in range(4)}
    assert set(out["ms"]) == expected and f"{out['cluster']}/{out['shape']}" in out["ms"]
    assert (batch.cluster, batch.pcg_shape) == (out["cluster"], out["shape"])


def test_pcg_launch_shapes_agree(tmp_path, monkeypatch) -> None:
    """Every launch shape of the cluster PCG solves the same systems (same iteration
    counts up to the rounding of the CTA sums, solutions within 1e-9); the tuner's choice
    is persisted per edge mix and reused without timing."""
    models = _models([8, 16], 64)
    batch = R.RVEBatch(models, precision=64, linear_solver=R.LinearSolverOptions(cluster=4))
    batch.macro.copy_(torch.full((2, 6), 1.0e-3, dtype=torch.float64, device=batch.device))
    batch.dt.fill_(5.0e-6)
    b = batch.batch_struct(UPDATE)
    batch.residual(b, batch.w, None, None)
    sols = []
    for shape in range(4):
        batch.pcg_shape = shape
        batch.x.zero_()
        batch.pcg(b, batch.res, batch.x, batch.r, batch.p, batch.Ap, batch.nrve, batch.sys_rve, batch.sys_off,
                  batch.pcg_status, batch.pcg_iters, batch.pcg_rel, batch.pcg_xnorm)  # fmt: skip
        torch.cuda.synchronize()
        assert torch.all(batch.pcg_status == 0)
        sols.append((batch.x.cpu().numpy(), batch.pcg_iters.cpu().numpy()))
    for x, its in sols[1:]:
        np.testing.assert_allclose(x, sols[0][0], rtol=1e-9, atol=1e-9 * np.abs(sols[0][0]).max())
        assert np.abs(its - sols[0][1]).max() <= 2
    monkeypatch.setenv("CIB_TUNING_CACHE", str(tmp_path / "tuning.json"))
    first = R.tune_pcg_cluster(batch, UPDATE)
    assert not first["cached"] and (tmp_path / "tuning.json").exists()
    again = R.tune_pcg_cluster(R.RVEBatch(models, precision=64), UPDATE)
    assert again["cached"] and (again["cluster"], again["shape"]) == (first["cluster"], first["shape"])


def test_saved_state_resumes_bitwise(tmp_path) -> None:
    models = _models([8, 12], 64)
    strains = np.random.default_rng(5).normal(0.0, 1.5e-3, size=(2, 6))
    a = R.RVEBatch(models, precision=64)
    a.macro.copy_(torch.as_tensor(strains, device=a.device))
    a.dt.fill_(5.0e-6)
    R.solve_batch_step(a, models[0].newton_settings, UPDATE, False)
    a.commit()
    a.save_state(tmp_path / "rve_state.npz")
    b = R.RVEBatch(models, precision=64)
    b.load_state(tmp_path / "rve_state.npz")
    for batch in (a, b):
        batch.macro.copy_(torch.as_tensor(2.0 * strains, device=batch.device))
        batch.dt.fill_(5.0e-6)
        R.solve_batch_step(batch, models[0].newton_settings, UPDATE, False)
        batch.response(batch.batch_struct(UPDATE), batch.w, None, None)
    assert torch.equal(a.sums, b.sums) and torch.equal(a.w, b.w)
    with pytest.raises(ValueError, match="layout"):
        R.RVEBatch(_models([8], 64), precision=64).load_state(tmp_path / "rve_state.npz")


@pytest.mark.parametrize("precision,tol", [(64, 1e-6), (32, 1e-4)])
def test_inexact_newton_forcing_reaches_the_same_state(precision: int, tol: float) -> None:
    """Eisenstat-Walker PCG tolerances: the Newton convergence tests are unchanged, so the
    homogenised stress agrees within the parity tolerances, with fewer PCG iterations."""
    edges = [8, 12, 16, 8]
    models = _models(edges, precision)
    strains = np.random.default_rng(6).normal(0.0, 1.5e-3, size=(len(edges), 6))
    out = {}
    for forcing in (None, "eisenstat_walker"):
        batch = R.RVEBatch(models, precision=precision, linear_solver=R.LinearSolverOptions(forcing=forcing))
        batch.macro.copy_(torch.as_tensor(strains, device=batch.device))
        batch.dt.fill_(5.0e-6)
        res = R.solve_batch_step(batch, models[0].newton_settings, UPDATE, False)
        batch.response(batch.batch_struct(UPDATE), batch.w, None, None)
        vol = torch.as_tensor(batch.volumes, device=batch.device)[:, None]
        out[forcing] = ((batch.sums[:, R.RS_SIGMA : R.RS_SIGMA + 6] / vol).cpu().numpy(), res)
    ref, res_ref = out[None]
    got, res = out["eisenstat_walker"]
    assert np.all(np.abs(got - ref) <= tol * np.abs(ref).max(axis=1, keepdims=True))
    assert res.pcg_iterations.sum() < res_ref.pcg_iterations.sum()
