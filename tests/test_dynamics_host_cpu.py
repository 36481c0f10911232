"""CPU test of the host logic of concrete_impact_b200.dynamics (Newton loop, Armijo, step
control, energy and field histories) against the reference's golden implicit Newmark runs.

The device pieces are replaced by CPU stand-ins with the same interface: the macro
operators (consistent mass in the tangent's CSR pattern, Newmark kinematics and residual,
the effective-tangent solve, here a direct solve) and the Hex8 material assembly (the
oracle's J2 points).  What remains is exactly the driver code that runs on the GPU path,
so its decisions -- accepted times, cutbacks, Newton and Armijo counts, histories -- are
checked here without a GPU.
"""

from __future__ import annotations

import math
from types import SimpleNamespace

import numpy as np
import pytest
import torch
from scipy.sparse import coo_matrix, csr_matrix
from scipy.sparse.linalg import spsolve

import concrete_impact_b200.dynamics as D
from concrete_impact_b200.assembly import NonlinearSolidAssemblyResult
from concrete_impact_b200.materials import MaterialState, MaterialUpdateSettings
from concrete_impact_b200.rve import ArmijoSettings, NonlinearNewtonSettings
from conftest import load_case
from oracle import j2vp as oj
from oracle import newmark as on
from oracle.rve import box_mesh


class HostOperators:
    """CPU stand-in for dynamics.MacroOperators (float64 torch tensors on the host)."""

    def __init__(self, nodes, elements, density, fixed) -> None:
        self.bar = on.Bar(nodes, elements, density)
        n = self.bar.n_dof
        self.n = n
        pattern = coo_matrix((np.ones(self.bar.rows.size), (self.bar.rows, self.bar.cols)), shape=(n, n)).tocsr()
        pattern.sort_indices()
        self.indptr, self.indices = pattern.indptr, pattern.indices
        self.rows = np.repeat(np.arange(n), np.diff(self.indptr))
        self.cache = SimpleNamespace(csr_indptr=self.indptr, csr_indices=self.indices)
        self.mass = torch.as_tensor(self.values(self.bar.mass))
        self.free_np = np.ones(n, dtype=bool)
        self.free_np[fixed] = False
        self.fixed = torch.as_tensor(np.asarray(fixed, dtype=np.int64))
        self.weights = torch.as_tensor(self.bar.weights)
        self.volume = float(self.bar.weights.sum())
        self.device = torch.device("cpu")
        self.linear_iterations = 0

    def values(self, matrix) -> np.ndarray:
        return np.asarray(matrix.tocsr()[self.rows, self.indices]).ravel()

    def matrix(self, values) -> csr_matrix:
        return csr_matrix((np.asarray(values), self.indices, self.indptr), shape=(self.n, self.n))

    def vector(self, values) -> torch.Tensor:
        t = values if isinstance(values, torch.Tensor) else torch.as_tensor(np.asarray(values, dtype=np.float64))
        return t.to(torch.float64).reshape(-1).clone()

    def spmv(self, values, x) -> torch.Tensor:
        return torch.as_tensor(self.matrix(values) @ x.numpy())

    def kinematics(self, u, u_pred, v_pred, beta_dt2, gamma_dt):
        a = (u - u_pred) / beta_dt2
        return a, v_pred + gamma_dt * a

    def residual(self, a, f_int, f_ext) -> torch.Tensor:
        r = torch.as_tensor(self.matrix(self.mass) @ a.numpy()) + f_int - f_ext
        r[torch.as_tensor(~self.free_np)] = 0.0
        return r

    def solve(self, k_values, beta_dt2, rhs):
        a = self.matrix(self.mass) / beta_dt2
        if k_values is not None:
            a = a + self.matrix(k_values)
        x = np.zeros(self.n)
        f = self.free_np
        x[f] = spsolve(a.tocsr()[f][:, f].tocsc(), rhs.numpy()[f])
        return torch.as_tensor(x), 0, 1, 0.0

    def integrate(self, density) -> float:
        return float(torch.dot(torch.as_tensor(np.asarray(density), dtype=torch.float64).reshape(-1), self.weights))


@pytest.fixture
def host_driver(monkeypatch):
    """Routes the driver's assembly to the oracle's J2 points; returns a runner."""
    ctx = {}

    def assemble(nodes, elements, material, committed, u, u_prev, dt, settings, cache, need_tangent=True):
        ops, point = ctx["ops"], ctx["point"]
        asm = ops.bar.assemble(point, committed.variables["oracle"], u.numpy(), u_prev.numpy(), dt, need_tangent)
        tangent = None
        if need_tangent:
            tangent = torch.sparse_csr_tensor(torch.as_tensor(ops.indptr), torch.as_tensor(ops.indices),
                                              torch.as_tensor(ops.values(asm["K"])), size=(ops.n, ops.n),
                                              check_invariants=False)  # fmt: skip
        t = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64))  # noqa: E731
        return NonlinearSolidAssemblyResult(
            internal_force=t(asm["f"]), tangent=tangent, state=MaterialState({"oracle": asm["state"]}), strains=None,
            strain_rates=None, stresses=t(asm["stress"]), diagnostics={"equivalent_plastic_strain": t(asm["eqps"])},
            free_energy=t(asm["psi"]), dissipation=t(asm["diss"]))  # fmt: skip

    monkeypatch.setattr(D, "assemble_hex8_material_response_cached", assemble)
    monkeypatch.setattr(D, "initialize_hex8_material_state",
                        lambda material, ne: MaterialState({"oracle": ctx["point"].initial_state(8 * ne)}))

    def run(name: str, record_fields: bool = True, adaptive: bool | None = None):
        g, meta = load_case(name)
        nodes, elements = box_mesh(meta["bar"]["lengths"], meta["bar"]["divisions"])
        density = meta["material"]["density"]
        ctx["point"] = on.PointJ2(oj.J2Params(**meta["material"]["params"]))
        ctx["ops"] = HostOperators(nodes, elements, density, g["fixed_dofs"])
        mesh = SimpleNamespace(nodes=nodes, elements=elements, material=SimpleNamespace(density=density))
        unit, amp, dur = torch.as_tensor(g["unit_force"]), meta["amplitude"], meta["duration"]

        def load(t):
            return (amp * math.sin(math.pi * t / dur) if 0.0 <= t <= dur else 0.0) * unit

        ts = D.TimeIntegrationSettings("newmark", meta["time_step"], meta["num_steps"], meta["beta"], meta["gamma"], 1.0,
                                       D.AdaptiveTimeStepSettings(enabled=meta["adaptive"] if adaptive is None
                                                                  else adaptive))  # fmt: skip
        newton = NonlinearNewtonSettings(*meta["newton"][:5], ArmijoSettings(enabled=meta["newton"][5]))
        n = ctx["ops"].n
        sol = D.solve_material_implicit_newmark(
            mesh, ts, np.zeros(n), np.zeros(n), D.DirichletDofSet(g["fixed_dofs"], np.zeros(g["fixed_dofs"].size)),
            load, "three_dimensional", MaterialUpdateSettings(*meta["update_settings"]), newton,
            record_fields=record_fields, operators=ctx["ops"])  # fmt: skip
        return sol, g, meta

    return run


@pytest.mark.parametrize("name", ["newmark_j2_bar_fixed", "newmark_j2_bar_adaptive"])
def test_driver_reproduces_reference_decisions_and_histories(host_driver, name) -> None:
    sol, g, meta = host_driver(name)
    np.testing.assert_array_equal(sol.times, g["times"])
    np.testing.assert_array_equal(sol.newton_iterations, g["newton_iterations"])
    np.testing.assert_array_equal(sol.rejected_step_counts, g["rejected_step_counts"])
    np.testing.assert_array_equal(sol.armijo_backtracks, g["armijo_backtracks"])
    np.testing.assert_array_equal(sol.accepted_time_steps, g["accepted_time_steps"])
    assert [list(r) for r in sol.rejected_reasons] == meta["rejected_reasons"]
    for key in ("displacement", "velocity", "acceleration", "stresses", "equivalent_plastic_strain", "kinetic_energy",
                "free_energy", "dissipated_energy", "external_work"):  # fmt: skip
        ref = g[key]
        np.testing.assert_allclose(getattr(sol, key), ref, rtol=0, atol=1e-11 * np.abs(ref).max(), err_msg=key)
    np.testing.assert_allclose(sol.energy_residual, g["energy_residual"], rtol=0,
                               atol=1e-11 * np.abs(g["external_work"]).max())  # fmt: skip


def test_driver_keeps_final_fields_only_when_asked(host_driver) -> None:
    full, _, _ = host_driver("newmark_j2_bar_fixed")
    last, _, _ = host_driver("newmark_j2_bar_fixed", record_fields=False)
    np.testing.assert_array_equal(last.times, full.times)
    assert last.displacement.shape == (1, full.displacement.shape[1])
    np.testing.assert_array_equal(last.displacement[0], full.displacement[-1])
    np.testing.assert_array_equal(last.kinetic_energy, full.kinetic_energy)


def test_driver_rejects_inhomogeneous_dirichlet_and_other_kinematics(host_driver) -> None:
    mesh = SimpleNamespace(nodes=np.zeros((8, 3)), elements=np.zeros((1, 8), dtype=np.int64),
                           material=SimpleNamespace(density=1.0))  # fmt: skip
    ts = D.TimeIntegrationSettings("newmark", 1e-6, 1, 0.25, 0.5, 1.0)
    newton = NonlinearNewtonSettings(5, 1e-6, 1e-8, 1e-14, 1e-8)
    with pytest.raises(ValueError, match="homogeneous"):
        D.solve_material_implicit_newmark(mesh, ts, np.zeros(24), np.zeros(24), D.DirichletDofSet(np.array([0]),
                                          np.array([1.0])), lambda t: np.zeros(24), "three_dimensional",
                                          MaterialUpdateSettings(50, 1e-10, 1e-12, 1e-10), newton)  # fmt: skip
    with pytest.raises(ValueError, match="three_dimensional"):
        D.solve_material_implicit_newmark(mesh, ts, np.zeros(24), np.zeros(24), D.DirichletDofSet(np.array([0]),
                                          np.array([0.0])), lambda t: np.zeros(24), "plane_strain",
                                          MaterialUpdateSettings(50, 1e-10, 1e-12, 1e-10), newton)  # fmt: skip


def test_unconverged_linear_solve_is_recoverable(host_driver, monkeypatch) -> None:
    """A Newton system whose PCG solve stops at its iteration limit (status 1) fails the step
    with the recoverable reason "linear_solver_not_converged": with fixed steps the error
    propagates, with adaptive steps the step is retried at half the size."""
    state = {"left": 1}
    original = HostOperators.solve

    def flaky(self, k_values, beta_dt2, rhs):
        x, status, iterations, rel = original(self, k_values, beta_dt2, rhs)
        if k_values is not None and state["left"] > 0:
            state["left"] -= 1
            return x, 1, 20000, 1e-3
        return x, status, iterations, rel

    monkeypatch.setattr(HostOperators, "solve", flaky)
    with pytest.raises(D.RecoverableNonlinearStepError) as info:
        host_driver("newmark_j2_bar_fixed")  # fixed steps: the failure propagates
    assert info.value.reason == "linear_solver_not_converged"
    assert info.value.diagnostics["linear_status"] == 1
    state["left"] = 1
    sol, g, _ = host_driver("newmark_j2_bar_fixed", adaptive=True)  # the first step is retried at half size
    assert sol.rejected_reasons[1][0] == "linear_solver_not_converged"
    assert sol.times[-1] == pytest.approx(g["times"][-1], rel=1e-12)
    assert sol.accepted_time_steps[1] == pytest.approx(0.5 * g["accepted_time_steps"][1], rel=1e-12)
