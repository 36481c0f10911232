"""Implicit Newmark material dynamics on the GPU (drop-in for fem.dynamics.material's
``solve_material_implicit_newmark``); with ``RVEHomogenizedMaterial`` at the macro points
it is implicit FE^2 with the RVE effective tangent.

Same arguments, step control and histories as the reference
(src/fem/dynamics/material.py:300-731, 732-927):

* Newmark predictor; full Newton on r = M a + f_int - f_ext over the free DOFs with the
  reference's scaled residual and increment tests, re-evaluated from the committed
  material state at every iterate; effective tangent K + M / (beta dt^2); optional Armijo
  line search on the residual merit (src/fem/solvers/line_search.py:40-67);
* convergence-driven step control: a recoverable failure cuts the step back, easy steps
  grow it (src/fem/solvers/time_step.py:12-31);
* kinetic energy with the consistent mass, free and dissipated energy, external work, the
  energy residual, incremental-work and activation measures, Newton iterations, Armijo
  backtracks and rejected steps per accepted state.

``mesh`` is the reference's preprocess bundle (``mesh_info.nodes``, ``mesh_info.elements``,
``material``) or any object with ``nodes``, ``elements`` and ``material``.  Each Newton
iterate runs on the device: Hex8 strains, the material update at every integration point
(the J2 kernels, or one device batch of periodic RVE solves), internal force and CSR
tangent (csrc/hex8.cu), then the Newmark kinematics, residual, effective tangent and a
Jacobi-preconditioned CG on the free DOFs (csrc/newmark.cu).  The consistent mass is
assembled once, in the CSR pattern of the tangent.

Deviation from the reference: the Newton systems are solved by PCG to a relative residual
of ``MacroLinearSolverOptions.relative_tolerance`` (1e-12) rather than factorised; a PCG
solve that does not converge raises ``RecoverableNonlinearStepError`` with reason
"linear_solver_not_converged" (a time-step cutback when adaptive stepping is on).
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from time import perf_counter
from typing import Any, Callable

import numpy as np
import torch

from . import _native
from .assembly import (
    MaterialAssemblyCache,
    NonlinearSolidAssemblyResult,
    assemble_hex8_material_response_cached,
    build_hex8_material_assembly_cache,
    initialize_hex8_material_state,
)
from .materials import MaterialState, MaterialUpdateSettings
from .rve import ArmijoSettings, NonlinearNewtonSettings

LoadFunction = Callable[[float], Any]

CSR_PCG_WORK_DOUBLES = 3 * 1024 + 8  # CIB_CSR_PCG_WORK_DOUBLES


# --------------------------------------------------------------------------------------
# Settings, errors and step-control rules (src/fem/solvers/data.py, time_step.py,
# line_search.py; src/fem/dynamics/material.py:56-69).


@dataclass(frozen=True)
class AdaptiveTimeStepSettings:
    """Convergence-driven implicit time-step controls."""

    enabled: bool = False
    minimum_factor: float = 1.0 / 16.0
    maximum_factor: float = 2.0
    cutback_factor: float = 0.5
    growth_factor: float = 2.0
    easy_iteration_limit: int = 4
    easy_step_count: int = 3

    def __post_init__(self) -> None:
        if not 0.0 < self.minimum_factor <= 1.0:
            raise ValueError("Adaptive minimum_factor must lie in (0, 1].")
        if self.maximum_factor < 1.0:
            raise ValueError("Adaptive maximum_factor must be at least one.")
        if not 0.0 < self.cutback_factor < 1.0:
            raise ValueError("Adaptive cutback_factor must lie in (0, 1).")
        if self.growth_factor <= 1.0:
            raise ValueError("Adaptive growth_factor must exceed one.")
        if self.easy_iteration_limit < 0 or self.easy_step_count <= 0:
            raise ValueError("Adaptive easy-step controls must be positive.")


@dataclass(frozen=True)
class TimeIntegrationSettings:
    """Time-integration settings (Newmark beta and gamma, nominal step and step count)."""

    scheme: str
    time_step: float
    num_steps: int
    beta: float
    gamma: float
    cfl_safety_factor: float
    adaptive: AdaptiveTimeStepSettings = field(default_factory=AdaptiveTimeStepSettings)


@dataclass(frozen=True)
class DirichletDofSet:
    """Prescribed degrees of freedom and values (homogeneous only for material dynamics)."""

    dofs: np.ndarray
    values: np.ndarray


@dataclass(frozen=True)
class MacroLinearSolverOptions:
    """Controls of the Jacobi-PCG solves of the macro Newton systems (no reference
    counterpart: the reference factorises).  The host reads the solver status every
    ``check_every`` iterations."""

    relative_tolerance: float = 1.0e-12
    max_iterations: int = 20000
    check_every: int = 16


class NonlinearStepConvergenceError(RuntimeError):
    """A failed global Newton step with structured diagnostics."""

    def __init__(self, reason: str, diagnostics: dict[str, object]) -> None:
        super().__init__(f"Implicit Newmark Newton failed: {reason}.")
        self.reason = reason
        self.diagnostics = diagnostics


class RecoverableNonlinearStepError(NonlinearStepConvergenceError):
    """A convergence failure eligible for a time-step cutback."""


class ArmijoLineSearchError(RuntimeError):
    """Exhaustion of the configured Armijo sequence."""

    def __init__(self, diagnostics: dict[str, float | int]) -> None:
        super().__init__("Armijo line search exhausted all configured candidates.")
        self.diagnostics = diagnostics


@dataclass(frozen=True)
class ArmijoResult:
    """One accepted line-search step."""

    step_length: float
    backtracks: int
    residual_norm: float


def cut_back_time_step(current_time_step: float, initial_time_step: float, settings: AdaptiveTimeStepSettings) -> float:
    """Reduce a rejected step without crossing the configured minimum."""
    return max(initial_time_step * settings.minimum_factor, current_time_step * settings.cutback_factor)


def grow_time_step(current_time_step: float, initial_time_step: float, settings: AdaptiveTimeStepSettings) -> float:
    """Increase an easy accepted step without crossing the configured maximum."""
    return min(initial_time_step * settings.maximum_factor, current_time_step * settings.growth_factor)


def perform_armijo_search(residual_norm: float, evaluate_residual_norm: Callable[[float], float],
                          settings: ArmijoSettings) -> ArmijoResult:  # fmt: skip
    """First step length 1, rho, rho^2, ... whose residual merit 0.5 ||r||^2 drops below
    0.5 ||r0||^2 - c s ||r0||^2.  Takes norms (the residuals stay on the device)."""
    current_merit = 0.5 * residual_norm**2
    last = math.inf
    for backtrack in range(settings.max_backtracks + 1):
        step = settings.reduction_factor**backtrack
        last = float(evaluate_residual_norm(step))
        if 0.5 * last**2 <= current_merit - settings.sufficient_decrease * step * residual_norm**2:
            return ArmijoResult(step, backtrack, last)
    raise ArmijoLineSearchError({"current_residual_norm": residual_norm, "current_merit": current_merit,
                                 "last_candidate_residual_norm": last, "max_backtracks": settings.max_backtracks})  # fmt: skip


@dataclass(frozen=True)
class MaterialDynamicSolution:
    """Histories of an implicit material-dynamics run (one row per accepted state).

    Per-DOF and per-point histories (displacement ... material_diagnostics) hold every
    accepted state when the run records fields, else the final state only."""

    times: np.ndarray
    displacement: np.ndarray
    velocity: np.ndarray
    acceleration: np.ndarray
    internal_force: np.ndarray
    external_force: np.ndarray
    stresses: np.ndarray
    equivalent_plastic_strain: np.ndarray
    kinetic_energy: np.ndarray
    free_energy: np.ndarray
    dissipated_energy: np.ndarray
    external_work: np.ndarray
    energy_residual: np.ndarray
    positive_incremental_work: np.ndarray
    negative_incremental_work: np.ndarray
    unloading_volume_fraction: np.ndarray
    viscoplastic_active_volume_fraction: np.ndarray
    minimum_yield_activation_margin: np.ndarray
    maximum_yield_activation_margin: np.ndarray
    newton_iterations: np.ndarray
    accepted_time_steps: np.ndarray
    rejected_step_counts: np.ndarray
    armijo_backtracks: np.ndarray
    rejected_reasons: tuple[tuple[str, ...], ...]
    material_diagnostics: dict[str, np.ndarray]
    integrator_diagnostics: dict[str, np.ndarray]
    final_state: MaterialState
    solve_time: float
    material_state_history: dict[str, np.ndarray] | None = None


# --------------------------------------------------------------------------------------
# Device operators of one mesh.


class MacroOperators:
    """Assembly cache, consistent mass (CSR values in the tangent's pattern), free-DOF
    mask and the PCG work vectors of one Hex8 mesh, all on the device."""

    def __init__(self, nodes, elements, density: float, fixed_dofs, cache: MaterialAssemblyCache | None = None,
                 linear_solver: MacroLinearSolverOptions | None = None) -> None:  # fmt: skip
        dev = _native.require_cuda()
        self.lib = _native.load_library()
        self.device = dev
        self.nodes = np.asarray(nodes.cpu() if isinstance(nodes, torch.Tensor) else nodes, dtype=np.float64)
        self.elements = np.asarray(elements.cpu() if isinstance(elements, torch.Tensor) else elements, dtype=np.int64)
        self.cache = cache if cache is not None else build_hex8_material_assembly_cache(self.nodes, self.elements)
        self.linear = linear_solver or MacroLinearSolverOptions()
        n = 3 * self.cache.node_count
        self.n = n
        self.indptr = torch.as_tensor(self.cache.csr_indptr, dtype=torch.int64, device=dev)
        self.indices = torch.as_tensor(self.cache.csr_indices, dtype=torch.int64, device=dev)
        nnz = int(self.cache.csr_indices.size)
        ne = int(self.elements.shape[0])
        f64 = dict(dtype=torch.float64, device=dev)
        me = torch.empty(ne * 576, **f64)
        self.mass = torch.empty(nnz, **f64)
        _native.check(self.lib.cib_hex8_mass_csr(ne, self.cache.jw.data_ptr(), float(density), nnz,
                                                 self.cache.csr_ptr.data_ptr(), self.cache.csr_list.data_ptr(),
                                                 me.data_ptr(), self.mass.data_ptr(), _native.stream_ptr()),
                      "cib_hex8_mass_csr")  # fmt: skip
        del me
        fixed = np.unique(np.asarray(fixed_dofs, dtype=np.int64))
        if fixed.size and (fixed.min() < 0 or fixed.max() >= n):
            raise ValueError("Dirichlet DOFs out of range.")
        free = np.ones(n, dtype=np.uint8)
        free[fixed] = 0
        self.fixed = torch.as_tensor(fixed, device=dev)
        self.free = torch.as_tensor(free, device=dev)
        self.weights = self.cache.jw.reshape(-1)
        self.volume = float(self.weights.sum())
        self.values = torch.empty(nnz, **f64)
        self.dinv = torch.empty(n, **f64)
        self.r, self.z, self.p, self.q = (torch.empty(n, **f64) for _ in range(4))
        self.work = torch.zeros(CSR_PCG_WORK_DOUBLES, **f64)
        self.linear_iterations = 0

    def vector(self, values: Any) -> torch.Tensor:
        """A length-3N float64 device vector (copied from host arrays)."""
        t = values if isinstance(values, torch.Tensor) else torch.as_tensor(np.asarray(values, dtype=np.float64))
        t = t.to(device=self.device, dtype=torch.float64).contiguous().reshape(-1)
        if t.numel() != self.n:
            raise ValueError(f"expected {self.n} DOF values, got {t.numel()}")
        return t

    def spmv(self, values: torch.Tensor, x: torch.Tensor) -> torch.Tensor:
        y = torch.empty(self.n, dtype=torch.float64, device=self.device)
        _native.check(self.lib.cib_csr_spmv(self.n, self.indptr.data_ptr(), self.indices.data_ptr(), values.data_ptr(),
                                            x.data_ptr(), y.data_ptr(), _native.stream_ptr()), "cib_csr_spmv")  # fmt: skip
        return y

    def kinematics(self, u, u_pred, v_pred, beta_dt2: float, gamma_dt: float):
        a = torch.empty(self.n, dtype=torch.float64, device=self.device)
        v = torch.empty_like(a)
        _native.check(self.lib.cib_newmark_kinematics(self.n, u.data_ptr(), u_pred.data_ptr(), v_pred.data_ptr(),
                                                      beta_dt2, gamma_dt, a.data_ptr(), v.data_ptr(),
                                                      _native.stream_ptr()), "cib_newmark_kinematics")  # fmt: skip
        return a, v

    def residual(self, a, f_int, f_ext) -> torch.Tensor:
        r = torch.empty(self.n, dtype=torch.float64, device=self.device)
        _native.check(self.lib.cib_newmark_residual(self.n, self.indptr.data_ptr(), self.indices.data_ptr(),
                                                    self.mass.data_ptr(), a.data_ptr(), f_int.data_ptr(),
                                                    f_ext.data_ptr(), self.free.data_ptr(), r.data_ptr(),
                                                    _native.stream_ptr()), "cib_newmark_residual")  # fmt: skip
        return r

    def solve(self, k_values: torch.Tensor | None, beta_dt2: float, rhs: torch.Tensor) -> tuple[torch.Tensor, int, int, float]:
        """x on the free DOFs of (K + M / beta_dt2) x = rhs (K None: M / beta_dt2); 0 on the
        fixed DOFs.  Returns x, status (0 converged, 1 iteration limit, 2 breakdown),
        iterations and the relative residual."""
        lib = self.lib
        stream = _native.stream_ptr()
        kp = k_values.data_ptr() if k_values is not None else None
        _native.check(lib.cib_newmark_effective_tangent(self.n, self.indptr.data_ptr(), self.indices.data_ptr(), kp,
                                                        self.mass.data_ptr(), beta_dt2, self.free.data_ptr(),
                                                        self.values.data_ptr(), self.dinv.data_ptr(), stream),
                      "cib_newmark_effective_tangent")  # fmt: skip
        x = torch.empty(self.n, dtype=torch.float64, device=self.device)
        status, iterations, rel = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_double(0.0)
        opts = self.linear
        _native.check(lib.cib_csr_pcg(self.n, self.indptr.data_ptr(), self.indices.data_ptr(), self.values.data_ptr(),
                                      self.free.data_ptr(), self.dinv.data_ptr(), rhs.data_ptr(), x.data_ptr(),
                                      self.r.data_ptr(), self.z.data_ptr(), self.p.data_ptr(), self.q.data_ptr(),
                                      self.work.data_ptr(), float(opts.relative_tolerance), int(opts.max_iterations),
                                      int(opts.check_every), ctypes.byref(status), ctypes.byref(iterations),
                                      ctypes.byref(rel), stream), "cib_csr_pcg")  # fmt: skip
        self.linear_iterations += int(iterations.value)
        return x, int(status.value), int(iterations.value), float(rel.value)

    def integrate(self, density: Any) -> float:
        """Sum over integration points of density * J w (integrate_quadrature_density)."""
        d = density if isinstance(density, torch.Tensor) else torch.as_tensor(np.asarray(density, dtype=np.float64))
        return float(torch.dot(d.to(self.device, torch.float64).reshape(-1), self.weights))


# --------------------------------------------------------------------------------------
# The solver.


@dataclass
class _StepState:
    time: float
    displacement: torch.Tensor
    velocity: torch.Tensor
    acceleration: torch.Tensor
    material_state: MaterialState
    assembly: NonlinearSolidAssemblyResult


@dataclass
class _Interval:
    state: _StepState
    dissipation_increment: float
    external_work_increment: float
    newton_iterations: int
    armijo_backtracks: int


def _mesh_fields(mesh) -> tuple[np.ndarray, np.ndarray, Any]:
    info = getattr(mesh, "mesh_info", None)
    if info is not None:
        if getattr(info, "dimension", 3) != 3:
            raise ValueError("The GPU material dynamics needs a three-dimensional Hex8 mesh.")
        nodes, elements = info.nodes, info.elements
    else:
        nodes, elements = mesh.nodes, mesh.elements
    elements = np.asarray(elements)
    if elements.ndim != 2 or elements.shape[1] != 8:
        raise ValueError("The GPU material dynamics needs Hex8 elements (E, 8).")
    return np.asarray(nodes, dtype=np.float64), elements.astype(np.int64), mesh.material


class _Trial:
    """Evaluates Newmark trials of one step from its committed start state."""

    def __init__(self, ops: MacroOperators, mesh_nodes, mesh_elements, material, start: _StepState,
                 dt: float, beta: float, gamma: float, external: torch.Tensor, kinematics: str,
                 update_settings: MaterialUpdateSettings) -> None:  # fmt: skip
        self.ops, self.nodes, self.elements, self.material = ops, mesh_nodes, mesh_elements, material
        self.start, self.dt, self.external = start, dt, external
        self.kinematics, self.update_settings = kinematics, update_settings
        self.beta_dt2 = beta * dt**2
        self.gamma_dt = gamma * dt
        self.u_pred = start.displacement + dt * start.velocity + dt**2 * (0.5 - beta) * start.acceleration
        self.v_pred = start.velocity + dt * (1.0 - gamma) * start.acceleration

    def __call__(self, u: torch.Tensor, need_tangent: bool = True):
        assembly = assemble_hex8_material_response_cached(
            self.nodes, self.elements, self.material, self.start.material_state, u, self.start.displacement, self.dt,
            self.update_settings, self.ops.cache, need_tangent)  # fmt: skip
        a, v = self.ops.kinematics(u, self.u_pred, self.v_pred, self.beta_dt2, self.gamma_dt)
        r = self.ops.residual(a, assembly.internal_force, self.external)
        return a, v, assembly, r


def solve_material_implicit_newmark(
    mesh,
    time_settings: TimeIntegrationSettings,
    initial_displacement,
    initial_velocity,
    dirichlet: DirichletDofSet,
    load_function: LoadFunction,
    kinematics: str,
    update_settings: MaterialUpdateSettings,
    newton_settings: NonlinearNewtonSettings,
    progress_callback: Callable[[dict[str, Any]], None] | None = None,
    linear_solver: MacroLinearSolverOptions | None = None,
    record_fields: bool = True,
    operators: MacroOperators | None = None,
) -> MaterialDynamicSolution:
    """Material dynamics by implicit Newmark with the reference's nonlinear controls
    (src/fem/dynamics/material.py:300-443).  ``load_function(t)`` returns the external
    force vector (3N; host array or device tensor).  ``operators`` reuses the device
    operators of an earlier run on the same mesh and Dirichlet set."""
    if np.any(np.asarray(dirichlet.values) != 0.0):
        raise ValueError("Material dynamics currently requires homogeneous Dirichlet values.")
    if kinematics != "three_dimensional":
        raise ValueError("The GPU Hex8 material dynamics supports kinematics='three_dimensional' only.")
    start_time = perf_counter()
    nodes, elements, material = _mesh_fields(mesh)
    ops = operators or MacroOperators(nodes, elements, material.density, dirichlet.dofs, linear_solver=linear_solver)
    dt0 = float(time_settings.time_step)
    final_time = dt0 * time_settings.num_steps
    u = ops.vector(initial_displacement).clone()
    v = ops.vector(initial_velocity).clone()
    u[ops.fixed] = 0.0
    v[ops.fixed] = 0.0
    state0 = initialize_hex8_material_state(material, int(elements.shape[0]))
    assembly = assemble_hex8_material_response_cached(nodes, elements, material, state0, u, u, dt0, update_settings,
                                                      ops.cache, True)  # fmt: skip
    external = ops.vector(load_function(0.0))
    a, status, _, _ = ops.solve(None, 1.0, external - assembly.internal_force)
    if status != 0:
        raise RuntimeError("The consistent-mass solve for the initial acceleration did not converge.")
    current = _StepState(0.0, u, v, a, assembly.state, assembly)
    rec = _Recorder(ops, load_function, record_fields)
    rec.record(current, None)
    pending: list[str] = []
    dt = dt0
    minimum = dt0 * time_settings.adaptive.minimum_factor
    easy = 0
    adaptive = time_settings.adaptive
    while current.time < final_time:
        trial_dt = min(dt, final_time - current.time)
        try:
            interval = _solve_implicit_step(ops, nodes, elements, material, current, trial_dt, load_function, kinematics,
                                            update_settings, newton_settings, time_settings.beta, time_settings.gamma)  # fmt: skip
        except RecoverableNonlinearStepError as error:
            if not adaptive.enabled:
                raise
            pending.append(error.reason)
            if trial_dt <= minimum:
                error.diagnostics["minimum_time_step"] = minimum
                error.diagnostics["rejected_reasons"] = tuple(pending)
                raise
            dt = cut_back_time_step(trial_dt, dt0, adaptive)
            easy = 0
            continue
        current = interval.state
        rec.record(current, interval, rejected=tuple(pending))
        if progress_callback is not None:
            progress_callback({"stage": "material_dynamics", "scheme": "implicit_newmark",
                               "accepted_step": rec.accepted, "nominal_total_steps": time_settings.num_steps,
                               "physical_time": current.time, "final_time": final_time,
                               "newton_iterations": interval.newton_iterations,
                               "armijo_backtracks": interval.armijo_backtracks,
                               "elapsed_seconds": perf_counter() - start_time})  # fmt: skip
        easy_step = (not pending and interval.armijo_backtracks == 0
                     and interval.newton_iterations <= adaptive.easy_iteration_limit)  # fmt: skip
        easy = easy + 1 if easy_step else 0
        pending = []
        if adaptive.enabled and easy >= adaptive.easy_step_count:
            dt = grow_time_step(trial_dt, dt0, adaptive)
            easy = 0
        else:
            dt = trial_dt
    return rec.solution(current, perf_counter() - start_time)


def _solve_implicit_step(ops: MacroOperators, nodes, elements, material, start: _StepState, time_step: float,
                         load_function: LoadFunction, kinematics: str, update_settings: MaterialUpdateSettings,
                         newton: NonlinearNewtonSettings, beta: float, gamma: float) -> _Interval:  # fmt: skip
    """One implicit Newmark step from a committed state (src/fem/dynamics/material.py:446-662)."""
    if newton.max_iterations <= 0:
        raise ValueError("Implicit Newmark requires max_iterations > 0.")
    target_time = start.time + time_step
    external = ops.vector(load_function(target_time))
    trial = _Trial(ops, nodes, elements, material, start, time_step, beta, gamma, external, kinematics, update_settings)
    u = trial.u_pred.clone()
    u[ops.fixed] = 0.0
    initial_norm = None
    last_increment_norm = math.inf
    last_residual_norm = math.inf
    last_increment = torch.zeros(ops.n, dtype=torch.float64, device=ops.device)
    backtracks = 0
    residual_tolerance = increment_tolerance = 0.0
    assembly = None

    def accept(a, v, asm, iteration) -> _Interval:
        dissipation = time_step * ops.integrate(asm.dissipation)
        previous = ops.vector(load_function(start.time))
        work = float(0.5 * torch.dot(previous + external, u - start.displacement))
        return _Interval(_StepState(target_time, u, v, a, asm.state, asm), dissipation, work, iteration, backtracks)

    for iteration in range(newton.max_iterations + 1):
        a, v, assembly, residual = trial(u)
        norms = torch.stack([torch.linalg.vector_norm(residual), torch.linalg.vector_norm(u)]).cpu().numpy()
        residual_norm, displacement_norm = float(norms[0]), float(norms[1])
        last_residual_norm = residual_norm
        if initial_norm is None:
            initial_norm = residual_norm
        residual_tolerance = max(newton.residual_absolute_tolerance, newton.residual_relative_tolerance * initial_norm)
        increment_tolerance = max(newton.increment_absolute_tolerance,
                                  newton.increment_relative_tolerance * max(displacement_norm, 1.0))  # fmt: skip
        if residual_norm <= residual_tolerance and (iteration == 0 or last_increment_norm <= increment_tolerance):
            return accept(a, v, assembly, iteration)
        if iteration == newton.max_iterations:
            break
        increment, status, pcg_iterations, pcg_rel = ops.solve(assembly.tangent.values(), beta * time_step**2, -residual)
        if not bool(torch.isfinite(increment).all()):
            raise NonlinearStepConvergenceError("non_finite_increment", _failure_diagnostics(
                target_time, time_step, iteration, residual_norm, residual_tolerance, increment, increment_tolerance,
                u, assembly))  # fmt: skip
        if status != 0:
            diag = _failure_diagnostics(target_time, time_step, iteration, residual_norm, residual_tolerance, increment,
                                        increment_tolerance, u, assembly)  # fmt: skip
            diag.update(linear_status=status, linear_iterations=pcg_iterations, linear_relative_residual=pcg_rel)
            raise RecoverableNonlinearStepError("linear_solver_not_converged", diag)
        increment_norm = float(torch.linalg.vector_norm(increment))
        if residual_norm <= residual_tolerance and increment_norm <= increment_tolerance:
            return accept(a, v, assembly, iteration)
        step = 1.0
        if newton.armijo.enabled:
            base = u

            def candidate_norm(step_length: float) -> float:
                return float(torch.linalg.vector_norm(trial(base + step_length * increment, need_tangent=False)[3]))

            try:
                search = perform_armijo_search(residual_norm, candidate_norm, newton.armijo)
            except ArmijoLineSearchError as error:
                diag = _failure_diagnostics(target_time, time_step, iteration, residual_norm, residual_tolerance,
                                            increment, increment_tolerance, u, assembly)  # fmt: skip
                diag["armijo"] = error.diagnostics
                raise RecoverableNonlinearStepError("armijo_exhausted", diag) from error
            step = search.step_length
            backtracks += search.backtracks
        accepted = increment if step == 1.0 else step * increment
        u = u + accepted
        last_increment = accepted
        last_increment_norm = float(torch.linalg.vector_norm(accepted))
    raise RecoverableNonlinearStepError("maximum_iterations_exceeded", _failure_diagnostics(
        target_time, time_step, newton.max_iterations, last_residual_norm, residual_tolerance, last_increment,
        increment_tolerance, u, assembly))  # fmt: skip


def _failure_diagnostics(target_time, time_step, iteration, residual_norm, residual_tolerance, increment,
                         increment_tolerance, displacement, assembly) -> dict[str, object]:  # fmt: skip
    """Global Newton failure snapshot (src/fem/dynamics/material.py:704-729); the increment
    vector itself is included for meshes of at most 4096 DOFs."""
    out: dict[str, object] = {
        "algorithm": "implicit_newmark_full_step_newton", "target_time": target_time, "time_step": time_step,
        "iteration": iteration, "residual_norm": residual_norm, "residual_tolerance": residual_tolerance,
        "increment_norm": float(torch.linalg.vector_norm(increment)), "increment_tolerance": increment_tolerance,
        "displacement_norm": float(torch.linalg.vector_norm(displacement)),
    }  # fmt: skip
    if increment.numel() <= 4096:
        out["increment"] = increment.cpu().tolist()
    if assembly is not None:
        stresses = assembly.stresses
        out["maximum_absolute_stress"] = float(torch.as_tensor(stresses).abs().max())
        if assembly.tangent is not None and hasattr(assembly.tangent, "values"):
            tan = assembly.tangent
            rows = torch.repeat_interleave(torch.arange(tan.shape[0], device=tan.device), tan.crow_indices().diff())
            diag = tan.values()[tan.col_indices() == rows]
            out["minimum_tangent_diagonal"] = float(diag.min())
    return out


_ACTIVITY = ("incremental_work_density", "viscoplastic_active", "yield_activation_margin")


class _Recorder:
    """Histories of the accepted states (src/fem/dynamics/material.py:732-927)."""

    def __init__(self, ops: MacroOperators, load_function: LoadFunction, record_fields: bool,
                 lumped_mass: torch.Tensor | None = None, record_state: bool = False) -> None:  # fmt: skip
        self.ops, self.load, self.fields = ops, load_function, record_fields
        self.lumped = lumped_mass  # explicit runs: kinetic energy with the lumped mass
        self.record_state = record_state
        self.rows: list[dict[str, Any]] = []
        self.accepted = 0

    def record(self, state: _StepState, interval: _Interval | None, rejected: tuple[str, ...] = ()) -> None:
        ops, asm = self.ops, state.assembly
        if self.lumped is not None:
            kinetic = 0.5 * float(torch.sum(self.lumped * state.velocity**2))
        else:
            kinetic = 0.5 * float(torch.dot(state.velocity, ops.spmv(ops.mass, state.velocity)))
        row: dict[str, Any] = {
            "time": state.time, "kinetic": kinetic, "free": ops.integrate(asm.free_energy),
            "dissipation": interval.dissipation_increment if interval else 0.0,
            "work": interval.external_work_increment if interval else 0.0,
            "newton": interval.newton_iterations if interval else 0,
            "armijo": interval.armijo_backtracks if interval else 0, "rejected": rejected,
        }  # fmt: skip
        diags = asm.diagnostics
        if all(k in diags for k in _ACTIVITY):
            work = torch.as_tensor(diags["incremental_work_density"], device=ops.device, dtype=torch.float64)
            active = torch.as_tensor(diags["viscoplastic_active"], device=ops.device, dtype=torch.float64)
            margin = torch.as_tensor(diags["yield_activation_margin"], device=ops.device, dtype=torch.float64)
            row["pos"] = ops.integrate(work.clamp(min=0.0))
            row["neg"] = ops.integrate(work.clamp(max=0.0))
            row["unload"] = ops.integrate((work < 0.0).to(torch.float64)) / ops.volume
            row["active"] = ops.integrate(active) / ops.volume
            row["mmin"], row["mmax"] = float(margin.min()), float(margin.max())
        if interval is not None:
            self.accepted += 1
        row["fields"] = self._fields(state) if self.fields else None
        if self.record_state:
            row["state"] = {k: (v.cpu().numpy() if isinstance(v, torch.Tensor) else np.asarray(v)).copy()
                            for k, v in state.material_state.variables.items()}  # fmt: skip
        self.last = state
        self.rows.append(row)

    def _fields(self, state: _StepState) -> dict[str, np.ndarray]:
        asm = state.assembly
        host = lambda t: (t.cpu().numpy() if isinstance(t, torch.Tensor) else np.asarray(t)).copy()  # noqa: E731
        if "equivalent_plastic_strain" in asm.diagnostics:
            eqps = host(asm.diagnostics["equivalent_plastic_strain"])
        elif "equivalent_plastic_strain" in state.material_state.variables:
            eqps = host(state.material_state.variables["equivalent_plastic_strain"])
        else:
            eqps = np.zeros(int(np.asarray(asm.stresses.shape)[0]))
        n_points = int(asm.stresses.shape[0])
        return {
            "u": host(state.displacement), "v": host(state.velocity), "a": host(state.acceleration),
            "f_int": host(asm.internal_force), "f_ext": host(self.ops.vector(self.load(state.time))),
            "stress": host(asm.stresses), "eqps": eqps,
            "diag": {k: host(val) for k, val in asm.diagnostics.items() if tuple(np.shape(val)) == (n_points,)},
            "psi": host(asm.free_energy), "diss": host(asm.dissipation),
        }  # fmt: skip

    def solution(self, final: _StepState, solve_time: float, integrator: dict | None = None) -> MaterialDynamicSolution:
        rows = self.rows
        steps = len(rows)
        col = lambda k, default=0.0: np.asarray([r.get(k, default) for r in rows], dtype=np.float64)  # noqa: E731
        times = col("time")
        kinetic, free = col("kinetic"), col("free")
        dissipated = np.cumsum(col("dissipation"))
        work = np.cumsum(col("work"))
        residual = kinetic + free + dissipated - work - (kinetic[0] + free[0])
        kept = [r["fields"] for r in rows] if self.fields else [self._fields(self.last)]
        stack = lambda k: np.stack([f[k] for f in kept])  # noqa: E731
        diag_names = sorted(set(kept[0]["diag"]).intersection(*[f["diag"] for f in kept]))
        material_diagnostics = {k: np.stack([f["diag"][k] for f in kept]) for k in diag_names}
        material_diagnostics["free_energy_density"] = stack("psi")
        material_diagnostics["dissipation_density"] = stack("diss")
        accepted_steps = np.zeros(steps)
        accepted_steps[1:] = np.diff(times)
        final_state = MaterialState({k: (v.cpu().numpy() if isinstance(v, torch.Tensor) else v)
                                     for k, v in final.material_state.variables.items()})  # fmt: skip
        return MaterialDynamicSolution(
            times=times, displacement=stack("u"), velocity=stack("v"), acceleration=stack("a"),
            internal_force=stack("f_int"), external_force=stack("f_ext"), stresses=stack("stress"),
            equivalent_plastic_strain=stack("eqps"), kinetic_energy=kinetic, free_energy=free,
            dissipated_energy=dissipated, external_work=work, energy_residual=residual,
            positive_incremental_work=col("pos"), negative_incremental_work=col("neg"),
            unloading_volume_fraction=col("unload"), viscoplastic_active_volume_fraction=col("active"),
            minimum_yield_activation_margin=col("mmin"), maximum_yield_activation_margin=col("mmax"),
            newton_iterations=col("newton").astype(np.int64), accepted_time_steps=accepted_steps,
            rejected_step_counts=np.asarray([len(r["rejected"]) for r in rows], dtype=np.int64),
            armijo_backtracks=col("armijo").astype(np.int64),
            rejected_reasons=tuple(r["rejected"] for r in rows), material_diagnostics=material_diagnostics,
            integrator_diagnostics=(integrator if integrator is not None else
                                    {"linear_iterations": np.asarray([self.ops.linear_iterations], dtype=np.int64)}),
            final_state=final_state, solve_time=solve_time,
            material_state_history=({k: np.stack([r["state"][k] for r in rows]) for k in rows[0]["state"]}
                                    if self.record_state else None),
        )  # fmt: skip


# --------------------------------------------------------------------------------------
# Explicit velocity-Verlet material dynamics (src/fem/dynamics/material.py:89-297) and its
# CFL check (src/fem/dynamics/stability.py:34-100).

# Hex8 element edges in the reference's node order (stability.py EDGE_NODE_TABLE["hex8"]).
HEX8_EDGES = ((0, 1), (0, 2), (1, 3), (2, 3), (4, 5), (4, 6), (5, 7), (6, 7), (0, 4), (1, 5), (2, 6), (3, 7))


@dataclass(frozen=True)
class StabilityReport:
    """Explicit CFL data: smallest element edge, material wave-speed bound, stable step."""

    minimum_length: float
    maximum_wave_speed: float
    stable_time_step: float
    requested_time_step: float


def compute_explicit_stability_report(mesh, time_settings: TimeIntegrationSettings) -> StabilityReport:
    """cfl_safety_factor x the smallest Hex8 edge / the material's maximum wave speed."""
    nodes, elements, material = _mesh_fields(mesh)
    edges = np.asarray(HEX8_EDGES)
    vectors = nodes[elements[:, edges[:, 1]]] - nodes[elements[:, edges[:, 0]]]
    minimum_length = float(np.sqrt(np.min(np.einsum("eki,eki->ek", vectors, vectors))))
    speed = float(material.maximum_wave_speed)
    return StabilityReport(minimum_length, speed, time_settings.cfl_safety_factor * minimum_length / speed,
                           time_settings.time_step)  # fmt: skip


def check_explicit_stability(mesh, time_settings: TimeIntegrationSettings) -> StabilityReport:
    """Raise ValueError when the requested explicit step exceeds the CFL bound."""
    report = compute_explicit_stability_report(mesh, time_settings)
    if time_settings.time_step > report.stable_time_step:
        raise ValueError("Explicit time step violates the CFL stability bound: "
                         f"dt={time_settings.time_step:.6e}, dt_crit={report.stable_time_step:.6e}.")  # fmt: skip
    return report


def solve_material_explicit(
    mesh,
    time_settings: TimeIntegrationSettings,
    initial_displacement,
    initial_velocity,
    dirichlet: DirichletDofSet,
    load_function: LoadFunction,
    kinematics: str,
    update_settings: MaterialUpdateSettings,
    progress_callback: Callable[[dict[str, Any]], None] | None = None,
    residual_corrector=None,
    correction_controls=None,
    record_material_state_history: bool = False,
    record_fields: bool = True,
    operators: MacroOperators | None = None,
) -> MaterialDynamicSolution:
    """Material dynamics by explicit velocity Verlet with the row-sum lumped mass
    (src/fem/dynamics/material.py:89-297), same arguments and histories as the reference.

    Every step runs on the device: the Verlet predictor (``cib_verlet_predict``), Hex8
    strains, the material update at every integration point (J2 kernels, or one device
    batch of periodic RVE solves for ``RVEHomogenizedMaterial``: explicit FE^2), internal
    force, and the corrector with the next load (``cib_verlet_correct``).  The lumped mass
    is the row sum of the consistent mass, assembled on the device.  The reference's
    optional velocity-Verlet residual corrector (a surrogate hook) is not supported.
    ``record_fields`` False keeps the per-DOF and per-point histories of the final state
    only (scalar histories are always complete)."""
    if np.any(np.asarray(dirichlet.values) != 0.0):
        raise ValueError("Material dynamics currently requires homogeneous Dirichlet values.")
    stability = check_explicit_stability(mesh, time_settings)
    if residual_corrector is None and correction_controls is not None:
        raise ValueError("Correction controls require an enabled residual corrector.")
    if residual_corrector is not None:
        raise NotImplementedError("The velocity-Verlet residual corrector is not supported on the GPU path.")
    if kinematics != "three_dimensional":
        raise ValueError("The GPU Hex8 material dynamics supports kinematics='three_dimensional' only.")
    start_time = perf_counter()
    nodes, elements, material = _mesh_fields(mesh)
    ops = operators or MacroOperators(nodes, elements, material.density, dirichlet.dofs)
    lib, dev = ops.lib, ops.device
    dt = float(time_settings.time_step)
    steps = int(time_settings.num_steps)
    lumped = ops.spmv(ops.mass, torch.ones(ops.n, dtype=torch.float64, device=dev))
    fixed = (1 - ops.free).to(torch.uint8).contiguous()
    u = ops.vector(initial_displacement).clone()
    v = ops.vector(initial_velocity).clone()
    u[ops.fixed] = 0.0
    v[ops.fixed] = 0.0
    state = initialize_hex8_material_state(material, int(elements.shape[0]))
    assembly = assemble_hex8_material_response_cached(nodes, elements, material, state, u, u, dt, update_settings,
                                                      ops.cache, False)  # fmt: skip
    external = ops.vector(load_function(0.0))
    a = (external - assembly.internal_force) / lumped
    a[ops.fixed] = 0.0
    current = _StepState(0.0, u, v, a, assembly.state, assembly)
    rec = _Recorder(ops, load_function, record_fields, lumped_mass=lumped, record_state=record_material_state_history)
    rec.record(current, None)
    stream = _native.stream_ptr
    for step in range(steps):
        t1 = (step + 1) * dt
        u1 = torch.empty_like(u)
        _native.check(lib.cib_verlet_predict(ops.n, current.displacement.data_ptr(), current.velocity.data_ptr(),
                                             current.acceleration.data_ptr(), fixed.data_ptr(), dt, u1.data_ptr(),
                                             stream()), "cib_verlet_predict")  # fmt: skip
        asm = assemble_hex8_material_response_cached(nodes, elements, material, current.material_state, u1,
                                                     current.displacement, dt, update_settings, ops.cache, False)  # fmt: skip
        external1 = ops.vector(load_function(t1))
        a1, v1 = torch.empty_like(u), torch.empty_like(u)
        _native.check(lib.cib_verlet_correct(ops.n, external1.data_ptr(), 1.0, asm.internal_force.data_ptr(),
                                             lumped.data_ptr(), fixed.data_ptr(), dt, current.acceleration.data_ptr(),
                                             current.velocity.data_ptr(), a1.data_ptr(), v1.data_ptr(), stream()),
                      "cib_verlet_correct")  # fmt: skip
        dissipation = dt * ops.integrate(asm.dissipation)
        work = float(0.5 * torch.dot(external + external1, u1 - current.displacement))
        current = _StepState(t1, u1, v1, a1, asm.state, asm)
        rec.record(current, _Interval(current, dissipation, work, 0, 0))
        external = external1
        if progress_callback is not None:
            progress_callback({"stage": "material_dynamics", "scheme": "explicit", "accepted_step": step + 1,
                               "nominal_total_steps": steps, "physical_time": t1, "final_time": steps * dt,
                               "newton_iterations": 0, "armijo_backtracks": 0,
                               "elapsed_seconds": perf_counter() - start_time})  # fmt: skip
    del stability  # checked above; the reference returns no integrator diagnostics without a corrector
    return rec.solution(current, perf_counter() - start_time, integrator={})
