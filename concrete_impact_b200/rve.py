"""Periodic Hex8 RVE solve on the GPU (drop-in for the reference's fem.rve).

Mirrors, with the same names, fields, argument meaning and error behaviour:

* ``build_structured_hex8_box`` -- src/fem/mesh/structured.py:36-80
* ``PeriodicConstraint``, ``build_structured_hex8_periodic_constraint``,
  ``compute_periodic_fluctuation_error`` -- src/fem/rve/data.py:24-38, periodic.py:20-169
* ``ArmijoSettings``, ``NonlinearNewtonSettings`` -- src/fem/solvers/data.py:32-94
* ``RVERequest``, ``RVEState``, ``RVEResponse``, ``RVEPathResult``, ``StructuredHex8RVE``,
  ``RVEOperatorCache``, ``RVEExecutionSettings`` -- src/fem/rve/data.py:41-138
* ``RVEEquilibriumError``, ``initialize_rve_state``, ``solve_rve_microequilibrium``,
  ``build_rve_operator_cache`` -- src/fem/rve/solver.py:36-388
* ``iterate_prescribed_rve_path``, ``solve_prescribed_rve_path`` -- src/fem/rve/path.py:47-123

The Newton iteration follows solver.py:62-227 step for step (residual and increment tests,
Armijo residual-merit backtracking, failure reasons).  Each iteration runs the fused
residual kernel, a deterministic periodic gather and a Jacobi-PCG solve of the reduced
tangent on the device (``libcib200.so``); the reference's sparse direct solve is not used.
The GPU solver handles structured periodic boxes (the meshes built by
``build_structured_hex8_box``) whose material is a J2 viscoplastic or linear elastic model
or a ``PhasedMaterialModel`` of those, for one RVE or a batch of RVEs of different sizes.
"""

from __future__ import annotations

import ctypes
import json
import math
import os
from collections.abc import Callable, Iterator
from dataclasses import dataclass, field
from pathlib import Path
from time import perf_counter
from typing import Any, Literal

import numpy as np
import torch
from scipy.sparse import coo_matrix, csr_matrix

from . import _native
from .materials import (
    J2ViscoplasticMaterial,
    LinearElasticMaterial,
    MaterialPointConvergenceError,
    MaterialPointRequest,
    MaterialResponseRequirements,
    MaterialState,
    MaterialUpdateSettings,
    PhasedMaterialModel,
    _j2_failure,
    _Io,
    encode_phase_state_key,
)

MAX_PHASES = 8
NOUT = 130
# slots of the per-RVE reduction (csrc/rve.cuh)
RS_SIGMA, RS_PSI, RS_DISS, RS_MICRO_WORK, RS_POS_WORK, RS_NEG_WORK = 0, 6, 7, 8, 9, 10
RS_UNLOAD, RS_ACTIVE, RS_EQPS, RS_VW, RS_FNORM2, RS_FACE, RS_PERIODIC, RS_PHASE = 11, 12, 13, 14, 20, 21, 39, 40
RS_PHASE_STRIDE = 10
RS_MARGIN_MIN, RS_MARGIN_MAX, RS_QMAX = 120, 121, 122


# --------------------------------------------------------------------------------------
# Mesh and periodic constraint (host set-up, once per RVE geometry).


def build_structured_hex8_box(lengths: tuple[float, float, float], divisions: tuple[int, int, int]):
    """Tensor-product Hex8 box: lexicographic nodes i + (nx+1)(j + (ny+1)k), elements likewise."""
    nx, ny, nz = divisions
    xs = np.linspace(0.0, lengths[0], nx + 1)
    ys = np.linspace(0.0, lengths[1], ny + 1)
    zs = np.linspace(0.0, lengths[2], nz + 1)
    zz, yy, xx = np.meshgrid(zs, ys, xs, indexing="ij")
    nodes = np.column_stack([xx.ravel(), yy.ravel(), zz.ravel()])
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()

    def nid(a, b, c):
        return a + (nx + 1) * (b + (ny + 1) * c)

    elements = np.column_stack([
        nid(i, j, k), nid(i + 1, j, k), nid(i, j + 1, k), nid(i + 1, j + 1, k),
        nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i, j + 1, k + 1), nid(i + 1, j + 1, k + 1),
    ]).astype(np.int64)  # fmt: skip
    return nodes, elements


@dataclass(frozen=True)
class PeriodicConstraint:
    """Exact periodic elimination operators for one structured box."""

    transformation: csr_matrix
    affine_matrix: np.ndarray
    equivalence_class_ids: np.ndarray
    representative_nodes: np.ndarray
    reference_class: int
    divisions: tuple[int, int, int]
    opposite_face_nodes: tuple


def build_structured_hex8_periodic_constraint(nodes: np.ndarray, divisions: tuple[int, int, int]) -> PeriodicConstraint:
    """Periodic classes (i%nx) + nx((j%ny) + ny(k%nz)), T without the reference class, affine A."""
    nx, ny, nz = divisions
    expected = (nx + 1) * (ny + 1) * (nz + 1)
    if nodes.shape != (expected, 3):
        raise ValueError("Structured periodic constraint received an incompatible node array.")
    if min(divisions) <= 0:
        raise ValueError("Structured periodic constraint requires positive divisions.")
    kk, jj, ii = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
    class_ids = (ii % nx) + nx * ((jj % ny) + ny * (kk % nz))
    faces = []
    for axis, idx in enumerate((ii, jj, kk)):
        faces.append((np.flatnonzero(idx == 0), np.flatnonzero(idx == divisions[axis])))
    return build_periodic_constraint_from_classes(nodes, class_ids, divisions, tuple(faces))


def build_periodic_constraint_from_classes(nodes, class_ids, divisions, opposite_face_nodes) -> PeriodicConstraint:
    """Elimination operators from topology-provided classes (periodic.py:50-104)."""
    unique, normalized = np.unique(class_ids, return_inverse=True)
    if unique.size == 0:
        raise ValueError("Periodic constraint requires at least one equivalence class.")
    class_ids = normalized.astype(np.int64)
    count = unique.size
    representatives = np.full(count, -1, dtype=np.int64)
    first = np.unique(class_ids, return_index=True)[1]
    representatives[class_ids[first]] = first
    reference_class = int(class_ids[opposite_face_nodes[0][0][0]])
    reduced = np.full(count, -1, dtype=np.int64)
    keep = np.arange(count) != reference_class
    reduced[keep] = np.arange(count - 1)
    node_ids = np.flatnonzero(class_ids != reference_class)
    rows = (3 * node_ids[:, None] + np.arange(3)[None, :]).ravel()
    cols = (3 * reduced[class_ids[node_ids]][:, None] + np.arange(3)[None, :]).ravel()
    t = coo_matrix((np.ones(rows.size), (rows, cols)), shape=(3 * nodes.shape[0], 3 * (count - 1))).tocsr()
    return PeriodicConstraint(t, _build_affine_matrix(nodes), class_ids, representatives, reference_class,
                              tuple(divisions), tuple(opposite_face_nodes))  # fmt: skip


def _build_affine_matrix(nodes: np.ndarray) -> np.ndarray:
    """Nodal map of engineering strain (xx, yy, zz, yz, xz, xy) to displacement (periodic.py:153-169)."""
    rel = nodes - np.min(nodes, axis=0)
    x, y, z = rel[:, 0], rel[:, 1], rel[:, 2]
    a = np.zeros((3 * nodes.shape[0], 6))
    a[0::3, 0], a[0::3, 4], a[0::3, 5] = x, 0.5 * z, 0.5 * y
    a[1::3, 1], a[1::3, 3], a[1::3, 5] = y, 0.5 * z, 0.5 * x
    a[2::3, 2], a[2::3, 3], a[2::3, 4] = z, 0.5 * y, 0.5 * x
    return a


def compute_periodic_fluctuation_error(displacement, macro_strain, constraint: PeriodicConstraint) -> float:
    """Largest mismatch of the fluctuation within each periodic class."""
    fluctuation = (np.asarray(displacement) - constraint.affine_matrix @ np.asarray(macro_strain)).reshape(-1, 3)
    rep = constraint.representative_nodes[constraint.equivalence_class_ids]
    return float(np.max(np.linalg.norm(fluctuation - fluctuation[rep], axis=1), initial=0.0))


# --------------------------------------------------------------------------------------
# Settings and containers.


@dataclass(frozen=True)
class ArmijoSettings:
    """Residual-merit Armijo line-search settings."""

    enabled: bool = False
    sufficient_decrease: float = 1.0e-4
    reduction_factor: float = 0.5
    max_backtracks: int = 20

    def __post_init__(self) -> None:
        if not 0.0 < self.sufficient_decrease < 1.0:
            raise ValueError("Armijo sufficient_decrease must lie in (0, 1).")
        if not 0.0 < self.reduction_factor < 1.0:
            raise ValueError("Armijo reduction_factor must lie in (0, 1).")
        if self.max_backtracks < 0:
            raise ValueError("Armijo max_backtracks must be nonnegative.")


@dataclass(frozen=True)
class NonlinearNewtonSettings:
    """Scaled Newton convergence settings."""

    max_iterations: int
    residual_absolute_tolerance: float
    residual_relative_tolerance: float
    increment_absolute_tolerance: float
    increment_relative_tolerance: float
    armijo: ArmijoSettings = field(default_factory=ArmijoSettings)


@dataclass(frozen=True)
class LinearSolverOptions:
    """Matrix-free PCG controls of the reduced tangent solves (no reference counterpart:
    the reference solves directly).  ``relative_tolerance`` None picks 1e-11 for float64
    element kernels and 1e-6 for float32.  ``cluster`` is the number of CTAs (1, 2, 4, 8;
    one thread-block cluster) that share each linear system, or "auto" for a choice from
    the batch's RVE sizes; ``tune_pcg_cluster`` measures the choice instead.  ``forcing``
    "eisenstat_walker" solves the Newton systems only as accurately as the Newton
    iteration needs (the relative tolerance follows the residual's decrease, down to
    ``relative_tolerance``); the Newton convergence tests are unchanged."""

    relative_tolerance: float | None = None
    max_iterations: int = 5000
    cluster: int | str = 1
    forcing: str | None = None  # "eisenstat_walker": inexact Newton, see solve_batch_step


@dataclass(frozen=True)
class RVERequest:
    """One strain-driven RVE update request."""

    macro_strain: Any
    time_step: float
    material_update_settings: MaterialUpdateSettings
    requirements: MaterialResponseRequirements = field(default_factory=lambda: MaterialResponseRequirements(tangent=True))


@dataclass(frozen=True)
class RVEState:
    """Committed microstate and converged periodic fluctuation."""

    material_state: MaterialState
    macro_strain: Any
    fluctuation_dofs: Any


@dataclass(frozen=True)
class RVEResponse:
    """Homogenised and microscopic outputs of one RVE update."""

    macro_stress: Any
    effective_tangent: Any | None
    state: RVEState
    displacement: Any
    micro_strains: Any
    micro_stresses: Any
    micro_diagnostics: dict[str, Any]
    free_energy_density: float
    dissipation_density: float
    phase_diagnostics: dict[str, dict[str, Any]]
    diagnostics: dict[str, Any]


@dataclass(frozen=True)
class RVEPathResult:
    """Accepted responses along one macro-strain path."""

    times: Any
    responses: tuple[RVEResponse, ...]
    validation_diagnostics: dict[str, Any] = field(default_factory=dict)


@dataclass(frozen=True)
class StructuredHex8RVE:
    """One structured periodic Hex8 RVE definition."""

    nodes: np.ndarray
    elements: np.ndarray
    divisions: tuple[int, int, int]
    material: Any
    constraint: PeriodicConstraint
    newton_settings: NonlinearNewtonSettings
    element_phase_ids: np.ndarray | None = None
    element_densities: np.ndarray | None = None
    phase_names: tuple[str, ...] = ()
    quadrature_order: int = 2
    hill_mandel_power_scale: float = 1.0


@dataclass(frozen=True)
class RVEOperatorCache:
    """Geometry and phase data reused by one RVE (GPU: the device batch of this RVE)."""

    quadrature_weights: np.ndarray
    volume: float
    point_phase_ids: np.ndarray
    batch: Any = None


@dataclass(frozen=True)
class RVEExecutionSettings:
    """Execution of macro-point RVEs.  On the GPU every macro point of a call is solved in
    one device batch; ``serial`` and ``process_pool`` are accepted for API compatibility
    and run the same batched device path (the worker count is validated as before)."""

    backend: Literal["serial", "process_pool"] = "serial"
    workers: int = 1
    threads_per_worker: int = 1

    def __post_init__(self) -> None:
        if self.workers <= 0:
            raise ValueError("RVE execution workers must be positive.")
        if self.threads_per_worker <= 0:
            raise ValueError("RVE execution threads_per_worker must be positive.")
        if self.backend == "serial" and self.workers != 1:
            raise ValueError("Serial RVE execution requires exactly one worker.")


class RVEEquilibriumError(RuntimeError):
    """A failed periodic microequilibrium solve with diagnostics."""

    def __init__(self, reason: str, diagnostics: dict[str, Any]) -> None:
        super().__init__(f"RVE microequilibrium failed: {reason}.")
        self.reason = reason
        self.diagnostics = diagnostics


# --------------------------------------------------------------------------------------
# Material table of a model.


def _phases_of(model: StructuredHex8RVE) -> tuple[list[tuple[str, Any]], np.ndarray]:
    """(phase name, material) list and the per-element phase ids of the GPU layout."""
    material = model.material
    n_el = model.elements.shape[0]
    if isinstance(material, PhasedMaterialModel):
        point_phase = np.asarray(material.point_phase_ids).reshape(n_el, 8)
        if np.any(point_phase != point_phase[:, :1]):
            raise NotImplementedError("The GPU RVE solver needs one phase per element.")
        phases = [(p.name, p.material) for p in material.phases]
        element_phase = point_phase[:, 0].astype(np.uint8)
    else:
        phases = [("domain", material)]
        element_phase = np.zeros(n_el, dtype=np.uint8)
    if len(phases) > MAX_PHASES:
        raise NotImplementedError(f"At most {MAX_PHASES} phases are supported.")
    for _, mat in phases:
        if not isinstance(mat, (J2ViscoplasticMaterial, LinearElasticMaterial)):
            raise NotImplementedError(f"GPU RVE phases must be J2 viscoplastic or linear elastic, not {type(mat).__name__}.")
    return phases, element_phase


def _phase_struct(mat) -> _native.PhaseMaterialC:
    if isinstance(mat, J2ViscoplasticMaterial):
        return _native.PhaseMaterialC(1, 0, _native.material_struct(mat))
    params = _native.J2VPMaterialC(float(mat.young_modulus), float(mat.poisson_ratio), 1.0, 0.0, 1.0, 1.0, 1.0)
    return _native.PhaseMaterialC(0, 0, params)


def _check_structured(model: StructuredHex8RVE) -> tuple[float, float, float]:
    """Element edge lengths of a structured box mesh (raises for other meshes)."""
    nx, ny, nz = model.divisions
    if min(nx, ny, nz) <= 0:
        raise NotImplementedError("The GPU RVE solver needs a structured box (positive divisions).")
    lengths = np.ptp(model.nodes, axis=0)
    ref_nodes, ref_elements = build_structured_hex8_box(tuple(lengths), (nx, ny, nz))
    origin = np.min(model.nodes, axis=0)
    if model.nodes.shape != ref_nodes.shape or not np.allclose(model.nodes - origin, ref_nodes, rtol=0, atol=1e-12 * max(lengths)):
        raise NotImplementedError("The GPU RVE solver needs the nodes of build_structured_hex8_box.")
    if not np.array_equal(model.elements, ref_elements):
        raise NotImplementedError("The GPU RVE solver needs the element order of build_structured_hex8_box.")
    if model.quadrature_order != 2:
        raise NotImplementedError("The GPU RVE solver uses the 2x2x2 Gauss rule.")
    return float(lengths[0] / nx), float(lengths[1] / ny), float(lengths[2] / nz)


# --------------------------------------------------------------------------------------
# Device batch.


class RVEBatch:
    """Device buffers and kernels for a batch of structured periodic RVEs.

    All RVEs share the phase materials (same model family) but may differ in divisions and
    lengths.  State arrays are SoA over all Gauss points; periodic vectors are float64.
    ``precision`` 64 or 32 selects the element arithmetic (history stays float64).
    ``device_control`` runs each Newton solve without Armijo search as one CUDA graph whose
    iterations are decided on the device (``cib_rve_newton_graph_*``): one launch and one
    read-back per step instead of two host round trips per Newton iteration.
    """

    def __init__(self, models: list[StructuredHex8RVE], precision: int = 64,
                 linear_solver: LinearSolverOptions | None = None, device_control: bool = False) -> None:  # fmt: skip
        if not models:
            raise ValueError("an RVE batch needs at least one model")
        self.device = _native.require_cuda()
        self.lib = _native.load_library()
        self.models = models
        self.precision = int(precision)
        if self.precision not in (32, 64):
            raise ValueError("precision must be 32 or 64")
        self.dtype = torch.float64 if self.precision == 64 else torch.float32
        self.linear = linear_solver or LinearSolverOptions()
        self.rtol = self.linear.relative_tolerance
        if self.rtol is None:
            self.rtol = 1.0e-11 if self.precision == 64 else 1.0e-6
        phases0, _ = _phases_of(models[0])
        self.phases = phases0
        descs, phase_arrays, offsets = [], [], []
        off = 0
        self.max_nxy = 1
        checked: dict[int, tuple] = {}
        for m in models:
            key = id(m)
            if key not in checked:  # a model object repeated in the batch is validated once
                ph, el_phase = _phases_of(m)
                if [type(x[1]) for x in ph] != [type(x[1]) for x in phases0] or [x[1] for x in ph] != [x[1] for x in phases0]:
                    raise ValueError("all RVEs of a batch must share the phase materials")
                checked[key] = (el_phase, _check_structured(m))
            el_phase, (hx, hy, hz) = checked[key]
            nx, ny, nz = m.divisions
            descs.append(_native.RVEDescC(nx, ny, nz, 0, off, hx, hy, hz))
            phase_arrays.append(el_phase)
            offsets.append(off)
            off += nx * ny * nz
            self.max_nxy = max(self.max_nxy, nx * ny)
        self.nrve = len(models)
        self.nelem = off
        self.elem_offsets = np.asarray(offsets, dtype=np.int64)
        self.elem_counts = np.asarray([int(np.prod(m.divisions)) for m in models], dtype=np.int64)
        self.volumes = np.asarray([d.hx * d.hy * d.hz * c for d, c in zip(descs, self.elem_counts)])
        self.cell_volume = np.asarray([d.hx * d.hy * d.hz / 8.0 for d in descs])
        dev, f64 = self.device, torch.float64
        desc_bytes = np.frombuffer(b"".join(bytes(d) for d in descs), dtype=np.uint8)
        self.desc = torch.as_tensor(desc_bytes.copy(), device=dev)
        self.phase = torch.as_tensor(np.concatenate(phase_arrays), device=dev)
        g = 8 * self.nelem
        n3 = 3 * self.nelem

        def z(*shape, dtype=f64):
            return torch.zeros(shape, dtype=dtype, device=dev)

        # committed and trial Gauss-point state
        self.ep_n, self.q_n, self.vpm_n = z(6, g, dtype=self.dtype), z(g), z(g)
        self.ep, self.q, self.vpm = z(6, g, dtype=self.dtype), z(g), z(g)
        self.stress = z(6, g, dtype=self.dtype)
        self.tparam = z(8, g, dtype=self.dtype)
        self.tflag = z(g, dtype=torch.uint8)
        self.fe, self.de = z(24 * self.nelem), z(24 * self.nelem)
        # periodic vectors
        self.w_n, self.w, self.w_out = z(n3), z(n3), z(n3)
        self.res, self.dinv = z(n3), z(n3)
        self.x, self.r, self.p, self.Ap = z(n3), z(n3), z(n3), z(n3)
        self.macro, self.macro_n, self.dt = z(self.nrve, 6), z(self.nrve, 6), z(self.nrve)
        self.alpha = z(self.nrve)
        self.active = torch.ones(self.nrve, dtype=torch.int32, device=dev)
        self.fail = torch.empty(self.nrve, dtype=torch.int64, device=dev)
        self.rnorm2, self.wnorm2, self.class_max = z(self.nrve), z(self.nrve), z(self.nrve)
        self.pcg_status = torch.zeros(self.nrve, dtype=torch.int32, device=dev)
        self.pcg_iters = torch.zeros(self.nrve, dtype=torch.int32, device=dev)
        self.pcg_rel, self.pcg_xnorm = z(self.nrve), z(self.nrve)
        self.sums = z(self.nrve, NOUT)
        self.sys_rve = torch.arange(self.nrve, dtype=torch.int32, device=dev)
        self.sys_off = torch.as_tensor(3 * self.elem_offsets, device=dev)
        self._tangent_buffers = None
        self.settings = MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)
        self.min_nz = int(min(m.divisions[2] for m in models))
        c = self.linear.cluster
        self.cluster = auto_pcg_cluster(self) if c == "auto" else self.check_cluster(int(c))
        self._batch_struct = None
        self.pcg_shape = 0
        self.device_control = bool(device_control)
        self.live_mask = torch.ones(self.nrve, dtype=torch.int32, device=dev)
        self._graphs: dict = {}

    # -- C structs ---------------------------------------------------------------------
    def batch_struct(self, settings: MaterialUpdateSettings, prefix: int | None = None) -> _native.RVEBatchC:
        """The C view of the batch; ``prefix`` restricts it to RVEs [0, prefix) (the kernels
        that cover every element or node of a batch then launch over that range only)."""
        b = _native.RVEBatchC()
        m = self.nrve if prefix is None else int(prefix)
        b.nrve = m
        b.nphase = len(self.phases)
        b.nelem = self.nelem if m == self.nrve else int(self.elem_offsets[m]) if m < self.nrve else self.nelem
        b.point_stride = 8 * self.nelem  # the Gauss-point arrays keep the whole batch's layout
        b.precision = self.precision
        b.max_nxy = self.max_nxy
        b.desc = self.desc.data_ptr()
        b.phase = self.phase.data_ptr()
        for i, (_, mat) in enumerate(self.phases):
            b.mats[i] = _phase_struct(mat)
        b.settings = _native.settings_struct(settings)
        b.plastic_strain_n = self.ep_n.data_ptr()
        b.eqps_n = self.q_n.data_ptr()
        b.vpm_n = self.vpm_n.data_ptr()
        b.plastic_strain = self.ep.data_ptr()
        b.eqps = self.q.data_ptr()
        b.vpm = self.vpm.data_ptr()
        b.stress = self.stress.data_ptr()
        b.tparam = self.tparam.data_ptr()
        b.tflag = self.tflag.data_ptr()
        b.fe = self.fe.data_ptr()
        b.de = self.de.data_ptr()
        return b

    # -- kernels -----------------------------------------------------------------------
    def residual(self, b, w: torch.Tensor, dw: torch.Tensor | None, alpha: torch.Tensor | None) -> None:
        self.fail.fill_(-1)
        code = self.lib.cib_rve_residual(
            ctypes.byref(b), self.dt.data_ptr(), self.macro.data_ptr(), w.data_ptr(), _native.ptr(dw),
            _native.ptr(alpha), self.active.data_ptr(), self.fail.data_ptr(), _native.stream_ptr(),
        )  # fmt: skip
        _native.check(code, "cib_rve_residual")
        code = self.lib.cib_rve_gather(
            ctypes.byref(b), w.data_ptr(), _native.ptr(dw), _native.ptr(alpha), self.active.data_ptr(),
            self.res.data_ptr(), self.dinv.data_ptr(), self.rnorm2.data_ptr(), self.wnorm2.data_ptr(),
            self.class_max.data_ptr(), self.w_out.data_ptr(), _native.stream_ptr(),
        )  # fmt: skip
        _native.check(code, "cib_rve_gather")

    def pcg_launch(self) -> int:
        """The ``cluster`` argument of cib_rve_pcg_cluster: CTAs per system in bits 0-3, the
        launch shape (threads per CTA / register cap) in bits 4-7."""
        return int(self.cluster) | (int(self.pcg_shape) << 4)

    def check_cluster(self, cluster: int) -> int:
        if cluster not in (1, 2, 4, 8):
            raise ValueError("the PCG cluster size must be 1, 2, 4 or 8")
        if cluster > self.min_nz:
            raise ValueError(f"PCG cluster {cluster} needs every RVE to have at least {cluster} element layers in z")
        return cluster

    def pcg(self, b, rhs: torch.Tensor, x, r, p, Ap, nsys: int, sys_rve, sys_off, status, iters, rel, xnorm,
            rtol: float | None = None) -> None:  # fmt: skip
        code = self.lib.cib_rve_pcg_cluster(
            ctypes.byref(b), nsys, sys_rve.data_ptr(), sys_off.data_ptr(), self.active.data_ptr(), rhs.data_ptr(),
            self.dinv.data_ptr(), x.data_ptr(), r.data_ptr(), p.data_ptr(), Ap.data_ptr(),
            float(self.rtol if rtol is None else rtol),
            int(self.linear.max_iterations), self.pcg_launch(), status.data_ptr(), iters.data_ptr(), rel.data_ptr(),
            xnorm.data_ptr(), _native.stream_ptr(),
        )  # fmt: skip
        _native.check(code, "cib_rve_pcg_cluster")

    def effective_tangent(self, b) -> torch.Tensor:
        """(R, 6, 6) condensed tangent of the last residual pass (solver.py:438-461)."""
        if self._tangent_buffers is None:
            dev = self.device
            n18 = 18 * self.nelem
            zz = lambda n: torch.zeros(n, dtype=torch.float64, device=dev)  # noqa: E731
            sys_rve = torch.arange(self.nrve, dtype=torch.int32, device=dev).repeat_interleave(6)
            offs = torch.as_tensor(
                np.concatenate([18 * o + 3 * c * np.arange(6) for o, c in zip(self.elem_offsets, self.elem_counts)]),
                device=dev,
            )
            self._tangent_buffers = {
                "fe6": zz(6 * 24 * self.nelem), "rhs": zz(n18), "x": zz(n18), "r": zz(n18), "p": zz(n18),
                "Ap": zz(n18), "kee": zz(36 * self.nrve), "ceff": zz(36 * self.nrve), "sys_rve": sys_rve,
                "sys_off": offs, "status": torch.zeros(6 * self.nrve, dtype=torch.int32, device=dev),
                "iters": torch.zeros(6 * self.nrve, dtype=torch.int32, device=dev), "rel": zz(6 * self.nrve),
                "xnorm": zz(6 * self.nrve),
            }  # fmt: skip
        t = self._tangent_buffers
        code = self.lib.cib_rve_tangent_rhs(ctypes.byref(b), self.active.data_ptr(), t["fe6"].data_ptr(),
                                            t["rhs"].data_ptr(), t["kee"].data_ptr(), _native.stream_ptr())  # fmt: skip
        _native.check(code, "cib_rve_tangent_rhs")
        self.pcg(b, t["rhs"], t["x"], t["r"], t["p"], t["Ap"], 6 * self.nrve, t["sys_rve"], t["sys_off"], t["status"],
                 t["iters"], t["rel"], t["xnorm"])  # fmt: skip
        code = self.lib.cib_rve_tangent_finish(ctypes.byref(b), self.active.data_ptr(), t["rhs"].data_ptr(),
                                               t["x"].data_ptr(), t["kee"].data_ptr(), t["ceff"].data_ptr(),
                                               _native.stream_ptr())  # fmt: skip
        _native.check(code, "cib_rve_tangent_finish")
        return t["ceff"].view(self.nrve, 6, 6)

    def response(self, b, w: torch.Tensor, point_out: torch.Tensor | None, diag: torch.Tensor | None) -> None:
        code = self.lib.cib_rve_response(
            ctypes.byref(b), self.dt.data_ptr(), self.macro.data_ptr(), self.macro_n.data_ptr(), w.data_ptr(),
            self.w_n.data_ptr(), self.active.data_ptr(), self.sums.data_ptr(), _native.ptr(point_out),
            _native.ptr(diag), _native.stream_ptr(),
        )  # fmt: skip
        _native.check(code, "cib_rve_response")

    def newton_graph(self, newton: NonlinearNewtonSettings, update_settings: MaterialUpdateSettings,
                     prefix: int | None = None) -> "_NewtonGraph":  # fmt: skip
        """The device-controlled Newton graph for these settings (built once, then reused;
        the PCG cluster size and tolerances in force and the RVE prefix it covers are part
        of the key)."""
        prefix = self.nrve if prefix is None else int(prefix)
        key = (tuple(_newton_key(newton)), repr(update_settings), self.pcg_launch(), float(self.rtol),
               int(self.linear.max_iterations), self.linear.forcing, prefix)  # fmt: skip
        graph = self._graphs.get(key)
        if graph is None:
            graph = _NewtonGraph(self, newton, update_settings, prefix)
            self._graphs[key] = graph
        return graph

    def save_state(self, path) -> None:
        """Write the committed state of every RVE (history, fluctuation, macro strain) to an
        .npz file, for resuming long runs."""
        np.savez(path, ep_n=self.ep_n.cpu().numpy(), q_n=self.q_n.cpu().numpy(), vpm_n=self.vpm_n.cpu().numpy(),
                 w_n=self.w_n.cpu().numpy(), macro_n=self.macro_n.cpu().numpy(),
                 elem_counts=self.elem_counts, precision=self.precision)  # fmt: skip

    def load_state(self, path) -> None:
        """Restore a committed state written by ``save_state`` for the same batch layout."""
        data = np.load(path)
        if not np.array_equal(data["elem_counts"], self.elem_counts) or int(data["precision"]) != self.precision:
            raise ValueError("the saved state belongs to a batch of another layout or precision")
        for name in ("ep_n", "q_n", "vpm_n", "w_n", "macro_n"):
            getattr(self, name).copy_(torch.as_tensor(data[name], device=self.device))

    def commit(self) -> None:
        """Accept the trial state of every RVE as the committed state."""
        self.ep_n.copy_(self.ep)
        self.q_n.copy_(self.q)
        self.vpm_n.copy_(self.vpm)
        self.w_n.copy_(self.w)
        self.macro_n.copy_(self.macro)


def _live_prefix(batch: RVEBatch, live_mask) -> int:
    """Smallest power of two (capped at the batch size) covering every live RVE: a fallback
    pool whose first slots are in use launches over those slots only."""
    if live_mask is None:
        return batch.nrve
    live = np.flatnonzero(np.asarray(live_mask, dtype=bool))
    if live.size == 0:
        return min(1, batch.nrve)
    need = int(live[-1]) + 1
    return min(batch.nrve, 1 << (need - 1).bit_length())


# --------------------------------------------------------------------------------------
# Device-controlled Newton solve: one CUDA graph per step (csrc/rve_newton.cu).

_CTL = 16  # control words ahead of the per-RVE records in the graph's workspaces


def _newton_key(newton: NonlinearNewtonSettings) -> list:
    return [int(newton.max_iterations), float(newton.residual_absolute_tolerance),
            float(newton.residual_relative_tolerance), float(newton.increment_absolute_tolerance),
            float(newton.increment_relative_tolerance)]  # fmt: skip


class _NewtonGraph:
    """Workspaces and the instantiated graph of ``cib_rve_newton_graph_create``."""

    def __init__(self, batch: RVEBatch, newton: NonlinearNewtonSettings, update_settings: MaterialUpdateSettings,
                 prefix: int) -> None:  # fmt: skip
        lib = batch.lib
        self.prefix = prefix
        n_int, n_double = ctypes.c_int64(), ctypes.c_int64()
        lib.cib_rve_newton_workspace(prefix, ctypes.byref(n_int), ctypes.byref(n_double))
        dev = batch.device
        self.iwork = torch.zeros(n_int.value, dtype=torch.int32, device=dev)
        self.dwork = torch.zeros(n_double.value, dtype=torch.float64, device=dev)
        self.batch = batch
        self.b = batch.batch_struct(update_settings, prefix)
        s = _native.RVENewtonC()
        s.max_iterations = int(newton.max_iterations)
        s.inexact = 1 if batch.linear.forcing == "eisenstat_walker" else 0
        s.residual_absolute_tolerance = float(newton.residual_absolute_tolerance)
        s.residual_relative_tolerance = float(newton.residual_relative_tolerance)
        s.increment_absolute_tolerance = float(newton.increment_absolute_tolerance)
        s.increment_relative_tolerance = float(newton.increment_relative_tolerance)
        s.pcg_rtol = float(batch.rtol)
        s.pcg_maxit = int(batch.linear.max_iterations)
        s.cluster = batch.pcg_launch()
        for name, tensor in (("time_step", batch.dt), ("macro", batch.macro), ("w_n", batch.w_n), ("w", batch.w),
                             ("w_out", batch.w_out), ("x", batch.x), ("r", batch.r), ("p", batch.p), ("Ap", batch.Ap),
                             ("residual", batch.res), ("dinv", batch.dinv), ("rnorm2", batch.rnorm2),
                             ("wnorm2", batch.wnorm2), ("class_max", batch.class_max), ("alpha", batch.alpha),
                             ("active", batch.active), ("live_mask", batch.live_mask), ("fail", batch.fail),
                             ("sys_rve", batch.sys_rve), ("sys_off", batch.sys_off), ("pcg_status", batch.pcg_status),
                             ("pcg_iterations", batch.pcg_iters), ("pcg_rel_residual", batch.pcg_rel),
                             ("pcg_xnorm", batch.pcg_xnorm), ("iwork", self.iwork), ("dwork", self.dwork)):  # fmt: skip
            setattr(s, name, tensor.data_ptr())
        self.struct = s
        handle = ctypes.c_void_p()
        torch.cuda.synchronize()
        _native.check(lib.cib_rve_newton_graph_create(ctypes.byref(self.b), ctypes.byref(s), ctypes.byref(handle)),
                      "cib_rve_newton_graph_create")  # fmt: skip
        self.handle = handle
        self.lib = lib

    def launch(self) -> None:
        _native.check(self.lib.cib_rve_newton_graph_launch(self.handle, _native.stream_ptr()),
                      "cib_rve_newton_graph_launch")  # fmt: skip

    def __del__(self) -> None:
        handle = getattr(self, "handle", None)
        if handle is not None and handle.value:
            self.lib.cib_rve_newton_graph_destroy(handle)
            self.handle = None


def _solve_batch_step_graph(batch: RVEBatch, newton: NonlinearNewtonSettings, update_settings: MaterialUpdateSettings,
                            failure_context, live_mask) -> BatchStepResult:  # fmt: skip
    """solve_batch_step on the device: one graph launch, one read-back of the records."""
    R = batch.nrve
    prefix = _live_prefix(batch, live_mask)
    graph = batch.newton_graph(newton, update_settings, prefix)
    if live_mask is None:
        batch.live_mask.fill_(1)
    else:
        batch.live_mask.copy_(torch.as_tensor(np.asarray(live_mask, dtype=np.int32), device=batch.device))
    graph.launch()
    if prefix < R:  # RVEs beyond the prefix take no part: inactive, as in the host loop
        batch.active[prefix:] = 0
    iw = graph.iwork.cpu().numpy()
    R = prefix
    batch.last_graph_iterations = int(iw[0])  # loop bodies run (for launch accounting)
    dw = graph.dwork.cpu().numpy()
    its, pcg = iw[_CTL : _CTL + R].astype(np.int64), iw[_CTL + R : _CTL + 2 * R].astype(np.int64)
    rnorm, tol = dw[_CTL : _CTL + R], dw[_CTL + R : _CTL + 2 * R]
    inc, inc_tol = dw[_CTL + 2 * R : _CTL + 3 * R], dw[_CTL + 3 * R : _CTL + 4 * R]
    error, r, info = int(iw[1]), int(iw[2]), int(iw[3])
    if error == 1:
        if failure_context is not None:
            raise failure_context(r, info)
        raise MaterialPointConvergenceError("RVE material point failed.", "material_point_failure",
                                            {"rve_index": r, "point_id": info})  # fmt: skip
    if error == 3:  # found by the check of the last iteration; the loop counter was advanced after it
        raise RVEEquilibriumError("maximum_iterations_exceeded", _failure_diag(batch, r, int(iw[0]) - 1, rnorm[r],
                                                                               tol[r], inc[r], inc_tol[r]))  # fmt: skip
    if error == 2:
        d = _failure_diag(batch, r, int(iw[0]) - 1, rnorm[r], tol[r], float(inc[r]), inc_tol[r])
        d["linear_solver_status"] = info
        raise RVEEquilibriumError("non_finite_increment", d)
    full = batch.nrve
    live = np.ones(full, dtype=bool) if live_mask is None else np.asarray(live_mask, dtype=bool)

    def padded(v, dtype=None):  # per-RVE records of the whole batch (zeros beyond the prefix)
        out = np.zeros(full, dtype=dtype or v.dtype)
        out[:R] = v
        return out

    return BatchStepResult(padded(its), np.zeros(full, dtype=np.int64), np.where(live, padded(rnorm), 0.0),
                           np.where(live, padded(tol), 0.0), padded(pcg))  # fmt: skip


# --------------------------------------------------------------------------------------
# Newton driver (solver.py:62-227), vectorised over the RVEs of a batch.


@dataclass
class BatchStepResult:
    """Per-RVE outcome of one batched step (arrays of length R)."""

    newton_iterations: np.ndarray
    armijo_backtracks: np.ndarray
    residual_norm: np.ndarray
    residual_tolerance: np.ndarray
    pcg_iterations: np.ndarray
    sums: np.ndarray | None = None
    effective_tangent: torch.Tensor | None = None


def solve_batch_step(
    batch: RVEBatch,
    newton: NonlinearNewtonSettings,
    update_settings: MaterialUpdateSettings,
    need_tangent: bool,
    point_out: torch.Tensor | None = None,
    diag: torch.Tensor | None = None,
    failure_context: Callable[[int, int], Exception] | None = None,
    live_mask: np.ndarray | None = None,
    timers: dict | None = None,
) -> BatchStepResult:
    """Solve the microequilibrium of every RVE of the batch from its committed state.

    ``batch.macro`` / ``batch.dt`` hold the request; ``batch.w`` starts at the committed
    fluctuation.  On success the trial state of every RVE is its converged state (not yet
    committed).  ``live_mask`` restricts the solve to some RVEs; the others are left
    untouched and stay inactive (``batch.active``) for the response and tangent kernels.
    ``timers``, when given, collects CUDA event pairs around the residual and PCG launches
    (keys "residual", "pcg"; read them after a synchronize).
    """
    if batch.device_control and not newton.armijo.enabled and timers is None:
        return _solve_batch_step_graph(batch, newton, update_settings, failure_context, live_mask)
    R = batch.nrve
    prefix = _live_prefix(batch, live_mask)
    b = batch.batch_struct(update_settings, prefix)
    batch.w.copy_(batch.w_n)
    done = np.zeros(R, dtype=bool) if live_mask is None else ~np.asarray(live_mask, dtype=bool)
    final_active = None if live_mask is None else np.asarray(live_mask, dtype=bool).copy()
    init_norm = np.full(R, np.nan)
    last_inc = np.full(R, np.inf)
    backtracks = np.zeros(R, dtype=np.int64)
    iters_out = np.zeros(R, dtype=np.int64)
    res_out = np.zeros(R)
    tol_out = np.zeros(R)
    pcg_total = np.zeros(R, dtype=np.int64)
    _set_active(batch, ~done)
    ns = newton
    inexact = batch.linear.forcing == "eisenstat_walker"
    if batch.linear.forcing not in (None, "eisenstat_walker"):
        raise ValueError(f"unknown forcing {batch.linear.forcing!r}")
    prev_rnorm = np.full(R, np.nan)
    eta = 0.1
    for iteration in range(ns.max_iterations + 1):
        _timed(timers, "residual", lambda: batch.residual(b, batch.w, None, None))
        rn2, wn2, fail = (t.cpu().numpy() for t in (batch.rnorm2, batch.wnorm2, batch.fail))
        live = ~done
        _raise_material_failure(batch, fail, live, failure_context)
        rnorm = np.sqrt(rn2)
        first = np.isnan(init_norm) & live
        init_norm[first] = rnorm[first]
        tol = np.maximum(ns.residual_absolute_tolerance, ns.residual_relative_tolerance * init_norm)
        inc_tol = np.maximum(ns.increment_absolute_tolerance, ns.increment_relative_tolerance * np.maximum(np.sqrt(wn2), 1.0))
        conv = live & (rnorm <= tol) & ((iteration == 0) | (last_inc <= inc_tol))
        _finish(batch, conv, done, iteration, rnorm, tol, iters_out, res_out, tol_out)
        live = ~done
        if not live.any():
            break
        if iteration == ns.max_iterations:
            r = int(np.flatnonzero(live)[0])
            raise RVEEquilibriumError("maximum_iterations_exceeded", _failure_diag(batch, r, iteration, rnorm[r], tol[r],
                                                                                   last_inc[r], inc_tol[r]))  # fmt: skip
        _set_active(batch, live)
        rtol = None
        if inexact:
            # Eisenstat-Walker choice 2 (gamma 0.9, alpha 2) over the live RVEs, with its
            # safeguard, capped at 0.1 and floored at the solver's own tolerance
            seen = live & np.isfinite(prev_rnorm) & (prev_rnorm > 0)
            if seen.any():
                ratio = float(np.max(rnorm[seen] / prev_rnorm[seen]))
                new_eta = 0.9 * ratio**2
                if 0.9 * eta**2 > 0.1:
                    new_eta = max(new_eta, 0.9 * eta**2)
                eta = min(new_eta, 0.1)
            rtol = max(float(batch.rtol), eta)
        prev_rnorm = np.where(live, rnorm, prev_rnorm)
        _timed(timers, "pcg", lambda: batch.pcg(b, batch.res, batch.x, batch.r, batch.p, batch.Ap, prefix, batch.sys_rve,
                                                batch.sys_off, batch.pcg_status, batch.pcg_iters, batch.pcg_rel,
                                                batch.pcg_xnorm, rtol))  # fmt: skip
        status, piters, xnorm = (t.cpu().numpy() for t in (batch.pcg_status, batch.pcg_iters, batch.pcg_xnorm))
        pcg_total[live] += piters[live]
        bad = live & ((status == 2) | ~np.isfinite(xnorm))
        if bad.any():
            r = int(np.flatnonzero(bad)[0])
            d = _failure_diag(batch, r, iteration, rnorm[r], tol[r], float(xnorm[r]), inc_tol[r])
            d["linear_solver_status"] = int(status[r])
            raise RVEEquilibriumError("non_finite_increment", d)
        # increment dw = -x; second convergence test uses the unapplied increment
        conv2 = live & (rnorm <= tol) & (xnorm <= inc_tol)
        _finish(batch, conv2, done, iteration, rnorm, tol, iters_out, res_out, tol_out, restore=True)
        live = ~done
        if not live.any():
            break
        steps = np.ones(R)
        if ns.armijo.enabled:
            steps, bts = _armijo(batch, b, live, rnorm, ns.armijo, iteration, tol, xnorm, inc_tol)
            backtracks[live] += bts[live]
        alpha = torch.as_tensor(np.where(live, -steps, 0.0), device=batch.device)
        batch.alpha.copy_(alpha)
        _set_active(batch, live)
        _axpy_commit(batch, b)
        last_inc = np.where(live, steps * xnorm, last_inc)
    if final_active is None:
        batch.active.fill_(1)
    else:
        _set_active(batch, final_active)
    return BatchStepResult(iters_out, backtracks, res_out, tol_out, pcg_total)


def auto_pcg_cluster(batch: RVEBatch) -> int:
    """Cluster size from the batch's sizes: doubled while the largest RVE has at least
    2 x 1,728 elements (a 12^3 block) per CTA, at most 8 and at most the smallest number
    of z layers."""
    largest = int(batch.elem_counts.max())
    c = 1
    while c < 8 and 2 * c <= batch.min_nz and largest >= 1728 * 2 * c:
        c *= 2
    return c


PCG_SHAPES = {0: "256 threads, default register cap", 1: "128 threads, 4 (FP64: 2) CTAs per SM",
              2: "512 threads, 1 CTA per SM", 3: "256 threads, the other register cap (FP32: 1, FP64: 2 CTAs per SM)"}


def _tuning_path() -> Path:
    base = os.environ.get("CIB_TUNING_CACHE")
    if base:
        return Path(base)
    return Path(os.environ.get("XDG_CACHE_HOME", Path.home() / ".cache")) / "cib200" / "pcg_tuning.json"


def _edge_mix_key(batch: RVEBatch) -> str:
    """The tuning key of a batch: precision, GPU name and the multiset of RVE divisions."""
    mix: dict[str, int] = {}
    for m in batch.models:
        d = "x".join(str(int(v)) for v in m.divisions)
        mix[d] = mix.get(d, 0) + 1
    name = torch.cuda.get_device_name(batch.device)
    return f"f{batch.precision}|{name}|" + ",".join(f"{k}:{mix[k]}" for k in sorted(mix))


def tune_pcg_cluster(batch: RVEBatch, update_settings: MaterialUpdateSettings, candidates=(1, 2, 4, 8),
                     shapes=(0, 1, 2, 3), persist: bool = True) -> dict:  # fmt: skip
    """Time one PCG solve of the batch's current Newton system (a residual pass at the
    committed fluctuation) for every admissible cluster size x launch shape (threads per
    CTA and register cap, ``PCG_SHAPES``; shapes apply to cluster sizes above 1) and keep
    the fastest.  The solves write only work vectors; the batch's state is unchanged.
    With ``persist`` the choice is stored per edge mix (precision, GPU, RVE divisions) in
    a JSON file (``$CIB_TUNING_CACHE``, else ``~/.cache/cib200/pcg_tuning.json``) and a
    later call for the same mix takes it from there without timing.  Returns
    {"cluster": c, "shape": s, "ms": {"c/s": milliseconds}, "cached": bool, "key": key}."""
    key = _edge_mix_key(batch)
    path = _tuning_path()
    table = {}
    if persist and path.exists():
        try:
            table = json.loads(path.read_text())
        except ValueError:
            table = {}
    hit = table.get(key)
    if persist and hit and hit["cluster"] in candidates and hit["cluster"] <= batch.min_nz and hit["shape"] in shapes:
        batch.cluster, batch.pcg_shape = int(hit["cluster"]), int(hit["shape"])
        return {"cluster": batch.cluster, "shape": batch.pcg_shape, "ms": hit.get("ms", {}), "cached": True, "key": key}
    b = batch.batch_struct(update_settings)
    saved = (batch.cluster, batch.pcg_shape)
    batch.w.copy_(batch.w_n)
    batch.residual(b, batch.w, None, None)
    timings: dict[str, float] = {}
    for c in candidates:
        if c > batch.min_nz:
            continue
        for shape in (shapes if c > 1 else (0,)):
            batch.cluster, batch.pcg_shape = c, shape
            for rep in range(2):  # the first run also sets the launch attributes
                start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                start.record()
                batch.pcg(b, batch.res, batch.x, batch.r, batch.p, batch.Ap, batch.nrve, batch.sys_rve, batch.sys_off,
                          batch.pcg_status, batch.pcg_iters, batch.pcg_rel, batch.pcg_xnorm)  # fmt: skip
                end.record()
                torch.cuda.synchronize()
            timings[f"{c}/{shape}"] = start.elapsed_time(end)
    if timings:
        best = min(timings, key=timings.get)
        batch.cluster, batch.pcg_shape = (int(v) for v in best.split("/"))
    else:
        batch.cluster, batch.pcg_shape = saved
    if persist and timings:
        table[key] = {"cluster": batch.cluster, "shape": batch.pcg_shape, "ms": timings}
        try:
            path.parent.mkdir(parents=True, exist_ok=True)
            path.write_text(json.dumps(table, indent=1, sort_keys=True))
        except OSError:
            pass  # a read-only cache location only loses the persistence
    return {"cluster": batch.cluster, "shape": batch.pcg_shape, "ms": timings, "cached": False, "key": key}


def _timed(timers: dict | None, key: str, fn) -> None:
    if timers is None:
        fn()
        return
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    fn()
    end.record()
    timers.setdefault(key, []).append((start, end))


def _set_active(batch: RVEBatch, mask: np.ndarray) -> None:
    batch.active.copy_(torch.as_tensor(mask.astype(np.int32), device=batch.device))


def _axpy_commit(batch: RVEBatch, b) -> None:
    """w <- w + alpha dw (dw = x) for the active RVEs, through the gather kernel's w_out."""
    code = batch.lib.cib_rve_gather(
        ctypes.byref(b), batch.w.data_ptr(), batch.x.data_ptr(), batch.alpha.data_ptr(), batch.active.data_ptr(),
        batch.res.data_ptr(), batch.dinv.data_ptr(), batch.rnorm2.data_ptr(), batch.wnorm2.data_ptr(),
        batch.class_max.data_ptr(), batch.w_out.data_ptr(), _native.stream_ptr(),
    )  # fmt: skip
    _native.check(code, "cib_rve_gather")
    mask = batch.active.bool().repeat_interleave(torch.as_tensor(3 * batch.elem_counts, device=batch.device))
    batch.w.copy_(torch.where(mask, batch.w_out, batch.w))


def _finish(batch, conv, done, iteration, rnorm, tol, iters_out, res_out, tol_out, restore: bool = False) -> None:
    """Mark converged RVEs; their current trial state (last residual pass) is the answer."""
    if not conv.any():
        return
    done |= conv
    iters_out[conv] = iteration
    res_out[conv] = rnorm[conv]
    tol_out[conv] = tol[conv]


def _armijo(batch, b, live, rnorm, settings: ArmijoSettings, iteration, tol, xnorm, inc_tol):
    """Residual-merit backtracking (line_search.py:40-67) for every live RVE at once."""
    R = batch.nrve
    steps = np.ones(R)
    bts = np.zeros(R, dtype=np.int64)
    searching = live.copy()
    merit = 0.5 * rnorm**2
    last = np.full(R, np.inf)
    for backtrack in range(settings.max_backtracks + 1):
        step = settings.reduction_factor**backtrack
        _set_active(batch, searching)
        batch.alpha.copy_(torch.full((R,), -step, dtype=torch.float64, device=batch.device))
        batch.residual(b, batch.w, batch.x, batch.alpha)
        cand = np.sqrt(batch.rnorm2.cpu().numpy())
        last = np.where(searching, cand, last)
        ok = searching & (0.5 * cand**2 <= merit - settings.sufficient_decrease * step * rnorm**2)
        steps[ok] = step
        bts[ok] = backtrack
        searching &= ~ok
        if not searching.any():
            return steps, bts
    r = int(np.flatnonzero(searching)[0])
    d = _failure_diag(batch, r, iteration, rnorm[r], tol[r], float(xnorm[r]), inc_tol[r])
    d["armijo"] = {"current_residual_norm": float(rnorm[r]), "current_merit": float(merit[r]),
                   "last_candidate_residual_norm": float(last[r]), "max_backtracks": settings.max_backtracks}  # fmt: skip
    raise RVEEquilibriumError("armijo_exhausted", d)


def _failure_diag(batch, r, iteration, rnorm, tol, inc, inc_tol) -> dict[str, Any]:
    stress = batch.stress[:, 8 * batch.elem_offsets[r] : 8 * (batch.elem_offsets[r] + batch.elem_counts[r])]
    return {
        "algorithm": "periodic_rve_microequilibrium_newton",
        "macro_strain": batch.macro[r].cpu().tolist(),
        "time_step": float(batch.dt[r].item()),
        "iteration": int(iteration),
        "residual_norm": float(rnorm),
        "residual_tolerance": float(tol),
        "increment_norm": float(inc),
        "increment_tolerance": float(inc_tol),
        "maximum_absolute_stress": float(stress.abs().max().item()),
        "rve_index": int(r),
    }


def _raise_material_failure(batch, fail, live, failure_context) -> None:
    bad = live & (fail != -1)
    if not bad.any():
        return
    r = int(np.flatnonzero(bad)[0])
    local_point = int(fail[r])
    if failure_context is not None:
        raise failure_context(r, local_point)
    raise MaterialPointConvergenceError("RVE material point failed.", "material_point_failure",
                                        {"rve_index": r, "point_id": local_point})  # fmt: skip


# --------------------------------------------------------------------------------------
# Single-RVE drop-in API.


def is_structured_box(model: StructuredHex8RVE) -> bool:
    """True when the model is a structured box of build_structured_hex8_box (the batched
    box path); other meshes take the general-mesh path of ``rve_general``."""
    try:
        _check_structured(model)
    except NotImplementedError:
        return False
    return True


def build_rve_operator_cache(model: StructuredHex8RVE, precision: int = 64,
                             linear_solver: LinearSolverOptions | None = None) -> RVEOperatorCache:  # fmt: skip
    """Geometry, quadrature weights, phase map and the device batch of one RVE (for a
    general mesh: its general-mesh operators, FP64)."""
    if not is_structured_box(model):
        from .rve_general import GeneralRVEOperators

        if precision != 64:
            raise NotImplementedError("General-mesh RVEs are solved in FP64 only.")
        opts = linear_solver or LinearSolverOptions()
        ops = GeneralRVEOperators(model, opts.relative_tolerance or 1.0e-11, opts.max_iterations)
        phase_ids = (np.zeros(model.elements.shape[0], dtype=np.int64) if model.element_phase_ids is None
                     else np.asarray(model.element_phase_ids, dtype=np.int64))  # fmt: skip
        return RVEOperatorCache(ops.weights_host, ops.volume, np.repeat(phase_ids, 8), ops)
    hx, hy, hz = _check_structured(model)
    n_el = model.elements.shape[0]
    weights = np.full(8 * n_el, hx * hy * hz / 8.0)
    phase_ids = (np.zeros(n_el, dtype=np.int64) if model.element_phase_ids is None
                 else np.asarray(model.element_phase_ids, dtype=np.int64))  # fmt: skip
    batch = RVEBatch([model], precision=precision, linear_solver=linear_solver)
    return RVEOperatorCache(weights, float(np.sum(weights)), np.repeat(phase_ids, 8), batch)


def initialize_rve_state(model: StructuredHex8RVE) -> RVEState:
    """Zero committed state: material state of every Gauss point, zero strain and fluctuation."""
    material_state = model.material.initialize_state(8 * model.elements.shape[0])
    independent = model.constraint.transformation.shape[1]
    return RVEState(material_state, np.zeros(6), np.zeros(independent))


def _phase_points(model: StructuredHex8RVE) -> list[np.ndarray]:
    """Global Gauss-point ids of each phase, in the reference's compact order."""
    phases, el_phase = _phases_of(model)
    point_phase = np.repeat(el_phase.astype(np.int64), 8)
    return [np.flatnonzero(point_phase == i) for i in range(len(phases))]


def _load_state(cache: RVEOperatorCache, model: StructuredHex8RVE, state: RVEState) -> _Io:
    """Copy a reference-shaped committed state into the batch's committed buffers."""
    batch: RVEBatch = cache.batch
    io = _Io(state.fluctuation_dofs)
    dev = batch.device
    ep = torch.zeros((8 * batch.nelem, 6), dtype=torch.float64, device=dev)
    q = torch.zeros(8 * batch.nelem, dtype=torch.float64, device=dev)
    vpm = torch.zeros(8 * batch.nelem, dtype=torch.float64, device=dev)
    phases, _ = _phases_of(model)
    points = _phase_points(model)
    variables = state.material_state.variables
    phased = isinstance(model.material, PhasedMaterialModel)
    for (name, mat), ids in zip(phases, points):
        if not isinstance(mat, J2ViscoplasticMaterial):
            continue
        key = (lambda v: encode_phase_state_key(name, v)) if phased else (lambda v: v)
        idx = torch.as_tensor(ids, device=dev)
        ep.index_copy_(0, idx, io.to_device(variables[key("plastic_strain")], (ids.size, 6)))
        q.index_copy_(0, idx, io.to_device(variables[key("equivalent_plastic_strain")], (ids.size,)))
        vpm.index_copy_(0, idx, io.to_device(variables[key("viscoplastic_multiplier")], (ids.size,)))
    batch.ep_n.copy_(ep.T.to(batch.dtype))
    batch.q_n.copy_(q)
    batch.vpm_n.copy_(vpm)
    w = torch.zeros(3 * batch.nelem, dtype=torch.float64, device=dev)
    w[3:] = io.to_device(state.fluctuation_dofs).reshape(-1)
    batch.w_n.copy_(w)
    batch.macro_n[0].copy_(io.to_device(state.macro_strain).reshape(6))
    return io


def _trial_material_state(cache: RVEOperatorCache, model: StructuredHex8RVE, io: _Io) -> MaterialState:
    batch: RVEBatch = cache.batch
    phases, _ = _phases_of(model)
    points = _phase_points(model)
    phased = isinstance(model.material, PhasedMaterialModel)
    ep = batch.ep.T.to(torch.float64)
    out: dict[str, Any] = {}
    for (name, mat), ids in zip(phases, points):
        if not isinstance(mat, J2ViscoplasticMaterial):
            continue
        key = (lambda v: encode_phase_state_key(name, v)) if phased else (lambda v: v)
        idx = torch.as_tensor(ids, device=batch.device)
        out[key("plastic_strain")] = io.out(ep.index_select(0, idx).contiguous())
        out[key("equivalent_plastic_strain")] = io.out(batch.q.index_select(0, idx).contiguous())
        out[key("viscoplastic_multiplier")] = io.out(batch.vpm.index_select(0, idx).contiguous())
    return MaterialState(out)


def solve_rve_microequilibrium(
    model: StructuredHex8RVE,
    request: RVERequest,
    committed_state: RVEState,
    operator_cache: RVEOperatorCache | None = None,
) -> RVEResponse:
    """Solve one strain-driven periodic RVE update from a committed state on the GPU."""
    macro = np.asarray(request.macro_strain.cpu() if isinstance(request.macro_strain, torch.Tensor)
                       else request.macro_strain, dtype=np.float64)  # fmt: skip
    if macro.shape != (6,):
        raise ValueError("RVE macro strain must have shape (6,).")
    if request.time_step <= 0.0:
        raise ValueError("RVE time step must be positive.")
    if operator_cache is None or operator_cache.batch is None:
        operator_cache = build_rve_operator_cache(model)
    if not isinstance(operator_cache.batch, RVEBatch):
        from .rve_general import solve_general_rve_microequilibrium

        return solve_general_rve_microequilibrium(model, request, committed_state, operator_cache.batch)
    batch: RVEBatch = operator_cache.batch
    io = _load_state(operator_cache, model, committed_state)
    batch.macro[0].copy_(torch.as_tensor(macro, device=batch.device))
    batch.dt.fill_(float(request.time_step))
    g = 8 * batch.nelem
    point_out = torch.empty((14, g), dtype=torch.float64, device=batch.device)
    diag = torch.empty((_native.J2_NDIAG, g), dtype=torch.float64, device=batch.device)

    def failure(r: int, local_point: int) -> Exception:
        return _rve_point_failure(model, batch, request, committed_state, local_point, io)

    result = solve_batch_step(batch, model.newton_settings, request.material_update_settings, False,
                              failure_context=failure)  # fmt: skip
    b = batch.batch_struct(request.material_update_settings)
    batch.response(b, batch.w, point_out, diag)
    tangent = None
    if request.requirements.tangent:
        tangent = batch.effective_tangent(b)[0]
    return _build_response(model, operator_cache, request, committed_state, macro, result, 0, point_out, diag,
                           tangent, io)  # fmt: skip


def _rve_point_failure(model, batch: RVEBatch, request, committed_state, local_point: int, io) -> Exception:
    """The reference's MaterialPointConvergenceError for a failed micro point, with the
    element/quadrature context of nonlinear_solid.py:338-348."""
    phases, el_phase = _phases_of(model)
    point_phase = np.repeat(el_phase.astype(np.int64), 8)
    ph = int(point_phase[local_point])
    _, mat = phases[ph]
    # strain of the failing point: ebar + B_q w_e, restated on the host for this one point
    e, q = divmod(local_point, 8)
    nx, ny, nz = model.divisions
    i, j, k = e % nx, (e // nx) % ny, e // (nx * ny)
    hx, hy, hz = _check_structured(model)
    w = batch.w.cpu().numpy()
    ebar = batch.macro[0].cpu().numpy()
    eps = ebar.copy()
    gp = 1.0 / math.sqrt(3.0)
    xi, eta, zeta = (gp if q & 4 else -gp), (gp if q & 2 else -gp), (gp if q & 1 else -gp)
    for a in range(8):
        sx, sy, sz = (1 if a & 1 else -1), (1 if a & 2 else -1), (1 if a & 4 else -1)
        gx = 0.125 * sx * (1 + sy * eta) * (1 + sz * zeta) * 2 / hx
        gy = 0.125 * sy * (1 + sx * xi) * (1 + sz * zeta) * 2 / hy
        gz = 0.125 * sz * (1 + sx * xi) * (1 + sy * eta) * 2 / hz
        node = ((i + (a & 1)) % nx) + nx * (((j + ((a >> 1) & 1)) % ny) + ny * ((k + ((a >> 2) & 1)) % nz))
        u = w[3 * node : 3 * node + 3]
        eps += np.asarray([gx * u[0], gy * u[1], gz * u[2], gz * u[1] + gy * u[2], gz * u[0] + gx * u[2],
                           gy * u[0] + gx * u[1]])  # fmt: skip
    ids = _phase_points(model)[ph]
    phase_local = int(np.searchsorted(ids, local_point))
    strain = eps.reshape(1, 6)
    dev = batch.device
    eps_t = torch.as_tensor(strain, device=dev)
    ep0 = batch.ep_n[:, local_point].double().reshape(1, 6).contiguous()
    q0 = batch.q_n[local_point : local_point + 1].contiguous()
    req = MaterialPointRequest(strain, None, request.time_step, "three_dimensional", request.material_update_settings)
    err = _j2_failure(mat, req, strain, eps_t, None, ep0, q0, 0, _native.settings_struct(request.material_update_settings),
                      _native.material_struct(mat), _Io(eps_t))  # fmt: skip
    if isinstance(err, MaterialPointConvergenceError):
        err = err.with_context(point_id=phase_local, strain=eps.tolist())
        err = err.with_context(element_id=phase_local // 8, quadrature_id=phase_local % 8)
    return err


def _build_response(model, cache: RVEOperatorCache, request, committed, macro, result: BatchStepResult, r: int,
                    point_out, diag, tangent, io) -> RVEResponse:  # fmt: skip
    """Assemble the reference's RVEResponse from the device reduction (solver.py:253-364)."""
    batch: RVEBatch = cache.batch
    s = batch.sums[r].cpu().numpy()
    volume = float(batch.volumes[r])
    macro_stress = s[RS_SIGMA : RS_SIGMA + 6] / volume
    virtual = s[RS_VW : RS_VW + 6] / volume
    macro_n = np.asarray(batch.macro_n[r].cpu().numpy())
    macro_work = float(macro_stress @ (macro - macro_n))
    micro_work = float(s[RS_MICRO_WORK] / volume)
    hm_res = macro_work - micro_work
    hm_err = abs(hm_res) / (abs(macro_work) + abs(micro_work) + model.hill_mandel_power_scale * request.time_step)
    face = s[RS_FACE : RS_FACE + 18].reshape(3, 2, 3)
    reaction = max(float(np.linalg.norm(m + p)) / max(float(np.linalg.norm(m) + np.linalg.norm(p)), 1.0) for m, p in face)
    class_reaction = float(batch.class_max[r].item()) / max(math.sqrt(s[RS_FNORM2]), 1.0)
    phases, _ = _phases_of(model)
    has_j2 = any(isinstance(m, J2ViscoplasticMaterial) for _, m in phases)
    if not has_j2:
        raise ValueError("RVE J2 diagnostics require incremental_work_density.")
    mmin, mmax = float(s[RS_MARGIN_MIN]), float(s[RS_MARGIN_MAX])
    available = np.isfinite(mmin)
    state = RVEState(_trial_material_state(cache, model, io), io.out(torch.as_tensor(macro, device=batch.device)),
                     io.out(batch.w[3 * batch.elem_offsets[r] + 3 : 3 * (batch.elem_offsets[r] + batch.elem_counts[r])].clone()))  # fmt: skip
    # per-point fields in the reference's (n_points, .) layout
    g0, g1 = 8 * batch.elem_offsets[r], 8 * (batch.elem_offsets[r] + batch.elem_counts[r])
    micro_strains = io.out(point_out[0:6, g0:g1].T.contiguous())
    micro_stresses = io.out(batch.stress[:, g0:g1].T.to(torch.float64).contiguous())
    micro_diag = _micro_diagnostics(model, diag[:, g0:g1], batch.tflag[g0:g1], io)
    phase_diag = _phase_diagnostics(model, s, volume, micro_state_keys=state.material_state.variables)
    displacement = _nodal_displacement(model, batch.w[3 * batch.elem_offsets[r] : 3 * (batch.elem_offsets[r] + batch.elem_counts[r])],
                                       macro, io)  # fmt: skip
    diagnostics = {
        "micro_residual_norm": float(result.residual_norm[r]),
        "micro_residual_tolerance": float(result.residual_tolerance[r]),
        "newton_iterations": int(result.newton_iterations[r]),
        "armijo_backtracks": int(result.armijo_backtracks[r]),
        "volume": volume,
        "virtual_work_stress_error": float(np.linalg.norm(virtual - macro_stress)),
        "periodic_fluctuation_error": float(s[RS_PERIODIC]),
        "reaction_antiperiodicity_error": reaction,
        "periodic_class_reaction_error": class_reaction,
        "macro_work_increment": macro_work,
        "micro_work_increment": micro_work,
        "hill_mandel_residual": hm_res,
        "hill_mandel_error": hm_err,
        "positive_work_density": float(s[RS_POS_WORK] / volume),
        "negative_work_density": float(s[RS_NEG_WORK] / volume),
        "unloading_volume_fraction": float(s[RS_UNLOAD] / volume),
        "viscoplastic_active_volume_fraction": float(s[RS_ACTIVE] / volume),
        "yield_activation_margin_available": int(available),
        "minimum_yield_activation_margin": mmin if available else np.nan,
        "maximum_yield_activation_margin": mmax if available else np.nan,
        "linear_solver_iterations": int(result.pcg_iterations[r]),
    }
    return RVEResponse(
        macro_stress=io.out(torch.as_tensor(macro_stress, device=batch.device)),
        effective_tangent=None if tangent is None else io.out(tangent.clone()),
        state=state,
        displacement=displacement,
        micro_strains=micro_strains,
        micro_stresses=micro_stresses,
        micro_diagnostics=micro_diag,
        free_energy_density=float(s[RS_PSI] / volume),
        dissipation_density=float(s[RS_DISS] / volume),
        phase_diagnostics=phase_diag,
        diagnostics=diagnostics,
    )


def _micro_diagnostics(model, diag: torch.Tensor, tflag: torch.Tensor, io) -> dict[str, Any]:
    """The assembly's per-point diagnostics dict with the reference's keys."""
    names = _native.j2_diagnostic_names()
    phases, el_phase = _phases_of(model)
    point_phase = np.repeat(el_phase.astype(np.int64), 8)
    phased = isinstance(model.material, PhasedMaterialModel)
    j2_points = np.zeros(point_phase.size, dtype=bool)
    for i, (_, m) in enumerate(phases):
        if isinstance(m, J2ViscoplasticMaterial):
            j2_points |= point_phase == i
    any_active = bool((tflag.cpu().numpy()[j2_points] > 0).any())
    keep = []
    for i, name in enumerate(names):
        if name == "viscoplastic_hv" and not any_active:
            continue
        keep.append(i)
    rows = diag[keep]
    if phased:
        # phase-local elastic points carry only the elastic-phase keys; others are NaN
        pass
    out = io.out(rows.contiguous())
    return {names[i]: out[slot] for slot, i in enumerate(keep)}


def _phase_diagnostics(model, s, volume, micro_state_keys) -> dict[str, dict[str, Any]]:
    phases, _ = _phases_of(model)
    if model.element_phase_ids is None:
        names = ("domain",)
    else:
        names = model.phase_names
    out = {}
    for i, name in enumerate(names):
        p = s[RS_PHASE + RS_PHASE_STRIDE * i : RS_PHASE + RS_PHASE_STRIDE * (i + 1)]
        vol = float(p[0])
        if model.element_phase_ids is None:
            fields = tuple(micro_state_keys)
        else:
            fields = tuple(k for k in micro_state_keys if k.startswith(f"phase_{name}__"))
        out[name] = {
            "volume": vol,
            "volume_fraction": vol / volume,
            "average_stress": p[1:7] / vol if vol > 0 else np.full(6, np.nan),
            "free_energy_density": float(p[7] / vol) if vol > 0 else np.nan,
            "dissipation_density": float(p[8] / vol) if vol > 0 else np.nan,
            "state_fields": fields,
        }
    return out


def _nodal_displacement(model, w_rve: torch.Tensor, macro: np.ndarray, io) -> Any:
    """u = T w + A ebar at every physical node (solver.py:88)."""
    c = model.constraint
    w_full = w_rve.reshape(-1, 3)
    cls = torch.as_tensor(c.equivalence_class_ids, device=w_rve.device)
    fluct = w_full.index_select(0, cls).reshape(-1)
    aff = torch.as_tensor(c.affine_matrix @ macro, device=w_rve.device)
    return io.out(fluct + aff)


# --------------------------------------------------------------------------------------
# Path drivers (path.py:47-123).


@dataclass(frozen=True)
class AcceptedRVEPathStep:
    """One accepted prescribed-path step."""

    step_id: int
    time: float
    time_step: float
    previous_state: RVEState
    response: RVEResponse


@dataclass(frozen=True)
class SolverProgressEvent:
    """Progress event of one accepted step (src/fem/solvers/progress.py:16)."""

    stage: str
    scheme: str
    accepted_step: int
    nominal_total_steps: int
    physical_time: float
    final_time: float
    newton_iterations: int
    armijo_backtracks: int
    elapsed_seconds: float
    residual_norm: float
    residual_tolerance: float


def iterate_prescribed_rve_path(model, times, macro_strains, update_settings, progress_callback=None
                                ) -> Iterator[AcceptedRVEPathStep]:  # fmt: skip
    """Yield accepted RVE steps of a prescribed macro-strain path."""
    times = np.asarray(times, dtype=np.float64)
    macro_strains = np.asarray(macro_strains, dtype=np.float64)
    if times.ndim != 1 or macro_strains.shape != (times.size, 6):
        raise ValueError("Prescribed RVE path requires time (n,) and strain (n, 6).")
    time_steps = np.diff(times)
    if times.size < 2 or np.any(time_steps <= 0.0):
        raise ValueError("Prescribed RVE path requires at least two increasing times.")
    cache = build_rve_operator_cache(model)
    start = perf_counter()
    state = initialize_rve_state(model)
    for step_id, dt in enumerate(time_steps, start=1):
        previous = state
        response = solve_rve_microequilibrium(
            model, RVERequest(macro_strains[step_id], float(dt), update_settings), state, cache
        )
        state = response.state
        if progress_callback is not None:
            progress_callback(SolverProgressEvent(
                "rve_path", "quasi_static_microequilibrium", step_id, time_steps.size, float(times[step_id]),
                float(times[-1]), int(response.diagnostics["newton_iterations"]),
                int(response.diagnostics["armijo_backtracks"]), perf_counter() - start,
                float(response.diagnostics["micro_residual_norm"]),
                float(response.diagnostics["micro_residual_tolerance"])))  # fmt: skip
        yield AcceptedRVEPathStep(step_id, float(times[step_id]), float(dt), previous, response)


def solve_prescribed_rve_path(model, times, macro_strains, update_settings, progress_callback=None) -> RVEPathResult:
    """Solve and commit every accepted point of one prescribed strain path."""
    accepted = tuple(iterate_prescribed_rve_path(model, times, macro_strains, update_settings, progress_callback))
    return RVEPathResult(np.asarray([s.time for s in accepted]), tuple(s.response for s in accepted))
