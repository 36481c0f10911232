"""Material-point protocol and GPU material models (drop-in for the reference's fem.materials).

Mirrors the reference's containers and models with the same names, fields, argument
meaning and error behaviour:

* ``MaterialUpdateSettings``, ``MaterialState``, ``MaterialResponseRequirements``,
  ``MaterialPointRequest``, ``MaterialPointResponse`` -- src/fem/materials/data.py:17-65
* ``MaterialPointConvergenceError`` -- src/fem/materials/errors.py:15-47
* ``J2ViscoplasticMaterial`` (+ ``build_j2_viscoplastic_material``) --
  src/fem/materials/plasticity.py:80-117, 223-256
* ``LinearElasticMaterial`` -- src/fem/materials/linear_elastic.py:25-100
* ``PhasedMaterialModel``, ``RVEPhase``, phase-key helpers -- src/fem/materials/phased.py:27-199

Arrays may be NumPy arrays (host; results come back as NumPy) or CUDA torch tensors
(results stay on the device).  Every update runs the sm_100a kernels of ``libcib200.so``;
there is no CPU path.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import Any, Protocol

import numpy as np
import torch

from . import _native

VOIGT_DIM = 6


# --------------------------------------------------------------------------------------
# Containers (src/fem/materials/data.py).


@dataclass(frozen=True)
class MaterialUpdateSettings:
    """Local constitutive integration settings."""

    max_iterations: int
    yield_relative_tolerance: float
    residual_absolute_tolerance: float
    residual_relative_tolerance: float


@dataclass(frozen=True)
class MaterialState:
    """Integration-point internal variables (NumPy arrays or CUDA tensors)."""

    variables: dict[str, Any]


@dataclass(frozen=True)
class MaterialResponseRequirements:
    """Optional constitutive outputs required by one caller."""

    tangent: bool = False
    free_energy: bool = False
    dissipation: bool = False


DEFAULT_RESPONSE_REQUIREMENTS = MaterialResponseRequirements()


@dataclass(frozen=True)
class MaterialPointRequest:
    """Input path data for one material-point update."""

    strains: Any
    strain_rates: Any | None
    time_step: float
    kinematics: str
    update_settings: MaterialUpdateSettings


@dataclass(frozen=True)
class MaterialPointResponse:
    """Output data from one material-point update."""

    stresses: Any
    state: MaterialState
    tangents: Any | None = None
    free_energy: Any | None = None
    dissipation: Any | None = None
    diagnostics: dict[str, Any] = field(default_factory=dict)


class MaterialModel(Protocol):
    """Local material update protocol."""

    @property
    def name(self) -> str: ...

    @property
    def density(self) -> float: ...

    @property
    def maximum_wave_speed(self) -> float: ...

    def initialize_state(self, n_points: int) -> MaterialState: ...

    def update(
        self,
        request: MaterialPointRequest,
        state: MaterialState,
        requirements: MaterialResponseRequirements = DEFAULT_RESPONSE_REQUIREMENTS,
    ) -> MaterialPointResponse: ...


def compute_isotropic_pressure_wave_speed(young_modulus: float, poisson_ratio: float, density: float) -> float:
    """Isotropic three-dimensional longitudinal wave speed."""
    bulk_modulus = young_modulus / (3.0 * (1.0 - 2.0 * poisson_ratio))
    shear_modulus = young_modulus / (2.0 * (1.0 + poisson_ratio))
    return float(math.sqrt((bulk_modulus + 4.0 * shear_modulus / 3.0) / density))


# --------------------------------------------------------------------------------------
# Errors (src/fem/materials/errors.py).


class MaterialPointConvergenceError(RuntimeError):
    """One failed material-point nonlinear update with serialisable diagnostics."""

    def __init__(self, message: str, reason: str, diagnostics: dict[str, Any]) -> None:
        super().__init__(message)
        self.reason = reason
        self.diagnostics = _to_serializable(diagnostics)

    def with_context(self, **context: Any) -> MaterialPointConvergenceError:
        """The same failure enriched with outer-layer context."""
        return MaterialPointConvergenceError(str(self), self.reason, {**self.diagnostics, **context})


def _to_serializable(value: Any) -> Any:
    if isinstance(value, dict):
        return {str(key): _to_serializable(item) for key, item in value.items()}
    if isinstance(value, (list, tuple)):
        return [_to_serializable(item) for item in value]
    if hasattr(value, "item"):
        return _to_serializable(value.item())
    if isinstance(value, float) and not math.isfinite(value):
        return str(value)
    return value


# --------------------------------------------------------------------------------------
# Host <-> device plumbing.


class _Io:
    """Moves request arrays to the GPU and results back to the caller's array type."""

    def __init__(self, like: Any) -> None:
        self.device = _native.require_cuda()
        self.host = not isinstance(like, torch.Tensor)

    def to_device(self, array: Any, shape: tuple[int, ...] | None = None) -> torch.Tensor:
        if isinstance(array, torch.Tensor):
            tensor = array.to(device=self.device, dtype=torch.float64)
        else:
            tensor = torch.as_tensor(np.asarray(array, dtype=np.float64), device=self.device)
        tensor = tensor.contiguous()
        if shape is not None:
            tensor = tensor.reshape(shape)
        return tensor

    def out(self, tensor: torch.Tensor | None) -> Any:
        if tensor is None:
            return None
        return tensor.cpu().numpy() if self.host else tensor

    def empty(self, *shape: int) -> torch.Tensor:
        return torch.empty(shape, dtype=torch.float64, device=self.device)


def _require_six_component_strains(strains: Any) -> Any:
    if len(strains.shape) != 2 or strains.shape[1] != VOIGT_DIM:
        raise ValueError("Plastic materials require strain arrays with shape (n_points, 6).")
    return strains


def _new_flags(device: torch.device) -> torch.Tensor:
    """[first_failure (all bits set = none), active_count] as int64 on the device."""
    flags = torch.zeros(2, dtype=torch.int64, device=device)
    flags[0] = -1
    return flags


# --------------------------------------------------------------------------------------
# J2 viscoplastic material (src/fem/materials/plasticity.py).


@dataclass(frozen=True)
class J2ViscoplasticMaterial:
    """Rate-dependent (Perzyna) J2 viscoplasticity with linear isotropic hardening."""

    name: str
    density: float
    young_modulus: float
    poisson_ratio: float
    yield_stress: float
    hardening_modulus: float
    time_scale: float
    reference_stress: float
    rate_exponent: float

    @property
    def maximum_wave_speed(self) -> float:
        """Elastic longitudinal wave-speed bound."""
        return compute_isotropic_pressure_wave_speed(self.young_modulus, self.poisson_ratio, self.density)

    @property
    def shear_modulus(self) -> float:
        return self.young_modulus / (2.0 * (1.0 + self.poisson_ratio))

    def initialize_state(self, n_points: int) -> MaterialState:
        """Zero plastic strain, equivalent plastic strain and viscoplastic multiplier."""
        return MaterialState(
            variables={
                "plastic_strain": np.zeros((n_points, VOIGT_DIM), dtype=np.float64),
                "equivalent_plastic_strain": np.zeros(n_points, dtype=np.float64),
                "viscoplastic_multiplier": np.zeros(n_points, dtype=np.float64),
            }
        )

    def update(
        self,
        request: MaterialPointRequest,
        state: MaterialState,
        requirements: MaterialResponseRequirements = DEFAULT_RESPONSE_REQUIREMENTS,
    ) -> MaterialPointResponse:
        """Update stresses and history on the GPU; the committed state is never written."""
        return j2vp_update_points(self, request, state, requirements)


def build_j2_viscoplastic_material(material_spec: dict[str, object]) -> J2ViscoplasticMaterial:
    """Build and validate a rate-dependent J2 material from a dictionary."""
    material = J2ViscoplasticMaterial(
        name=str(material_spec["name"]),
        density=float(material_spec["density"]),
        young_modulus=float(material_spec["young_modulus"]),
        poisson_ratio=float(material_spec["poisson_ratio"]),
        yield_stress=float(material_spec["yield_stress"]),
        hardening_modulus=float(material_spec["hardening_modulus"]),
        time_scale=float(material_spec["time_scale"]),
        reference_stress=float(material_spec["reference_stress"]),
        rate_exponent=float(material_spec["rate_exponent"]),
    )
    validate_j2_viscoplastic_material(material)
    return material


def validate_j2_viscoplastic_material(material: J2ViscoplasticMaterial) -> None:
    """Physical parameter checks of plasticity.py:239-256."""
    if material.young_modulus <= 0.0:
        raise ValueError("J2 viscoplasticity requires young_modulus > 0.")
    if not -1.0 < material.poisson_ratio < 0.5:
        raise ValueError("J2 viscoplasticity requires -1 < poisson_ratio < 0.5.")
    if material.yield_stress <= 0.0:
        raise ValueError("J2 viscoplasticity requires yield_stress > 0.")
    if material.hardening_modulus < 0.0:
        raise ValueError("J2 viscoplasticity requires hardening_modulus >= 0.")
    if material.time_scale <= 0.0:
        raise ValueError("J2 viscoplasticity requires time_scale > 0.")
    if material.reference_stress <= 0.0:
        raise ValueError("J2 viscoplasticity requires reference_stress > 0.")
    if material.rate_exponent < 1.0:
        raise ValueError("J2 viscoplasticity requires rate_exponent >= 1.")


def j2vp_update_points(
    material: J2ViscoplasticMaterial,
    request: MaterialPointRequest,
    state: MaterialState,
    requirements: MaterialResponseRequirements,
) -> MaterialPointResponse:
    """Batch driver of the reference's _update_points (plasticity.py:343-431) on the GPU."""
    if request.kinematics != "three_dimensional":
        raise ValueError("Plastic material updates currently require three_dimensional kinematics.")
    strains = _require_six_component_strains(request.strains)
    n = int(strains.shape[0])
    io = _Io(strains)
    lib = _native.load_library()
    eps = io.to_device(strains, (n, 6))
    rate = None if request.strain_rates is None else io.to_device(request.strain_rates, (n, 6))
    ep0 = io.to_device(state.variables["plastic_strain"], (n, 6))
    q0 = io.to_device(state.variables["equivalent_plastic_strain"], (n,))
    vpm0 = io.to_device(state.variables["viscoplastic_multiplier"], (n,))
    stress, ep1, q1, vpm1 = io.empty(n, 6), io.empty(n, 6), io.empty(n), io.empty(n)
    tangent = io.empty(n, 6, 6) if requirements.tangent else None
    psi, diss, diag = io.empty(n), io.empty(n), io.empty(_native.J2_NDIAG, n)
    flags = _new_flags(io.device)
    mat_c = _native.material_struct(material)
    set_c = _native.settings_struct(request.update_settings)
    dt = float(request.time_step)
    if n > 0:
        code = lib.cib_j2vp_update(
            ctypes.byref(mat_c), ctypes.byref(set_c), n, dt,
            _native.ptr(eps), _native.ptr(rate), _native.ptr(ep0), _native.ptr(q0), _native.ptr(vpm0),
            _native.ptr(stress), _native.ptr(ep1), _native.ptr(q1), _native.ptr(vpm1), _native.ptr(tangent),
            _native.ptr(psi), _native.ptr(diss), _native.ptr(diag),
            flags.data_ptr() + 8, flags.data_ptr(), _native.stream_ptr(),
        )  # fmt: skip
        _native.check(code, "cib_j2vp_update")
    first_failure, active = (int(v) for v in flags.cpu().tolist())
    if first_failure != -1:
        raise _j2_failure(material, request, strains, eps, rate, ep0, q0, first_failure, set_c, mat_c, io)
    variables = {name: values for name, values in state.variables.items()}
    variables["plastic_strain"] = io.out(ep1)
    variables["equivalent_plastic_strain"] = io.out(q1)
    variables["viscoplastic_multiplier"] = io.out(vpm1)
    diagnostics: dict[str, Any] = {}
    if n > 0:
        names = _native.j2_diagnostic_names()
        keep = [i for i, name in enumerate(names) if _keep_j2_diagnostic(name, active, rate is not None)]
        rows = io.out(diag[keep])
        for slot, i in enumerate(keep):
            diagnostics[names[i]] = rows[slot]
    return MaterialPointResponse(
        stresses=io.out(stress),
        state=MaterialState(variables),
        tangents=io.out(tangent) if requirements.tangent else None,
        free_energy=io.out(psi) if requirements.free_energy else None,
        dissipation=io.out(diss) if requirements.dissipation else None,
        diagnostics=diagnostics,
    )


def _keep_j2_diagnostic(name: str, active_points: int, has_rates: bool) -> bool:
    """Which keys the reference dict holds: viscoplastic_hv only once a point went viscous,
    the increment diagnostics only when strain rates are given."""
    if name == "viscoplastic_hv":
        return active_points > 0
    if name in ("incremental_work_density", "equivalent_stress_increment"):
        return has_rates
    return True


def _j2_failure(material, request, strains, eps, rate, ep0, q0, point, set_c, mat_c, io) -> Exception:
    """Build the reference's exception for the first failing point (plasticity.py:363-406)."""
    lib = _native.load_library()
    record = torch.zeros(ctypes.sizeof(_native.J2VPFailureC), dtype=torch.uint8, device=io.device)
    code = lib.cib_j2vp_diagnose_point(
        ctypes.byref(mat_c), ctypes.byref(set_c), int(eps.shape[0]), float(request.time_step),
        _native.ptr(eps), _native.ptr(rate), _native.ptr(ep0), _native.ptr(q0), int(point),
        record.data_ptr(), _native.stream_ptr(),
    )  # fmt: skip
    _native.check(code, "cib_j2vp_diagnose_point")
    rec = _native.J2VPFailureC.from_buffer_copy(bytes(record.cpu().numpy()))
    reason = _native.j2_reason(rec.reason)
    strain_row = np.asarray(eps[point].cpu().numpy(), dtype=np.float64).tolist()
    context = {
        "material_name": material.name,
        "material_type": type(material).__name__,
        "point_id": int(point),
        "time_step": request.time_step,
        "kinematics": request.kinematics,
        "strain": strain_row,
    }
    if rec.reason == 15:
        return RuntimeError("J2 viscoplastic tangent requires positive corrected overstress.")
    if rec.algorithm == 1:
        finite = reason == "non_finite_j2_invariant"
        error = MaterialPointConvergenceError(
            "J2 equivalent-stress invariant is non-finite." if finite else "J2 equivalent-stress invariant is negative.",
            reason,
            {"algorithm": "j2_equivalent_stress", "radicand": rec.radicand,
             "deviatoric_stress": list(rec.deviatoric_stress)},
        )  # fmt: skip
        return error.with_context(**context)
    if rec.algorithm == 2:
        error = MaterialPointConvergenceError(
            "J2 viscoplasticity received an invalid yield activation tolerance.",
            reason,
            {"algorithm": "j2_viscoplastic_yield_activation",
             "yield_relative_tolerance": request.update_settings.yield_relative_tolerance,
             "yield_scale": rec.yield_scale, "yield_activation_threshold": rec.yield_activation_threshold,
             "trial_yield_value": rec.trial_yield},
        )  # fmt: skip
        return error.with_context(**context)
    if reason == "invalid_iteration_limit":
        diagnostics: dict[str, Any] = {"algorithm": "j2_viscoplastic_local_newton", "max_iterations": rec.max_iterations}
    elif reason == "non_finite_problem_scale":
        diagnostics = {"algorithm": "j2_viscoplastic_local_newton", "physical_upper_bound": rec.physical_upper_bound,
                       "residual_tolerance": rec.residual_tolerance}  # fmt: skip
    else:
        diagnostics = {
            "algorithm": "j2_viscoplastic_local_newton",
            "iteration": rec.iteration,
            "max_iterations": rec.max_iterations,
            "time_step": rec.time_step,
            "rate_exponent": material.rate_exponent,
            "time_scale": material.time_scale,
            "reference_stress": material.reference_stress,
            "yield_stress": material.yield_stress,
            "hardening_modulus": material.hardening_modulus,
            "shear_modulus": rec.shear_modulus,
            "hardening_slope": rec.hardening_slope,
            "trial_yield": rec.trial_yield,
            "physical_lower_bound": 0.0,
            "physical_upper_bound": rec.physical_upper_bound,
            "plastic_multiplier": rec.plastic_multiplier,
            "corrected_overstress": rec.corrected_overstress,
            "residual": rec.residual if rec.has_residual else None,
            "residual_tolerance": rec.residual_tolerance,
            "derivative": rec.derivative if rec.has_derivative else None,
            "newton_candidate": rec.newton_candidate if rec.has_newton_candidate else None,
        }
    error = MaterialPointConvergenceError(f"J2 viscoplastic local Newton failed: {reason}.", reason, diagnostics)
    error = error.with_context(
        trial_equivalent_stress=rec.trial_equivalent_stress,
        yield_radius=rec.yield_radius,
        equivalent_plastic_strain=rec.equivalent_plastic_strain,
        trial_stress=list(rec.trial_stress),
    )
    return error.with_context(**context)


# --------------------------------------------------------------------------------------
# Linear elasticity (src/fem/materials/linear_elastic.py).


@dataclass(frozen=True)
class LinearElasticMaterial:
    """Linear elastic material parameters."""

    name: str
    density: float
    young_modulus: float
    poisson_ratio: float

    @property
    def maximum_wave_speed(self) -> float:
        return compute_isotropic_pressure_wave_speed(self.young_modulus, self.poisson_ratio, self.density)

    def initialize_state(self, n_points: int) -> MaterialState:
        """Linear elasticity carries no internal variables."""
        return MaterialState(variables={})

    def update(
        self,
        request: MaterialPointRequest,
        state: MaterialState,
        requirements: MaterialResponseRequirements = DEFAULT_RESPONSE_REQUIREMENTS,
    ) -> MaterialPointResponse:
        """Stress, tangent and energy at linear elastic points (three-dimensional)."""
        return evaluate_linear_elastic_points(request, self, state, requirements)


def build_linear_elastic_material(material_spec: dict[str, Any]) -> LinearElasticMaterial:
    """Build a linear elastic material definition."""
    return LinearElasticMaterial(
        name=str(material_spec["name"]),
        density=float(material_spec["density"]),
        young_modulus=float(material_spec["young_modulus"]),
        poisson_ratio=float(material_spec["poisson_ratio"]),
    )


def evaluate_linear_elastic_points(
    request: MaterialPointRequest,
    material: LinearElasticMaterial,
    state: MaterialState,
    requirements: MaterialResponseRequirements = DEFAULT_RESPONSE_REQUIREMENTS,
    increment_diagnostics: bool = False,
) -> tuple[MaterialPointResponse, dict[str, Any]] | MaterialPointResponse:
    """GPU evaluation of linear_elastic.py:74-100 (three-dimensional kinematics).

    With ``increment_diagnostics`` the elastic-phase work/stress-change diagnostics of
    phased.py:172-191 are returned alongside the response.
    """
    if request.kinematics != "three_dimensional":
        raise ValueError("The GPU linear elastic update supports three_dimensional kinematics.")
    strains = request.strains
    n = int(strains.shape[0])
    io = _Io(strains)
    lib = _native.load_library()
    eps = io.to_device(strains, (n, 6))
    rate = None if request.strain_rates is None else io.to_device(request.strain_rates, (n, 6))
    stress = io.empty(n, 6)
    tangent = io.empty(n, 6, 6) if requirements.tangent else None
    psi = io.empty(n) if requirements.free_energy else None
    diss = io.empty(n) if requirements.dissipation else None
    inc = io.empty(2, n) if (increment_diagnostics and rate is not None) else None
    if n > 0:
        code = lib.cib_linear_elastic_update(
            float(material.young_modulus), float(material.poisson_ratio), n, float(request.time_step),
            _native.ptr(eps), _native.ptr(rate), _native.ptr(stress), _native.ptr(tangent), _native.ptr(psi),
            _native.ptr(diss), _native.ptr(inc), _native.stream_ptr(),
        )  # fmt: skip
        _native.check(code, "cib_linear_elastic_update")
    response = MaterialPointResponse(
        stresses=io.out(stress),
        state=state,
        tangents=io.out(tangent),
        free_energy=io.out(psi),
        dissipation=io.out(diss),
    )
    if not increment_diagnostics:
        return response
    extra: dict[str, Any] = {}
    if inc is not None:
        rows = io.out(inc)
        extra = {"incremental_work_density": rows[0], "equivalent_stress_increment": rows[1]}
    return response, extra


# --------------------------------------------------------------------------------------
# Phased material (src/fem/materials/phased.py).


@dataclass(frozen=True)
class RVEPhase:
    """One named material phase."""

    name: str
    material: MaterialModel


@dataclass(frozen=True)
class PhasedMaterialModel:
    """Dispatch fixed integration-point subsets to phase material models."""

    name: str
    phases: tuple[RVEPhase, ...]
    point_phase_ids: Any
    effective_density: float

    @property
    def density(self) -> float:
        return self.effective_density

    @property
    def maximum_wave_speed(self) -> float:
        return max(phase.material.maximum_wave_speed for phase in self.phases)

    def initialize_state(self, n_points: int) -> MaterialState:
        """Phase-local state arrays under ``phase_<name>__<variable>`` keys."""
        phase_ids = np.asarray(self.point_phase_ids)
        if n_points != phase_ids.size:
            raise ValueError("Phased material point count does not match its phase map.")
        variables: dict[str, Any] = {}
        for phase_id, phase in enumerate(self.phases):
            count = int(np.count_nonzero(phase_ids == phase_id))
            for name, values in phase.material.initialize_state(count).variables.items():
                variables[encode_phase_state_key(phase.name, name)] = values
        return MaterialState(variables)

    def update(
        self,
        request: MaterialPointRequest,
        state: MaterialState,
        requirements: MaterialResponseRequirements = DEFAULT_RESPONSE_REQUIREMENTS,
    ) -> MaterialPointResponse:
        """Update every phase on the GPU and scatter back to the common point order."""
        strains = request.strains
        point_count, component_count = strains.shape
        phase_ids = np.asarray(self.point_phase_ids)
        if point_count != phase_ids.size:
            raise ValueError("Phased material request does not match its fixed phase map.")
        io = _Io(strains)
        eps = io.to_device(strains, (point_count, component_count))
        rates = None if request.strain_rates is None else io.to_device(request.strain_rates, eps.shape)
        stresses = torch.zeros_like(eps)
        tangents = (
            torch.zeros((point_count, component_count, component_count), dtype=torch.float64, device=io.device)
            if requirements.tangent
            else None
        )
        free_energy = torch.zeros(point_count, dtype=torch.float64, device=io.device) if requirements.free_energy else None
        dissipation = torch.zeros(point_count, dtype=torch.float64, device=io.device) if requirements.dissipation else None
        next_variables: dict[str, Any] = {}
        phase_diagnostics: list[tuple[torch.Tensor, dict[str, Any]]] = []
        for phase_id, phase in enumerate(self.phases):
            ids = torch.as_tensor(np.flatnonzero(phase_ids == phase_id), device=io.device)
            phase_state = _decode_phase_state(state, phase.name)
            phase_request = MaterialPointRequest(
                strains=eps.index_select(0, ids),
                strain_rates=None if rates is None else rates.index_select(0, ids),
                time_step=request.time_step,
                kinematics=request.kinematics,
                update_settings=request.update_settings,
            )
            device_state = MaterialState({k: io.to_device(v) for k, v in phase_state.variables.items()})
            diagnostics: dict[str, Any]
            if isinstance(phase.material, LinearElasticMaterial):
                if request.strain_rates is None or not requirements.tangent:
                    raise ValueError("Elastic RVE phase diagnostics require strain rates and tangents.")
                response, extra = evaluate_linear_elastic_points(
                    phase_request, phase.material, device_state, requirements, increment_diagnostics=True
                )
                diagnostics = dict(response.diagnostics)
                diagnostics.update(extra)
                diagnostics["viscoplastic_active"] = torch.zeros(ids.numel(), dtype=torch.float64, device=io.device)
            else:
                response = phase.material.update(phase_request, device_state, requirements)
                diagnostics = dict(response.diagnostics)
            stresses.index_copy_(0, ids, response.stresses)
            if tangents is not None:
                if response.tangents is None:
                    raise ValueError("Phased material requested a tangent but received None.")
                tangents.index_copy_(0, ids, response.tangents)
            if free_energy is not None:
                if response.free_energy is None:
                    raise ValueError("Phased material requested free energy but received None.")
                free_energy.index_copy_(0, ids, response.free_energy)
            if dissipation is not None:
                if response.dissipation is None:
                    raise ValueError("Phased material requested dissipation but received None.")
                dissipation.index_copy_(0, ids, response.dissipation)
            for name, values in response.state.variables.items():
                next_variables[encode_phase_state_key(phase.name, name)] = io.out(values)
            phase_diagnostics.append((ids, diagnostics))
        names = sorted(set().union(*(d.keys() for _, d in phase_diagnostics)))
        combined = {name: torch.full((point_count,), float("nan"), dtype=torch.float64, device=io.device) for name in names}
        for ids, diagnostics in phase_diagnostics:
            for name, values in diagnostics.items():
                combined[name].index_copy_(0, ids, io.to_device(values))
        return MaterialPointResponse(
            stresses=io.out(stresses),
            state=MaterialState(next_variables),
            tangents=io.out(tangents),
            free_energy=io.out(free_energy),
            dissipation=io.out(dissipation),
            diagnostics={name: io.out(values) for name, values in combined.items()},
        )


def _decode_phase_state(state: MaterialState, phase_name: str) -> MaterialState:
    prefix = f"phase_{phase_name}__"
    return MaterialState(
        {name.removeprefix(prefix): values for name, values in state.variables.items() if name.startswith(prefix)}
    )


def encode_phase_state_key(phase_name: str, variable_name: str) -> str:
    """Stable phase namespace key with a double-underscore separator."""
    return f"phase_{phase_name}__{variable_name}"


def decode_phase_state_key(key: str) -> tuple[str, str]:
    """Decode one phase namespace key or reject an incompatible name."""
    prefix, variable_name = key.split("__", maxsplit=1)
    if not prefix.startswith("phase_"):
        raise ValueError(f"Invalid phased material state key: {key}.")
    return prefix.removeprefix("phase_"), variable_name
