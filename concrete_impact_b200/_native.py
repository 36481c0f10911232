"""ctypes binding of ``libcib200.so`` (the C ABI declared in ``include/cib200.h``).

The library is built in-tree by :mod:`concrete_impact_b200.build`.  Loading it needs no
GPU; every compute entry point does, and :func:`require_cuda` makes that failure loud:
there is no CPU fallback anywhere in this package.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import torch

LIB_PATH = Path(__file__).resolve().parent / "libcib200.so"
CIB_NO_FAILURE = 0xFFFFFFFFFFFFFFFF
J2_NDIAG = 22


class J2VPMaterialC(ctypes.Structure):
    """``cib_j2vp_material``."""

    _fields_ = [
        ("young_modulus", ctypes.c_double),
        ("poisson_ratio", ctypes.c_double),
        ("yield_stress", ctypes.c_double),
        ("hardening_modulus", ctypes.c_double),
        ("time_scale", ctypes.c_double),
        ("reference_stress", ctypes.c_double),
        ("rate_exponent", ctypes.c_double),
    ]


class UpdateSettingsC(ctypes.Structure):
    """``cib_update_settings``."""

    _fields_ = [
        ("max_iterations", ctypes.c_int32),
        ("pad_", ctypes.c_int32),
        ("yield_relative_tolerance", ctypes.c_double),
        ("residual_absolute_tolerance", ctypes.c_double),
        ("residual_relative_tolerance", ctypes.c_double),
    ]


class J2VPFailureC(ctypes.Structure):
    """``cib_j2vp_failure``."""

    _fields_ = [
        ("reason", ctypes.c_int32),
        ("iteration", ctypes.c_int32),
        ("max_iterations", ctypes.c_int32),
        ("algorithm", ctypes.c_int32),
        ("time_step", ctypes.c_double),
        ("shear_modulus", ctypes.c_double),
        ("hardening_slope", ctypes.c_double),
        ("trial_yield", ctypes.c_double),
        ("physical_upper_bound", ctypes.c_double),
        ("plastic_multiplier", ctypes.c_double),
        ("corrected_overstress", ctypes.c_double),
        ("residual", ctypes.c_double),
        ("residual_tolerance", ctypes.c_double),
        ("derivative", ctypes.c_double),
        ("newton_candidate", ctypes.c_double),
        ("radicand", ctypes.c_double),
        ("yield_scale", ctypes.c_double),
        ("yield_activation_threshold", ctypes.c_double),
        ("trial_equivalent_stress", ctypes.c_double),
        ("yield_radius", ctypes.c_double),
        ("equivalent_plastic_strain", ctypes.c_double),
        ("trial_stress", ctypes.c_double * 6),
        ("deviatoric_stress", ctypes.c_double * 6),
        ("has_residual", ctypes.c_int32),
        ("has_derivative", ctypes.c_int32),
        ("has_newton_candidate", ctypes.c_int32),
        ("pad_", ctypes.c_int32),
    ]


class RVEDescC(ctypes.Structure):
    """``cib_rve_desc``."""

    _fields_ = [
        ("nx", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("nz", ctypes.c_int32),
        ("pad_", ctypes.c_int32),
        ("elem_offset", ctypes.c_int64),
        ("hx", ctypes.c_double),
        ("hy", ctypes.c_double),
        ("hz", ctypes.c_double),
    ]


class PhaseMaterialC(ctypes.Structure):
    """``cib_phase_material``."""

    _fields_ = [("kind", ctypes.c_int32), ("pad_", ctypes.c_int32), ("params", J2VPMaterialC)]


RVE_MAX_PHASES = 8


class RVEBatchC(ctypes.Structure):
    """``cib_rve_batch``."""

    _fields_ = [
        ("nrve", ctypes.c_int32),
        ("nphase", ctypes.c_int32),
        ("nelem", ctypes.c_int64),
        ("precision", ctypes.c_int32),
        ("max_nxy", ctypes.c_int32),
        ("desc", ctypes.c_void_p),
        ("phase", ctypes.c_void_p),
        ("mats", PhaseMaterialC * RVE_MAX_PHASES),
        ("settings", UpdateSettingsC),
        ("plastic_strain_n", ctypes.c_void_p),
        ("eqps_n", ctypes.c_void_p),
        ("vpm_n", ctypes.c_void_p),
        ("plastic_strain", ctypes.c_void_p),
        ("eqps", ctypes.c_void_p),
        ("vpm", ctypes.c_void_p),
        ("stress", ctypes.c_void_p),
        ("tparam", ctypes.c_void_p),
        ("tflag", ctypes.c_void_p),
        ("fe", ctypes.c_void_p),
        ("de", ctypes.c_void_p),
        ("point_stride", ctypes.c_int64),
    ]


class RVENewtonC(ctypes.Structure):
    """``cib_rve_newton``: settings and device buffers of the device-controlled Newton solve."""

    _fields_ = [
        ("max_iterations", ctypes.c_int32),
        ("inexact", ctypes.c_int32),
        ("residual_absolute_tolerance", ctypes.c_double),
        ("residual_relative_tolerance", ctypes.c_double),
        ("increment_absolute_tolerance", ctypes.c_double),
        ("increment_relative_tolerance", ctypes.c_double),
        ("pcg_rtol", ctypes.c_double),
        ("pcg_maxit", ctypes.c_int32),
        ("cluster", ctypes.c_int32),
    ] + [(name, ctypes.c_void_p) for name in (
        "time_step", "macro", "w_n", "w", "w_out", "x", "r", "p", "Ap", "residual", "dinv", "rnorm2", "wnorm2",
        "class_max", "alpha", "active", "live_mask", "fail", "sys_rve", "sys_off", "pcg_status", "pcg_iterations",
        "pcg_rel_residual", "pcg_xnorm", "iwork", "dwork")]  # fmt: skip


class RNOWindowC(ctypes.Structure):
    """``cib_rno_window``."""

    _fields_ = [
        ("B", ctypes.c_int32),
        ("T", ctypes.c_int32),
        ("hidden", ctypes.c_int32),
        ("loss_scale", ctypes.c_float),
        ("ldt", ctypes.c_int64),
        ("strain", ctypes.c_void_p),
        ("rate", ctypes.c_void_p),
        ("coef", ctypes.c_void_p),
        ("target", ctypes.c_void_p),
        ("z", ctypes.c_void_p),
        ("W", ctypes.c_void_p * 4),
        ("Wt", ctypes.c_void_p * 4),
        ("bias", ctypes.c_void_p * 4),
        ("skip", ctypes.c_void_p),
        ("Z", ctypes.c_void_p * 3),
        ("Xt", ctypes.c_void_p),
        ("Ht", ctypes.c_void_p * 3),
        ("stress", ctypes.c_void_p),
        ("gS", ctypes.c_void_p),
        ("loss_part", ctypes.c_void_p),
        ("dYt", ctypes.c_void_p),
        ("dZt", ctypes.c_void_p * 3),
        ("err", ctypes.c_void_p),
    ]


class EnergyRNOC(ctypes.Structure):
    """``cib_energy_rno``."""

    _fields_ = [
        ("hidden", ctypes.c_int32),
        ("layers", ctypes.c_int32),
        ("latent", ctypes.c_int32),
        ("integrator", ctypes.c_int32),
        ("reference_time_scale", ctypes.c_double),
        ("params", ctypes.c_void_p),
        ("strain_scale", ctypes.c_void_p),
    ]


_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_D = ctypes.c_double
_I = ctypes.c_int

# name -> (restype, argtypes); every symbol declared in include/cib200.h.
SIGNATURES: dict[str, tuple[object, list[object]]] = {
    "cib_j2vp_update_soa_f64": (_I, [_P, _P, _I64, _I64, _D] + [_P] * 10),
    "cib_j2vp_update_soa_f32": (_I, [_P, _P, _I64, _I64, _D] + [_P] * 10),
    "cib_j2vp_update_soa_compact_f64": (_I, [_P, _P, _I64, _I64, _D] + [_P] * 10),
    "cib_j2vp_update_soa_compact_f32": (_I, [_P, _P, _I64, _I64, _D] + [_P] * 10),
    "cib_j2vp_update": (_I, [_P, _P, _I64, _D] + [_P] * 16),
    "cib_j2vp_diagnose_point": (_I, [_P, _P, _I64, _D, _P, _P, _P, _P, _I64, _P, _P]),
    "cib_linear_elastic_update": (_I, [_D, _D, _I64, _D] + [_P] * 8),
    "cib_copy_rows_async": (_I, [_P, _I64, _P, _I64, _I64, _I64, _I, _P]),
    "cib_hex8_geometry": (_I, [_I64] + [_P] * 6),
    "cib_hex8_strains": (_I, [_I64, _P, _P, _P, _P, _D, _P, _P, _P]),
    "cib_hex8_internal_force": (_I, [_I64, _I64] + [_P] * 8),
    "cib_hex8_tangent_csr": (_I, [_I64, _P, _P, _P, _I64, _P, _P, _P, _P, _P]),
    "cib_mlp_gemm": (_I, [ctypes.c_int32] * 4 + [_P, ctypes.c_int32, _P, ctypes.c_int32, ctypes.c_int32, _P, _P,
                          ctypes.c_int32, _P, ctypes.c_int32, _P, ctypes.c_int32, _P, ctypes.c_int32,
                          ctypes.c_int32, _P, _P]),
    "cib_splitk_reduce": (_I, [ctypes.c_int32] * 3 + [_P, ctypes.c_int32, _P, ctypes.c_int32, _P]),
    "cib_rno_input": (_I, [ctypes.c_int32, _P, _P, _P, _P, _P, ctypes.c_int32, ctypes.c_int32, _P]),
    "cib_rno_forward_tail": (_I, [ctypes.c_int32, _P, _P, _P, _P, _P, _P, ctypes.c_float, _P, _P]),
    "cib_rno_backward_head": (_I, [ctypes.c_int32, _P, _P, _P, _P, _P, ctypes.c_int32, ctypes.c_int32, _P]),
    "cib_rno_backward_tail": (_I, [ctypes.c_int32, _P, _P, _P, _P]),
    "cib_row_sum_bf16": (_I, [ctypes.c_int32, ctypes.c_int32, _P, ctypes.c_int32, _P, _P]),
    "cib_adam_step": (_I, [ctypes.c_int32, ctypes.c_int32, _P, _P, _P, _P] + [ctypes.c_float] * 4
                      + [_P, _P, ctypes.c_int32, _P, ctypes.c_int32, _P]),
    "cib_counter_increment": (_I, [_P, _P]),
    "cib_rno_window_forward": (_I, [_P, _P]),
    "cib_rno_window_backward": (_I, [_P, _P]),
    "cib_rno_gate_prepare": (_I, [_I64, _P, _P, _D, _D, _P, _D] + [_P] * 7),
    "cib_rno_gate_finish": (_I, [_I64, _P, _D, _P, _P, _P, _P, _P]),
    "cib_verlet_predict": (_I, [_I64, _P, _P, _P, _P, _D, _P, _P]),
    "cib_verlet_correct": (_I, [_I64, _P, _D, _P, _P, _P, _D, _P, _P, _P, _P, _P]),
    "cib_hex8_mass_csr": (_I, [_I64, _P, _D, _I64, _P, _P, _P, _P, _P]),
    "cib_csr_gather": (_I, [_I64] + [_P] * 5),
    "cib_energy_rno_param_count": (_I64, [ctypes.c_int32] * 3),
    "cib_energy_rno_anchors": (_I, [_P, _P, _P]),
    "cib_energy_rno_update": (_I, [_P, _I64] + [_P] * 10),
    "cib_energy_rno_tangent": (_I, [_P, _I64] + [_P] * 5),
    "cib_newmark_kinematics": (_I, [_I64, _P, _P, _P, _D, _D, _P, _P, _P]),
    "cib_newmark_residual": (_I, [_I64] + [_P] * 9),
    "cib_newmark_effective_tangent": (_I, [_I64, _P, _P, _P, _P, _D, _P, _P, _P, _P]),
    "cib_csr_spmv": (_I, [_I64] + [_P] * 6),
    "cib_csr_pcg": (_I, [_I64] + [_P] * 12 + [_D, ctypes.c_int32, ctypes.c_int32] + [_P] * 4),
    "cib_rve_residual": (_I, [_P] * 9),
    "cib_rve_gather": (_I, [_P] * 12),
    "cib_rve_pcg": (_I, [_P, ctypes.c_int32] + [_P] * 9 + [_D, ctypes.c_int32] + [_P] * 5),
    "cib_rve_pcg_cluster": (_I, [_P, ctypes.c_int32] + [_P] * 9 + [_D, ctypes.c_int32, ctypes.c_int32] + [_P] * 5),
    "cib_rve_pcg_noalloc": (_I, [_P, ctypes.c_int32, _P, _P, _P, _I64, _P, _P, _P, _D, ctypes.c_int32] + [_P] * 5),
    "cib_rve_tangent_rhs": (_I, [_P] * 6),
    "cib_rve_tangent_finish": (_I, [_P] * 7),
    "cib_rve_response": (_I, [_P] * 11),
    "cib_rve_newton_workspace": (None, [ctypes.c_int32, _P, _P]),
    "cib_rve_newton_graph_create": (_I, [_P, _P, _P]),
    "cib_rve_newton_graph_launch": (_I, [_P, _P]),
    "cib_rve_newton_graph_destroy": (_I, [_P]),
    "cib_j2_diagnostic_name": (ctypes.c_char_p, [_I]),
    "cib_j2_reason": (ctypes.c_char_p, [_I]),
    "cib_last_cuda_error": (_I, []),
    "cib_version": (ctypes.c_char_p, []),
}

_LIB: ctypes.CDLL | None = None


def load_library() -> ctypes.CDLL:
    """Load ``libcib200.so`` and bind every declared symbol (raises if missing)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m concrete_impact_b200.build` "
            "(this package has no CPU fallback)."
        )
    lib = ctypes.CDLL(os.fspath(LIB_PATH), mode=ctypes.RTLD_GLOBAL)
    for name, (restype, argtypes) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    _LIB = lib
    return lib


def require_cuda() -> torch.device:
    """Return the current CUDA device or raise: the kernels have no CPU path."""
    if not torch.cuda.is_available():
        raise RuntimeError("concrete_impact_b200 kernels need a CUDA device (sm_100a); none is available.")
    return torch.device("cuda", torch.cuda.current_device())


def ptr(tensor: torch.Tensor | None) -> int | None:
    """Device pointer of a tensor (None passes NULL)."""
    return None if tensor is None else tensor.data_ptr()


def stream_ptr(stream: torch.cuda.Stream | None = None) -> int:
    """Raw ``cudaStream_t`` of a torch stream (current stream by default)."""
    stream = torch.cuda.current_stream() if stream is None else stream
    return stream.cuda_stream


LAUNCHED = [0]  # entry-point calls that returned 0 (each launches at most one kernel)


def check(code: int, what: str) -> None:
    """Raise on a non-zero return code of an entry point; count the successful ones."""
    if code == 0:
        LAUNCHED[0] += 1
        return
    cuda = load_library().cib_last_cuda_error()
    raise RuntimeError(f"{what} failed with code {code} (last CUDA error {cuda}).")


def j2_diagnostic_names() -> list[str]:
    """Names of the diagnostic rows written by ``cib_j2vp_update``, in row order."""
    lib = load_library()
    return [lib.cib_j2_diagnostic_name(i).decode() for i in range(J2_NDIAG)]


def j2_reason(code: int) -> str:
    """Reference reason string of a per-point status code."""
    return load_library().cib_j2_reason(code).decode()


def material_struct(material) -> J2VPMaterialC:
    """``cib_j2vp_material`` from a J2ViscoplasticMaterial-like object."""
    return J2VPMaterialC(
        float(material.young_modulus),
        float(material.poisson_ratio),
        float(material.yield_stress),
        float(material.hardening_modulus),
        float(material.time_scale),
        float(material.reference_stress),
        float(material.rate_exponent),
    )


def settings_struct(settings) -> UpdateSettingsC:
    """``cib_update_settings`` from a MaterialUpdateSettings-like object."""
    return UpdateSettingsC(
        int(settings.max_iterations),
        0,
        float(settings.yield_relative_tolerance),
        float(settings.residual_absolute_tolerance),
        float(settings.residual_relative_tolerance),
    )
