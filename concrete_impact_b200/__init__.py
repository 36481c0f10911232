"""B200-native (sm_100a) Gauss-point return map and periodic-RVE solve for concrete FE^2.

Drop-in for the reference's material-update, element-assembly and RVE/FE^2 driver API
(zhenhao2049/concrete_impact_ai, src/fem).  The compute path is hand-written CUDA in
``libcib200.so`` (C ABI: ``include/cib200.h``); Python here is the host-side mirror of the
reference interface and owns device memory and streams through PyTorch.
"""

from . import _native
from .materials import (
    DEFAULT_RESPONSE_REQUIREMENTS,
    J2ViscoplasticMaterial,
    LinearElasticMaterial,
    MaterialModel,
    MaterialPointConvergenceError,
    MaterialPointRequest,
    MaterialPointResponse,
    MaterialResponseRequirements,
    MaterialState,
    MaterialUpdateSettings,
    PhasedMaterialModel,
    RVEPhase,
    build_j2_viscoplastic_material,
    build_linear_elastic_material,
    compute_isotropic_pressure_wave_speed,
    decode_phase_state_key,
    encode_phase_state_key,
)

__all__ = [
    "DEFAULT_RESPONSE_REQUIREMENTS",
    "J2ViscoplasticMaterial",
    "LinearElasticMaterial",
    "MaterialModel",
    "MaterialPointConvergenceError",
    "MaterialPointRequest",
    "MaterialPointResponse",
    "MaterialResponseRequirements",
    "MaterialState",
    "MaterialUpdateSettings",
    "PhasedMaterialModel",
    "RVEPhase",
    "build_j2_viscoplastic_material",
    "build_linear_elastic_material",
    "compute_isotropic_pressure_wave_speed",
    "decode_phase_state_key",
    "encode_phase_state_key",
    "load_library",
]

load_library = _native.load_library
