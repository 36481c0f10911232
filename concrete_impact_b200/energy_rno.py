"""The reference's energy-based RVE-RNO surrogate on the GPU (inference).

Drop-in for ``EnergyDissipationRVERNO`` (src/concrete_impact/nn/models/rve_rno.py:162-476),
``load_rve_rno_state_dict`` and ``RVERNOMaterialAdapter``
(src/concrete_impact/nn/deployment.py:30-165): the same configuration fields, state-dict
key names, anchors, update results and material-point protocol, so a model trained by the
reference (its ``best_model.pt``) runs at FE^2 macro points on the device.  The update is one
FP32 kernel (csrc/energy_rno.cu) per call: per point, the equilibrium and non-equilibrium
potentials with their hand-written input gradients, the state-evolution network and the
forward-Euler latent step.

``compute_tangent`` adds the algorithmic tangent d stress / d strain, computed by a second
kernel with forward-over-reverse second derivatives of the three networks (the reference
differentiates the stress with autograd).  Scope: ``direct_rate`` evolution, FP32 models;
training stays with the reference (the surrogate this package trains is
``rno.RNOSurrogate``).
"""

from __future__ import annotations

import ctypes
import json
from dataclasses import dataclass, field
from pathlib import Path
from typing import Any

import numpy as np
import torch

from . import _native
from .materials import (
    DEFAULT_RESPONSE_REQUIREMENTS,
    MaterialPointRequest,
    MaterialPointResponse,
    MaterialResponseRequirements,
    MaterialState,
)

INTEGRATORS = {"cs_semi_implicit_forward_euler": 0, "current_state_stress_forward_euler": 1}
NETWORKS = (("equilibrium_energy.network.network", False), ("nonequilibrium_energy.network.network", False),
            ("state_evolution.network", True))  # fmt: skip


class SurrogateCapabilityError(RuntimeError):
    """A requested output that the surrogate does not provide."""


@dataclass(frozen=True)
class RVERNOModelConfig:
    """The energy-based RVE-RNO architecture (src/concrete_impact/nn/config.py:91-116)."""

    family: str
    time_representation: str
    integrator: str
    evolution: str
    reference_time_scale: float
    latent_dimension: int
    hidden_size: int
    hidden_layers: int
    activation: str
    strain_input_scale: tuple[float, ...] = (1.0, 1.0, 1.0, 1.0, 1.0, 1.0)
    dtype: str = "float32"
    device: str = "cuda"

    def __post_init__(self) -> None:
        if len(self.strain_input_scale) != 6 or any(not s > 0.0 for s in self.strain_input_scale):
            raise ValueError("RVE-RNO strain input scale must contain six positive values.")
        if self.family != "energy_rve_rno" or self.activation != "silu" or self.time_representation != "continuous":
            raise ValueError("Only the continuous-time SiLU energy_rve_rno family is defined.")
        if self.integrator not in INTEGRATORS:
            raise ValueError(f"Unknown RVE-RNO integrator {self.integrator!r}.")
        if self.evolution not in ("direct_rate", "mobility_gradient"):
            raise ValueError(f"Unknown RVE-RNO evolution {self.evolution!r}.")
        if not self.reference_time_scale > 0.0 or self.latent_dimension <= 0 or self.hidden_size <= 0 \
                or self.hidden_layers <= 0:
            raise ValueError("RVE-RNO sizes and the reference time scale must be positive.")


@dataclass(frozen=True)
class EnergyAnchors:
    """Zero-state energy values and strain gradients, packed as in cib_energy_rno_anchors."""

    packed: torch.Tensor  # (14,) float32 on the device

    @property
    def equilibrium_value(self) -> torch.Tensor:
        return self.packed[0]

    @property
    def equilibrium_strain_gradient(self) -> torch.Tensor:
        return self.packed[1:7]

    @property
    def nonequilibrium_value(self) -> torch.Tensor:
        return self.packed[7]

    @property
    def nonequilibrium_strain_gradient(self) -> torch.Tensor:
        return self.packed[8:14]


@dataclass(frozen=True)
class RVERNOUpdateBatch:
    """One batched update (rve_rno.py:34-45)."""

    stress: torch.Tensor
    latent_state: torch.Tensor
    state_rate: torch.Tensor
    dimensionless_state_rate: torch.Tensor
    dissipation: torch.Tensor
    free_energy: torch.Tensor
    thermodynamic_violation: torch.Tensor
    nonequilibrium_energy_increment: torch.Tensor
    tangent: torch.Tensor | None = None


def pack_state_dict(config: RVERNOModelConfig, state_dict: dict[str, Any], strict: bool = True) -> np.ndarray:
    """The kernel's parameter array: for the equilibrium, non-equilibrium and evolution
    networks in turn, per hidden layer W (torch layout), W^T and bias, then the output
    weights and bias (zeros for the two potentials), all FP32."""
    c = config
    sizes = ((6, 1), (6 + c.latent_dimension, 1), (6 + c.latent_dimension, c.latent_dimension))
    parts, used = [], set()

    def arr(key: str) -> np.ndarray:
        v = state_dict[key]
        return np.asarray(v.detach().cpu() if isinstance(v, torch.Tensor) else v, dtype=np.float32)

    for (prefix, out_bias), (n_in, n_out) in zip(NETWORKS, sizes):
        for layer in range(c.hidden_layers):
            w, b = arr(f"{prefix}.{2 * layer}.weight"), arr(f"{prefix}.{2 * layer}.bias")
            if w.shape != (c.hidden_size, n_in if layer == 0 else c.hidden_size) or b.shape != (c.hidden_size,):
                raise ValueError(f"RVE-RNO weight {prefix}.{2 * layer} has an unexpected shape {w.shape}.")
            parts += [w.ravel(), np.ascontiguousarray(w.T).ravel(), b]
            used |= {f"{prefix}.{2 * layer}.weight", f"{prefix}.{2 * layer}.bias"}
        key = f"{prefix}.{2 * c.hidden_layers}"
        wo = arr(f"{key}.weight")
        if wo.shape != (n_out, c.hidden_size):
            raise ValueError(f"RVE-RNO weight {key} has an unexpected shape {wo.shape}.")
        bo = arr(f"{key}.bias") if out_bias else np.zeros(n_out, dtype=np.float32)
        parts += [wo.ravel(), bo]
        used |= {f"{key}.weight"} | ({f"{key}.bias"} if out_bias else set())
    extra = set(state_dict) - used
    if strict and extra:
        raise KeyError(f"Unexpected RVE-RNO state-dict keys: {sorted(extra)}")
    return np.concatenate(parts)


class EnergyDissipationRVERNO:
    """Energy-derived stress and forward-Euler latent evolution, evaluated by one kernel."""

    def __init__(self, config: RVERNOModelConfig) -> None:
        if config.evolution != "direct_rate":
            raise NotImplementedError("The GPU RVE-RNO implements the direct_rate evolution.")
        if config.dtype != "float32":
            raise NotImplementedError("The GPU RVE-RNO evaluates FP32 models.")
        if config.hidden_size > 128 or config.latent_dimension > 8:
            raise NotImplementedError("The GPU RVE-RNO supports hidden_size <= 128 and latent_dimension <= 8.")
        self.config = config
        self.device = _native.require_cuda()
        self.lib = _native.load_library()
        count = int(self.lib.cib_energy_rno_param_count(config.hidden_size, config.hidden_layers,
                                                        config.latent_dimension))  # fmt: skip
        self.params = torch.zeros(count, dtype=torch.float32, device=self.device)
        self.strain_scale = torch.as_tensor(config.strain_input_scale, dtype=torch.float32, device=self.device)
        self.loaded = False

    @property
    def dtype(self) -> torch.dtype:
        return torch.float32

    def _struct(self) -> _native.EnergyRNOC:
        c = self.config
        return _native.EnergyRNOC(c.hidden_size, c.hidden_layers, c.latent_dimension, INTEGRATORS[c.integrator],
                                  float(c.reference_time_scale), self.params.data_ptr(), self.strain_scale.data_ptr())

    def load_state_dict(self, state_dict: dict[str, Any], strict: bool = True) -> None:
        """Pack the reference's state dict (torch or NumPy arrays, its key names)."""
        packed = pack_state_dict(self.config, state_dict, strict)
        if packed.size != self.params.numel():
            raise ValueError("RVE-RNO state dict does not match the configured architecture.")
        self.params.copy_(torch.as_tensor(packed))
        self.loaded = True

    def eval(self) -> EnergyDissipationRVERNO:
        return self

    def prepare_energy_anchors(self) -> EnergyAnchors:
        """Zero-state anchors, evaluated by the update kernel on a zero point."""
        self._require_loaded()
        out = torch.empty(14, dtype=torch.float32, device=self.device)
        m = self._struct()
        _native.check(self.lib.cib_energy_rno_anchors(ctypes.byref(m), out.data_ptr(), _native.stream_ptr()),
                      "cib_energy_rno_anchors")  # fmt: skip
        return EnergyAnchors(out)

    def initial_state_batch(self, batch_size: int) -> torch.Tensor:
        return torch.zeros((batch_size, self.config.latent_dimension), dtype=torch.float32, device=self.device)

    def update_batch(self, strain, previous_latent, time_step, anchors: EnergyAnchors | None = None,
                     compute_tangent: bool = False) -> RVERNOUpdateBatch:  # fmt: skip
        """Update all points at one time index (rve_rno.py:249-313).  ``compute_tangent``
        adds the algorithmic tangent d stress / d strain (n, 6, 6) from the second-derivative
        kernel (cib_energy_rno_tangent), in place of the reference's autograd rows."""
        self._require_loaded()
        f32 = lambda a: (a if isinstance(a, torch.Tensor) else torch.as_tensor(np.asarray(a))).to(  # noqa: E731
            device=self.device, dtype=torch.float32).contiguous()
        eps, z, dt = f32(strain), f32(previous_latent), f32(time_step)
        n, L = eps.shape[0], self.config.latent_dimension
        if eps.shape != (n, 6):
            raise ValueError(f"RVE-RNO strain must have shape [B, 6], received {tuple(eps.shape)}.")
        if z.shape != (n, L):
            raise ValueError("RVE-RNO latent state must have shape [B, latent_dimension].")
        if dt.shape != (n,):
            raise ValueError("RVE-RNO time step must have shape [B].")
        anchors = anchors or self.prepare_energy_anchors()
        out = {k: torch.empty(shape, dtype=torch.float32, device=self.device)
               for k, shape in (("stress", (n, 6)), ("latent", (n, L)), ("rate", (n, L)), ("dimless", (n, L)),
                                ("scalars", (4, n)))}  # fmt: skip
        m = self._struct()
        _native.check(self.lib.cib_energy_rno_update(ctypes.byref(m), n, eps.data_ptr(), z.data_ptr(), dt.data_ptr(),
                                                     anchors.packed.data_ptr(), out["stress"].data_ptr(),
                                                     out["latent"].data_ptr(), out["rate"].data_ptr(),
                                                     out["dimless"].data_ptr(), out["scalars"].data_ptr(),
                                                     _native.stream_ptr()), "cib_energy_rno_update")  # fmt: skip
        tangent = None
        if compute_tangent:
            tangent = torch.empty((n, 6, 6), dtype=torch.float32, device=self.device)
            _native.check(self.lib.cib_energy_rno_tangent(ctypes.byref(m), n, eps.data_ptr(), z.data_ptr(),
                                                          dt.data_ptr(), tangent.data_ptr(), _native.stream_ptr()),
                          "cib_energy_rno_tangent")  # fmt: skip
        s = out["scalars"]
        return RVERNOUpdateBatch(out["stress"], out["latent"], out["rate"], out["dimless"], s[0], s[1], s[2], s[3],
                                 tangent)

    def update(self, strain, previous_latent, time_step, compute_tangent: bool = False, context=None):
        """Batch of one (rve_rno.py:420-453)."""
        res = self.update_batch(torch.as_tensor(np.asarray(strain, dtype=np.float32)).reshape(1, 6),
                                torch.as_tensor(np.asarray(previous_latent, dtype=np.float32)).reshape(1, -1),
                                torch.as_tensor([float(time_step)], dtype=torch.float32), None, compute_tangent)  # fmt: skip
        return RVERNOUpdateBatch(*(getattr(res, f)[0] if getattr(res, f) is not None else None
                                   for f in RVERNOUpdateBatch.__dataclass_fields__))

    def _require_loaded(self) -> None:
        if not self.loaded:
            raise RuntimeError("Load the RVE-RNO weights (load_state_dict) before evaluating it.")


def load_rve_rno_state_dict(model_config: RVERNOModelConfig, model_path: str | Path,
                            metadata_path: str | Path) -> EnergyDissipationRVERNO:  # fmt: skip
    """Load one trained RVE-RNO after the reference's strict architecture matching
    (src/concrete_impact/nn/deployment.py:30-65)."""
    metadata = json.loads(Path(metadata_path).read_text(encoding="utf-8"))
    expected = {"model_family": model_config.family, "integrator": model_config.integrator,
                "evolution": model_config.evolution, "reference_time_scale": model_config.reference_time_scale,
                "latent_dimension": model_config.latent_dimension, "hidden_size": model_config.hidden_size,
                "hidden_layers": model_config.hidden_layers, "activation": model_config.activation,
                "strain_input_scale": tuple(model_config.strain_input_scale), "dtype": model_config.dtype,
                "deployment_integrator": "explicit_only"}  # fmt: skip
    received = {k: metadata.get(k, (1.0,) * 6 if k == "strain_input_scale" else None) for k in expected}
    received["strain_input_scale"] = tuple(received["strain_input_scale"])
    if received != expected:
        raise ValueError("RVE-RNO artifact metadata does not match the requested architecture: "
                         f"expected={expected}; received={received}.")  # fmt: skip
    checkpoint = torch.load(Path(model_path), map_location="cpu", weights_only=True)
    model = EnergyDissipationRVERNO(model_config)
    model.load_state_dict(checkpoint["model_state_dict"], strict=True)
    return model


@dataclass
class RVERNOMaterialAdapter:
    """A trained RVE-RNO through the material-point protocol (deployment.py:68-165)."""

    model: EnergyDissipationRVERNO
    name: str
    density: float
    maximum_wave_speed: float
    _anchors: EnergyAnchors | None = field(default=None, repr=False)

    def __post_init__(self) -> None:
        if self.density <= 0.0 or self.maximum_wave_speed <= 0.0:
            raise ValueError("RVE-RNO density and wave-speed bound must be positive.")

    def initialize_state(self, n_points: int) -> MaterialState:
        return MaterialState({"latent_state": np.zeros((n_points, self.model.config.latent_dimension))})

    def update(self, request: MaterialPointRequest, state: MaterialState,
               requirements: MaterialResponseRequirements = DEFAULT_RESPONSE_REQUIREMENTS) -> MaterialPointResponse:  # fmt: skip
        if request.kinematics != "three_dimensional":
            raise ValueError("Fixed-cell RVE-RNO currently requires three-dimensional strain.")
        latent = state.variables["latent_state"]
        if request.strains.shape[0] != latent.shape[0]:
            raise ValueError("RVE-RNO strain and latent-state point counts differ.")
        host = not isinstance(request.strains, torch.Tensor)
        if self._anchors is None:
            self._anchors = self.model.prepare_energy_anchors()
        n = int(request.strains.shape[0])
        res = self.model.update_batch(request.strains, latent,
                                      torch.full((n,), float(request.time_step), dtype=torch.float32), self._anchors,
                                      compute_tangent=requirements.tangent)  # fmt: skip
        if requirements.tangent and res.tangent is None:
            raise SurrogateCapabilityError("RVE-RNO tangent was requested but not returned.")
        out = (lambda t: t.double().cpu().numpy()) if host else (lambda t: t.double())  # noqa: E731
        return MaterialPointResponse(
            stresses=out(res.stress), state=MaterialState({"latent_state": out(res.latent_state)}),
            tangents=out(res.tangent) if requirements.tangent else None,
            dissipation=out(res.dissipation) if requirements.dissipation else None,
            free_energy=out(res.free_energy) if requirements.free_energy else None,
            diagnostics={"thermodynamic_violation": out(res.thermodynamic_violation),
                         "nonequilibrium_energy_increment": out(res.nonequilibrium_energy_increment)},
        )  # fmt: skip
