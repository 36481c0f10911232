"""FE^2 macro material: one independent periodic RVE per macro integration point.

Drop-in for the reference's RVEHomogenizedMaterial (src/fem/rve/material.py:40-264): the
same state keys (``rve_macro_strain``, ``rve_fluctuation_dofs``, ``rve_material__<key>``),
outputs and macro diagnostics.  Where the reference solves the macro points' RVEs one by
one (serially or in a process pool), here every macro point of an update call is one RVE
of a single device batch: one launch per kernel advances all of them together.  RVEs on
general meshes (the cylindrical O-grid RVE) are solved point by point with the
general-mesh device path, as the reference's serial loop (material.py:113-215).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

import numpy as np
import torch

from .materials import (
    DEFAULT_RESPONSE_REQUIREMENTS,
    J2ViscoplasticMaterial,
    MaterialPointRequest,
    MaterialPointResponse,
    MaterialResponseRequirements,
    MaterialState,
    PhasedMaterialModel,
    _Io,
    encode_phase_state_key,
)
from .rve import (
    RS_ACTIVE,
    RS_EQPS,
    RS_MARGIN_MIN,
    RS_MICRO_WORK,
    RS_NEG_WORK,
    RS_PHASE,
    RS_PHASE_STRIDE,
    RS_POS_WORK,
    RS_PSI,
    RS_DISS,
    RS_QMAX,
    RS_SIGMA,
    LinearSolverOptions,
    RVEBatch,
    RVEExecutionSettings,
    StructuredHex8RVE,
    _phase_points,
    _phases_of,
    initialize_rve_state,
    solve_batch_step,
)

_COMPONENTS = ("xx", "yy", "zz", "yz", "xz", "xy")


@dataclass(frozen=True)
class RVEHomogenizedMaterial:
    """A fixed quasi-static RVE exposed through the material-point protocol."""

    model: StructuredHex8RVE
    name: str
    execution_settings: RVEExecutionSettings = field(default_factory=RVEExecutionSettings)
    precision: int = 64
    linear_solver: LinearSolverOptions | None = None
    _batches: dict = field(default_factory=dict, init=False, repr=False, compare=False)

    @property
    def density(self) -> float:
        return float(self.model.material.density)

    @property
    def maximum_wave_speed(self) -> float:
        return float(self.model.material.maximum_wave_speed)

    @property
    def young_modulus(self) -> float:
        return float(self.model.material.young_modulus)

    @property
    def poisson_ratio(self) -> float:
        return float(self.model.material.poisson_ratio)

    def initialize_state(self, n_points: int) -> MaterialState:
        """One independent committed RVE state per macro point (material.py:94-111)."""
        prototype = initialize_rve_state(self.model)
        variables = {
            "rve_macro_strain": np.repeat(np.asarray(prototype.macro_strain)[None, :], n_points, axis=0),
            "rve_fluctuation_dofs": np.repeat(np.asarray(prototype.fluctuation_dofs)[None, :], n_points, axis=0),
        }
        for name, values in prototype.material_state.variables.items():
            variables[f"rve_material__{name}"] = np.repeat(np.asarray(values)[None, ...], n_points, axis=0)
        return MaterialState(variables)

    def _batch(self, n: int) -> RVEBatch:
        if n not in self._batches:
            self._batches[n] = RVEBatch([self.model] * n, precision=self.precision, linear_solver=self.linear_solver)
        return self._batches[n]

    def update(
        self,
        request: MaterialPointRequest,
        state: MaterialState,
        requirements: MaterialResponseRequirements = DEFAULT_RESPONSE_REQUIREMENTS,
    ) -> MaterialPointResponse:
        """Solve the RVEs of every macro integration point in one device batch."""
        from .rve import is_structured_box

        if not is_structured_box(self.model):
            return self._update_general(request, state, requirements)
        n = int(request.strains.shape[0])
        io = _Io(request.strains)
        batch = self._batch(n)
        dev = batch.device
        E = int(np.prod(self.model.divisions))
        g = 8 * E
        phases, _ = _phases_of(self.model)
        points = _phase_points(self.model)
        phased = isinstance(self.model.material, PhasedMaterialModel)
        v = state.variables
        # committed states -> device SoA (RVE i owns elements [i E, (i+1) E))
        ep = torch.zeros((n, g, 6), dtype=torch.float64, device=dev)
        q = torch.zeros((n, g), dtype=torch.float64, device=dev)
        vpm = torch.zeros((n, g), dtype=torch.float64, device=dev)
        for (pname, mat), ids in zip(phases, points):
            if not isinstance(mat, J2ViscoplasticMaterial):
                continue
            key = (lambda s: f"rve_material__{encode_phase_state_key(pname, s)}") if phased else (lambda s: f"rve_material__{s}")
            idx = torch.as_tensor(ids, device=dev)
            ep[:, idx] = io.to_device(v[key("plastic_strain")], (n, ids.size, 6))
            q[:, idx] = io.to_device(v[key("equivalent_plastic_strain")], (n, ids.size))
            vpm[:, idx] = io.to_device(v[key("viscoplastic_multiplier")], (n, ids.size))
        batch.ep_n.copy_(ep.reshape(n * g, 6).T.to(batch.dtype))
        batch.q_n.copy_(q.reshape(-1))
        batch.vpm_n.copy_(vpm.reshape(-1))
        w = torch.zeros((n, E, 3), dtype=torch.float64, device=dev)
        w.view(n, 3 * E)[:, 3:] = io.to_device(v["rve_fluctuation_dofs"], (n, 3 * E - 3))
        batch.w_n.copy_(w.reshape(-1))
        batch.macro_n.copy_(io.to_device(v["rve_macro_strain"], (n, 6)))
        batch.macro.copy_(io.to_device(request.strains, (n, 6)))
        batch.dt.fill_(float(request.time_step))
        result = solve_batch_step(batch, self.model.newton_settings, request.update_settings, False)
        b = batch.batch_struct(request.update_settings)
        batch.response(b, batch.w, None, None)
        tangent = batch.effective_tangent(b).clone() if requirements.tangent else None
        sums = batch.sums.cpu().numpy()
        volume = float(batch.volumes[0])
        stresses = sums[:, RS_SIGMA : RS_SIGMA + 6] / volume
        # next state
        nxt: dict[str, Any] = {"rve_macro_strain": io.out(batch.macro.clone()),
                               "rve_fluctuation_dofs": io.out(batch.w.view(n, 3 * E)[:, 3:].contiguous())}  # fmt: skip
        ep1 = batch.ep.T.to(torch.float64).reshape(n, g, 6)
        q1 = batch.q.reshape(n, g)
        vpm1 = batch.vpm.reshape(n, g)
        for (pname, mat), ids in zip(phases, points):
            if not isinstance(mat, J2ViscoplasticMaterial):
                continue
            key = (lambda s: f"rve_material__{encode_phase_state_key(pname, s)}") if phased else (lambda s: f"rve_material__{s}")
            idx = torch.as_tensor(ids, device=dev)
            nxt[key("plastic_strain")] = io.out(ep1[:, idx].contiguous())
            nxt[key("equivalent_plastic_strain")] = io.out(q1[:, idx].contiguous())
            nxt[key("viscoplastic_multiplier")] = io.out(vpm1[:, idx].contiguous())
        diagnostics = self._macro_diagnostics(sums, volume, result, request, batch)
        return MaterialPointResponse(
            stresses=io.out(torch.as_tensor(stresses, device=dev)),
            state=MaterialState(nxt),
            tangents=None if tangent is None else io.out(tangent),
            free_energy=io.out(torch.as_tensor(sums[:, RS_PSI] / volume, device=dev)) if requirements.free_energy else None,
            dissipation=io.out(torch.as_tensor(sums[:, RS_DISS] / volume, device=dev)) if requirements.dissipation else None,
            diagnostics={k: io.out(torch.as_tensor(val, device=dev)) for k, val in diagnostics.items()},
        )

    def _macro_diagnostics(self, sums, volume, result, request, batch) -> dict[str, np.ndarray]:
        """Macro-point reduction of the RVE diagnostics (material.py:218-264)."""
        n = sums.shape[0]
        macro = batch.macro.cpu().numpy()
        macro_n = batch.macro_n.cpu().numpy()
        stress = sums[:, RS_SIGMA : RS_SIGMA + 6] / volume
        macro_work = np.einsum("ij,ij->i", stress, macro - macro_n)
        micro_work = sums[:, RS_MICRO_WORK] / volume
        hm = np.abs(macro_work - micro_work) / (np.abs(macro_work) + np.abs(micro_work)
                                                + self.model.hill_mandel_power_scale * request.time_step)  # fmt: skip
        out = {
            "incremental_work_density": (sums[:, RS_POS_WORK] + sums[:, RS_NEG_WORK]) / volume,
            "viscoplastic_active": sums[:, RS_ACTIVE] / volume,
            "yield_activation_margin": np.where(np.isfinite(sums[:, RS_MARGIN_MIN]), sums[:, RS_MARGIN_MIN], np.nan),
            "micro_newton_iterations": result.newton_iterations.astype(np.float64),
            "micro_armijo_backtracks": result.armijo_backtracks.astype(np.float64),
            "hill_mandel_error": hm,
        }
        phases, _ = _phases_of(self.model)
        if not isinstance(self.model.material, PhasedMaterialModel) and isinstance(self.model.material, J2ViscoplasticMaterial):
            out["equivalent_plastic_strain"] = sums[:, RS_EQPS] / volume
        for i, pname in enumerate(self.model.phase_names):
            p = sums[:, RS_PHASE + RS_PHASE_STRIDE * i : RS_PHASE + RS_PHASE_STRIDE * (i + 1)]
            pv = p[:, 0]
            out[f"phase_{pname}__volume_fraction"] = pv / volume
            for c, comp in enumerate(_COMPONENTS):
                out[f"phase_{pname}__stress_{comp}"] = p[:, 1 + c] / pv
            if isinstance(phases[i][1], J2ViscoplasticMaterial):
                out[f"phase_{pname}__equivalent_plastic_strain"] = p[:, 9] / pv
                out[f"phase_{pname}__maximum_equivalent_plastic_strain"] = sums[:, RS_QMAX + i]
        return dict(sorted(out.items()))

    def _update_general(self, request, state, requirements) -> MaterialPointResponse:
        """One general-mesh RVE solve per macro point from its committed state, in point order."""
        from .rve import RVERequest, RVEState, build_rve_operator_cache, solve_rve_microequilibrium

        if "general" not in self._batches:
            self._batches["general"] = build_rve_operator_cache(self.model, linear_solver=self.linear_solver)
        cache = self._batches["general"]
        n = int(request.strains.shape[0])
        host = not isinstance(request.strains, torch.Tensor)
        variables = state.variables
        copy = lambda v: v.clone() if isinstance(v, torch.Tensor) else np.array(v, copy=True)  # noqa: E731
        nxt = {k: copy(v) for k, v in variables.items()}
        stresses = np.zeros((n, 6))
        tangents = np.zeros((n, 6, 6)) if requirements.tangent else None
        psi = np.zeros(n) if requirements.free_energy else None
        diss = np.zeros(n) if requirements.dissipation else None
        rows = []
        for i in range(n):
            committed = RVEState(
                MaterialState({k.removeprefix("rve_material__"): v[i] for k, v in variables.items()
                               if k.startswith("rve_material__")}),
                variables["rve_macro_strain"][i], variables["rve_fluctuation_dofs"][i])  # fmt: skip
            resp = solve_rve_microequilibrium(self.model, RVERequest(request.strains[i], request.time_step,
                                                                     request.update_settings, requirements),
                                              committed, cache)  # fmt: skip
            stresses[i] = _host(resp.macro_stress)
            if tangents is not None:
                tangents[i] = _host(resp.effective_tangent)
            if psi is not None:
                psi[i] = resp.free_energy_density
            if diss is not None:
                diss[i] = resp.dissipation_density
            nxt["rve_macro_strain"][i] = _like(resp.state.macro_strain, nxt["rve_macro_strain"])
            nxt["rve_fluctuation_dofs"][i] = _like(resp.state.fluctuation_dofs, nxt["rve_fluctuation_dofs"])
            for k, v in resp.state.material_state.variables.items():
                nxt[f"rve_material__{k}"][i] = _like(v, nxt[f"rve_material__{k}"])
            rows.append(_general_macro_diagnostics(resp, self.model, cache))
        names = sorted(set().union(*(r.keys() for r in rows)))
        dev = None if host else request.strains.device
        out = (lambda a: a) if host else (lambda a: None if a is None else torch.as_tensor(a, device=dev))  # noqa: E731
        return MaterialPointResponse(
            stresses=out(stresses), state=MaterialState(nxt), tangents=out(tangents), free_energy=out(psi),
            dissipation=out(diss), diagnostics={k: out(np.asarray([r[k] for r in rows])) for k in names},
        )  # fmt: skip

    def close(self) -> None:
        """Release the device batches."""
        self._batches.clear()


def _host(value) -> np.ndarray:
    return value.detach().cpu().numpy() if isinstance(value, torch.Tensor) else np.asarray(value)


def _like(value, target):
    """``value`` in the array type of ``target`` (host array or device tensor)."""
    if isinstance(target, torch.Tensor):
        return torch.as_tensor(_host(value), dtype=target.dtype, device=target.device)
    return _host(value)


def _general_macro_diagnostics(response, model, cache) -> dict[str, float]:
    """The reference's reduction of one RVE response to macro-point values (material.py:218-264)."""
    d = response.diagnostics
    out = {
        "incremental_work_density": float(d["positive_work_density"] + d["negative_work_density"]),
        "viscoplastic_active": float(d["viscoplastic_active_volume_fraction"]),
        "yield_activation_margin": float(d["minimum_yield_activation_margin"]),
        "micro_newton_iterations": float(d["newton_iterations"]),
        "micro_armijo_backtracks": float(d["armijo_backtracks"]),
        "hill_mandel_error": float(d["hill_mandel_error"]),
    }
    weights = np.asarray(cache.quadrature_weights)
    state = response.state.material_state.variables
    if "equivalent_plastic_strain" in state:
        out["equivalent_plastic_strain"] = float(np.sum(_host(state["equivalent_plastic_strain"]) * weights) / np.sum(weights))
    stresses = _host(response.micro_stresses)
    for phase_id, name in enumerate(model.phase_names):
        mask = np.asarray(cache.point_phase_ids) == phase_id
        pw = weights[mask]
        out[f"phase_{name}__volume_fraction"] = float(np.sum(pw) / np.sum(weights))
        phase_stress = np.sum(stresses[mask] * pw[:, None], axis=0) / np.sum(pw)
        for comp, value in zip(_COMPONENTS, phase_stress):
            out[f"phase_{name}__stress_{comp}"] = float(value)
        key = f"phase_{name}__equivalent_plastic_strain"
        if key in state:
            q = _host(state[key])
            out[key] = float(np.sum(q * pw) / np.sum(pw))
            out[f"phase_{name}__maximum_equivalent_plastic_strain"] = float(np.max(q))
    return out


__all__ = ["RVEHomogenizedMaterial", "build_rve_operator_cache"]
