"""Training data for the surrogate, generated by the batched GPU RVE solver.

Restates the reference's path-data generation (iterate_prescribed_rve_path driven over
random macro strain paths, src/concrete_impact/experiments/rve_response_generation.py:74-212
and src/fem/rve/path.py:47-100), with all paths of a set advanced together: one RVE per
path in one ``RVEBatch``, one batched Newton solve per time index.  Each path is a
piecewise-linear 6-component macro strain history (``random_strain_path``) with its own
amplitude (|strain| <= ``max_abs``) and strain rate, so the set spans the slow/fast and
small/large loadings a macro point meets.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, Sequence

import numpy as np
import torch

from .materials import MaterialUpdateSettings
from .rno import RNODataset, RNOScales
from .rve import RS_SIGMA, NonlinearNewtonSettings, RVEBatch, StructuredHex8RVE, solve_batch_step
from .rve_builders import random_strain_path


@dataclass(frozen=True)
class PathSetSpec:
    """Random path family: ``paths`` paths of ``steps`` steps, seeds ``seed``, ``seed`` + 1, ...;
    per-path amplitude log-uniform in ``amplitude`` and strain rate log-uniform in
    ``rate_range`` (1/s)."""

    paths: int
    steps: int = 200
    seed: int = 20000
    segments: int = 4
    amplitude: tuple[float, float] = (5.0e-4, 1.0e-2)
    rate_range: tuple[float, float] = (1.0, 1000.0)


def draw_paths(spec: PathSetSpec) -> tuple[np.ndarray, np.ndarray]:
    """(times (P, T+1), strains (P, T+1, 6)) of the path family."""
    times = np.empty((spec.paths, spec.steps + 1))
    strains = np.empty((spec.paths, spec.steps + 1, 6))
    lo, hi = np.log(spec.amplitude[0]), np.log(spec.amplitude[1])
    for p in range(spec.paths):
        amp = float(np.exp(np.random.default_rng(spec.seed + p + 7_000_000).uniform(lo, hi)))
        times[p], strains[p] = random_strain_path(spec.seed + p, spec.steps, spec.segments, amp, spec.rate_range)
    return times, strains


def generate_rve_paths(
    models: StructuredHex8RVE | Sequence[StructuredHex8RVE],
    spec: PathSetSpec,
    update_settings: MaterialUpdateSettings,
    newton: NonlinearNewtonSettings | None = None,
    precision: int = 32,
    progress: Callable[[int, int], None] | None = None,
    stats: list | None = None,
) -> RNODataset:
    """Solve every path of ``spec`` on its RVE (one model for all paths, or one per path)
    and return the homogenised stresses as a device dataset (stress at step 0 is zero).
    ``stats``, when given, receives per step (max Newton iterations, mean PCG iterations)."""
    if isinstance(models, StructuredHex8RVE):
        models = [models] * spec.paths
    if len(models) != spec.paths:
        raise ValueError("give one RVE model or one per path")
    newton = newton or models[0].newton_settings
    times, strains = draw_paths(spec)
    batch = RVEBatch(list(models), precision=precision)
    dev = batch.device
    strain_d = torch.as_tensor(strains, device=dev)
    dt_d = torch.as_tensor(np.diff(times, axis=1), device=dev)
    stress = torch.zeros_like(strain_d)
    vol = torch.as_tensor(batch.volumes, device=dev)[:, None]
    for t in range(1, spec.steps + 1):
        batch.macro.copy_(strain_d[:, t])
        batch.dt.copy_(dt_d[:, t - 1])
        res = solve_batch_step(batch, newton, update_settings, False)
        if stats is not None:
            stats.append((int(res.newton_iterations.max()), float(res.pcg_iterations.mean())))
        batch.response(batch.batch_struct(update_settings), batch.w, None, None)
        stress[:, t] = batch.sums[:, RS_SIGMA : RS_SIGMA + 6] / vol
        batch.commit()
        if progress is not None:
            progress(t, spec.steps)
    return RNODataset(strain_d, stress, dt_d)


def impact_paths(
    model: StructuredHex8RVE,
    amplitudes: Sequence[float],
    steps: int,
    update_settings: MaterialUpdateSettings,
    divisions=(32, 2, 2),
    lengths=(0.32, 0.02, 0.02),
    density: float = 2400.0,
    duration: float = 50.0e-6,
    dt: float | None = None,
    precision: int = 32,
    point_stride: int = 1,
) -> RNODataset:
    """Macro strain and homogenised stress histories at the macro points of direct FE^2
    bar runs, one run per half-sine pressure amplitude -- the reference's impact_path data
    source (macro paths extracted from direct explicit FE^2,
    src/concrete_impact/experiments/rve_response_generation.py:898-940 and
    rve_path_generation.py:44-47).  Every ``point_stride``-th macro point gives one path of
    ``steps`` steps (neighbouring points of one run carry nearly the same history)."""
    from .fe2 import DirectRVEPoints, ExplicitFE2, build_macro_bar, half_sine_pressure, stable_time_step

    bar = build_macro_bar(divisions, lengths, density)
    if dt is None:
        dt = stable_time_step(bar, model.material.maximum_wave_speed, 0.5)
    strains, stresses = [], []
    for amp in amplitudes:
        fe2 = ExplicitFE2(bar, DirectRVEPoints(model, bar.points, update_settings, precision=precision), dt,
                          lambda t, a=float(amp): half_sine_pressure(t, a, duration))  # fmt: skip
        keep = torch.arange(0, bar.points, point_stride, device=bar.fixed.device)
        e = torch.zeros((keep.numel(), steps + 1, 6), dtype=torch.float64, device=bar.fixed.device)
        s = torch.zeros_like(e)
        for t in range(1, steps + 1):
            fe2.step()
            e[:, t] = fe2.strain[keep]
            s[:, t] = fe2.last_stress[keep]
        strains.append(e)
        stresses.append(s)
        del fe2
    strain = torch.cat(strains)
    return RNODataset(strain, torch.cat(stresses), torch.full((strain.shape[0], steps), float(dt), dtype=torch.float64,
                                                              device=strain.device))  # fmt: skip


def concat_datasets(*sets: RNODataset) -> RNODataset:
    """Paths of several sets with the same number of steps, in order."""
    return RNODataset(torch.cat([d.strain for d in sets]), torch.cat([d.stress for d in sets]),
                      torch.cat([d.dt for d in sets]))  # fmt: skip


def split_dataset(data: RNODataset, validation: int) -> tuple[RNODataset, RNODataset]:
    """First P - ``validation`` paths for training, the rest for validation."""
    k = data.paths - validation
    return (RNODataset(data.strain[:k], data.stress[:k], data.dt[:k]),
            RNODataset(data.strain[k:], data.stress[k:], data.dt[k:]))  # fmt: skip


def input_envelope(scales: RNOScales, data: RNODataset, per_component: bool = False):
    """(max |normalised strain|, max |normalised rate|) over the training paths: the region
    in which the surrogate's answers are trusted by the macro error gate.  With
    ``per_component`` each entry is a list of the six component maxima."""
    if per_component:
        strain = (data.strain.abs().amax(dim=(0, 1)) / scales.strain).tolist()
        rate = (data.rates().abs().amax(dim=(0, 1)) / scales.rate).tolist()
        return strain, rate
    strain = float((data.strain.abs().amax() / scales.strain).item())
    rate = float((data.rates().abs().amax() / scales.rate).item())
    return strain, rate


def relative_stress_error(pred: torch.Tensor, target: torch.Tensor) -> float:
    """||pred - target||_F / ||target||_F over all points, steps and components."""
    t = target.double()
    return float(((pred.double() - t).norm() / t.norm().clamp_min(1e-300)).item())
