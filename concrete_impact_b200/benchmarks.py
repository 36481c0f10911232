"""Standard workloads of the RVE solver, the surrogate and FE^2, timed on the device.

Counterparts of the reference's benchmark drivers (src/concrete_impact/benchmarks/
rve_heterogeneous.py, dynamic_viscoplastic.py) for the concrete RVE of this package:

* ``rve_path_workload`` -- one 8^3 two-phase RVE (aggregate spheres at 40 % volume, seed 0)
  under uniaxial compression to -0.5 % in 100 steps at 10 /s with the other five macro
  strain components free (zero macro stress), FP64, Newton relative tolerance 1e-8.
* ``rve_batch_workload`` -- 256 RVEs with edges drawn from {8, 12, 16, 20, 24}, each on its
  own random piecewise-linear macro strain path (4 segments, |strain| <= 1 %, strain rate
  log-uniform in 1..1000 /s, 200 steps), all advanced by one batched Newton solve per
  time index with FP32 element kernels and FP64 reductions.

Each returns a dict of measured quantities; ``bench.py --workload`` prints them as its
JSON line.  Timing uses CUDA events around whole steps on the current stream.
"""

from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np
import torch

from .materials import MaterialUpdateSettings
from .rve import (
    RS_SIGMA,
    RVEBatch,
    StructuredHex8RVE,
    build_rve_operator_cache,
    initialize_rve_state,
    solve_batch_step,
    solve_rve_microequilibrium,
)
from .rve_builders import (
    build_two_phase_sphere_rve,
    config0_materials,
    default_newton,
    fp32_newton,
    random_strain_path,
    solve_mixed_control_step,
    uniaxial_path,
)

UPDATE_SETTINGS = MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)
EDGES = (8, 12, 16, 20, 24)


def concrete_rve(edge: int = 8, seed: int = 0, precision: int = 64) -> StructuredHex8RVE:
    """Unit-cube concrete RVE: mortar (J2 Perzyna) with 40 % aggregate spheres."""
    mortar, aggregate = config0_materials()
    newton = default_newton() if precision == 64 else fp32_newton()
    return build_two_phase_sphere_rve((edge, edge, edge), mortar, aggregate, newton, seed=seed)


def _elapsed_ms(fn) -> float:
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    fn()
    end.record()
    torch.cuda.synchronize()
    return start.elapsed_time(end)


def rve_path_workload(steps: int = 100) -> dict:
    """The mixed-control uniaxial compression path of one 8^3 RVE (FP64)."""
    model = concrete_rve(8, 0, 64)
    cache = build_rve_operator_cache(model)
    times, exx = uniaxial_path(steps)
    solves: list[tuple[int, int]] = []
    out: dict = {}

    def solve(request, state):
        r = solve_rve_microequilibrium(model, request, state, cache)
        solves.append((int(r.diagnostics["newton_iterations"]), int(r.diagnostics["linear_solver_iterations"])))
        return r

    def run() -> None:
        state = initialize_rve_state(model)
        guess = np.zeros(6)
        stress, strain = [], []
        for step in range(1, steps + 1):
            res = solve_mixed_control_step(solve, state, {0: float(exx[step])}, guess, float(times[step] - times[step - 1]),
                                           UPDATE_SETTINGS, stress_tolerance=1.0e-6 * 20.0e6)  # fmt: skip
            state = res.response.state
            guess = res.macro_strain
            stress.append(np.asarray(res.response.macro_stress, dtype=np.float64))
            strain.append(guess.copy())
        out["macro_stress"] = np.asarray(stress)
        out["macro_strain"] = np.asarray(strain)
        out["times"] = times

    wall0 = time.perf_counter()
    ms = _elapsed_ms(run)
    out.update({"ms": ms, "wall_s": time.perf_counter() - wall0, "steps": steps, "solves": len(solves),
                "newton_iterations": int(sum(s[0] for s in solves)), "pcg_iterations": int(sum(s[1] for s in solves)),
                "gauss_points": int(8 * model.elements.shape[0])})  # fmt: skip
    # residual passes: one per Newton iteration plus the converged pass, per solve
    out["gp_evaluations"] = (out["newton_iterations"] + len(solves)) * out["gauss_points"]
    return out


@dataclass
class RVEBatchSetup:
    models: list[StructuredHex8RVE]
    times: np.ndarray  # (R, T+1)
    strains: np.ndarray  # (R, T+1, 6)


def rve_batch_setup(n_rve: int = 256, steps: int = 200, edges=EDGES, base_seed: int = 1000) -> RVEBatchSetup:
    """Per RVE i: edge uniform from ``edges`` (seed base_seed + i), sphere layout seed i,
    macro path seed 5000 + i."""
    models, times, strains = [], [], []
    for i in range(n_rve):
        edge = int(np.random.default_rng(base_seed + i).choice(edges))
        models.append(concrete_rve(edge, i, 32))
        t, e = random_strain_path(5000 + i, steps, 4, 1.0e-2, (1.0, 1000.0))
        times.append(t)
        strains.append(e)
    return RVEBatchSetup(models, np.asarray(times), np.asarray(strains))


def rve_batch_workload(setup: RVEBatchSetup, warmup: int, timed: int, precision: int = 32) -> dict:
    """Advance every RVE of the batch ``warmup`` path steps untimed, then ``timed`` steps
    timed; one step = one batched Newton solve (+ homogenisation and commit) per time index.
    Each step copies its macro strains and time steps from pinned host memory and reads the
    homogenised stresses back (the caller's view of the batched API)."""
    batch = RVEBatch(setup.models, precision=precision)
    dev = batch.device
    strain_h = torch.as_tensor(setup.strains).pin_memory()
    dt_h = torch.as_tensor(np.diff(setup.times, axis=1)).pin_memory()
    stress_h = torch.empty((batch.nrve, 6), dtype=torch.float64).pin_memory()
    newton = setup.models[0].newton_settings
    gp = 8 * batch.elem_counts
    counts = {"gp_evaluations": 0, "newton_max": 0, "pcg_max": 0, "pcg_total": 0, "pcg_element_iterations": 0}
    vol = torch.as_tensor(batch.volumes, device=dev)[:, None]
    timers: dict = {}

    def step(t: int, record: bool) -> None:
        batch.macro.copy_(strain_h[:, t], non_blocking=True)
        batch.dt.copy_(dt_h[:, t - 1], non_blocking=True)
        res = solve_batch_step(batch, newton, UPDATE_SETTINGS, False, timers=timers if record else None)
        batch.response(batch.batch_struct(UPDATE_SETTINGS), batch.w, None, None)
        stress_h.copy_(batch.sums[:, RS_SIGMA : RS_SIGMA + 6] / vol)
        batch.commit()
        if record:
            passes = res.newton_iterations + 1 + res.armijo_backtracks
            counts["gp_evaluations"] += int((passes * gp).sum())
            counts["newton_max"] = max(counts["newton_max"], int(res.newton_iterations.max()))
            counts["pcg_max"] = max(counts["pcg_max"], int(res.pcg_iterations.max()))
            counts["pcg_total"] += int(res.pcg_iterations.sum())
            counts["pcg_element_iterations"] += int((res.pcg_iterations * batch.elem_counts).sum())

    for t in range(1, warmup + 1):
        step(t, False)
    ms = _elapsed_ms(lambda: [step(t, True) for t in range(warmup + 1, warmup + timed + 1)])
    kernel_ms = {k: float(sum(a.elapsed_time(b) for a, b in v)) for k, v in timers.items()}
    launches = {k: len(v) for k, v in timers.items()}
    plastic = float(batch.tflag.float().mean().item())
    return {"ms": ms, "rve_steps": batch.nrve * timed, "gauss_points": int(gp.sum()), "elements": int(batch.nelem),
            "stress_last": stress_h.numpy().copy(), "kernel_ms": kernel_ms, "kernel_launches": launches,
            "plastic_fraction": plastic, "h2d_bytes_per_step": int(batch.nrve * 7 * 8),
            "d2h_bytes_per_step": int(batch.nrve * 6 * 8), **counts}  # fmt: skip
