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
* ``rno_training_workload`` -- 2000 RVE paths x 200 steps from the batched solver, then
  surrogate training (MLP 18-128-128-128-12, BF16, batch 512 paths, TBPTT 50, Adam) scored
  on held-out paths solved in FP64.
* ``train_fe2_surrogate`` / ``fe2_accuracy`` / ``fe2_speed`` -- the explicit impact bar
  (64 x 16 x 16 Hex8, 0.01 m elements, half-sine 50 MPa over 50 us, density 2400) with the
  surrogate at every macro point behind the error gate, checked against all-direct FE^2
  and timed against it.
* ``ogrid_rve_path_workload`` -- the cylindrical O-grid two-phase RVE (32 circumferential,
  8 radial, 8 axial divisions: 2,560 elements, 30 % inclusion) along a 20-step compression
  path through solve_prescribed_rve_path (general-mesh device path, FP64).
* ``energy_rno_workload`` -- the reference's trained energy-based RVE-RNO (4 x 128 SiLU
  networks) at the 131,072 macro points of the 64 x 16 x 16 bar: one update_batch per step
  along seeded strain ramps, FP32.
* ``implicit_fe2_workload`` -- implicit FE^2 through solve_material_implicit_newmark: a
  16 x 4 x 4 Hex8 bar (0.01 m elements, 2,048 macro points) with an 8^3 concrete RVE (FP64)
  at every point, average-acceleration Newmark at 5 us under a half-sine 40 MPa pulse.

Each returns a dict of measured quantities; ``bench.py --workload`` prints them as its
JSON line.  Timing uses CUDA events around whole steps on the current stream.
"""

from __future__ import annotations

import time
from dataclasses import dataclass

import numpy as np
import torch

from . import _native
from .materials import MaterialUpdateSettings
from .rve import (
    RS_SIGMA,
    LinearSolverOptions,
    RVEBatch,
    StructuredHex8RVE,
    build_rve_operator_cache,
    initialize_rve_state,
    solve_batch_step,
    solve_rve_microequilibrium,
    tune_pcg_cluster,
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


def rve_path_workload(steps: int = 100, cluster: int = 1) -> dict:
    """The mixed-control uniaxial compression path of one 8^3 RVE (FP64); ``cluster`` CTAs
    share its PCG solves."""
    model = concrete_rve(8, 0, 64)
    cache = build_rve_operator_cache(model, linear_solver=LinearSolverOptions(cluster=cluster))
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
    calls0 = _native.LAUNCHED[0]
    ms = _elapsed_ms(run)
    out["launches"] = _native.LAUNCHED[0] - calls0
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


def rve_batch_workload(setup: RVEBatchSetup, warmup: int, timed: int, precision: int = 32, tune: bool = True,
                       forcing: str | None = "eisenstat_walker", device_control: bool = True,
                       breakdown_steps: int = 2) -> dict:  # fmt: skip
    """Advance every RVE of the batch ``warmup`` path steps untimed, then ``timed`` steps
    timed; one step = one batched Newton solve (+ homogenisation and commit) per time index.
    Each step copies its macro strains and time steps from pinned host memory and reads the
    homogenised stresses back (the caller's view of the batched API).  With ``tune`` the PCG
    cluster size is measured (``tune_pcg_cluster``) on the first timed step's system before
    the timed region.  ``forcing`` selects the inexact-Newton PCG tolerance
    (LinearSolverOptions.forcing).  With ``device_control`` every step's Newton solve is one
    CUDA graph launch (decisions on the device); ``breakdown_steps`` further steps then run
    through the host-driven loop with CUDA events around its residual and PCG launches, for
    the per-kernel times (the graph hides them)."""
    batch = RVEBatch(setup.models, precision=precision, linear_solver=LinearSolverOptions(forcing=forcing),
                     device_control=device_control)  # fmt: skip
    dev = batch.device
    strain_h = torch.as_tensor(setup.strains).pin_memory()
    dt_h = torch.as_tensor(np.diff(setup.times, axis=1)).pin_memory()
    stress_h = torch.empty((batch.nrve, 6), dtype=torch.float64).pin_memory()
    newton = setup.models[0].newton_settings
    gp = 8 * batch.elem_counts
    keys = ("gp_evaluations", "newton_max", "pcg_max", "pcg_total", "pcg_element_iterations", "graph_loops")
    counts = dict.fromkeys(keys, 0)
    breakdown = dict.fromkeys(keys, 0)
    vol = torch.as_tensor(batch.volumes, device=dev)[:, None]
    timers: dict = {}

    def step(t: int, tally: dict | None, step_timers: dict | None = None) -> None:
        batch.macro.copy_(strain_h[:, t], non_blocking=True)
        batch.dt.copy_(dt_h[:, t - 1], non_blocking=True)
        res = solve_batch_step(batch, newton, UPDATE_SETTINGS, False, timers=step_timers)
        batch.response(batch.batch_struct(UPDATE_SETTINGS), batch.w, None, None)
        stress_h.copy_(batch.sums[:, RS_SIGMA : RS_SIGMA + 6] / vol)
        batch.commit()
        if tally is not None:
            passes = res.newton_iterations + 1 + res.armijo_backtracks
            tally["gp_evaluations"] += int((passes * gp).sum())
            tally["newton_max"] = max(tally["newton_max"], int(res.newton_iterations.max()))
            tally["pcg_max"] = max(tally["pcg_max"], int(res.pcg_iterations.max()))
            tally["pcg_total"] += int(res.pcg_iterations.sum())
            tally["pcg_element_iterations"] += int((res.pcg_iterations * batch.elem_counts).sum())
            if batch.device_control:
                tally["graph_loops"] += batch.last_graph_iterations

    for t in range(1, warmup + 1):
        step(t, None)
    tuning = None
    if tune:
        batch.macro.copy_(strain_h[:, warmup + 1])
        batch.dt.copy_(dt_h[:, warmup])
        tuning = tune_pcg_cluster(batch, UPDATE_SETTINGS, persist=False)  # measured in every run
    if device_control:  # build the step's graph outside the timed region
        batch.newton_graph(newton, UPDATE_SETTINGS)
    calls0 = _native.LAUNCHED[0]
    last = warmup + timed
    ms = _elapsed_ms(lambda: [step(t, counts, None if device_control else timers)
                              for t in range(warmup + 1, last + 1)])  # fmt: skip
    launched = _native.LAUNCHED[0] - calls0
    if device_control:  # a graph launch runs init + 7 kernels per loop + finish
        launched += 7 * counts["graph_loops"] + timed
    breakdown_range = range(warmup + 1, last + 1)
    if device_control:
        # per-kernel times from further steps through the host-driven loop (the same kernels
        # and decisions, with CUDA events around its residual and PCG launches), untimed
        batch.device_control = False
        breakdown_range = range(last + 1, min(last + breakdown_steps, setup.strains.shape[1] - 1) + 1)
        for t in breakdown_range:
            step(t, breakdown, timers)
        batch.device_control = True
    else:
        breakdown = dict(counts)
    kernel_ms = {k: float(sum(a.elapsed_time(b) for a, b in v)) for k, v in timers.items()}
    launches = {k: len(v) for k, v in timers.items()}
    plastic = float(batch.tflag.float().mean().item())
    return {"ms": ms, "rve_steps": batch.nrve * timed, "gauss_points": int(gp.sum()), "elements": int(batch.nelem),
            "stress_last": stress_h.numpy().copy(), "kernel_ms": kernel_ms, "kernel_launches": launches,
            "plastic_fraction": plastic, "h2d_bytes_per_step": int(batch.nrve * 7 * 8),
            "d2h_bytes_per_step": int(batch.nrve * 6 * 8), "pcg_cluster": int(batch.cluster), "pcg_shape": int(batch.pcg_shape), "tuning": tuning,
            "forcing": forcing, "device_control": device_control,
            "launches": launched, "breakdown": {"steps": len(breakdown_range), **breakdown},
            **counts}  # fmt: skip


# ---------------------------------------------------------------------------------------
# Surrogate training on RVE paths.

RNO_FORWARD_FLOP = 2 * (18 * 128 + 128 * 128 * 2 + 128 * 12)  # 73,216 per path-step (unpadded)
RNO_TRAIN_FLOP = 3 * RNO_FORWARD_FLOP  # forward + input-gradient + weight-gradient products


def effective_elastic_tangent(model: StructuredHex8RVE) -> np.ndarray:
    """The RVE's homogenised elastic stiffness: the effective tangent of one FP64 solve at a
    strain far below yield (solve_rve_microequilibrium with the tangent requested)."""
    from .materials import MaterialResponseRequirements
    from .rve import RVERequest

    cache = build_rve_operator_cache(model)
    req = RVERequest(np.full(6, 1.0e-9), 1.0e-6, UPDATE_SETTINGS, MaterialResponseRequirements(tangent=True))
    return np.asarray(solve_rve_microequilibrium(model, req, initialize_rve_state(model), cache).effective_tangent)


def rno_training_workload(paths: int = 2000, steps: int = 200, epochs: int = 300, warmup_epochs: int = 1,
                          val_paths: int = 256, config=None) -> dict:  # fmt: skip
    """Generate ``paths`` RVE paths (8^3 concrete RVE, FP32 solver), train the surrogate
    (batch 512 paths, TBPTT 50, Adam) for ``warmup_epochs`` + ``epochs`` epochs, timing the
    latter, and score it on ``val_paths`` held-out paths solved in FP64."""
    from .rno import RNOConfig, RNOScales, RNOSurrogate
    from .rno_data import PathSetSpec, generate_rve_paths, relative_stress_error

    out: dict = {}
    model32, model64 = concrete_rve(8, 0, 32), concrete_rve(8, 0, 64)
    t0 = time.perf_counter()
    data = generate_rve_paths(model32, PathSetSpec(paths, steps, seed=20000), UPDATE_SETTINGS, precision=32)
    torch.cuda.synchronize()
    out["data_generation_s"] = time.perf_counter() - t0
    val = generate_rve_paths(model64, PathSetSpec(val_paths, steps, seed=30000), UPDATE_SETTINGS, precision=64)
    scales = RNOScales.from_data(data.strain[:, 1:], data.rates(), data.stress[:, 1:])
    rno = RNOSurrogate(config or RNOConfig(), scales)
    c_eff = torch.as_tensor(effective_elastic_tangent(model64), device=val.strain.device)
    target = val.stress[:, 1:]
    out["error_untrained"] = relative_stress_error(rno.rollout(val), target)
    out["error_elastic"] = relative_stress_error(val.strain[:, 1:] @ c_eff.T, target)
    history = rno.fit(data, warmup_epochs)
    calls0 = _native.LAUNCHED[0]
    rno.window_step(rno.config.tbptt_steps, min(rno.config.batch_paths, paths))  # eager: count its launches
    per_window = _native.LAUNCHED[0] - calls0
    c = rno.config
    batch = min(c.batch_paths, paths)
    batches = paths // batch
    ms = _elapsed_ms(lambda: history.extend(rno.fit(data, epochs)))
    path_steps = epochs * batches * batch * steps
    out.update({"train_ms": ms, "path_steps": path_steps, "epochs": epochs,
                "windows": epochs * batches * (steps // c.tbptt_steps), "loss_first": history[0],
                "loss_last": history[-1], "error_trained": relative_stress_error(rno.rollout(val), target),
                "flop": path_steps * RNO_TRAIN_FLOP, "model": rno,
                "launches": per_window * epochs * batches * (steps // c.tbptt_steps)})  # fmt: skip
    out["inference"] = rno_inference_workload(rno)
    return out


def rno_inference_workload(rno, points: int = 131072, steps: int = 50, warmup: int = 3) -> dict:
    """Surrogate inference at ``points`` macro points (the 64 x 16 x 16 bar's Gauss points):
    ``steps`` chained fused steps (latent carried from step to step) on seeded normalised
    inputs, CUDA-event timed; one launch per step."""
    g = torch.Generator(device="cuda").manual_seed(11)
    strain = torch.randn((points, 6), generator=g, device="cuda", dtype=torch.float32)
    rate = torch.randn((points, 6), generator=g, device="cuda", dtype=torch.float32)
    coef = torch.full((points,), 0.01, dtype=torch.float32, device="cuda")
    z = torch.zeros((2, points, 6), dtype=torch.float32, device="cuda")
    stress = torch.empty((points, 6), dtype=torch.float32, device="cuda")

    def step() -> None:
        rno.predict_normalized(strain, rate, coef, z, stress)
        z[0].copy_(z[1])

    for _ in range(warmup):
        step()
    calls0 = _native.LAUNCHED[0]
    ms = _elapsed_ms(lambda: [step() for _ in range(steps)])
    if int(rno.err.item()) != 0:
        raise RuntimeError("a tensor-core wait timed out in the surrogate inference kernel")
    return {"ms_per_step": ms / steps, "points": points, "steps": steps, "launches": _native.LAUNCHED[0] - calls0,
            "flop_per_step": points * RNO_FORWARD_FLOP}  # fmt: skip


# ---------------------------------------------------------------------------------------
# FE^2 explicit impact: surrogate-driven vs direct RVE macro points.


@dataclass(frozen=True)
class FE2Recipe:
    """How the deployed surrogate is trained: random 6-component RVE paths (general states;
    they also keep the surrogate stable when a macro solver drives it) plus impact paths taken
    from direct FE^2 runs of a calibration bar at other pulse amplitudes (the reference's
    impact_path data source).  The calibration bar has a confined core (64 x 8 x 8): a
    surrogate calibrated on a 64 x 2 x 2 bar, all free surface, reached 2.2 % open-loop
    error on that bar but 10.7 % on the 64 x 16 x 16 bar."""

    random_paths: int = 1000
    random_amplitude: tuple[float, float] = (2.0e-4, 5.0e-3)
    path_steps: int = 400
    impact_amplitudes: tuple[float, ...] = (20.0e6, 30.0e6, 40.0e6, 60.0e6, 70.0e6, 80.0e6)
    calibration_divisions: tuple[int, int, int] = (64, 8, 8)
    point_stride: int = 16
    epochs: int = 1500
    tau_ref: float = 1.0e-4
    learning_rate: float = 1.0e-3
    final_lr_fraction: float = 0.02
    input_noise: float = 0.0


def train_fe2_surrogate(recipe: FE2Recipe, log=None):
    """Data generation and training for the FE^2 surrogate; returns (rno, envelope, info)."""
    import math

    from .rno import RNOConfig, RNOScales, RNOSurrogate
    from .rno_data import PathSetSpec, concat_datasets, generate_rve_paths, impact_paths, input_envelope

    model32 = concrete_rve(8, 0, 32)
    info: dict = {}
    t0 = time.perf_counter()
    sets = []
    if recipe.random_paths:
        spec = PathSetSpec(recipe.random_paths, recipe.path_steps, seed=20000, amplitude=tuple(recipe.random_amplitude))
        sets.append(generate_rve_paths(model32, spec, UPDATE_SETTINGS, precision=32))
    if recipe.impact_amplitudes:
        lengths = tuple(0.01 * d for d in recipe.calibration_divisions)
        sets.append(impact_paths(model32, recipe.impact_amplitudes, recipe.path_steps, UPDATE_SETTINGS,
                                 divisions=recipe.calibration_divisions, lengths=lengths, precision=32,
                                 point_stride=recipe.point_stride))  # fmt: skip
    data = concat_datasets(*sets)
    torch.cuda.synchronize()
    info["data_generation_s"] = time.perf_counter() - t0
    info["training_paths"] = data.paths
    scales = RNOScales.from_data(data.strain[:, 1:], data.rates(), data.stress[:, 1:])
    rno = RNOSurrogate(RNOConfig(tau_ref=recipe.tau_ref, learning_rate=recipe.learning_rate), scales)
    lr0, frac, E = recipe.learning_rate, recipe.final_lr_fraction, recipe.epochs
    schedule = lambda e: lr0 * (frac + (1.0 - frac) * 0.5 * (1.0 + math.cos(math.pi * e / max(E, 1))))  # noqa: E731
    t0 = time.perf_counter()
    history = rno.fit(data, E, lr_schedule=schedule, log=log, input_noise=recipe.input_noise)
    torch.cuda.synchronize()
    info["training_s"] = time.perf_counter() - t0
    info["loss_first_last"] = [history[0], history[-1]] if history else None
    return rno, input_envelope(scales, data, per_component=True), info


def save_surrogate(path: str, rno, envelope) -> None:
    """Weights, scales, latent time scale and gate envelope of a trained surrogate."""
    state = rno.state_dict()
    state["tau_ref"] = torch.tensor(rno.config.tau_ref, dtype=torch.float64)
    e, r = (np.asarray(v, dtype=np.float64).reshape(-1) for v in envelope)
    state["envelope"] = torch.as_tensor(np.stack(np.broadcast_arrays(e, r)))
    torch.save(state, path)


def load_surrogate(path: str):
    """(rno, envelope) from ``save_surrogate``."""
    from .rno import RNOConfig, RNOSurrogate

    state = torch.load(path, map_location="cpu")
    rno = RNOSurrogate(RNOConfig(tau_ref=float(state["tau_ref"])))
    rno.load_state_dict(state)
    env = state["envelope"]
    return rno, (env[0].tolist(), env[1].tolist())


def _record_run(fe2, steps: int) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """Run ``steps`` steps; (stress (steps, P, 6), displacement (steps, 3N), macro strain
    (steps, P, 6)) at every step."""
    stress = torch.empty((steps, fe2.bar.points, 6), dtype=torch.float64, device=fe2.u.device)
    strain = torch.empty_like(stress)
    disp = torch.empty((steps, fe2.u.numel()), dtype=torch.float64, device=fe2.u.device)
    for t in range(steps):
        fe2.step()
        stress[t] = fe2.last_stress
        strain[t] = fe2.strain
        disp[t] = fe2.u
    return stress, disp, strain


def fe2_accuracy(rno, envelope, steps: int = 400, divisions=(64, 2, 2), precision_direct: int = 64,
                 fallback_capacity: int | None = None) -> dict:  # fmt: skip
    """Surrogate FE^2 (with the error gate and direct fallback) against all-direct FE^2 on
    the same bar (0.01 m elements, half-sine 50 MPa, 50 us): relative Frobenius errors of
    the macro stress and displacement histories."""
    from .fe2 import DirectRVEPoints, ExplicitFE2, RNOPoints, build_macro_bar, stable_time_step
    from .rno import RNODataset
    from .rno_data import relative_stress_error

    model_ref = concrete_rve(8, 0, precision_direct)
    lengths = tuple(0.01 * d for d in divisions)
    bar = build_macro_bar(divisions, lengths, 2400.0)
    dt = stable_time_step(bar, model_ref.material.maximum_wave_speed, 0.5)
    direct = ExplicitFE2(bar, DirectRVEPoints(model_ref, bar.points, UPDATE_SETTINGS, precision=precision_direct), dt)
    s_ref, u_ref, e_ref = _record_run(direct, steps)
    del direct
    # open loop: the surrogate alone along the direct run's macro strain histories
    zeros = torch.zeros((bar.points, 1, 6), dtype=torch.float64, device=e_ref.device)
    paths = RNODataset(torch.cat([zeros, e_ref.transpose(0, 1)], dim=1), torch.cat([zeros, s_ref.transpose(0, 1)], dim=1),
                       torch.full((bar.points, steps), dt, dtype=torch.float64, device=e_ref.device))  # fmt: skip
    open_loop = relative_stress_error(rno.rollout(paths), paths.stress[:, 1:])
    gate = RNOPoints(rno, bar.points, envelope, concrete_rve(8, 0, 32), UPDATE_SETTINGS,
                     fallback_capacity=fallback_capacity or bar.points)  # fmt: skip
    surrogate = ExplicitFE2(bar, gate, dt)
    s_rno, u_rno, _ = _record_run(surrogate, steps)
    return {"steps": steps, "divisions": list(divisions), "dt": dt, "points": bar.points,
            "homogenised_stress_error_open_loop": open_loop,
            "stress_error": relative_stress_error(s_rno, s_ref), "displacement_error": relative_stress_error(u_rno, u_ref),
            "flagged_points": int(gate.slots_used), "fallback_steps": int(gate.fallback_steps),
            "stress_rms_pa": float(s_ref.pow(2).mean().sqrt().item())}  # fmt: skip


def fe2_closed_loop(rno, envelope, steps: int = 400, divisions=(64, 16, 16), fallback_capacity: int = 32768) -> dict:
    """Surrogate FE^2 against all-direct FE^2 (FP32 RVEs; FP64 RVEs of all 131,072 points do
    not fit in HBM) on the full bar over ``steps`` steps from rest: relative Frobenius
    errors of the macro stress and displacement histories (closed loop), and of the
    surrogate alone along the direct run's strain histories (open loop)."""
    from .fe2 import DirectRVEPoints, ExplicitFE2, RNOPoints, build_macro_bar, stable_time_step
    from .rno import RNODataset
    from .rno_data import relative_stress_error

    model32 = concrete_rve(8, 0, 32)
    lengths = tuple(0.01 * d for d in divisions)
    bar = build_macro_bar(divisions, lengths, 2400.0)
    dt = stable_time_step(bar, model32.material.maximum_wave_speed, 0.5)
    t0 = time.perf_counter()
    direct = ExplicitFE2(bar, DirectRVEPoints(model32, bar.points, UPDATE_SETTINGS, precision=32), dt)
    s_ref, u_ref, e_ref = _record_run(direct, steps)
    del direct
    torch.cuda.empty_cache()
    direct_s = time.perf_counter() - t0
    zeros = torch.zeros((bar.points, 1, 6), dtype=torch.float64, device=e_ref.device)
    paths = RNODataset(torch.cat([zeros, e_ref.transpose(0, 1)], dim=1), torch.cat([zeros, s_ref.transpose(0, 1)], dim=1),
                       torch.full((bar.points, steps), dt, dtype=torch.float64, device=e_ref.device))  # fmt: skip
    open_loop = relative_stress_error(rno.rollout(paths), paths.stress[:, 1:])
    del paths
    gate = RNOPoints(rno, bar.points, envelope, model32, UPDATE_SETTINGS, fallback_capacity=fallback_capacity)
    surrogate = ExplicitFE2(bar, gate, dt)
    s_rno, u_rno, _ = _record_run(surrogate, steps)
    out = {"steps": steps, "divisions": list(divisions), "dt": dt, "points": bar.points,
           "homogenised_stress_error_open_loop": open_loop,
           "stress_error": relative_stress_error(s_rno, s_ref), "displacement_error": relative_stress_error(u_rno, u_ref),
           "flagged_points": int(gate.slots_used), "direct_reference": "all-direct FE2, FP32 8^3 RVEs",
           "direct_run_s": direct_s, "stress_rms_pa": float(s_ref.pow(2).mean().sqrt().item())}  # fmt: skip
    del surrogate, gate, s_ref, u_ref, e_ref, s_rno, u_rno
    torch.cuda.empty_cache()
    return out


def fe2_judged(rno, envelope, steps: int = 5000, warmup: int = 5, divisions=(64, 16, 16), sample: int = 256,
               every: int = 1, threshold: float | None = 0.05, fallback_capacity: int = 32768, seed: int = 0) -> dict:  # fmt: skip
    """Surrogate FE^2 on the full bar with the runtime judge (``SurrogateJudge``: FP64
    direct RVEs at ``sample`` seeded macro points, every ``every`` steps): macro steps/s
    with the judge's cost included, the judged homogenised-stress error over the run and
    the escalations to the fallback pool."""
    from .fe2 import ExplicitFE2, RNOPoints, SurrogateJudge, build_macro_bar, stable_time_step

    model32 = concrete_rve(8, 0, 32)
    lengths = tuple(0.01 * d for d in divisions)
    bar = build_macro_bar(divisions, lengths, 2400.0)
    dt = stable_time_step(bar, model32.material.maximum_wave_speed, 0.5)
    judge = SurrogateJudge(concrete_rve(8, 0, 64), bar.points, UPDATE_SETTINGS, sample=sample, every=every,
                           threshold=threshold, seed=seed)  # fmt: skip
    gate = RNOPoints(rno, bar.points, envelope, model32, UPDATE_SETTINGS, fallback_capacity=fallback_capacity,
                     judge=judge)  # fmt: skip
    fe2 = ExplicitFE2(bar, gate, dt)
    fe2.run(warmup)
    ms = _elapsed_ms(lambda: fe2.run(steps))
    hist = judge.history
    picks = sorted({0, len(hist) // 4, len(hist) // 2, 3 * len(hist) // 4, len(hist) - 1}) if hist else []
    out = {"steps": steps, "ms": ms, "steps_per_s": steps / (ms / 1e3), "sample": int(judge.points.numel()),
           "every": every, "threshold": threshold, "judge_steps": judge.judge_steps, "judged_error": judge.error,
           "worst_point_error": max((h[2] for h in hist), default=0.0), "escalations": gate.escalations,
           "flagged_points": int(gate.slots_used),
           "history": [{"step": hist[i][0], "error": hist[i][1], "worst_point": hist[i][2]} for i in picks],
           "judge_precision": "FP64 direct 8^3 RVEs (the reference's precision)"}  # fmt: skip
    del fe2, gate, judge
    torch.cuda.empty_cache()
    return out


def fe2_speed(rno, envelope, rno_steps: int = 5000, rno_warmup: int = 5, direct_steps: int = 3,
              divisions=(64, 16, 16), fallback_capacity: int = 32768, time_limit_s: float = 180.0) -> dict:  # fmt: skip
    """Macro steps/s of surrogate FE^2 (``rno_steps`` steps) and of all-direct FE^2 (FP32 RVEs,
    ``direct_steps`` steps from rest) on the full bar, CUDA-event timed."""
    from .fe2 import DirectRVEPoints, ExplicitFE2, RNOPoints, build_macro_bar, stable_time_step

    model32 = concrete_rve(8, 0, 32)
    lengths = tuple(0.01 * d for d in divisions)
    bar = build_macro_bar(divisions, lengths, 2400.0)
    dt = stable_time_step(bar, model32.material.maximum_wave_speed, 0.5)
    gate = RNOPoints(rno, bar.points, envelope, model32, UPDATE_SETTINGS, fallback_capacity=fallback_capacity)
    fe2 = ExplicitFE2(bar, gate, dt)
    fe2.run(rno_warmup)
    done = [0]
    wall0 = time.perf_counter()

    def run() -> None:
        # chunks of 250 steps; stop early once the wall time passes the limit (many flagged
        # points make every step a batched RVE solve)
        while done[0] < rno_steps:
            n = min(250, rno_steps - done[0])
            fe2.run(n)
            done[0] += n
            if done[0] < rno_steps:
                torch.cuda.synchronize()
                if time.perf_counter() - wall0 > time_limit_s:
                    break

    calls0 = _native.LAUNCHED[0]
    rno_ms = _elapsed_ms(run)
    out = {"launches": _native.LAUNCHED[0] - calls0, "points": bar.points, "dt": dt, "rno_steps": done[0], "rno_steps_requested": rno_steps, "rno_ms": rno_ms,
           "rno_steps_per_s": done[0] / (rno_ms / 1e3), "flagged_points": int(gate.slots_used),
           "fallback_steps": int(gate.fallback_steps), "simulated_time_s": (rno_warmup + done[0]) * dt}  # fmt: skip
    del fe2, gate
    torch.cuda.empty_cache()
    if direct_steps > 0:
        direct = ExplicitFE2(bar, DirectRVEPoints(model32, bar.points, UPDATE_SETTINGS, precision=32), dt)
        per_step = [_elapsed_ms(direct.step) for _ in range(direct_steps)]
        out.update({"direct_steps": direct_steps, "direct_ms": per_step,
                    "direct_steps_per_s": direct_steps / (sum(per_step) / 1e3)})  # fmt: skip
        del direct
        torch.cuda.empty_cache()
    return out


class _CountingMaterial:
    """Delegates to a material and counts the macro points it solves."""

    def __init__(self, inner) -> None:
        self.inner = inner
        self.points = 0
        self.calls = 0

    def __getattr__(self, name):
        return getattr(self.inner, name)

    def update(self, request, state, requirements=None):
        self.points += int(request.strains.shape[0])
        self.calls += 1
        return self.inner.update(request, state, requirements) if requirements is not None else self.inner.update(
            request, state)


def implicit_fe2_workload(steps: int = 5, warmup: int = 3, divisions=(16, 4, 4), time_step: float = 5.0e-6,
                          amplitude: float = 40.0e6, duration: float = 50.0e-6, forcing: str | None = None) -> dict:  # fmt: skip
    """Accepted macro steps/s of implicit FE^2 (solve_material_implicit_newmark with an 8^3
    concrete RVE at every macro point, FP64), through the public call with host arrays in
    (initial fields, load vectors) and out (the recorded histories).  A ``warmup``-step run
    from rest precedes the timed ``steps``-step run from rest; CUDA events bracket the call.
    ``forcing`` "eisenstat_walker" solves the RVE Newton systems inexactly (same RVE
    convergence tests; see LinearSolverOptions)."""
    from types import SimpleNamespace

    from .dynamics import (DirichletDofSet, MacroOperators, TimeIntegrationSettings,
                           solve_material_implicit_newmark)  # fmt: skip
    from .fe2 import build_macro_bar, half_sine_pressure
    from .rve import ArmijoSettings, NonlinearNewtonSettings
    from .rve_material import RVEHomogenizedMaterial

    model = concrete_rve(8, 0, 64)
    linear = LinearSolverOptions(forcing=forcing) if forcing else None
    material = _CountingMaterial(RVEHomogenizedMaterial(model, "concrete_rve_8", linear_solver=linear))
    lengths = tuple(0.01 * d for d in divisions)
    bar = build_macro_bar(divisions, lengths, material.density)
    fixed = np.flatnonzero(bar.fixed.cpu().numpy())
    unit = bar.unit_force.cpu().numpy()
    mesh = SimpleNamespace(nodes=bar.nodes, elements=bar.elements, material=material)
    h2d = [0]

    def load(t: float) -> np.ndarray:
        f = half_sine_pressure(t, amplitude, duration) * unit
        h2d[0] += f.nbytes
        return f

    n = 3 * bar.nodes.shape[0]
    newton = NonlinearNewtonSettings(20, 1.0e-3, 1.0e-8, 1.0e-14, 1.0e-8, ArmijoSettings(enabled=False))
    dirichlet = DirichletDofSet(fixed, np.zeros(fixed.size))
    ops = MacroOperators(bar.nodes, bar.elements, material.density, fixed, cache=bar.cache)

    def call(k: int):
        return solve_material_implicit_newmark(mesh, TimeIntegrationSettings("newmark", time_step, k, 0.25, 0.5, 1.0),
                                               np.zeros(n), np.zeros(n), dirichlet, load, "three_dimensional",
                                               UPDATE_SETTINGS, newton, operators=ops)  # fmt: skip

    call(warmup)
    material.points = material.calls = 0
    h2d[0] = 0
    calls0 = _native.LAUNCHED[0]
    pcg0 = ops.linear_iterations
    box: dict = {}
    ms = _elapsed_ms(lambda: box.setdefault("sol", call(steps)))
    sol = box["sol"]
    accepted = int(sol.times.size - 1)
    record_bytes = sum(getattr(sol, k).nbytes for k in ("displacement", "velocity", "acceleration", "internal_force",
                                                         "external_force", "stresses", "equivalent_plastic_strain"))
    out = {"ms": ms, "steps": accepted, "points": bar.points, "rve_elements": int(np.prod(model.divisions)),
           "rve_solves": material.points, "material_calls": material.calls,
           "newton_iterations": sol.newton_iterations[1:].tolist(), "macro_pcg_iterations": ops.linear_iterations - pcg0,
           "launches": _native.LAUNCHED[0] - calls0, "h2d_bytes": h2d[0], "d2h_record_bytes": int(record_bytes),
           "tip_displacement": float(sol.displacement[-1][3 * int(np.argmax(bar.nodes[:, 0]))]),
           "dissipated_energy": float(sol.dissipated_energy[-1]), "external_work": float(sol.external_work[-1]),
           "energy_residual": float(sol.energy_residual[-1]), "time_step": time_step}  # fmt: skip
    material.inner.close()
    return out


OGRID_DIRECTION = np.asarray([-1.0, 0.22, 0.22, 0.05, -0.03, 0.08])


def ogrid_rve(circumferential: int = 32, radial: int = 8, axial: int = 8):
    """Cylindrical O-grid concrete RVE: mortar matrix (J2 Perzyna), elastic aggregate
    cylinder at 30 % of the unit cell, Newton relative tolerance 1e-8."""
    from .rve_builders import build_cylindrical_ogrid_hex8, build_cylindrical_two_phase_rve

    mortar, aggregate = config0_materials()
    mesh = build_cylindrical_ogrid_hex8((1.0, 1.0, 1.0), 0.3, circumferential, radial, axial)
    return mesh, build_cylindrical_two_phase_rve(mesh, mortar, aggregate, default_newton(), 1.0)


def ogrid_path(steps: int, final_amplitude: float = 2.5e-3, time_step: float = 5.0e-6):
    """Times and macro strains of a proportional compression path from rest."""
    times = time_step * np.arange(steps + 1)
    strains = np.outer(np.linspace(0.0, final_amplitude, steps + 1), OGRID_DIRECTION)
    return times, strains


def ogrid_rve_path_workload(steps: int = 20, warmup: int = 3) -> dict:
    """Accepted RVE steps/s of the O-grid RVE along ``ogrid_path(steps)`` through
    solve_prescribed_rve_path; a ``warmup``-step path first, CUDA events around the call."""
    from .rve import solve_prescribed_rve_path

    mesh, model = ogrid_rve()
    solve_prescribed_rve_path(model, *ogrid_path(warmup), UPDATE_SETTINGS)
    times, strains = ogrid_path(steps)
    calls0 = _native.LAUNCHED[0]
    box: dict = {}
    ms = _elapsed_ms(lambda: box.setdefault("r", solve_prescribed_rve_path(model, times, strains, UPDATE_SETTINGS)))
    result = box["r"]
    newton = [int(r.diagnostics["newton_iterations"]) for r in result.responses]
    return {"ms": ms, "steps": len(result.responses), "elements": int(model.elements.shape[0]),
            "dofs": 3 * int(model.nodes.shape[0]), "newton_iterations": newton,
            "evaluations": 8 * int(model.elements.shape[0]) * (sum(newton) + len(newton)),
            "launches": _native.LAUNCHED[0] - calls0, "macro_stress": [np.asarray(r.macro_stress).tolist() for r in result.responses],
            "times": times, "strains": strains, "mesh": mesh}  # fmt: skip



def energy_rno_flop(hidden: int = 128, layers: int = 4, latent: int = 6) -> int:
    """Multiply-adds x 2 of one update: four network passes (equilibrium, non-equilibrium at
    the previous and candidate states, evolution) and three input-gradient passes."""
    def hidden_macs(n_in: int) -> int:
        return n_in * hidden + (layers - 1) * hidden * hidden

    forward = hidden_macs(6) + hidden + 2 * (hidden_macs(6 + latent) + hidden) + hidden_macs(6 + latent) + latent * hidden
    backward = hidden_macs(6) + 2 * hidden_macs(6 + latent)
    return 2 * (forward + backward)


def energy_rno_workload(state_dict: dict, config, points: int = 131072, steps: int = 50, warmup: int = 3) -> dict:
    """Update throughput of the energy-based RVE-RNO at ``points`` macro points: ``steps``
    chained updates along seeded strain ramps (dt 1e-4 s), CUDA-event timed."""
    from .energy_rno import EnergyDissipationRVERNO

    model = EnergyDissipationRVERNO(config)
    model.load_state_dict(state_dict)
    anchors = model.prepare_energy_anchors()
    g = torch.Generator(device="cuda").manual_seed(7)
    target = 5.0e-3 * torch.randn((points, 6), generator=g, device="cuda", dtype=torch.float32)
    dt = torch.full((points,), 1.0e-4, dtype=torch.float32, device="cuda")
    latent = model.initial_state_batch(points)
    for k in range(warmup):
        latent = model.update_batch(target * (k + 1) / (warmup + steps), latent, dt, anchors).latent_state
    calls0 = _native.LAUNCHED[0]
    box = {"z": latent}

    def run() -> None:
        z = box["z"]
        for k in range(steps):
            z = model.update_batch(target * (warmup + k + 1) / (warmup + steps), z, dt, anchors).latent_state
        box["z"] = z

    ms = _elapsed_ms(run)
    return {"ms": ms, "steps": steps, "points": points, "launches": _native.LAUNCHED[0] - calls0,
            "flop_per_point": energy_rno_flop(config.hidden_size, config.hidden_layers, config.latent_dimension),
            "latent_abs_max": float(box["z"].abs().max())}  # fmt: skip


def gemm_weight_gradient_workload(rows: int = 25600, splits: int = 50, steps: int = 20, warmup: int = 3) -> dict:
    """The training window's weight-gradient product on its own: dW (128 x 128) = dZ^T H over
    ``rows`` = T B rows (TBPTT 50 x batch 512), split-K over ``splits`` CTAs (the split the
    surrogate uses), fp32 partials; CUDA-event timed per launch."""
    from . import mlp

    g = torch.Generator(device="cuda").manual_seed(3)
    a = torch.randn((128, rows), generator=g, device="cuda").to(torch.bfloat16)
    b = torch.randn((128, rows), generator=g, device="cuda").to(torch.bfloat16)
    part = torch.empty((splits * 128, 128), dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    for _ in range(warmup):
        mlp.gemm(mlp.EPI_PARTIAL, a, b, c=part, splits=splits, err=err)
    ms = _elapsed_ms(lambda: [mlp.gemm(mlp.EPI_PARTIAL, a, b, c=part, splits=splits, err=err) for _ in range(steps)])
    if int(err.item()) != 0:
        raise RuntimeError("a tensor-core wait timed out in the GEMM")
    flop = 2.0 * 128 * 128 * rows
    return {"ms_per_launch": ms / steps, "rows": rows, "splits": splits, "tflops": flop / (ms / steps * 1e-3) / 1e12}


def _main(argv: list[str] | None = None) -> None:
    """``python -m concrete_impact_b200.benchmarks rno_inference|gemm_wgrad [steps]``: time one
    surrogate kernel on its own and print a JSON line (randomly initialised weights: the
    kernels and their work are those of a trained surrogate)."""
    import json
    import sys

    args = sys.argv[1:] if argv is None else argv
    steps = int(args[1]) if len(args) > 1 else 50
    if args and args[0] == "rno_inference":
        from .rno import RNOConfig, RNOSurrogate

        print(json.dumps(rno_inference_workload(RNOSurrogate(RNOConfig(seed=1)), steps=steps)))
    elif args and args[0] == "gemm_wgrad":
        print(json.dumps(gemm_weight_gradient_workload(steps=steps)))
    else:
        raise SystemExit("usage: python -m concrete_impact_b200.benchmarks rno_inference|gemm_wgrad [steps]")


if __name__ == "__main__":
    _main()
