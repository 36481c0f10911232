"""The workloads of ``bench.py --workload rve_path|rve_batch|rno_train|fe2|implicit_fe2|rve_ogrid``
(one JSON line on rank 0).

* rve_path  -- one 8^3 two-phase concrete RVE, mixed-control uniaxial compression to
  -0.5 % in 100 steps at 10 /s (free components at zero macro stress), FP64.  Metric:
  accepted RVE path steps per second through the single-RVE public API
  (solve_rve_microequilibrium inside the mixed-control outer Newton).
* rve_batch -- 256 concrete RVEs of edges {8, 12, 16, 20, 24}, each on its own random
  macro strain path; one batched Newton solve per time index, FP32 element kernels and
  FP64 reductions.  Metric: micro Gauss-point return-map evaluations per second inside
  the Newton solves (all residual passes of all RVEs), with accepted RVE steps/s beside it.
* rno_train -- 2000 RVE paths x 200 steps generated by the batched solver, then surrogate
  training; metric: training path-steps/s, with the held-out FP64 error beside it.
* fe2       -- the 64x16x16 impact bar with surrogate macro points behind the error gate;
  metric: macro steps/s, with all-direct FE^2 timed beside it and the surrogate's error
  against all-direct FP64 FE^2 on a 64x2x2 bar.
* rve_ogrid -- the cylindrical O-grid two-phase RVE (2,560 general Hex8 elements) along a
  20-step compression path; metric: accepted RVE steps/s through solve_prescribed_rve_path.
* rno_energy -- the reference's trained energy-based RVE-RNO at 131,072 macro points, 50
  chained updates (weights from tests/golden/rno_energy_c48.npz); metric: point-updates/s.
* implicit_fe2 -- implicit Newmark FE^2 (solve_material_implicit_newmark) on a 16x4x4 bar
  with an 8^3 concrete RVE (FP64) at each of the 2,048 macro points; metric: accepted macro
  steps/s through the public call (host arrays in and out), RVE solves/s beside it.

CPU baselines, each timed on the host on a bounded sample: the NumPy/SciPy oracle of the
reference's RVE solve (direct sparse solves, the reference's algorithm) for rve_path,
rve_batch, fe2 and implicit_fe2, its general-mesh form for rve_ogrid, and the torch
training loop on the host (oracle/rno_torch.py) for rno_train.
Multi-GPU runs are replicas: every rank runs the same workload, rank 0 prints.
"""

from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

EDGES = (8, 12, 16, 20, 24)


def _oracle_for(model, newton_rel: float):
    from oracle import j2vp as oj
    from oracle.rve import OraclePhase, OracleRVE, RVEOracle

    newton = {"max_iterations": 25, "residual_absolute_tolerance": 1.0e-6, "residual_relative_tolerance": newton_rel,
              "increment_absolute_tolerance": 1.0e-14, "increment_relative_tolerance": 1.0e-10, "armijo": None}  # fmt: skip
    phases = [OraclePhase("j2", oj.mortar_params()), OraclePhase("elastic", None, 50.0e9, 0.2)]
    return RVEOracle(OracleRVE(tuple(model.divisions), (1.0, 1.0, 1.0), phases, np.asarray(model.element_phase_ids), newton))


def _peak() -> tuple[float, str]:
    from bench import hbm_peak

    return hbm_peak()


def _line(args, metric, value, unit, workload, extra) -> dict:
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "data": "synthetic (seeded sphere layouts and macro strain paths)"}  # fmt: skip
    line["config"] = {"workload": workload, "parallelism": f"replicas x{args.gpus}"}
    line.update(extra)
    return line


# ---------------------------------------------------------------------------------------
# rve_path


def _rve_path_cpu(gpu_out: dict, sample_steps: int = 3) -> dict:
    """The oracle's solve on the GPU run's converged macro strains for the first steps;
    per-solve time times the GPU run's solve count estimates the path."""
    from concrete_impact_b200.benchmarks import concrete_rve

    model = concrete_rve(8, 0, 64)
    oracle = _oracle_for(model, 1.0e-8)
    state = oracle.initial_state()
    times = gpu_out["times"]
    diffs = []
    t0 = time.perf_counter()
    for step in range(1, sample_steps + 1):
        res = oracle.solve(gpu_out["macro_strain"][step - 1], float(times[step] - times[step - 1]), state, True)
        state = res["state"]
        ref = res["macro_stress"]
        diffs.append(float(np.abs(gpu_out["macro_stress"][step - 1] - ref).max() / max(np.abs(ref).max(), 1.0)))
    per_solve = (time.perf_counter() - t0) / sample_steps
    est = per_solve * gpu_out["solves"]
    return {"value": gpu_out["steps"] / est, "unit": "RVE steps/s", "cores": 1, "kind": "port",
            "sample": f"oracle (NumPy/SciPy direct solves) on the first {sample_steps} path steps at the GPU run's "
                      f"converged macro strains, {per_solve:.3f} s per solve x {gpu_out['solves']} solves",
            "max_rel_stress_diff_vs_oracle": max(diffs)}  # fmt: skip


def run_rve_path(args: argparse.Namespace) -> None:
    import torch

    from concrete_impact_b200.benchmarks import rve_path_workload

    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    from bench import ClockSampler

    cluster = int(os.environ.get("CIB_RVE_PATH_CLUSTER", "8"))
    rve_path_workload(max(args.warmup, 1), cluster)  # warm-up: a short path
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
        out = rve_path_workload(args.steps, cluster)
    if rank != 0:
        return
    cpu = None if args.no_cpu_baseline else _rve_path_cpu(out)
    ref, meta = _golden("rve_path_uniaxial_8")
    parity = {"max_rel_stress_diff_vs_reference": None}
    if ref is not None and len(out["macro_stress"]) >= meta["steps"]:
        got = np.asarray(out["macro_stress"][: meta["steps"]])
        scale = np.abs(ref["macro_stress"]).max(axis=1)
        parity = {"max_rel_stress_diff_vs_reference": float((np.abs(got - ref["macro_stress"]).max(axis=1) / scale).max()),
                  "sample": f"first {meta['steps']} steps against the reference's solve_rve_microequilibrium in the "
                            "same mixed-control loop"}  # fmt: skip
    seconds = out["ms"] / 1e3
    value = out["steps"] / seconds
    # one 8^3 RVE occupies at most one cluster of CTAs: a latency-bound solve, not a
    # bandwidth workload, so no roofline fraction is claimed
    peak, kind = _peak()
    line = _line(args, "accepted RVE steps/s (8^3 concrete RVE, mixed-control uniaxial path, FP64)", value,
                 "RVE steps/s", "rve_path: 8^3 two-phase RVE, seed 0, uniaxial compression -0.5 % in 100 steps at 10/s",
                 {"ms_per_step": out["ms"] / out["steps"], "dtype": "f64", "pcg_cluster": cluster, "parity": parity,
                  "gp_evaluations_per_s": out["gp_evaluations"] / seconds,
                  "solves": out["solves"], "newton_iterations": out["newton_iterations"],
                  "pcg_iterations": out["pcg_iterations"],
                  "final_macro_stress_xx_pa": float(out["macro_stress"][-1][0]),
                  "roofline": {"bound": "hbm", "achieved": None, "peak": peak, "unit": "GB/s", "frac": None,
                               "traffic": None, "peak_kind": kind,
                               "note": "one RVE = one CTA or one cluster per kernel: latency-bound, not a bandwidth workload"},
                  "gpu_launches": out["launches"],
                  "e2e": {"value": value, "unit": "RVE steps/s", "h2d_bytes_per_step": 6 * 8 * (out["solves"] // out["steps"] + 1),
                          "d2h_bytes_per_step": (6 + 36) * 8 * (out["solves"] // out["steps"] + 1),
                          "path": "solve_rve_microequilibrium (host arrays in and out) in the mixed-control loop"},
                  "clocks": clocks.summary(), "cpu_baseline": cpu})  # fmt: skip
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# rve_batch

PCG_TANGENT_BYTES_PER_GP = 8 * 4  # FP32 tangent parameters (n[6], f, c) of a plastic point
PCG_VECTOR_BYTES_PER_ELEMENT = 10 * 3 * 8  # p gather, Ap write, x/r/p/dinv/Ap updates, FP64
# Residual pass (rve_residual_kernel + gather), FP32 elements, per element of an active RVE:
# 8 points x (committed state read: plastic strain 24 + eqps 8 + multiplier 8; trial write:
# plastic strain 24 + eqps 8 + multiplier 8 + stress 24 + tangent data 32 + flag 1) + one
# node's fluctuation 24 + element forces and diagonals 2 x 192 written + phase 1 = 1,505 B;
# the gather reads the 384 B back and writes residual, inverse diagonal and trial w (72 B)
# and reads w (24 B) = 480 B.
RESIDUAL_BYTES_PER_ELEMENT_F32 = 8 * (40 + 97) + 24 + 384 + 1 + 480


def _rve_batch_cpu(setup, sample_edges=(8, 12)) -> dict:
    """The oracle on one RVE of each sample edge for the first two path steps; time per
    element-step scaled to the batch's element count (direct sparse solves grow faster
    than linearly in the element count, so the scaled estimate favours the CPU)."""
    picked = []
    for edge in sample_edges:
        for i, m in enumerate(setup.models):
            if m.divisions[0] == edge:
                picked.append(i)
                break
    elements, seconds = 0, 0.0
    for i in picked:
        model = setup.models[i]
        oracle = _oracle_for(model, 1.0e-6)
        state = oracle.initial_state()
        t0 = time.perf_counter()
        for step in (1, 2):
            res = oracle.solve(setup.strains[i, step], float(setup.times[i, step] - setup.times[i, step - 1]), state, False)
            state = res["state"]
        seconds += time.perf_counter() - t0
        elements += 2 * int(np.prod(model.divisions))
    per_element_step = seconds / elements
    total_elements = sum(int(np.prod(m.divisions)) for m in setup.models)
    return {"per_element_step_s": per_element_step, "total_elements": total_elements, "picked": picked,
            "sample_seconds": seconds}  # fmt: skip


def _golden(name: str):
    """Arrays and metadata of a committed golden run of the reference (tests/golden)."""
    from pathlib import Path

    root = Path(__file__).resolve().parent / "tests" / "golden"
    manifest = json.loads((root / "manifest.json").read_text())
    if name not in manifest or not (root / f"{name}.npz").exists():
        return None, None
    with np.load(root / f"{name}.npz") as data:
        return {k: data[k] for k in data.files}, manifest[name]


def _rve_batch_reference_parity(precision: int = 32, forcing: str | None = "eisenstat_walker") -> dict:
    """The workload's RVEs of every edge (the reference's own solves, tests/golden
    rve_batch_edge*) re-solved as one uneven batch with the workload's settings: the largest
    relative homogenised-stress difference over members and steps."""
    import torch

    from concrete_impact_b200.benchmarks import UPDATE_SETTINGS, concrete_rve
    from concrete_impact_b200.rve import RS_SIGMA, LinearSolverOptions, RVEBatch, solve_batch_step

    cases = [_golden(f"rve_batch_edge{e}") for e in EDGES]
    if any(a is None for a, _ in cases):
        return {"max_rel_stress_diff_vs_reference": None, "note": "reference golden runs not present"}
    models = [concrete_rve(m["edge"], m["layout_seed"], precision) for _, m in cases]
    batch = RVEBatch(models, precision=precision, linear_solver=LinearSolverOptions(cluster="auto", forcing=forcing),
                     device_control=True)  # fmt: skip
    vol = torch.as_tensor(batch.volumes, device=batch.device)[:, None]
    worst = 0.0
    for step in range(cases[0][0]["macro_strain"].shape[0]):
        batch.macro.copy_(torch.as_tensor(np.stack([a["macro_strain"][step] for a, _ in cases]), device=batch.device))
        batch.dt.copy_(torch.as_tensor([a["time_step"][step] for a, _ in cases], device=batch.device))
        solve_batch_step(batch, models[0].newton_settings, UPDATE_SETTINGS, False)
        batch.response(batch.batch_struct(UPDATE_SETTINGS), batch.w, None, None)
        got = (batch.sums[:, RS_SIGMA : RS_SIGMA + 6] / vol).cpu().numpy()
        batch.commit()
        for r, (a, _) in enumerate(cases):
            ref = a["macro_stress"][step]
            worst = max(worst, float(np.abs(got[r] - ref).max() / np.abs(ref).max()))
    return {"max_rel_stress_diff_vs_reference": worst,
            "sample": "one RVE of each edge 8..24 of this workload (its layout and path), time indices 0, 10, 20, 30, "
                      "against the reference's solve_rve_microequilibrium (FP64 direct solves)"}  # fmt: skip


def run_rve_batch(args: argparse.Namespace) -> None:
    import torch

    from bench import ClockSampler
    from concrete_impact_b200.benchmarks import rve_batch_setup, rve_batch_workload

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    setup = rve_batch_setup(getattr(args, "rves", 256), 200)
    forcing = os.environ.get("CIB_RVE_FORCING", "eisenstat_walker") or None
    with ClockSampler(local) as clocks:
        out = rve_batch_workload(setup, args.warmup, args.steps, forcing=forcing)
    if rank != 0:
        return
    seconds = out["ms"] / 1e3
    value = out["gp_evaluations"] / seconds
    peak, kind = _peak()
    bd = out["breakdown"]  # the steps whose kernels were timed one by one
    pcg_ms = out["kernel_ms"].get("pcg", 0.0)
    pcg_bytes = bd["pcg_element_iterations"] * (8 * PCG_TANGENT_BYTES_PER_GP * out["plastic_fraction"]
                                                + PCG_VECTOR_BYTES_PER_ELEMENT)  # fmt: skip
    achieved = pcg_bytes / (pcg_ms / 1e3) / 1e9 if pcg_ms > 0 else None
    res_ms = out["kernel_ms"].get("residual", 0.0)
    res_bytes = bd["gp_evaluations"] / 8 * RESIDUAL_BYTES_PER_ELEMENT_F32
    res_achieved = res_bytes / (res_ms / 1e3) / 1e9 if res_ms > 0 else None
    cpu = None
    if not args.no_cpu_baseline:
        c = _rve_batch_cpu(setup)
        cpu_rve_steps = 1.0 / (c["per_element_step_s"] * c["total_elements"] / len(setup.models))
        cpu = {"value": cpu_rve_steps, "unit": "RVE steps/s", "cores": 1, "kind": "port",
               "sample": f"oracle (NumPy/SciPy, direct solves) on RVEs {c['picked']} (edges 8 and 12), first 2 path "
                         f"steps, {c['per_element_step_s'] * 1e6:.1f} us per element-step scaled to "
                         f"{c['total_elements']:,} elements"}  # fmt: skip
    rve_steps_s = out["rve_steps"] / seconds
    parity = _rve_batch_reference_parity()
    line = _line(args, "micro Gauss-point evaluations/s inside the batched RVE Newton solve (256 uneven RVEs)", value,
                 "GP/s", "rve_batch: 256 two-phase RVEs, edges {8,12,16,20,24}, random 4-segment paths, FP32 elements",
                 {"ms_per_step": out["ms"] / args.steps, "dtype": "f32 elements, f64 reductions and history",
                  "accepted_rve_steps_per_s": rve_steps_s, "elements": out["elements"],
                  "gauss_points": out["gauss_points"], "newton_max": out["newton_max"], "pcg_max": out["pcg_max"],
                  "pcg_total": out["pcg_total"], "plastic_fraction": out["plastic_fraction"],
                  "pcg_cluster": out["pcg_cluster"], "pcg_shape": out["pcg_shape"],
                  "pcg_tuning": {"ms": (out["tuning"] or {}).get("ms"), "cached": (out["tuning"] or {}).get("cached"),
                                 "key": "cluster size / launch shape (0: 256 threads default cap, 1: 128 threads, "
                                        "2: 512 threads, 3: 256 threads other register cap)"},
                  "newton_forcing": out["forcing"], "parity": parity,
                  "newton_control": ("device: one CUDA graph per step (conditional while loop over the Newton "
                                     "iterations; residual, gather x2, check, PCG, update, axpy kernels per iteration)"
                                     if out["device_control"] else "host loop (two read-backs per Newton iteration)"),
                  "graph_launches_per_step": 1 if out["device_control"] else 0,
                  "host_syncs_per_step": 2 if out["device_control"] else None,
                  "graph_loop_iterations": out["graph_loops"],
                  "kernel_ms": out["kernel_ms"], "kernel_launches": out["kernel_launches"],
                  "kernel_breakdown_steps": bd["steps"],
                  "residual_roofline": {"bound": "hbm", "achieved": res_achieved, "peak": peak, "unit": "GB/s",
                                        "frac": None if res_achieved is None else res_achieved / peak,
                                        "kernel": "rve_residual_kernel<float> + rve_gather_nodes/norms_kernel",
                                        "bytes_per_element": RESIDUAL_BYTES_PER_ELEMENT_F32,
                                        "algorithmic_bytes": res_bytes},
                  "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                               "frac": None if achieved is None else achieved / peak, "traffic": None,
                               "peak_kind": kind, "kernel": "rve_pcg_cluster_kernel<float> (rve_pcg_kernel at cluster 1)",
                               "algorithmic_bytes": pcg_bytes,
                               "note": "algorithmic bytes of all PCG iterations over the PCG launches' event time; "
                                       "small RVEs stay in L2"},
                  "gpu_launches": out["launches"],
                  "e2e": {"value": value, "unit": "GP/s", "h2d_bytes_per_step": out["h2d_bytes_per_step"],
                          "d2h_bytes_per_step": out["d2h_bytes_per_step"],
                          "path": "pinned host macro strains -> batched Newton -> pinned host stresses, every step"},
                  "clocks": clocks.summary(), "cpu_baseline": cpu})  # fmt: skip
    if cpu is not None:
        line["speedup_rve_steps_vs_cpu"] = rve_steps_s / cpu["value"]
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# rno_train


def _tensor_peak() -> tuple[float, str]:
    from pathlib import Path

    path = Path(__file__).resolve().parent / "MEASURED_PEAKS.json"
    if path.exists():
        try:
            return float(json.loads(path.read_text())["bf16_tflops"]), "measured"
        except (KeyError, ValueError):
            pass
    return 1590.0, "fallback"


def _rno_train_cpu(windows: int = 6) -> dict:
    """The training loop in torch on the host (the reference's way of training its
    surrogate), same network, batch 512, TBPTT 50, float32, all host threads."""
    import torch

    from oracle.rno_torch import train_windows

    g = torch.Generator().manual_seed(0)
    shape = (600, 200, 6)
    out = train_windows(torch.randn(shape, generator=g), torch.randn(shape, generator=g), torch.randn(shape, generator=g),
                        torch.rand(shape[:2], generator=g) * 0.1, windows=windows)  # fmt: skip
    return {"value": out["path_steps"] / out["seconds"], "unit": "path-steps/s", "cores": out["threads"], "kind": "port",
            "sample": f"{windows} TBPTT windows of 512 paths x 50 steps, torch float32 autograd + Adam on the host "
                      "(oracle/rno_torch.py)"}  # fmt: skip


def _fe2_cpu(solves: int = 3) -> dict:
    """Direct FE^2 on the host: the oracle's 8^3 RVE solve (the reference's algorithm, FP64
    direct sparse solves) timed per solve; one solve per macro point per step, spread over
    all host cores without loss (which favours the CPU)."""
    from concrete_impact_b200.benchmarks import concrete_rve

    oracle = _oracle_for(concrete_rve(8, 0, 64), 1.0e-8)
    state = oracle.initial_state()
    t0 = time.perf_counter()
    for k in range(1, solves + 1):
        macro = np.array([-1.0e-3, 2.0e-4, 2.0e-4, 0.0, 0.0, 0.0]) * k / solves
        state = oracle.solve(macro, 1.0e-6, state, False)["state"]
    per_solve = (time.perf_counter() - t0) / solves
    cores = os.cpu_count() or 1
    return {"value": cores / (131072 * per_solve), "unit": "macro steps/s", "cores": cores, "kind": "port",
            "sample": f"oracle 8^3 RVE solves ({per_solve:.3f} s each, {solves} loading steps) x 131,072 macro points "
                      f"per step / {cores} cores"}  # fmt: skip


def _rno_inference_line(inf: dict, peak: float, kind: str) -> dict:
    """The trained surrogate's fused inference step at the 131,072 Gauss points of the
    64 x 16 x 16 macro bar (one persistent rno_window_forward launch per step)."""
    seconds = inf["ms_per_step"] / 1e3
    achieved = inf["flop_per_step"] / seconds / 1e12
    return {"points": inf["points"], "ms_per_step": inf["ms_per_step"], "points_per_s": inf["points"] / seconds,
            "steps_timed": inf["steps"], "launches": inf["launches"],
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "peak_kind": f"{kind} (cuBLAS bf16, burst)",
                         "note": "73,216 FLOP per point-step (unpadded MLP); the bias + exact-GELU epilogue on "
                                 "CUDA cores bounds the step"}}  # fmt: skip


def run_rno_train(args: argparse.Namespace) -> None:
    import torch

    from bench import ClockSampler
    from concrete_impact_b200.benchmarks import rno_training_workload

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    with ClockSampler(local) as clocks:
        out = rno_training_workload(epochs=args.steps, warmup_epochs=args.warmup)
    if rank != 0:
        return
    seconds = out["train_ms"] / 1e3
    value = out["path_steps"] / seconds
    peak, kind = _tensor_peak()
    achieved = out["flop"] / seconds / 1e12
    line = _line(args, "surrogate training throughput (path-steps/s; BF16 tcgen05 forward+backward, TBPTT 50, "
                       "batch 512, Adam)", value, "path-steps/s",
                 "rno_train: 2000 RVE paths x 200 steps (8^3 concrete RVE, FP32 solver), MLP 18-128-128-128-12 GELU",
                 {"ms_per_step": out["train_ms"] / max(out["epochs"], 1),
                  "dtype": "bf16 weights/activations, fp32 accumulation",
                  "epochs_timed": out["epochs"], "windows_timed": out["windows"],
                  "data_generation_s": out["data_generation_s"],
                  "val_error": {"trained": out["error_trained"], "untrained": out["error_untrained"],
                                "elastic_predictor": out["error_elastic"],
                                "note": "relative Frobenius stress error on 256 held-out paths solved in FP64"},
                  "loss_first_last": [out["loss_first"], out["loss_last"]],
                  "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                               "frac": achieved / peak, "traffic": None, "peak_kind": f"{kind} (cuBLAS bf16, burst)",
                               "kernel": "rno_window_forward/backward + split-K weight-gradient GEMMs",
                               "note": "219,648 FLOP per path-step; the time recursion leaves B/128 CTAs per step"},
                  "gpu_launches": out["launches"],
                  "inference": _rno_inference_line(out["inference"], peak, kind),
                  "e2e": {"value": value, "unit": "path-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 8,
                          "path": "device-resident dataset; one loss read-back per epoch"},
                  "clocks": clocks.summary(), "cpu_baseline": None if args.no_cpu_baseline else _rno_train_cpu()})  # fmt: skip
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# fe2


def _progress(stage: str, seconds: float, payload: dict) -> None:
    """Intermediate results on stderr, so that a run that stops later still reports them."""
    import sys

    sys.stderr.write(json.dumps({"stage": stage, "elapsed_s": seconds, **payload}, default=str) + "\n")
    sys.stderr.flush()


def _fe2_roofline(steps_per_s: float) -> dict:
    """Surrogate FLOPs of a macro step (131,072 points x the MLP's 73,216) over the whole
    step's time, against the bf16 tensor peak."""
    from concrete_impact_b200.benchmarks import RNO_FORWARD_FLOP

    peak, kind = _tensor_peak()
    achieved = steps_per_s * 131072 * RNO_FORWARD_FLOP / 1e12
    return {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": None, "peak_kind": f"{kind} (cuBLAS bf16, burst)",
            "note": "per step: one persistent fused surrogate launch (1,024 tiles of 128 points on one CTA per SM), "
                    "the gate kernels, and the macro Hex8 and Verlet kernels; time is the whole step's"}


def run_fe2(args: argparse.Namespace) -> None:
    """Train the surrogate (random + impact calibration paths), check it against all-direct
    FE^2 (FP64 RVEs) on a 64x2x2 bar, then time surrogate FE^2 on the 64x16x16 bar for
    ``--steps`` macro steps and all-direct FE^2 (FP32 RVEs) on the same bar for a short
    window from rest.  CIB_FE2_RECIPE (JSON of FE2Recipe fields), CIB_FE2_ACCURACY_STEPS and
    CIB_FE2_DIRECT_STEPS override the defaults; CIB_FE2_SAVE / CIB_FE2_LOAD store or reuse
    the trained surrogate.  On the full bar it also compares surrogate FE^2 with all-direct
    FE^2 over CIB_FE2_FULL_STEPS steps (default 200; 0 skips it) and runs the surrogate with
    the runtime judge (256 FP64 direct RVEs at seeded points: measuring every step, measuring
    every 10 steps, and escalating every 10 steps), whose homogenised-stress error and cost
    the line reports."""
    import torch

    from bench import ClockSampler
    from concrete_impact_b200.benchmarks import (
        FE2Recipe,
        fe2_accuracy,
        fe2_closed_loop,
        fe2_judged,
        fe2_speed,
        load_surrogate,
        save_surrogate,
        train_fe2_surrogate,
    )

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    fields = json.loads(os.environ.get("CIB_FE2_RECIPE", "{}"))
    recipe = FE2Recipe(**{k: tuple(v) if isinstance(v, list) else v for k, v in fields.items()})
    t0 = time.perf_counter()
    if os.environ.get("CIB_FE2_LOAD"):
        rno, envelope = load_surrogate(os.environ["CIB_FE2_LOAD"])
        info = {"loaded": os.environ["CIB_FE2_LOAD"]}
    else:
        rno, envelope, info = train_fe2_surrogate(recipe)
        if os.environ.get("CIB_FE2_SAVE"):
            save_surrogate(os.environ["CIB_FE2_SAVE"], rno, envelope)
    _progress("trained", time.perf_counter() - t0, info)
    acc = fe2_accuracy(rno, envelope, steps=int(os.environ.get("CIB_FE2_ACCURACY_STEPS", "400")))
    _progress("accuracy", time.perf_counter() - t0, acc)
    full = None
    if int(os.environ.get("CIB_FE2_FULL_STEPS", "200")) > 0:
        full = fe2_closed_loop(rno, envelope, steps=int(os.environ.get("CIB_FE2_FULL_STEPS", "200")))
        _progress("closed_loop_full_bar", time.perf_counter() - t0, full)
    with ClockSampler(local) as clocks:
        speed = fe2_speed(rno, envelope, rno_steps=args.steps, rno_warmup=args.warmup,
                          direct_steps=int(os.environ.get("CIB_FE2_DIRECT_STEPS", "3")))  # fmt: skip
        # the judge measuring every step (exact FP64 reference of the sampled points), every 10
        # steps (one RVE step per 10 macro steps), and every 10 steps with escalation
        judged = [fe2_judged(rno, envelope, steps=args.steps, warmup=args.warmup, every=every, threshold=threshold)
                  for every, threshold in ((1, None), (10, None), (10, 0.05))]  # fmt: skip
    _progress("judged", time.perf_counter() - t0, {"judged": judged})
    if rank != 0:
        return
    value = speed["rno_steps_per_s"]
    direct = speed.get("direct_steps_per_s")
    line = _line(args, "FE2 macro steps/s with surrogate macro points (64x16x16 Hex8 bar, 131,072 macro GP, "
                       "8^3 RVE fallback)", value, "macro steps/s",
                 "fe2: velocity-Verlet bar 0.64x0.16x0.16 m, half-sine 50 MPa 50 us, rho 2400, CFL 0.5",
                 {"ms_per_step": speed["rno_ms"] / max(speed["rno_steps"], 1), "dtype": "bf16 surrogate, f64 macro fields",
                  "direct_steps_per_s": direct, "speedup_vs_direct": value / direct if direct else None,
                  "direct_ms_per_step": speed.get("direct_ms"), "accuracy": acc,
                  "accuracy_full_bar": full, "judged_runs": judged,
                  "speedup_vs_direct_with_judge": {f"every_{j['every']}_{'escalating' if j['threshold'] else 'measuring'}":
                                                   (j["steps_per_s"] / direct if direct else None) for j in judged},
                  "training": {**info, "recipe": recipe.__dict__, "envelope": envelope},
                  "gate": {"flagged_points": speed["flagged_points"], "fallback_steps": speed["fallback_steps"]},
                  "simulated_time_s": speed["simulated_time_s"],
                  "roofline": _fe2_roofline(value),
                  "gpu_launches": speed["launches"],
                  "e2e": {"value": value, "unit": "macro steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                          "path": "ExplicitFE2.run on device-resident macro fields"},
                  "clocks": clocks.summary(), "cpu_baseline": None if args.no_cpu_baseline else _fe2_cpu()})  # fmt: skip
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# rve_ogrid


def _rve_ogrid_cpu(gpu_out: dict | None = None, sample_steps: int = 2) -> dict:
    """The general-mesh RVE oracle (NumPy/SciPy, direct solves) on the first steps of the
    same path; per-step time times the path's steps."""
    from concrete_impact_b200.benchmarks import ogrid_path, ogrid_rve
    from oracle import j2vp as oj
    from oracle.rve import OraclePhase
    from oracle.rve_general import general_rve_oracle

    mesh, model = ogrid_rve()
    newton = {"max_iterations": 25, "residual_absolute_tolerance": 1.0e-6, "residual_relative_tolerance": 1.0e-8,
              "increment_absolute_tolerance": 1.0e-14, "increment_relative_tolerance": 1.0e-10, "armijo": None}  # fmt: skip
    oracle = general_rve_oracle(mesh.nodes, mesh.elements, mesh.periodic_class_ids, int(mesh.opposite_face_nodes[0][0][0]),
                                [OraclePhase("j2", oj.mortar_params()), OraclePhase("elastic", None, 50.0e9, 0.2)],
                                mesh.element_phase_ids, newton)  # fmt: skip
    steps = 20 if gpu_out is None else gpu_out["steps"]
    times, strains = ogrid_path(steps)
    state = oracle.initial_state()
    diffs = []
    t0 = time.perf_counter()
    for k in range(1, sample_steps + 1):
        out = oracle.solve(strains[k], float(times[k] - times[k - 1]), state, True)
        state = out["state"]
        if gpu_out is not None:
            ref = np.asarray(gpu_out["macro_stress"][k - 1])
            diffs.append(float(np.abs(out["macro_stress"] - ref).max() / np.abs(ref).max()))
    per_step = (time.perf_counter() - t0) / sample_steps
    line = {"value": 1.0 / per_step, "unit": "RVE steps/s", "cores": 1, "kind": "port",
            "sample": f"general-mesh RVE oracle on the first {sample_steps} path steps, {per_step:.3f} s per step"}  # fmt: skip
    if diffs:
        line["max_rel_stress_diff_vs_oracle"] = max(diffs)
    return line


def run_rve_ogrid(args: argparse.Namespace) -> None:
    import torch

    from bench import ClockSampler
    from concrete_impact_b200.benchmarks import ogrid_rve_path_workload

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    with ClockSampler(local) as clocks:
        out = ogrid_rve_path_workload(steps=args.steps, warmup=args.warmup)
    if rank != 0:
        return
    seconds = out["ms"] / 1e3
    value = out["steps"] / seconds
    line = _line(args, "accepted RVE steps/s (cylindrical O-grid two-phase RVE, general Hex8 mesh, FP64)", value,
                 "RVE steps/s", f"rve_ogrid: 32x8x8 O-grid, {out['elements']} elements, {out['dofs']} DOF, 30 % "
                                "aggregate cylinder, proportional compression to 2.5e-3 in 20 steps, dt 5 us",
                 {"ms_per_step": out["ms"] / max(out["steps"], 1), "dtype": "f64",
                  "gp_evaluations_per_s": out["evaluations"] / seconds, "newton_iterations": out["newton_iterations"],
                  "final_macro_stress_pa": out["macro_stress"][-1],
                  "roofline": {"bound": "hbm", "achieved": None, "peak": None, "unit": "GB/s", "frac": None,
                               "traffic": None, "note": "one small RVE: launch- and latency-bound CSR kernels"},
                  "gpu_launches": out["launches"],
                  "e2e": {"value": value, "unit": "RVE steps/s", "h2d_bytes_per_step": 6 * 8,
                          "d2h_bytes_per_step": (6 + 36) * 8,
                          "path": "solve_prescribed_rve_path with host arrays in and out (value and e2e are one measurement)"},
                  "clocks": clocks.summary(), "cpu_baseline": None if args.no_cpu_baseline else _rve_ogrid_cpu(out)})  # fmt: skip
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# rno_energy


def _energy_case():
    from pathlib import Path

    from concrete_impact_b200.energy_rno import RVERNOModelConfig

    here = Path(__file__).resolve().parent / "tests" / "golden"
    meta = json.loads((here / "manifest.json").read_text())["rno_energy_c48"]
    with np.load(here / "rno_energy_c48.npz") as data:
        state_dict = {k[3:]: data[k] for k in data.files if k.startswith("w__")}
    return state_dict, RVERNOModelConfig(**{k: v for k, v in meta["model"].items() if k != "device"})


def _rno_energy_cpu(points: int = 2048) -> dict:
    """The NumPy oracle (float64, the reference's update) on a bounded sample of points."""
    from oracle import rno_energy as oe

    state_dict, cfg = _energy_case()
    rng = np.random.default_rng(7)
    strain = 5.0e-3 * rng.standard_normal((points, 6))
    latent = np.zeros((points, 6))
    anchor = oe.anchors(state_dict, 6)
    from threadpoolctl import threadpool_limits

    with threadpool_limits(1):
        t0 = time.perf_counter()
        oe.update(state_dict, strain, latent, np.full(points, 1.0e-4), cfg.reference_time_scale, cfg.integrator,
                  anchor=anchor)  # fmt: skip
        seconds = time.perf_counter() - t0
    return {"value": points / seconds, "unit": "point-updates/s", "cores": 1, "kind": "port",
            "sample": f"NumPy oracle (float64, one BLAS thread), one update of {points} points ({seconds:.2f} s)"}  # fmt: skip


def run_rno_energy(args: argparse.Namespace) -> None:
    import torch

    from bench import ClockSampler
    from concrete_impact_b200.benchmarks import energy_rno_workload

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    state_dict, cfg = _energy_case()
    with ClockSampler(local) as clocks:
        out = energy_rno_workload(state_dict, cfg, steps=args.steps, warmup=args.warmup)
    if rank != 0:
        return
    seconds = out["ms"] / 1e3
    value = out["points"] * out["steps"] / seconds
    achieved = value * out["flop_per_point"] / 1e12
    line = _line(args, "energy-based RVE-RNO point-updates/s (the reference's trained c48 model, 131,072 macro "
                       "points, FP32)", value, "point-updates/s",
                 "rno_energy: EnergyDissipationRVERNO 4x128 SiLU, latent 6, direct_rate, current-state integrator",
                 {"ms_per_step": out["ms"] / max(out["steps"], 1), "dtype": "f32",
                  "flop_per_point_update": out["flop_per_point"],
                  "roofline": {"bound": "fp32 cuda cores", "achieved": achieved, "peak": None, "unit": "TFLOP/s",
                               "frac": None, "traffic": None,
                               "note": "FP32 SIMT kernel; no measured FP32 CUDA-core peak for the denominator"},
                  "gpu_launches": out["launches"],
                  "e2e": {"value": value, "unit": "point-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                          "path": "update_batch on device-resident strains and latent states"},
                  "clocks": clocks.summary(), "cpu_baseline": None if args.no_cpu_baseline else _rno_energy_cpu()})  # fmt: skip
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# implicit_fe2

IMPLICIT_FE2_POINTS = 2048
IMPLICIT_FE2_EVALUATIONS = 3  # material evaluations per macro step assumed without a GPU run


def _implicit_fe2_cpu(solves_per_step: float, solves: int = 3) -> dict:
    """Implicit FE^2 on the host: the oracle's 8^3 RVE solve with its effective tangent (the
    reference's algorithm, FP64 direct sparse solves) timed per solve, times the RVE solves
    of one macro step, spread over all host cores without loss (which favours the CPU)."""
    from concrete_impact_b200.benchmarks import concrete_rve

    oracle = _oracle_for(concrete_rve(8, 0, 64), 1.0e-8)
    state = oracle.initial_state()
    t0 = time.perf_counter()
    for k in range(1, solves + 1):
        macro = np.array([-1.0e-3, 2.0e-4, 2.0e-4, 0.0, 0.0, 0.0]) * k / solves
        state = oracle.solve(macro, 5.0e-6, state, True)["state"]
    per_solve = (time.perf_counter() - t0) / solves
    cores = os.cpu_count() or 1
    return {"value": cores / (solves_per_step * per_solve), "unit": "macro steps/s", "cores": cores, "kind": "port",
            "sample": f"oracle 8^3 RVE solves with effective tangent ({per_solve:.3f} s each, {solves} loading "
                      f"steps) x {solves_per_step:.0f} RVE solves per macro step / {cores} cores"}  # fmt: skip


def run_implicit_fe2(args: argparse.Namespace) -> None:
    import torch

    from bench import ClockSampler
    from concrete_impact_b200.benchmarks import implicit_fe2_workload

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    forcing = os.environ.get("CIB_IMPLICIT_FE2_FORCING", "eisenstat_walker")  # "none": exact RVE PCG solves
    with ClockSampler(local) as clocks:
        out = implicit_fe2_workload(steps=args.steps, warmup=args.warmup, forcing=None if forcing == "none" else forcing)
    if rank != 0:
        return
    seconds = out["ms"] / 1e3
    value = out["steps"] / seconds
    per_step = out["rve_solves"] / max(out["steps"], 1)
    line = _line(args, "implicit FE2 accepted macro steps/s (16x4x4 Hex8 bar, 2,048 macro points, 8^3 concrete RVE "
                       "per point, FP64, Newmark average acceleration)", value, "macro steps/s",
                 "implicit_fe2: bar 0.16x0.04x0.04 m, x = 0 fixed, half-sine 40 MPa over 50 us, dt 5 us, "
                 f"macro Newton rel 1e-8, RVE Newton rel 1e-8, RVE linear forcing {forcing}",
                 {"ms_per_step": out["ms"] / max(out["steps"], 1), "dtype": "f64",
                  "rve_solves_per_s": out["rve_solves"] / seconds, "rve_solves_per_step": per_step,
                  "micro_gp_per_rve": 8 * out["rve_elements"], "newton_iterations": out["newton_iterations"],
                  "macro_pcg_iterations": out["macro_pcg_iterations"], "material_calls": out["material_calls"],
                  "tip_displacement_m": out["tip_displacement"], "dissipated_energy_j": out["dissipated_energy"],
                  "energy_residual_j": out["energy_residual"],
                  "roofline": {"bound": "hbm", "achieved": None, "peak": None, "unit": "GB/s", "frac": None,
                               "traffic": None, "kernel": "rve_pcg (batched RVE Newton solves)",
                               "note": "dominated by the batched RVE solves, whose PCG is latency-bound "
                                       "(profiles/rve_pcg_cluster_batch256.md)"},
                  "gpu_launches": out["launches"],
                  "e2e": {"value": value, "unit": "macro steps/s",
                          "h2d_bytes_per_step": out["h2d_bytes"] // max(out["steps"], 1),
                          "d2h_bytes_per_step": out["d2h_record_bytes"] // max(out["steps"] + 1, 1),
                          "path": "solve_material_implicit_newmark with host initial fields, host load vectors and "
                                  "host histories; the whole call is the timed region (value and e2e are one measurement)"},
                  "clocks": clocks.summary(),
                  "cpu_baseline": None if args.no_cpu_baseline else _implicit_fe2_cpu(per_step)})  # fmt: skip
    print(json.dumps(line), flush=True)


def run_reference(args: argparse.Namespace) -> None:
    """``--impl reference``: the oracle alone on the workload's CPU sample (rank 0)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    if args.workload in ("rno_train", "fe2", "implicit_fe2", "rve_ogrid", "rno_energy"):
        if args.workload == "rno_energy":
            c = _rno_energy_cpu()
        elif args.workload == "implicit_fe2":
            c = _implicit_fe2_cpu(float(IMPLICIT_FE2_POINTS * IMPLICIT_FE2_EVALUATIONS))
        elif args.workload == "rve_ogrid":
            c = _rve_ogrid_cpu()
        else:
            c = _rno_train_cpu() if args.workload == "rno_train" else _fe2_cpu()
        value, unit, sample = c["value"], c["unit"], c["sample"]
        metric = {"rno_train": "surrogate training throughput (torch on the host)",
                  "fe2": "direct FE2 macro steps/s (oracle RVE solves on the host)",
                  "implicit_fe2": "implicit FE2 macro steps/s (oracle RVE solves with effective tangents on the host, "
                                  f"{IMPLICIT_FE2_EVALUATIONS} material evaluations per step)",
                  "rve_ogrid": "accepted RVE steps/s (general-mesh RVE oracle, cylindrical O-grid)",
                  "rno_energy": "energy-based RVE-RNO point-updates/s (NumPy oracle on the host)"}[args.workload]  # fmt: skip
        line = {"impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32" if args.workload == "rno_train" else "f64", "data": "synthetic",
                "config": {"workload": args.workload}, "cpu_baseline": c,
                "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}  # fmt: skip
        print(json.dumps(line), flush=True)
        return
    if args.workload == "rve_batch":
        from concrete_impact_b200.benchmarks import concrete_rve
        from concrete_impact_b200.rve_builders import random_strain_path

        class _Setup:
            pass

        setup = _Setup()
        setup.models, times, strains = [], [], []
        for i in range(256):
            edge = int(np.random.default_rng(1000 + i).choice(EDGES))
            if edge > 12:
                continue
            setup.models.append(concrete_rve(edge, i, 32))
            t, e = random_strain_path(5000 + i, 200, 4, 1.0e-2, (1.0, 1000.0))
            times.append(t)
            strains.append(e)
            if len({m.divisions[0] for m in setup.models}) == 2:
                break
        setup.times, setup.strains = np.asarray(times), np.asarray(strains)
        c = _rve_batch_cpu(setup)
        value = 1.0 / (c["per_element_step_s"] * 5632.0)  # mean elements per RVE of the workload
        unit, metric = "RVE steps/s", "accepted RVE steps/s (oracle, mean-size RVE of the 256-RVE workload)"
        sample = f"oracle on edges 8 and 12, 2 steps each, {c['per_element_step_s'] * 1e6:.1f} us per element-step"
    else:
        from concrete_impact_b200.rve_builders import uniaxial_path

        times, exx = uniaxial_path(100)
        from concrete_impact_b200.benchmarks import concrete_rve

        oracle = _oracle_for(concrete_rve(8, 0, 64), 1.0e-8)
        state = oracle.initial_state()
        t0 = time.perf_counter()
        for step in (1, 2, 3):
            macro = np.zeros(6)
            macro[0] = exx[step]
            macro[1] = macro[2] = -0.2 * exx[step]
            state = oracle.solve(macro, float(times[step] - times[step - 1]), state, True)["state"]
        per_solve = (time.perf_counter() - t0) / 3
        value = 1.0 / (3.0 * per_solve)  # about three mixed-control solves per path step
        unit, metric = "RVE steps/s", "accepted RVE steps/s (oracle, 8^3 RVE, mixed-control path)"
        sample = f"oracle, 3 solves on the uniaxial path, {per_solve:.3f} s per solve, 3 solves per step"
    line = {"impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": {"workload": args.workload},
            "cpu_baseline": {"value": value, "unit": unit, "cores": 1, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}  # fmt: skip
    print(json.dumps(line), flush=True)


def run(args: argparse.Namespace) -> None:
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "rve_path":
        run_rve_path(args)
    elif args.workload == "rve_batch":
        run_rve_batch(args)
    elif args.workload == "rno_train":
        run_rno_train(args)
    elif args.workload == "fe2":
        run_fe2(args)
    elif args.workload == "implicit_fe2":
        run_implicit_fe2(args)
    elif args.workload == "rve_ogrid":
        run_rve_ogrid(args)
    elif args.workload == "rno_energy":
        run_rno_energy(args)
    else:
        raise SystemExit(f"unknown workload {args.workload}")
