"""The RVE workloads of ``bench.py --workload rve_path|rve_batch`` (one JSON line on rank 0).

* rve_path  -- one 8^3 two-phase concrete RVE, mixed-control uniaxial compression to
  -0.5 % in 100 steps at 10 /s (free components at zero macro stress), FP64.  Metric:
  accepted RVE path steps per second through the single-RVE public API
  (solve_rve_microequilibrium inside the mixed-control outer Newton).
* rve_batch -- 256 concrete RVEs of edges {8, 12, 16, 20, 24}, each on its own random
  macro strain path; one batched Newton solve per time index, FP32 element kernels and
  FP64 reductions.  Metric: micro Gauss-point return-map evaluations per second inside
  the Newton solves (all residual passes of all RVEs), with accepted RVE steps/s beside it.

The CPU baseline of both is the NumPy/SciPy oracle of the reference's RVE solve (direct
sparse solves, the reference's algorithm) timed on the host on a bounded sample.
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
            "max_rel_stress_diff_vs_gpu": max(diffs)}  # fmt: skip


def run_rve_path(args: argparse.Namespace) -> None:
    import torch

    from concrete_impact_b200.benchmarks import rve_path_workload

    rank = int(os.environ.get("RANK", "0"))
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    from bench import ClockSampler

    rve_path_workload(max(args.warmup, 1))  # warm-up: a short path
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clocks:
        out = rve_path_workload(args.steps)
    if rank != 0:
        return
    cpu = None if args.no_cpu_baseline else _rve_path_cpu(out)
    seconds = out["ms"] / 1e3
    value = out["steps"] / seconds
    # dominant work: the Newton residual passes (984 algorithmic bytes per element, FP64
    # element state counted at 8 bytes) -- one CTA per system, so the fraction is small
    peak, kind = _peak()
    line = _line(args, "accepted RVE steps/s (8^3 concrete RVE, mixed-control uniaxial path, FP64)", value,
                 "RVE steps/s", "rve_path: 8^3 two-phase RVE, seed 0, uniaxial compression -0.5 % in 100 steps at 10/s",
                 {"ms_per_step": out["ms"] / out["steps"], "dtype": "f64",
                  "gp_evaluations_per_s": out["gp_evaluations"] / seconds,
                  "solves": out["solves"], "newton_iterations": out["newton_iterations"],
                  "pcg_iterations": out["pcg_iterations"],
                  "final_macro_stress_xx_pa": float(out["macro_stress"][-1][0]),
                  "roofline": {"bound": "hbm", "achieved": None, "peak": peak, "unit": "GB/s", "frac": None,
                               "traffic": None, "peak_kind": kind,
                               "note": "one RVE = one CTA per kernel: latency-bound, not a bandwidth workload"},
                  "gpu_launches": None,
                  "e2e": {"value": value, "unit": "RVE steps/s", "h2d_bytes_per_step": 6 * 8 * (out["solves"] // out["steps"] + 1),
                          "d2h_bytes_per_step": (6 + 36) * 8 * (out["solves"] // out["steps"] + 1),
                          "path": "solve_rve_microequilibrium (host arrays in and out) in the mixed-control loop"},
                  "clocks": clocks.summary(), "cpu_baseline": cpu})  # fmt: skip
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# rve_batch

PCG_TANGENT_BYTES_PER_GP = 8 * 4  # FP32 tangent parameters (n[6], f, c) of a plastic point
PCG_VECTOR_BYTES_PER_ELEMENT = 10 * 3 * 8  # p gather, Ap write, x/r/p/dinv/Ap updates, FP64


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


def run_rve_batch(args: argparse.Namespace) -> None:
    import torch

    from bench import ClockSampler
    from concrete_impact_b200.benchmarks import rve_batch_setup, rve_batch_workload

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    setup = rve_batch_setup(256, 200)
    with ClockSampler(local) as clocks:
        out = rve_batch_workload(setup, args.warmup, args.steps)
    if rank != 0:
        return
    seconds = out["ms"] / 1e3
    value = out["gp_evaluations"] / seconds
    peak, kind = _peak()
    pcg_ms = out["kernel_ms"].get("pcg", 0.0)
    pcg_bytes = out["pcg_element_iterations"] * (8 * PCG_TANGENT_BYTES_PER_GP * out["plastic_fraction"]
                                                 + PCG_VECTOR_BYTES_PER_ELEMENT)  # fmt: skip
    achieved = pcg_bytes / (pcg_ms / 1e3) / 1e9 if pcg_ms > 0 else None
    cpu = None
    if not args.no_cpu_baseline:
        c = _rve_batch_cpu(setup)
        cpu_rve_steps = 1.0 / (c["per_element_step_s"] * c["total_elements"] / len(setup.models))
        cpu = {"value": cpu_rve_steps, "unit": "RVE steps/s", "cores": 1, "kind": "port",
               "sample": f"oracle (NumPy/SciPy, direct solves) on RVEs {c['picked']} (edges 8 and 12), first 2 path "
                         f"steps, {c['per_element_step_s'] * 1e6:.1f} us per element-step scaled to "
                         f"{c['total_elements']:,} elements"}  # fmt: skip
    rve_steps_s = out["rve_steps"] / seconds
    line = _line(args, "micro Gauss-point evaluations/s inside the batched RVE Newton solve (256 uneven RVEs)", value,
                 "GP/s", "rve_batch: 256 two-phase RVEs, edges {8,12,16,20,24}, random 4-segment paths, FP32 elements",
                 {"ms_per_step": out["ms"] / args.steps, "dtype": "f32 elements, f64 reductions and history",
                  "accepted_rve_steps_per_s": rve_steps_s, "elements": out["elements"],
                  "gauss_points": out["gauss_points"], "newton_max": out["newton_max"], "pcg_max": out["pcg_max"],
                  "pcg_total": out["pcg_total"], "plastic_fraction": out["plastic_fraction"],
                  "kernel_ms": out["kernel_ms"], "kernel_launches": out["kernel_launches"],
                  "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                               "frac": None if achieved is None else achieved / peak, "traffic": None,
                               "peak_kind": kind, "kernel": "rve_pcg_kernel<float>",
                               "algorithmic_bytes": pcg_bytes,
                               "note": "algorithmic bytes of all PCG iterations over the PCG launches' event time; "
                                       "small RVEs stay in L2"},
                  "gpu_launches": sum(out["kernel_launches"].values()),
                  "e2e": {"value": value, "unit": "GP/s", "h2d_bytes_per_step": out["h2d_bytes_per_step"],
                          "d2h_bytes_per_step": out["d2h_bytes_per_step"],
                          "path": "pinned host macro strains -> batched Newton -> pinned host stresses, every step"},
                  "clocks": clocks.summary(), "cpu_baseline": cpu})  # fmt: skip
    if cpu is not None:
        line["speedup_rve_steps_vs_cpu"] = rve_steps_s / cpu["value"]
    print(json.dumps(line), flush=True)


def run_reference(args: argparse.Namespace) -> None:
    """``--impl reference``: the oracle alone on the workload's CPU sample (rank 0)."""
    if int(os.environ.get("RANK", "0")) != 0:
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
    else:
        raise SystemExit(f"unknown workload {args.workload}")
