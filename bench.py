"""Benchmark of the batched J2 Perzyna return map on B200 (one JSON line on rank 0).

Workload: the isolated batched return map, 16,777,216 Gauss points in structure-of-arrays
layout, state (stress 6, plastic strain 6, equivalent plastic strain 1), strain increments
N(0, 2e-4^2) per component, dt = 1e-5 s, equivalent plastic strain U[0, 0.01], stress a
random deviatoric direction at q = U[0.8, 1.0] x yield radius (mortar: E 25 GPa, nu 0.2,
sigma_y 20 MPa, H 2 GPa, eta 1e-3 s, m = 1).  A step is one pass over the batch with the
consistent tangent written (the reference's `J2ViscoplasticMaterial.update` with
tangent=True).  Headline precision is float64 (the reference's); the float32 variant of
the method is reported alongside.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload return_map|rve_path|rve_batch|rno_train|fe2|implicit_fe2|rve_ogrid|rno_energy]

Under torchrun each rank updates its own batch of the same size (independent points:
weak scaling, no collective on the data path); rank 0 prints the line.  The other
workloads (the RVE path, the 256-RVE batch, surrogate training, explicit and implicit
FE^2, the cylindrical O-grid RVE path) are in bench_workloads.py.
"""

from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

REPO = Path(__file__).resolve().parent
N_POINTS = 16_777_216
BYTES_PER_POINT = {"f64": 544, "f32": 280}  # algorithmic bytes per point with tangent
METRIC = "Gauss-point updates/s (batched J2 Perzyna return map with consistent tangent)"
UNIT = "GP/s"
WORKLOAD = "isolated batched return map, 16,777,216 GP SoA, FP64 state, tangent written"
FALLBACK_HBM_GBS = 6650.0
# (timed steps, warm-up steps) per workload when not given on the command line
WORKLOAD_DEFAULTS = {"return_map": (200, 5), "rve_path": (100, 3), "rve_batch": (5, 3), "rno_train": (300, 1),
                     "fe2": (5000, 5), "implicit_fe2": (10, 3), "rve_ogrid": (20, 3), "rno_energy": (50, 3)}


def parse_args() -> argparse.Namespace:
    parser = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    parser.add_argument("--gpus", type=int, default=1)
    parser.add_argument("--steps", type=int, default=None)
    parser.add_argument("--warmup", type=int, default=None)
    parser.add_argument("--workload", choices=tuple(WORKLOAD_DEFAULTS), default="return_map")
    parser.add_argument("--impl", choices=("ours", "reference"), default="ours")
    parser.add_argument("--points", type=int, default=N_POINTS, help=argparse.SUPPRESS)
    parser.add_argument("--e2e-steps", type=int, default=3)
    parser.add_argument("--no-cpu-baseline", action="store_true", help=argparse.SUPPRESS)
    # rve_batch: number of RVEs (256 is the workload; fewer for a small profiling case)
    parser.add_argument("--rves", type=int, default=256, help=argparse.SUPPRESS)
    args = parser.parse_args()
    steps, warmup = WORKLOAD_DEFAULTS[args.workload]
    args.steps = steps if args.steps is None else args.steps
    args.warmup = warmup if args.warmup is None else args.warmup
    return args


# ---------------------------------------------------------------------------------------
# Reference arm: the reference's per-point CPU execution, ported (the reference checkout
# does not exist on the GPU machine), over all host cores in a spawn pool as the
# reference's own process-pool backend runs it.

_WORKER: dict = {}


def _ref_worker_init(points: int, seed: int) -> None:
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    sys.path.insert(0, str(REPO))
    import numpy as np

    from oracle import j2vp as oj

    inputs = oj.config1_inputs(points, seed=seed)
    p = oj.mortar_params()
    c = oj.elasticity_matrix(p.young_modulus, p.poisson_ratio)
    strain = inputs["stress"] @ np.linalg.inv(c).T + inputs["plastic_strain"] + inputs["dstrain"]
    _WORKER.update(p=p, strain=strain, ep=inputs["plastic_strain"], q=inputs["eqps"], dt=inputs["dt"])


def _ref_task(_: int) -> int:
    from oracle.j2vp_loop import update_points_loop

    w = _WORKER
    update_points_loop(w["p"], w["strain"], w["ep"], w["q"], w["dt"], None)
    return int(w["strain"].shape[0])


def run_reference(args: argparse.Namespace) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    per_task = 1024  # points per worker per step (~40 ms of one core)
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores, initializer=_ref_worker_init, initargs=(per_task, 1234)) as pool:
        for _ in range(max(args.warmup, 1)):
            pool.map(_ref_task, range(cores))
        times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            done = sum(pool.map(_ref_task, range(cores)))
            times.append(time.perf_counter() - t0)
    total = sum(times)
    value = done * len(times) / total
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded; no dataset involved)",
        "config": {"workload": WORKLOAD, "points_per_gpu": args.points, "parallelism": f"host process pool x{cores}",
                   "sample_points_per_step": done},
        "cpu_baseline": {
            "value": value,
            "unit": UNIT,
            "cores": cores,
            "kind": "port",
            "sample": f"{per_task} points per worker per step x {cores} spawn workers = {done} points per step, a "
            "bounded sample of the 16,777,216-point workload; per-point loop port of J2ViscoplasticMaterial.update "
            "(strain_rates=None, tangent) -- oracle/j2vp_loop.py",
        },
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# Clock sampling during the timed region.


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while active."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")  # fmt: skip

    def __init__(self, local_rank: int) -> None:
        visible = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
        self.gpu_index = visible[local_rank] if local_rank < len(visible) else str(local_rank)
        self.proc = None
        self.file = None

    def __enter__(self) -> ClockSampler:
        exe = shutil.which("nvidia-smi")
        if exe:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                [exe, f"--id={self.gpu_index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL,
            )  # fmt: skip
            time.sleep(0.3)
        return self

    def __exit__(self, *exc) -> None:
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self) -> dict:
        if self.file is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.file.flush()
        rows = [r.split(",") for r in Path(self.file.name).read_text().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows]
        mx = max(float(r[2]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip().lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows)}  # fmt: skip


# ---------------------------------------------------------------------------------------
# Our arm.


def hbm_peak() -> tuple[float, str]:
    path = REPO / "MEASURED_PEAKS.json"
    if path.exists():
        try:
            return float(json.loads(path.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kind: str) -> float | None:
    """DRAM bytes per point of the SoA kernel from the committed ncu summary, if any."""
    path = REPO / "profiles" / "j2vp_soa_traffic.json"
    if not path.exists():
        return None
    data = json.loads(path.read_text())
    return data.get(kind, {}).get("dram_bytes_per_point")


def cpu_baseline_c(n_sample: int) -> dict:
    """The C oracle (OpenMP, all host threads) on a bounded sample of the workload."""
    import numpy as np

    from oracle import j2vp as oj
    from oracle.native import j2vp_incremental_c, max_threads

    inputs = oj.config1_inputs(n_sample, seed=99)
    de = np.ascontiguousarray(inputs["dstrain"].T)
    s0 = np.ascontiguousarray(inputs["stress"].T)
    ep0 = np.ascontiguousarray(inputs["plastic_strain"].T)
    p = oj.mortar_params()
    j2vp_incremental_c(p, inputs["dt"], de[:, :1024].copy(), s0[:, :1024].copy(), ep0[:, :1024].copy(), inputs["eqps"][:1024].copy())
    reps, t_total = 0, 0.0
    while t_total < 8.0 and reps < 50:
        t0 = time.perf_counter()
        j2vp_incremental_c(p, inputs["dt"], de, s0, ep0, inputs["eqps"])
        t_total += time.perf_counter() - t0
        reps += 1
    threads = max_threads()
    return {
        "value": n_sample * reps / t_total,
        "unit": UNIT,
        "cores": threads,
        "kind": "port",
        "sample": f"{reps} passes over {n_sample:,} points of the same workload, float64, tangent written; "
        "plain-C restatement (oracle/j2vp_oracle.c, gcc -O3 -fopenmp)",
    }


def max_over_ranks(value: float, dist, device) -> float:
    """The largest of every rank's value (one all-reduce; ``dist`` None = one process)."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_ours(args: argparse.Namespace) -> None:
    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    cpu_line = None
    if rank == 0 and not args.no_cpu_baseline:
        cpu_line = cpu_baseline_c(1 << 21)  # before the first GPU call
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    from concrete_impact_b200 import batched
    from concrete_impact_b200.materials import J2ViscoplasticMaterial, MaterialUpdateSettings
    from oracle import j2vp as oj

    mp_ = oj.mortar_params()
    material = J2ViscoplasticMaterial("mortar", 2200.0, mp_.young_modulus, mp_.poisson_ratio, mp_.yield_stress,
                                      mp_.hardening_modulus, mp_.time_scale, mp_.reference_stress, mp_.rate_exponent)  # fmt: skip
    settings = MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)
    n = args.points
    dt = 1.0e-5

    def make_inputs(dtype):
        g = torch.Generator(device=dev)
        g.manual_seed(1234 + rank)
        q = torch.rand(n, generator=g, device=dev, dtype=torch.float64) * 0.01
        d = torch.randn((6, n), generator=g, device=dev, dtype=torch.float64)
        d[:3] -= d[:3].mean(dim=0, keepdim=True)
        qd = torch.sqrt(1.5 * ((d[:3] ** 2).sum(0) + 2.0 * (d[3:] ** 2).sum(0)))
        radius = mp_.yield_stress + mp_.hardening_modulus * q
        s = d * ((0.8 + 0.2 * torch.rand(n, generator=g, device=dev, dtype=torch.float64)) * radius / qd)
        de = torch.randn((6, n), generator=g, device=dev, dtype=torch.float64) * 2.0e-4
        del d, qd
        return de.to(dtype).contiguous(), batched.SoAState(s.to(dtype).contiguous(),
                                                           torch.zeros((6, n), device=dev, dtype=dtype), q)  # fmt: skip

    def device_timed(dtype):
        de, st0 = make_inputs(dtype)
        st1 = batched.SoAState.empty(n, dtype, dev)
        tan = torch.empty((36, n), device=dev, dtype=dtype)
        flags = batched._flags(dev)
        states = [st0, st1]
        stream = torch.cuda.current_stream()
        for i in range(args.warmup):
            batched.launch_j2vp_soa(material, settings, dt, de, states[i % 2], states[(i + 1) % 2], tan, flags)
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        for i in range(args.steps):
            starts[i].record(stream)
            batched.launch_j2vp_soa(material, settings, dt, de, states[i % 2], states[(i + 1) % 2], tan, flags)
            ends[i].record(stream)
        t_end.record(stream)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        total_ms = t_start.elapsed_time(t_end)
        kernel_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
        failures = int(flags[0].item())
        active = None
        del de, states, st0, st1, tan
        torch.cuda.empty_cache()
        return total_ms, kernel_ms, failures, active

    def e2e_timed(dtype, compact: bool = False):
        """Host-resident batch: pinned host SoA in, pinned host SoA + tangent out (36 rows,
        or the 8-row compact form)."""
        de_d, st_d = make_inputs(dtype)
        de_h = de_d.cpu().pin_memory()
        st_h = batched.SoAState(st_d.stress.cpu().pin_memory(), st_d.plastic_strain.cpu().pin_memory(),
                                st_d.eqps.cpu().pin_memory())  # fmt: skip
        del de_d, st_d
        torch.cuda.empty_cache()
        out_h = batched.SoAState(torch.empty((6, n), dtype=dtype).pin_memory(), torch.empty((6, n), dtype=dtype).pin_memory(),
                                 torch.empty(n, dtype=torch.float64).pin_memory())  # fmt: skip
        tan_h = torch.empty((8 if compact else 36, n), dtype=dtype).pin_memory()
        pipe = batched.J2HostPipeline(material, settings, dtype, chunk=1 << 20, compact_tangent=compact)
        pipe.run(dt, de_h, st_h, out_h, tan_h)  # warm-up
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        fails = -1
        for _ in range(args.e2e_steps):
            fails = max(fails, pipe.run(dt, de_h, st_h, out_h, tan_h))
        elapsed = time.perf_counter() - t0
        h2d, d2h = batched.J2HostPipeline.bytes_per_point(dtype, True, compact)
        launches = math.ceil(n / pipe.chunk) * args.e2e_steps
        del pipe, de_h, st_h, out_h, tan_h
        torch.cuda.empty_cache()
        return elapsed, h2d * n, d2h * n, fails, launches

    peak, peak_kind = hbm_peak()
    with ClockSampler(local_rank) as clocks:
        total64, kms64, fail64, _ = device_timed(torch.float64)
        total32, kms32, fail32, _ = device_timed(torch.float32)
    e2e_s, h2d_b, d2h_b, e2e_fail, e2e_launches = e2e_timed(torch.float64)
    e2e_more = {}
    for key, dtype, compact in (("f64_compact_tangent", torch.float64, True), ("f32", torch.float32, False),
                                ("f32_compact_tangent", torch.float32, True)):  # fmt: skip
        secs, hb, db, fl, _ = e2e_timed(dtype, compact)
        e2e_fail = max(e2e_fail, fl)
        e2e_more[key] = (secs, hb, db)

    def reduce_max(x: float) -> float:
        return max_over_ranks(x, dist, dev)

    total64 = reduce_max(total64)
    total32 = reduce_max(total32)
    e2e_s = reduce_max(e2e_s)
    e2e_more = {k: (reduce_max(v[0]), v[1], v[2]) for k, v in e2e_more.items()}
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return
    if fail64 != -1 or fail32 != -1 or e2e_fail != -1:
        raise SystemExit(f"return map reported failing points: {fail64}, {fail32}, {e2e_fail}")
    value64 = world * n * args.steps / (total64 / 1e3)
    value32 = world * n * args.steps / (total32 / 1e3)
    k64 = statistics.mean(kms64)
    k32 = statistics.mean(kms32)
    ach64 = BYTES_PER_POINT["f64"] * n / (k64 / 1e3) / 1e9
    ach32 = BYTES_PER_POINT["f32"] * n / (k32 / 1e3) / 1e9
    t64 = ncu_traffic("f64")
    line = {
        "metric": METRIC,
        "value": value64,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total64 / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded on device; distributions of the isolated return-map workload)",
        "config": {"workload": WORKLOAD, "points_per_gpu": n, "parallelism": f"replicas x{world}",
                   "l2": "inputs larger than L2 (2.5 GB read per step)", "state": "ping-pong committed/trial buffers"},  # fmt: skip
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": ach64, "peak": peak, "unit": "GB/s", "frac": ach64 / peak,
                     "peak_kind": f"{peak_kind} (copy bandwidth, burst)",
                     "traffic": None if t64 is None else t64 * n,
                     "algorithmic_bytes_per_launch": BYTES_PER_POINT["f64"] * n,
                     "kernel": "j2vp_soa_kernel<double,2,1>", "mean_launch_ms": k64},  # fmt: skip
        "variants": {"f32": {"value": value32, "unit": UNIT, "ms_per_step": total32 / args.steps,
                             "roofline": {"achieved": ach32, "peak": peak, "frac": ach32 / peak,
                                          "traffic": None if ncu_traffic("f32") is None else ncu_traffic("f32") * n,
                                          "algorithmic_bytes_per_launch": BYTES_PER_POINT["f32"] * n,
                                          "mean_launch_ms": k32},
                             "dtype": "f32 state and tangent, f64 equivalent plastic strain"}},  # fmt: skip
        "e2e": {"value": world * n * args.e2e_steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d_b,
                "d2h_bytes_per_step": d2h_b, "path": "J2HostPipeline: pinned host SoA -> cib_j2vp_update_soa_f64 -> pinned host",
                "steps": args.e2e_steps, "gpu_launches": e2e_launches,
                "variants": {k: {"value": world * n * args.e2e_steps / v[0], "h2d_bytes_per_step": v[1],
                                 "d2h_bytes_per_step": v[2],
                                 "path": ("J2HostPipeline, compact tangent (n, f, c: 8 values instead of 36)"
                                          if "compact" in k else "J2HostPipeline") + (", FP32 state" if "f32" in k
                                                                                      else "")}
                             for k, v in e2e_more.items()}},  # fmt: skip
        "clocks": clocks.summary(),
        "cpu_baseline": cpu_line,
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    args = parse_args()
    sys.path.insert(0, str(REPO))
    if args.workload != "return_map":
        import bench_workloads

        bench_workloads.run(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
