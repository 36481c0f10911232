"""CPU tests of host-side helpers: the PCG cluster-size heuristic, the FP32 Newton settings,
the host training-loop baseline and the kernel-timer command line."""

from __future__ import annotations

from types import SimpleNamespace

import numpy as np
import torch

from concrete_impact_b200.rve import auto_pcg_cluster
from concrete_impact_b200.rve_builders import default_newton, fp32_newton
from oracle.rno_torch import train_windows


def _batch(edges):
    counts = np.asarray([e ** 3 for e in edges], dtype=np.int64)
    return SimpleNamespace(elem_counts=counts, min_nz=min(edges))


def test_auto_cluster_follows_the_largest_rve_and_the_thinnest() -> None:
    assert auto_pcg_cluster(_batch([8, 8])) == 1
    assert auto_pcg_cluster(_batch([8, 12])) == 1  # 1,728 elements: one CTA's share
    assert auto_pcg_cluster(_batch([8, 16])) == 2
    assert auto_pcg_cluster(_batch([8, 20])) == 4
    assert auto_pcg_cluster(_batch([8, 24])) == 8
    assert auto_pcg_cluster(_batch([4, 24])) == 4  # at most the smallest z layer count
    assert auto_pcg_cluster(_batch([2, 24])) == 2


def test_fp32_newton_tolerance_scales_with_the_traction_resultant() -> None:
    n32, n64 = fp32_newton(), default_newton()
    assert n32.residual_absolute_tolerance == 1e-6 * 20.0e6
    assert fp32_newton(40.0e6, 0.5).residual_absolute_tolerance == 1e-6 * 20.0e6
    assert n32.residual_relative_tolerance == 1e-6 and n64.residual_relative_tolerance == 1e-8


def test_host_training_loop_learns_a_linear_map() -> None:
    g = torch.Generator().manual_seed(0)
    P, T = 64, 50
    strain = torch.randn((P, T, 6), generator=g)
    rate = torch.zeros((P, T, 6))
    stress = 0.5 * strain
    coef = torch.full((P, T), 0.01)
    out = train_windows(strain, rate, stress, coef, windows=30, batch=64, tbptt=50, lr=3e-3, threads=2)
    assert out["path_steps"] == 30 * 64 * 50 and out["seconds"] > 0
    assert out["loss_last"] < 0.2 * out["loss_first"]


def test_kernel_timer_cli_names_its_workloads() -> None:
    """``python -m concrete_impact_b200.benchmarks`` refuses an unknown workload with its usage
    line (the timed workloads themselves need a GPU)."""
    import pytest

    from concrete_impact_b200.benchmarks import _main

    with pytest.raises(SystemExit) as info:
        _main(["unknown"])
    assert "rno_inference|gemm_wgrad" in str(info.value)
