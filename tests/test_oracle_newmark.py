"""CPU tests of the implicit Newmark oracle (oracle/newmark.py) and the host-side step
control of concrete_impact_b200.dynamics.

The oracle is pinned to the reference's own solve_material_implicit_newmark
(src/fem/dynamics/material.py:300-731), run by tests/golden/make_golden.py on pressure-pulse
bars: J2 Perzyna points with fixed steps, adaptive steps with Armijo and a two-iteration
Newton budget (cutbacks and growth), and FE2 with a two-phase 4^3 RVE at every point (the
first step here; the whole run takes minutes on the CPU).
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import load_case
from oracle import fe2 as of
from oracle import j2vp as oj
from oracle import newmark as on
from oracle.rve import OraclePhase, OracleRVE, RVEOracle, box_mesh

HISTORIES = ("displacement", "velocity", "acceleration", "stresses", "kinetic_energy", "free_energy",
             "dissipated_energy", "external_work")  # fmt: skip
NEWTON_KEYS = ("max_iterations", "residual_absolute_tolerance", "residual_relative_tolerance",
               "increment_absolute_tolerance", "increment_relative_tolerance")  # fmt: skip


def oracle_setup(name: str):
    """Oracle bar, point material, load, Newton settings and golden arrays of one case."""
    g, meta = load_case(name)
    nodes, elements = box_mesh(meta["bar"]["lengths"], meta["bar"]["divisions"])
    if "rve" in meta:
        r = meta["rve"]
        mortar = oj.J2Params(25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0)
        rve = OracleRVE(tuple(r["divisions"]), (1.0, 1.0, 1.0),
                        [OraclePhase("j2", mortar), OraclePhase("elastic", None, 50.0e9, 0.2)], g["element_phase"],
                        dict(zip(NEWTON_KEYS, r["newton"][:5]), armijo=None))  # fmt: skip
        material, density = on.PointRVE(RVEOracle(rve)), r["density"]
    else:
        material, density = on.PointJ2(oj.J2Params(**meta["material"]["params"])), meta["material"]["density"]
    unit, amp, dur = g["unit_force"], meta["amplitude"], meta["duration"]

    def load(t):
        return (amp * math.sin(math.pi * t / dur) if 0.0 <= t <= dur else 0.0) * unit

    newton = dict(zip(NEWTON_KEYS, meta["newton"][:5]))
    newton["armijo"] = dict(sufficient_decrease=1.0e-4, reduction_factor=0.5, max_backtracks=20) if meta["newton"][5] else None
    return on.Bar(nodes, elements, density), material, load, newton, g, meta


def _compare(out, g, steps=None, tol=1.0e-12):
    sl = slice(None) if steps is None else slice(0, steps + 1)
    np.testing.assert_array_equal(out["times"], g["times"][sl])
    np.testing.assert_array_equal(out["newton_iterations"], g["newton_iterations"][sl])
    np.testing.assert_array_equal(out["rejected_step_counts"], g["rejected_step_counts"][sl])
    np.testing.assert_array_equal(out["armijo_backtracks"], g["armijo_backtracks"][sl])
    for key in HISTORIES:
        ref = g[key][sl]
        scale = max(float(np.abs(ref).max()), 1e-300)
        np.testing.assert_allclose(out[key], ref, rtol=0, atol=tol * scale, err_msg=key)


@pytest.mark.parametrize("name", ["newmark_j2_bar_fixed", "newmark_j2_bar_adaptive"])
def test_oracle_matches_reference_newmark_j2(name) -> None:
    bar, material, load, newton, g, meta = oracle_setup(name)
    out = on.implicit_newmark(bar, material, g["fixed_dofs"], load, meta["time_step"], meta["num_steps"], 0.25, 0.5,
                              newton, on.Adaptive(enabled=meta["adaptive"]))  # fmt: skip
    _compare(out, g)
    assert [list(r) for r in out["rejected_reasons"]] == meta["rejected_reasons"]
    np.testing.assert_allclose(out["energy_residual"], g["energy_residual"], rtol=0,
                               atol=1e-11 * float(np.abs(g["external_work"]).max()))  # fmt: skip
    if meta["adaptive"]:
        assert meta["rejected"] > 0 and len(set(np.round(np.diff(out["times"]), 12))) > 2


def test_oracle_matches_reference_fe2_first_step() -> None:
    bar, material, load, newton, g, meta = oracle_setup("newmark_fe2_bar")
    dt = meta["time_step"]
    out = on.implicit_newmark(bar, material, g["fixed_dofs"], load, dt, 1, 0.25, 0.5, newton)
    _compare(out, g, steps=1, tol=1e-12)
    assert g["newton_iterations"][1] >= 1  # the step used the RVE effective tangents


def test_consistent_mass_rows_sum_to_lumped_mass() -> None:
    rng = np.random.default_rng(3)
    nodes, elements = box_mesh((0.3, 0.2, 0.1), (3, 2, 2))
    nodes = nodes + rng.uniform(-0.01, 0.01, nodes.shape)  # distorted hexahedra
    m = on.consistent_mass(nodes, elements, 2400.0)
    np.testing.assert_allclose(np.asarray(m.sum(axis=1)).ravel(), of.lumped_mass(nodes, elements, 2400.0), rtol=1e-13)
    assert abs(m - m.T).max() <= 1e-14 * abs(m).max()
    _, det = of.b_matrices(nodes, elements)
    assert m.sum() == pytest.approx(3 * 2400.0 * det.sum(), rel=1e-13)


def test_step_control_rules_and_armijo_search() -> None:
    from concrete_impact_b200.dynamics import (AdaptiveTimeStepSettings, ArmijoLineSearchError, cut_back_time_step,
                                               grow_time_step, perform_armijo_search)  # fmt: skip
    from concrete_impact_b200.rve import ArmijoSettings

    s = AdaptiveTimeStepSettings(enabled=True)
    assert cut_back_time_step(1.0e-6, 1.0e-6, s) == 0.5e-6
    assert cut_back_time_step(0.1e-6, 1.0e-6, s) == 1.0e-6 / 16.0
    assert grow_time_step(0.5e-6, 1.0e-6, s) == 1.0e-6
    assert grow_time_step(1.5e-6, 1.0e-6, s) == 2.0e-6
    for bad in (dict(minimum_factor=0.0), dict(maximum_factor=0.5), dict(cutback_factor=1.0), dict(growth_factor=1.0),
                dict(easy_step_count=0)):  # fmt: skip
        with pytest.raises(ValueError):
            AdaptiveTimeStepSettings(**bad)
    # residual norm of a candidate step s along a direction that overshoots: |1 - 3 s|
    res = perform_armijo_search(1.0, lambda step: abs(1.0 - 3.0 * step), ArmijoSettings(enabled=True))
    assert (res.step_length, res.backtracks) == (0.5, 1)
    with pytest.raises(ArmijoLineSearchError):
        perform_armijo_search(1.0, lambda step: 2.0, ArmijoSettings(enabled=True, max_backtracks=3))


def test_average_acceleration_conserves_energy_on_an_elastic_bar() -> None:
    """Newmark with beta = 1/4, gamma = 1/2 conserves the discrete energy of a linear
    system: with the J2 yield stress out of reach the oracle's energy residual (kinetic +
    free + dissipated - external work) stays at roundoff over a pulse and its free
    vibration."""
    nodes, elements = box_mesh((0.06, 0.01, 0.01), (6, 1, 1))
    elastic = oj.J2Params(25.0e9, 0.2, 1.0e12, 2.0e9, 1.0e-3, 1.0e12, 1.0)
    bar = on.Bar(nodes, elements, 2200.0)
    fixed = (3 * np.flatnonzero(np.isclose(nodes[:, 0], 0.0))[:, None] + np.arange(3)).ravel()
    unit = np.zeros(3 * nodes.shape[0])
    unit[3 * np.flatnonzero(np.isclose(nodes[:, 0], 0.06))] = -1.0e-4 / 4.0

    def load(t):
        return (5.0e6 * math.sin(math.pi * t / 10.0e-6) if t <= 10.0e-6 else 0.0) * unit

    newton = dict(max_iterations=10, residual_absolute_tolerance=1e-9, residual_relative_tolerance=1e-12,
                  increment_absolute_tolerance=1e-16, increment_relative_tolerance=1e-12, armijo=None)  # fmt: skip
    out = on.implicit_newmark(bar, on.PointJ2(elastic), fixed, load, 2.0e-6, 30, 0.25, 0.5, newton)
    assert np.all(out["dissipated_energy"] == 0.0)
    assert np.abs(out["energy_residual"]).max() <= 1e-9 * out["external_work"].max()
    assert out["kinetic_energy"][-1] > 0.0  # still vibrating after the pulse
