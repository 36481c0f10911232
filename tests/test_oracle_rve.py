"""CPU tests: the RVE oracle against the reference's own RVE solves (golden vectors)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import j2vp as oj
from oracle.rve import OraclePhase, OracleRVE, RVEOracle
from tests.conftest import load_case

MORTAR = oj.mortar_params()


def oracle_for(name: str) -> tuple[RVEOracle, dict, dict]:
    arrays, meta = load_case(name)
    div = tuple(meta["divisions"])
    mi, ra, rr, ia, ir, armijo = meta["newton"]
    newton = {"max_iterations": mi, "residual_absolute_tolerance": ra, "residual_relative_tolerance": rr,
              "increment_absolute_tolerance": ia, "increment_relative_tolerance": ir,
              "armijo": {"sufficient_decrease": 1e-4, "reduction_factor": 0.5, "max_backtracks": 20} if armijo else None}  # fmt: skip
    if meta["kind"] == "homogeneous":
        phases = [OraclePhase("j2", oj.J2Params(**meta["material"]["params"]))]
        element_phase = np.zeros(int(np.prod(div)), dtype=np.int64)
    else:
        phases = [OraclePhase("j2", MORTAR), OraclePhase("elastic", None, 50.0e9, 0.2)]
        element_phase = arrays["element_phase"]
    return RVEOracle(OracleRVE(div, (1.0, 1.0, 1.0), phases, element_phase, newton)), arrays, meta


def _state_key(meta, name):
    return f"state__{name}" if meta["kind"] == "homogeneous" else f"state__phase_matrix__{name}"


@pytest.mark.parametrize("name", ["rve_homogeneous_1", "rve_homogeneous_2", "rve_two_phase_4", "rve_two_phase_8"])
def test_rve_oracle_matches_reference_path(name: str) -> None:
    oracle, arrays, meta = oracle_for(name)
    state = oracle.initial_state()
    j2_points = np.flatnonzero(oracle.point_phase == 0)
    for step in range(meta["steps"]):
        p = f"s{step}__"
        out = oracle.solve(arrays[p + "macro_strain"], meta["time_step"], state)
        ref = arrays[p + "macro_stress"]
        np.testing.assert_allclose(out["macro_stress"], ref, rtol=1e-9, atol=1e-10 * np.abs(ref).max())
        tan = arrays[p + "effective_tangent"]
        np.testing.assert_allclose(out["effective_tangent"], tan, rtol=1e-7, atol=1e-9 * np.abs(tan).max())
        ref_eqps = arrays[p + _state_key(meta, "equivalent_plastic_strain")]
        np.testing.assert_allclose(out["state"]["eqps"][j2_points], ref_eqps, rtol=1e-7, atol=1e-12)
        sc = meta["scalars"][step]
        assert out["newton_iterations"] == sc["newton_iterations"]
        np.testing.assert_allclose(out["free_energy_density"], sc["free_energy_density"], rtol=1e-9)
        state = out["state"]
