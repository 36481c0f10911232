"""CPU: the benchmarked RVE configurations' inputs and the RVE oracle against the
reference's own runs (tests/golden groups rve_batch and rve_path).

The sphere layouts and macro paths that the workloads generate are the ones the golden
runs used; the NumPy/SciPy oracle reproduces the reference's homogenised stress on the 8^3
member of the uneven batch (1e-9) -- the larger members take minutes per step in the
oracle's direct solves and are checked on the GPU only.
"""

from __future__ import annotations

import numpy as np

from concrete_impact_b200.benchmarks import concrete_rve
from concrete_impact_b200.rve_builders import random_strain_path
from oracle import j2vp as oj
from oracle.rve import OraclePhase, OracleRVE, RVEOracle
from tests.conftest import golden_names, load_case


def test_batch_members_are_workload_rves() -> None:
    names = golden_names("rve_batch_edge")
    assert len(names) == 5
    for name in names:
        arrays, meta = load_case(name)
        edge, index = meta["edge"], meta["workload_index"]
        assert int(np.random.default_rng(1000 + index).choice((8, 12, 16, 20, 24))) == edge
        model = concrete_rve(edge, index, 32)
        assert np.array_equal(model.element_phase_ids, arrays["element_phase"])
        times, strains = random_strain_path(5000 + index, 200, 4, 1.0e-2, (1.0, 1000.0))
        ti = np.asarray(meta["time_indices"])
        np.testing.assert_array_equal(strains[ti[1:]], arrays["macro_strain"])


def test_oracle_reproduces_reference_on_the_8_cube_batch_member() -> None:
    arrays, meta = load_case("rve_batch_edge8")
    mi, ra, rr, ia, ir, _ = meta["newton"]
    newton = {"max_iterations": mi, "residual_absolute_tolerance": ra, "residual_relative_tolerance": rr,
              "increment_absolute_tolerance": ia, "increment_relative_tolerance": ir, "armijo": None}  # fmt: skip
    phases = [OraclePhase("j2", oj.mortar_params()), OraclePhase("elastic", None, 50.0e9, 0.2)]
    oracle = RVEOracle(OracleRVE((8, 8, 8), (1.0, 1.0, 1.0), phases, arrays["element_phase"].astype(np.int64), newton))
    state = oracle.initial_state()
    for step in range(arrays["macro_strain"].shape[0]):
        res = oracle.solve(arrays["macro_strain"][step], float(arrays["time_step"][step]), state, False)
        ref = arrays["macro_stress"][step]
        assert np.abs(res["macro_stress"] - ref).max() <= 1e-9 * np.abs(ref).max()
        assert res["newton_iterations"] == meta["newton_iterations"][step]
        state = res["state"]


def test_mixed_control_golden_is_the_uniaxial_ramp() -> None:
    arrays, meta = load_case("rve_path_uniaxial_8")
    assert np.array_equal(concrete_rve(8, 0, 64).element_phase_ids, arrays["element_phase"])
    exx = np.linspace(0.0, -5.0e-3, 101)[1 : meta["steps"] + 1]
    np.testing.assert_array_equal(arrays["macro_strain"][:, 0], exx)
    free = np.abs(arrays["macro_stress"][:, 1:]).max()
    assert free <= meta["stress_tolerance"]
