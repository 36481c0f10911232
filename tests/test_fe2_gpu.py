"""GPU tests of the explicit FE^2 macro dynamics and the surrogate's training data.

* the velocity-Verlet kernels against their formula;
* a linear elastic bar against the NumPy oracle of solve_material_explicit
  (material.py:164-219) with its own lumped mass and face pressure;
* FE^2 with one single-phase RVE per macro point against the same bar with the J2 point
  law (a homogeneous RVE reproduces its material point, test_rve.py's RVE == point pin);
* the surrogate's error gate: flagged points are answered by the direct RVE solve;
* the RVE path generator against the oracle's point-law path for a single-phase RVE.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from concrete_impact_b200 import _native  # noqa: E402
from concrete_impact_b200.fe2 import (  # noqa: E402
    SurrogateJudge,
    DirectRVEPoints,
    ExplicitFE2,
    MaterialPoints,
    RNOPoints,
    build_macro_bar,
    half_sine_pressure,
    stable_time_step,
)
from concrete_impact_b200.materials import (  # noqa: E402
    J2ViscoplasticMaterial,
    LinearElasticMaterial,
    MaterialUpdateSettings,
    compute_isotropic_pressure_wave_speed,
)
from concrete_impact_b200.rno import RNOConfig, RNOScales, RNOSurrogate  # noqa: E402
from concrete_impact_b200.rno_data import PathSetSpec, draw_paths, generate_rve_paths, input_envelope  # noqa: E402
from concrete_impact_b200.rve import NonlinearNewtonSettings  # noqa: E402
from concrete_impact_b200.rve_builders import build_structured_rve, default_newton  # noqa: E402
from oracle import fe2 as of  # noqa: E402
from oracle import j2vp as oj  # noqa: E402

SETTINGS = MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)
MORTAR = J2ViscoplasticMaterial("mortar", 2400.0, 25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0)


def _pulse(duration):
    return lambda t: half_sine_pressure(t, 50.0e6, duration)


def test_verlet_kernels_match_formula() -> None:
    lib = _native.load_library()
    g = torch.Generator(device="cuda").manual_seed(0)
    n = 10_007
    u, v, a, fu, fi = (torch.randn(n, generator=g, device="cuda", dtype=torch.float64) for _ in range(5))
    m = torch.rand(n, generator=g, device="cuda", dtype=torch.float64) + 0.5
    fixed = (torch.rand(n, generator=g, device="cuda") < 0.1).to(torch.uint8)
    dt, p = 1.3e-3, 2.5
    un, an, vn = torch.empty_like(u), torch.empty_like(u), torch.empty_like(u)
    sp = _native.stream_ptr()
    _native.check(lib.cib_verlet_predict(n, u.data_ptr(), v.data_ptr(), a.data_ptr(), fixed.data_ptr(), dt,
                                         un.data_ptr(), sp), "predict")  # fmt: skip
    _native.check(lib.cib_verlet_correct(n, fu.data_ptr(), p, fi.data_ptr(), m.data_ptr(), fixed.data_ptr(), dt,
                                         a.data_ptr(), v.data_ptr(), an.data_ptr(), vn.data_ptr(), sp), "correct")  # fmt: skip
    keep = fixed == 0
    ref_u = torch.where(keep, u + dt * v + 0.5 * dt * dt * a, 0.0)
    ref_a = torch.where(keep, (p * fu - fi) / m, 0.0)
    ref_v = torch.where(keep, v + 0.5 * dt * (a + ref_a), 0.0)
    for got, ref in ((un, ref_u), (an, ref_a), (vn, ref_v)):
        torch.testing.assert_close(got, ref, rtol=1e-14, atol=1e-14)
    assert lib.cib_verlet_predict(-1, u.data_ptr(), v.data_ptr(), a.data_ptr(), fixed.data_ptr(), dt, un.data_ptr(), sp) != 0


def test_macro_bar_mass_and_load_match_oracle() -> None:
    div, lengths = (6, 3, 2), (0.06, 0.03, 0.02)
    bar = build_macro_bar(div, lengths, 2400.0)
    np.testing.assert_allclose(bar.mass.cpu().numpy(), of.lumped_mass(bar.nodes, bar.elements, 2400.0), rtol=1e-13)
    np.testing.assert_allclose(bar.unit_force.cpu().numpy(), of.face_pressure_force(bar.nodes, lengths, div),
                               rtol=1e-13, atol=1e-18)  # fmt: skip


def test_elastic_bar_matches_numpy_oracle() -> None:
    div, lengths, rho, E, nu = (8, 2, 2), (0.08, 0.02, 0.02), 2400.0, 30.0e9, 0.2
    bar = build_macro_bar(div, lengths, rho)
    c = compute_isotropic_pressure_wave_speed(E, nu, rho)
    dt = stable_time_step(bar, c, 0.5)
    steps, pulse = 80, _pulse(20 * dt)
    solver = ExplicitFE2(bar, MaterialPoints(LinearElasticMaterial("elastic", rho, E, nu), bar.points, SETTINGS), dt, pulse)
    solver.run(steps)
    u_ref, v_ref, _ = of.explicit_elastic_bar(div, lengths, rho, E, nu, dt, steps, pulse)
    u = solver.u.cpu().numpy()
    assert np.abs(u_ref).max() > 0
    np.testing.assert_allclose(u, u_ref, rtol=0, atol=1e-10 * np.abs(u_ref).max())
    np.testing.assert_allclose(solver.v.cpu().numpy(), v_ref, rtol=0, atol=1e-10 * np.abs(v_ref).max())


@pytest.mark.parametrize("precision,tol", [(64, 1e-6), (32, 1e-4)])
def test_direct_rve_fe2_matches_point_law(precision: int, tol: float) -> None:
    div, lengths = (4, 1, 1), (0.04, 0.01, 0.01)
    bar = build_macro_bar(div, lengths, 2400.0)
    dt = stable_time_step(bar, MORTAR.maximum_wave_speed, 0.5)
    steps, pulse = 24, _pulse(16 * dt)
    point = ExplicitFE2(bar, MaterialPoints(MORTAR, bar.points, SETTINGS), dt, pulse)
    # a homogeneous RVE's residual is pure roundoff: FP32 needs an absolute force tolerance
    # (50 N against element forces of ~5e6 N on the unit cell)
    newton = default_newton() if precision == 64 else NonlinearNewtonSettings(25, 50.0, 1.0e-6, 1.0e-14, 1.0e-6)
    rve = build_structured_rve((2, 2, 2), MORTAR, newton)
    direct = ExplicitFE2(bar, DirectRVEPoints(rve, bar.points, SETTINGS, precision=precision, chunk=24), dt, pulse)
    point.run(steps)
    direct.run(steps)
    s_ref = point.last_stress.cpu().numpy()
    assert np.abs(s_ref).max() > 20.0e6  # the pulse drives the points past yield
    np.testing.assert_allclose(direct.last_stress.cpu().numpy(), s_ref, rtol=0, atol=tol * np.abs(s_ref).max())
    u_ref = point.u.cpu().numpy()
    np.testing.assert_allclose(direct.u.cpu().numpy(), u_ref, rtol=0, atol=tol * np.abs(u_ref).max())


def _untrained_rno() -> RNOSurrogate:
    return RNOSurrogate(RNOConfig(seed=5), RNOScales(1e-3, 10.0, 20.0e6))


def test_rno_gate_flagging_every_point_reproduces_direct_fe2() -> None:
    div, lengths = (4, 1, 1), (0.04, 0.01, 0.01)
    bar = build_macro_bar(div, lengths, 2400.0)
    dt = stable_time_step(bar, MORTAR.maximum_wave_speed, 0.5)
    steps, pulse = 12, _pulse(16 * dt)
    rve = build_structured_rve((2, 2, 2), MORTAR, default_newton())
    direct = ExplicitFE2(bar, DirectRVEPoints(rve, bar.points, SETTINGS, precision=64), dt, pulse)
    # a negative envelope flags every point at the first step (zero elapsed time, so the
    # catch-up step is the ordinary first step)
    gated = RNOPoints(_untrained_rno(), bar.points, (-1.0, -1.0), rve, SETTINGS, fallback_capacity=bar.points + 5,
                      precision=64)  # fmt: skip
    fe2 = ExplicitFE2(bar, gated, dt, pulse)
    direct.run(steps)
    fe2.run(steps)
    assert gated.slots_used == bar.points
    assert bool(gated.flagged.all())
    torch.testing.assert_close(fe2.last_stress, direct.last_stress, rtol=1e-12, atol=1e-6)
    torch.testing.assert_close(fe2.u, direct.u, rtol=1e-12, atol=1e-18)


def test_rno_gate_capacity_and_untouched_points() -> None:
    div, lengths = (4, 1, 1), (0.04, 0.01, 0.01)
    bar = build_macro_bar(div, lengths, 2400.0)
    dt = stable_time_step(bar, MORTAR.maximum_wave_speed, 0.5)
    rve = build_structured_rve((2, 2, 2), MORTAR, default_newton())
    rno = _untrained_rno()
    # a huge envelope never flags: the answers are the surrogate's
    free = RNOPoints(rno, bar.points, (1e30, 1e30), rve, SETTINGS, fallback_capacity=4)
    fe2 = ExplicitFE2(bar, free, dt, _pulse(16 * dt))
    fe2.run(6)
    assert free.slots_used == 0 and free.fallback_steps == 0
    # a negative envelope with a too-small pool raises
    tight = RNOPoints(rno, bar.points, (-1.0, -1.0), rve, SETTINGS, fallback_capacity=4)
    fe2 = ExplicitFE2(bar, tight, dt, _pulse(16 * dt))
    with pytest.raises(RuntimeError, match="fallback pool"):
        fe2.step()


def test_gate_kernels_match_formula() -> None:
    lib = _native.load_library()
    g = torch.Generator(device="cuda").manual_seed(4)
    n = 1000
    strain = torch.randn((n, 6), generator=g, device="cuda", dtype=torch.float64) * 1e-3
    rate = torch.randn((n, 6), generator=g, device="cuda", dtype=torch.float64) * 50.0
    strain[7, 2] = float("nan")
    lim = torch.tensor([2.0] * 6 + [2.5] * 6, dtype=torch.float64, device="cuda")
    flagged = (torch.rand(n, generator=g, device="cuda") < 0.2).to(torch.uint8)
    xn, rn, sn = (torch.empty((n, 6), dtype=torch.float32, device="cuda") for _ in range(3))
    cf = torch.empty(n, dtype=torch.float32, device="cuda")
    fresh = torch.zeros(n, dtype=torch.uint8, device="cuda")
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.empty((n, 6), dtype=torch.float64, device="cuda")
    sp = _native.stream_ptr()
    _native.check(lib.cib_rno_gate_prepare(n, strain.data_ptr(), rate.data_ptr(), 1e-3, 40.0, lim.data_ptr(), 0.25,
                                           flagged.data_ptr(), xn.data_ptr(), rn.data_ptr(), cf.data_ptr(),
                                           fresh.data_ptr(), count.data_ptr(), sp), "prepare")  # fmt: skip
    en, rnr = strain / 1e-3, rate / 40.0
    over = ~((en.abs() <= 2.0).all(1) & (rnr.abs() <= 2.5).all(1))
    expect = over & (flagged == 0)
    assert torch.equal(fresh.bool(), expect) and int(count.item()) == int(expect.sum())
    torch.testing.assert_close(rn, rnr.float())
    assert bool((cf == 0.25).all())
    sn.copy_(torch.randn((n, 6), generator=g, device="cuda"))
    sn[11, 0] = float("inf")
    before = fresh.clone()
    _native.check(lib.cib_rno_gate_finish(n, sn.data_ptr(), 2.0e7, flagged.data_ptr(), fresh.data_ptr(),
                                          count.data_ptr(), out.data_ptr(), sp), "finish")  # fmt: skip
    torch.testing.assert_close(out[:11], sn[:11].double() * 2.0e7)
    extra = int((~before.bool() & (flagged == 0))[11])
    assert bool(fresh[11]) == bool(flagged[11] == 0) and int(count.item()) == int(expect.sum()) + extra


def test_rno_gate_flags_non_finite_answers() -> None:
    div, lengths = (4, 1, 1), (0.04, 0.01, 0.01)
    bar = build_macro_bar(div, lengths, 2400.0)
    dt = stable_time_step(bar, MORTAR.maximum_wave_speed, 0.5)
    rve = build_structured_rve((2, 2, 2), MORTAR, default_newton())
    rno = _untrained_rno()
    rno.layers[3].b.fill_(float("nan"))  # every answer of the surrogate is NaN
    gated = RNOPoints(rno, bar.points, (1e30, 1e30), rve, SETTINGS, fallback_capacity=bar.points, precision=64)
    fe2 = ExplicitFE2(bar, gated, dt, _pulse(16 * dt))
    fe2.run(3)
    assert gated.slots_used == bar.points
    assert bool(torch.isfinite(fe2.last_stress).all()) and bool(torch.isfinite(fe2.u).all())


def test_generated_paths_of_single_phase_rve_match_point_law() -> None:
    rve = build_structured_rve((2, 2, 2), MORTAR, default_newton())
    spec = PathSetSpec(paths=5, steps=12, seed=31, amplitude=(2e-3, 5e-3), rate_range=(10.0, 1000.0))
    data = generate_rve_paths(rve, spec, SETTINGS, precision=64)
    times, strains = draw_paths(spec)
    p = oj.mortar_params()
    for k in range(spec.paths):
        ep, q, vpm = np.zeros((1, 6)), np.zeros(1), np.zeros(1)
        for t in range(1, spec.steps + 1):
            out = oj.update_reference_form(p, strains[k, t][None], ep, q, vpm, float(times[k, t] - times[k, t - 1]))
            ep, q, vpm = out["plastic_strain"], out["equivalent_plastic_strain"], out["viscoplastic_multiplier"]
            ref = out["stresses"][0]
            got = data.stress[k, t].cpu().numpy()
            np.testing.assert_allclose(got, ref, rtol=0, atol=1e-6 * max(np.abs(ref).max(), 1e6))
    np.testing.assert_allclose(data.strain.cpu().numpy(), strains)
    env = input_envelope(RNOScales(1e-3, 10.0, 1e7), data)
    assert env[0] > 0 and env[1] > 0


def test_judge_measures_the_delivered_stress_against_direct_rves() -> None:
    """The runtime judge's RVEs follow the sampled points' macro strains: with every point
    flagged to the (FP64) fallback pool the delivered stress is the direct one, so the
    judged error is at roundoff; with a huge envelope the untrained surrogate delivers, and
    the judge reports its error (the same relative Frobenius error as the delivered stress
    against independent direct RVEs at those points) and escalates the worst points, whose
    answers are the direct ones from then on."""
    div, lengths = (4, 1, 1), (0.04, 0.01, 0.01)
    bar = build_macro_bar(div, lengths, 2400.0)
    dt = stable_time_step(bar, MORTAR.maximum_wave_speed, 0.5)
    rve = build_structured_rve((2, 2, 2), MORTAR, default_newton())
    steps, pulse = 10, _pulse(16 * dt)
    judge = SurrogateJudge(rve, bar.points, SETTINGS, sample=8, every=1, threshold=None, stress_floor=1.0, seed=3)
    gated = RNOPoints(_untrained_rno(), bar.points, (-1.0, -1.0), rve, SETTINGS, fallback_capacity=bar.points,
                      precision=64, judge=judge)  # fmt: skip
    ExplicitFE2(bar, gated, dt, pulse).run(steps)
    assert judge.judge_steps == steps and judge.error < 1e-10
    # surrogate answers, judged against independent direct RVEs along the same histories
    judge = SurrogateJudge(rve, bar.points, SETTINGS, sample=8, every=1, threshold=None, stress_floor=1.0, seed=3)
    free = RNOPoints(_untrained_rno(), bar.points, (1e30, 1e30), rve, SETTINGS, fallback_capacity=bar.points,
                     precision=64, judge=judge)  # fmt: skip
    fe2 = ExplicitFE2(bar, free, dt, pulse)
    shadow = DirectRVEPoints(rve, int(judge.points.numel()), SETTINGS, precision=64)
    err2 = ref2 = 0.0
    for _ in range(steps):
        fe2.step()
        direct = shadow.stress(fe2.strain[judge.points], fe2.rate[judge.points], dt)
        shadow.commit()
        d = fe2.last_stress[judge.points] - direct
        err2 += float((d * d).sum())
        ref2 += float((direct * direct).sum())
    assert judge.error == pytest.approx((err2 / ref2) ** 0.5, rel=1e-9)
    assert judge.error > 0.05 and free.escalations == 0
    # a threshold below that error escalates the sampled points to the fallback pool
    judge = SurrogateJudge(rve, bar.points, SETTINGS, sample=8, every=1, threshold=0.05, stress_floor=1.0, seed=3)
    esc = RNOPoints(_untrained_rno(), bar.points, (1e30, 1e30), rve, SETTINGS, fallback_capacity=bar.points,
                    precision=64, judge=judge)  # fmt: skip
    fe2 = ExplicitFE2(bar, esc, dt, pulse)
    fe2.run(steps)
    assert esc.escalations > 0 and esc.slots_used == esc.escalations
    escalated = judge.points[judge.escalated]
    assert bool(esc.flagged[escalated].all())
    # escalated points carry the judge's RVE history: their answers equal the judge's
    fe2.step()
    torch.testing.assert_close(fe2.last_stress[escalated], judge.reference[judge.escalated], rtol=1e-9, atol=1e-3)
