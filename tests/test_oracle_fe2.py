"""CPU tests of the explicit-dynamics oracle (mass, face load, stiffness, Verlet)."""

from __future__ import annotations

import numpy as np

from oracle import fe2 as of
from oracle.rve import box_mesh


def test_lumped_mass_and_face_load_totals() -> None:
    lengths, div = (0.08, 0.03, 0.02), (8, 3, 2)
    nodes, elements = box_mesh(lengths, div)
    m = of.lumped_mass(nodes, elements, 2400.0)
    assert np.isclose(m[0::3].sum(), 2400.0 * np.prod(lengths), rtol=1e-13)
    f = of.face_pressure_force(nodes, lengths, div)
    assert np.isclose(f.sum(), -lengths[1] * lengths[2], rtol=1e-13)
    # only x components on the x = L face carry the load
    loaded = np.flatnonzero(f)
    assert np.all(loaded % 3 == 0) and np.allclose(nodes[loaded // 3, 0], lengths[0])


def test_stiffness_has_rigid_body_null_space() -> None:
    nodes, elements = box_mesh((0.04, 0.02, 0.02), (4, 2, 2))
    k = of.elastic_stiffness(nodes, elements, 30.0e9, 0.2)
    scale = abs(k).max()
    for comp in range(3):
        t = np.zeros(3 * nodes.shape[0])
        t[comp::3] = 1.0
        assert np.abs(k @ t).max() <= 1e-12 * scale
    # infinitesimal rotation about z: u = (-y, x, 0)
    r = np.zeros(3 * nodes.shape[0])
    r[0::3], r[1::3] = -nodes[:, 1], nodes[:, 0]
    assert np.abs(k @ r).max() <= 1e-10 * scale


def test_elastic_wave_front_speed() -> None:
    """The compressive front reaches the middle of the bar after about L / (2 c_p)."""
    lengths, div, rho, E, nu = (0.4, 0.02, 0.02), (40, 2, 2), 2400.0, 30.0e9, 0.2
    c_p = np.sqrt(E * (1 - nu) / ((1 + nu) * (1 - 2 * nu)) / rho)
    dt = 0.5 * 0.01 / c_p
    steps = int(round(0.5 * lengths[0] / c_p / dt))
    u, _, _ = of.explicit_elastic_bar(div, lengths, rho, E, nu, dt, steps, lambda t: 1.0e6)
    nodes, _ = box_mesh(lengths, div)
    ux = u[0::3]
    front = ux[np.isclose(nodes[:, 0], 0.1)]  # a quarter of the bar from the fixed end: not reached
    mid = ux[np.isclose(nodes[:, 0], 0.3)]  # reached
    assert np.abs(front).max() < 1e-3 * np.abs(mid).max()
    assert np.all(mid < 0)


def test_explicit_j2_oracle_reproduces_reference_run() -> None:
    """The oracle's velocity Verlet with J2 points reproduces the reference's own
    solve_material_explicit run (tests/golden explicit_j2_bar) to 1e-11 of each history's
    maximum; its lumped mass and face load are the reference's."""
    import math

    from oracle import j2vp as oj
    from tests.conftest import load_case

    g, meta = load_case("explicit_j2_bar")
    div, lengths = tuple(meta["bar"]["divisions"]), tuple(meta["bar"]["lengths"])
    nodes, elements = box_mesh(lengths, div)
    np.testing.assert_allclose(of.face_pressure_force(nodes, lengths, div), g["unit_force"], rtol=0, atol=1e-18)
    amp, dur = meta["amplitude"], meta["duration"]

    def load(t):
        return (amp * math.sin(math.pi * t / dur) if 0.0 <= t <= dur else 0.0) * g["unit_force"]

    h = of.explicit_j2_bar(div, lengths, oj.mortar_params(), meta["material"]["density"], meta["time_step"],
                           meta["num_steps"], load, g["fixed_dofs"])  # fmt: skip
    for ours, ref in (("u", "displacement"), ("v", "velocity"), ("a", "acceleration"), ("stresses", "stresses"),
                      ("eqps", "equivalent_plastic_strain"), ("kinetic", "kinetic_energy"),
                      ("dissipated", "dissipated_energy"), ("work", "external_work")):
        np.testing.assert_allclose(h[ours], g[ref], rtol=0, atol=1e-11 * np.abs(g[ref]).max(), err_msg=ref)
    assert g["equivalent_plastic_strain"].max() > 1e-4
