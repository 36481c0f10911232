"""CPU tests of the cylindrical O-grid RVE builders and the general-mesh RVE oracle.

Pinned to the reference itself (tests/golden/make_golden.py runs its
build_cylindrical_ogrid_hex8, build_cylindrical_two_phase_rve and solve_rve_microequilibrium):
the mesh, its phases, periodic classes and opposite faces are reproduced exactly, and the
oracle's RVE solves on it match the reference's homogenised stress, effective tangent and
fluctuation along a three-step compression path.
"""

from __future__ import annotations

import numpy as np
import pytest

from concrete_impact_b200.materials import J2ViscoplasticMaterial, LinearElasticMaterial
from concrete_impact_b200.rve import NonlinearNewtonSettings
from concrete_impact_b200.rve_builders import build_cylindrical_ogrid_hex8, build_cylindrical_two_phase_rve
from conftest import load_case
from oracle import j2vp as oj
from oracle.rve import OraclePhase
from oracle.rve_general import general_rve_oracle

NEWTON_KEYS = ("max_iterations", "residual_absolute_tolerance", "residual_relative_tolerance",
               "increment_absolute_tolerance", "increment_relative_tolerance")  # fmt: skip


def _mesh(meta):
    s = meta["mesh"]
    return build_cylindrical_ogrid_hex8(s["lengths"], s["inclusion_volume_fraction"], s["circumferential_divisions"],
                                        s["matrix_radial_divisions"], s["axial_divisions"])  # fmt: skip


def test_ogrid_mesh_matches_reference() -> None:
    g, meta = load_case("rve_ogrid_cylinder")
    mesh = _mesh(meta)
    np.testing.assert_array_equal(mesh.nodes, g["nodes"])
    np.testing.assert_array_equal(mesh.elements, g["elements"])
    np.testing.assert_array_equal(mesh.element_phase_ids, g["element_phase_ids"])
    np.testing.assert_array_equal(mesh.periodic_class_ids, g["periodic_class_ids"])
    for axis, (minus, plus) in zip("xyz", mesh.opposite_face_nodes):
        np.testing.assert_array_equal(minus, g[f"face_{axis}_minus"])
        np.testing.assert_array_equal(plus, g[f"face_{axis}_plus"])
    assert mesh.analytic_inclusion_area == pytest.approx(meta["analytic_inclusion_area"], rel=1e-15)
    assert mesh.discrete_inclusion_area == pytest.approx(meta["discrete_inclusion_area"], rel=1e-13)


def test_cylindrical_rve_builder_matches_reference() -> None:
    g, meta = load_case("rve_ogrid_cylinder")
    mortar = J2ViscoplasticMaterial("mortar", 2200.0, 25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0)
    aggregate = LinearElasticMaterial("aggregate", 2600.0, 50.0e9, 0.2)
    model = build_cylindrical_two_phase_rve(_mesh(meta), mortar, aggregate, NonlinearNewtonSettings(25, 1e-6, 1e-8,
                                                                                                     1e-14, 1e-10), 1.0)
    assert model.material.density == pytest.approx(meta["effective_density"], rel=1e-13)
    assert model.divisions == (0, 0, 0)
    c = model.constraint
    assert c.transformation.shape == (3 * g["nodes"].shape[0], 3 * (int(g["periodic_class_ids"].max())))
    assert c.reference_class == int(g["periodic_class_ids"][g["face_x_minus"][0]])
    # every node of a class carries the class's fluctuation: T has one entry per non-reference node DOF
    per_row = np.diff(c.transformation.indptr)
    ref_nodes = np.flatnonzero(c.equivalence_class_ids == c.reference_class)
    assert np.all(per_row.reshape(-1, 3)[ref_nodes] == 0) and per_row.sum() == 3 * (g["nodes"].shape[0] - ref_nodes.size)


def test_ogrid_mesh_rejects_invalid_divisions() -> None:
    with pytest.raises(ValueError, match="divisible by four"):
        build_cylindrical_ogrid_hex8((1.0, 1.0, 1.0), 0.3, 6, 2, 2)
    with pytest.raises(ValueError, match="positive"):
        build_cylindrical_ogrid_hex8((1.0, 1.0, 1.0), 0.3, 8, 0, 2)
    with pytest.raises(ValueError, match="intersects"):
        build_cylindrical_ogrid_hex8((1.0, 1.0, 1.0), 0.9, 8, 2, 2)


def test_general_oracle_matches_reference_ogrid_rve() -> None:
    g, meta = load_case("rve_ogrid_cylinder")
    phases = [OraclePhase("j2", oj.J2Params(25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0)),
              OraclePhase("elastic", None, 50.0e9, 0.2)]  # fmt: skip
    oracle = general_rve_oracle(g["nodes"], g["elements"], g["periodic_class_ids"], int(g["face_x_minus"][0]), phases,
                                g["element_phase_ids"], dict(zip(NEWTON_KEYS, meta["newton"][:5]), armijo=None))  # fmt: skip
    state = oracle.initial_state()
    for step in range(meta["steps"]):
        out = oracle.solve(g[f"s{step}__macro_strain"], meta["time_step"], state, True)
        state = out["state"]
        assert out["newton_iterations"] == meta["scalars"][step]["newton_iterations"]
        for key, ref in (("macro_stress", g[f"s{step}__macro_stress"]), ("effective_tangent", g[f"s{step}__effective_tangent"])):
            np.testing.assert_allclose(out[key], ref, rtol=0, atol=1e-13 * np.abs(ref).max(), err_msg=key)
        np.testing.assert_allclose(state["w"], g[f"s{step}__fluctuation"], rtol=0,
                                   atol=1e-12 * np.abs(g[f"s{step}__fluctuation"]).max())  # fmt: skip


@pytest.mark.parametrize("divisions", [(8, 2, 2), (16, 4, 3), (32, 8, 2)])
def test_ogrid_meshes_are_valid_periodic_cells(divisions) -> None:
    """Positive Jacobians, the cell volume, an inclusion area converging to the target
    fraction, and periodic classes that pair every boundary node with its images."""
    from oracle.rve import b_matrices

    c, r, a = divisions
    mesh = build_cylindrical_ogrid_hex8((1.0, 0.8, 0.5), 0.3, c, r, a)
    _, det = b_matrices(mesh.nodes, mesh.elements)
    assert det.min() > 0.0
    assert det.sum() == pytest.approx(1.0 * 0.8 * 0.5, rel=1e-12)
    # the inscribed polygon of c sides misses O(1/c^2) of the circle's area
    assert 0.0 < 1.0 - mesh.discrete_inclusion_area / (0.3 * 0.8) < {8: 0.1, 16: 0.04, 32: 0.01}[c]
    cls = mesh.periodic_class_ids
    for (minus, plus), axis in zip(mesh.opposite_face_nodes, range(3)):
        np.testing.assert_array_equal(cls[minus], cls[plus])
        shift = mesh.nodes[plus] - mesh.nodes[minus]
        np.testing.assert_allclose(shift[:, axis], (1.0, 0.8, 0.5)[axis], rtol=1e-12)
        np.testing.assert_allclose(np.delete(shift, axis, axis=1), 0.0, atol=1e-12)
