"""CPU tests of the RVE host-side set-up: mesh, periodic constraint, builders, settings."""

from __future__ import annotations

import numpy as np
import pytest

from concrete_impact_b200 import rve as R
from concrete_impact_b200.rve_builders import draw_spheres, random_strain_path, sphere_phase_map
from oracle.rve import box_mesh, periodic_operators


@pytest.mark.parametrize("divisions", [(1, 1, 1), (2, 2, 2), (4, 4, 4), (3, 4, 5)])
def test_structured_periodic_constraint_merges_faces_edges_and_corners(divisions) -> None:
    """Reference tests/unit/fem/test_rve.py:36 (class count, T, affine consistency)."""
    macro = np.asarray([0.01, -0.003, 0.002, 0.004, -0.006, 0.008])
    nodes, elements = R.build_structured_hex8_box((1.0, 1.0, 1.0), divisions)
    ref_nodes, ref_elements = box_mesh((1.0, 1.0, 1.0), divisions)
    np.testing.assert_array_equal(nodes, ref_nodes)
    np.testing.assert_array_equal(elements, ref_elements)
    c = R.build_structured_hex8_periodic_constraint(nodes, divisions)
    count = int(np.prod(divisions))
    assert np.unique(c.equivalence_class_ids).size == count
    assert c.transformation.shape == (3 * nodes.shape[0], 3 * (count - 1))
    if count > 1:
        assert np.linalg.matrix_rank(c.transformation.toarray()) == 3 * (count - 1)
    t, a, cls = periodic_operators(nodes, divisions)
    assert (c.transformation != t).nnz == 0
    np.testing.assert_array_equal(c.affine_matrix, a)
    np.testing.assert_array_equal(c.equivalence_class_ids, cls)
    assert c.reference_class == 0
    disp = c.affine_matrix @ macro
    rep = c.representative_nodes[c.equivalence_class_ids]
    diff = disp.reshape(-1, 3) - disp.reshape(-1, 3)[rep]
    aff = (c.affine_matrix.reshape(-1, 3, 6) - c.affine_matrix.reshape(-1, 3, 6)[rep]) @ macro
    np.testing.assert_allclose(diff, aff, atol=1e-14)
    assert R.compute_periodic_fluctuation_error(disp, macro, c) <= 1e-15


def test_settings_validation_matches_reference() -> None:
    with pytest.raises(ValueError, match="sufficient_decrease"):
        R.ArmijoSettings(sufficient_decrease=1.0)
    with pytest.raises(ValueError, match="reduction_factor"):
        R.ArmijoSettings(reduction_factor=0.0)
    with pytest.raises(ValueError, match="max_backtracks"):
        R.ArmijoSettings(max_backtracks=-1)
    with pytest.raises(ValueError, match="exactly one worker"):
        R.RVEExecutionSettings(backend="serial", workers=2)


def test_sphere_layout_is_seeded_periodic_and_near_target_fraction() -> None:
    a, b = draw_spheres(5), draw_spheres(5)
    np.testing.assert_array_equal(a.centres, b.centres)
    assert 0.38 <= a.sphere_fraction <= 0.42
    d = a.centres[:, None, :] - a.centres[None, :, :]
    d -= np.round(d)
    dist = np.linalg.norm(d, axis=2) + np.eye(len(a.radii)) * 10
    assert np.all(dist >= a.radii[:, None] + a.radii[None, :] - 1e-12)
    phase = sphere_phase_map((12, 12, 12), a)
    assert abs(phase.mean() - a.sphere_fraction) < 0.05


def test_random_strain_path_bounds_and_rate() -> None:
    times, strains = random_strain_path(3, steps=200)
    assert strains.shape == (201, 6) and np.all(np.abs(strains) <= 1e-2 + 1e-15)
    assert np.all(np.diff(times) > 0)
    rate = np.linalg.norm(np.diff(strains, axis=0), axis=1) / np.diff(times)
    assert 1.0 <= rate.mean() <= 1000.0
