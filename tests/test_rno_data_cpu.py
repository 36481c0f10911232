"""CPU tests of the surrogate's data-path helpers (path families, envelopes, errors)."""

from __future__ import annotations

import numpy as np
import torch

from concrete_impact_b200.rno import RNODataset, RNOScales
from concrete_impact_b200.rno_data import PathSetSpec, concat_datasets, draw_paths, input_envelope, relative_stress_error


def test_path_family_is_seeded_bounded_and_monotone_in_time() -> None:
    spec = PathSetSpec(paths=12, steps=40, seed=77, amplitude=(1e-3, 4e-3), rate_range=(10.0, 100.0))
    t1, e1 = draw_paths(spec)
    t2, e2 = draw_paths(spec)
    assert np.array_equal(t1, t2) and np.array_equal(e1, e2)
    assert t1.shape == (12, 41) and e1.shape == (12, 41, 6)
    assert np.all(np.diff(t1, axis=1) > 0) and np.all(e1[:, 0] == 0)
    assert np.abs(e1).max() <= 4e-3 + 1e-15
    # strain rate along each path equals the drawn constant rate (arc length per time)
    speed = np.linalg.norm(np.diff(e1, axis=1), axis=2) / np.diff(t1, axis=1)
    assert np.all(speed.max(axis=1) >= 10.0 * (1 - 1e-9)) and np.all(speed.max(axis=1) <= 100.0 * (1 + 1e-9))


def test_envelopes_and_errors() -> None:
    strain = torch.zeros((3, 5, 6), dtype=torch.float64)
    strain[1, 2, 4] = -2.0
    strain[2, 3, 0] = 1.0
    data = RNODataset(strain, torch.ones_like(strain), torch.full((3, 4), 0.5, dtype=torch.float64))
    scales = RNOScales(2.0, 1.0, 1.0)
    e, r = input_envelope(scales, data)
    assert e == 1.0 and r == 4.0  # max |strain| / 2; max |rate| = |-2| / 0.5 (one step)
    ec, rc = input_envelope(scales, data, per_component=True)
    assert ec == [0.5, 0.0, 0.0, 0.0, 1.0, 0.0] and rc[4] == 4.0 and rc[0] == 2.0
    both = concat_datasets(data, data)
    assert both.paths == 6 and both.steps == 4
    assert abs(relative_stress_error(data.stress * 1.01, data.stress) - 0.01) < 1e-12
