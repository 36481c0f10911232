"""NumPy/SciPy oracle of the periodic RVE solve on general Hex8 meshes -- test
infrastructure only.

The RVE oracle of ``oracle.rve`` (Newton with direct solves, response, effective tangent)
on any mesh with topology-provided periodic classes, with the elimination operators of the
reference's build_periodic_constraint_from_classes (src/fem/rve/periodic.py:50-104): every
node of a class shares the class's fluctuation, the class of the first node of the x-minus
face is eliminated, and u = T w + A ebar with the affine map of periodic.py:153-169.
"""

from __future__ import annotations

import numpy as np
from scipy.sparse import coo_matrix

from .rve import OracleRVE, RVEOracle, b_matrices


def periodic_operators_from_classes(nodes: np.ndarray, class_ids: np.ndarray, reference_node: int):
    """(T, A, normalised class ids) for classes given per node."""
    _, cls = np.unique(class_ids, return_inverse=True)
    count = int(cls.max()) + 1
    ref = int(cls[reference_node])
    reduced = np.full(count, -1, dtype=np.int64)
    reduced[np.arange(count) != ref] = np.arange(count - 1)
    node_ids = np.flatnonzero(cls != ref)
    rows = (3 * node_ids[:, None] + np.arange(3)).ravel()
    cols = (3 * reduced[cls[node_ids]][:, None] + np.arange(3)).ravel()
    t = coo_matrix((np.ones(rows.size), (rows, cols)), shape=(3 * nodes.shape[0], 3 * (count - 1))).tocsr()
    rel = nodes - nodes.min(axis=0)
    a = np.zeros((3 * nodes.shape[0], 6))
    a[0::3, 0], a[0::3, 4], a[0::3, 5] = rel[:, 0], 0.5 * rel[:, 2], 0.5 * rel[:, 1]
    a[1::3, 1], a[1::3, 3], a[1::3, 5] = rel[:, 1], 0.5 * rel[:, 2], 0.5 * rel[:, 0]
    a[2::3, 2], a[2::3, 3], a[2::3, 4] = rel[:, 2], 0.5 * rel[:, 1], 0.5 * rel[:, 0]
    return t, a, cls


def general_rve_oracle(nodes: np.ndarray, elements: np.ndarray, class_ids: np.ndarray, reference_node: int,
                       phases, element_phase: np.ndarray, newton: dict) -> RVEOracle:  # fmt: skip
    """An RVEOracle whose mesh, geometry and periodic operators are the given ones."""
    oracle = RVEOracle.__new__(RVEOracle)
    oracle.rve = OracleRVE((0, 0, 0), tuple(np.ptp(nodes, axis=0)), list(phases), np.asarray(element_phase), newton)
    oracle.nodes, oracle.elements = np.asarray(nodes, dtype=np.float64), np.asarray(elements, dtype=np.int64)
    oracle.t, oracle.a, oracle.cls = periodic_operators_from_classes(oracle.nodes, class_ids, reference_node)
    oracle.b, oracle.jw = b_matrices(oracle.nodes, oracle.elements)
    oracle.weights = oracle.jw.reshape(-1)
    oracle.volume = float(oracle.weights.sum())
    e = oracle.elements.shape[0]
    oracle.dofs = (3 * oracle.elements[:, :, None] + np.arange(3)).reshape(-1, 24)
    oracle.point_phase = np.repeat(np.asarray(element_phase), 8)
    oracle.rows = np.repeat(oracle.dofs, 24, axis=1).ravel()
    oracle.cols = np.tile(oracle.dofs, (1, 24)).ravel()
    oracle.n_gp = 8 * e
    return oracle
