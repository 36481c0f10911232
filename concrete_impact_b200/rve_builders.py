"""Builders and drivers around the periodic RVE solve.

* ``sphere_phase_map`` / ``build_two_phase_sphere_rve`` -- two-phase concrete RVE on a
  structured box: an element belongs to the aggregate phase when its centroid lies in one
  of a set of non-overlapping, periodically wrapped spheres with radii U[r_min, r_max],
  drawn by seeded rejection until the spheres' volume reaches the target fraction.  The
  reference builds its two-phase RVEs from a cylindrical O-grid
  (src/fem/rve/builders.py:22-78); this box builder keeps its PhasedMaterialModel layout
  (phase names, point_phase_ids, effective density; src/fem/materials/phased.py:36-66).
* ``build_structured_rve`` -- single-material structured RVE as in the reference's tests
  (tests/unit/fem/test_rve.py:223-246).
* ``solve_mixed_control_step`` -- one macro step where some macro strain components are
  prescribed and the others are free (their macro stress vanishes), solved by an outer
  Newton on the RVE's effective tangent around solve_rve_microequilibrium.
* ``random_strain_path`` -- piecewise-linear 6-component macro strain path with a
  prescribed strain rate, for batched path generation.
* ``build_cylindrical_ogrid_hex8`` / ``build_cylindrical_two_phase_rve`` -- the reference's
  cylindrical two-phase RVE (src/fem/mesh/structured.py:83-154, 157-316;
  src/fem/rve/builders.py:22-78): a centred z-cylinder inclusion meshed as a mapped square
  core, a square annulus of matrix blended from the core boundary to the cell boundary,
  extruded along z, with union-find periodic classes.  Same node, element and class
  numbering as the reference (the RVE solve and its golden data index by them); solved by
  the general-mesh RVE path of ``rve_general``.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Callable

import numpy as np

from .materials import MaterialResponseRequirements, PhasedMaterialModel, RVEPhase
from .rve import (
    NonlinearNewtonSettings,
    RVERequest,
    RVEResponse,
    RVEState,
    StructuredHex8RVE,
    build_periodic_constraint_from_classes,
    build_structured_hex8_box,
    build_structured_hex8_periodic_constraint,
)


@dataclass(frozen=True)
class SphereLayout:
    """Spheres (centres, radii) of a periodic unit-cell inclusion layout."""

    centres: np.ndarray
    radii: np.ndarray
    target_fraction: float
    sphere_fraction: float


def draw_spheres(seed: int, target_fraction: float = 0.4, r_min: float = 0.08, r_max: float = 0.15,
                 lengths=(1.0, 1.0, 1.0), candidates_per_sphere: int = 4096, batch: int = 512) -> SphereLayout:  # fmt: skip
    """Seeded random placement of non-overlapping periodic spheres, largest first.

    Radii U[r_min, r_max] are drawn until their total volume reaches the target fraction
    of the box, then placed in decreasing size: each sphere takes the first of its seeded
    candidate centres (drawn in batches) that clears every sphere placed before it
    (minimum-image distance).  A sphere with no clear candidate is dropped, so the
    achieved fraction can fall slightly short of the target near jamming."""
    rng = np.random.default_rng(seed)
    box = np.asarray(lengths, dtype=np.float64)
    volume = float(np.prod(box))
    radii_drawn: list[float] = []
    total = 0.0
    while total < target_fraction * volume:
        r = float(rng.uniform(r_min, r_max))
        radii_drawn.append(r)
        total += 4.0 / 3.0 * np.pi * r**3
    order = sorted(radii_drawn, reverse=True)
    centres = np.zeros((0, 3))
    radii = np.zeros(0)
    for r in order:
        placed = False
        for _ in range(max(1, candidates_per_sphere // batch)):
            c = rng.uniform(0.0, 1.0, size=(batch, 3)) * box
            if radii.size:
                d = c[:, None, :] - centres[None, :, :]
                d -= box * np.round(d / box)
                ok = ~np.any(np.einsum("ijk,ijk->ij", d, d) < (radii[None, :] + r) ** 2, axis=1)
            else:
                ok = np.ones(batch, dtype=bool)
            hit = np.flatnonzero(ok)
            if hit.size:
                centres = np.vstack([centres, c[hit[0]]])
                radii = np.append(radii, r)
                placed = True
                break
        if not placed:
            continue
    filled = float(np.sum(4.0 / 3.0 * np.pi * radii**3))
    return SphereLayout(centres, radii, target_fraction, filled / volume)


def sphere_phase_map(divisions, layout: SphereLayout, lengths=(1.0, 1.0, 1.0)) -> np.ndarray:
    """Element phase ids: 1 (aggregate) where the element centroid lies in a sphere, else 0."""
    nx, ny, nz = divisions
    box = np.asarray(lengths, dtype=np.float64)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    centroids = np.column_stack([(i.ravel() + 0.5) * box[0] / nx, (j.ravel() + 0.5) * box[1] / ny,
                                 (k.ravel() + 0.5) * box[2] / nz])  # fmt: skip
    inside = np.zeros(centroids.shape[0], dtype=bool)
    for c, r in zip(layout.centres, layout.radii):
        d = centroids - c
        d -= box * np.round(d / box)
        inside |= np.einsum("ij,ij->i", d, d) <= r * r
    return inside.astype(np.int64)


def build_structured_rve(divisions, material, newton_settings: NonlinearNewtonSettings, lengths=(1.0, 1.0, 1.0),
                         hill_mandel_power_scale: float = 1.0) -> StructuredHex8RVE:  # fmt: skip
    """Single-material structured periodic RVE."""
    nodes, elements = build_structured_hex8_box(tuple(lengths), tuple(divisions))
    constraint = build_structured_hex8_periodic_constraint(nodes, tuple(divisions))
    return StructuredHex8RVE(nodes, elements, tuple(divisions), material, constraint, newton_settings,
                             hill_mandel_power_scale=hill_mandel_power_scale)  # fmt: skip


def build_two_phase_sphere_rve(divisions, matrix_material, inclusion_material, newton_settings: NonlinearNewtonSettings,
                               seed: int, target_fraction: float = 0.4, r_min: float = 0.08, r_max: float = 0.15,
                               lengths=(1.0, 1.0, 1.0), hill_mandel_power_scale: float = 1.0,
                               phase_names=("matrix", "inclusion")) -> StructuredHex8RVE:  # fmt: skip
    """Two-phase periodic box RVE: phase 0 matrix (mortar), phase 1 inclusion (aggregate)."""
    nodes, elements = build_structured_hex8_box(tuple(lengths), tuple(divisions))
    layout = draw_spheres(seed, target_fraction, r_min, r_max, lengths)
    element_phase = sphere_phase_map(divisions, layout, lengths)
    n_el = elements.shape[0]
    frac = element_phase.mean() if n_el else 0.0
    density = matrix_material.density * (1.0 - frac) + inclusion_material.density * frac
    phased = PhasedMaterialModel(
        name=f"{matrix_material.name}__{inclusion_material.name}",
        phases=(RVEPhase(phase_names[0], matrix_material), RVEPhase(phase_names[1], inclusion_material)),
        point_phase_ids=np.repeat(element_phase, 8),
        effective_density=float(density),
    )
    constraint = build_structured_hex8_periodic_constraint(nodes, tuple(divisions))
    return StructuredHex8RVE(
        nodes, elements, tuple(divisions), phased, constraint, newton_settings,
        element_phase_ids=element_phase,
        element_densities=np.where(element_phase == 0, matrix_material.density, inclusion_material.density),
        phase_names=tuple(phase_names), hill_mandel_power_scale=hill_mandel_power_scale,
    )  # fmt: skip


@dataclass(frozen=True)
class MixedControlResult:
    """Outcome of one mixed strain/stress controlled macro step."""

    response: RVEResponse
    macro_strain: np.ndarray
    outer_iterations: int
    free_stress_norm: float


def solve_mixed_control_step(
    solve: Callable[[RVERequest, RVEState], RVEResponse],
    state: RVEState,
    prescribed: dict[int, float],
    guess: np.ndarray,
    time_step: float,
    update_settings,
    stress_tolerance: float,
    max_outer: int = 20,
) -> MixedControlResult:
    """Find the free macro strain components so that their macro stress vanishes.

    ``solve(request, state)`` is one RVE microequilibrium solve from the committed state
    (e.g. solve_rve_microequilibrium with a bound model and cache).  Each outer iteration
    corrects the free components with the effective tangent's free-free block.
    """
    strain = np.asarray(guess, dtype=np.float64).copy()
    for comp, value in prescribed.items():
        strain[comp] = value
    free = [c for c in range(6) if c not in prescribed]
    response = None
    norm = np.inf
    for outer in range(1, max_outer + 1):
        response = solve(RVERequest(strain.copy(), time_step, update_settings,
                                    MaterialResponseRequirements(tangent=True)), state)  # fmt: skip
        stress = np.asarray(response.macro_stress, dtype=np.float64)
        norm = float(np.linalg.norm(stress[free]))
        if norm <= stress_tolerance:
            return MixedControlResult(response, strain, outer, norm)
        tangent = np.asarray(response.effective_tangent, dtype=np.float64)
        strain[free] -= np.linalg.solve(tangent[np.ix_(free, free)], stress[free])
    raise RuntimeError(f"mixed control did not converge: free stress norm {norm:.3e} after {max_outer} iterations")


def random_strain_path(seed: int, steps: int = 200, segments: int = 4, max_abs: float = 1.0e-2,
                       rate_range=(1.0, 1000.0)) -> tuple[np.ndarray, np.ndarray]:  # fmt: skip
    """Piecewise-linear macro strain path: ``segments`` vertices uniform in the ball of
    radius ``max_abs`` (6 components, then clipped to |strain| <= max_abs), strain rate
    log-uniform in ``rate_range`` (1/s); returns (times (steps+1,), strains (steps+1, 6))."""
    rng = np.random.default_rng(seed)
    vertices = [np.zeros(6)]
    for _ in range(segments):
        v = rng.standard_normal(6)
        v *= rng.uniform(0.0, 1.0) ** (1.0 / 6.0) * max_abs / np.linalg.norm(v)
        vertices.append(np.clip(v, -max_abs, max_abs))
    vertices = np.asarray(vertices)
    seg_len = np.linalg.norm(np.diff(vertices, axis=0), axis=1)
    arc = np.concatenate([[0.0], np.cumsum(seg_len)])
    s = np.linspace(0.0, arc[-1], steps + 1)
    strains = np.column_stack([np.interp(s, arc, vertices[:, c]) for c in range(6)])
    rate = float(np.exp(rng.uniform(np.log(rate_range[0]), np.log(rate_range[1]))))
    times = s / rate
    if times[-1] == 0.0:
        times = np.arange(steps + 1, dtype=np.float64) * 1e-6
    return times, strains


def config0_materials():
    """Mortar (J2 Perzyna) and aggregate (linear elastic) of the concrete RVE, SI units."""
    from .materials import J2ViscoplasticMaterial, LinearElasticMaterial

    mortar = J2ViscoplasticMaterial("mortar", 2200.0, 25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0)
    aggregate = LinearElasticMaterial("aggregate", 2600.0, 50.0e9, 0.2)
    return mortar, aggregate


def default_newton(armijo: bool = False) -> NonlinearNewtonSettings:
    """Newton settings of the concrete RVE runs (relative residual tolerance 1e-8)."""
    from .rve import ArmijoSettings

    return NonlinearNewtonSettings(25, 1.0e-6, 1.0e-8, 1.0e-14, 1.0e-10, ArmijoSettings(enabled=armijo))


def fp32_newton(stress_scale: float = 20.0e6, face_area: float = 1.0, armijo: bool = False) -> NonlinearNewtonSettings:
    """Newton settings for FP32 element kernels.  The residual of an FP32 stress field has a
    roundoff floor of about 1e-7 of the element forces, which a tolerance relative to a small
    step's initial residual can fall below; the absolute tolerance is therefore 1e-6 of the
    traction resultant ``stress_scale`` * ``face_area`` (20 N on a unit cell at 20 MPa)."""
    from .rve import ArmijoSettings

    return NonlinearNewtonSettings(25, 1.0e-6 * stress_scale * face_area, 1.0e-6, 1.0e-14, 1.0e-6,
                                   ArmijoSettings(enabled=armijo))  # fmt: skip


def uniaxial_path(steps: int = 100, final_strain: float = -5.0e-3, rate: float = 10.0) -> tuple[np.ndarray, np.ndarray]:
    """Times and prescribed xx strain of the uniaxial compression ramp."""
    exx = np.linspace(0.0, final_strain, steps + 1)
    times = np.abs(exx) / rate
    return times, exx


def describe(model: StructuredHex8RVE) -> dict[str, Any]:
    """Small summary of a two-phase RVE (phase fractions, sizes)."""
    phase = model.element_phase_ids
    return {"divisions": model.divisions, "elements": int(model.elements.shape[0]),
            "inclusion_fraction": float(np.mean(phase)) if phase is not None else 0.0}  # fmt: skip


# --------------------------------------------------------------------------------------
# Cylindrical O-grid RVE.


@dataclass(frozen=True)
class CylindricalOGridHex8Mesh:
    """Conforming Hex8 mesh of a periodic box with a centred z-cylinder inclusion."""

    nodes: np.ndarray
    elements: np.ndarray
    element_phase_ids: np.ndarray
    periodic_class_ids: np.ndarray
    opposite_face_nodes: tuple
    analytic_inclusion_area: float
    discrete_inclusion_area: float


def _ring_keys(c: int) -> list[tuple[int, int]]:
    """Core-boundary grid keys (i, j), counterclockwise from (0, 0), each once."""
    return ([(i, 0) for i in range(c)] + [(c, j) for j in range(c)] + [(i, c) for i in range(c, 0, -1)]
            + [(0, j) for j in range(c, 0, -1)])  # fmt: skip


def _ogrid_section(lx: float, ly: float, radius: float, c: int, m: int):
    """Cross-section nodes (2D), quads, quad phases (1 core, 0 matrix) and the outer-ring
    node -> grid key map.  Core node (i, j) is j (c + 1) + i at radius * (xi sqrt(1 - eta^2/2),
    eta sqrt(1 - xi^2/2)); matrix ring r (1..m) blends each boundary key's core node towards
    the cell boundary point (lx xi / 2, ly eta / 2) with weight r / m."""
    t = np.linspace(-1.0, 1.0, c + 1)
    xi, eta = np.meshgrid(t, t, indexing="xy")  # [j, i]
    core = np.column_stack([(radius * xi * np.sqrt(1.0 - 0.5 * eta**2)).ravel(),
                            (radius * eta * np.sqrt(1.0 - 0.5 * xi**2)).ravel()])  # fmt: skip
    cid = lambda i, j: j * (c + 1) + i  # noqa: E731
    quads = [[cid(i, j), cid(i + 1, j), cid(i, j + 1), cid(i + 1, j + 1)] for j in range(c) for i in range(c)]
    phases = [1] * len(quads)
    keys = _ring_keys(c)
    ring_size = len(keys)
    inner_ids = np.asarray([cid(i, j) for i, j in keys])
    inner = core[inner_ids]
    outer = np.column_stack([0.5 * lx * t[[i for i, _ in keys]], 0.5 * ly * t[[j for _, j in keys]]])
    points = [core]
    previous = inner_ids
    count = core.shape[0]
    for r in range(1, m + 1):
        f = r / m
        points.append((1.0 - f) * inner + f * outer)
        current = count + np.arange(ring_size)
        count += ring_size
        nxt = (np.arange(ring_size) + 1) % ring_size
        quads.extend(np.column_stack([previous[nxt], previous, current[nxt], current]).tolist())
        phases.extend([0] * ring_size)
        previous = current
    outer_keys = {int(node): key for node, key in zip(previous, keys)}
    return np.vstack(points), np.asarray(quads, dtype=np.int64), np.asarray(phases, dtype=np.int64), outer_keys


def _ogrid_periodic_classes(cross_count: int, layers: int, outer_keys: dict):
    """Union-find periodic classes (x, y pairs per layer in key order, then z pairs; the
    second root is linked under the first) numbered by ascending root, and the opposite
    face node lists."""
    parent = np.arange((layers + 1) * cross_count, dtype=np.int64)

    def root(a: int) -> int:
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = int(parent[a])
        return a

    def link(a: int, b: int) -> None:
        ra, rb = root(a), root(b)
        if ra != rb:
            parent[rb] = ra

    c = max(max(k) for k in outer_keys.values())
    side = {name: {} for name in ("x-", "x+", "y-", "y+")}
    for node, (i, j) in outer_keys.items():
        if i == 0:
            side["x-"][j] = node
        if i == c:
            side["x+"][j] = node
        if j == 0:
            side["y-"][i] = node
        if j == c:
            side["y+"][i] = node
    faces = {name: [] for name in side}
    for layer in range(layers + 1):
        off = layer * cross_count
        for axis in ("x", "y"):
            minus, plus = side[axis + "-"], side[axis + "+"]
            for key in sorted(minus):
                link(off + minus[key], off + plus[key])
                faces[axis + "-"].append(off + minus[key])
                faces[axis + "+"].append(off + plus[key])
    for node in range(cross_count):
        link(node, layers * cross_count + node)
    roots = np.asarray([root(a) for a in range(parent.size)], dtype=np.int64)
    class_ids = np.unique(roots, return_inverse=True)[1].astype(np.int64)
    bottom = np.arange(cross_count, dtype=np.int64)
    face_nodes = ((np.asarray(faces["x-"], dtype=np.int64), np.asarray(faces["x+"], dtype=np.int64)),
                  (np.asarray(faces["y-"], dtype=np.int64), np.asarray(faces["y+"], dtype=np.int64)),
                  (bottom, layers * cross_count + bottom))  # fmt: skip
    return class_ids, face_nodes


def build_cylindrical_ogrid_hex8(lengths, inclusion_volume_fraction: float, circumferential_divisions: int,
                                 matrix_radial_divisions: int, axial_divisions: int) -> CylindricalOGridHex8Mesh:  # fmt: skip
    """Centred z-cylinder O-grid of a periodic box, extruded in axial_divisions layers.

    Radius sqrt(f lx ly / pi); circumferential_divisions / 4 core divisions per side."""
    if circumferential_divisions % 4 != 0:
        raise ValueError("O-grid circumferential divisions must be divisible by four.")
    if matrix_radial_divisions <= 0 or axial_divisions <= 0:
        raise ValueError("O-grid radial and axial divisions must be positive.")
    lx, ly, lz = (float(v) for v in lengths)
    radius = float(np.sqrt(inclusion_volume_fraction * lx * ly / np.pi))
    if radius >= 0.5 * min(lx, ly):
        raise ValueError("Cylindrical inclusion intersects the periodic cell boundary.")
    section, quads, phases, outer_keys = _ogrid_section(lx, ly, radius, circumferential_divisions // 4,
                                                         matrix_radial_divisions)  # fmt: skip
    nc = section.shape[0]
    layers = axial_divisions
    z = lz * np.arange(layers + 1) / layers
    nodes = np.column_stack([np.tile(section, (layers + 1, 1)), np.repeat(z, nc)])
    base = (np.arange(layers) * nc)[:, None, None]
    elements = np.concatenate([base + quads[None, :, :], base + nc + quads[None, :, :]], axis=2).reshape(-1, 8)
    element_phase = np.tile(phases, layers)
    class_ids, face_nodes = _ogrid_periodic_classes(nc, layers, outer_keys)
    q = section[quads[phases == 1]]  # (k, 4, 2): two triangles (0, 1, 2) and (1, 3, 2)
    tri = lambda a, b, o: 0.5 * np.abs((a[:, 0] - o[:, 0]) * (b[:, 1] - o[:, 1]) - (a[:, 1] - o[:, 1]) * (b[:, 0] - o[:, 0]))  # noqa: E731,E501
    area = float(np.sum(tri(q[:, 1], q[:, 2], q[:, 0]) + tri(q[:, 3], q[:, 2], q[:, 1])))
    return CylindricalOGridHex8Mesh(nodes, elements.astype(np.int64), element_phase.astype(np.int64), class_ids,
                                    face_nodes, float(np.pi * radius**2), area)  # fmt: skip


def _element_volumes(nodes: np.ndarray, elements: np.ndarray) -> np.ndarray:
    """Sum over the 2x2x2 Gauss points of det J per Hex8 element (host set-up)."""
    g = 1.0 / np.sqrt(3.0)
    pts = np.asarray([(a, b, c) for a in (-g, g) for b in (-g, g) for c in (-g, g)])
    signs = np.asarray([[(-1.0, 1.0)[(a >> d) & 1] for d in range(3)] for a in range(8)])
    f = 1.0 + pts[:, None, :] * signs[None, :, :]
    dref = np.stack([0.125 * signs[None, :, 0] * f[:, :, 1] * f[:, :, 2], 0.125 * signs[None, :, 1] * f[:, :, 0] * f[:, :, 2],
                     0.125 * signs[None, :, 2] * f[:, :, 0] * f[:, :, 1]], axis=2)  # fmt: skip
    jac = np.einsum("eai,qaj->eqij", nodes[elements], dref)
    return np.linalg.det(jac).sum(axis=1)


def build_cylindrical_two_phase_rve(mesh: CylindricalOGridHex8Mesh, matrix_material, inclusion_material,
                                    newton_settings: NonlinearNewtonSettings, hill_mandel_power_scale: float,
                                    quadrature_order: int = 2) -> StructuredHex8RVE:  # fmt: skip
    """Two-phase RVE on an O-grid: phase 0 matrix, phase 1 the cylindrical inclusion, the
    effective density volume-weighted, periodic classes from the mesh topology."""
    volumes = _element_volumes(mesh.nodes, mesh.elements)
    vm = float(np.sum(volumes[mesh.element_phase_ids == 0]))
    vi = float(np.sum(volumes[mesh.element_phase_ids == 1]))
    density = (matrix_material.density * vm + inclusion_material.density * vi) / (vm + vi)
    phased = PhasedMaterialModel(
        name=f"{matrix_material.name}__{inclusion_material.name}",
        phases=(RVEPhase("matrix", matrix_material), RVEPhase("inclusion", inclusion_material)),
        point_phase_ids=np.repeat(mesh.element_phase_ids, 8),
        effective_density=density,
    )
    constraint = build_periodic_constraint_from_classes(mesh.nodes, mesh.periodic_class_ids, (0, 0, 0),
                                                        mesh.opposite_face_nodes)  # fmt: skip
    return StructuredHex8RVE(
        nodes=mesh.nodes, elements=mesh.elements, divisions=(0, 0, 0), material=phased, constraint=constraint,
        newton_settings=newton_settings, element_phase_ids=mesh.element_phase_ids,
        element_densities=np.where(mesh.element_phase_ids == 0, matrix_material.density, inclusion_material.density),
        phase_names=("matrix", "inclusion"), quadrature_order=quadrature_order,
        hill_mandel_power_scale=hill_mandel_power_scale,
    )  # fmt: skip
