"""Hex8 material-response assembly on the GPU (drop-in for fem.assembly.nonlinear_solid).

Same names, arguments and results as the reference
(src/fem/assembly/nonlinear_solid.py:36-180): ``MaterialAssemblyCache``,
``NonlinearSolidAssemblyResult``, ``initialize_hex8_material_state``,
``build_hex8_material_assembly_cache``, ``assemble_hex8_material_response`` and
``assemble_hex8_material_response_cached``, for any Hex8 mesh and any material that
implements the material protocol on the GPU (this package's models).

The cache keeps the physical shape-function gradients on the device (192 doubles per
element) plus the node and CSR gather lists of the mesh, built once; ``b_matrices`` is
materialised only when read.  Strains, internal force and the CSR tangent are computed by
the kernels of ``csrc/hex8.cu`` with a deterministic (fixed-order, atomic-free) assembly.
"""

from __future__ import annotations

import warnings
from dataclasses import dataclass, field
from typing import Any

import numpy as np
import torch
from scipy.sparse import csr_matrix

from . import _native
from .materials import (
    MaterialModel,
    MaterialPointConvergenceError,
    MaterialPointRequest,
    MaterialResponseRequirements,
    MaterialState,
    MaterialUpdateSettings,
    _Io,
)

QUADRATURE_POINTS = 8


@dataclass(frozen=True)
class NonlinearSolidAssemblyResult:
    """One nonlinear solid assembly result."""

    internal_force: Any
    tangent: Any
    state: MaterialState
    strains: Any
    strain_rates: Any
    stresses: Any
    diagnostics: dict[str, Any]
    free_energy: Any
    dissipation: Any


@dataclass(frozen=True)
class MaterialAssemblyCache:
    """Displacement-strain operators and quadrature weights of one Hex8 mesh (device)."""

    grads: torch.Tensor  # (E, 8, 8, 3) dN/dx
    jw: torch.Tensor  # (E, 8)
    elements: torch.Tensor  # (E, 8) int64
    node_count: int
    node_ptr: torch.Tensor
    node_list: torch.Tensor
    csr_indptr: np.ndarray
    csr_indices: np.ndarray
    csr_ptr: torch.Tensor
    csr_list: torch.Tensor
    _host: dict = field(default_factory=dict, repr=False, compare=False)

    @property
    def jacobian_weights(self) -> np.ndarray:
        """(E, 8) det J times the Gauss weight."""
        if "jw" not in self._host:
            self._host["jw"] = self.jw.cpu().numpy()
        return self._host["jw"]

    @property
    def b_matrices(self) -> np.ndarray:
        """(E, 8, 6, 24) strain-displacement matrices (materialised on first access)."""
        if "b" not in self._host:
            g = self.grads.cpu().numpy()
            e = g.shape[0]
            b = np.zeros((e, 8, 6, 24))
            gx, gy, gz = g[..., 0], g[..., 1], g[..., 2]
            for a in range(8):
                b[:, :, 0, 3 * a], b[:, :, 1, 3 * a + 1], b[:, :, 2, 3 * a + 2] = gx[:, :, a], gy[:, :, a], gz[:, :, a]
                b[:, :, 3, 3 * a + 1], b[:, :, 3, 3 * a + 2] = gz[:, :, a], gy[:, :, a]
                b[:, :, 4, 3 * a], b[:, :, 4, 3 * a + 2] = gz[:, :, a], gx[:, :, a]
                b[:, :, 5, 3 * a], b[:, :, 5, 3 * a + 1] = gy[:, :, a], gx[:, :, a]
            self._host["b"] = b
        return self._host["b"]


def initialize_hex8_material_state(material: MaterialModel, element_count: int, quadrature_order: int = 2) -> MaterialState:
    """Integration-point state for Hex8 elements (8 points per element)."""
    _require_order(quadrature_order)
    return material.initialize_state(element_count * QUADRATURE_POINTS)


def _require_order(order: int) -> None:
    if order != 2:
        raise NotImplementedError("The GPU Hex8 assembly uses the 2x2x2 Gauss rule (quadrature_order=2).")


def build_hex8_material_assembly_cache(nodes, elements, quadrature_order: int = 2) -> MaterialAssemblyCache:
    """Geometry on the device plus the mesh's deterministic gather lists."""
    _require_order(quadrature_order)
    dev = _native.require_cuda()
    lib = _native.load_library()
    nodes_h = np.ascontiguousarray(np.asarray(nodes.cpu() if isinstance(nodes, torch.Tensor) else nodes, dtype=np.float64))
    el_h = np.ascontiguousarray(np.asarray(elements.cpu() if isinstance(elements, torch.Tensor) else elements, dtype=np.int64))
    ne, nn = el_h.shape[0], nodes_h.shape[0]
    nodes_d = torch.as_tensor(nodes_h, device=dev)
    el_d = torch.as_tensor(el_h, device=dev)
    grads = torch.empty((ne, 8, 8, 3), dtype=torch.float64, device=dev)
    jw = torch.empty((ne, 8), dtype=torch.float64, device=dev)
    bad = torch.zeros(1, dtype=torch.int64, device=dev)
    code = lib.cib_hex8_geometry(ne, nodes_d.data_ptr(), el_d.data_ptr(), grads.data_ptr(), jw.data_ptr(),
                                 bad.data_ptr(), _native.stream_ptr())  # fmt: skip
    _native.check(code, "cib_hex8_geometry")
    if int(bad.item()) > 0:
        raise ValueError("Hex8 nonlinear assembly requires positive Jacobian.")
    # node gather list: slots 8 e + a grouped by node, ascending slot order
    slots = np.arange(8 * ne, dtype=np.int64)
    node_of = el_h.reshape(-1)
    order = np.argsort(node_of, kind="stable")
    node_ptr = np.zeros(nn + 1, dtype=np.int64)
    np.add.at(node_ptr, node_of + 1, 1)
    node_ptr = np.cumsum(node_ptr)
    # CSR pattern of the 3N x 3N tangent and the (e, i, j) contributions of every entry
    dofs = (3 * el_h[:, :, None] + np.arange(3)).reshape(ne, 24)
    rows = np.repeat(dofs, 24, axis=1).reshape(-1)
    cols = np.tile(dofs, (1, 24)).reshape(-1)
    key = rows * (3 * nn) + cols
    korder = np.argsort(key, kind="stable")
    ukey, start = np.unique(key[korder], return_index=True)
    csr_ptr = np.append(start, key.size).astype(np.int64)
    urow = ukey // (3 * nn)
    indptr = np.zeros(3 * nn + 1, dtype=np.int64)
    np.add.at(indptr, urow + 1, 1)
    indptr = np.cumsum(indptr)
    return MaterialAssemblyCache(
        grads, jw, el_d, nn,
        torch.as_tensor(node_ptr, device=dev), torch.as_tensor(slots[order], device=dev),
        indptr, (ukey % (3 * nn)).astype(np.int64),
        torch.as_tensor(csr_ptr, device=dev), torch.as_tensor(korder.astype(np.int64), device=dev),
    )  # fmt: skip


def assemble_hex8_material_response(nodes, elements, material, committed_state, displacement, previous_displacement,
                                    time_step, update_settings: MaterialUpdateSettings, need_tangent: bool = True,
                                    quadrature_order: int = 2) -> NonlinearSolidAssemblyResult:  # fmt: skip
    """Assemble internal force and tangent from material-point responses."""
    cache = build_hex8_material_assembly_cache(nodes, elements, quadrature_order)
    return assemble_hex8_material_response_cached(nodes, elements, material, committed_state, displacement,
                                                  previous_displacement, time_step, update_settings, cache,
                                                  need_tangent)  # fmt: skip


def assemble_hex8_material_response_cached(nodes, elements, material, committed_state, displacement,
                                           previous_displacement, time_step, update_settings: MaterialUpdateSettings,
                                           cache: MaterialAssemblyCache,
                                           need_tangent: bool = True) -> NonlinearSolidAssemblyResult:  # fmt: skip
    """Strains -> material update -> internal force and CSR tangent, all on the device."""
    lib = _native.load_library()
    io = _Io(displacement)
    dev = cache.grads.device
    ne = int(cache.elements.shape[0])
    npts = 8 * ne
    u = io.to_device(displacement, (3 * cache.node_count,))
    up = io.to_device(previous_displacement, (3 * cache.node_count,))
    strains = torch.empty((npts, 6), dtype=torch.float64, device=dev)
    rates = torch.empty((npts, 6), dtype=torch.float64, device=dev)
    code = lib.cib_hex8_strains(ne, cache.elements.data_ptr(), cache.grads.data_ptr(), u.data_ptr(), up.data_ptr(),
                                float(time_step), strains.data_ptr(), rates.data_ptr(), _native.stream_ptr())  # fmt: skip
    _native.check(code, "cib_hex8_strains")
    request = MaterialPointRequest(strains, rates, time_step, "three_dimensional", update_settings)
    device_state = MaterialState({k: io.to_device(v) for k, v in committed_state.variables.items()})
    try:
        response = material.update(request, device_state,
                                   MaterialResponseRequirements(tangent=need_tangent, free_energy=True, dissipation=True))  # fmt: skip
    except MaterialPointConvergenceError as error:
        pid = int(error.diagnostics["point_id"])
        raise error.with_context(element_id=pid // QUADRATURE_POINTS, quadrature_id=pid % QUADRATURE_POINTS) from error
    if need_tangent and response.tangents is None:
        raise ValueError("Material assembly requested a tangent but received None.")
    if response.free_energy is None:
        raise ValueError("Material assembly requested free energy but received None.")
    if response.dissipation is None:
        raise ValueError("Material assembly requested dissipation but received None.")
    stress = io.to_device(response.stresses, (npts, 6))
    fe = torch.empty(npts * 3, dtype=torch.float64, device=dev)
    force = torch.empty(3 * cache.node_count, dtype=torch.float64, device=dev)
    code = lib.cib_hex8_internal_force(ne, cache.node_count, cache.grads.data_ptr(), cache.jw.data_ptr(),
                                       stress.data_ptr(), cache.node_ptr.data_ptr(), cache.node_list.data_ptr(),
                                       fe.data_ptr(), force.data_ptr(), _native.stream_ptr())  # fmt: skip
    _native.check(code, "cib_hex8_internal_force")
    tangent: Any = None
    n_dof = 3 * cache.node_count
    if need_tangent:
        tan = io.to_device(response.tangents, (npts, 6, 6))
        nnz = int(cache.csr_indices.size)
        ke = torch.empty(ne * 576, dtype=torch.float64, device=dev)
        values = torch.empty(nnz, dtype=torch.float64, device=dev)
        code = lib.cib_hex8_tangent_csr(ne, cache.grads.data_ptr(), cache.jw.data_ptr(), tan.data_ptr(), nnz,
                                        cache.csr_ptr.data_ptr(), cache.csr_list.data_ptr(), ke.data_ptr(),
                                        values.data_ptr(), _native.stream_ptr())  # fmt: skip
        _native.check(code, "cib_hex8_tangent_csr")
        if io.host:
            tangent = csr_matrix((values.cpu().numpy(), cache.csr_indices, cache.csr_indptr), shape=(n_dof, n_dof))
        else:
            # the pattern is the cache's own sorted CSR pattern: skip torch's invariant check
            # (and its notices that CSR support is beta and the check is off)
            with warnings.catch_warnings():
                warnings.simplefilter("ignore", UserWarning)
                tangent = torch.sparse_csr_tensor(torch.as_tensor(cache.csr_indptr, device=dev),
                                                  torch.as_tensor(cache.csr_indices, device=dev), values,
                                                  size=(n_dof, n_dof), check_invariants=False)  # fmt: skip
    else:
        tangent = csr_matrix((n_dof, n_dof)) if io.host else None
    return NonlinearSolidAssemblyResult(
        internal_force=io.out(force),
        tangent=tangent,
        state=MaterialState({k: io.out(v) if isinstance(v, torch.Tensor) else v for k, v in response.state.variables.items()}),
        strains=io.out(strains),
        strain_rates=io.out(rates),
        stresses=io.out(stress),
        diagnostics={k: io.out(v) if isinstance(v, torch.Tensor) else v for k, v in response.diagnostics.items()},
        free_energy=io.out(io.to_device(response.free_energy)),
        dissipation=io.out(io.to_device(response.dissipation)),
    )
