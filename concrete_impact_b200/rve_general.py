"""Periodic RVE solve on general Hex8 meshes on the GPU.

The reference's solve_rve_microequilibrium (src/fem/rve/solver.py:62-227), its response
(_build_rve_response, :253-364), effective tangent (_compute_effective_tangent, :438-461)
and reaction checks (:464-494) for any mesh whose periodic classes come with the mesh --
the cylindrical O-grid RVE of ``rve_builders.build_cylindrical_ogrid_hex8`` and other
unstructured cells.  ``rve.solve_rve_microequilibrium`` and ``rve.build_rve_operator_cache``
dispatch here for every model that is not a structured box.

The structured-box batch (``rve.RVEBatch``) relies on identical box elements; a general mesh
has per-element geometry, so each Newton iterate runs the general Hex8 kernels:
``u = T w + A ebar`` as two CSR products, the Hex8 assembly with the material at every
Gauss point (strains, material update, internal force, CSR tangent K), ``r = T^T f``, the
reduced tangent ``T^T K T`` gathered from K's values in a fixed order (``cib_csr_gather``;
T is a 0/1 matrix, so every reduced entry is a sum of K entries), and its Jacobi-PCG solve
(``cib_csr_pcg``) in place of the reference's direct factorisation.  The effective tangent
takes six K products with the columns of A, their reductions and six PCG solves; it uses
``K_ew = K_we^T`` (K is symmetric for the J2 and elastic tangents).
"""

from __future__ import annotations

import ctypes
import math
from typing import Any

import numpy as np
import torch
from scipy.sparse import csr_matrix

from . import _native
from .assembly import assemble_hex8_material_response_cached, build_hex8_material_assembly_cache
from .materials import MaterialState, _Io

CSR_PCG_WORK_DOUBLES = 3 * 1024 + 8  # CIB_CSR_PCG_WORK_DOUBLES


class _DeviceCSR:
    """A CSR matrix on the device with y = M x through cib_csr_spmv."""

    def __init__(self, matrix, device) -> None:
        m = csr_matrix(matrix)
        m.sort_indices()
        self.rows, self.cols = m.shape
        self.indptr = torch.as_tensor(m.indptr.astype(np.int64), device=device)
        self.indices = torch.as_tensor(m.indices.astype(np.int64), device=device)
        self.values = torch.as_tensor(m.data.astype(np.float64), device=device)
        self.device = device

    def mv(self, lib, x: torch.Tensor) -> torch.Tensor:
        y = torch.empty(self.rows, dtype=torch.float64, device=self.device)
        if self.rows:
            _native.check(lib.cib_csr_spmv(self.rows, self.indptr.data_ptr(), self.indices.data_ptr(),
                                           self.values.data_ptr(), x.contiguous().data_ptr(), y.data_ptr(),
                                           _native.stream_ptr()), "cib_csr_spmv")  # fmt: skip
        return y


class _ReducedSystem:
    """Jacobi-PCG on a CSR system whose rows are all free (the reduced periodic tangent)."""

    def __init__(self, indptr: np.ndarray, indices: np.ndarray, n: int, device, relative_tolerance: float,
                 max_iterations: int) -> None:  # fmt: skip
        self.n = n
        self.indptr = torch.as_tensor(indptr.astype(np.int64), device=device)
        self.indices = torch.as_tensor(indices.astype(np.int64), device=device)
        f64 = dict(dtype=torch.float64, device=device)
        self.values = torch.empty(int(indices.size), **f64)
        self.dinv = torch.empty(n, **f64)
        self.free = torch.ones(n, dtype=torch.uint8, device=device)
        self.r, self.z, self.p, self.q = (torch.empty(n, **f64) for _ in range(4))
        self.work = torch.zeros(CSR_PCG_WORK_DOUBLES, **f64)
        self.rtol, self.maxit = relative_tolerance, max_iterations
        self.device = device
        self.iterations = 0

    def prepare(self, lib, values: torch.Tensor) -> None:
        """Copy the matrix values (values / 1) and form the Jacobi inverse diagonal."""
        _native.check(lib.cib_newmark_effective_tangent(self.n, self.indptr.data_ptr(), self.indices.data_ptr(), None,
                                                        values.data_ptr(), 1.0, self.free.data_ptr(),
                                                        self.values.data_ptr(), self.dinv.data_ptr(),
                                                        _native.stream_ptr()), "cib_newmark_effective_tangent")  # fmt: skip

    def solve(self, lib, rhs: torch.Tensor) -> tuple[torch.Tensor, int, int, float]:
        x = torch.empty(self.n, dtype=torch.float64, device=self.device)
        status, iterations, rel = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_double(0.0)
        _native.check(lib.cib_csr_pcg(self.n, self.indptr.data_ptr(), self.indices.data_ptr(), self.values.data_ptr(),
                                      self.free.data_ptr(), self.dinv.data_ptr(), rhs.contiguous().data_ptr(),
                                      x.data_ptr(), self.r.data_ptr(), self.z.data_ptr(), self.p.data_ptr(),
                                      self.q.data_ptr(), self.work.data_ptr(), float(self.rtol), int(self.maxit), 16,
                                      ctypes.byref(status), ctypes.byref(iterations), ctypes.byref(rel),
                                      _native.stream_ptr()), "cib_csr_pcg")  # fmt: skip
        self.iterations += int(iterations.value)
        return x, int(status.value), int(iterations.value), float(rel.value)


class GeneralRVEOperators:
    """Device operators of one general-mesh RVE: the Hex8 assembly cache, T, T^T, A, A^T as
    CSR, the reduced tangent's pattern and gather lists, and the PCG work vectors."""

    def __init__(self, model, relative_tolerance: float = 1.0e-11, max_iterations: int = 20000) -> None:
        if model.quadrature_order != 2:
            raise NotImplementedError("The GPU RVE solver uses the 2x2x2 Gauss rule.")
        dev = _native.require_cuda()
        self.lib = _native.load_library()
        self.device = dev
        self.cache = build_hex8_material_assembly_cache(model.nodes, model.elements)
        weights = self.cache.jw.reshape(-1).cpu().numpy()
        if np.any(weights <= 0.0):
            raise ValueError("RVE operator cache requires strictly positive quadrature weights.")
        self.weights_host = weights
        self.weights = self.cache.jw.reshape(-1)
        self.volume = float(np.sum(weights))
        c = model.constraint
        t = csr_matrix(c.transformation)
        a = np.asarray(c.affine_matrix, dtype=np.float64)
        self.n, self.m = t.shape
        self.T, self.Tt = _DeviceCSR(t, dev), _DeviceCSR(t.T, dev)
        self.A, self.At = _DeviceCSR(a, dev), _DeviceCSR(a.T, dev)
        self.A_cols = torch.as_tensor(np.ascontiguousarray(a.T), device=dev)  # (6, 3N)
        # reduced DOF of every physical DOF (-1 for the eliminated reference class)
        red = np.full(self.n, -1, dtype=np.int64)
        has = np.diff(t.indptr) > 0
        red[has] = t.indices[t.indptr[:-1][has]]
        kp, ki = self.cache.csr_indptr, self.cache.csr_indices
        rows = np.repeat(np.arange(self.n), np.diff(kp))
        rr, rc = red[rows], red[ki]
        keep = np.flatnonzero((rr >= 0) & (rc >= 0))
        key = rr[keep] * max(self.m, 1) + rc[keep]
        order = np.argsort(key, kind="stable")
        ukey, start = np.unique(key[order], return_index=True)
        self.gather_ptr = torch.as_tensor(np.append(start, key.size).astype(np.int64), device=dev)
        self.gather_list = torch.as_tensor(keep[order].astype(np.int64), device=dev)
        urow = ukey // max(self.m, 1)
        indptr = np.zeros(self.m + 1, dtype=np.int64)
        np.add.at(indptr, urow + 1, 1)
        self.reduced = _ReducedSystem(np.cumsum(indptr), ukey % max(self.m, 1), self.m, dev, relative_tolerance,
                                      max_iterations)  # fmt: skip
        self.reduced_values = torch.empty(int(ukey.size), dtype=torch.float64, device=dev)
        self.class_ids = np.asarray(c.equivalence_class_ids, dtype=np.int64)
        self.faces = [(np.asarray(mi, dtype=np.int64), np.asarray(pl, dtype=np.int64)) for mi, pl in c.opposite_face_nodes]

    def gather_reduced(self, k_values: torch.Tensor) -> torch.Tensor:
        """Values of T^T K T from the values of K (fixed-order sums)."""
        nnz = int(self.reduced_values.numel())
        _native.check(self.lib.cib_csr_gather(nnz, self.gather_ptr.data_ptr(), self.gather_list.data_ptr(),
                                              k_values.contiguous().data_ptr(), self.reduced_values.data_ptr(),
                                              _native.stream_ptr()), "cib_csr_gather")  # fmt: skip
        return self.reduced_values

    def spmv_k(self, tangent, x: torch.Tensor) -> torch.Tensor:
        y = torch.empty(self.n, dtype=torch.float64, device=self.device)
        _native.check(self.lib.cib_csr_spmv(self.n, tangent.crow_indices().data_ptr(), tangent.col_indices().data_ptr(),
                                            tangent.values().data_ptr(), x.contiguous().data_ptr(), y.data_ptr(),
                                            _native.stream_ptr()), "cib_csr_spmv")  # fmt: skip
        return y


def _failure(request, iteration, residual_norm, residual_tolerance, increment_norm, increment_tolerance,
             assembly) -> dict[str, Any]:  # fmt: skip
    """The reference's RVE Newton failure snapshot (src/fem/rve/solver.py:497-518)."""
    tan = assembly.tangent
    rows = torch.repeat_interleave(torch.arange(tan.shape[0], device=tan.device), tan.crow_indices().diff())
    diag = tan.values()[tan.col_indices() == rows]
    return {"algorithm": "periodic_rve_microequilibrium_newton", "macro_strain": np.asarray(request.macro_strain).tolist(),
            "time_step": request.time_step, "iteration": iteration, "residual_norm": residual_norm,
            "residual_tolerance": residual_tolerance, "increment_norm": increment_norm,
            "increment_tolerance": increment_tolerance,
            "maximum_absolute_stress": float(torch.as_tensor(assembly.stresses).abs().max()),
            "minimum_tangent_diagonal": float(diag.min())}  # fmt: skip


def solve_general_rve_microequilibrium(model, request, committed_state, ops: GeneralRVEOperators):
    """One strain-driven periodic RVE update on a general mesh (solver.py:62-227)."""
    from .dynamics import ArmijoLineSearchError, perform_armijo_search
    from .rve import RVEEquilibriumError

    lib, dev = ops.lib, ops.device
    macro = np.asarray(request.macro_strain.cpu() if isinstance(request.macro_strain, torch.Tensor)
                       else request.macro_strain, dtype=np.float64)  # fmt: skip
    io = _Io(committed_state.fluctuation_dofs)
    ebar = torch.as_tensor(macro, device=dev)
    w = io.to_device(committed_state.fluctuation_dofs).reshape(-1).clone()
    u_prev = ops.T.mv(lib, w) + ops.A.mv(lib, io.to_device(committed_state.macro_strain).reshape(6))
    newton = model.newton_settings
    initial = None
    last_increment_norm = math.inf
    backtracks = 0

    def trial(fluct: torch.Tensor, need_tangent: bool = True):  # candidates too (solver.py:176-204, 229-251)
        u = ops.T.mv(lib, fluct) + ops.A.mv(lib, ebar)
        asm = assemble_hex8_material_response_cached(model.nodes, model.elements, model.material,
                                                     committed_state.material_state, u, u_prev, request.time_step,
                                                     request.material_update_settings, ops.cache, need_tangent)  # fmt: skip
        return u, asm, ops.Tt.mv(lib, asm.internal_force)

    for iteration in range(newton.max_iterations + 1):
        u, asm, r = trial(w)
        norms = torch.stack([torch.linalg.vector_norm(r), torch.linalg.vector_norm(w)]).cpu().numpy()
        rn, wn = float(norms[0]), float(norms[1])
        if initial is None:
            initial = rn
        tol = max(newton.residual_absolute_tolerance, newton.residual_relative_tolerance * initial)
        inc_tol = max(newton.increment_absolute_tolerance, newton.increment_relative_tolerance * max(wn, 1.0))
        if rn <= tol and (iteration == 0 or last_increment_norm <= inc_tol):
            return _general_response(model, request, committed_state, macro, w, u, asm, iteration, backtracks, rn, tol,
                                     ops, io)  # fmt: skip
        if iteration == newton.max_iterations:
            raise RVEEquilibriumError("maximum_iterations_exceeded",
                                      _failure(request, iteration, rn, tol, last_increment_norm, inc_tol, asm))  # fmt: skip
        ops.reduced.prepare(lib, ops.gather_reduced(asm.tangent.values()))
        inc, status, pcg_iterations, pcg_rel = ops.reduced.solve(lib, -r)
        inc_norm = float(torch.linalg.vector_norm(inc))
        if not math.isfinite(inc_norm):
            raise RVEEquilibriumError("non_finite_increment", _failure(request, iteration, rn, tol, inc_norm, inc_tol, asm))
        if status != 0:
            d = _failure(request, iteration, rn, tol, inc_norm, inc_tol, asm)
            d.update(linear_solver_status=status, linear_solver_iterations=pcg_iterations,
                     linear_solver_relative_residual=pcg_rel)  # fmt: skip
            raise RVEEquilibriumError("linear_solver_not_converged", d)
        if rn <= tol and inc_norm <= inc_tol:
            return _general_response(model, request, committed_state, macro, w, u, asm, iteration, backtracks, rn, tol,
                                     ops, io)  # fmt: skip
        step = 1.0
        if newton.armijo.enabled:
            base = w
            try:
                search = perform_armijo_search(
                    rn, lambda s: float(torch.linalg.vector_norm(trial(base + s * inc)[2])),
                    newton.armijo)  # fmt: skip
            except ArmijoLineSearchError as error:
                d = _failure(request, iteration, rn, tol, inc_norm, inc_tol, asm)
                d["armijo"] = error.diagnostics
                raise RVEEquilibriumError("armijo_exhausted", d) from error
            step = search.step_length
            backtracks += search.backtracks
        accepted = inc if step == 1.0 else step * inc
        w = w + accepted
        last_increment_norm = float(torch.linalg.vector_norm(accepted))
    raise AssertionError("RVE Newton loop ended without a convergence decision.")


def effective_tangent(ops: GeneralRVEOperators, tangent) -> torch.Tensor:
    """(K_ee - K_we^T K_ww^-1 K_we) / V with K_ww = T^T K T, K_we = T^T K A, K_ee = A^T K A."""
    from .rve import RVEEquilibriumError

    lib = ops.lib
    ka = torch.stack([ops.spmv_k(tangent, ops.A_cols[j]) for j in range(6)])  # (6, 3N)
    k_ee = ops.A_cols @ ka.T
    if ops.m == 0:
        return k_ee / ops.volume
    k_we = torch.stack([ops.Tt.mv(lib, ka[j]) for j in range(6)])  # (6, m)
    ops.reduced.prepare(lib, ops.gather_reduced(tangent.values()))
    sens = []
    for j in range(6):
        x, status, _, _ = ops.reduced.solve(lib, k_we[j])
        if status != 0 or not bool(torch.isfinite(x).all()):
            raise RVEEquilibriumError("non_finite_effective_tangent_sensitivity", {"reduced_dof_count": ops.m})
        sens.append(x)
    return (k_ee - k_we @ torch.stack(sens).T) / ops.volume


def _general_response(model, request, committed, macro, w, u, asm, iterations, backtracks, rn, tol, ops, io):
    """The reference's RVEResponse of a converged microstate (solver.py:253-364)."""
    from .rve import RVEResponse, RVEState

    lib = ops.lib
    wts = ops.weights
    vol = ops.volume
    stress = torch.as_tensor(asm.stresses, device=ops.device)
    macro_stress = (stress * wts[:, None]).sum(0) / vol
    virtual = ops.At.mv(lib, asm.internal_force) / vol
    tangent = effective_tangent(ops, asm.tangent) if request.requirements.tangent else None
    strains = torch.as_tensor(asm.strains, device=ops.device)
    rates = torch.as_tensor(asm.strain_rates, device=ops.device)
    increment = strains - (strains - request.time_step * rates)
    micro_work = float(((stress * increment).sum(1) * wts).sum() / vol)
    macro_n = np.asarray(committed.macro_strain.cpu() if isinstance(committed.macro_strain, torch.Tensor)
                         else committed.macro_strain, dtype=np.float64)  # fmt: skip
    macro_stress_h = macro_stress.cpu().numpy()
    macro_work = float(macro_stress_h @ (macro - macro_n))
    hm_res = macro_work - micro_work
    hm_err = abs(hm_res) / (abs(macro_work) + abs(micro_work) + model.hill_mandel_power_scale * request.time_step)
    diag = asm.diagnostics
    if "incremental_work_density" not in diag:
        raise ValueError("RVE J2 diagnostics require incremental_work_density.")
    if "viscoplastic_active" not in diag:
        raise ValueError("RVE J2 diagnostics require viscoplastic_active.")
    work = torch.as_tensor(diag["incremental_work_density"], device=ops.device)
    active = torch.as_tensor(diag["viscoplastic_active"], device=ops.device)
    f_host = asm.internal_force.cpu().numpy()
    u_host = u.cpu().numpy()
    nodal = f_host.reshape(-1, 3)
    fluct = (u_host - model.constraint.affine_matrix @ macro).reshape(-1, 3)
    rep = model.constraint.representative_nodes[ops.class_ids]
    periodic_error = float(np.max(np.linalg.norm(fluct - fluct[rep], axis=1), initial=0.0))
    reaction = 0.0
    for minus, plus in ops.faces:
        fm, fp = nodal[minus].sum(0), nodal[plus].sum(0)
        reaction = max(reaction, float(np.linalg.norm(fm + fp)) / max(float(np.linalg.norm(fm) + np.linalg.norm(fp)), 1.0))
    class_force = np.zeros((int(ops.class_ids.max()) + 1, 3))
    np.add.at(class_force, ops.class_ids, nodal)
    class_reaction = float(np.max(np.linalg.norm(class_force, axis=1))) / max(float(np.linalg.norm(f_host)), 1.0)
    margin = torch.as_tensor(diag.get("yield_activation_margin", torch.full_like(wts, float("nan"))), device=ops.device)
    finite = margin[torch.isfinite(margin)]
    available = finite.numel() > 0
    psi = torch.as_tensor(asm.free_energy, device=ops.device)
    diss = torch.as_tensor(asm.dissipation, device=ops.device)
    material_state = MaterialState({k: io.out(torch.as_tensor(v, device=ops.device)) if isinstance(v, torch.Tensor) else v
                                    for k, v in asm.state.variables.items()})  # fmt: skip
    state = RVEState(material_state, io.out(torch.as_tensor(macro, device=ops.device)), io.out(w.clone()))
    diagnostics = {
        "micro_residual_norm": rn,
        "micro_residual_tolerance": tol,
        "newton_iterations": iterations,
        "armijo_backtracks": backtracks,
        "volume": vol,
        "virtual_work_stress_error": float(torch.linalg.vector_norm(virtual - macro_stress)),
        "periodic_fluctuation_error": periodic_error,
        "reaction_antiperiodicity_error": reaction,
        "periodic_class_reaction_error": class_reaction,
        "macro_work_increment": macro_work,
        "micro_work_increment": micro_work,
        "hill_mandel_residual": hm_res,
        "hill_mandel_error": hm_err,
        "positive_work_density": float((work.clamp(min=0.0) * wts).sum() / vol),
        "negative_work_density": float((work.clamp(max=0.0) * wts).sum() / vol),
        "unloading_volume_fraction": float(wts[work < 0.0].sum() / vol),
        "viscoplastic_active_volume_fraction": float(wts[active > 0.5].sum() / vol),
        "yield_activation_margin_available": int(available),
        "minimum_yield_activation_margin": float(finite.min()) if available else np.nan,
        "maximum_yield_activation_margin": float(finite.max()) if available else np.nan,
        "linear_solver_iterations": ops.reduced.iterations,
    }
    return RVEResponse(
        macro_stress=io.out(macro_stress), effective_tangent=None if tangent is None else io.out(tangent),
        state=state, displacement=io.out(u), micro_strains=io.out(strains), micro_stresses=io.out(stress),
        micro_diagnostics={k: io.out(torch.as_tensor(v, device=ops.device)) for k, v in diag.items()},
        free_energy_density=float((psi * wts).sum() / vol), dissipation_density=float((diss * wts).sum() / vol),
        phase_diagnostics=_phase_diagnostics(model, asm, stress, psi, diss, wts, vol), diagnostics=diagnostics,
    )  # fmt: skip


def _phase_diagnostics(model, asm, stress, psi, diss, wts, vol) -> dict[str, dict[str, Any]]:
    """Phase volumes, average stresses, energies and state-field names (solver.py:391-435)."""
    n_el = model.elements.shape[0]
    if model.element_phase_ids is None:
        point_phase = np.zeros(8 * n_el, dtype=np.int64)
        names: tuple[str, ...] = ("domain",)
    else:
        point_phase = np.repeat(np.asarray(model.element_phase_ids, dtype=np.int64), 8)
        names = model.phase_names
    out = {}
    for i, name in enumerate(names):
        mask = torch.as_tensor(point_phase == i, device=stress.device)
        pw = wts[mask]
        pv = float(pw.sum())
        fields = (tuple(asm.state.variables) if model.element_phase_ids is None
                  else tuple(k for k in asm.state.variables if k.startswith(f"phase_{name}__")))  # fmt: skip
        out[name] = {
            "volume": pv,
            "volume_fraction": pv / vol,
            "average_stress": ((stress[mask] * pw[:, None]).sum(0) / pv).cpu().numpy(),
            "free_energy_density": float((psi[mask] * pw).sum() / pv),
            "dissipation_density": float((diss[mask] * pw).sum() / pv),
            "state_fields": fields,
        }
    return out

