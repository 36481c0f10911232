"""CPU test of the host logic of the general-mesh RVE path (concrete_impact_b200.rve_general)
on the reference's cylindrical O-grid RVE.

The device is replaced by CPU stand-ins with the same interfaces: the C entry points the
path calls (CSR product, fixed-order gather, Jacobi set-up, PCG -- here a direct solve)
act on host memory through their pointer arguments, and the Hex8 assembly is the general
oracle's (oracle/rve_general.py).  What remains is the driver code of the GPU path: the
periodic operators and the reduced-tangent pattern and gather lists built from the
tangent's CSR layout, the Newton loop, the effective tangent and the response.  It must
reproduce the reference's golden solves.
"""

from __future__ import annotations

import ctypes
from types import SimpleNamespace

import numpy as np
import pytest
import torch
from scipy.sparse import coo_matrix, csr_matrix
from scipy.sparse.linalg import spsolve

import concrete_impact_b200.rve_general as G
from concrete_impact_b200 import _native
from concrete_impact_b200.assembly import NonlinearSolidAssemblyResult
from concrete_impact_b200.materials import (J2ViscoplasticMaterial, LinearElasticMaterial, MaterialResponseRequirements,
                                            MaterialState, MaterialUpdateSettings)  # fmt: skip
from concrete_impact_b200.rve import NonlinearNewtonSettings, RVERequest, initialize_rve_state
from concrete_impact_b200.rve_builders import build_cylindrical_ogrid_hex8, build_cylindrical_two_phase_rve
from conftest import load_case
from oracle import j2vp as oj
from oracle.rve import OraclePhase
from oracle.rve_general import general_rve_oracle


def _f64(ptr: int, n: int) -> np.ndarray:
    return np.ctypeslib.as_array((ctypes.c_double * max(n, 1)).from_address(ptr))[:n]


def _i64(ptr: int, n: int) -> np.ndarray:
    return np.ctypeslib.as_array((ctypes.c_int64 * max(n, 1)).from_address(ptr))[:n]


def _u8(ptr: int, n: int) -> np.ndarray:
    return np.ctypeslib.as_array((ctypes.c_uint8 * max(n, 1)).from_address(ptr))[:n]


class HostLibrary:
    """The C entry points of the general-mesh path, acting on host memory."""

    @staticmethod
    def _csr(n, indptr, indices, values):
        ip = _i64(indptr, n + 1).copy()
        nnz = int(ip[-1])
        ix = _i64(indices, nnz).copy()
        return ip, ix, _f64(values, nnz).copy()

    def cib_csr_spmv(self, n, indptr, indices, values, x, y, stream):
        ip, ix, v = self._csr(n, indptr, indices, values)
        cols = int(ix.max()) + 1 if ix.size else 0
        _f64(y, n)[:] = csr_matrix((v, ix, ip), shape=(n, cols)) @ _f64(x, cols)
        return 0

    def cib_csr_gather(self, nnz, ptr, lst, src, dst, stream):
        p = _i64(ptr, nnz + 1).copy()
        idx = _i64(lst, int(p[-1])).copy()
        s = _f64(src, int(idx.max()) + 1 if idx.size else 0)
        _f64(dst, nnz)[:] = [s[idx[p[k]:p[k + 1]]].sum() for k in range(nnz)]
        return 0

    def cib_newmark_effective_tangent(self, n, indptr, indices, k_values, m_values, beta_dt2, free, out, dinv, stream):
        ip, ix, m = self._csr(n, indptr, indices, m_values)
        k = _f64(k_values, m.size) if k_values else 0.0
        vals = k + m / beta_dt2
        _f64(out, m.size)[:] = vals
        diag = csr_matrix((vals, ix, ip), shape=(n, n)).diagonal()
        _f64(dinv, n)[:] = np.where(_u8(free, n) != 0, 1.0 / diag, 0.0)
        return 0

    def cib_csr_pcg(self, n, indptr, indices, values, free, dinv, b, x, r, z, p, q, work, rtol, maxit, check_every,
                    status, iterations, rel, stream):  # fmt: skip
        ip, ix, v = self._csr(n, indptr, indices, values)
        _f64(x, n)[:] = spsolve(csr_matrix((v, ix, ip), shape=(n, n)).tocsc(), _f64(b, n).copy())
        ctypes.cast(status, ctypes.POINTER(ctypes.c_int32))[0] = 0
        ctypes.cast(iterations, ctypes.POINTER(ctypes.c_int32))[0] = 1
        ctypes.cast(rel, ctypes.POINTER(ctypes.c_double))[0] = 0.0
        return 0


def _byref_address(obj) -> int:
    return ctypes.addressof(obj._obj) if hasattr(obj, "_obj") else int(obj)


class _Lib(HostLibrary):
    """Adapts ctypes.byref arguments to the addresses the stand-ins take."""

    def cib_csr_pcg(self, *args):
        args = list(args)
        for i in (16, 17, 18):
            args[i] = _byref_address(args[i])
        return super().cib_csr_pcg(*args)


@pytest.fixture
def host_general(monkeypatch):
    g, meta = load_case("rve_ogrid_cylinder")
    phases = [OraclePhase("j2", oj.J2Params(25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0)),
              OraclePhase("elastic", None, 50.0e9, 0.2)]  # fmt: skip
    oracle = general_rve_oracle(g["nodes"], g["elements"], g["periodic_class_ids"], int(g["face_x_minus"][0]), phases,
                                g["element_phase_ids"], {})  # fmt: skip
    n = 3 * g["nodes"].shape[0]
    pattern = coo_matrix((np.ones(oracle.rows.size), (oracle.rows, oracle.cols)), shape=(n, n)).tocsr()
    pattern.sort_indices()
    rows = np.repeat(np.arange(n), np.diff(pattern.indptr))

    def cache(nodes, elements):
        return SimpleNamespace(csr_indptr=pattern.indptr.astype(np.int64), csr_indices=pattern.indices.astype(np.int64),
                               jw=torch.as_tensor(oracle.jw))  # fmt: skip

    def assemble(nodes, elements, material, committed, u, u_prev, dt, settings, c, need_tangent=True):
        st = committed.variables.get("oracle") or oracle.initial_state()
        asm = oracle.assemble(u.numpy(), u_prev.numpy(), dt, st)
        t = lambda a: torch.as_tensor(np.asarray(a, dtype=np.float64))  # noqa: E731
        k = asm["K"].tocsr()
        tangent = torch.sparse_csr_tensor(torch.as_tensor(pattern.indptr.astype(np.int64)),
                                          torch.as_tensor(pattern.indices.astype(np.int64)),
                                          t(np.asarray(k[rows, pattern.indices]).ravel()), size=(n, n),
                                          check_invariants=False)  # fmt: skip
        diag = {"incremental_work_density": t(asm["iwd"]), "viscoplastic_active": t(asm["active"]),
                "yield_activation_margin": t(asm["margin"])}  # fmt: skip
        return NonlinearSolidAssemblyResult(t(asm["f"]), tangent, MaterialState({"oracle": asm["state"]}), t(asm["eps"]),
                                            t(asm["rate"]), t(asm["stress"]), diag, t(asm["psi"]), t(asm["diss"]))  # fmt: skip

    monkeypatch.setattr(_native, "require_cuda", lambda: torch.device("cpu"))
    monkeypatch.setattr(_native, "load_library", lambda: _Lib())
    monkeypatch.setattr(_native, "stream_ptr", lambda stream=None: 0)
    monkeypatch.setattr(G, "build_hex8_material_assembly_cache", cache)
    monkeypatch.setattr(G, "assemble_hex8_material_response_cached", assemble)
    s = meta["mesh"]
    mesh = build_cylindrical_ogrid_hex8(s["lengths"], s["inclusion_volume_fraction"], s["circumferential_divisions"],
                                        s["matrix_radial_divisions"], s["axial_divisions"])  # fmt: skip
    mortar = J2ViscoplasticMaterial("mortar", 2200.0, 25.0e9, 0.2, 20.0e6, 2.0e9, 1.0e-3, 20.0e6, 1.0)
    aggregate = LinearElasticMaterial("aggregate", 2600.0, 50.0e9, 0.2)
    model = build_cylindrical_two_phase_rve(mesh, mortar, aggregate, NonlinearNewtonSettings(*meta["newton"][:5]), 1.0)
    return model, G.GeneralRVEOperators(model), g, meta


def test_general_path_reproduces_reference_ogrid_solves(host_general) -> None:
    model, ops, g, meta = host_general
    state = initialize_rve_state(model)
    state = type(state)(MaterialState({}), state.macro_strain, state.fluctuation_dofs)
    update = MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)
    for step in range(meta["steps"]):
        request = RVERequest(g[f"s{step}__macro_strain"], meta["time_step"], update, MaterialResponseRequirements(tangent=True))
        out = G.solve_general_rve_microequilibrium(model, request, state, ops)
        state = out.state
        ref = meta["scalars"][step]
        assert out.diagnostics["newton_iterations"] == ref["newton_iterations"]
        for key, tol in (("macro_stress", 1e-12), ("effective_tangent", 1e-12), ("displacement", 1e-12)):
            r = g[f"s{step}__{key}"]
            np.testing.assert_allclose(np.asarray(getattr(out, key)), r, rtol=0, atol=tol * np.abs(r).max(), err_msg=key)
        np.testing.assert_allclose(np.asarray(out.state.fluctuation_dofs), g[f"s{step}__fluctuation"], rtol=0,
                                   atol=1e-12 * np.abs(g[f"s{step}__fluctuation"]).max())  # fmt: skip
        for key in ("viscoplastic_active_volume_fraction", "positive_work_density", "negative_work_density",
                    "unloading_volume_fraction", "macro_work_increment", "micro_work_increment"):  # fmt: skip
            assert out.diagnostics[key] == pytest.approx(ref[key], rel=1e-10, abs=1e-12), key
        # consistency measures at roundoff level: both sides are tiny, not equal
        scale = float(np.abs(g[f"s{step}__macro_stress"]).max())
        assert out.diagnostics["virtual_work_stress_error"] <= 1e-12 * scale
        for key in ("hill_mandel_error", "reaction_antiperiodicity_error", "periodic_class_reaction_error"):
            assert out.diagnostics[key] <= 1e-9 and ref[key] <= 1e-9, key
        assert out.diagnostics["periodic_fluctuation_error"] <= 1e-15
        assert out.free_energy_density == pytest.approx(ref["free_energy_density"], rel=1e-12)
        assert out.dissipation_density == pytest.approx(ref["dissipation_density"], rel=1e-10, abs=1e-6)
