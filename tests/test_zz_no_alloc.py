"""GPU test of cib_rve_pcg_noalloc, the RVE PCG solve that allocates nothing.

It is meant for callers that cannot allocate device memory (allocator hooks, frameworks
that forbid device allocations after start-up); its work vectors live in a fixed 1.5 MiB
array inside the library.  The test calls it twice in a row through the C ABI on the same
systems as the ordinary entry point cib_rve_pcg (whose work vectors the caller allocates)
and requires the same solutions (tolerance rtol 1e-12 of the largest entry; the arithmetic
is the same, so they agree to the bit in practice), iteration counts and statuses.  This
file is collected after every other test file.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

import concrete_impact_b200 as cib
from concrete_impact_b200 import _native
from concrete_impact_b200 import rve as R
from concrete_impact_b200.rve_builders import build_two_phase_sphere_rve, config0_materials

pytestmark = pytest.mark.gpu

MAX_VEC = 65536


def _prepared_batch() -> R.RVEBatch:
    """Two two-phase RVEs after one residual pass, so the tangent data and residual exist."""
    mortar, aggregate = config0_materials()
    newton = R.NonlinearNewtonSettings(25, 1.0e-6, 1.0e-8, 1.0e-14, 1.0e-10)
    models = [build_two_phase_sphere_rve((n, n, n), mortar, aggregate, newton, seed=s) for n, s in ((4, 11), (6, 12))]
    batch = R.RVEBatch(models)
    batch.macro.copy_(torch.as_tensor([[-1.2e-3, 2.5e-4, 2.5e-4, 0, 1e-4, 0], [8e-4, -2e-4, -2e-4, 3e-4, 0, 0]],
                                      device=batch.device))  # fmt: skip
    batch.dt.copy_(torch.as_tensor([5e-6, 1e-5], device=batch.device))
    settings = cib.MaterialUpdateSettings(50, 1.0e-10, 1.0e-12, 1.0e-10)
    batch.residual(batch.batch_struct(settings), batch.w, None, None)
    batch._settings_used = settings
    return batch


def _outputs(batch: R.RVEBatch):
    dev = batch.device
    n = batch.nrve
    return (torch.full((3 * batch.nelem,), float("nan"), dtype=torch.float64, device=dev),
            torch.full((n,), -7, dtype=torch.int32, device=dev), torch.full((n,), -7, dtype=torch.int32, device=dev),
            torch.zeros(n, dtype=torch.float64, device=dev), torch.zeros(n, dtype=torch.float64, device=dev))  # fmt: skip


def test_noalloc_pcg_matches_allocating_entry_on_two_calls_in_a_row() -> None:
    batch = _prepared_batch()
    lib = _native.load_library()
    b = batch.batch_struct(batch._settings_used)
    vec_len = 3 * batch.nelem
    assert vec_len <= MAX_VEC
    # reference: the ordinary entry point with caller-allocated work vectors
    x_ref, st_ref, it_ref, rel_ref, xn_ref = _outputs(batch)
    batch.pcg(b, batch.res, x_ref, batch.r, batch.p, batch.Ap, batch.nrve, batch.sys_rve, batch.sys_off, st_ref,
              it_ref, rel_ref, xn_ref)  # fmt: skip
    torch.cuda.synchronize()
    assert torch.all(st_ref == 0), st_ref
    for _call in range(2):
        x, st, it, rel, xn = _outputs(batch)
        code = lib.cib_rve_pcg_noalloc(
            ctypes.byref(b), batch.nrve, batch.sys_rve.data_ptr(), batch.sys_off.data_ptr(), batch.active.data_ptr(),
            vec_len, batch.res.data_ptr(), batch.dinv.data_ptr(), x.data_ptr(), float(batch.rtol),
            int(batch.linear.max_iterations), st.data_ptr(), it.data_ptr(), rel.data_ptr(), xn.data_ptr(),
            _native.stream_ptr(),
        )  # fmt: skip
        assert code == 0
        torch.cuda.synchronize()
        xr = x_ref.cpu().numpy()
        np.testing.assert_allclose(x.cpu().numpy(), xr, rtol=1e-12, atol=1e-12 * np.abs(xr).max())
        assert torch.equal(st, st_ref) and torch.equal(it, it_ref)
        np.testing.assert_allclose(xn.cpu().numpy(), xn_ref.cpu().numpy(), rtol=1e-12)
        np.testing.assert_allclose(rel.cpu().numpy(), rel_ref.cpu().numpy(), rtol=1e-9, atol=1e-300)


def test_noalloc_pcg_rejects_sizes_beyond_its_work_array() -> None:
    batch = _prepared_batch()
    lib = _native.load_library()
    b = batch.batch_struct(batch._settings_used)
    x, st, it, rel, xn = _outputs(batch)
    code = lib.cib_rve_pcg_noalloc(
        ctypes.byref(b), batch.nrve, batch.sys_rve.data_ptr(), batch.sys_off.data_ptr(), batch.active.data_ptr(),
        MAX_VEC + 1, batch.res.data_ptr(), batch.dinv.data_ptr(), x.data_ptr(), 1e-10, 100, st.data_ptr(),
        it.data_ptr(), rel.data_ptr(), xn.data_ptr(), _native.stream_ptr(),
    )  # fmt: skip
    assert code == -3  # CIB_ERANGE: nothing launched
    assert torch.all(st == -7)


def test_noalloc_pcg_skips_a_system_whose_offset_leaves_the_work_array() -> None:
    """A system offset that would put r, p, Ap past vec_len is refused by the kernel's own
    bounds check (status 3, nothing written); the other system is solved as usual."""
    batch = _prepared_batch()
    lib = _native.load_library()
    b = batch.batch_struct(batch._settings_used)
    vec_len = 3 * batch.nelem
    x_ref, st_ref, it_ref, rel_ref, xn_ref = _outputs(batch)
    batch.pcg(b, batch.res, x_ref, batch.r, batch.p, batch.Ap, batch.nrve, batch.sys_rve, batch.sys_off, st_ref,
              it_ref, rel_ref, xn_ref)  # fmt: skip
    bad_off = batch.sys_off.clone()
    bad_off[1] = vec_len - 3  # the second RVE's 3 E entries would run past the end
    x, st, it, rel, xn = _outputs(batch)
    code = lib.cib_rve_pcg_noalloc(
        ctypes.byref(b), batch.nrve, batch.sys_rve.data_ptr(), bad_off.data_ptr(), batch.active.data_ptr(),
        vec_len, batch.res.data_ptr(), batch.dinv.data_ptr(), x.data_ptr(), float(batch.rtol),
        int(batch.linear.max_iterations), st.data_ptr(), it.data_ptr(), rel.data_ptr(), xn.data_ptr(),
        _native.stream_ptr(),
    )  # fmt: skip
    assert code == 0
    torch.cuda.synchronize()
    assert st.cpu().tolist() == [0, 3] and int(it[1]) == 0
    n0 = 3 * int(batch.elem_counts[0])
    np.testing.assert_allclose(x[:n0].cpu().numpy(), x_ref[:n0].cpu().numpy(), rtol=1e-12,
                               atol=1e-12 * float(x_ref.abs().max()))  # fmt: skip
    assert torch.isnan(x[n0:]).all()  # the skipped system's solution was never written
