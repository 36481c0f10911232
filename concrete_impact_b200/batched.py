"""Batched return map on device-resident structure-of-arrays state, and a host pipeline.

``j2vp_update_soa`` is the streaming entry for large batches (millions of Gauss points)
whose state already lives in HBM: component c of point p sits at ``[c, p]`` of a (6, n)
tensor.  It computes the same update as J2ViscoplasticMaterial.update of the reference
(src/fem/materials/plasticity.py:343-431) in the incremental, stress-carried form:
the trial stress is ``stress_n + C dstrain``.

``J2HostPipeline`` runs the same kernel on batches held in pinned host memory: the batch
is cut into chunks whose host-to-device copy, kernel and device-to-host copy run on three
streams, so PCIe transfers in both directions overlap each other and the kernel.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _native
from .materials import J2ViscoplasticMaterial, MaterialPointConvergenceError, MaterialUpdateSettings, _j2_failure

_KIND_H2D = 1
_KIND_D2H = 2


def _flags(device: torch.device) -> torch.Tensor:
    flags = torch.zeros(2, dtype=torch.int64, device=device)
    flags[0] = -1
    return flags


@dataclass
class SoAState:
    """Device-resident state of a batch of J2 points (SoA)."""

    stress: torch.Tensor  # (6, n), float32 or float64
    plastic_strain: torch.Tensor  # (6, n), same dtype
    eqps: torch.Tensor  # (n,), float64 (history is always double)

    @staticmethod
    def empty(n: int, dtype: torch.dtype, device: torch.device) -> SoAState:
        return SoAState(
            torch.empty((6, n), dtype=dtype, device=device),
            torch.empty((6, n), dtype=dtype, device=device),
            torch.empty((n,), dtype=torch.float64, device=device),
        )


def _entry(dtype: torch.dtype, compact: bool = False):
    lib = _native.load_library()
    if dtype == torch.float64:
        return lib.cib_j2vp_update_soa_compact_f64 if compact else lib.cib_j2vp_update_soa_f64
    if dtype == torch.float32:
        return lib.cib_j2vp_update_soa_compact_f32 if compact else lib.cib_j2vp_update_soa_f32
    raise TypeError(f"unsupported dtype {dtype}; use float32 or float64")


def expand_compact_tangent(compact: torch.Tensor, material: J2ViscoplasticMaterial) -> torch.Tensor:
    """(36, n) consistent tangent from the compact (8, n) rows n (6), f, c:
    C = K 1(x)1 + f P + c n(x)n (plasticity.py:929-963 in factored form)."""
    e, nu = float(material.young_modulus), float(material.poisson_ratio)
    bulk = e / (3.0 * (1.0 - 2.0 * nu))
    n, f, c = compact[:6], compact[6], compact[7]
    p = torch.zeros((6, 6), dtype=compact.dtype, device=compact.device)
    p[:3, :3] = -1.0 / 3.0
    p[range(3), range(3)] = 2.0 / 3.0
    p[range(3, 6), range(3, 6)] = 0.5
    vol = torch.zeros((6, 6), dtype=compact.dtype, device=compact.device)
    vol[:3, :3] = bulk
    out = vol.reshape(36, 1) + p.reshape(36, 1) * f[None, :] + c[None, :] * (n[:, None, :] * n[None, :, :]).reshape(36, -1)
    return out


def launch_j2vp_soa(
    material: J2ViscoplasticMaterial,
    settings: MaterialUpdateSettings,
    time_step: float,
    dstrain: torch.Tensor,
    state_n: SoAState,
    state: SoAState,
    tangent: torch.Tensor | None,
    flags: torch.Tensor,
    stream: torch.cuda.Stream | None = None,
    count: int | None = None,
) -> None:
    """Asynchronous launch (no host sync).  ``flags[0]`` receives the lowest failing index.

    The (6, ld) / (36, ld) tensors may hold more columns than the ``count`` points updated
    (default: all ld columns); the leading dimension is the tensors' row length.  A tangent
    of 8 rows receives the compact form (n (6), f, c; ``expand_compact_tangent``).
    """
    ld = int(dstrain.shape[1])
    n = ld if count is None else int(count)
    if not 0 <= n <= ld:
        raise ValueError("count must lie in [0, ld].")
    for t in (dstrain, state_n.stress, state_n.plastic_strain, state.stress, state.plastic_strain):
        if t.shape != (6, ld) or not t.is_contiguous() or t.dtype != dstrain.dtype:
            raise ValueError("SoA arrays must be contiguous (6, ld) tensors of one dtype.")
    for t in (state_n.eqps, state.eqps):
        if t.shape[0] < n or t.dtype != torch.float64 or not t.is_contiguous():
            raise ValueError("equivalent plastic strain must be a contiguous float64 tensor of >= count points.")
    if tangent is not None and (tangent.shape not in ((36, ld), (8, ld)) or not tangent.is_contiguous()
                                or tangent.dtype != dstrain.dtype):  # fmt: skip
        raise ValueError("tangent must be a contiguous (36, ld) (full) or (8, ld) (compact) tensor of the state dtype.")
    compact = tangent is not None and tangent.shape[0] == 8
    mat_c = _native.material_struct(material)
    set_c = _native.settings_struct(settings)
    code = _entry(dstrain.dtype, compact)(
        ctypes.byref(mat_c), ctypes.byref(set_c), n, ld, float(time_step),
        dstrain.data_ptr(), state_n.stress.data_ptr(), state_n.plastic_strain.data_ptr(), state_n.eqps.data_ptr(),
        state.stress.data_ptr(), state.plastic_strain.data_ptr(), state.eqps.data_ptr(), _native.ptr(tangent),
        flags.data_ptr(), _native.stream_ptr(stream),
    )  # fmt: skip
    _native.check(code, "cib_j2vp_update_soa")


def j2vp_update_soa(
    material: J2ViscoplasticMaterial,
    settings: MaterialUpdateSettings,
    time_step: float,
    dstrain: torch.Tensor,
    state_n: SoAState,
    with_tangent: bool = True,
) -> tuple[SoAState, torch.Tensor | None]:
    """Update a device-resident batch; returns (new state, tangent (36, n) or None).

    Raises MaterialPointConvergenceError for the first failing point, like the reference.
    The committed state ``state_n`` is never written.
    """
    _native.require_cuda()
    n = int(dstrain.shape[1])
    state = SoAState.empty(n, dstrain.dtype, dstrain.device)
    tangent = torch.empty((36, n), dtype=dstrain.dtype, device=dstrain.device) if with_tangent else None
    flags = _flags(dstrain.device)
    if n > 0:
        launch_j2vp_soa(material, settings, time_step, dstrain, state_n, state, tangent, flags)
        first = int(flags[0].item())
        if first != -1:
            raise soa_failure(material, settings, time_step, dstrain, state_n, first)
    return state, tangent


def soa_failure(material, settings, time_step, dstrain, state_n, point: int) -> Exception:
    """Exception of the reference for one failed point of an SoA batch.

    The point is restated in the reference's total-strain form (strain = C^-1 stress_n +
    plastic_strain_n + dstrain) and its failure snapshot is taken by the device.
    """
    from .materials import MaterialPointRequest, _Io

    g = material.young_modulus / (2.0 * (1.0 + material.poisson_ratio))
    lam = material.young_modulus * material.poisson_ratio / ((1.0 + material.poisson_ratio) * (1.0 - 2.0 * material.poisson_ratio))
    c = np.zeros((6, 6))
    c[:3, :3] = lam
    c[[0, 1, 2], [0, 1, 2]] += 2.0 * g
    c[[3, 4, 5], [3, 4, 5]] = g
    s = state_n.stress[:, point].double().cpu().numpy()
    ep = state_n.plastic_strain[:, point].double().cpu().numpy()
    de = dstrain[:, point].double().cpu().numpy()
    strain = (np.linalg.solve(c, s) + ep + de).reshape(1, 6)
    io = _Io(torch.empty(0, device=dstrain.device))
    eps = io.to_device(strain)
    request = MaterialPointRequest(strain, None, time_step, "three_dimensional", settings)
    ep0 = io.to_device(ep.reshape(1, 6))
    q0 = io.to_device(state_n.eqps[point : point + 1])
    error = _j2_failure(material, request, strain, eps, None, ep0, q0, 0, _native.settings_struct(settings),
                        _native.material_struct(material), io)  # fmt: skip
    if isinstance(error, MaterialPointConvergenceError):
        error = error.with_context(point_id=int(point))
    return error


def copy_rows_async(dst: int, dst_pitch: int, src: int, src_pitch: int, row_bytes: int, rows: int, kind: int,
                    stream: torch.cuda.Stream) -> None:  # fmt: skip
    """Strided 2-D copy (one cudaMemcpy2DAsync) between host and device."""
    lib = _native.load_library()
    code = lib.cib_copy_rows_async(dst, dst_pitch, src, src_pitch, row_bytes, rows, kind, _native.stream_ptr(stream))
    _native.check(code, "cib_copy_rows_async")


class J2HostPipeline:
    """Return map over a batch held in pinned host memory (SoA, (6, n) rows).

    Chunks of ``chunk`` points are copied in on one stream, updated on a second and
    copied out on a third, with two device buffer sets in flight.  Results land in the
    caller's pinned host output arrays; ``run`` returns after the last copy finished.
    ``compact_tangent`` returns the tangent as 8 rows (n, f, c) instead of 36, which cuts
    the device-to-host traffic per point from 48 to 20 values.
    """

    def __init__(self, material: J2ViscoplasticMaterial, settings: MaterialUpdateSettings, dtype: torch.dtype,
                 chunk: int = 1 << 20, with_tangent: bool = True, buffers: int = 2,
                 compact_tangent: bool = False) -> None:  # fmt: skip
        self.device = _native.require_cuda()
        self.material = material
        self.settings = settings
        self.dtype = dtype
        self.chunk = int(chunk)
        self.with_tangent = with_tangent
        self.tangent_rows = 8 if compact_tangent else 36
        self.h2d = torch.cuda.Stream()
        self.compute = torch.cuda.Stream()
        self.d2h = torch.cuda.Stream()
        self.sets = []
        for _ in range(buffers):
            self.sets.append(
                {
                    "de": torch.empty((6, self.chunk), dtype=dtype, device=self.device),
                    "in": SoAState.empty(self.chunk, dtype, self.device),
                    "out": SoAState.empty(self.chunk, dtype, self.device),
                    "tan": (torch.empty((self.tangent_rows, self.chunk), dtype=dtype, device=self.device)
                            if with_tangent else None),
                    "loaded": torch.cuda.Event(),
                    "computed": torch.cuda.Event(),
                    "drained": torch.cuda.Event(),
                    "used": False,
                }
            )
        self.flags = _flags(self.device)

    @staticmethod
    def bytes_per_point(dtype: torch.dtype, with_tangent: bool, compact_tangent: bool = False) -> tuple[int, int]:
        """(host-to-device, device-to-host) bytes per point."""
        w = 8 if dtype == torch.float64 else 4
        rows = (8 if compact_tangent else 36) if with_tangent else 0
        return 18 * w + 8, (12 + rows) * w + 8

    def run(self, time_step: float, dstrain: torch.Tensor, state_n: SoAState, state: SoAState,
            tangent: torch.Tensor | None) -> int:  # fmt: skip
        """Update host arrays (pinned, contiguous) in place of ``state``/``tangent``; returns
        the lowest failing point index or -1."""
        n = int(dstrain.shape[1])
        w = dstrain.element_size()
        self.flags[0] = -1
        caller = torch.cuda.current_stream()
        self.h2d.wait_stream(caller)
        self.compute.wait_stream(caller)
        for start in range(0, n, self.chunk):
            count = min(self.chunk, n - start)
            buf = self.sets[(start // self.chunk) % len(self.sets)]
            if buf["used"]:
                self.h2d.wait_event(buf["drained"])
            buf["used"] = True

            def rows_in(dst: torch.Tensor, src: torch.Tensor, nrows: int, width: int) -> None:
                copy_rows_async(dst.data_ptr(), self.chunk * width, src.data_ptr() + start * width, n * width,
                                count * width, nrows, _KIND_H2D, self.h2d)  # fmt: skip

            rows_in(buf["de"], dstrain, 6, w)
            rows_in(buf["in"].stress, state_n.stress, 6, w)
            rows_in(buf["in"].plastic_strain, state_n.plastic_strain, 6, w)
            rows_in(buf["in"].eqps, state_n.eqps, 1, 8)
            buf["loaded"].record(self.h2d)
            self.compute.wait_event(buf["loaded"])
            launch_j2vp_soa(self.material, self.settings, time_step, buf["de"], buf["in"], buf["out"], buf["tan"],
                            self.flags, self.compute, count=count)  # fmt: skip
            buf["computed"].record(self.compute)
            self.d2h.wait_event(buf["computed"])

            def rows_out(dst: torch.Tensor, src: torch.Tensor, nrows: int, width: int) -> None:
                copy_rows_async(dst.data_ptr() + start * width, n * width, src.data_ptr(), self.chunk * width,
                                count * width, nrows, _KIND_D2H, self.d2h)  # fmt: skip

            rows_out(state.stress, buf["out"].stress, 6, w)
            rows_out(state.plastic_strain, buf["out"].plastic_strain, 6, w)
            rows_out(state.eqps, buf["out"].eqps, 1, 8)
            if tangent is not None and buf["tan"] is not None:
                rows_out(tangent, buf["tan"], self.tangent_rows, w)
            buf["drained"].record(self.d2h)
        self.d2h.synchronize()
        return int(self.flags[0].item())
