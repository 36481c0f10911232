"""Host wrappers of the tensor-core MLP GEMM (``cib_mlp_gemm``) used by the surrogate."""

from __future__ import annotations

import torch

from . import _native

EPI_F32, EPI_BIAS_F32, EPI_BIAS_GELU, EPI_GELU_BWD, EPI_PARTIAL = 0, 1, 2, 3, 4


def _ld(t: torch.Tensor) -> int:
    return int(t.stride(0))


def gemm(
    epilogue: int,
    a: torch.Tensor,
    b: torch.Tensor,
    *,
    n: int | None = None,
    bias: torch.Tensor | None = None,
    c: torch.Tensor | None = None,
    z: torch.Tensor | None = None,
    h: torch.Tensor | None = None,
    ht: torch.Tensor | None = None,
    row_offset: int = 0,
    splits: int = 1,
    err: torch.Tensor,
    rows: int | None = None,
    stream: torch.cuda.Stream | None = None,
) -> None:
    """Launch C = A B^T with an epilogue (asynchronous).  ``a``: (M, K) bf16, ``b``: (N, K)
    bf16, both row-major with unit column stride; outputs per the epilogue."""
    m = int(a.shape[0]) if rows is None else int(rows)
    k = int(a.shape[1])
    n = int(b.shape[0]) if n is None else int(n)
    for t in (a, b):
        if t.dtype != torch.bfloat16 or t.stride(1) != 1:
            raise ValueError("GEMM operands must be bf16 with unit column stride")
    code = _native.load_library().cib_mlp_gemm(
        int(epilogue), m, n, k, a.data_ptr(), _ld(a), b.data_ptr(), _ld(b), int(splits), _native.ptr(bias),
        _native.ptr(c), 0 if c is None else _ld(c), _native.ptr(z), 0 if z is None else _ld(z), _native.ptr(h),
        0 if h is None else _ld(h), _native.ptr(ht), 0 if ht is None else _ld(ht), int(row_offset), err.data_ptr(),
        _native.stream_ptr(stream),
    )  # fmt: skip
    _native.check(code, "cib_mlp_gemm")


def splitk_reduce(partial: torch.Tensor, splits: int, m: int, n: int, out: torch.Tensor,
                  stream: torch.cuda.Stream | None = None) -> None:  # fmt: skip
    """out (m, n) = sum of the ``splits`` fp32 partial tiles in ``partial`` (fixed order)."""
    code = _native.load_library().cib_splitk_reduce(m, n, splits, partial.data_ptr(), int(partial.shape[-1]),
                                                    out.data_ptr(), _ld(out), _native.stream_ptr(stream))  # fmt: skip
    _native.check(code, "cib_splitk_reduce")
