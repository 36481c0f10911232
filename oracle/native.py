"""Build and bind the plain-C oracle (``oracle/j2vp_oracle.c``) -- test infrastructure only.

``build_oracle()`` compiles it with gcc (-O3 -fopenmp) into ``oracle/_build/``;
``j2vp_incremental_c`` runs it on (6, n) float64 SoA NumPy arrays.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "j2vp_oracle.c"
OUT_DIR = HERE / "_build"
LIB = OUT_DIR / "libj2vp_oracle.so"


class OracleParams(ctypes.Structure):
    _fields_ = [
        ("young_modulus", ctypes.c_double),
        ("poisson_ratio", ctypes.c_double),
        ("yield_stress", ctypes.c_double),
        ("hardening_modulus", ctypes.c_double),
        ("time_scale", ctypes.c_double),
        ("reference_stress", ctypes.c_double),
        ("rate_exponent", ctypes.c_double),
        ("max_iterations", ctypes.c_int),
        ("yield_relative_tolerance", ctypes.c_double),
        ("residual_absolute_tolerance", ctypes.c_double),
        ("residual_relative_tolerance", ctypes.c_double),
    ]


def build_oracle(force: bool = False) -> Path:
    """Compile the C oracle if the shared object is missing or stale."""
    OUT_DIR.mkdir(exist_ok=True)
    if force or not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
        tmp = LIB.with_suffix(".so.tmp")
        cmd = ["gcc", "-O3", "-march=x86-64-v2", "-fopenmp", "-fPIC", "-shared", str(SRC), "-o", str(tmp), "-lm"]
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


_lib: ctypes.CDLL | None = None


def _load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(os.fspath(build_oracle()))
        lib.oracle_j2vp_incremental.restype = ctypes.c_int64
        lib.oracle_j2vp_incremental.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double] + [ctypes.c_void_p] * 9 + [ctypes.c_int]
        lib.oracle_max_threads.restype = ctypes.c_int
        _lib = lib
    return _lib


def max_threads() -> int:
    return int(_load().oracle_max_threads())


def j2vp_incremental_c(params, dt: float, dstrain, stress_n, plastic_strain_n, eqps_n, with_tangent=True,
                       threads: int = 0) -> dict:  # fmt: skip
    """Run the C oracle on SoA (6, n) float64 arrays; returns outputs and per-point status."""
    lib = _load()
    de = np.ascontiguousarray(dstrain, dtype=np.float64)
    n = de.shape[1]
    s0 = np.ascontiguousarray(stress_n, dtype=np.float64)
    ep0 = np.ascontiguousarray(plastic_strain_n, dtype=np.float64)
    q0 = np.ascontiguousarray(eqps_n, dtype=np.float64)
    s1 = np.empty((6, n))
    ep1 = np.empty((6, n))
    q1 = np.empty(n)
    tan = np.empty((36, n)) if with_tangent else None
    status = np.empty(n, dtype=np.int32)
    p = OracleParams(params.young_modulus, params.poisson_ratio, params.yield_stress, params.hardening_modulus,
                     params.time_scale, params.reference_stress, params.rate_exponent, params.max_iterations,
                     params.yield_relative_tolerance, params.residual_absolute_tolerance,
                     params.residual_relative_tolerance)  # fmt: skip
    lib.oracle_j2vp_incremental(
        ctypes.byref(p), n, float(dt), de.ctypes.data, s0.ctypes.data, ep0.ctypes.data, q0.ctypes.data,
        s1.ctypes.data, ep1.ctypes.data, q1.ctypes.data, None if tan is None else tan.ctypes.data,
        status.ctypes.data, int(threads),
    )  # fmt: skip
    return {"stress": s1, "plastic_strain": ep1, "eqps": q1, "tangent": tan, "status": status}
