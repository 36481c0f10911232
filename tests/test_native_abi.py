"""CPU tests of the C ABI: the library loads and exports every symbol of include/cib200.h."""

from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from concrete_impact_b200 import _native
from concrete_impact_b200.materials import (
    J2ViscoplasticMaterial,
    MaterialPointRequest,
    MaterialUpdateSettings,
    build_j2_viscoplastic_material,
)

REPO = Path(__file__).resolve().parents[1]


def _declared_functions() -> set[str]:
    text = (REPO / "include" / "cib200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(cib_[a-z0-9_]+)\s*\(", text))


def test_library_exports_every_declared_symbol() -> None:
    lib = _native.load_library()
    declared = _declared_functions()
    assert declared, "no declarations parsed"
    for name in sorted(declared):
        assert hasattr(lib, name), name
    # and nm agrees (dynamic symbol table, C linkage)
    out = subprocess.run(["nm", "-D", "--defined-only", str(_native.LIB_PATH)], capture_output=True, text=True, check=True)
    exported = set(re.findall(r"\bT (cib_[a-z0-9_]+)$", out.stdout, flags=re.M))
    assert declared <= exported, declared - exported
    assert set(_native.SIGNATURES) == declared


def _declared_prototypes() -> dict[str, int]:
    """Parameter count of every cib_ function prototype in the header."""
    text = (REPO / "include" / "cib200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(cib_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text, flags=re.S):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_ctypes_signatures_match_header_prototypes() -> None:
    """Every ctypes binding passes exactly the C prototype's number of arguments."""
    protos = _declared_prototypes()
    assert set(protos) == set(_native.SIGNATURES)
    for name, count in protos.items():
        assert len(_native.SIGNATURES[name][1]) == count, (name, count, len(_native.SIGNATURES[name][1]))


def test_struct_layouts_match_header() -> None:
    """ctypes mirrors of the C structs have the C sizes (no silent padding mismatch)."""
    assert ctypes.sizeof(_native.J2VPMaterialC) == 7 * 8
    assert ctypes.sizeof(_native.UpdateSettingsC) == 8 + 3 * 8
    assert ctypes.sizeof(_native.J2VPFailureC) == 16 + 17 * 8 + 12 * 8 + 16


def test_names_and_reasons_need_no_gpu() -> None:
    names = _native.j2_diagnostic_names()
    from oracle.j2vp import DIAGNOSTIC_NAMES, REASONS

    assert names == DIAGNOSTIC_NAMES
    assert [_native.j2_reason(i) for i in range(len(REASONS))] == REASONS
    assert _native.load_library().cib_version().decode().startswith("cib200")


def test_argument_errors_are_rejected_without_a_launch() -> None:
    lib = _native.load_library()
    m = _native.J2VPMaterialC(25e9, 0.2, 20e6, 2e9, 1e-3, 20e6, 1.0)
    s = _native.UpdateSettingsC(50, 0, 1e-10, 1e-12, 1e-10)
    # null buffers and negative sizes come back as CIB_EINVAL (-1)
    assert lib.cib_j2vp_update_soa_f64(ctypes.byref(m), ctypes.byref(s), 16, 16, 1e-5, *([None] * 10)) == -1
    assert lib.cib_j2vp_update_soa_f64(ctypes.byref(m), ctypes.byref(s), -1, 0, 1e-5, *([None] * 10)) == -1
    assert lib.cib_j2vp_update(ctypes.byref(m), ctypes.byref(s), 4, 1e-5, *([None] * 16)) == -1
    assert lib.cib_copy_rows_async(None, 8, None, 8, 8, 1, 1, None) == -1
    # zero points is a no-op success
    assert lib.cib_j2vp_update_soa_f32(ctypes.byref(m), ctypes.byref(s), 0, 0, 1e-5, *([1] * 9), None, None, None) == 0


def test_kinematics_and_shape_contract_errors_precede_the_gpu() -> None:
    material = J2ViscoplasticMaterial("m", 1.0, 1000.0, 0.25, 1.0, 1.0, 1.0, 1.0, 1.0)
    settings = MaterialUpdateSettings(50, 1e-10, 1e-12, 1e-10)
    state = material.initialize_state(2)
    with pytest.raises(ValueError, match="three_dimensional"):
        material.update(MaterialPointRequest(np.zeros((2, 6)), None, 1.0, "plane_strain", settings), state)
    with pytest.raises(ValueError, match=r"\(n_points, 6\)"):
        material.update(MaterialPointRequest(np.zeros((2, 3)), None, 1.0, "three_dimensional", settings), state)


def test_material_validation_matches_reference_messages() -> None:
    base = dict(name="m", density=1.0, young_modulus=1.0, poisson_ratio=0.2, yield_stress=1.0, hardening_modulus=0.0,
                time_scale=1.0, reference_stress=1.0, rate_exponent=1.0)  # fmt: skip
    build_j2_viscoplastic_material(base)
    for key, value, message in [("young_modulus", 0.0, "young_modulus > 0"), ("poisson_ratio", 0.5, "poisson_ratio"),
                                ("rate_exponent", 0.5, "rate_exponent >= 1"), ("time_scale", 0.0, "time_scale > 0")]:  # fmt: skip
        with pytest.raises(ValueError, match=message):
            build_j2_viscoplastic_material({**base, key: value})


def test_struct_layouts_match_c_header(tmp_path) -> None:
    """sizeof/offsetof of the C structs (compiled from include/cib200.h with the host C
    compiler) equal the ctypes mirrors' layouts."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    checks = {
        "cib_rve_batch": (_native.RVEBatchC, ["nelem", "desc", "mats", "settings", "plastic_strain_n", "de"]),
        "cib_rno_window": (_native.RNOWindowC, ["ldt", "strain", "W", "Wt", "bias", "skip", "Z", "Xt", "Ht", "stress",
                                                "loss_part", "dYt", "dZt", "err"]),
        "cib_phase_material": (_native.PhaseMaterialC, ["params"]),
    }
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "cib200.h"', "int main(void) {"]
    for name, (_, fields) in checks.items():
        lines.append(f'  printf("{name} %zu\\n", sizeof({name}));')
        for f in fields:
            lines.append(f'  printf("{name}.{f} %zu\\n", offsetof({name}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    include = Path(__file__).resolve().parent.parent / "include"
    subprocess.run([cc, f"-I{include}", str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines())
    for name, (cls, fields) in checks.items():
        assert int(got[name]) == ctypes.sizeof(cls), name
        for f in fields:
            assert int(got[f"{name}.{f}"]) == getattr(cls, f).offset, f"{name}.{f}"


def test_sizes_beyond_32_bit_indexing_are_refused_without_a_launch() -> None:
    """The surrogate's elementwise entry points index with 32-bit ints; batches whose
    element count would overflow come back as CIB_ERANGE (-3) before any CUDA call."""
    lib = _native.load_library()
    big = 2**31 // 16  # B * 32 inputs per row overflows int32
    fake = 256  # never dereferenced: the size check comes first
    assert lib.cib_rno_input(big, fake, fake, fake, fake, None, 0, 0, None) == -3
    assert lib.cib_rno_backward_tail(big, fake, fake, fake, None) == -3
    assert lib.cib_rno_forward_tail(2**31 // 8, fake, None, fake, fake, fake, None, 1.0, None, None) == -3
    assert lib.cib_adam_step(65536, 65536, fake, fake, fake, fake, 1e-3, 0.9, 0.999, 1e-8, fake, None, 0, None, 0,
                             None) == -3  # fmt: skip
    assert lib.cib_splitk_reduce(65536, 65536, 1, fake, 65536, fake, 65536, None) == -3


def test_tensor_core_entry_points_check_their_contracts_before_the_gpu() -> None:
    """The tcgen05 GEMM and the fused surrogate window reject shapes outside their tile
    contract (N a multiple of 16 up to 128, K a multiple of 16, 16-byte aligned rows, width
    128) with CIB_EINVAL, and treat an empty batch as a no-op, all before any CUDA call."""
    lib = _native.load_library()
    fake = 256  # 16-byte aligned, never dereferenced
    gemm = lib.cib_mlp_gemm
    # epilogue, M, N, K, A, lda, B, ldb, splits, bias, C, ldc, Z, ldz, H, ldh, Ht, ldht, row_offset, err, stream
    ok = dict(M=128, N=128, K=64, lda=64, ldb=64)

    def call(**kw):
        a = {**ok, **kw}
        return gemm(0, a["M"], a["N"], a["K"], fake, a["lda"], fake, a["ldb"], 1, None, fake, a["N"], None, 0, None, 0,
                    None, 0, 0, fake, None)  # fmt: skip

    assert call(N=24) == -1 and call(N=144) == -1 and call(K=8) == -1 and call(lda=60) == -1 and call(ldb=72 + 4) == -1
    assert call(M=0) == 0  # empty: no launch
    w = _native.RNOWindowC()
    w.B, w.T, w.hidden = 0, 1, 128
    w.strain = w.rate = w.coef = w.z = w.err = fake
    for i in range(4):
        w.W[i], w.bias[i] = fake, fake
    assert lib.cib_rno_window_forward(ctypes.byref(w), None) == 0  # empty batch
    w.hidden = 96
    assert lib.cib_rno_window_forward(ctypes.byref(w), None) == -1  # the fused kernels are width 128
    w.hidden, w.B, w.gS = 128, 4, fake
    assert lib.cib_rno_window_forward(ctypes.byref(w), None) == -1  # loss gradient without a target
