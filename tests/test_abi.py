"""CPU-side checks of the C ABI: the library loads without a GPU, exports every
symbol include/mojoblas_gpu.h declares, and rejects invalid arguments with the
reference's Netlib `info` numbering before touching the device."""
import re
from pathlib import Path

import numpy as np
import pytest

import mojoblas_b200 as mb
from mojoblas_b200 import _lib as L

HEADER = Path(__file__).resolve().parents[1] / "include" / "mojoblas_gpu.h"


def declared_symbols():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(mbg_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = L.load()
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_symbols()) <= set(L.SIGNATURES), set(declared_symbols()) - set(L.SIGNATURES)


def test_version_and_status_strings():
    lib = L.load()
    assert lib.mbg_version() >= 100
    assert L.status_string(0) == "success"
    assert "Netlib" in L.status_string(3)
    assert L.status_string(L.MBG_ERR_TIMEOUT)


Z = np.zeros(64, dtype=np.float32)
D = np.zeros(64, dtype=np.float64)


@pytest.mark.parametrize("args,info", [
    (("X", "N", 2, 2, 2, 1.0, Z, 2, Z, 2, 0.0, Z, 2), 1),
    (("N", "q", 2, 2, 2, 1.0, Z, 2, Z, 2, 0.0, Z, 2), 2),
    (("N", "N", -1, 2, 2, 1.0, Z, 2, Z, 2, 0.0, Z, 2), 3),
    (("N", "N", 2, -1, 2, 1.0, Z, 2, Z, 2, 0.0, Z, 2), 4),
    (("N", "N", 2, 2, -1, 1.0, Z, 2, Z, 2, 0.0, Z, 2), 5),
    (("N", "N", 3, 2, 2, 1.0, Z, 2, Z, 2, 0.0, Z, 3), 8),
    (("T", "N", 2, 2, 3, 1.0, Z, 2, Z, 3, 0.0, Z, 2), 8),
    (("N", "N", 2, 2, 3, 1.0, Z, 2, Z, 2, 0.0, Z, 2), 10),
    (("N", "T", 2, 3, 2, 1.0, Z, 2, Z, 2, 0.0, Z, 2), 10),
    (("N", "N", 3, 2, 2, 1.0, Z, 3, Z, 2, 0.0, Z, 2), 13),
])
def test_gemm_info_codes(args, info, capsys):
    assert mb.gemm(*args) == info
    assert f"gemm: Info {info}" in capsys.readouterr().out


def test_gemm_double_and_modes_info():
    assert mb.gemm("N", "N", 2, 2, 2, 1.0, D, 1, D, 2, 0.0, D, 2) == 8
    assert mb.gemm("N", "N", 2, 2, 2, 1.0, Z, 1, Z, 2, 0.0, Z, 2, mode=mb.BF16X3) == 8
    assert mb.gemm("N", "N", 2, 2, 2, 1.0, D, 2, D, 1, 0.0, D, 2, mode=mb.OZAKI) == 10


@pytest.mark.parametrize("args,info", [
    (("X", "N", 2, 2, 1.0, Z, 2, 0.0, Z, 2), 1),
    (("L", "X", 2, 2, 1.0, Z, 2, 0.0, Z, 2), 2),
    (("L", "N", -2, 2, 1.0, Z, 2, 0.0, Z, 2), 3),
    (("L", "N", 2, -2, 1.0, Z, 2, 0.0, Z, 2), 4),
    (("L", "N", 3, 2, 1.0, Z, 2, 0.0, Z, 3), 7),
    (("U", "T", 2, 3, 1.0, Z, 2, 0.0, Z, 2), 7),
    (("U", "N", 3, 2, 1.0, Z, 3, 0.0, Z, 2), 10),
])
def test_syrk_info_codes(args, info):
    assert mb.syrk(*args) == info


@pytest.mark.parametrize("args,info", [
    (("X", "L", "N", "N", 2, 2, 1.0, Z, 2, Z, 2), 1),
    (("L", "X", "N", "N", 2, 2, 1.0, Z, 2, Z, 2), 2),
    (("L", "L", "X", "N", 2, 2, 1.0, Z, 2, Z, 2), 3),
    (("L", "L", "N", "X", 2, 2, 1.0, Z, 2, Z, 2), 4),
    (("L", "L", "N", "N", -1, 2, 1.0, Z, 2, Z, 2), 5),
    (("L", "L", "N", "N", 2, -1, 1.0, Z, 2, Z, 2), 6),
    (("L", "L", "N", "N", 3, 2, 1.0, Z, 2, Z, 3), 9),
    (("R", "L", "N", "N", 2, 3, 1.0, Z, 2, Z, 2), 9),
    (("L", "L", "N", "N", 3, 2, 1.0, Z, 3, Z, 2), 11),
])
def test_trsm_info_codes(args, info):
    assert mb.trsm(*args) == info


def test_quick_returns_touch_no_device():
    # m == 0 / n == 0 / syrk alpha == 0 and beta == 1 return before any CUDA call
    assert mb.gemm("N", "N", 0, 5, 5, 1.0, Z, 1, Z, 5, 0.0, Z, 1) == 0
    assert mb.gemm("T", "N", 4, 0, 5, 1.0, Z, 5, Z, 5, 0.0, Z, 4) == 0
    assert mb.syrk("L", "N", 0, 3, 1.0, Z, 1, 0.0, Z, 1) == 0
    assert mb.syrk("L", "N", 3, 3, 0.0, Z, 3, 1.0, Z, 3) == 0
    assert mb.trsm("L", "L", "N", "N", 0, 3, 1.0, Z, 1, Z, 1) == 0
    assert mb.trsm("R", "U", "T", "U", 3, 0, 1.0, Z, 1, Z, 3) == 0


def test_invalid_mode_rejected():
    lib = L.load()
    assert lib.mbg_sgemm_ex(9, b"N", b"N", 1, 1, 1, 1.0, Z.ctypes.data, 1, Z.ctypes.data, 1, 0.0,
                            Z.ctypes.data, 1) == L.MBG_ERR_INVALID_MODE
    assert lib.mbg_dgemm_ex(L.MODE_OZAKI, 1, b"N", b"N", 1, 1, 1, 1.0, D.ctypes.data, 1,
                            D.ctypes.data, 1, 0.0, D.ctypes.data, 1) == L.MBG_ERR_INVALID_MODE
    assert lib.mbg_dgemm_ex(L.MODE_OZAKI, 9, b"N", b"N", 1, 1, 1, 1.0, D.ctypes.data, 1,
                            D.ctypes.data, 1, 0.0, D.ctypes.data, 1) == L.MBG_ERR_INVALID_MODE


def test_cuda_failure_is_reported_not_silent():
    """Without a usable GPU a compute call must fail loudly (no CPU fallback)."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    a = np.ones((2, 2), np.float32, order="F")
    with pytest.raises(mb.MbgError):
        mb.gemm("N", "N", 2, 2, 2, 1.0, a, 2, a, 2, 0.0, a.copy(order="F"), 2)


@pytest.mark.parametrize("args,info", [
    (("X", "U", 2, 2, 1.0, Z, 2, Z, 2, 0.0, Z, 2), 1),
    (("L", "X", 2, 2, 1.0, Z, 2, Z, 2, 0.0, Z, 2), 2),
    (("L", "U", -1, 2, 1.0, Z, 2, Z, 2, 0.0, Z, 2), 3),
    (("L", "U", 2, -1, 1.0, Z, 2, Z, 2, 0.0, Z, 2), 4),
    (("L", "U", 3, 2, 1.0, Z, 2, Z, 3, 0.0, Z, 3), 7),
    (("R", "U", 2, 3, 1.0, Z, 2, Z, 2, 0.0, Z, 2), 7),
    (("L", "U", 3, 2, 1.0, Z, 3, Z, 2, 0.0, Z, 3), 9),
    (("L", "U", 3, 2, 1.0, Z, 3, Z, 3, 0.0, Z, 2), 12),
])
def test_symm_info_codes(args, info, capsys):
    """Numbering of mojoBLAS symm (src/level3/symm.mojo:69-86)."""
    assert mb.symm(*args) == info
    assert f"symm: Info {info}" in capsys.readouterr().out


@pytest.mark.parametrize("args,info", [
    (("X", "N", 2, 2, 1.0, Z, 2, Z, 2, 0.0, Z, 2), 1),
    (("U", "X", 2, 2, 1.0, Z, 2, Z, 2, 0.0, Z, 2), 2),
    (("U", "N", -1, 2, 1.0, Z, 2, Z, 2, 0.0, Z, 2), 3),
    (("U", "N", 2, -1, 1.0, Z, 2, Z, 2, 0.0, Z, 2), 4),
    (("U", "N", 3, 2, 1.0, Z, 2, Z, 3, 0.0, Z, 3), 7),
    (("U", "T", 2, 3, 1.0, Z, 2, Z, 3, 0.0, Z, 2), 7),
    (("U", "C", 2, 3, 1.0, Z, 3, Z, 2, 0.0, Z, 2), 9),
    (("U", "N", 3, 2, 1.0, Z, 3, Z, 3, 0.0, Z, 2), 12),
])
def test_syr2k_info_codes(args, info):
    """Numbering of mojoBLAS syr2k (src/level3/syr2k.mojo:69-93)."""
    assert mb.syr2k(*args) == info


@pytest.mark.parametrize("args,info", [
    (("X", "L", "N", "N", 2, 2, 1.0, Z, 2, Z, 2), 1),
    (("L", "X", "N", "N", 2, 2, 1.0, Z, 2, Z, 2), 2),
    (("L", "L", "X", "N", 2, 2, 1.0, Z, 2, Z, 2), 3),
    (("L", "L", "N", "X", 2, 2, 1.0, Z, 2, Z, 2), 4),
    (("L", "L", "N", "N", -1, 2, 1.0, Z, 2, Z, 2), 5),
    (("L", "L", "N", "N", 2, -1, 1.0, Z, 2, Z, 2), 6),
    (("L", "L", "N", "N", 3, 2, 1.0, Z, 2, Z, 3), 9),
    (("R", "L", "N", "N", 2, 3, 1.0, Z, 2, Z, 2), 9),
    (("L", "L", "N", "N", 3, 2, 1.0, Z, 3, Z, 2), 11),
])
def test_trmm_info_codes(args, info):
    """Numbering of mojoBLAS trmm (src/level3/trmm.mojo:63-89)."""
    assert mb.trmm(*args) == info


def test_neighbour_quick_returns_and_modes():
    # m == 0 / n == 0 / alpha == 0 and beta == 1 return before any CUDA call
    assert mb.symm("L", "U", 0, 3, 1.0, Z, 1, Z, 1, 0.0, Z, 1) == 0
    assert mb.symm("R", "L", 3, 3, 0.0, Z, 3, Z, 3, 1.0, Z, 3) == 0
    assert mb.syr2k("L", "N", 0, 3, 1.0, Z, 1, Z, 1, 0.0, Z, 1) == 0
    assert mb.syr2k("U", "T", 3, 3, 0.0, Z, 3, Z, 3, 1.0, Z, 3) == 0
    assert mb.trmm("L", "L", "N", "N", 0, 3, 1.0, Z, 1, Z, 1) == 0
    assert mb.trmm("R", "U", "T", "U", 3, 0, 1.0, Z, 1, Z, 3) == 0
    lib = L.load()
    p = Z.ctypes.data
    assert lib.mbg_ssymm_ex(L.MODE_OZAKI, b"L", b"U", 1, 1, 1.0, p, 1, p, 1, 0.0, p, 1) == L.MBG_ERR_INVALID_MODE
    assert lib.mbg_dsyr2k_ex(L.MODE_BF16X6, 8, b"L", b"N", 1, 1, 1.0, p, 1, p, 1, 0.0, p, 1) == \
        L.MBG_ERR_INVALID_MODE
    assert lib.mbg_dtrmm_ex(L.MODE_OZAKI, 1, b"L", b"L", b"N", b"N", 1, 1, 1.0, p, 1, p, 1) == \
        L.MBG_ERR_INVALID_MODE


@pytest.mark.parametrize("args,info", [
    (("n", 2, 2, 1.0, Z, 2, Z, 1, 0.0, Z, 1), 1),   # upper case only, as the reference checks it
    (("X", 2, 2, 1.0, Z, 2, Z, 1, 0.0, Z, 1), 1),
    (("N", -1, 2, 1.0, Z, 2, Z, 1, 0.0, Z, 1), 2),
    (("N", 2, -1, 1.0, Z, 2, Z, 1, 0.0, Z, 1), 3),
    (("T", 3, 2, 1.0, Z, 2, Z, 1, 0.0, Z, 1), 6),
    (("N", 2, 2, 1.0, Z, 2, Z, 0, 0.0, Z, 1), 8),
    (("C", 2, 2, 1.0, Z, 2, Z, 1, 0.0, Z, 0), 11),
])
def test_gemv_info_codes(args, info, capsys):
    """Numbering of mojoBLAS gemv (src/level2/gemv.mojo:69-84)."""
    assert mb.gemv(*args) == info
    assert f"gemv: Info {info}" in capsys.readouterr().out


@pytest.mark.parametrize("args,info", [
    (("X", "N", "N", 2, Z, 2, Z, 1), 1),
    (("U", "X", "N", 2, Z, 2, Z, 1), 2),
    (("U", "n", "X", 2, Z, 2, Z, 1), 3),
    (("U", "N", "N", -1, Z, 2, Z, 1), 4),
    (("l", "t", "u", 3, Z, 2, Z, 1), 6),
    (("U", "N", "N", 2, Z, 2, Z, 0), 8),
])
def test_trsv_info_codes(args, info):
    """Numbering of mojoBLAS trsv (src/level2/trsv.mojo:56-79)."""
    assert mb.trsv(*args) == info


def test_level2_quick_returns_touch_no_device():
    assert mb.gemv("N", 0, 3, 1.0, Z, 1, Z, 1, 0.0, Z, 1) == 0
    assert mb.gemv("T", 3, 0, 1.0, Z, 3, Z, 1, 0.0, Z, 1) == 0
    assert mb.gemv("N", 3, 3, 0.0, Z, 3, Z, 1, 1.0, Z, 1) == 0
    assert mb.trsv("L", "N", "N", 0, Z, 1, Z, 1) == 0


def test_noalloc_rejects_huge_dimensions_before_device_work():
    """Dimensions near INT64_MAX cannot wrap the no-allocation entry point's scratch
    size into a small number: they are rejected with MBG_ERR_SCRATCH_LIMIT before any
    pointer is inspected or any device work is queued (no GPU needed)."""
    lib = L.load()
    huge = (1 << 62) + 5
    for m, n, k in ((huge, 64, 64), (64, huge, 64), (64, 64, huge)):
        lda = m
        ldb = k
        st = lib.mbg_sgemm_ex_noalloc(L.MODE_BF16X6, b"N", b"N", m, n, k, 1.0, None, lda, None, ldb, 0.0, None, m)
        assert st == L.MBG_ERR_SCRATCH_LIMIT, (m, n, k, st)
        assert "scratch limit" in L.last_error()
