"""The tuning table's file reader (mbg_load_tuning), on the CPU: the library loads
without a GPU and the table is host state.

* The shipped table (mojoblas_b200/tuning_b200.json) applies exactly its
  top-level keys; its nested measurements and device name are skipped.
* In a JSON object only top-level integer members are applied: string, boolean,
  non-integral and nested values are skipped wherever they stand, and a key
  name inside a nested object is not applied.
* Plain "key value" lines, with '#' comments; a value must be a whole integer.
* Unknown keys and out-of-range values are ignored; a file that applies nothing,
  or that cannot be opened, is an error.
"""
import json

import pytest

from mojoblas_b200 import _lib as L

KEYS = ("trsm_tc_min_k", "grouped_gemm_tile", "trsm_leaf_ctas", "trsm_block_rows", "trsm_block_min_cols",
        "plain_fp64_simt", "plain_fp32_staged")


@pytest.fixture
def lib():
    lib = L.load()
    saved = {k: lib.mbg_get_tuning(k.encode()) for k in KEYS}
    yield lib
    for k, v in saved.items():
        assert lib.mbg_set_tuning(k.encode(), v) == 0


def table(lib):
    return {k: lib.mbg_get_tuning(k.encode()) for k in KEYS}


def load(lib, path):
    return lib.mbg_load_tuning(str(path).encode())


def test_shipped_table(lib):
    shipped = json.loads(L.TUNING_PATH.read_text())
    top = {k: v for k, v in shipped.items() if k in KEYS}
    assert top and "_measurements" in shipped
    for k in top:  # move every key away from the file's value first
        lib.mbg_set_tuning(k.encode(), 128 if k == "grouped_gemm_tile" else 7)
    assert load(lib, L.TUNING_PATH) == 0
    got = table(lib)
    assert all(got[k] == v for k, v in top.items()), (got, top)


def test_json_skips_non_integer_and_nested_values(lib, tmp_path):
    f = tmp_path / "t.json"
    f.write_text(json.dumps({
        "_device": "NVIDIA B200",            # a string value before the keys
        "trsm_tc_min_k": 300,
        "_notes": {"trsm_block_rows": 128},  # a key name inside a nested object
        "trsm_block_min_cols": 2.5,          # not an integer
        "_list": [1, 2, {"trsm_leaf_ctas": 9}],
        "plain_fp64_simt": True,
        "trsm_leaf_ctas": 40,
        "unknown_key": 3,
        "grouped_gemm_tile": 96,             # out of range: ignored
    }, indent=1))
    lib.mbg_set_tuning(b"trsm_block_rows", 512)
    lib.mbg_set_tuning(b"trsm_block_min_cols", 64)
    lib.mbg_set_tuning(b"grouped_gemm_tile", 64)
    lib.mbg_set_tuning(b"plain_fp64_simt", 0)
    assert load(lib, f) == 0
    got = table(lib)
    assert got["trsm_tc_min_k"] == 300 and got["trsm_leaf_ctas"] == 40
    assert got["trsm_block_rows"] == 512 and got["trsm_block_min_cols"] == 64
    assert got["grouped_gemm_tile"] == 64 and got["plain_fp64_simt"] == 0


def test_plain_lines(lib, tmp_path):
    f = tmp_path / "t.txt"
    f.write_text("# autotuner output\ntrsm_block_rows 256   # fused blocks\n\ntrsm_tc_min_k 1024\n"
                 "trsm_block_min_cols 32abc\nplain_fp32_staged 1\n")
    lib.mbg_set_tuning(b"trsm_block_min_cols", 64)
    assert load(lib, f) == 0
    got = table(lib)
    assert got["trsm_block_rows"] == 256 and got["trsm_tc_min_k"] == 1024 and got["plain_fp32_staged"] == 1
    assert got["trsm_block_min_cols"] == 64  # "32abc" is not an integer


def test_errors(lib, tmp_path):
    assert load(lib, tmp_path / "missing.json") < 0
    assert "cannot open" in L.last_error()
    f = tmp_path / "none.json"
    f.write_text('{"unknown": 1, "trsm_block_rows": "512"}')
    before = table(lib)
    assert load(lib, f) < 0
    assert table(lib) == before
