"""include/mojoblas_gpu.h is a C header: a C99 program that includes it compiles
with warnings as errors, links against the library and runs without a GPU
(version, status text, Netlib argument checks and quick returns, which touch no
device), as a C caller or an FFI stub generator would use it."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
LIB_DIR = ROOT / "mojoblas_b200"

PROGRAM = r"""
#include <stdio.h>
#include <string.h>
#include "mojoblas_gpu.h"

int main(void) {
    float a[4] = {0}, c[4] = {0};
    double d[4] = {0};
    if (mbg_version() < 100) return 1;
    if (strlen(mbg_status_string(0)) == 0) return 2;
    /* argument checks come before any device work: Netlib positions */
    if (mbg_sgemm('X', 'N', 2, 2, 2, 1.0f, a, 2, a, 2, 0.0f, c, 2) != 1) return 3;
    if (mbg_dgemm('N', 'N', 2, 2, 2, 1.0, d, 1, d, 2, 0.0, d, 2) != 8) return 4;
    if (mbg_ssyrk('L', 'N', 2, 2, 1.0f, a, 1, 0.0f, c, 2) != 7) return 5;
    if (mbg_dtrsm('L', 'L', 'N', 'Q', 2, 2, 1.0, d, 2, d, 2) != 4) return 6;
    if (mbg_strsv('U', 'N', 'N', 2, a, 2, c, 0) != 8) return 7;
    if (mbg_dgemv('n', 2, 2, 1.0, d, 2, d, 1, 0.0, d, 1) != 1) return 8;  /* upper case only */
    /* quick returns (m == 0, alpha == 0 with beta == 1) */
    if (mbg_sgemm('N', 'N', 0, 2, 2, 1.0f, a, 1, a, 2, 0.0f, c, 1) != 0) return 9;
    if (mbg_dsymm_ex(MBG_MODE_OZAKI, 7, 'L', 'U', 2, 0, 1.0, d, 2, d, 2, 0.0, d, 2) != 0) return 10;
    if (mbg_set_tuning("trsm_block_rows", 512) != 0 || mbg_get_tuning("trsm_block_rows") != 512) return 11;
    if (mbg_get_tuning("no_such_key") != -1) return 12;
    printf("ok\n");
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_header_compiles_as_c_and_links(tmp_path):
    if not (LIB_DIR / "libmojoblas_gpu.so").exists():
        pytest.skip("library not built")
    src = tmp_path / "abi.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "abi"
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", str(ROOT / "include"), str(src),
           "-L", str(LIB_DIR), "-lmojoblas_gpu", f"-Wl,-rpath,{LIB_DIR}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0 and run.stdout.strip() == "ok", (run.returncode, run.stdout, run.stderr)
