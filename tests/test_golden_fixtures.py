"""The committed known-answer fixtures are exactly what the committed generator
extracts from the reference's own tests (tests/test_level3.mojo,
tests/test_level2.mojo, tests/test_level2_extended.mojo).  Runs only when the
environment variable MOJOBLAS_REFERENCE names the reference's source tree;
elsewhere (a GPU host) the fixtures are used as committed."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

HERE = Path(__file__).parent / "golden"
REF = Path(os.environ["MOJOBLAS_REFERENCE"]) if os.environ.get("MOJOBLAS_REFERENCE") else None


@pytest.mark.skipif(REF is None or not (REF / "tests" / "test_level3.mojo").exists(),
                    reason="MOJOBLAS_REFERENCE does not name the reference's source tree")
def test_fixtures_regenerate_identically(tmp_path):
    script = tmp_path / "make_known_answers.py"
    script.write_text((HERE / "make_known_answers.py").read_text())
    subprocess.run([sys.executable, str(script), str(REF)], check=True, capture_output=True)
    for name in ("level3_known_answers.json", "level2_known_answers.json"):
        made = json.loads((tmp_path / name).read_text())
        committed = json.loads((HERE / name).read_text())
        assert made == committed, name
