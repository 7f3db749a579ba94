"""The committed known-answer fixtures are exactly what the committed generator
extracts from the reference's own tests (tests/test_level3.mojo,
tests/test_level2.mojo, tests/test_level2_extended.mojo).  Runs only where the
reference's source tree is present; elsewhere (a GPU host) the fixtures are used
as committed."""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

HERE = Path(__file__).parent / "golden"
REF = Path(os.environ.get("MOJOBLAS_REFERENCE", "/root/reference"))


@pytest.mark.skipif(not (REF / "tests" / "test_level3.mojo").exists(), reason="reference source tree absent")
def test_fixtures_regenerate_identically(tmp_path):
    script = tmp_path / "make_known_answers.py"
    script.write_text((HERE / "make_known_answers.py").read_text())
    subprocess.run([sys.executable, str(script), str(REF)], check=True, capture_output=True)
    for name in ("level3_known_answers.json", "level2_known_answers.json"):
        made = json.loads((tmp_path / name).read_text())
        committed = json.loads((HERE / name).read_text())
        assert made == committed, name
