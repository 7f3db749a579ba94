"""Generate tests/golden/level3_known_answers.json and level2_known_answers.json
from the reference's own tests.

The reference's level-3 tests (mojoBLAS tests/test_level3.mojo) hard-code tiny
column-major inputs and the expected outputs of gemm / syrk / trsm / trmm / symm /
syr2k; its level-2 tests (tests/test_level2.mojo, tests/test_level2_extended.mojo)
do the same for gemv and trsv, among others.  Mojo cannot run in this container,
so this script reads those files as text, replays each test's assignments and
records the call and its expected values.  The JSON it writes is committed;
nothing reads the reference at test time.

Run:  python tests/golden/make_known_answers.py path/to/mojoBLAS
(or set MOJOBLAS_REFERENCE to the mojoBLAS source tree and omit the argument)
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

ROUTINES = ("gemm", "syrk", "trsm", "trmm", "symm", "syr2k")
LEVEL2_ROUTINES = ("gemv", "trsv")


def _split_args(s: str) -> list[str]:
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "([":
            depth += 1
        elif ch in ")]":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur.strip())
    return out


def _eval(expr: str, env: dict):
    expr = expr.strip()
    m = re.fullmatch(r"(?:Float32|Float64|Scalar\[DType\.float(?:32|64)\])\((.*)\)", expr)
    if m:
        return float(_eval(m.group(1), env))
    if re.fullmatch(r'"[^"]*"', expr):
        return expr.strip('"')
    return eval(expr, {"__builtins__": {}, "max": max, "min": min}, env)  # ints / floats / names


def parse(path: Path, routines=ROUTINES) -> list[dict]:
    text = path.read_text()
    cases = []
    for fm in re.finditer(r"^def (test_\w+)\(\) raises:\n(.*?)(?=^def |\Z)", text, re.S | re.M):
        name, body = fm.group(1), fm.group(2)
        first = body.find("(")
        lines = [ln.split("#")[0].rstrip() for ln in body.splitlines()]
        env: dict = {}
        arrays: dict = {}
        dtype = None
        call = None
        asserts = []
        i = 0
        while i < len(lines):
            ln = lines[i].strip()
            i += 1
            if not ln:
                continue
            m = re.fullmatch(r"var (\w+) = alloc\[Scalar\[DType\.(float32|float64)\]\]\((.*)\)", ln)
            if m:
                arrays[m.group(1)] = [None] * int(_eval(m.group(3), env))
                dtype = m.group(2)
                continue
            m = re.fullmatch(r"var (\w+) = (.+)", ln)
            if m:
                env[m.group(1)] = _eval(m.group(2), env)
                continue
            m = re.fullmatch(r"for (\w+) in range\((.+)\):", ln)
            if m:
                body_ln = lines[i].strip()
                i += 1
                bm = re.fullmatch(r"(\w+)\[(\w+)\] = (.+)", body_ln)
                assert bm and bm.group(2) == m.group(1), (name, body_ln)
                for idx in range(int(_eval(m.group(2), env))):
                    arrays[bm.group(1)][idx] = float(_eval(bm.group(3), env))
                continue
            m = re.fullmatch(r"(\w+)\[(\d+)\] = (.+)", ln)
            if m and m.group(1) in arrays:
                arrays[m.group(1)][int(m.group(2))] = float(_eval(m.group(3), env))
                continue
            m = re.match(r"(%s)(\[DType\.(float32|float64)\])?\($" % "|".join(routines), ln) or \
                re.match(r"(%s)(\[DType\.(float32|float64)\])?\((.*)\)$" % "|".join(routines), ln)
            if m:
                routine = m.group(1)
                if ln.endswith("("):  # call spans lines
                    argtxt = ""
                    while not lines[i].strip().startswith(")"):
                        argtxt += lines[i].strip() + " "
                        i += 1
                    i += 1
                else:
                    argtxt = m.group(4)
                args = []
                for a in _split_args(argtxt):
                    if a in arrays:
                        args.append({"array": a})
                    else:
                        args.append(_eval(a, env))
                call = {"routine": routine, "args": args}
                if m.group(3):
                    dtype = m.group(3)
                continue
            m = re.fullmatch(r"assert_almost_equal\((\w+)\[(\d+)\], (Float32|Float64)\(([-\d.e]+)\)(?:, atol=([-\d.e]+))?\)", ln)
            if m:
                asserts.append({"array": m.group(1), "index": int(m.group(2)),
                                "expected": float(m.group(4)),
                                "atol": float(m.group(5)) if m.group(5) else None})
                continue
        if call is None:
            continue
        for k, v in arrays.items():
            arrays[k] = [0.0 if x is None else x for x in v]  # never read: unassigned entries
        cases.append({"test": name, "source_line": text[: fm.start()].count("\n") + 1,
                      "dtype": dtype, "call": call, "inputs": arrays, "asserts": asserts})
    return cases


def main() -> None:
    import os
    where = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MOJOBLAS_REFERENCE")
    if not where:
        sys.exit("usage: make_known_answers.py path/to/mojoBLAS (or set MOJOBLAS_REFERENCE)")
    root = Path(where)
    src = root / "tests" / "test_level3.mojo"
    cases = parse(src)
    out = {
        "source": "mojoBLAS tests/test_level3.mojo (known answers, column-major)",
        "default_float32_tolerance": "assert_almost_equal defaults: atol=1e-8, rtol=1e-5",
        "cases": cases,
    }
    dst = Path(__file__).with_name("level3_known_answers.json")
    dst.write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {len(cases)} cases to {dst}")
    cases2 = []
    for name in ("test_level2.mojo", "test_level2_extended.mojo"):
        for c in parse(root / "tests" / name, LEVEL2_ROUTINES):
            c["file"] = f"tests/{name}"
            cases2.append(c)
    out2 = {
        "source": "mojoBLAS tests/test_level2.mojo and tests/test_level2_extended.mojo (gemv / trsv known "
                  "answers, column-major)",
        "default_float32_tolerance": "assert_almost_equal defaults: atol=1e-8, rtol=1e-5",
        "cases": cases2,
    }
    dst2 = Path(__file__).with_name("level2_known_answers.json")
    dst2.write_text(json.dumps(out2, indent=1) + "\n")
    print(f"wrote {len(cases2)} cases to {dst2}")


if __name__ == "__main__":
    main()
