"""Generates tests/golden/solve_jl.json from the reference's own test file.

FixedEffects.jl's only numeric pins live in test/solve.jl: the 10-observation
input ``x``, the two fixed effects ``p1 = repeat(1:5, inner = 2)`` and
``p2 = repeat(1:5, outer = 2)``, the golden OLS residuals ``r_ols`` and the
interaction vector of the interacted-FE cases.  This script reads that file as
text (it runs no reference code), evaluates the few ``repeat(a:b, inner|outer
= n)`` expressions it contains, and writes the values as JSON.

Usage (in a checkout that has the reference project next to it):
    python tests/golden/make_golden.py /path/to/FixedEffects.jl
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

_NUM = r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?"


def _vector(src: str, name: str):
    m = re.search(rf"^\s*{name}\s*=\s*\[([^\]]*)\]", src, re.M)
    if not m:
        raise SystemExit(f"{name} not found")
    return [float(t) for t in re.findall(_NUM, m.group(1))]


def _repeat(src: str, name: str):
    m = re.search(rf"^\s*{name}\s*=\s*repeat\((\d+):(\d+),\s*(inner|outer)\s*=\s*(\d+)\)",
                  src, re.M)
    if not m:
        raise SystemExit(f"{name} not found")
    a, b, kind, n = int(m.group(1)), int(m.group(2)), m.group(3), int(m.group(4))
    base = list(range(a, b + 1))
    if kind == "inner":
        return [v for v in base for _ in range(n)]
    return base * n


def main(ref_root: str) -> None:
    solve = Path(ref_root) / "test" / "solve.jl"
    src = solve.read_text()
    out = {
        "source": "test/solve.jl (FixedEffects.jl v3.1.0)",
        "p1": _repeat(src, "p1"),
        "p2": _repeat(src, "p2"),
        "x": _vector(src, "x"),
        "r_ols": _vector(src, "r_ols"),
        "interaction": _vector(src, "interaction"),
        "weights_linear": list(range(1, 11)),
        "notes": {
            "x, p1, p2, r_ols": "test/solve.jl:3-7",
            "solve_coefficients! reproduces r_ols": "test/solve.jl:9-12",
            "solve_residuals! == r_ols (Vector/Pooled/Categorical)": "test/solve.jl:15-24",
            "Float32 on each backend == Float32.(r_ols)": "test/solve.jl:27-38",
            "length mismatch error": "test/solve.jl:41-42",
            "update_weights! round trip (unasserted upstream)": "test/solve.jl:45-55",
            "interacted FE converges": "test/solve.jl:57-61",
            "interacted + plain on same refs converges": "test/solve.jl:63-66",
        },
    }
    dst = Path(__file__).resolve().parent / "solve_jl.json"
    dst.write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {dst}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/FixedEffects.jl")
    main(sys.argv[1])
