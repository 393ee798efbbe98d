"""Writes tests/golden/reference_cases.json from reference_cases.py.

    python tests/golden/make_golden.py

The expected rows are the reference test suite's own known answers: each case's `expected()` runs the
same CPU loops its test in cuda_engine/tests/test_gpu_executor.cpp (or test_gpu_filter.cu) uses to
build its expectation. Nothing here runs this engine or the oracle.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
sys.path.insert(0, str(HERE))

from golden_util import encode_expected  # noqa: E402
from reference_cases import CASES  # noqa: E402


def main() -> None:
    out = {}
    for name, (line, build) in CASES.items():
        _plan, _inputs, expected = build()
        fx = encode_expected(expected())
        fx["reference"] = line
        out[name] = fx
    path = HERE / "reference_cases.json"
    path.write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
    print(f"wrote {len(out)} cases to {path} ({path.stat().st_size} bytes)")


if __name__ == "__main__":
    main()
