"""The plan oracle reproduces every known answer of the reference engine's test suite
(cuda_engine/tests/test_gpu_executor.cpp, test_gpu_filter.cu), re-expressed in tests/golden/."""
import pytest

from golden_util import check
from reference_cases import CASES
from oracle.plan_oracle import OracleRefusal, evaluate


@pytest.mark.parametrize("name", sorted(CASES))
def test_plan_oracle_matches_reference_known_answers(name, golden):
    line, build = CASES[name]
    plan, inputs, _ = build()
    try:
        cols = evaluate(plan, inputs)
        success, error = True, ""
    except OracleRefusal as e:
        cols, success, error = [], False, str(e)

    class _C:
        def __init__(self, c):
            self.data = c.data
            self.validity = c.valid
    mismatch = check(golden[name], success, error, [_C(c) for c in cols])
    assert mismatch is None, f"{name} ({line}): {mismatch}"
