"""The engine (through the C ABI) reproduces every known answer of the reference engine's test suite,
re-expressed in tests/golden/ -- the same fixtures the oracle is pinned against."""
import pytest

from golden_util import check
from reference_cases import CASES

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(CASES))
def test_engine_matches_reference_known_answers(name, golden):
    from vectisdb_b200 import GpuEngine
    line, build = CASES[name]
    plan, inputs, _ = build()
    result = GpuEngine.instance().execute_plan(plan, inputs)
    mismatch = check(golden[name], result.success, result.error_message, result.columns)
    assert mismatch is None, f"{name} ({line}): {mismatch}"


def test_repeated_execution_hits_kernel_cache():
    """test_gpu_executor.cpp:421 -- the second identical run reuses the compiled module."""
    from vectisdb_b200 import GpuEngine
    from vectisdb_b200.engine import kernel_cache_stats
    _, build = CASES["repeated_execution_hits_kernel_cache"]
    plan, inputs, _ = build()
    GpuEngine.instance().execute_plan(plan, inputs)
    before = kernel_cache_stats()
    for _ in range(3):
        r = GpuEngine.instance().execute_plan(plan, inputs)
        assert r.success
    after = kernel_cache_stats()
    assert after.hits >= before.hits + 3
    assert after.compiles == before.compiles
