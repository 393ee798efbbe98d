"""The C++ shim that binds the reference's DuckDB extension to this engine (integration/gpu_engine_vgpu.cpp)
compiles against the reference's unchanged engine headers and include/vgpu.h: every declaration it
defines (GpuEngine::ExecutePlan, the cost-model and routing helpers, GpuColumnCache) matches the
reference's signatures. Skipped where the reference's sources are not on disk."""
import os
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
REFERENCE = Path(os.environ.get("VGPU_REFERENCE_ROOT", "/root/reference"))
HEADERS = REFERENCE / "cuda_engine" / "include"
CUDA_INCLUDE = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "include"


@pytest.mark.skipif(not (HEADERS / "gpu_engine.hpp").exists(), reason="reference engine headers not present")
@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not installed")
def test_shim_compiles_against_the_reference_headers():
    r = subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-Wall", "-Werror", f"-I{HEADERS}",
                        f"-I{ROOT / 'include'}", f"-I{CUDA_INCLUDE}", str(ROOT / "integration" / "gpu_engine_vgpu.cpp")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_shim_defines_every_entry_point_the_extension_calls():
    src = (ROOT / "integration" / "gpu_engine_vgpu.cpp").read_text()
    for decl in ("GpuEngine::ExecutePlan", "GpuEngine::Instance", "bool IsRowIndependent(",
                 "GpuWorkingSetEstimate EstimateWorkingSet(", "GpuPlanShape AnalyzePlanShape(",
                 "uint64_t EstimateColumnsSize(", "ExecutionMode DetermineExecutionMode(",
                 "GpuColumnCache::BeginStaging", "GpuColumnCache::StageChunk", "GpuColumnCache::CommitStaging",
                 "GpuColumnCache::AbortStaging", "GpuColumnCache::ReplayableChunkRows", "GpuColumnCache::TryGetChunk",
                 "GpuColumnCache::InvalidateTable", "GpuColumnCache::InvalidateAll", "GpuColumnCache::CurrentBytes",
                 "GpuColumnCache::TableGeneration"):
        assert decl in src, decl
