// cost_model.hpp -- peak device bytes of one plan execution, re-derived from this engine's own
// allocation sites (the role of the reference's EstimateWorkingSet, cuda_engine/src/gpu_cost_model.cpp:78-147).
// Used by routing (headroom checks) and by the serving admission controller.
#pragma once

#include <string>
#include <vector>

#include "plan.hpp"

namespace vgpu {

//! Row counts and widths come from each SCAN's input (`scan_rows`, `scan_widths`, traversal order) when
//! given, else from the nodes' estimated_rows / estimated_row_width_bytes; a SCAN marked in
//! `scan_resident` (cache-served or device-memory inputs) is borrowed, not copied, and charges nothing.
//! A GROUP BY's estimated_rows is its group count. Chunk-capped when the plan is row-independent and
//! max_chunk_rows > 0.
vgpu_working_set EstimateWorkingSet(const PlanNode &plan, uint64_t max_chunk_rows,
                                    const std::vector<uint64_t> *scan_rows = nullptr,
                                    const std::vector<uint32_t> *scan_widths = nullptr,
                                    const std::vector<bool> *scan_resident = nullptr);

//! The estimate for one execution with its actual inputs and options: rows and widths from the
//! inputs (or the cached columns a cache-served scan reads), SCANs over cache-served or device-memory
//! columns charging nothing.
vgpu_working_set EstimateWorkingSetFor(const PlanNode &plan, const std::vector<vgpu_column> &inputs,
                                       bool serve_from_cache);

//! Work-to-data ratio of a plan from its advisory fields (the reference's AnalyzePlanShape,
//! cuda_engine/include/gpu_engine.hpp:284-329): the routing input of the extension's table checker.
vgpu_plan_shape AnalyzePlanShape(const PlanNode &plan);

//! Bytes of every SCAN's columns: estimated_rows x row width, width 0 counting as 8 bytes
//! (EstimateColumnsSize, gpu_engine.hpp:342).
uint64_t EstimateColumnsSize(const PlanNode &plan);

//! PIPELINE_STREAM_UNCACHED when the scanned columns exceed vram_budget x threshold and a budget is
//! given, else PIPELINE_STREAM_CACHED (DetermineExecutionMode, gpu_engine.hpp:344-348).
vgpu_execution_mode DetermineExecutionMode(const PlanNode &plan, uint64_t vram_budget, double threshold);

//! Generated source for the topmost pipeline of `plan` using only input descriptors (no device):
//! lets a host without a GPU check that every fused kernel compiles. Group keys are assumed to span
//! 16 bits each.
std::string GenerateSourceText(const PlanNode &plan, const std::vector<vgpu_column> &inputs);

} // namespace vgpu
