// cost_model.hpp -- peak device bytes of one plan execution, re-derived from this engine's own
// allocation sites (the role of the reference's EstimateWorkingSet, cuda_engine/src/gpu_cost_model.cpp:78-147).
// Used by routing (headroom checks) and by the serving admission controller.
#pragma once

#include <string>
#include <vector>

#include "plan.hpp"

namespace vgpu {

//! Row counts come from each SCAN's input (`scan_rows`, traversal order) when given, else from the
//! nodes' estimated_rows. Chunk-capped when the plan is row-independent and max_chunk_rows > 0.
vgpu_working_set EstimateWorkingSet(const PlanNode &plan, uint64_t max_chunk_rows,
                                    const std::vector<uint64_t> *scan_rows = nullptr,
                                    const std::vector<uint32_t> *scan_widths = nullptr);

//! Generated source for the topmost pipeline of `plan` using only input descriptors (no device):
//! lets a host without a GPU check that every fused kernel compiles. Group keys are assumed to span
//! 16 bits each.
std::string GenerateSourceText(const PlanNode &plan, const std::vector<vgpu_column> &inputs);

} // namespace vgpu
