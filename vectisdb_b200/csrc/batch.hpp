// batch.hpp -- many group-by queries in one persistent launch.
//
// The batching form the engine adds beside one-query-per-launch: queries whose plans differ only
// in their numeric literals (the same template) share one NVRTC kernel that reads each query's
// constants, column pointers and key packing from a query table, and one persistent launch walks a
// (query, row tile) queue for all of them. The launch pair (aggregate, finalize) is captured in a
// CUDA graph and replayed while the batch's columns stay where they are. Tile geometry (block,
// items per thread, rows per tile, shared-table slots) comes from the autotuner.
#pragma once

#include <string>
#include <vector>

#include "executor.hpp"

namespace vgpu {

struct BatchOptions {
	int block = 0;      // 0 = autotuned / default
	int items = 0;
	int tile_rows = 0;
	int smem_slots = 0;
	bool use_graph = true;
	bool autotune = false;  // measure the candidate geometries now (else reuse a tuned entry or defaults)
};

struct BatchStats {
	uint64_t batched = 0;    // queries run by the batch kernel
	uint64_t fallback = 0;   // queries run one by one (shape outside the batch form)
	uint64_t templates = 0;  // distinct templates (one kernel each)
	uint64_t graph_replays = 0;
	int block = 0, items = 0, tile_rows = 0, smem_slots = 0;  // geometry of the last template
};

//! Plans converted, templated and signed once for repeated execution (a prepared batch).
struct PreparedPlan {
	std::shared_ptr<PlanNode> plan;
	const PlanNode *scan = nullptr;  // the SCAN leaf when the plan has the batch form
	std::shared_ptr<PlanNode> templ;
	std::vector<char> ptypes;
	std::vector<uint64_t> params;
	std::string sig_base;
};
struct PreparedBatch {
	std::vector<PreparedPlan> plans;
};
std::shared_ptr<PreparedBatch> PrepareBatch(const std::vector<std::shared_ptr<PlanNode>> &plans);
std::vector<ExecResult> ExecutePrepared(const PreparedBatch &batch, const std::vector<std::vector<vgpu_column>> &inputs,
                                        const ExecOptions &options, const BatchOptions &bopts, cudaStream_t stream,
                                        BatchStats *stats);

//! Executes every plan over its inputs; results in plan order. Queries of the form
//! GROUP_BY(keys) <- FILTER/PROJECTION* <- SCAN, with pass-through integer keys and no NULLs, run in
//! the batch kernel; any other plan runs through ExecutePlan. Throws Error on failure.
std::vector<ExecResult> ExecuteBatch(const std::vector<std::shared_ptr<PlanNode>> &plans,
                                     const std::vector<std::vector<vgpu_column>> &inputs, const ExecOptions &options,
                                     const BatchOptions &bopts, cudaStream_t stream, BatchStats *stats);

//! Numeric literals of an expression source replaced by typed reads of a per-query parameter
//! (vgpu_qpd / qpf / qpi / qpu / qpl / qpul (j)). Array indices of inputs[...] stay literal.
struct TemplatedSource {
	std::string text;
	std::vector<char> types;        // 'd' double, 'f' float, 'i' int, 'u' unsigned, 'l' long long, 'L' u64
	std::vector<uint64_t> values;   // bit patterns
};
TemplatedSource TemplateLiterals(const std::string &source, int first_index);

//! Drops every cached batch (graphs, query tables, accumulators) and the in-memory tuning table.
void ClearBatchCaches();

} // namespace vgpu
