// executor.hpp -- runs a plan on the device: the role of the reference's ExecuteGpuPlan /
// ExecuteNode (cuda_engine/src/gpu_executor.cu:748-966), re-designed around fused NVRTC pipelines.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "codegen.hpp"
#include "plan.hpp"
#include "runtime.hpp"

namespace vgpu {

//! A device column. `valid` is a byte-per-row null mask (nullptr = no NULLs). Buffers are owned by the
//! execution's arena unless borrowed (caller inputs, cache entries).
struct DevColumn {
	std::string name;
	ValueType type = ValueType::INT32;
	uint64_t rows = 0;
	void *data = nullptr;
	uint8_t *valid = nullptr;
	bool has_stats = false;
	int64_t min = 0, max = 0;
};
using Relation = std::vector<DevColumn>;

struct HostColumnOut {
	std::string name;
	ValueType type;
	uint64_t rows = 0;
	std::vector<uint8_t> data;
	std::shared_ptr<uint8_t> host;  // page-locked copy of the values (used instead of `data` when set)
	std::vector<uint8_t> validity; // empty = all valid
	void *device_data = nullptr;   // set when the result stays on the device
	uint8_t *device_validity = nullptr;
};

struct ExecOptions {
	bool stage_scan_to_cache = false;
	bool serve_whole_scan_from_cache = false;
	int64_t cache_chunk_index = -1;
	bool output_on_device = false;
	bool no_sync = false;
};

struct ExecResult {
	std::vector<HostColumnOut> columns;
	std::vector<void *> device_buffers; // owned device memory (device output mode)
	std::vector<std::shared_ptr<void>> keepalive; // device memory shared with other results (batches)
	cudaStream_t stream = nullptr;
	// Device u64 with the row count of every column, not read yet (device output without a sync): the
	// columns' `rows` are their capacity until it is. It is also listed in device_buffers.
	void *pending_rows = nullptr;
	int pending_rows_bytes = 8;  // its width: 8 (u64) or 4 (u32)
};

//! Validates a GROUP_BY_AGGREGATE node against its input pipeline and returns its aggregate spec;
//! `key_cols` receives the visible column of each group key. Throws Error(VGPU_ERR_UNSUPPORTED /
//! INVALID_ARGUMENT) for what this GPU path does not model.
PipelineCodegen::GroupBySpec ValidateGroupBy(const PlanNode &node, const PipelineCodegen &cg, std::vector<int> &key_cols);

//! Drops every dense join table kept across executions (their memory is freed once no execution holds
//! it). Called when cached base columns are invalidated.
void ClearJoinTables();

//! Executes `plan` over `inputs`. Throws Error on any failure (nothing partial escapes).
ExecResult ExecutePlan(const PlanNode &plan, const std::vector<vgpu_column> &inputs, const ExecOptions &options,
                       cudaStream_t stream);

} // namespace vgpu
