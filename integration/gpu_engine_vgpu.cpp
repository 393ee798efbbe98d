// gpu_engine_vgpu.cpp -- the reference extension's engine interface over the vgpu C ABI.
//
// Compiled in place of the reference's cuda_engine/src/gpu_engine.cpp, gpu_cost_model.cpp and
// gpu_column_cache.cpp, against the reference's UNCHANGED headers (cuda_engine/include/gpu_engine.hpp,
// gpu_column_cache.hpp) and this repository's include/vgpu.h, and linked with libvgpu.so instead of
// the cuda_engine target, it gives the DuckDB extension (extension/src/physical_gpu_execute.cpp:245-274,
// table_checker.cpp:449-499, the optimizer hook gpu_offload_extension.cpp:1415-1443) this engine with no
// change on its side:
//
//   g++ -std=c++17 -c -I<reference>/cuda_engine/include -Iinclude -I<cuda>/include gpu_engine_vgpu.cpp
//
// Every call flattens the reference's GpuPlanNode tree into the ABI's node array (the enums have the same
// order on both sides), calls the C function, and maps the status back to the reference's contract:
// ExecutePlan never throws and reports refusals as success=false with the engine's message, which the
// extension turns into a CPU fallback.
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "gpu_column_cache.hpp"  // the reference's headers, unchanged
#include "gpu_engine.hpp"
#include "vgpu.h"

namespace vector_gpu {

namespace {

//! Owns the flattened form of one plan for the duration of one call.
struct Flat {
	std::vector<vgpu_plan_node> nodes;
	std::vector<std::vector<uint32_t>> kids;
	std::vector<std::vector<const char *>> names;
	std::vector<std::vector<vgpu_expr>> exprs;
	std::vector<std::vector<vgpu_aggregate>> aggs;
	vgpu_plan plan {};

	const char *const *Names(const std::vector<std::string> &v) {
		names.emplace_back();
		for (auto &s : v) names.back().push_back(s.c_str());
		return names.back().data();
	}
	uint32_t Add(const GpuPlanNode &n) {
		const uint32_t id = static_cast<uint32_t>(nodes.size());
		nodes.emplace_back();
		std::vector<uint32_t> children;
		for (auto &c : n.children) children.push_back(Add(*c));
		kids.push_back(children);
		vgpu_plan_node &o = nodes[id];
		o = {};
		o.op = static_cast<uint32_t>(n.op_type);
		o.n_children = static_cast<uint32_t>(children.size());
		o.children = kids.back().data();
		o.catalog = n.table.catalog.c_str();
		o.schema = n.table.schema.c_str();
		o.table = n.table.table.c_str();
		o.column_names = Names(n.column_names);
		o.n_column_names = static_cast<uint32_t>(n.column_names.size());
		exprs.emplace_back();
		for (auto &e : n.expressions) {
			exprs.back().push_back({e.generated_cuda_source.c_str(), Names(e.input_columns),
			                        static_cast<uint32_t>(e.input_columns.size()), static_cast<uint32_t>(e.output_type),
			                        static_cast<uint32_t>(e.window_primitive), e.estimated_ops_per_row});
		}
		o.expressions = exprs.back().data();
		o.n_expressions = static_cast<uint32_t>(n.expressions.size());
		o.build_keys = Names(n.build_keys);
		o.n_build_keys = static_cast<uint32_t>(n.build_keys.size());
		o.probe_keys = Names(n.probe_keys);
		o.n_probe_keys = static_cast<uint32_t>(n.probe_keys.size());
		o.output_columns = Names(n.output_columns);
		o.n_output_columns = static_cast<uint32_t>(n.output_columns.size());
		o.group_keys = Names(n.group_keys);
		o.n_group_keys = static_cast<uint32_t>(n.group_keys.size());
		aggs.emplace_back();
		for (auto &a : n.aggregates) {
			aggs.back().push_back({static_cast<uint32_t>(a.kind), static_cast<uint32_t>(a.output_type),
			                       a.input_column.c_str()});
		}
		o.aggregates = aggs.back().data();
		o.n_aggregates = static_cast<uint32_t>(n.aggregates.size());
		o.estimated_rows = n.estimated_rows;
		o.estimated_row_width_bytes = n.estimated_row_width_bytes;
		o.aggregate_exprs = Names(n.aggregate_exprs);
		o.n_aggregate_exprs = static_cast<uint32_t>(n.aggregate_exprs.size());
		return id;
	}
	//! The ABI plan; the vectors are filled before their data is taken (Add may reallocate them).
	const vgpu_plan *Of(const GpuPlanNode &root) {
		nodes.reserve(64);
		kids.reserve(64);
		names.reserve(512);
		exprs.reserve(64);
		aggs.reserve(64);
		const uint32_t r = Add(root);
		plan.nodes = nodes.data();
		plan.n_nodes = static_cast<uint32_t>(nodes.size());
		plan.root = r;
		return &plan;
	}
};

size_t ValueWidth(uint32_t type) {
	switch (type) {
	case VGPU_HUGEINT:
		return 16;
	case VGPU_INT64:
	case VGPU_FLOAT64:
		return 8;
	case VGPU_INT16:
		return 2;
	case VGPU_BOOLEAN:
		return 1;
	default:
		return 4;
	}
}

vgpu_table_ref Ref(const GpuTableRef &t) {
	return {t.catalog.c_str(), t.schema.c_str(), t.table.c_str()};
}

} // namespace

// ---- GpuEngine (cuda_engine/include/gpu_engine.hpp:389-402) -----------------------------------------

GpuEngine &GpuEngine::Instance() {
	static GpuEngine engine;
	return engine;
}

GpuExecutionResult GpuEngine::ExecutePlan(const GpuPlanNode &plan, const std::vector<GpuColumn> &inputs,
                                          const GpuExecuteOptions &options) {
	GpuExecutionResult result;
	Flat flat;
	const vgpu_plan *p = flat.Of(plan);
	std::vector<vgpu_column> in;
	in.reserve(inputs.size());
	for (auto &c : inputs) {
		in.push_back({c.name.c_str(), static_cast<uint32_t>(c.type), VGPU_MEM_HOST, c.data, c.validity, c.row_count});
	}
	vgpu_exec_options o;
	vgpu_exec_options_init(&o);
	o.stage_scan_to_cache = options.stage_scan_to_cache ? 1 : 0;
	o.serve_whole_scan_from_cache = options.serve_whole_scan_from_cache ? 1 : 0;
	o.cache_chunk_index = options.cache_chunk_index;
	vgpu_result *r = nullptr;
	if (vgpu_execute_plan(p, in.data(), in.size(), &o, &r) != VGPU_OK) {
		result.success = false;
		result.error_message = vgpu_last_error();  // the caller falls back to DuckDB's CPU path
		return result;
	}
	const size_t n = vgpu_result_column_count(r);
	result.owned_buffers.reserve(2 * n);  // column pointers below point into these buffers
	for (size_t i = 0; i < n; i++) {
		vgpu_column c;
		vgpu_result_get_column(r, i, &c);
		const auto *bytes = static_cast<const uint8_t *>(c.data);
		result.owned_buffers.emplace_back(bytes, bytes + c.row_count * ValueWidth(c.type));
		GpuColumn col;
		col.name = c.name;
		col.type = static_cast<GpuValueType>(c.type);
		col.data = result.owned_buffers.back().data();
		col.row_count = c.row_count;
		if (c.validity != nullptr) {
			result.owned_buffers.emplace_back(c.validity, c.validity + (c.row_count + 7) / 8);
			col.validity = result.owned_buffers.back().data();
		}
		result.columns.push_back(std::move(col));
	}
	vgpu_result_free(r);
	result.success = true;
	return result;
}

// ---- Cost model and routing helpers (gpu_engine.hpp:241-348) -----------------------------------------

bool IsRowIndependent(const GpuPlanNode &node) {
	Flat flat;
	return vgpu_is_row_independent(flat.Of(node)) != 0;
}

GpuWorkingSetEstimate EstimateWorkingSet(const GpuPlanNode &plan, uint64_t max_chunk_rows) {
	thread_local std::string largest;  // the reference's field is a C string the caller does not own
	Flat flat;
	vgpu_working_set w {};
	GpuWorkingSetEstimate out;
	if (vgpu_estimate_working_set(flat.Of(plan), max_chunk_rows, &w) != VGPU_OK) {
		out.total_bytes = UINT64_MAX;  // a plan the estimator rejects reads as "does not fit"
		out.largest_operator = "INVALID";
		return out;
	}
	largest.assign(w.largest_operator, strnlen(w.largest_operator, sizeof(w.largest_operator)));
	out.total_bytes = w.total_bytes;
	out.chunk_capped = w.chunk_capped != 0;
	out.largest_operator = largest.c_str();
	out.largest_bytes = w.largest_bytes;
	return out;
}

GpuPlanShape AnalyzePlanShape(const GpuPlanNode &plan) {
	Flat flat;
	vgpu_plan_shape s {};
	vgpu_analyze_plan_shape(flat.Of(plan), &s);  // fails only on a malformed plan: s stays zero
	GpuPlanShape out;
	out.scanned_rows = s.scanned_rows;
	out.scanned_bytes = s.scanned_bytes;
	out.max_rows = s.max_rows;
	out.total_ops = s.total_ops;
	out.ops_per_scanned_row = s.ops_per_scanned_row;
	out.ops_per_scanned_byte = s.ops_per_scanned_byte;
	out.amplification = s.amplification;
	out.density = static_cast<GpuWorkDensity>(s.density);
	return out;
}

uint64_t EstimateColumnsSize(const GpuPlanNode &plan) {
	Flat flat;
	uint64_t bytes = 0;
	vgpu_estimate_columns_size(flat.Of(plan), &bytes);
	return bytes;
}

ExecutionMode DetermineExecutionMode(const GpuPlanNode &plan, uint64_t vram_budget, double threshold) {
	Flat flat;
	uint32_t mode = VGPU_MODE_PIPELINE_STREAM_CACHED;
	vgpu_determine_execution_mode(flat.Of(plan), vram_budget, threshold, &mode, nullptr);
	return static_cast<ExecutionMode>(mode);
}

// ---- GpuColumnCache (cuda_engine/include/gpu_column_cache.hpp:107-196) --------------------------------
// The engine keeps the cache; this class forwards to it. A staged chunk's device buffers pass to the
// cache's ownership in the reference, so they are freed here once the engine has copied them.

GpuColumnCache::GpuColumnCache() = default;

GpuColumnCache &GpuColumnCache::Instance() {
	static GpuColumnCache cache;
	return cache;
}

void GpuColumnCache::EnsureInitialized(double fraction_of_vram) {
	vgpu_cache_init(fraction_of_vram);
}

void GpuColumnCache::BeginStaging(const GpuTableRef &table) {
	const vgpu_table_ref t = Ref(table);
	vgpu_cache_begin_staging(&t);
}

bool GpuColumnCache::StageChunk(const GpuTableRef &table, const std::string &column_name,
                                const GpuColumnChunk &chunk) {
	const vgpu_table_ref t = Ref(table);
	std::vector<uint8_t> bitmap;
	if (chunk.device_validity != nullptr && chunk.row_count > 0) {
		// the engine takes validity as an Arrow bitmap: pack the chunk's byte-per-row flags on the host
		std::vector<uint8_t> bytes(chunk.row_count);
		cudaMemcpy(bytes.data(), chunk.device_validity, chunk.row_count, cudaMemcpyDeviceToHost);
		bitmap.assign((chunk.row_count + 7) / 8, 0);
		for (uint64_t i = 0; i < chunk.row_count; i++) bitmap[i / 8] |= static_cast<uint8_t>((bytes[i] != 0) << (i % 8));
	}
	std::vector<uint8_t> host(chunk.data_bytes);
	if (chunk.data_bytes) cudaMemcpy(host.data(), chunk.device_data, chunk.data_bytes, cudaMemcpyDeviceToHost);
	const vgpu_column c {column_name.c_str(), static_cast<uint32_t>(chunk.type), VGPU_MEM_HOST, host.data(),
	                     bitmap.empty() ? nullptr : bitmap.data(), chunk.row_count};
	int accepted = 0;
	const bool ok = vgpu_cache_stage_chunk(&t, &c, &accepted) == VGPU_OK && accepted != 0;
	cudaFree(chunk.device_data);  // ownership passed with the call, whatever its outcome
	if (chunk.device_validity != nullptr) cudaFree(chunk.device_validity);
	return ok;
}

void GpuColumnCache::CommitStaging(const GpuTableRef &table, uint64_t scanned_rows) {
	const vgpu_table_ref t = Ref(table);
	vgpu_cache_commit_staging(&t, scanned_rows);
}

void GpuColumnCache::AbortStaging(const GpuTableRef &table) {
	const vgpu_table_ref t = Ref(table);
	vgpu_cache_abort_staging(&t);
}

std::vector<uint64_t> GpuColumnCache::ReplayableChunkRows(const GpuTableRef &table,
                                                          const std::vector<std::string> &column_names) {
	const vgpu_table_ref t = Ref(table);
	std::vector<const char *> names;
	for (auto &n : column_names) names.push_back(n.c_str());
	std::vector<uint64_t> rows(4096);
	size_t count = 0;
	if (vgpu_cache_replayable_chunk_rows(&t, names.data(), names.size(), rows.data(), rows.size(), &count) != VGPU_OK) {
		return {};
	}
	rows.resize(count < rows.size() ? count : rows.size());
	return rows;
}

bool GpuColumnCache::TryGetChunk(const GpuTableRef &table, const std::string &column_name, uint64_t chunk_index,
                                 GpuColumnChunk &out_chunk) {
	const vgpu_table_ref t = Ref(table);
	vgpu_column c {};
	int found = 0;
	if (vgpu_cache_try_get_chunk(&t, column_name.c_str(), chunk_index, &c, &found) != VGPU_OK || !found) return false;
	out_chunk.device_data = const_cast<void *>(c.data);  // a borrow, as in the reference
	out_chunk.device_validity = nullptr;
	out_chunk.row_count = c.row_count;
	out_chunk.data_bytes = c.row_count * ValueWidth(c.type);
	out_chunk.validity_bytes = 0;
	out_chunk.type = static_cast<GpuValueType>(c.type);
	return true;
}

void GpuColumnCache::InvalidateTable(const GpuTableRef &table) {
	const vgpu_table_ref t = Ref(table);
	vgpu_cache_invalidate_table(&t);
}

void GpuColumnCache::InvalidateAll() {
	vgpu_cache_invalidate_all();
}

uint64_t GpuColumnCache::CurrentBytes() const {
	return vgpu_cache_current_bytes();
}

uint64_t GpuColumnCache::TableGeneration(const GpuTableRef &table) const {
	const vgpu_table_ref t = Ref(table);
	return vgpu_cache_table_generation(&t);
}

} // namespace vector_gpu
