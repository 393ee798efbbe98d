// abi.cpp -- the extern "C" boundary (include/vgpu.h). Every entry point catches everything: no C++
// exception and no process abort ever crosses into the caller; failures become a status code plus a
// thread-local message (the reference's success=false + error_message contract,
// cuda_engine/src/gpu_engine.cpp:41-52).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "column_cache.hpp"
#include "cost_model.hpp"
#include "translator.hpp"
#include "batch.hpp"
#include "server.hpp"
#include "stream_pipeline.hpp"
#include "executor.hpp"
#include "plan.hpp"
#include "runtime.hpp"
#include "shard.hpp"

namespace vgpu {
std::string Sha256Hex(const void *data, size_t n);
}

using namespace vgpu;

struct vgpu_result {
	ExecResult exec;
	std::vector<std::string> names;
	std::mutex rows_mu;  // guards the first read of a row count left on the device
};

namespace {

thread_local std::string g_last_error;

template <typename F> vgpu_status Guard(F &&f) {
	try {
		g_last_error.clear();
		f();
		return VGPU_OK;
	} catch (const Error &e) {
		g_last_error = e.what();
		return e.status();
	} catch (const std::bad_alloc &) {
		g_last_error = "host allocation failed";
		return VGPU_ERR_OUT_OF_MEMORY;
	} catch (const std::exception &e) {
		g_last_error = e.what();
		return VGPU_ERR_INTERNAL;
	} catch (...) {
		g_last_error = "unknown internal error";
		return VGPU_ERR_INTERNAL;
	}
}

} // namespace

namespace vgpu {
void SetLastError(const std::string &message) {
	g_last_error = message;
}
} // namespace vgpu

namespace {

TableRef ToTable(const vgpu_table_ref *t) {
	if (t == nullptr) Fail(VGPU_ERR_INVALID_ARGUMENT, "null table reference");
	return TableRef {t->catalog ? t->catalog : "", t->schema ? t->schema : "", t->table ? t->table : ""};
}

} // namespace

extern "C" {

int vgpu_abi_version(void) {
	return VGPU_ABI_VERSION;
}

const char *vgpu_last_error(void) {
	return g_last_error.c_str();
}

const char *vgpu_status_string(vgpu_status status) {
	switch (status) {
	case VGPU_OK:
		return "OK";
	case VGPU_ERR_INVALID_ARGUMENT:
		return "INVALID_ARGUMENT";
	case VGPU_ERR_UNSUPPORTED:
		return "UNSUPPORTED";
	case VGPU_ERR_CUDA:
		return "CUDA";
	case VGPU_ERR_OUT_OF_MEMORY:
		return "OUT_OF_MEMORY";
	case VGPU_ERR_COMPILE:
		return "COMPILE";
	case VGPU_ERR_NOT_READY:
		return "NOT_READY";
	case VGPU_ERR_TIMEOUT:
		return "TIMEOUT";
	case VGPU_ERR_REJECTED:
		return "REJECTED";
	case VGPU_ERR_INTERNAL:
		return "INTERNAL";
	}
	return "UNKNOWN";
}

void vgpu_exec_options_init(vgpu_exec_options *o) {
	if (!o) return;
	std::memset(o, 0, sizeof(*o));
	o->cache_chunk_index = -1;
	o->output_memory = VGPU_MEM_HOST;
}

vgpu_status vgpu_execute_plan(const vgpu_plan *plan, const vgpu_column *inputs, size_t n_inputs,
                              const vgpu_exec_options *options, vgpu_result **out) {
	return Guard([&] {
		if (out == nullptr) Fail(VGPU_ERR_INVALID_ARGUMENT, "null result pointer");
		*out = nullptr;
		if (n_inputs > 0 && inputs == nullptr) Fail(VGPU_ERR_INVALID_ARGUMENT, "null inputs with nonzero count");
		auto root = ConvertPlan(plan);
		RefuseWindowPrimitives(*root);  // before anything touches the device
		ExecOptions eo;
		cudaStream_t stream = nullptr;
		if (options) {
			eo.stage_scan_to_cache = options->stage_scan_to_cache != 0;
			eo.serve_whole_scan_from_cache = options->serve_whole_scan_from_cache != 0;
			eo.cache_chunk_index = options->cache_chunk_index;
			eo.output_on_device = options->output_memory == VGPU_MEM_DEVICE;
			eo.no_sync = (options->flags & VGPU_EXEC_NO_SYNC) != 0;
			stream = static_cast<cudaStream_t>(options->stream);
			if (eo.serve_whole_scan_from_cache && eo.cache_chunk_index >= 0) {
				Fail(VGPU_ERR_INVALID_ARGUMENT, "serve_whole_scan_from_cache and cache_chunk_index are exclusive");
			}
			if (eo.stage_scan_to_cache) {
				Fail(VGPU_ERR_UNSUPPORTED, "stage_scan_to_cache: stage columns with vgpu_cache_stage_chunk");
			}
		}
		if (stream == nullptr) stream = Runtime::Get().default_stream();
		std::vector<vgpu_column> in(inputs, inputs + n_inputs);
		auto *r = new vgpu_result();
		try {
			r->exec = ExecutePlan(*root, in, eo, stream);
		} catch (...) {
			delete r;
			throw;
		}
		*out = r;
	});
}

void vgpu_batch_options_init(vgpu_batch_options *options) {
	if (!options) return;
	std::memset(options, 0, sizeof(*options));
	options->use_graph = 1;
}

struct vgpu_batch {
	std::shared_ptr<PreparedBatch> prepared;
};

namespace {

void RunPreparedBatch(const PreparedBatch &pb, const vgpu_column *const *inputs, const size_t *n_inputs,
                      const vgpu_exec_options *options, const vgpu_batch_options *batch_options,
                      vgpu_result **results, vgpu_batch_stats *stats) {
	const size_t n_plans = pb.plans.size();
	if (n_plans > 0 && results == nullptr) Fail(VGPU_ERR_INVALID_ARGUMENT, "null results");
	for (size_t i = 0; i < n_plans; i++) results[i] = nullptr;
	std::vector<std::vector<vgpu_column>> ins(n_plans);
	for (size_t i = 0; i < n_plans; i++) {
		const size_t k = n_inputs ? n_inputs[i] : 0;
		if (k > 0 && (inputs == nullptr || inputs[i] == nullptr)) Fail(VGPU_ERR_INVALID_ARGUMENT, "null inputs with nonzero count");
		if (k > 0) ins[i].assign(inputs[i], inputs[i] + k);
	}
	ExecOptions eo;
	cudaStream_t stream = nullptr;
	if (options) {
		eo.serve_whole_scan_from_cache = options->serve_whole_scan_from_cache != 0;
		eo.cache_chunk_index = options->cache_chunk_index;
		eo.stage_scan_to_cache = options->stage_scan_to_cache != 0;
		eo.output_on_device = options->output_memory == VGPU_MEM_DEVICE;
		stream = static_cast<cudaStream_t>(options->stream);
	}
	if (stream == nullptr) stream = Runtime::Get().default_stream();
	BatchOptions bo;
	if (batch_options) {
		bo.block = batch_options->block;
		bo.items = batch_options->items;
		bo.tile_rows = batch_options->tile_rows;
		bo.smem_slots = batch_options->smem_slots;
		bo.use_graph = batch_options->use_graph != 0;
		bo.autotune = batch_options->autotune != 0;
	}
	BatchStats st;
	auto out = ExecutePrepared(pb, ins, eo, bo, stream, &st);
	for (size_t i = 0; i < n_plans; i++) {
		auto *r = new vgpu_result();
		r->exec = std::move(out[i]);
		results[i] = r;
	}
	if (stats) {
		stats->batched = st.batched;
		stats->fallback = st.fallback;
		stats->templates = st.templates;
		stats->graph_replays = st.graph_replays;
		stats->block = st.block;
		stats->items = st.items;
		stats->tile_rows = st.tile_rows;
		stats->smem_slots = st.smem_slots;
	}
}

std::shared_ptr<PreparedBatch> PrepareFromAbi(const vgpu_plan *const *plans, size_t n_plans) {
	if (n_plans > 0 && plans == nullptr) Fail(VGPU_ERR_INVALID_ARGUMENT, "null plans");
	std::vector<std::shared_ptr<PlanNode>> roots;
	for (size_t i = 0; i < n_plans; i++) roots.push_back(ConvertPlan(plans[i]));
	return PrepareBatch(roots);
}

} // namespace

vgpu_status vgpu_batch_prepare(const vgpu_plan *const *plans, size_t n_plans, vgpu_batch **out) {
	return Guard([&] {
		if (!out) Fail(VGPU_ERR_INVALID_ARGUMENT, "null batch pointer");
		*out = nullptr;
		auto *b = new vgpu_batch();
		try {
			b->prepared = PrepareFromAbi(plans, n_plans);
		} catch (...) {
			delete b;
			throw;
		}
		*out = b;
	});
}

size_t vgpu_batch_size(const vgpu_batch *batch) {
	return batch && batch->prepared ? batch->prepared->plans.size() : 0;
}

vgpu_status vgpu_batch_execute(vgpu_batch *batch, const vgpu_column *const *inputs, const size_t *n_inputs,
                               const vgpu_exec_options *options, const vgpu_batch_options *batch_options,
                               vgpu_result **results, vgpu_batch_stats *stats) {
	return Guard([&] {
		if (!batch || !batch->prepared) Fail(VGPU_ERR_INVALID_ARGUMENT, "null batch");
		RunPreparedBatch(*batch->prepared, inputs, n_inputs, options, batch_options, results, stats);
	});
}

void vgpu_batch_free(vgpu_batch *batch) {
	delete batch;
}

vgpu_status vgpu_execute_batch(const vgpu_plan *const *plans, const vgpu_column *const *inputs,
                               const size_t *n_inputs, size_t n_plans, const vgpu_exec_options *options,
                               const vgpu_batch_options *batch_options, vgpu_result **results,
                               vgpu_batch_stats *stats) {
	return Guard([&] {
		auto pb = PrepareFromAbi(plans, n_plans);
		RunPreparedBatch(*pb, inputs, n_inputs, options, batch_options, results, stats);
	});
}

struct vgpu_pipeline {
	std::unique_ptr<StreamPipeline> p;
	size_t outstanding = 0;  // results handed out and not yet released
};

struct vgpu_pipeline_result {
	vgpu_pipeline *owner = nullptr;
	int stage = -1;
};

int vgpu_pipeline_supports(const vgpu_plan *plan) {
	try {
		auto root = ConvertPlan(plan);
		return StreamPipeline::Supports(*root) ? 1 : 0;
	} catch (...) {
		return 0;
	}
}

vgpu_status vgpu_pipeline_create(const vgpu_plan *plan, const char *const *input_names, const int32_t *input_types,
                                 size_t n_inputs, uint64_t max_rows_per_batch, int32_t depth, vgpu_pipeline **out) {
	return Guard([&] {
		if (!out || (n_inputs > 0 && (!input_names || !input_types))) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		*out = nullptr;
		std::vector<std::string> names;
		std::vector<ValueType> types;
		for (size_t i = 0; i < n_inputs; i++) {
			if (!input_names[i]) Fail(VGPU_ERR_INVALID_ARGUMENT, "null input name");
			if (!IsValidValueType(input_types[i])) Fail(VGPU_ERR_INVALID_ARGUMENT, "input type out of range");
			names.push_back(input_names[i]);
			types.push_back(static_cast<ValueType>(input_types[i]));
		}
		auto *p = new vgpu_pipeline();
		try {
			p->p.reset(new StreamPipeline(ConvertPlan(plan), names, types, max_rows_per_batch, depth > 0 ? depth : 3));
		} catch (...) {
			delete p;
			throw;
		}
		*out = p;
	});
}

size_t vgpu_pipeline_output_count(const vgpu_pipeline *pipeline) {
	return pipeline && pipeline->p ? pipeline->p->output_types().size() : 0;
}

int32_t vgpu_pipeline_output_type(const vgpu_pipeline *pipeline, size_t index) {
	if (!pipeline || !pipeline->p || index >= pipeline->p->output_types().size()) return -1;
	return static_cast<int32_t>(pipeline->p->output_types()[index]);
}

void vgpu_pipeline_poll(vgpu_pipeline *pipeline) {
	if (pipeline && pipeline->p) pipeline->p->Poll();
}

int vgpu_pipeline_can_submit(vgpu_pipeline *pipeline) {
	return pipeline && pipeline->p && pipeline->p->CanSubmit() ? 1 : 0;
}

vgpu_status vgpu_pipeline_submit(vgpu_pipeline *pipeline, const vgpu_column *columns, size_t n_columns,
                                 uint64_t row_count) {
	return Guard([&] {
		if (!pipeline || !pipeline->p || (n_columns > 0 && !columns)) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		pipeline->p->Submit(std::vector<vgpu_column>(columns, columns + n_columns), row_count);
	});
}

namespace {
vgpu_status PipelineTake(vgpu_pipeline *pipeline, vgpu_pipeline_result **out, bool wait) {
	return Guard([&] {
		if (!pipeline || !pipeline->p || !out) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		*out = nullptr;
		const int s = pipeline->p->Take(wait);
		if (s < 0) return;
		auto *r = new vgpu_pipeline_result();
		r->owner = pipeline;
		r->stage = s;
		pipeline->outstanding++;
		*out = r;
	});
}
} // namespace

vgpu_status vgpu_pipeline_try_take(vgpu_pipeline *pipeline, vgpu_pipeline_result **out) {
	return PipelineTake(pipeline, out, false);
}

vgpu_status vgpu_pipeline_take_blocking(vgpu_pipeline *pipeline, vgpu_pipeline_result **out) {
	return PipelineTake(pipeline, out, true);
}

size_t vgpu_pipeline_in_flight(const vgpu_pipeline *pipeline) {
	return pipeline && pipeline->p ? pipeline->p->in_flight() : 0;
}

uint64_t vgpu_pipeline_result_rows(const vgpu_pipeline_result *result) {
	return result && result->owner ? result->owner->p->StageRows(result->stage) : 0;
}

size_t vgpu_pipeline_result_column_count(const vgpu_pipeline_result *result) {
	return result && result->owner ? result->owner->p->output_types().size() : 0;
}

vgpu_status vgpu_pipeline_result_get_column(const vgpu_pipeline_result *result, size_t index, vgpu_column *out) {
	return Guard([&] {
		if (!result || !result->owner || !out) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		auto &p = *result->owner->p;
		if (index >= p.output_types().size()) Fail(VGPU_ERR_INVALID_ARGUMENT, "column index out of range");
		auto v = p.StageOutput(result->stage, index);
		std::memset(out, 0, sizeof(*out));
		out->name = p.output_names()[index].c_str();
		out->type = static_cast<int32_t>(p.output_types()[index]);
		out->data = v.data;
		out->validity = v.validity;
		out->row_count = p.StageRows(result->stage);
		out->memory = VGPU_MEM_HOST;
	});
}

void vgpu_pipeline_result_release(vgpu_pipeline_result *result) {
	if (!result) return;
	if (result->owner && result->owner->p) {
		result->owner->p->Release(result->stage);
		result->owner->outstanding--;
	}
	delete result;
}

void vgpu_pipeline_destroy(vgpu_pipeline *pipeline) {
	try {
		delete pipeline;
	} catch (...) {
	}
}

struct vgpu_server {
	std::unique_ptr<Server> server;
};

void vgpu_server_options_init(vgpu_server_options *options) {
	if (!options) return;
	std::memset(options, 0, sizeof(*options));
	options->slots = 4;
	options->batch_max = 64;
}

vgpu_status vgpu_server_create(const vgpu_server_options *options, vgpu_server **out) {
	return Guard([&] {
		if (!out) Fail(VGPU_ERR_INVALID_ARGUMENT, "null server pointer");
		*out = nullptr;
		ServerOptions so;
		if (options) {
			so.slots = options->slots;
			so.batch_max = options->batch_max;
			so.memory_budget = options->memory_budget_bytes;
		}
		auto *s = new vgpu_server();
		try {
			s->server.reset(new Server(so));
		} catch (...) {
			delete s;
			throw;
		}
		*out = s;
	});
}

vgpu_status vgpu_server_submit(vgpu_server *server, const vgpu_plan *plan, const vgpu_column *inputs, size_t n_inputs,
                               const vgpu_exec_options *options, uint64_t *request_id) {
	return Guard([&] {
		if (!server || !request_id) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		if (n_inputs > 0 && inputs == nullptr) Fail(VGPU_ERR_INVALID_ARGUMENT, "null inputs with nonzero count");
		ExecOptions eo;
		if (options) {
			eo.serve_whole_scan_from_cache = options->serve_whole_scan_from_cache != 0;
			eo.cache_chunk_index = options->cache_chunk_index;
			eo.output_on_device = options->output_memory == VGPU_MEM_DEVICE;
			if (options->stage_scan_to_cache) Fail(VGPU_ERR_UNSUPPORTED, "serving does not stage scans to the cache");
			if (eo.serve_whole_scan_from_cache && eo.cache_chunk_index >= 0) {
				Fail(VGPU_ERR_INVALID_ARGUMENT, "serve_whole_scan_from_cache and cache_chunk_index are exclusive");
			}
		}
		std::vector<vgpu_column> in(inputs, inputs + n_inputs);
		*request_id = server->server->Submit(ConvertPlan(plan), std::move(in), eo);
	});
}

vgpu_status vgpu_server_wait(vgpu_server *server, uint64_t request_id, double timeout_ms, vgpu_result **result,
                             vgpu_request_info *info, int *done) {
	return Guard([&] {
		if (!server || !done) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		*done = 0;
		if (result) *result = nullptr;
		ExecResult r;
		RequestInfo ri;
		if (!server->server->Wait(request_id, timeout_ms, &r, &ri)) return;
		*done = 1;
		if (info) {
			std::memset(info, 0, sizeof(*info));
			info->status = ri.status;
			info->batch_size = static_cast<int32_t>(ri.batch_size);
			info->queued_ms = ri.queued_ms;
			info->run_ms = ri.run_ms;
			info->estimated_bytes = ri.estimated_bytes;
			std::snprintf(info->error, sizeof(info->error), "%s", ri.error.c_str());
		}
		if (ri.status == VGPU_OK && result) {
			auto *res = new vgpu_result();
			res->exec = std::move(r);
			*result = res;
		} else {
			for (void *p : r.device_buffers) Runtime::Get().allocator().Free(p, r.stream);
		}
	});
}

vgpu_status vgpu_server_stats_get(vgpu_server *server, vgpu_server_stats *out) {
	return Guard([&] {
		if (!server || !out) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		ServerStats s = server->server->Stats();
		out->submitted = s.submitted;
		out->completed = s.completed;
		out->failed = s.failed;
		out->rejected = s.rejected;
		out->batches = s.batches;
		out->batched_requests = s.batched_requests;
		out->in_flight = s.in_flight;
		out->queued = s.queued;
		out->reserved_bytes = s.reserved_bytes;
		out->peak_reserved_bytes = s.peak_reserved_bytes;
		out->budget_bytes = s.budget_bytes;
		out->peak_in_flight = s.peak_in_flight;
	});
}

void vgpu_server_destroy(vgpu_server *server) {
	try {
		delete server;
	} catch (...) {
	}
}

vgpu_status vgpu_batch_template(const char *source, char *out, size_t capacity, size_t *length, size_t *n_params) {
	return Guard([&] {
		if (!source) Fail(VGPU_ERR_INVALID_ARGUMENT, "null source");
		TemplatedSource t = TemplateLiterals(source, 0);
		if (length) *length = t.text.size();
		if (n_params) *n_params = t.types.size();
		if (out && capacity > 0) {
			const size_t k = std::min(capacity - 1, t.text.size());
			std::memcpy(out, t.text.data(), k);
			out[k] = '\0';
		}
	});
}

vgpu_status vgpu_copy_to_host(void *dst, const void *src, size_t bytes, void *stream) {
	return Guard([&] {
		if (bytes == 0) return;
		if (!dst || !src) Fail(VGPU_ERR_INVALID_ARGUMENT, "null pointer");
		cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : Runtime::Get().default_stream();
		VGPU_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
		VGPU_CUDA(cudaStreamSynchronize(s));
	});
}

vgpu_status vgpu_batch_clear(void) {
	return Guard([&] { ClearBatchCaches(); });
}

size_t vgpu_result_column_count(const vgpu_result *result) {
	return result ? result->exec.columns.size() : 0;
}

namespace {

// A result whose execution left its row count on the device (device output without a sync) reads it
// now, once: the stream's work up to the count is waited for here instead of in the execution.
void ResolveRows(const vgpu_result *result) {
	auto *r = const_cast<vgpu_result *>(result);  // results are created mutable; the API hands out const views
	std::lock_guard<std::mutex> lock(r->rows_mu);
	if (!r->exec.pending_rows) return;
	const size_t width = r->exec.pending_rows_bytes == 4 ? 4 : 8;
	auto word = PinnedPool::Get().Acquire(sizeof(uint64_t));
	VGPU_CUDA(cudaMemcpyAsync(word.get(), r->exec.pending_rows, width, cudaMemcpyDeviceToHost, r->exec.stream));
	VGPU_CUDA(cudaStreamSynchronize(r->exec.stream));
	uint64_t rows = 0;
	if (width == 4) {
		uint32_t v;
		std::memcpy(&v, word.get(), sizeof(v));
		rows = v;
	} else {
		std::memcpy(&rows, word.get(), sizeof(rows));
	}
	for (auto &c : r->exec.columns) c.rows = rows;
	r->exec.pending_rows = nullptr;  // its buffer is freed with the result
}

} // namespace

vgpu_status vgpu_result_get_column(const vgpu_result *result, size_t index, vgpu_column *out) {
	return Guard([&] {
		if (!result || !out) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		ResolveRows(result);
		if (index >= result->exec.columns.size()) Fail(VGPU_ERR_INVALID_ARGUMENT, "column index out of range");
		const HostColumnOut &c = result->exec.columns[index];
		out->name = c.name.c_str();
		out->type = static_cast<uint32_t>(c.type);
		out->row_count = c.rows;
		if (c.device_data != nullptr) {
			out->memory = VGPU_MEM_DEVICE;
			out->data = c.device_data;
			out->validity = c.device_validity;
		} else {
			out->memory = VGPU_MEM_HOST;
			out->data = c.host ? static_cast<const void *>(c.host.get()) : (c.data.empty() ? nullptr : c.data.data());
			out->validity = c.validity.empty() ? nullptr : c.validity.data();
		}
	});
}

vgpu_status vgpu_result_column_range(const vgpu_result *result, size_t index, uint64_t offset, uint64_t count,
                                     vgpu_column *out) {
	return Guard([&] {
		if (!result || !out) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		vgpu_column whole;
		if (vgpu_result_get_column(result, index, &whole) != VGPU_OK) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "vgpu_result_column_range: column index out of range");
		}
		if (offset > whole.row_count || count > whole.row_count - offset) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "vgpu_result_column_range: rows [" + std::to_string(offset) + ", " +
			                                    std::to_string(offset + count) + ") exceed the column's " +
			                                    std::to_string(whole.row_count));
		}
		if (whole.validity != nullptr && offset % 64 != 0) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "vgpu_result_column_range: a column with validity is sliced at multiples "
			                                "of 64 rows (whole validity words)");
		}
		*out = whole;
		out->row_count = count;
		const size_t width = TypeSize(static_cast<ValueType>(whole.type));
		if (whole.data) out->data = static_cast<const uint8_t *>(whole.data) + offset * width;
		if (whole.validity) out->validity = whole.validity + offset / 8;
	});
}

void vgpu_result_free(vgpu_result *result) {
	if (!result) return;
	try {
		for (void *p : result->exec.device_buffers) {
			Runtime::Get().allocator().Free(p, result->exec.stream);
		}
	} catch (...) {
	}
	delete result;
}

vgpu_status vgpu_set_device(int device) {
	return Guard([&] { Runtime::Get().SetDevice(device); });
}

vgpu_status vgpu_get_device_info(vgpu_device_info *out) {
	return Guard([&] {
		if (!out) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		const auto &p = Runtime::Get().props();
		std::memset(out, 0, sizeof(*out));
		out->device = p.device;
		out->sm_count = p.sm_count;
		out->cc_major = p.cc_major;
		out->cc_minor = p.cc_minor;
		out->total_memory = p.total_memory;
		size_t free_b = 0, total_b = 0;
		VGPU_CUDA(cudaMemGetInfo(&free_b, &total_b));
		out->free_memory = free_b;
		out->l2_bytes = p.l2_bytes;
		out->smem_per_block_optin = p.smem_optin;
		std::snprintf(out->name, sizeof(out->name), "%s", p.name.c_str());
	});
}

vgpu_status vgpu_synchronize(void *stream) {
	return Guard([&] {
		cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : Runtime::Get().default_stream();
		VGPU_CUDA(cudaStreamSynchronize(s));
	});
}

vgpu_status vgpu_profile_enable(int enable) {
	return Guard([&] { Runtime::Get().profiler().Enable(enable != 0); });
}

vgpu_status vgpu_profile_collect(vgpu_kernel_timing *out, size_t capacity, size_t *count) {
	return Guard([&] {
		auto v = Runtime::Get().profiler().Collect();
		if (count) *count = v.size();
		for (size_t i = 0; i < v.size() && i < capacity && out; i++) out[i] = v[i];
	});
}

uint64_t vgpu_launch_count(void) {
	return Runtime::Get().launches();
}

void vgpu_sha256_hex(const void *data, size_t n, char *out) {
	if (!out) return;
	std::string h = Sha256Hex(data, data ? n : 0);
	std::memcpy(out, h.c_str(), 65);
}

vgpu_status vgpu_kernel_cache_stats_get(vgpu_kernel_cache_stats *out) {
	return Guard([&] {
		if (!out) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		*out = Runtime::Get().modules().Stats();
	});
}

vgpu_status vgpu_nvrtc_compile_check(const char *source, size_t *cubin_bytes) {
	return Guard([&] {
		if (!source) Fail(VGPU_ERR_INVALID_ARGUMENT, "null source");
		const char *arch = std::getenv("VGPU_NVRTC_ARCH");
		auto cubin = CompileToCubin(source, arch ? arch : "sm_100a", nullptr);
		if (cubin_bytes) *cubin_bytes = cubin.size();
	});
}

vgpu_status vgpu_generate_source(const vgpu_plan *plan, const vgpu_column *inputs, size_t n_inputs, char *out,
                                 size_t capacity, size_t *length) {
	return Guard([&] {
		auto root = ConvertPlan(plan);
		std::vector<vgpu_column> in(inputs, inputs + n_inputs);
		std::string src = GenerateSourceText(*root, in);
		if (length) *length = src.size();
		if (out && capacity > 0) {
			size_t n = std::min(capacity - 1, src.size());
			std::memcpy(out, src.data(), n);
			out[n] = '\0';
		}
	});
}

int vgpu_is_row_independent(const vgpu_plan *plan) {
	try {
		auto root = ConvertPlan(plan);
		return IsRowIndependent(*root) ? 1 : 0;
	} catch (...) {
		return 0;
	}
}

vgpu_status vgpu_estimate_working_set(const vgpu_plan *plan, uint64_t max_chunk_rows, vgpu_working_set *out) {
	return Guard([&] {
		if (!out) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		auto root = ConvertPlan(plan);
		*out = EstimateWorkingSet(*root, max_chunk_rows);
	});
}

vgpu_status vgpu_estimate_working_set_for(const vgpu_plan *plan, const vgpu_column *inputs, size_t n_inputs,
                                          const vgpu_exec_options *options, vgpu_working_set *out) {
	return Guard([&] {
		if (!out || (n_inputs && !inputs)) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		auto root = ConvertPlan(plan);
		std::vector<vgpu_column> in(inputs, inputs + n_inputs);
		*out = EstimateWorkingSetFor(*root, in, options && options->serve_whole_scan_from_cache);
	});
}

vgpu_status vgpu_translate_expression(const vgpu_bexpr *nodes, uint32_t n_nodes, uint32_t root, uint32_t flags,
                                      char *statement, size_t statement_cap, size_t *statement_len, char *inputs,
                                      size_t inputs_cap, size_t *inputs_len, uint32_t *n_inputs,
                                      uint32_t *output_type) {
	return Guard([&] {
		const TranslatedExpr t = TranslateExpression(nodes, n_nodes, root, flags);
		std::string names;
		for (auto &n : t.inputs) {
			names += n;
			names.push_back('\0');
		}
		if (statement_len) *statement_len = t.statement.size() + 1;
		if (inputs_len) *inputs_len = names.size();
		if (n_inputs) *n_inputs = static_cast<uint32_t>(t.inputs.size());
		if (output_type) *output_type = static_cast<uint32_t>(t.output_type);
		if (!statement || statement_cap < t.statement.size() + 1 || (!names.empty() && (!inputs || inputs_cap < names.size()))) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "vgpu_translate_expression: output buffer too small");
		}
		std::memcpy(statement, t.statement.c_str(), t.statement.size() + 1);
		if (!names.empty()) std::memcpy(inputs, names.data(), names.size());
	});
}

vgpu_status vgpu_analyze_plan_shape(const vgpu_plan *plan, vgpu_plan_shape *out) {
	return Guard([&] {
		if (!out) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		auto root = ConvertPlan(plan);
		*out = AnalyzePlanShape(*root);
	});
}

vgpu_status vgpu_estimate_columns_size(const vgpu_plan *plan, uint64_t *out) {
	return Guard([&] {
		if (!out) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		auto root = ConvertPlan(plan);
		*out = EstimateColumnsSize(*root);
	});
}

vgpu_status vgpu_determine_execution_mode(const vgpu_plan *plan, uint64_t vram_budget, double threshold,
                                          uint32_t *mode, uint64_t *columns_size) {
	return Guard([&] {
		if (!mode) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		auto root = ConvertPlan(plan);
		*mode = DetermineExecutionMode(*root, vram_budget, threshold);
		if (columns_size) *columns_size = EstimateColumnsSize(*root);
	});
}

vgpu_status vgpu_memory_set_budget(uint64_t bytes) {
	return Guard([&] {
		Runtime::Get().EnsureDevice();
		Runtime::Get().allocator().SetBudget(bytes);
	});
}

vgpu_status vgpu_memory_stats_get(vgpu_memory_stats *out) {
	return Guard([&] {
		if (!out) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		Runtime::Get().EnsureDevice();
		*out = Runtime::Get().allocator().Stats();
	});
}

vgpu_status vgpu_memory_reset_peak(void) {
	return Guard([&] {
		Runtime::Get().EnsureDevice();
		Runtime::Get().allocator().ResetPeak();
	});
}

int vgpu_memory_has_headroom(uint64_t bytes) {
	try {
		Runtime::Get().EnsureDevice();
		return Runtime::Get().allocator().HasHeadroom(bytes) ? 1 : 0;
	} catch (...) {
		return 0;
	}
}

vgpu_status vgpu_cache_init(double fraction_of_vram) {
	return Guard([&] { ColumnCache::Get().EnsureInitialized(fraction_of_vram); });
}

vgpu_status vgpu_cache_begin_staging(const vgpu_table_ref *table) {
	return Guard([&] { ColumnCache::Get().BeginStaging(ToTable(table)); });
}

vgpu_status vgpu_cache_stage_chunk(const vgpu_table_ref *table, const vgpu_column *chunk, int *accepted) {
	return Guard([&] {
		if (!chunk) Fail(VGPU_ERR_INVALID_ARGUMENT, "null chunk");
		bool ok = ColumnCache::Get().StageChunk(ToTable(table), *chunk);
		if (accepted) *accepted = ok ? 1 : 0;
	});
}

vgpu_status vgpu_cache_commit_staging(const vgpu_table_ref *table, uint64_t scanned_rows) {
	return Guard([&] { ColumnCache::Get().CommitStaging(ToTable(table), scanned_rows); });
}

vgpu_status vgpu_cache_abort_staging(const vgpu_table_ref *table) {
	return Guard([&] { ColumnCache::Get().AbortStaging(ToTable(table)); });
}

vgpu_status vgpu_cache_replayable_chunk_rows(const vgpu_table_ref *table, const char *const *column_names,
                                             size_t n_columns, uint64_t *rows, size_t capacity, size_t *count) {
	return Guard([&] {
		std::vector<std::string> cols;
		for (size_t i = 0; i < n_columns; i++) cols.emplace_back(column_names[i] ? column_names[i] : "");
		auto v = ColumnCache::Get().ReplayableChunkRows(ToTable(table), cols);
		if (count) *count = v.size();
		for (size_t i = 0; i < v.size() && i < capacity && rows; i++) rows[i] = v[i];
	});
}

vgpu_status vgpu_cache_try_get_chunk(const vgpu_table_ref *table, const char *column_name, uint64_t chunk_index,
                                     vgpu_column *out, int *found) {
	return Guard([&] {
		if (!out || !column_name) Fail(VGPU_ERR_INVALID_ARGUMENT, "null argument");
		DevColumn c;
		bool ok = ColumnCache::Get().TryGetChunk(ToTable(table), column_name, chunk_index, c);
		if (found) *found = ok ? 1 : 0;
		if (ok) {
			out->name = column_name;
			out->type = static_cast<uint32_t>(c.type);
			out->memory = VGPU_MEM_DEVICE;
			out->data = c.data;
			out->validity = nullptr; // internal byte masks are not an Arrow bitmap; not exposed
			out->row_count = c.rows;
		}
	});
}

vgpu_status vgpu_cache_invalidate_table(const vgpu_table_ref *table) {
	return Guard([&] {
		ColumnCache::Get().InvalidateTable(ToTable(table));
		ClearJoinTables();
	});
}

vgpu_status vgpu_cache_invalidate_all(void) {
	return Guard([&] {
		ColumnCache::Get().InvalidateAll();
		ClearJoinTables();
	});
}

uint64_t vgpu_cache_current_bytes(void) {
	try {
		return ColumnCache::Get().CurrentBytes();
	} catch (...) {
		return 0;
	}
}

uint64_t vgpu_cache_table_generation(const vgpu_table_ref *table) {
	try {
		return ColumnCache::Get().Generation(ToTable(table));
	} catch (...) {
		return 0;
	}
}

int32_t vgpu_shard_words(const int32_t *kinds, int32_t n_values) {
	if (n_values < 0 || (n_values > 0 && !kinds)) return 0;
	return ShardWords(kinds, n_values);
}

vgpu_status vgpu_shard_route(const vgpu_column *keys, int32_t n_keys, const int64_t *key_min, const int32_t *key_shift,
                             const vgpu_column *values, const int32_t *kinds, int32_t n_values, uint64_t rows,
                             int32_t world, int64_t *send, uint64_t *send_counts, void *stream) {
	return Guard([&] {
		if (!keys || !key_min || !key_shift || !send_counts || (n_values > 0 && (!values || !kinds))) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "vgpu_shard_route: null argument");
		}
		Runtime::Get().EnsureDevice();
		cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : Runtime::Get().default_stream();
		ShardRoute(keys, n_keys, key_min, key_shift, values, kinds, n_values, rows, static_cast<uint32_t>(world), send,
		           send_counts, s);
	});
}

vgpu_status vgpu_shard_columns(const int64_t *recv, uint64_t rows, int32_t words, int64_t *out, void *stream) {
	return Guard([&] {
		Runtime::Get().EnsureDevice();
		cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : Runtime::Get().default_stream();
		ShardColumns(recv, rows, words, out, s);
	});
}

vgpu_status vgpu_shard_finish(const vgpu_shard_output *outs, int32_t n_outs, uint64_t rows, void *stream) {
	return Guard([&] {
		if (n_outs < 0 || (n_outs > 0 && !outs)) Fail(VGPU_ERR_INVALID_ARGUMENT, "vgpu_shard_finish: null argument");
		Runtime::Get().EnsureDevice();
		cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : Runtime::Get().default_stream();
		ShardFinish(outs, n_outs, rows, s);
	});
}

} // extern "C"
