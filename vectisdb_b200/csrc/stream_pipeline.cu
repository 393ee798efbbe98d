// stream_pipeline.cu -- see stream_pipeline.hpp.
#include "stream_pipeline.hpp"

#include <algorithm>
#include <cstring>

#include "kernels.hpp"

namespace vgpu {

namespace {

constexpr int kBlock = 256;
constexpr int kItems = 4;

// The projection chain from the top node down to the SCAN, or false.
bool Chain(const PlanNode &plan, std::vector<const PlanNode *> &chain, const PlanNode **scan) {
	const PlanNode *cur = &plan;
	while (cur->op == OpType::PROJECTION) {
		if (cur->children.size() != 1 || cur->expressions.empty()) return false;
		chain.push_back(cur);
		cur = cur->children[0].get();
	}
	if (cur->op != OpType::SCAN || chain.empty()) return false;
	*scan = cur;
	return true;
}

} // namespace

bool StreamPipeline::Supports(const PlanNode &plan) {
	std::vector<const PlanNode *> chain;
	const PlanNode *scan = nullptr;
	if (!Chain(plan, chain, &scan)) return false;
	std::vector<std::string> below = scan->column_names;
	for (auto it = chain.rbegin(); it != chain.rend(); ++it) {
		std::vector<std::string> names;
		const bool top = *it == chain.front();
		for (size_t i = 0; i < (*it)->expressions.size(); i++) {
			const auto &e = (*it)->expressions[i];
			// RUNNING_SUM: a running total of a numeric output column (the chain runs fused, so only the
			// top level's outputs are materialized to scan).
			if (e.window != VGPU_WINDOW_NONE) {
				if (!top || e.output_type == ValueType::BOOLEAN || e.output_type == ValueType::DICTIONARY_STRING ||
				    e.output_type == ValueType::HUGEINT) {
					return false;
				}
			}
			for (auto &in : e.input_columns) {
				if (std::find(below.begin(), below.end(), in) == below.end()) return false;
			}
			if (!IsValidValueType(static_cast<int>(e.output_type)) || e.output_type == ValueType::HUGEINT ||
			    TypeSize(e.output_type) == 0) {
				return false;
			}
			names.push_back("col" + std::to_string(i));
		}
		below = names;
	}
	return true;
}

StreamPipeline::StreamPipeline(std::shared_ptr<PlanNode> plan, const std::vector<std::string> &input_names,
                               const std::vector<ValueType> &input_types, uint64_t max_rows_per_batch, int depth)
    : plan_(std::move(plan)), in_names_(input_names), in_types_(input_types), max_rows_(max_rows_per_batch),
      depth_(static_cast<size_t>(std::max(1, depth))) {
	if (!Supports(*plan_)) {
		Fail(VGPU_ERR_UNSUPPORTED, "gpu_stream_pipeline: the plan is not a chain of projections over a scan");
	}
	if (input_names.size() != input_types.size() || input_names.empty() || input_names.size() > 64) {
		Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_stream_pipeline: 1..64 input columns, one type per name");
	}
	if (max_rows_ == 0 || max_rows_ >= (1ull << 32)) {
		Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_stream_pipeline: max_rows_per_batch must be in [1, 2^32)");
	}
	std::vector<const PlanNode *> chain;
	const PlanNode *scan = nullptr;
	Chain(*plan_, chain, &scan);
	if (scan->column_names != in_names_) {
		Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_stream_pipeline: input names differ from the plan's scan columns");
	}
	for (auto t : in_types_) {
		if (!IsValidValueType(static_cast<int>(t)) || t == ValueType::HUGEINT) {
			Fail(VGPU_ERR_UNSUPPORTED, "gpu_stream_pipeline: unsupported input type");
		}
	}
	Runtime::Get().EnsureDevice();
	const Variant &v0 = GetVariant(0);  // compile (or fetch) the no-NULL kernel now: fail here, not mid-scan
	(void)v0;
	for (auto &e : chain.front()->expressions) {
		if (e.window != VGPU_WINDOW_NONE) window_cols_.push_back(out_types_.size());
		out_types_.push_back(e.output_type);
	}
	for (size_t i = 0; i < out_types_.size(); i++) out_names_.push_back("col" + std::to_string(i));
	for (cudaStream_t *s : {&s_h2d_, &s_exec_, &s_d2h_}) VGPU_CUDA(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking));
	auto &al = Runtime::Get().allocator();
	auto dev = [&](size_t bytes) {
		void *p = al.Alloc(std::max<size_t>(bytes, 16), s_exec_);
		device_owned_.push_back(p);
		return p;
	};
	auto host = [&](size_t bytes) {
		void *p = nullptr;
		VGPU_CUDA(cudaMallocHost(&p, std::max<size_t>(bytes, 16)));
		host_owned_.push_back(p);
		return p;
	};
	const size_t bm = (max_rows_ + 7) / 8;
	stages_.resize(depth_ + 1);
	for (auto &st : stages_) {
		for (auto t : in_types_) {
			st.in_host.push_back(host(max_rows_ * TypeSize(t)));
			st.in_dev.push_back(dev(max_rows_ * TypeSize(t)));
			st.in_bitmap_host.push_back(host(bm));
			st.in_bitmap_dev.push_back(dev(bm));
			st.in_valid_dev.push_back(dev(max_rows_));
		}
		for (auto t : out_types_) {
			st.out_dev.push_back(dev(max_rows_ * TypeSize(t)));
			st.out_valid_dev.push_back(dev(max_rows_));
			st.out_bitmap_dev.push_back(dev(bm));
			st.out_host.push_back(host(max_rows_ * TypeSize(t)));
			st.out_bitmap_host.push_back(host(bm));
		}
		for (cudaEvent_t *e : {&st.h2d, &st.exec, &st.d2h}) VGPU_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
	}
	for (size_t i = 0; i < stages_.size(); i++) free_.push_back(static_cast<int>(i));
	if (!window_cols_.empty()) {
		// one running state per RUNNING_SUM column, starting at zero; one scratch (batches run in order
		// on the compute stream, so they share it)
		for (size_t c : window_cols_) {
			running_state_.push_back(dev(TypeSize(out_types_[c])));
			VGPU_CUDA(cudaMemsetAsync(running_state_.back(), 0, TypeSize(out_types_[c]), s_exec_));
		}
		running_scratch_ = dev(kern::RunningSumScratchBytes(max_rows_));
	}
	VGPU_CUDA(cudaStreamSynchronize(s_exec_));
}

StreamPipeline::~StreamPipeline() {
	for (cudaStream_t s : {s_h2d_, s_exec_, s_d2h_}) {
		if (s) cudaStreamSynchronize(s);
	}
	auto &al = Runtime::Get().allocator();
	for (void *p : device_owned_) {
		try {
			al.Free(p, s_exec_);
		} catch (...) {
		}
	}
	if (s_exec_) cudaStreamSynchronize(s_exec_);
	for (void *p : host_owned_) cudaFreeHost(p);
	for (auto &st : stages_) {
		for (cudaEvent_t e : {st.h2d, st.exec, st.d2h}) {
			if (e) cudaEventDestroy(e);
		}
	}
	for (cudaStream_t s : {s_h2d_, s_exec_, s_d2h_}) {
		if (s) cudaStreamDestroy(s);
	}
}

const StreamPipeline::Variant &StreamPipeline::GetVariant(uint64_t null_mask) {
	auto it = variants_.find(null_mask);
	if (it != variants_.end()) return it->second;
	std::vector<const PlanNode *> chain;
	const PlanNode *scan = nullptr;
	Chain(*plan_, chain, &scan);
	std::reverse(chain.begin(), chain.end());
	PipelineSpec spec;
	spec.chain = chain;
	for (size_t i = 0; i < in_names_.size(); i++) {
		SourceColumn sc;
		sc.name = in_names_[i];
		sc.type = in_types_[i];
		sc.nullable = ((null_mask >> i) & 1ull) != 0;
		spec.sources.push_back(sc);
	}
	PipelineCodegen cg(spec);
	std::vector<int> outs;
	for (size_t i = 0; i < cg.visible().size(); i++) outs.push_back(static_cast<int>(i));
	Geometry g;
	g.block = kBlock;
	g.items = kItems;
	Variant v;
	v.module = Runtime::Get().modules().GetOrCompile(cg.EmitMaterialize(outs, g));
	for (auto &c : cg.visible()) v.out_nullable.push_back(c.nullable);
	v.cb = cg.ConsumerBase();
	return variants_.emplace(null_mask, std::move(v)).first->second;
}

bool StreamPipeline::CanSubmit() const {
	return !free_.empty() && fifo_.size() < depth_;
}

void StreamPipeline::Submit(const std::vector<vgpu_column> &cols, uint64_t rows) {
	if (!CanSubmit()) {
		Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_stream_pipeline: no free stage (take results before submitting more)");
	}
	if (cols.size() != in_names_.size()) Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_stream_pipeline: column count mismatch");
	if (rows > max_rows_) Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_stream_pipeline: batch larger than max_rows_per_batch");
	uint64_t mask = 0;
	for (size_t i = 0; i < cols.size(); i++) {
		const vgpu_column &c = cols[i];
		if (!c.name || in_names_[i] != c.name) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_stream_pipeline: column " + std::to_string(i) + " should be '" +
			                                    in_names_[i] + "'");
		}
		if (c.type != static_cast<int32_t>(in_types_[i])) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_stream_pipeline: column '" + in_names_[i] + "' type mismatch");
		}
		if (c.memory == VGPU_MEM_DEVICE) Fail(VGPU_ERR_UNSUPPORTED, "gpu_stream_pipeline: batches are host columns");
		if (c.row_count < rows || (rows > 0 && c.data == nullptr)) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_stream_pipeline: column '" + in_names_[i] + "' shorter than the batch");
		}
		if (c.validity) mask |= 1ull << i;
	}
	const Variant &v = GetVariant(mask);
	for (size_t c : window_cols_) {
		if (v.out_nullable[c]) {
			Fail(VGPU_ERR_UNSUPPORTED, "gpu_stream_pipeline: RUNNING_SUM over a batch with NULL inputs is not supported");
		}
	}
	const int s = free_.front();
	free_.pop_front();
	Stage &st = stages_[s];
	st.rows = rows;
	st.out_nullable = v.out_nullable;
	const size_t bm = (rows + 7) / 8;
	// upload (through this stage's pinned buffers: the caller's memory is free when we return)
	for (size_t i = 0; i < cols.size(); i++) {
		const size_t bytes = rows * TypeSize(in_types_[i]);
		if (bytes) {
			std::memcpy(st.in_host[i], cols[i].data, bytes);
			VGPU_CUDA(cudaMemcpyAsync(st.in_dev[i], st.in_host[i], bytes, cudaMemcpyHostToDevice, s_h2d_));
		}
		if (cols[i].validity && bm) {
			std::memcpy(st.in_bitmap_host[i], cols[i].validity, bm);
			VGPU_CUDA(cudaMemcpyAsync(st.in_bitmap_dev[i], st.in_bitmap_host[i], bm, cudaMemcpyHostToDevice, s_h2d_));
		}
	}
	VGPU_CUDA(cudaEventRecord(st.h2d, s_h2d_));
	// compute: one fused kernel for the whole chain
	VGPU_CUDA(cudaStreamWaitEvent(s_exec_, st.h2d, 0));
	if (rows > 0) {
		for (size_t i = 0; i < cols.size(); i++) {
			if ((mask >> i) & 1u) kern::UnpackValidity(static_cast<uint8_t *>(st.in_bitmap_dev[i]),
			                                           static_cast<uint8_t *>(st.in_valid_dev[i]), rows, s_exec_);
		}
		uint64_t w[128];
		std::memset(w, 0, sizeof(w));
		w[0] = rows;
		for (size_t i = 0; i < cols.size(); i++) {
			w[2 + 2 * i] = reinterpret_cast<uint64_t>(st.in_dev[i]);
			w[3 + 2 * i] = ((mask >> i) & 1u) ? reinterpret_cast<uint64_t>(st.in_valid_dev[i]) : 0;
		}
		for (size_t c = 0; c < out_types_.size(); c++) {
			w[v.cb + 1 + 2 * c] = reinterpret_cast<uint64_t>(st.out_dev[c]);
			w[v.cb + 2 + 2 * c] = v.out_nullable[c] ? reinterpret_cast<uint64_t>(st.out_valid_dev[c]) : 0;
		}
		const uint64_t tile = kBlock * kItems;
		const unsigned grid = static_cast<unsigned>(
		    std::max<uint64_t>(1, std::min<uint64_t>((rows + tile - 1) / tile, uint64_t(Runtime::Get().props().sm_count) * 8)));
		{
			LaunchScope scope("vgpu_mat_write", s_exec_, 0, rows);
			void *params[] = {w};
			Runtime::Get().LaunchModuleKernel(v.module->Get("vgpu_mat_write"), dim3(grid), dim3(kBlock), 0, s_exec_, params);
		}
		for (size_t k = 0; k < window_cols_.size(); k++) {
			const size_t c = window_cols_[k];
			kern::RunningSum(st.out_dev[c], out_types_[c], rows, running_state_[k], running_scratch_, s_exec_);
		}
		for (size_t c = 0; c < out_types_.size(); c++) {
			if (v.out_nullable[c]) kern::PackValidity(static_cast<uint8_t *>(st.out_valid_dev[c]),
			                                          static_cast<uint8_t *>(st.out_bitmap_dev[c]), rows, s_exec_);
		}
	}
	VGPU_CUDA(cudaEventRecord(st.exec, s_exec_));
	// download into this stage's pinned outputs
	VGPU_CUDA(cudaStreamWaitEvent(s_d2h_, st.exec, 0));
	for (size_t c = 0; c < out_types_.size(); c++) {
		const size_t bytes = rows * TypeSize(out_types_[c]);
		if (bytes) VGPU_CUDA(cudaMemcpyAsync(st.out_host[c], st.out_dev[c], bytes, cudaMemcpyDeviceToHost, s_d2h_));
		if (v.out_nullable[c] && bm) {
			VGPU_CUDA(cudaMemcpyAsync(st.out_bitmap_host[c], st.out_bitmap_dev[c], bm, cudaMemcpyDeviceToHost, s_d2h_));
		}
	}
	VGPU_CUDA(cudaEventRecord(st.d2h, s_d2h_));
	fifo_.push_back(s);
}

int StreamPipeline::Take(bool wait) {
	if (fifo_.empty()) return -1;
	const int s = fifo_.front();
	if (wait) {
		VGPU_CUDA(cudaEventSynchronize(stages_[s].d2h));
	} else {
		const cudaError_t e = cudaEventQuery(stages_[s].d2h);
		if (e == cudaErrorNotReady) return -1;
		if (e != cudaSuccess) VGPU_CUDA(e);
	}
	fifo_.pop_front();
	return s;
}

void StreamPipeline::Release(int stage) {
	if (stage < 0 || stage >= static_cast<int>(stages_.size())) return;
	if (std::find(free_.begin(), free_.end(), stage) != free_.end()) return;
	free_.push_back(stage);
}

StreamPipeline::OutView StreamPipeline::StageOutput(int stage, size_t column) const {
	const Stage &st = stages_.at(stage);
	OutView v;
	v.data = st.out_host.at(column);
	v.validity = st.out_nullable.at(column) ? static_cast<const uint8_t *>(st.out_bitmap_host.at(column)) : nullptr;
	return v;
}

} // namespace vgpu
