// stream_pipeline.hpp -- GpuStreamPipeline (cuda_engine/include/gpu_stream_pipeline.hpp:122-208,
// cuda_engine/src/gpu_stream_pipeline.cu:347-837), re-designed for this engine.
//
// Batches of a row-independent projection chain (PROJECTION* over SCAN, no filter: the output row
// count is the input's, so downloads never wait on a count) flow through three non-blocking streams:
// upload of batch N+2, the fused kernel of batch N+1 and download of batch N overlap, ordered only by
// per-stage events. Differences from the reference: the whole chain is ONE fused kernel per batch
// (the reference launches one kernel per expression per level); inputs are staged through the
// pipeline's own pinned buffers, so the caller's buffers are free again when Submit returns; NULLs
// are handled (byte masks on the device, Arrow bitmaps at both ends). Every buffer is allocated at
// construction (depth + 1 stage sets: one more than in flight, for the result the consumer holds).
// A top-level expression marked RUNNING_SUM (the reference's window primitive,
// gpu_stream_pipeline.cu:133-166, 700-704) leaves the running total of its values over every batch
// submitted so far: each batch is scanned on the compute stream after the fused kernel, continuing from
// a state kept on the device (integers wrap in their width, floats add in their own precision).
// Externally serialized: one call at a time.
#pragma once

#include <deque>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "codegen.hpp"
#include "plan.hpp"
#include "runtime.hpp"

namespace vgpu {

class StreamPipeline {
public:
	//! PROJECTION+ over a SCAN, every level with at least one expression whose inputs resolve against
	//! the level below, fixed-width output types; RUNNING_SUM only on top-level INT16/INT32/INT64/
	//! FLOAT32/FLOAT64 outputs (a batch whose window column would carry NULLs is refused at Submit).
	static bool Supports(const PlanNode &plan);

	StreamPipeline(std::shared_ptr<PlanNode> plan, const std::vector<std::string> &input_names,
	               const std::vector<ValueType> &input_types, uint64_t max_rows_per_batch, int depth = 3);
	~StreamPipeline();
	StreamPipeline(const StreamPipeline &) = delete;
	StreamPipeline &operator=(const StreamPipeline &) = delete;

	const std::vector<ValueType> &output_types() const {
		return out_types_;
	}
	const std::vector<std::string> &output_names() const {
		return out_names_;
	}
	void Poll() {
	}
	bool CanSubmit() const;
	//! Queues one batch (host columns in the declared order; names and types checked). Returns once
	//! the work is queued; the caller's buffers may be reused immediately.
	void Submit(const std::vector<vgpu_column> &columns, uint64_t rows);
	//! The oldest batch's stage when its download finished (or after waiting for it when `wait`);
	//! -1 when nothing is in flight (or, without waiting, not finished yet).
	int Take(bool wait);
	void Release(int stage);
	size_t in_flight() const {
		return fifo_.size();
	}

	struct OutView {
		const void *data = nullptr;
		const uint8_t *validity = nullptr;  // Arrow bitmap or nullptr
	};
	uint64_t StageRows(int stage) const {
		return stages_.at(stage).rows;
	}
	OutView StageOutput(int stage, size_t column) const;

private:
	struct Variant {
		std::shared_ptr<Module> module;
		std::vector<bool> out_nullable;
		int cb = 0;
	};
	struct Stage {
		std::vector<void *> in_host, in_dev, in_bitmap_host, in_bitmap_dev, in_valid_dev;
		std::vector<void *> out_dev, out_valid_dev, out_bitmap_dev, out_host, out_bitmap_host;
		std::vector<bool> out_nullable;
		cudaEvent_t h2d = nullptr, exec = nullptr, d2h = nullptr;
		uint64_t rows = 0;
	};
	const Variant &GetVariant(uint64_t null_mask);

	std::shared_ptr<PlanNode> plan_;
	std::vector<std::string> in_names_;
	std::vector<ValueType> in_types_;
	std::vector<std::string> out_names_;
	std::vector<ValueType> out_types_;
	uint64_t max_rows_;
	size_t depth_;
	std::map<uint64_t, Variant> variants_;
	std::vector<Stage> stages_;
	std::deque<int> free_, fifo_;
	cudaStream_t s_h2d_ = nullptr, s_exec_ = nullptr, s_d2h_ = nullptr;
	std::vector<void *> device_owned_, host_owned_;
	std::vector<size_t> window_cols_;      // output columns carrying RUNNING_SUM
	std::vector<void *> running_state_;    // per window column: the total so far (device, its type)
	void *running_scratch_ = nullptr;      // per-tile totals of the batch being scanned
};

} // namespace vgpu
