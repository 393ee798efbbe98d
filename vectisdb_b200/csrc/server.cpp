// server.cpp -- see server.hpp.
#include "server.hpp"

#include <algorithm>
#include <chrono>
#include <cstdlib>

#include "batch.hpp"
#include "column_cache.hpp"
#include "cost_model.hpp"

namespace vgpu {

using Clock = std::chrono::steady_clock;

struct Server::Request {
	uint64_t id = 0;
	std::shared_ptr<PlanNode> plan;
	std::vector<vgpu_column> inputs;
	ExecOptions options;
	uint64_t est = 0;
	std::string tmpl;  // batch template ("" = not the batch form)
	Clock::time_point submitted, admitted, finished;
	bool done = false;
	ExecResult result;
	RequestInfo info;
};

namespace {

double Ms(Clock::time_point a, Clock::time_point b) {
	return std::chrono::duration<double, std::milli>(b - a).count();
}

} // namespace

Server::Server(const ServerOptions &options) : options_(options) {
	if (options_.slots < 1) options_.slots = 1;
	if (options_.batch_max < 1) options_.batch_max = 1;
	auto &rt = Runtime::Get();
	rt.EnsureDevice();
	const uint64_t allocator_budget = rt.allocator().Stats().budget_bytes;
	const uint64_t default_budget = 120ull << 30;
	budget_ = options_.memory_budget ? options_.memory_budget : std::min(default_budget, allocator_budget);
	stats_.budget_bytes = budget_;
	// Concurrent requests hold more device memory together than one at a time, and a pool that has to
	// grow or remap pages while they run stalls every slot's allocations: map half the admission
	// budget up front (what admitted requests hold at once stays under the budget).
	if (options_.slots > 1) {
		rt.allocator().Reserve(budget_ / 2, rt.default_stream());
		VGPU_CUDA(cudaStreamSynchronize(rt.default_stream()));
	}
	for (int s = 0; s < options_.slots; s++) workers_.emplace_back([this, s] { WorkerLoop(s); });
}

Server::~Server() {
	{
		std::lock_guard<std::mutex> lock(mu_);
		stop_ = true;
	}
	work_cv_.notify_all();
	for (auto &t : workers_) t.join();
	auto &al = Runtime::Get().allocator();
	for (auto &kv : requests_) {
		for (void *p : kv.second->result.device_buffers) {
			try {
				al.Free(p, kv.second->result.stream);
			} catch (...) {
			}
		}
	}
}

uint64_t Server::Estimate(const PlanNode &plan, const std::vector<vgpu_column> &inputs, const ExecOptions &options) {
	// what the execution allocates: cache-served and device-memory columns are borrowed, not copied
	return EstimateWorkingSetFor(plan, inputs, options.serve_whole_scan_from_cache).total_bytes;
}

uint64_t Server::Submit(std::shared_ptr<PlanNode> plan, std::vector<vgpu_column> inputs, const ExecOptions &options) {
	auto req = std::make_shared<Request>();
	req->plan = std::move(plan);
	req->inputs = std::move(inputs);
	req->options = options;
	req->options.no_sync = false;
	req->submitted = Clock::now();
	req->est = Estimate(*req->plan, req->inputs, req->options);
	req->info.estimated_bytes = req->est;
	// Only small requests batch: the batch launch pays off by sharing one launch among queries that are
	// each too small to fill the GPU; a large request's own kernels fill it at least as well and run
	// beside the other slots' work (VGPU_SERVE_BATCH_ROWS: the largest input that still batches).
	uint64_t rows = 0;
	for (auto &c : req->inputs) rows = std::max<uint64_t>(rows, c.row_count);
	static const uint64_t batch_rows = [] {
		const char *env = std::getenv("VGPU_SERVE_BATCH_ROWS");
		return env ? std::strtoull(env, nullptr, 10) : (1ull << 21);
	}();
	if (options_.batch_max > 1 && options.cache_chunk_index < 0 && rows <= batch_rows) {
		auto pb = PrepareBatch({req->plan});
		if (pb->plans[0].scan) req->tmpl = pb->plans[0].sig_base;
	}
	std::lock_guard<std::mutex> lock(mu_);
	req->id = next_id_++;
	requests_[req->id] = req;
	stats_.submitted++;
	if (req->est > budget_) {
		req->done = true;
		req->finished = req->admitted = req->submitted;
		req->info.status = VGPU_ERR_OUT_OF_MEMORY;
		req->info.error = "serving: estimated working set of " + std::to_string(req->est) +
		                  " bytes exceeds the admission budget of " + std::to_string(budget_) + " bytes";
		stats_.rejected++;
		done_cv_.notify_all();
		return req->id;
	}
	queue_.push_back(req);
	work_cv_.notify_one();
	return req->id;
}

// Admission, in arrival order: the head request when it fits in what the budget has left (or when
// nothing runs, so a request below the budget always gets in); then, if its template batches, the
// queued requests of the same template that also fit.
std::vector<std::shared_ptr<Server::Request>> Server::AdmitLocked() {
	std::vector<std::shared_ptr<Request>> job;
	if (queue_.empty()) return job;
	auto head = queue_.front();
	if (reserved_ + head->est > budget_ && reserved_ > 0) return job;
	queue_.pop_front();
	job.push_back(head);
	reserved_ += head->est;
	if (options_.batch_max > 1 && !head->tmpl.empty() && template_batches_[head->tmpl] > 0) {
		for (auto it = queue_.begin(); it != queue_.end() && static_cast<int>(job.size()) < options_.batch_max;) {
			auto &r = *it;
			if (r->tmpl == head->tmpl && r->options.output_on_device == head->options.output_on_device &&
			    r->options.serve_whole_scan_from_cache == head->options.serve_whole_scan_from_cache &&
			    reserved_ + r->est <= budget_) {
				reserved_ += r->est;
				job.push_back(r);
				it = queue_.erase(it);
			} else {
				++it;
			}
		}
	}
	const auto now = Clock::now();
	for (auto &r : job) r->admitted = now;
	return job;
}

void Server::WorkerLoop(int slot) {
	(void)slot;
	cudaStream_t stream = nullptr;
	try {
		Runtime::Get().EnsureDevice();
		VGPU_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
	} catch (...) {
		return;
	}
	while (true) {
		std::vector<std::shared_ptr<Request>> job;
		{
			std::unique_lock<std::mutex> lock(mu_);
			work_cv_.wait(lock, [&] {
				if (stop_) return true;
				if (queue_.empty()) return false;
				return reserved_ == 0 || reserved_ + queue_.front()->est <= budget_;
			});
			if (stop_ && queue_.empty()) break;
			job = AdmitLocked();
			if (job.empty()) continue;
			stats_.in_flight += job.size();
			stats_.peak_in_flight = std::max(stats_.peak_in_flight, stats_.in_flight);
			stats_.peak_reserved_bytes = std::max(stats_.peak_reserved_bytes, reserved_);
		}
		// Run the job: a template whose batching is still unknown runs its first request through the
		// batch path alone to learn whether the batch kernel takes it.
		const auto &head = job.front();
		bool learn = false;
		bool as_batch = job.size() > 1;
		if (!as_batch && options_.batch_max > 1 && !head->tmpl.empty()) {
			std::lock_guard<std::mutex> lock(mu_);
			learn = template_batches_[head->tmpl] == 0;
			as_batch = learn;
		}
		int batched = 0;  // +1: the batch form took the job, -1: it ran one by one
		std::vector<ExecResult> results(job.size());
		std::vector<int> status(job.size(), VGPU_OK);
		std::vector<std::string> errors(job.size());
		if (as_batch) {
			try {
				std::vector<std::shared_ptr<PlanNode>> plans;
				std::vector<std::vector<vgpu_column>> ins;
				for (auto &r : job) {
					plans.push_back(r->plan);
					ins.push_back(r->inputs);
				}
				BatchOptions bo;
				bo.use_graph = false;  // compositions change from launch to launch
				BatchStats st;
				results = ExecutePrepared(*PrepareBatch(plans), ins, head->options, bo, stream, &st);
				batched = st.batched > 0 ? 1 : -1;
			} catch (const Error &e) {
				for (size_t i = 0; i < job.size(); i++) {
					status[i] = e.status();
					errors[i] = e.what();
				}
			} catch (const std::exception &e) {
				for (size_t i = 0; i < job.size(); i++) {
					status[i] = VGPU_ERR_INTERNAL;
					errors[i] = e.what();
				}
			}
		} else {
			for (size_t i = 0; i < job.size(); i++) {
				try {
					results[i] = ExecutePlan(*job[i]->plan, job[i]->inputs, job[i]->options, stream);
				} catch (const Error &e) {
					status[i] = e.status();
					errors[i] = e.what();
				} catch (const std::exception &e) {
					status[i] = VGPU_ERR_INTERNAL;
					errors[i] = e.what();
				}
			}
		}
		cudaStreamSynchronize(stream);
		const auto now = Clock::now();
		{
			std::lock_guard<std::mutex> lock(mu_);
			if (learn && batched != 0) template_batches_[head->tmpl] = batched;
			for (size_t i = 0; i < job.size(); i++) {
				auto &r = job[i];
				reserved_ -= r->est;
				r->result = std::move(results[i]);
				r->info.status = status[i];
				r->info.error = errors[i];
				r->info.batch_size = job.size();
				r->info.queued_ms = Ms(r->submitted, r->admitted);
				r->info.run_ms = Ms(r->admitted, now);
				r->finished = now;
				r->done = true;
				stats_.completed++;
				if (status[i] != VGPU_OK) stats_.failed++;
			}
			stats_.in_flight -= job.size();
			if (job.size() > 1) {
				stats_.batches++;
				stats_.batched_requests += job.size();
			}
		}
		done_cv_.notify_all();
		work_cv_.notify_all();
	}
	if (stream) cudaStreamDestroy(stream);
}

bool Server::Wait(uint64_t id, double timeout_ms, ExecResult *result, RequestInfo *info) {
	std::unique_lock<std::mutex> lock(mu_);
	auto it = requests_.find(id);
	if (it == requests_.end()) Fail(VGPU_ERR_INVALID_ARGUMENT, "serving: unknown or already collected request id");
	auto req = it->second;
	auto ready = [&] { return req->done; };
	if (timeout_ms < 0) {
		done_cv_.wait(lock, ready);
	} else if (!done_cv_.wait_for(lock, std::chrono::duration<double, std::milli>(timeout_ms), ready)) {
		return false;
	}
	if (result) *result = std::move(req->result);
	if (info) *info = req->info;
	requests_.erase(id);
	return true;
}

ServerStats Server::Stats() {
	std::lock_guard<std::mutex> lock(mu_);
	ServerStats s = stats_;
	s.queued = queue_.size();
	s.reserved_bytes = reserved_;
	return s;
}

} // namespace vgpu
