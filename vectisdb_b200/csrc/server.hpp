// server.hpp -- serving: admission against a device-memory budget and continuous batching.
//
// Requests (plans with their inputs) are queued on submit and admitted in arrival order whenever a
// worker slot is free and the request's estimated working set (the cost model's peak device bytes)
// fits in what the budget has left; the slots run on their own CUDA streams, so admitted requests
// overlap on the device, and a request that arrives while others run starts as soon as a slot and
// memory free up. When the head request's plan template is one the batch kernel takes, the queued
// requests of the same template join it (continuous batching) and run as one batched launch. The
// serial executor of the reference host (one request at a time) is this server with one slot and
// no batching.
#pragma once

#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "executor.hpp"

namespace vgpu {

struct ServerOptions {
	int slots = 4;
	uint64_t memory_budget = 0;  // 0 = min(120 GB, the allocator's budget)
	int batch_max = 64;          // 1 = never batch
};

struct RequestInfo {
	int status = 0;              // vgpu_status of the request
	std::string error;
	double queued_ms = 0;        // submit -> admission
	double run_ms = 0;           // admission -> completion
	uint64_t batch_size = 1;     // requests in the launch that ran it
	uint64_t estimated_bytes = 0;
};

struct ServerStats {
	uint64_t submitted = 0, completed = 0, failed = 0, rejected = 0;
	uint64_t batches = 0, batched_requests = 0;
	uint64_t in_flight = 0, queued = 0;
	uint64_t reserved_bytes = 0, peak_reserved_bytes = 0, budget_bytes = 0;
	uint64_t peak_in_flight = 0;
};

class Server {
public:
	explicit Server(const ServerOptions &options);
	~Server();
	Server(const Server &) = delete;
	Server &operator=(const Server &) = delete;

	//! Queues a request; returns its id. Host inputs must stay valid until Wait returns for it.
	uint64_t Submit(std::shared_ptr<PlanNode> plan, std::vector<vgpu_column> inputs, const ExecOptions &options);
	//! Blocks until the request is done (or timeout_ms passes: returns false). Moves the result out.
	bool Wait(uint64_t id, double timeout_ms, ExecResult *result, RequestInfo *info);
	ServerStats Stats();

private:
	struct Request;
	void WorkerLoop(int slot);
	std::vector<std::shared_ptr<Request>> AdmitLocked();
	uint64_t Estimate(const PlanNode &plan, const std::vector<vgpu_column> &inputs, const ExecOptions &options);

	ServerOptions options_;
	uint64_t budget_ = 0;
	std::mutex mu_;
	std::condition_variable work_cv_, done_cv_;
	std::deque<std::shared_ptr<Request>> queue_;
	std::map<uint64_t, std::shared_ptr<Request>> requests_;
	std::map<std::string, int> template_batches_;  // +1 batches, -1 does not
	uint64_t next_id_ = 1;
	uint64_t reserved_ = 0;
	bool stop_ = false;
	ServerStats stats_;
	std::vector<std::thread> workers_;
};

} // namespace vgpu
