// runtime.hpp -- process-wide device state of the engine: the device and its properties, the
// stream-ordered device allocator with a hard budget, NVRTC compilation and the CUBIN module cache,
// the per-launch profiler and the launch counter.
#pragma once

#include <atomic>
#include <cstdint>
#include <list>
#include <memory>
#include <functional>
#include <map>
#include <tuple>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>

#include "common.hpp"

namespace vgpu {

struct DeviceProps {
	int device = 0;
	int sm_count = 0;
	int cc_major = 0;
	int cc_minor = 0;
	size_t smem_optin = 0;
	size_t l2_bytes = 0;
	size_t total_memory = 0;
	std::string name;
};

// ---- Device allocator -------------------------------------------------------------------------
//! Stream-ordered device memory (cudaMallocAsync on the device's memory pool, which keeps freed
//! blocks cached so steady-state execution does not go back to the driver) with a hard byte budget
//! checked before every allocation. The budget replaces the reference's per-plan cudaMalloc arena
//! (cuda_engine/src/gpu_executor_internal.hpp:37-59) and its headroom oracle (src/rmm_pool.cpp).
//! Page-locked host buffers for results copied to the host, reused across calls (the role of the
//! reference's PinnedBufferPool, src/pinned_buffer_pool.cpp:78-116): a device->host copy into pinned
//! memory runs at link speed, and page-locking a fresh buffer per result would cost more than the copy.
//! Buffers come back to the pool when the last owner lets go and are handed out again to any request
//! of at least half their size (sizes round up to eighths of a power of two), so results of varying
//! sizes reuse page-locked memory instead of pinning more: pinning costs far more than the copy, and
//! freeing page-locked memory synchronizes the device. At most the cache budget stays cached (16 GiB,
//! VECTOR_GPU_PINNED_CACHE_MB to change it); beyond it a returned buffer is freed.
class PinnedPool {
public:
	static PinnedPool &Get();
	std::shared_ptr<uint8_t> Acquire(size_t bytes);

private:
	void Return(void *p, size_t cls);
	size_t Budget();
	std::mutex mu_;
	std::multimap<size_t, void *> free_;
	size_t cached_ = 0;
	size_t budget_ = 0;
};

class DeviceAllocator {
public:
	void *Alloc(size_t bytes, cudaStream_t stream);
	void Free(void *ptr, cudaStream_t stream);
	void SetBudget(uint64_t bytes);
	uint64_t Budget();
	//! Maps `bytes` (within the budget) into the stream-ordered pool ahead of use, so requests that
	//! come later find free ranges without the pool remapping pages (a server about to run many
	//! requests at once reserves what they will hold together).
	void Reserve(uint64_t bytes, cudaStream_t stream);
	bool HasHeadroom(uint64_t bytes);
	vgpu_memory_stats Stats();
	//! Restarts the peak at the bytes in use now (the pool's reserve is unaffected).
	void ResetPeak();

private:
	void EnsureBudgetLocked();
	void GrowReserve(uint64_t in_use, cudaStream_t stream);
	void ReserveLocked(uint64_t want, cudaStream_t stream);
	std::mutex mu_;
	bool budget_set_ = false;
	uint64_t budget_ = 0;
	uint64_t reserve_target_ = 0;  // pool bytes kept mapped (see GrowReserve)
	uint64_t in_use_ = 0;
	uint64_t peak_ = 0;
	uint64_t allocations_ = 0;
	uint64_t failed_ = 0;
	std::unordered_map<void *, size_t> sizes_;
};

// ---- Reader marks -------------------------------------------------------------------------------
//! An event recorded on a stream after the last kernel of one execution that read long-lived device
//! buffers (committed cache columns, kept join tables). The free of such a buffer is enqueued on the
//! runtime's stream after a wait on every mark its readers left, so it is ordered after their kernels
//! without synchronizing the device or the readers' streams.
class StreamMark {
public:
	StreamMark() = default;
	StreamMark(const StreamMark &) = delete;
	StreamMark &operator=(const StreamMark &) = delete;
	~StreamMark() {
		if (ev_) cudaEventDestroy(ev_);  // a wait already enqueued on it still holds
	}
	//! A mark after the work enqueued on `stream` so far; nullptr when no event could be made, in which
	//! case `stream` has been synchronized instead (the reads are then over).
	static std::shared_ptr<StreamMark> After(cudaStream_t stream);
	//! True once the marked work has finished (a not-ready query leaves no error behind).
	bool Done() const;
	void WaitOn(cudaStream_t stream) const {
		cudaStreamWaitEvent(stream, ev_, 0);
	}

private:
	cudaEvent_t ev_ = nullptr;
};

//! Marks of the executions that read one buffer; finished marks are dropped as new ones arrive.
class ReaderMarks {
public:
	void Add(const std::shared_ptr<StreamMark> &m);
	//! Enqueues on `stream` a wait for every reader still marked.
	void WaitAll(cudaStream_t stream);

private:
	std::mutex mu_;
	std::vector<std::shared_ptr<StreamMark>> marks_;
};

// ---- Per-execution arena -----------------------------------------------------------------------
//! Every temporary one execution allocates, released stream-ordered when the execution ends (so the
//! release needs no device synchronization). `Release` hands a buffer's ownership to the caller.
class Arena {
public:
	explicit Arena(cudaStream_t stream) : stream_(stream) {
	}
	~Arena();
	Arena(const Arena &) = delete;
	Arena &operator=(const Arena &) = delete;

	void *Alloc(size_t bytes);
	template <typename T> T *AllocT(size_t count) {
		return static_cast<T *>(Alloc(count * sizeof(T)));
	}
	//! Stops tracking `ptr`: it survives the arena (used for results left on the device).
	void Release(void *ptr);
	//! Hands `ptr` to the caller when the arena owns it (true); false for memory it does not own or
	//! has already handed over.
	bool Take(void *ptr);
	void FreeNow(void *ptr);
	cudaStream_t stream() const {
		return stream_;
	}

private:
	cudaStream_t stream_;
	std::vector<void *> owned_;
};

// ---- Compiled modules ----------------------------------------------------------------------------
struct Module {
	CUmodule module = nullptr;
	std::unordered_map<std::string, CUfunction> functions;  // guarded by mu (modules are shared across threads)
	std::mutex mu;
	size_t cubin_bytes = 0;
	CUfunction Get(const std::string &name);
};

//! NVRTC front end: source -> CUBIN for the running device's arch (sm_100a on B200), strict FP
//! (--fmad=false, so a*b+c rounds twice exactly as the CPU does), the shared device library
//! supplied as an in-memory header. Throws Error(VGPU_ERR_COMPILE) with the log.
std::vector<char> CompileToCubin(const std::string &source, const std::string &arch, std::string *log);

//! LRU of loaded modules keyed by SHA-256 of (source, options) -- KernelCache
//! (cuda_engine/src/kernel_cache.cpp:171-218) -- backed by an on-disk CUBIN cache
//! (VECTOR_GPU_KERNEL_CACHE_DIR). Blobs are opaque: written and loaded, never inspected.
class ModuleCache {
public:
	std::shared_ptr<Module> GetOrCompile(const std::string &source);
	//! The module for `memo_key` (a description that determines the generated source): the source is
	//! generated and hashed only the first time a key is seen in this process.
	std::shared_ptr<Module> GetOrCompileMemo(const std::string &memo_key, const std::function<std::string()> &source);
	vgpu_kernel_cache_stats Stats();

private:
	std::mutex mu_;
	std::unordered_map<std::string, std::shared_ptr<Module>> memo_;
	std::list<std::string> lru_;
	std::unordered_map<std::string, std::pair<std::shared_ptr<Module>, std::list<std::string>::iterator>> map_;
	vgpu_kernel_cache_stats stats_ {};
	static constexpr size_t kCapacity = 256;
};

// ---- Profiler --------------------------------------------------------------------------------------
struct LaunchRecord {
	std::string name;
	cudaEvent_t start = nullptr, stop = nullptr;
	uint64_t bytes = 0, rows = 0;
};

class Profiler {
public:
	bool enabled() const {
		return enabled_.load(std::memory_order_relaxed);
	}
	void Enable(bool on) {
		enabled_.store(on);
	}
	//! Returns an index to pass to End, or -1 when disabled.
	int Begin(const char *name, cudaStream_t stream, uint64_t bytes, uint64_t rows);
	void End(int index, cudaStream_t stream);
	//! Replaces a record's algorithmic bytes once the host knows them (after a later read-back).
	void SetBytes(int index, uint64_t bytes);
	std::vector<vgpu_kernel_timing> Collect();

private:
	std::atomic<bool> enabled_ {false};
	std::mutex mu_;
	std::vector<LaunchRecord> records_;
	std::vector<cudaEvent_t> free_events_;
	cudaEvent_t GetEventLocked();
};

//! RAII profile scope around one launch (or a short group of launches).
class LaunchScope {
public:
	LaunchScope(const char *name, cudaStream_t stream, uint64_t bytes = 0, uint64_t rows = 0);
	~LaunchScope();
	int index() const {
		return index_;
	}

private:
	int index_;
	cudaStream_t stream_;
};

// ---- Runtime singleton ---------------------------------------------------------------------------
class Runtime {
public:
	static Runtime &Get();

	void EnsureDevice();
	const DeviceProps &props();
	cudaStream_t default_stream();
	DeviceAllocator &allocator() {
		return allocator_;
	}
	ModuleCache &modules() {
		return modules_;
	}
	Profiler &profiler() {
		return profiler_;
	}
	void CountLaunch(uint64_t n = 1) {
		launches_.fetch_add(n, std::memory_order_relaxed);
	}
	uint64_t launches() const {
		return launches_.load();
	}
	void SetDevice(int device);
	std::string arch();

	//! Launches a kernel of a loaded module (driver API via cudaGetDriverEntryPoint, so the library
	//! has no link-time dependency on libcuda and loads on machines without a GPU).
	void LaunchModuleKernel(CUfunction f, dim3 grid, dim3 block, size_t smem, cudaStream_t stream, void **args);
	CUmodule LoadCubin(const void *image);
	CUfunction ModuleFunction(CUmodule m, const char *name);
	void UnloadModule(CUmodule m);
	int MaxActiveBlocks(CUfunction f, int block, size_t smem);

private:
	Runtime() = default;
	void LoadDriverEntryPoints();
	std::mutex mu_;
	bool initialized_ = false;
	std::atomic<bool> ready_ {false};  // initialized_, readable without mu_
	int requested_device_ = 0;
	DeviceProps props_;
	cudaStream_t stream_ = nullptr;
	DeviceAllocator allocator_;
	ModuleCache modules_;
	Profiler profiler_;
	std::atomic<uint64_t> launches_ {0};

	// driver entry points
	bool driver_loaded_ = false;
	CUresult (*cuModuleLoadData_)(CUmodule *, const void *) = nullptr;
	CUresult (*cuModuleGetFunction_)(CUfunction *, CUmodule, const char *) = nullptr;
	CUresult (*cuModuleUnload_)(CUmodule) = nullptr;
	CUresult (*cuLaunchKernel_)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
	                            CUstream, void **, void **) = nullptr;
	CUresult (*cuFuncSetAttribute_)(CUfunction, CUfunction_attribute, int) = nullptr;
	CUresult (*cuGetErrorString_)(CUresult, const char **) = nullptr;
	CUresult (*cuOccupancyMaxActiveBlocksPerMultiprocessor_)(int *, CUfunction, int, size_t) = nullptr;
	void DriverCheck(CUresult r, const char *what);
	// occupancy answers (and the shared-memory attribute set) per (function, block, dynamic shared
	// bytes): the driver queries cost tens of microseconds per query otherwise
	std::mutex occ_mu_;
	std::map<std::tuple<CUfunction, int, size_t>, int> occ_;
	std::map<CUfunction, size_t> smem_attr_;  // the dynamic shared-memory limit set per function
	void EnsureSmemAttribute(CUfunction f, size_t smem);
};

} // namespace vgpu
