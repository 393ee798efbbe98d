// runtime.cpp -- device selection, allocator, NVRTC + module cache, profiler.
#include "runtime.hpp"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <dlfcn.h>
#include <mutex>
#include <sys/stat.h>

#include <nvrtc.h>

namespace vgpu {

std::string Sha256Hex(const void *data, size_t n);

// The device library source, embedded at build time so NVRTC can include it by name.
#include "device_lib_embed.inc"

// ============================================================================================
// PinnedPool

PinnedPool &PinnedPool::Get() {
	static PinnedPool *p = new PinnedPool();
	return *p;
}

size_t PinnedPool::Budget() {
	if (budget_ == 0) {
		budget_ = 16ull << 30;
		if (const char *env = std::getenv("VECTOR_GPU_PINNED_CACHE_MB")) {
			const unsigned long long mb = std::strtoull(env, nullptr, 10);
			if (mb > 0) budget_ = static_cast<size_t>(mb) << 20;
		}
	}
	return budget_;
}

std::shared_ptr<uint8_t> PinnedPool::Acquire(size_t bytes) {
	// size class: at least 64 KiB, rounded up to an eighth of the power of two at or below it
	size_t cls = 64 * 1024;
	if (bytes > cls) {
		size_t top = 1;
		while ((top << 1) <= bytes) top <<= 1;
		const size_t step = std::max<size_t>(top / 8, 1);
		cls = (bytes + step - 1) / step * step;
	}
	void *p = nullptr;
	size_t got = cls;
	{
		std::lock_guard<std::mutex> lock(mu_);
		auto it = free_.lower_bound(cls);  // the smallest cached buffer that holds the request ...
		if (it != free_.end() && it->first <= 2 * cls) {  // ... unless it is over twice the size
			p = it->second;
			got = it->first;
			cached_ -= got;
			free_.erase(it);
		}
	}
	if (!p) VGPU_CUDA(cudaMallocHost(&p, cls));
	return std::shared_ptr<uint8_t>(static_cast<uint8_t *>(p), [this, got](uint8_t *q) { Return(q, got); });
}

void PinnedPool::Return(void *p, size_t cls) {
	{
		std::lock_guard<std::mutex> lock(mu_);
		if (cached_ + cls <= Budget()) {
			free_.emplace(cls, p);
			cached_ += cls;
			return;
		}
	}
	cudaFreeHost(p);
}

// ============================================================================================
// DeviceAllocator

void DeviceAllocator::EnsureBudgetLocked() {
	if (budget_set_) {
		return;
	}
	double fraction = 0.85;
	if (const char *env = std::getenv("VECTOR_GPU_VRAM_FRACTION")) {
		double f = std::atof(env);
		if (f > 0.0 && f <= 1.0) {
			fraction = f;
		}
	}
	size_t free_bytes = 0, total_bytes = 0;
	VGPU_CUDA(cudaMemGetInfo(&free_bytes, &total_bytes));
	budget_ = static_cast<uint64_t>(static_cast<double>(free_bytes) * fraction);
	budget_set_ = true;
}

// The stream-ordered pool keeps what it has mapped (release threshold at the maximum), but a request
// larger than any of its free ranges makes it unmap free blocks and map their pages again for the new
// range: UVM driver calls that blocked the calling thread for 30 ms to 1 s at a time on the B200s
// (seen with 4 GB partition intermediates). So the pool's reserve is kept at twice the peak bytes in
// use (within the budget, in 1 GiB steps), grown ahead of the request by one allocation released at
// once in stream order: requests then find a free range without remapping.
void DeviceAllocator::GrowReserve(uint64_t in_use, cudaStream_t stream) {
	constexpr uint64_t kStep = 1ull << 30;
	ReserveLocked(std::min<uint64_t>(budget_, (2 * in_use + kStep - 1) / kStep * kStep), stream);
}

void DeviceAllocator::Reserve(uint64_t bytes, cudaStream_t stream) {
	std::lock_guard<std::mutex> lock(mu_);
	EnsureBudgetLocked();
	ReserveLocked(std::min<uint64_t>(budget_, bytes), stream);
}

void DeviceAllocator::ReserveLocked(uint64_t want, cudaStream_t stream) {
	if (want <= reserve_target_) return;
	cudaMemPool_t pool;
	int device = 0;
	if (cudaGetDevice(&device) != cudaSuccess || cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) {
		cudaGetLastError();
		return;
	}
	uint64_t reserved = 0;
	cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
	reserve_target_ = want;
	if (reserved >= want) return;
	void *block = nullptr;
	if (cudaMallocAsync(&block, want - reserved, stream) == cudaSuccess) {
		cudaFreeAsync(block, stream);
	} else {
		cudaGetLastError();  // no room to grow ahead: requests map on demand, as before
	}
}

void *DeviceAllocator::Alloc(size_t bytes, cudaStream_t stream) {
	if (bytes == 0) {
		bytes = 16; // a valid, distinct pointer for empty columns
	}
	bytes = (bytes + 255) & ~size_t(255);
	{
		std::lock_guard<std::mutex> lock(mu_);
		EnsureBudgetLocked();
		if (in_use_ + bytes > budget_) {
			failed_++;
			Fail(VGPU_ERR_OUT_OF_MEMORY, "device memory budget exhausted: need " + std::to_string(bytes) +
			                                 " more bytes with " + std::to_string(in_use_) + " of " +
			                                 std::to_string(budget_) + " in use");
		}
		in_use_ += bytes;
		peak_ = std::max(peak_, in_use_);
		allocations_++;
		if (2 * in_use_ > reserve_target_) GrowReserve(in_use_, stream);
	}
	void *ptr = nullptr;
	cudaError_t err = cudaMallocAsync(&ptr, bytes, stream);
	if (err != cudaSuccess) {
		cudaGetLastError();
		std::lock_guard<std::mutex> lock(mu_);
		in_use_ -= bytes;
		failed_++;
		Fail(err == cudaErrorMemoryAllocation ? VGPU_ERR_OUT_OF_MEMORY : VGPU_ERR_CUDA,
		     std::string("cudaMallocAsync(") + std::to_string(bytes) + "): " + cudaGetErrorString(err));
	}
	std::lock_guard<std::mutex> lock(mu_);
	sizes_[ptr] = bytes;
	return ptr;
}

void DeviceAllocator::Free(void *ptr, cudaStream_t stream) {
	if (ptr == nullptr) {
		return;
	}
	size_t bytes = 0;
	{
		std::lock_guard<std::mutex> lock(mu_);
		auto it = sizes_.find(ptr);
		if (it == sizes_.end()) {
			return; // not ours: never free foreign memory
		}
		bytes = it->second;
		sizes_.erase(it);
		in_use_ -= bytes;
	}
	cudaFreeAsync(ptr, stream);
}

void DeviceAllocator::SetBudget(uint64_t bytes) {
	std::lock_guard<std::mutex> lock(mu_);
	if (bytes == 0) {
		budget_set_ = false;
		EnsureBudgetLocked();
	} else {
		budget_ = bytes;
		budget_set_ = true;
	}
}

uint64_t DeviceAllocator::Budget() {
	std::lock_guard<std::mutex> lock(mu_);
	EnsureBudgetLocked();
	return budget_;
}

bool DeviceAllocator::HasHeadroom(uint64_t bytes) {
	std::lock_guard<std::mutex> lock(mu_);
	EnsureBudgetLocked();
	return in_use_ + bytes <= budget_;
}

vgpu_memory_stats DeviceAllocator::Stats() {
	std::lock_guard<std::mutex> lock(mu_);
	EnsureBudgetLocked();
	vgpu_memory_stats s;
	s.budget_bytes = budget_;
	s.in_use_bytes = in_use_;
	s.peak_bytes = peak_;
	s.allocations = allocations_;
	s.failed_allocations = failed_;
	return s;
}

void DeviceAllocator::ResetPeak() {
	std::lock_guard<std::mutex> lock(mu_);
	peak_ = in_use_;
}

// ============================================================================================
// Arena

Arena::~Arena() {
	auto &alloc = Runtime::Get().allocator();
	for (void *p : owned_) {
		alloc.Free(p, stream_);
	}
}

void *Arena::Alloc(size_t bytes) {
	void *p = Runtime::Get().allocator().Alloc(bytes, stream_);
	owned_.push_back(p);
	return p;
}

void Arena::Release(void *ptr) {
	auto it = std::find(owned_.begin(), owned_.end(), ptr);
	if (it != owned_.end()) {
		owned_.erase(it);
	}
}

bool Arena::Take(void *ptr) {
	auto it = std::find(owned_.begin(), owned_.end(), ptr);
	if (it == owned_.end()) return false;
	owned_.erase(it);
	return true;
}

void Arena::FreeNow(void *ptr) {
	auto it = std::find(owned_.begin(), owned_.end(), ptr);
	if (it != owned_.end()) {
		owned_.erase(it);
		Runtime::Get().allocator().Free(ptr, stream_);
	}
}

// ============================================================================================
// NVRTC

// NVRTC is bound at run time from the CUDA toolkit the engine was built against (a full path, local
// symbols), not through the dynamic linker: a process that already holds another NVRTC of the same
// soname (PyTorch ships one) would otherwise hand the engine that copy, whose PTX assembler may not
// know the sm_100 instruction forms the generated kernels use. VGPU_NVRTC_LIBRARY overrides the path.
#ifndef VGPU_CUDA_LIB_DIR
#define VGPU_CUDA_LIB_DIR "/usr/local/cuda/lib64"
#endif

namespace {

struct NvrtcApi {
	decltype(&nvrtcCreateProgram) create = nullptr;
	decltype(&nvrtcCompileProgram) compile = nullptr;
	decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
	decltype(&nvrtcGetProgramLog) log = nullptr;
	decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
	decltype(&nvrtcGetCUBIN) cubin = nullptr;
	decltype(&nvrtcDestroyProgram) destroy = nullptr;
	decltype(&nvrtcGetErrorString) error_string = nullptr;
	decltype(&nvrtcVersion) version = nullptr;
};

const NvrtcApi &Nvrtc() {
	static std::mutex mu;
	static NvrtcApi api;
	static bool loaded = false;
	std::lock_guard<std::mutex> lock(mu);
	if (loaded) {
		return api;
	}
	const char *env = std::getenv("VGPU_NVRTC_LIBRARY");
	const std::string path = env ? env : VGPU_CUDA_LIB_DIR "/libnvrtc.so.12";
	void *h = dlopen(path.c_str(), RTLD_NOW | RTLD_LOCAL);
	if (!h) {
		const char *err = dlerror();
		Fail(VGPU_ERR_COMPILE, "cannot load NVRTC from " + path + ": " + (err ? err : "unknown error"));
	}
	NvrtcApi a;
	auto bind = [&](auto &fn, const char *name) {
		fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
		if (!fn) Fail(VGPU_ERR_COMPILE, std::string("NVRTC library ") + path + " lacks " + name);
	};
	bind(a.create, "nvrtcCreateProgram");
	bind(a.compile, "nvrtcCompileProgram");
	bind(a.log_size, "nvrtcGetProgramLogSize");
	bind(a.log, "nvrtcGetProgramLog");
	bind(a.cubin_size, "nvrtcGetCUBINSize");
	bind(a.cubin, "nvrtcGetCUBIN");
	bind(a.destroy, "nvrtcDestroyProgram");
	bind(a.error_string, "nvrtcGetErrorString");
	bind(a.version, "nvrtcVersion");
	api = a;
	loaded = true;
	return api;
}

} // namespace

#define VGPU_NVRTC(call)                                                                                      \
	do {                                                                                                       \
		nvrtcResult _r = (call);                                                                               \
		if (_r != NVRTC_SUCCESS) {                                                                             \
			Fail(VGPU_ERR_COMPILE, std::string(#call) + ": " + Nvrtc().error_string(_r));                      \
		}                                                                                                      \
	} while (0)

std::vector<char> CompileToCubin(const std::string &source, const std::string &arch, std::string *log_out) {
	const NvrtcApi &nv = Nvrtc();
	nvrtcProgram prog = nullptr;
	const char *header_sources[] = {kDeviceLibSource};
	const char *header_names[] = {"vgpu_device_lib.cuh"};
	VGPU_NVRTC(nv.create(&prog, source.c_str(), "vgpu_fused.cu", 1, header_sources, header_names));
	std::string arch_opt = "--gpu-architecture=" + arch;
	std::vector<const char *> opts = {arch_opt.c_str(), "--fmad=false", "-std=c++17", "-DVGPU_NVRTC=1",
	                                  "--extra-device-vectorization", "-lineinfo"};
	nvrtcResult r = nv.compile(prog, static_cast<int>(opts.size()), opts.data());
	size_t log_size = 0;
	nv.log_size(prog, &log_size);
	std::string log;
	if (log_size > 1) {
		log.resize(log_size);
		nv.log(prog, &log[0]);
	}
	if (log_out) {
		*log_out = log;
	}
	if (r != NVRTC_SUCCESS) {
		nv.destroy(&prog);
		Fail(VGPU_ERR_COMPILE, "NVRTC compilation failed:\n" + log + "\n--- generated source ---\n" + source);
	}
	size_t cubin_size = 0;
	VGPU_NVRTC(nv.cubin_size(prog, &cubin_size));
	std::vector<char> cubin(cubin_size);
	VGPU_NVRTC(nv.cubin(prog, cubin.data()));
	nv.destroy(&prog);
	return cubin;
}

// ============================================================================================
// ModuleCache

CUfunction Module::Get(const std::string &name) {
	std::lock_guard<std::mutex> lock(mu);
	auto it = functions.find(name);
	if (it != functions.end()) {
		return it->second;
	}
	CUfunction f = Runtime::Get().ModuleFunction(module, name.c_str());
	functions[name] = f;
	return f;
}

namespace {

std::string CacheDir() {
	if (const char *env = std::getenv("VECTOR_GPU_KERNEL_CACHE_DIR")) {
		return env;
	}
	const char *home = std::getenv("HOME");
	return std::string(home ? home : "/tmp") + "/.cache/vectisdb_b200/cubin";
}

void MakeDirs(const std::string &path) {
	std::string cur;
	std::stringstream ss(path);
	std::string part;
	if (!path.empty() && path[0] == '/') {
		cur = "/";
	}
	while (std::getline(ss, part, '/')) {
		if (part.empty()) {
			continue;
		}
		cur += part + "/";
		mkdir(cur.c_str(), 0755);
	}
}

bool ReadFile(const std::string &path, std::vector<char> &out) {
	std::ifstream f(path, std::ios::binary);
	if (!f) {
		return false;
	}
	f.seekg(0, std::ios::end);
	auto size = f.tellg();
	if (size <= 0) {
		return false;
	}
	out.resize(static_cast<size_t>(size));
	f.seekg(0);
	f.read(out.data(), size);
	return static_cast<bool>(f);
}

} // namespace

std::shared_ptr<Module> ModuleCache::GetOrCompileMemo(const std::string &memo_key,
                                                      const std::function<std::string()> &source) {
	{
		std::lock_guard<std::mutex> lock(mu_);
		auto it = memo_.find(memo_key);
		if (it != memo_.end()) {
			stats_.hits++;
			return it->second;
		}
	}
	auto module = GetOrCompile(source());
	std::lock_guard<std::mutex> lock(mu_);
	if (memo_.size() >= 4096) memo_.clear();
	memo_[memo_key] = module;
	return module;
}

std::shared_ptr<Module> ModuleCache::GetOrCompile(const std::string &source) {
	auto &rt = Runtime::Get();
	const std::string arch = rt.arch();
	// the generated source includes the device library by name: its text is part of the key too, so a
	// cached CUBIN built against another version of it is never reused
	static const std::string lib_hash = Sha256Hex(kDeviceLibSource, sizeof(kDeviceLibSource) - 1);
	const std::string keyed = source + "\n//arch=" + arch + " fmad=false lib=" + lib_hash;
	const std::string key = Sha256Hex(keyed.data(), keyed.size());
	{
		std::lock_guard<std::mutex> lock(mu_);
		auto it = map_.find(key);
		if (it != map_.end()) {
			lru_.splice(lru_.begin(), lru_, it->second.second);
			stats_.hits++;
			return it->second.first;
		}
		stats_.misses++;
	}
	std::vector<char> cubin;
	const std::string dir = CacheDir();
	const std::string path = dir + "/" + key + ".cubin";
	bool from_disk = ReadFile(path, cubin);
	if (!from_disk) {
		auto t0 = std::chrono::steady_clock::now();
		cubin = CompileToCubin(source, arch, nullptr);
		double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
		{
			std::lock_guard<std::mutex> lock(mu_);
			stats_.compiles++;
			stats_.compile_ms_total += ms;
		}
		MakeDirs(dir);
		const std::string tmp = path + ".tmp" + std::to_string(reinterpret_cast<uintptr_t>(&cubin));
		std::ofstream f(tmp, std::ios::binary);
		if (f) {
			f.write(cubin.data(), static_cast<std::streamsize>(cubin.size()));
			f.close();
			std::rename(tmp.c_str(), path.c_str());
		}
	}
	auto module = std::make_shared<Module>();
	try {
		module->module = rt.LoadCubin(cubin.data());
	} catch (const Error &) {
		if (!from_disk) {
			throw;
		}
		// A stale or truncated cache file: recompile once.
		std::remove(path.c_str());
		cubin = CompileToCubin(source, arch, nullptr);
		module->module = rt.LoadCubin(cubin.data());
	}
	module->cubin_bytes = cubin.size();
	std::lock_guard<std::mutex> lock(mu_);
	if (from_disk) {
		stats_.disk_hits++;
	}
	auto it = map_.find(key);
	if (it != map_.end()) {
		// Another thread loaded it meanwhile; keep theirs, drop ours.
		rt.UnloadModule(module->module);
		return it->second.first;
	}
	lru_.push_front(key);
	map_[key] = {module, lru_.begin()};
	while (map_.size() > kCapacity) {
		auto victim = lru_.back();
		lru_.pop_back();
		auto vit = map_.find(victim);
		if (vit != map_.end()) {
			// Modules in use elsewhere stay alive through their shared_ptr; the CUmodule is unloaded only
			// when the last user lets go (see ~ModuleHolder below via custom deleter semantics).
			map_.erase(vit);
		}
	}
	stats_.entries = map_.size();
	return module;
}

vgpu_kernel_cache_stats ModuleCache::Stats() {
	std::lock_guard<std::mutex> lock(mu_);
	stats_.entries = map_.size();
	return stats_;
}

// ============================================================================================
// Profiler

cudaEvent_t Profiler::GetEventLocked() {
	if (!free_events_.empty()) {
		cudaEvent_t e = free_events_.back();
		free_events_.pop_back();
		return e;
	}
	cudaEvent_t e = nullptr;
	VGPU_CUDA(cudaEventCreate(&e));
	return e;
}

int Profiler::Begin(const char *name, cudaStream_t stream, uint64_t bytes, uint64_t rows) {
	if (!enabled()) {
		return -1;
	}
	std::lock_guard<std::mutex> lock(mu_);
	LaunchRecord rec;
	rec.name = name;
	rec.bytes = bytes;
	rec.rows = rows;
	rec.start = GetEventLocked();
	rec.stop = GetEventLocked();
	cudaEventRecord(rec.start, stream);
	records_.push_back(rec);
	return static_cast<int>(records_.size() - 1);
}

void Profiler::End(int index, cudaStream_t stream) {
	if (index < 0) {
		return;
	}
	std::lock_guard<std::mutex> lock(mu_);
	if (index < static_cast<int>(records_.size())) {
		cudaEventRecord(records_[index].stop, stream);
	}
}

void Profiler::SetBytes(int index, uint64_t bytes) {
	if (index < 0) {
		return;
	}
	std::lock_guard<std::mutex> lock(mu_);
	if (index < static_cast<int>(records_.size())) {
		records_[index].bytes = bytes;
	}
}

std::vector<vgpu_kernel_timing> Profiler::Collect() {
	std::lock_guard<std::mutex> lock(mu_);
	std::vector<vgpu_kernel_timing> out;
	for (auto &rec : records_) {
		cudaEventSynchronize(rec.stop);
		float ms = 0.f;
		cudaEventElapsedTime(&ms, rec.start, rec.stop);
		vgpu_kernel_timing t;
		std::memset(&t, 0, sizeof(t));
		std::snprintf(t.name, sizeof(t.name), "%s", rec.name.c_str());
		t.ms = ms;
		t.bytes = rec.bytes;
		t.rows = rec.rows;
		out.push_back(t);
		free_events_.push_back(rec.start);
		free_events_.push_back(rec.stop);
	}
	records_.clear();
	return out;
}

LaunchScope::LaunchScope(const char *name, cudaStream_t stream, uint64_t bytes, uint64_t rows) : stream_(stream) {
	index_ = Runtime::Get().profiler().Begin(name, stream, bytes, rows);
	Runtime::Get().CountLaunch();
}

LaunchScope::~LaunchScope() {
	Runtime::Get().profiler().End(index_, stream_);
}

// ============================================================================================
// Runtime

Runtime &Runtime::Get() {
	static Runtime *rt = new Runtime(); // never destroyed: outlives static destructors that free memory
	return *rt;
}

void Runtime::SetDevice(int device) {
	std::lock_guard<std::mutex> lock(mu_);
	if (initialized_ && device != requested_device_) {
		Fail(VGPU_ERR_INVALID_ARGUMENT, "vgpu_set_device: the engine is already bound to device " +
		                                    std::to_string(requested_device_));
	}
	requested_device_ = device;
}

void Runtime::EnsureDevice() {
	// after initialization: no lock, and a device switch only when this thread's current device differs
	// (concurrent serving threads call this on every step)
	if (ready_.load(std::memory_order_acquire)) {
		int current = -1;
		if (cudaGetDevice(&current) != cudaSuccess || current != props_.device) VGPU_CUDA(cudaSetDevice(props_.device));
		return;
	}
	std::lock_guard<std::mutex> lock(mu_);
	if (initialized_) {
		VGPU_CUDA(cudaSetDevice(props_.device));
		return;
	}
	int count = 0;
	cudaError_t err = cudaGetDeviceCount(&count);
	if (err != cudaSuccess || count == 0) {
		cudaGetLastError();
		Fail(VGPU_ERR_CUDA, std::string("no CUDA device available: ") + cudaGetErrorString(err));
	}
	if (requested_device_ < 0 || requested_device_ >= count) {
		Fail(VGPU_ERR_INVALID_ARGUMENT, "device index out of range");
	}
	VGPU_CUDA(cudaSetDevice(requested_device_));
	cudaDeviceProp prop;
	VGPU_CUDA(cudaGetDeviceProperties(&prop, requested_device_));
	props_.device = requested_device_;
	props_.sm_count = prop.multiProcessorCount;
	props_.cc_major = prop.major;
	props_.cc_minor = prop.minor;
	props_.smem_optin = prop.sharedMemPerBlockOptin;
	props_.l2_bytes = prop.l2CacheSize;
	props_.total_memory = prop.totalGlobalMem;
	props_.name = prop.name;
	VGPU_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
	// Keep freed blocks in the pool: steady-state executions then allocate without driver calls.
	cudaMemPool_t pool;
	VGPU_CUDA(cudaDeviceGetDefaultMemPool(&pool, requested_device_));
	uint64_t threshold = UINT64_MAX;
	VGPU_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
	LoadDriverEntryPoints();
	initialized_ = true;
	ready_.store(true, std::memory_order_release);
}

const DeviceProps &Runtime::props() {
	EnsureDevice();
	return props_;
}

cudaStream_t Runtime::default_stream() {
	EnsureDevice();
	return stream_;
}

std::string Runtime::arch() {
	if (const char *env = std::getenv("VGPU_NVRTC_ARCH")) {
		return env;
	}
	EnsureDevice();
	// Blackwell datacenter parts take the arch-specific target (tcgen05/TMA features); others the
	// plain one. Only sm_100a is a supported deployment target of this engine.
	std::string a = "sm_" + std::to_string(props_.cc_major) + std::to_string(props_.cc_minor);
	if (props_.cc_major == 10 && props_.cc_minor == 0) {
		a += "a";
	}
	return a;
}

void Runtime::LoadDriverEntryPoints() {
	if (driver_loaded_) {
		return;
	}
	auto get = [](const char *name, void **fn) {
		cudaDriverEntryPointQueryResult q;
		cudaError_t err = cudaGetDriverEntryPoint(name, fn, cudaEnableDefault, &q);
		if (err != cudaSuccess || q != cudaDriverEntryPointSuccess || *fn == nullptr) {
			cudaGetLastError();
			Fail(VGPU_ERR_CUDA, std::string("driver entry point unavailable: ") + name);
		}
	};
	get("cuModuleLoadData", reinterpret_cast<void **>(&cuModuleLoadData_));
	get("cuModuleGetFunction", reinterpret_cast<void **>(&cuModuleGetFunction_));
	get("cuModuleUnload", reinterpret_cast<void **>(&cuModuleUnload_));
	get("cuLaunchKernel", reinterpret_cast<void **>(&cuLaunchKernel_));
	get("cuFuncSetAttribute", reinterpret_cast<void **>(&cuFuncSetAttribute_));
	get("cuGetErrorString", reinterpret_cast<void **>(&cuGetErrorString_));
	get("cuOccupancyMaxActiveBlocksPerMultiprocessor",
	    reinterpret_cast<void **>(&cuOccupancyMaxActiveBlocksPerMultiprocessor_));
	driver_loaded_ = true;
}

void Runtime::DriverCheck(CUresult r, const char *what) {
	if (r == CUDA_SUCCESS) {
		return;
	}
	const char *msg = "unknown";
	if (cuGetErrorString_) {
		cuGetErrorString_(r, &msg);
	}
	Fail(r == CUDA_ERROR_OUT_OF_MEMORY ? VGPU_ERR_OUT_OF_MEMORY : VGPU_ERR_CUDA, std::string(what) + ": " + msg);
}

CUmodule Runtime::LoadCubin(const void *image) {
	EnsureDevice();
	CUmodule m = nullptr;
	DriverCheck(cuModuleLoadData_(&m, image), "cuModuleLoadData");
	return m;
}

CUfunction Runtime::ModuleFunction(CUmodule m, const char *name) {
	CUfunction f = nullptr;
	DriverCheck(cuModuleGetFunction_(&f, m, name), "cuModuleGetFunction");
	return f;
}

void Runtime::UnloadModule(CUmodule m) {
	if (m && cuModuleUnload_) {
		cuModuleUnload_(m);
		std::lock_guard<std::mutex> lock(occ_mu_);
		occ_.clear();  // a later module's functions may reuse these handles
		smem_attr_.clear();
	}
}

void Runtime::EnsureSmemAttribute(CUfunction f, size_t smem) {
	if (smem <= 32 * 1024) return;
	{
		std::lock_guard<std::mutex> lock(occ_mu_);
		auto it = smem_attr_.find(f);
		if (it != smem_attr_.end() && it->second >= smem) return;
	}
	DriverCheck(cuFuncSetAttribute_(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, static_cast<int>(smem)),
	            "cuFuncSetAttribute(max dynamic smem)");
	std::lock_guard<std::mutex> lock(occ_mu_);
	smem_attr_[f] = smem;
}

void Runtime::LaunchModuleKernel(CUfunction f, dim3 grid, dim3 block, size_t smem, cudaStream_t stream, void **args) {
	EnsureSmemAttribute(f, smem);
	DriverCheck(cuLaunchKernel_(f, grid.x, grid.y, grid.z, block.x, block.y, block.z, static_cast<unsigned>(smem),
	                            reinterpret_cast<CUstream>(stream), args, nullptr),
	            "cuLaunchKernel");
}

int Runtime::MaxActiveBlocks(CUfunction f, int block, size_t smem) {
	const auto key = std::make_tuple(f, block, smem);
	{
		std::lock_guard<std::mutex> lock(occ_mu_);
		auto it = occ_.find(key);
		if (it != occ_.end()) return it->second;
	}
	EnsureSmemAttribute(f, smem);
	int n = 0;
	DriverCheck(cuOccupancyMaxActiveBlocksPerMultiprocessor_(&n, f, block, smem), "cuOccupancyMaxActiveBlocks");
	std::lock_guard<std::mutex> lock(occ_mu_);
	if (occ_.size() >= 4096) occ_.clear();  // bounded: functions of unloaded modules leave stale keys
	occ_[key] = n;
	return n;
}

// ---- Reader marks -------------------------------------------------------------------------------

std::shared_ptr<StreamMark> StreamMark::After(cudaStream_t stream) {
	auto m = std::make_shared<StreamMark>();
	if (cudaEventCreateWithFlags(&m->ev_, cudaEventDisableTiming) != cudaSuccess ||
	    cudaEventRecord(m->ev_, stream) != cudaSuccess) {
		cudaGetLastError();
		cudaStreamSynchronize(stream);
		return nullptr;
	}
	return m;
}

bool StreamMark::Done() const {
	const cudaError_t e = cudaEventQuery(ev_);
	if (e == cudaErrorNotReady) cudaGetLastError();  // a status, not an error: leave none behind
	return e != cudaErrorNotReady;
}

void ReaderMarks::Add(const std::shared_ptr<StreamMark> &m) {
	if (!m) return;
	std::lock_guard<std::mutex> lock(mu_);
	marks_.erase(std::remove_if(marks_.begin(), marks_.end(), [](const std::shared_ptr<StreamMark> &r) { return r->Done(); }),
	             marks_.end());
	marks_.push_back(m);
}

void ReaderMarks::WaitAll(cudaStream_t stream) {
	std::lock_guard<std::mutex> lock(mu_);
	for (auto &m : marks_) m->WaitOn(stream);
	marks_.clear();
}

} // namespace vgpu
