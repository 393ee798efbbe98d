// noalloc.cu -- a group-by entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc: code running inside a host callback or a CUDA-graph-driven
// loop, a process whose memory is reserved up front by another allocator, or a caller holding a
// device-wide lock that an allocation (which may synchronize the device) would deadlock on. For them
// vgpu_group_by_count_sum_noalloc computes SELECT k, COUNT(*), SUM(v) GROUP BY k over a small key
// range with every temporary in the fixed array below; inputs and outputs are the caller's.
//
// The array is file-scope device memory: every GPU that loads this library holds it
// (kNoAllocMaxDomain * 16 + 8 bytes, about 1 MiB) until the process exits. Host code may not use the
// symbol itself as an address -- there it is only a host-side stand-in -- so the device address is
// looked up once per device with cudaGetSymbolAddress, with that device current. That address belongs
// to the device's context of the time: a cudaDeviceReset makes it stale, so the entry point is not for
// use after a reset in the same process. SUM(v) accumulates with FP64 atomics, so its last bits depend
// on the order they land in and vary between calls.
#include <cstdint>
#include <mutex>

#include <cuda_runtime.h>

#include "common.hpp"

namespace vgpu {

namespace {

constexpr uint32_t kNoAllocMaxDomain = 1u << 16;
constexpr int kMaxDevices = 64;
constexpr int kBlock = 256;

// [0, D): per-key counts; [D, 2D): per-key sums (double bits); [2D]: unused pad for alignment.
static __device__ __align__(256) unsigned long long g_noalloc_scratch[2 * kNoAllocMaxDomain + 1];

std::mutex g_setup_mu;
void *g_scratch_ptr[kMaxDevices] = {};

void *ScratchForCurrentDevice(int device) {
	std::lock_guard<std::mutex> lock(g_setup_mu);
	if (g_scratch_ptr[device] == nullptr) {
		void *ptr = nullptr;
		cudaError_t err = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
		if (err != cudaSuccess || ptr == nullptr) {
			cudaGetLastError();
			Fail(VGPU_ERR_CUDA, std::string("vgpu_group_by_count_sum_noalloc: cudaGetSymbolAddress failed: ") +
			                        cudaGetErrorString(err));
		}
		g_scratch_ptr[device] = ptr;
	}
	return g_scratch_ptr[device];
}

__global__ void ClearScratch(unsigned long long *scratch, uint32_t domain) {
	for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < 2 * domain; i += gridDim.x * blockDim.x) {
		scratch[i] = 0ull;
	}
}

__global__ void __launch_bounds__(kBlock) Accumulate(const int32_t *keys, const double *values, uint64_t n,
                                                     int32_t key_min, uint32_t domain, unsigned long long *scratch) {
	unsigned long long *counts = scratch;
	double *sums = reinterpret_cast<double *>(scratch + domain);
	for (uint64_t i = blockIdx.x * (uint64_t)kBlock + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kBlock) {
		const int64_t slot = static_cast<int64_t>(keys[i]) - key_min;
		if (slot < 0 || slot >= static_cast<int64_t>(domain)) continue; // outside the declared key range
		atomicAdd(&counts[slot], 1ull);
		atomicAdd(&sums[slot], values[i]);
	}
}

// One CTA: writes the non-empty groups in key order and their number.
__global__ void __launch_bounds__(1024) Compact(const unsigned long long *scratch, uint32_t domain, int32_t key_min,
                                                int32_t *out_keys, int64_t *out_counts, double *out_sums,
                                                uint64_t *out_groups) {
	__shared__ uint32_t warp_sums[32];
	const unsigned long long *counts = scratch;
	const double *sums = reinterpret_cast<const double *>(scratch + domain);
	const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
	uint64_t base = 0;
	for (uint32_t c0 = 0; c0 < domain; c0 += blockDim.x) {
		const uint32_t s = c0 + threadIdx.x;
		const bool live = s < domain && counts[s] != 0;
		const uint32_t ballot = __ballot_sync(0xffffffffu, live);
		if (lane == 0) warp_sums[warp] = __popc(ballot);
		__syncthreads();
		uint32_t before = 0, total = 0;
		for (int w = 0; w < static_cast<int>(blockDim.x >> 5); w++) {
			if (w < warp) before += warp_sums[w];
			total += warp_sums[w];
		}
		if (live) {
			const uint64_t pos = base + before + __popc(ballot & ((1u << lane) - 1u));
			out_keys[pos] = key_min + static_cast<int32_t>(s);
			out_counts[pos] = static_cast<int64_t>(counts[s]);
			out_sums[pos] = sums[s];
		}
		base += total;
		__syncthreads();
	}
	if (threadIdx.x == 0) *out_groups = base;
}

} // namespace

} // namespace vgpu

// The library-wide thread-local last-error buffer lives in abi.cpp; this entry point reports through it.
namespace vgpu {
void SetLastError(const std::string &message);
}

extern "C" vgpu_status vgpu_group_by_count_sum_noalloc(const int32_t *keys, const double *values, uint64_t n,
                                                       int32_t key_min, uint32_t domain, int32_t *out_keys,
                                                       int64_t *out_counts, double *out_sums, uint64_t *out_groups,
                                                       void *stream) {
	using namespace vgpu;
	try {
		if (domain == 0 || domain > kNoAllocMaxDomain) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "vgpu_group_by_count_sum_noalloc: domain " + std::to_string(domain) +
			                                    " is outside [1, " + std::to_string(kNoAllocMaxDomain) +
			                                    "], the size of its fixed scratch array");
		}
		if ((n > 0 && (keys == nullptr || values == nullptr)) || out_keys == nullptr || out_counts == nullptr ||
		    out_sums == nullptr || out_groups == nullptr) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "vgpu_group_by_count_sum_noalloc: null pointer argument");
		}
		int device = 0;
		VGPU_CUDA(cudaGetDevice(&device));
		if (device < 0 || device >= kMaxDevices) Fail(VGPU_ERR_INVALID_ARGUMENT, "device index out of range");
		auto *scratch = static_cast<unsigned long long *>(ScratchForCurrentDevice(device));
		cudaStream_t s = static_cast<cudaStream_t>(stream);
		ClearScratch<<<(2 * domain + kBlock - 1) / kBlock, kBlock, 0, s>>>(scratch, domain);
		if (n > 0) {
			int sms = 148;
			cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
			uint64_t grid = (n + kBlock - 1) / kBlock;
			grid = grid < static_cast<uint64_t>(sms) * 8 ? grid : static_cast<uint64_t>(sms) * 8;
			Accumulate<<<static_cast<unsigned>(grid), kBlock, 0, s>>>(keys, values, n, key_min, domain, scratch);
		}
		Compact<<<1, 1024, 0, s>>>(scratch, domain, key_min, out_keys, out_counts, out_sums, out_groups);
		VGPU_CUDA(cudaGetLastError());
		SetLastError("");
		return VGPU_OK;
	} catch (const Error &e) {
		SetLastError(e.what());
		return e.status();
	} catch (const std::exception &e) {
		SetLastError(e.what());
		return VGPU_ERR_INTERNAL;
	}
}
