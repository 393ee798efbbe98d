// kernels.cu -- precompiled device primitives (see kernels.hpp).
#include "kernels.hpp"

#include <algorithm>

#include <type_traits>

#include <utility>

#include "device_lib.cuh"

namespace vgpu {
namespace kern {

using namespace vgpu_dev;

namespace {

constexpr int kScanBlock = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanBlock * kScanItems;

unsigned GridFor(uint64_t n, int block) {
	uint64_t g = (n + block - 1) / block;
	if (g == 0) {
		g = 1;
	}
	const uint64_t cap = static_cast<uint64_t>(Runtime::Get().props().sm_count) * 32;
	return static_cast<unsigned>(g < cap ? g : cap);
}

template <typename T> __device__ __forceinline__ T BlockScanExclusive(T v, T *scratch /*33*/, T *total) {
	const int lane = threadIdx.x & 31;
	const int warp = threadIdx.x >> 5;
	const int nwarps = blockDim.x >> 5;
	T x = v;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		T y = __shfl_up_sync(0xffffffffu, x, o);
		if (lane >= o) x += y;
	}
	if (lane == 31) scratch[warp] = x;
	__syncthreads();
	if (warp == 0) {
		T w = (lane < nwarps) ? scratch[lane] : T(0);
		T s = w;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			T y = __shfl_up_sync(0xffffffffu, s, o);
			if (lane >= o) s += y;
		}
		if (lane < nwarps) scratch[lane] = s - w;
		if (lane == 31) scratch[32] = s;
	}
	__syncthreads();
	T r = scratch[warp] + x - v;
	*total = scratch[32];
	__syncthreads();
	return r;
}

template <typename T> __global__ void __launch_bounds__(kScanBlock) ScanTileSums(const T *in, uint64_t n, T *sums) {
	__shared__ T scratch[33];
	const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile + static_cast<uint64_t>(threadIdx.x) * kScanItems;
	T local = 0;
#pragma unroll
	for (int i = 0; i < kScanItems; i++) {
		if (base + i < n) local += in[base + i];
	}
	T total;
	BlockScanExclusive<T>(local, scratch, &total);
	if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// Single CTA: exclusive scan of the tile sums in place, grand total to *total.
template <typename T> __global__ void __launch_bounds__(1024) ScanSums(T *sums, uint64_t count, T *total) {
	__shared__ T scratch[33];
	T carry = 0;
	for (uint64_t c0 = 0; c0 < count; c0 += blockDim.x) {
		const uint64_t i = c0 + threadIdx.x;
		T v = i < count ? sums[i] : T(0);
		T chunk_total;
		T ex = BlockScanExclusive<T>(v, scratch, &chunk_total);
		if (i < count) sums[i] = carry + ex;
		carry += chunk_total;
	}
	if (threadIdx.x == 0 && total) *total = carry;
}

template <typename T>
__global__ void __launch_bounds__(kScanBlock) ScanApply(const T *in, T *out, uint64_t n, const T *sums) {
	__shared__ T scratch[33];
	const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kScanTile + static_cast<uint64_t>(threadIdx.x) * kScanItems;
	T vals[kScanItems];
	T local = 0;
#pragma unroll
	for (int i = 0; i < kScanItems; i++) {
		vals[i] = base + i < n ? in[base + i] : T(0);
		local += vals[i];
	}
	T total;
	T run = BlockScanExclusive<T>(local, scratch, &total) + sums[blockIdx.x];
#pragma unroll
	for (int i = 0; i < kScanItems; i++) {
		if (base + i < n) out[base + i] = run;
		run += vals[i];
	}
}

// Values one CTA scans in one launch (16 per thread): the tile counts of a materialization of up to
// 2^24 rows. The three-launch form costs more in launches than in work at these sizes.
constexpr int kSmallScanItems = 16;
constexpr uint64_t kSmallScanMax = 1024 * kSmallScanItems;

// Single CTA, in place allowed: each thread loads a run of up to 16 consecutive values at once (all
// loads issued before any is used), the block scans the run sums, then each thread writes its run's
// exclusive prefixes from registers (every read precedes the block scan's barrier, every write follows).
template <typename T> __global__ void __launch_bounds__(1024) ScanSmall(const T *in, T *out, uint64_t n, T *total) {
	__shared__ T scratch[33];
	const uint64_t per = (n + blockDim.x - 1) / blockDim.x;
	const uint64_t b = static_cast<uint64_t>(threadIdx.x) * per;
	T vals[kSmallScanItems];
	T local = 0;
#pragma unroll
	for (int k = 0; k < kSmallScanItems; k++) {
		const uint64_t i = b + k;
		vals[k] = (static_cast<uint64_t>(k) < per && i < n) ? in[i] : T(0);
		local += vals[k];
	}
	T all;
	T run = BlockScanExclusive<T>(local, scratch, &all);
#pragma unroll
	for (int k = 0; k < kSmallScanItems; k++) {
		const uint64_t i = b + k;
		if (static_cast<uint64_t>(k) < per && i < n) {
			out[i] = run;
			run += vals[k];
		}
	}
	if (threadIdx.x == 0 && total) *total = all;
}

template <typename T> void ExclusiveScan(const T *in, T *out, uint64_t n, T *total, Arena &arena) {
	cudaStream_t s = arena.stream();
	if (n <= kSmallScanMax) {
		LaunchScope scope("scan_small", s, 2 * n * sizeof(T), n);
		ScanSmall<T><<<1, 1024, 0, s>>>(in, out, n, total);
		VGPU_CUDA(cudaGetLastError());
		return;
	}
	const uint64_t tiles = n == 0 ? 1 : (n + kScanTile - 1) / kScanTile;
	T *sums = arena.AllocT<T>(tiles);
	{
		LaunchScope scope("scan_tiles", s, n * sizeof(T), n);
		ScanTileSums<T><<<static_cast<unsigned>(tiles), kScanBlock, 0, s>>>(in, n, sums);
	}
	{
		LaunchScope scope("scan_sums", s, tiles * sizeof(T), tiles);
		ScanSums<T><<<1, 1024, 0, s>>>(sums, tiles, total);
	}
	if (n > 0) {
		LaunchScope scope("scan_apply", s, 2 * n * sizeof(T), n);
		ScanApply<T><<<static_cast<unsigned>(tiles), kScanBlock, 0, s>>>(in, out, n, sums);
	}
	VGPU_CUDA(cudaGetLastError());
}

__global__ void UnpackValidityKernel(const uint8_t *bitmap, uint8_t *bytes, uint64_t n) {
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
		bytes[i] = (bitmap[i >> 3] >> (i & 7)) & 1u;
	}
}

__global__ void PackValidityKernel(const uint8_t *bytes, uint8_t *bitmap, uint64_t n) {
	const uint64_t nbytes = (n + 7) / 8;
	for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nbytes; b += (uint64_t)gridDim.x * blockDim.x) {
		uint8_t v = 0;
		for (int k = 0; k < 8; k++) {
			uint64_t i = b * 8 + k;
			if (i < n && bytes[i]) v |= static_cast<uint8_t>(1u << k);
		}
		bitmap[b] = v;
	}
}

template <typename T> __global__ void GatherKernel(const T *src, const uint32_t *idx, uint64_t n, T *dst) {
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
		dst[i] = src[idx[i]];
	}
}

template <typename T> __global__ void WidenKernel(const T *src, uint64_t n, uint64_t *dst) {
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
		dst[i] = static_cast<uint64_t>(src[i]);
	}
}

// The CTA's smallest and largest value (unsigned) folded into out[0] / out[1] with one atomic pair per
// CTA: per-warp atomics on two words serialize at L2 once thousands of warps reach them.
template <typename U>
__device__ __forceinline__ void BlockMinMaxToGlobal(U mn, U mx, U *out) {
	__shared__ U smn[32], smx[32];
	for (int o = 16; o > 0; o >>= 1) {
		const U a = __shfl_xor_sync(0xffffffffu, mn, o);
		const U b = __shfl_xor_sync(0xffffffffu, mx, o);
		mn = a < mn ? a : mn;
		mx = b > mx ? b : mx;
	}
	const unsigned warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	if (lane == 0) {
		smn[warp] = mn;
		smx[warp] = mx;
	}
	__syncthreads();
	if (warp == 0) {
		const unsigned nw = (blockDim.x + 31) >> 5;
		mn = lane < nw ? smn[lane] : smn[0];
		mx = lane < nw ? smx[lane] : smx[0];
		for (int o = 16; o > 0; o >>= 1) {
			const U a = __shfl_xor_sync(0xffffffffu, mn, o);
			const U b = __shfl_xor_sync(0xffffffffu, mx, o);
			mn = a < mn ? a : mn;
			mx = b > mx ? b : mx;
		}
		if (lane == 0) {
			atomicMin(&out[0], mn);
			atomicMax(&out[1], mx);
		}
	}
}

__global__ void MinMaxKernel(const uint64_t *keys, uint64_t n, uint64_t *minmax) {
	unsigned long long mn = ~0ull, mx = 0;
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
		const unsigned long long k = keys[i];
		mn = k < mn ? k : mn;
		mx = k > mx ? k : mx;
	}
	BlockMinMaxToGlobal<unsigned long long>(mn, mx, reinterpret_cast<unsigned long long *>(minmax));
}

// Keys zero-extended to 64 bits and their range in one pass (the widening and the range the dense join
// tables need).
template <typename T> __global__ void WidenMinMaxKernel(const T *src, uint64_t n, uint64_t *dst, uint64_t *minmax) {
	unsigned long long mn = ~0ull, mx = 0;
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
		const unsigned long long k = static_cast<uint64_t>(src[i]);
		dst[i] = k;
		mn = k < mn ? k : mn;
		mx = k > mx ? k : mx;
	}
	BlockMinMaxToGlobal<unsigned long long>(mn, mx, reinterpret_cast<unsigned long long *>(minmax));
}

template <typename T> __global__ void MinMaxSignedKernel(const T *data, uint64_t n, int64_t *out) {
	int64_t mn = INT64_MAX, mx = INT64_MIN;
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
		const int64_t v = static_cast<int64_t>(data[i]);
		mn = v < mn ? v : mn;
		mx = v > mx ? v : mx;
	}
	for (int o = 16; o > 0; o >>= 1) {
		int64_t a = __shfl_xor_sync(0xffffffffu, mn, o);
		int64_t b = __shfl_xor_sync(0xffffffffu, mx, o);
		mn = a < mn ? a : mn;
		mx = b > mx ? b : mx;
	}
	if ((threadIdx.x & 31) == 0) {
		atomicMin(reinterpret_cast<long long *>(&out[0]), static_cast<long long>(mn));
		atomicMax(reinterpret_cast<long long *>(&out[1]), static_cast<long long>(mx));
	}
}

__global__ void InitMinMaxSignedKernel(int64_t *out) {
	out[0] = INT64_MAX;
	out[1] = INT64_MIN;
}

__global__ void InitMinMaxKernel(uint64_t *minmax) {
	minmax[0] = ~0ull;
	minmax[1] = 0ull;
}

__global__ void SubtractBiasKernel(uint64_t *keys, uint64_t n, uint64_t bias) {
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
		keys[i] -= bias;
	}
}

__global__ void IotaKernel(uint32_t *out, uint64_t n) {
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
		out[i] = static_cast<uint32_t>(i);
	}
}

// ---- LSD radix sort: 8-bit digits, stable warp-ordered local ranking ----------------------------

constexpr int kSortBlock = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortBlock * kSortItems;
constexpr int kSortWarps = kSortBlock / 32;

__device__ __forceinline__ uint32_t LaneMaskLt() {
	uint32_t m;
	asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
	return m;
}

__global__ void __launch_bounds__(kSortBlock) RadixHistKernel(const uint64_t *keys, uint64_t n, int shift,
                                                              uint32_t *hist, uint32_t ntiles) {
	__shared__ uint32_t counts[256];
	for (int i = threadIdx.x; i < 256; i += kSortBlock) counts[i] = 0;
	__syncthreads();
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const uint64_t base = static_cast<uint64_t>(blockIdx.x) * kSortTile + static_cast<uint64_t>(warp) * 32 * kSortItems;
#pragma unroll 4
	for (int k = 0; k < kSortItems; k++) {
		const uint64_t idx = base + static_cast<uint64_t>(k) * 32 + lane;
		const bool valid = idx < n;
		const uint32_t active = __ballot_sync(0xffffffffu, valid);
		if (valid) {
			const uint32_t d = static_cast<uint32_t>(keys[idx] >> shift) & 255u;
			const uint32_t peers = __match_any_sync(active, d);
			if ((peers & LaneMaskLt()) == 0) atomicAdd(&counts[d], static_cast<uint32_t>(__popc(peers)));
		}
	}
	__syncthreads();
	for (int d = threadIdx.x; d < 256; d += kSortBlock) hist[static_cast<uint64_t>(d) * ntiles + blockIdx.x] = counts[d];
}

// Scatter of one pass: the tile's keys are ranked stably (warp-ordered: a warp's items in order, warps
// in order), placed in shared memory in digit order, then written out by consecutive threads to
// consecutive positions of each digit's run, so the global stores are coalesced runs instead of one
// scattered store per key.
__global__ void __launch_bounds__(kSortBlock) RadixScatterKernel(const uint64_t *kin, const uint32_t *vin,
                                                                 uint64_t *kout, uint32_t *vout, uint64_t n, int shift,
                                                                 const uint32_t *offsets, uint32_t ntiles) {
	__shared__ uint32_t wcount[kSortWarps][256];
	__shared__ uint32_t tile_start[256];  // first local position of each digit in the tile
	__shared__ uint32_t global_start[256];
	__shared__ uint64_t skeys[kSortTile];  // the tile in digit order: keys, then (reused) values
	__shared__ uint8_t sdig[kSortTile];
	for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortBlock) (&wcount[0][0])[i] = 0;
	__syncthreads();
	const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
	const uint64_t tile0 = static_cast<uint64_t>(blockIdx.x) * kSortTile;
	const uint64_t base = tile0 + static_cast<uint64_t>(warp) * 32 * kSortItems;
	uint64_t keys[kSortItems];
	uint32_t vals[kSortItems];
	uint32_t rank[kSortItems];
#pragma unroll
	for (int k = 0; k < kSortItems; k++) {
		const uint64_t idx = base + static_cast<uint64_t>(k) * 32 + lane;
		const bool valid = idx < n;
		keys[k] = valid ? kin[idx] : 0ull;
		vals[k] = valid ? vin[idx] : 0u;
	}
#pragma unroll
	for (int k = 0; k < kSortItems; k++) {
		const uint64_t idx = base + static_cast<uint64_t>(k) * 32 + lane;
		const bool valid = idx < n;
		const uint32_t active = __ballot_sync(0xffffffffu, valid);
		uint32_t peers = 0, d = 0;
		if (valid) {
			d = static_cast<uint32_t>(keys[k] >> shift) & 255u;
			peers = __match_any_sync(active, d);
			rank[k] = wcount[warp][d] + static_cast<uint32_t>(__popc(peers & LaneMaskLt()));
		}
		__syncwarp();
		if (valid && (peers & LaneMaskLt()) == 0) wcount[warp][d] += static_cast<uint32_t>(__popc(peers));
		__syncwarp();
	}
	__syncthreads();
	if (threadIdx.x < 256) {  // per digit: warps' starts within the digit, the digit's count in the tile
		uint32_t run = 0;
		for (int w = 0; w < kSortWarps; w++) {
			const uint32_t c = wcount[w][threadIdx.x];
			wcount[w][threadIdx.x] = run;
			run += c;
		}
		tile_start[threadIdx.x] = run;  // the count, turned into a start below
		global_start[threadIdx.x] = offsets[static_cast<uint64_t>(threadIdx.x) * ntiles + blockIdx.x];
	}
	__syncthreads();
	if (threadIdx.x < 32) {  // exclusive scan of the 256 digit counts by one warp (8 per lane)
		uint32_t c[8], sum = 0;
#pragma unroll
		for (int j = 0; j < 8; j++) {
			c[j] = tile_start[threadIdx.x * 8 + j];
			sum += c[j];
		}
		uint32_t incl = sum;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
			if (lane >= o) incl += y;
		}
		uint32_t run = incl - sum;
#pragma unroll
		for (int j = 0; j < 8; j++) {
			tile_start[threadIdx.x * 8 + j] = run;
			run += c[j];
		}
	}
	__syncthreads();
	uint32_t lpos[kSortItems];
#pragma unroll
	for (int k = 0; k < kSortItems; k++) {
		const uint64_t idx = base + static_cast<uint64_t>(k) * 32 + lane;
		if (idx < n) {
			const uint32_t d = static_cast<uint32_t>(keys[k] >> shift) & 255u;
			lpos[k] = tile_start[d] + wcount[warp][d] + rank[k];
			skeys[lpos[k]] = keys[k];
			sdig[lpos[k]] = static_cast<uint8_t>(d);
		}
	}
	__syncthreads();
	const uint32_t valid_rows = static_cast<uint32_t>(n - tile0 < kSortTile ? n - tile0 : kSortTile);
	for (uint32_t i = threadIdx.x; i < valid_rows; i += kSortBlock) {
		const uint32_t d = sdig[i];
		kout[global_start[d] + (i - tile_start[d])] = skeys[i];
	}
	__syncthreads();
	uint32_t *svals = reinterpret_cast<uint32_t *>(skeys);
#pragma unroll
	for (int k = 0; k < kSortItems; k++) {
		const uint64_t idx = base + static_cast<uint64_t>(k) * 32 + lane;
		if (idx < n) svals[lpos[k]] = vals[k];
	}
	__syncthreads();
	for (uint32_t i = threadIdx.x; i < valid_rows; i += kSortBlock) {
		const uint32_t d = sdig[i];
		vout[global_start[d] + (i - tile_start[d])] = svals[i];
	}
}

// ---- join -----------------------------------------------------------------------------------------

// Load-balanced expansion of the match pairs (a merge path over the left rows' output offsets): each
// CTA owns a fixed tile of output positions, finds once which left rows those positions span, stages
// those rows' offsets in shared memory (when they fit) and every thread places its outputs by a search
// there; writes are coalesced across the tile. Left rows with no match share an offset with the next
// row, so "last row whose offset <= o" skips them.
constexpr int kExpandBlock = 256;
constexpr int kExpandItems = 8;
constexpr int kExpandTile = kExpandBlock * kExpandItems;
constexpr int kExpandWindow = 4096;

__device__ __forceinline__ uint64_t LastAtMost(const uint64_t *offsets, uint64_t a, uint64_t b, uint64_t o) {
	// offsets[a] <= o; returns the last index in [a, b) with offsets[index] <= o
	uint64_t lo = a + 1, hi = b;
	while (lo < hi) {
		const uint64_t mid = (lo + hi) >> 1;
		if (offsets[mid] <= o) lo = mid + 1;
		else hi = mid;
	}
	return lo - 1;
}

__global__ void __launch_bounds__(kExpandBlock) JoinExpandKernel(const uint64_t *offsets, const uint64_t *lower,
                                                                 uint64_t n_left, const uint32_t *sorted_perm,
                                                                 uint64_t total, uint32_t *out_left, uint32_t *out_right) {
	__shared__ uint64_t s_off[kExpandWindow];
	__shared__ uint64_t s_first, s_end;
	for (uint64_t tile = blockIdx.x; tile * kExpandTile < total; tile += gridDim.x) {
		const uint64_t o_begin = tile * kExpandTile;
		const uint64_t o_last = o_begin + kExpandTile < total ? o_begin + kExpandTile - 1 : total - 1;
		if (threadIdx.x == 0) {
			const uint64_t first = LastAtMost(offsets, 0, n_left, o_begin);
			s_first = first;
			s_end = LastAtMost(offsets, first, n_left, o_last) + 1;
		}
		__syncthreads();
		const uint64_t first = s_first, end = s_end, window = end - first;
		const bool staged = window <= kExpandWindow;
		if (staged) {
			for (uint64_t r = threadIdx.x; r < window; r += kExpandBlock) s_off[r] = offsets[first + r];
		}
		__syncthreads();
		for (int t = 0; t < kExpandItems; ++t) {
			const uint64_t o = o_begin + static_cast<uint64_t>(t) * kExpandBlock + threadIdx.x;
			if (o > o_last) break;
			uint64_t i;
			if (staged) {
				uint32_t lo = 1, hi = static_cast<uint32_t>(window);
				while (lo < hi) {
					const uint32_t mid = (lo + hi) >> 1;
					if (s_off[mid] <= o) lo = mid + 1;
					else hi = mid;
				}
				i = first + lo - 1;
			} else {
				i = LastAtMost(offsets, first, end, o);
			}
			const uint64_t j = o - (staged ? s_off[i - first] : offsets[i]);
			out_left[o] = static_cast<uint32_t>(i);
			out_right[o] = sorted_perm[lower[i] + j];
		}
		__syncthreads();
	}
}

// Each probe key's run in the sorted right keys through a radix directory (see vgpu_join_run): shift 0
// indexes the directory by the key itself, so the run is read, not searched.
__global__ void JoinRunKernel(const uint64_t *probe, uint64_t n_probe, const uint64_t *sorted, const uint32_t *dir,
                              uint64_t nb, uint32_t shift, uint64_t bias, uint64_t *lower, uint64_t *count) {
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_probe; i += (uint64_t)gridDim.x * blockDim.x) {
		const uint64_t k = probe[i] - bias;  // below the bias wraps past every bucket: no match
		const uint64_t b = k >> shift;
		uint64_t lo = 0, c = 0;
		if (b < nb) {
			uint64_t a = dir[b], e = dir[b + 1];
			if (shift != 0) {
				uint64_t hi = e;
				while (a < hi) {
					const uint64_t mid = (a + hi) >> 1;
					if (sorted[mid] < k) a = mid + 1;
					else hi = mid;
				}
				uint64_t up = a;
				hi = e;
				while (up < hi) {
					const uint64_t mid = (up + hi) >> 1;
					if (sorted[mid] <= k) up = mid + 1;
					else hi = mid;
				}
				e = up;
			}
			lo = a;
			c = e - a;
		}
		lower[i] = lo;
		count[i] = c;
	}
}

// Radix directory over a sorted key array (see vgpu_join_find): position i writes the entries of the
// buckets that start at i, so every one of the nb + 1 entries is written exactly once.
__global__ void JoinDirectoryKernel(const uint64_t *sorted, uint64_t n, uint32_t shift, uint64_t nb, uint32_t *dir) {
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i <= n; i += (uint64_t)gridDim.x * blockDim.x) {
		const uint64_t lo = i == 0 ? 0 : (sorted[i - 1] >> shift) + 1;
		const uint64_t hi = i == n ? nb : (sorted[i] >> shift);
		for (uint64_t b = lo; b <= hi && b <= nb; ++b) dir[b] = static_cast<uint32_t>(i);
	}
}

// Dense key tables: entry of (biased) key k = row index + 1, or (1 << 32 | value) with the row's
// value inlined; a key met twice counts as a duplicate (compare-and-swap from empty).
__global__ void JoinDenseRowsKernel(const uint64_t *keys, uint64_t n, uint64_t bias, uint32_t *table, uint32_t *dups) {
	uint32_t local = 0;
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
		if (atomicCAS(&table[keys[i] - bias], 0u, static_cast<uint32_t>(i + 1)) != 0u) local++;
	}
	if (local) atomicAdd(dups, local);
}

template <typename T>
__global__ void JoinDenseInlineKernel(const uint64_t *keys, const T *values, uint64_t n, uint64_t bias,
                                      unsigned long long *table, uint32_t *dups) {
	uint32_t local = 0;
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
		const unsigned long long e = (1ull << 32) | static_cast<unsigned long long>(values[i]);
		if (atomicCAS(&table[keys[i] - bias], 0ull, e) != 0ull) local++;
	}
	if (local) atomicAdd(dups, local);
}

template <typename T> __global__ void ValueBitsKernel(const T *values, uint64_t n, uint32_t *bounds) {
	unsigned int lo = 0xffffffffu, hi = 0;
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
		const unsigned int bits = static_cast<uint32_t>(values[i]);
		lo = bits < lo ? bits : lo;
		hi = bits > hi ? bits : hi;
	}
	BlockMinMaxToGlobal<unsigned int>(lo, hi, bounds);
}

// Compact inline table: entry = value bits - vmin in E (all ones = no key), filled by compare-and-swap
// from the marker; a key met twice counts in *dups. One-byte entries swap their 32-bit word (bounded
// retries while neighbours change it; running out counts as a duplicate, so the caller falls back).
template <typename T, typename E>
__global__ void JoinDenseCompactKernel(const uint64_t *keys, const T *values, uint64_t n, uint64_t bias, uint32_t vmin,
                                       E *table, uint32_t *dups) {
	uint32_t local = 0;
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
		const uint32_t entry = static_cast<uint32_t>(values[i]) - vmin;
		E *slot = table + (keys[i] - bias);
		if constexpr (sizeof(E) == 4) {
			if (atomicCAS(reinterpret_cast<unsigned int *>(slot), 0xffffffffu, entry) != 0xffffffffu) local++;
		} else if constexpr (sizeof(E) == 2) {
			if (atomicCAS(reinterpret_cast<unsigned short *>(slot), static_cast<unsigned short>(0xffffu),
			              static_cast<unsigned short>(entry)) != 0xffffu) {
				local++;
			}
		} else {
			unsigned int *word = reinterpret_cast<unsigned int *>(reinterpret_cast<uintptr_t>(slot) & ~uintptr_t(3));
			const uint32_t sh = static_cast<uint32_t>(reinterpret_cast<uintptr_t>(slot) & 3u) * 8u;
			uint32_t old = *reinterpret_cast<volatile unsigned int *>(word);
			bool done = false;
			for (int t = 0; t < 4096 && !done; ++t) {
				if (((old >> sh) & 0xffu) != 0xffu) break;  // taken: a duplicate key
				const uint32_t want = (old & ~(0xffu << sh)) | ((entry & 0xffu) << sh);
				const uint32_t prev = atomicCAS(word, old, want);
				done = prev == old;
				old = prev;
			}
			if (!done) local++;
		}
	}
	if (local) atomicAdd(dups, local);
}

__global__ void CountAdjacentEqualKernel(const uint64_t *sorted, uint64_t n, uint32_t *out) {
	uint32_t local = 0;
	for (uint64_t i = 1 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
		local += sorted[i] == sorted[i - 1] ? 1u : 0u;
	}
	if (local) atomicAdd(out, local);
}

// Longest run of equal keys in a sorted array: every run start finds its end by a galloping then a
// binary search, and the lengths meet in one atomic maximum.
__global__ void MaxRunLengthKernel(const uint64_t *sorted, uint64_t n, uint32_t *out) {
	uint32_t local = 0;
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
		const uint64_t k = sorted[i];
		if (i > 0 && sorted[i - 1] == k) continue;
		// gallop: `good` holds k, `bad` is the first probe past the run (or n)
		uint64_t good = i, step = 1, bad = n;
		while (good + step < n) {
			if (sorted[good + step] != k) {
				bad = good + step;
				break;
			}
			good += step;
			step <<= 1;
		}
		// the run ends in (good, bad]: binary search for the first position without k
		uint64_t a = good + 1, b = bad;
		while (a < b) {
			const uint64_t mid = (a + b) >> 1;
			if (sorted[mid] == k) a = mid + 1;
			else b = mid;
		}
		const uint64_t len = a - i;
		local = max(local, len > 0xffffffffull ? 0xffffffffu : static_cast<uint32_t>(len));
	}
	if (local) atomicMax(out, local);
}

// Work list of a partitioned aggregation pass. Item = (partition, first row, end row, split index or
// ~0). Partitions above `split_rows` rows become ceil(size / split_rows) chunks sharing one split
// index; everything is ordered longest first by size class (chunks of split partitions, then
// partitions by descending floor(log2(size))), so the longest items start first and the persistent
// CTAs finish together. Empty partitions produce no item. One CTA.
constexpr int kPlanBlock = 1024;

__global__ void __launch_bounds__(kPlanBlock) PlanWorkKernel(const uint32_t *offsets, uint64_t stride, uint32_t P,
                                                             const uint32_t *total_rows, uint32_t min_split,
                                                             uint32_t ctas, uint4 *items, uint32_t *counts,
                                                             uint32_t *split_info, uint32_t max_split) {
	__shared__ uint32_t cls_count[34];
	__shared__ uint32_t cls_cursor[34];
	__shared__ uint32_t n_split;
	__shared__ uint32_t split_rows;
	if (threadIdx.x < 34) cls_count[threadIdx.x] = 0;
	if (threadIdx.x == 0) {
		n_split = 0;
		// chunks small enough that every CTA gets several items on average
		const uint32_t total = *total_rows;
		// rounded up, so fewer than 4 * ctas partitions exceed it: the caller sizes the split tables from
		// that bound without reading the plan back
		const uint64_t quarter = 4ull * (ctas ? ctas : 1);
		const uint32_t even = static_cast<uint32_t>((total + quarter - 1) / quarter);
		split_rows = even > min_split ? even : min_split;
	}
	__syncthreads();
	const uint32_t total = *total_rows;
	const uint32_t S = split_rows;
	for (uint32_t p = threadIdx.x; p < P; p += blockDim.x) {
		const uint32_t r0 = offsets[static_cast<uint64_t>(p) * stride];
		const uint32_t r1 = p + 1 < P ? offsets[static_cast<uint64_t>(p + 1) * stride] : total;
		const uint32_t size = r1 - r0;
		if (size == 0) continue;
		const bool split = size > S;
		const uint32_t nch = split ? (size + S - 1) / S : 1u;
		const int cls = split ? 33 : 31 - __clz(size);
		atomicAdd(&cls_count[cls], nch);
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		uint32_t run = 0;
		for (int c = 33; c >= 0; --c) {
			cls_cursor[c] = run;
			run += cls_count[c];
		}
		counts[0] = run;
	}
	__syncthreads();
	for (uint32_t p = threadIdx.x; p < P; p += blockDim.x) {
		const uint32_t r0 = offsets[static_cast<uint64_t>(p) * stride];
		const uint32_t r1 = p + 1 < P ? offsets[static_cast<uint64_t>(p + 1) * stride] : total;
		const uint32_t size = r1 - r0;
		if (size == 0) continue;
		const bool split = size > S;
		const uint32_t nch = split ? (size + S - 1) / S : 1u;
		const int cls = split ? 33 : 31 - __clz(size);
		const uint32_t pos = atomicAdd(&cls_cursor[cls], nch);
		uint32_t sidx = ~0u;
		if (split) {
			sidx = atomicAdd(&n_split, 1u);
			if (sidx < max_split) {
				split_info[2 * sidx] = nch;
				split_info[2 * sidx + 1] = 0;
			}
		}
		for (uint32_t c = 0; c < nch; ++c) {
			const uint32_t a = r0 + c * S;
			const uint32_t b = (c + 1 == nch) ? r1 : a + S;
			items[pos + c] = make_uint4(p, a, b, sidx);
		}
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		counts[1] = n_split;
		counts[3] = *total_rows;  // read back with the split count: the partitioned row count
	}
}

} // namespace

void JoinDirectory(const uint64_t *sorted, uint64_t n, uint32_t shift, uint64_t nb, uint32_t *dir, cudaStream_t stream) {
	LaunchScope scope("join_directory", stream, n * 8 + (nb + 1) * 4, n);
	JoinDirectoryKernel<<<GridFor(n + 1, 256), 256, 0, stream>>>(sorted, n, shift, nb, dir);
	VGPU_CUDA(cudaGetLastError());
}

void JoinDenseRows(const uint64_t *keys, uint64_t n, uint64_t range, uint32_t *table, uint32_t *dups,
                   cudaStream_t stream, uint64_t bias) {
	LaunchScope scope("join_dense_table", stream, n * 12 + (range + 1) * 4, n);
	VGPU_CUDA(cudaMemsetAsync(table, 0, (range + 1) * 4, stream));
	VGPU_CUDA(cudaMemsetAsync(dups, 0, 4, stream));
	JoinDenseRowsKernel<<<GridFor(n, 256), 256, 0, stream>>>(keys, n, bias, table, dups);
	VGPU_CUDA(cudaGetLastError());
}

void JoinDenseInline(const uint64_t *keys, const void *values, size_t width, uint64_t n, uint64_t range,
                     uint64_t *table, uint32_t *dups, cudaStream_t stream, uint64_t bias) {
	LaunchScope scope("join_dense_table", stream, n * (8 + width) + (range + 1) * 8, n);
	VGPU_CUDA(cudaMemsetAsync(table, 0, (range + 1) * 8, stream));
	VGPU_CUDA(cudaMemsetAsync(dups, 0, 4, stream));
	auto *t = reinterpret_cast<unsigned long long *>(table);
	const unsigned grid = GridFor(n, 256);
	switch (width) {
	case 1:
		JoinDenseInlineKernel<uint8_t><<<grid, 256, 0, stream>>>(keys, static_cast<const uint8_t *>(values), n, bias, t, dups);
		break;
	case 2:
		JoinDenseInlineKernel<uint16_t><<<grid, 256, 0, stream>>>(keys, static_cast<const uint16_t *>(values), n, bias, t, dups);
		break;
	case 4:
		JoinDenseInlineKernel<uint32_t><<<grid, 256, 0, stream>>>(keys, static_cast<const uint32_t *>(values), n, bias, t, dups);
		break;
	default:
		Fail(VGPU_ERR_INTERNAL, "dense inline join table: value width must be 1, 2 or 4 bytes");
	}
	VGPU_CUDA(cudaGetLastError());
}

void ValueBits(const void *values, size_t width, uint64_t n, uint32_t *bounds, cudaStream_t stream) {
	VGPU_CUDA(cudaMemsetAsync(bounds, 0xff, 4, stream));
	VGPU_CUDA(cudaMemsetAsync(bounds + 1, 0, 4, stream));
	if (n == 0) return;
	LaunchScope scope("value_bits", stream, n * width, n);
	const unsigned grid = std::min<unsigned>(GridFor(n, 256), 1184);
	switch (width) {
	case 1: ValueBitsKernel<uint8_t><<<grid, 256, 0, stream>>>(static_cast<const uint8_t *>(values), n, bounds); break;
	case 2: ValueBitsKernel<uint16_t><<<grid, 256, 0, stream>>>(static_cast<const uint16_t *>(values), n, bounds); break;
	case 4: ValueBitsKernel<uint32_t><<<grid, 256, 0, stream>>>(static_cast<const uint32_t *>(values), n, bounds); break;
	default: Fail(VGPU_ERR_INTERNAL, "value bits: width must be 1, 2 or 4 bytes");
	}
	VGPU_CUDA(cudaGetLastError());
}

// Multi-match inline table: entry[k] = the key's match count in the low `cbits` bits, then one
// `vbits`-bit slot per match holding value bits - vmin (the matches of a key in no particular order).
// A match reserves its slot by adding 1 to the count and then ORs its value into that slot; a key
// with more than rmax matches (rmax < 2^cbits, so the count never wraps before it is seen) counts in
// *overflow and the table is not valid.
template <typename T, typename E>
__global__ void JoinDenseMultiKernel(const uint64_t *keys, const T *values, uint64_t n, uint64_t bias, uint32_t vmin,
                                     uint32_t vbits, uint32_t cbits, uint32_t rmax, E *table, uint32_t *overflow) {
	const E cmask = (E(1) << cbits) - 1;
	uint32_t local = 0;
	for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
		E *slot = table + (keys[i] - bias);
		const E old = atomicAdd(slot, E(1));
		const uint32_t j = static_cast<uint32_t>(old & cmask);
		if (j >= rmax) {
			local++;
			continue;
		}
		const E v = static_cast<E>(static_cast<uint32_t>(values[i]) - vmin);
		atomicOr(slot, v << (cbits + j * vbits));
	}
	if (local) atomicAdd(overflow, local);
}

namespace {
template <typename E>
void LaunchDenseCompact(const uint64_t *keys, const void *values, size_t vwidth, uint64_t n, uint64_t bias, uint32_t vmin,
                        E *table, uint32_t *dups, cudaStream_t stream) {
	const unsigned grid = GridFor(n, 256);
	switch (vwidth) {
	case 1:
		JoinDenseCompactKernel<uint8_t, E><<<grid, 256, 0, stream>>>(keys, static_cast<const uint8_t *>(values), n, bias,
		                                                             vmin, table, dups);
		break;
	case 2:
		JoinDenseCompactKernel<uint16_t, E><<<grid, 256, 0, stream>>>(keys, static_cast<const uint16_t *>(values), n,
		                                                              bias, vmin, table, dups);
		break;
	case 4:
		JoinDenseCompactKernel<uint32_t, E><<<grid, 256, 0, stream>>>(keys, static_cast<const uint32_t *>(values), n,
		                                                              bias, vmin, table, dups);
		break;
	default:
		Fail(VGPU_ERR_INTERNAL, "compact join table: value width must be 1, 2 or 4 bytes");
	}
}
} // namespace

void JoinDenseCompact(const uint64_t *keys, const void *values, size_t vwidth, uint64_t n, uint64_t range,
                      uint32_t vmin, void *table, size_t width, uint32_t *dups, cudaStream_t stream, uint64_t bias) {
	LaunchScope scope("join_dense_table", stream, n * (8 + vwidth) + (range + 1) * width, n);
	VGPU_CUDA(cudaMemsetAsync(table, 0xff, (range + 1) * width, stream));
	VGPU_CUDA(cudaMemsetAsync(dups, 0, 4, stream));
	switch (width) {
	case 1: LaunchDenseCompact(keys, values, vwidth, n, bias, vmin, static_cast<uint8_t *>(table), dups, stream); break;
	case 2: LaunchDenseCompact(keys, values, vwidth, n, bias, vmin, static_cast<uint16_t *>(table), dups, stream); break;
	case 4: LaunchDenseCompact(keys, values, vwidth, n, bias, vmin, static_cast<uint32_t *>(table), dups, stream); break;
	default: Fail(VGPU_ERR_INTERNAL, "compact join table: width must be 1, 2 or 4 bytes");
	}
	VGPU_CUDA(cudaGetLastError());
}

void JoinDenseMulti(const uint64_t *keys, const void *values, size_t vwidth, uint64_t n, uint64_t range, uint32_t vmin,
                    uint32_t vbits, uint32_t cbits, uint32_t rmax, void *table, bool wide, uint32_t *overflow,
                    cudaStream_t stream, uint64_t bias) {
	const size_t ew = wide ? 8 : 4;
	if (cbits < 1 || cbits > 3 || rmax >= (1u << cbits) || cbits + rmax * vbits > ew * 8) {
		Fail(VGPU_ERR_INTERNAL, "multi-match join table: slots do not fit the entry");
	}
	LaunchScope scope("join_dense_multi", stream, n * (8 + vwidth) + (range + 1) * ew, n);
	VGPU_CUDA(cudaMemsetAsync(table, 0, (range + 1) * ew, stream));
	VGPU_CUDA(cudaMemsetAsync(overflow, 0, 4, stream));
	const unsigned grid = GridFor(n, 256);
	auto launch = [&](auto *tab) {
		using E = std::remove_pointer_t<decltype(tab)>;
		switch (vwidth) {
		case 1:
			JoinDenseMultiKernel<uint8_t, E><<<grid, 256, 0, stream>>>(keys, static_cast<const uint8_t *>(values), n, bias,
			                                                           vmin, vbits, cbits, rmax, tab, overflow);
			break;
		case 2:
			JoinDenseMultiKernel<uint16_t, E><<<grid, 256, 0, stream>>>(keys, static_cast<const uint16_t *>(values), n,
			                                                            bias, vmin, vbits, cbits, rmax, tab, overflow);
			break;
		case 4:
			JoinDenseMultiKernel<uint32_t, E><<<grid, 256, 0, stream>>>(keys, static_cast<const uint32_t *>(values), n,
			                                                            bias, vmin, vbits, cbits, rmax, tab, overflow);
			break;
		default:
			Fail(VGPU_ERR_INTERNAL, "multi-match join table: value width must be 1, 2 or 4 bytes");
		}
	};
	if (wide) {
		launch(static_cast<unsigned long long *>(table));
	} else {
		launch(static_cast<unsigned int *>(table));
	}
	VGPU_CUDA(cudaGetLastError());
}

void CountAdjacentEqual(const uint64_t *sorted, uint64_t n, uint32_t *out, cudaStream_t stream) {
	VGPU_CUDA(cudaMemsetAsync(out, 0, 4, stream));
	if (n < 2) return;
	LaunchScope scope("count_adjacent_equal", stream, n * 8, n);
	CountAdjacentEqualKernel<<<GridFor(n, 256), 256, 0, stream>>>(sorted, n, out);
	VGPU_CUDA(cudaGetLastError());
}

void MaxRunLength(const uint64_t *sorted, uint64_t n, uint32_t *out, cudaStream_t stream) {
	VGPU_CUDA(cudaMemsetAsync(out, 0, 4, stream));
	if (n == 0) return;
	LaunchScope scope("max_run_length", stream, n * 8, n);
	MaxRunLengthKernel<<<GridFor(n, 256), 256, 0, stream>>>(sorted, n, out);
	VGPU_CUDA(cudaGetLastError());
}

uint64_t PlanWorkCapacity(uint32_t P, uint64_t rows, uint32_t min_split) {
	return static_cast<uint64_t>(P) + rows / (min_split ? min_split : 1) + 1;
}

namespace {
constexpr int kHeavyBlock = 1024;
constexpr uint32_t kHeavyBins = 1024;  // counts at or above the last bin share it
constexpr int kHeavyUnroll = 8;        // sample slots per thread and batch

__device__ uint64_t HeavyBlockSum(uint64_t v, uint64_t *scratch) {
	for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
	if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = v;
	__syncthreads();
	uint64_t total = 0;
	for (uint32_t w = 0; w < blockDim.x / 32; ++w) total += scratch[w];
	__syncthreads();
	return total;
}

__global__ void __launch_bounds__(kHeavyBlock) HeavySelectKernel(const uint64_t *keys, uint32_t *counts, uint32_t SC,
                                                                 uint32_t *hmap, uint32_t dbits, uint32_t *hkeys,
                                                                 uint32_t K, uint32_t min_count, bool require_cover,
                                                                 uint32_t *n_heavy) {
	__shared__ uint32_t hist[kHeavyBins];
	__shared__ uint64_t scratch[32];
	__shared__ uint32_t threshold, n_keys;
	const uint32_t dmask = (1u << dbits) - 1;
	constexpr uint32_t kWon = 0x80000000u;
	constexpr int kBatch = kHeavyUnroll;
	for (uint32_t b = threadIdx.x; b < kHeavyBins; b += blockDim.x) hist[b] = 0;
	if (threadIdx.x == 0) n_keys = 0;
	__syncthreads();
	// Every pass walks the table in batches of kBatch slots per thread, loads first (one CTA: the
	// loads of a batch must be in flight together). SC is a multiple of kBatch * blockDim.x, so every
	// lane of a warp runs every iteration.
	const uint32_t step = kBatch * blockDim.x;
	uint64_t sampled = 0;
	for (uint32_t base = threadIdx.x; base < SC; base += step) {
		uint32_t c[kBatch];
#pragma unroll
		for (int j = 0; j < kBatch; ++j) {
			const uint32_t s = base + j * blockDim.x;
			c[j] = keys[s] == ~0ull ? 0u : counts[s];
		}
#pragma unroll
		for (int j = 0; j < kBatch; ++j) {
			// most sampled keys share a few small counts: lanes of one bin add once
			const uint32_t bin = c[j] < kHeavyBins ? c[j] : kHeavyBins - 1;
			const uint32_t peers = __match_any_sync(0xffffffffu, bin);
			if (bin && static_cast<uint32_t>(__ffs(peers) - 1) == (threadIdx.x & 31)) atomicAdd(&hist[bin], __popc(peers));
			sampled += c[j];
		}
	}
	sampled = HeavyBlockSum(sampled, scratch);
	if (threadIdx.x == 0) {
		// the smallest threshold whose keys fit in K (bins summed from the top)
		uint32_t t = kHeavyBins, keys_at = 0;
		while (t > min_count && keys_at + hist[t - 1] <= K) {
			keys_at += hist[t - 1];
			--t;
		}
		threshold = t;
	}
	__syncthreads();
	const uint32_t t = threshold;
	// claim each candidate's partition; the winner marks its sample slot
	for (uint32_t base = threadIdx.x; base < SC; base += step) {
		uint64_t k[kBatch];
		uint32_t c[kBatch];
#pragma unroll
		for (int j = 0; j < kBatch; ++j) {
			k[j] = keys[base + j * blockDim.x];
			c[j] = counts[base + j * blockDim.x];
		}
#pragma unroll
		for (int j = 0; j < kBatch; ++j) {
			if (k[j] == ~0ull || c[j] < t) continue;
			const uint32_t p = static_cast<uint32_t>(k[j] >> dbits);
			if (atomicCAS(&hmap[p], ~0u, 0xfffe0000u | (static_cast<uint32_t>(k[j]) & dmask)) == ~0u) {
				counts[base + j * blockDim.x] = c[j] | kWon;
			}
		}
	}
	__syncthreads();
	uint64_t covered = 0;
	for (uint32_t base = threadIdx.x; base < SC; base += step) {
		uint32_t c[kBatch];
#pragma unroll
		for (int j = 0; j < kBatch; ++j) c[j] = counts[base + j * blockDim.x];
#pragma unroll
		for (int j = 0; j < kBatch; ++j) {
			if (!(c[j] & kWon)) continue;
			const uint32_t s = base + j * blockDim.x;
			const uint64_t k = keys[s];
			const uint32_t p = static_cast<uint32_t>(k >> dbits);
			const uint32_t idx = atomicAdd(&n_keys, 1u);
			if (idx < K) {
				hmap[p] = (idx << 16) | (static_cast<uint32_t>(k) & dmask);
				hkeys[idx] = static_cast<uint32_t>(k);
				covered += c[j] & ~kWon;
			} else {
				hmap[p] = ~0u;
				counts[s] = c[j] & ~kWon;
			}
		}
	}
	covered = HeavyBlockSum(covered, scratch);
	const bool drop = require_cover && covered * 10 < sampled;
	if (drop) {
		for (uint32_t s = threadIdx.x; s < SC; s += blockDim.x) {
			if (counts[s] & kWon) hmap[static_cast<uint32_t>(keys[s] >> dbits)] = ~0u;
		}
	}
	if (threadIdx.x == 0) *n_heavy = drop ? 0u : (n_keys < K ? n_keys : K);
}
} // namespace

void HeavySelect(const uint64_t *sample_keys, uint32_t *sample_counts, uint32_t SC, uint32_t *hmap, uint32_t dbits,
                 uint32_t *heavy_keys, uint32_t K, uint32_t min_count, bool require_cover, uint32_t *n_heavy,
                 cudaStream_t stream) {
	if (SC % (kHeavyBlock * kHeavyUnroll) != 0) {
		Fail(VGPU_ERR_INTERNAL, "heavy_select: sample table size must be a multiple of 8192");
	}
	LaunchScope scope("heavy_select", stream, static_cast<uint64_t>(SC) * 12, SC);
	HeavySelectKernel<<<1, kHeavyBlock, 0, stream>>>(sample_keys, sample_counts, SC, hmap, dbits, heavy_keys, K,
	                                                 min_count < 1 ? 1u : min_count, require_cover, n_heavy);
	VGPU_CUDA(cudaGetLastError());
}

void PlanWork(const uint32_t *offsets, uint64_t stride, uint32_t P, const uint32_t *total_rows, uint32_t min_split,
              uint32_t ctas, void *items, uint32_t *counts, uint32_t *split_info, uint32_t max_split,
              cudaStream_t stream) {
	LaunchScope scope("plan_work", stream, static_cast<uint64_t>(P) * 8, P);
	PlanWorkKernel<<<1, kPlanBlock, 0, stream>>>(offsets, stride, P, total_rows, min_split, ctas,
	                                             static_cast<uint4 *>(items), counts, split_info, max_split);
	VGPU_CUDA(cudaGetLastError());
}

void ExclusiveScanU32(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *total, Arena &arena) {
	ExclusiveScan<uint32_t>(in, out, n, total, arena);
}

void ExclusiveScanU64(const uint64_t *in, uint64_t *out, uint64_t n, uint64_t *total, Arena &arena) {
	ExclusiveScan<uint64_t>(in, out, n, total, arena);
}

void UnpackValidity(const uint8_t *bitmap, uint8_t *bytes, uint64_t n, cudaStream_t stream) {
	if (n == 0) return;
	LaunchScope scope("unpack_validity", stream, n / 8 + n, n);
	UnpackValidityKernel<<<GridFor(n, 256), 256, 0, stream>>>(bitmap, bytes, n);
	VGPU_CUDA(cudaGetLastError());
}

void PackValidity(const uint8_t *bytes, uint8_t *bitmap, uint64_t n, cudaStream_t stream) {
	if (n == 0) return;
	LaunchScope scope("pack_validity", stream, n + n / 8, n);
	PackValidityKernel<<<GridFor((n + 7) / 8, 256), 256, 0, stream>>>(bytes, bitmap, n);
	VGPU_CUDA(cudaGetLastError());
}

void Gather(const void *src, size_t width, const uint32_t *idx, uint64_t n, void *dst, cudaStream_t stream) {
	if (n == 0) return;
	LaunchScope scope("gather", stream, n * (width * 2 + 4), n);
	const unsigned grid = GridFor(n, 256);
	switch (width) {
	case 1:
		GatherKernel<uint8_t><<<grid, 256, 0, stream>>>(static_cast<const uint8_t *>(src), idx, n, static_cast<uint8_t *>(dst));
		break;
	case 2:
		GatherKernel<uint16_t><<<grid, 256, 0, stream>>>(static_cast<const uint16_t *>(src), idx, n, static_cast<uint16_t *>(dst));
		break;
	case 4:
		GatherKernel<uint32_t><<<grid, 256, 0, stream>>>(static_cast<const uint32_t *>(src), idx, n, static_cast<uint32_t *>(dst));
		break;
	case 8:
		GatherKernel<uint64_t><<<grid, 256, 0, stream>>>(static_cast<const uint64_t *>(src), idx, n, static_cast<uint64_t *>(dst));
		break;
	case 16:
		GatherKernel<uint4><<<grid, 256, 0, stream>>>(static_cast<const uint4 *>(src), idx, n, static_cast<uint4 *>(dst));
		break;
	default:
		Fail(VGPU_ERR_INTERNAL, "gather: unsupported width");
	}
	VGPU_CUDA(cudaGetLastError());
}

void WidenKeys(const void *src, size_t width, uint64_t n, uint64_t *dst, cudaStream_t stream) {
	if (n == 0) return;
	LaunchScope scope("widen_keys", stream, n * (width + 8), n);
	const unsigned grid = GridFor(n, 256);
	switch (width) {
	case 1:
		WidenKernel<uint8_t><<<grid, 256, 0, stream>>>(static_cast<const uint8_t *>(src), n, dst);
		break;
	case 2:
		WidenKernel<uint16_t><<<grid, 256, 0, stream>>>(static_cast<const uint16_t *>(src), n, dst);
		break;
	case 4:
		WidenKernel<uint32_t><<<grid, 256, 0, stream>>>(static_cast<const uint32_t *>(src), n, dst);
		break;
	case 8:
		WidenKernel<uint64_t><<<grid, 256, 0, stream>>>(static_cast<const uint64_t *>(src), n, dst);
		break;
	default:
		Fail(VGPU_ERR_INTERNAL, "widen: unsupported width");
	}
	VGPU_CUDA(cudaGetLastError());
}

void MinMaxU64(const uint64_t *keys, uint64_t n, uint64_t *minmax, cudaStream_t stream) {
	LaunchScope scope("minmax", stream, n * 8, n);
	InitMinMaxKernel<<<1, 1, 0, stream>>>(minmax);
	if (n > 0) {
		const unsigned grid = std::min<unsigned>(GridFor(n, 256), Runtime::Get().props().sm_count * 8);
		MinMaxKernel<<<grid, 256, 0, stream>>>(keys, n, minmax);
	}
	VGPU_CUDA(cudaGetLastError());
}

void WidenKeysMinMax(const void *src, size_t width, uint64_t n, uint64_t *dst, uint64_t *minmax, cudaStream_t stream) {
	InitMinMaxKernel<<<1, 1, 0, stream>>>(minmax);
	if (n == 0) {
		VGPU_CUDA(cudaGetLastError());
		return;
	}
	LaunchScope scope("widen_keys", stream, n * (width + 8), n);
	const unsigned grid = std::min<unsigned>(GridFor(n, 256), Runtime::Get().props().sm_count * 8);
	switch (width) {
	case 1:
		WidenMinMaxKernel<uint8_t><<<grid, 256, 0, stream>>>(static_cast<const uint8_t *>(src), n, dst, minmax);
		break;
	case 2:
		WidenMinMaxKernel<uint16_t><<<grid, 256, 0, stream>>>(static_cast<const uint16_t *>(src), n, dst, minmax);
		break;
	case 4:
		WidenMinMaxKernel<uint32_t><<<grid, 256, 0, stream>>>(static_cast<const uint32_t *>(src), n, dst, minmax);
		break;
	case 8:
		WidenMinMaxKernel<uint64_t><<<grid, 256, 0, stream>>>(static_cast<const uint64_t *>(src), n, dst, minmax);
		break;
	default:
		Fail(VGPU_ERR_INTERNAL, "widen: unsupported width");
	}
	VGPU_CUDA(cudaGetLastError());
}

void MinMaxSigned(const void *data, int type, uint64_t n, int64_t *out, cudaStream_t stream) {
	LaunchScope scope("minmax_signed", stream, n * 8, n);
	InitMinMaxSignedKernel<<<1, 1, 0, stream>>>(out);
	if (n > 0) {
		const unsigned grid = GridFor(n, 256);
		switch (static_cast<ValueType>(type)) {
		case ValueType::INT16:
			MinMaxSignedKernel<int16_t><<<grid, 256, 0, stream>>>(static_cast<const int16_t *>(data), n, out);
			break;
		case ValueType::INT32:
		case ValueType::DICTIONARY_STRING:
			MinMaxSignedKernel<int32_t><<<grid, 256, 0, stream>>>(static_cast<const int32_t *>(data), n, out);
			break;
		case ValueType::INT64:
			MinMaxSignedKernel<int64_t><<<grid, 256, 0, stream>>>(static_cast<const int64_t *>(data), n, out);
			break;
		case ValueType::BOOLEAN:
			MinMaxSignedKernel<uint8_t><<<grid, 256, 0, stream>>>(static_cast<const uint8_t *>(data), n, out);
			break;
		default:
			Fail(VGPU_ERR_INTERNAL, "min/max statistics need an integer column");
		}
	}
	VGPU_CUDA(cudaGetLastError());
}

void RadixSortPairs(uint64_t *keys, uint32_t *values, uint64_t *keys_alt, uint32_t *values_alt, uint64_t n, int bits,
                    Arena &arena) {
	if (n <= 1 || bits <= 0) return;
	cudaStream_t s = arena.stream();
	const uint64_t ntiles64 = (n + kSortTile - 1) / kSortTile;
	if (ntiles64 > 0xffffffffull) Fail(VGPU_ERR_UNSUPPORTED, "radix sort: too many rows");
	const uint32_t ntiles = static_cast<uint32_t>(ntiles64);
	uint32_t *hist = arena.AllocT<uint32_t>(static_cast<size_t>(ntiles) * 256);
	uint32_t *total = arena.AllocT<uint32_t>(1);
	uint64_t *kin = keys, *kout = keys_alt;
	uint32_t *vin = values, *vout = values_alt;
	const int passes = (bits + 7) / 8;
	for (int p = 0; p < passes; p++) {
		const int shift = 8 * p;
		{
			LaunchScope scope("radix_hist", s, n * 8, n);
			RadixHistKernel<<<ntiles, kSortBlock, 0, s>>>(kin, n, shift, hist, ntiles);
		}
		ExclusiveScanU32(hist, hist, static_cast<uint64_t>(ntiles) * 256, total, arena);
		{
			LaunchScope scope("radix_scatter", s, n * 24, n);
			RadixScatterKernel<<<ntiles, kSortBlock, 0, s>>>(kin, vin, kout, vout, n, shift, hist, ntiles);
		}
		VGPU_CUDA(cudaGetLastError());
		std::swap(kin, kout);
		std::swap(vin, vout);
	}
	if (kin != keys) {
		VGPU_CUDA(cudaMemcpyAsync(keys, kin, n * 8, cudaMemcpyDeviceToDevice, s));
		VGPU_CUDA(cudaMemcpyAsync(values, vin, n * 4, cudaMemcpyDeviceToDevice, s));
	}
}

void SubtractBias(uint64_t *keys, uint64_t n, uint64_t bias, cudaStream_t stream) {
	if (n == 0 || bias == 0) return;
	LaunchScope scope("subtract_bias", stream, n * 16, n);
	SubtractBiasKernel<<<GridFor(n, 256), 256, 0, stream>>>(keys, n, bias);
	VGPU_CUDA(cudaGetLastError());
}

void Iota(uint32_t *out, uint64_t n, cudaStream_t stream) {
	if (n == 0) return;
	LaunchScope scope("iota", stream, n * 4, n);
	IotaKernel<<<GridFor(n, 256), 256, 0, stream>>>(out, n);
	VGPU_CUDA(cudaGetLastError());
}

void JoinExpand(const uint64_t *offsets, const uint64_t *lower, uint64_t n_left, const uint32_t *sorted_perm,
                uint64_t total, uint32_t *out_left, uint32_t *out_right, cudaStream_t stream) {
	if (total == 0) return;
	LaunchScope scope("join_expand", stream, total * 8, total);
	const uint64_t tiles = (total + kExpandTile - 1) / kExpandTile;
	const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(tiles, 148ull * 8));
	JoinExpandKernel<<<grid, kExpandBlock, 0, stream>>>(offsets, lower, n_left, sorted_perm, total, out_left, out_right);
	VGPU_CUDA(cudaGetLastError());
}

void JoinRuns(const uint64_t *probe, uint64_t n_probe, const uint64_t *sorted, const uint32_t *dir, uint64_t nb,
              uint32_t shift, uint64_t bias, uint64_t *lower, uint64_t *count, cudaStream_t stream) {
	if (n_probe == 0) return;
	LaunchScope scope("join_runs", stream, n_probe * 24, n_probe);
	JoinRunKernel<<<GridFor(n_probe, 256), 256, 0, stream>>>(probe, n_probe, sorted, dir, nb, shift, bias, lower, count);
	VGPU_CUDA(cudaGetLastError());
}

// ---- running total (the stream pipeline's RUNNING_SUM window primitive) ----------------------------
//
// Three passes over tiles of 4096 values (1024 threads x 4 consecutive values): each tile's total; one
// block turning the totals into per-tile starting values that continue from the carried state; each
// tile's inclusive scan from its starting value. Integer values are summed as unsigned words of at
// least their width (wrap-around, truncated on store), floats in their own type.

namespace {

constexpr int kSumThreads = 1024;
constexpr int kSumItems = 4;
constexpr uint64_t kSumTile = uint64_t(kSumThreads) * kSumItems;

template <class T, class A> __device__ __forceinline__ A SumLoad(const T *p) {
	if constexpr (sizeof(T) == 2) {
		return static_cast<A>(static_cast<uint16_t>(*p));
	} else if constexpr (std::is_integral<T>::value) {
		return static_cast<A>(*p);
	} else {
		return *p;
	}
}

template <class T, class A> __device__ __forceinline__ void SumStore(T *p, A v) {
	*p = static_cast<T>(v);
}

// Block-wide scan of one value per thread (1024 threads): inclusive and exclusive prefixes and the
// block total, all in the same addition order.
template <class A> __device__ void SumBlockScan(A x, A *warp_sums, A &incl, A &excl, A &total) {
	const int lane = threadIdx.x & 31;
	const int warp = threadIdx.x >> 5;
	for (int d = 1; d < 32; d <<= 1) {
		const A y = __shfl_up_sync(0xffffffffu, x, d);
		if (lane >= d) x = static_cast<A>(x + y);
	}
	A prev = __shfl_up_sync(0xffffffffu, x, 1);
	if (lane == 31) warp_sums[warp] = x;
	__syncthreads();
	if (warp == 0) {
		A w = warp_sums[lane];
		for (int d = 1; d < 32; d <<= 1) {
			const A y = __shfl_up_sync(0xffffffffu, w, d);
			if (lane >= d) w = static_cast<A>(w + y);
		}
		warp_sums[lane] = w;
	}
	__syncthreads();
	if (warp == 0) {
		incl = x;
		excl = lane == 0 ? A(0) : prev;
	} else {
		const A before = warp_sums[warp - 1];
		incl = static_cast<A>(before + x);
		excl = lane == 0 ? before : static_cast<A>(before + prev);
	}
	total = warp_sums[31];
	__syncthreads();  // warp_sums is rewritten by the next call
}

template <class T, class A>
__global__ void __launch_bounds__(kSumThreads) SumTileTotalsKernel(const T *data, uint64_t rows, A *totals) {
	__shared__ A warp_sums[32];
	const uint64_t base = blockIdx.x * kSumTile + uint64_t(threadIdx.x) * kSumItems;
	A s = A(0);
	for (int j = 0; j < kSumItems; j++) {
		if (base + j < rows) s = static_cast<A>(s + SumLoad<T, A>(data + base + j));
	}
	A incl, excl, total;
	SumBlockScan(s, warp_sums, incl, excl, total);
	if (threadIdx.x == 0) totals[blockIdx.x] = total;
}

// One block: totals[i] becomes the value before tile i (the carried state plus the tiles before it).
template <class T, class A>
__global__ void __launch_bounds__(kSumThreads) SumTileStartsKernel(A *totals, uint64_t tiles, const T *state) {
	__shared__ A warp_sums[32];
	A carry = SumLoad<T, A>(state);
	for (uint64_t c = 0; c < tiles; c += kSumThreads) {
		const uint64_t i = c + threadIdx.x;
		const A x = i < tiles ? totals[i] : A(0);
		A incl, excl, chunk;
		SumBlockScan(x, warp_sums, incl, excl, chunk);
		if (i < tiles) totals[i] = static_cast<A>(carry + excl);
		carry = static_cast<A>(carry + chunk);
	}
}

template <class T, class A>
__global__ void __launch_bounds__(kSumThreads) SumTileScanKernel(T *data, uint64_t rows, const A *starts, T *state) {
	__shared__ A warp_sums[32];
	const uint64_t base = blockIdx.x * kSumTile + uint64_t(threadIdx.x) * kSumItems;
	A v[kSumItems];
	A s = A(0);
	for (int j = 0; j < kSumItems; j++) {
		v[j] = base + j < rows ? SumLoad<T, A>(data + base + j) : A(0);
		s = static_cast<A>(s + v[j]);
	}
	A incl, excl, total;
	SumBlockScan(s, warp_sums, incl, excl, total);
	A run = static_cast<A>(starts[blockIdx.x] + excl);
	for (int j = 0; j < kSumItems; j++) {
		run = static_cast<A>(run + v[j]);
		if (base + j < rows) {
			SumStore<T, A>(data + base + j, run);
			if (base + j == rows - 1) SumStore<T, A>(state, run);
		}
	}
}

template <class T, class A> void RunningSumTyped(void *data, uint64_t rows, void *state, void *scratch, cudaStream_t stream) {
	const uint64_t tiles = (rows + kSumTile - 1) / kSumTile;
	T *d = static_cast<T *>(data);
	T *st = static_cast<T *>(state);
	A *sums = static_cast<A *>(scratch);
	SumTileTotalsKernel<T, A><<<static_cast<unsigned>(tiles), kSumThreads, 0, stream>>>(d, rows, sums);
	SumTileStartsKernel<T, A><<<1, kSumThreads, 0, stream>>>(sums, tiles, st);
	SumTileScanKernel<T, A><<<static_cast<unsigned>(tiles), kSumThreads, 0, stream>>>(d, rows, sums, st);
	VGPU_CUDA(cudaGetLastError());
}

} // namespace

size_t RunningSumScratchBytes(uint64_t rows) {
	return static_cast<size_t>((rows + kSumTile - 1) / kSumTile) * sizeof(uint64_t) + 16;
}

void RunningSum(void *data, ValueType t, uint64_t rows, void *state, void *scratch, cudaStream_t stream) {
	if (rows == 0) return;
	if (rows >= (1ull << 32)) Fail(VGPU_ERR_INVALID_ARGUMENT, "running sum: at most 2^32 - 1 rows per call");
	LaunchScope scope("vgpu_running_sum", stream, 2 * rows * TypeSize(t) + rows * TypeSize(t), rows);
	switch (t) {
	case ValueType::INT16:
		RunningSumTyped<int16_t, uint32_t>(data, rows, state, scratch, stream);
		break;
	case ValueType::INT32:
		RunningSumTyped<int32_t, uint32_t>(data, rows, state, scratch, stream);
		break;
	case ValueType::INT64:
		RunningSumTyped<int64_t, uint64_t>(data, rows, state, scratch, stream);
		break;
	case ValueType::FLOAT32:
		RunningSumTyped<float, float>(data, rows, state, scratch, stream);
		break;
	case ValueType::FLOAT64:
		RunningSumTyped<double, double>(data, rows, state, scratch, stream);
		break;
	default:
		Fail(VGPU_ERR_UNSUPPORTED, std::string("running sum: unsupported type ") + TypeName(t));
	}
}

} // namespace kern
} // namespace vgpu
