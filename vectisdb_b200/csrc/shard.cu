// shard.cu -- the exchange step of a GROUP BY split by rows across GPUs, on the device.
//
// Each rank runs the GROUP BY on its own rows (the engine, partial states: AVG as SUM + COUNT), then:
//   1. ShardRoute packs every partial group into one row of 64-bit words -- the packed key, then each
//      partial state as words that merge by plain SUM / MIN / MAX over INT64 or FLOAT64 columns -- and
//      writes the rows ordered by the rank that owns the key (mix64(packed key) mod world);
//   2. the rows cross the ranks with one NCCL all-to-all (the caller's, over torch.distributed);
//   3. ShardColumns turns the received rows into one device column per word, which the engine's GROUP
//      BY re-aggregates on the owning rank;
//   4. ShardFinish turns the re-aggregated words back into the query's output columns.
// Words per partial state (the kinds of vectisdb_b200/distributed.py, same order):
//   SUM_F64  1: the double's bits (re-aggregated as a FLOAT64 SUM);
//   SUM_I128 4: the 128-bit sum as 32-bit chunks c0..c2 (unsigned) and c3 (signed), each re-aggregated
//              as an exact INT64 SUM (fewer than 2^31 partials per group cannot overflow) and carried
//              back into 128 bits at the end;
//   COUNT    1: the count (INT64 SUM);
//   MIN/MAX  1: the value sign-extended to INT64 (INT64 MIN/MAX);
//   MIN_F64/MAX_F64 1: an int64 whose signed order is the float's order (INT64 MIN/MAX).
// The owner hash is the one the host-side merge uses (distributed._owner), so both send every group to
// the same rank.
#include <algorithm>
#include <cstring>

#include "common.hpp"
#include "device_lib.cuh"
#include "kernels.hpp"
#include "runtime.hpp"
#include "shard.hpp"

namespace vgpu {
namespace {

using vgpu_dev::i128_to_double;
using vgpu_dev::mix64;

constexpr int kRouteBlock = 256;
constexpr int kMaxKeys = 8;
constexpr int kMaxValues = 32;

struct KeySpec {
	const void *data[kMaxKeys];
	int64_t min[kMaxKeys];
	int32_t width[kMaxKeys];  // 1, 2, 4 or 8 bytes, signed
	int32_t shift[kMaxKeys];
	int32_t n;
};

struct ValueSpec {
	const void *data[kMaxValues];
	int32_t kind[kMaxValues];
	int32_t type[kMaxValues];  // ValueType of the partial column
	int32_t n;
	int32_t words;
};

__device__ __forceinline__ int64_t LoadSigned(const void *p, int width, uint64_t i) {
	switch (width) {
	case 1:
		return static_cast<const int8_t *>(p)[i];
	case 2:
		return static_cast<const int16_t *>(p)[i];
	case 4:
		return static_cast<const int32_t *>(p)[i];
	default:
		return static_cast<const int64_t *>(p)[i];
	}
}

__device__ __forceinline__ uint64_t PackedKey(const KeySpec &k, uint64_t i) {
	uint64_t packed = 0;
	for (int j = 0; j < k.n; j++) {
		packed |= static_cast<uint64_t>(LoadSigned(k.data[j], k.width[j], i) - k.min[j]) << k.shift[j];
	}
	return packed;
}

__device__ __forceinline__ int64_t OrderBits(double v) {
	const int64_t b = __double_as_longlong(v);
	return b < 0 ? (b ^ 0x7FFFFFFFFFFFFFFFll) : b;
}

// Rows [c * chunk, min((c + 1) * chunk, rows)) belong to CTA c; counts are rank-major ([rank][cta]) so
// one exclusive scan gives every (rank, CTA) its first output row.
__global__ void __launch_bounds__(kRouteBlock) RouteCountKernel(KeySpec keys, uint64_t rows, uint64_t chunk,
                                                                uint32_t world, uint64_t *counts) {
	extern __shared__ uint32_t hist[];
	for (uint32_t r = threadIdx.x; r < world; r += blockDim.x) hist[r] = 0;
	__syncthreads();
	const uint64_t begin = blockIdx.x * chunk;
	const uint64_t end = begin + chunk < rows ? begin + chunk : rows;
	for (uint64_t i = begin + threadIdx.x; i < end; i += blockDim.x) {
		atomicAdd(&hist[mix64(PackedKey(keys, i)) % world], 1u);
	}
	__syncthreads();
	for (uint32_t r = threadIdx.x; r < world; r += blockDim.x) counts[static_cast<uint64_t>(r) * gridDim.x + blockIdx.x] = hist[r];
}

__global__ void RouteTotalsKernel(const uint64_t *offsets, uint32_t ctas, uint32_t world, uint64_t rows, uint64_t *totals) {
	const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
	if (r >= world) return;
	const uint64_t a = offsets[static_cast<uint64_t>(r) * ctas];
	const uint64_t b = r + 1 < world ? offsets[static_cast<uint64_t>(r + 1) * ctas] : rows;
	totals[r] = b - a;
}

__global__ void __launch_bounds__(kRouteBlock) RouteScatterKernel(KeySpec keys, ValueSpec vals, uint64_t rows,
                                                                  uint64_t chunk, uint32_t world,
                                                                  const uint64_t *offsets, int64_t *send) {
	extern __shared__ uint32_t cursor[];
	for (uint32_t r = threadIdx.x; r < world; r += blockDim.x) cursor[r] = 0;
	__syncthreads();
	const uint64_t begin = blockIdx.x * chunk;
	const uint64_t end = begin + chunk < rows ? begin + chunk : rows;
	const uint32_t W = static_cast<uint32_t>(vals.words);
	for (uint64_t i = begin + threadIdx.x; i < end; i += blockDim.x) {
		const uint64_t packed = PackedKey(keys, i);
		const uint32_t owner = static_cast<uint32_t>(mix64(packed) % world);
		const uint64_t at = offsets[static_cast<uint64_t>(owner) * gridDim.x + blockIdx.x] + atomicAdd(&cursor[owner], 1u);
		int64_t *row = send + at * W;
		row[0] = static_cast<int64_t>(packed);
		uint32_t w = 1;
		for (int j = 0; j < vals.n; j++) {
			const void *p = vals.data[j];
			switch (vals.kind[j]) {
			case kShardSumI128: {
				const uint64_t lo = static_cast<const uint64_t *>(p)[2 * i];
				const int64_t hi = static_cast<const int64_t *>(p)[2 * i + 1];
				row[w] = static_cast<int64_t>(lo & 0xFFFFFFFFull);
				row[w + 1] = static_cast<int64_t>(lo >> 32);
				row[w + 2] = static_cast<int64_t>(static_cast<uint64_t>(hi) & 0xFFFFFFFFull);
				row[w + 3] = hi >> 32;
				w += 4;
				break;
			}
			case kShardMinF64:
			case kShardMaxF64: {
				const double v = vals.type[j] == static_cast<int32_t>(ValueType::FLOAT32)
				                     ? static_cast<double>(static_cast<const float *>(p)[i])
				                     : static_cast<const double *>(p)[i];
				row[w++] = OrderBits(v);
				break;
			}
			case kShardSumF64:
				row[w++] = static_cast<const int64_t *>(p)[i];
				break;
			default: {  // COUNT, MIN, MAX: integers sign-extended
				const int t = vals.type[j];
				const int width = t == static_cast<int32_t>(ValueType::BOOLEAN)   ? 1
				                  : t == static_cast<int32_t>(ValueType::INT16) ? 2
				                  : t == static_cast<int32_t>(ValueType::INT64) ? 8
				                                                                : 4;
				row[w++] = LoadSigned(p, width, i);
				break;
			}
			}
		}
	}
}

// [rows][W] row-major -> W columns of `rows` values, through a shared-memory tile so both the reads and
// the writes are coalesced.
constexpr int kTileRows = 128;
__global__ void __launch_bounds__(256) ColumnsKernel(const int64_t *in, uint64_t rows, uint32_t W, int64_t *out) {
	extern __shared__ int64_t tile[];  // kTileRows * W
	const uint64_t r0 = static_cast<uint64_t>(blockIdx.x) * kTileRows;
	const uint32_t n = static_cast<uint32_t>(rows - r0 < kTileRows ? rows - r0 : kTileRows);
	for (uint32_t i = threadIdx.x; i < n * W; i += blockDim.x) tile[i] = in[r0 * W + i];
	__syncthreads();
	for (uint32_t i = threadIdx.x; i < n * W; i += blockDim.x) {
		const uint32_t w = i / n, r = i % n;
		out[static_cast<uint64_t>(w) * rows + r0 + r] = tile[static_cast<uint64_t>(r) * W + w];
	}
}

// 128-bit value from the sums of its four 32-bit chunks (c0..c2 from non-negative chunks, c3 signed).
__device__ __forceinline__ void CarryChunks(int64_t s0, int64_t s1, int64_t s2, int64_t s3, uint64_t *lo, int64_t *hi) {
	int64_t t = s0;
	const uint64_t w0 = static_cast<uint64_t>(t) & 0xFFFFFFFFull;
	t = s1 + (t >> 32);
	const uint64_t w1 = static_cast<uint64_t>(t) & 0xFFFFFFFFull;
	t = s2 + (t >> 32);
	const uint64_t w2 = static_cast<uint64_t>(t) & 0xFFFFFFFFull;
	t = s3 + (t >> 32);
	*lo = w0 | (w1 << 32);
	*hi = static_cast<int64_t>(w2 | (static_cast<uint64_t>(t) << 32));
}

struct FinishOp {
	int32_t op;
	int32_t width;          // KEY: output bytes
	int32_t shift, bits;    // KEY
	int64_t min;            // KEY
	const void *src[4];     // the re-aggregated columns read
	int32_t src_hugeint[4]; // 1: the column is a HUGEINT sum (read its low word)
	const void *count;      // AVG: the merged count (HUGEINT sum or INT64)
	int32_t count_hugeint;
	void *dst;
};

__device__ __forceinline__ int64_t Word(const void *p, int hugeint, uint64_t i) {
	return hugeint ? static_cast<const int64_t *>(p)[2 * i] : static_cast<const int64_t *>(p)[i];
}

__global__ void FinishKernel(FinishOp f, uint64_t rows) {
	const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
	if (i >= rows) return;
	switch (f.op) {
	case kShardOutKey: {
		const uint64_t packed = static_cast<uint64_t>(Word(f.src[0], 0, i));
		const uint64_t mask = f.bits >= 64 ? ~0ull : ((1ull << f.bits) - 1);
		const int64_t v = static_cast<int64_t>((packed >> f.shift) & mask) + f.min;
		switch (f.width) {
		case 1:
			static_cast<int8_t *>(f.dst)[i] = static_cast<int8_t>(v);
			break;
		case 2:
			static_cast<int16_t *>(f.dst)[i] = static_cast<int16_t>(v);
			break;
		case 4:
			static_cast<int32_t *>(f.dst)[i] = static_cast<int32_t>(v);
			break;
		default:
			static_cast<int64_t *>(f.dst)[i] = v;
		}
		break;
	}
	case kShardOutI128:
	case kShardOutAvgI128: {
		uint64_t lo;
		int64_t hi;
		CarryChunks(Word(f.src[0], f.src_hugeint[0], i), Word(f.src[1], f.src_hugeint[1], i),
		            Word(f.src[2], f.src_hugeint[2], i), Word(f.src[3], f.src_hugeint[3], i), &lo, &hi);
		if (f.op == kShardOutI128) {
			static_cast<uint64_t *>(f.dst)[2 * i] = lo;
			static_cast<int64_t *>(f.dst)[2 * i + 1] = hi;
		} else {
			static_cast<double *>(f.dst)[i] =
			    i128_to_double(lo, hi) / static_cast<double>(Word(f.count, f.count_hugeint, i));
		}
		break;
	}
	case kShardOutAvgF64:
		static_cast<double *>(f.dst)[i] =
		    __longlong_as_double(Word(f.src[0], f.src_hugeint[0], i)) / static_cast<double>(Word(f.count, f.count_hugeint, i));
		break;
	case kShardOutF64FromOrder: {
		const int64_t b = Word(f.src[0], f.src_hugeint[0], i);
		static_cast<int64_t *>(f.dst)[i] = b < 0 ? (b ^ 0x7FFFFFFFFFFFFFFFll) : b;
		break;
	}
	default:  // kShardOutWord: a 64-bit word as it is (FLOAT64 sums, INT64 counts, MIN/MAX)
		static_cast<int64_t *>(f.dst)[i] = Word(f.src[0], f.src_hugeint[0], i);
	}
}

int KeyWidth(ValueType t) {
	switch (t) {
	case ValueType::BOOLEAN:
		return 1;
	case ValueType::INT16:
		return 2;
	case ValueType::INT32:
	case ValueType::DICTIONARY_STRING:
		return 4;
	case ValueType::INT64:
		return 8;
	default:
		return 0;
	}
}

} // namespace

int ShardWords(const int32_t *kinds, int n_values) {
	int w = 1;
	for (int j = 0; j < n_values; j++) w += kinds[j] == kShardSumI128 ? 4 : 1;
	return w;
}

void ShardRoute(const vgpu_column *keys, int n_keys, const int64_t *key_min, const int32_t *key_shift,
                const vgpu_column *values, const int32_t *kinds, int n_values, uint64_t rows, uint32_t world,
                int64_t *send, uint64_t *send_counts, cudaStream_t stream) {
	if (n_keys < 1 || n_keys > kMaxKeys) Fail(VGPU_ERR_INVALID_ARGUMENT, "shard route: 1 to 8 key columns");
	if (n_values < 0 || n_values > kMaxValues) Fail(VGPU_ERR_INVALID_ARGUMENT, "shard route: at most 32 partial states");
	if (world < 1 || world > 4096) Fail(VGPU_ERR_INVALID_ARGUMENT, "shard route: world size 1 to 4096");
	KeySpec ks{};
	ks.n = n_keys;
	for (int j = 0; j < n_keys; j++) {
		const auto t = static_cast<ValueType>(keys[j].type);
		ks.width[j] = KeyWidth(t);
		if (!ks.width[j]) Fail(VGPU_ERR_UNSUPPORTED, "shard route: key columns must be integer-typed");
		if (keys[j].validity) Fail(VGPU_ERR_UNSUPPORTED, "shard route: NULL group keys do not merge here");
		if (rows && !keys[j].data) Fail(VGPU_ERR_INVALID_ARGUMENT, "shard route: null key column");
		if (key_shift[j] < 0 || key_shift[j] > 63) Fail(VGPU_ERR_INVALID_ARGUMENT, "shard route: key shift out of range");
		ks.data[j] = keys[j].data;
		ks.min[j] = key_min[j];
		ks.shift[j] = key_shift[j];
	}
	ValueSpec vs{};
	vs.n = n_values;
	for (int j = 0; j < n_values; j++) {
		const auto t = static_cast<ValueType>(values[j].type);
		const int k = kinds[j];
		bool ok = false;
		switch (k) {
		case kShardSumF64:
			ok = t == ValueType::FLOAT64;
			break;
		case kShardSumI128:
			ok = t == ValueType::HUGEINT;
			break;
		case kShardMinF64:
		case kShardMaxF64:
			ok = t == ValueType::FLOAT64 || t == ValueType::FLOAT32;
			break;
		case kShardCount:
		case kShardMin:
		case kShardMax:
			ok = KeyWidth(t) != 0;
			break;
		default:
			Fail(VGPU_ERR_INVALID_ARGUMENT, "shard route: unknown partial-state kind " + std::to_string(k));
		}
		if (!ok) Fail(VGPU_ERR_UNSUPPORTED, "shard route: partial state " + std::to_string(j) + " has a type its kind does not take");
		if (values[j].validity) Fail(VGPU_ERR_UNSUPPORTED, "shard route: NULL aggregate values do not merge here");
		if (rows && !values[j].data) Fail(VGPU_ERR_INVALID_ARGUMENT, "shard route: null partial-state column");
		vs.data[j] = values[j].data;
		vs.kind[j] = k;
		vs.type[j] = values[j].type;
	}
	vs.words = ShardWords(kinds, n_values);
	if (rows == 0) {
		std::fill(send_counts, send_counts + world, 0ull);
		return;
	}
	if (!send) Fail(VGPU_ERR_INVALID_ARGUMENT, "shard route: null send buffer");
	const auto &props = Runtime::Get().props();
	const uint64_t max_ctas = static_cast<uint64_t>(props.sm_count) * 4;
	const uint64_t ctas = std::max<uint64_t>(1, std::min<uint64_t>(max_ctas, (rows + 4 * kRouteBlock - 1) / (4 * kRouteBlock)));
	const uint64_t chunk = (rows + ctas - 1) / ctas;
	const size_t smem = world * sizeof(uint32_t);
	Arena arena(stream);
	uint64_t *counts = arena.AllocT<uint64_t>(ctas * world + 1);
	uint64_t *totals = arena.AllocT<uint64_t>(world);
	{
		LaunchScope scope("shard_route_count", stream, rows * 8ull * n_keys, rows);
		RouteCountKernel<<<static_cast<unsigned>(ctas), kRouteBlock, smem, stream>>>(ks, rows, chunk, world, counts);
		VGPU_CUDA(cudaGetLastError());
	}
	kern::ExclusiveScanU64(counts, counts, ctas * world, counts + ctas * world, arena);
	RouteTotalsKernel<<<(world + 255) / 256, 256, 0, stream>>>(counts, static_cast<uint32_t>(ctas), world, rows, totals);
	VGPU_CUDA(cudaGetLastError());
	{
		LaunchScope scope("shard_route_scatter", stream, rows * (8ull * n_keys + 8ull * vs.words * 2), rows);
		RouteScatterKernel<<<static_cast<unsigned>(ctas), kRouteBlock, smem, stream>>>(ks, vs, rows, chunk, world, counts, send);
		VGPU_CUDA(cudaGetLastError());
	}
	VGPU_CUDA(cudaMemcpyAsync(send_counts, totals, world * sizeof(uint64_t), cudaMemcpyDeviceToHost, stream));
	VGPU_CUDA(cudaStreamSynchronize(stream));
}

void ShardColumns(const int64_t *recv, uint64_t rows, int words, int64_t *out, cudaStream_t stream) {
	if (words < 1 || words > 256) Fail(VGPU_ERR_INVALID_ARGUMENT, "shard columns: 1 to 256 words per row");
	if (rows == 0) return;
	if (!recv || !out) Fail(VGPU_ERR_INVALID_ARGUMENT, "shard columns: null buffer");
	const size_t smem = static_cast<size_t>(kTileRows) * words * sizeof(int64_t);
	if (smem > 48 * 1024) VGPU_CUDA(cudaFuncSetAttribute(ColumnsKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
	LaunchScope scope("shard_columns", stream, rows * words * 16ull, rows);
	ColumnsKernel<<<static_cast<unsigned>((rows + kTileRows - 1) / kTileRows), 256, smem, stream>>>(recv, rows, static_cast<uint32_t>(words), out);
	VGPU_CUDA(cudaGetLastError());
}

void ShardFinish(const vgpu_shard_output *outs, int n_outs, uint64_t rows, cudaStream_t stream) {
	if (rows == 0) return;
	for (int o = 0; o < n_outs; o++) {
		const vgpu_shard_output &s = outs[o];
		FinishOp f{};
		f.op = s.op;
		f.dst = s.dst;
		if (!f.dst) Fail(VGPU_ERR_INVALID_ARGUMENT, "shard finish: null output column");
		const int nsrc = s.op == kShardOutI128 || s.op == kShardOutAvgI128 ? 4 : 1;
		for (int j = 0; j < nsrc; j++) {
			const auto t = static_cast<ValueType>(s.src[j].type);
			if (!s.src[j].data) Fail(VGPU_ERR_INVALID_ARGUMENT, "shard finish: null input column");
			if (t != ValueType::HUGEINT && t != ValueType::INT64 && t != ValueType::FLOAT64) {
				Fail(VGPU_ERR_UNSUPPORTED, "shard finish: inputs are INT64, FLOAT64 or HUGEINT sums");
			}
			f.src[j] = s.src[j].data;
			f.src_hugeint[j] = t == ValueType::HUGEINT;
		}
		switch (s.op) {
		case kShardOutKey:
			f.width = KeyWidth(static_cast<ValueType>(s.key_type));
			if (!f.width) Fail(VGPU_ERR_UNSUPPORTED, "shard finish: key columns are integer-typed");
			if (s.key_shift < 0 || s.key_shift > 63 || s.key_bits < 0 || s.key_bits > 64) {
				Fail(VGPU_ERR_INVALID_ARGUMENT, "shard finish: key shift/bits out of range");
			}
			f.shift = s.key_shift;
			f.bits = s.key_bits;
			f.min = s.key_min;
			break;
		case kShardOutAvgF64:
		case kShardOutAvgI128: {
			const auto ct = static_cast<ValueType>(s.count.type);
			if (!s.count.data || (ct != ValueType::HUGEINT && ct != ValueType::INT64)) {
				Fail(VGPU_ERR_INVALID_ARGUMENT, "shard finish: AVG needs the merged count (INT64 or HUGEINT)");
			}
			f.count = s.count.data;
			f.count_hugeint = ct == ValueType::HUGEINT;
			break;
		}
		case kShardOutI128:
		case kShardOutWord:
		case kShardOutF64FromOrder:
			break;
		default:
			Fail(VGPU_ERR_INVALID_ARGUMENT, "shard finish: unknown output op " + std::to_string(s.op));
		}
		LaunchScope scope("shard_finish", stream, rows * 8ull * (nsrc + 1), rows);
		FinishKernel<<<static_cast<unsigned>((rows + 255) / 256), 256, 0, stream>>>(f, rows);
		VGPU_CUDA(cudaGetLastError());
	}
}

} // namespace vgpu
