// device_lib.cuh -- device-side building blocks shared by the precompiled kernels (nvcc) and the
// per-query kernels generated at run time (NVRTC, where this file is handed over as an in-memory
// header). It therefore uses no host or standard-library headers: builtin types and CUDA intrinsics
// only.
#pragma once

namespace vgpu_dev {

typedef unsigned long long u64;
typedef long long i64;
typedef unsigned int u32;
typedef unsigned short u16;
typedef unsigned char u8;

// Argument block every generated kernel takes by value: pointers, sizes and bit-cast constants, one
// 64-bit word each. Keeps the host side free of per-kernel struct layouts.
struct KArgs {
	u64 w[128];
};

// ---------------------------------------------------------------------------------------------
// Bit casts

template <typename T> __device__ __forceinline__ T from_bits(u64 b);
template <> __device__ __forceinline__ bool from_bits<bool>(u64 b) { return (b & 0xffull) != 0; }
template <> __device__ __forceinline__ signed char from_bits<signed char>(u64 b) { return (signed char)(b & 0xff); }
template <> __device__ __forceinline__ unsigned char from_bits<unsigned char>(u64 b) { return (unsigned char)(b & 0xff); }
template <> __device__ __forceinline__ char from_bits<char>(u64 b) { return (char)(b & 0xff); }
template <> __device__ __forceinline__ short from_bits<short>(u64 b) { return (short)(u16)(b & 0xffff); }
template <> __device__ __forceinline__ unsigned short from_bits<unsigned short>(u64 b) { return (u16)(b & 0xffff); }
template <> __device__ __forceinline__ int from_bits<int>(u64 b) { return (int)(u32)b; }
template <> __device__ __forceinline__ u32 from_bits<u32>(u64 b) { return (u32)b; }
template <> __device__ __forceinline__ float from_bits<float>(u64 b) { return __int_as_float((int)(u32)b); }
template <> __device__ __forceinline__ i64 from_bits<i64>(u64 b) { return (i64)b; }
template <> __device__ __forceinline__ u64 from_bits<u64>(u64 b) { return b; }
template <> __device__ __forceinline__ double from_bits<double>(u64 b) { return __longlong_as_double((i64)b); }

template <typename T> __device__ __forceinline__ u64 to_bits(T v);
template <> __device__ __forceinline__ u64 to_bits<bool>(bool v) { return v ? 1ull : 0ull; }
template <> __device__ __forceinline__ u64 to_bits<signed char>(signed char v) { return (u64)(u8)v; }
template <> __device__ __forceinline__ u64 to_bits<unsigned char>(unsigned char v) { return (u64)v; }
template <> __device__ __forceinline__ u64 to_bits<char>(char v) { return (u64)(u8)v; }
template <> __device__ __forceinline__ u64 to_bits<unsigned short>(unsigned short v) { return (u64)v; }
template <> __device__ __forceinline__ u64 to_bits<short>(short v) { return (u64)(u16)v; }
template <> __device__ __forceinline__ u64 to_bits<int>(int v) { return (u64)(u32)v; }
template <> __device__ __forceinline__ u64 to_bits<u32>(u32 v) { return (u64)v; }
template <> __device__ __forceinline__ u64 to_bits<float>(float v) { return (u64)(u32)__float_as_int(v); }
template <> __device__ __forceinline__ u64 to_bits<i64>(i64 v) { return (u64)v; }
template <> __device__ __forceinline__ u64 to_bits<u64>(u64 v) { return v; }
template <> __device__ __forceinline__ u64 to_bits<double>(double v) { return (u64)__double_as_longlong(v); }

// Reinterprets the storage of a value of type S as type T of the same size (the reference kernels read
// a column through whatever pointer type the expression casts it to).
template <typename T, typename S> __device__ __forceinline__ T reinterpret_value(S v) {
	return from_bits<T>(to_bits<S>(v));
}

// ---------------------------------------------------------------------------------------------
// Coalesced row loads: R consecutive rows of one column per thread, 128-bit vectors where the
// address allows it, streaming cache policy (each input byte is read exactly once per launch).

__device__ __forceinline__ uint4 ld_stream_v4(const void *p) {
	uint4 r;
	asm("ld.global.cs.v4.u32 {%0,%1,%2,%3}, [%4];"
	             : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
	             : "l"(p));
	return r;
}
__device__ __forceinline__ uint2 ld_stream_v2(const void *p) {
	uint2 r;
	asm("ld.global.cs.v2.u32 {%0,%1}, [%2];" : "=r"(r.x), "=r"(r.y) : "l"(p));
	return r;
}
__device__ __forceinline__ u32 ld_stream_u32(const void *p) {
	u32 r;
	asm("ld.global.cs.u32 %0, [%1];" : "=r"(r) : "l"(p));
	return r;
}

template <typename T> __device__ __forceinline__ T ld_scalar(const T *p) {
	return *p;
}

// Extracts element `i` (of size sizeof(T)) from a little-endian array of 32-bit words.
template <typename T> __device__ __forceinline__ T word_element(const u32 *words, int i) {
	if (sizeof(T) == 8) {
		u64 b = (u64)words[2 * i] | ((u64)words[2 * i + 1] << 32);
		return from_bits<T>(b);
	} else if (sizeof(T) == 4) {
		return from_bits<T>((u64)words[i]);
	} else if (sizeof(T) == 2) {
		u32 w = words[i >> 1];
		return from_bits<T>((u64)((w >> ((i & 1) * 16)) & 0xffffu));
	} else {
		u32 w = words[i >> 2];
		return from_bits<T>((u64)((w >> ((i & 3) * 8)) & 0xffu));
	}
}

template <typename T, int R>
__device__ __forceinline__ void load_rows(const T *__restrict__ base, u64 row0, u64 n, T (&out)[R]) {
	constexpr int BYTES = (int)sizeof(T) * R;
	const T *p = base + row0;
	const u64 addr = (u64)p;
	if (row0 + R <= n && (BYTES % 16 == 0) && (addr & 15ull) == 0) {
		u32 words[BYTES / 4];
#pragma unroll
		for (int q = 0; q < BYTES / 16; ++q) {
			uint4 v = ld_stream_v4(reinterpret_cast<const char *>(p) + 16 * q);
			words[4 * q + 0] = v.x;
			words[4 * q + 1] = v.y;
			words[4 * q + 2] = v.z;
			words[4 * q + 3] = v.w;
		}
#pragma unroll
		for (int r = 0; r < R; ++r) out[r] = word_element<T>(words, r);
	} else if (row0 + R <= n && BYTES == 8 && (addr & 7ull) == 0) {
		u32 words[2];
		uint2 v = ld_stream_v2(p);
		words[0] = v.x;
		words[1] = v.y;
#pragma unroll
		for (int r = 0; r < R; ++r) out[r] = word_element<T>(words, r);
	} else {
#pragma unroll
		for (int r = 0; r < R; ++r) out[r] = (row0 + r < n) ? ld_scalar(p + r) : T();
	}
}

// ---------------------------------------------------------------------------------------------
// Tile staging through shared memory: column chunks of a tile move with bulk asynchronous copies
// (cp.async.bulk, the TMA engine's 1-D form) whose completion an mbarrier counts in bytes, so a CTA
// partitions one tile from registers while the next ones are in flight. Every wait is bounded.

__device__ __forceinline__ u32 smem_addr(const void *p) { return (u32)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void stage_barrier_init(u64 *bar) {
	asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

// Makes initialized barriers visible to the copy engine (call once, after the inits, before a sync).
__device__ __forceinline__ void stage_barrier_fence() {
	asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
	asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Thread that issues a stage's copies: announces the stage's byte count on its barrier (one arrival).
__device__ __forceinline__ void stage_expect(u64 *bar, u32 bytes) {
	asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// `bytes` (a multiple of 16) from 16-byte aligned global `src` to 16-byte aligned shared `dst`.
__device__ __forceinline__ void stage_copy(void *dst, const void *src, u32 bytes, u64 *bar) {
	asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
	                 smem_addr(dst)),
	             "l"(src), "r"(bytes), "r"(smem_addr(bar))
	             : "memory");
}

__device__ __forceinline__ bool stage_try_wait(u64 *bar, u32 parity) {
	u32 done;
	asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
	             : "=r"(done)
	             : "r"(smem_addr(bar)), "r"(parity)
	             : "memory");
	return done != 0;
}

__device__ __forceinline__ u64 global_ns() {
	u64 t;
	asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
	return t;
}

// Waits for the barrier phase of the given parity to complete; false after about one second (or 2^26
// polls) without it: the caller records an error and gives up on the tile.
__device__ __forceinline__ bool stage_wait(u64 *bar, u32 parity) {
	if (stage_try_wait(bar, parity)) return true;
	const u64 t0 = global_ns();
	for (u32 i = 0; i < (1u << 26); ++i) {
		if (stage_try_wait(bar, parity)) return true;
		if (global_ns() - t0 > 1000000000ull) return false;
	}
	return false;
}

// R consecutive elements of a staged column (16-byte aligned when R * sizeof(T) is a multiple of 16).
template <typename T, int R> __device__ __forceinline__ void load_stage(const T *p, T (&out)[R]) {
	constexpr int BYTES = (int)sizeof(T) * R;
	if constexpr (BYTES % 16 == 0) {
		u32 words[BYTES / 4];
#pragma unroll
		for (int q = 0; q < BYTES / 16; ++q) {
			const uint4 v = reinterpret_cast<const uint4 *>(p)[q];
			words[4 * q + 0] = v.x;
			words[4 * q + 1] = v.y;
			words[4 * q + 2] = v.z;
			words[4 * q + 3] = v.w;
		}
#pragma unroll
		for (int r = 0; r < R; ++r) out[r] = word_element<T>(words, r);
	} else {
#pragma unroll
		for (int r = 0; r < R; ++r) out[r] = p[r];
	}
}

// Fixed-size row records (W 32-bit words, W a multiple of 4; records 32-byte aligned when W is a
// multiple of 8). A 32-byte record moves as one 256-bit access (sm_100 global vector width): one
// store request per scattered record instead of two half-sector ones, and one fully coalesced load
// per warp of consecutive records.
template <int W> __device__ __forceinline__ void store_record(void *dst, const u32 (&w)[W]) {
	if constexpr (W % 8 == 0) {
#pragma unroll
		for (int q = 0; q < W / 8; ++q) {
			asm volatile("st.global.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(reinterpret_cast<char *>(dst) + 32 * q),
			             "r"(w[8 * q]), "r"(w[8 * q + 1]), "r"(w[8 * q + 2]), "r"(w[8 * q + 3]), "r"(w[8 * q + 4]),
			             "r"(w[8 * q + 5]), "r"(w[8 * q + 6]), "r"(w[8 * q + 7])
			             : "memory");
		}
	} else {
#pragma unroll
		for (int q = 0; q < W / 4; ++q) {
			asm volatile("st.global.v4.u32 [%0], {%1,%2,%3,%4};" ::"l"(reinterpret_cast<char *>(dst) + 16 * q),
			             "r"(w[4 * q]), "r"(w[4 * q + 1]), "r"(w[4 * q + 2]), "r"(w[4 * q + 3])
			             : "memory");
		}
	}
}
template <int W> __device__ __forceinline__ void load_record(const void *src, u32 (&w)[W]) {
	if constexpr (W % 8 == 0) {
#pragma unroll
		for (int q = 0; q < W / 8; ++q) {
			asm volatile("ld.global.cs.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
			             : "=r"(w[8 * q]), "=r"(w[8 * q + 1]), "=r"(w[8 * q + 2]), "=r"(w[8 * q + 3]), "=r"(w[8 * q + 4]),
			               "=r"(w[8 * q + 5]), "=r"(w[8 * q + 6]), "=r"(w[8 * q + 7])
			             : "l"(reinterpret_cast<const char *>(src) + 32 * q));
		}
	} else {
#pragma unroll
		for (int q = 0; q < W / 4; ++q) {
			uint4 v = ld_stream_v4(reinterpret_cast<const char *>(src) + 16 * q);
			w[4 * q] = v.x;
			w[4 * q + 1] = v.y;
			w[4 * q + 2] = v.z;
			w[4 * q + 3] = v.w;
		}
	}
}

// Byte-per-row validity (the engine's internal null mask layout). nullptr = all valid.
template <int R>
__device__ __forceinline__ void load_valid(const u8 *__restrict__ base, u64 row0, u64 n, bool (&out)[R]) {
	if (base == nullptr) {
#pragma unroll
		for (int r = 0; r < R; ++r) out[r] = true;
		return;
	}
#pragma unroll
	for (int r = 0; r < R; ++r) out[r] = (row0 + r < n) ? (base[row0 + r] != 0) : false;
}

// ---------------------------------------------------------------------------------------------
// Block-wide exclusive scan of one u32 per thread (blockDim.x a multiple of 32, <= 1024).
// `scratch` needs 33 words of shared memory. Returns the exclusive prefix; *total gets the sum.

__device__ __forceinline__ u32 block_exclusive_scan(u32 v, u32 *scratch, u32 *total) {
	const int lane = threadIdx.x & 31;
	const int warp = threadIdx.x >> 5;
	const int nwarps = blockDim.x >> 5;
	u32 x = v;
#pragma unroll
	for (int o = 1; o < 32; o <<= 1) {
		u32 y = __shfl_up_sync(0xffffffffu, x, o);
		if (lane >= o) x += y;
	}
	if (lane == 31) scratch[warp] = x;
	__syncthreads();
	if (warp == 0) {
		u32 w = (lane < nwarps) ? scratch[lane] : 0u;
		u32 s = w;
#pragma unroll
		for (int o = 1; o < 32; o <<= 1) {
			u32 y = __shfl_up_sync(0xffffffffu, s, o);
			if (lane >= o) s += y;
		}
		if (lane < nwarps) scratch[lane] = s - w;
		if (lane == 31) scratch[32] = s;
	}
	__syncthreads();
	u32 result = scratch[warp] + x - v;
	*total = scratch[32];
	__syncthreads();
	return result;
}

// ---------------------------------------------------------------------------------------------
// Atomics

// Exact 128-bit accumulation from 64-bit atomics. Order-independent: every add's carry out of the
// low word is computed against the value that add actually replaced, so the high word receives the
// true total of carries whatever the interleaving.
__device__ __forceinline__ void atomic_add_i128(u64 *lo, i64 *hi, i64 x) {
	const u64 ux = (u64)x;
	const u64 old = atomicAdd(lo, ux);
	const u64 sum = old + ux;
	i64 hi_add = (x < 0 ? -1 : 0) + (sum < old ? 1 : 0);
	if (hi_add != 0) atomicAdd(reinterpret_cast<u64 *>(hi), (u64)hi_add);
}

// Same, adding an already-128-bit partial (lo, hi).
__device__ __forceinline__ void atomic_add_i128_pair(u64 *lo, i64 *hi, u64 add_lo, i64 add_hi) {
	const u64 old = atomicAdd(lo, add_lo);
	const u64 sum = old + add_lo;
	i64 hi_add = add_hi + (sum < old ? 1 : 0);
	if (hi_add != 0) atomicAdd(reinterpret_cast<u64 *>(hi), (u64)hi_add);
}

// Exact 128-bit accumulation into four 32-bit words (w0 least significant) with native 32-bit shared
// atomics only: each word's carry is computed against the value that add replaced and passed to the
// next word, so the words hold the true total under any interleaving (carry out of bit 127 wraps,
// i.e. the sum is mod 2^128 like the addends). Non-negative addends below 2^32 cost one atomic.
__device__ __forceinline__ u32 add_word_carry(u32 *w, u64 t) {
	if (t == 0) return 0u;
	if (t == (1ull << 32)) return 1u;
	const u32 x = (u32)t;
	const u32 old = atomicAdd(w, x);
	return (u32)(old + x) < old ? 1u : 0u;
}
__device__ __forceinline__ void atomic_add_i128_u32x4(u32 *w0, u32 *w1, u32 *w2, u32 *w3, u64 lo, i64 hi) {
	u32 c = add_word_carry(w0, (u64)(u32)lo);
	c = add_word_carry(w1, (u64)(u32)(lo >> 32) + c);
	c = add_word_carry(w2, (u64)(u32)(u64)hi + c);
	const u32 top = (u32)((u64)hi >> 32) + c;
	if (top) atomicAdd(w3, top);
}

__device__ __forceinline__ void atomic_min_i64(i64 *p, i64 v) { atomicMin(reinterpret_cast<long long *>(p), (long long)v); }
__device__ __forceinline__ void atomic_max_i64(i64 *p, i64 v) { atomicMax(reinterpret_cast<long long *>(p), (long long)v); }

// ---------------------------------------------------------------------------------------------
// Equi-join lookup into a sorted unique key array through a radix directory: dir[b] is the first
// position whose key >> shift >= b (dir[nb] = n), so a probe key's candidates are one bucket, which
// a short binary search finishes. Keys are biased by the sorted side's minimum (u64 arithmetic);
// a probe key below that minimum wraps to a bucket past nb and misses. Returns the position or -1.
// Dense forms (tables indexed by the biased key over the whole range, nb entries): shift == 0xff,
// dir holds row index + 1 of the key's right row (0 = no key); shift == 0xfe, `sorted` is reused as a
// u64 table holding (1 << 32 | the right column's 32-bit value) (0 = no key), returned as is;
// shift == 0xfd / 0xfc / 0xfb, `sorted` is a u8 / u16 / u32 table of value bits minus `aux` (all ones =
// no key), returned in the 0xfe form. `aux` is the directory word (the directory pointer otherwise).
__device__ __forceinline__ long long vgpu_join_find(u64 k, const u64 *__restrict__ sorted, u64 aux, u64 nb, u32 shift) {
	const u32 *__restrict__ dir = (const u32 *)aux;
	if (shift == 0xffu) {
		if (k >= nb) return -1ll;
		const u32 p = dir[k];
		return p == 0u ? -1ll : (long long)(p - 1u);
	}
	if (shift == 0xfeu) {
		if (k >= nb) return -1ll;
		const u64 e = sorted[k];
		return e == 0ull ? -1ll : (long long)e;
	}
	if (shift >= 0xfbu) {
		if (k >= nb) return -1ll;
		u32 e;
		// random reads of an L2-resident table: loaded through L2 only (nothing to reuse in L1)
		if (shift == 0xfdu) {
			e = __ldcg((const unsigned char *)sorted + k);
			if (e == 0xffu) return -1ll;
		} else if (shift == 0xfcu) {
			e = __ldcg((const unsigned short *)sorted + k);
			if (e == 0xffffu) return -1ll;
		} else {
			e = __ldcg((const unsigned int *)sorted + k);
			if (e == 0xffffffffu) return -1ll;
		}
		return (long long)((1ull << 32) | (u64)(u32)(e + (u32)aux));
	}
	const u64 b = k >> shift;
	if (b >= nb) return -1ll;
	u32 lo = dir[b];
	const u32 end = dir[b + 1];
	u32 hi = end;
	while (lo < hi) {
		const u32 mid = (lo + hi) >> 1;
		if (sorted[mid] < k) lo = mid + 1;
		else hi = mid;
	}
	return (lo < end && sorted[lo] == k) ? (long long)lo : -1ll;
}

// The run of right rows whose (biased) key equals k in a sorted key array that may repeat keys, through
// the radix directory above: returns the run's first position and sets *count to its length, or
// returns -1 (count 0) when k is absent. With shift == 0 the directory is indexed by the key itself
// (one bucket per key value), so the run is the whole bucket: two adjacent loads and no search.
__device__ __forceinline__ long long vgpu_join_run(u64 k, const u64 *__restrict__ sorted, const u32 *__restrict__ dir,
                                                   u64 nb, u32 shift, u32 *count) {
	const u64 b = k >> shift;
	*count = 0u;
	if (b >= nb) return -1ll;
	const u32 lo0 = dir[b], end = dir[b + 1];
	if (shift == 0u) {
		*count = end - lo0;
		return end > lo0 ? (long long)lo0 : -1ll;
	}
	u32 lo = lo0, hi = end;
	while (lo < hi) {  // first position with key >= k
		const u32 mid = (lo + hi) >> 1;
		if (sorted[mid] < k) lo = mid + 1;
		else hi = mid;
	}
	u32 up = lo, top = end;
	while (up < top) {  // first position with key > k
		const u32 mid = (up + top) >> 1;
		if (sorted[mid] <= k) up = mid + 1;
		else top = mid;
	}
	*count = up - lo;
	return up > lo ? (long long)lo : -1ll;
}

// A probe key's entry in the dense multi-match inline table (the join words: table, vmin, entries and
// the spec byte (wide << 7) | (vbits << 2) | (cbits - 1)): the entry, with *count = its match count (0
// for a key outside the table or without matches). Match j's value bits are vmin plus the vbits-bit
// slot at bit cbits + j * vbits.
__device__ __forceinline__ u64 vgpu_join_minline(u64 k, const void *__restrict__ table, u64 entries, u32 spec,
                                                 u32 *count) {
	*count = 0u;
	if (k >= entries) return 0ull;
	const u32 cbits = (spec & 3u) + 1u;
	const u64 e = (spec & 0x80u) ? __ldcg((const unsigned long long *)table + k) : (u64)__ldcg((const unsigned int *)table + k);
	*count = (u32)(e & ((1ull << cbits) - 1ull));
	return e;
}

__device__ __forceinline__ u32 vgpu_join_minline_value(u64 e, u32 j, u32 spec, u32 vmin) {
	const u32 cbits = (spec & 3u) + 1u, vbits = (spec >> 2) & 31u;
	return vmin + (u32)((e >> (cbits + j * vbits)) & ((1ull << vbits) - 1ull));
}

// ---------------------------------------------------------------------------------------------
// Hashing of packed group keys

__device__ __forceinline__ u64 mix64(u64 k) {
	k ^= k >> 33;
	k *= 0xff51afd7ed558ccdull;
	k ^= k >> 33;
	k *= 0xc4ceb9fe1a85ec53ull;
	k ^= k >> 33;
	return k;
}

// Partition of a packed key: the top `bits` of the mixed key. Bucket-table slots use the low bits of
// the same mix, so the two are independent.
__device__ __forceinline__ u32 partition_of(u64 key, int bits) {
	return bits == 0 ? 0u : (u32)(mix64(key) >> (64 - bits));
}

// ---------------------------------------------------------------------------------------------
// int128 -> double, correctly rounded (round to nearest even), from the two's-complement halves.
// The magnitude is normalised so its top bit is bit 127; the upper 64 bits, with every lower bit
// folded into bit 0 as a sticky bit, convert exactly like the full value would (the rounding point
// sits at bit 11 of that word), and the power-of-two rescale is exact.
__device__ __forceinline__ double i128_to_double(u64 lo, i64 hi) {
	const bool neg = hi < 0;
	u64 mlo = lo, mhi = (u64)hi;
	if (neg) {
		mlo = ~mlo + 1ull;
		mhi = ~mhi + (mlo == 0 ? 1ull : 0ull);
	}
	double mag;
	if (mhi == 0) {
		mag = (double)mlo;
	} else {
		const int s = __clzll((long long)mhi);
		u64 top = s == 0 ? mhi : ((mhi << s) | (mlo >> (64 - s)));
		const u64 rest = s == 0 ? mlo : (mlo << s);
		if (rest != 0) top |= 1ull;
		const double scale = __longlong_as_double((long long)((u64)(1023 + 64 - s) << 52));
		mag = (double)top * scale;
	}
	return neg ? -mag : mag;
}

} // namespace vgpu_dev
