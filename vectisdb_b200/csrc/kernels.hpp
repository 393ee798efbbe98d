// kernels.hpp -- precompiled (nvcc, sm_100a) device primitives used by the executor. Every entry
// point launches on the given stream, takes temporaries from the given arena and never synchronizes.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "runtime.hpp"

namespace vgpu {
namespace kern {

//! out[i] = sum(in[0..i)), *total = sum(in) (device scalar). In-place (out == in) is allowed.
void ExclusiveScanU32(const uint32_t *in, uint32_t *out, uint64_t n, uint32_t *total, Arena &arena);
void ExclusiveScanU64(const uint64_t *in, uint64_t *out, uint64_t n, uint64_t *total, Arena &arena);

//! Running total in place: data[i] = *state + data[0] + ... + data[i] for `rows` values of type `t`
//! (INT16/INT32/INT64 wrapping in their width, FLOAT32/FLOAT64 in their own precision), then
//! *state = data[rows - 1] (device scalar of type `t`), so consecutive calls continue one total.
//! `scratch` holds RunningSumScratchBytes(rows) bytes. Three launches, no host synchronization.
size_t RunningSumScratchBytes(uint64_t rows);
void RunningSum(void *data, ValueType t, uint64_t rows, void *state, void *scratch, cudaStream_t stream);

//! Arrow LSB-first bitmap <-> one byte per row.
void UnpackValidity(const uint8_t *bitmap, uint8_t *bytes, uint64_t n, cudaStream_t stream);
void PackValidity(const uint8_t *bytes, uint8_t *bitmap, uint64_t n, cudaStream_t stream);

//! dst[o] = src[idx[o]] for `width`-byte values (1, 2, 4, 8 or 16).
void Gather(const void *src, size_t width, const uint32_t *idx, uint64_t n, void *dst, cudaStream_t stream);

//! Raw key bits zero-extended to 64 bits (the reference's WidenKeyKernel semantics,
//! cuda_engine/src/operators/gpu_groupby.cu:76-94), plus the range of the widened values.
void WidenKeys(const void *src, size_t width, uint64_t n, uint64_t *dst, cudaStream_t stream);
void MinMaxU64(const uint64_t *keys, uint64_t n, uint64_t *minmax /* device [2] */, cudaStream_t stream);
//! WidenKeys and MinMaxU64 of the widened keys in one pass.
void WidenKeysMinMax(const void *src, size_t width, uint64_t n, uint64_t *dst, uint64_t *minmax, cudaStream_t stream);

//! Signed range of an integer/boolean column: out[0] = min, out[1] = max (device i64[2]).
void MinMaxSigned(const void *data, int type /* ValueType */, uint64_t n, int64_t *out, cudaStream_t stream);

//! Stable LSD radix sort of (key, value) pairs over the low `bits` bits of the keys (8-bit digits).
//! Results end in (keys, values); (keys_alt, values_alt) are the ping-pong buffers.
void RadixSortPairs(uint64_t *keys, uint32_t *values, uint64_t *keys_alt, uint32_t *values_alt, uint64_t n, int bits,
                    Arena &arena);

//! keys[i] -= bias (normalizes a key range to start at zero before sorting).
void SubtractBias(uint64_t *keys, uint64_t n, uint64_t bias, cudaStream_t stream);
void Iota(uint32_t *out, uint64_t n, cudaStream_t stream);

//! Left row i owns outputs [offsets[i], offsets[i + 1]) (offsets ascending, offsets[0] = 0): output o
//! becomes (i, sorted_perm[lower[i] + o - offsets[i]]). Load-balanced: fixed tiles of outputs per CTA,
//! the left rows a tile spans staged in shared memory.
void JoinExpand(const uint64_t *offsets, const uint64_t *lower, uint64_t n_left, const uint32_t *sorted_perm,
                uint64_t total, uint32_t *out_left, uint32_t *out_right, cudaStream_t stream);
//! For each probe key (widened): the first position of its run of equal keys in `sorted` (normalized by
//! `bias`) and the run's length, through the radix directory `dir` (nb buckets of key >> shift).
void JoinRuns(const uint64_t *probe, uint64_t n_probe, const uint64_t *sorted, const uint32_t *dir, uint64_t nb,
              uint32_t shift, uint64_t bias, uint64_t *lower, uint64_t *count, cudaStream_t stream);

//! Radix directory of a sorted (biased) key array: dir[b] = first position whose key >> shift >= b,
//! for b in [0, nb]; dir needs nb + 1 entries and nb must exceed every key >> shift.
void JoinDirectory(const uint64_t *sorted, uint64_t n, uint32_t shift, uint64_t nb, uint32_t *dir, cudaStream_t stream);
//! Dense join tables over keys - bias all <= range (`bias`: the keys' minimum, subtracted on the fly;
//! 0 for keys already biased), range + 1 entries, built without sorting:
//! table[k] = row index + 1 of key k (0 = none), or (1 << 32 | value) with a <= 4-byte value of that
//! row inlined. *dups = keys met more than once (then the table is not a valid lookup).
void JoinDenseRows(const uint64_t *keys, uint64_t n, uint64_t range, uint32_t *table, uint32_t *dups,
                   cudaStream_t stream, uint64_t bias = 0);
void JoinDenseInline(const uint64_t *keys, const void *values, size_t width, uint64_t n, uint64_t range,
                     uint64_t *table, uint32_t *dups, cudaStream_t stream, uint64_t bias = 0);
//! Smallest and largest raw bits (zero-extended to 32) of a 1-, 2- or 4-byte column: bounds[0], bounds[1].
void ValueBits(const void *values, size_t width, uint64_t n, uint32_t *bounds, cudaStream_t stream);
//! The inline table in `width` (1, 2 or 4) bytes per key: table[k] = value bits - vmin, all ones = no
//! key (every value's offset must stay below that marker). *dups = keys met more than once.
void JoinDenseCompact(const uint64_t *keys, const void *values, size_t vwidth, uint64_t n, uint64_t range,
                      uint32_t vmin, void *table, size_t width, uint32_t *dups, cudaStream_t stream,
                      uint64_t bias = 0);
//! Dense multi-match table over (biased) keys <= range, built without sorting, for a join that contributes
//! one right column of at most 4 bytes: entry[k] (4 bytes, or 8 when `wide`) holds k's match count in its
//! low `cbits` bits (1..3) and one `vbits`-bit slot per match above them, each the value bits - vmin. A key
//! with more than `rmax` matches (rmax < 2^cbits, cbits + rmax * vbits within the entry) counts in
//! *overflow, and the table is then not valid.
void JoinDenseMulti(const uint64_t *keys, const void *values, size_t vwidth, uint64_t n, uint64_t range, uint32_t vmin,
                    uint32_t vbits, uint32_t cbits, uint32_t rmax, void *table, bool wide, uint32_t *overflow,
                    cudaStream_t stream, uint64_t bias = 0);
//! *out = number of positions i > 0 with sorted[i] == sorted[i - 1].
void CountAdjacentEqual(const uint64_t *sorted, uint64_t n, uint32_t *out, cudaStream_t stream);
//! *out = the length of the longest run of equal keys in `sorted` (saturating at 2^32 - 1).
void MaxRunLength(const uint64_t *sorted, uint64_t n, uint32_t *out, cudaStream_t stream);

//! Work list of a partitioned aggregation pass over `P` partitions whose row ranges start at
//! offsets[p * stride] (the last ends at *total_rows): 16-byte items (partition, first row, end row,
//! split index or ~0u), longest first, into `items` (capacity PlanWorkCapacity). Partitions larger
//! than max(min_split, ceil(total / (4 * ctas))) rows are split into chunks (so at most 4 * ctas and
//! at most total / min_split partitions are split); chunks of one partition share a
//! split index s with split_info[2s] = chunk count and split_info[2s+1] = 0 (a completion counter).
//! counts[0] = items, counts[1] = split partitions (split_info is written for the first max_split),
//! counts[3] = *total_rows.
//! Heavy keys of a direct-partitioned group-by from a sample: sample_keys/sample_counts ([SC], key ~0
//! = empty) hold the sampled rows' mixed keys and counts (the counts are used as scratch). Keys seen
//! at least t times, t >= min_count the smallest threshold that selects at most K keys, claim their
//! partition (key >> dbits; the first claim wins, one heavy key per partition): hmap[p] = (index << 16)
//! | (key & (2^dbits - 1)), heavy_keys[index] = key, *n_heavy = keys selected. hmap must hold ~0 on
//! entry. With require_cover, a selection covering under a tenth of the sampled rows is dropped.
void HeavySelect(const uint64_t *sample_keys, uint32_t *sample_counts, uint32_t SC, uint32_t *hmap, uint32_t dbits,
                 uint32_t *heavy_keys, uint32_t K, uint32_t min_count, bool require_cover, uint32_t *n_heavy,
                 cudaStream_t stream);
uint64_t PlanWorkCapacity(uint32_t P, uint64_t rows, uint32_t min_split);
void PlanWork(const uint32_t *offsets, uint64_t stride, uint32_t P, const uint32_t *total_rows, uint32_t min_split,
              uint32_t ctas, void *items, uint32_t *counts, uint32_t *split_info, uint32_t max_split,
              cudaStream_t stream);

} // namespace kern
} // namespace vgpu
