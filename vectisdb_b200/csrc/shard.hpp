// shard.hpp -- the device side of the exchange step of a GROUP BY split by rows across GPUs
// (vgpu_shard_* in include/vgpu.h). The reference runs on one device and has no such step.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "vgpu.h"

namespace vgpu {

// Partial-state kinds (vgpu_shard_kind) and output ops (vgpu_shard_op).
constexpr int kShardSumF64 = VGPU_SHARD_SUM_F64, kShardSumI128 = VGPU_SHARD_SUM_I128, kShardCount = VGPU_SHARD_COUNT,
              kShardMin = VGPU_SHARD_MIN, kShardMax = VGPU_SHARD_MAX, kShardMinF64 = VGPU_SHARD_MIN_F64,
              kShardMaxF64 = VGPU_SHARD_MAX_F64;
constexpr int kShardOutWord = VGPU_SHARD_OUT_WORD, kShardOutKey = VGPU_SHARD_OUT_KEY, kShardOutI128 = VGPU_SHARD_OUT_I128,
              kShardOutAvgF64 = VGPU_SHARD_OUT_AVG_F64, kShardOutAvgI128 = VGPU_SHARD_OUT_AVG_I128,
              kShardOutF64FromOrder = VGPU_SHARD_OUT_F64_FROM_ORDER;

//! 64-bit words per exchanged row: the packed key, then 4 per SUM_I128 and 1 per other kind.
int ShardWords(const int32_t *kinds, int n_values);
//! Routes partial groups to their owner ranks (one synchronization of `stream`, for the counts).
void ShardRoute(const vgpu_column *keys, int n_keys, const int64_t *key_min, const int32_t *key_shift,
                const vgpu_column *values, const int32_t *kinds, int n_values, uint64_t rows, uint32_t world,
                int64_t *send, uint64_t *send_counts, cudaStream_t stream);
//! Received rows ([rows][words], row-major) to `words` columns of `rows` int64 values each.
void ShardColumns(const int64_t *recv, uint64_t rows, int words, int64_t *out, cudaStream_t stream);
//! The query's output columns from the re-aggregated words.
void ShardFinish(const vgpu_shard_output *outs, int n_outs, uint64_t rows, cudaStream_t stream);

} // namespace vgpu
