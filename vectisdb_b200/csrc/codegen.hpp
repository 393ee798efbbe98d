// codegen.hpp -- per-query CUDA source generation for NVRTC.
//
// A "pipeline" is a chain of FILTER/PROJECTION nodes over a source relation (scanned columns, a
// materialized intermediate, or the virtual pair space of a CROSS_PRODUCT). The generator walks the
// chain symbolically and emits ONE kernel body that loads each needed source column once (128-bit
// coalesced loads, R consecutive rows per thread), evaluates every predicate and projection in
// registers, and hands the surviving rows to a consumer: compaction into dense output columns, key
// statistics, or a group-by (direct shared-memory tables or radix partitioning).
//
// Expression sources keep the reference's contract (cuda_engine/src/code_generator.cpp:269-310 and
// extension/src/expression_translator.cpp:311-315): a statement reading ((const T*)inputs[i])[row] and
// writing ((T*)out)[idx]. The generator rewrites those two access forms into register values.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "plan.hpp"

namespace vgpu {

struct SourceColumn {
	std::string name;
	ValueType type = ValueType::INT32;
	bool nullable = false;
	int side = 0; // CROSS_PRODUCT pipelines: 0 = left (row / m), 1 = right (row % m)
};

struct PipelineSpec {
	std::vector<SourceColumn> sources;
	bool cross = false;
	// Equi-join source: row r is left row r; side-1 sources are the sorted right side's columns, read at
	// the position of the left key's match (source join_key) in the unique sorted right keys; rows
	// without a match are filtered out.
	bool join = false;
	int join_key = -1;
	// The lookup returns the (single, <= 4-byte) right column's value itself instead of a position.
	bool join_inline = false;
	// multi-match join whose right column sits inline in a dense table, one slot per match (join_multi set
	// too): join words 0 = table, 1 = the column's smallest value bits, 3 = entries << 8 | spec byte
	bool join_minline = false;
	// Right keys repeat: the lookup returns the run of equal keys in the sorted right side (start and
	// length), and every left row expands into one pipeline item per match, in sorted right order.
	// Consumers that support it: materialization, key statistics, the one-pass group-by.
	bool join_multi = false;
	std::vector<const PlanNode *> chain; // FILTER / PROJECTION nodes, bottom-up
};

struct PipeColumn {
	std::string name;
	ValueType type = ValueType::INT32;
	int source = -1;    // >= 0: pass-through of that source column
	std::string value;  // C expression for item r
	std::string valid;  // C bool expression for item r ("true" when never NULL)
	bool nullable = false;
};

//! Launch geometry of one generated kernel.
struct Geometry {
	int block = 256;
	int items = 4; // consecutive rows per thread
	// Direct-partitioned partition passes only: full tiles arrive through two shared-memory stages
	// filled by bulk asynchronous copies (plain columns, 16-byte aligned, no NULLs, no join source).
	bool staged = false;
	// > 0: CTAs per SM the partition kernels are compiled for (__launch_bounds__ minimum blocks).
	int min_blocks = 0;
	int tile() const {
		return block * items;
	}
};

// Reserved KArgs words of the group-by kernels: the data-dependent key packing travels as arguments
// so one compiled kernel serves every instance of a plan shape. Key j: [kKeyWord + 3j] minimum,
// [+1] shift, [+2] mask (up to kMaxPackedKeys keys); the direct-partitioned mix: [kMixWord] odd
// multiplier, [+1] its inverse, [+2] key mask. Ordinary arguments stay below kKeyWord.
constexpr int kKeyWord = 96;
constexpr int kMaxPackedKeys = 8;
constexpr int kMixWord = 120;
// Join-source words: [kJoinWord] sorted right keys (u64, biased), [+1] radix directory (u32),
// [+2] bias (the right minimum), [+3] shift | bucket count << 8.
constexpr int kJoinWord = 123;

// KArgs word layout shared by every pipeline kernel:
//   w[0] = rows (pairs n*m for CROSS), w[1] = right rows m (CROSS) else 0,
//   w[2 + 2*i] = source i data pointer, w[3 + 2*i] = source i byte-validity pointer (or 0),
//   w[ConsumerBase() + k] = consumer arguments documented per Emit* function.
class PipelineCodegen {
public:
	explicit PipelineCodegen(const PipelineSpec &spec);

	const std::vector<PipeColumn> &visible() const {
		return visible_;
	}
	bool has_filter() const {
		return has_filter_;
	}
	int FindVisible(const std::string &name) const;
	int ConsumerBase() const {
		return 2 + 2 * static_cast<int>(spec_.sources.size());
	}

	//! vgpu_mat_count(tile_counts u32* @+0) and vgpu_mat_write(tile_offsets u32* @+0,
	//! then per output column c: data @+1+2c, byte-validity @+2+2c). Without a filter only
	//! vgpu_mat_write exists and writes row-aligned.
	std::string EmitMaterialize(const std::vector<int> &out_columns, const Geometry &g) const;

	//! vgpu_stats: per column c, atomic min/max of the (integer) value over every row < n into
	//! i64 mins @+2c and maxs @+2c+1 (pointers to device i64). Ignores predicates (a superset bound).
	std::string EmitStats(const std::vector<int> &columns, const Geometry &g) const;

	struct GroupKey {
		int column;     // visible column index
		int64_t min;    // value offset
		int shift;      // bit position in the packed key
		int bits;       // width
	};
	struct AggSpec {
		AggKind kind;
		int column = -1; // visible column (-1 for COUNT_STAR)
		ValueType input_type = ValueType::INT64;
		ValueType output_type = ValueType::INT64;
		// One-pass group-by, MIN/MAX: >= 0 keeps the shared-memory state as a 32-bit offset from the
		// value in this argument word (the input's minimum; its range spans less than 2^32).
		int narrow_word = -1;
	};
	struct GroupBySpec {
		std::vector<GroupKey> keys;
		std::vector<AggSpec> aggs;
		uint64_t domain = 1; // number of packed key values (direct strategy)
		int partition_bits = 0;
		int table_capacity = 4096; // bucket hash-table slots (partitioned strategy)
		int bucket_threads = 128;  // tier-1 bucket CTA size (partitioned strategy)
		// Direct-partitioned strategy (direct_bits > 0): the packed key (key_bits wide) is mixed by an
		// odd multiplier mod 2^key_bits (a bijection); the top bits pick the partition and the low
		// direct_bits index a dense shared-memory table, so no hashing or probing is needed.
		int direct_bits = 0;
		int key_bits = 0;
		uint64_t key_mult = 1, key_mult_inv = 1;
		// Heavy-key pre-aggregation (direct-partitioned only, > 0 = the most heavy keys, at most one
		// per partition): rows of the query's most frequent keys are folded into per-CTA shared
		// partial states during the scatter and leave as one partial record per key and CTA instead
		// of one record per row.
		int heavy_slots = 0;
		// FP64 sums accumulate in a per-CTA table in global memory (it stays in L2) with fire-and-forget
		// reductions, instead of shared-memory compare-and-swap loops. Direct-partitioned bucket pass:
		// the region (CTAs x FP64 fields x slots doubles) is zero on entry and left zero. One-pass
		// group-by: argument word cb+2+F+outputs, CTAs x FP64 fields x D doubles, set by each CTA.
		bool f64_l2 = false;
		// Heavy-key partition scatter: lanes of a warp step with the same heavy key combine their rows by
		// shuffles and one lane updates the CTA's partial state (fewer, uncontended shared atomics).
		bool heavy_warp = false;
		// Direct-partitioned bucket pass without the warp's equal-slot grouping and hot-key register run:
		// every record updates its slot with shared atomics (cheaper once heavy keys are pre-aggregated).
		bool bucket_plain = false;
		// One-pass group-by: fewer than 2^32 items feed it (a multi-match join source counts its matches
		// too), so shared counts add without carries.
		bool narrow_count = false;
		// One-pass group-by: no aggregate reads the row count (no COUNT, no AVG), so the count word only
		// marks a group as present -- a plain store of 1, not an atomic add.
		bool count_as_flag = false;
		// One-pass group-by: the count (narrow or a flag) takes 4 bytes per slot in shared memory instead
		// of 8 (the tables shrink, more CTAs fit on an SM).
		bool count32 = false;
	};

	//! Group-by kernels (see executor for the argument layout), all in one translation unit:
	//!  direct: vgpu_gb_direct_init, vgpu_gb_direct (+ vgpu_gb_direct_final unless DirectFinalFused)
	//!  partitioned: vgpu_gb_part_count, vgpu_gb_part_scatter, vgpu_gb_bucket (+ _retry, _global)
	//!  direct-partitioned: vgpu_gb_part_count, vgpu_gb_part_scatter, vgpu_gb_dtab_init, vgpu_gb_dbucket
	std::string EmitGroupBy(const GroupBySpec &gb, bool partitioned, const Geometry &g) const;

	//! Word offsets inside one query's row of a batch query table (see EmitBatchGroupBy).
	struct BatchLayout {
		int qwords = 0;
		int key_base = 0;
		int dom_base = 0;
		int param_base = 0;
	};
	//! Batched group-by over many queries sharing this plan template (literals read from the query
	//! table through vgpu_qp*): vgpu_batch_init, vgpu_batch_gb (persistent over (query, tile) items),
	//! vgpu_batch_final (one CTA per query).
	std::string EmitBatchGroupBy(const GroupBySpec &gb, const Geometry &g, int tile_rows, int smem_slots,
	                             const BatchLayout &L) const;
	//! Number of 8-byte per-group aggregate state fields (excluding the key), as laid out by EmitGroupBy.
	static int StateWords(const GroupBySpec &gb);
	//! Shared-memory bytes per slot of a direct-partitioned table (32-bit count and sum words).
	static int DirectSlotBytes(const GroupBySpec &gb);
	//! FP64 sum fields of a group-by's state (the per-CTA region of f64_l2 holds one table each).
	static int F64Fields(const GroupBySpec &gb);
	//! Dynamic shared memory of the one-pass group-by's tables over `domain` slots.
	static uint64_t DirectSmemBytes(const GroupBySpec &gb, uint64_t domain);
	//! One-pass group-by: the last CTA to finish its merge compacts the groups (no separate final
	//! launch), counting finished CTAs in a u32 ticket at argument word cb + 3 + F + outputs, which
	//! vgpu_gb_direct_init zeroes. Only while that word lies below the reserved key words.
	bool DirectFinalFused(const GroupBySpec &gb) const {
		return ConsumerBase() + 3 + StateWords(gb) + static_cast<int>(gb.keys.size() + gb.aggs.size()) < kKeyWord;
	}
	//! Shared-memory bytes of one heavy key's partial state in the heavy partition passes (row count,
	//! partial state of every aggregate).
	static int HeavySlotBytes(const GroupBySpec &gb);
	//! Bytes per row of one staged tile of the partition count (`scatter` false) or scatter pass: the
	//! source columns that pass reads.
	int StageRowBytes(const GroupBySpec &gb, bool scatter) const;
	//! Byte stride of one partitioned-intermediate record (packed key + carried values, 32-byte multiple).
	int RecordStride(const GroupBySpec &gb) const;

private:
	void Resolve();
	std::string EmitExpression(const Expr &expr, const std::vector<PipeColumn> &cols, int index);
	std::string Prologue() const;
	std::string LoadBlock(const Geometry &g, const std::vector<bool> &needed, bool chunked) const;
	//! Opens the per-item loop of a tile: `row`, `keep` and (for a multi-match join source) the loop over
	//! the row's matches with the needed right columns loaded at each; ItemClose closes what it opened.
	std::string ItemOpen(const Geometry &g, const std::vector<bool> &needed) const;
	std::string ItemClose() const;
	std::vector<bool> NeededSources(const std::vector<int> &extra_columns) const;

	PipelineSpec spec_;
	std::vector<PipeColumn> visible_;
	bool has_filter_ = false;
	std::string chain_code_;               // per-item code computing keep + expression values
	std::vector<std::vector<int>> chain_uses_; // per expression: source columns it reads (transitively)
	std::vector<bool> chain_sources_;      // sources read by the chain itself
	int expr_count_ = 0;
};

//! Everything a PipelineSpec contributes to generated code (sources, source kind, the chain's
//! expressions), as a compact key: equal keys generate equal code.
std::string SpecKey(const PipelineSpec &spec);
//! The same for a group-by consumer: key columns, aggregates, strategy and table parameters.
std::string GroupByKey(const PipelineCodegen::GroupBySpec &gb, bool partitioned);
//! A code generator for `spec`, shared by every pipeline with the same SpecKey (the chain's nodes are
//! read only while it is built).
std::shared_ptr<const PipelineCodegen> CodegenFor(const PipelineSpec &spec);

//! Registers the reference access forms of an expression source: returns the rewritten statement or
//! throws Error(VGPU_ERR_UNSUPPORTED) when the source uses inputs/out/row/idx any other way.
struct RewrittenExpr {
	std::string statement;                 // writes `vgpu_out`, reads `vgpu_in_<i>`
	std::vector<std::string> input_ctypes; // C type each inputs[i] is read as ("" = unused)
	std::string output_ctype;
};
RewrittenExpr RewriteExpression(const std::string &source, size_t n_inputs);

size_t CTypeSize(const std::string &ctype);

} // namespace vgpu
