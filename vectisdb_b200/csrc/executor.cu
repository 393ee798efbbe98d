// executor.cu -- plan execution (see executor.hpp).
//
// Operator mapping to the reference engine (cuda_engine/src):
//   SCAN                -> gpu_executor.cu:368-643   (H2D / cache serving; validity unpacked to bytes)
//   FILTER/PROJECTION   -> gpu_executor.cu:645-746   (one fused NVRTC kernel per chain, stable compaction)
//   GROUP_BY_AGGREGATE  -> operators/gpu_groupby.cu  (direct shared-memory tables when the packed key
//                          domain is small, else radix partitioning + per-partition hash tables)
//   HASH_JOIN           -> operators/gpu_hash_join.cu (sort-merge: LSD radix sort of the right side,
//                          per-left-row search, load-balanced expansion, gathers)
//   CROSS_PRODUCT       -> operators/gpu_cross_join.cu (left-major virtual pair space fed straight into
//                          the fused pipeline, so a filter above it never materializes the n*m pairs)
#include "executor.hpp"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <list>
#include <map>
#include <set>
#include <unordered_map>

#include "column_cache.hpp"
#include "kernels.hpp"

namespace vgpu {

namespace {

constexpr uint64_t kMaxOutputRows = 1ull << 32; // same backstop as the reference's join/cross caps
// Longest run of one right key a fused multi-match join source takes (one thread walks a row's run).
constexpr uint32_t kMaxJoinRun = 1u << 16;

struct KArgsHost {
	uint64_t w[128];
	int used = 0;
	KArgsHost() {
		std::memset(w, 0, sizeof(w));
	}
	void Set(int i, uint64_t v) {
		if (i >= kKeyWord) Fail(VGPU_ERR_UNSUPPORTED, "generated kernel needs more than 96 argument words");
		SetWord(i, v);
	}
	//! Reserved words (key packing, diagnostics) at or above kKeyWord.
	void SetWord(int i, uint64_t v) {
		w[i] = v;
		used = std::max(used, i + 1);
	}
	void SetPtr(int i, const void *p) {
		Set(i, reinterpret_cast<uint64_t>(p));
	}
};

// Returns the launch's profiler record (-1 when profiling is off), for Profiler::SetBytes.
int LaunchGenerated(Module &m, const char *name, dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                    KArgsHost &args, uint64_t bytes, uint64_t rows) {
	CUfunction f = m.Get(name);
	LaunchScope scope(name, stream, bytes, rows);
	void *params[] = {args.w};
	Runtime::Get().LaunchModuleKernel(f, grid, block, smem, stream, params);
	return scope.index();
}

// Key packing of a group-by into its kernels' reserved argument words (see kKeyWord).
void SetKeyWords(KArgsHost &k, const PipelineCodegen::GroupBySpec &gb) {
	if (gb.keys.size() > static_cast<size_t>(kMaxPackedKeys)) {
		Fail(VGPU_ERR_UNSUPPORTED, "gpu_groupby: more than 8 group keys");
	}
	for (size_t j = 0; j < gb.keys.size(); j++) {
		const auto &key = gb.keys[j];
		k.SetWord(kKeyWord + 3 * static_cast<int>(j), static_cast<uint64_t>(key.min));
		k.SetWord(kKeyWord + 3 * static_cast<int>(j) + 1, static_cast<uint64_t>(key.shift));
		k.SetWord(kKeyWord + 3 * static_cast<int>(j) + 2, key.bits >= 64 ? ~0ull : ((1ull << key.bits) - 1));
	}
	if (gb.direct_bits > 0) {
		k.SetWord(kMixWord, gb.key_mult);
		k.SetWord(kMixWord + 1, gb.key_mult_inv);
		k.SetWord(kMixWord + 2, gb.key_bits >= 64 ? ~0ull : ((1ull << gb.key_bits) - 1));
	}
}

// Most heavy keys one direct-partitioned group-by pre-aggregates (VGPU_GB_HEAVY_KEYS overrides 512).
uint32_t HeavyKeyCap() {
	if (const char *env = std::getenv("VGPU_GB_HEAVY_KEYS")) {
		return static_cast<uint32_t>(std::min<uint64_t>(4096, std::max<uint64_t>(1, std::strtoull(env, nullptr, 10))));
	}
	return 512;
}

int BitsFor(uint64_t range) {
	int b = 0;
	while (b < 64 && (range >> b) != 0) {
		b++;
	}
	return b;
}

uint64_t NextPow2(uint64_t x) {
	uint64_t p = 1;
	while (p < x) p <<= 1;
	return p;
}

uint64_t FloorPow2(uint64_t x) {
	uint64_t p = 1;
	while ((p << 1) <= x) p <<= 1;
	return p;
}

// Dense join tables built from cache-owned columns, kept across executions and keyed by the columns'
// identities (ColumnCache::Identify: contents behind an identity never change), so a repeated join with
// the same right side skips its key widening, range passes, read-back and table build. LRU over at most
// 2 GiB of tables. A table is freed when the cache has let go of it and no execution holds it, on the
// runtime's stream after the events its readers recorded (CachedJoinTable::AddReader).

struct CachedJoinTable {
	void *table = nullptr;
	uint64_t bytes = 0;
	uint64_t words[4] = {0, 0, 0, 0};  // join words; [2] (the key bias) is `bias`
	uint64_t bias = 0;
	bool inline_value = false;
	bool multi_inline = false;  // the multi-match inline table (one value slot per match)
	bool cached = false;  // held by the cache (guarded by the cache's mutex)
	//! Marks left by the executions that read the table: the free waits for all of them, wherever the
	//! last reference is dropped (an eviction by another query, a cache clear, or the reader itself).
	ReaderMarks readers;
	// Freed when the last holder lets go, on the runtime's stream, after every reader's mark.
	~CachedJoinTable() {
		if (!table) return;
		try {
			cudaStream_t s = Runtime::Get().default_stream();
			readers.WaitAll(s);
			Runtime::Get().allocator().Free(table, s);
		} catch (...) {
			// a destructor must not throw; a failing free leaves the bytes to the pool's teardown
		}
	}
};

class JoinTableCache {
public:
	static JoinTableCache &Get() {
		static JoinTableCache *cache = new JoinTableCache();  // never destroyed: outlives static teardown
		return *cache;
	}
	std::shared_ptr<CachedJoinTable> Find(const std::string &key) {
		std::lock_guard<std::mutex> lock(mu_);
		auto it = map_.find(key);
		if (it == map_.end()) return nullptr;
		lru_.splice(lru_.begin(), lru_, it->second.second);
		return it->second.first;
	}
	void Insert(const std::string &key, const std::shared_ptr<CachedJoinTable> &t) {
		std::lock_guard<std::mutex> lock(mu_);
		if (t->bytes > kCapacity || map_.count(key)) return;
		while (bytes_ + t->bytes > kCapacity && !lru_.empty()) EvictLocked(lru_.back());
		lru_.push_front(key);
		map_[key] = {t, lru_.begin()};
		bytes_ += t->bytes;
		t->cached = true;
	}
	void Clear() {
		std::lock_guard<std::mutex> lock(mu_);
		while (!lru_.empty()) EvictLocked(lru_.back());
	}

private:
	static constexpr uint64_t kCapacity = 2ull << 30;
	void EvictLocked(const std::string &key) {
		auto it = map_.find(key);
		it->second.first->cached = false;
		bytes_ -= it->second.first->bytes;
		lru_.erase(it->second.second);
		map_.erase(it);
	}
	std::mutex mu_;
	uint64_t bytes_ = 0;
	std::list<std::string> lru_;
	std::unordered_map<std::string, std::pair<std::shared_ptr<CachedJoinTable>, std::list<std::string>::iterator>> map_;
};

class Executor {
public:
	Executor(const std::vector<vgpu_column> &inputs, const ExecOptions &options, cudaStream_t stream, bool nulls_ok)
	    : inputs_(inputs), options_(options), stream_(stream), arena_(stream), nulls_supported_(nulls_ok) {
	}
	~Executor() {
		ReleaseHolds();
	}
	Executor(const Executor &) = delete;
	Executor &operator=(const Executor &) = delete;

	Relation Exec(const PlanNode &node);
	Arena &arena() {
		return arena_;
	}
	//! The plan's root: the node whose outputs become the result.
	void SetRoot(const PlanNode *root) {
		root_ = root;
	}
	//! Device word holding the row count of every result column when the execution left it there
	//! (taken from the arena: the result owns it), else nullptr.
	void *deferred_rows() const {
		return deferred_rows_;
	}
	int deferred_rows_bytes() const {
		return deferred_rows_bytes_;
	}

private:
	struct PipelineInput {
		PipelineSpec spec;
		std::vector<DevColumn> sources; // parallel to spec.sources
		uint64_t rows = 0;              // pairs for CROSS
		uint64_t right_rows = 0;
		uint64_t join_words[4] = {0, 0, 0, 0};  // join source: sorted keys, directory, bias, shift | nb << 8
	};

	Relation Scan(const PlanNode &node);
	//! `multi_ok`: the consumer accepts a join source whose right keys repeat (join_multi). `any_order`:
	//! it also takes a row's matches in any order (an aggregation), so they may come from the dense
	//! multi-match inline table, whose slots are filled in no particular order.
	PipelineInput BuildPipeline(const PlanNode &top, std::vector<const PlanNode *> chain_top_down, bool multi_ok = false,
	                            bool any_order = false);
	//! A pipeline with no chain over the columns of a relation.
	PipelineInput PipelineOver(const Relation &rel);
	//! `at_root`: the outputs are the plan's result (their row count may stay on the device).
	Relation Materialize(PipelineInput &pin, const std::vector<int> &out_cols, const std::vector<std::string> &names,
	                     bool at_root = false);
	Relation RunChain(const PlanNode &node);
	Relation GroupBy(const PlanNode &node);
	Relation Join(const PlanNode &node);
	Relation JoinMaterialize(const PlanNode &node, Relation &left, Relation &right);
	Relation JoinForPipeline(const PlanNode &node, PipelineInput &pin, bool *fused, bool multi_ok, bool any_order);
	Relation GroupByPipeline(const PlanNode &node, PipelineInput &pin);
	Relation CrossProduct(const PlanNode &node);
	void ComputeStats(PipelineInput &pin, const PipelineCodegen &cg, const std::vector<int> &cols,
	                  std::vector<std::pair<int64_t, int64_t>> &out);
	void FillArgs(const PipelineInput &pin, KArgsHost &args);
	uint64_t DirectBuckets(Module &module, const PipelineCodegen::GroupBySpec &gb, const PipelineInput &pin, uint64_t P,
	                       uint64_t G, const uint32_t *offsets, const uint32_t *total, const char *records, uint64_t n,
	                       uint64_t RS, Relation &out, int out_words, int threads, uint32_t *status,
	                       uint32_t *status_host);
	uint64_t ReadU64(const void *dev);
	uint32_t ReadU32(const void *dev);
	//! Heavy keys chosen for the partition passes of a direct-partitioned group-by (no module: none).
	//! The selection stays on the device: hmap, the key list and its length are kernel inputs.
	struct HeavyPlan {
		std::shared_ptr<Module> module;  // the heavy variant of the group-by kernels
		uint32_t *hmap = nullptr;        // [P] (state index << 16) | slot, or ~0
		uint32_t *keys = nullptr;        // [max_keys] mixed keys
		uint32_t *count = nullptr;       // selected keys (<= max_keys)
		uint32_t *overflow = nullptr;    // set when an integer partial sum leaves 64 bits (status word)
		uint32_t max_keys = 0;
		uint64_t state_bytes = 0;        // per heavy key
		size_t smem(uint64_t P) const {
			const uint64_t hoff = ((P + 32) * 4 + 15) & ~uint64_t(15);
			const uint64_t soff = (hoff + 4 * P + 4ull * max_keys + 15) & ~uint64_t(15);
			return static_cast<size_t>(soff + max_keys * state_bytes);
		}
	};
	using GroupByCompiler = std::function<std::shared_ptr<Module>(const PipelineCodegen::GroupBySpec &)>;
	HeavyPlan PlanHeavy(const PipelineCodegen::GroupBySpec &gb, const PipelineCodegen &cg, const PipelineInput &pin,
	                    const GroupByCompiler &compile, const Geometry &g, int cb, uint64_t P, uint64_t ntiles,
	                    uint64_t extra_smem);

	const std::vector<vgpu_column> &inputs_;
	//! Long-lived buffers this execution's kernels read -- kept join tables and committed cache columns
	//! -- get a mark recorded after its last kernel, which their frees wait for; the references then
	//! drop without waiting for the stream (with VGPU_EXEC_NO_SYNC the execution returns before its
	//! kernels finish), and whoever frees such a buffer later (an eviction, an invalidation, this
	//! execution dropping a table's last reference) frees it only after those kernels.
	void ReleaseHolds() {
		if (holds_.empty() && cache_reads_.empty()) return;
		// A stream with nothing left to run has finished every read (the usual case: the execution read
		// a group or row count back), so no mark is needed for the readers.
		const cudaError_t idle = cudaStreamQuery(stream_);
		if (idle == cudaSuccess) {
			holds_.clear();
			cache_reads_.clear();
			return;
		}
		if (idle == cudaErrorNotReady) cudaGetLastError();  // a status, not an error: leave none behind
		auto mark = StreamMark::After(stream_);
		for (auto &h : holds_) h->readers.Add(mark);
		holds_.clear();
		if (mark) ColumnCache::Get().AddReaders(cache_reads_, mark);
		cache_reads_.clear();
	}
	std::vector<const void *> cache_reads_;  // device data this execution read that may be cache-owned
	std::vector<std::shared_ptr<CachedJoinTable>> holds_;  // kept join tables in use by this execution
	ExecOptions options_;
	cudaStream_t stream_;
	Arena arena_;
	size_t cursor_ = 0;
	bool nulls_supported_;
	const PlanNode *root_ = nullptr;
	void *deferred_rows_ = nullptr;
	int deferred_rows_bytes_ = 8;
	//! The root's outputs stay on the device and the caller does not wait (device output, no sync): a
	//! row count nothing after the root needs stays on the device too, read when the result's columns
	//! are first asked for, the columns sized for `capacity_bytes` meanwhile. False when the count must
	//! be read now.
	bool DeferRows(void *count, int bytes, uint64_t capacity_bytes) {
		if (!(options_.output_on_device && options_.no_sync) || deferred_rows_) return false;
		if (!Runtime::Get().allocator().HasHeadroom(capacity_bytes)) return false;
		if (!arena_.Take(count)) return false;
		deferred_rows_ = count;
		deferred_rows_bytes_ = bytes;
		return true;
	}
};

// Counts are read through a pooled page-locked word: a copy into pageable memory takes the driver's
// staged path, slower for a few bytes than a direct write into pinned memory.
uint64_t Executor::ReadU64(const void *dev) {
	auto word = PinnedPool::Get().Acquire(sizeof(uint64_t));
	VGPU_CUDA(cudaMemcpyAsync(word.get(), dev, sizeof(uint64_t), cudaMemcpyDeviceToHost, stream_));
	VGPU_CUDA(cudaStreamSynchronize(stream_));
	uint64_t v;
	std::memcpy(&v, word.get(), sizeof(v));
	return v;
}

uint32_t Executor::ReadU32(const void *dev) {
	auto word = PinnedPool::Get().Acquire(sizeof(uint32_t));
	VGPU_CUDA(cudaMemcpyAsync(word.get(), dev, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
	VGPU_CUDA(cudaStreamSynchronize(stream_));
	uint32_t v;
	std::memcpy(&v, word.get(), sizeof(v));
	return v;
}

// ---- SCAN ------------------------------------------------------------------------------------------

Relation Executor::Scan(const PlanNode &node) {
	Relation out;
	if (options_.serve_whole_scan_from_cache || options_.cache_chunk_index >= 0) {
		auto &cache = ColumnCache::Get();
		for (auto &name : node.column_names) {
			DevColumn col;
			bool ok = options_.cache_chunk_index >= 0
			              ? cache.TryGetChunk(node.table, name, static_cast<uint64_t>(options_.cache_chunk_index), col)
			              : cache.GetWhole(node.table, name, col);
			if (!ok) {
				Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_executor: column '" + name + "' of table '" + node.table.ToString() +
				                                    "' was expected to be cache-resident but is no longer present -- "
				                                    "retry the query");
			}
			if (col.valid != nullptr && !nulls_supported_) {
				Fail(VGPU_ERR_UNSUPPORTED, "gpu_executor: cached column '" + name +
				                               "' contains NULLs, which this operator does not model");
			}
			cache_reads_.push_back(col.data);
			out.push_back(col);
		}
		return out;
	}
	for (size_t i = 0; i < node.column_names.size(); i++) {
		if (cursor_ >= inputs_.size()) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_executor: plan expects more scanned columns than were supplied");
		}
		const vgpu_column &in = inputs_[cursor_++];
		if (!IsValidValueType(in.type)) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_executor: input column type out of range");
		}
		DevColumn col;
		col.name = in.name ? in.name : "";
		col.type = static_cast<ValueType>(in.type);
		col.rows = in.row_count;
		if (in.validity != nullptr && !nulls_supported_) {
			Fail(VGPU_ERR_UNSUPPORTED,
			     "gpu_executor: column '" + col.name + "' contains NULLs, which this operator does not model");
		}
		const size_t bytes = static_cast<size_t>(in.row_count) * TypeSize(col.type);
		if (bytes > 0 && in.data == nullptr) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_executor: column '" + col.name + "' has rows but no data");
		}
		if (in.memory == VGPU_MEM_DEVICE) {
			col.data = const_cast<void *>(in.data);
			if (col.data != nullptr) cache_reads_.push_back(col.data);  // may be rows of a cached column
			if (col.data == nullptr) {
				col.data = arena_.Alloc(16);
			} else if (in.validity == nullptr && IsIntegerKeyType(col.type)) {
				// rows of a cached column (a borrowed prefix, say): its range covers theirs, so group-by key
				// packing needs no statistics pass
				col.has_stats = ColumnCache::Get().BoundsOf(col.data, col.type, col.rows, &col.min, &col.max);
			}
		} else {
			col.data = arena_.Alloc(bytes);
			if (bytes > 0) {
				VGPU_CUDA(cudaMemcpyAsync(col.data, in.data, bytes, cudaMemcpyHostToDevice, stream_));
			}
		}
		if (in.validity != nullptr && in.row_count > 0) {
			const size_t vbytes = (in.row_count + 7) / 8;
			const uint8_t *bitmap = in.validity;
			if (in.memory != VGPU_MEM_DEVICE) {
				uint8_t *dev_bitmap = arena_.AllocT<uint8_t>(vbytes);
				VGPU_CUDA(cudaMemcpyAsync(dev_bitmap, in.validity, vbytes, cudaMemcpyHostToDevice, stream_));
				bitmap = dev_bitmap;
			}
			col.valid = arena_.AllocT<uint8_t>(in.row_count);
			kern::UnpackValidity(bitmap, col.valid, in.row_count, stream_);
		}
		out.push_back(col);
	}
	return out;
}

// ---- pipelines -------------------------------------------------------------------------------------

void Executor::FillArgs(const PipelineInput &pin, KArgsHost &args) {
	args.Set(0, pin.rows);
	args.Set(1, pin.right_rows);
	if (pin.spec.join) {
		for (int i = 0; i < 4; i++) args.SetWord(kJoinWord + i, pin.join_words[i]);
	}
	for (size_t i = 0; i < pin.sources.size(); i++) {
		args.SetPtr(2 + 2 * static_cast<int>(i), pin.sources[i].data);
		args.SetPtr(3 + 2 * static_cast<int>(i), pin.sources[i].valid);
	}
}

Executor::PipelineInput Executor::BuildPipeline(const PlanNode &top, std::vector<const PlanNode *> chain, bool multi_ok,
                                                bool any_order) {
	// `top` is the first non-FILTER/PROJECTION node below the chain.
	PipelineInput pin;
	std::reverse(chain.begin(), chain.end()); // bottom-up
	pin.spec.chain = chain;
	if (top.op == OpType::CROSS_PRODUCT) {
		if (top.children.size() != 2) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_executor: CROSS_PRODUCT expects exactly two children");
		}
		if (top.output_columns.empty()) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_cross_join: node has no output columns");
		}
		Relation left = Exec(*top.children[0]);
		Relation right = Exec(*top.children[1]);
		if (left.empty() || right.empty()) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_cross_join: both inputs must produce at least one column");
		}
		const uint64_t ln = left.front().rows, rn = right.front().rows;
		for (auto &c : left) {
			if (c.rows != ln) Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_cross_join: left input column '" + c.name + "' row count mismatch");
		}
		for (auto &c : right) {
			if (c.rows != rn) Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_cross_join: right input column '" + c.name + "' row count mismatch");
		}
		for (auto &name : top.output_columns) {
			const DevColumn *l = nullptr, *r = nullptr;
			for (auto &c : left) if (c.name == name) { l = &c; break; }
			for (auto &c : right) if (c.name == name) { r = &c; break; }
			if (l && r) {
				Fail(VGPU_ERR_UNSUPPORTED, "gpu_cross_join: output column '" + name + "' is ambiguous (present on both sides)");
			}
			if (!l && !r) {
				Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_cross_join: output column '" + name + "' not found on either side");
			}
			SourceColumn sc;
			sc.name = name;
			sc.type = (l ? l : r)->type;
			sc.nullable = (l ? l : r)->valid != nullptr;
			sc.side = l ? 0 : 1;
			pin.spec.sources.push_back(sc);
			pin.sources.push_back(*(l ? l : r));
		}
		pin.spec.cross = true;
		if (ln == 0 || rn == 0) {
			pin.rows = 0;
			pin.right_rows = std::max<uint64_t>(rn, 1);
		} else {
			if (ln > kMaxOutputRows / rn || ln * rn > kMaxOutputRows) {
				Fail(VGPU_ERR_UNSUPPORTED, "gpu_cross_join: cross product of " + std::to_string(ln) + " x " +
				                               std::to_string(rn) + " rows is too large for GPU execution");
			}
			pin.rows = ln * rn;
			pin.right_rows = rn;
		}
		return pin;
	}
	Relation rel;
	if (top.op == OpType::HASH_JOIN) {
		bool fused = false;
		rel = JoinForPipeline(top, pin, &fused, multi_ok, any_order);
		if (fused) return pin;
	} else {
		rel = top.op == OpType::SCAN ? Scan(top) : Exec(top);
	}
	PipelineInput over = PipelineOver(rel);
	over.spec.chain = pin.spec.chain;
	return over;
}

Executor::PipelineInput Executor::PipelineOver(const Relation &rel) {
	PipelineInput pin;
	uint64_t rows = rel.empty() ? 0 : rel.front().rows;
	for (auto &c : rel) {
		if (c.rows != rows) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_executor: input column '" + c.name + "' row count mismatch");
		}
		SourceColumn sc;
		sc.name = c.name;
		sc.type = c.type;
		sc.nullable = c.valid != nullptr;
		pin.spec.sources.push_back(sc);
		pin.sources.push_back(c);
	}
	pin.rows = rows;
	return pin;
}

Relation Executor::Materialize(PipelineInput &pin, const std::vector<int> &out_cols,
                               const std::vector<std::string> &names, bool at_root) {
	auto cgp = CodegenFor(pin.spec);
	const PipelineCodegen &cg = *cgp;
	Geometry g;
	g.block = 256;
	g.items = 4;
	std::string mkey = "mat|" + SpecKey(pin.spec) + "|outs:";
	for (int c : out_cols) mkey += std::to_string(c) + ",";
	mkey += "|g:" + std::to_string(g.block) + "x" + std::to_string(g.items);
	auto module = Runtime::Get().modules().GetOrCompileMemo(mkey, [&] { return cg.EmitMaterialize(out_cols, g); });
	const uint64_t n = pin.rows;
	const uint64_t ntiles = (n + g.tile() - 1) / g.tile();
	const int sms = Runtime::Get().props().sm_count;
	const unsigned grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ntiles, uint64_t(sms) * 8)));
	const int cb = cg.ConsumerBase();
	uint64_t out_rows = n;
	void *tile_offsets = nullptr;
	if (cg.has_filter() && n > 0) {
		uint64_t in_bytes = 0;
		for (auto &s : pin.sources) in_bytes += s.rows * TypeSize(s.type);
		KArgsHost a;
		FillArgs(pin, a);
		if (pin.spec.join_multi) {  // 64-bit tile counts: the matches can outnumber the rows
			uint64_t *tile_counts = arena_.AllocT<uint64_t>(ntiles);
			uint64_t *total = arena_.AllocT<uint64_t>(1);
			a.SetPtr(cb, tile_counts);
			LaunchGenerated(*module, "vgpu_mat_count", grid, g.block, 0, stream_, a, in_bytes, n);
			kern::ExclusiveScanU64(tile_counts, tile_counts, ntiles, total, arena_);
			out_rows = ReadU64(total);
			if (out_rows >= kMaxOutputRows) {
				Fail(VGPU_ERR_UNSUPPORTED, "gpu_hash_join: join produces " + std::to_string(out_rows) +
				                               " rows, more than this GPU path materializes");
			}
			tile_offsets = tile_counts;
		} else {
			uint32_t *tile_counts = arena_.AllocT<uint32_t>(ntiles);
			uint32_t *total = arena_.AllocT<uint32_t>(1);
			a.SetPtr(cb, tile_counts);
			LaunchGenerated(*module, "vgpu_mat_count", grid, g.block, 0, stream_, a, in_bytes, n);
			kern::ExclusiveScanU32(tile_counts, tile_counts, ntiles, total, arena_);
			// at the root, outputs without NULL masks may take a row per input row and leave the count
			// on the device
			bool defer = at_root;
			uint64_t row_bytes = 0;
			for (int c : out_cols) {
				defer = defer && !cg.visible()[c].nullable;
				row_bytes += TypeSize(cg.visible()[c].type);
			}
			if (defer && DeferRows(total, 4, n * row_bytes)) {
				out_rows = n;
			} else {
				out_rows = ReadU32(total);
			}
			tile_offsets = tile_counts;
		}
	}
	Relation out;
	KArgsHost a;
	FillArgs(pin, a);
	a.SetPtr(cb, tile_offsets);
	for (size_t c = 0; c < out_cols.size(); c++) {
		const auto &vc = cg.visible()[out_cols[c]];
		DevColumn col;
		col.name = names[c];
		col.type = vc.type;
		col.rows = out_rows;
		col.data = arena_.Alloc(out_rows * TypeSize(vc.type));
		if (vc.nullable) {
			col.valid = arena_.AllocT<uint8_t>(out_rows);
		}
		if (vc.source >= 0 && pin.sources[vc.source].has_stats) {
			col.has_stats = true;
			col.min = pin.sources[vc.source].min;
			col.max = pin.sources[vc.source].max;
		}
		a.SetPtr(cb + 1 + 2 * static_cast<int>(c), col.data);
		a.SetPtr(cb + 2 + 2 * static_cast<int>(c), col.valid);
		out.push_back(col);
	}
	if (n > 0 && (out_rows > 0 || !cg.has_filter())) {
		LaunchGenerated(*module, "vgpu_mat_write", grid, g.block, 0, stream_, a, 0, n);
	}
	return out;
}

Relation Executor::RunChain(const PlanNode &node) {
	std::vector<const PlanNode *> chain;
	const PlanNode *cur = &node;
	while (cur->op == OpType::FILTER || cur->op == OpType::PROJECTION) {
		if (cur->children.size() != 1) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, std::string("gpu_executor: ") +
			                                    (cur->op == OpType::FILTER ? "FILTER" : "PROJECTION") +
			                                    " expects exactly one child");
		}
		chain.push_back(cur);
		cur = cur->children[0].get();
	}
	PipelineInput pin = BuildPipeline(*cur, chain, true);
	auto probe_cg = CodegenFor(pin.spec);
	const PipelineCodegen &probe = *probe_cg;
	std::vector<int> outs;
	std::vector<std::string> names;
	for (size_t i = 0; i < probe.visible().size(); i++) {
		outs.push_back(static_cast<int>(i));
		names.push_back(probe.visible()[i].name);
	}
	return Materialize(pin, outs, names, &node == root_);
}

Relation Executor::CrossProduct(const PlanNode &node) {
	PipelineInput pin = BuildPipeline(node, {});
	std::vector<int> outs;
	std::vector<std::string> names;
	for (size_t i = 0; i < pin.spec.sources.size(); i++) {
		outs.push_back(static_cast<int>(i));
		names.push_back(pin.spec.sources[i].name);
	}
	return Materialize(pin, outs, names);
}

void Executor::ComputeStats(PipelineInput &pin, const PipelineCodegen &cg, const std::vector<int> &cols,
                            std::vector<std::pair<int64_t, int64_t>> &out) {
	out.assign(cols.size(), {0, 0});
	std::vector<int> missing;
	std::vector<size_t> missing_pos;
	for (size_t i = 0; i < cols.size(); i++) {
		const auto &vc = cg.visible()[cols[i]];
		if (vc.source >= 0 && pin.sources[vc.source].has_stats) {
			out[i] = {pin.sources[vc.source].min, pin.sources[vc.source].max};
		} else {
			missing.push_back(cols[i]);
			missing_pos.push_back(i);
		}
	}
	if (missing.empty()) {
		return;
	}
	Geometry g;
	g.block = 256;
	g.items = 4;
	std::string skey = "stats|" + SpecKey(pin.spec) + "|cols:";
	for (int c : missing) skey += std::to_string(c) + ",";
	auto module = Runtime::Get().modules().GetOrCompileMemo(skey, [&] { return cg.EmitStats(missing, g); });
	int64_t *mm = arena_.AllocT<int64_t>(2 * missing.size());
	std::vector<int64_t> init(2 * missing.size());
	for (size_t i = 0; i < missing.size(); i++) {
		init[2 * i] = INT64_MAX;
		init[2 * i + 1] = INT64_MIN;
	}
	VGPU_CUDA(cudaMemcpyAsync(mm, init.data(), init.size() * 8, cudaMemcpyHostToDevice, stream_));
	KArgsHost a;
	FillArgs(pin, a);
	const int cb = cg.ConsumerBase();
	for (size_t i = 0; i < missing.size(); i++) {
		a.SetPtr(cb + 2 * static_cast<int>(i), mm + 2 * i);
		a.SetPtr(cb + 2 * static_cast<int>(i) + 1, mm + 2 * i + 1);
	}
	const uint64_t ntiles = (pin.rows + g.tile() - 1) / g.tile();
	const unsigned grid = static_cast<unsigned>(
	    std::max<uint64_t>(1, std::min<uint64_t>(ntiles, uint64_t(Runtime::Get().props().sm_count) * 8)));
	if (pin.rows > 0) {
		LaunchGenerated(*module, "vgpu_stats", grid, g.block, 0, stream_, a, 0, pin.rows);
	}
	std::vector<int64_t> host(2 * missing.size());
	VGPU_CUDA(cudaMemcpyAsync(host.data(), mm, host.size() * 8, cudaMemcpyDeviceToHost, stream_));
	VGPU_CUDA(cudaStreamSynchronize(stream_));
	for (size_t i = 0; i < missing.size(); i++) {
		out[missing_pos[i]] = {host[2 * i], host[2 * i + 1]};
	}
}

// ---- GROUP BY --------------------------------------------------------------------------------------

// Group-by validation shared by the single-query and batched paths. Mirrors
// operators/gpu_groupby.cu:224-299 and :320-350.
PipelineCodegen::GroupBySpec ValidateGroupByNode(const PlanNode &node, const PipelineCodegen &cg,
                                                 std::vector<int> &key_cols) {
	auto find = [&](const std::string &name, const char *what) {
		int c = cg.FindVisible(name);
		if (c < 0) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, std::string("gpu_groupby: ") + what + " column '" + name + "' not found");
		}
		return c;
	};
	// Validation mirrors operators/gpu_groupby.cu:224-299 and :320-350.
	key_cols.clear();
	for (auto &k : node.group_keys) {
		int c = find(k, "group key");
		const ValueType t = cg.visible()[c].type;
		if (!IsIntegerKeyType(t)) {
			Fail(VGPU_ERR_UNSUPPORTED, "gpu_groupby: group key '" + k +
			                               "' is not an integer/boolean column, which this GPU path requires");
		}
		key_cols.push_back(c);
	}
	PipelineCodegen::GroupBySpec gb;
	for (auto &agg : node.aggregates) {
		PipelineCodegen::AggSpec s;
		s.kind = agg.kind;
		s.output_type = agg.output_type;
		if (agg.kind == AggKind::COUNT_STAR) {
			if (agg.output_type != ValueType::INT64) Fail(VGPU_ERR_UNSUPPORTED, "gpu_groupby: COUNT(*) must produce INT64");
			gb.aggs.push_back(s);
			continue;
		}
		s.column = find(agg.input_column, "aggregate input");
		s.input_type = cg.visible()[s.column].type;
		const ValueType in = s.input_type;
		switch (agg.kind) {
		case AggKind::COUNT:
			if (agg.output_type != ValueType::INT64) Fail(VGPU_ERR_UNSUPPORTED, "gpu_groupby: COUNT must produce INT64");
			break;
		case AggKind::SUM:
			if (IsFloatType(in)) {
				if (agg.output_type != ValueType::FLOAT64) {
					Fail(VGPU_ERR_UNSUPPORTED, "gpu_groupby: SUM on this GPU path supports only FLOAT/DOUBLE input "
					                           "producing DOUBLE");
				}
			} else if (in == ValueType::INT16 || in == ValueType::INT32 || in == ValueType::INT64) {
				// DuckDB: SUM over INTEGER/BIGINT/DECIMAL(<=18) returns a 128-bit integer (exact).
				if (agg.output_type != ValueType::HUGEINT) {
					Fail(VGPU_ERR_UNSUPPORTED, "gpu_groupby: SUM over an integer column must produce HUGEINT");
				}
			} else {
				Fail(VGPU_ERR_UNSUPPORTED, "gpu_groupby: SUM on this GPU path supports only FLOAT/DOUBLE input "
				                           "producing DOUBLE");
			}
			break;
		case AggKind::AVG:
			if (agg.output_type != ValueType::FLOAT64) Fail(VGPU_ERR_UNSUPPORTED, "gpu_groupby: AVG must produce DOUBLE");
			if (!(in == ValueType::INT16 || in == ValueType::INT32 || in == ValueType::INT64 || IsFloatType(in))) {
				Fail(VGPU_ERR_UNSUPPORTED, "gpu_groupby: AVG supports numeric columns only");
			}
			break;
		case AggKind::MIN:
		case AggKind::MAX:
			if (agg.output_type != in) {
				Fail(VGPU_ERR_UNSUPPORTED, "gpu_groupby: MIN/MAX output type must match its input column type");
			}
			if (!IsIntegerKeyType(in)) {
				Fail(VGPU_ERR_UNSUPPORTED, "gpu_groupby: MIN/MAX on this GPU path supports only integer/boolean columns");
			}
			break;
		default:
			break;
		}
		gb.aggs.push_back(s);
	}
	return gb;
}

Relation Executor::GroupBy(const PlanNode &node) {
	if (node.children.size() != 1) {
		Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_executor: GROUP_BY_AGGREGATE expects exactly one child");
	}
	if (node.group_keys.empty() && node.aggregates.empty()) {
		Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_groupby: node has neither group keys nor aggregates");
	}
	std::vector<const PlanNode *> chain;
	const PlanNode *cur = node.children[0].get();
	while (cur->op == OpType::FILTER || cur->op == OpType::PROJECTION) {
		if (cur->children.size() != 1) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_executor: FILTER/PROJECTION expects exactly one child");
		}
		chain.push_back(cur);
		cur = cur->children[0].get();
	}
	PipelineInput pin = BuildPipeline(*cur, chain, true, true);
	return GroupByPipeline(node, pin);
}

Relation Executor::GroupByPipeline(const PlanNode &node, PipelineInput &pin) {
	auto cgp = CodegenFor(pin.spec);
	const PipelineCodegen &cg = *cgp;
	if (cg.visible().empty()) {
		Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_groupby: input operator produced no columns to group");
	}
	std::vector<int> key_cols;
	PipelineCodegen::GroupBySpec gb = ValidateGroupByNode(node, cg, key_cols);
	const uint64_t n = pin.rows;
	auto empty_result = [&]() {
		Relation out;
		for (size_t i = 0; i < key_cols.size(); i++) {
			DevColumn c;
			c.name = node.group_keys[i];
			c.type = cg.visible()[key_cols[i]].type;
			c.rows = 0;
			c.data = arena_.Alloc(0);
			out.push_back(c);
		}
		for (size_t i = 0; i < node.aggregates.size(); i++) {
			DevColumn c;
			c.name = "agg_" + std::to_string(i);
			c.type = node.aggregates[i].output_type;
			c.rows = 0;
			c.data = arena_.Alloc(0);
			out.push_back(c);
		}
		return out;
	};
	const char *kEmptyGlobal = "gpu_groupby: global aggregate over an empty input needs NULL results, which this GPU "
	                           "path cannot represent";
	if (n == 0) {
		if (node.group_keys.empty()) Fail(VGPU_ERR_UNSUPPORTED, kEmptyGlobal);
		return empty_result();
	}
	// Key packing from the key ranges.
	std::vector<std::pair<int64_t, int64_t>> ranges;
	ComputeStats(pin, cg, key_cols, ranges);
	int shift = 0;
	for (size_t i = 0; i < key_cols.size(); i++) {
		PipelineCodegen::GroupKey k;
		k.column = key_cols[i];
		k.min = ranges[i].first;
		const uint64_t span = static_cast<uint64_t>(ranges[i].second) - static_cast<uint64_t>(ranges[i].first);
		k.bits = BitsFor(span);
		k.shift = shift;
		shift += k.bits;
		gb.keys.push_back(k);
	}
	if (shift > 63) {
		Fail(VGPU_ERR_UNSUPPORTED, "gpu_groupby: the group key ranges need " + std::to_string(shift) +
		                               " bits packed, more than the 63 this path supports");
	}
	const auto &props = Runtime::Get().props();
	const int F = PipelineCodegen::StateWords(gb);
	const uint64_t domain = 1ull << shift;
	const bool direct = domain * static_cast<uint64_t>(F) * 8 <= 96 * 1024;  // 8-byte words per slot bound the choice
	// FP64 sums of the one-pass group-by in L2-resident per-CTA tables (VGPU_GB_DIRECT_F64_L2=1)
	const char *env_dl2 = std::getenv("VGPU_GB_DIRECT_F64_L2");
	const int direct_f64 = PipelineCodegen::F64Fields(gb);
	const bool direct_l2 = direct && direct_f64 > 0 && env_dl2 && std::strcmp(env_dl2, "1") == 0;
	if (!direct && pin.spec.join_multi) {
		// the partitioned strategies take one item per input row: expand the join's matches into a
		// relation first, then group that
		std::vector<int> outs;
		std::vector<std::string> names;
		for (size_t i = 0; i < cg.visible().size(); i++) {
			outs.push_back(static_cast<int>(i));
			names.push_back(cg.visible()[i].name);
		}
		Relation flat = Materialize(pin, outs, names);
		PipelineInput over = PipelineOver(flat);
		return GroupByPipeline(node, over);
	}
	const int key_words = static_cast<int>(gb.keys.size());
	const int out_words = key_words + static_cast<int>(gb.aggs.size());
	gb.domain = domain;

	// Output columns, sized for the largest possible group count.
	const uint64_t cap_rows = direct ? domain : std::min<uint64_t>(domain, n);
	Relation out;
	for (size_t i = 0; i < key_cols.size(); i++) {
		DevColumn c;
		c.name = node.group_keys[i];
		c.type = cg.visible()[key_cols[i]].type;
		c.data = arena_.Alloc(cap_rows * TypeSize(c.type));
		c.has_stats = true;
		c.min = ranges[i].first;
		c.max = ranges[i].second;
		out.push_back(c);
	}
	for (size_t i = 0; i < node.aggregates.size(); i++) {
		DevColumn c;
		c.name = "agg_" + std::to_string(i);
		c.type = node.aggregates[i].output_type;
		c.data = arena_.Alloc(cap_rows * TypeSize(c.type));
		out.push_back(c);
	}
	uint64_t in_bytes = 0;
	for (auto &s : pin.sources) in_bytes += s.rows * TypeSize(s.type);
	const int cb = cg.ConsumerBase();
	uint64_t groups = 0;

	if (direct) {
		// a CTA's table sees at most n items (a multi-match join source can expand past n: keep carries)
		gb.narrow_count = !pin.spec.join_multi && n < (1ull << 32);
		gb.count_as_flag = true;  // unless an aggregate reads the count
		for (auto &ag : gb.aggs) {
			if (ag.kind == AggKind::COUNT || ag.kind == AggKind::COUNT_STAR || ag.kind == AggKind::AVG) gb.count_as_flag = false;
		}
		// 4-byte count slots pay where each probe row expands into several updates (the multi-match join
		// source: the fourth CTA per SM hides their latency); over single rows the extra CTAs' table merges
		// cost more than they hide (a 2^28-row probe into 4096 groups: 1.45 -> 1.51 ms)
		gb.count32 = pin.spec.join_multi;
		gb.f64_l2 = direct_l2;
		// MIN/MAX over a cached integer column whose values span less than 2^32: the shared tables hold
		// 32-bit offsets from the column's minimum (native 32-bit atomics on the slot's low word instead
		// of 64-bit ones), the minimum in an argument word after the compaction ticket.
		std::vector<std::pair<int, int64_t>> narrow_args;
		if (cg.DirectFinalFused(gb)) {
			int word = cb + 4 + F + out_words;
			for (auto &ag : gb.aggs) {
				if (ag.kind != AggKind::MIN && ag.kind != AggKind::MAX) continue;
				if (ag.input_type != ValueType::INT16 && ag.input_type != ValueType::INT32 &&
				    ag.input_type != ValueType::INT64) {
					continue;
				}
				const PipeColumn &vc = cg.visible()[ag.column];
				if (vc.nullable || vc.source < 0 || vc.type != ag.input_type) continue;
				const DevColumn &src = pin.sources[vc.source];
				if (!src.has_stats || src.max < src.min ||
				    static_cast<uint64_t>(src.max) - static_cast<uint64_t>(src.min) > 0xffffffffull) {
					continue;
				}
				if (word >= kKeyWord) break;
				ag.narrow_word = word;
				narrow_args.emplace_back(word++, src.min);
			}
		}
		Geometry g;
		g.block = 512;
		g.items = 4;  // also for a join source (a fused 2^28-row probe: 4 rows per thread 1.68 ms, 8 1.71 ms)
		if (const char *env = std::getenv("VGPU_GB_DIRECT_ITEMS")) {  // tuning override
			g.items = std::max(1, std::min(32, std::atoi(env)));
		}
		if (const char *env = std::getenv("VGPU_GB_DIRECT_BLOCK")) {  // tuning override (whole warps)
			g.block = std::max(64, std::min(1024, std::atoi(env))) / 32 * 32;
		}
		const std::string gkey = SpecKey(pin.spec) + "|" + GroupByKey(gb, false) + "|g:" + std::to_string(g.block) + "x" +
		                         std::to_string(g.items);
		auto module = Runtime::Get().modules().GetOrCompileMemo(gkey, [&] { return cg.EmitGroupBy(gb, false, g); });
		uint64_t *fields = arena_.AllocT<uint64_t>(domain * F);
		uint64_t *count = arena_.AllocT<uint64_t>(1);
		KArgsHost a;
		FillArgs(pin, a);
		SetKeyWords(a, gb);
		a.Set(cb, domain);
		for (int f = 0; f < F; f++) a.SetPtr(cb + 1 + f, fields + domain * f);
		for (int w = 0; w < out_words; w++) a.SetPtr(cb + 1 + F + w, out[w].data);
		a.SetPtr(cb + 1 + F + out_words, count);
		const bool fused_final = cg.DirectFinalFused(gb);
		if (fused_final) a.SetPtr(cb + 3 + F + out_words, arena_.AllocT<uint32_t>(1));  // finished-CTA ticket
		for (auto &na : narrow_args) a.Set(na.first, static_cast<uint64_t>(na.second));
		const unsigned init_grid = static_cast<unsigned>(std::min<uint64_t>((domain + 255) / 256, 1024));
		LaunchGenerated(*module, "vgpu_gb_direct_init", init_grid, 256, 0, stream_, a, domain * F * 8, domain);
		const size_t smem = static_cast<size_t>(PipelineCodegen::DirectSmemBytes(gb, domain));
		CUfunction f = module->Get("vgpu_gb_direct");
		int occ = std::max(1, Runtime::Get().MaxActiveBlocks(f, g.block, smem));
		const uint64_t ntiles = (n + g.tile() - 1) / g.tile();
		const unsigned grid =
		    static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ntiles, uint64_t(props.sm_count) * occ)));
		if (direct_l2) a.SetPtr(cb + 2 + F + out_words, arena_.AllocT<uint64_t>(uint64_t(grid) * direct_f64 * domain));
		LaunchGenerated(*module, "vgpu_gb_direct", grid, g.block, smem, stream_, a, in_bytes, n);
		if (!fused_final) LaunchGenerated(*module, "vgpu_gb_direct_final", 1, 1024, 0, stream_, a, domain * F * 8, domain);
		if (&node == root_ && !node.group_keys.empty() && DeferRows(count, 8, 0)) {
			groups = domain;  // the columns already hold a slot per key value
		} else {
			groups = ReadU64(count);
		}
	} else {
		// Partitioned. Tier-1 bucket tables are small (about 48 KB, 128 threads per CTA, several CTAs per
		// SM): few warps share a table, so same-slot atomics of moderately heavy keys queue behind at most
		// four warps. Partitions are sized so a tier-1 table would run half full at the key-range bound;
		// the ones that do not fit are retried on the device with the largest shared-memory table.
		const uint64_t slot_bytes = (1 + F) * 8;
		const uint64_t smem_cap = std::min<uint64_t>(props.smem_optin > 4096 ? props.smem_optin - 4096 : 48 * 1024,
		                                             200 * 1024);
		uint64_t C2 = std::max<uint64_t>(256, FloorPow2(smem_cap / slot_bytes));
		if (const char *env = std::getenv("VGPU_GB_RETRY_SLOTS")) {  // tuning/testing override (power of two)
			C2 = std::min<uint64_t>(C2, std::max<uint64_t>(64, FloorPow2(std::strtoull(env, nullptr, 10))));
		}
		uint64_t C = std::min<uint64_t>(C2, std::max<uint64_t>(256, FloorPow2((48 * 1024) / slot_bytes)));
		if (const char *env = std::getenv("VGPU_GB_TABLE_SLOTS")) {  // tuning override (power of two)
			C = std::min<uint64_t>(C2, std::max<uint64_t>(256, FloorPow2(std::strtoull(env, nullptr, 10))));
		}
		const uint64_t expected_groups = std::min<uint64_t>(domain, n);
		uint64_t P = NextPow2(std::max<uint64_t>(1, (expected_groups + C / 2 - 1) / (C / 2)));
		P = std::min<uint64_t>(P, 16384);
		if (const char *env = std::getenv("VGPU_GB_PARTITIONS")) {  // tuning override (power of two)
			P = std::min<uint64_t>(16384, std::max<uint64_t>(1, FloorPow2(std::strtoull(env, nullptr, 10))));
		}
		// Direct-partitioned when the packed key space is dense enough to be walked slot by slot
		// (at most 4 slots per input row) and splits into at most 2^14 partitions of the largest
		// shared-memory table: a row then costs no hashing and no probing.
		const uint64_t dslot = static_cast<uint64_t>(PipelineCodegen::DirectSlotBytes(gb));
		const int dbits_max = BitsFor(FloorPow2(smem_cap / dslot)) - 1;
		bool dpart = shift <= dbits_max + 14 && domain <= 4 * n;
		if (const char *env = std::getenv("VGPU_GB_STRATEGY")) {  // testing override: "hash" or "direct"
			if (std::strcmp(env, "hash") == 0) dpart = false;
			if (std::strcmp(env, "direct") == 0) dpart = shift <= dbits_max + 14;
		}
		if (dpart) {
			// the table size depends on the plan shape only (slot bytes), not on the data, so every
			// instance of a query shape reuses one compiled kernel
			int dbits = dbits_max;
			if (const char *env = std::getenv("VGPU_GB_DIRECT_BITS")) {  // tuning override
				dbits = std::min(dbits_max, std::max(5, std::atoi(env)));
			}
			dbits = std::max(dbits, shift - 14);  // at most 2^14 partitions (the partition histograms)
			gb.direct_bits = dbits;
			gb.key_bits = shift;
			// FP64 sums of the bucket pass in L2 through reductions (VGPU_GB_F64_L2=0: shared CAS loops)
			const char *env_l2 = std::getenv("VGPU_GB_F64_L2");
			gb.f64_l2 = PipelineCodegen::F64Fields(gb) > 0 && !(env_l2 && std::strcmp(env_l2, "0") == 0);
			// without heavy-key pre-aggregation the bucket pass groups equal slots per warp step (hot keys);
			// VGPU_GB_BUCKET_PLAIN=1 makes every record update its slot itself
			const char *env_plain = std::getenv("VGPU_GB_BUCKET_PLAIN");
			gb.bucket_plain = env_plain && std::strcmp(env_plain, "1") == 0;
			const uint64_t mask = (1ull << shift) - 1;
			const uint64_t M = (0x9e3779b97f4a7c15ull & mask) | 1ull;
			uint64_t inv = M;  // Newton iteration for the inverse mod 2^64: each step doubles the valid bits
			for (int it = 0; it < 6; it++) inv *= 2 - M * inv;
			gb.key_mult = M;
			gb.key_mult_inv = inv & mask;
			P = 1ull << std::max(0, shift - dbits);
		}
		int pbits = BitsFor(P - 1);
		if (P == 1) pbits = 0;
		gb.partition_bits = pbits;
		gb.table_capacity = static_cast<int>(C);
		int T1 = gb.direct_bits > 0 ? 1024 : 128;
		if (const char *env = std::getenv("VGPU_GB_BUCKET_THREADS")) {  // tuning override (128..1024)
			T1 = static_cast<int>(std::min<uint64_t>(1024, std::max<uint64_t>(128, FloorPow2(std::strtoull(env, nullptr, 10)))));
		}
		gb.bucket_threads = T1;
		Geometry g;
		g.block = 256;
		g.items = 8;
		// Staged tiles (direct-partitioned): the partition passes' full tiles arrive in shared memory by
		// bulk asynchronous copies, two tiles ahead, instead of as per-thread loads. Needs plain columns
		// (no join or cross-product source, no NULLs) whose base addresses are 16-byte aligned, and room
		// for two stages beside the counters and the heavy-key state. 1024 threads × 2 rows per tile.
		// VGPU_GB_STAGED=0 turns it off.
		const char *staged_env = std::getenv("VGPU_GB_STAGED");
		bool staged = gb.direct_bits > 0 && !pin.spec.join && !pin.spec.cross && cb + 14 < kKeyWord &&
		              !(staged_env && std::strcmp(staged_env, "0") == 0);
		for (auto &src : pin.sources) {
			if (src.valid || (reinterpret_cast<uintptr_t>(src.data) & 15u) != 0) staged = false;
		}
		if (staged) {
			// 32 warps per SM (one CTA, registers capped at 64 per thread): the passes are latency-bound on
			// shared-memory atomics, so more warps beat more rows per thread
			g.block = 1024;
			g.items = 2;
			g.min_blocks = 1;
		}
		// tuning overrides: threads per CTA (128..1024), rows per thread (1..8), CTAs per SM to compile for
		if (const char *env = std::getenv("VGPU_GB_PART_BLOCK")) {
			g.block = static_cast<int>(std::min<uint64_t>(1024, std::max<uint64_t>(128, FloorPow2(std::strtoull(env, nullptr, 10)))));
		}
		if (const char *env = std::getenv("VGPU_GB_PART_ITEMS")) {
			g.items = static_cast<int>(std::min<uint64_t>(8, std::max<uint64_t>(1, FloorPow2(std::strtoull(env, nullptr, 10)))));
		}
		if (const char *env = std::getenv("VGPU_GB_PART_MINB")) g.min_blocks = std::max(0, std::min(4, std::atoi(env)));
		// bytes of the two stages of the count and the scatter pass
		uint64_t stage2_count = staged ? 2ull * g.tile() * cg.StageRowBytes(gb, false) : 0;
		uint64_t stage2_scatter = staged ? 2ull * g.tile() * cg.StageRowBytes(gb, true) : 0;
		if (staged) {
			// room for the stages beside the counters and, should heavy keys be chosen, their state:
			// pre-aggregation saves more than staging, so staging yields when both do not fit
			HeavyPlan room;
			room.max_keys = HeavyKeyCap();
			room.state_bytes = static_cast<uint64_t>(PipelineCodegen::HeavySlotBytes(gb));
			if (room.smem(P) + 128 + stage2_scatter + 1024 > static_cast<uint64_t>(props.smem_optin)) {
				staged = false;
				stage2_count = stage2_scatter = 0;
				g.block = 256;
				g.items = 8;
				g.min_blocks = 0;
			}
		}
		g.staged = staged;
		auto compile = [&](const PipelineCodegen::GroupBySpec &spec) {
			const std::string gkey = SpecKey(pin.spec) + "|" + GroupByKey(spec, true) + "|g:" + std::to_string(g.block) +
			                         "x" + std::to_string(g.items) + (g.staged ? "s" : "") + "m" + std::to_string(g.min_blocks);
			return Runtime::Get().modules().GetOrCompileMemo(gkey, [&] { return cg.EmitGroupBy(spec, true, g); });
		};
		const uint64_t ntiles = (n + g.tile() - 1) / g.tile();
		if (n >= (1ull << 32)) Fail(VGPU_ERR_UNSUPPORTED, "gpu_groupby: more than 2^32 input rows");
		// Records of the partitioned intermediate: packed key + carried values, RS bytes each.
		const uint64_t RS = static_cast<uint64_t>(cg.RecordStride(gb));
		const size_t part_smem = (P + 32) * 4;  // partition counters + per-lane dummies for filtered rows
		// Heavy-key pre-aggregation (direct-partitioned): a sample of tiles finds the most frequent keys,
		// whose rows the partition passes fold into per-CTA shared partial states; each CTA then writes
		// one partial record per such key instead of one record per row.
		HeavyPlan heavy = PlanHeavy(gb, cg, pin, compile, g, cb, P, ntiles, staged ? 128 + stage2_scatter : 0);
		// status words read back once per attempt: [0, 6) the bucket pass's plan and group count,
		// [6] heavy-key partial overflow, [7] staging error
		uint32_t *status = arena_.AllocT<uint32_t>(8);
		uint32_t status_host[8];
		VGPU_CUDA(cudaMemsetAsync(status, 0, 32, stream_));
		if (heavy.module) heavy.overflow = status + 6;
		uint32_t *stage_err = staged ? status + 7 : nullptr;
		for (int attempt = 0;; ++attempt) {
			const bool use_heavy = heavy.module && attempt == 0;
			auto module = use_heavy ? heavy.module : compile(gb);
			const size_t smem = use_heavy ? heavy.smem(P) : part_smem;
			// stages after the counters (and heavy-key state), 128-byte aligned
			const size_t stage_off = staged ? ((smem + 127) & ~size_t(127)) : 0;
			const size_t smem_count = staged ? stage_off + stage2_count : smem;
			const size_t smem_scatter = staged ? stage_off + stage2_scatter : smem;
			CUfunction fcount = module->Get("vgpu_gb_part_count");
			int occ = std::max(1, Runtime::Get().MaxActiveBlocks(fcount, g.block, smem_count));
			occ = std::min(occ, std::max(1, Runtime::Get().MaxActiveBlocks(module->Get("vgpu_gb_part_scatter"), g.block,
			                                                             smem_scatter)));
			if (const char *env = std::getenv("VGPU_GB_PART_OCC")) {  // tuning override: CTAs per SM
				occ = std::min(occ, std::max(1, std::atoi(env)));
			}
			const uint64_t G = std::max<uint64_t>(1, std::min<uint64_t>(ntiles, uint64_t(props.sm_count) * occ));
			const uint64_t tpc = (ntiles + G - 1) / G;
			// every CTA writes one partial record per heavy key
			const uint64_t n_rec = n + (use_heavy ? G * heavy.max_keys : 0);
			if (n_rec >= (1ull << 32)) Fail(VGPU_ERR_UNSUPPORTED, "gpu_groupby: more than 2^32 partition records");
			uint32_t *offsets = arena_.AllocT<uint32_t>(P * G);
			uint32_t *total = arena_.AllocT<uint32_t>(1);
			KArgsHost a;
			FillArgs(pin, a);
			SetKeyWords(a, gb);
			a.Set(cb, P);
			a.Set(cb + 1, static_cast<uint64_t>(pbits));
			a.Set(cb + 2, tpc);
			a.SetPtr(cb + 3, offsets);
			if (use_heavy) {
				a.SetPtr(cb + 5, heavy.hmap);
				a.SetPtr(cb + 10, heavy.overflow);
				a.SetPtr(cb + 11, heavy.keys);
				a.SetPtr(cb + 12, heavy.count);
			}
			if (staged) {
				a.Set(cb + 13, stage_off);
				a.SetPtr(cb + 14, stage_err);
			}
			LaunchGenerated(*module, "vgpu_gb_part_count", static_cast<unsigned>(G), g.block, smem_count, stream_, a,
			                in_bytes, n);
			kern::ExclusiveScanU32(offsets, offsets, P * G, total, arena_);
			char *records = static_cast<char *>(arena_.Alloc(n_rec * RS));
			a.SetPtr(cb + 4, records);
			const int scatter_rec = LaunchGenerated(*module, "vgpu_gb_part_scatter", static_cast<unsigned>(G), g.block,
			                                        smem_scatter, stream_, a, in_bytes, n);
			if (gb.direct_bits > 0) {
				groups = DirectBuckets(*module, gb, pin, P, G, offsets, total, records, n_rec, RS, out, out_words, T1,
				                       status, status_host);
				if (staged && status_host[7] != 0) {
					Fail(VGPU_ERR_CUDA, "gpu_groupby: a staged tile copy did not complete within a second");
				}
				// the scatter's bytes: the columns it reads once and the records it wrote
				Runtime::Get().profiler().SetBytes(scatter_rec, in_bytes + static_cast<uint64_t>(status_host[3]) * RS);
				if (use_heavy && status_host[6] != 0) continue;  // a partial sum left 64 bits: redo plainly
				for (auto &c : out) c.rows = groups;
				return out;
			}
			// bucket tables. control: [0] work counter, [1] overflow count, [2] retry count, [3] retry work
			// counter, [4, 4+P) overflow flags, [4+P, 4+2P) retry list.
			const int W = cb + 6;
			const int L = W + 4 + out_words;
			uint32_t *control = arena_.AllocT<uint32_t>(4 + 2 * P);
			uint64_t *out_count = arena_.AllocT<uint64_t>(1);
			VGPU_CUDA(cudaMemsetAsync(control, 0, (4 + 2 * P) * 4, stream_));
			VGPU_CUDA(cudaMemsetAsync(out_count, 0, 8, stream_));
			KArgsHost b;
			FillArgs(pin, b);
			SetKeyWords(b, gb);
			b.Set(cb, P);
			b.Set(cb + 1, C);
			b.SetPtr(cb + 2, offsets);
			b.Set(cb + 3, G);
			b.SetPtr(cb + 4, total);
			b.SetPtr(cb + 5, records);
			b.SetPtr(W, control);           // work counter
			b.SetPtr(W + 1, control + 4);   // overflow flags [P]
			b.SetPtr(W + 2, control + 1);   // overflow count
			b.SetPtr(W + 3, out_count);
			for (int w = 0; w < out_words; w++) b.SetPtr(W + 4 + w, out[w].data);
			b.SetPtr(L + 5, control + 4 + P);  // retry list
			b.SetPtr(L + 6, control + 2);      // retry count
			b.SetPtr(L + 7, control + 3);      // retry work counter
			b.Set(L + 8, C2);
			const uint64_t part_bytes = n * RS;
			// VGPU_DEBUG_BUCKET=<file>: per-partition rows, groups and cycle counts of the bucket pass.
			const char *debug_path = std::getenv("VGPU_DEBUG_BUCKET");
			uint64_t *debug = nullptr;
			if (debug_path) {
				debug = arena_.AllocT<uint64_t>(P * 8);
				VGPU_CUDA(cudaMemsetAsync(debug, 0, P * 64, stream_));
				b.SetWord(127, reinterpret_cast<uint64_t>(debug));
			}
			{
				const size_t smem1 = static_cast<size_t>(slot_bytes * C);
				CUfunction fb = module->Get("vgpu_gb_bucket");
				const int occ1 = std::max(1, Runtime::Get().MaxActiveBlocks(fb, T1, smem1));
				const unsigned grid1 = static_cast<unsigned>(std::min<uint64_t>(P, uint64_t(props.sm_count) * occ1));
				LaunchGenerated(*module, "vgpu_gb_bucket", grid1, T1, smem1, stream_, b, part_bytes, n);
			}
			{
				const size_t smem2 = static_cast<size_t>(slot_bytes * C2);
				CUfunction fr = module->Get("vgpu_gb_bucket_retry");
				const int occ2 = std::max(1, Runtime::Get().MaxActiveBlocks(fr, 512, smem2));
				LaunchGenerated(*module, "vgpu_gb_bucket_retry", static_cast<unsigned>(props.sm_count * occ2), 512, smem2,
				                stream_, b, 0, 0);
			}
			if (debug) {
				std::vector<uint64_t> h(P * 8);
				VGPU_CUDA(cudaMemcpyAsync(h.data(), debug, P * 64, cudaMemcpyDeviceToHost, stream_));
				VGPU_CUDA(cudaStreamSynchronize(stream_));
				if (FILE *f = std::fopen(debug_path, "w")) {
					for (uint64_t p = 0; p < P; p++) {
						std::fprintf(f, "%llu %llu %llu %llu %llu %llu %llu\n", (unsigned long long)p,
						             (unsigned long long)h[p * 8], (unsigned long long)h[p * 8 + 1],
						             (unsigned long long)h[p * 8 + 2], (unsigned long long)h[p * 8 + 3],
						             (unsigned long long)h[p * 8 + 4], (unsigned long long)h[p * 8 + 5]);
					}
					std::fclose(f);
				}
			}
			const uint32_t overflowed = ReadU32(control + 1);
			if (overflowed > 0) {
				// Partitions with more distinct keys than a shared-memory table holds: redo them with a
				// global-memory table sized from the partition's row count.
				std::vector<uint32_t> flags(P), offs(P * G);
				uint32_t total_rows = ReadU32(total);
				VGPU_CUDA(cudaMemcpyAsync(flags.data(), control + 4, P * 4, cudaMemcpyDeviceToHost, stream_));
				VGPU_CUDA(cudaMemcpyAsync(offs.data(), offsets, P * G * 4, cudaMemcpyDeviceToHost, stream_));
				VGPU_CUDA(cudaStreamSynchronize(stream_));
				std::vector<uint32_t> list, caps;
				std::vector<uint64_t> tab_off;
				uint64_t words = 0;
				for (uint64_t p = 0; p < P; p++) {
					if (!flags[p]) continue;
					const uint32_t start = offs[p * G];
					const uint32_t end = p + 1 < P ? offs[(p + 1) * G] : total_rows;
					const uint64_t cap = NextPow2(std::max<uint64_t>(64, 2ull * (end - start)));
					list.push_back(static_cast<uint32_t>(p));
					caps.push_back(static_cast<uint32_t>(cap));
					tab_off.push_back(words);
					words += cap * (1 + F);
				}
				uint64_t *tables = arena_.AllocT<uint64_t>(words);
				uint32_t *d_list = arena_.AllocT<uint32_t>(list.size());
				uint32_t *d_caps = arena_.AllocT<uint32_t>(caps.size());
				uint64_t *d_off = arena_.AllocT<uint64_t>(tab_off.size());
				VGPU_CUDA(cudaMemcpyAsync(d_list, list.data(), list.size() * 4, cudaMemcpyHostToDevice, stream_));
				VGPU_CUDA(cudaMemcpyAsync(d_caps, caps.data(), caps.size() * 4, cudaMemcpyHostToDevice, stream_));
				VGPU_CUDA(cudaMemcpyAsync(d_off, tab_off.data(), tab_off.size() * 8, cudaMemcpyHostToDevice, stream_));
				VGPU_CUDA(cudaMemsetAsync(control + 1, 0, 4, stream_));
				b.SetPtr(L, d_list);
				b.Set(L + 1, list.size());
				b.SetPtr(L + 2, tables);
				b.SetPtr(L + 3, d_off);
				b.SetPtr(L + 4, d_caps);
				LaunchGenerated(*module, "vgpu_gb_bucket_global",
				                static_cast<unsigned>(std::min<uint64_t>(list.size(), uint64_t(props.sm_count) * 2)), 512, 0,
				                stream_, b, 0, 0);
				if (ReadU32(control + 1) != 0) {
					Fail(VGPU_ERR_INTERNAL, "gpu_groupby: global-table fallback overflowed");
				}
			}
			groups = ReadU64(out_count);
			break;
		}
	}
	if (node.group_keys.empty() && groups == 0) {
		Fail(VGPU_ERR_UNSUPPORTED, kEmptyGlobal);
	}
	for (auto &c : out) c.rows = groups;
	return out;
}

// Heavy keys of a direct-partitioned group-by. Eligible when every carried value is 8 bytes wide and
// feeds exactly one aggregate (its partial state then fits the value's record slot), no input has
// NULLs, the mixed key leaves bit 31 of the record's key word free for the partial-record flag and a
// table slot fits 15 bits. 64 tiles spread over the input are sampled on the device; keys seen often
// enough that one CTA's share of their rows beats its one partial record are selected (at most 512,
// one per partition), and the selection is dropped on the device when they cover under a tenth of
// the sampled rows. VGPU_GB_HEAVY: 0 = off, 2 = always, whatever the input size and coverage (testing).
Executor::HeavyPlan Executor::PlanHeavy(const PipelineCodegen::GroupBySpec &gb, const PipelineCodegen &cg,
                                        const PipelineInput &pin, const GroupByCompiler &compile, const Geometry &g,
                                        int cb, uint64_t P, uint64_t ntiles, uint64_t extra_smem) {
	HeavyPlan none;
	int mode = 1;
	if (const char *env = std::getenv("VGPU_GB_HEAVY")) mode = std::atoi(env);
	if (mode == 0 || gb.direct_bits <= 0 || gb.direct_bits > 15 || gb.key_bits > 31 || cb + 12 >= kKeyWord) return none;
	if (mode == 1 && pin.rows < (1ull << 22)) return none;  // small inputs: sampling costs more than it saves
	for (auto &s : pin.sources) {
		if (s.valid) return none;
	}
	std::map<int, int> uses;
	for (auto &a : gb.aggs) {
		if (a.column < 0 || a.kind == AggKind::COUNT || a.kind == AggKind::COUNT_STAR) continue;
		if (TypeSize(cg.visible()[a.column].type) != 8 || ++uses[a.column] > 1) return none;
	}
	const auto &props = Runtime::Get().props();
	const uint32_t K = HeavyKeyCap();
	PipelineCodegen::GroupBySpec gbh = gb;
	gbh.heavy_slots = static_cast<int>(K);
	{  // heavy rows combined per warp step before the shared atomics (VGPU_GB_HEAVY_WARP=0: one update per row)
		const char *env = std::getenv("VGPU_GB_HEAVY_WARP");
		gbh.heavy_warp = !(env && std::strcmp(env, "0") == 0);
		// with the hot keys pre-aggregated, the bucket pass's records update their slots one by one: the
		// warp's equal-slot grouping costs more than the contention it saves (0.69 vs 0.89 ms on c1);
		// VGPU_GB_BUCKET_PLAIN=0 keeps the grouping
		const char *env_plain = std::getenv("VGPU_GB_BUCKET_PLAIN");
		gbh.bucket_plain = !(env_plain && std::strcmp(env_plain, "0") == 0);
	}
	HeavyPlan hp;
	hp.max_keys = K;
	hp.state_bytes = static_cast<uint64_t>(PipelineCodegen::HeavySlotBytes(gbh));
	if (hp.smem(P) + extra_smem + 1024 > static_cast<size_t>(props.smem_optin)) return none;
	hp.module = compile(gbh);
	const uint32_t SC = 1u << 16;
	uint64_t *skeys = arena_.AllocT<uint64_t>(SC);
	uint32_t *scount = arena_.AllocT<uint32_t>(SC);
	hp.hmap = arena_.AllocT<uint32_t>(P);
	hp.keys = arena_.AllocT<uint32_t>(K);
	hp.count = arena_.AllocT<uint32_t>(1);  // selected keys (the caller points `overflow` at its status block)
	VGPU_CUDA(cudaMemsetAsync(skeys, 0xff, static_cast<size_t>(SC) * 8, stream_));
	VGPU_CUDA(cudaMemsetAsync(scount, 0, static_cast<size_t>(SC) * 4, stream_));
	VGPU_CUDA(cudaMemsetAsync(hp.hmap, 0xff, P * 4, stream_));
	VGPU_CUDA(cudaMemsetAsync(hp.count, 0, 4, stream_));
	const uint64_t samples = std::min<uint64_t>(ntiles, 64);
	const uint64_t stride = ntiles / samples;
	KArgsHost a;
	FillArgs(pin, a);
	SetKeyWords(a, gbh);
	a.SetPtr(cb + 6, skeys);
	a.SetPtr(cb + 7, scount);
	a.Set(cb + 8, SC);
	a.Set(cb + 9, stride);
	const uint64_t sampled_rows = samples * static_cast<uint64_t>(g.tile());
	LaunchGenerated(*hp.module, "vgpu_gb_sample", static_cast<unsigned>(samples), g.block, 0, stream_, a, 0, sampled_rows);
	// a key seen c times in the sample has about c * ntiles / samples rows, spread over about
	// 2 * sm_count CTAs: selected when that is at least two rows per CTA
	const uint64_t ctas = 2ull * props.sm_count;
	uint32_t min_count = static_cast<uint32_t>(std::max<uint64_t>(2, (2 * ctas * samples + ntiles - 1) / ntiles));
	if (mode == 2) min_count = 1;
	kern::HeavySelect(skeys, scount, SC, hp.hmap, static_cast<uint32_t>(gb.direct_bits), hp.keys, K, min_count,
	                  mode != 2, hp.count, stream_);
	return hp;
}

// Bucket pass of the direct-partitioned group-by: a longest-first work list of (partition, row range)
// items, partitions too large for one CTA split into chunks merged through global tables, then one
// persistent launch over the list. Returns the group count.
// `status` (device, 8 words, the caller's flags in [6] and [7]) holds the work plan's counts in [0, 4)
// and the group count in [4, 6); it is read back once, into `status_host`, after the bucket pass --
// the only host round trip of the pass.
uint64_t Executor::DirectBuckets(Module &module, const PipelineCodegen::GroupBySpec &gb, const PipelineInput &pin,
                                 uint64_t P, uint64_t G, const uint32_t *offsets, const uint32_t *total,
                                 const char *records, uint64_t n, uint64_t RS, Relation &out, int out_words,
                                 int threads, uint32_t *status, uint32_t *status_host) {
	const auto &props = Runtime::Get().props();
	const uint64_t D = 1ull << gb.direct_bits;
	const uint64_t F = static_cast<uint64_t>(PipelineCodegen::StateWords(gb));
	const size_t smem = static_cast<size_t>(D * PipelineCodegen::DirectSlotBytes(gb));
	CUfunction fb = module.Get("vgpu_gb_dbucket");
	const int occ = Runtime::Get().MaxActiveBlocks(fb, threads, smem);
	if (occ < 1) Fail(VGPU_ERR_UNSUPPORTED, "gpu_groupby: direct-partitioned table does not fit on an SM");
	const uint32_t ctas = static_cast<uint32_t>(props.sm_count * occ);
	uint32_t min_split = 16384;
	if (const char *env = std::getenv("VGPU_GB_SPLIT_ROWS")) {  // testing/tuning override
		min_split = static_cast<uint32_t>(std::max<uint64_t>(256, std::strtoull(env, nullptr, 10)));
	}
	const uint64_t cap = kern::PlanWorkCapacity(static_cast<uint32_t>(P), n, min_split);
	// Split partitions: each has more than max(min_split, ceil(rows / (4 * ctas))) rows, so there are
	// fewer than this many, and their tables are sized without reading the plan back.
	const uint32_t max_split = static_cast<uint32_t>(std::min<uint64_t>({P, 4ull * ctas, n / min_split + 1}));
	void *items = arena_.Alloc(cap * 16);
	uint32_t *control = status;  // [0] items, [1] split partitions, [2] work counter, [3] partitioned rows
	uint32_t *split_info = arena_.AllocT<uint32_t>(2ull * max_split);
	uint64_t *out_count = reinterpret_cast<uint64_t *>(status + 4);
	VGPU_CUDA(cudaMemsetAsync(status, 0, 24, stream_));
	kern::PlanWork(offsets, G, static_cast<uint32_t>(P), total, min_split, ctas, items, control, split_info, max_split,
	               stream_);
	uint64_t *gtab = arena_.AllocT<uint64_t>(static_cast<uint64_t>(max_split) * F * D);
	const int cb = 2 + 2 * static_cast<int>(pin.sources.size());  // first consumer argument word
	KArgsHost b;
	FillArgs(pin, b);
	SetKeyWords(b, gb);
	b.SetPtr(cb, items);
	b.SetPtr(cb + 1, control);
	b.SetPtr(cb + 2, records);
	b.SetPtr(cb + 3, gtab);
	b.SetPtr(cb + 4, split_info);
	b.SetPtr(cb + 5, control + 2);
	b.SetPtr(cb + 6, out_count);
	b.SetPtr(cb + 7, control + 1);
	for (int w = 0; w < out_words; w++) b.SetPtr(cb + 8 + w, out[w].data);
	if (gb.f64_l2) {  // per-CTA FP64 sum tables (the kernel clears its own on entry and leaves them clear)
		const uint64_t nf = static_cast<uint64_t>(PipelineCodegen::F64Fields(gb));
		b.SetPtr(cb + 8 + out_words, arena_.Alloc(static_cast<uint64_t>(ctas) * nf * D * 8));
	}
	{
		// initializes the tables of the splits the plan made (a count it reads on the device)
		const uint64_t words = static_cast<uint64_t>(max_split) * F * D;
		const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((words + 255) / 256, uint64_t(props.sm_count) * 8));
		LaunchGenerated(module, "vgpu_gb_dtab_init", grid, 256, 0, stream_, b, 0, 0);
	}
	const int rec = LaunchGenerated(module, "vgpu_gb_dbucket", ctas, threads, smem, stream_, b, n * RS, n);
	VGPU_CUDA(cudaMemcpyAsync(status_host, status, 32, cudaMemcpyDeviceToHost, stream_));
	VGPU_CUDA(cudaStreamSynchronize(stream_));
	if (status_host[1] > max_split) {
		Fail(VGPU_ERR_INTERNAL, "gpu_groupby: work plan produced more splits than its bound");
	}
	const uint64_t groups = static_cast<uint64_t>(status_host[4]) | (static_cast<uint64_t>(status_host[5]) << 32);
	uint64_t out_row = 0;
	for (int w = 0; w < out_words; w++) out_row += TypeSize(out[w].type);
	Runtime::Get().profiler().SetBytes(rec, status_host[3] * RS + groups * out_row);  // records in, groups out
	return groups;
}

// ---- HASH_JOIN (sort-merge) ------------------------------------------------------------------------

Relation Executor::Join(const PlanNode &node) {
	if (node.children.size() != 2) {
		Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_executor: HASH_JOIN expects exactly two children");
	}
	if (node.build_keys.size() != 1 || node.probe_keys.size() != 1) {
		Fail(VGPU_ERR_UNSUPPORTED, "gpu_hash_join: this GPU path joins on exactly one equality key column");
	}
	if (node.output_columns.empty()) {
		Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_hash_join: node has no output columns");
	}
	Relation left = Exec(*node.children[0]);
	Relation right = Exec(*node.children[1]);
	return JoinMaterialize(node, left, right);
}

// A join under a pipeline (filter, projection or group-by above it). When the right side's keys are
// unique -- every left row has at most one match, the common key/foreign-key case -- the join is a
// virtual source of the pipeline: left row r is output row r, its right columns are read at its
// match in the sorted right side (a radix directory over the sorted keys, then a short binary search;
// right columns gathered into sorted order once), and rows without a match are filtered out. The
// match pairs are never materialized. Otherwise the join output is materialized as usual.
Relation Executor::JoinForPipeline(const PlanNode &node, PipelineInput &pin, bool *fused, bool multi_ok,
                                   bool any_order) {
	*fused = false;
	if (node.children.size() != 2) {
		Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_executor: HASH_JOIN expects exactly two children");
	}
	if (node.build_keys.size() != 1 || node.probe_keys.size() != 1) {
		Fail(VGPU_ERR_UNSUPPORTED, "gpu_hash_join: this GPU path joins on exactly one equality key column");
	}
	if (node.output_columns.empty()) {
		Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_hash_join: node has no output columns");
	}
	Relation left = Exec(*node.children[0]);
	Relation right = Exec(*node.children[1]);
	const DevColumn *lk = nullptr, *rk = nullptr;
	for (auto &c : left) if (c.name == node.build_keys[0]) { lk = &c; break; }
	for (auto &c : right) if (c.name == node.probe_keys[0]) { rk = &c; break; }
	const char *env = std::getenv("VGPU_JOIN_FUSED");  // "0": always materialize (testing)
	const bool allowed = !(env && std::strcmp(env, "0") == 0);
	if (!allowed || !lk || !rk || lk->type != rk->type || !IsIntegerKeyType(lk->type) || lk->rows == 0 ||
	    rk->rows == 0 || lk->rows >= (1ull << 32) || rk->rows >= (1ull << 32) || rk->valid || lk->valid) {
		return JoinMaterialize(node, left, right);
	}
	std::vector<const DevColumn *> outs;
	std::vector<int> side;
	for (auto &name : node.output_columns) {
		const DevColumn *l = nullptr, *r = nullptr;
		for (auto &c : left) if (c.name == name) { l = &c; break; }
		for (auto &c : right) if (c.name == name) { r = &c; break; }
		if (!l == !r) return JoinMaterialize(node, left, right);  // missing or ambiguous: its error path
		outs.push_back(l ? l : r);
		side.push_back(l ? 0 : 1);
	}
	const uint64_t ln = lk->rows, rn = rk->rows;
	const size_t kw = TypeSize(rk->type);
	// The join contributes one right column of at most 4 bytes without NULLs: its value can be inlined
	// into a dense key table; the value bits' bounds come back with the key range.
	const DevColumn *inline_col = nullptr;
	{
		size_t right_outs = 0;
		for (size_t i = 0; i < outs.size(); i++) {
			if (side[i] == 1) {
				right_outs++;
				inline_col = outs[i];
			}
		}
		if (right_outs != 1 || TypeSize(inline_col->type) > 4 || TypeSize(inline_col->type) == 3 || inline_col->valid) {
			inline_col = nullptr;
		}
	}
	auto add_sources = [&](bool sorted_side, const uint32_t *perm) {
		for (size_t i = 0; i < outs.size(); i++) {
			DevColumn c = *outs[i];
			c.name = node.output_columns[i];
			if (side[i] == 1 && sorted_side) {  // right columns in sorted-key order
				const size_t w = TypeSize(c.type);
				void *dst = arena_.Alloc(rn * w);
				kern::Gather(outs[i]->data, w, perm, rn, dst, stream_);
				c.data = dst;
				if (outs[i]->valid) {
					uint8_t *v = arena_.AllocT<uint8_t>(rn);
					kern::Gather(outs[i]->valid, 1, perm, rn, v, stream_);
					c.valid = v;
				}
			}
			SourceColumn sc;
			sc.name = c.name;
			sc.type = c.type;
			sc.nullable = c.valid != nullptr;
			sc.side = side[i];
			pin.spec.sources.push_back(sc);
			pin.sources.push_back(c);
		}
	};
	// A right side read from the column cache: its dense table may already be kept (see JoinTableCache).
	std::string cache_key;
	{
		const std::string idk = ColumnCache::Get().Identify(rk->data, rk->type, rn);
		const std::string idv = inline_col ? ColumnCache::Get().Identify(inline_col->data, inline_col->type, rn) : "";
		const char *env_c = std::getenv("VGPU_JOIN_COMPACT");
		const char *env_keep = std::getenv("VGPU_JOIN_CACHE");  // "0": build every time (measurement, testing)
		const bool keep_allowed = !(env_keep && std::strcmp(env_keep, "0") == 0);
		if (keep_allowed && !idk.empty() && (!inline_col || !idv.empty())) {
			cache_key = idk + "|" + idv + "|" + std::to_string(inline_col ? static_cast<int>(inline_col->type) : -1) + "|" +
			            (env_c ? env_c : "");
		}
	}
	uint64_t bias = 0;
	std::shared_ptr<CachedJoinTable> hit = cache_key.empty() ? nullptr : JoinTableCache::Get().Find(cache_key);
	if (hit && hit->multi_inline && !(multi_ok && any_order)) hit = nullptr;  // built again in right-side order
	if (hit) {
		holds_.push_back(hit);
		add_sources(false, nullptr);
		pin.spec.join_inline = hit->inline_value;
		pin.spec.join_multi = pin.spec.join_minline = hit->multi_inline;
		pin.join_words[0] = hit->words[0];
		pin.join_words[1] = hit->words[1];
		pin.join_words[3] = hit->words[3];
		bias = hit->bias;
	} else {
		// a dense table just built: handed from the execution's arena to the cache
		auto keep = [&](void *table, uint64_t bytes, bool inline_value, bool multi_inline = false) {
			if (cache_key.empty()) return;
			arena_.Release(table);
			auto t = std::make_shared<CachedJoinTable>();
			t->table = table;
			t->bytes = bytes;
			t->inline_value = inline_value;
			t->multi_inline = multi_inline;
			t->bias = bias;
			t->words[0] = pin.join_words[0];
			t->words[1] = pin.join_words[1];
			t->words[3] = pin.join_words[3];
			holds_.push_back(t);
			JoinTableCache::Get().Insert(cache_key, t);
		};
		uint64_t *rw = arena_.AllocT<uint64_t>(rn);
		uint64_t *mm = arena_.AllocT<uint64_t>(3);  // key min, key max, value bits (min, max)
		kern::WidenKeysMinMax(rk->data, kw, rn, rw, mm, stream_);
		if (inline_col) kern::ValueBits(inline_col->data, TypeSize(inline_col->type), rn, reinterpret_cast<uint32_t *>(mm + 2), stream_);
		uint64_t host_mm[3] = {0, 0, 0};
		VGPU_CUDA(cudaMemcpyAsync(host_mm, mm, inline_col ? 24 : 16, cudaMemcpyDeviceToHost, stream_));
		VGPU_CUDA(cudaStreamSynchronize(stream_));
		bias = host_mm[0];
		const uint64_t range = host_mm[1] - host_mm[0];
		const uint32_t vmin = static_cast<uint32_t>(host_mm[2]), vmax = static_cast<uint32_t>(host_mm[2] >> 32);
		const int bits = BitsFor(range);
		// the dense tables subtract the bias as they index; the sorted form below works on biased keys
		uint32_t *dups = arena_.AllocT<uint32_t>(1);
		bool built = false;
		// Dense keys (range within 4x the key count, at most 2^28): a table indexed by the key over the whole
		// range, filled without sorting. It holds the right row index, or -- when the join contributes one
		// right column of at most 4 bytes -- that column's value itself, so a probe row costs one random
		// read; the value is stored as its offset from the smallest value in the fewest bytes that hold every
		// offset (all ones marks a missing key), so the table of a small-valued column stays in L2. A key met
		// twice (many-to-many) falls back to the sorted form below.
		// More right rows than key values: some key repeats for sure, so no unique-key table is tried.
		const bool surely_repeated = rn > range + 1;
		if (range < (1ull << 28) && range < 4 * rn && !surely_repeated) {
			const uint64_t span = static_cast<uint64_t>(vmax) - vmin;
			const size_t width = !inline_col ? 0 : span < 0xffull ? 1 : span < 0xffffull ? 2 : span < 0xffffffffull ? 4 : 8;
			const char *env_c = std::getenv("VGPU_JOIN_COMPACT");  // "0": 8-byte inline entries (testing)
			const bool compact = width != 0 && width != 8 && !(env_c && std::strcmp(env_c, "0") == 0);
			if (compact) {
				void *table = arena_.Alloc((range + 1) * width);
				kern::JoinDenseCompact(rw, inline_col->data, TypeSize(inline_col->type), rn, range, vmin, table, width, dups,
				                       stream_, bias);
				if (ReadU32(dups) == 0) {
					add_sources(false, nullptr);
					pin.spec.join_inline = true;
					pin.join_words[0] = reinterpret_cast<uint64_t>(table);
					pin.join_words[1] = vmin;
					pin.join_words[3] = (width == 1 ? 0xfdu : width == 2 ? 0xfcu : 0xfbu) | ((range + 1) << 8);
					built = true;
					keep(table, (range + 1) * width, true);
				}
			} else if (inline_col) {
				uint64_t *table = arena_.AllocT<uint64_t>(range + 1);
				kern::JoinDenseInline(rw, inline_col->data, TypeSize(inline_col->type), rn, range, table, dups, stream_, bias);
				if (ReadU32(dups) == 0) {
					add_sources(false, nullptr);
					pin.spec.join_inline = true;
					pin.join_words[0] = reinterpret_cast<uint64_t>(table);
					pin.join_words[1] = 0;
					pin.join_words[3] = 0xfeu | ((range + 1) << 8);
					built = true;
					keep(table, (range + 1) * 8, true);
				}
			} else {
				uint32_t *table = arena_.AllocT<uint32_t>(range + 1);
				kern::JoinDenseRows(rw, rn, range, table, dups, stream_, bias);
				if (ReadU32(dups) == 0) {
					add_sources(false, nullptr);
					pin.join_words[0] = 0;
					pin.join_words[1] = reinterpret_cast<uint64_t>(table);
					pin.join_words[3] = 0xffu | ((range + 1) << 8);
					built = true;
					keep(table, (range + 1) * 4, false);
				}
			}
		}
		// Repeated right keys with few matches each and one narrow right column: the dense table holds every
		// match's value inline (a count, then one slot per match), still filled without sorting -- 4-byte
		// entries when two matches fit, else 8-byte ones; a key with more matches than fit falls back to the
		// sorted form.
		const uint64_t mspan = static_cast<uint64_t>(vmax) - vmin;
		if (!built && multi_ok && any_order && inline_col && range < (1ull << 28) && range < 4 * rn &&
		    mspan < (1ull << 30)) {
			const uint32_t vbits = std::max(1, BitsFor(mspan));
			uint32_t *overflow = arena_.AllocT<uint32_t>(1);
			for (int wide = 0; wide < 2 && !built; wide++) {
				const uint32_t ebits = wide ? 64 : 32, cbits = wide ? 3 : 2;
				const uint32_t rmax = std::min<uint32_t>((1u << cbits) - 1, (ebits - cbits) / vbits);
				if (rmax < 2) continue;
				const uint64_t bytes = (range + 1) * (wide ? 8 : 4);
				void *table = arena_.Alloc(bytes);
				kern::JoinDenseMulti(rw, inline_col->data, TypeSize(inline_col->type), rn, range, vmin, vbits, cbits, rmax,
				                     table, wide != 0, overflow, stream_, bias);
				if (ReadU32(overflow) == 0) {
					add_sources(false, nullptr);
					pin.spec.join_multi = pin.spec.join_minline = true;
					pin.join_words[0] = reinterpret_cast<uint64_t>(table);
					pin.join_words[1] = vmin;
					pin.join_words[3] = ((range + 1) << 8) | (wide ? 0x80u : 0u) | (vbits << 2) | (cbits - 1);
					built = true;
					keep(table, bytes, false, true);
				} else {
					arena_.FreeNow(table);
				}
			}
		}
		if (!built) {
			// Sorted form: LSD radix sort of the right keys, uniqueness check, radix directory over the sorted
			// keys (at most 2^22 buckets), right columns gathered into sorted order once.
			kern::SubtractBias(rw, rn, bias, stream_);
			uint32_t *perm = arena_.AllocT<uint32_t>(rn);
			kern::Iota(perm, rn, stream_);
			uint64_t *rw_alt = arena_.AllocT<uint64_t>(rn);
			uint32_t *perm_alt = arena_.AllocT<uint32_t>(rn);
			kern::RadixSortPairs(rw, perm, rw_alt, perm_alt, rn, bits, arena_);
			arena_.FreeNow(rw_alt);
			arena_.FreeNow(perm_alt);
			kern::CountAdjacentEqual(rw, rn, dups, stream_);
			bool multi = false;
			if (ReadU32(dups) != 0) {
				// Right keys repeat: a consumer that takes one item per match reads each probe row's run of
				// equal keys (sorted right order); runs longer than kMaxJoinRun go to the load-balanced
				// materializing join instead, which spreads one row's matches over many threads.
				if (!multi_ok) return JoinMaterialize(node, left, right);
				uint32_t *maxrun = arena_.AllocT<uint32_t>(1);
				kern::MaxRunLength(rw, rn, maxrun, stream_);
				if (ReadU32(maxrun) > kMaxJoinRun) return JoinMaterialize(node, left, right);
				multi = true;
			}
			// a dense key range gets one directory bucket per key value (the run is the bucket)
			const bool dense_runs = multi && range < (1ull << 28) && range < 4 * rn;
			const uint32_t shift = dense_runs ? 0u : bits > 22 ? static_cast<uint32_t>(bits - 22) : 0u;
			const uint64_t nb = (range >> shift) + 1;
			uint32_t *dir = arena_.AllocT<uint32_t>(nb + 1);
			kern::JoinDirectory(rw, rn, shift, nb, dir, stream_);
			add_sources(true, perm);
			pin.join_words[0] = reinterpret_cast<uint64_t>(rw);
			pin.join_words[1] = reinterpret_cast<uint64_t>(dir);
			pin.join_words[3] = shift | (nb << 8);
			pin.spec.join_multi = multi;
		}
	}
	pin.join_words[2] = bias;
	SourceColumn key;
	key.name = "__vgpu_join_key";
	key.type = lk->type;
	key.side = 0;
	pin.spec.join_key = static_cast<int>(pin.spec.sources.size());
	pin.spec.sources.push_back(key);
	DevColumn kc = *lk;
	kc.name = key.name;
	pin.sources.push_back(kc);
	pin.spec.join = true;
	pin.rows = ln;
	pin.right_rows = 0;
	*fused = true;
	return {};
}

// The join's output relation: right side sorted by key, per-left-row search, load-balanced expansion
// of the match pairs, gathers of the output columns.
Relation Executor::JoinMaterialize(const PlanNode &node, Relation &left, Relation &right) {
	auto find = [](const Relation &rel, const std::string &name, const char *side) -> const DevColumn & {
		for (auto &c : rel) {
			if (c.name == name) return c;
		}
		Fail(VGPU_ERR_INVALID_ARGUMENT, std::string("gpu_hash_join: ") + side + " key column '" + name + "' not found");
	};
	const DevColumn &lk = find(left, node.build_keys[0], "left");
	const DevColumn &rk = find(right, node.probe_keys[0], "right");
	for (auto *k : {&lk, &rk}) {
		if (!IsIntegerKeyType(k->type)) {
			Fail(VGPU_ERR_UNSUPPORTED, std::string("gpu_hash_join: ") + (k == &lk ? "left" : "right") +
			                               " join key is not an integer/boolean column, which this GPU path requires");
		}
	}
	if (lk.type != rk.type) {
		Fail(VGPU_ERR_UNSUPPORTED, "gpu_hash_join: join key columns must have the same type on both sides");
	}
	std::vector<const DevColumn *> sources;
	std::vector<bool> from_left;
	for (auto &name : node.output_columns) {
		const DevColumn *l = nullptr, *r = nullptr;
		for (auto &c : left) if (c.name == name) { l = &c; break; }
		for (auto &c : right) if (c.name == name) { r = &c; break; }
		if (l && r) Fail(VGPU_ERR_UNSUPPORTED, "gpu_hash_join: output column '" + name + "' is ambiguous (present on both sides)");
		if (!l && !r) Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_hash_join: output column '" + name + "' not found on either side");
		sources.push_back(l ? l : r);
		from_left.push_back(l != nullptr);
	}
	const uint64_t ln = lk.rows, rn = rk.rows;
	auto make_out = [&](uint64_t rows) {
		Relation out;
		for (size_t i = 0; i < sources.size(); i++) {
			DevColumn c;
			c.name = node.output_columns[i];
			c.type = sources[i]->type;
			c.rows = rows;
			c.data = arena_.Alloc(rows * TypeSize(c.type));
			c.has_stats = sources[i]->has_stats;
			c.min = sources[i]->min;
			c.max = sources[i]->max;
			out.push_back(c);
		}
		return out;
	};
	if (ln == 0 || rn == 0) {
		return make_out(0);
	}
	if (ln >= (1ull << 32) || rn >= (1ull << 32)) Fail(VGPU_ERR_UNSUPPORTED, "gpu_hash_join: side too large");
	const size_t kw = TypeSize(lk.type);
	uint64_t *lw = arena_.AllocT<uint64_t>(ln);
	uint64_t *rw = arena_.AllocT<uint64_t>(rn);
	kern::WidenKeys(lk.data, kw, ln, lw, stream_);
	uint64_t *mm = arena_.AllocT<uint64_t>(2);
	kern::WidenKeysMinMax(rk.data, kw, rn, rw, mm, stream_);
	uint64_t host_mm[2];
	VGPU_CUDA(cudaMemcpyAsync(host_mm, mm, 16, cudaMemcpyDeviceToHost, stream_));
	VGPU_CUDA(cudaStreamSynchronize(stream_));
	const uint64_t bias = host_mm[0];
	const int bits = BitsFor(host_mm[1] - host_mm[0]);
	kern::SubtractBias(rw, rn, bias, stream_);
	uint32_t *perm = arena_.AllocT<uint32_t>(rn);
	kern::Iota(perm, rn, stream_);
	uint64_t *rw_alt = arena_.AllocT<uint64_t>(rn);
	uint32_t *perm_alt = arena_.AllocT<uint32_t>(rn);
	kern::RadixSortPairs(rw, perm, rw_alt, perm_alt, rn, bits, arena_);
	arena_.FreeNow(rw_alt);
	arena_.FreeNow(perm_alt);
	// each left key's run of equal right keys through a radix directory: one bucket per key value when
	// the key range is dense (the run is read, not searched), else 2^22 buckets and a short search
	const uint64_t range = host_mm[1] - host_mm[0];
	const uint32_t shift = (range < (1ull << 28) && range < 4 * rn) ? 0u : bits > 22 ? static_cast<uint32_t>(bits - 22) : 0u;
	const uint64_t nb = (range >> shift) + 1;
	uint32_t *dir = arena_.AllocT<uint32_t>(nb + 1);
	kern::JoinDirectory(rw, rn, shift, nb, dir, stream_);
	uint64_t *lower = arena_.AllocT<uint64_t>(ln);
	uint64_t *counts = arena_.AllocT<uint64_t>(ln);
	kern::JoinRuns(lw, ln, rw, dir, nb, shift, bias, lower, counts, stream_);
	uint64_t *total = arena_.AllocT<uint64_t>(1);
	kern::ExclusiveScanU64(counts, counts, ln, total, arena_);
	const uint64_t total_rows = ReadU64(total);
	if (total_rows > kMaxOutputRows) {
		Fail(VGPU_ERR_UNSUPPORTED, "gpu_hash_join: join result of " + std::to_string(total_rows) +
		                               " rows is too large for GPU execution");
	}
	Relation out = make_out(total_rows);
	if (total_rows == 0) return out;
	uint32_t *out_left = arena_.AllocT<uint32_t>(total_rows);
	uint32_t *out_right = arena_.AllocT<uint32_t>(total_rows);
	kern::JoinExpand(counts, lower, ln, perm, total_rows, out_left, out_right, stream_);
	for (size_t i = 0; i < sources.size(); i++) {
		kern::Gather(sources[i]->data, TypeSize(sources[i]->type), from_left[i] ? out_left : out_right, total_rows,
		             out[i].data, stream_);
	}
	return out;
}

Relation Executor::Exec(const PlanNode &node) {
	switch (node.op) {
	case OpType::SCAN:
		return Scan(node);
	case OpType::FILTER:
	case OpType::PROJECTION:
		return RunChain(node);
	case OpType::GROUP_BY_AGGREGATE:
		return GroupBy(node);
	case OpType::HASH_JOIN:
		return Join(node);
	case OpType::CROSS_PRODUCT:
		return CrossProduct(node);
	}
	Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_executor: unknown GpuOpType value");
}

} // namespace

void ClearJoinTables() {
	JoinTableCache::Get().Clear();
}

PipelineCodegen::GroupBySpec ValidateGroupBy(const PlanNode &node, const PipelineCodegen &cg, std::vector<int> &key_cols) {
	return ValidateGroupByNode(node, cg, key_cols);
}

ExecResult ExecutePlan(const PlanNode &plan, const std::vector<vgpu_column> &inputs, const ExecOptions &options,
                       cudaStream_t stream) {
	RefuseWindowPrimitives(plan);
	Runtime::Get().EnsureDevice();
	Executor ex(inputs, options, stream, IsRowIndependent(plan));
	ex.SetRoot(&plan);
	Relation rel = ex.Exec(plan);
	ExecResult result;
	result.stream = stream;
	if (void *rows = ex.deferred_rows()) {
		result.pending_rows = rows;
		result.pending_rows_bytes = ex.deferred_rows_bytes();
		result.device_buffers.push_back(rows);
	}
	for (auto &c : rel) {
		HostColumnOut o;
		o.name = c.name;
		o.type = c.type;
		o.rows = c.rows;
		const size_t bytes = c.rows * TypeSize(c.type);
		if (options.output_on_device) {
			// A buffer the execution allocated itself passes to the result as it is; anything else (borrowed
			// inputs, cache entries, a buffer already handed to another column) is copied, so the result
			// never aliases memory it does not own.
			void *d = nullptr;
			if (bytes && ex.arena().Take(c.data)) {
				d = c.data;
			} else {
				d = Runtime::Get().allocator().Alloc(bytes, stream);
				if (bytes) VGPU_CUDA(cudaMemcpyAsync(d, c.data, bytes, cudaMemcpyDeviceToDevice, stream));
			}
			result.device_buffers.push_back(d);
			o.device_data = d;
			if (c.valid) {
				const size_t vb = (c.rows + 7) / 8;
				uint8_t *bm = static_cast<uint8_t *>(Runtime::Get().allocator().Alloc(vb, stream));
				result.device_buffers.push_back(bm);
				kern::PackValidity(c.valid, bm, c.rows, stream);
				o.device_validity = bm;
			}
		} else {
			if (bytes) {
				o.host = PinnedPool::Get().Acquire(bytes);
				VGPU_CUDA(cudaMemcpyAsync(o.host.get(), c.data, bytes, cudaMemcpyDeviceToHost, stream));
			}
			if (c.valid && c.rows > 0) {
				const size_t vb = (c.rows + 7) / 8;
				uint8_t *bm = ex.arena().AllocT<uint8_t>(vb);
				kern::PackValidity(c.valid, bm, c.rows, stream);
				o.validity.resize(vb);
				VGPU_CUDA(cudaMemcpyAsync(o.validity.data(), bm, vb, cudaMemcpyDeviceToHost, stream));
			}
		}
		result.columns.push_back(std::move(o));
	}
	if (!(options.output_on_device && options.no_sync)) {
		VGPU_CUDA(cudaStreamSynchronize(stream));
	}
	return result;
}

} // namespace vgpu
