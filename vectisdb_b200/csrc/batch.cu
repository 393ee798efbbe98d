// batch.cu -- many group-by queries in one persistent launch (see batch.hpp).
#include "batch.hpp"

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <list>
#include <map>
#include <mutex>
#include <sstream>

#include "column_cache.hpp"
#include "kernels.hpp"

namespace vgpu {

std::string Sha256Hex(const void *data, size_t n);

namespace {

bool IdentChar(char c) {
	return std::isalnum(static_cast<unsigned char>(c)) || c == '_';
}

uint64_t NextPow2(uint64_t x) {
	uint64_t p = 1;
	while (p < x) p <<= 1;
	return p;
}

int BitsFor(uint64_t range) {
	int b = 0;
	while (b < 64 && (range >> b) != 0) b++;
	return b;
}

// ---- templates ------------------------------------------------------------------------------------

// Deep copy of a plan with every expression source's literals templated; parameters are numbered in
// traversal order (children first, then the node's expressions).
std::shared_ptr<PlanNode> TemplatePlan(const PlanNode &n, std::vector<char> &types, std::vector<uint64_t> &values) {
	auto c = std::make_shared<PlanNode>(n);
	c->children.clear();
	for (auto &ch : n.children) c->children.push_back(TemplatePlan(*ch, types, values));
	for (auto &e : c->expressions) {
		TemplatedSource t = TemplateLiterals(e.source, static_cast<int>(types.size()));
		e.source = t.text;
		types.insert(types.end(), t.types.begin(), t.types.end());
		values.insert(values.end(), t.values.begin(), t.values.end());
	}
	return c;
}

void Signature(const PlanNode &n, std::ostringstream &o) {
	o << "op" << static_cast<int>(n.op) << "{cols:";
	for (auto &s : n.column_names) o << s << ",";
	o << "|exprs:";
	for (auto &e : n.expressions) {
		o << static_cast<int>(e.output_type) << ":" << e.source << "(";
		for (auto &i : e.input_columns) o << i << ",";
		o << ");";
	}
	o << "|keys:";
	for (auto &k : n.group_keys) o << k << ",";
	o << "|aggs:";
	for (auto &a : n.aggregates) o << static_cast<int>(a.kind) << ":" << a.input_column << ":" << static_cast<int>(a.output_type) << ";";
	o << "|out:";
	for (auto &s : n.output_columns) o << s << ",";
	for (auto &ch : n.children) Signature(*ch, o);
	o << "}";
}

// ---- per-query preparation ---------------------------------------------------------------------

struct Prepared {
	size_t index = 0;
	bool batchable = false;
	std::shared_ptr<PlanNode> templ;
	std::vector<char> ptypes;
	std::vector<uint64_t> params;
	std::vector<DevColumn> sources;
	std::string sig;
	uint64_t rows = 0;
};

// The batch form: GROUP_BY(keys) <- FILTER/PROJECTION* <- SCAN. Returns the SCAN leaf or nullptr.
const PlanNode *BatchShape(const PlanNode &root) {
	if (root.op != OpType::GROUP_BY_AGGREGATE || root.group_keys.empty() || root.children.size() != 1) return nullptr;
	const PlanNode *cur = root.children[0].get();
	while (cur->op == OpType::FILTER || cur->op == OpType::PROJECTION) {
		if (cur->children.size() != 1) return nullptr;
		cur = cur->children[0].get();
	}
	return cur->op == OpType::SCAN ? cur : nullptr;
}

// ---- autotuner ---------------------------------------------------------------------------------

struct Geometry4 {
	int block = 256, items = 4, tile_rows = 16384, smem_slots = 2048;
	std::string ToString() const {
		return std::to_string(block) + " " + std::to_string(items) + " " + std::to_string(tile_rows) + " " +
		       std::to_string(smem_slots);
	}
};

// Best geometry per (template, device), measured on a real batch; kept in memory and, when
// VGPU_AUTOTUNE_FILE names a file, loaded from and appended to it ("key block items tile slots ms").
class Autotuner {
public:
	bool Lookup(const std::string &key, Geometry4 &g) {
		std::lock_guard<std::mutex> lock(mu_);
		LoadLocked();
		auto it = table_.find(key);
		if (it == table_.end()) return false;
		g = it->second;
		return true;
	}
	void Record(const std::string &key, const Geometry4 &g, double ms) {
		std::lock_guard<std::mutex> lock(mu_);
		LoadLocked();
		table_[key] = g;
		if (const char *path = std::getenv("VGPU_AUTOTUNE_FILE")) {
			std::ofstream f(path, std::ios::app);
			if (f) f << key << " " << g.ToString() << " " << ms << "\n";
		}
	}
	void Clear() {
		std::lock_guard<std::mutex> lock(mu_);
		table_.clear();
		loaded_ = true;
	}

private:
	void LoadLocked() {
		if (loaded_) return;
		loaded_ = true;
		const char *path = std::getenv("VGPU_AUTOTUNE_FILE");
		if (!path) return;
		std::ifstream f(path);
		std::string key;
		Geometry4 g;
		double ms;
		while (f >> key >> g.block >> g.items >> g.tile_rows >> g.smem_slots >> ms) table_[key] = g;
	}
	std::mutex mu_;
	bool loaded_ = false;
	std::map<std::string, Geometry4> table_;
};

Autotuner &Tuner() {
	static Autotuner *t = new Autotuner();
	return *t;
}

// ---- cached batch launches ---------------------------------------------------------------------

// Device state of one batch (one template, fixed columns, constants and geometry): query table,
// tile list, accumulators (left at identity by the finalize kernel), output pointer table and the
// captured graph. Reused while a call presents the same batch again.
struct BatchEntry {
	std::string key;
	std::shared_ptr<Module> module;
	uint64_t *qtab = nullptr, *acc = nullptr, *counts = nullptr, *outp = nullptr;
	uint32_t *work = nullptr;
	void *tiles = nullptr;
	uint64_t *counts_host = nullptr, *outp_host = nullptr;  // pinned (cached entries) or into host_stage
	std::vector<uint64_t> host_stage;                        // transient entries
	bool pinned = true;
	cudaGraphExec_t graph = nullptr;
	bool initialized = false;
	uint64_t nq = 0, ntiles = 0, acc_words = 0, out_rows = 0, in_bytes = 0, rows = 0;
	unsigned grid = 0;
	size_t smem = 0;
	Geometry4 geo;
	std::vector<uint64_t> out_base, out_cap;
	int F = 0;

	void Release(cudaStream_t stream) {
		auto &al = Runtime::Get().allocator();
		if (graph) cudaGraphExecDestroy(graph);
		graph = nullptr;
		for (void *p : {static_cast<void *>(qtab), static_cast<void *>(acc), static_cast<void *>(counts),
		                static_cast<void *>(outp), static_cast<void *>(work), tiles}) {
			if (p) al.Free(p, stream);
		}
		if (pinned && counts_host) cudaFreeHost(counts_host);
		if (pinned && outp_host) cudaFreeHost(outp_host);
		qtab = acc = counts = outp = nullptr;
		work = nullptr;
		tiles = nullptr;
		counts_host = outp_host = nullptr;
	}
};

class BatchCache {
public:
	std::shared_ptr<BatchEntry> Find(const std::string &key) {
		std::lock_guard<std::mutex> lock(mu_);
		for (auto it = lru_.begin(); it != lru_.end(); ++it) {
			if ((*it)->key == key) {
				auto e = *it;
				lru_.erase(it);
				lru_.push_front(e);
				return e;
			}
		}
		return nullptr;
	}
	void Insert(const std::shared_ptr<BatchEntry> &e, cudaStream_t stream) {
		std::lock_guard<std::mutex> lock(mu_);
		lru_.push_front(e);
		// evict least recently used entries that no caller holds (a tuning run keeps its best one)
		for (auto it = lru_.end(); lru_.size() > kMaxEntries && it != lru_.begin();) {
			--it;
			if (it->use_count() > 1) continue;
			VGPU_CUDA(cudaStreamSynchronize(stream));
			(*it)->Release(stream);
			it = lru_.erase(it);
		}
	}
	void Clear(cudaStream_t stream) {
		std::lock_guard<std::mutex> lock(mu_);
		if (!lru_.empty()) VGPU_CUDA(cudaDeviceSynchronize());
		for (auto &e : lru_) e->Release(stream);
		lru_.clear();
	}

private:
	static constexpr size_t kMaxEntries = 16;
	std::mutex mu_;
	std::list<std::shared_ptr<BatchEntry>> lru_;
};

BatchCache &Cache() {
	static BatchCache *c = new BatchCache();
	return *c;
}

struct DeviceBuffers {
	std::vector<void *> ptrs;
	cudaStream_t stream = nullptr;
	~DeviceBuffers() {
		try {
			for (void *p : ptrs) Runtime::Get().allocator().Free(p, stream);
		} catch (...) {
		}
	}
};

void LaunchRaw(Module &m, const char *name, unsigned grid, unsigned block, size_t smem, cudaStream_t stream,
               uint64_t (&w)[128]) {
	CUfunction f = m.Get(name);
	void *params[] = {w};
	Runtime::Get().LaunchModuleKernel(f, dim3(grid), dim3(block), smem, stream, params);
}

// One template's queries through the batch kernel. Returns false (nothing launched) when the
// template is outside the batch form; then every query of it runs alone.
bool RunTemplate(const std::vector<Prepared *> &qs, const ExecOptions &options, const BatchOptions &bopts,
                 cudaStream_t stream, std::vector<ExecResult> &results, BatchStats *stats) {
	Prepared &q0 = *qs.front();
	const PlanNode &root = *q0.templ;
	std::vector<const PlanNode *> chain;
	const PlanNode *cur = root.children[0].get();
	while (cur->op == OpType::FILTER || cur->op == OpType::PROJECTION) {
		chain.push_back(cur);
		cur = cur->children[0].get();
	}
	std::reverse(chain.begin(), chain.end());
	PipelineSpec spec;
	spec.chain = chain;
	for (auto &s : q0.sources) {
		SourceColumn sc;
		sc.name = s.name;
		sc.type = s.type;
		spec.sources.push_back(sc);
	}
	std::unique_ptr<PipelineCodegen> cg;
	PipelineCodegen::GroupBySpec gb;
	std::vector<int> key_cols;
	try {
		cg.reset(new PipelineCodegen(spec));
		gb = ValidateGroupBy(root, *cg, key_cols);
	} catch (const Error &) {
		return false;
	}
	for (int c : key_cols) {
		if (cg->visible()[c].source < 0) return false;  // computed keys: no column statistics to pack by
		PipelineCodegen::GroupKey k;
		k.column = c;
		gb.keys.push_back(k);
	}
	const int nsrc = static_cast<int>(q0.sources.size());
	const int nkeys = static_cast<int>(key_cols.size());
	const int nparams = static_cast<int>(q0.params.size());
	PipelineCodegen::BatchLayout L;
	L.key_base = 1 + 2 * nsrc;
	L.dom_base = L.key_base + 2 * nkeys;
	L.param_base = L.dom_base + 4;
	L.qwords = L.param_base + nparams;
	const int F = PipelineCodegen::StateWords(gb);
	const auto &props = Runtime::Get().props();

	// Key statistics (cached columns carry them; others are measured, one sync for all).
	Arena arena(stream);
	std::vector<std::vector<std::pair<int64_t, int64_t>>> ranges(qs.size(), std::vector<std::pair<int64_t, int64_t>>(nkeys));
	std::vector<std::pair<size_t, int>> pending;
	int64_t *mm = nullptr;
	for (size_t qi = 0; qi < qs.size(); qi++) {
		for (int j = 0; j < nkeys; j++) {
			const DevColumn &src = qs[qi]->sources[cg->visible()[key_cols[j]].source];
			if (src.has_stats) {
				ranges[qi][j] = {src.min, src.max};
			} else {
				pending.push_back({qi, j});
			}
		}
	}
	if (!pending.empty()) {
		mm = arena.AllocT<int64_t>(2 * pending.size());
		for (size_t p = 0; p < pending.size(); p++) {
			const DevColumn &src = qs[pending[p].first]->sources[cg->visible()[key_cols[pending[p].second]].source];
			kern::MinMaxSigned(src.data, static_cast<int>(src.type), src.rows, mm + 2 * p, stream);
		}
		std::vector<int64_t> host(2 * pending.size());
		VGPU_CUDA(cudaMemcpyAsync(host.data(), mm, host.size() * 8, cudaMemcpyDeviceToHost, stream));
		VGPU_CUDA(cudaStreamSynchronize(stream));
		for (size_t p = 0; p < pending.size(); p++) {
			ranges[pending[p].first][pending[p].second] = {host[2 * p], host[2 * p + 1]};
		}
	}

	// Query table rows, largest queries first in the tile queue.
	const uint64_t kMaxBits = 22;
	std::vector<size_t> order;
	std::vector<uint64_t> dom(qs.size(), 0);
	std::vector<Prepared *> fitting;
	for (size_t qi = 0; qi < qs.size(); qi++) {
		uint64_t b = 0;
		for (int j = 0; j < nkeys; j++) {
			const auto &r = ranges[qi][j];
			if (r.first > r.second) continue;  // no rows
			b += BitsFor(static_cast<uint64_t>(r.second) - static_cast<uint64_t>(r.first));
		}
		dom[qi] = 1ull << std::min<uint64_t>(b, 63);
		if (b <= kMaxBits) fitting.push_back(qs[qi]);
		order.push_back(qi);
	}
	// A key space wider than the batch accumulators take belongs to the partitioned single-query
	// path: such queries leave the batch (they run alone afterwards) and the rest stay together.
	if (fitting.empty()) return false;
	if (fitting.size() != qs.size()) return RunTemplate(fitting, options, bopts, stream, results, stats);
	std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return qs[a]->rows > qs[b]->rows; });

	Geometry4 geo;
	const std::string tune_key = Sha256Hex(q0.sig.data(), q0.sig.size()).substr(0, 24) + "_sm" +
	                             std::to_string(props.cc_major) + std::to_string(props.cc_minor);
	bool have_tuned = Tuner().Lookup(tune_key, geo);
	(void)have_tuned;
	if (bopts.block) geo.block = bopts.block;
	if (bopts.items) geo.items = bopts.items;
	if (bopts.tile_rows) geo.tile_rows = bopts.tile_rows;
	if (bopts.smem_slots) geo.smem_slots = bopts.smem_slots;
	const uint64_t smem_cap = props.smem_optin > 2048 ? props.smem_optin - 2048 : 48 * 1024;

	std::vector<Geometry4> candidates;
	if (bopts.autotune) {
		for (auto bi : std::vector<std::pair<int, int>>{{256, 4}, {256, 8}, {512, 4}}) {
			for (int tile : {16384, 65536}) {
				for (int slots : {1024, 4096}) {
					Geometry4 c;
					c.block = bi.first;
					c.items = bi.second;
					c.tile_rows = tile;
					c.smem_slots = slots;
					candidates.push_back(c);
				}
			}
		}
	}
	candidates.push_back(geo);

	uint64_t in_bytes = 0, total_rows = 0;
	for (auto *q : qs) {
		total_rows += q->rows;
		for (auto &s : q->sources) in_bytes += q->rows * TypeSize(s.type);
	}

	auto build_entry = [&](Geometry4 g) -> std::shared_ptr<BatchEntry> {
		g.block = std::max(64, std::min(1024, g.block));
		g.items = std::max(1, std::min(16, g.items));
		g.tile_rows = static_cast<int>(NextPow2(std::max(1024, g.tile_rows)));
		g.smem_slots = static_cast<int>(NextPow2(std::max(32, g.smem_slots)));
		while (static_cast<uint64_t>(g.smem_slots) * F * 8 > smem_cap && g.smem_slots > 32) g.smem_slots >>= 1;
		// query table and tiles
		std::vector<uint64_t> qt(qs.size() * L.qwords, 0);
		std::vector<uint32_t> tl;
		std::vector<uint64_t> out_base(qs.size()), out_cap(qs.size());
		uint64_t acc_words = 0, out_rows = 0, ntiles = 0;
		for (size_t qi = 0; qi < qs.size(); qi++) {
			uint64_t *row = qt.data() + qi * L.qwords;
			row[0] = qs[qi]->rows;
			for (int i = 0; i < nsrc; i++) row[1 + 2 * i] = reinterpret_cast<uint64_t>(qs[qi]->sources[i].data);
			uint32_t shift = 0;
			for (int j = 0; j < nkeys; j++) {
				const auto &r = ranges[qi][j];
				const uint32_t kb = r.first > r.second ? 0u : static_cast<uint32_t>(BitsFor(static_cast<uint64_t>(r.second) - static_cast<uint64_t>(r.first)));
				row[L.key_base + 2 * j] = static_cast<uint64_t>(r.first > r.second ? 0 : r.first);
				row[L.key_base + 2 * j + 1] = shift | (kb << 8);
				shift += kb;
			}
			row[L.dom_base] = dom[qi];
			row[L.dom_base + 1] = acc_words;
			row[L.dom_base + 2] = out_rows;
			row[L.dom_base + 3] = dom[qi] <= static_cast<uint64_t>(g.smem_slots) ? 1 : 0;
			for (int p = 0; p < nparams; p++) row[L.param_base + p] = qs[qi]->params[p];
			out_base[qi] = out_rows;
			out_cap[qi] = std::max<uint64_t>(1, std::min<uint64_t>(dom[qi], qs[qi]->rows));
			acc_words += dom[qi];
			out_rows += out_cap[qi];
		}
		for (size_t qi : order) {
			const uint64_t t = (qs[qi]->rows + g.tile_rows - 1) / g.tile_rows;
			for (uint64_t k = 0; k < t; k++) {
				tl.push_back(static_cast<uint32_t>(qi));
				tl.push_back(static_cast<uint32_t>(k));
			}
			ntiles += t;
		}
		// Without a graph to replay (a composition that changes from call to call, as in serving) the
		// entry is transient: no cache lookup, no pinned staging, freed when the call ends.
		const bool transient = !bopts.use_graph && !bopts.autotune;
		std::string key = transient ? std::string()
		                            : q0.sig + "#" + g.ToString() + "#" + Sha256Hex(qt.data(), qt.size() * 8) +
		                                  Sha256Hex(tl.data(), tl.size() * 4);
		if (!transient) {
			if (auto e = Cache().Find(key)) return e;
		}
		auto e = std::make_shared<BatchEntry>();
		e->key = key;
		e->geo = g;
		e->F = F;
		e->nq = qs.size();
		e->ntiles = ntiles;
		e->acc_words = std::max<uint64_t>(1, acc_words);
		e->out_rows = out_rows;
		e->out_base = out_base;
		e->out_cap = out_cap;
		e->in_bytes = in_bytes;
		e->rows = total_rows;
		Geometry geom;
		geom.block = g.block;
		geom.items = g.items;
		e->module = Runtime::Get().modules().GetOrCompile(cg->EmitBatchGroupBy(gb, geom, g.tile_rows, g.smem_slots, L));
		e->smem = static_cast<size_t>(g.smem_slots) * F * 8;
		const int occ = Runtime::Get().MaxActiveBlocks(e->module->Get("vgpu_batch_gb"), g.block, e->smem);
		if (occ < 1) Fail(VGPU_ERR_UNSUPPORTED, "batch: kernel geometry does not fit on an SM");
		e->grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(ntiles, uint64_t(props.sm_count) * occ)));
		auto &al = Runtime::Get().allocator();
		const size_t out_words = gb.keys.size() + gb.aggs.size();
		e->qtab = static_cast<uint64_t *>(al.Alloc(qt.size() * 8, stream));
		e->tiles = al.Alloc(std::max<size_t>(8, tl.size() * 4), stream);
		e->acc = static_cast<uint64_t *>(al.Alloc(e->acc_words * F * 8, stream));
		e->counts = static_cast<uint64_t *>(al.Alloc(qs.size() * 8, stream));
		e->outp = static_cast<uint64_t *>(al.Alloc(out_words * 8, stream));
		e->work = static_cast<uint32_t *>(al.Alloc(16, stream));
		if (transient) {
			e->pinned = false;
			e->host_stage.assign(qs.size() + out_words, 0);
			e->counts_host = e->host_stage.data();
			e->outp_host = e->host_stage.data() + qs.size();
		} else {
			VGPU_CUDA(cudaMallocHost(&e->counts_host, qs.size() * 8));
			VGPU_CUDA(cudaMallocHost(&e->outp_host, out_words * 8));
		}
		VGPU_CUDA(cudaMemcpyAsync(e->qtab, qt.data(), qt.size() * 8, cudaMemcpyHostToDevice, stream));
		if (!tl.empty()) VGPU_CUDA(cudaMemcpyAsync(e->tiles, tl.data(), tl.size() * 4, cudaMemcpyHostToDevice, stream));
		VGPU_CUDA(cudaStreamSynchronize(stream));  // host staging vectors go out of scope
		if (!transient) Cache().Insert(e, stream);
		return e;
	};

	auto fill_args = [&](BatchEntry &e, uint64_t (&w)[128]) {
		std::memset(w, 0, sizeof(w));
		w[0] = e.nq;
		w[1] = reinterpret_cast<uint64_t>(e.qtab);
		w[2] = reinterpret_cast<uint64_t>(e.tiles);
		w[3] = e.ntiles;
		w[4] = reinterpret_cast<uint64_t>(e.work);
		w[5] = reinterpret_cast<uint64_t>(e.acc);
		w[6] = e.acc_words;
		w[7] = reinterpret_cast<uint64_t>(e.outp);
		w[8] = reinterpret_cast<uint64_t>(e.counts);
	};
	// The launches of one batch run: work counter reset, aggregate, finalize.
	auto enqueue = [&](BatchEntry &e, bool scoped) {
		uint64_t w[128];
		fill_args(e, w);
		VGPU_CUDA(cudaMemsetAsync(e.work, 0, 4, stream));
		if (scoped) {
			{
				LaunchScope scope("vgpu_batch_gb", stream, e.in_bytes, e.rows);
				LaunchRaw(*e.module, "vgpu_batch_gb", e.grid, e.geo.block, e.smem, stream, w);
			}
			LaunchScope scope("vgpu_batch_final", stream, e.acc_words * e.F * 8, e.acc_words);
			LaunchRaw(*e.module, "vgpu_batch_final", static_cast<unsigned>(e.nq), 1024, 0, stream, w);
		} else {
			LaunchRaw(*e.module, "vgpu_batch_gb", e.grid, e.geo.block, e.smem, stream, w);
			LaunchRaw(*e.module, "vgpu_batch_final", static_cast<unsigned>(e.nq), 1024, 0, stream, w);
		}
	};
	auto init_if_needed = [&](BatchEntry &e) {
		if (e.initialized) return;
		uint64_t w[128];
		fill_args(e, w);
		const uint64_t words = e.acc_words * e.F;
		const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((words + 255) / 256, uint64_t(props.sm_count) * 8));
		LaunchScope scope("vgpu_batch_init", stream, words * 8, 0);
		LaunchRaw(*e.module, "vgpu_batch_init", std::max(1u, grid), 256, 0, stream, w);
		e.initialized = true;
	};

	// Tuning: each candidate runs the real batch (discarding its output) and is timed on the stream.
	std::shared_ptr<BatchEntry> best;
	double best_ms = 1e30;
	const size_t out_words = gb.keys.size() + gb.aggs.size();
	if (candidates.size() > 1) {
		DeviceBuffers scratch_out;
		scratch_out.stream = stream;
		uint64_t max_out = 0;
		cudaEvent_t e0, e1;
		VGPU_CUDA(cudaEventCreate(&e0));
		VGPU_CUDA(cudaEventCreate(&e1));
		for (auto &c : candidates) {
			auto e = build_entry(c);
			if (e->out_rows > max_out) {
				for (void *p : scratch_out.ptrs) Runtime::Get().allocator().Free(p, stream);
				scratch_out.ptrs.clear();
				max_out = e->out_rows;
				for (size_t w = 0; w < out_words; w++) scratch_out.ptrs.push_back(Runtime::Get().allocator().Alloc(max_out * 16, stream));
			}
			for (size_t w = 0; w < out_words; w++) e->outp_host[w] = reinterpret_cast<uint64_t>(scratch_out.ptrs[w]);
			VGPU_CUDA(cudaMemcpyAsync(e->outp, e->outp_host, out_words * 8, cudaMemcpyHostToDevice, stream));
			init_if_needed(*e);
			enqueue(*e, false);
			float ms_best = 1e30f;
			for (int rep = 0; rep < 2; rep++) {
				VGPU_CUDA(cudaEventRecord(e0, stream));
				enqueue(*e, false);
				VGPU_CUDA(cudaEventRecord(e1, stream));
				VGPU_CUDA(cudaEventSynchronize(e1));
				float ms = 0;
				VGPU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
				ms_best = std::min(ms_best, ms);
			}
			if (ms_best < best_ms) {
				best_ms = ms_best;
				best = e;
			}
		}
		cudaEventDestroy(e0);
		cudaEventDestroy(e1);
		VGPU_CUDA(cudaStreamSynchronize(stream));
		Tuner().Record(tune_key, best->geo, best_ms);
	} else {
		best = build_entry(candidates.front());
	}
	BatchEntry &e = *best;

	// Outputs of this call, shared by its queries' results.
	auto holder = std::make_shared<DeviceBuffers>();
	holder->stream = stream;
	std::vector<ValueType> out_types;
	std::vector<std::string> out_names;
	for (int j = 0; j < nkeys; j++) {
		out_types.push_back(cg->visible()[key_cols[j]].type);
		out_names.push_back(root.group_keys[j]);
	}
	for (size_t i = 0; i < root.aggregates.size(); i++) {
		out_types.push_back(root.aggregates[i].output_type);
		out_names.push_back("agg_" + std::to_string(i));
	}
	for (size_t w = 0; w < out_words; w++) {
		holder->ptrs.push_back(Runtime::Get().allocator().Alloc(std::max<uint64_t>(1, e.out_rows) * TypeSize(out_types[w]), stream));
		e.outp_host[w] = reinterpret_cast<uint64_t>(holder->ptrs[w]);
	}
	VGPU_CUDA(cudaMemcpyAsync(e.outp, e.outp_host, out_words * 8, cudaMemcpyHostToDevice, stream));
	init_if_needed(e);
	const bool can_graph = bopts.use_graph && stream != nullptr && stream != cudaStreamLegacy && stream != cudaStreamPerThread;
	if (can_graph) {
		if (!e.graph) {
			cudaGraph_t g = nullptr;
			VGPU_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
			try {
				enqueue(e, false);
			} catch (...) {
				cudaStreamEndCapture(stream, &g);
				if (g) cudaGraphDestroy(g);
				throw;
			}
			VGPU_CUDA(cudaStreamEndCapture(stream, &g));
			cudaError_t err = cudaGraphInstantiate(&e.graph, g, 0);
			cudaGraphDestroy(g);
			if (err != cudaSuccess) {
				e.graph = nullptr;
				Fail(VGPU_ERR_CUDA, std::string("batch: graph instantiation failed: ") + cudaGetErrorString(err));
			}
		} else if (stats) {
			stats->graph_replays++;
		}
		LaunchScope scope("vgpu_batch_graph", stream, e.in_bytes, e.rows);
		Runtime::Get().CountLaunch(2);  // the aggregate and finalize kernels inside the graph
		VGPU_CUDA(cudaGraphLaunch(e.graph, stream));
	} else {
		enqueue(e, true);
	}
	VGPU_CUDA(cudaMemcpyAsync(e.counts_host, e.counts, e.nq * 8, cudaMemcpyDeviceToHost, stream));
	std::vector<std::vector<uint8_t>> host_out;
	if (!options.output_on_device) {
		host_out.resize(out_words);
		for (size_t w = 0; w < out_words; w++) {
			host_out[w].resize(e.out_rows * TypeSize(out_types[w]));
			VGPU_CUDA(cudaMemcpyAsync(host_out[w].data(), holder->ptrs[w], host_out[w].size(), cudaMemcpyDeviceToHost, stream));
		}
	}
	VGPU_CUDA(cudaStreamSynchronize(stream));

	for (size_t qi = 0; qi < qs.size(); qi++) {
		ExecResult r;
		r.stream = stream;
		const uint64_t cnt = e.counts_host[qi];
		if (cnt > e.out_cap[qi]) Fail(VGPU_ERR_INTERNAL, "batch: group count beyond its output capacity");
		for (size_t w = 0; w < out_words; w++) {
			HostColumnOut c;
			c.name = out_names[w];
			c.type = out_types[w];
			c.rows = cnt;
			const size_t width = TypeSize(out_types[w]);
			if (options.output_on_device) {
				c.device_data = static_cast<char *>(holder->ptrs[w]) + e.out_base[qi] * width;
			} else {
				const uint8_t *src = host_out[w].data() + e.out_base[qi] * width;
				c.data.assign(src, src + cnt * width);
			}
			r.columns.push_back(std::move(c));
		}
		if (options.output_on_device) r.keepalive.push_back(holder);
		results[qs[qi]->index] = std::move(r);
	}
	if (!e.pinned) e.Release(stream);  // transient: every copy out of it has completed
	if (stats) {
		stats->batched += qs.size();
		stats->templates++;
		stats->block = e.geo.block;
		stats->items = e.geo.items;
		stats->tile_rows = e.geo.tile_rows;
		stats->smem_slots = e.geo.smem_slots;
	}
	return true;
}

} // namespace

TemplatedSource TemplateLiterals(const std::string &src, int first_index) {
	TemplatedSource t;
	std::string out;
	const size_t n = src.size();
	size_t i = 0;
	while (i < n) {
		const char c = src[i];
		if (std::isalpha(static_cast<unsigned char>(c)) || c == '_') {
			size_t j = i;
			while (j < n && IdentChar(src[j])) j++;
			out.append(src, i, j - i);
			i = j;
			continue;
		}
		const bool starts_num = std::isdigit(static_cast<unsigned char>(c)) ||
		                        (c == '.' && i + 1 < n && std::isdigit(static_cast<unsigned char>(src[i + 1])));
		if (!starts_num) {
			out.push_back(c);
			i++;
			continue;
		}
		size_t j = i;
		bool is_float = false, hex = false;
		if (c == '0' && j + 1 < n && (src[j + 1] == 'x' || src[j + 1] == 'X')) {
			hex = true;
			j += 2;
			while (j < n && std::isxdigit(static_cast<unsigned char>(src[j]))) j++;
		} else {
			while (j < n && std::isdigit(static_cast<unsigned char>(src[j]))) j++;
			if (j < n && src[j] == '.') {
				is_float = true;
				j++;
				while (j < n && std::isdigit(static_cast<unsigned char>(src[j]))) j++;
			}
			if (j < n && (src[j] == 'e' || src[j] == 'E')) {
				size_t k = j + 1;
				if (k < n && (src[k] == '+' || src[k] == '-')) k++;
				if (k < n && std::isdigit(static_cast<unsigned char>(src[k]))) {
					is_float = true;
					j = k;
					while (j < n && std::isdigit(static_cast<unsigned char>(src[j]))) j++;
				}
			}
		}
		const size_t num_end = j;
		while (j < n && std::strchr("uUlLfF", src[j]) != nullptr) j++;
		const std::string number = src.substr(i, num_end - i);
		std::string suffix;
		for (size_t k = num_end; k < j; k++) suffix.push_back(static_cast<char>(std::tolower(static_cast<unsigned char>(src[k]))));
		const std::string literal = src.substr(i, j - i);
		// the index of an inputs[...] access stays literal
		size_t p = out.size();
		while (p > 0 && std::isspace(static_cast<unsigned char>(out[p - 1]))) p--;
		bool in_index = p >= 1 && out[p - 1] == '[';
		if (in_index) {
			size_t q = p - 1;
			while (q > 0 && std::isspace(static_cast<unsigned char>(out[q - 1]))) q--;
			const size_t e = q;
			while (q > 0 && IdentChar(out[q - 1])) q--;
			in_index = out.compare(q, e - q, "inputs") == 0;
		}
		if (in_index || (j < n && IdentChar(src[j]))) {
			out += literal;
			i = j;
			continue;
		}
		char type = 0;
		uint64_t bits = 0;
		if (is_float && !hex) {
			if (suffix == "f") {
				const float f = std::strtof(number.c_str(), nullptr);
				uint32_t b;
				std::memcpy(&b, &f, 4);
				bits = b;
				type = 'f';
			} else if (suffix.empty()) {
				const double d = std::strtod(number.c_str(), nullptr);
				std::memcpy(&bits, &d, 8);
				type = 'd';
			}
		} else if (!is_float && suffix.find('f') == std::string::npos) {
			errno = 0;
			const unsigned long long v = std::strtoull(number.c_str(), nullptr, 0);
			if (errno == 0) {
				const bool has_u = suffix.find('u') != std::string::npos;
				const bool has_l = suffix.find('l') != std::string::npos;
				const bool decimal = !hex && !(number.size() > 1 && number[0] == '0');
				if (!has_u && !has_l) {
					if (v <= static_cast<unsigned long long>(INT_MAX)) type = 'i';
					else if (!decimal && v <= UINT_MAX) type = 'u';
					else if (v <= static_cast<unsigned long long>(LLONG_MAX)) type = 'l';
					else if (!decimal) type = 'L';
				} else if (has_u && !has_l) {
					type = v <= UINT_MAX ? 'u' : 'L';
				} else if (has_l && !has_u) {
					if (v <= static_cast<unsigned long long>(LLONG_MAX)) type = 'l';
					else if (!decimal) type = 'L';
				} else {
					type = 'L';
				}
				bits = v;
			}
		}
		if (!type) {
			out += literal;
			i = j;
			continue;
		}
		const int idx = first_index + static_cast<int>(t.types.size());
		const char *fn = type == 'd' ? "vgpu_qpd" : type == 'f' ? "vgpu_qpf" : type == 'i' ? "vgpu_qpi"
		                 : type == 'u' ? "vgpu_qpu" : type == 'l' ? "vgpu_qpl" : "vgpu_qpul";
		out += std::string(fn) + "(" + std::to_string(idx) + ")";
		t.types.push_back(type);
		t.values.push_back(bits);
		i = j;
	}
	t.text = out;
	return t;
}

void ClearBatchCaches() {
	Cache().Clear(Runtime::Get().default_stream());
	Tuner().Clear();
}

std::shared_ptr<PreparedBatch> PrepareBatch(const std::vector<std::shared_ptr<PlanNode>> &plans) {
	auto pb = std::make_shared<PreparedBatch>();
	for (auto &plan : plans) {
		PreparedPlan pp;
		pp.plan = plan;
		pp.scan = HasWindowPrimitive(*plan) ? nullptr : BatchShape(*plan);  // one by one: refused there
		if (pp.scan) {
			pp.templ = TemplatePlan(*plan, pp.ptypes, pp.params);
			std::ostringstream sig;
			Signature(*pp.templ, sig);
			sig << "|params:" << std::string(pp.ptypes.begin(), pp.ptypes.end());
			pp.sig_base = sig.str();
		}
		pb->plans.push_back(std::move(pp));
	}
	return pb;
}

std::vector<ExecResult> ExecuteBatch(const std::vector<std::shared_ptr<PlanNode>> &plans,
                                     const std::vector<std::vector<vgpu_column>> &inputs, const ExecOptions &options,
                                     const BatchOptions &bopts, cudaStream_t stream, BatchStats *stats) {
	return ExecutePrepared(*PrepareBatch(plans), inputs, options, bopts, stream, stats);
}

std::vector<ExecResult> ExecutePrepared(const PreparedBatch &pb, const std::vector<std::vector<vgpu_column>> &inputs,
                                        const ExecOptions &options, const BatchOptions &bopts, cudaStream_t stream,
                                        BatchStats *stats) {
	const size_t nplans = pb.plans.size();
	if (nplans != inputs.size()) Fail(VGPU_ERR_INVALID_ARGUMENT, "batch: one input list per plan");
	if (options.cache_chunk_index >= 0 || options.stage_scan_to_cache) {
		Fail(VGPU_ERR_UNSUPPORTED, "batch: chunked cache serving and staging run through vgpu_execute_plan");
	}
	std::vector<ExecResult> results(nplans);
	std::vector<Prepared> prep(nplans);
	Arena arena(stream);  // device copies of host inputs, alive until the batch has run
	for (size_t i = 0; i < nplans; i++) {
		Prepared &p = prep[i];
		p.index = i;
		const PreparedPlan &pp = pb.plans[i];
		const PlanNode *scan = pp.scan;
		if (!scan) continue;
		bool ok = true;
		std::vector<DevColumn> cols;
		for (size_t k = 0; k < scan->column_names.size() && ok; k++) {
			DevColumn col;
			if (options.serve_whole_scan_from_cache) {
				ok = ColumnCache::Get().GetWhole(scan->table, scan->column_names[k], col) && col.valid == nullptr;
			} else {
				if (k >= inputs[i].size()) {
					ok = false;
					break;
				}
				const vgpu_column &in = inputs[i][k];
				if (in.validity != nullptr || !IsValidValueType(in.type)) {
					ok = false;
					break;
				}
				col.name = in.name ? in.name : "";
				col.type = static_cast<ValueType>(in.type);
				col.rows = in.row_count;
				const size_t bytes = static_cast<size_t>(in.row_count) * TypeSize(col.type);
				if (in.memory == VGPU_MEM_DEVICE) {
					col.data = const_cast<void *>(in.data);
				} else {
					col.data = arena.Alloc(bytes);
					if (bytes) VGPU_CUDA(cudaMemcpyAsync(col.data, in.data, bytes, cudaMemcpyHostToDevice, stream));
				}
				if (bytes && col.data == nullptr) ok = false;
			}
			if (ok && !cols.empty() && col.rows != cols.front().rows) ok = false;
			cols.push_back(col);
		}
		if (!ok || cols.empty()) continue;
		p.sources = cols;
		p.rows = cols.front().rows;
		p.templ = pp.templ;
		p.ptypes = pp.ptypes;
		p.params = pp.params;
		std::ostringstream sig;
		sig << pp.sig_base << "|types:";
		for (auto &c : cols) sig << static_cast<int>(c.type) << ",";
		p.sig = sig.str();
		p.batchable = true;
	}
	// Batch entries (output tables, captured graphs) are shared state: one batch runs at a time.
	static std::mutex batch_mu;
	std::lock_guard<std::mutex> lock(batch_mu);
	std::map<std::string, std::vector<Prepared *>> groups;
	for (auto &p : prep) {
		if (p.batchable) groups[p.sig].push_back(&p);
	}
	std::vector<bool> done(nplans, false);
	for (auto &kv : groups) {
		if (RunTemplate(kv.second, options, bopts, stream, results, stats)) {
			// batched queries always carry their key and aggregate columns; the rest run alone below
			for (auto *p : kv.second) done[p->index] = !results[p->index].columns.empty();
		}
	}
	VGPU_CUDA(cudaStreamSynchronize(stream));
	for (size_t i = 0; i < nplans; i++) {
		if (done[i]) continue;
		results[i] = ExecutePlan(*pb.plans[i].plan, inputs[i], options, stream);
		if (stats) stats->fallback++;
	}
	return results;
}

} // namespace vgpu
