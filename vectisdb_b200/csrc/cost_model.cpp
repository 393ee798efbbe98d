// cost_model.cpp -- see cost_model.hpp.
#include "cost_model.hpp"

#include <algorithm>
#include <cstdio>
#include <cstring>

#include "codegen.hpp"
#include "column_cache.hpp"

namespace vgpu {

namespace {

struct Estimate {
	uint64_t rows = 0;
	uint64_t width = 0; // bytes per output row
};

uint64_t SatAdd(uint64_t a, uint64_t b) {
	return a > UINT64_MAX - b ? UINT64_MAX : a + b;
}

uint64_t SatMul(uint64_t a, uint64_t b) {
	if (a == 0 || b == 0) return 0;
	return a > UINT64_MAX / b ? UINT64_MAX : a * b;
}

// Byte width of one value of a plan-level type (HUGEINT sums are 16 bytes, key types unknown here
// count as 8).
uint64_t ValueBytes(ValueType t) {
	return TypeSize(t);
}

// Walk of the plan that charges what this engine's executor allocates for it (its arena and the result
// buffers), operator by operator. A FILTER / PROJECTION chain, and a join or cross product under one,
// is one fused kernel pipeline: it allocates only where its rows are materialized -- at the plan's root,
// or as the right (build) side of a join -- while under a GROUP BY it streams straight into the
// aggregation and allocates nothing per row.
struct Walker {
	uint64_t cap = 0;
	const std::vector<uint64_t> *scan_rows;
	const std::vector<uint32_t> *scan_widths;
	const std::vector<bool> *scan_resident;
	size_t scan_index = 0;
	vgpu_working_set ws {};

	void Charge(const char *op, uint64_t bytes) {
		ws.total_bytes = SatAdd(ws.total_bytes, bytes);
		if (bytes > ws.largest_bytes) {
			ws.largest_bytes = bytes;
			std::snprintf(ws.largest_operator, sizeof(ws.largest_operator), "%s", op);
		}
	}

	uint64_t Capped(uint64_t r) {
		if (cap && r > cap) {
			ws.chunk_capped = 1;
			r = cap;
		}
		return r;
	}

	// `materialize`: this node's rows become device columns (the root, a join's build side, a cross
	// product's sides); otherwise they stream into the pipeline above.
	Estimate Walk(const PlanNode &n, bool materialize) {
		Estimate e;
		switch (n.op) {
		case OpType::SCAN: {
			uint64_t rows = n.estimated_rows;
			uint64_t width = n.estimated_row_width_bytes ? n.estimated_row_width_bytes : 8 * n.column_names.size();
			bool resident = false;
			if (scan_rows && scan_index < scan_rows->size()) rows = (*scan_rows)[scan_index];
			if (scan_widths && scan_index < scan_widths->size()) width = (*scan_widths)[scan_index];
			if (scan_resident && scan_index < scan_resident->size()) resident = (*scan_resident)[scan_index];
			scan_index++;
			e.rows = Capped(rows);
			e.width = width;
			// host columns are copied to the device; resident ones (cache-served, device inputs) are borrowed
			if (!resident) Charge("SCAN", SatMul(e.rows, width));
			return e;
		}
		case OpType::FILTER:
		case OpType::PROJECTION: {
			Estimate c = n.children.empty() ? Estimate {} : Walk(*n.children[0], false);
			e.rows = c.rows;
			if (n.op == OpType::FILTER && n.estimated_rows) e.rows = std::min(c.rows, Capped(n.estimated_rows));
			if (n.op == OpType::PROJECTION) {
				e.width = 0;
				for (auto &x : n.expressions) e.width += ValueBytes(x.output_type);
				if (e.width == 0) e.width = 8;
			} else {
				e.width = c.width;
			}
			if (materialize) {  // dense outputs plus per-tile counts of the compaction
				Charge(n.op == OpType::FILTER ? "FILTER" : "PROJECTION", SatAdd(SatMul(e.rows, e.width), e.rows / 256 + 64));
			}
			return e;
		}
		case OpType::GROUP_BY_AGGREGATE: {
			Estimate c = n.children.empty() ? Estimate {} : Walk(*n.children[0], false);
			// state words per group: COUNT, then one per FP64 sum / MIN / MAX and two per integer sum
			uint64_t fields = 1, carried = 8, out_width = 8 * n.group_keys.size();
			for (auto &a : n.aggregates) {
				out_width += ValueBytes(a.output_type);
				if (a.kind == AggKind::COUNT || a.kind == AggKind::COUNT_STAR) continue;
				carried += 8;
				const bool int_sum = (a.kind == AggKind::SUM || a.kind == AggKind::AVG) && a.output_type == ValueType::HUGEINT;
				fields += int_sum ? 2 : 1;
			}
			const uint64_t groups = n.estimated_rows ? std::min(c.rows, n.estimated_rows) : c.rows;
			uint64_t bytes;
			if (SatMul(groups, fields * 8) <= 96 * 1024) {
				// one pass: per-CTA shared tables, one global table over the key domain, outputs
				bytes = SatAdd(SatMul(groups, fields * 8 + out_width), 64);
			} else {
				// partitioned: one record per passing row (packed key + carried values, 32-byte aligned),
				// outputs per group, per-(partition, CTA) offsets, tables of split partitions
				const uint64_t record = (carried + 31) / 32 * 32;
				bytes = SatMul(c.rows, record);
				bytes = SatAdd(bytes, SatMul(groups, out_width));
				// (at most 2^14 partitions x the CTAs' counters, bounded by the rows), and the split tables
				// (one per partition chunk of at least 16384 rows, at most 4 per SM of 148)
				bytes = SatAdd(bytes, std::min<uint64_t>(16384ull * 2048 * 4 / 8, SatMul(c.rows, 8)));
				bytes = SatAdd(bytes, SatMul(fields * 8 * 4096, std::min<uint64_t>(4 * 148, c.rows / 16384 + 1)));
			}
			e.rows = groups;
			e.width = out_width;
			Charge("GROUP_BY_AGGREGATE", bytes);
			return e;
		}
		case OpType::HASH_JOIN: {
			Estimate l = n.children.size() > 0 ? Walk(*n.children[0], !materialize ? false : true) : Estimate {};
			Estimate r = n.children.size() > 1 ? Walk(*n.children[1], true) : Estimate {};
			const uint64_t out_width = 8 * std::max<size_t>(1, n.output_columns.size());
			uint64_t bytes;
			if (!materialize) {
				// the join as a pipeline source: right keys widened, their range, a dense table (at most
				// 8 bytes per key of the range) or sorted keys with a radix directory
				bytes = SatMul(r.rows, 32);
				e.rows = n.estimated_rows ? Capped(n.estimated_rows) : l.rows;
			} else {
				// materializing: both sides' keys widened, the right side sorted with a permutation and
				// its double buffers, per-left-row ranges, one index pair and the output columns per match
				const uint64_t out_rows = n.estimated_rows ? Capped(n.estimated_rows) : std::max(l.rows, r.rows);
				bytes = SatAdd(SatMul(l.rows, 24), SatMul(r.rows, 24));
				bytes = SatAdd(bytes, SatMul(out_rows, out_width + 8));
				e.rows = out_rows;
			}
			e.width = out_width;
			Charge("HASH_JOIN", bytes);
			return e;
		}
		case OpType::CROSS_PRODUCT: {
			Estimate l = n.children.size() > 0 ? Walk(*n.children[0], true) : Estimate {};
			Estimate r = n.children.size() > 1 ? Walk(*n.children[1], true) : Estimate {};
			e.rows = SatMul(l.rows, r.rows);
			e.width = 8 * std::max<size_t>(1, n.output_columns.size());
			// a virtual pair space under a pipeline; materialized only at the root
			if (materialize) Charge("CROSS_PRODUCT", SatMul(e.rows, e.width));
			return e;
		}
		}
		return e;
	}
};

} // namespace

vgpu_working_set EstimateWorkingSet(const PlanNode &plan, uint64_t max_chunk_rows,
                                    const std::vector<uint64_t> *scan_rows,
                                    const std::vector<uint32_t> *scan_widths,
                                    const std::vector<bool> *scan_resident) {
	Walker w;
	w.cap = IsRowIndependent(plan) ? max_chunk_rows : 0;
	w.scan_rows = scan_rows;
	w.scan_widths = scan_widths;
	w.scan_resident = scan_resident;
	std::memset(&w.ws, 0, sizeof(w.ws));
	w.Walk(plan, true);
	return w.ws;
}

vgpu_working_set EstimateWorkingSetFor(const PlanNode &plan, const std::vector<vgpu_column> &inputs,
                                       bool serve_from_cache) {
	std::vector<const PlanNode *> scans;
	CollectScans(plan, scans);
	std::vector<uint64_t> rows;
	std::vector<uint32_t> widths;
	std::vector<bool> resident;
	size_t cursor = 0;
	for (auto *scan : scans) {
		uint64_t r = 0;
		uint32_t w = 0;
		bool res = true;
		for (auto &name : scan->column_names) {
			if (serve_from_cache) {
				DevColumn col;
				if (ColumnCache::Get().GetWhole(scan->table, name, col)) {
					r = col.rows;
					w += static_cast<uint32_t>(TypeSize(col.type));
				}
			} else if (cursor < inputs.size()) {
				const vgpu_column &in = inputs[cursor++];
				r = in.row_count;
				if (IsValidValueType(in.type)) w += static_cast<uint32_t>(TypeSize(static_cast<ValueType>(in.type)));
				if (in.memory != VGPU_MEM_DEVICE) res = false;
			}
		}
		rows.push_back(r);
		widths.push_back(w);
		resident.push_back(res);
	}
	return EstimateWorkingSet(plan, 0, &rows, &widths, &resident);
}

namespace {

uint64_t ScanWidth(const PlanNode &n) {
	return n.estimated_row_width_bytes ? n.estimated_row_width_bytes : 8;
}

// Post-order walk: SCAN leaves add their rows and bytes; every node may raise max_rows and adds its
// expressions' price times the rows they run over (a FILTER tests every row entering it).
void Shape(const PlanNode &n, vgpu_plan_shape &s) {
	for (auto &c : n.children) Shape(*c, s);
	if (n.op == OpType::SCAN) {
		s.scanned_rows = SatAdd(s.scanned_rows, n.estimated_rows);
		s.scanned_bytes = SatAdd(s.scanned_bytes, SatMul(n.estimated_rows, ScanWidth(n)));
	}
	s.max_rows = std::max<uint64_t>(s.max_rows, n.estimated_rows);
	double price = 0.0;
	for (auto &e : n.expressions) price += e.ops_per_row;
	if (price != 0.0) {
		uint64_t rows = n.estimated_rows;
		if (n.op == OpType::FILTER) rows = n.children.empty() ? 0 : n.children[0]->estimated_rows;
		s.total_ops += price * static_cast<double>(rows);
	}
}

} // namespace

vgpu_plan_shape AnalyzePlanShape(const PlanNode &plan) {
	vgpu_plan_shape s;
	std::memset(&s, 0, sizeof(s));
	Shape(plan, s);
	// Nothing scanned means nothing to amortise: the ratios fall back to the numerators themselves.
	const double rows = static_cast<double>(s.scanned_rows);
	const double bytes = static_cast<double>(s.scanned_bytes);
	s.amplification = s.scanned_rows ? static_cast<double>(s.max_rows) / rows : static_cast<double>(s.max_rows);
	s.ops_per_scanned_row = s.scanned_rows ? s.total_ops / rows : s.total_ops;
	s.ops_per_scanned_byte = s.scanned_bytes ? s.total_ops / bytes : s.total_ops;
	// Nothing priced is "unmeasured", never "cheap" (a group-by over a cross product carries no
	// expression yet does the most work of all).
	if (s.total_ops == 0.0) {
		s.density = VGPU_DENSITY_INCONCLUSIVE;
	} else if (s.ops_per_scanned_row >= VGPU_OFFLOAD_OPS_PER_ROW) {
		s.density = VGPU_DENSITY_SUFFICIENT;
	} else if (s.ops_per_scanned_row < VGPU_MIN_OPS_PER_SCANNED_ROW) {
		s.density = VGPU_DENSITY_INSUFFICIENT;
	} else {
		s.density = VGPU_DENSITY_INCONCLUSIVE;
	}
	return s;
}

uint64_t EstimateColumnsSize(const PlanNode &plan) {
	uint64_t total = plan.op == OpType::SCAN ? SatMul(plan.estimated_rows, ScanWidth(plan)) : 0;
	for (auto &c : plan.children) total = SatAdd(total, EstimateColumnsSize(*c));
	return total;
}

vgpu_execution_mode DetermineExecutionMode(const PlanNode &plan, uint64_t vram_budget, double threshold) {
	const double size = static_cast<double>(EstimateColumnsSize(plan));
	if (vram_budget > 0 && size > static_cast<double>(vram_budget) * threshold) {
		return VGPU_MODE_PIPELINE_STREAM_UNCACHED;
	}
	return VGPU_MODE_PIPELINE_STREAM_CACHED;
}

std::string GenerateSourceText(const PlanNode &plan, const std::vector<vgpu_column> &inputs) {
	const PlanNode *gb = nullptr;
	const PlanNode *cur = &plan;
	if (cur->op == OpType::GROUP_BY_AGGREGATE) {
		gb = cur;
		if (cur->children.size() != 1) Fail(VGPU_ERR_INVALID_ARGUMENT, "GROUP_BY expects one child");
		cur = cur->children[0].get();
	}
	std::vector<const PlanNode *> chain;
	while (cur->op == OpType::FILTER || cur->op == OpType::PROJECTION) {
		if (cur->children.size() != 1) Fail(VGPU_ERR_INVALID_ARGUMENT, "chain node expects one child");
		chain.push_back(cur);
		cur = cur->children[0].get();
	}
	std::reverse(chain.begin(), chain.end());
	PipelineSpec spec;
	spec.chain = chain;
	if (cur->op == OpType::HASH_JOIN) {
		// a join source over two SCANs: left columns, then the right output columns, then the left key;
		// the one-match and the multi-match lookups are both generated
		if (cur->children.size() != 2 || cur->children[0]->op != OpType::SCAN || cur->children[1]->op != OpType::SCAN ||
		    cur->build_keys.size() != 1) {
			Fail(VGPU_ERR_UNSUPPORTED, "source generation without a device covers joins of two SCANs");
		}
		const auto &ln = cur->children[0]->column_names, &rn = cur->children[1]->column_names;
		if (inputs.size() < ln.size() + rn.size()) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "plan expects more scanned columns than were supplied");
		}
		auto input_of = [&](const std::string &name, int *side) -> const vgpu_column * {
			for (size_t i = 0; i < ln.size(); i++) {
				if (ln[i] == name) { *side = 0; return &inputs[i]; }
			}
			for (size_t i = 0; i < rn.size(); i++) {
				if (rn[i] == name) { *side = 1; return &inputs[ln.size() + i]; }
			}
			Fail(VGPU_ERR_INVALID_ARGUMENT, "join column '" + name + "' not found");
		};
		for (auto &name : cur->output_columns) {
			int side = 0;
			const vgpu_column *in = input_of(name, &side);
			SourceColumn s;
			s.name = name;
			s.type = static_cast<ValueType>(in->type);
			s.nullable = in->validity != nullptr;
			s.side = side;
			spec.sources.push_back(s);
		}
		int side = 0;
		const vgpu_column *key = input_of(cur->build_keys[0], &side);
		SourceColumn k;
		k.name = "__vgpu_join_key";
		k.type = static_cast<ValueType>(key->type);
		spec.join_key = static_cast<int>(spec.sources.size());
		spec.sources.push_back(k);
		spec.join = true;
	} else if (cur->op != OpType::SCAN) {
		Fail(VGPU_ERR_UNSUPPORTED, "source generation without a device covers pipelines over a SCAN or a join");
	} else {
		if (inputs.size() < cur->column_names.size()) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "plan expects more scanned columns than were supplied");
		}
		for (size_t i = 0; i < cur->column_names.size(); i++) {
			SourceColumn s;
			s.name = inputs[i].name ? inputs[i].name : "";
			s.type = static_cast<ValueType>(inputs[i].type);
			s.nullable = inputs[i].validity != nullptr;
			spec.sources.push_back(s);
		}
	}
	PipelineCodegen cg(spec);
	Geometry g;
	if (spec.join) {
		PipelineSpec multi = spec;
		multi.join_multi = true;
		PipelineCodegen cgm(multi);
		PipelineSpec minline = multi;  // ... with the right column inline, one slot per match
		minline.join_minline = true;
		PipelineCodegen cgi(minline);
		std::vector<int> outs;
		for (size_t i = 0; i < cg.visible().size(); i++) outs.push_back(static_cast<int>(i));
		std::string text = cg.EmitMaterialize(outs, g) + "\n//@@VGPU_TU@@\n" + cgm.EmitMaterialize(outs, g) +
		                   "\n//@@VGPU_TU@@\n" + cgm.EmitStats(outs, g) + "\n//@@VGPU_TU@@\n" +
		                   cgi.EmitMaterialize(outs, g);
		if (!gb) return text;
		PipelineCodegen::GroupBySpec spec_gb;
		int shift = 0;
		for (auto &kname : gb->group_keys) {
			PipelineCodegen::GroupKey key;
			key.column = cg.FindVisible(kname);
			if (key.column < 0) Fail(VGPU_ERR_INVALID_ARGUMENT, "group key '" + kname + "' not found");
			key.min = 0;
			key.bits = 16;
			key.shift = shift;
			shift += 16;
			spec_gb.keys.push_back(key);
		}
		for (auto &a : gb->aggregates) {
			PipelineCodegen::AggSpec as;
			as.kind = a.kind;
			as.output_type = a.output_type;
			if (a.kind != AggKind::COUNT_STAR) {
				as.column = cg.FindVisible(a.input_column);
				if (as.column < 0) Fail(VGPU_ERR_INVALID_ARGUMENT, "aggregate input '" + a.input_column + "' not found");
				as.input_type = cg.visible()[as.column].type;
			}
			spec_gb.aggs.push_back(as);
		}
		Geometry gj;
		gj.block = 512;
		gj.items = 8;
		return text + "\n//@@VGPU_TU@@\n" + cg.EmitGroupBy(spec_gb, false, gj) + "\n//@@VGPU_TU@@\n" +
		       cgm.EmitGroupBy(spec_gb, false, gj) + "\n//@@VGPU_TU@@\n" + cgi.EmitGroupBy(spec_gb, false, gj);
	}
	if (!gb) {
		std::vector<int> outs;
		for (size_t i = 0; i < cg.visible().size(); i++) outs.push_back(static_cast<int>(i));
		return cg.EmitMaterialize(outs, g);
	}
	PipelineCodegen::GroupBySpec spec_gb;
	int shift = 0;
	for (auto &k : gb->group_keys) {
		PipelineCodegen::GroupKey key;
		key.column = cg.FindVisible(k);
		if (key.column < 0) Fail(VGPU_ERR_INVALID_ARGUMENT, "group key '" + k + "' not found");
		key.min = 0;
		key.bits = 16;
		key.shift = shift;
		shift += 16;
		spec_gb.keys.push_back(key);
	}
	for (auto &a : gb->aggregates) {
		PipelineCodegen::AggSpec s;
		s.kind = a.kind;
		s.output_type = a.output_type;
		if (a.kind != AggKind::COUNT_STAR) {
			s.column = cg.FindVisible(a.input_column);
			if (s.column < 0) Fail(VGPU_ERR_INVALID_ARGUMENT, "aggregate input '" + a.input_column + "' not found");
			s.input_type = cg.visible()[s.column].type;
		}
		spec_gb.aggs.push_back(s);
	}
	g.block = 512;
	std::vector<int> key_columns;
	for (auto &k : spec_gb.keys) key_columns.push_back(k.column);
	Geometry gs;
	// Direct-partitioned variant: 2^12-slot tables over the 16-bit-per-key packing.
	PipelineCodegen::GroupBySpec spec_dp = spec_gb;
	spec_dp.direct_bits = 12;
	spec_dp.key_bits = shift;
	spec_dp.key_mult = (0x9e3779b97f4a7c15ull & (shift >= 64 ? ~0ull : (1ull << shift) - 1)) | 1ull;
	spec_dp.key_mult_inv = 1;
	spec_dp.bucket_threads = 1024;
	// ... and its heavy-key variant (sampling kernel, pre-aggregating partition passes)
	PipelineCodegen::GroupBySpec spec_hv = spec_dp;
	spec_hv.heavy_slots = 512;
	spec_hv.heavy_warp = true;
	PipelineCodegen::GroupBySpec spec_plain = spec_dp;
	spec_plain.bucket_plain = true;
	spec_hv.f64_l2 = PipelineCodegen::F64Fields(spec_hv) > 0;  // FP64 sums of its bucket pass in L2
	PipelineCodegen::GroupBySpec spec_nc = spec_gb;
	spec_nc.narrow_count = true;  // one-pass tables whose counts take no carries
	spec_nc.count_as_flag = true;  // ... or are presence flags
	spec_nc.f64_l2 = PipelineCodegen::F64Fields(spec_nc) > 0;  // ... and FP64 sums in L2
	if (cg.DirectFinalFused(spec_nc)) {  // ... and integer MIN/MAX as 32-bit offsets
		int word = cg.ConsumerBase() + 4 + PipelineCodegen::StateWords(spec_nc) +
		           static_cast<int>(spec_nc.keys.size() + spec_nc.aggs.size());
		for (auto &a : spec_nc.aggs) {
			const bool narrowable = (a.kind == AggKind::MIN || a.kind == AggKind::MAX) &&
			                        (a.input_type == ValueType::INT16 || a.input_type == ValueType::INT32 ||
			                         a.input_type == ValueType::INT64);
			if (narrowable && word < kKeyWord) a.narrow_word = word++;
		}
	}
	// ... and both with tiles staged through shared memory by bulk copies
	Geometry gst = g;
	gst.items = 4;
	gst.staged = true;
	// Separate translation units, separated by a marker line: direct, partitioned, key statistics,
	// direct-partitioned, direct-partitioned with heavy keys, the last two staged, the plain bucket pass,
	// and the direct one with narrow counts and MIN/MAX.
	return cg.EmitGroupBy(spec_gb, false, g) + "\n//@@VGPU_TU@@\n" + cg.EmitGroupBy(spec_gb, true, g) +
	       "\n//@@VGPU_TU@@\n" + cg.EmitStats(key_columns, gs) + "\n//@@VGPU_TU@@\n" +
	       cg.EmitGroupBy(spec_dp, true, g) + "\n//@@VGPU_TU@@\n" + cg.EmitGroupBy(spec_hv, true, g) +
	       "\n//@@VGPU_TU@@\n" + cg.EmitGroupBy(spec_dp, true, gst) + "\n//@@VGPU_TU@@\n" +
	       cg.EmitGroupBy(spec_hv, true, gst) + "\n//@@VGPU_TU@@\n" + cg.EmitGroupBy(spec_plain, true, g) +
	       "\n//@@VGPU_TU@@\n" + cg.EmitGroupBy(spec_nc, false, g);
}

} // namespace vgpu
