// cost_model.cpp -- see cost_model.hpp.
#include "cost_model.hpp"

#include <algorithm>
#include <cstdio>
#include <cstring>

#include "codegen.hpp"

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

struct Walker {
	uint64_t cap = 0;
	const std::vector<uint64_t> *scan_rows;
	const std::vector<uint32_t> *scan_widths;
	size_t scan_index = 0;
	vgpu_working_set ws {};

	void Charge(const char *op, uint64_t bytes) {
		ws.total_bytes = SatAdd(ws.total_bytes, bytes);
		if (bytes > ws.largest_bytes) {
			ws.largest_bytes = bytes;
			std::snprintf(ws.largest_operator, sizeof(ws.largest_operator), "%s", op);
		}
	}

	uint64_t Rows(const PlanNode &n, uint64_t fallback) {
		uint64_t r = n.estimated_rows ? n.estimated_rows : fallback;
		if (cap && r > cap) {
			ws.chunk_capped = 1;
			r = cap;
		}
		return r;
	}

	Estimate Walk(const PlanNode &n) {
		Estimate e;
		switch (n.op) {
		case OpType::SCAN: {
			uint64_t rows = n.estimated_rows;
			uint64_t width = n.estimated_row_width_bytes ? n.estimated_row_width_bytes : 8 * n.column_names.size();
			if (scan_rows && scan_index < scan_rows->size()) rows = (*scan_rows)[scan_index];
			if (scan_widths && scan_index < scan_widths->size()) width = (*scan_widths)[scan_index];
			scan_index++;
			if (cap && rows > cap) {
				ws.chunk_capped = 1;
				rows = cap;
			}
			e.rows = rows;
			e.width = width;
			Charge("SCAN", SatMul(rows, width));
			return e;
		}
		case OpType::FILTER:
		case OpType::PROJECTION: {
			Estimate c = n.children.empty() ? Estimate {} : Walk(*n.children[0]);
			e.rows = c.rows;
			e.width = n.op == OpType::PROJECTION ? 8 * std::max<size_t>(1, n.expressions.size()) : c.width;
			// dense outputs plus per-tile counts
			Charge(n.op == OpType::FILTER ? "FILTER" : "PROJECTION", SatAdd(SatMul(e.rows, e.width), e.rows / 256 + 64));
			return e;
		}
		case OpType::GROUP_BY_AGGREGATE: {
			Estimate c = n.children.empty() ? Estimate {} : Walk(*n.children[0]);
			const uint64_t out_width = 8 * (n.group_keys.size() + n.aggregates.size()) + 8;
			// partitioned strategy: packed key + carried values per row, bucket outputs sized by rows
			uint64_t carried = 8;
			for (auto &a : n.aggregates) {
				if (a.kind != AggKind::COUNT && a.kind != AggKind::COUNT_STAR) carried += 8;
			}
			uint64_t bytes = SatAdd(SatMul(c.rows, carried), SatMul(c.rows, out_width));
			// partition offsets: (partitions <= 2^14, about one per 1024 rows) x (CTAs <= 2048) x 4 B
			bytes = SatAdd(bytes, SatMul(std::min<uint64_t>(16384, std::max<uint64_t>(1, c.rows / 1024)), 2048ull * 4));
			e.rows = n.estimated_rows ? n.estimated_rows : c.rows;
			e.width = out_width;
			Charge("GROUP_BY_AGGREGATE", bytes);
			return e;
		}
		case OpType::HASH_JOIN: {
			Estimate l = n.children.size() > 0 ? Walk(*n.children[0]) : Estimate {};
			Estimate r = n.children.size() > 1 ? Walk(*n.children[1]) : Estimate {};
			// widened keys + search results (left), widened keys + permutation + sort buffers (right)
			uint64_t bytes = SatAdd(SatMul(l.rows, 24), SatMul(r.rows, 24));
			const uint64_t out_rows = Rows(n, std::max(l.rows, r.rows));
			const uint64_t out_width = 8 * std::max<size_t>(1, n.output_columns.size());
			bytes = SatAdd(bytes, SatMul(out_rows, out_width + 8));
			e.rows = out_rows;
			e.width = out_width;
			Charge("HASH_JOIN", bytes);
			return e;
		}
		case OpType::CROSS_PRODUCT: {
			Estimate l = n.children.size() > 0 ? Walk(*n.children[0]) : Estimate {};
			Estimate r = n.children.size() > 1 ? Walk(*n.children[1]) : Estimate {};
			e.rows = SatMul(l.rows, r.rows);
			e.width = 8 * std::max<size_t>(1, n.output_columns.size());
			Charge("CROSS_PRODUCT", SatMul(e.rows, e.width));
			return e;
		}
		}
		return e;
	}
};

} // namespace

vgpu_working_set EstimateWorkingSet(const PlanNode &plan, uint64_t max_chunk_rows,
                                    const std::vector<uint64_t> *scan_rows,
                                    const std::vector<uint32_t> *scan_widths) {
	Walker w;
	w.cap = IsRowIndependent(plan) ? max_chunk_rows : 0;
	w.scan_rows = scan_rows;
	w.scan_widths = scan_widths;
	std::memset(&w.ws, 0, sizeof(w.ws));
	w.Walk(plan);
	return w.ws;
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
	if (cur->op != OpType::SCAN) {
		Fail(VGPU_ERR_UNSUPPORTED, "source generation without a device covers pipelines over a SCAN");
	}
	std::reverse(chain.begin(), chain.end());
	PipelineSpec spec;
	spec.chain = chain;
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
	PipelineCodegen cg(spec);
	Geometry g;
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
	// ... and both with tiles staged through shared memory by bulk copies
	Geometry gst = g;
	gst.items = 4;
	gst.staged = true;
	// Separate translation units, separated by a marker line: direct, partitioned, key statistics,
	// direct-partitioned, direct-partitioned with heavy keys, the last two staged.
	return cg.EmitGroupBy(spec_gb, false, g) + "\n//@@VGPU_TU@@\n" + cg.EmitGroupBy(spec_gb, true, g) +
	       "\n//@@VGPU_TU@@\n" + cg.EmitStats(key_columns, gs) + "\n//@@VGPU_TU@@\n" +
	       cg.EmitGroupBy(spec_dp, true, g) + "\n//@@VGPU_TU@@\n" + cg.EmitGroupBy(spec_hv, true, g) +
	       "\n//@@VGPU_TU@@\n" + cg.EmitGroupBy(spec_dp, true, gst) + "\n//@@VGPU_TU@@\n" +
	       cg.EmitGroupBy(spec_hv, true, gst);
}

} // namespace vgpu
