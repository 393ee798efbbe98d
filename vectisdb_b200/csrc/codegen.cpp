// codegen.cpp -- see codegen.hpp.
#include "codegen.hpp"

#include <algorithm>
#include <mutex>
#include <cctype>
#include <map>
#include <regex>
#include <set>
#include <sstream>

namespace vgpu {

size_t CTypeSize(const std::string &ctype) {
	static const std::map<std::string, size_t> sizes = {
	    {"bool", 1},          {"char", 1},          {"signed char", 1},         {"unsigned char", 1},
	    {"short", 2},         {"unsigned short", 2}, {"int", 4},                {"unsigned int", 4},
	    {"unsigned", 4},      {"float", 4},         {"long long", 8},           {"unsigned long long", 8},
	    {"double", 8},        {"long", 8},          {"long long int", 8},       {"short int", 2}};
	auto it = sizes.find(ctype);
	return it == sizes.end() ? 0 : it->second;
}

namespace {

std::string NormalizeCType(std::string t) {
	// collapse internal whitespace
	std::string out;
	bool space = false;
	for (char c : t) {
		if (c == ' ' || c == '\t' || c == '\n') {
			space = !out.empty();
			continue;
		}
		if (space) {
			out += ' ';
			space = false;
		}
		out += c;
	}
	if (out == "long long int") {
		out = "long long";
	}
	if (out == "short int") {
		out = "short";
	}
	if (out == "unsigned") {
		out = "unsigned int";
	}
	if (out == "long") {
		out = "long long";
	}
	return out;
}

bool ContainsWord(const std::string &s, const std::string &word) {
	size_t pos = 0;
	while ((pos = s.find(word, pos)) != std::string::npos) {
		bool left_ok = pos == 0 || !(std::isalnum(static_cast<unsigned char>(s[pos - 1])) || s[pos - 1] == '_');
		size_t end = pos + word.size();
		bool right_ok = end >= s.size() || !(std::isalnum(static_cast<unsigned char>(s[end])) || s[end] == '_');
		if (left_ok && right_ok) {
			return true;
		}
		pos = end;
	}
	return false;
}

} // namespace

RewrittenExpr RewriteExpression(const std::string &source, size_t n_inputs) {
	static const std::regex input_re(
	    R"(\(\s*\(\s*const\s+([A-Za-z_][A-Za-z_0-9 ]*?)\s*\*\s*\)\s*inputs\s*\[\s*(\d+)\s*\]\s*\)\s*\[\s*row\s*\])");
	static const std::regex output_re(R"(\(\s*\(\s*([A-Za-z_][A-Za-z_0-9 ]*?)\s*\*\s*\)\s*out\s*\)\s*\[\s*idx\s*\])");
	RewrittenExpr rw;
	rw.input_ctypes.assign(n_inputs, "");
	std::string s;
	{
		std::string rest = source;
		std::smatch m;
		while (std::regex_search(rest, m, input_re)) {
			size_t index = std::stoul(m[2].str());
			if (index >= n_inputs) {
				Fail(VGPU_ERR_INVALID_ARGUMENT, "expression reads inputs[" + std::to_string(index) + "] but lists only " +
				                                    std::to_string(n_inputs) + " input columns");
			}
			std::string ctype = NormalizeCType(m[1].str());
			if (!rw.input_ctypes[index].empty() && rw.input_ctypes[index] != ctype) {
				Fail(VGPU_ERR_UNSUPPORTED, "expression reads inputs[" + std::to_string(index) + "] as two different types");
			}
			rw.input_ctypes[index] = ctype;
			s += m.prefix().str();
			s += "vgpu_in_" + std::to_string(index);
			rest = m.suffix().str();
		}
		s += rest;
	}
	std::smatch m;
	std::string out;
	int writes = 0;
	{
		std::string rest = s;
		while (std::regex_search(rest, m, output_re)) {
			std::string ctype = NormalizeCType(m[1].str());
			if (!rw.output_ctype.empty() && rw.output_ctype != ctype) {
				Fail(VGPU_ERR_UNSUPPORTED, "expression writes out[] as two different types");
			}
			rw.output_ctype = ctype;
			out += m.prefix().str();
			out += "vgpu_out";
			rest = m.suffix().str();
			writes++;
		}
		out += rest;
	}
	if (writes == 0) {
		Fail(VGPU_ERR_UNSUPPORTED, "expression source does not write ((T*)out)[idx]: " + source);
	}
	for (const char *word : {"inputs", "out", "row", "idx", "sel", "input_valid", "out_valid"}) {
		if (ContainsWord(out, word)) {
			Fail(VGPU_ERR_UNSUPPORTED, std::string("expression source uses '") + word +
			                               "' outside the ((const T*)inputs[i])[row] / ((T*)out)[idx] forms: " +
			                               source);
		}
	}
	if (CTypeSize(rw.output_ctype) == 0) {
		Fail(VGPU_ERR_UNSUPPORTED, "expression writes an unsupported C type '" + rw.output_ctype + "'");
	}
	for (auto &t : rw.input_ctypes) {
		if (!t.empty() && CTypeSize(t) == 0) {
			Fail(VGPU_ERR_UNSUPPORTED, "expression reads an unsupported C type '" + t + "'");
		}
	}
	rw.statement = out;
	return rw;
}

// ============================================================================================
// PipelineCodegen

PipelineCodegen::PipelineCodegen(const PipelineSpec &spec) : spec_(spec) {
	for (auto &src : spec_.sources) {
		if (src.type == ValueType::HUGEINT) {
			Fail(VGPU_ERR_UNSUPPORTED, "column '" + src.name + "': HUGEINT columns cannot feed a fused pipeline");
		}
	}
	Resolve();
}

int PipelineCodegen::FindVisible(const std::string &name) const {
	for (size_t i = 0; i < visible_.size(); i++) {
		if (visible_[i].name == name) {
			return static_cast<int>(i);
		}
	}
	return -1;
}

std::string PipelineCodegen::EmitExpression(const Expr &expr, const std::vector<PipeColumn> &cols, int k) {
	RewrittenExpr rw = RewriteExpression(expr.source, expr.input_columns.size());
	std::ostringstream o;
	const char *out_c = CudaTypeName(expr.output_type);
	if (expr.output_type == ValueType::HUGEINT) {
		Fail(VGPU_ERR_UNSUPPORTED, "expressions producing HUGEINT are not supported");
	}
	if (CTypeSize(rw.output_ctype) != TypeSize(expr.output_type)) {
		Fail(VGPU_ERR_UNSUPPORTED, "expression writes " + rw.output_ctype + " into a " + TypeName(expr.output_type) +
		                               " result");
	}
	o << "\t\t" << out_c << " e" << k << ";\n\t\t{\n";
	std::vector<std::string> valids;
	for (size_t i = 0; i < expr.input_columns.size(); i++) {
		if (rw.input_ctypes[i].empty()) {
			continue;
		}
		const std::string &name = expr.input_columns[i];
		const PipeColumn *col = nullptr;
		for (auto &c : cols) {
			if (c.name == name) {
				col = &c;
				break;
			}
		}
		if (!col) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_executor: expression input column '" + name + "' not found");
		}
		if (CTypeSize(rw.input_ctypes[i]) != TypeSize(col->type)) {
			Fail(VGPU_ERR_UNSUPPORTED, "expression reads column '" + name + "' (" + TypeName(col->type) + ") as " +
			                               rw.input_ctypes[i]);
		}
		o << "\t\t\tconst " << rw.input_ctypes[i] << " vgpu_in_" << i << " = vgpu_dev::reinterpret_value<"
		  << rw.input_ctypes[i] << ", " << CudaTypeName(col->type) << ">(" << col->value << ");\n";
		if (col->nullable) {
			valids.push_back("(" + col->valid + ")");
		}
	}
	o << "\t\t\t" << rw.output_ctype << " vgpu_out;\n";
	o << "\t\t\t" << rw.statement << "\n";
	o << "\t\t\te" << k << " = vgpu_dev::reinterpret_value<" << out_c << ", " << rw.output_ctype << ">(vgpu_out);\n";
	o << "\t\t}\n";
	o << "\t\tconst bool ev" << k << " = ";
	if (valids.empty()) {
		o << "true";
	} else {
		for (size_t i = 0; i < valids.size(); i++) {
			o << (i ? " && " : "") << valids[i];
		}
	}
	o << ";\n";
	return o.str();
}

void PipelineCodegen::Resolve() {
	std::vector<PipeColumn> cols;
	for (size_t i = 0; i < spec_.sources.size(); i++) {
		PipeColumn c;
		c.name = spec_.sources[i].name;
		c.type = spec_.sources[i].type;
		c.source = static_cast<int>(i);
		c.value = "s" + std::to_string(i) + "[r]";
		c.nullable = spec_.sources[i].nullable;
		c.valid = c.nullable ? "sv" + std::to_string(i) + "[r]" : "true";
		cols.push_back(c);
	}
	chain_sources_.assign(spec_.sources.size(), false);
	std::ostringstream code;
	if (spec_.join) {
		// left rows without a match in the right side are not join output rows
		if (spec_.join_key < 0 || spec_.join_key >= static_cast<int>(spec_.sources.size())) {
			Fail(VGPU_ERR_INTERNAL, "join pipeline without a key source");
		}
		code << "\t\tkeep = keep && (jm[r] >= 0);\n";
		chain_sources_[spec_.join_key] = true;
		has_filter_ = true;
	}
	// Sources read by each visible column (transitively through projections).
	std::vector<std::set<int>> deps(cols.size());
	for (size_t i = 0; i < cols.size(); i++) {
		deps[i].insert(static_cast<int>(i));
	}
	for (const PlanNode *node : spec_.chain) {
		if (node->op == OpType::FILTER) {
			for (auto &expr : node->expressions) {
				if (expr.output_type != ValueType::BOOLEAN) {
					Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_executor: FILTER predicate did not evaluate to BOOLEAN");
				}
				int k = expr_count_++;
				code << EmitExpression(expr, cols, k);
				code << "\t\tkeep = keep && ev" << k << " && e" << k << ";\n";
				for (auto &in : expr.input_columns) {
					for (size_t c = 0; c < cols.size(); c++) {
						if (cols[c].name == in) {
							for (int s : deps[c]) {
								chain_sources_[s] = true;
							}
							break;
						}
					}
				}
			}
			if (!node->expressions.empty()) {
				has_filter_ = true;
			}
		} else if (node->op == OpType::PROJECTION) {
			std::vector<PipeColumn> next;
			std::vector<std::set<int>> next_deps;
			for (size_t i = 0; i < node->expressions.size(); i++) {
				auto &expr = node->expressions[i];
				int k = expr_count_++;
				code << EmitExpression(expr, cols, k);
				PipeColumn c;
				c.name = "col" + std::to_string(i);
				c.type = expr.output_type;
				c.value = "e" + std::to_string(k);
				c.valid = "ev" + std::to_string(k);
				std::set<int> d;
				bool nullable = false;
				for (auto &in : expr.input_columns) {
					for (size_t cc = 0; cc < cols.size(); cc++) {
						if (cols[cc].name == in) {
							d.insert(deps[cc].begin(), deps[cc].end());
							nullable |= cols[cc].nullable;
							break;
						}
					}
				}
				// The chain code evaluates every projection, so every source it reads must be loaded
				// (loads whose values end up unused are dead code the compiler drops).
				for (int s : d) {
					chain_sources_[s] = true;
				}
				c.nullable = nullable;
				if (!nullable) {
					c.valid = "true";
				}
				// An identity projection (out = in, same type) passes its source column through, so the
				// source's statistics (key ranges for group-by packing) still describe it.
				if (expr.input_columns.size() == 1) {
					RewrittenExpr rw = RewriteExpression(expr.source, 1);
					std::string st;
					for (char ch : rw.statement) {
						if (!std::isspace(static_cast<unsigned char>(ch))) st += ch;
					}
					if (st == "vgpu_out=vgpu_in_0;" && rw.input_ctypes[0] == rw.output_ctype) {
						for (size_t cc = 0; cc < cols.size(); cc++) {
							if (cols[cc].name == expr.input_columns[0] && cols[cc].source >= 0 &&
							    cols[cc].type == expr.output_type) {
								c.source = cols[cc].source;
							}
						}
					}
				}
				next.push_back(c);
				next_deps.push_back(d);
			}
			cols = std::move(next);
			deps = std::move(next_deps);
		} else {
			Fail(VGPU_ERR_INTERNAL, "pipeline chain may hold only FILTER/PROJECTION nodes");
		}
	}
	visible_ = cols;
	chain_uses_.clear();
	for (auto &d : deps) {
		chain_uses_.emplace_back(d.begin(), d.end());
	}
	chain_code_ = code.str();
}

std::vector<bool> PipelineCodegen::NeededSources(const std::vector<int> &extra_columns) const {
	std::vector<bool> needed = chain_sources_;
	for (int c : extra_columns) {
		for (int s : chain_uses_[c]) {
			needed[s] = true;
		}
	}
	return needed;
}

std::string PipelineCodegen::Prologue() const {
	return "#include \"vgpu_device_lib.cuh\"\n"
	       "using namespace vgpu_dev;\n"
	       "__device__ __forceinline__ double __vgpu_radians(double d) { return d * 0.017453292519943295; }\n"
	       "__device__ __forceinline__ double __vgpu_degrees(double r) { return r * 57.29577951308232; }\n";
}

std::string PipelineCodegen::LoadBlock(const Geometry &g, const std::vector<bool> &needed, bool chunked) const {
	(void)chunked;
	std::ostringstream o;
	o << "\t\tconst u64 row0 = tile * (u64)" << g.tile() << " + (u64)threadIdx.x * " << g.items << ";\n";
	if (spec_.cross) {
		o << "\t\tu64 li[" << g.items << "], rj[" << g.items << "];\n";
		o << "\t\t{ u64 i0 = row0 / m; u64 j0 = row0 - i0 * m;\n";
		o << "\t\t#pragma unroll\n\t\tfor (int r = 0; r < " << g.items
		  << "; ++r) { li[r] = i0; rj[r] = j0; if (++j0 == m) { j0 = 0; ++i0; } } }\n";
	}
	for (size_t i = 0; i < spec_.sources.size(); i++) {
		if (!needed[i]) {
			continue;
		}
		const auto &src = spec_.sources[i];
		const char *t = CudaTypeName(src.type);
		const int w = 2 + 2 * static_cast<int>(i);
		o << "\t\t" << t << " s" << i << "[" << g.items << "];\n";
		if (src.nullable) {
			o << "\t\tbool sv" << i << "[" << g.items << "];\n";
		}
		if (spec_.join) {
			// left columns at the left rows; right columns come from the lookup below
			if (src.side == 0) {
				o << "\t\tload_rows<" << t << ", " << g.items << ">((const " << t << "*)a.w[" << w << "], row0, n, s" << i
				  << ");\n";
				if (src.nullable) {
					o << "\t\tload_valid<" << g.items << ">((const u8*)a.w[" << w + 1 << "], row0, n, sv" << i << ");\n";
				}
			}
		} else if (!spec_.cross) {
			o << "\t\tload_rows<" << t << ", " << g.items << ">((const " << t << "*)a.w[" << w << "], row0, n, s" << i
			  << ");\n";
			if (src.nullable) {
				o << "\t\tload_valid<" << g.items << ">((const u8*)a.w[" << w + 1 << "], row0, n, sv" << i << ");\n";
			}
		} else {
			const char *idx = src.side == 0 ? "li[r]" : "rj[r]";
			o << "\t\t#pragma unroll\n\t\tfor (int r = 0; r < " << g.items << "; ++r) {\n";
			o << "\t\t\ts" << i << "[r] = (row0 + r < n) ? ((const " << t << "*)a.w[" << w << "])[" << idx << "] : ("
			  << t << ")0;\n";
			if (src.nullable) {
				o << "\t\t\tsv" << i << "[r] = (row0 + r < n) ? (((const u8*)a.w[" << w + 1 << "])[" << idx
				  << "] != 0) : false;\n";
			}
			o << "\t\t}\n";
		}
	}
	if (spec_.join) {
		// each item's match in the sorted right side, then the right columns at that position
		const int key = spec_.join_key;
		// keys widen by zero extension of their width, as the sorted side was widened
		const size_t kw = TypeSize(spec_.sources[key].type);
		const char *ut = kw == 1 ? "u8" : kw == 2 ? "unsigned short" : kw == 4 ? "u32" : "u64";
		if (spec_.join_minline) {
			// the key's entry in the dense multi-match inline table: match count and one value slot per match
			o << "\t\tlong long jm[" << g.items << "];\n\t\tu32 jc[" << g.items << "];\n\t\tu64 je[" << g.items << "];\n"
			  << "\t\t#pragma unroll\n\t\tfor (int r = 0; r < " << g.items << "; ++r) {\n"
			  << "\t\t\tu32 c_ = 0u;\n"
			  << "\t\t\tje[r] = row0 + r < n ? vgpu_join_minline((u64)(" << ut << ")s" << key << "[r] - a.w[" << kJoinWord + 2
			  << "], (const void*)a.w[" << kJoinWord << "], a.w[" << kJoinWord + 3 << "] >> 8, (u32)(a.w[" << kJoinWord + 3
			  << "] & 0xffu), &c_) : 0ull;\n"
			  << "\t\t\tjc[r] = c_;\n\t\t\tjm[r] = c_ ? 0ll : -1ll;\n\t\t}\n";
			return o.str();
		}
		if (spec_.join_multi) {
			// the run of equal keys: start and length (0 = no match); the right columns are read per match
			o << "\t\tlong long jm[" << g.items << "];\n\t\tu32 jc[" << g.items << "];\n"
			  << "\t\t#pragma unroll\n\t\tfor (int r = 0; r < " << g.items << "; ++r) {\n"
			  << "\t\t\tu32 c_ = 0u;\n"
			  << "\t\t\tjm[r] = row0 + r < n ? vgpu_join_run((u64)(" << ut << ")s" << key << "[r] - a.w[" << kJoinWord + 2
			  << "], (const u64*)a.w[" << kJoinWord << "], (const u32*)a.w[" << kJoinWord + 1 << "], a.w[" << kJoinWord + 3
			  << "] >> 8, (u32)(a.w[" << kJoinWord + 3 << "] & 0xffu), &c_) : -1ll;\n"
			  << "\t\t\tjc[r] = c_;\n\t\t}\n";
			return o.str();
		}
		o << "\t\tlong long jm[" << g.items << "];\n"
		  << "\t\t#pragma unroll\n\t\tfor (int r = 0; r < " << g.items << "; ++r) {\n"
		  << "\t\t\tjm[r] = row0 + r < n ? vgpu_join_find((u64)(" << ut << ")s" << key << "[r] - a.w[" << kJoinWord + 2
		  << "], (const u64*)a.w[" << kJoinWord << "], a.w[" << kJoinWord + 1 << "], a.w[" << kJoinWord + 3
		  << "] >> 8, (u32)(a.w[" << kJoinWord + 3 << "] & 0xffu)) : -1ll;\n\t\t}\n";
		for (size_t i = 0; i < spec_.sources.size(); i++) {
			const auto &src = spec_.sources[i];
			if (!needed[i] || src.side != 1) continue;
			const char *t = CudaTypeName(src.type);
			const int w = 2 + 2 * static_cast<int>(i);
			if (spec_.join_inline) {
				o << "\t\t#pragma unroll\n\t\tfor (int r = 0; r < " << g.items << "; ++r) s" << i << "[r] = jm[r] >= 0 ? from_bits<"
				  << t << ">((u64)(u32)jm[r]) : (" << t << ")0;\n";
				continue;
			}
			o << "\t\t#pragma unroll\n\t\tfor (int r = 0; r < " << g.items << "; ++r) s" << i << "[r] = jm[r] >= 0 ? ((const "
			  << t << "*)a.w[" << w << "])[jm[r]] : (" << t << ")0;\n";
			if (src.nullable) {
				o << "\t\t#pragma unroll\n\t\tfor (int r = 0; r < " << g.items << "; ++r) sv" << i
				  << "[r] = jm[r] >= 0 ? (((const u8*)a.w[" << w + 1 << "])[jm[r]] != 0) : false;\n";
			}
		}
	}
	return o.str();
}

std::string PipelineCodegen::ItemOpen(const Geometry &g, const std::vector<bool> &needed) const {
	std::ostringstream o;
	o << "\t\t#pragma unroll\n\t\tfor (int r = 0; r < " << g.items << "; ++r) {\n\t\tconst u64 row = row0 + r; (void)row;\n";
	if (!spec_.join_multi) {
		o << "\t\tbool keep = row < n;\n";
		return o.str();
	}
	// one item per match of the row's key, right columns read at the match's sorted position
	o << "\t\tconst u32 jn_ = (row < n && jm[r] >= 0) ? jc[r] : 0u;\n"
	  << "\t\tfor (u32 jx_ = 0; jx_ < jn_; ++jx_) {\n"
	  << "\t\tconst u64 jp_ = (u64)jm[r] + jx_; (void)jp_;\n";
	for (size_t i = 0; i < spec_.sources.size(); i++) {
		const auto &src = spec_.sources[i];
		if (!needed[i] || src.side != 1) continue;
		const char *t = CudaTypeName(src.type);
		if (spec_.join_minline) {  // the (single) right column from the match's slot of the entry
			o << "\t\ts" << i << "[r] = from_bits<" << t << ">((u64)vgpu_join_minline_value(je[r], jx_, (u32)(a.w["
			  << kJoinWord + 3 << "] & 0xffu), (u32)a.w[" << kJoinWord + 1 << "]));\n";
			continue;
		}
		const int w = 2 + 2 * static_cast<int>(i);
		o << "\t\ts" << i << "[r] = ((const " << t << "*)a.w[" << w << "])[jp_];\n";
		if (src.nullable) o << "\t\tsv" << i << "[r] = ((const u8*)a.w[" << w + 1 << "])[jp_] != 0;\n";
	}
	o << "\t\tbool keep = true;\n";
	return o.str();
}

std::string PipelineCodegen::ItemClose() const {
	return spec_.join_multi ? "\t\t}\n\t\t}\n" : "\t\t}\n";
}

namespace {

// KArgs word carrying the optional bucket diagnostics buffer (0 = off).
constexpr int kDebugWord = 127;

const char *kKernelHead = "\tconst u64 n = a.w[0];\n\tconst u64 m = a.w[1];\n\t(void)m;\n";

} // namespace

std::string PipelineCodegen::EmitMaterialize(const std::vector<int> &outs, const Geometry &g) const {
	std::ostringstream o;
	o << Prologue();
	const int cb = ConsumerBase();
	std::vector<int> out_cols = outs;
	auto needed = NeededSources(out_cols);
	const std::string loads = LoadBlock(g, needed, false);
	// tile counts and offsets: 32-bit, or 64-bit when a multi-match join source can expand past 2^32 rows
	const char *cnt_t = spec_.join_multi ? "u64" : "u32";
	if (has_filter_) {
		const auto count_needed = NeededSources({});
		o << "extern \"C\" __global__ void __launch_bounds__(" << g.block << ") vgpu_mat_count(KArgs a) {\n"
		  << kKernelHead << "\t__shared__ u32 scan_scratch[33];\n"
		  << "\t" << cnt_t << " *tile_counts = (" << cnt_t << "*)a.w[" << cb << "];\n"
		  << "\tconst u64 ntiles = (n + " << g.tile() - 1 << ") / " << g.tile() << ";\n"
		  << "\tfor (u64 tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {\n"
		  << LoadBlock(g, count_needed, false) << "\t\tu32 cnt = 0;\n"
		  << ItemOpen(g, count_needed) << chain_code_ << "\t\tcnt += keep ? 1u : 0u;\n" << ItemClose()
		  << "\t\tu32 total; block_exclusive_scan(cnt, scan_scratch, &total);\n"
		  << "\t\tif (threadIdx.x == 0) tile_counts[tile] = total;\n\t}\n}\n\n";
	}
	o << "extern \"C\" __global__ void __launch_bounds__(" << g.block << ") vgpu_mat_write(KArgs a) {\n"
	  << kKernelHead << "\t__shared__ u32 scan_scratch[33];\n"
	  << "\tconst " << cnt_t << " *tile_offsets = (const " << cnt_t << "*)a.w[" << cb << "]; (void)tile_offsets;\n"
	  << "\tconst u64 ntiles = (n + " << g.tile() - 1 << ") / " << g.tile() << ";\n"
	  << "\tfor (u64 tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {\n"
	  << loads;
	if (spec_.join_multi) {
		// a row's matches are not bounded: count this thread's outputs, then evaluate again and write
		o << "\t\tu32 cnt = 0;\n" << ItemOpen(g, needed) << chain_code_ << "\t\tcnt += keep ? 1u : 0u;\n" << ItemClose()
		  << "\t\tu32 total; u64 pos = (u64)block_exclusive_scan(cnt, scan_scratch, &total) + tile_offsets[tile];\n"
		  << ItemOpen(g, needed) << chain_code_ << "\t\tif (keep) {\n";
		for (size_t c = 0; c < out_cols.size(); c++) {
			const auto &col = visible_[out_cols[c]];
			int w = cb + 1 + 2 * static_cast<int>(c);
			o << "\t\t\t((" << CudaTypeName(col.type) << "*)a.w[" << w << "])[pos] = " << col.value << ";\n";
			if (col.nullable) {
				o << "\t\t\tif (a.w[" << w + 1 << "]) ((u8*)a.w[" << w + 1 << "])[pos] = (" << col.valid << ") ? 1 : 0;\n";
			}
		}
		o << "\t\t\t++pos;\n\t\t}\n" << ItemClose() << "\t}\n}\n";
		return o.str();
	}
	o << "\t\tbool kv[" << g.items << "];\n";
	for (size_t c = 0; c < out_cols.size(); c++) {
		const auto &col = visible_[out_cols[c]];
		o << "\t\t" << CudaTypeName(col.type) << " o" << c << "[" << g.items << "];\n";
		if (col.nullable) {
			o << "\t\tbool ov" << c << "[" << g.items << "];\n";
		}
	}
	o << "\t\tu32 cnt = 0;\n" << ItemOpen(g, needed) << chain_code_ << "\t\tkv[r] = keep;\n\t\tcnt += keep ? 1u : 0u;\n";
	for (size_t c = 0; c < out_cols.size(); c++) {
		const auto &col = visible_[out_cols[c]];
		o << "\t\to" << c << "[r] = " << col.value << ";\n";
		if (col.nullable) {
			o << "\t\tov" << c << "[r] = " << col.valid << ";\n";
		}
	}
	o << ItemClose();
	// A filtered tile's kept rows are contiguous in the output: they are placed in shared memory by
	// rank, then written out as one coalesced run per column (the per-thread stores would leave each
	// warp's sectors partly written by several instructions). Only while the staging fits 32 KB, and
	// not over a cross product, whose predicate keeps few of the pairs it computes: there the extra
	// barrier costs more than the sparse stores (4096 x 4096 pairs keeping 1 in 13: 0.046 -> 0.050 ms
	// staged; a filter + projection of 2^24 rows keeping 43%: 0.116 -> 0.103 ms).
	uint64_t stage_bytes = 0;
	for (int c : out_cols) {
		const auto &col = visible_[c];
		stage_bytes += static_cast<uint64_t>(g.tile()) * (TypeSize(col.type) + (col.nullable ? 1 : 0));
	}
	if (has_filter_ && !spec_.cross && stage_bytes <= 32 * 1024) {
		for (size_t c = 0; c < out_cols.size(); c++) {
			const auto &col = visible_[out_cols[c]];
			o << "\t\t__shared__ __align__(16) " << CudaTypeName(col.type) << " vgpu_st" << c << "[" << g.tile() << "];\n";
			if (col.nullable) o << "\t\t__shared__ u8 vgpu_sv" << c << "[" << g.tile() << "];\n";
		}
		o << "\t\tu32 total; u32 rank = block_exclusive_scan(cnt, scan_scratch, &total);\n"
		  << "\t\t#pragma unroll\n\t\tfor (int r = 0; r < " << g.items << "; ++r) {\n\t\t\tif (kv[r]) {\n";
		for (size_t c = 0; c < out_cols.size(); c++) {
			o << "\t\t\t\tvgpu_st" << c << "[rank] = o" << c << "[r];\n";
			if (visible_[out_cols[c]].nullable) o << "\t\t\t\tvgpu_sv" << c << "[rank] = ov" << c << "[r] ? 1 : 0;\n";
		}
		o << "\t\t\t\t++rank;\n\t\t\t}\n\t\t}\n\t\t__syncthreads();\n"
		  << "\t\tconst u64 base = tile_offsets[tile];\n"
		  << "\t\tfor (u32 i = threadIdx.x; i < total; i += " << g.block << ") {\n";
		for (size_t c = 0; c < out_cols.size(); c++) {
			const auto &col = visible_[out_cols[c]];
			int w = cb + 1 + 2 * static_cast<int>(c);
			o << "\t\t\t((" << CudaTypeName(col.type) << "*)a.w[" << w << "])[base + i] = vgpu_st" << c << "[i];\n";
			if (col.nullable) {
				o << "\t\t\tif (a.w[" << w + 1 << "]) ((u8*)a.w[" << w + 1 << "])[base + i] = vgpu_sv" << c << "[i];\n";
			}
		}
		o << "\t\t}\n\t\t__syncthreads();  // the next tile reuses the staging\n\t}\n}\n";
		return o.str();
	}
	if (has_filter_) {
		o << "\t\tu32 total; u32 pos = block_exclusive_scan(cnt, scan_scratch, &total) + tile_offsets[tile];\n";
	} else {
		o << "\t\tu64 pos = row0;\n";
	}
	o << "\t\t#pragma unroll\n\t\tfor (int r = 0; r < " << g.items << "; ++r) {\n\t\t\tif (kv[r]) {\n";
	for (size_t c = 0; c < out_cols.size(); c++) {
		const auto &col = visible_[out_cols[c]];
		int w = cb + 1 + 2 * static_cast<int>(c);
		o << "\t\t\t\t((" << CudaTypeName(col.type) << "*)a.w[" << w << "])[pos] = o" << c << "[r];\n";
		if (col.nullable) {
			o << "\t\t\t\tif (a.w[" << w + 1 << "]) ((u8*)a.w[" << w + 1 << "])[pos] = ov" << c << "[r] ? 1 : 0;\n";
		}
	}
	if (has_filter_) {
		o << "\t\t\t\t++pos;\n\t\t\t}\n";
	} else {
		o << "\t\t\t}\n\t\t\t++pos;\n";
	}
	o << "\t\t}\n\t}\n}\n";
	return o.str();
}

std::string PipelineCodegen::EmitStats(const std::vector<int> &columns, const Geometry &g) const {
	std::ostringstream o;
	o << Prologue();
	const int cb = ConsumerBase();
	auto needed = NeededSources(columns);
	// Predicates are not applied: the bound must hold for every row the consumer could see, and a
	// superset bound is still a valid one.
	std::vector<bool> load_needed(spec_.sources.size(), false);
	for (int c : columns) {
		for (int s : chain_uses_[c]) {
			load_needed[s] = true;
		}
	}
	// The chain code may reference any source the chain touches; load those too.
	for (size_t i = 0; i < load_needed.size(); i++) {
		load_needed[i] = load_needed[i] || needed[i];
	}
	o << "extern \"C\" __global__ void __launch_bounds__(" << g.block << ") vgpu_stats(KArgs a) {\n" << kKernelHead;
	for (size_t c = 0; c < columns.size(); c++) {
		o << "\ti64 mn" << c << " = 0x7fffffffffffffffLL, mx" << c << " = (-0x7fffffffffffffffLL - 1);\n";
	}
	o << "\tconst u64 ntiles = (n + " << g.tile() - 1 << ") / " << g.tile() << ";\n"
	  << "\tfor (u64 tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {\n"
	  << LoadBlock(g, load_needed, false) << ItemOpen(g, load_needed) << chain_code_ << "\t\tif (row < n) {\n";
	for (size_t c = 0; c < columns.size(); c++) {
		const auto &col = visible_[columns[c]];
		o << "\t\t\t{ const i64 x = (i64)(" << col.value << "); mn" << c << " = x < mn" << c << " ? x : mn" << c
		  << "; mx" << c << " = x > mx" << c << " ? x : mx" << c << "; }\n";
	}
	o << "\t\t}\n" << ItemClose() << "\t}\n";
	for (size_t c = 0; c < columns.size(); c++) {
		o << "\tfor (int off = 16; off > 0; off >>= 1) {\n"
		  << "\t\ti64 a1 = __shfl_xor_sync(0xffffffffu, mn" << c << ", off); mn" << c << " = a1 < mn" << c << " ? a1 : mn"
		  << c << ";\n"
		  << "\t\ti64 b1 = __shfl_xor_sync(0xffffffffu, mx" << c << ", off); mx" << c << " = b1 > mx" << c << " ? b1 : mx"
		  << c << ";\n\t}\n"
		  << "\tif ((threadIdx.x & 31) == 0) { atomic_min_i64((i64*)a.w[" << cb + 2 * c << "], mn" << c
		  << "); atomic_max_i64((i64*)a.w[" << cb + 2 * c + 1 << "], mx" << c << "); }\n";
	}
	o << "}\n";
	return o.str();
}

// ---------------------------------------------------------------------------------------------
// Group-by

namespace {

struct Field {
	std::string kind; // "cnt", "f64", "lo", "hi", "min", "max"
	int agg = -1;
	// One-pass group-by, MIN/MAX in shared memory: >= 0 keeps the value as a 32-bit offset from the
	// minimum in argument word `narrow_word` (the low word of the slot, updated by native 32-bit atomics).
	int narrow_word = -1;
};

std::vector<Field> StateFields(const PipelineCodegen::GroupBySpec &gb) {
	std::vector<Field> f;
	f.push_back({"cnt", -1});
	for (size_t i = 0; i < gb.aggs.size(); i++) {
		auto &a = gb.aggs[i];
		int ai = static_cast<int>(i);
		switch (a.kind) {
		case AggKind::COUNT_STAR:
		case AggKind::COUNT:
			break;
		case AggKind::SUM:
		case AggKind::AVG:
			if (IsFloatType(a.input_type)) {
				f.push_back({"f64", ai});
			} else {
				f.push_back({"lo", ai});
				f.push_back({"hi", ai});
			}
			break;
		case AggKind::MIN:
			f.push_back({"min", ai});
			break;
		case AggKind::MAX:
			f.push_back({"max", ai});
			break;
		}
	}
	return f;
}

int FieldIndex(const std::vector<Field> &fields, const std::string &kind, int agg) {
	for (size_t i = 0; i < fields.size(); i++) {
		if (fields[i].kind == kind && fields[i].agg == agg) {
			return static_cast<int>(i);
		}
	}
	return -1;
}

std::string InitValue(const Field &f) {
	if (f.narrow_word >= 0) {
		return f.kind == "min" ? "0xffffffffull" : "0ull";
	}
	if (f.kind == "min") {
		return "0x7fffffffffffffffull";
	}
	if (f.kind == "max") {
		return "0x8000000000000000ull";
	}
	return "0ull"; // cnt, f64 (+0.0 bit pattern), lo, hi
}

// Update of table T (u64 arrays T_f at slot S) with the value expression `v` of aggregate field f.
// `shared`: the table is in shared memory, where a count moves as a 32-bit atomic on its low word with
// an explicit carry into the high word (cheaper there than a 64-bit atomic, and exact).
// `narrow_count`: fewer than 2^32 rows reach the table, so the low word never carries and the count
// is a plain 32-bit add whose result nothing waits for.
std::string UpdateCode(const std::vector<Field> &fields, const std::string &tab, const std::string &slot,
                       const std::vector<std::string> &agg_values, bool shared, bool narrow_count = false,
                       bool count_as_flag = false) {
	std::ostringstream o;
	for (size_t i = 0; i < fields.size(); i++) {
		auto &f = fields[i];
		std::string p = tab + std::to_string(i) + " + " + slot;
		if ((f.kind == "min" || f.kind == "max") && shared && f.narrow_word >= 0) {
			o << "\t\t\tatomic" << (f.kind == "min" ? "Min" : "Max") << "((u32*)(" << p << "), (u32)((i64)("
			  << agg_values[f.agg] << ") - (i64)a.w[" << f.narrow_word << "]));\n";
		} else if (f.kind == "cnt" && shared && count_as_flag) {
			o << "\t\t\t*(u32*)(" << p << ") = 1u;\n";
		} else if (f.kind == "cnt" && shared && narrow_count) {
			o << "\t\t\tatomicAdd((u32*)(" << p << "), 1u);\n";
		} else if (f.kind == "cnt" && shared) {
			o << "\t\t\t{ u32 *w_ = (u32*)(" << p << "); if (atomicAdd(w_, 1u) == 0xffffffffu) atomicAdd(w_ + 1, 1u); }\n";
		} else if (f.kind == "cnt") {
			o << "\t\t\tatomicAdd(" << p << ", 1ull);\n";
		} else if (f.kind == "f64") {
			o << "\t\t\tatomicAdd((double*)(" << p << "), (double)(" << agg_values[f.agg] << "));\n";
		} else if (f.kind == "lo") {
			std::string phi = tab + std::to_string(i + 1) + " + " + slot;
			o << "\t\t\tatomic_add_i128(" << p << ", (i64*)(" << phi << "), (i64)(" << agg_values[f.agg] << "));\n";
		} else if (f.kind == "min") {
			o << "\t\t\tatomic_min_i64((i64*)(" << p << "), (i64)(" << agg_values[f.agg] << "));\n";
		} else if (f.kind == "max") {
			o << "\t\t\tatomic_max_i64((i64*)(" << p << "), (i64)(" << agg_values[f.agg] << "));\n";
		}
	}
	return o.str();
}

// Merge of source table slot into destination table slot (both u64 field arrays).
// `l2_src`: FP64 sum fields of the source live in global memory updated by reductions; they are read
// through L2 (__ldcg), past any line this SM's L1 might hold.
std::string MergeCode(const std::vector<Field> &fields, const std::string &src, const std::string &ss,
                      const std::string &dst, const std::string &ds, bool l2_src = false) {
	std::ostringstream o;
	for (size_t i = 0; i < fields.size(); i++) {
		auto &f = fields[i];
		std::string ps = src + std::to_string(i) + "[" + ss + "]";
		if (l2_src && f.kind == "f64") ps = "__ldcg(&" + ps + ")";
		std::string pd = dst + std::to_string(i) + " + " + ds;
		if (f.kind == "cnt") {
			o << "\t\t\tatomicAdd(" << pd << ", " << ps << ");\n";
		} else if (f.kind == "f64") {
			o << "\t\t\tatomicAdd((double*)(" << pd << "), __longlong_as_double((i64)" << ps << "));\n";
		} else if (f.kind == "lo") {
			std::string ps_hi = src + std::to_string(i + 1) + "[" + ss + "]";
			std::string pd_hi = dst + std::to_string(i + 1) + " + " + ds;
			o << "\t\t\tatomic_add_i128_pair(" << pd << ", (i64*)(" << pd_hi << "), " << ps << ", (i64)" << ps_hi
			  << ");\n";
		} else if (f.kind == "min" || f.kind == "max") {
			const std::string v = f.narrow_word >= 0
			                          ? "(i64)(u32)" + ps + " + (i64)a.w[" + std::to_string(f.narrow_word) + "]"
			                          : "(i64)" + ps;
			o << "\t\t\tatomic_" << f.kind << "_i64((i64*)(" << pd << "), " << v << ");\n";
		}
	}
	return o.str();
}

// Writes the finalized outputs of one group from table T slot `s` to output row `pos`.
// Outputs start at word `out_base`: keys first, then aggregates (HUGEINT outputs are 16 bytes/row).
std::string FinalizeCode(const PipelineCodegen::GroupBySpec &gb, const std::vector<Field> &fields,
                         const std::vector<PipeColumn> &visible, const std::string &tab, const std::string &s,
                         const std::string &key, const std::string &pos, int out_base,
                         const std::string &out_array = "a.w") {
	std::ostringstream o;
	int w = out_base;
	for (auto &k : gb.keys) {
		const auto &col = visible[k.column];
		const char *t = CudaTypeName(col.type);
		const int j = static_cast<int>(&k - gb.keys.data());
		o << "\t\t\t((" << t << "*)" << out_array << "[" << w << "])[" << pos << "] = (" << t << ")((i64)((" << key
		  << " >> (u32)a.w[" << kKeyWord + 3 * j + 1 << "]) & a.w[" << kKeyWord + 3 * j + 2 << "]) + (i64)a.w["
		  << kKeyWord + 3 * j << "]);\n";
		w++;
	}
	const std::string cnt = tab + "0[" + s + "]";
	for (size_t i = 0; i < gb.aggs.size(); i++) {
		auto &a = gb.aggs[i];
		int ai = static_cast<int>(i);
		std::string out = out_array + "[" + std::to_string(w) + "]";
		switch (a.kind) {
		case AggKind::COUNT_STAR:
		case AggKind::COUNT:
			o << "\t\t\t((i64*)" << out << ")[" << pos << "] = (i64)" << cnt << ";\n";
			break;
		case AggKind::SUM:
		case AggKind::AVG: {
			bool avg = a.kind == AggKind::AVG;
			if (IsFloatType(a.input_type)) {
				int f = FieldIndex(fields, "f64", ai);
				std::string sum = "__longlong_as_double((i64)" + tab + std::to_string(f) + "[" + s + "])";
				if (avg) {
					o << "\t\t\t((double*)" << out << ")[" << pos << "] = " << sum << " / (double)" << cnt << ";\n";
				} else {
					o << "\t\t\t((double*)" << out << ")[" << pos << "] = " << sum << ";\n";
				}
			} else {
				int f = FieldIndex(fields, "lo", ai);
				std::string lo = tab + std::to_string(f) + "[" + s + "]";
				std::string hi = "(i64)" + tab + std::to_string(f + 1) + "[" + s + "]";
				if (avg) {
					o << "\t\t\t((double*)" << out << ")[" << pos << "] = i128_to_double(" << lo << ", " << hi
					  << ") / (double)" << cnt << ";\n";
				} else if (a.output_type == ValueType::HUGEINT) {
					o << "\t\t\t((u64*)" << out << ")[2 * (" << pos << ")] = " << lo << ";\n";
					o << "\t\t\t((u64*)" << out << ")[2 * (" << pos << ") + 1] = (u64)" << hi << ";\n";
				} else {
					o << "\t\t\t((double*)" << out << ")[" << pos << "] = i128_to_double(" << lo << ", " << hi << ");\n";
				}
			}
			break;
		}
		case AggKind::MIN:
		case AggKind::MAX: {
			int f = FieldIndex(fields, a.kind == AggKind::MIN ? "min" : "max", ai);
			const char *t = CudaTypeName(a.output_type);
			o << "\t\t\t((" << t << "*)" << out << ")[" << pos << "] = (" << t << ")(i64)" << tab << f << "[" << s << "];\n";
			break;
		}
		}
		w++;
	}
	return o.str();
}

} // namespace

int PipelineCodegen::StateWords(const GroupBySpec &gb) {
	return static_cast<int>(StateFields(gb).size());
}

int PipelineCodegen::DirectSlotBytes(const GroupBySpec &gb) {
	int bytes = 0;
	for (auto &f : StateFields(gb)) {
		if (f.kind == "cnt") bytes += 4;
		if ((f.kind == "f64" && !gb.f64_l2) || f.kind == "min" || f.kind == "max") bytes += 8;
		if (f.kind == "lo") bytes += 16;
	}
	return bytes;
}

uint64_t PipelineCodegen::DirectSmemBytes(const GroupBySpec &gb, uint64_t domain) {
	const int F = static_cast<int>(StateFields(gb).size());
	const int shared64 = F - 1 - (gb.f64_l2 ? F64Fields(gb) : 0);
	const bool c32 = gb.count32 && (gb.narrow_count || gb.count_as_flag);
	return domain * (static_cast<uint64_t>(shared64) * 8 + (c32 ? 4 : 8));
}

int PipelineCodegen::F64Fields(const GroupBySpec &gb) {
	int n = 0;
	for (auto &f : StateFields(gb)) n += f.kind == "f64" ? 1 : 0;
	return n;
}

int PipelineCodegen::HeavySlotBytes(const GroupBySpec &gb) {
	int bytes = 4;
	for (auto &a : gb.aggs) {
		if (a.column < 0 || a.kind == AggKind::COUNT || a.kind == AggKind::COUNT_STAR) continue;
		const bool int_sum = (a.kind == AggKind::SUM || a.kind == AggKind::AVG) && !IsFloatType(a.input_type);
		bytes += int_sum ? 16 : 8;
	}
	return bytes;
}

int PipelineCodegen::StageRowBytes(const GroupBySpec &gb, bool scatter) const {
	std::vector<int> used;
	for (auto &k : gb.keys) used.push_back(k.column);
	if (scatter) {
		for (auto &a : gb.aggs) {
			if (a.column >= 0) used.push_back(a.column);
		}
	}
	const auto needed = NeededSources(used);
	int bytes = 0;
	for (size_t i = 0; i < spec_.sources.size(); i++) {
		if (needed[i]) bytes += static_cast<int>(TypeSize(spec_.sources[i].type));
	}
	return bytes;
}

int PipelineCodegen::RecordStride(const GroupBySpec &gb) const {
	// Same layout rule as EmitGroupBy: key u64, then each distinct carried value column at its
	// natural alignment, rounded up to 32 bytes.
	std::vector<int> value_cols;
	for (auto &a : gb.aggs) {
		if (a.column >= 0 && (a.kind != AggKind::COUNT && a.kind != AggKind::COUNT_STAR) &&
		    std::find(value_cols.begin(), value_cols.end(), a.column) == value_cols.end()) {
			value_cols.push_back(a.column);
		}
	}
	int off = 8;
	for (int c : value_cols) {
		const int w = static_cast<int>(TypeSize(visible_[c].type));
		off = (off + w - 1) / w * w + w;
	}
	return (off + 31) / 32 * 32;
}

std::string PipelineCodegen::EmitGroupBy(const GroupBySpec &gb, bool partitioned, const Geometry &g) const {
	std::ostringstream o;
	o << Prologue();
	const int cb = ConsumerBase();
	const auto fields = StateFields(gb);
	const int F = static_cast<int>(fields.size());
	// Columns the consumer reads: keys and aggregate inputs.
	std::vector<int> used;
	for (auto &k : gb.keys) {
		used.push_back(k.column);
	}
	for (auto &a : gb.aggs) {
		if (a.column >= 0) {
			used.push_back(a.column);
		}
	}
	auto needed = NeededSources(used);
	// Distinct aggregate input columns (the values a partitioned scatter carries).
	std::vector<int> value_cols;
	for (auto &a : gb.aggs) {
		if (a.column >= 0 && (a.kind != AggKind::COUNT && a.kind != AggKind::COUNT_STAR) &&
		    std::find(value_cols.begin(), value_cols.end(), a.column) == value_cols.end()) {
			value_cols.push_back(a.column);
		}
	}
	std::ostringstream pack;
	pack << "(0ull";
	for (auto &k : gb.keys) {
		const int j = static_cast<int>(&k - gb.keys.data());
		pack << " | ((u64)((i64)(" << visible_[k.column].value << ") - (i64)a.w[" << kKeyWord + 3 * j << "]) << (u32)a.w["
		     << kKeyWord + 3 * j + 1 << "])";
	}
	pack << ")";
	auto value_of = [&](int agg_index, bool from_partition) -> std::string {
		const auto &a = gb.aggs[agg_index];
		if (a.column < 0) {
			return "0";
		}
		if (!from_partition) {
			return visible_[a.column].value;
		}
		int vi = static_cast<int>(std::find(value_cols.begin(), value_cols.end(), a.column) - value_cols.begin());
		return "((const " + std::string(CudaTypeName(visible_[a.column].type)) + "*)vin" + std::to_string(vi) + ")[i]";
	};
	std::vector<std::string> pipe_values, part_values;
	for (size_t i = 0; i < gb.aggs.size(); i++) {
		pipe_values.push_back(value_of(static_cast<int>(i), false));
		part_values.push_back(value_of(static_cast<int>(i), true));
	}
	const std::string tile_loop_head = "\tconst u64 ntiles = (n + " + std::to_string(g.tile() - 1) + ") / " +
	                                   std::to_string(g.tile()) + ";\n";
	const std::string item_head = "\t\t#pragma unroll\n\t\tfor (int r = 0; r < " + std::to_string(g.items) +
	                              "; ++r) {\n\t\tconst u64 row = row0 + r; (void)row;\n\t\tbool keep = row < n;\n";
	const int out_words = static_cast<int>(gb.keys.size() + gb.aggs.size());

	if (!partitioned) {
		// ---- direct: packed key is the slot of a dense table of `domain` groups ----
		// args: cb+0 = D, cb+1+f = global field arrays, then (final) outputs, then count ptr.
		const bool fused = DirectFinalFused(gb);
		const int ticket = cb + 3 + F + out_words;
		// the shared tables' view of the fields: MIN/MAX the executor narrowed to 32-bit offsets
		std::vector<Field> dfields = fields;
		for (auto &f : dfields) {
			if (f.kind == "min" || f.kind == "max") f.narrow_word = gb.aggs[f.agg].narrow_word;
		}
		o << "extern \"C\" __global__ void vgpu_gb_direct_init(KArgs a) {\n"
		  << "\tconst u64 D = a.w[" << cb << "];\n";
		if (fused) o << "\tif (blockIdx.x == 0 && threadIdx.x == 0) *(u32*)a.w[" << ticket << "] = 0u;\n";
		o << "\tfor (u64 s = blockIdx.x * (u64)blockDim.x + threadIdx.x; s < D; s += (u64)gridDim.x * blockDim.x) {\n";
		for (int f = 0; f < F; f++) {
			o << "\t\t((u64*)a.w[" << cb + 1 + f << "])[s] = " << InitValue(fields[f]) << ";\n";
		}
		o << "\t}\n}\n\n";
		// With f64_l2 the FP64 sums leave shared memory (where an FP64 atomic add is a compare-and-swap
		// loop) for this CTA's own region of a global array (arg cb+2+F+out_words), updated by native L2
		// reductions; the region stays L2-resident (D * 8 bytes per sum and CTA).
		const bool l2 = gb.f64_l2;
		const int nl2 = l2 ? F64Fields(gb) : 0;
		o << "extern \"C\" __global__ void __launch_bounds__(" << g.block << ") vgpu_gb_direct(KArgs a) {\n"
		  << kKernelHead << "\textern __shared__ __align__(16) u64 vgpu_smem[];\n"
		  << "\tconst u64 D = a.w[" << cb << "];\n";
		// A count that never carries (fewer than 2^32 rows) or only marks presence needs 32 bits: with
		// count32 its array goes after the 64-bit ones, in 4 bytes per slot (DirectSmemBytes sizes the
		// launch alike).
		const bool c32 = gb.count32 && (gb.narrow_count || gb.count_as_flag);
		int sh = 0;
		for (int f = 0, gl = 0; f < F; f++) {
			if (l2 && fields[f].kind == "f64") {
				o << "\tu64 *T" << f << " = (u64*)a.w[" << cb + 2 + F + out_words << "] + ((u64)blockIdx.x * " << nl2
				  << " + " << gl++ << ") * D;\n";
			} else if (!(c32 && f == 0)) {
				o << "\tu64 *T" << f << " = vgpu_smem + " << sh++ << " * D;\n";
			}
		}
		if (c32) o << "\tu32 *T0 = (u32*)(vgpu_smem + " << sh << " * D);\n";
		o << "\tfor (u64 s = threadIdx.x; s < D; s += " << g.block << ") {\n";
		for (int f = 0; f < F; f++) {
			o << "\t\tT" << f << "[s] = " << InitValue(dfields[f]) << ";\n";
		}
		o << "\t}\n\t__syncthreads();\n" << tile_loop_head
		  << "\tfor (u64 tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {\n"
		  << LoadBlock(g, needed, false) << ItemOpen(g, needed) << chain_code_ << "\t\tif (keep) {\n"
		  << "\t\t\tconst u64 slot = " << pack.str() << ";\n"
		  << UpdateCode(dfields, "T", "slot", pipe_values, true, gb.narrow_count, gb.count_as_flag) << "\t\t}\n" << ItemClose()
		  << "\t}\n"
		  << (l2 ? "\t__threadfence();  // this thread's reductions are performed before the sums are read\n" : "")
		  << "\t__syncthreads();\n";
		for (int f = 0; f < F; f++) {
			o << "\tu64 *G" << f << " = (u64*)a.w[" << cb + 1 + f << "];\n";
		}
		o << "\tfor (u64 s = threadIdx.x; s < D; s += " << g.block << ") {\n\t\tif (T0[s] != 0) {\n"
		  << MergeCode(dfields, "T", "s", "G", "s", l2) << "\t\t}\n\t}\n";
		// final: one CTA compacts the non-empty groups in key order. Fused, it is the CTA whose merge
		// finished last: every thread fences its merge atomics before the CTA takes a ticket, and the
		// last CTA fences again before reading the global tables (which no CTA has loaded through L1:
		// the merges are atomics).
		if (fused) {
			o << "\t__threadfence();\n\t__syncthreads();\n\t__shared__ u32 vgpu_last;\n"
			  << "\tif (threadIdx.x == 0) vgpu_last = atomicAdd((u32*)a.w[" << ticket
			  << "], 1u) == gridDim.x - 1 ? 1u : 0u;\n"
			  << "\t__syncthreads();\n\tif (vgpu_last == 0u) return;\n\t__threadfence();\n"
			  << "\t__shared__ u32 scan_scratch[33];\n";
		} else {
			o << "}\n\n";
			o << "extern \"C\" __global__ void vgpu_gb_direct_final(KArgs a) {\n"
			  << "\t__shared__ u32 scan_scratch[33];\n"
			  << "\tconst u64 D = a.w[" << cb << "];\n";
			for (int f = 0; f < F; f++) {
				o << "\tconst u64 *G" << f << " = (const u64*)a.w[" << cb + 1 + f << "];\n";
			}
		}
		o << "\tu64 base = 0;\n"
		  << "\tfor (u64 c0 = 0; c0 < D; c0 += blockDim.x) {\n"
		  << "\t\tconst u64 s = c0 + threadIdx.x;\n"
		  << "\t\tconst bool live = s < D && G0[s] != 0;\n"
		  << "\t\tu32 total; const u32 off = block_exclusive_scan(live ? 1u : 0u, scan_scratch, &total);\n"
		  << "\t\tif (live) {\n\t\t\tconst u64 pos = base + off;\n\t\t\tconst u64 key = s;\n"
		  << FinalizeCode(gb, fields, visible_, "G", "s", "key", "pos", cb + 1 + F) << "\t\t}\n"
		  << "\t\tbase += total;\n\t}\n"
		  << "\tif (threadIdx.x == 0) *(u64*)a.w[" << cb + 1 + F + out_words << "] = base;\n}\n";
		return o.str();
	}

	if (spec_.join_multi) {
		Fail(VGPU_ERR_INTERNAL, "partitioned group-by over a multi-match join source (materialize the join first)");
	}
	// ---- partitioned: radix partition on the mixed key, then one hash table per partition ----
	// The intermediate is one fixed-size record per qualifying row: the packed key (u64) at byte 0,
	// then each carried value at its natural width and alignment, stride RS a multiple of 32 bytes so
	// every row's write covers whole sectors (no partial-sector read-modify-writes in DRAM however
	// scattered the partitions are).
	struct RecSlot {
		int col, offset, width;
	};
	std::vector<RecSlot> rec;
	int roff = 8;
	for (int c : value_cols) {
		const int w = static_cast<int>(TypeSize(visible_[c].type));
		roff = (roff + w - 1) / w * w;
		rec.push_back({c, roff, w});
		roff += w;
	}
	const int RS = (roff + 31) / 32 * 32;
	const int RW = RS / 4;
	auto rec_value = [&](int col, const std::string &words) -> std::string {
		for (auto &s : rec) {
			if (s.col != col) continue;
			const char *t = CudaTypeName(visible_[col].type);
			const int wi = s.offset / 4, sh = (s.offset % 4) * 8;
			std::string bits;
			if (s.width == 8) {
				bits = "((u64)" + words + "[" + std::to_string(wi) + "] | ((u64)" + words + "[" + std::to_string(wi + 1) +
				       "] << 32))";
			} else if (s.width == 4) {
				bits = "(u64)" + words + "[" + std::to_string(wi) + "]";
			} else {
				const char *mask = s.width == 2 ? "0xffffu" : "0xffu";
				bits = "(u64)((" + words + "[" + std::to_string(wi) + "] >> " + std::to_string(sh) + ") & " + mask + ")";
			}
			return "from_bits<" + std::string(t) + ">(" + bits + ")";
		}
		return "0";
	};
	// Partition of a row: top bits of the mixed key (hashed strategy), or of the bijectively mixed key
	// whose low direct_bits are the table slot (direct-partitioned strategy; the record then carries the
	// mixed key).
	const bool dpart = gb.direct_bits > 0;
	const std::string part_of_pack = dpart ? "(u32)(vgpu_dmix(a, " + pack.str() + ") >> " + std::to_string(gb.direct_bits) + ")"
	                                       : "partition_of(" + pack.str() + ", pbits)";
	const std::string key_of_pack = dpart ? "vgpu_dmix(a, " + pack.str() + ")" : pack.str();
	if (dpart) {
		// multiplier, inverse and key mask come with the arguments, so the kernel does not depend on the data
		o << "__device__ __forceinline__ u64 vgpu_dmix(const KArgs &a, u64 k) { return (k * a.w[" << kMixWord
		  << "]) & a.w[" << kMixWord + 2 << "]; }\n"
		  << "__device__ __forceinline__ u64 vgpu_dunmix(const KArgs &a, u64 k) { return (k * a.w[" << kMixWord + 1
		  << "]) & a.w[" << kMixWord + 2 << "]; }\n\n";
	}
	// Staged tiles (g.staged, direct-partitioned count and scatter): args cb+13 = byte offset of the two
	// stages in dynamic shared memory, cb+14 = error flag (u32*). A full tile's needed columns land in
	// stage (local tile index & 1) by bulk copies that thread 0 issues two tiles ahead; the tail tile
	// uses plain loads. A wait that gives up sets the flag and ends the CTA's tile loop.
	std::vector<int> key_cols_used;
	for (auto &k : gb.keys) key_cols_used.push_back(k.column);
	const auto needed_count = NeededSources(key_cols_used);
	struct StageCol {
		int src, off, chunk;
	};
	auto stage_layout = [&](const std::vector<bool> &nd, int *stage_bytes) {
		std::vector<StageCol> cols;
		int off = 0;
		for (size_t i = 0; i < spec_.sources.size(); i++) {
			if (!nd[i]) continue;
			const int chunk = static_cast<int>(TypeSize(spec_.sources[i].type)) * g.tile();
			cols.push_back({static_cast<int>(i), off, chunk});
			off += chunk;
		}
		*stage_bytes = off;
		return cols;
	};
	auto stage_issue = [&](const std::vector<bool> &nd, const std::string &li, const std::string &t) {
		int sb = 0;
		const auto cols = stage_layout(nd, &sb);
		std::ostringstream r;
		r << "{ const u32 s_ = (u32)(" << li << ") & 1u; u64 *b_ = &vgpu_bar[s_]; char *d_ = vgpu_stage + s_ * " << sb
		  << "u;\n"
		  << "\t\t\tasm volatile(\"fence.proxy.async.shared::cta;\" ::: \"memory\");\n"
		  << "\t\t\tstage_expect(b_, " << sb << "u);\n";
		for (auto &c : cols) {
			r << "\t\t\tstage_copy(d_ + " << c.off << ", (const char*)a.w[" << 2 + 2 * c.src << "] + (" << t << ") * (u64)"
			  << c.chunk << ", " << c.chunk << "u, b_);\n";
		}
		r << "\t\t\tvgpu_pend |= 1u << s_; }\n";
		return r.str();
	};
	auto stage_prologue = [&](const std::vector<bool> &nd, const char *smem_name) {
		if (!g.staged) return std::string();
		std::ostringstream r;
		r << "\t__shared__ __align__(8) u64 vgpu_bar[2];\n"
		  << "\tchar *vgpu_stage = (char*)" << smem_name << " + a.w[" << cb + 13 << "];\n"
		  << "\tconst u64 vgpu_full = n / " << g.tile() << "ull;\n"
		  << "\tconst u64 vgpu_t0 = blockIdx.x * tpc;\n"
		  << "\tu32 vgpu_pend = 0, vgpu_phase = 0;\n\tbool vgpu_failed = false;\n"
		  << "\tif (threadIdx.x == 0) { stage_barrier_init(&vgpu_bar[0]); stage_barrier_init(&vgpu_bar[1]); "
		     "stage_barrier_fence(); }\n"
		  << "\t__syncthreads();\n"
		  << "\tif (threadIdx.x == 0) {\n"
		  << "\t\tfor (u32 j_ = 0; j_ < 2u; ++j_) {\n"
		  << "\t\t\tconst u64 t_ = vgpu_t0 + j_;\n"
		  << "\t\t\tif (t_ < t_end && t_ < vgpu_full) " << stage_issue(nd, "j_", "t_") << "\t\t}\n\t}\n";
		return r.str();
	};
	auto tile_load = [&](const std::vector<bool> &nd) {
		if (!g.staged) return LoadBlock(g, nd, true);
		int sb = 0;
		const auto cols = stage_layout(nd, &sb);
		std::ostringstream r;
		r << "\t\tconst u64 row0 = tile * (u64)" << g.tile() << " + (u64)threadIdx.x * " << g.items << ";\n";
		for (auto &c : cols) {
			r << "\t\t" << CudaTypeName(spec_.sources[c.src].type) << " s" << c.src << "[" << g.items << "];\n";
		}
		r << "\t\tconst u32 vgpu_li = (u32)(tile - vgpu_t0);\n"
		  << "\t\tif (tile < vgpu_full) {\n"
		  << "\t\t\tconst u32 s_ = vgpu_li & 1u;\n"
		  << "\t\t\tif (stage_wait(&vgpu_bar[s_], (vgpu_li >> 1) & 1u)) {\n"
		  << "\t\t\t\tif (threadIdx.x == 0) { vgpu_pend &= ~(1u << s_); vgpu_phase ^= 1u << s_; }\n"
		  << "\t\t\t} else {\n\t\t\t\tvgpu_failed = true;\n\t\t\t}\n"
		  << "\t\t\tconst char *b_ = vgpu_stage + s_ * " << sb << "u;\n";
		for (auto &c : cols) {
			const char *t = CudaTypeName(spec_.sources[c.src].type);
			r << "\t\t\tload_stage<" << t << ", " << g.items << ">((const " << t << "*)(b_ + " << c.off
			  << ") + threadIdx.x * " << g.items << ", s" << c.src << ");\n";
		}
		r << "\t\t} else {\n";
		for (auto &c : cols) {
			const char *t = CudaTypeName(spec_.sources[c.src].type);
			r << "\t\t\tload_rows<" << t << ", " << g.items << ">((const " << t << "*)a.w[" << 2 + 2 * c.src
			  << "], row0, n, s" << c.src << ");\n";
		}
		r << "\t\t}\n"
		  << "\t\tif (__syncthreads_or(vgpu_failed)) { vgpu_failed = true; break; }\n"
		  << "\t\tif (threadIdx.x == 0 && tile + 2 < t_end && tile + 2 < vgpu_full) "
		  << stage_issue(nd, "vgpu_li + 2u", "tile + 2");
		return r.str();
	};
	auto stage_epilogue = [&]() {
		if (!g.staged) return std::string();
		std::ostringstream r;
		r << "\tif (vgpu_failed && threadIdx.x == 0) {\n"
		  << "\t\tatomicOr((u32*)a.w[" << cb + 14 << "], 1u);\n"
		  << "\t\tfor (u32 s_ = 0; s_ < 2u; ++s_) {\n"
		  << "\t\t\tif (vgpu_pend & (1u << s_)) (void)stage_wait(&vgpu_bar[s_], (vgpu_phase >> s_) & 1u);\n"
		  << "\t\t}\n\t}\n";
		return r.str();
	};
	// part_count / part_scatter args: cb+0 = P, cb+1 = pbits, cb+2 = tiles per CTA,
	//   cb+3 = counts/offsets (u32, [p * G + cta]), cb+4 = records out.
	if (dpart && gb.heavy_slots > 0) {
		// ---- heavy-key variants of the partition passes ----
		// A partition holds at most one heavy key: hmap[p] = (state index << 16) | the key's slot in
		// partition p, or ~0 (a slot is below 2^15, so ~0 never matches). Heavy rows fold into the
		// CTA's partial state of their key; each CTA then writes one partial record per heavy key.
		// Extra args: cb+5 = hmap (u32 [P]), cb+6 = sample keys (u64 [SC]), cb+7 = sample counts
		// (u32 [SC]), cb+8 = SC, cb+9 = sampled tile stride, cb+10 = overflow flag (u32*),
		// cb+11 = heavy keys (u32 [K], mixed keys), cb+12 = heavy key count (u32*).
		const int K = gb.heavy_slots;
		const int dbits = gb.direct_bits;
		const std::string dmask = std::to_string((1u << dbits) - 1) + "u";
		// per-CTA partial state of each heavy key: 8-byte arrays (FP64 sums, MIN/MAX) then 32-bit arrays
		// (COUNT, four words per integer SUM)
		struct HArr {
			std::string name, type;
			int bytes;
		};
		std::vector<HArr> harr;
		std::vector<std::string> hkind(gb.aggs.size());
		for (size_t i = 0; i < gb.aggs.size(); i++) {
			const auto &ag = gb.aggs[i];
			if (ag.column < 0 || ag.kind == AggKind::COUNT || ag.kind == AggKind::COUNT_STAR) continue;
			const std::string is = std::to_string(i);
			if (ag.kind == AggKind::MIN || ag.kind == AggKind::MAX) {
				hkind[i] = ag.kind == AggKind::MIN ? "min" : "max";
				harr.push_back({"HM" + is, "i64", 8});
			} else if (IsFloatType(ag.input_type)) {
				hkind[i] = "f64";
				harr.push_back({"HF" + is, "double", 8});
			} else {
				hkind[i] = "int";
			}
		}
		harr.push_back({"HC", "u32", 4});
		for (size_t i = 0; i < gb.aggs.size(); i++) {
			if (hkind[i] != "int") continue;
			for (int w = 0; w < 4; w++) harr.push_back({"HW" + std::to_string(i) + "_" + std::to_string(w), "u32", 4});
		}
		// shared layout after the P + 32 counters: hmap [P], heavy keys [K], then the state arrays
		// (16-byte aligned; the host sizes the launch with the same rule)
		std::ostringstream hdecl;
		hdecl << "\tconst u32 hoff = ((P + 32u) * 4u + 15u) & ~15u;\n"
		      << "\tu32 *vgpu_hmap = (u32*)((char*)vgpu_smem + hoff);\n"
		      << "\tu32 *vgpu_hkeys = vgpu_hmap + P;\n"
		      << "\tchar *vgpu_hstate = (char*)vgpu_smem + ((hoff + 4u * P + " << 4 * K << "u + 15u) & ~15u);\n"
		      << "\tconst u32 nheavy = *(const u32*)a.w[" << cb + 12 << "];\n";
		uint64_t hbytes = 0;
		for (auto &ar : harr) {
			hdecl << "\t" << ar.type << " *" << ar.name << " = (" << ar.type << "*)(vgpu_hstate + " << hbytes << ");\n";
			hbytes += static_cast<uint64_t>(K) * ar.bytes;
		}
		auto heavy_load = [&](bool with_state) {
			std::ostringstream r;
			r << "\tfor (u32 p = threadIdx.x; p < P; p += blockDim.x) vgpu_hmap[p] = ((const u32*)a.w[" << cb + 5
			  << "])[p];\n"
			  << "\tfor (u32 h = threadIdx.x; h < nheavy; h += blockDim.x) {\n"
			  << "\t\tvgpu_hkeys[h] = ((const u32*)a.w[" << cb + 11 << "])[h];\n";
			if (with_state) {
				for (auto &ar : harr) {
					std::string init = "0";
					if (ar.name.rfind("HM", 0) == 0) {
						const int ai = std::stoi(ar.name.substr(2));
						init = hkind[ai] == "min" ? "0x7fffffffffffffffLL" : "(-0x7fffffffffffffffLL - 1)";
					}
					r << "\t\t" << ar.name << "[h] = (" << ar.type << ")" << init << ";\n";
				}
			}
			r << "\t}\n";
			return r.str();
		};
		const std::string mixed = "vgpu_dmix(a, " + pack.str() + ")";
		// a kept row's heavy-state index, or -1 (one map load per row)
		o << "__device__ __forceinline__ int vgpu_heavy_slot(const u32 *hmap, u64 k) {\n"
		  << "\tconst u32 e = hmap[(u32)(k >> " << dbits << ")];\n"
		  << "\treturn (e & 0xffffu) == ((u32)k & " << dmask << ") ? (int)(e >> 16) : -1;\n}\n\n";
		const std::string heavy_of = "vgpu_heavy_slot(vgpu_hmap, k0)";
		// sample: one tile per CTA at a stride, counts of the mixed keys of the kept rows
		o << "extern \"C\" __global__ void __launch_bounds__(" << g.block << (g.min_blocks > 0 ? ", " + std::to_string(g.min_blocks) : std::string()) << ") vgpu_gb_sample(KArgs a) {\n"
		  << kKernelHead
		  << "\tu64 *skeys = (u64*)a.w[" << cb + 6 << "];\n\tu32 *scount = (u32*)a.w[" << cb + 7 << "];\n"
		  << "\tconst u32 SC = (u32)a.w[" << cb + 8 << "];\n"
		  << "\tconst u64 tile = (u64)blockIdx.x * a.w[" << cb + 9 << "];\n"
		  << LoadBlock(g, needed, true) << item_head << chain_code_ << "\t\tif (keep) {\n"
		  << "\t\t\tconst u64 k = " << mixed << ";\n"
		  << "\t\t\tu32 s = (u32)mix64(k) & (SC - 1);\n"
		  // a short probe: a key that finds no slot within 8 is a rare one in a table that filled up
		  // (many distinct keys), which no heavy-key selection would pick
		  << "\t\t\t#pragma unroll 1\n\t\t\tfor (int i = 0; i < 8; ++i) {\n"
		  << "\t\t\t\tconst u64 prev = atomicCAS((unsigned long long*)&skeys[s], ~0ull, k);\n"
		  << "\t\t\t\tif (prev == ~0ull || prev == k) { atomicAdd(&scount[s], 1u); break; }\n"
		  << "\t\t\t\ts = (s + 1) & (SC - 1);\n\t\t\t}\n"
		  << "\t\t}\n\t\t}\n}\n\n";
		// count: heavy rows are not counted; every CTA reserves one partial record per heavy key
		o << "extern \"C\" __global__ void __launch_bounds__(" << g.block << (g.min_blocks > 0 ? ", " + std::to_string(g.min_blocks) : std::string()) << ") vgpu_gb_part_count(KArgs a) {\n"
		  << kKernelHead << "\textern __shared__ __align__(16) u32 vgpu_smem[];\n\tu32 *vgpu_hist = vgpu_smem;\n"
		  << "\tconst u32 P = (u32)a.w[" << cb << "]; const int pbits = (int)a.w[" << cb + 1 << "]; (void)pbits;\n"
		  << "\tconst u64 tpc = a.w[" << cb + 2 << "];\n"
		  << hdecl.str()
		  << "\tfor (u32 p = threadIdx.x; p < P; p += " << g.block << ") vgpu_hist[p] = 0;\n"
		  << heavy_load(false) << "\t__syncthreads();\n"
		  << tile_loop_head
		  << "\tconst u64 t_end = (blockIdx.x + 1) * tpc < ntiles ? (blockIdx.x + 1) * tpc : ntiles;\n"
		  << stage_prologue(needed_count, "vgpu_smem")
		  << "\tfor (u64 tile = blockIdx.x * tpc; tile < t_end; ++tile) {\n"
		  << tile_load(needed_count) << item_head << chain_code_ << "\t\tif (keep) {\n"
		  << "\t\t\tconst u64 k0 = " << mixed << ";\n"
		  << "\t\t\tif (" << heavy_of << " < 0) atomicAdd(&vgpu_hist[(u32)(k0 >> " << dbits << ")], 1u);\n"
		  << "\t\t}\n\t\t}\n\t}\n" << stage_epilogue() << "\t__syncthreads();\n"
		  << "\tfor (u32 h = threadIdx.x; h < nheavy; h += blockDim.x) atomicAdd(&vgpu_hist[vgpu_hkeys[h] >> " << dbits
		  << "], 1u);\n"
		  << "\t__syncthreads();\n"
		  << "\tu32 *counts = (u32*)a.w[" << cb + 3 << "];\n"
		  << "\tfor (u32 p = threadIdx.x; p < P; p += " << g.block
		  << ") counts[(u64)p * gridDim.x + blockIdx.x] = vgpu_hist[p];\n}\n\n";
		// scatter: heavy rows fold into the CTA's partial state, the rest are records; then one partial
		// record per heavy key (flag bit 31 of the key word, row count in the next word, each aggregate's
		// partial state in its value column's slot)
		std::ostringstream hupd;
		hupd << "\t\t\t\tatomicAdd(&HC[h], 1u);\n";
		for (size_t i = 0; i < gb.aggs.size(); i++) {
			if (hkind[i].empty()) continue;
			const std::string is = std::to_string(i);
			const std::string v = visible_[gb.aggs[i].column].value;
			if (hkind[i] == "int") {
				hupd << "\t\t\t\t{ const i64 x_ = (i64)(" << v << "); atomic_add_i128_u32x4(&HW" << is << "_0[h], &HW" << is
				     << "_1[h], &HW" << is << "_2[h], &HW" << is << "_3[h], (u64)x_, x_ < 0 ? -1 : 0); }\n";
			} else if (hkind[i] == "f64") {
				hupd << "\t\t\t\tatomicAdd(&HF" << is << "[h], (double)(" << v << "));\n";
			} else {
				hupd << "\t\t\t\tatomic_" << hkind[i] << "_i64(&HM" << is << "[h], (i64)(" << v << "));\n";
			}
		}
		// Warp-aggregated form (gb.heavy_warp): the lanes of a step holding the same heavy key (found with
		// __match_any_sync) fold their rows into the group's lowest lane by shuffles -- count, 128-bit
		// integer sums, FP64 sums, MIN/MAX -- and that lane alone updates the shared state, so a hot key
		// costs one set of shared atomics per warp step instead of one per row.
		std::ostringstream hgrp;
		hgrp << "\t\t\tconst u32 ln_ = threadIdx.x & 31u, lead_ = __ffs(hpeers_) - 1u;\n"
		     << "\t\t\tu32 gc_ = 1u;\n";
		for (size_t i = 0; i < gb.aggs.size(); i++) {
			if (hkind[i].empty()) continue;
			const std::string is = std::to_string(i);
			const std::string v = visible_[gb.aggs[i].column].value;
			if (hkind[i] == "int") {
				hgrp << "\t\t\tu64 glo" << is << " = (u64)(i64)(" << v << "); i64 ghi" << is << " = ((i64)(" << v
				     << ") < 0) ? -1 : 0;\n";
			} else if (hkind[i] == "f64") {
				hgrp << "\t\t\tdouble gf" << is << " = (double)(" << v << ");\n";
			} else {
				hgrp << "\t\t\ti64 gm" << is << " = (i64)(" << v << ");\n";
			}
		}
		hgrp << "\t\t\tfor (u32 m_ = hpeers_ & ~(1u << lead_); m_; m_ &= m_ - 1u) {\n"
		     << "\t\t\t\tconst u32 src_ = __ffs(m_) - 1u;\n"
		     << "\t\t\t\tconst bool me_ = ln_ == lead_;\n"
		     << "\t\t\t\tgc_ += me_ ? 1u : 0u;\n";
		for (size_t i = 0; i < gb.aggs.size(); i++) {
			if (hkind[i].empty()) continue;
			const std::string is = std::to_string(i);
			if (hkind[i] == "int") {
				hgrp << "\t\t\t\t{ const u64 ol_ = __shfl_sync(hpeers_, glo" << is << ", src_); const i64 oh_ = __shfl_sync(hpeers_, ghi"
				     << is << ", src_);\n\t\t\t\t  if (me_) { const u64 nl_ = glo" << is << " + ol_; ghi" << is
				     << " += oh_ + (nl_ < glo" << is << " ? 1 : 0); glo" << is << " = nl_; } }\n";
			} else if (hkind[i] == "f64") {
				hgrp << "\t\t\t\t{ const double o_ = __shfl_sync(hpeers_, gf" << is << ", src_); if (me_) gf" << is << " += o_; }\n";
			} else {
				const char *op = hkind[i] == "min" ? "<" : ">";
				hgrp << "\t\t\t\t{ const i64 o_ = __shfl_sync(hpeers_, gm" << is << ", src_); if (me_ && o_ " << op << " gm" << is
				     << ") gm" << is << " = o_; }\n";
			}
		}
		hgrp << "\t\t\t}\n\t\t\tif (ln_ == lead_) {\n\t\t\t\tatomicAdd(&HC[h], gc_);\n";
		for (size_t i = 0; i < gb.aggs.size(); i++) {
			if (hkind[i].empty()) continue;
			const std::string is = std::to_string(i);
			if (hkind[i] == "int") {
				hgrp << "\t\t\t\tatomic_add_i128_u32x4(&HW" << is << "_0[h], &HW" << is << "_1[h], &HW" << is << "_2[h], &HW" << is
				     << "_3[h], glo" << is << ", ghi" << is << ");\n";
			} else if (hkind[i] == "f64") {
				hgrp << "\t\t\t\tatomicAdd(&HF" << is << "[h], gf" << is << ");\n";
			} else {
				hgrp << "\t\t\t\tatomic_" << hkind[i] << "_i64(&HM" << is << "[h], gm" << is << ");\n";
			}
		}
		hgrp << "\t\t\t}\n";
		std::ostringstream hflush;
		hflush << "\t\t\tu32 rw[" << RW << "];\n"
		       << "\t\t\t#pragma unroll\n\t\t\tfor (int q = 0; q < " << RW << "; ++q) rw[q] = 0u;\n"
		       << "\t\t\trw[0] = k | 0x80000000u; rw[1] = HC[h];\n";
		for (auto &sl : rec) {
			int ai = -1;
			for (size_t i = 0; i < gb.aggs.size(); i++) {
				if (!hkind[i].empty() && gb.aggs[i].column == sl.col) ai = static_cast<int>(i);
			}
			if (ai < 0) continue;
			const std::string is = std::to_string(ai);
			const int wi = sl.offset / 4;
			std::string bits;
			if (hkind[ai] == "int") {
				bits = "((u64)HW" + is + "_0[h] | ((u64)HW" + is + "_1[h] << 32))";
				// the partial travels as a 64-bit value: a sum outside that range flags the launch,
				// whose caller then runs the query without pre-aggregation
				hflush << "\t\t\tif (HW" << is << "_2[h] != ((HW" << is << "_1[h] & 0x80000000u) ? 0xffffffffu : 0u) || HW"
				       << is << "_3[h] != HW" << is << "_2[h]) atomicOr((u32*)a.w[" << cb + 10 << "], 1u);\n";
			} else if (hkind[ai] == "f64") {
				bits = "(u64)__double_as_longlong(HF" + is + "[h])";
			} else {
				bits = "(u64)HM" + is + "[h]";
			}
			hflush << "\t\t\t{ const u64 b = " << bits << "; rw[" << wi << "] = (u32)b; rw[" << wi + 1
			       << "] = (u32)(b >> 32); }\n";
		}
		o << "extern \"C\" __global__ void __launch_bounds__(" << g.block << (g.min_blocks > 0 ? ", " + std::to_string(g.min_blocks) : std::string()) << ") vgpu_gb_part_scatter(KArgs a) {\n"
		  << kKernelHead << "\textern __shared__ __align__(16) u32 vgpu_smem[];\n\tu32 *vgpu_cursor = vgpu_smem;\n"
		  << "\tconst u32 P = (u32)a.w[" << cb << "]; const int pbits = (int)a.w[" << cb + 1 << "]; (void)pbits;\n"
		  << "\tconst u64 tpc = a.w[" << cb + 2 << "];\n"
		  << "\tconst u32 *offsets = (const u32*)a.w[" << cb + 3 << "];\n"
		  << "\tchar *rec_out = (char*)a.w[" << cb + 4 << "];\n"
		  << hdecl.str()
		  << "\tfor (u32 p = threadIdx.x; p < P; p += " << g.block
		  << ") vgpu_cursor[p] = offsets[(u64)p * gridDim.x + blockIdx.x];\n"
		  << heavy_load(true) << "\t__syncthreads();\n"
		  << tile_loop_head
		  << "\tconst u64 t_end = (blockIdx.x + 1) * tpc < ntiles ? (blockIdx.x + 1) * tpc : ntiles;\n"
		  << stage_prologue(needed, "vgpu_smem")
		  << "\tfor (u64 tile = blockIdx.x * tpc; tile < t_end; ++tile) {\n"
		  << tile_load(needed)
		  << "\t\tu32 vgpu_pos[" << g.items << "];\n\t\tint vgpu_hv[" << g.items << "];\n\t\tu64 vgpu_k[" << g.items
		  << "];\n"
		  << item_head << chain_code_
		  << "\t\tconst u64 k0 = " << mixed << ";\n"
		  << "\t\tvgpu_k[r] = k0;\n"
		  << "\t\tvgpu_hv[r] = keep ? " << heavy_of << " : -1;\n"
		  << "\t\tvgpu_pos[r] = atomicAdd(&vgpu_cursor[keep && vgpu_hv[r] < 0 ? (u32)(k0 >> " << dbits
		  << ") : P + (threadIdx.x & 31u)], 1u);\n"
		  << "\t\t}\n"
		  << item_head << chain_code_;
		if (gb.heavy_warp) {
			// every lane of the warp reaches the match (the item loop has no divergent exit)
			o << "\t\tconst int hh_ = keep ? vgpu_hv[r] : -1;\n"
			  << "\t\tconst u32 hpeers_ = __match_any_sync(0xffffffffu, hh_);\n"
			  << "\t\tif (hh_ >= 0) {\n\t\t\tconst int h = hh_;\n" << hgrp.str() << "\t\t} else if (keep) {\n\t\t{\n";
		} else {
			o << "\t\tif (keep) {\n"
			  << "\t\t\tconst int h = vgpu_hv[r];\n"
			  << "\t\t\tif (h >= 0) {\n" << hupd.str() << "\t\t\t} else {\n";
		}
		o << "\t\t\tconst u64 key = vgpu_k[r];\n"
		  << "\t\t\tconst u32 pos = vgpu_pos[r];\n"
		  << "\t\t\tu32 rw[" << RW << "];\n"
		  << "\t\t\t#pragma unroll\n\t\t\tfor (int q = 0; q < " << RW << "; ++q) rw[q] = 0u;\n"
		  << "\t\t\trw[0] = (u32)key; rw[1] = (u32)(key >> 32);\n";
		for (auto &sl : rec) {
			const auto &col = visible_[sl.col];
			const int wi = sl.offset / 4, sh = (sl.offset % 4) * 8;
			o << "\t\t\t{ const u64 b = to_bits<" << CudaTypeName(col.type) << ">(" << col.value << ");\n";
			if (sl.width == 8) {
				o << "\t\t\t  rw[" << wi << "] = (u32)b; rw[" << wi + 1 << "] = (u32)(b >> 32); }\n";
			} else if (sl.width == 4) {
				o << "\t\t\t  rw[" << wi << "] = (u32)b; }\n";
			} else {
				o << "\t\t\t  rw[" << wi << "] |= ((u32)b & " << (sl.width == 2 ? "0xffffu" : "0xffu") << ") << " << sh
				  << "; }\n";
			}
		}
		o << "\t\t\tstore_record<" << RW << ">(rec_out + (u64)pos * " << RS << ", rw);\n"
		  << "\t\t\t}\n\t\t}\n\t\t}\n\t}\n"
		  << stage_epilogue() << "\t__syncthreads();\n"
		  << "\tfor (u32 h = threadIdx.x; h < nheavy; h += blockDim.x) {\n"
		  << "\t\tconst u32 k = vgpu_hkeys[h];\n"
		  << "\t\tconst u32 pos = atomicAdd(&vgpu_cursor[k >> " << dbits << "], 1u);\n"
		  << "\t\t{\n" << hflush.str()
		  << "\t\t\tstore_record<" << RW << ">(rec_out + (u64)pos * " << RS << ", rw);\n\t\t}\n\t}\n}\n\n";
	} else {
	o << "extern \"C\" __global__ void __launch_bounds__(" << g.block << (g.min_blocks > 0 ? ", " + std::to_string(g.min_blocks) : std::string()) << ") vgpu_gb_part_count(KArgs a) {\n"
	  << kKernelHead << "\textern __shared__ __align__(16) u32 vgpu_hist[];\n"
	  << "\tconst u32 P = (u32)a.w[" << cb << "]; const int pbits = (int)a.w[" << cb + 1 << "];\n"
	  << "\tconst u64 tpc = a.w[" << cb + 2 << "];\n"
	  << "\tfor (u32 p = threadIdx.x; p < P; p += " << g.block << ") vgpu_hist[p] = 0;\n\t__syncthreads();\n"
	  << tile_loop_head
	  << "\tconst u64 t_end = (blockIdx.x + 1) * tpc < ntiles ? (blockIdx.x + 1) * tpc : ntiles;\n"
	  << stage_prologue(needed_count, "vgpu_hist")
	  << "\tfor (u64 tile = blockIdx.x * tpc; tile < t_end; ++tile) {\n"
	  << tile_load(needed_count) << item_head << chain_code_ << "\t\tif (keep) {\n"
	  << "\t\t\tatomicAdd(&vgpu_hist[" << part_of_pack << "], 1u);\n"
	  << "\t\t}\n\t\t}\n\t}\n" << stage_epilogue() << "\t__syncthreads();\n"
	  << "\tu32 *counts = (u32*)a.w[" << cb + 3 << "];\n"
	  << "\tfor (u32 p = threadIdx.x; p < P; p += " << g.block
	  << ") counts[(u64)p * gridDim.x + blockIdx.x] = vgpu_hist[p];\n}\n\n";

	o << "extern \"C\" __global__ void __launch_bounds__(" << g.block << (g.min_blocks > 0 ? ", " + std::to_string(g.min_blocks) : std::string()) << ") vgpu_gb_part_scatter(KArgs a) {\n"
	  << kKernelHead << "\textern __shared__ __align__(16) u32 vgpu_cursor[];\n"
	  << "\tconst u32 P = (u32)a.w[" << cb << "]; const int pbits = (int)a.w[" << cb + 1 << "];\n"
	  << "\tconst u64 tpc = a.w[" << cb + 2 << "];\n"
	  << "\tconst u32 *offsets = (const u32*)a.w[" << cb + 3 << "];\n"
	  << "\tchar *rec_out = (char*)a.w[" << cb + 4 << "];\n"
	  << "\tfor (u32 p = threadIdx.x; p < P; p += " << g.block
	  << ") vgpu_cursor[p] = offsets[(u64)p * gridDim.x + blockIdx.x];\n\t__syncthreads();\n"
	  << tile_loop_head
	  << "\tconst u64 t_end = (blockIdx.x + 1) * tpc < ntiles ? (blockIdx.x + 1) * tpc : ntiles;\n"
	  << stage_prologue(needed, "vgpu_cursor")
	  << "\tfor (u64 tile = blockIdx.x * tpc; tile < t_end; ++tile) {\n"
	  << tile_load(needed)
	  // every item's cursor reservation first, branch-free (rows that are filtered out add to a per-lane
	  // dummy counter past P), so the tile's shared atomics are in flight together; then the records
	  << "\t\tu32 vgpu_pos[" << g.items << "];\n\t\tu64 vgpu_k[" << g.items << "];\n"
	  << item_head << chain_code_
	  << "\t\tconst u64 k0 = " << key_of_pack << ";\n"
	  << "\t\tvgpu_k[r] = k0;\n"
	  << "\t\tvgpu_pos[r] = atomicAdd(&vgpu_cursor[keep ? "
	  << (dpart ? "(u32)(k0 >> " + std::to_string(gb.direct_bits) + ")" : std::string("partition_of(k0, pbits)"))
	  << " : P + (threadIdx.x & 31u)], 1u);\n"
	  << "\t\t}\n"
	  << item_head << chain_code_ << "\t\tif (keep) {\n"
	  << "\t\t\tconst u64 key = vgpu_k[r];\n"
	  << "\t\t\tconst u32 pos = vgpu_pos[r];\n"
	  << "\t\t\tu32 rw[" << RW << "];\n"
	  << "\t\t\t#pragma unroll\n\t\t\tfor (int q = 0; q < " << RW << "; ++q) rw[q] = 0u;\n"
	  << "\t\t\trw[0] = (u32)key; rw[1] = (u32)(key >> 32);\n";
	for (auto &s : rec) {
		const auto &col = visible_[s.col];
		const int wi = s.offset / 4, sh = (s.offset % 4) * 8;
		o << "\t\t\t{ const u64 b = to_bits<" << CudaTypeName(col.type) << ">(" << col.value << ");\n";
		if (s.width == 8) {
			o << "\t\t\t  rw[" << wi << "] = (u32)b; rw[" << wi + 1 << "] = (u32)(b >> 32); }\n";
		} else if (s.width == 4) {
			o << "\t\t\t  rw[" << wi << "] = (u32)b; }\n";
		} else {
			o << "\t\t\t  rw[" << wi << "] |= ((u32)b & " << (s.width == 2 ? "0xffffu" : "0xffu") << ") << " << sh
			  << "; }\n";
		}
	}
	o << "\t\t\tstore_record<" << RW << ">(rec_out + (u64)pos * " << RS << ", rw);\n"
	  << "\t\t}\n\t\t}\n\t}\n" << stage_epilogue() << "}\n\n";

	}

	// bucket: args cb+0 = P, cb+1 = C (smem table slots), cb+2 = offsets (u32 [p*G]), cb+3 = G,
	//   cb+4 = total ptr (u32*), cb+5 = records, then W = cb+6: work counter (u32*), W+1 overflow flags
	//   (u32 [P]), W+2 overflow count (u32*), W+3 output count (u64*), W+4.. outputs. Global-table
	//   variant: W+4+outs = partition list (u32*), +1 list length, +2 table base (u64*), +3 per-entry
	//   table offsets (u64*), +4 capacities (u32*).
	// Rows are read warp-contiguously: lane i of a warp takes record base + 32q + i, four 32-record
	// steps per iteration with their loads hoisted. Lanes holding equal keys are found with
	// __match_any_sync; when some group spans at least 4 lanes (a heavy key) the groups are combined by a
	// rank tree of shuffles, so only each group's first lane updates the table. Counts are 32-bit
	// atomics on the low half of the count word (a partition holds fewer than 2^32 rows).
	const int W = cb + 6;
	const int OUT = W + 4;
	std::ostringstream gdecl, gcomb, gupd, gxor, wdecl, wacc, wflush, wvars;
	gdecl << "\t\t\tu32 gc = valid ? 1u : 0u;\n";
	gxor << "\t\t\t\t\tgc += __shfl_xor_sync(0xffffffffu, gc, d);\n";
	wdecl << "\tu64 my_pk = ~0ull; u64 wc = 0; u32 free_mask = 0xffu;\n"
	      << "\tu64 pk_[8];\n\t#pragma unroll\n\tfor (int j = 0; j < 8; ++j) pk_[j] = ~0ull;\n";
	wacc << "\t\t\t\t{ const u32 t_ = __shfl_sync(0xffffffffu, gc, src_); if (have_) wc += t_; }\n";
	wflush << "\t\t\tatomicAdd((u32*)(T0 + s_), (u32)wc);\n";
	gcomb << "\t\t\t\t\t{ const u32 o_ = __shfl_sync(0xffffffffu, gc, src_); if (take) gc += o_; }\n";
	gupd << "\t\t\t\t\tatomicAdd((u32*)(T0 + s_), gc);\n";
	for (int f = 1; f < F; f++) {
		const auto &fd = fields[f];
		const std::string v = "v" + std::to_string(fd.agg);
		if (fd.kind == "f64") {
			gdecl << "\t\t\tdouble gf" << f << " = valid ? (double)" << v << " : 0.0;\n";
			gcomb << "\t\t\t\t\t{ const double o_ = __shfl_sync(0xffffffffu, gf" << f << ", src_); if (take) gf" << f
			      << " += o_; }\n";
			gupd << "\t\t\t\t\tatomicAdd((double*)(T" << f << " + s_), gf" << f << ");\n";
			gxor << "\t\t\t\t\tgf" << f << " += __shfl_xor_sync(0xffffffffu, gf" << f << ", d);\n";
			wdecl << "\tdouble wf" << f << " = 0.0;\n";
			wvars << "\tdouble wf" << f << " = 0.0;\n";
			wacc << "\t\t\t\t{ const double t_ = __shfl_sync(0xffffffffu, gf" << f << ", src_); if (have_) wf" << f << " += t_; }\n";
			wflush << "\t\t\tatomicAdd((double*)(T" << f << " + s_), wf" << f << ");\n";
		} else if (fd.kind == "lo") {
			gdecl << "\t\t\tu64 glo" << f << " = valid ? (u64)(i64)" << v << " : 0ull; i64 ghi" << f << " = (valid && (i64)"
			      << v << " < 0) ? -1 : 0;\n";
			gcomb << "\t\t\t\t\t{ const u64 ol_ = __shfl_sync(0xffffffffu, glo" << f
			      << ", src_); const i64 oh_ = __shfl_sync(0xffffffffu, ghi" << f << ", src_);\n"
			      << "\t\t\t\t\t  if (take) { const u64 nl_ = glo" << f << " + ol_; ghi" << f << " += oh_ + (nl_ < glo" << f
			      << " ? 1 : 0); glo" << f << " = nl_; } }\n";
			gupd << "\t\t\t\t\tatomic_add_i128_pair(T" << f << " + s_, (i64*)(T" << f + 1 << " + s_), glo" << f << ", ghi"
			     << f << ");\n";
			gxor << "\t\t\t\t\t{ const u64 ol_ = __shfl_xor_sync(0xffffffffu, glo" << f
			     << ", d); const i64 oh_ = __shfl_xor_sync(0xffffffffu, ghi" << f << ", d); const u64 nl_ = glo" << f
			     << " + ol_; ghi" << f << " += oh_ + (nl_ < glo" << f << " ? 1 : 0); glo" << f << " = nl_; }\n";
			wdecl << "\tu64 wlo" << f << " = 0; i64 whi" << f << " = 0;\n";
			wvars << "\tu64 wlo" << f << " = 0; i64 whi" << f << " = 0;\n";
			wacc << "\t\t\t\t{ const u64 ol_ = __shfl_sync(0xffffffffu, glo" << f
			     << ", src_); const i64 oh_ = __shfl_sync(0xffffffffu, ghi" << f << ", src_);\n"
			     << "\t\t\t\t  if (have_) { const u64 nl_ = wlo" << f << " + ol_; whi" << f << " += oh_ + (nl_ < wlo" << f
			     << " ? 1 : 0); wlo" << f << " = nl_; } }\n";
			wflush << "\t\t\tatomic_add_i128_pair(T" << f << " + s_, (i64*)(T" << f + 1 << " + s_), wlo" << f << ", whi" << f
			       << ");\n";
		} else if (fd.kind == "min" || fd.kind == "max") {
			const char *op = fd.kind == "min" ? "<" : ">";
			const char *ident = fd.kind == "min" ? "0x7fffffffffffffffLL" : "(-0x7fffffffffffffffLL - 1)";
			gdecl << "\t\t\ti64 gm" << f << " = valid ? (i64)" << v << " : " << ident << ";\n";
			gcomb << "\t\t\t\t\t{ const i64 o_ = __shfl_sync(0xffffffffu, gm" << f << ", src_); if (take && o_ " << op
			      << " gm" << f << ") gm" << f << " = o_; }\n";
			gupd << "\t\t\t\t\tatomic_" << fd.kind << "_i64((i64*)(T" << f << " + s_), gm" << f << ");\n";
			gxor << "\t\t\t\t\t{ const i64 o_ = __shfl_xor_sync(0xffffffffu, gm" << f << ", d); if (o_ " << op << " gm" << f
			     << ") gm" << f << " = o_; }\n";
			wdecl << "\ti64 wm" << f << " = " << ident << ";\n";
			wvars << "\ti64 wm" << f << " = " << ident << ";\n";
			wacc << "\t\t\t\t{ const i64 t_ = __shfl_sync(0xffffffffu, gm" << f << ", src_); if (have_ && t_ " << op << " wm" << f
			     << ") wm" << f << " = t_; }\n";
			wflush << "\t\t\tatomic_" << fd.kind << "_i64((i64*)(T" << f << " + s_), wm" << f << ");\n";
		}
	}
	if (dpart) {
		// ---- direct-partitioned buckets ----
		// args: cb+0 = work items (uint4: partition, first row, end row, split index or ~0),
		//   cb+1 = item count (u32*), cb+2 = records, cb+3 = global tables of split partitions (u64,
		//   [split][field][D]), cb+4 = split info (u32 [2s] chunks, [2s+1] completed chunks),
		//   cb+5 = work counter (u32*), cb+6 = output count (u64*), cb+7 = split partition count (u32*,
		//   read by the init kernel), cb+8.. outputs.
		// Shared table of D slots, one array per state word: 8-byte arrays (FP64 sums, MIN/MAX) first,
		// then 32-bit arrays (COUNT, and four words per integer SUM accumulated with 32-bit atomics).
		const int dbits = gb.direct_bits;
		const uint64_t D = 1ull << dbits;
		struct DArr {
			std::string name, type;
			int bytes;
		};
		std::vector<DArr> arrs;
		for (int f = 0; f < F; f++) {
			const auto &fd = fields[f];
			if (fd.kind == "f64" && !gb.f64_l2) arrs.push_back({"DF" + std::to_string(f), "double", 8});
			if (fd.kind == "min" || fd.kind == "max") arrs.push_back({"DM" + std::to_string(f), "i64", 8});
		}
		for (int f = 0; f < F; f++) {
			const auto &fd = fields[f];
			if (fd.kind == "cnt") arrs.push_back({"DC", "u32", 4});
			if (fd.kind == "lo") {
				for (int w = 0; w < 4; w++) arrs.push_back({"DW" + std::to_string(f) + "_" + std::to_string(w), "u32", 4});
			}
		}
		std::ostringstream decl;  // array pointers into the shared table `sm`
		uint64_t off = 0;
		for (auto &ar : arrs) {
			decl << "\t" << ar.type << " *" << ar.name << " = (" << ar.type << "*)(sm + " << off << ");\n";
			off += D * ar.bytes;
		}
		// FP64 sums in the CTA's own tables of the global region (L2-resident: reductions, no CAS loops)
		const int OUTD_ = cb + 8;
		const int SCR = OUTD_ + static_cast<int>(gb.keys.size() + gb.aggs.size());
		if (gb.f64_l2) {
			int fi = 0;
			const int nf = F64Fields(gb);
			for (int f = 0; f < F; f++) {
				if (fields[f].kind != "f64") continue;
				decl << "\tdouble *DF" << f << " = (double*)a.w[" << SCR << "] + ((u64)blockIdx.x * " << nf << "u + " << fi
				     << "u) * " << D << "ull;\n";
				fi++;
			}
		}
		// a sum field's current value (the global tables are read past L1: reductions land in L2)
		auto f64_load = [&](int f, const std::string &sv) {
			return gb.f64_l2 ? "__ldcg(&DF" + std::to_string(f) + "[" + sv + "])" : "DF" + std::to_string(f) + "[" + sv + "]";
		};
		auto reset_slot = [&](const std::string &sv) {
			std::ostringstream r;
			for (int f = 0; f < F; f++) {
				const auto &fd = fields[f];
				if (fd.kind == "cnt") r << "\t\t\tDC[" << sv << "] = 0u;\n";
				if (fd.kind == "f64") r << "\t\t\tDF" << f << "[" << sv << "] = 0.0;\n";
				if (fd.kind == "min" || fd.kind == "max") {
					r << "\t\t\tDM" << f << "[" << sv << "] = (i64)" << InitValue(fd) << ";\n";
				}
				if (fd.kind == "lo") {
					for (int w = 0; w < 4; w++) r << "\t\t\tDW" << f << "_" << w << "[" << sv << "] = 0u;\n";
				}
			}
			return r.str();
		};
		// slot state in the u64 field format of the other strategies (S<f>[0])
		auto load_slot = [&](const std::string &sv) {
			std::ostringstream r;
			for (int f = 0; f < F; f++) {
				const auto &fd = fields[f];
				if (fd.kind == "cnt") r << "\t\t\tS" << f << "[0] = (u64)DC[" << sv << "];\n";
				if (fd.kind == "f64") r << "\t\t\tS" << f << "[0] = (u64)__double_as_longlong(" << f64_load(f, sv) << ");\n";
				if (fd.kind == "min" || fd.kind == "max") r << "\t\t\tS" << f << "[0] = (u64)DM" << f << "[" << sv << "];\n";
				if (fd.kind == "lo") {
					r << "\t\t\tS" << f << "[0] = (u64)DW" << f << "_0[" << sv << "] | ((u64)DW" << f << "_1[" << sv
					  << "] << 32);\n"
					  << "\t\t\tS" << f + 1 << "[0] = (u64)DW" << f << "_2[" << sv << "] | ((u64)DW" << f << "_3[" << sv
					  << "] << 32);\n";
				}
			}
			return r.str();
		};
		// update of slot `sv` with the register partials of prefix `g` (group) or `w` (hot run)
		auto update = [&](const std::string &pre, const std::string &sv) {
			std::ostringstream r;
			for (int f = 0; f < F; f++) {
				const auto &fd = fields[f];
				const std::string fs = std::to_string(f);
				if (fd.kind == "cnt") r << "\t\t\t\tatomicAdd(&DC[" << sv << "], (u32)" << pre << "c);\n";
				if (fd.kind == "f64") r << "\t\t\t\tatomicAdd(&DF" << fs << "[" << sv << "], " << pre << "f" << fs << ");\n";
				if (fd.kind == "min" || fd.kind == "max") {
					r << "\t\t\t\tatomic_" << fd.kind << "_i64(&DM" << fs << "[" << sv << "], " << pre << "m" << fs << ");\n";
				}
				if (fd.kind == "lo") {
					r << "\t\t\t\tatomic_add_i128_u32x4(&DW" << fs << "_0[" << sv << "], &DW" << fs << "_1[" << sv << "], &DW" << fs
					  << "_2[" << sv << "], &DW" << fs << "_3[" << sv << "], " << pre << "lo" << fs << ", " << pre << "hi" << fs
					  << ");\n";
				}
			}
			return r.str();
		};
		std::ostringstream sdecl;
		for (int f = 0; f < F; f++) sdecl << (f ? ", " : "\t\t\tu64 ") << "S" << f << "[1]";
		sdecl << ";\n";
		std::ostringstream gptr;  // global table arrays of split index `sidx`
		for (int f = 0; f < F; f++) {
			gptr << "\tu64 *G" << f << " = (u64*)a.w[" << cb + 3 << "] + ((u64)sidx * " << F << " + " << f << ") * " << D
			     << "ull;\n";
		}
		const int OUTD = cb + 8;
		// compaction of live groups into the outputs: `live` and `load` are per-slot code, `key`
		// the packed key of slot s; two passes with one output reservation per item
		auto compaction = [&](const std::string &live, const std::string &load, const std::string &reset) {
			std::ostringstream r;
			r << "\t{\n\tu32 mine = 0;\n"
			  << "\tfor (u32 c0 = warp * 32u; c0 < " << D << "u; c0 += nwarps * 32u) { const u32 s = c0 + lane; mine += __popc(__ballot_sync(0xffffffffu, "
			  << live << ")); }\n"
			  << "\tif (lane == 0) warp_live[warp] = mine;\n\t__syncthreads();\n"
			  << "\tu32 before = 0, total = 0;\n"
			  << "\tfor (u32 w_ = 0; w_ < nwarps; ++w_) { const u32 x_ = warp_live[w_]; before += w_ < warp ? x_ : 0u; total += x_; }\n"
			  << "\tif (threadIdx.x == 0) out_base = atomicAdd((unsigned long long*)a.w[" << cb + 6
			  << "], (unsigned long long)total);\n\t__syncthreads();\n"
			  << "\tu64 run = out_base + before;\n"
			  << "\tfor (u32 c0 = warp * 32u; c0 < " << D << "u; c0 += nwarps * 32u) {\n"
			  << "\t\tconst u32 s = c0 + lane;\n"
			  << "\t\tconst bool lv = " << live << ";\n"
			  << "\t\tconst u32 live_mask = __ballot_sync(0xffffffffu, lv);\n"
			  << "\t\tif (lv) {\n" << sdecl.str() << load
			  << "\t\t\tconst u64 pos = run + __popc(live_mask & ((1u << lane) - 1u));\n"
			  << "\t\t\tconst u64 key = vgpu_dunmix(a, ((u64)p << " << dbits << ") | s);\n"
			  << FinalizeCode(gb, fields, visible_, "S", "0", "key", "pos", OUTD) << reset << "\t\t}\n"
			  << "\t\trun += __popc(live_mask);\n\t}\n\t__syncthreads();\n\t}\n";
			return r.str();
		};
		std::ostringstream gload;
		for (int f = 0; f < F; f++) gload << "\t\t\tS" << f << "[0] = __ldcg(G" << f << " + s);\n";
		// Groups spanning 4+ lanes are combined one at a time by a full-warp xor butterfly in which the
		// group's lanes contribute their values and the others the identity: every lane ends with the
		// group total and the group's lowest lane keeps it. A step whose 32 rows share one key takes
		// exactly one butterfly; a step of distinct keys takes none.
		std::ostringstream tinit, txor, ttake;
		tinit << "\t\t\t\t\tu32 tc = mem ? gc : 0u;\n";
		txor << "\t\t\t\t\t\ttc += __shfl_xor_sync(0xffffffffu, tc, d);\n";
		ttake << "\t\t\t\t\t\tgc = tc;\n";
		for (int f = 1; f < F; f++) {
			const auto &fd = fields[f];
			const std::string fs = std::to_string(f);
			if (fd.kind == "f64") {
				tinit << "\t\t\t\t\tdouble tf" << fs << " = mem ? gf" << fs << " : 0.0;\n";
				txor << "\t\t\t\t\t\ttf" << fs << " += __shfl_xor_sync(0xffffffffu, tf" << fs << ", d);\n";
				ttake << "\t\t\t\t\t\tgf" << fs << " = tf" << fs << ";\n";
			} else if (fd.kind == "lo") {
				tinit << "\t\t\t\t\tu64 tlo" << fs << " = mem ? glo" << fs << " : 0ull; i64 thi" << fs << " = mem ? ghi" << fs
				      << " : 0;\n";
				txor << "\t\t\t\t\t\t{ const u64 ol_ = __shfl_xor_sync(0xffffffffu, tlo" << fs
				     << ", d); const i64 oh_ = __shfl_xor_sync(0xffffffffu, thi" << fs << ", d); const u64 nl_ = tlo" << fs
				     << " + ol_; thi" << fs << " += oh_ + (nl_ < tlo" << fs << " ? 1 : 0); tlo" << fs << " = nl_; }\n";
				ttake << "\t\t\t\t\t\tglo" << fs << " = tlo" << fs << "; ghi" << fs << " = thi" << fs << ";\n";
			} else if (fd.kind == "min" || fd.kind == "max") {
				const char *op = fd.kind == "min" ? "<" : ">";
				const char *ident = fd.kind == "min" ? "0x7fffffffffffffffLL" : "(-0x7fffffffffffffffLL - 1)";
				tinit << "\t\t\t\t\ti64 tm" << fs << " = mem ? gm" << fs << " : " << ident << ";\n";
				txor << "\t\t\t\t\t\t{ const i64 o_ = __shfl_xor_sync(0xffffffffu, tm" << fs << ", d); if (o_ " << op
				     << " tm" << fs << ") tm" << fs << " = o_; }\n";
				ttake << "\t\t\t\t\t\tgm" << fs << " = tm" << fs << ";\n";
			}
		}

		o << "__device__ __forceinline__ void vgpu_dslot_reset(const KArgs &a, char *sm, u32 s) {\n\t(void)a;\n" << decl.str() << reset_slot("s")
		  << "}\n\n";
		o << "__device__ __forceinline__ void vgpu_ditem(const KArgs &a, const uint4 it, char *sm) {\n"
		  << "\t__shared__ u32 warp_live[32];\n\t__shared__ u64 out_base;\n\t__shared__ bool last_chunk;\n"
		  << "\tconst u32 p = it.x, sidx = it.w;\n"
		  << "\tconst u64 start = it.y, end = it.z;\n"
		  << "\tconst char *recs = (const char*)a.w[" << cb + 2 << "];\n"
		  << "\tconst u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;\n"
		  << decl.str()
		  // hot run: the first key of a step whose group spans 8+ lanes; later groups of it add into lane
		  // 0's registers instead of the table (FP64 shared adds are CAS loops that serialize on one word)
		  << "\tu32 hot = ~0u; u64 wc = 0;\n" << wvars.str()
		  << "\tfor (u64 base = start + (u64)warp * 128ull; base < end; base += (u64)nwarps * 128ull) {\n"
		  << "\t\tu32 rw[4][" << RW << "];\n"
		  << "\t\t#pragma unroll\n\t\tfor (int q = 0; q < 4; ++q) {\n"
		  << "\t\t\tconst u64 i = base + 32ull * q + lane;\n"
		  << "\t\t\tload_record<" << RW << ">(recs + (i < end ? i : end - 1) * " << RS << ", rw[q]);\n\t\t}\n"
		  << "\t\t#pragma unroll\n\t\tfor (int q = 0; q < 4; ++q) {\n";
		if (gb.heavy_slots > 0) {
			// partial records of heavy keys: bit 31 of the key word, row count in the next word (0: the
			// key had no rows in that CTA, the record holds identities and is skipped)
			o << "\t\t\tconst bool part_rec = (rw[q][0] & 0x80000000u) != 0u;\n"
			  << "\t\t\tconst bool valid = base + 32ull * q + lane < end && !(part_rec && rw[q][1] == 0u);\n";
		} else {
			o << "\t\t\tconst bool valid = base + 32ull * q + lane < end;\n";
		}
		o << "\t\t\tconst u32 slot = valid ? (rw[q][0] & " << D - 1 << "u) : 0xffffffffu;\n";
		for (size_t i = 0; i < gb.aggs.size(); i++) {
			const auto &ag = gb.aggs[i];
			if (ag.column >= 0 && ag.kind != AggKind::COUNT && ag.kind != AggKind::COUNT_STAR) {
				o << "\t\t\tconst " << CudaTypeName(visible_[ag.column].type) << " v" << i << " = "
				  << rec_value(ag.column, "rw[q]") << ";\n";
			}
		}
		std::string gd = gdecl.str();
		if (gb.heavy_slots > 0) {
			const std::string one = "u32 gc = valid ? 1u : 0u;";
			gd.replace(gd.find(one), one.size(), "u32 gc = valid ? (part_rec ? rw[q][1] : 1u) : 0u;");
		}
		o << gd;
		if (gb.bucket_plain) {  // every record updates its slot itself: no warp grouping, no hot run
			o << "\t\t\tif (valid) {\n" << update("g", "slot") << "\t\t\t}\n";
		} else {
		o << "\t\t\tconst u32 peers = __match_any_sync(0xffffffffu, slot);\n"
		  << "\t\t\tbool leader = true;\n"
		  << "\t\t\tfor (u32 todo = __ballot_sync(0xffffffffu, __popc(peers) >= 4); todo;) {\n"
		  << "\t\t\t\tconst u32 src_ = __ffs(todo) - 1;\n"
		  << "\t\t\t\tconst u32 gmask = __shfl_sync(0xffffffffu, peers, src_);\n"
		  << "\t\t\t\tconst bool mem = (gmask >> lane) & 1u;\n"
		  << "\t\t\t\t{\n" << tinit.str()
		  << "\t\t\t\t\t#pragma unroll\n\t\t\t\t\tfor (int d = 16; d > 0; d >>= 1) {\n" << txor.str()
		  << "\t\t\t\t\t}\n"
		  << "\t\t\t\t\tif (mem) {\n" << ttake.str() << "\t\t\t\t\t\tleader = lane == src_;\n\t\t\t\t\t}\n"
		  << "\t\t\t\t}\n"
		  << "\t\t\t\ttodo &= ~gmask;\n"
		  << "\t\t\t}\n"
		  << "\t\t\tconst u32 hm = __ballot_sync(0xffffffffu, valid && leader && slot == hot);\n"
		  << "\t\t\tfor (u32 m_ = hm; m_; m_ &= m_ - 1) {\n"
		  << "\t\t\t\tconst u32 src_ = __ffs(m_) - 1; const bool have_ = lane == 0;\n" << wacc.str() << "\t\t\t}\n"
		  << "\t\t\tif (hm & (1u << lane)) leader = false;\n"
		  << "\t\t\tif (hot == ~0u) {\n"
		  << "\t\t\t\tconst u32 cand = __ballot_sync(0xffffffffu, valid && leader && __popc(peers) >= 8);\n"
		  << "\t\t\t\tif (cand) {\n"
		  << "\t\t\t\t\tconst u32 src_ = __ffs(cand) - 1; const bool have_ = lane == 0;\n"
		  << "\t\t\t\t\thot = __shfl_sync(0xffffffffu, slot, src_);\n" << wacc.str()
		  << "\t\t\t\t\tif (lane == src_) leader = false;\n"
		  << "\t\t\t\t}\n\t\t\t}\n"
		  << "\t\t\tif (valid && leader) {\n" << update("g", "slot") << "\t\t\t}\n";
		}
		o << "\t\t}\n\t}\n"
		  << "\tif (hot != ~0u && lane == 0) {\n" << update("w", "hot") << "\t}\n"
		  << (gb.f64_l2 ? "\t__threadfence();  // this thread's reductions are performed before the tables are read\n" : "")
		  << "\t__syncthreads();\n"
		  << "\tif (sidx == ~0u) {\n"
		  << compaction("DC[s] != 0u", load_slot("s"), reset_slot("s"))
		  << "\t\treturn;\n\t}\n"
		  << "\t// a chunk of a split partition: fold the table into the partition's global table; the last\n"
		  << "\t// chunk to finish writes the partition's groups\n"
		  << gptr.str()
		  << "\tfor (u32 s = threadIdx.x; s < " << D << "u; s += blockDim.x) {\n"
		  << "\t\tif (DC[s] != 0u) {\n" << sdecl.str() << load_slot("s") << MergeCode(fields, "S", "0", "G", "s")
		  << reset_slot("s") << "\t\t}\n\t}\n"
		  << "\t__threadfence();\n\t__syncthreads();\n"
		  << "\tif (threadIdx.x == 0) {\n"
		  << "\t\tu32 *info = (u32*)a.w[" << cb + 4 << "] + 2ull * sidx;\n"
		  << "\t\tlast_chunk = atomicAdd(info + 1, 1u) + 1u == info[0];\n\t}\n"
		  << "\t__syncthreads();\n"
		  << "\tif (!last_chunk) return;\n"
		  << "\t__threadfence();\n"
		  << compaction("__ldcg(G0 + s) != 0ull", gload.str(), "")
		  << "}\n\n";
		// global tables of split partitions: identity values
		o << "extern \"C\" __global__ void vgpu_gb_dtab_init(KArgs a) {\n"
		  << "\tu64 *g = (u64*)a.w[" << cb + 3 << "];\n"
		  << "\tconst u64 total = (u64)*(const u32*)a.w[" << cb + 7 << "] * " << F * D << "ull;\n"
		  << "\tfor (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < total; i += (u64)gridDim.x * blockDim.x) {\n"
		  << "\t\tconst u32 f = (u32)((i / " << D << "ull) % " << F << "u);\n"
		  << "\t\tu64 v = 0ull;\n";
		for (int f = 0; f < F; f++) {
			o << "\t\tif (f == " << f << "u) v = " << InitValue(fields[f]) << ";\n";
		}
		o << "\t\tg[i] = v;\n\t}\n}\n\n";
		o << "extern \"C\" __global__ void __launch_bounds__(" << gb.bucket_threads << ") vgpu_gb_dbucket(KArgs a) {\n"
		  << "\textern __shared__ __align__(16) char vgpu_dsm[];\n"
		  << "\t__shared__ u32 cur;\n"
		  << "\tfor (u32 s = threadIdx.x; s < " << D << "u; s += blockDim.x) vgpu_dslot_reset(a, vgpu_dsm, s);\n"
		  << "\tconst u32 n_items = *(const u32*)a.w[" << cb + 1 << "];\n"
		  << "\tconst uint4 *items = (const uint4*)a.w[" << cb << "];\n"
		  << "\twhile (true) {\n"
		  << "\t\tif (threadIdx.x == 0) cur = atomicAdd((u32*)a.w[" << cb + 5 << "], 1u);\n"
		  << (gb.f64_l2 ? "\t\t__threadfence();  // resets of the global sums land before the next reductions\n" : "")
		  << "\t\t__syncthreads();\n"
		  << "\t\tconst u32 i = cur;\n"
		  << "\t\t__syncthreads();\n"
		  << "\t\tif (i >= n_items) break;\n"
		  << "\t\tvgpu_ditem(a, items[i], vgpu_dsm);\n"
		  << "\t}\n}\n";
		return o.str();
	}
	o << "__device__ __forceinline__ int vgpu_find_slot(u64 *K, u32 C, u64 key, u32 limit) {\n"
	  << "\tu32 slot = (u32)mix64(key) & (C - 1);\n"
	  << "\tfor (u32 probe = 0; probe < limit; ++probe) {\n"
	  << "\t\tconst u64 cur = *(volatile u64*)&K[slot];\n"
	  << "\t\tif (cur == key) return (int)slot;\n"
	  << "\t\tif (cur == ~0ull) {\n"
	  << "\t\t\tconst u64 prev = atomicCAS((unsigned long long*)&K[slot], ~0ull, key);\n"
	  << "\t\t\tif (prev == ~0ull || prev == key) return (int)slot;\n"
	  << "\t\t}\n"
	  << "\t\tslot = (slot + 1) & (C - 1);\n"
	  << "\t}\n\treturn -1;\n}\n\n";
	{
		o << "__device__ __forceinline__ void vgpu_table_reset(u64 *tab, u32 C, u32 s) {\n\ttab[s] = ~0ull;\n";
		for (int f = 0; f < F; f++) {
			o << "\ttab[(u64)" << f + 1 << " * C + s] = " << InitValue(fields[f]) << ";\n";
		}
		o << "}\n\n__device__ __forceinline__ void vgpu_table_init(u64 *tab, u32 C) {\n"
		  << "\tfor (u32 s = threadIdx.x; s < C; s += blockDim.x) vgpu_table_reset(tab, C, s);\n\t__syncthreads();\n}\n\n";
	}
	// probe runs longer than `limit` count as overflow: shared-memory tables give up after 64 probes
	// (the partition is then retried with a larger table), global-memory tables probe all C slots
	o << "__device__ __forceinline__ void vgpu_bucket_process(const KArgs &a, u32 p, u64 *tab, u32 C, u32 limit, bool *overflow) {\n"
	  << "\tconst u32 P = (u32)a.w[" << cb << "];\n"
	  << "\tconst u32 *offsets = (const u32*)a.w[" << cb + 2 << "];\n"
	  << "\tconst u64 G = a.w[" << cb + 3 << "];\n"
	  << "\tconst u32 total_rows = *(const u32*)a.w[" << cb + 4 << "];\n"
	  << "\tconst char *recs = (const char*)a.w[" << cb + 5 << "];\n"
	  << "\tconst u64 start = offsets[(u64)p * G];\n"
	  << "\tconst u64 end = (p + 1 < P) ? offsets[(u64)(p + 1) * G] : total_rows;\n"
	  << "\tconst u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;\n"
	  << "\tconst long long dbg_t0 = clock64();\n"
	  << "\tu64 *K = tab;\n";
	for (int f = 0; f < F; f++) {
		o << "\tu64 *T" << f << " = tab + (u64)" << f + 1 << " * C;\n";
	}
	// The table is clean on entry (vgpu_table_init once per CTA; compaction resets what it visits).
	// A warp keeps up to 8 pending runs for frequent keys: entry j lives in lane j (key my_pk, totals in
	// its w* registers; every lane holds the 8 keys in pk_). A key is adopted once one of its groups
	// spans 3 lanes of a step; later groups of that key are added in registers, so frequent keys cost no
	// table atomics until the partition ends (64-bit and FP64 shared atomics are CAS loops that
	// serialize badly on one hot word).
	o << wdecl.str()
	  << "\tfor (u64 base = start + (u64)warp * 128ull; base < end; base += (u64)nwarps * 128ull) {\n"
	  << "\t\t// this table cannot hold the partition: stop early (one decision per warp, so the warp's\n"
	  << "\t\t// lanes never split across the full-warp match/ballot/shuffle operations below)\n"
	  << "\t\tif (__any_sync(0xffffffffu, *(volatile bool *)overflow)) break;\n"
	  << "\t\tu32 rw[4][" << RW << "];\n"
	  << "\t\t#pragma unroll\n\t\tfor (int q = 0; q < 4; ++q) {\n"
	  << "\t\t\tconst u64 i = base + 32ull * q + lane;\n"
	  << "\t\t\tload_record<" << RW << ">(recs + (i < end ? i : end - 1) * " << RS << ", rw[q]);\n\t\t}\n"
	  << "\t\t#pragma unroll\n\t\tfor (int q = 0; q < 4; ++q) {\n"
	  << "\t\t\tconst bool valid = base + 32ull * q + lane < end;\n"
	  << "\t\t\tconst u64 key = valid ? ((u64)rw[q][0] | ((u64)rw[q][1] << 32)) : ~0ull;\n";
	for (size_t i = 0; i < gb.aggs.size(); i++) {
		const auto &ag = gb.aggs[i];
		if (ag.column >= 0 && ag.kind != AggKind::COUNT && ag.kind != AggKind::COUNT_STAR) {
			o << "\t\t\tconst " << CudaTypeName(visible_[ag.column].type) << " v" << i << " = "
			  << rec_value(ag.column, "rw[q]") << ";\n";
		}
	}
	o << gdecl.str()
	  << "\t\t\tconst u32 peers = __match_any_sync(0xffffffffu, key);\n"
	  << "\t\t\tbool leader = true;\n"
	  << "\t\t\tif (peers == 0xffffffffu) {\n"
	  << "\t\t\t\t#pragma unroll\n\t\t\t\tfor (int d = 16; d > 0; d >>= 1) {\n" << gxor.str() << "\t\t\t\t}\n"
	  << "\t\t\t\tleader = lane == 0;\n"
	  << "\t\t\t} else if (__ballot_sync(0xffffffffu, __popc(peers) >= 4)) {\n"
	  << "\t\t\t\tconst u32 rank = __popc(peers & ((1u << lane) - 1u));\n"
	  << "\t\t\t\tconst u32 size = __popc(peers);\n"
	  << "\t\t\t\t#pragma unroll\n\t\t\t\tfor (u32 d = 1; d < 32; d <<= 1) {\n"
	  << "\t\t\t\t\tconst u32 want = rank + d;\n"
	  << "\t\t\t\t\tconst bool take = ((rank & (2 * d - 1)) == 0) && want < size;\n"
	  << "\t\t\t\t\tconst u32 src_ = want < size ? __fns(peers, 0, (int)want + 1) : lane;\n"
	  << gcomb.str()
	  << "\t\t\t\t}\n"
	  << "\t\t\t\tleader = rank == 0;\n"
	  << "\t\t\t}\n"
	  << "\t\t\t// groups whose key is pending hand their totals to the entry's lane\n"
	  << "\t\t\tint pidx = -1;\n"
	  << "\t\t\t#pragma unroll\n\t\t\tfor (int j = 0; j < 8; ++j) pidx = (valid && key == pk_[j]) ? j : pidx;\n"
	  << "\t\t\tconst bool absorb = valid && leader && pidx >= 0;\n"
	  << "\t\t\t// one pass per absorbing lane (warp-uniform count): every one of them is added\n"
	  << "\t\t\tfor (u32 am_ = __ballot_sync(0xffffffffu, absorb); am_; am_ &= am_ - 1) {\n"
	  << "\t\t\t\tconst u32 src_ = __ffs(am_) - 1;\n"
	  << "\t\t\t\tconst bool have_ = (int)lane == __shfl_sync(0xffffffffu, pidx, src_);\n" << wacc.str()
	  << "\t\t\t}\n"
	  << "\t\t\tif (absorb) leader = false;\n"
	  << "\t\t\t// adopt one new frequent key per step while entries are free\n"
	  << "\t\t\tif (free_mask) {\n"
	  << "\t\t\t\tconst u32 cand = __ballot_sync(0xffffffffu, valid && leader && __popc(peers) >= 3);\n"
	  << "\t\t\t\tif (cand) {\n"
	  << "\t\t\t\t\tconst u32 c_ = __ffs(cand) - 1, e_ = __ffs(free_mask) - 1;\n"
	  << "\t\t\t\t\tconst u64 nk_ = __shfl_sync(0xffffffffu, key, c_);\n"
	  << "\t\t\t\t\t#pragma unroll\n\t\t\t\t\tfor (int j = 0; j < 8; ++j) if ((u32)j == e_) pk_[j] = nk_;\n"
	  << "\t\t\t\t\tfree_mask &= ~(1u << e_);\n"
	  << "\t\t\t\t\tconst u32 src_ = c_; const bool have_ = lane == e_;\n"
	  << "\t\t\t\t\tif (have_) my_pk = nk_;\n" << wacc.str()
	  << "\t\t\t\t\tif (lane == c_) leader = false;\n"
	  << "\t\t\t\t}\n"
	  << "\t\t\t}\n"
	  << "\t\t\tif (valid && leader) {\n"
	  << "\t\t\t\tconst int s_ = vgpu_find_slot(K, C, key, limit);\n"
	  << "\t\t\t\tif (s_ < 0) { *overflow = true; } else {\n"
	  << gupd.str() << "\t\t\t\t}\n\t\t\t}\n\t\t}\n\t}\n"
	  << "\tif (my_pk != ~0ull) {\n"
	  << "\t\tconst int s_ = vgpu_find_slot(K, C, my_pk, limit);\n"
	  << "\t\tif (s_ < 0) { *overflow = true; } else {\n" << wflush.str() << "\t\t}\n\t}\n"
	  << "\t__syncthreads();\n"
	  << "\tconst long long dbg_t1 = clock64();\n"
	  << "\tif (*overflow) { vgpu_table_init(tab, C); return; }\n"
	  << "\t// compaction: 32-slot chunks round-robin over warps; pass 1 counts live slots per warp, one\n"
	  << "\t// reservation for the partition, pass 2 writes each live slot and resets it for the next one\n"
	  << "\t__shared__ u32 warp_live[32];\n\t__shared__ u64 out_base;\n"
	  << "\tu32 mine = 0;\n"
	  << "\tfor (u32 c0 = warp * 32u; c0 < C; c0 += nwarps * 32u) mine += __popc(__ballot_sync(0xffffffffu, K[c0 + lane] != ~0ull));\n"
	  << "\tif (lane == 0) warp_live[warp] = mine;\n"
	  << "\t__syncthreads();\n"
	  << "\tu32 before = 0, total = 0;\n"
	  << "\tfor (u32 w_ = 0; w_ < nwarps; ++w_) { const u32 x_ = warp_live[w_]; before += w_ < warp ? x_ : 0u; total += x_; }\n"
	  << "\tif (threadIdx.x == 0) out_base = atomicAdd((unsigned long long*)a.w[" << W + 3
	  << "], (unsigned long long)total);\n"
	  << "\t__syncthreads();\n"
	  << "\tu64 run = out_base + before;\n"
	  << "\tfor (u32 c0 = warp * 32u; c0 < C; c0 += nwarps * 32u) {\n"
	  << "\t\tconst u32 s = c0 + lane;\n"
	  << "\t\tconst u64 key = K[s];\n"
	  << "\t\tconst u32 live_mask = __ballot_sync(0xffffffffu, key != ~0ull);\n"
	  << "\t\tif (key != ~0ull) {\n"
	  << "\t\t\tconst u64 pos = run + __popc(live_mask & ((1u << lane) - 1u));\n"
	  << FinalizeCode(gb, fields, visible_, "T", "s", "key", "pos", OUT)
	  << "\t\t\tvgpu_table_reset(tab, C, s);\n\t\t}\n"
	  << "\t\trun += __popc(live_mask);\n\t}\n\t__syncthreads();\n"
	  << "\t// optional per-partition diagnostics (rows, groups, row-loop and compaction cycles, block)\n"
	  << "\tif (threadIdx.x == 0 && a.w[" << kDebugWord << "]) {\n"
	  << "\t\tu64 *d = (u64*)a.w[" << kDebugWord << "] + 8ull * p;\n"
	  << "\t\td[0] = end - start; d[1] = total; d[2] = (u64)(dbg_t1 - dbg_t0); d[3] = (u64)(clock64() - dbg_t1);\n"
	  << "\t\td[4] = blockIdx.x; d[5] = blockDim.x;\n\t}\n"
	  << "}\n\n";

	const int L = OUT + out_words;
	// Tier 1: every partition, small shared-memory table (C from the arguments, any block size).
	// Partitions it cannot hold go to a device-side retry list instead of failing.
	o << "extern \"C\" __global__ void __launch_bounds__(" << gb.bucket_threads << ") vgpu_gb_bucket(KArgs a) {\n"
	  << "\textern __shared__ __align__(16) u64 vgpu_tab[];\n"
	  << "\t__shared__ u32 cur_p;\n\t__shared__ bool overflow;\n"
	  << "\tconst u32 P = (u32)a.w[" << cb << "]; const u32 C = (u32)a.w[" << cb + 1 << "];\n"
	  << "\tu32 next_p = 0;\n"
	  << "\tif (threadIdx.x == 0) { cur_p = atomicAdd((u32*)a.w[" << W << "], 1u); overflow = false; }\n"
	  << "\tvgpu_table_init(vgpu_tab, C);\n"
	  << "\twhile (true) {\n"
	  << "\t\tconst u32 p = cur_p;\n"
	  << "\t\tif (p >= P) break;\n"
	  << "\t\t// the next partition's index is claimed now; its result is only needed after this one\n"
	  << "\t\tif (threadIdx.x == 0) next_p = atomicAdd((u32*)a.w[" << W << "], 1u);\n"
	  << "\t\tvgpu_bucket_process(a, p, vgpu_tab, C, C < 64u ? C : 64u, &overflow);\n"
	  << "\t\tif (threadIdx.x == 0) {\n"
	  << "\t\t\tif (overflow) { ((u32*)a.w[" << L + 5 << "])[atomicAdd((u32*)a.w[" << L + 6 << "], 1u)] = p; }\n"
	  << "\t\t\toverflow = false;\n\t\t\tcur_p = next_p;\n\t\t}\n"
	  << "\t\t__syncthreads();\n\t}\n}\n\n";

	// Tier 2: the retry list with the largest shared-memory table (C2). Partitions that still do not
	// fit are flagged for the host's global-memory pass.
	o << "extern \"C\" __global__ void __launch_bounds__(512, 1) vgpu_gb_bucket_retry(KArgs a) {\n"
	  << "\textern __shared__ __align__(16) u64 vgpu_tab[];\n"
	  << "\t__shared__ u32 cur_i;\n\t__shared__ bool overflow;\n"
	  << "\tconst u32 C = (u32)a.w[" << L + 8 << "];\n"
	  << "\tconst u32 n_retry = *(volatile u32*)a.w[" << L + 6 << "];\n"
	  << "\tif (n_retry == 0) return;\n"
	  << "\tvgpu_table_init(vgpu_tab, C);\n"
	  << "\twhile (true) {\n"
	  << "\t\tif (threadIdx.x == 0) { cur_i = atomicAdd((u32*)a.w[" << L + 7 << "], 1u); overflow = false; }\n"
	  << "\t\t__syncthreads();\n"
	  << "\t\tconst u32 i = cur_i;\n"
	  << "\t\tif (i >= n_retry) break;\n"
	  << "\t\tconst u32 p = ((const u32*)a.w[" << L + 5 << "])[i];\n"
	  << "\t\tvgpu_bucket_process(a, p, vgpu_tab, C, C < 64u ? C : 64u, &overflow);\n"
	  << "\t\tif (threadIdx.x == 0 && overflow) { ((u32*)a.w[" << W + 1 << "])[p] = 1u; atomicAdd((u32*)a.w[" << W + 2
	  << "], 1u); }\n"
	  << "\t\t__syncthreads();\n\t}\n}\n\n";

	o << "extern \"C\" __global__ void __launch_bounds__(512, 1) vgpu_gb_bucket_global(KArgs a) {\n"
	  << "\t__shared__ bool overflow;\n"
	  << "\tconst u32 *list = (const u32*)a.w[" << L << "];\n"
	  << "\tconst u32 nlist = (u32)a.w[" << L + 1 << "];\n"
	  << "\tu64 *tables = (u64*)a.w[" << L + 2 << "];\n"
	  << "\tconst u64 *tab_off = (const u64*)a.w[" << L + 3 << "];\n"
	  << "\tconst u32 *caps = (const u32*)a.w[" << L + 4 << "];\n"
	  << "\tfor (u32 e = blockIdx.x; e < nlist; e += gridDim.x) {\n"
	  << "\t\tif (threadIdx.x == 0) overflow = false;\n"
	  << "\t\tvgpu_table_init(tables + tab_off[e], caps[e]);\n"
	  << "\t\tvgpu_bucket_process(a, list[e], tables + tab_off[e], caps[e], caps[e], &overflow);\n"
	  << "\t\tif (threadIdx.x == 0 && overflow) atomicAdd((u32*)a.w[" << W + 2 << "], 1u);\n"
	  << "\t\t__syncthreads();\n\t}\n}\n";
	return o.str();
}

std::string PipelineCodegen::EmitBatchGroupBy(const GroupBySpec &gb, const Geometry &g, int tile_rows, int smem_slots,
                                              const BatchLayout &L) const {
	// One kernel for every query of a batch that shares this plan template. Query q's columns, key
	// packing, table placement and literal constants come from its row of the query table (L.qwords
	// u64 words): [0] rows, [1+2i] source i data, [2+2i] source i validity (unused), [key_base+2j]
	// key j minimum, [key_base+2j+1] key j shift | bits << 8, [dom_base] table slots D,
	// [dom_base+1] accumulator offset, [dom_base+2] output row offset, [dom_base+3] 1 = shared-memory
	// table, [param_base..] the literal constants as 64-bit patterns.
	// vgpu_batch_gb args: w[0] queries, w[1] query table, w[2] tiles (uint2 query, tile), w[3] tiles,
	//   w[4] tile work counter (u32*, zero at launch), w[5] accumulators (u64, F arrays of w[6] words), w[6] accumulator words
	//   per field, w[7] output pointer table (u64 [out words]), w[8] group counts (u64 [queries]).
	std::ostringstream o;
	o << Prologue();
	o << "#define vgpu_qpd(j) __longlong_as_double((long long)vgpu_qp[(j)])\n"
	  << "#define vgpu_qpf(j) __int_as_float((int)(u32)vgpu_qp[(j)])\n"
	  << "#define vgpu_qpi(j) ((int)(long long)vgpu_qp[(j)])\n"
	  << "#define vgpu_qpu(j) ((unsigned)vgpu_qp[(j)])\n"
	  << "#define vgpu_qpl(j) ((long long)vgpu_qp[(j)])\n"
	  << "#define vgpu_qpul(j) ((unsigned long long)vgpu_qp[(j)])\n\n";
	const auto fields = StateFields(gb);
	const int F = static_cast<int>(fields.size());
	std::vector<int> used;
	for (auto &k : gb.keys) used.push_back(k.column);
	for (auto &a : gb.aggs) {
		if (a.column >= 0) used.push_back(a.column);
	}
	auto needed = NeededSources(used);
	std::ostringstream pack;
	pack << "(0ull";
	for (size_t j = 0; j < gb.keys.size(); j++) {
		const auto &k = gb.keys[j];
		pack << " | ((u64)((i64)(" << visible_[k.column].value << ") - (i64)qp[" << L.key_base + 2 * j
		     << "]) << ((u32)qp[" << L.key_base + 2 * j + 1 << "] & 0xffu))";
	}
	pack << ")";
	std::vector<std::string> values;
	for (auto &a : gb.aggs) values.push_back(a.column >= 0 ? visible_[a.column].value : "0");
	const int T = smem_slots;
	o << "extern \"C\" __global__ void __launch_bounds__(" << g.block << ") vgpu_batch_gb(KArgs a) {\n"
	  << "\textern __shared__ __align__(16) u64 vgpu_smem[];\n"
	  << "\tconst u64 *qtab = (const u64*)a.w[1];\n"
	  << "\tconst uint2 *tiles = (const uint2*)a.w[2];\n"
	  << "\tconst u64 ntiles = a.w[3];\n\tu32 *work = (u32*)a.w[4];\n\t__shared__ u32 cur_t;\n"
	  << "\tu64 *acc = (u64*)a.w[5];\n\tconst u64 ACC = a.w[6];\n";
	for (int f = 0; f < F; f++) o << "\tu64 *T" << f << " = vgpu_smem + " << f * T << ";\n";
	o << "\tfor (u32 s = threadIdx.x; s < " << T << "u; s += blockDim.x) {\n";
	for (int f = 0; f < F; f++) o << "\t\tT" << f << "[s] = " << InitValue(fields[f]) << ";\n";
	o << "\t}\n\t__syncthreads();\n"
	  << "\tu32 cur_q = 0xffffffffu; bool cur_sm = false; u64 cur_d = 0;\n";
	for (int f = 0; f < F; f++) o << "\tu64 *G" << f << " = acc;\n";
	std::ostringstream flush;
	flush << "\t\t\t__syncthreads();\n"
	      << "\t\t\tfor (u32 s = threadIdx.x; s < (u32)cur_d; s += blockDim.x) {\n\t\t\t\tif (T0[s] != 0) {\n"
	      << MergeCode(fields, "T", "s", "G", "s");
	for (int f = 0; f < F; f++) flush << "\t\t\t\tT" << f << "[s] = " << InitValue(fields[f]) << ";\n";
	flush << "\t\t\t\t}\n\t\t\t}\n\t\t\t__syncthreads();\n";
	// tiles are claimed one at a time from a counter (queries differ in size by orders of magnitude;
	// the queue lists the largest queries first)
	o << "\twhile (true) {\n"
	  << "\t\tif (threadIdx.x == 0) cur_t = atomicAdd(work, 1u);\n"
	  << "\t\t__syncthreads();\n"
	  << "\t\tconst u64 t = cur_t;\n"
	  << "\t\t__syncthreads();\n"
	  << "\t\tif (t >= ntiles) break;\n"
	  << "\t\tconst uint2 tl = tiles[t];\n"
	  << "\t\tconst u64 *qp = qtab + (u64)tl.x * " << L.qwords << "ull;\n"
	  << "\t\tif (tl.x != cur_q) {\n"
	  << "\t\t\t// the CTA moves to another query: its shared table goes to the previous query's accumulators\n"
	  << "\t\t\tif (cur_sm) {\n" << flush.str() << "\t\t\t}\n"
	  << "\t\t\tcur_q = tl.x; cur_d = qp[" << L.dom_base << "]; cur_sm = qp[" << L.dom_base + 3 << "] != 0;\n";
	for (int f = 0; f < F; f++) {
		o << "\t\t\tG" << f << " = acc + " << f << "ull * ACC + qp[" << L.dom_base + 1 << "];\n";
	}
	o << "\t\t}\n"
	  << "\t\tconst u64 *vgpu_qp = qp + " << L.param_base << ";\n\t\t(void)vgpu_qp;\n"
	  << "\t\tconst u64 n = qp[0];\n"
	  << "\t\tconst u64 t0 = (u64)tl.y * " << tile_rows << "ull;\n"
	  << "\t\tconst u64 t1 = t0 + " << tile_rows << "ull < n ? t0 + " << tile_rows << "ull : n;\n"
	  << "\t\tfor (u64 sub = t0; sub < t1; sub += " << g.tile() << "ull) {\n"
	  << "\t\tconst u64 row0 = sub + (u64)threadIdx.x * " << g.items << ";\n";
	for (size_t i = 0; i < spec_.sources.size(); i++) {
		if (!needed[i]) continue;
		const char *t = CudaTypeName(spec_.sources[i].type);
		o << "\t\t" << t << " s" << i << "[" << g.items << "];\n"
		  << "\t\tload_rows<" << t << ", " << g.items << ">((const " << t << "*)qp[" << 1 + 2 * i << "], row0, t1, s" << i
		  << ");\n";
	}
	o << "\t\t#pragma unroll\n\t\tfor (int r = 0; r < " << g.items << "; ++r) {\n"
	  << "\t\tconst u64 row = row0 + r; (void)row;\n\t\tbool keep = row < t1;\n"
	  << chain_code_ << "\t\tif (keep) {\n"
	  << "\t\t\tconst u64 slot = " << pack.str() << ";\n"
	  << "\t\t\tif (cur_sm) {\n" << UpdateCode(fields, "T", "slot", values, true) << "\t\t\t} else {\n"
	  << UpdateCode(fields, "G", "slot", values, false) << "\t\t\t}\n"
	  << "\t\t}\n\t\t}\n\t\t}\n\t}\n"
	  << "\tif (cur_sm) {\n" << flush.str() << "\t}\n}\n\n";

	// accumulators to identity (first use of a batch's buffers; the final kernel resets what it reads)
	o << "extern \"C\" __global__ void vgpu_batch_init(KArgs a) {\n"
	  << "\tu64 *acc = (u64*)a.w[5];\n\tconst u64 ACC = a.w[6];\n"
	  << "\tfor (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < " << F
	  << "ull * ACC; i += (u64)gridDim.x * blockDim.x) {\n\t\tconst u64 f = i / ACC;\n\t\tu64 v = 0ull;\n";
	for (int f = 0; f < F; f++) o << "\t\tif (f == " << f << "ull) v = " << InitValue(fields[f]) << ";\n";
	o << "\t\tacc[i] = v;\n\t}\n}\n\n";

	// one CTA per query: its live slots, in key order, into the outputs; the accumulators are reset
	GroupBySpec aggs_only = gb;
	aggs_only.keys.clear();
	const int nk = static_cast<int>(gb.keys.size());
	o << "extern \"C\" __global__ void __launch_bounds__(1024) vgpu_batch_final(KArgs a) {\n"
	  << "\t__shared__ u32 scan_scratch[33];\n"
	  << "\tconst u32 q = blockIdx.x;\n"
	  << "\tconst u64 *qp = (const u64*)a.w[1] + (u64)q * " << L.qwords << "ull;\n"
	  << "\tu64 *acc = (u64*)a.w[5];\n\tconst u64 ACC = a.w[6];\n"
	  << "\tconst u64 *outp = (const u64*)a.w[7];\n"
	  << "\tconst u64 D = qp[" << L.dom_base << "], outb = qp[" << L.dom_base + 2 << "];\n";
	for (int f = 0; f < F; f++) o << "\tu64 *G" << f << " = acc + " << f << "ull * ACC + qp[" << L.dom_base + 1 << "];\n";
	o << "\tu64 base = 0;\n"
	  << "\tfor (u64 c0 = 0; c0 < D; c0 += blockDim.x) {\n"
	  << "\t\tconst u64 s = c0 + threadIdx.x;\n"
	  << "\t\tconst bool live = s < D && G0[s] != 0;\n"
	  << "\t\tu32 total; const u32 off = block_exclusive_scan(live ? 1u : 0u, scan_scratch, &total);\n"
	  << "\t\tif (live) {\n\t\t\tconst u64 pos = outb + base + off;\n\t\t\tconst u64 key = s;\n";
	for (int j = 0; j < nk; j++) {
		const char *t = CudaTypeName(visible_[gb.keys[j].column].type);
		o << "\t\t\t{ const u32 sb = (u32)qp[" << L.key_base + 2 * j + 1 << "]; const u32 bits = sb >> 8;\n"
		  << "\t\t\t  const u64 mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1ull);\n"
		  << "\t\t\t  ((" << t << "*)outp[" << j << "])[pos] = (" << t << ")((i64)((key >> (sb & 0xffu)) & mask) + (i64)qp["
		  << L.key_base + 2 * j << "]); }\n";
	}
	o << FinalizeCode(aggs_only, fields, visible_, "G", "s", "key", "pos", nk, "outp") << "\t\t}\n"
	  << "\t\tif (s < D) {\n";
	for (int f = 0; f < F; f++) o << "\t\t\tG" << f << "[s] = " << InitValue(fields[f]) << ";\n";
	o << "\t\t}\n\t\tbase += total;\n\t}\n"
	  << "\tif (threadIdx.x == 0) ((u64*)a.w[8])[q] = base;\n}\n";
	return o.str();
}

std::string SpecKey(const PipelineSpec &spec) {
	std::ostringstream o;
	o << "src:";
	for (auto &sc : spec.sources) {
		o << sc.name << '/' << static_cast<int>(sc.type) << '/' << sc.nullable << '/' << sc.side << ';';
	}
	o << "|cross:" << spec.cross << "|join:" << spec.join << '/' << spec.join_key << '/' << spec.join_inline << '/' << spec.join_multi << '/' << spec.join_minline << "|chain:";
	for (const PlanNode *n : spec.chain) {
		o << static_cast<int>(n->op) << '{';
		for (auto &e : n->expressions) {
			o << static_cast<int>(e.output_type) << ':' << e.source.size() << ':' << e.source << '(';
			for (auto &in : e.input_columns) o << in << ',';
			o << ')';
		}
		o << '}';
	}
	return o.str();
}

std::string GroupByKey(const PipelineCodegen::GroupBySpec &gb, bool partitioned) {
	std::ostringstream o;
	o << "gb:" << partitioned << "|keys:";
	for (auto &k : gb.keys) o << k.column << ',';
	o << "|aggs:";
	for (auto &a : gb.aggs) {
		o << static_cast<int>(a.kind) << '/' << a.column << '/' << static_cast<int>(a.input_type) << '/'
		  << static_cast<int>(a.output_type) << '/' << a.narrow_word << ';';
	}
	o << "|db:" << gb.direct_bits << "|bt:" << gb.bucket_threads << "|hv:" << gb.heavy_slots << "|f64l2:" << gb.f64_l2 << "|hw:" << gb.heavy_warp << "|bp:" << gb.bucket_plain << "|nc:" << gb.narrow_count << "|cf:" << gb.count_as_flag << "|c32:" << gb.count32;
	return o.str();
}

std::shared_ptr<const PipelineCodegen> CodegenFor(const PipelineSpec &spec) {
	static std::mutex mu;
	static std::map<std::string, std::shared_ptr<const PipelineCodegen>> memo;
	const std::string key = SpecKey(spec);
	{
		std::lock_guard<std::mutex> lock(mu);
		auto it = memo.find(key);
		if (it != memo.end()) return it->second;
	}
	auto cg = std::make_shared<const PipelineCodegen>(spec);
	std::lock_guard<std::mutex> lock(mu);
	if (memo.size() >= 4096) memo.clear();  // bounded: plan shapes seen by one process are few
	memo.emplace(key, cg);
	return cg;
}

} // namespace vgpu
