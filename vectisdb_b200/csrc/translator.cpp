// translator.cpp -- bound expression tree -> the CUDA statement the engine's plans carry.
//
// The reference's DuckDB extension lowers each bound expression (BoundColumnRef, BoundConstant,
// BoundComparison, BoundFunction) into one C statement `((T*)out)[idx] = ...;` that reads
// `((const T*)inputs[i])[row]` (extension/src/expression_translator.cpp:287-460, 489-493). The same
// rules are restated here over a plain-data tree (vgpu_bexpr, include/vgpu.h) so a host that binds
// SQL itself -- DuckDB's optimizer hook, or any other planner -- gets the statement text, the ordered
// input columns and the output type the engine's expression contract expects:
//   - column references read [row] (the original row under late materialization), one inputs[] slot
//     per distinct column, in first-reference order;
//   - constants: INT16/INT32 plain, INT64 with LL, FLOAT with a decimal point and f (9 digits), DOUBLE
//     with 17 digits, BOOLEAN true/false; NULL and non-finite constants are refused;
//   - comparisons `(l op r)`; arithmetic `(l op r)` and unary minus `(-x)`; `%` on floats as fmod;
//   - casts only where the C conversion agrees with DuckDB's CAST (widening integers, integer or
//     BOOLEAN to floating, FLOAT to DOUBLE); narrowing and float->integer are refused;
//   - DOUBLE math functions by DuckDB name (ln -> log, log -> log10, ceiling -> ceil, ...), abs kept
//     in its input type; with the FP32 relaxation flag they run in float, with the strict-FP flag only
//     the correctly rounded ones (sqrt, floor, ceil, radians, degrees) are accepted.
#include <cmath>
#include <cstring>
#include <iomanip>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include "translator.hpp"

namespace vgpu {

namespace {

const char *TypeNameOrRefuse(ValueType t) {
	if (t == ValueType::DICTIONARY_STRING || t == ValueType::HUGEINT) {
		Fail(VGPU_ERR_UNSUPPORTED, std::string("expression_translator: ") +
		                               (t == ValueType::HUGEINT ? "HUGEINT" : "dictionary string") +
		                               " values are not usable in a fused arithmetic/comparison expression");
	}
	return CudaTypeName(t);
}

bool CastAgrees(ValueType from, ValueType to) {
	if (from == to) return true;
	switch (from) {
	case ValueType::BOOLEAN:
	case ValueType::INT16:
		return to == ValueType::INT32 || to == ValueType::INT64 || to == ValueType::FLOAT32 || to == ValueType::FLOAT64;
	case ValueType::INT32:
		return to == ValueType::INT64 || to == ValueType::FLOAT32 || to == ValueType::FLOAT64;
	case ValueType::INT64:
		return to == ValueType::FLOAT32 || to == ValueType::FLOAT64;
	case ValueType::FLOAT32:
		return to == ValueType::FLOAT64;
	default:
		return false;
	}
}

const char *MathFunction(const std::string &name, size_t arity, bool fp32) {
	static const std::map<std::string, std::pair<const char *, const char *>> unary = {
	    {"sqrt", {"sqrt", "sqrtf"}},   {"exp", {"exp", "expf"}},       {"ln", {"log", "logf"}},
	    {"log10", {"log10", "log10f"}}, {"log", {"log10", "log10f"}},   {"log2", {"log2", "log2f"}},
	    {"sin", {"sin", "sinf"}},      {"cos", {"cos", "cosf"}},       {"tan", {"tan", "tanf"}},
	    {"asin", {"asin", "asinf"}},   {"acos", {"acos", "acosf"}},    {"atan", {"atan", "atanf"}},
	    {"floor", {"floor", "floorf"}}, {"ceil", {"ceil", "ceilf"}},   {"ceiling", {"ceil", "ceilf"}},
	    {"radians", {"__vgpu_radians", "__vgpu_radians"}}, {"degrees", {"__vgpu_degrees", "__vgpu_degrees"}}};
	static const std::map<std::string, std::pair<const char *, const char *>> binary = {
	    {"pow", {"pow", "powf"}}, {"power", {"pow", "powf"}}, {"atan2", {"atan2", "atan2f"}}};
	const auto &table = arity == 1 ? unary : binary;
	if (arity != 1 && arity != 2) return nullptr;
	auto it = table.find(name);
	if (it == table.end()) return nullptr;
	return fp32 ? it->second.second : it->second.first;
}

std::string FloatLiteral(double v, int precision, const char *suffix) {
	if (std::isnan(v) || std::isinf(v)) {
		Fail(VGPU_ERR_UNSUPPORTED, "expression_translator: non-finite floating constants have no CUDA literal");
	}
	std::ostringstream o;
	o << std::setprecision(precision) << v;
	std::string t = o.str();
	if (t.find('.') == std::string::npos && t.find('e') == std::string::npos && t.find('E') == std::string::npos) {
		t += ".0";
	}
	return t + suffix;
}

struct Translator {
	const vgpu_bexpr *nodes;
	uint32_t n;
	bool fp32;
	bool strict;
	std::vector<std::string> inputs;
	std::map<std::string, size_t> slot;
	int depth = 0;

	const vgpu_bexpr &Node(uint32_t i) {
		if (i >= n) Fail(VGPU_ERR_INVALID_ARGUMENT, "expression_translator: child index out of range");
		return nodes[i];
	}
	static ValueType TypeOf(const vgpu_bexpr &e) {
		if (!IsValidValueType(e.return_type)) Fail(VGPU_ERR_INVALID_ARGUMENT, "expression_translator: type out of range");
		return static_cast<ValueType>(e.return_type);
	}

	std::string Go(uint32_t i) {
		if (++depth > 256) Fail(VGPU_ERR_INVALID_ARGUMENT, "expression_translator: expression nested too deeply");
		std::string s = One(Node(i));
		--depth;
		return s;
	}

	std::string One(const vgpu_bexpr &e) {
		const ValueType t = TypeOf(e);
		const std::string name = e.name ? e.name : "";
		switch (e.kind) {
		case VGPU_BEXPR_COLUMN: {
			if (name.empty()) Fail(VGPU_ERR_INVALID_ARGUMENT, "expression_translator: column reference without a name");
			auto it = slot.find(name);
			size_t s;
			if (it != slot.end()) {
				s = it->second;
			} else {
				s = inputs.size();
				inputs.push_back(name);
				slot[name] = s;
			}
			return std::string("((const ") + TypeNameOrRefuse(t) + "*)inputs[" + std::to_string(s) + "])[row]";
		}
		case VGPU_BEXPR_CONSTANT: {
			if (e.is_null) Fail(VGPU_ERR_UNSUPPORTED, "expression_translator: NULL constants are not supported in GPU expressions");
			switch (t) {
			case ValueType::INT16:
				return std::to_string(static_cast<int16_t>(e.i64));
			case ValueType::INT32:
				return std::to_string(static_cast<int32_t>(e.i64));
			case ValueType::INT64:
				return std::to_string(e.i64) + "LL";
			case ValueType::FLOAT32:
				return FloatLiteral(static_cast<double>(static_cast<float>(e.f64)), 9, "f");
			case ValueType::FLOAT64:
				return FloatLiteral(e.f64, 17, "");
			case ValueType::BOOLEAN:
				return e.i64 ? "true" : "false";
			default:
				TypeNameOrRefuse(t);
			}
			Fail(VGPU_ERR_UNSUPPORTED, "expression_translator: constant of this type is not representable");
		}
		case VGPU_BEXPR_COMPARE: {
			static const std::map<std::string, const char *> ops = {{"=", "=="}, {"==", "=="}, {"!=", "!="}, {"<>", "!="},
			                                                      {"<", "<"},   {">", ">"},   {"<=", "<="}, {">=", ">="}};
			auto it = ops.find(name);
			if (it == ops.end()) Fail(VGPU_ERR_UNSUPPORTED, "expression_translator: unsupported comparison operator: " + name);
			if (e.n_children != 2 || e.children == nullptr) {
				Fail(VGPU_ERR_INVALID_ARGUMENT, "expression_translator: comparison needs two operands");
			}
			const std::string l = Go(e.children[0]), r = Go(e.children[1]);
			return "(" + l + " " + it->second + " " + r + ")";
		}
		case VGPU_BEXPR_FUNCTION:
			return Function(e, t, name);
		default:
			Fail(VGPU_ERR_UNSUPPORTED, "expression_translator: unsupported expression class " + std::to_string(e.kind));
		}
	}

	std::string Function(const vgpu_bexpr &e, ValueType t, const std::string &name) {
		const uint32_t k = e.n_children;
		if (k > 0 && e.children == nullptr) Fail(VGPU_ERR_INVALID_ARGUMENT, "expression_translator: children missing");
		if (name == "__cast") {
			if (k != 1) Fail(VGPU_ERR_INVALID_ARGUMENT, "expression_translator: cast with unexpected arity");
			const ValueType from = TypeOf(Node(e.children[0]));
			if (!CastAgrees(from, t)) {
				Fail(VGPU_ERR_UNSUPPORTED, std::string("expression_translator: cast from ") + CudaTypeName(from) + " to " +
				                               CudaTypeName(t) + " does not agree with DuckDB's CAST for every value");
			}
			const std::string x = Go(e.children[0]);
			if (from == t) return x;
			return std::string("((") + TypeNameOrRefuse(t) + ")(" + x + "))";
		}
		if (const char *fn = MathFunction(name, k, false)) {
			if (t != ValueType::FLOAT64) {
				Fail(VGPU_ERR_UNSUPPORTED, "expression_translator: GPU math function '" + name + "' is supported only where it returns DOUBLE");
			}
			// correctly rounded on both sides (or plain arithmetic); the transcendentals differ by about an ulp
			static const std::set<std::string> exact = {"sqrt", "floor", "ceil", "ceiling", "radians", "degrees"};
			if (strict && !exact.count(name)) {
				Fail(VGPU_ERR_UNSUPPORTED, "expression_translator: strict FP is requested and '" + name +
				                               "' is not bit-identical to the CPU implementation");
			}
			if (fp32) {
				std::string call = std::string("(double)(") + MathFunction(name, k, true) + "(";
				for (uint32_t c = 0; c < k; c++) call += (c ? ", " : "") + std::string("(float)(") + Go(e.children[c]) + ")";
				return call + "))";
			}
			std::string call = std::string(fn) + "(";
			for (uint32_t c = 0; c < k; c++) call += (c ? ", " : "") + std::string("(double)(") + Go(e.children[c]) + ")";
			return call + ")";
		}
		if (name == "abs" && k == 1) {
			const std::string x = Go(e.children[0]);
			if (t == ValueType::FLOAT64 || t == ValueType::FLOAT32) return "fabs((double)(" + x + "))";
			if (t == ValueType::INT32 || t == ValueType::INT64) return "((" + x + ") < 0 ? -(" + x + ") : (" + x + "))";
			Fail(VGPU_ERR_UNSUPPORTED, "expression_translator: GPU abs supports numeric types only");
		}
		if (name == "%") {
			if (k != 2) Fail(VGPU_ERR_INVALID_ARGUMENT, "expression_translator: modulo with unexpected arity");
			const ValueType lt = TypeOf(Node(e.children[0]));
			const std::string l = Go(e.children[0]), r = Go(e.children[1]);
			if (lt == ValueType::FLOAT64 || lt == ValueType::FLOAT32) return "fmod((double)(" + l + "), (double)(" + r + "))";
			return "(" + l + " % " + r + ")";
		}
		if (name == "+" || name == "-" || name == "*" || name == "/") {
			if (k == 2) {
				const std::string l = Go(e.children[0]), r = Go(e.children[1]);
				return "(" + l + " " + name + " " + r + ")";
			}
			if (k == 1 && name == "-") return "(-" + Go(e.children[0]) + ")";
			Fail(VGPU_ERR_UNSUPPORTED, "expression_translator: unsupported arity for GPU arithmetic function: " + name);
		}
		Fail(VGPU_ERR_UNSUPPORTED, "expression_translator: unsupported function for GPU expression: " + name);
	}
};

} // namespace

TranslatedExpr TranslateExpression(const vgpu_bexpr *nodes, uint32_t n_nodes, uint32_t root, uint32_t flags) {
	if (nodes == nullptr || root >= n_nodes) Fail(VGPU_ERR_INVALID_ARGUMENT, "expression_translator: empty expression");
	Translator tr {nodes, n_nodes, (flags & VGPU_TRANSLATE_FP32) != 0, (flags & VGPU_TRANSLATE_STRICT_FP) != 0, {}, {}, 0};
	TranslatedExpr out;
	const std::string body = tr.Go(root);
	out.output_type = static_cast<ValueType>(nodes[root].return_type);
	out.statement = std::string("((") + TypeNameOrRefuse(out.output_type) + "*)out)[idx] = " + body + ";";
	out.inputs = std::move(tr.inputs);
	return out;
}

} // namespace vgpu
