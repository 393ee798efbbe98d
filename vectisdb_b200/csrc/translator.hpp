// translator.hpp -- bound expression tree -> engine expression statement (see translator.cpp).
#pragma once

#include <string>
#include <vector>

#include "common.hpp"

namespace vgpu {

struct TranslatedExpr {
	std::string statement;           // ((T*)out)[idx] = ...;
	std::vector<std::string> inputs; // column names, one per inputs[] slot
	ValueType output_type = ValueType::INT32;
};

//! The reference extension's TranslateExpression + WrapAsOutputStatement over a vgpu_bexpr tree
//! (`nodes[root]` is the expression; children are node indices). Throws Error(VGPU_ERR_UNSUPPORTED)
//! with the reference's refusal reasons for shapes it does not lower.
TranslatedExpr TranslateExpression(const vgpu_bexpr *nodes, uint32_t n_nodes, uint32_t root, uint32_t flags);

} // namespace vgpu
