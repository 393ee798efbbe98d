// plan.cpp -- ABI plan conversion and structural helpers.
#include "plan.hpp"

#include <functional>

namespace vgpu {

namespace {

std::vector<std::string> Names(const char *const *names, uint32_t n, const char *what) {
	std::vector<std::string> out;
	if (n == 0) {
		return out;
	}
	if (names == nullptr) {
		Fail(VGPU_ERR_INVALID_ARGUMENT, std::string("plan: null ") + what + " array with nonzero count");
	}
	out.reserve(n);
	for (uint32_t i = 0; i < n; i++) {
		if (names[i] == nullptr) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, std::string("plan: null entry in ") + what);
		}
		out.emplace_back(names[i]);
	}
	return out;
}

std::string Str(const char *s) {
	return s ? std::string(s) : std::string();
}

} // namespace

std::shared_ptr<PlanNode> ConvertPlan(const vgpu_plan *plan) {
	if (plan == nullptr || plan->nodes == nullptr || plan->n_nodes == 0) {
		Fail(VGPU_ERR_INVALID_ARGUMENT, "plan: empty plan");
	}
	if (plan->root >= plan->n_nodes) {
		Fail(VGPU_ERR_INVALID_ARGUMENT, "plan: root index out of range");
	}
	std::vector<int> visiting(plan->n_nodes, 0);
	std::function<std::shared_ptr<PlanNode>(uint32_t, int)> build = [&](uint32_t index, int depth) {
		if (depth > 256) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "plan: nesting deeper than 256 levels");
		}
		if (visiting[index]) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "plan: node " + std::to_string(index) + " is part of a cycle");
		}
		visiting[index] = 1;
		const vgpu_plan_node &src = plan->nodes[index];
		auto node = std::make_shared<PlanNode>();
		if (src.op > VGPU_OP_CROSS_PRODUCT) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "plan: unknown op type " + std::to_string(src.op));
		}
		node->op = static_cast<OpType>(src.op);
		node->table = TableRef {Str(src.catalog), Str(src.schema), Str(src.table)};
		node->column_names = Names(src.column_names, src.n_column_names, "column_names");
		if (src.n_expressions > 0 && src.expressions == nullptr) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "plan: null expressions array");
		}
		for (uint32_t i = 0; i < src.n_expressions; i++) {
			const vgpu_expr &e = src.expressions[i];
			Expr expr;
			if (e.source == nullptr) {
				Fail(VGPU_ERR_INVALID_ARGUMENT, "plan: expression without source");
			}
			if (!IsValidValueType(e.output_type)) {
				Fail(VGPU_ERR_INVALID_ARGUMENT, "plan: expression output type out of range");
			}
			expr.source = e.source;
			expr.input_columns = Names(e.input_columns, e.n_input_columns, "expression inputs");
			expr.output_type = static_cast<ValueType>(e.output_type);
			expr.ops_per_row = e.estimated_ops_per_row;
			if (e.window_primitive > VGPU_WINDOW_RUNNING_SUM) {
				Fail(VGPU_ERR_INVALID_ARGUMENT, "plan: expression window primitive out of range");
			}
			expr.window = e.window_primitive;
			node->expressions.push_back(std::move(expr));
		}
		node->build_keys = Names(src.build_keys, src.n_build_keys, "build_keys");
		node->probe_keys = Names(src.probe_keys, src.n_probe_keys, "probe_keys");
		node->output_columns = Names(src.output_columns, src.n_output_columns, "output_columns");
		node->group_keys = Names(src.group_keys, src.n_group_keys, "group_keys");
		if (src.n_aggregates > 0 && src.aggregates == nullptr) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "plan: null aggregates array");
		}
		for (uint32_t i = 0; i < src.n_aggregates; i++) {
			const vgpu_aggregate &a = src.aggregates[i];
			if (a.kind > VGPU_AGG_AVG || !IsValidValueType(a.output_type)) {
				Fail(VGPU_ERR_INVALID_ARGUMENT, "plan: aggregate kind or output type out of range");
			}
			Aggregate agg;
			agg.kind = static_cast<AggKind>(a.kind);
			agg.output_type = static_cast<ValueType>(a.output_type);
			agg.input_column = Str(a.input_column);
			node->aggregates.push_back(std::move(agg));
		}
		node->aggregate_exprs = Names(src.aggregate_exprs, src.n_aggregate_exprs, "aggregate_exprs");
		if (!node->aggregate_exprs.empty() && node->aggregate_exprs.size() != node->aggregates.size()) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "gpu_groupby: aggregates and aggregate_exprs disagree in length");
		}
		node->estimated_rows = src.estimated_rows;
		node->estimated_row_width_bytes = src.estimated_row_width_bytes;
		if (src.n_children > 0 && src.children == nullptr) {
			Fail(VGPU_ERR_INVALID_ARGUMENT, "plan: null children array");
		}
		for (uint32_t i = 0; i < src.n_children; i++) {
			uint32_t child = src.children[i];
			if (child >= plan->n_nodes) {
				Fail(VGPU_ERR_INVALID_ARGUMENT, "plan: child index out of range");
			}
			node->children.push_back(build(child, depth + 1));
		}
		visiting[index] = 0;
		return node;
	};
	return build(plan->root, 0);
}

void CollectScans(const PlanNode &node, std::vector<const PlanNode *> &out) {
	if (node.op == OpType::SCAN) {
		out.push_back(&node);
		return;
	}
	for (auto &child : node.children) {
		CollectScans(*child, out);
	}
}

// IsRowIndependent (cuda_engine/include/gpu_engine.hpp:239-248): SCAN/PROJECTION are row-wise and
// FILTER only drops rows; every other operator combines rows and must see its input whole.
bool HasWindowPrimitive(const PlanNode &node) {
	for (auto &e : node.expressions) {
		if (e.window != VGPU_WINDOW_NONE) return true;
	}
	for (auto &c : node.children) {
		if (HasWindowPrimitive(*c)) return true;
	}
	return false;
}

void RefuseWindowPrimitives(const PlanNode &node) {
	if (HasWindowPrimitive(node)) {
		Fail(VGPU_ERR_UNSUPPORTED, "gpu_executor: RUNNING_SUM window expressions are not supported by this engine");
	}
}

bool IsRowIndependent(const PlanNode &node) {
	switch (node.op) {
	case OpType::SCAN:
		return true;
	case OpType::FILTER:
	case OpType::PROJECTION:
		for (auto &child : node.children) {
			if (!IsRowIndependent(*child)) {
				return false;
			}
		}
		return true;
	default:
		return false;
	}
}

} // namespace vgpu
