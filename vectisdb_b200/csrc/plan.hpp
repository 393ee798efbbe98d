// plan.hpp -- the engine's own plan IR, converted from the C ABI's flat node array. Mirrors the
// reference's GpuPlanNode (cuda_engine/include/gpu_engine.hpp:135-185) with children as owned pointers.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "common.hpp"

namespace vgpu {

enum class OpType : uint8_t {
	SCAN = VGPU_OP_SCAN,
	FILTER = VGPU_OP_FILTER,
	PROJECTION = VGPU_OP_PROJECTION,
	HASH_JOIN = VGPU_OP_HASH_JOIN,
	GROUP_BY_AGGREGATE = VGPU_OP_GROUP_BY_AGGREGATE,
	CROSS_PRODUCT = VGPU_OP_CROSS_PRODUCT,
};

enum class AggKind : uint8_t {
	COUNT_STAR = VGPU_AGG_COUNT_STAR,
	COUNT = VGPU_AGG_COUNT,
	SUM = VGPU_AGG_SUM,
	MIN = VGPU_AGG_MIN,
	MAX = VGPU_AGG_MAX,
	AVG = VGPU_AGG_AVG,
};

struct Expr {
	std::string source;
	std::vector<std::string> input_columns;
	ValueType output_type = ValueType::FLOAT64;
	double ops_per_row = 0.0;  // caller's price of one row (routing only); 0 = not priced
	uint32_t window = VGPU_WINDOW_NONE;  // vgpu_window_primitive
};

struct Aggregate {
	AggKind kind = AggKind::COUNT_STAR;
	std::string input_column;
	ValueType output_type = ValueType::INT64;
};

struct TableRef {
	std::string catalog, schema, table;
	bool operator==(const TableRef &o) const {
		return catalog == o.catalog && schema == o.schema && table == o.table;
	}
	std::string ToString() const {
		return catalog + "." + schema + "." + table;
	}
};

struct PlanNode {
	OpType op = OpType::SCAN;
	std::vector<std::shared_ptr<PlanNode>> children;
	TableRef table;
	std::vector<std::string> column_names;
	std::vector<Expr> expressions;
	std::vector<std::string> build_keys;
	std::vector<std::string> probe_keys;
	std::vector<std::string> output_columns;
	std::vector<std::string> group_keys;
	std::vector<Aggregate> aggregates;
	std::vector<std::string> aggregate_exprs;  // descriptors only: never executed
	uint64_t estimated_rows = 0;
	uint32_t estimated_row_width_bytes = 0;
};

//! Converts and validates the ABI plan: indices in range, no cycles (each node reachable once from
//! the root along a tree), enums in range. Throws Error(VGPU_ERR_INVALID_ARGUMENT).
std::shared_ptr<PlanNode> ConvertPlan(const vgpu_plan *plan);

//! Number of SCAN leaves in traversal order (children[0] before children[1]).
void CollectScans(const PlanNode &node, std::vector<const PlanNode *> &out);

bool IsRowIndependent(const PlanNode &node);

//! True when an expression anywhere in the plan carries a window primitive (RUNNING_SUM).
bool HasWindowPrimitive(const PlanNode &node);

//! Fails with VGPU_ERR_UNSUPPORTED when the plan carries a window primitive: only the stream pipeline
//! keeps a running total across calls, and running one as a plain expression would be wrong.
void RefuseWindowPrimitives(const PlanNode &node);

} // namespace vgpu
