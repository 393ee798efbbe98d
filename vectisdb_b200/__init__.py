"""B200-native GPU execution path for DuckDB's data-parallel hot path.

The engine is libvgpu.so (include/vgpu.h, CUDA for sm_100a); this package holds its Python mirror of
the reference engine interface (`engine`), the ctypes ABI (`abi`), the synthetic workload generators
(`workloads`) and the build script (`build`).
"""
from .engine import (  # noqa: F401
    BatchOptions,
    PreparedBatch,
    Server,
    StreamPipeline,
    batch_clear,
    batch_template,
    device_to_host,
    ColumnCache,
    DeviceResult,
    ExecuteOptions,
    GpuAggregate,
    GpuAggregateKind,
    GpuColumn,
    GpuEngine,
    GpuExecutionResult,
    GpuExpr,
    GpuOpType,
    GpuPlanNode,
    GpuTableRef,
    GpuValueType,
    make_aggregate,
    make_column,
    make_cross_product,
    make_device_column,
    make_expr,
    make_filter,
    make_group_by,
    make_join,
    make_projection,
    make_scan,
)
