/*
 * vgpu.h -- C ABI of the B200-native DuckDB GPU execution path (libvgpu.so).
 *
 * Everything crosses this boundary as plain C: POD structs, raw pointers, sizes and integer status
 * codes. No C++ types, no exceptions, no torch types. A failed call returns a status other than
 * VGPU_OK and leaves a human-readable message in a thread-local buffer (vgpu_last_error()).
 *
 * The plan IR mirrors the reference engine boundary, cuda_engine/include/gpu_engine.hpp:
 *   vgpu_op_type          <- GpuOpType            (gpu_engine.hpp:14-21)
 *   vgpu_value_type       <- GpuValueType         (gpu_engine.hpp:29-38)
 *   vgpu_hugeint          <- GpuHugeInt           (gpu_engine.hpp:40-47)
 *   vgpu_expr             <- GpuExpr              (gpu_engine.hpp:56-80)
 *   vgpu_aggregate_kind   <- GpuAggregateKind     (gpu_engine.hpp:85-92)
 *   vgpu_aggregate        <- GpuAggregate         (gpu_engine.hpp:96-104)
 *   vgpu_plan_node        <- GpuPlanNode          (gpu_engine.hpp:135-185), children by index
 *   vgpu_column           <- GpuColumn            (gpu_engine.hpp:199-213)
 *   vgpu_result           <- GpuExecutionResult   (gpu_engine.hpp:215-222)
 *   vgpu_exec_options     <- GpuExecuteOptions    (gpu_engine.hpp:357-385)
 */
#ifndef VGPU_H_
#define VGPU_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VGPU_ABI_VERSION 2

typedef enum vgpu_status {
	VGPU_OK = 0,
	VGPU_ERR_INVALID_ARGUMENT = 1, /* malformed plan, null pointer, size mismatch */
	VGPU_ERR_UNSUPPORTED = 2,      /* a shape this engine refuses cleanly (caller falls back to CPU) */
	VGPU_ERR_CUDA = 3,             /* CUDA runtime / driver failure */
	VGPU_ERR_OUT_OF_MEMORY = 4,    /* device budget exhausted or allocation failed */
	VGPU_ERR_COMPILE = 5,          /* NVRTC rejected generated source */
	VGPU_ERR_NOT_READY = 6,        /* non-blocking query: work not finished yet */
	VGPU_ERR_TIMEOUT = 7,          /* a bounded wait gave up */
	VGPU_ERR_REJECTED = 8,         /* admission control refused the request */
	VGPU_ERR_INTERNAL = 9
} vgpu_status;

/* GpuOpType, same order (gpu_engine.hpp:14-21). */
typedef enum vgpu_op_type {
	VGPU_OP_SCAN = 0,
	VGPU_OP_FILTER = 1,
	VGPU_OP_PROJECTION = 2,
	VGPU_OP_HASH_JOIN = 3,
	VGPU_OP_GROUP_BY_AGGREGATE = 4,
	VGPU_OP_CROSS_PRODUCT = 5
} vgpu_op_type;

/* GpuValueType, same order (gpu_engine.hpp:29-38). */
typedef enum vgpu_value_type {
	VGPU_INT16 = 0,
	VGPU_INT32 = 1,
	VGPU_INT64 = 2,
	VGPU_FLOAT32 = 3,
	VGPU_FLOAT64 = 4,
	VGPU_BOOLEAN = 5,
	VGPU_DICTIONARY_STRING = 6,
	VGPU_HUGEINT = 7
} vgpu_value_type;

/* GpuHugeInt (gpu_engine.hpp:40-47): two's-complement 128-bit integer, little-endian halves. */
typedef struct vgpu_hugeint {
	uint64_t lower;
	int64_t upper;
} vgpu_hugeint;

/* GpuAggregateKind, same order (gpu_engine.hpp:85-92). */
typedef enum vgpu_aggregate_kind {
	VGPU_AGG_COUNT_STAR = 0,
	VGPU_AGG_COUNT = 1,
	VGPU_AGG_SUM = 2,
	VGPU_AGG_MIN = 3,
	VGPU_AGG_MAX = 4,
	VGPU_AGG_AVG = 5
} vgpu_aggregate_kind;

/* GpuWindowPrimitive (gpu_engine.hpp:48-51) */
typedef enum vgpu_window_primitive {
	VGPU_WINDOW_NONE = 0,
	VGPU_WINDOW_RUNNING_SUM = 1
} vgpu_window_primitive;

/* GpuExpr (gpu_engine.hpp:56-80). `source` is a CUDA statement that reads its inputs as
 * ((const T*)inputs[i])[row] and writes ((T*)out)[idx], exactly the form the reference's
 * expression translator emits (extension/src/expression_translator.cpp:311-315, 489-493). */
typedef struct vgpu_expr {
	const char *source;
	const char *const *input_columns;
	uint32_t n_input_columns;
	uint32_t output_type; /* vgpu_value_type */
	/* GpuExpr::window_primitive (gpu_engine.hpp:48-51, 67): vgpu_window_primitive. RUNNING_SUM asks for
	 * the running total of the expression across every row streamed so far. The stream pipeline computes
	 * it for top-level INT16/INT32/INT64/FLOAT32/FLOAT64 outputs of batches without NULLs (integers wrap
	 * in their width); vgpu_execute_plan, batches and serving refuse it with VGPU_ERR_UNSUPPORTED. */
	uint32_t window_primitive;
	/* GpuExpr::estimated_ops_per_row (gpu_engine.hpp:79): weighted operations per row, priced by the
	 * caller's translator; 0 = not priced. Read only by vgpu_analyze_plan_shape. */
	double estimated_ops_per_row;
} vgpu_expr;

/* GpuAggregate (gpu_engine.hpp:96-104). input_column is NULL/empty for COUNT_STAR. */
typedef struct vgpu_aggregate {
	uint32_t kind;        /* vgpu_aggregate_kind */
	uint32_t output_type; /* vgpu_value_type */
	const char *input_column;
} vgpu_aggregate;

/* GpuPlanNode (gpu_engine.hpp:135-185) flattened: children are indices into vgpu_plan.nodes.
 * Output naming follows the reference: PROJECTION emits "col<i>", GROUP_BY emits its key names then
 * "agg_<i>", FILTER passes its child's columns through, joins emit `output_columns`. */
typedef struct vgpu_plan_node {
	uint32_t op; /* vgpu_op_type */
	uint32_t n_children;
	const uint32_t *children;
	/* SCAN */
	const char *catalog;
	const char *schema;
	const char *table;
	const char *const *column_names;
	uint32_t n_column_names;
	/* FILTER / PROJECTION */
	const vgpu_expr *expressions;
	uint32_t n_expressions;
	/* HASH_JOIN: build_keys name children[0] columns, probe_keys children[1] columns */
	const char *const *build_keys;
	uint32_t n_build_keys;
	const char *const *probe_keys;
	uint32_t n_probe_keys;
	/* HASH_JOIN / CROSS_PRODUCT */
	const char *const *output_columns;
	uint32_t n_output_columns;
	/* GROUP_BY_AGGREGATE */
	const char *const *group_keys;
	uint32_t n_group_keys;
	const vgpu_aggregate *aggregates;
	uint32_t n_aggregates;
	/* cost-model inputs (advisory) */
	uint64_t estimated_rows;
	uint32_t estimated_row_width_bytes;
	/* GROUP_BY_AGGREGATE: GpuPlanNode::aggregate_exprs (gpu_engine.hpp:181), one human-readable
	 * descriptor per aggregate, or none; any other count is a malformed plan (gpu_groupby.cu:311-312). */
	const char *const *aggregate_exprs;
	uint32_t n_aggregate_exprs;
} vgpu_plan_node;

typedef struct vgpu_plan {
	const vgpu_plan_node *nodes;
	uint32_t n_nodes;
	uint32_t root;
} vgpu_plan;

typedef enum vgpu_memory {
	VGPU_MEM_HOST = 0,  /* pageable or pinned host memory */
	VGPU_MEM_DEVICE = 1 /* device memory of the current device */
} vgpu_memory;

/* GpuColumn (gpu_engine.hpp:199-213). Validity: NULL = no nulls; otherwise an Arrow LSB-first
 * bitmap (bit set = valid) living in the same memory space as `data`. */
typedef struct vgpu_column {
	const char *name;
	uint32_t type;   /* vgpu_value_type */
	uint32_t memory; /* vgpu_memory */
	const void *data;
	const uint8_t *validity;
	uint64_t row_count;
} vgpu_column;

/* GpuExecuteOptions (gpu_engine.hpp:357-385) plus placement controls. */
typedef struct vgpu_exec_options {
	int32_t stage_scan_to_cache;         /* hand every SCAN column to the open cache staging slot */
	int32_t serve_whole_scan_from_cache; /* read every SCAN leaf from the committed cache entry */
	int64_t cache_chunk_index;           /* >=0: serve chunk i of the cache entry (row-independent plans) */
	int32_t output_memory;               /* VGPU_MEM_HOST (default) or VGPU_MEM_DEVICE */
	int32_t flags;                       /* VGPU_EXEC_* bits */
	void *stream;                        /* cudaStream_t to run on; NULL = the engine's own stream */
} vgpu_exec_options;

/* Device output only: return without synchronizing the stream. A root GROUP BY on the one-pass path,
 * or a root FILTER/PROJECTION chain whose outputs have no NULL masks, then leaves its row count on the
 * device too: until vgpu_result_get_column (or _column_range) first reads the result, which waits for
 * the stream, the columns are sized for every key value (every input row). */
#define VGPU_EXEC_NO_SYNC 1u

void vgpu_exec_options_init(vgpu_exec_options *options);

typedef struct vgpu_result vgpu_result;

/* GpuEngine::ExecutePlan (gpu_engine.hpp:389-402; cuda_engine/src/gpu_engine.cpp:37-74).
 * SCAN leaves consume `inputs` positionally in traversal order, children[0] before children[1]
 * (cuda_engine/src/gpu_executor_internal.hpp:97). Host inputs are read during the call only. */
vgpu_status vgpu_execute_plan(const vgpu_plan *plan, const vgpu_column *inputs, size_t n_inputs,
                              const vgpu_exec_options *options, vgpu_result **out);

/* GpuExecutionResult::columns (gpu_engine.hpp:215-222). Column pointers stay valid until
 * vgpu_result_free; their memory space is vgpu_exec_options.output_memory. Device results keep the
 * buffers the execution wrote its outputs into (no copy), which a GROUP BY sizes for the largest
 * group count its key ranges allow: free a device result once it has been read. */
size_t vgpu_result_column_count(const vgpu_result *result);
vgpu_status vgpu_result_get_column(const vgpu_result *result, size_t index, vgpu_column *out);
/* Rows [offset, offset + count) of result column `index` as borrowed pointers into the result (no copy):
 * the emission of STANDARD_VECTOR_SIZE chunks (extension/src/physical_gpu_execute.cpp:506-517). Values
 * are laid out as DuckDB's flat vectors hold them (HUGEINT as hugeint_t {lower, upper}), and the
 * validity bitmap, LSB first with bit set = valid, is byte for byte DuckDB's 64-bit validity words, so a
 * column with validity is sliced at multiples of 64 rows (a 2048-row chunk is 32 whole words). */
vgpu_status vgpu_result_column_range(const vgpu_result *result, size_t index, uint64_t offset, uint64_t count,
                                     vgpu_column *out);
void vgpu_result_free(vgpu_result *result);

/* Copies `bytes` of device memory (a device-resident result column, for instance) to host memory,
 * ordered after the work already queued on `stream` (NULL = the engine's stream); returns when the
 * copy is complete. No single reference counterpart: the reference always returns host columns. */
vgpu_status vgpu_copy_to_host(void *dst, const void *src, size_t bytes, void *stream);

/* Thread-local message describing the last failed call on this thread ("" if none). */
const char *vgpu_last_error(void);
const char *vgpu_status_string(vgpu_status status);
int vgpu_abi_version(void);

/* ---- Device, streams and timing plumbing ---------------------------------------------------- */

/* Device properties the engine sized itself against (device 0 unless vgpu_set_device was called). */
typedef struct vgpu_device_info {
	int32_t device;
	int32_t sm_count;
	int32_t cc_major;
	int32_t cc_minor;
	uint64_t total_memory;
	uint64_t free_memory;
	uint64_t l2_bytes;
	uint64_t smem_per_block_optin;
	char name[128];
} vgpu_device_info;

vgpu_status vgpu_set_device(int device);
vgpu_status vgpu_get_device_info(vgpu_device_info *out);
vgpu_status vgpu_synchronize(void *stream);

/* Per-launch device timing of the engine's own kernels (CUDA events on the launching stream).
 * While enabled, every launch records a start/stop event pair; vgpu_profile_collect synchronizes
 * and returns (name, milliseconds, algorithmic bytes) per launch since the last collect. */
typedef struct vgpu_kernel_timing {
	char name[48];
	float ms;
	uint64_t bytes;
	uint64_t rows;
} vgpu_kernel_timing;

vgpu_status vgpu_profile_enable(int enable);
vgpu_status vgpu_profile_collect(vgpu_kernel_timing *out, size_t capacity, size_t *count);
/* Number of engine kernels launched since process start (all streams). */
uint64_t vgpu_launch_count(void);

/* ---- Kernel cache (cuda_engine/include/code_generator.hpp:30-155, kernel_cache.hpp:29-66) ---- */

/* SHA-256 of `n` bytes as 64 lowercase hex characters plus NUL (KernelCache::HashSource,
 * cuda_engine/src/kernel_cache.cpp:20-146). `out` must hold 65 bytes. */
void vgpu_sha256_hex(const void *data, size_t n, char *out);

typedef struct vgpu_kernel_cache_stats {
	uint64_t entries;
	uint64_t hits;
	uint64_t misses;
	uint64_t disk_hits;
	uint64_t compiles;
	double compile_ms_total;
} vgpu_kernel_cache_stats;

vgpu_status vgpu_kernel_cache_stats_get(vgpu_kernel_cache_stats *out);
/* Compiles `source` (a whole translation unit) with NVRTC for sm_100a without loading it. Usable on
 * a machine without a GPU; returns VGPU_ERR_COMPILE with the NVRTC log on failure. */
vgpu_status vgpu_nvrtc_compile_check(const char *source, size_t *cubin_bytes);
/* Generates (but does not compile) the fused source the engine would build for `plan`; writes at
 * most `capacity` bytes including the NUL and reports the full length in *length. */
vgpu_status vgpu_generate_source(const vgpu_plan *plan, const vgpu_column *inputs, size_t n_inputs,
                                 char *out, size_t capacity, size_t *length);

/* ---- Expression translation (extension/src/expression_translator.cpp:287-460, 489-493) ----------
 * A bound expression (DuckDB's BoundColumnRef / BoundConstant / BoundComparison / BoundFunction) as a
 * node array; `children` index into the same array. The translation is the statement the engine's
 * vgpu_expr contract carries, the ordered input columns it reads and its output type. */
typedef enum vgpu_bexpr_kind {
	VGPU_BEXPR_COLUMN = 0,   /* name = the scanned column; return_type its type */
	VGPU_BEXPR_CONSTANT = 1, /* integer/BOOLEAN value in i64, FLOAT/DOUBLE in f64; is_null refuses */
	VGPU_BEXPR_COMPARE = 2,  /* name = "=", "!=", "<>", "<", ">", "<=", ">="; two children */
	VGPU_BEXPR_FUNCTION = 3  /* name = DuckDB function ("+", "-", "*", "/", "%", "__cast", "abs", "sqrt", "ln", ...) */
} vgpu_bexpr_kind;

typedef struct vgpu_bexpr {
	uint32_t kind;        /* vgpu_bexpr_kind */
	uint32_t return_type; /* vgpu_value_type of the expression's DuckDB return type */
	const char *name;
	const uint32_t *children;
	uint32_t n_children;
	uint32_t is_null;
	int64_t i64;
	double f64;
} vgpu_bexpr;

#define VGPU_TRANSLATE_FP32 1u      /* VECTOR_GPU_FP32_RELAXATION: math functions in float */
#define VGPU_TRANSLATE_STRICT_FP 2u /* VECTOR_GPU_STRICT_FP: only the bit-exact math functions */

/* TranslateExpression + WrapAsOutputStatement: writes the statement ('\0'-terminated) into `statement`
 * and the input column names, each '\0'-terminated one after another, into `inputs`; *n_inputs and
 * *output_type receive their count and the output type. VGPU_ERR_UNSUPPORTED (with the reason in
 * vgpu_last_error) for shapes the GPU path does not lower; VGPU_ERR_INVALID_ARGUMENT when a buffer is
 * too small (the needed sizes are in *statement_len / *inputs_len). */
vgpu_status vgpu_translate_expression(const vgpu_bexpr *nodes, uint32_t n_nodes, uint32_t root, uint32_t flags,
                                      char *statement, size_t statement_cap, size_t *statement_len, char *inputs,
                                      size_t inputs_cap, size_t *inputs_len, uint32_t *n_inputs,
                                      uint32_t *output_type);

/* ---- Cost model (cuda_engine/include/gpu_engine.hpp:187-348; src/gpu_cost_model.cpp) ------- */

typedef struct vgpu_working_set {
	uint64_t total_bytes; /* saturates at UINT64_MAX */
	int32_t chunk_capped;
	uint64_t largest_bytes;
	char largest_operator[32];
} vgpu_working_set;

/* IsRowIndependent (gpu_engine.hpp:248) */
int vgpu_is_row_independent(const vgpu_plan *plan);
/* EstimateWorkingSet (gpu_engine.hpp:341), re-derived for this engine's own allocation sites. */
vgpu_status vgpu_estimate_working_set(const vgpu_plan *plan, uint64_t max_chunk_rows, vgpu_working_set *out);
/* The same estimate for one execution with its actual inputs and options (no reference counterpart:
 * the reference's caller passes the plan alone): rows and widths from `inputs` (or from the cached
 * columns a cache-served scan reads); scans over cache-served or device-memory columns are borrowed
 * and charge nothing. The serving admission controller uses it. */
vgpu_status vgpu_estimate_working_set_for(const vgpu_plan *plan, const vgpu_column *inputs, size_t n_inputs,
                                          const vgpu_exec_options *options, vgpu_working_set *out);

/* Routing helpers the extension's table checker calls (extension/src/table_checker.cpp:400, 485-499).
 * Plain arithmetic over the plan's advisory fields; no device is touched. */

/* ExecutionMode (gpu_engine.hpp:23-27) */
typedef enum vgpu_execution_mode {
	VGPU_MODE_PIPELINE_STREAM_CACHED = 0,
	VGPU_MODE_PIPELINE_STREAM_UNCACHED = 1,
	VGPU_MODE_BATCH_DISPATCH = 2
} vgpu_execution_mode;

/* GpuWorkDensity (gpu_engine.hpp:250-264) */
typedef enum vgpu_work_density {
	VGPU_DENSITY_INSUFFICIENT = 0, /* priced, below VGPU_MIN_OPS_PER_SCANNED_ROW */
	VGPU_DENSITY_INCONCLUSIVE = 1, /* between the thresholds, or nothing priced at all */
	VGPU_DENSITY_SUFFICIENT = 2    /* at or above VGPU_OFFLOAD_OPS_PER_ROW */
} vgpu_work_density;

/* The reference's routing thresholds (gpu_engine.hpp:269, 279), kept so its routing decides alike. */
#define VGPU_MIN_OPS_PER_SCANNED_ROW 3.0
#define VGPU_OFFLOAD_OPS_PER_ROW 10.0

/* GpuPlanShape (gpu_engine.hpp:284-317) */
typedef struct vgpu_plan_shape {
	uint64_t scanned_rows;  /* sum of SCAN estimated_rows (saturating) */
	uint64_t scanned_bytes; /* sum of SCAN rows x row width (width 0 counts as 8 bytes) */
	uint64_t max_rows;      /* largest estimated_rows of any node */
	double total_ops;       /* sum over nodes of (sum of their expressions' ops per row) x rows evaluated */
	double ops_per_scanned_row;
	double ops_per_scanned_byte;
	uint32_t density; /* vgpu_work_density */
	double amplification; /* max_rows / scanned_rows (max_rows when nothing is scanned) */
} vgpu_plan_shape;

/* AnalyzePlanShape (gpu_engine.hpp:329). A FILTER's expressions are charged over the rows entering it
 * (its child's estimated_rows), every other node's over its own estimated_rows. */
vgpu_status vgpu_analyze_plan_shape(const vgpu_plan *plan, vgpu_plan_shape *out);
/* EstimateColumnsSize (gpu_engine.hpp:342): sum of SCAN rows x row width (width 0 counts as 8 bytes). */
vgpu_status vgpu_estimate_columns_size(const vgpu_plan *plan, uint64_t *out);
/* DetermineExecutionMode (gpu_engine.hpp:348): PIPELINE_STREAM_UNCACHED when vram_budget > 0 and the
 * scanned columns exceed vram_budget x threshold (the reference's default threshold is 0.75), else
 * PIPELINE_STREAM_CACHED. `columns_size` (optional) receives the estimate it compared. */
vgpu_status vgpu_determine_execution_mode(const vgpu_plan *plan, uint64_t vram_budget, double threshold,
                                          uint32_t *mode, uint64_t *columns_size);

/* ---- Device memory budget (cuda_engine/include/rmm_pool.hpp:32-141) -------------------------- */

typedef struct vgpu_memory_stats {
	uint64_t budget_bytes;
	uint64_t in_use_bytes;
	uint64_t peak_bytes;
	uint64_t allocations;
	uint64_t failed_allocations;
} vgpu_memory_stats;

/* 0 = derive from VECTOR_GPU_VRAM_FRACTION (default 0.85) of free memory at first use. */
vgpu_status vgpu_memory_set_budget(uint64_t bytes);
vgpu_status vgpu_memory_stats_get(vgpu_memory_stats *out);
/* Restarts peak_bytes at the bytes in use now, so that the peak of the next calls can be read back
 * (the reference samples cudaMemGetInfo for this, cuda_engine/tests/test_gpu_cost_model.cpp:16-40). */
vgpu_status vgpu_memory_reset_peak(void);
/* HasHeadroomFor (cuda_engine/src/rmm_pool.cpp:172-191) */
int vgpu_memory_has_headroom(uint64_t bytes);

/* ---- Device column cache (cuda_engine/include/gpu_column_cache.hpp:107-281) ------------------ */

typedef struct vgpu_table_ref {
	const char *catalog;
	const char *schema;
	const char *table;
} vgpu_table_ref;

/* EnsureInitialized: fraction of free device memory (VECTOR_GPU_CACHE_FRACTION / _MB override). */
vgpu_status vgpu_cache_init(double fraction_of_vram);
vgpu_status vgpu_cache_begin_staging(const vgpu_table_ref *table);
/* StageChunk: copies (H2D or D2D) `chunk` into cache-owned device memory as the next chunk of the
 * column. *accepted = 1 when staged, 0 when declined (no open slot, type mismatch, budget). */
vgpu_status vgpu_cache_stage_chunk(const vgpu_table_ref *table, const vgpu_column *chunk, int *accepted);
vgpu_status vgpu_cache_commit_staging(const vgpu_table_ref *table, uint64_t scanned_rows);
vgpu_status vgpu_cache_abort_staging(const vgpu_table_ref *table);
/* ReplayableChunkRows: writes up to `capacity` chunk row counts; *count = number of chunks (0 on miss). */
vgpu_status vgpu_cache_replayable_chunk_rows(const vgpu_table_ref *table, const char *const *column_names,
                                             size_t n_columns, uint64_t *rows, size_t capacity, size_t *count);
/* TryGetChunk: borrow of the device buffer (valid until the next evicting call). */
vgpu_status vgpu_cache_try_get_chunk(const vgpu_table_ref *table, const char *column_name, uint64_t chunk_index,
                                     vgpu_column *out, int *found);
vgpu_status vgpu_cache_invalidate_table(const vgpu_table_ref *table);
vgpu_status vgpu_cache_invalidate_all(void);
uint64_t vgpu_cache_current_bytes(void);
uint64_t vgpu_cache_table_generation(const vgpu_table_ref *table);

/* ---- Host ingest (extension/src/vector_converter.cpp:87-273, gpu_batch_accumulator.cpp:126-249) -----
 * One vector of a scanned chunk in DuckDB's UnifiedVectorFormat: logical row i reads physical index
 * sel[i] (identity when sel is NULL; 0 for every row of a constant vector); validity holds DuckDB's
 * 64-bit mask words by physical index, LSB first, bit set = valid (NULL = all valid). */
typedef struct vgpu_vector {
	const void *data;
	const uint32_t *sel;
	const uint64_t *validity;
	uint32_t constant;
} vgpu_vector;

/* ConvertVectorToGpuColumn: `count` logical rows (through row_sel first, when given) of a vector of
 * `type` into dense out_data and, when out_validity is given, an Arrow LSB-first bitmap (bit set =
 * valid); *any_null says whether a NULL was met (the reference attaches the bitmap only then). */
vgpu_status vgpu_convert_vector(const vgpu_vector *vector, uint32_t type, uint64_t count, const uint32_t *row_sel,
                                void *out_data, uint8_t *out_validity, int *any_null);

/* The accumulator + upload of a scan into the device column cache: chunks appended to a handle are
 * converted into page-locked batches of batch_rows rows; each full batch is uploaded asynchronously on
 * the handle's own stream and staged in the cache as one chunk per column (no second copy), so the
 * conversion of the next batch overlaps the transfer. vgpu_ingest_finish uploads the rest, waits and
 * commits the table (replacing the re-staged columns, keeping the others); a handle destroyed before
 * finishing aborts its staging. One handle per table scan; calls on one handle are serialized. */
typedef struct vgpu_ingest vgpu_ingest;
vgpu_status vgpu_ingest_create(const vgpu_table_ref *table, const char *const *names, const int32_t *types,
                               size_t n_columns, uint64_t batch_rows, vgpu_ingest **out);
/* `vectors` holds one vector per column; `row_sel` (optional) selects `count` rows of the chunk. */
vgpu_status vgpu_ingest_append(vgpu_ingest *ingest, const vgpu_vector *vectors, uint64_t count,
                               const uint32_t *row_sel);
vgpu_status vgpu_ingest_finish(vgpu_ingest *ingest, uint64_t *rows);
void vgpu_ingest_destroy(vgpu_ingest *ingest);

/* ---- Stream pipeline (GpuStreamPipeline, cuda_engine/include/gpu_stream_pipeline.hpp:122-208) -------
 * A row-independent projection chain (PROJECTION+ over SCAN, no filter) run batch by batch with upload,
 * compute and download of consecutive batches overlapping on three streams. vgpu_pipeline_create
 * allocates every buffer (depth + 1 stages of max_rows_per_batch rows) and compiles the fused kernel,
 * failing there rather than mid-scan. Batches are host columns in the declared order (names and
 * types checked); their memory may be reused as soon as vgpu_pipeline_submit returns. Results come
 * back in submission order, in pinned host memory owned by the result's stage, valid until
 * vgpu_pipeline_result_release. Columns are named col0, col1, ... (the top projection's
 * expressions). Externally serialized: one call at a time on a pipeline. */
typedef struct vgpu_pipeline vgpu_pipeline;
typedef struct vgpu_pipeline_result vgpu_pipeline_result;
/* GpuStreamPipeline::Supports (gpu_stream_pipeline.hpp:138-145): 1 when the plan has the shape. */
int vgpu_pipeline_supports(const vgpu_plan *plan);
/* Constructor (gpu_stream_pipeline.hpp:147-157); depth = batches in flight (0 = 3). */
vgpu_status vgpu_pipeline_create(const vgpu_plan *plan, const char *const *input_names, const int32_t *input_types,
                                 size_t n_inputs, uint64_t max_rows_per_batch, int32_t depth, vgpu_pipeline **out);
size_t vgpu_pipeline_output_count(const vgpu_pipeline *pipeline);
int32_t vgpu_pipeline_output_type(const vgpu_pipeline *pipeline, size_t index);
/* Poll / CanSubmit (gpu_stream_pipeline.hpp:163-176). */
void vgpu_pipeline_poll(vgpu_pipeline *pipeline);
int vgpu_pipeline_can_submit(vgpu_pipeline *pipeline);
/* Submit (gpu_stream_pipeline.hpp:178-186): queues one batch of `row_count` rows. */
vgpu_status vgpu_pipeline_submit(vgpu_pipeline *pipeline, const vgpu_column *columns, size_t n_columns,
                                 uint64_t row_count);
/* TryTake / TakeBlocking (gpu_stream_pipeline.hpp:188-199): *out = the oldest batch's result, or NULL
 * (not finished yet / nothing in flight). */
vgpu_status vgpu_pipeline_try_take(vgpu_pipeline *pipeline, vgpu_pipeline_result **out);
vgpu_status vgpu_pipeline_take_blocking(vgpu_pipeline *pipeline, vgpu_pipeline_result **out);
size_t vgpu_pipeline_in_flight(const vgpu_pipeline *pipeline);
uint64_t vgpu_pipeline_result_rows(const vgpu_pipeline_result *result);
size_t vgpu_pipeline_result_column_count(const vgpu_pipeline_result *result);
vgpu_status vgpu_pipeline_result_get_column(const vgpu_pipeline_result *result, size_t index, vgpu_column *out);
/* GpuStreamResult::Reset: returns the stage for reuse. */
void vgpu_pipeline_result_release(vgpu_pipeline_result *result);
void vgpu_pipeline_destroy(vgpu_pipeline *pipeline);

/* ---- Batching: many queries in one persistent, graph-captured launch ------------------------------
 * No single reference function: this is the batching form added beside the reference's
 * one-plan-per-call ExecutePlan (gpu_engine.hpp:389-402). Plans of the form GROUP_BY(keys) <-
 * FILTER/PROJECTION* <- SCAN whose expression sources differ only in numeric literals share one
 * kernel; a persistent launch walks a (query, row tile) queue over all of them and one CTA per
 * query writes its groups. The launch pair is captured in a CUDA graph on `options->stream` and
 * replayed while a later call presents the same batch (same columns, constants and geometry).
 * Other plans run one by one through vgpu_execute_plan. results[i] belongs to plans[i]; each is
 * freed with vgpu_result_free. Device results of one call share buffers that live until the last
 * of them is freed. */
typedef struct vgpu_batch_options {
	int32_t block;      /* threads per CTA; 0 = tuned or default */
	int32_t items;      /* consecutive rows per thread; 0 = tuned or default */
	int32_t tile_rows;  /* rows per queue item; 0 = tuned or default */
	int32_t smem_slots; /* shared-memory table slots (queries with larger key spaces use global tables) */
	int32_t use_graph;  /* capture and replay the launch pair in a CUDA graph (needs a non-legacy stream) */
	int32_t autotune;   /* time the candidate geometries on this batch now and remember the best */
} vgpu_batch_options;

typedef struct vgpu_batch_stats {
	uint64_t batched;       /* queries run by the batch kernel */
	uint64_t fallback;      /* queries run one by one */
	uint64_t templates;     /* distinct templates, one kernel each */
	uint64_t graph_replays; /* graph launches that reused a captured graph */
	int32_t block, items, tile_rows, smem_slots; /* geometry used for the last template */
} vgpu_batch_stats;

void vgpu_batch_options_init(vgpu_batch_options *options);

/* A prepared batch: the plans converted, templated and grouped once, for repeated execution (the
 * per-call work is then resolving the columns and launching). Freed with vgpu_batch_free. */
typedef struct vgpu_batch vgpu_batch;
vgpu_status vgpu_batch_prepare(const vgpu_plan *const *plans, size_t n_plans, vgpu_batch **out);
size_t vgpu_batch_size(const vgpu_batch *batch);
vgpu_status vgpu_batch_execute(vgpu_batch *batch, const vgpu_column *const *inputs, const size_t *n_inputs,
                               const vgpu_exec_options *options, const vgpu_batch_options *batch_options,
                               vgpu_result **results, vgpu_batch_stats *stats);
void vgpu_batch_free(vgpu_batch *batch);
/* One-shot form: prepare, execute, free. */
vgpu_status vgpu_execute_batch(const vgpu_plan *const *plans, const vgpu_column *const *inputs,
                               const size_t *n_inputs, size_t n_plans, const vgpu_exec_options *options,
                               const vgpu_batch_options *batch_options, vgpu_result **results,
                               vgpu_batch_stats *stats);
/* The template of one expression source: its numeric literals replaced by per-query parameter reads
 * (inputs[...] indices stay literal). Writes up to `capacity` bytes (NUL-terminated) and the number
 * of parameters. Host-only; for tests and plan inspection. */
vgpu_status vgpu_batch_template(const char *source, char *out, size_t capacity, size_t *length, size_t *n_params);
/* Drops cached batch graphs and buffers and the in-memory autotuning table. */
vgpu_status vgpu_batch_clear(void);

/* ---- Serving: admission against a device-memory budget, continuous batching ---------------------
 * No single reference counterpart: the reference host runs one query at a time
 * (extension/include/vector_gpu_host.hpp:71-76). A server owns `slots` worker threads, each with
 * its own CUDA stream. Requests queue on submit and are admitted in arrival order while a slot is
 * free and their estimated working set (vgpu_estimate_working_set, with the real input sizes) fits
 * in what the budget has left; admitted requests run concurrently on the device. Queued requests
 * whose plan has the batch form and shares the head request's template are admitted with it and run
 * as one batched launch. A request whose estimate exceeds the whole budget completes at once with
 * VGPU_ERR_OUT_OF_MEMORY. Host inputs must stay valid until vgpu_server_wait reports the request
 * done; plans are copied at submit. */
typedef struct vgpu_server_options {
	int32_t slots;                /* requests running at once (default 4) */
	int32_t batch_max;            /* most requests in one batched launch; 1 = no batching (default 64) */
	uint64_t memory_budget_bytes; /* admission budget; 0 = min(120 GiB, the allocator budget) */
} vgpu_server_options;

typedef struct vgpu_request_info {
	int32_t status;           /* vgpu_status of the request */
	int32_t batch_size;       /* requests in the launch that ran it */
	double queued_ms;         /* submit -> admission */
	double run_ms;            /* admission -> completion */
	uint64_t estimated_bytes; /* working-set estimate used for admission */
	char error[256];
} vgpu_request_info;

typedef struct vgpu_server_stats {
	uint64_t submitted, completed, failed, rejected;
	uint64_t batches, batched_requests;
	uint64_t in_flight, queued;
	uint64_t reserved_bytes, peak_reserved_bytes, budget_bytes;
	uint64_t peak_in_flight;
} vgpu_server_stats;

typedef struct vgpu_server vgpu_server;
void vgpu_server_options_init(vgpu_server_options *options);
vgpu_status vgpu_server_create(const vgpu_server_options *options, vgpu_server **out);
vgpu_status vgpu_server_submit(vgpu_server *server, const vgpu_plan *plan, const vgpu_column *inputs, size_t n_inputs,
                               const vgpu_exec_options *options, uint64_t *request_id);
/* Waits up to timeout_ms (< 0 = no limit). *done = 1 when the request finished: then *result holds
 * its columns (NULL if it failed; see info->status / info->error) and the id is released. */
vgpu_status vgpu_server_wait(vgpu_server *server, uint64_t request_id, double timeout_ms, vgpu_result **result,
                             vgpu_request_info *info, int *done);
vgpu_status vgpu_server_stats_get(vgpu_server *server, vgpu_server_stats *out);
/* Finishes the queued and running requests, then stops the workers. */
void vgpu_server_destroy(vgpu_server *server);

/* ---- Group-by without device allocation ------------------------------------------------------
 * No counterpart in the reference. For callers that cannot call cudaMalloc (a host callback or a
 * graph-driven loop, a process whose device memory another allocator has reserved, a caller holding a
 * lock an allocation could deadlock on): SELECT k, COUNT(*), SUM(v) GROUP BY k over keys in
 * [key_min, key_min + domain), domain <= 65536. All pointers are device memory the caller owns;
 * out_keys/out_counts/out_sums hold `domain` entries and receive the non-empty groups in key order,
 * *out_groups their number. Rows with keys outside the range are skipped. Temporaries live in a fixed
 * file-scope device array (about 1 MiB, held by every GPU that loads the library until exit), so the
 * call allocates nothing; a larger domain is rejected with VGPU_ERR_INVALID_ARGUMENT. The first call
 * on a device looks up that array's device address (cudaGetSymbolAddress) and should come before any
 * stream capture. Work is queued on `stream` (NULL = legacy default stream) and not synchronized.
 * Every call shares the one array, which keeps the last call's contents: calls whose work overlaps on
 * the GPU (different streams, no ordering between them) race and corrupt each other's results.
 * SUM(v) is accumulated with FP64 atomics, so its order -- and its last bits -- vary from call to call
 * (COUNT is exact). The looked-up address belongs to the device's current context: after a
 * cudaDeviceReset (or any reset of the primary context) in the same process it is stale, so do not
 * call this entry point after such a reset. */
vgpu_status vgpu_group_by_count_sum_noalloc(const int32_t *keys, const double *values, uint64_t n, int32_t key_min,
                                            uint32_t domain, int32_t *out_keys, int64_t *out_counts,
                                            double *out_sums, uint64_t *out_groups, void *stream);

/* ---- Sharded GROUP BY: the exchange step on the device -----------------------------------------
 * No counterpart in the reference, which runs on one device (cuda_engine/src/code_generator.cpp:53
 * takes device 0). A GROUP BY split by rows across GPUs (one process per GPU) runs the plan on each
 * rank's rows with partial states (AVG as SUM + COUNT), routes every partial group to the rank owning
 * its key with vgpu_shard_route, moves the rows with one all-to-all (NCCL, the caller's), turns the
 * received rows into columns with vgpu_shard_columns, re-aggregates them with vgpu_execute_plan (a
 * GROUP BY over the key word: SUM over FLOAT64 words and over INT64 count / 128-bit-chunk words, MIN
 * and MAX over INT64 words) and builds the output columns with vgpu_shard_finish. All buffers are
 * device memory; NULL keys or partial states are refused. */
typedef enum vgpu_shard_kind {
	VGPU_SHARD_SUM_F64 = 0,  /* FLOAT64 sum: 1 word (its bits; merged by a FLOAT64 SUM) */
	VGPU_SHARD_SUM_I128 = 1, /* HUGEINT sum: 4 words, 32-bit chunks c0..c2 unsigned, c3 signed (INT64 SUMs) */
	VGPU_SHARD_COUNT = 2,    /* integer count: 1 word (INT64 SUM) */
	VGPU_SHARD_MIN = 3,      /* integer MIN / MAX: 1 word, sign-extended (INT64 MIN / MAX) */
	VGPU_SHARD_MAX = 4,
	VGPU_SHARD_MIN_F64 = 5,  /* FLOAT32/FLOAT64 MIN / MAX: 1 word whose signed order is the float order */
	VGPU_SHARD_MAX_F64 = 6
} vgpu_shard_kind;

/* 64-bit words per exchanged row: 1 (the packed key) + 4 per SUM_I128 + 1 per other kind. */
int32_t vgpu_shard_words(const int32_t *kinds, int32_t n_values);

/* Packs `rows` partial groups -- key columns keys[0..n_keys) (integer types), packed as the sum of
 * (key_j - key_min[j]) << key_shift[j], and partial states values[0..n_values) of kinds[] -- into rows
 * of vgpu_shard_words() int64 words, written to `send` (device, rows x words, row-major) grouped by
 * owner rank (mix64(packed key) mod world, mix64 = MurmurHash3's 64-bit finalizer): the rows for rank
 * r start after send_counts[0..r). send_counts (host, `world` entries) receives the rows per rank.
 * Queued on `stream` (NULL = the runtime's stream), which is synchronized once for the counts. */
vgpu_status vgpu_shard_route(const vgpu_column *keys, int32_t n_keys, const int64_t *key_min, const int32_t *key_shift,
                             const vgpu_column *values, const int32_t *kinds, int32_t n_values, uint64_t rows,
                             int32_t world, int64_t *send, uint64_t *send_counts, void *stream);

/* Received rows (device, rows x words, row-major) to `words` device columns of `rows` int64 values:
 * column j at out + j * rows. Queued on `stream`, not synchronized. */
vgpu_status vgpu_shard_columns(const int64_t *recv, uint64_t rows, int32_t words, int64_t *out, void *stream);

typedef enum vgpu_shard_op {
	VGPU_SHARD_OUT_WORD = 0,          /* src[0]'s 64-bit word (the low word of a HUGEINT sum) */
	VGPU_SHARD_OUT_KEY = 1,           /* key column: ((src[0] >> key_shift) & (2^key_bits - 1)) + key_min, as key_type */
	VGPU_SHARD_OUT_I128 = 2,          /* HUGEINT from the sums of its four chunk words src[0..3] */
	VGPU_SHARD_OUT_AVG_F64 = 3,       /* FLOAT64: src[0] (a FLOAT64 sum) / count */
	VGPU_SHARD_OUT_AVG_I128 = 4,      /* FLOAT64: the 128-bit sum of src[0..3] rounded to nearest double, / count */
	VGPU_SHARD_OUT_F64_FROM_ORDER = 5 /* FLOAT64 from an order-preserving word (MIN_F64 / MAX_F64) */
} vgpu_shard_op;

typedef struct vgpu_shard_output {
	int32_t op;          /* vgpu_shard_op */
	int32_t key_type;    /* OUT_KEY: the key column's vgpu_value_type */
	int32_t key_shift;   /* OUT_KEY */
	int32_t key_bits;    /* OUT_KEY */
	int64_t key_min;     /* OUT_KEY */
	vgpu_column src[4];  /* re-aggregated columns read (INT64, FLOAT64 or HUGEINT sums; device) */
	vgpu_column count;   /* AVG ops: the merged count column (INT64 or HUGEINT) */
	void *dst;           /* device output, `rows` values of the op's type */
} vgpu_shard_output;

/* Writes each output of outs[0..n_outs) for `rows` merged groups. Queued on `stream`, not synchronized. */
vgpu_status vgpu_shard_finish(const vgpu_shard_output *outs, int32_t n_outs, uint64_t rows, void *stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* VGPU_H_ */
