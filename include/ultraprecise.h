/*
 * ultraprecise.h — C ABI of the B200 exact-decimal execution path.
 *
 * Every entry point takes plain pointers and sizes.  Device buffers are owned
 * by the caller unless an entry point says otherwise; launches are ordered on
 * the caller's CUDA stream (passed as `void*`, a cudaStream_t) and never
 * synchronise implicitly.  No exception crosses this boundary: every function
 * returns an up_status, and up_last_error_message() gives the detail of the
 * last failure on the calling thread.
 *
 * Reference interfaces replaced (file:line in lx0623/UltraPrecise):
 *   - compact decimal layout, GetDecimalRealBytes
 *       src/datatypes/decimal.hxx:91-92,126-128; src/datatypes/decimal.cu:92,464-467
 *   - precision -> limb table                  src/AriesDataType.cu:7-16
 *   - type derivation / AlignOptimize           src/AriesEngineWrapper/AriesEngineShell.cpp:90-685
 *   - JIT compile + module cache                src/CudaAcc/DynamicKernel.h:50-117, DynamicKernel.cu:61-158
 *   - expression kernel launch (CallKernel)     src/CudaAcc/DynamicKernel.cu:281-338
 *   - expression node (AEExprCalcNode)          src/AriesEngine/AriesExprCalcNode.h:242-295
 *   - kernel input iterator                     src/AriesColumnDataIterator.hxx:8-41
 *   - grouped SUM/COUNT (AggregateColumnData)   src/CudaAcc/AriesSqlOperator_group.cu:360-424
 *   - AVG division (DivisionInt64)              src/CudaAcc/AriesSqlOperator_helpers.cu:717-763
 */
#ifndef ULTRAPRECISE_H_
#define ULTRAPRECISE_H_

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UP_ABI_VERSION 1

/* ------------------------------------------------------------------ status */
typedef int32_t up_status;
enum {
    UP_OK = 0,
    UP_ERR_INVALID_ARG = 1,   /* bad pointer, size, precision, tree shape */
    UP_ERR_UNSUPPORTED = 2,   /* valid request outside what this build implements */
    UP_ERR_CUDA = 3,          /* a CUDA runtime call failed */
    UP_ERR_COMPILE = 4,       /* NVRTC rejected the generated kernel */
    UP_ERR_NO_MEMORY = 5,     /* device or host allocation failed / admission refused */
    UP_ERR_TIMEOUT = 6,       /* a bounded wait ran out */
    UP_ERR_QUEUE_FULL = 7,    /* serving queue has no free slot */
    UP_ERR_NOT_READY = 8,     /* asynchronous result not complete yet */
    UP_ERR_NO_DEVICE = 9      /* no CUDA device visible */
};

/* Per-launch device error word bits (OR-ed over all rows).  The reference
 * drops its decimal error byte at store time (AriesDecimal.hxx:308-313); this
 * path reports it instead. */
enum {
    UP_ROWERR_OVERFLOW = 1u,     /* the value did not fit the compact field: bits were lost */
    UP_ROWERR_DIV_BY_ZERO = 2u,  /* a divisor was zero (ERR_DIV_BY_ZERO, decimal.hxx:28) */
    UP_ROWERR_DOMAIN = 4u,       /* an input outside the supported domain (e.g. bad group id) */
    UP_ROWERR_TIMEOUT = 8u       /* a bounded wait in the kernel ran out: the launch's results are incomplete */
};

const char* up_status_string(up_status s);
const char* up_last_error_message(void);
int32_t up_abi_version(void);

/* -------------------------------------------------------- compact layout */
/* Bytes per compact value of precision p: the reference table for p < 300
 * (decimal.cu:92), ceil((bitlen(10^p-1)+1)/8) beyond it.  Returns -1 for p<1. */
int32_t up_compact_bytes(int32_t precision);
/* The reference's precision -> 32-bit word table (AriesDataType.cu:7); for
 * p >= 300 ceil((bitlen(10^p-1)+1)/32).  Used only to report the reference's
 * own limb choice; this path sizes limbs from value bounds. */
int32_t up_precision_words(int32_t precision);
/* Largest precision this build accepts. */
int32_t up_max_precision(void);

/* ---------------------------------------------------------- expressions */
enum {
    UP_NODE_COLUMN = 0,   /* input column `column` */
    UP_NODE_CONST = 1,    /* decimal constant: const_sign, scale, const_limbs */
    UP_NODE_INT = 2,      /* integer literal (only before up_expr_align_optimize) */
    UP_NODE_ADD = 3,
    UP_NODE_SUB = 4,
    UP_NODE_MUL = 5,
    UP_NODE_DIV = 6,
    UP_NODE_MOD = 7,
    UP_NODE_LT = 10,      /* comparisons produce one byte per row: 0 / 1 */
    UP_NODE_LE = 11,
    UP_NODE_GT = 12,
    UP_NODE_GE = 13,
    UP_NODE_EQ = 14,
    UP_NODE_NE = 15,
    UP_NODE_AND = 16,     /* AND / OR of two boolean nodes (comparisons or AND/OR): one byte per row, */
    UP_NODE_OR = 17,      /* the reference's and_or_expr kernels (AriesExprCalcNode.cpp:667-760) */
    UP_NODE_RESCALE = 20  /* extension: truncate toward zero (or widen) to `scale` */
};

#define UP_CONST_MAX_LIMBS 128

/* One node of a typed expression tree (or DAG: a node may be shared).
 * Nodes are referenced by index; `left`/`right` are -1 when unused.
 * `precision`/`scale` are the node's result type (filled by
 * up_expr_derive_types for inner nodes; given for COLUMN and CONST).
 * `reverse` negates the node's value (the reference's value_reverse,
 * AriesCommonExpr.cpp:1678-1680). */
typedef struct up_expr_node {
    int32_t kind;
    int32_t left;
    int32_t right;
    int32_t column;
    int32_t precision;
    int32_t scale;
    int32_t reverse;
    int32_t const_sign;
    int32_t const_nlimbs;
    int64_t int_value;                         /* UP_NODE_INT */
    uint32_t const_limbs[UP_CONST_MAX_LIMBS];  /* little-endian magnitude */
} up_expr_node;

/* Column type descriptor for compile-time typing. */
typedef struct up_col_type {
    int32_t precision;
    int32_t scale;
    int32_t nullable;   /* 1: values are preceded by a flag byte */
} up_col_type;

/* Fill precision/scale of every inner node with the reference rules
 * (AriesEngineShell.cpp:90-144): ADD/SUB p = max(p1-s1,p2-s2)+1+max(s1,s2);
 * MUL p = p1+p2, s = s1+s2; DIV p = p1-p2+s2+5, s = s1+4; MOD p = p2, s = 0. */
up_status up_expr_derive_types(up_expr_node* nodes, int32_t n_nodes, int32_t root,
                               const up_col_type* cols, int32_t n_cols);

/* The reference's AlignOptimize rewrite (AriesEngineShell.cpp:244-685):
 * a-b -> a+(-b), n-ary flattening, addends sorted by scale, integer/decimal
 * constant folding, zero elimination, left-deep rebuild, re-typing.
 * Writes at most `cap` nodes to `out`. */
up_status up_expr_align_optimize(const up_expr_node* in, int32_t n_in, int32_t root,
                                 const up_col_type* cols, int32_t n_cols,
                                 up_expr_node* out, int32_t cap, int32_t* n_out, int32_t* out_root);

/* ------------------------------------------------------------- columns */
/* Kernel input: the AriesColumnDataIterator shape (AriesColumnDataIterator.hxx:8-41).
 * Fast path: `data` non-NULL, n_blocks == 0, indices == NULL: rows are
 * contiguous, `value_bytes` apart.  Block path: `blocks` is a DEVICE array of
 * n_blocks block pointers and `block_prefix` a DEVICE array of n_blocks+1 row
 * prefix sums.  `indices` (DEVICE, int32) maps row i to a data row; -1 = NULL. */
typedef struct up_column {
    const void* data;
    const void* const* blocks;
    const int64_t* block_prefix;
    int32_t n_blocks;
    const int32_t* indices;
    int32_t precision;
    int32_t scale;
    int32_t value_bytes;   /* must equal up_compact_bytes(precision) (+1 if nullable) */
    int32_t nullable;
} up_column;

/* ------------------------------------------------ JIT expression module */
typedef struct up_module up_module;

typedef struct up_compile_opts {
    int32_t threads_per_value;   /* 0 = autotuned default; else 1,2,4,8,16,32 */
    int32_t block_threads;       /* 0 = default */
    int32_t flags;               /* reserved, 0 */
} up_compile_opts;

/* Compile a typed expression (root = result) into a CUDA kernel for sm_100a.
 * The module cache is keyed by the generated source; compiling the same
 * expression twice returns a module sharing one cubin. */
up_status up_module_compile(const up_expr_node* nodes, int32_t n_nodes, int32_t root,
                            const up_col_type* cols, int32_t n_cols,
                            const up_compile_opts* opts, up_module** out);
/* Result type of the module: precision, scale, bytes per output row. */
up_status up_module_result_type(const up_module* m, int32_t* precision, int32_t* scale,
                                int32_t* value_bytes);
/* Generated CUDA source (AEExprCalcNode::GetCudaKernelCode); returns the
 * length; copies at most cap-1 bytes + NUL when buf is non-NULL. */
int64_t up_module_source(const up_module* m, char* buf, int64_t cap);
/* Launch over `rows` rows.  `out` is a device buffer of rows*value_bytes.
 * `err_word` (device uint32, may be NULL) receives UP_ROWERR_* bits OR-ed. */
up_status up_expr_launch(up_module* m, const up_column* in, int32_t n_in, int64_t rows,
                         void* out, uint32_t* err_word, void* stream);
/* One launch over n_req requests of the same expression module: request k
 * reads columns in[k*n_in .. k*n_in+n_in) over rows[k] rows and writes outs[k];
 * errs[k] (device uint32, may be NULL) receives its row errors.  Requests of
 * contiguous non-null columns on a one-thread-per-value module share one
 * kernel (virtual tiles over all requests); otherwise each request is launched
 * on its own.  Results equal launching each request alone.  The request
 * descriptors go through a stream-ordered allocation.  No counterpart in the
 * reference (one kernel per expression and call, DynamicKernel.cu:281-338). */
up_status up_expr_launch_many(up_module* m, const up_column* in, int32_t n_in, const int64_t* rows, int32_t n_req,
                              void* const* outs, uint32_t* const* errs, void* stream);

/* Threads that cooperate on one value in the module's kernel (1: one thread
 * per value; 2..32: the cooperative form), as chosen at compile time. */
int32_t up_module_threads_per_value(const up_module* m);
void up_module_release(up_module* m);
/* Number of cached compiled kernels; clears the cache when clear != 0. */
int32_t up_module_cache_size(int32_t clear);

/* ------------------------------------------------- grouped aggregation */
enum { UP_AGG_COUNT = 0, UP_AGG_SUM = 1, UP_AGG_AVG = 2 };

/* Output image of SUM/AVG per group: the reference's nullable_type<Decimal>
 * (kernel_segreduce.hxx:609-612): flag, sign, prec, frac, error, v[32]. */
#define UP_AGG_DECIMAL_BYTES 133

/* Exact grouped aggregation of compact decimal columns by dense group id.
 * vals[k] with kinds[k]; group_ids is a DEVICE int32 array of `rows` ids in
 * [0, n_groups); outs[k] is a DEVICE buffer of n_groups*133 bytes (SUM/AVG)
 * or n_groups int64 (COUNT; vals[k] ignored).  Scratch is allocated
 * stream-ordered by the library. */
up_status up_group_agg(const up_column* vals, const int32_t* kinds, int32_t n_vals,
                       const int32_t* group_ids, int32_t n_groups, int64_t rows,
                       void* const* outs, uint32_t* err_word, void* stream);

/* AggregateColumnData form (AriesSqlOperator_group.cu:360-424): rows are
 * visited through `associated` (DEVICE int32 permutation) and grouped by
 * `group_starts` (DEVICE int32, n_groups ascending segment starts).  One
 * aggregate per call; `out` as in up_group_agg. */
up_status up_aggregate_column_data(const up_column* src, int32_t kind,
                                   const int32_t* associated, const int32_t* group_starts,
                                   int32_t n_groups, int64_t rows, void* out,
                                   uint32_t* err_word, void* stream);

/* DivisionInt64 (AriesSqlOperator_helpers.cu:717): out[i] = sums[i] / counts[i]
 * with the reference's divide rule (scale+4, half-up); 133-byte images. */
up_status up_division_int64(const void* sums, const int64_t* counts, int32_t n,
                            void* out, void* stream);

/* Dense group ids from up to 4 fixed-width byte key columns (CHAR(n), n<=8
 * bytes per key column, total <= 2 bytes handled by a direct table; wider
 * keys by sort).  Ids follow ascending key order, like the reference's
 * sort-based GroupColumns (AriesSqlOperator_group.cu:14-54).
 * key_cols: DEVICE pointers; key_bytes: bytes per key column.  Writes
 * `group_ids` (DEVICE int32, rows), *n_groups, and optionally the distinct
 * keys (DEVICE, n_groups * sum(key_bytes)) into `group_keys`. */
up_status up_group_ids_from_keys(const void* const* key_cols, const int32_t* key_bytes,
                                 int32_t n_keys, int64_t rows, int32_t* group_ids,
                                 int32_t* n_groups, void* group_keys, void* stream);

/* The grouping of up_group_ids_from_keys without the per-row id array: one
 * pass over the key bytes marks the keys present, and `key_table` (DEVICE
 * int32, UP_KEY_TABLE_ENTRIES entries) receives in entries [0, 65536) each
 * possible key's dense id in ascending key order (-1 where absent), in
 * entries [65536, 65536 + n_groups) the key of each id, and the group count
 * in entry UP_KEY_TABLE_COUNT.  A key is its bytes in column order, most
 * significant first.  Synchronises `stream` to return *n_groups. */
#define UP_KEY_TABLE_ENTRIES 131088
#define UP_KEY_TABLE_COUNT 131072 /* entry holding the group count */
up_status up_group_table_from_keys(const void* const* key_cols, const int32_t* key_bytes,
                                   int32_t n_keys, int64_t rows, int32_t* key_table,
                                   int32_t* n_groups, void* group_keys, void* stream);

/* up_query_launch with the GROUP BY keys read by the query kernel itself
 * (GroupColumns + AggregateColumnData fused, AriesSqlOperator_group.cu:14-54,
 * 360-424): each row's group is key_table[key] of its key bytes, so no group
 * id array is written or read.  Key columns: one of 1 or 2 bytes, or two of 1
 * byte (DEVICE); key_table and n_groups from up_group_table_from_keys. */
up_status up_query_launch_keys(up_module* query, const up_column* in, int32_t n_in, int64_t rows,
                               const void* const* key_cols, const int32_t* key_bytes, int32_t n_keys,
                               const int32_t* key_table, int32_t n_groups, void* const* outs,
                               uint32_t* err_word, void* stream);

/* The same pair without a round trip to the host: the table call does not
 * synchronise, and the query reads the group count from the table on the
 * device, choosing its accumulation mode there.  Outputs are sized for
 * `max_groups` groups (1..65536); a count above it sets UP_ROWERR_DOMAIN and
 * leaves the outputs unwritten.  The group count is read back by the caller
 * from entry UP_KEY_TABLE_COUNT when it needs it. */
up_status up_group_table_from_keys_async(const void* const* key_cols, const int32_t* key_bytes,
                                         int32_t n_keys, int64_t rows, int32_t* key_table,
                                         void* group_keys, void* stream);
up_status up_query_launch_keys_async(up_module* query, const up_column* in, int32_t n_in, int64_t rows,
                                     const void* const* key_cols, const int32_t* key_bytes, int32_t n_keys,
                                     const int32_t* key_table, int32_t max_groups, void* const* outs,
                                     uint32_t* err_word, void* stream);

/* ------------------------------------- fused expression + group aggregate */
typedef struct up_query_agg {
    int32_t kind;       /* UP_AGG_* */
    int32_t root;       /* expression root node index (ignored for COUNT) */
} up_query_agg;

/* One kernel computes every aggregate's expression per row and accumulates
 * it by group without materialising the expression results. */
up_status up_query_compile(const up_expr_node* nodes, int32_t n_nodes,
                           const up_col_type* cols, int32_t n_cols,
                           const up_query_agg* aggs, int32_t n_aggs,
                           const up_compile_opts* opts, up_module** out);
up_status up_query_launch(up_module* m, const up_column* in, int32_t n_in, int64_t rows,
                          const int32_t* group_ids, int32_t n_groups,
                          void* const* outs, uint32_t* err_word, void* stream);

/* up_query_launch for callers that cannot allocate device memory (no
 * counterpart in the reference; the reference allocates its aggregation
 * buffers itself).  Same arguments and results as up_query_launch, but the
 * per-group accumulators live in an 8 MiB file-scope device array of the
 * library instead of stream-ordered allocations, so the call performs no
 * cudaMalloc/cudaFree and no allocating library call.  Requests whose
 * accumulators do not fit (n_groups x accumulator bytes + 8 bytes per group)
 * fail with UP_ERR_INVALID_ARG.  Every GPU that loads the library holds the
 * array until exit; all calls share it, each call clears what it uses on its
 * stream, and calls that overlap on the GPU race.  Every call looks the
 * array's address up in the current context (the first one on a device also
 * loads the library's module there): make the first call on a device before
 * any stream capture. */
up_status up_query_launch_noalloc(up_module* m, const up_column* in, int32_t n_in, int64_t rows,
                                  const int32_t* group_ids, int32_t n_groups,
                                  void* const* outs, uint32_t* err_word, void* stream);

/* Launch over columns in HOST memory (page-locked for full speed): the rows
 * are cut into chunks whose inputs are copied in, computed and copied back
 * out on three streams, so copies in, kernels and copies out of successive
 * chunks overlap.  Contiguous non-null columns (up_column.data is the host
 * pointer); host_out receives rows * value_bytes.  chunk_rows 0 = about 64 MB
 * of input per chunk.  Returns when host_out holds every row; *err_word
 * (host, may be NULL) receives the OR of the row errors. */
up_status up_expr_launch_host(up_module* m, const up_column* host_in, int32_t n_in, int64_t rows,
                              void* host_out, uint32_t* err_word, int64_t chunk_rows);

/* ---------------------------------------------------- decimal text in/out */
/* Parse decimal text into a compact DECIMAL(precision, scale) column, as the
 * reference's CSV import does (Decimal(precision, scale, mode, str),
 * decimal.cu:158-165; StringToDecimal :2980-3025; cast :471-533): field r is
 * text[offsets[r] .. offsets[r+1]) (DEVICE buffers; offsets has rows+1
 * entries); an optional '-', digits, at most one '.'; extra fraction digits
 * are cut off (truncation), missing ones padded.  Other characters flag
 * UP_ROWERR_DOMAIN (the row stores 0); lost magnitude bits flag
 * UP_ROWERR_OVERFLOW.  precision <= 1000, fields of up to 1500 digits. */
up_status up_parse_decimal(const char* text, const int64_t* offsets, int64_t rows, int32_t precision, int32_t scale,
                           void* out, uint32_t* err_word, void* stream);

/* Characters one formatted value of DECIMAL(precision, .) can need. */
int32_t up_format_width(int32_t precision, int32_t hex);

/* Format a compact column into fixed-width slots of `width` characters (DEVICE
 * out_text of rows*width bytes; out_len[r] = characters written, -1 when the
 * slot is too small).  hex != 0: the reference's output image
 * (Decimal::GetDecimal, decimal.cu:362-398: sign, 8 upper-case hex digits per
 * limb from the highest nonzero one, "(fff)" scale); hex == 0: the decimal
 * string ("-123.4500"), which parses back to the same bytes. */
up_status up_format_decimal(const void* compact, int64_t rows, int32_t precision, int32_t scale, int32_t hex,
                            char* out_text, int32_t width, int32_t* out_len, void* stream);

/* --------------------------------------------------------------- filters */
/* Row selection (FilterFlags / FilterAssociated, AriesSqlOperator_filter.h:15-19):
 * the indices of the rows whose flag byte is nonzero, in row order, into
 * `indices` (DEVICE, room for `rows` entries); *count (DEVICE int64) receives
 * how many.  `flags` is typically the output of a module whose root is a
 * comparison or an AND/OR of comparisons.  rows <= 2^31-1. */
up_status up_filter_flags(const uint8_t* flags, int64_t rows, int32_t* indices, int64_t* count, void* stream);

/* ------------------------------------------------------------ utilities */
/* Measured device facts used by the roofline report. */
typedef struct up_device_info {
    int32_t sm_count;
    int32_t cc_major, cc_minor;
    int64_t free_bytes, total_bytes;
    char name[128];
} up_device_info;
up_status up_device_query(int32_t device, up_device_info* info);

#ifdef __cplusplus
}
#endif
#endif /* ULTRAPRECISE_H_ */
