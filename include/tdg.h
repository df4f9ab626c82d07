/*
 * tdg.h -- C ABI of the sm_100a kernels behind td_execute.
 *
 * Plain C: device pointers, sizes, status codes and an opaque stream handle
 * (a cudaStream_t passed as void*).  No C++ or torch types cross this line.
 * The host executor (teide_b200/csrc/host/exec.c) lowers a Teide DAG into
 * these calls; tests and the benchmark call them directly through ctypes.
 *
 * Each entry point replaces one executor loop of Teide's CPU engine
 * (src/ops/exec.c in TeideDB/teide); the replaced lines are cited beside it.
 * Status codes are td_err_t values (0 = ok).
 *
 * Memory: the caller owns every buffer.  Functions that need scratch memory
 * come with a *_plan call that reports the bytes required; the caller passes
 * a device buffer of at least that size as `ws`.  Nothing here allocates
 * device memory except the tdg_*_static entry point documented at its
 * declaration, which allocates nothing at all.
 */
#ifndef TDG_H
#define TDG_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t tdg_status;

/* A device-resident column: element data in Teide's td_t layout (dense,
 * element size from the type tag, SYM width from attrs). */
typedef struct tdg_col {
    const void* data;
    int8_t      type;      /* TD_I64, TD_F64, TD_I32, TD_SYM, ... */
    uint8_t     attrs;     /* TD_SYM_W* for TD_SYM */
    uint8_t     side;      /* join/group inputs: 0 = probe (left) row, 1 = build (right) row */
    uint8_t     pad[5];
} tdg_col;

/* ---- expression programs --------------------------------------------------
 * A predicate or computed value is a straight-line program of at most
 * TDG_MAX_INS instructions; instruction k writes register k.  Values are I64
 * or F64 (kind 0 / 1) as in Teide's expression VM (exec.c:760-918): columns
 * load as I64 unless F64, mixed comparisons and arithmetic promote to F64,
 * DIV always yields F64, comparisons and AND/OR/NOT yield 0/1 as I64. */
enum {
    TDG_X_COL = 1,   /* imm = column index into cols[]          */
    TDG_X_CONST,     /* imm = value bits (I64, or F64 bits)      */
    TDG_X_EQ, TDG_X_NE, TDG_X_LT, TDG_X_LE, TDG_X_GT, TDG_X_GE,
    TDG_X_AND, TDG_X_OR, TDG_X_NOT,
    TDG_X_ADD, TDG_X_SUB, TDG_X_MUL, TDG_X_DIV, TDG_X_MOD,
    TDG_X_NEG, TDG_X_ABS, TDG_X_MIN2, TDG_X_MAX2,
    TDG_X_TOF64, TDG_X_TOI64
};
#define TDG_MAX_INS   24
#define TDG_MAX_XCOLS 8

typedef struct tdg_ins {
    uint8_t op;        /* TDG_X_* */
    uint8_t a, b;      /* source registers */
    uint8_t kind;      /* result kind: 0 = I64, 1 = F64 */
    uint8_t pad[4];
    int64_t imm;
} tdg_ins;

typedef struct tdg_expr {
    int32_t n_ins;
    int32_t n_cols;
    int32_t out;       /* result register */
    int32_t pad;
    tdg_col cols[TDG_MAX_XCOLS];
    tdg_ins ins[TDG_MAX_INS];
} tdg_expr;

/* ---- basic services --------------------------------------------------------- */

/* min and max over n rows of an integer-class column, written as two int64
 * to d_out[0..1] (INT64_MAX / INT64_MIN when n == 0).  Feeds the
 * direct-array decision of exec_group (exec.c:5970-6010, minmax_scan_fn
 * 4544-4604). */
tdg_status tdg_minmax(tdg_col col, int64_t n, int64_t* d_out, void* stream);

/* Evaluate `e` over n rows into a dense column `out` of kind 0 (int64),
 * 1 (double) or 2 (bool bytes).  Replaces expr_eval_full (exec.c:1254-1273). */
tdg_status tdg_eval(const tdg_expr* e, int64_t n, void* out, int32_t out_kind, void* stream);

/* out[r] = vals[p] for starts[p] <= r < starts[p + 1] (p < n_runs, starts
 * ascending, starts[n_runs] = n; elements of esz = 1, 2, 4 or 8 bytes):
 * a column given as runs written out per row -- a partitioned table's
 * MAPCOMMON key, one value per partition.  Replaces materialize_mapcommon
 * (exec.c:201-243). */
tdg_status tdg_expand_runs(const void* vals, int32_t esz, const int64_t* starts, int64_t n_runs,
                           void* out, int64_t n, void* stream);

/* ---- selection (filter) -----------------------------------------------------
 * A row is selected when `pred` (may be NULL) is non-zero and, if `sel_in` is
 * given, its bit in that TD_SEL bit array is set. */

/* TD_SEL block body on the device for n rows: bits[ceil(n/64)],
 * seg_flags[ceil(n/1024)], seg_popcnt[ceil(n/1024)] and total (one int64).
 * Replaces expr_eval_full + td_sel_from_pred + td_sel_recompute
 * (exec.c:11717-11731, sel.c:77-161). */
tdg_status tdg_select_bitmap(int64_t n, const tdg_expr* pred, const uint64_t* sel_in,
                             uint64_t* bits, uint8_t* seg_flags, uint16_t* seg_popcnt,
                             int64_t* d_total, void* stream);

/* Stable compaction of the selected rows of n_cols columns.  Two calls:
 * tdg_select_count fills ws (tdg_select_ws_bytes(n) bytes) and writes the
 * number of selected rows to d_count; tdg_select_gather then writes the
 * selected rows, in row order, to dst[c] (element size of src[c]).
 * Replaces exec_filter / sel_compact / multi_gather_fn (exec.c:2065-2224,
 * 2328-2480, 1852-1899). */
size_t     tdg_select_ws_bytes(int64_t n);
tdg_status tdg_select_count(int64_t n, const tdg_expr* pred, const uint64_t* sel_in,
                            void* ws, int64_t* d_count, void* stream);
tdg_status tdg_select_gather(int64_t n, const tdg_expr* pred, const uint64_t* sel_in,
                             const void* ws, int32_t n_cols, const tdg_col* src,
                             void* const* dst, void* stream);

/* ---- group-by ----------------------------------------------------------------
 * Keys and aggregate inputs are columns (side 0 for a plain group-by).
 * Aggregates: OP_SUM, OP_COUNT, OP_MIN, OP_MAX, OP_AVG (td.h opcodes).
 * Output: one row per non-empty group; key columns keep their element type,
 * SUM is I64 (F64 for F64 input), COUNT I64, AVG F64, MIN/MAX the input
 * type class (I64 or F64) -- emit_agg_columns, exec.c:4632-4773.
 * Integer SUM wraps (two's complement) exactly like the CPU loops. */
#define TDG_MAX_KEYS 8
#define TDG_MAX_AGGS 8

typedef struct tdg_agg {
    int32_t op;
    int32_t pad;
    tdg_col in;        /* ignored for OP_COUNT */
} tdg_agg;

typedef struct tdg_group_desc {
    int64_t nrows;
    int32_t n_keys;
    int32_t n_aggs;
    tdg_col keys[TDG_MAX_KEYS];
    tdg_agg aggs[TDG_MAX_AGGS];
    /* key statistics: when have_range is set, key k lies in
     * [key_min[k], key_max[k]] for every row (from tdg_minmax or table
     * statistics).  Enables the direct-array method. */
    int32_t have_range;
    int32_t pad;
    int64_t key_min[TDG_MAX_KEYS];
    int64_t key_max[TDG_MAX_KEYS];
} tdg_group_desc;

enum { TDG_GROUP_DIRECT = 1, TDG_GROUP_HASH = 2 };

typedef struct tdg_group_plan {
    int32_t method;        /* TDG_GROUP_DIRECT or TDG_GROUP_HASH */
    int32_t smem;          /* 1 when accumulators are privatized in shared memory */
    int64_t n_slots;       /* direct-array slots or hash-table capacity */
    int64_t max_groups;    /* capacity each output column must have */
    size_t  ws_bytes;      /* scratch the run needs */
    int32_t ctas_per_sm;   /* launch shape of the streaming kernel (the vector forms of the
                              group-by and of the fused join probe): persistent CTAs per SM,
                              0 = as many as fit.  tdg_group_plan_make sets 0; the host's
                              autotuner picks it per shape class. */
    int32_t pad;
} tdg_group_plan;

typedef struct tdg_group_out {
    void*    keys[TDG_MAX_KEYS];   /* max_groups elements of the key's type */
    void*    aggs[TDG_MAX_AGGS];   /* max_groups 8-byte values */
    int64_t* d_n_groups;           /* one int64: groups written */
} tdg_group_out;

/* Choose the method and size the scratch for a group-by.  `hint_groups` is
 * an upper bound on the number of groups if the caller knows one (else 0).
 * Replaces exec_group's dispatch (exec.c:5542-6879: DA at 5948-6404,
 * radix hash table at 6406-6667). */
tdg_status tdg_group_plan_make(const tdg_group_desc* d, int64_t hint_groups,
                               tdg_group_plan* plan);

/* Run a fused select + group-by over d->nrows rows and emit the groups.
 * Direct arrays emit in ascending composite-key order; the hash method emits
 * in table order.  Returns TD_ERR_RANGE if the hash table overflowed (the
 * caller re-plans with a larger hint) and TD_ERR_DOMAIN if a key fell outside
 * the declared range. */
tdg_status tdg_group_run(const tdg_group_desc* d, const tdg_expr* pred, const uint64_t* sel_in,
                         const tdg_group_plan* plan, void* ws, const tdg_group_out* out,
                         void* stream);

/* Group-by that allocates nothing.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc -- an engine embedded in a process
 * whose device memory belongs to another runtime's caching allocator (a
 * cudaMalloc there fails or fragments that pool), or a latency-critical path
 * that cannot take cudaMalloc's implicit device synchronization.  Same inputs,
 * outputs and results as tdg_group_run, but the scratch comes from an array of
 * TDG_STATIC_SCRATCH_BYTES compiled into the library, which every GPU that
 * loads the library holds until the process exits.  `out` must hold
 * plan.max_groups rows, where tdg_group_plan_make(d, 0, &plan) gives the plan
 * (and its ws_bytes); a group-by that needs more scratch than the array holds
 * is refused with TD_ERR_RANGE.  Each call waits for its stream before it
 * returns (it reads the group count and the error word back), so no call may
 * be made while its stream is being captured into a CUDA graph.  Every call
 * shares the array, and each call re-initializes what it reads, but calls
 * that overlap on the GPU race: serialize them. */
#define TDG_STATIC_SCRATCH_BYTES (16u << 20)
tdg_status tdg_group_run_static(const tdg_group_desc* d, const tdg_expr* pred, const uint64_t* sel_in,
                                const tdg_group_out* out, void* stream);

/* ---- join ----------------------------------------------------------------------
 * Equi-join of a probe (left) side against a build (right) side on n_keys
 * key columns.  join_type 0 = inner, 1 = left outer, 2 = full outer.
 * Row ids are int32 (Teide caps both sides at INT32_MAX rows, exec.c:8139). */
typedef struct tdg_join_desc {
    int64_t n_left;
    int64_t n_right;
    int32_t n_keys;
    int32_t join_type;
    tdg_col lkeys[TDG_MAX_KEYS];
    tdg_col rkeys[TDG_MAX_KEYS];
    /* single integer key statistics of the build side (enables a direct map) */
    int32_t have_range;
    int32_t flags;         /* TDG_JOIN_PREBUILT, or 0 */
    int64_t rkey_min, rkey_max;
} tdg_join_desc;

/* tdg_join_desc.flags: the join workspace already holds this build side's
 * payload map, made by tdg_join_payload_build for the same join and group
 * descriptors.  tdg_join_group_run then reads the map and writes nothing to
 * the join workspace, so concurrent runs may share one. */
#define TDG_JOIN_PREBUILT 1

enum { TDG_JOIN_DIRECT = 1, TDG_JOIN_HASH = 2 };

typedef struct tdg_join_plan {
    int32_t method;        /* TDG_JOIN_DIRECT (key - min indexes the map) or TDG_JOIN_HASH */
    int32_t pad;
    int64_t n_slots;
    size_t  ws_bytes;
} tdg_join_plan;

/* Replaces radix_join_bits / the partition plan (exec.c:7456-7471, 8179-8200). */
tdg_status tdg_join_plan_make(const tdg_join_desc* d, tdg_join_plan* plan);

/* Build the device hash table over the build side.  Replaces
 * join_radix_partition + the build half of join_radix_build_probe_fn
 * (exec.c:7626-7742, 7824-7950) and join_build_fn (7974-8006). */
tdg_status tdg_join_build(const tdg_join_desc* d, const tdg_join_plan* plan, void* ws, void* stream);

/* Materialized join, two calls.  tdg_join_count writes the number of output
 * rows to d_count; tdg_join_emit writes them: left columns gathered by probe
 * row, right columns by build row (zero-filled where a side is unmatched in
 * an outer join).  Output order is probe-row order, then unmatched build rows
 * (full join).  Replaces the probe + consolidation + gather of exec_join
 * (exec.c:8296-8368, 8607-8728). */
tdg_status tdg_join_count(const tdg_join_desc* d, const tdg_join_plan* plan, void* ws,
                          const tdg_expr* lpred, const uint64_t* lsel, int64_t* d_count,
                          void* stream);
tdg_status tdg_join_emit(const tdg_join_desc* d, const tdg_join_plan* plan, void* ws,
                         const tdg_expr* lpred, const uint64_t* lsel,
                         int32_t n_lcols, const tdg_col* lsrc, void* const* ldst,
                         int32_t n_rcols, const tdg_col* rsrc, void* const* rdst,
                         void* stream);

/* Fused build + probe + group-by: every joined row (probe rows passing
 * lpred/lsel) is aggregated directly, with no join output materialized.  Key
 * and aggregate columns of `g` name their side (tdg_col.side); g->nrows is an
 * upper bound on joined rows.  This call builds the join table itself (do not
 * call tdg_join_build first): when the build keys are dense and unique and
 * the group-by is a direct array fed by probe-side values, the table stores
 * each key's group slot and the probe reads nothing else from the build
 * side.  Replaces exec_join followed by exec_group on its result. */
tdg_status tdg_join_group_run(const tdg_join_desc* d, const tdg_join_plan* jplan, void* jws,
                              const tdg_expr* lpred, const uint64_t* lsel,
                              const tdg_group_desc* g, const tdg_group_plan* gplan, void* gws,
                              const tdg_group_out* out, void* stream);

/* ---- hash table ------------------------------------------------------------------
 * The open-addressing table the hash group-by and hash join build on, as an
 * entry point: finds or inserts n key tuples (n_keys int64 key columns laid
 * out column-wise in kv, kv[k * n + i]) in a caller-owned table of `cap`
 * slots (a power of two): state[cap] (0 empty, 1 being written, 2 ready) and
 * keys[n_keys * cap].  d_slot[i] receives tuple i's slot, or -1.  A thread
 * that meets a slot in state 1 polls it at most spin_limit times (0: the
 * library's limit, 2^20) before it fails that row with TD_ERR_IO, so a
 * writer that never publishes ends the kernel with an error instead of a
 * hang.  Returns the first error recorded (TD_ERR_RANGE: table full);
 * d_err is one device int32 of scratch.  Synchronizes the stream.
 * Replaces the find-or-insert of group_probe_entry (exec.c:4131-4170). */
tdg_status tdg_hash_upsert(uint32_t* state, int64_t* keys, uint64_t cap, int32_t n_keys,
                           const int64_t* kv, int64_t n, int32_t spin_limit, int64_t* d_slot,
                           int32_t* d_err, void* stream);

/* The build pass of the fused join -> group-by, on its own: when the shape
 * qualifies for the payload map (unique dense integer build keys, a direct
 * group-by fed by probe-side values -- the case tdg_join_group_run probes
 * with one 4-byte map read per row), writes the map into jws and sets *used
 * to 1; otherwise (or when a build key repeats) sets *used to 0.  A caller
 * that keeps jws may then run any number of probes against it with
 * TDG_JOIN_PREBUILT -- a server answering many join queries over one
 * resident build table builds it once.  Synchronizes the stream.  The map
 * is the build half of join_radix_build_probe_fn (exec.c:7824-7950). */
tdg_status tdg_join_payload_build(const tdg_join_desc* d, const tdg_join_plan* jp, void* jws,
                                  const tdg_group_desc* g, const tdg_group_plan* gp, int32_t* used,
                                  void* stream);

/* ---- sort ------------------------------------------------------------------------
 * tdg_sort_perm: the stable permutation that orders n rows by keys[0..n_keys)
 * (keys[0] most significant).  Replaces exec_sort (exec.c:3370-3862) for
 * the key types I64, TIMESTAMP, I32, DATE, TIME, F64, SYM, BOOL, U8 and I16.
 * Each key is encoded as radix_encode_fn does (exec.c:2739-2840): DESC
 * complements the code (equal keys keep their row order), F64 follows IEEE
 * order with NaN first or last by nulls_first, and SYM sorts by
 * sym_rank[id], a device array holding the rank of each intern id's string
 * (build_enum_rank, exec.c:2876-2975); BOOL / U8 compare unsigned and I16
 * signed (sort_cmp, exec.c:2503-2558).  -0.0 sorts before +0.0 where Teide
 * radix-sorts (one key of a radix type, more than 64 rows) and equals it
 * elsewhere, as in Teide's comparator sort.  perm receives n int64 row
 * indices; ws is tdg_sort_ws_bytes(n) device bytes.  The stream is
 * synchronized once per key (the key's range sets how many digits to sort).
 * Other key types return TD_ERR_NYI.
 * tdg_gather: out[i] = in[perm[i]] for i < n_out, for any element width. */
#define TDG_MAX_SORT_KEYS 16

typedef struct tdg_sort_key {
    tdg_col         col;
    const uint32_t* sym_rank;     /* SYM keys: rank by string of every intern id; NULL otherwise */
    uint8_t         desc;
    uint8_t         nulls_first;
    uint8_t         pad[6];
} tdg_sort_key;

size_t     tdg_sort_ws_bytes(int64_t n);
tdg_status tdg_sort_perm(const tdg_sort_key* keys, int32_t n_keys, int64_t n, void* ws, int64_t* perm, void* stream);
tdg_status tdg_gather(const tdg_col* in, const int64_t* perm, int64_t n_out, void* out, void* stream);

/* ---- batched group-by ------------------------------------------------------------
 * Many independent group-bys of one shape -- one integer key column with a
 * known range, aggregates over one value column -- run as ONE persistent
 * kernel that pulls (query, tile) work items from a queue, so thousands of
 * small or uneven queries cost one launch instead of thousands.  No
 * counterpart in Teide's CPU engine (each query there is its own
 * exec_group call, exec.c:5542).
 *
 * tdg_batch_prepare uploads the work description into ws (it synchronizes);
 * tdg_batch_run is asynchronous, allocates nothing and never synchronizes,
 * so a caller can capture it in a CUDA graph once and replay it.
 * Output: rows grouped by query (query order), keys ascending within a
 * query; columns query index, key, one 8-byte column per aggregate. */
typedef struct tdg_batch_query {
    tdg_col key;           /* integer key column */
    tdg_col val;           /* value column the aggregates read */
    int64_t nrows;
    int64_t key_min;       /* every key k satisfies key_min <= k < key_min + n_slots */
    int64_t n_slots;
} tdg_batch_query;

typedef struct tdg_batch_desc {
    int32_t n_queries;
    int32_t n_aggs;        /* OP_SUM, OP_COUNT, OP_MIN, OP_MAX, OP_AVG over val */
    int32_t agg_ops[TDG_MAX_AGGS];
    const tdg_batch_query* queries;   /* host array of n_queries */
} tdg_batch_desc;

typedef struct tdg_batch_plan {
    int64_t tile_rows;     /* rows per work item (autotuned) */
    int32_t ctas_per_sm;   /* persistent CTAs per SM (autotuned) */
    int32_t smem_slots;    /* queries with at most this many slots aggregate in shared memory */
    int64_t n_items;
    int64_t total_slots;   /* capacity each output column needs */
    size_t  ws_bytes;
    int32_t n_queries;
    int32_t n_aggs;
    int32_t agg_ops[TDG_MAX_AGGS];
    int32_t val_f64;       /* the value columns are F64 (all queries alike) */
    int32_t words;         /* 8-byte words per slot record */
    int32_t threads;       /* threads per persistent CTA */
    int32_t smem_bytes;    /* dynamic shared memory per CTA */
    int32_t query_base;    /* added to every emitted query index (0 from plan_make;
                              a caller running a batch in parts sets it per part) */
    int32_t n_pieces;      /* emit units: each query's slots in pieces of 4096 */
    int32_t pad;
    const volatile int32_t* cancel;   /* device-readable word (mapped host memory) or NULL:
                                         once it reads nonzero the persistent kernel takes no
                                         further work item, so a cancelled run ends within one
                                         item per CTA (the caller reports TD_ERR_CANCEL) */
} tdg_batch_plan;

typedef struct tdg_batch_out {
    int64_t* query;                /* total_slots rows */
    int64_t* key;
    void*    aggs[TDG_MAX_AGGS];   /* 8-byte values (I64, or F64 when the value column is F64 / AVG) */
    int64_t* d_n_rows;             /* one int64: rows written */
} tdg_batch_out;

/* tile_rows / ctas_per_sm of 0 pick defaults.  ctas_per_sm also sets the
 * shared-memory budget of a persistent CTA: 1 -> 1024 threads and most of
 * the SM's shared memory, 2 -> 512 threads and half of it, otherwise 256
 * threads and 48 KB.  A query whose key range fits that budget is cut into
 * tiles of at least 8 rows per slot, so its shared aggregates are flushed
 * rarely. */
tdg_status tdg_batch_plan_make(const tdg_batch_desc* d, int64_t tile_rows, int32_t ctas_per_sm,
                               tdg_batch_plan* plan);
tdg_status tdg_batch_prepare(const tdg_batch_desc* d, const tdg_batch_plan* plan, void* ws, void* stream);
tdg_status tdg_batch_run(const tdg_batch_plan* plan, void* ws, const tdg_batch_out* out, void* stream);

/* Device properties used by the planners (SM count, shared memory). */
int32_t tdg_device_sm_count(void);

/* ---- instrumentation ----------------------------------------------------------
 * With timing on, each tdg_group_run / tdg_join_group_run records CUDA events
 * around its main streaming kernel (the fused select [+ probe] + aggregate
 * launch) on the stream it was given, and tdg_join_build around its build
 * kernel; the last durations are read back here in milliseconds.  Timing
 * adds no synchronization beyond the one each call already does, except in
 * tdg_batch_run, which waits for its aggregation kernel's end event (and
 * records nothing while its stream is being captured into a CUDA graph), and
 * tdg_sort_perm, which waits for its end event. */
void     tdg_set_timing(int32_t on);
int32_t  tdg_timing_enabled(void);
/* A host that replays captured tdg launches (a CUDA graph) counts them here. */
void     tdg_count_launches(uint64_t n);
float    tdg_last_main_ms(void);
float    tdg_last_build_ms(void);
float    tdg_last_sort_ms(void);    /* the last tdg_sort_perm (timing on), CUDA events */
/* Kernels launched by this library since the process started. */
uint64_t tdg_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* TDG_H */
