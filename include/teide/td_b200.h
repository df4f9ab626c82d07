/*
 * teide/td_b200.h -- extensions of the B200 executor beyond Teide's td.h.
 *
 * Teide keeps every table in host memory.  Here a table can be made
 * resident in the GPU's HBM so that repeated queries skip the host->device
 * copy; td_execute uses the resident copy of any column it finds.  Results
 * are always ordinary host td_t objects.
 */
#ifndef TD_B200_H
#define TD_B200_H

#include "teide/td.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Number of CUDA devices visible to the process (0 when none). */
int      td_gpu_device_count(void);

/* Make every column of `tbl` resident on the current GPU (uploads now and
 * computes per-column min/max statistics for integer columns).  The copy is
 * dropped by td_gpu_unpin, or when a column is freed or mutated through the
 * td_* API.  Writes made through td_data() after pinning are not seen:
 * unpin and pin again. */
td_err_t td_gpu_pin(td_t* tbl);
void     td_gpu_unpin(td_t* tbl);

/* Upper bound on device bytes the executor may hold (0 = no limit).  A query
 * that would exceed it fails with TD_ERR_OOM; resident tables count too. */
void     td_gpu_set_mem_limit(size_t bytes);

typedef struct {
    uint64_t h2d_bytes;        /* host->device bytes of the last td_execute */
    uint64_t d2h_bytes;        /* device->host bytes of the last td_execute */
    uint64_t kernel_calls;     /* tdg_* kernel entry points it called */
    uint64_t dev_bytes_live;   /* device bytes held now (resident + cached) */
    uint64_t dev_bytes_peak;
    int32_t  last_group_method;/* 1 direct array, 2 hash table, 0 none */
    int32_t  last_join_method; /* 1 direct map, 2 hash table, 0 none */
    int32_t  last_fused;       /* 1 when the last query ran a fused kernel */
    int32_t  pad;
} td_gpu_stats_t;

void     td_gpu_last_stats(td_gpu_stats_t* out);

/* Release cached device memory that no resident table uses. */
void     td_gpu_trim(void);

/* Device address of a column's resident copy (td_gpu_pin, or a result left
 * on the device), or NULL.  Valid while the column is resident. */
const void* td_gpu_col_data(td_t* col);

/* td_execute of a group-by whose result stays on the device: the returned
 * table has the result's columns, names, types and lengths, each resident
 * (td_gpu_col_data), but their host elements are NOT written until
 * td_gpu_fetch(tbl) copies them down.  For a consumer that continues on the
 * GPU -- a partial group-by that crosses NVLink to be merged on another GPU
 * -- so the rows never cross PCIe.  Roots other than td_group return
 * TD_ERR_NYI.  No counterpart in Teide. */
td_t*    td_execute_device(td_graph_t* g, td_op_t* root);
/* Copy every resident column of tbl (or the vector tbl) to its host elements. */
td_err_t td_gpu_fetch(td_t* tbl);

/* Run n group-by graphs as one batched GPU launch.  Each graph is a
 * td_group over its bound table with one integer key (td_scan) and
 * aggregates reading one value column (td_scan; COUNT may read anything),
 * with the same aggregate list and column types in every graph, and keys
 * dense enough for direct indexing (key range at most max(2^20, 4 x rows));
 * anything else returns TD_ERR_NYI (TD_ERR_TYPE for mixed column types).  The result is ONE table: "_query" (index into graphs), the key
 * column, then one column per aggregate (named as td_group names them), rows
 * grouped by query in argument order with keys ascending.  A repeated batch
 * (same tables, same key ranges) replays a cached CUDA graph; its tile size
 * and CTA count come from an autotuner whose choices persist in a JSON file
 * ($TD_TUNE_CACHE, else ~/.cache/teide_b200_tune.json). */
td_t*    td_execute_batch(td_graph_t** graphs, td_op_t** roots, int64_t n);
void     td_gpu_batch_cache_clear(void);

/* ---- serving: a request loop over resident tables ------------------------------
 * td_server_new starts `slots` worker threads.  Each pulls submitted requests
 * in arrival order and runs td_execute on its own CUDA stream, so up to
 * `slots` queries are in flight on the GPU at once and a request that arrives
 * while others run starts as soon as a slot frees up and its estimated device
 * bytes fit in the budget (hbm_budget, or 0 for 90% of the GPU's free memory
 * when the server starts).  The queue head is never bypassed; a request that
 * alone exceeds the budget runs when nothing else is in flight.  Requests of
 * one td_execute_batch shape (below) that wait behind each other run as one
 * batched launch, one at a time, each still getting its own result table.
 *
 * Each submitted graph must stay alive, and must not be executed elsewhere,
 * until td_server_wait has returned its result.  est_bytes = 0 asks
 * td_server_estimate.  td_server_submit returns a ticket >= 0, or a negated
 * td_err_t (TD_ERR_RANGE when queue_cap requests are already outstanding).
 * td_server_wait blocks until that ticket's result is ready and hands it to
 * the caller (release it with td_release); the times are CLOCK_MONOTONIC
 * nanoseconds.  td_server_free finishes every queued request, then stops. */
typedef struct td_server td_server_t;

typedef struct {
    int64_t submit_ns;          /* td_server_submit */
    int64_t start_ns;           /* a worker started td_execute */
    int64_t end_ns;             /* the result table was complete on the host */
    int64_t est_bytes;          /* device bytes reserved for it while it ran */
    int32_t status;             /* td_err_t of the execution */
    int32_t in_flight_at_start; /* queries running (itself included) when it started */
} td_server_timing_t;

typedef struct {
    uint64_t completed;
    int64_t  queued;            /* submitted, not yet started */
    int32_t  in_flight;
    int32_t  peak_in_flight;
    int32_t  slots;
    int32_t  pad;
    uint64_t budget_bytes;
    uint64_t reserved_bytes;
    uint64_t peak_reserved_bytes;
} td_server_stats_t;

td_server_t* td_server_new(int32_t slots, size_t hbm_budget, int64_t queue_cap);
int64_t      td_server_submit(td_server_t* s, td_graph_t* g, td_op_t* root, size_t est_bytes);
td_t*        td_server_wait(td_server_t* s, int64_t ticket, td_server_timing_t* timing);
/* n requests in one call (tickets[i] as td_server_submit returns them; the
 * call stops at the first refusal and returns how many were submitted), and
 * their results in one call (results[i], timings[i] may be NULL), in ticket
 * order: a client with many small queries pays one call, not n. */
int64_t      td_server_submit_many(td_server_t* s, td_graph_t** graphs, td_op_t** roots, int64_t n,
                                   int64_t* tickets);
void         td_server_wait_many(td_server_t* s, const int64_t* tickets, int64_t n, td_t** results,
                                 td_server_timing_t* timings);
void         td_server_stats(td_server_t* s, td_server_stats_t* out);
void         td_server_free(td_server_t* s);
/* Device bytes a query may need beyond resident columns: uploads of columns
 * that are not resident plus a per-row scratch bound (128 bytes per row of the
 * largest input table, 16 per row of the others). */
size_t       td_server_estimate(td_graph_t* g, td_op_t* root);

/* td_splay_load, then every column made resident in HBM (td_gpu_pin): a
 * splayed table straight into device memory.  No counterpart in Teide. */
td_t*        td_gpu_splay_load(const char* dir);
/* td_part_load, then every column made resident in HBM.  No counterpart in Teide. */
td_t*        td_gpu_part_load(const char* db_root, const char* table_name);

#ifdef __cplusplus
}
#endif

#endif /* TD_B200_H */
