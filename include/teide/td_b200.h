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

#ifdef __cplusplus
}
#endif

#endif /* TD_B200_H */
