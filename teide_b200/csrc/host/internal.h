/*
 * Internal declarations shared by the host-side C17 sources of
 * libteide_b200.so.  Nothing here is part of the public ABI.
 */
#ifndef TDB_INTERNAL_H
#define TDB_INTERNAL_H

#include "teide/td.h"
#include "teide/td_b200.h"
#include "tdg.h"
#include <stdatomic.h>

/* ---- heap ------------------------------------------------------------------
 * Every block carries a 64-byte hidden prefix in front of its td_t header.
 * Blocks of 2 MB and more come from mmap (pages committed on first touch)
 * and are page-locked on their first upload to the GPU, so host->device
 * copies of large columns run at PCIe/C2C link speed. */
typedef struct tdb_block_prefix {
    uint32_t magic;
    uint32_t kind;          /* TDB_BLK_MALLOC, TDB_BLK_MMAP or TDB_BLK_FILE */
    void*    raw;           /* start of the OS allocation */
    size_t   raw_size;      /* bytes of the OS allocation */
    _Atomic(size_t) pinned; /* bytes page-locked with cudaHostRegister */
    uint64_t serial;        /* allocation serial: device mirrors key on it */
    uint8_t  pad[24];
} tdb_block_prefix;

/* The header that follows the prefix must keep the 32-byte alignment td.h
 * declares for td_t (TD_ALIGN(32), td_data assumed 32-byte aligned): the
 * OS allocation is 64-byte (small blocks) or page aligned (large ones). */
_Static_assert(sizeof(tdb_block_prefix) == 64, "block prefix must be 64 bytes");

#define TDB_BLK_MAGIC 0x7D6B1C0Au
#define TDB_BLK_MALLOC 1u
#define TDB_BLK_MMAP   2u
#define TDB_BLK_FILE   3u       /* a column file mapped copy-on-write (td_col_mmap) */

/* The mapping at `base` (page aligned, `total` bytes) holds a column file at
 * base + 4096; its prefix goes at the end of the first (anonymous) page.
 * Returns the file's header as a heap block; td_free unmaps the whole range. */
td_t* tdb_file_block(void* base, size_t total);

static inline tdb_block_prefix* tdb_prefix(td_t* v) {
    return (tdb_block_prefix*)((char*)v - sizeof(tdb_block_prefix));
}

void     tdb_retain_owned_refs(td_t* v);
int      tdb_is_heap_block(td_t* v);
uint64_t tdb_block_serial(td_t* v);

/* ---- atoms / vectors -------------------------------------------------------- */
int64_t tdb_vec_capacity(td_t* v);
int     tdb_atom_numeric(td_t* a, double* f, int64_t* i, int* is_f64);

/* ---- graph ------------------------------------------------------------------ */
td_op_ext_t* tdb_find_ext(td_graph_t* g, uint32_t id);

/* ---- GPU residency (gpu.c) ---------------------------------------------------- */
typedef struct tdb_devcol {
    void*    dptr;      /* device copy of the element data */
    int64_t  len;
    int8_t   type;
    uint8_t  attrs;
    int      has_stats; /* min/max valid */
    int64_t  kmin, kmax;
} tdb_devcol;

/* execution context of one td_execute call */
typedef struct tdb_ctx {
    void*    stream;            /* cudaStream_t */
    int      device;
    /* transient device buffers freed at the end of the call */
    void**   tmp;
    int      n_tmp, cap_tmp;
    /* host->device bytes uploaded in this call (for statistics) */
    uint64_t h2d_bytes, d2h_bytes;
    int      n_scalar;          /* mapped host scalars handed out in this call */
    /* device->host copies queued into the staging buffer (tdb_d2h_async) */
#define TDB_PENDING 32
    struct { void* host; void* stage; size_t bytes; } pending[TDB_PENDING];
    int      n_pending;
    size_t   stage_used;
    size_t   out_used;          /* mapped result area handed out in this call (tdb_host_out) */
} tdb_ctx;

int      tdb_gpu_ensure(void);                 /* 0 ok, else td_err_t */
int      tdb_gpu_available(void);              /* 1 if a CUDA device exists */
void*    tdb_dev_alloc(tdb_ctx* c, size_t bytes);   /* transient, freed by ctx_end */
void*    tdb_dev_alloc_persistent(size_t bytes);
void     tdb_dev_free_persistent(void* p);
int      tdb_ctx_begin(tdb_ctx* c);
void     tdb_ctx_end(tdb_ctx* c);
int      tdb_ctx_sync(tdb_ctx* c);               /* 0 ok, else td_err_t */
/* An int64 in page-locked host memory that kernels can write through the
 * returned device pointer (*dev): once the stream has synchronized, the host
 * reads it with no copy.  Valid until the end of the call; NULL if none left. */
volatile int64_t* tdb_host_scalar(tdb_ctx* c, void** dev);
/* Page-locked, device-mapped host memory for small results (TDB_OUT_BYTES per
 * thread, handed out per call): kernels write it directly, so the host reads
 * it after the stream synchronizes with no copy.  NULL when it does not fit. */
#define TDB_OUT_BYTES ((size_t)1 << 20)
void*    tdb_host_out(tdb_ctx* c, size_t bytes, void** dev);
/* 1 when `p` lies in page-locked memory (a copy to it can be asynchronous). */
int      tdb_host_is_pinned(const void* p);
/* Device->host copy queued on the call's stream; tdb_ctx_sync completes it. */
int      tdb_d2h_async(tdb_ctx* c, void* host, const void* dev, size_t bytes);
/* device view of a host column, copied into *out; uploads it unless it is
 * resident.  want_stats asks for min/max of an integer column. */
int      tdb_col_device(tdb_ctx* c, td_t* col, int want_stats, tdb_devcol* out);
void     tdb_note_kernel(void);
void     tdb_note_methods(int group, int join, int fused);
void     tdb_reset_methods(void);
int      tdb_d2h(tdb_ctx* c, void* host, const void* dev, size_t bytes);
int      tdb_h2d(tdb_ctx* c, void* dev, const void* host, size_t bytes);
void     tdb_mirror_forget(td_t* v);             /* host block freed or mutated */
int     tdb_adopt_mirror(tdb_ctx* c, td_t* host, void* dptr);
void     tdb_pin_host(td_t* v);                  /* page-lock a large host block */
int      tdb_check_cancel(void);
/* Device address of the cancel word (NULL before the GPU is initialized);
 * tdb_cancel_reset clears it and the host flag when a query starts. */
const volatile int32_t* tdb_cancel_word(void);
void     tdb_cancel_reset(void);

extern _Atomic(int) tdb_cancel_flag;

/* ---- executor ------------------------------------------------------------------ */
td_t* tdb_exec(td_graph_t* g, td_op_t* root, int dev_only);
/* Phase tracing: with TD_TRACE set in the environment, each call prints the
 * microseconds since this thread's td_execute began and a label to stderr. */
void  tdb_trace(const char* what);
void  tdb_trace_begin(void);

/* 1 when the column (or a slice's parent) has a resident device copy. */
int   tdb_col_resident(td_t* col);
/* Identity of a column's resident device copy: unique to that copy (a copy
 * made again after the column was freed, mutated or unpinned gets a new
 * one); 0 when the column has none or is a slice. */
uint64_t tdb_col_stamp(td_t* col);

/* ---- autotuner persistence (host/batch.c) ------------------------------------------
 * One JSON object in $TD_TUNE_CACHE (else ~/.cache/teide_b200_tune.json), one
 * entry per shape class: {"tile_rows": T, "ctas_per_sm": C}. */
int   tdb_tune_load(const char* key, int64_t* tile, int32_t* ctas);
void  tdb_tune_store(const char* key, int64_t tile, int32_t ctas);
/* Milliseconds the GPU spends on run(arg), queued on c's stream (CUDA events
 * on both sides); *st receives run's status.  Negative when not measured. */
float tdb_time_call(tdb_ctx* c, int (*run)(void*), void* arg, int* st);

/* ---- shared join builds (host/exec.c) ----------------------------------------------
 * While a thread's flag is set, fused join -> group-by queries over resident
 * build tables reuse one payload map per build side (td_server's workers set
 * it).  tdb_build_cache_clear frees every kept map. */
void  tdb_share_builds(int on);
/* Nonzero shape signature of a group graph td_execute_batch takes (aggregate
 * list, key and value column names and types), 0 otherwise; host-only. */
uint64_t tdb_batch_signature(td_graph_t* g, td_op_t* root);
/* td_execute_batch for a batch that will not repeat (no cached plan or CUDA
 * graph, no tuning run): td_server's packed requests. */
td_t* tdb_execute_batch_once(td_graph_t** graphs, td_op_t** roots, int64_t n);
void  tdb_build_cache_clear(void);

#endif
