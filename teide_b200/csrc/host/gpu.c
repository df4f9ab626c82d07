/*
 * Device residency for td_t columns: the device arena, host<->device copies,
 * resident (pinned) tables with per-column statistics, and the per-call
 * execution context.
 *
 * Teide keeps columns in its host buddy heap only (src/mem/heap.c).  Here a
 * column can additionally have a device mirror:
 *   - resident mirrors (td_gpu_pin) live until unpinned, or until the host
 *     block is freed or mutated through the td_* API (td_cow / td_vec_set /
 *     td_vec_append / td_vec_set_null all call tdb_mirror_forget);
 *   - transient mirrors are uploaded by one td_execute call and released when
 *     it returns.
 * Resident integer columns carry min/max statistics computed once at upload;
 * the group-by and join planners use them to choose direct arrays/maps.
 *
 * Device memory comes from a caching arena over cudaMalloc (freed blocks are
 * kept for reuse; td_gpu_trim returns them).  td_gpu_set_mem_limit caps the
 * bytes held, which is how out-of-memory handling is tested without
 * exhausting a real GPU.
 */

#include "internal.h"
#include <stdio.h>
#include <time.h>
#include <cuda_runtime_api.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

_Atomic(int) tdb_cancel_flag;

static pthread_mutex_t mu = PTHREAD_MUTEX_INITIALIZER;
static int gpu_probe = -1;        /* -1 unknown, else device count */
static int gpu_ready;

/* ---- device arena -------------------------------------------------------------- */
typedef struct { void* p; size_t sz; } dblk;
static dblk* freel; static int n_free, cap_free;
static dblk* live;  static int n_live, cap_live;
static size_t live_bytes, peak_bytes, cached_bytes, mem_limit;

static size_t round_sz(size_t n) {
    if (n < 512) return 512;
    if (n < ((size_t)2 << 20)) { size_t p = 512; while (p < n) p <<= 1; return p; }
    return (n + ((size_t)2 << 20) - 1) & ~(((size_t)2 << 20) - 1);
}

static int push(dblk** a, int* n, int* cap, void* p, size_t sz) {
    if (*n == *cap) {
        int nc = *cap ? *cap * 2 : 64;
        dblk* na = realloc(*a, (size_t)nc * sizeof(dblk));
        if (!na) return 0;
        *a = na; *cap = nc;
    }
    (*a)[(*n)++] = (dblk){p, sz};
    return 1;
}

static void release_cached_locked(void) {
    for (int i = 0; i < n_free; i++) cudaFree(freel[i].p);
    n_free = 0;
    cached_bytes = 0;
}

static void* arena_alloc(size_t bytes) {
    size_t sz = round_sz(bytes ? bytes : 1);
    pthread_mutex_lock(&mu);
    if (mem_limit && live_bytes + sz > mem_limit) { pthread_mutex_unlock(&mu); return NULL; }
    /* best fit among cached blocks up to twice the request: a new cudaMalloc
     * can synchronize the device and stall every other query's stream, which
     * costs far more than the unused tail of a larger block */
    int best = -1;
    for (int i = 0; i < n_free; i++)
        if (freel[i].sz >= sz && freel[i].sz <= 2 * sz + ((size_t)2 << 20) &&
            (best < 0 || freel[i].sz < freel[best].sz)) best = i;
    void* p = NULL;
    if (best >= 0) {
        p = freel[best].p;
        sz = freel[best].sz;
        cached_bytes -= sz;
        freel[best] = freel[--n_free];
    } else if (cudaMalloc(&p, sz) != cudaSuccess) {
        cudaGetLastError();
        release_cached_locked();
        if (cudaMalloc(&p, sz) != cudaSuccess) { cudaGetLastError(); p = NULL; }
    }
    if (p && !push(&live, &n_live, &cap_live, p, sz)) { cudaFree(p); p = NULL; }
    if (p) {
        live_bytes += sz;
        if (live_bytes > peak_bytes) peak_bytes = live_bytes;
    }
    pthread_mutex_unlock(&mu);
    return p;
}

static void arena_free(void* p) {
    if (!p) return;
    pthread_mutex_lock(&mu);
    for (int i = 0; i < n_live; i++) {
        if (live[i].p == p) {
            size_t sz = live[i].sz;
            live[i] = live[--n_live];
            live_bytes -= sz;
            if (push(&freel, &n_free, &cap_free, p, sz)) cached_bytes += sz;
            else cudaFree(p);
            break;
        }
    }
    pthread_mutex_unlock(&mu);
}

void td_gpu_trim(void) {
    pthread_mutex_lock(&mu);
    if (gpu_ready) release_cached_locked();
    pthread_mutex_unlock(&mu);
}

void td_gpu_set_mem_limit(size_t bytes) {
    pthread_mutex_lock(&mu);
    mem_limit = bytes;
    pthread_mutex_unlock(&mu);
}

void* tdb_dev_alloc_persistent(size_t bytes) { return arena_alloc(bytes); }
void  tdb_dev_free_persistent(void* p) { arena_free(p); }

/* ---- device presence ---------------------------------------------------------------- */
int tdb_gpu_available(void) {
    pthread_mutex_lock(&mu);
    if (gpu_probe < 0) {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); n = 0; }
        gpu_probe = n;
    }
    int n = gpu_probe;
    pthread_mutex_unlock(&mu);
    return n > 0;
}

int td_gpu_device_count(void) {
    tdb_gpu_available();
    return gpu_probe < 0 ? 0 : gpu_probe;
}

static int gpu_dev;                       /* the executor's device */
static _Thread_local int tls_dev_set;      /* this thread has made it current */

int tdb_gpu_ensure(void) {
    if (tls_dev_set) return TD_OK;
    if (!tdb_gpu_available()) return TD_ERR_IO;
    pthread_mutex_lock(&mu);
    if (!gpu_ready) {
        const char* env = getenv("TD_GPU_DEVICE");
        int dev = env ? atoi(env) : -1;
        if (dev >= 0) cudaSetDevice(dev);
        if (cudaFree(0) != cudaSuccess) { cudaGetLastError(); pthread_mutex_unlock(&mu); return TD_ERR_IO; }
        cudaGetDevice(&gpu_dev);
        gpu_ready = 1;
    }
    const int dev = gpu_dev;
    pthread_mutex_unlock(&mu);
    /* every thread that calls in (server workers included) works on the same
     * device as the first one, whatever its own current device was */
    if (cudaSetDevice(dev) != cudaSuccess) { cudaGetLastError(); return TD_ERR_IO; }
    tls_dev_set = 1;
    return TD_OK;
}

int tdb_check_cancel(void) { return atomic_load(&tdb_cancel_flag) ? TD_ERR_CANCEL : TD_OK; }

/* The cancel request as a word kernels can read: page-locked host memory
 * mapped into the device's address space, written by td_cancel and cleared
 * when a query starts, so a running persistent kernel sees it between work
 * items (Teide polls its flag per task and phase, pool.c:485-489,
 * exec.c:168-182). */
static volatile int32_t* cancel_h;
static void* cancel_d;

const volatile int32_t* tdb_cancel_word(void) {
    pthread_mutex_lock(&mu);
    if (!cancel_h && gpu_ready) {
        void* h = NULL;
        if (cudaHostAlloc(&h, 64, cudaHostAllocMapped | cudaHostAllocPortable) == cudaSuccess &&
            cudaHostGetDevicePointer(&cancel_d, h, 0) == cudaSuccess) {
            cancel_h = h;
            *cancel_h = atomic_load(&tdb_cancel_flag);
        } else {
            cudaGetLastError();
            if (h) cudaFreeHost(h);
            cancel_d = NULL;
        }
    }
    pthread_mutex_unlock(&mu);
    return cancel_h ? (const volatile int32_t*)cancel_d : NULL;
}

void tdb_cancel_reset(void) {
    atomic_store(&tdb_cancel_flag, 0);
    if (cancel_h) *cancel_h = 0;
}

/* ---- resident mirrors ------------------------------------------------------------------ */
typedef struct {
    td_t*      host;
    uint64_t   serial;
    tdb_devcol dc;
    size_t     bytes;
    uint64_t   stamp;     /* unique per mirror ever made (tdb_col_stamp) */
} mirror_t;

static uint64_t mirror_stamps;    /* under mu */

static mirror_t* mirrors; static int n_mir, cap_mir;

/* Hash index host pointer -> mirror slot (open addressing, -1 = empty).
 * Thousands of resident columns are common (one small table per batched
 * query), and every td_free asks whether its vector has a mirror, so the
 * lookup must not scan.  Inserts update the index in place; drops (rare)
 * mark it stale and the next lookup rebuilds it. */
static int* mh; static uint32_t mh_cap; static int mh_valid;

static uint32_t mh_slot(const td_t* v, uint32_t cap) {
    uint64_t x = (uint64_t)(uintptr_t)v;
    x ^= x >> 29;
    x *= 0x9E3779B97F4A7C15ull;
    return (uint32_t)(x >> 32) & (cap - 1);
}

static void mh_insert(int i) {
    uint32_t h = mh_slot(mirrors[i].host, mh_cap);
    while (mh[h] >= 0) h = (h + 1) & (mh_cap - 1);
    mh[h] = i;
}

static void mh_rebuild_locked(void) {
    uint32_t cap = 64;
    while (cap < (uint32_t)n_mir * 2 + 2) cap <<= 1;
    if (cap != mh_cap) {
        free(mh);
        mh = malloc((size_t)cap * sizeof(int));
        mh_cap = mh ? cap : 0;
    }
    mh_valid = 0;
    if (!mh) return;
    memset(mh, 0xFF, (size_t)mh_cap * sizeof(int));
    for (int i = 0; i < n_mir; i++) mh_insert(i);
    mh_valid = 1;
}

/* after mirrors[n_mir - 1] was appended */
static void mh_added_locked(void) {
    if (mh_valid && mh_cap >= (uint32_t)n_mir * 2 + 2) mh_insert(n_mir - 1);
    else mh_valid = 0;
}

/* Slot of v's mirror; any_serial also matches a mirror of an earlier block at v. */
static int lookup_locked(td_t* v, int any_serial) {
    if (!n_mir) return -1;
    const uint64_t s = any_serial ? 0 : tdb_block_serial(v);
    if (!mh_valid || mh_cap < (uint32_t)n_mir * 2 + 2) mh_rebuild_locked();
    if (!mh_valid) {
        for (int i = 0; i < n_mir; i++)
            if (mirrors[i].host == v && (any_serial || mirrors[i].serial == s)) return i;
        return -1;
    }
    for (uint32_t h = mh_slot(v, mh_cap);; h = (h + 1) & (mh_cap - 1)) {
        const int i = mh[h];
        if (i < 0) return -1;
        if (mirrors[i].host == v && (any_serial || mirrors[i].serial == s)) return i;
    }
}

static int find_mirror_locked(td_t* v) { return lookup_locked(v, 0); }

static void drop_mirror_locked(int i) {
    void* p = mirrors[i].dc.dptr;
    mirrors[i] = mirrors[--n_mir];
    mh_valid = 0;
    pthread_mutex_unlock(&mu);
    arena_free(p);
    pthread_mutex_lock(&mu);
}

void tdb_mirror_forget(td_t* v) {
    if (!v || TD_IS_ERR(v) || !n_mir) return;
    pthread_mutex_lock(&mu);
    for (int i = lookup_locked(v, 1); i >= 0; i = lookup_locked(v, 1)) drop_mirror_locked(i);
    pthread_mutex_unlock(&mu);
}

int tdb_col_resident(td_t* col) {
    if (col && !TD_IS_ERR(col) && (col->attrs & TD_ATTR_SLICE)) col = col->slice_parent;
    if (!col || TD_IS_ERR(col)) return 0;
    pthread_mutex_lock(&mu);
    const int r = find_mirror_locked(col) >= 0;
    pthread_mutex_unlock(&mu);
    return r;
}

void tdb_gpu_on_free(td_t* v, tdb_block_prefix* p) {
    (void)p;
    tdb_mirror_forget(v);
}

/* A large host block leaves the heap's cache for good: drop its page lock. */
void tdb_gpu_unpin_raw(void* raw) {
    cudaHostUnregister(raw);
    cudaGetLastError();
}

static size_t col_bytes(td_t* col) {
    return (size_t)col->len * td_sym_elem_size(col->type, col->attrs);
}

/* Page-lock a large host block once (the whole block: the heap reuses it for
 * any vector of the same size class), so copies to and from it run as DMA at
 * link speed instead of through a staging buffer. */
void tdb_pin_host(td_t* col) {
    if (!tdb_is_heap_block(col) || getenv("TD_GPU_NO_HOST_PIN")) return;
    tdb_block_prefix* p = tdb_prefix(col);
    if (p->kind != TDB_BLK_MMAP || atomic_load(&p->pinned)) return;
    if (cudaHostRegister(p->raw, p->raw_size, cudaHostRegisterPortable) == cudaSuccess)
        atomic_store(&p->pinned, p->raw_size);
    else
        cudaGetLastError();
}
#define pin_host tdb_pin_host

static int upload(tdb_ctx* c, td_t* col, tdb_devcol* out, int persistent) {
    size_t bytes = col_bytes(col);
    void* d = persistent ? arena_alloc(bytes) : tdb_dev_alloc(c, bytes);
    if (!d) return TD_ERR_OOM;
    if (bytes) {
        pin_host(col);
        if (cudaMemcpyAsync(d, td_data(col), bytes, cudaMemcpyHostToDevice, (cudaStream_t)c->stream) != cudaSuccess) {
            cudaGetLastError();
            if (persistent) arena_free(d);
            return TD_ERR_IO;
        }
        c->h2d_bytes += bytes;
    }
    memset(out, 0, sizeof(*out));
    out->dptr = d;
    out->len = col->len;
    out->type = col->type;
    out->attrs = col->attrs;
    return TD_OK;
}

static int is_int_type(int8_t t) {
    return t == TD_BOOL || t == TD_U8 || t == TD_CHAR || t == TD_I16 || t == TD_I32 || t == TD_I64 ||
           t == TD_DATE || t == TD_TIME || t == TD_TIMESTAMP || t == TD_SYM;
}

static int compute_stats(tdb_ctx* c, tdb_devcol* dc) {
    if (!is_int_type(dc->type)) return TD_OK;
    int64_t* d = tdb_dev_alloc(c, 16);
    if (!d) return TD_ERR_OOM;
    tdg_col col = { dc->dptr, dc->type, dc->attrs, 0, {0} };
    int st = tdg_minmax(col, dc->len, d, c->stream);
    if (st) return st;
    int64_t mm[2];
    st = tdb_d2h(c, mm, d, 16);
    if (st) return st;
    dc->kmin = mm[0];
    dc->kmax = mm[1];
    dc->has_stats = 1;
    return TD_OK;
}

/* ---- execution context ------------------------------------------------------------------- */
typedef struct { td_t* host; uint64_t serial; tdb_devcol dc; } tmirror_t;
static _Thread_local void* tls_stream;
static _Thread_local tmirror_t* tls_tm;
static _Thread_local int tls_ntm, tls_captm;

/* Trace points are buffered per thread and printed when the outermost call
 * returns ("td_execute returns"), so printing does not skew the intervals. */
static int trace_on = -1;
static _Thread_local struct timespec trace_t0;
static _Thread_local struct { const char* what; double us; } trace_buf[32];
static _Thread_local int trace_n;

void tdb_trace_begin(void) {
    if (trace_on < 0) trace_on = getenv("TD_TRACE") != NULL;
    if (trace_on) { clock_gettime(CLOCK_MONOTONIC, &trace_t0); trace_n = 0; }
}

void tdb_trace(const char* what) {
    if (trace_on <= 0) return;
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    const double us = (double)(t.tv_sec - trace_t0.tv_sec) * 1e6 + (double)(t.tv_nsec - trace_t0.tv_nsec) / 1e3;
    if (trace_n < 32) { trace_buf[trace_n].what = what; trace_buf[trace_n].us = us; trace_n++; }
    if (strcmp(what, "td_execute returns") == 0) {
        for (int i = 0; i < trace_n; i++) fprintf(stderr, "[td] %9.1f us  %s\n", trace_buf[i].us, trace_buf[i].what);
        trace_n = 0;
    }
}

static void tls_register(void);

int tdb_ctx_begin(tdb_ctx* c) {
    memset(c, 0, sizeof(*c));
    int st = tdb_gpu_ensure();
    if (st) return st;
    tls_register();
    if (!tls_stream) {
        cudaStream_t s;
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) { cudaGetLastError(); return TD_ERR_IO; }
        tls_stream = s;
    }
    c->stream = tls_stream;
    tls_ntm = 0;
    return TD_OK;
}

void* tdb_dev_alloc(tdb_ctx* c, size_t bytes) {
    void* p = arena_alloc(bytes);
    if (!p) return NULL;
    if (c->n_tmp == c->cap_tmp) {
        int nc = c->cap_tmp ? c->cap_tmp * 2 : 32;
        void** nt = realloc(c->tmp, (size_t)nc * sizeof(void*));
        if (!nt) { arena_free(p); return NULL; }
        c->tmp = nt; c->cap_tmp = nc;
    }
    c->tmp[c->n_tmp++] = p;
    return p;
}

static void finish_pending(tdb_ctx* c);

int tdb_ctx_sync(tdb_ctx* c) {
    if (cudaStreamSynchronize((cudaStream_t)c->stream) != cudaSuccess) { cudaGetLastError(); c->n_pending = 0; return TD_ERR_IO; }
    finish_pending(c);
    return TD_OK;
}

static td_gpu_stats_t last_stats;
static _Atomic(uint64_t) kernel_calls;
void tdb_note_kernel(void) { atomic_fetch_add(&kernel_calls, 1); }
void tdb_note_methods(int group, int join, int fused) {
    if (group) last_stats.last_group_method = group;
    if (join) last_stats.last_join_method = join;
    if (fused) last_stats.last_fused = fused;
}

void tdb_ctx_end(tdb_ctx* c) {
    if (c->stream) cudaStreamSynchronize((cudaStream_t)c->stream);
    finish_pending(c);
    for (int i = 0; i < c->n_tmp; i++) arena_free(c->tmp[i]);
    free(c->tmp);
    c->tmp = NULL;
    c->n_tmp = c->cap_tmp = 0;
    tls_ntm = 0;
    pthread_mutex_lock(&mu);
    last_stats.h2d_bytes = c->h2d_bytes;
    last_stats.d2h_bytes = c->d2h_bytes;
    last_stats.kernel_calls = atomic_exchange(&kernel_calls, 0);
    last_stats.dev_bytes_live = live_bytes;
    last_stats.dev_bytes_peak = peak_bytes;
    pthread_mutex_unlock(&mu);
}

void td_gpu_last_stats(td_gpu_stats_t* out) {
    if (!out) return;
    pthread_mutex_lock(&mu);
    *out = last_stats;
    pthread_mutex_unlock(&mu);
}

void tdb_reset_methods(void) {
    pthread_mutex_lock(&mu);
    last_stats.last_group_method = last_stats.last_join_method = last_stats.last_fused = 0;
    pthread_mutex_unlock(&mu);
}

/* Per-thread page-locked, device-mapped scalars (one page). */
#define TDB_SCALARS 64
static _Thread_local int64_t* tls_scalar_h;
static _Thread_local void* tls_scalar_d;

volatile int64_t* tdb_host_scalar(tdb_ctx* c, void** dev) {
    if (!tls_scalar_h) {
        void* h = NULL;
        if (cudaHostAlloc(&h, TDB_SCALARS * sizeof(int64_t), cudaHostAllocMapped) != cudaSuccess) {
            cudaGetLastError();
            return NULL;
        }
        void* d = NULL;
        if (cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) { cudaGetLastError(); cudaFreeHost(h); return NULL; }
        tls_scalar_h = h;
        tls_scalar_d = d;
    }
    if (c->n_scalar >= TDB_SCALARS) return NULL;
    const int i = c->n_scalar++;
    tls_scalar_h[i] = 0;
    *dev = (int64_t*)tls_scalar_d + i;
    return tls_scalar_h + i;
}

static _Thread_local char* tls_out_h;
static _Thread_local char* tls_out_d;

void* tdb_host_out(tdb_ctx* c, size_t bytes, void** dev) {
    if (!tls_out_h) {
        void* h = NULL;
        void* d = NULL;
        if (cudaHostAlloc(&h, TDB_OUT_BYTES, cudaHostAllocMapped) != cudaSuccess) { cudaGetLastError(); return NULL; }
        if (cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) { cudaGetLastError(); cudaFreeHost(h); return NULL; }
        tls_out_h = h;
        tls_out_d = d;
    }
    const size_t off = (c->out_used + 255) & ~(size_t)255;
    if (off + bytes > TDB_OUT_BYTES) return NULL;
    c->out_used = off + bytes;
    *dev = tls_out_d + off;
    return tls_out_h + off;
}

/* Per-thread page-locked staging for small device->host copies: a copy into
 * pageable memory is synchronous in CUDA, so queued copies land here and are
 * moved to their destinations when the call synchronizes. */
#define TDB_STAGE_BYTES ((size_t)16 << 20)
static _Thread_local char* tls_stage;

/* A thread that ran queries (a serve worker, a caller's thread) releases its
 * stream and page-locked buffers when it exits; every call on it has
 * synchronized by then. */
static pthread_key_t tls_key;
static pthread_once_t tls_once = PTHREAD_ONCE_INIT;
static int tls_key_ok;                  /* the key exists (set once, under pthread_once) */
static _Thread_local int tls_keyed;     /* this thread's release is registered */

static void tls_release(void* unused) {
    (void)unused;
    if (tls_stream) {
        cudaStreamSynchronize((cudaStream_t)tls_stream);
        cudaStreamDestroy((cudaStream_t)tls_stream);
        tls_stream = NULL;
    }
    if (tls_stage) { cudaFreeHost(tls_stage); tls_stage = NULL; }
    if (tls_out_h) { cudaFreeHost(tls_out_h); tls_out_h = tls_out_d = NULL; }
    if (tls_scalar_h) { cudaFreeHost(tls_scalar_h); tls_scalar_h = NULL; tls_scalar_d = NULL; }
    free(tls_tm);
    tls_tm = NULL;
    tls_ntm = tls_captm = 0;
    cudaGetLastError();
}

static void tls_make_key(void) {
    tls_key_ok = pthread_key_create(&tls_key, tls_release) == 0;
}

static void tls_register(void) {
    if (tls_keyed) return;
    pthread_once(&tls_once, tls_make_key);
    tls_keyed = 1;                      /* one attempt per thread */
    if (tls_key_ok) pthread_setspecific(tls_key, (void*)1);
}

int tdb_d2h_async(tdb_ctx* c, void* host, const void* dev, size_t bytes) {
    if (!bytes) return TD_OK;
    void* dst = host;
    const size_t off = (c->stage_used + 255) & ~(size_t)255;
    if (!tdb_host_is_pinned(host) && off + bytes <= TDB_STAGE_BYTES && c->n_pending < TDB_PENDING) {
        if (!tls_stage && cudaMallocHost((void**)&tls_stage, TDB_STAGE_BYTES) != cudaSuccess) {
            cudaGetLastError();
            tls_stage = NULL;
        }
        if (tls_stage) {
            dst = tls_stage + off;
            c->pending[c->n_pending].host = host;
            c->pending[c->n_pending].stage = dst;
            c->pending[c->n_pending].bytes = bytes;
            c->n_pending++;
            c->stage_used = off + bytes;
        }
    }
    if (cudaMemcpyAsync(dst, dev, bytes, cudaMemcpyDeviceToHost, (cudaStream_t)c->stream) != cudaSuccess) {
        cudaGetLastError();
        return TD_ERR_IO;
    }
    c->d2h_bytes += bytes;
    return TD_OK;
}

int tdb_host_is_pinned(const void* p) {
    struct cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) { cudaGetLastError(); return 0; }
    return a.type == cudaMemoryTypeHost;
}

static void finish_pending(tdb_ctx* c) {
    for (int i = 0; i < c->n_pending; i++) memcpy(c->pending[i].host, c->pending[i].stage, c->pending[i].bytes);
    c->n_pending = 0;
    c->stage_used = 0;
}

int tdb_d2h(tdb_ctx* c, void* host, const void* dev, size_t bytes) {
    if (!bytes) return TD_OK;
    if (cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, (cudaStream_t)c->stream) != cudaSuccess ||
        cudaStreamSynchronize((cudaStream_t)c->stream) != cudaSuccess) {
        cudaGetLastError();
        return TD_ERR_IO;
    }
    c->d2h_bytes += bytes;
    return TD_OK;
}

int tdb_h2d(tdb_ctx* c, void* dev, const void* host, size_t bytes) {
    if (!bytes) return TD_OK;
    if (cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, (cudaStream_t)c->stream) != cudaSuccess) {
        cudaGetLastError();
        return TD_ERR_IO;
    }
    c->h2d_bytes += bytes;
    return TD_OK;
}

static int is_parted(td_t* col) { return TD_IS_PARTED(col->type) || col->type == TD_MAPCOMMON; }

/* The device copy of a partitioned table's column, as one flat column of
 * its rows: a parted column's segments one after the other (uploaded, or
 * copied device to device when a segment is resident), a MAPCOMMON column's
 * partition keys each repeated over its partition's rows (tdg_expand_runs).
 * Replaces the concat fallback of exec_group_parted (exec.c:5462-5530) and
 * materialize_mapcommon (exec.c:201-243), on the device. */
static int flatten(tdb_ctx* c, td_t* col, tdb_devcol* out, int persistent) {
    memset(out, 0, sizeof(*out));
    const int64_t n = td_parted_nrows(col);
    td_t** kids = (td_t**)td_data(col);
    int st = TD_OK;
    void* d = NULL;
    if (col->type == TD_MAPCOMMON) {
        td_t* kv = kids[0];
        td_t* rc = kids[1];
        if (!kv || TD_IS_ERR(kv) || !rc || TD_IS_ERR(rc) || kv->len != rc->len || rc->type != TD_I64)
            return TD_ERR_CORRUPT;
        const int64_t np = kv->len;
        const size_t esz = td_sym_elem_size(kv->type, kv->attrs);
        const size_t bytes = n > 0 ? (size_t)n * esz : 1, vbytes = np > 0 ? (size_t)np * esz : 1;
        d = persistent ? arena_alloc(bytes) : tdb_dev_alloc(c, bytes);
        int64_t* starts = malloc((size_t)(np + 1) * 8);
        void* dv = tdb_dev_alloc(c, vbytes);
        int64_t* ds = tdb_dev_alloc(c, (size_t)(np + 1) * 8);
        if (!d || !starts || !dv || !ds) st = TD_ERR_OOM;
        if (!st) {
            starts[0] = 0;
            for (int64_t p = 0; p < np; p++) starts[p + 1] = starts[p] + ((const int64_t*)td_data(rc))[p];
            st = tdb_h2d(c, dv, td_data(kv), (size_t)np * esz);
            if (!st) st = tdb_h2d(c, ds, starts, (size_t)(np + 1) * 8);
            if (!st) st = tdb_ctx_sync(c);             /* the host arrays are copied before they are freed */
            if (!st) st = tdg_expand_runs(dv, (int32_t)esz, ds, np, d, n, c->stream);
        }
        free(starts);
        out->type = kv->type;
        out->attrs = kv->attrs;
    } else {
        td_t* first = NULL;
        for (int64_t p = 0; p < col->len && !first; p++) if (kids[p] && !TD_IS_ERR(kids[p])) first = kids[p];
        const int8_t base = (int8_t)TD_PARTED_BASETYPE(col->type);
        const uint8_t attrs = first ? first->attrs & TD_SYM_W_MASK : 0;
        const size_t esz = td_sym_elem_size(base, attrs);
        if (!esz) return TD_ERR_TYPE;
        for (int64_t p = 0; p < col->len; p++)
            if (kids[p] && !TD_IS_ERR(kids[p]) && (kids[p]->type != base ||
                                                   td_sym_elem_size(kids[p]->type, kids[p]->attrs) != esz))
                return TD_ERR_NYI;                         /* segments of different widths */
        const size_t bytes = n > 0 ? (size_t)n * esz : 1;
        d = persistent ? arena_alloc(bytes) : tdb_dev_alloc(c, bytes);
        if (!d) return TD_ERR_OOM;
        size_t off = 0;
        for (int64_t p = 0; p < col->len && !st; p++) {
            td_t* seg = kids[p];
            if (!seg || TD_IS_ERR(seg) || seg->len <= 0) continue;
            const size_t b = (size_t)seg->len * esz;
            tdb_devcol sd;
            if (tdb_col_resident(seg) && !tdb_col_device(c, seg, 0, &sd)) {
                if (cudaMemcpyAsync((char*)d + off, sd.dptr, b, cudaMemcpyDeviceToDevice, (cudaStream_t)c->stream) !=
                    cudaSuccess) { cudaGetLastError(); st = TD_ERR_IO; }
            } else {
                pin_host(seg);
                if (cudaMemcpyAsync((char*)d + off, td_data(seg), b, cudaMemcpyHostToDevice, (cudaStream_t)c->stream) !=
                    cudaSuccess) { cudaGetLastError(); st = TD_ERR_IO; }
                else c->h2d_bytes += b;
            }
            off += b;
        }
        out->type = base;
        out->attrs = attrs;
    }
    if (st) {
        if (persistent && d) arena_free(d);
        return st;
    }
    out->dptr = d;
    out->len = n;
    return TD_OK;
}

int tdb_col_device(tdb_ctx* c, td_t* col, int want_stats, tdb_devcol* out) {
    if (!col || TD_IS_ERR(col) || col->type <= 0 || col->type == TD_TABLE || col->type == TD_LIST ||
        col->type == TD_SEL)
        return TD_ERR_TYPE;
    if (col->attrs & TD_ATTR_SLICE) {
        /* a view into the parent's device copy; the parent's min/max bound
         * the slice's values, so they stay valid planning statistics */
        td_t* parent = col->slice_parent;
        if (!parent || TD_IS_ERR(parent) || (parent->attrs & TD_ATTR_SLICE)) return TD_ERR_NYI;
        if (col->slice_offset < 0 || col->slice_offset + col->len > parent->len) return TD_ERR_RANGE;
        int st = tdb_col_device(c, parent, want_stats, out);
        if (st) return st;
        out->dptr = (char*)out->dptr + (size_t)col->slice_offset * td_sym_elem_size(parent->type, parent->attrs);
        out->len = col->len;
        return TD_OK;
    }
    uint64_t serial = tdb_block_serial(col);
    const int64_t rows = td_parted_nrows(col);     /* a parted column's rows, else its length */
    pthread_mutex_lock(&mu);
    int i = find_mirror_locked(col);
    if (i >= 0 && mirrors[i].dc.len == rows) {
        *out = mirrors[i].dc;
        pthread_mutex_unlock(&mu);
        if (want_stats && !out->has_stats && is_int_type(out->type)) {
            int st = compute_stats(c, out);
            if (st) return st;
            pthread_mutex_lock(&mu);
            i = find_mirror_locked(col);
            if (i >= 0) mirrors[i].dc = *out;
            pthread_mutex_unlock(&mu);
        }
        return TD_OK;
    }
    pthread_mutex_unlock(&mu);
    for (int k = 0; k < tls_ntm; k++) {
        if (tls_tm[k].host == col && tls_tm[k].serial == serial && tls_tm[k].dc.len == rows) {
            if (want_stats && !tls_tm[k].dc.has_stats) {
                int st = compute_stats(c, &tls_tm[k].dc);
                if (st) return st;
            }
            *out = tls_tm[k].dc;
            return TD_OK;
        }
    }
    if (tls_ntm == tls_captm) {
        int nc = tls_captm ? tls_captm * 2 : 16;
        tmirror_t* nt = realloc(tls_tm, (size_t)nc * sizeof(tmirror_t));
        if (!nt) return TD_ERR_OOM;
        tls_tm = nt; tls_captm = nc;
    }
    tmirror_t* t = &tls_tm[tls_ntm];
    t->host = col;
    t->serial = serial;
    int st = is_parted(col) ? flatten(c, col, &t->dc, 0) : upload(c, col, &t->dc, 0);
    if (st) return st;
    if (want_stats) {
        st = compute_stats(c, &t->dc);
        if (st) return st;
    }
    tls_ntm++;
    *out = t->dc;
    return TD_OK;
}

uint64_t tdb_col_stamp(td_t* col) {
    if (!col || TD_IS_ERR(col) || (col->attrs & TD_ATTR_SLICE)) return 0;
    pthread_mutex_lock(&mu);
    const int i = find_mirror_locked(col);
    const uint64_t st = i >= 0 ? mirrors[i].stamp : 0;
    pthread_mutex_unlock(&mu);
    return st;
}

const void* td_gpu_col_data(td_t* col) {
    if (!col || TD_IS_ERR(col) || (col->attrs & TD_ATTR_SLICE)) return NULL;
    pthread_mutex_lock(&mu);
    const int i = find_mirror_locked(col);
    const void* p = i >= 0 ? mirrors[i].dc.dptr : NULL;
    pthread_mutex_unlock(&mu);
    return p;
}

td_err_t td_gpu_fetch(td_t* tbl) {
    if (!tbl || TD_IS_ERR(tbl)) return TD_ERR_TYPE;
    tdb_ctx c;
    int st = tdb_ctx_begin(&c);
    if (st) return (td_err_t)st;
    const int64_t nc = tbl->type == TD_TABLE ? td_table_ncols(tbl) : 1;
    for (int64_t j = 0; j < nc && !st; j++) {
        td_t* col = tbl->type == TD_TABLE ? td_table_get_col_idx(tbl, j) : tbl;
        const void* d = td_gpu_col_data(col);
        if (d) st = tdb_d2h_async(&c, td_data(col), d, col_bytes(col));
    }
    if (!st) st = tdb_ctx_sync(&c);
    tdb_ctx_end(&c);
    return (td_err_t)st;
}

/* Keep a device buffer this call produced as the resident mirror of the host
 * vector it was copied to: a later query over the result reads it from HBM.
 * The buffer leaves the call's transient list; it is freed with the host
 * vector (td_free) or by td_gpu_unpin.  Returns 1 when adopted. */
int tdb_adopt_mirror(tdb_ctx* c, td_t* host, void* dptr) {
    if (!host || TD_IS_ERR(host) || !dptr || getenv("TD_GPU_NO_RESULT_MIRROR")) return 0;
    int k = -1;
    for (int i = 0; i < c->n_tmp; i++) if (c->tmp[i] == dptr) { k = i; break; }
    if (k < 0) return 0;
    pthread_mutex_lock(&mu);
    if (n_mir == cap_mir) {
        int ncap = cap_mir ? cap_mir * 2 : 64;
        mirror_t* nm = realloc(mirrors, (size_t)ncap * sizeof(mirror_t));
        if (!nm) { pthread_mutex_unlock(&mu); return 0; }
        mirrors = nm; cap_mir = ncap;
    }
    tdb_devcol dc;
    memset(&dc, 0, sizeof(dc));
    dc.dptr = dptr; dc.len = host->len; dc.type = host->type; dc.attrs = host->attrs;
    mirrors[n_mir++] = (mirror_t){ host, tdb_block_serial(host), dc, col_bytes(host), ++mirror_stamps };
    mh_added_locked();
    pthread_mutex_unlock(&mu);
    c->tmp[k] = c->tmp[--c->n_tmp];
    return 1;
}

td_err_t td_gpu_pin(td_t* tbl) {
    if (!tbl || TD_IS_ERR(tbl)) return TD_ERR_TYPE;
    tdb_ctx c;
    int st = tdb_ctx_begin(&c);
    if (st) return (td_err_t)st;
    int64_t nc = tbl->type == TD_TABLE ? td_table_ncols(tbl) : 1;
    for (int64_t j = 0; j < nc && !st; j++) {
        td_t* col = tbl->type == TD_TABLE ? td_table_get_col_idx(tbl, j) : tbl;
        if (col && !TD_IS_ERR(col) && (col->attrs & TD_ATTR_SLICE)) col = col->slice_parent;  /* pin the data */
        if (!col || col->type <= 0 || col->type == TD_TABLE || col->type == TD_LIST) continue;
        pthread_mutex_lock(&mu);
        int have = find_mirror_locked(col) >= 0;
        pthread_mutex_unlock(&mu);
        if (have) continue;
        tdb_devcol dc;
        st = is_parted(col) ? flatten(&c, col, &dc, 1) : upload(&c, col, &dc, 1);
        if (st) break;
        st = compute_stats(&c, &dc);
        if (st) { arena_free(dc.dptr); break; }
        pthread_mutex_lock(&mu);
        if (n_mir == cap_mir) {
            int ncap = cap_mir ? cap_mir * 2 : 64;
            mirror_t* nm = realloc(mirrors, (size_t)ncap * sizeof(mirror_t));
            if (!nm) { pthread_mutex_unlock(&mu); arena_free(dc.dptr); st = TD_ERR_OOM; break; }
            mirrors = nm; cap_mir = ncap;
        }
        mirrors[n_mir++] = (mirror_t){ col, tdb_block_serial(col), dc, col_bytes(col), ++mirror_stamps };
        mh_added_locked();
        pthread_mutex_unlock(&mu);
    }
    tdb_ctx_end(&c);
    if (st) td_gpu_unpin(tbl);
    return (td_err_t)st;
}

void td_gpu_unpin(td_t* tbl) {
    if (!tbl || TD_IS_ERR(tbl)) return;
    if (tbl->type != TD_TABLE) { tdb_mirror_forget(tbl); return; }
    for (int64_t j = 0; j < td_table_ncols(tbl); j++) tdb_mirror_forget(td_table_get_col_idx(tbl, j));
}

float tdb_time_call(tdb_ctx* c, int (*run)(void*), void* arg, int* st) {
    cudaEvent_t a = NULL, b = NULL;
    cudaStream_t s = (cudaStream_t)c->stream;
    float ms = -1.f;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
        cudaGetLastError();
        if (a) cudaEventDestroy(a);
        *st = run(arg);
        return -1.f;
    }
    cudaEventRecord(a, s);
    *st = run(arg);
    cudaEventRecord(b, s);
    if (cudaEventSynchronize(b) != cudaSuccess || cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
        cudaGetLastError();
        ms = -1.f;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

/* ---- execution control ------------------------------------------------------------------- */
td_err_t td_pool_init(uint32_t n_workers) { (void)n_workers; return TD_OK; }
void td_pool_destroy(void) {}
void td_cancel(void) {
    atomic_store(&tdb_cancel_flag, 1);
    if (cancel_h) *cancel_h = 1;                 /* seen by running kernels that poll it */
}

uint32_t td_thread_count(void) { return 1; }
