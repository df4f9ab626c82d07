/*
 * td_execute_batch: many group-by graphs as one batched launch.
 *
 * Every graph must be a td_group over its bound table with one integer key
 * (td_scan) and aggregates that all read one value column (td_scan; COUNT may
 * read anything), with the same aggregate list in every graph.  The batch is
 * lowered to the tdg_batch_* kernels: one persistent kernel pulls
 * (query, tile) work items from a queue (tdg_batch.cu).
 *
 * Repeated batches are cheap: the last few batches' device work descriptions,
 * scratch and an instantiated CUDA graph of tdg_batch_run are cached, keyed
 * by the exact batch (device column addresses, row counts, key ranges,
 * aggregate list), so a repeated batch is one cudaGraphLaunch plus the
 * result copy.  Resident tables (td_gpu_pin) keep those addresses stable.
 *
 * Tile size and persistent CTAs per SM come from an autotuner: the first
 * time a batch of a given shape class runs, a few candidates are timed with
 * CUDA events and the fastest is stored in a JSON file ($TD_TUNE_CACHE, else
 * ~/.cache/teide_b200_tune.json) that later processes read.
 *
 * Result: one TD_TABLE with "_query" (I64, index of the graph), the key
 * column (named as the scanned key of the first graph) and one column per
 * aggregate (named like td_group's output), rows grouped by query in
 * argument order, keys ascending within a query.
 */
#include "internal.h"
#include <cuda_runtime_api.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <pthread.h>
#include <string.h>
#include <sys/stat.h>

#define BATCH_CACHE 4
#define BATCH_CHUNKS 8

/* One chunk of a batch: a contiguous range of its queries with its own work
 * description, scratch, outputs and captured CUDA graph. */
typedef struct {
    int32_t         q0, nq;
    tdg_batch_plan  plan;
    void*           ws;
    tdg_batch_out   out;
    void*           bufs[TDG_MAX_AGGS + 2];
    int             n_bufs;
    cudaGraphExec_t exec;
    uint64_t        launches;   /* kernels in the captured graph */
} bchunk_t;

typedef struct {
    uint64_t    sig;
    int64_t     n;
    int         used;           /* LRU stamp */
    int         n_chunks;
    bchunk_t    ch[BATCH_CHUNKS];
    int64_t*    h_rows;         /* page-locked, device-mapped: rows each chunk emitted */
    void*       d_rows;
    cudaEvent_t done[BATCH_CHUNKS];
    int64_t     total_slots;
} bcache_t;

static bcache_t bcache[BATCH_CACHE];
static int bstamp;
static pthread_mutex_t bcache_mu = PTHREAD_MUTEX_INITIALIZER;   /* cache + its graphs */

/* Signature of a batch: 8 bytes at a time (the query descriptors are 8-byte
 * multiples), a multiply-xorshift mix per word. */
static uint64_t sig64(uint64_t h, const void* p, size_t n) {
    const unsigned char* b = p;
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint64_t w;
        memcpy(&w, b + i, 8);
        h = (h ^ w) * 0x9E3779B97F4A7C15ULL;
        h ^= h >> 29;
    }
    for (; i < n; i++) h = (h ^ b[i]) * 1099511628211ULL;
    return h;
}

static void chunk_drop(bchunk_t* ch) {
    if (ch->exec) cudaGraphExecDestroy(ch->exec);
    tdb_dev_free_persistent(ch->ws);
    for (int i = 0; i < ch->n_bufs; i++) tdb_dev_free_persistent(ch->bufs[i]);
    memset(ch, 0, sizeof(*ch));
}

static void bcache_drop(bcache_t* e) {
    for (int i = 0; i < e->n_chunks; i++) {
        chunk_drop(&e->ch[i]);
        if (e->done[i]) cudaEventDestroy(e->done[i]);
    }
    if (e->h_rows) cudaFreeHost(e->h_rows);
    memset(e, 0, sizeof(*e));
}

/* ---- autotuner persistence ------------------------------------------------------ */
static void tune_path(char* buf, size_t n) {
    const char* env = getenv("TD_TUNE_CACHE");
    if (env && *env) { snprintf(buf, n, "%s", env); return; }
    const char* home = getenv("HOME");
    snprintf(buf, n, "%s/.cache/teide_b200_tune.json", home ? home : "/tmp");
}

/* Shape class of a batch: log2 buckets of query count, mean rows, mean slots. */
static void tune_key(const tdg_batch_desc* d, char* key, size_t n) {
    double rows = 0, slots = 0;
    for (int i = 0; i < d->n_queries; i++) { rows += (double)d->queries[i].nrows; slots += (double)d->queries[i].n_slots; }
    int q = d->n_queries > 0 ? (int)log2((double)d->n_queries) : 0;
    int r = d->n_queries > 0 && rows > 0 ? (int)log2(rows / d->n_queries) : 0;
    int s = d->n_queries > 0 && slots > 0 ? (int)log2(slots / d->n_queries) : 0;
    snprintf(key, n, "batch:q%d:r%d:s%d:a%d", q, r, s, d->n_aggs);
}

int tdb_tune_load(const char* key, int64_t* tile, int32_t* ctas) {
    char path[1024];
    tune_path(path, sizeof(path));
    FILE* f = fopen(path, "r");
    if (!f) return 0;
    char line[512];
    int found = 0;
    while (fgets(line, sizeof(line), f)) {
        char k[256];
        long long t;
        int c;
        if (sscanf(line, " \"%255[^\"]\": {\"tile_rows\": %lld, \"ctas_per_sm\": %d", k, &t, &c) == 3 &&
            strcmp(k, key) == 0) {
            *tile = t;
            *ctas = c;
            found = 1;
        }
    }
    fclose(f);
    return found;
}

void tdb_tune_store(const char* key, int64_t tile, int32_t ctas) {
    char path[1024], tmp[1100];
    tune_path(path, sizeof(path));
    /* keep other entries: one JSON object, one entry per line */
    char* lines[256];
    int n = 0;
    FILE* f = fopen(path, "r");
    if (f) {
        char line[512];
        while (n < 255 && fgets(line, sizeof(line), f)) {
            char k[256];
            if (sscanf(line, " \"%255[^\"]\":", k) == 1 && strcmp(k, key) != 0) {
                size_t l = strlen(line);
                while (l && (line[l - 1] == '\n' || line[l - 1] == ',')) line[--l] = 0;
                lines[n++] = strdup(line);
            }
        }
        fclose(f);
    }
    char mine[512];
    snprintf(mine, sizeof(mine), "  \"%s\": {\"tile_rows\": %lld, \"ctas_per_sm\": %d}", key, (long long)tile, ctas);
    lines[n++] = strdup(mine);
    char dir[1024];
    snprintf(dir, sizeof(dir), "%s", path);
    char* slash = strrchr(dir, '/');
    if (slash) { *slash = 0; mkdir(dir, 0755); }
    snprintf(tmp, sizeof(tmp), "%s.tmp", path);
    f = fopen(tmp, "w");
    if (f) {
        fprintf(f, "{\n");
        for (int i = 0; i < n; i++) fprintf(f, "%s%s\n", lines[i], i + 1 < n ? "," : "");
        fprintf(f, "}\n");
        fclose(f);
        rename(tmp, path);
    }
    for (int i = 0; i < n; i++) free(lines[i]);
}

/* ---- lowering ---------------------------------------------------------------------- */
typedef struct {
    tdg_batch_query q;
    int64_t key_name, val_name;
    int8_t key_type, val_type;
    uint8_t key_attrs, val_attrs;
} bq_host_t;

static int lower_one(tdb_ctx* c, td_graph_t* g, td_op_t* root, uint16_t* ops, int* n_ops, bq_host_t* out) {
    if (!root || root->opcode != OP_GROUP || !g->table) return TD_ERR_NYI;
    td_op_ext_t* ext = tdb_find_ext(g, root->id);
    if (!ext || ext->n_keys != 1 || ext->n_aggs < 1) return TD_ERR_NYI;
    td_op_ext_t* kx = tdb_find_ext(g, ext->keys[0]->id);
    if (!kx || kx->base.opcode != OP_SCAN) return TD_ERR_NYI;
    td_t* kcol = td_table_get_col(g->table, kx->sym);
    if (!kcol) return TD_ERR_SCHEMA;
    td_t* vcol = NULL;
    int64_t vname = -1;
    for (int a = 0; a < ext->n_aggs; a++) {
        td_op_ext_t* ax = tdb_find_ext(g, ext->agg_ins[a]->id);
        if (ext->agg_ops[a] == OP_COUNT && (!ax || ax->base.opcode != OP_SCAN)) continue;
        if (!ax || ax->base.opcode != OP_SCAN) return TD_ERR_NYI;
        td_t* v = td_table_get_col(g->table, ax->sym);
        if (!v) return TD_ERR_SCHEMA;
        if (vcol && v != vcol) return TD_ERR_NYI;
        vcol = v;
        vname = ax->sym;
    }
    if (!vcol) vcol = kcol, vname = kx->sym;
    if (*n_ops == 0) {
        *n_ops = ext->n_aggs;
        for (int a = 0; a < ext->n_aggs; a++) ops[a] = ext->agg_ops[a];
    } else {
        if (*n_ops != ext->n_aggs) return TD_ERR_NYI;
        for (int a = 0; a < ext->n_aggs; a++) if (ops[a] != ext->agg_ops[a]) return TD_ERR_NYI;
    }
    tdb_devcol dk, dv;
    int st = tdb_col_device(c, kcol, 1, &dk);
    if (!st) st = tdb_col_device(c, vcol, 0, &dv);
    if (st) return st;
    if (!dk.has_stats) return TD_ERR_TYPE;
    memset(out, 0, sizeof(*out));
    out->q.key = (tdg_col){ dk.dptr, dk.type, dk.attrs, 0, {0} };
    out->q.val = (tdg_col){ dv.dptr, dv.type, dv.attrs, 0, {0} };
    out->q.nrows = kcol->len;
    if (kcol->len == 0 || dk.kmax < dk.kmin) { out->q.key_min = 0; out->q.n_slots = 1; }
    else { out->q.key_min = dk.kmin; out->q.n_slots = dk.kmax - dk.kmin + 1; }
    out->key_name = kx->sym;
    out->val_name = vname;
    out->key_type = kcol->type;
    out->key_attrs = kcol->attrs & TD_SYM_W_MASK;
    out->val_type = vcol->type;
    out->val_attrs = vcol->attrs & TD_SYM_W_MASK;
    return TD_OK;
}

/* The shape of a group graph that td_execute_batch takes, as a nonzero
 * signature (0 when it takes no such graph): its aggregate list and its key
 * and value columns' names and types -- the output schema of the batch, so
 * graphs with equal signatures give the same columns batched or alone.
 * Host-only, no device work: the server calls it when a request arrives. */
uint64_t tdb_batch_signature(td_graph_t* g, td_op_t* root) {
    if (!g || !root || root->opcode != OP_GROUP || !g->table) return 0;
    td_op_ext_t* ext = tdb_find_ext(g, root->id);
    if (!ext || ext->n_keys != 1 || ext->n_aggs < 1 || ext->n_aggs > TDG_MAX_AGGS) return 0;
    td_op_ext_t* kx = tdb_find_ext(g, ext->keys[0]->id);
    if (!kx || kx->base.opcode != OP_SCAN) return 0;
    td_t* kcol = td_table_get_col(g->table, kx->sym);
    if (!kcol || TD_IS_ERR(kcol) || kcol->type <= 0 || kcol->type == TD_F64 || kcol->type >= TD_TABLE) return 0;
    td_t* vcol = NULL;
    int64_t vname = -1;
    for (int a = 0; a < ext->n_aggs; a++) {
        const uint16_t op = ext->agg_ops[a];
        if (op != OP_SUM && op != OP_COUNT && op != OP_MIN && op != OP_MAX && op != OP_AVG) return 0;
        td_op_ext_t* ax = tdb_find_ext(g, ext->agg_ins[a]->id);
        if (op == OP_COUNT && (!ax || ax->base.opcode != OP_SCAN)) continue;
        if (!ax || ax->base.opcode != OP_SCAN) return 0;
        td_t* v = td_table_get_col(g->table, ax->sym);
        if (!v || TD_IS_ERR(v) || (vcol && v != vcol)) return 0;
        vcol = v;
        vname = ax->sym;
    }
    if (!vcol) vcol = kcol, vname = kx->sym;
    if (vcol->type <= 0 || vcol->type >= TD_TABLE) return 0;
    const int64_t f[6] = { kx->sym, vname, kcol->type | (int64_t)(kcol->attrs & TD_SYM_W_MASK) << 8,
                           vcol->type | (int64_t)(vcol->attrs & TD_SYM_W_MASK) << 8, ext->n_aggs, 0 };
    uint64_t h = sig64(1469598103934665603ULL, f, sizeof(f));
    h = sig64(h, ext->agg_ops, sizeof(uint16_t) * (size_t)ext->n_aggs);
    return h ? h : 1;
}

static int alloc_outputs(bchunk_t* ch, int64_t* d_rows) {
    size_t rows = (size_t)(ch->plan.total_slots > 0 ? ch->plan.total_slots : 1);
    ch->n_bufs = 0;
    void** b = ch->bufs;
    if (!(b[ch->n_bufs++] = tdb_dev_alloc_persistent(rows * 8))) return TD_ERR_OOM;
    if (!(b[ch->n_bufs++] = tdb_dev_alloc_persistent(rows * 8))) return TD_ERR_OOM;
    ch->out.query = b[0];
    ch->out.key = b[1];
    ch->out.d_n_rows = d_rows;
    for (int a = 0; a < ch->plan.n_aggs; a++) {
        if (!(b[ch->n_bufs++] = tdb_dev_alloc_persistent(rows * 8))) return TD_ERR_OOM;
        ch->out.aggs[a] = b[ch->n_bufs - 1];
    }
    return TD_OK;
}

/* Time one configuration of the batch kernel (ms), or a negative value. */
static float time_config(tdb_ctx* c, const tdg_batch_desc* d, int64_t tile, int32_t ctas, bchunk_t* scratch) {
    tdg_batch_plan p;
    if (tdg_batch_plan_make(d, tile, ctas, &p)) return -1;
    void* ws = tdb_dev_alloc(c, p.ws_bytes);
    if (!ws) return -1;
    if (tdg_batch_prepare(d, &p, ws, c->stream)) return -1;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = -1;
    for (int rep = 0; rep < 3; rep++) {
        cudaEventRecord(a, (cudaStream_t)c->stream);
        int st = tdg_batch_run(&p, ws, &scratch->out, c->stream);
        cudaEventRecord(b, (cudaStream_t)c->stream);
        if (st || cudaEventSynchronize(b) != cudaSuccess) { best = -1; break; }
        float ms;
        cudaEventElapsedTime(&ms, a, b);
        if (rep > 0 && (best < 0 || ms < best)) best = ms;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return best;
}

/* Shape classes already looked up in the tuner's file by this process
 * (found or not), so a stream of one-off batches reads the file once per
 * class; callers hold bcache_mu. */
#define TUNE_MEMO 64
static struct { char key[64]; int64_t tile; int32_t ctas; int found; } tmemo[TUNE_MEMO];
static int n_tmemo;

static void autotune(tdb_ctx* c, const tdg_batch_desc* d, int64_t* tile, int32_t* ctas, int once) {
    char key[128];
    tune_key(d, key, sizeof(key));
    if (once) {
        for (int i = 0; i < n_tmemo; i++)
            if (!strcmp(tmemo[i].key, key)) {
                *tile = tmemo[i].found ? tmemo[i].tile : 0;
                *ctas = tmemo[i].found ? tmemo[i].ctas : 0;
                return;
            }
        const int found = tdb_tune_load(key, tile, ctas);
        if (!found) { *tile = 0; *ctas = 0; }
        if (n_tmemo < TUNE_MEMO && strlen(key) < sizeof(tmemo[0].key)) {
            snprintf(tmemo[n_tmemo].key, sizeof(tmemo[0].key), "%s", key);
            tmemo[n_tmemo].tile = *tile;
            tmemo[n_tmemo].ctas = *ctas;
            tmemo[n_tmemo].found = found;
            n_tmemo++;
        }
        return;                                    /* a one-off batch never times configurations */
    }
    if (tdb_tune_load(key, tile, ctas)) return;
    *tile = 0;
    *ctas = 0;
    if (getenv("TD_NO_AUTOTUNE")) return;
    bchunk_t scratch;
    memset(&scratch, 0, sizeof(scratch));
    int64_t* d_rows = tdb_dev_alloc(c, 8);
    if (!d_rows || tdg_batch_plan_make(d, 4096, 0, &scratch.plan) || alloc_outputs(&scratch, d_rows)) {
        chunk_drop(&scratch);
        return;
    }
    static const int64_t tiles[] = {4096, 16384, 65536};
    static const int32_t ctass[] = {0, 1, 2, 4};   /* 1 and 2: large shared-memory modes */
    float best = -1;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 4; j++) {
            float ms = time_config(c, d, tiles[i], ctass[j], &scratch);
            if (ms > 0 && (best < 0 || ms < best)) { best = ms; *tile = tiles[i]; *ctas = ctass[j]; }
        }
    chunk_drop(&scratch);
    if (best > 0) tdb_tune_store(key, *tile, *ctas);
}

static int64_t agg_out_name(uint16_t op, int64_t base) {
    const char* sfx = op == OP_SUM ? "_sum" : op == OP_COUNT ? "_count" : op == OP_AVG ? "_mean"
                    : op == OP_MIN ? "_min" : "_max";
    td_t* s = td_sym_str(base);
    char buf[300];
    int n = s ? (int)td_str_len(s) : 0;
    if (n > 250) n = 250;
    if (s) memcpy(buf, td_str_ptr(s), (size_t)n);
    memcpy(buf + n, sfx, strlen(sfx));
    return td_sym_intern(buf, (size_t)n + strlen(sfx));
}

/* once: a batch that will not repeat (td_server packing the requests that
 * wait in its queue): one chunk, run directly rather than captured into a CUDA
 * graph, outputs from the arena and the row count in a mapped scalar of the
 * call, nothing kept in the cache, and the defaults when its shape was never
 * tuned. */
static td_t* exec_batch(td_graph_t** graphs, td_op_t** roots, int64_t n, int once);

td_t* td_execute_batch(td_graph_t** graphs, td_op_t** roots, int64_t n) {
    return exec_batch(graphs, roots, n, 0);
}

td_t* tdb_execute_batch_once(td_graph_t** graphs, td_op_t** roots, int64_t n) {
    return exec_batch(graphs, roots, n, 1);
}

static td_t* exec_batch(td_graph_t** graphs, td_op_t** roots, int64_t n, int once) {
    if (!graphs || !roots || n < 0 || n > INT32_MAX) return TD_ERR_PTR(TD_ERR_RANGE);
    tdb_cancel_reset();
    tdb_trace_begin();
    tdb_ctx c;
    int st = tdb_ctx_begin(&c);
    if (st) return TD_ERR_PTR(st);
    pthread_mutex_lock(&bcache_mu);
    td_t* res = NULL;
    bchunk_t* once_ch = NULL;         /* the one-off chunk's arena buffers, freed at the end */
    bq_host_t* hq = calloc((size_t)(n ? n : 1), sizeof(bq_host_t));
    tdg_batch_query* qs = calloc((size_t)(n ? n : 1), sizeof(tdg_batch_query));
    uint16_t ops[TDG_MAX_AGGS];
    int n_ops = 0;
    if (!hq || !qs) { st = TD_ERR_OOM; goto done; }
    for (int64_t i = 0; i < n && !st; i++) {
        st = lower_one(&c, graphs[i], roots[i], ops, &n_ops, &hq[i]);
        qs[i] = hq[i].q;
        /* one output schema: every query's key and value columns share types */
        if (!st && i > 0 && (hq[i].key_type != hq[0].key_type || hq[i].key_attrs != hq[0].key_attrs ||
                             hq[i].val_type != hq[0].val_type || hq[i].val_attrs != hq[0].val_attrs))
            st = TD_ERR_TYPE;
    }
    if (st) goto done;
    if (n_ops > TDG_MAX_AGGS) { st = TD_ERR_NYI; goto done; }
    tdg_batch_desc d;
    memset(&d, 0, sizeof(d));
    d.n_queries = (int32_t)n;
    d.n_aggs = n_ops;
    for (int a = 0; a < n_ops; a++) d.agg_ops[a] = ops[a];
    d.queries = qs;

    /* Chunks: contiguous query ranges of about equal rows.  Each chunk's
     * results are copied to the host on a second stream while the next chunks
     * compute.  Timing (tdg_set_timing) runs one chunk so its kernel time
     * covers the whole batch. */
    const int timing = tdg_timing_enabled();
    int K = timing || once ? 1 : (int)(n / 64 < BATCH_CHUNKS ? n / 64 : BATCH_CHUNKS);
    if (K < 1) K = 1;
    bcache_t once_e;
    static _Thread_local cudaEvent_t once_done;
    uint64_t sig = sig64(1469598103934665603ULL, qs, sizeof(tdg_batch_query) * (size_t)n);
    sig = sig64(sig, &d.agg_ops, sizeof(d.agg_ops));
    sig = sig64(sig, &K, sizeof(K));
    bcache_t* e = NULL;
    for (int i = 0; i < BATCH_CACHE && !once; i++)
        if (bcache[i].n_chunks && bcache[i].sig == sig && bcache[i].n == n) e = &bcache[i];
    if (once) {
        memset(&once_e, 0, sizeof(once_e));
        e = &once_e;
        int64_t tile;
        int32_t ctas;
        autotune(&c, &d, &tile, &ctas, 1);
        void* d_rows = NULL;
        e->h_rows = (int64_t*)tdb_host_scalar(&c, &d_rows);
        e->d_rows = d_rows;
        if (!once_done && cudaEventCreateWithFlags(&once_done, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            once_done = NULL;
        }
        e->done[0] = once_done;
        bchunk_t* ch = &e->ch[0];
        once_ch = ch;
        e->n_chunks = 1;
        ch->nq = (int32_t)n;
        if (!e->h_rows || !once_done) st = TD_ERR_OOM;
        if (!st) st = tdg_batch_plan_make(&d, tile, ctas, &ch->plan);
        if (!st) {
            ch->plan.cancel = tdb_cancel_word();
            ch->ws = tdb_dev_alloc_persistent(ch->plan.ws_bytes);
            if (!ch->ws || alloc_outputs(ch, (int64_t*)e->d_rows)) st = TD_ERR_OOM;
        }
        if (!st) st = tdg_batch_prepare(&d, &ch->plan, ch->ws, c.stream);
        e->total_slots = ch->plan.total_slots;
        if (st) goto done;
    } else if (!e) {
        /* chunk boundaries: contiguous query ranges of about equal rows */
        int32_t q0s[BATCH_CHUNKS + 1];
        double total = 0, acc = 0;
        for (int64_t i = 0; i < n; i++) total += (double)qs[i].nrows + 1;
        int32_t q = 0;
        for (int k = 0; k < K; k++) {
            q0s[k] = q;
            const double goal = total * (k + 1) / K;
            while (q < n && (k == K - 1 || acc < goal)) { acc += (double)qs[q].nrows + 1; q++; }
        }
        q0s[K] = (int32_t)n;
        /* tile and CTAs tuned on a chunk: that is the launch that runs */
        tdg_batch_desc d0 = d;
        d0.n_queries = q0s[1] - q0s[0];
        d0.queries = qs;
        int64_t tile;
        int32_t ctas;
        autotune(&c, &d0, &tile, &ctas, 0);
        int victim = 0;
        for (int i = 1; i < BATCH_CACHE; i++) if (bcache[i].used < bcache[victim].used) victim = i;
        e = &bcache[victim];
        bcache_drop(e);
        e->sig = sig;
        e->n = n;
        void* h = NULL;
        if (cudaHostAlloc(&h, BATCH_CHUNKS * sizeof(int64_t), cudaHostAllocMapped) != cudaSuccess ||
            cudaHostGetDevicePointer(&e->d_rows, h, 0) != cudaSuccess) {
            cudaGetLastError();
            if (h) cudaFreeHost(h);
            memset(e, 0, sizeof(*e));
            st = TD_ERR_OOM;
            goto done;
        }
        e->h_rows = h;
        for (int k = 0; k < K && !st; k++) {
            bchunk_t* ch = &e->ch[k];
            e->n_chunks = k + 1;
            ch->q0 = q0s[k];
            ch->nq = q0s[k + 1] - q0s[k];
            tdg_batch_desc dc = d;
            dc.n_queries = ch->nq;
            dc.queries = qs + ch->q0;
            if (cudaEventCreateWithFlags(&e->done[k], cudaEventDisableTiming) != cudaSuccess) { cudaGetLastError(); st = TD_ERR_IO; break; }
            if ((st = tdg_batch_plan_make(&dc, tile, ctas, &ch->plan))) break;
            ch->plan.query_base = ch->q0;
            ch->plan.cancel = tdb_cancel_word();
            ch->ws = tdb_dev_alloc_persistent(ch->plan.ws_bytes);
            if (!ch->ws || alloc_outputs(ch, (int64_t*)e->d_rows + k)) { st = TD_ERR_OOM; break; }
            if ((st = tdg_batch_prepare(&dc, &ch->plan, ch->ws, c.stream))) break;
            e->total_slots += ch->plan.total_slots;
            /* capture the run once; replays reuse the instantiated graph */
            cudaGraph_t graph = NULL;
            cudaStream_t s = (cudaStream_t)c.stream;
            if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                uint64_t l0 = tdg_launch_count();
                int rs = tdg_batch_run(&ch->plan, ch->ws, &ch->out, c.stream);
                ch->launches = tdg_launch_count() - l0;
                if (cudaStreamEndCapture(s, &graph) == cudaSuccess && !rs && graph) {
                    if (cudaGraphInstantiate(&ch->exec, graph, 0) != cudaSuccess) ch->exec = NULL;
                }
                if (graph) cudaGraphDestroy(graph);
            }
            cudaGetLastError();
        }
        if (st) { bcache_drop(e); goto done; }
    }
    if (!once) e->used = ++bstamp;
    tdb_trace("batch lowered");
    if ((st = tdb_check_cancel())) goto done;
    tdb_note_kernel();
    cudaStream_t s = (cudaStream_t)c.stream;
    for (int k = 0; k < e->n_chunks && !st; k++) {
        bchunk_t* ch = &e->ch[k];
        if (ch->exec && !timing) {                /* timing runs the kernels directly */
            if (cudaGraphLaunch(ch->exec, s) != cudaSuccess) { cudaGetLastError(); st = TD_ERR_IO; break; }
            tdg_count_launches(ch->launches);
        } else if ((st = tdg_batch_run(&ch->plan, ch->ws, &ch->out, c.stream))) {
            break;
        }
        if (cudaEventRecord(e->done[k], s) != cudaSuccess) { cudaGetLastError(); st = TD_ERR_IO; }
    }
    if (st) goto done;
    tdb_trace("batch launched");

    /* device columns are 8 bytes wide; keys and MIN/MAX of narrower integer
     * columns are narrowed back to the column's type, as td_group returns them */
    typedef struct { int8_t t; uint8_t attrs; int64_t name; td_t* v; } outcol_t;
    outcol_t cols[TDG_MAX_AGGS + 2];
    memset(cols, 0, sizeof(cols));
    int nc = 0;
    cols[nc++] = (outcol_t){ TD_I64, 0, td_sym_intern("_query", 6), NULL };
    cols[nc++] = (outcol_t){ n ? hq[0].key_type : TD_I64, n ? hq[0].key_attrs : 0,
                             n ? hq[0].key_name : td_sym_intern("key", 3), NULL };
    for (int a = 0; a < n_ops; a++) {
        const int val_f64 = e->ch[0].plan.val_f64;
        int8_t t = ops[a] == OP_COUNT ? TD_I64 : (ops[a] == OP_AVG || val_f64) ? TD_F64
                 : (ops[a] == OP_SUM || !n) ? TD_I64 : hq[0].val_type;
        cols[nc++] = (outcol_t){ t, (ops[a] == OP_MIN || ops[a] == OP_MAX) && n ? hq[0].val_attrs : 0,
                                 agg_out_name(ops[a], n ? hq[0].val_name : 0), NULL };
    }
    tdb_trace("batch schema");
    /* wide host columns sized for every slot; lengths are set once known */
    const int64_t cap = e->total_slots > 0 ? e->total_slots : 1;
    for (int j = 0; j < nc && !st; j++) {
        const int wide = td_sym_elem_size(cols[j].t, cols[j].attrs) == 8;
        td_t* v = td_vec_new(wide ? cols[j].t : TD_I64, cap);
        if (!v || TD_IS_ERR(v)) { st = TD_ERR_OOM; break; }
        if (wide && cols[j].t == TD_SYM) v->attrs = cols[j].attrs;
        if ((size_t)cap * 8 >= ((size_t)8 << 20)) tdb_pin_host(v);
        cols[j].v = v;
    }
    tdb_trace("batch result vectors");
    static _Thread_local cudaStream_t copy_stream;
    if (!st && !copy_stream && cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        copy_stream = NULL;
        st = TD_ERR_IO;
    }
    int64_t rows = 0;
    for (int k = 0; k < e->n_chunks && !st; k++) {
        bchunk_t* ch = &e->ch[k];
        if (cudaEventSynchronize(e->done[k]) != cudaSuccess) { cudaGetLastError(); st = TD_ERR_IO; break; }
        tdb_trace("batch chunk computed");
        if ((st = tdb_check_cancel())) break;          /* the kernel stopped taking work: partial rows */
        const int64_t rk = ((volatile int64_t*)e->h_rows)[k];
        if (rk < 0) { st = TD_ERR_DOMAIN; break; }     /* a key outside its statistics */
        void* src[TDG_MAX_AGGS + 2];
        src[0] = ch->out.query;
        src[1] = ch->out.key;
        for (int a = 0; a < n_ops; a++) src[2 + a] = ch->out.aggs[a];
        for (int j = 0; j < nc && !st; j++)
            if (rk && cudaMemcpyAsync((char*)td_data(cols[j].v) + (size_t)rows * 8, src[j], (size_t)rk * 8,
                                      cudaMemcpyDeviceToHost, copy_stream) != cudaSuccess) { cudaGetLastError(); st = TD_ERR_IO; }
        rows += rk;
    }
    if (copy_stream && cudaStreamSynchronize(copy_stream) != cudaSuccess) { cudaGetLastError(); if (!st) st = TD_ERR_IO; }
    if (!st) c.d2h_bytes += (uint64_t)rows * 8 * (uint64_t)nc;
    tdb_trace("batch results copied");
    res = st ? NULL : td_table_new(2 + n_ops);
    if (!st && (!res || TD_IS_ERR(res))) { st = TD_ERR_OOM; res = NULL; }
    for (int j = 0; j < nc && !st; j++) {
        td_t* v = cols[j].v;
        v->len = rows;
        if (td_sym_elem_size(cols[j].t, cols[j].attrs) != 8) {
            td_t* nv = td_vec_new(cols[j].t, rows);
            if (!nv || TD_IS_ERR(nv)) { st = TD_ERR_OOM; break; }
            nv->len = rows;
            if (cols[j].t == TD_SYM) nv->attrs = cols[j].attrs;
            const int64_t* w = (const int64_t*)td_data(v);
            for (int64_t i = 0; i < rows; i++) {
                if (cols[j].t == TD_SYM) td_write_sym(td_data(nv), i, (uint64_t)w[i], TD_SYM, cols[j].attrs);
                else switch (td_elem_size(cols[j].t)) {
                    case 4: ((int32_t*)td_data(nv))[i] = (int32_t)w[i]; break;
                    case 2: ((int16_t*)td_data(nv))[i] = (int16_t)w[i]; break;
                    default: ((uint8_t*)td_data(nv))[i] = (uint8_t)w[i]; break;
                }
            }
            td_release(v);
            cols[j].v = v = nv;
        }
        td_t* r2 = td_table_add_col(res, cols[j].name, v);
        if (TD_IS_ERR(r2)) st = TD_ERR_CODE(r2); else res = r2;
    }
    for (int j = 0; j < nc; j++) if (cols[j].v) td_release(cols[j].v);
    tdb_trace("batch assembled");
done:
    if (once_ch) {
        cudaStreamSynchronize((cudaStream_t)c.stream);   /* nothing of the batch still running */
        cudaGetLastError();
        chunk_drop(once_ch);
    }
    pthread_mutex_unlock(&bcache_mu);
    if (st && res) { td_release(res); res = NULL; }
    free(hq);
    free(qs);
    tdb_ctx_end(&c);
    tdb_trace("td_execute returns");
    return st ? TD_ERR_PTR(st) : res;
}

void td_gpu_batch_cache_clear(void) {
    pthread_mutex_lock(&bcache_mu);
    for (int i = 0; i < BATCH_CACHE; i++) bcache_drop(&bcache[i]);
    pthread_mutex_unlock(&bcache_mu);
}
