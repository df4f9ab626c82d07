/*
 * td_server: a request loop over device-resident tables.
 *
 * Teide runs one td_execute at a time per caller; a serving process that
 * receives queries continuously would either serialize them (each waits for
 * all earlier ones) or oversubscribe the device.  Here a fixed set of worker
 * threads -- the server's slots -- pull requests in arrival order.  Each
 * worker has its own CUDA stream (the executor keeps one per thread), so the
 * kernels, copies and host-side planning of the queries in flight overlap on
 * the GPU, and a query that arrives while others run starts as soon as a slot
 * is free and its device memory fits: requests are admitted by an estimate of
 * the device bytes they need against a budget taken from the GPU's free HBM.
 * The head of the queue is never bypassed, so admission is FIFO; a request
 * whose estimate alone exceeds the budget runs when nothing else is in
 * flight.
 *
 * Small group-by requests of one shape -- one integer key, aggregates over one
 * value column, the same aggregate list and column names -- that wait in the
 * queue behind each other run together: a worker takes the head and every
 * queued request of its shape right behind it (up to SERVE_BATCH_MAX, within
 * the budget) into one td_execute_batch launch and splits the packed result
 * into one table per request, the columns td_execute returns.  Requests of
 * different sizes share the launch; the batch kernel balances their tiles.
 * One packed batch runs at a time: the batch-shaped requests that arrive
 * meanwhile wait at the head and leave together as the next batch.
 *
 * Join queries over the same resident build table share one payload map (the
 * build side's key -> group-slot map): the first query builds it into a kept
 * workspace and every later one only probes it (host/exec.c, shared join
 * builds), so a join request costs its probe and nothing for the build.
 *
 * Results are ordinary host td_t tables returned by td_server_wait, with the
 * request's submit / start / end times (CLOCK_MONOTONIC nanoseconds) so the
 * caller can compute latency percentiles.
 */
#include "internal.h"
#include <cuda_runtime_api.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef struct {
    int64_t             ticket;
    td_graph_t*         g;
    td_op_t*            root;
    uint64_t            sig;        /* td_execute_batch shape, 0 if none */
    size_t              est;
    int                 state;      /* 0 free, 1 queued, 2 running, 3 done */
    td_t*               result;
    td_server_timing_t  t;
} req_t;

struct td_server {
    pthread_mutex_t mu;
    pthread_cond_t  cv_work, cv_done;
    req_t*          ring;
    int64_t         cap;
    int64_t         next_ticket;    /* next ticket to hand out */
    int64_t         next_admit;     /* oldest ticket not yet admitted */
    int32_t         slots;
    pthread_t*      th;
    int32_t         n_th;
    int             stop;
    size_t          budget, reserved, peak_reserved;
    int32_t         in_flight, peak_in_flight;
    int32_t         batch_running;  /* a packed batch is in flight */
    uint64_t        completed;
};

static int64_t now_ns(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (int64_t)ts.tv_sec * 1000000000LL + ts.tv_nsec;
}

/* Requests a worker takes together at most, and the split of a batch's
 * packed result (rows of query i, keys ascending, _query column first) into
 * one table per request, with the columns td_execute would return. */
#define SERVE_BATCH_MAX 1024

static td_t* rows_of(td_t* b, int64_t r0, int64_t r1) {
    const int64_t nc = td_table_ncols(b);
    td_t* t = td_table_new(nc - 1);
    if (!t || TD_IS_ERR(t)) return TD_ERR_PTR(TD_ERR_OOM);
    for (int64_t j = 1; j < nc; j++) {
        td_t* c = td_table_get_col_idx(b, j);
        const size_t es = td_sym_elem_size(c->type, c->attrs);
        td_t* v = td_vec_new(c->type, r1 - r0 > 0 ? r1 - r0 : 1);
        if (!v || TD_IS_ERR(v)) { td_release(t); return TD_ERR_PTR(TD_ERR_OOM); }
        if (c->type == TD_SYM) v->attrs = c->attrs;
        if (r1 > r0) memcpy(td_data(v), (const char*)td_data(c) + (size_t)r0 * es, (size_t)(r1 - r0) * es);
        v->len = r1 - r0;
        td_t* t2 = td_table_add_col(t, td_table_col_name(b, j), v);
        td_release(v);
        if (TD_IS_ERR(t2)) { td_release(t); return t2; }
        t = t2;
    }
    return t;
}

/* Requests [i0, i1) of a packed result, their rows [lo[i], lo[i + 1]). */
typedef struct {
    td_t*          b;
    const int64_t* lo;
    int64_t        i0, i1;
    td_t**         out;
} split_job_t;

static void* split_range(void* arg) {
    split_job_t* j = arg;
    for (int64_t i = j->i0; i < j->i1; i++) j->out[i] = rows_of(j->b, j->lo[i], j->lo[i + 1]);
    return NULL;
}

/* Host threads that split one packed result: building a request's table (the
 * copy out of the packed columns and its allocations) is the served form's
 * bound once the batch itself is on the GPU, and it parallelizes (on 1024
 * small requests 8 threads measured 3.0-3.4x one query at a time, 4 threads
 * 1.9-3.0x). */
#define SPLIT_THREADS 8
#define SPLIT_MIN_PER_THREAD 128

/* The packed result b of n requests into one table per request (b released). */
static void split_batch(td_t* b, td_graph_t** gs, td_op_t** rs, int64_t n, td_t** out) {
    if (TD_IS_ERR(b)) {
        /* a cancel ends them all; any other refusal runs them one by one */
        for (int64_t i = 0; i < n; i++) out[i] = TD_ERR_CODE(b) == TD_ERR_CANCEL ? b : td_execute(gs[i], rs[i]);
        return;
    }
    const int64_t rows = td_table_ncols(b) > 0 ? td_table_get_col_idx(b, 0)->len : 0;
    const int64_t* q = rows ? (const int64_t*)td_data(td_table_get_col_idx(b, 0)) : NULL;
    int64_t* lo = malloc(((size_t)n + 1) * sizeof(int64_t));
    if (!lo) {
        for (int64_t i = 0; i < n; i++) out[i] = TD_ERR_PTR(TD_ERR_OOM);
        td_release(b);
        return;
    }
    int64_t r = 0;
    for (int64_t i = 0; i < n; i++) {
        lo[i] = r;
        while (r < rows && q[r] == i) r++;
    }
    lo[n] = r;
    int nt = (int)(n / SPLIT_MIN_PER_THREAD);
    if (nt < 1) nt = 1;
    if (nt > SPLIT_THREADS) nt = SPLIT_THREADS;
    split_job_t jobs[SPLIT_THREADS];
    pthread_t th[SPLIT_THREADS];
    int started[SPLIT_THREADS] = {0};
    for (int t = 0; t < nt; t++) {
        jobs[t] = (split_job_t){ b, lo, n * t / nt, n * (t + 1) / nt, out };
        if (t > 0) started[t] = pthread_create(&th[t], NULL, split_range, &jobs[t]) == 0;
    }
    split_range(&jobs[0]);
    for (int t = 1; t < nt; t++) {
        if (started[t]) pthread_join(th[t], NULL);
        else split_range(&jobs[t]);             /* no thread: this one does it */
    }
    free(lo);
    td_release(b);
}

static void* worker_main(void* arg) {
    td_server_t* s = arg;
    tdb_share_builds(1);                /* join queries over one build table share its map */
    int64_t* tix = malloc(SERVE_BATCH_MAX * sizeof(int64_t));
    td_graph_t** gs = malloc(SERVE_BATCH_MAX * sizeof(td_graph_t*));
    td_op_t** rs = malloc(SERVE_BATCH_MAX * sizeof(td_op_t*));
    td_t** res = malloc(SERVE_BATCH_MAX * sizeof(td_t*));
    pthread_mutex_lock(&s->mu);
    for (;;) {
        req_t* r = NULL;
        if (s->next_admit < s->next_ticket) {
            req_t* head = &s->ring[s->next_admit % s->cap];
            const int fits = s->reserved + head->est <= s->budget || s->in_flight == 0;
            /* one packed batch at a time (it fills the GPU): requests of a
             * batch shape queue behind it and leave together as the next one */
            const int wait_batch = head->sig && s->batch_running;
            if (s->in_flight < s->slots && fits && !wait_batch) r = head;
        }
        if (!r) {
            if (s->stop && s->next_admit >= s->next_ticket) break;
            pthread_cond_wait(&s->cv_work, &s->mu);
            continue;
        }
        /* the head, and behind it every queued request of the same batch shape
         * that fits the budget: they run as one td_execute_batch launch */
        const uint64_t sig = (tix && gs && rs && res) ? r->sig : 0;
        const int64_t now = now_ns();
        int64_t nb = 0;
        size_t est = 0;
        for (;;) {
            req_t* q = &s->ring[s->next_admit % s->cap];
            if (tix) tix[nb] = q->ticket;
            if (gs) gs[nb] = q->g;
            if (rs) rs[nb] = q->root;
            nb++;
            est += q->est;
            q->state = 2;
            q->t.start_ns = now;
            q->t.in_flight_at_start = s->in_flight + 1;
            s->next_admit++;
            if (!sig || nb >= SERVE_BATCH_MAX || s->next_admit >= s->next_ticket) break;
            const req_t* nx = &s->ring[s->next_admit % s->cap];
            if (nx->sig != sig || s->reserved + est + nx->est > s->budget) break;
        }
        s->in_flight++;
        s->reserved += est;
        if (sig) s->batch_running = 1;
        if (s->in_flight > s->peak_in_flight) s->peak_in_flight = s->in_flight;
        if (s->reserved > s->peak_reserved) s->peak_reserved = s->reserved;
        const int64_t ticket0 = r->ticket;
        td_graph_t* g0 = r->g;
        td_op_t* root0 = r->root;
        pthread_mutex_unlock(&s->mu);

        td_t* one = NULL;
        if (sig && nb > 1) {
            td_t* b = tdb_execute_batch_once(gs, rs, nb);
            /* the GPU is free: the next batch may start while this one's
             * result is split into its requests' tables */
            pthread_mutex_lock(&s->mu);
            s->batch_running = 0;
            pthread_cond_broadcast(&s->cv_work);
            pthread_mutex_unlock(&s->mu);
            split_batch(b, gs, rs, nb, res);
        } else if (sig) {
            res[0] = td_execute(g0, root0);
        } else {
            one = td_execute(g0, root0);
        }

        pthread_mutex_lock(&s->mu);
        const int64_t end = now_ns();
        for (int64_t i = 0; i < nb; i++) {
            req_t* d = &s->ring[(sig ? tix[i] : ticket0) % s->cap];
            d->result = sig ? res[i] : one;
            d->t.end_ns = end;
            d->t.status = TD_IS_ERR(d->result) ? (int32_t)TD_ERR_CODE(d->result) : 0;
            d->state = 3;
        }
        s->in_flight--;
        s->reserved -= est;
        if (sig && nb == 1) s->batch_running = 0;   /* a packed batch cleared it when its launch ended */
        s->completed += (uint64_t)nb;
        pthread_cond_broadcast(&s->cv_done);
        pthread_cond_broadcast(&s->cv_work);
    }
    pthread_mutex_unlock(&s->mu);
    free(tix);
    free(gs);
    free(rs);
    free(res);
    return NULL;
}

td_server_t* td_server_new(int32_t slots, size_t hbm_budget, int64_t queue_cap) {
    if (slots < 1 || slots > 256) return NULL;
    td_server_t* s = calloc(1, sizeof(*s));
    if (!s) return NULL;
    s->cap = queue_cap > 0 ? queue_cap : 65536;
    s->ring = calloc((size_t)s->cap, sizeof(req_t));
    s->th = calloc((size_t)slots, sizeof(pthread_t));
    if (!s->ring || !s->th) { free(s->ring); free(s->th); free(s); return NULL; }
    s->slots = slots;
    s->budget = hbm_budget;
    if (!s->budget) {
        /* 90% of the HBM free now: resident tables are already counted out */
        size_t fr = 0, tot = 0;
        if (tdb_gpu_ensure() == TD_OK && cudaMemGetInfo(&fr, &tot) == cudaSuccess) s->budget = fr / 10 * 9;
        else { cudaGetLastError(); s->budget = (size_t)-1; }
    }
    pthread_mutex_init(&s->mu, NULL);
    pthread_cond_init(&s->cv_work, NULL);
    pthread_cond_init(&s->cv_done, NULL);
    for (int32_t i = 0; i < slots; i++) {
        if (pthread_create(&s->th[i], NULL, worker_main, s) != 0) break;
        s->n_th++;
    }
    if (s->n_th != slots) { td_server_free(s); return NULL; }
    return s;
}

int64_t td_server_submit(td_server_t* s, td_graph_t* g, td_op_t* root, size_t est_bytes) {
    if (!s || !g || !root) return -(int64_t)TD_ERR_TYPE;
    if (!est_bytes) est_bytes = td_server_estimate(g, root);
    pthread_mutex_lock(&s->mu);
    if (s->stop) { pthread_mutex_unlock(&s->mu); return -(int64_t)TD_ERR_IO; }
    const int64_t t = s->next_ticket;
    req_t* r = &s->ring[t % s->cap];
    if (r->state != 0) { pthread_mutex_unlock(&s->mu); return -(int64_t)TD_ERR_RANGE; }  /* queue full */
    memset(r, 0, sizeof(*r));
    r->ticket = t;
    r->g = g;
    r->root = root;
    r->sig = tdb_batch_signature(g, root);
    r->est = est_bytes;
    r->state = 1;
    r->t.submit_ns = now_ns();
    r->t.est_bytes = (int64_t)est_bytes;
    s->next_ticket++;
    pthread_cond_signal(&s->cv_work);
    pthread_mutex_unlock(&s->mu);
    return t;
}

td_t* td_server_wait(td_server_t* s, int64_t ticket, td_server_timing_t* timing) {
    if (!s || ticket < 0) return TD_ERR_PTR(TD_ERR_RANGE);
    pthread_mutex_lock(&s->mu);
    req_t* r = &s->ring[ticket % s->cap];
    if (r->ticket != ticket || r->state == 0) { pthread_mutex_unlock(&s->mu); return TD_ERR_PTR(TD_ERR_RANGE); }
    while (r->state != 3) pthread_cond_wait(&s->cv_done, &s->mu);
    td_t* res = r->result;
    if (timing) *timing = r->t;
    r->state = 0;
    r->result = NULL;
    pthread_mutex_unlock(&s->mu);
    return res;
}

int64_t td_server_submit_many(td_server_t* s, td_graph_t** graphs, td_op_t** roots, int64_t n, int64_t* tickets) {
    if (!s || !graphs || !roots || !tickets || n < 0) return 0;
    int64_t i = 0;
    for (; i < n; i++) {
        tickets[i] = td_server_submit(s, graphs[i], roots[i], 0);
        if (tickets[i] < 0) break;
    }
    return i;
}

void td_server_wait_many(td_server_t* s, const int64_t* tickets, int64_t n, td_t** results,
                         td_server_timing_t* timings) {
    if (!s || !tickets) return;
    for (int64_t i = 0; i < n; i++) {
        td_t* r = td_server_wait(s, tickets[i], timings ? &timings[i] : NULL);
        if (results) results[i] = r;
        else if (r && !TD_IS_ERR(r)) td_release(r);
    }
}

void td_server_stats(td_server_t* s, td_server_stats_t* out) {
    if (!s || !out) return;
    pthread_mutex_lock(&s->mu);
    out->completed = s->completed;
    out->queued = s->next_ticket - s->next_admit;
    out->in_flight = s->in_flight;
    out->peak_in_flight = s->peak_in_flight;
    out->slots = s->slots;
    out->pad = 0;
    out->budget_bytes = s->budget;
    out->reserved_bytes = s->reserved;
    out->peak_reserved_bytes = s->peak_reserved;
    pthread_mutex_unlock(&s->mu);
}

void td_server_free(td_server_t* s) {
    if (!s) return;
    pthread_mutex_lock(&s->mu);
    s->stop = 1;                        /* workers drain the queue, then exit */
    pthread_cond_broadcast(&s->cv_work);
    pthread_mutex_unlock(&s->mu);
    for (int32_t i = 0; i < s->n_th; i++) pthread_join(s->th[i], NULL);
    tdb_build_cache_clear();
    for (int64_t i = 0; i < s->cap; i++)
        if (s->ring[i].state == 3 && s->ring[i].result && !TD_IS_ERR(s->ring[i].result)) td_release(s->ring[i].result);
    pthread_cond_destroy(&s->cv_work);
    pthread_cond_destroy(&s->cv_done);
    pthread_mutex_destroy(&s->mu);
    free(s->ring);
    free(s->th);
    free(s);
}

/* ---- admission estimate ----------------------------------------------------------- */

static void est_table(td_t* t, td_t** seen, int* n_seen, size_t* upload, int64_t* rows_max, int64_t* rows_sum) {
    if (!t || TD_IS_ERR(t) || t->type != TD_TABLE) return;
    for (int i = 0; i < *n_seen; i++) if (seen[i] == t) return;
    if (*n_seen < 64) seen[(*n_seen)++] = t;
    const int64_t rows = td_table_nrows(t);
    if (rows > *rows_max) *rows_max = rows;
    *rows_sum += rows;
    for (int64_t j = 0; j < td_table_ncols(t); j++) {
        td_t* c = td_table_get_col_idx(t, j);
        if (!c || TD_IS_ERR(c) || c->type <= 0 || c->type == TD_TABLE || c->type == TD_LIST) continue;
        if (!tdb_col_resident(c)) *upload += (size_t)c->len * td_sym_elem_size(c->type, c->attrs);
    }
}

size_t td_server_estimate(td_graph_t* g, td_op_t* root) {
    (void)root;
    if (!g) return 0;
    td_t* seen[64];
    int n_seen = 0;
    size_t upload = 0;
    int64_t rows_max = 0, rows_sum = 0;
    est_table(g->table, seen, &n_seen, &upload, &rows_max, &rows_sum);
    for (uint16_t i = 0; i < g->n_tables; i++) est_table(g->tables[i], seen, &n_seen, &upload, &rows_max, &rows_sum);
    for (uint32_t i = 0; i < g->ext_count; i++) {
        td_op_ext_t* x = g->ext_nodes[i];
        if (x && x->base.opcode == OP_CONST) est_table(x->literal, seen, &n_seen, &upload, &rows_max, &rows_sum);
    }
    /* columns not resident are uploaded; scratch (group records -- a direct
     * array holds at most two slots per row, 80 bytes at five words -- the
     * partitioned group-by's 20-byte entries, join map, selections, compacted
     * copies) is bounded by 128 bytes per row of the largest input and 16 per
     * row of the others */
    return upload + (size_t)rows_max * 128 + (size_t)(rows_sum - rows_max) * 16 + ((size_t)8 << 20);
}
