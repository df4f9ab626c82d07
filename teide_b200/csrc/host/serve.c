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
    uint64_t        completed;
};

static int64_t now_ns(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (int64_t)ts.tv_sec * 1000000000LL + ts.tv_nsec;
}

static void* worker_main(void* arg) {
    td_server_t* s = arg;
    tdb_share_builds(1);                /* join queries over one build table share its map */
    pthread_mutex_lock(&s->mu);
    for (;;) {
        req_t* r = NULL;
        if (s->next_admit < s->next_ticket) {
            req_t* head = &s->ring[s->next_admit % s->cap];
            const int fits = s->reserved + head->est <= s->budget || s->in_flight == 0;
            if (s->in_flight < s->slots && fits) r = head;
        }
        if (!r) {
            if (s->stop && s->next_admit >= s->next_ticket) break;
            pthread_cond_wait(&s->cv_work, &s->mu);
            continue;
        }
        s->next_admit++;
        s->in_flight++;
        s->reserved += r->est;
        if (s->in_flight > s->peak_in_flight) s->peak_in_flight = s->in_flight;
        if (s->reserved > s->peak_reserved) s->peak_reserved = s->reserved;
        r->state = 2;
        r->t.start_ns = now_ns();
        r->t.in_flight_at_start = s->in_flight;
        td_graph_t* g = r->g;
        td_op_t* root = r->root;
        const size_t est = r->est;
        const int64_t ticket = r->ticket;
        pthread_mutex_unlock(&s->mu);

        td_t* res = td_execute(g, root);

        pthread_mutex_lock(&s->mu);
        r = &s->ring[ticket % s->cap];
        r->result = res;
        r->t.end_ns = now_ns();
        r->t.status = TD_IS_ERR(res) ? (int32_t)TD_ERR_CODE(res) : 0;
        r->state = 3;
        s->in_flight--;
        s->reserved -= est;
        s->completed++;
        pthread_cond_broadcast(&s->cv_done);
        pthread_cond_broadcast(&s->cv_work);
    }
    pthread_mutex_unlock(&s->mu);
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
