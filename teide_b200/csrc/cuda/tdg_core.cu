// Core services: predicate analysis, launch sizing, column statistics,
// expression evaluation and selection (filter) kernels.
//
// Selection replaces three CPU loops of Teide's executor: the expression VM
// writing one BOOL byte per row (exec.c:1104-1196), the single-threaded
// byte-to-bit packing of td_sel_from_pred + td_sel_recompute (sel.c:77-161)
// and the sequential match-index build + gather of exec_filter / sel_compact
// (exec.c:2065-2224, 2328-2480).  Here one pass evaluates the predicate and
// packs bits with warp ballots, and compaction is a two-pass stable scatter.
#include "tdg_common.cuh"
#include <atomic>
#include <math.h>
#include <string.h>

namespace tdg {

// ---- host helpers -------------------------------------------------------------

static int g_sms = 0;

int sm_count() {
    if (!g_sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || g_sms <= 0)
            g_sms = 148;
    }
    return g_sms;
}

// Resident CTAs per SM of (kernel, threads, shared memory) on the current
// device; the occupancy query costs microseconds of host time, which sit on
// the critical path of a query's first launch, so each thread keeps its
// answers.
static int occupancy(const void* kernel, int threads, size_t smem) {
    struct Entry { const void* k; int threads; int dev; size_t smem; int per_sm; };
    constexpr int kCap = 64;
    static thread_local Entry cache[kCap];
    static thread_local int n_cached, next_victim;
    int dev = 0;
    cudaGetDevice(&dev);
    for (int i = 0; i < n_cached; i++) {
        const Entry& e = cache[i];
        if (e.k == kernel && e.threads == threads && e.smem == smem && e.dev == dev) return e.per_sm;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        return 1;                               // not cached: the next call asks again
    }
    // a full cache replaces its entries in turn
    int at;
    if (n_cached < kCap) {
        at = n_cached++;
    } else {
        at = next_victim;
        next_victim = (next_victim + 1) % kCap;
    }
    cache[at] = Entry{kernel, threads, dev, smem, per_sm};
    return per_sm;
}

int grid_for(const void* kernel, int threads, size_t smem, int64_t work_items) {
    const int per_sm = occupancy(kernel, threads, smem);
    int64_t g = (int64_t)per_sm * sm_count();
    int64_t need = (work_items + threads - 1) / threads;
    if (need < g) g = need < 1 ? 1 : need;
    return (int)g;
}

tdg_status launch_status() {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return E_OK;
    return e == cudaErrorMemoryAllocation ? E_OOM : E_IO;
}

static std::atomic<unsigned long long> g_launches{0};
static std::atomic<int> g_timing{0};
static std::atomic<float> g_main_ms{0.f}, g_build_ms{0.f};

static thread_local int t_timing_off = 0;
static thread_local int t_no_alloc = 0;
ThreadNoAlloc::ThreadNoAlloc() { t_no_alloc++; }
ThreadNoAlloc::~ThreadNoAlloc() { t_no_alloc--; }
bool no_alloc() { return t_no_alloc != 0; }

ThreadTimingOff::ThreadTimingOff() { t_timing_off++; }
ThreadTimingOff::~ThreadTimingOff() { t_timing_off--; }

void note_launch(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }
bool timing_on() { return g_timing.load(std::memory_order_relaxed) != 0 && t_timing_off == 0; }
void set_last_main_ms(float ms) { g_main_ms.store(ms); }
void set_last_build_ms(float ms) { g_build_ms.store(ms); }
static std::atomic<float> g_sort_ms{0.f};
void set_last_sort_ms(float ms) { g_sort_ms.store(ms); }

// CUDA events for the timers, kept per host thread and device: creating and
// destroying two events per timed launch cost several microseconds of host
// time before the launch.  Freed when the thread exits.
namespace {
struct EventPool {
    cudaEvent_t ev[16] = {};
    int dev[16] = {};
    bool used[16] = {};
    ~EventPool() {
        for (int i = 0; i < 16; i++)
            if (ev[i]) cudaEventDestroy(ev[i]);
    }
};
thread_local EventPool t_events;

cudaEvent_t event_take() {
    int dev = 0;
    cudaGetDevice(&dev);
    EventPool& P = t_events;
    for (int i = 0; i < 16; i++)
        if (P.ev[i] && !P.used[i] && P.dev[i] == dev) { P.used[i] = true; return P.ev[i]; }
    for (int i = 0; i < 16; i++)
        if (!P.ev[i]) {
            if (cudaEventCreate(&P.ev[i]) != cudaSuccess) { cudaGetLastError(); P.ev[i] = nullptr; return nullptr; }
            P.dev[i] = dev;
            P.used[i] = true;
            return P.ev[i];
        }
    cudaEvent_t e = nullptr;                    // pool full: a transient event
    if (cudaEventCreate(&e) != cudaSuccess) { cudaGetLastError(); return nullptr; }
    return e;
}

void event_give(cudaEvent_t e) {
    if (!e) return;
    EventPool& P = t_events;
    for (int i = 0; i < 16; i++)
        if (P.ev[i] == e) { P.used[i] = false; return; }
    cudaEventDestroy(e);
}
}  // namespace

void EventTimer::start(cudaStream_t s) {
    on = timing_on();
    if (!on) return;
    if (!a) a = event_take();
    if (!b) b = event_take();
    if (!a || !b) { on = false; return; }
    cudaEventRecord(a, s);
}
void EventTimer::stop(cudaStream_t s) {
    if (on) cudaEventRecord(b, s);
}
EventTimer::~EventTimer() {
    event_give(a);
    event_give(b);
}
float EventTimer::ms() {
    float t = 0.f;
    if (on && cudaEventElapsedTime(&t, a, b) != cudaSuccess) { cudaGetLastError(); t = 0.f; }
    event_give(a);
    event_give(b);
    a = b = nullptr;
    return t;
}

// Recognize AND-trees of (column CMP constant) comparisons.
static bool collect_terms(const tdg_expr* e, int reg, Pred* p) {
    const tdg_ins& I = e->ins[reg];
    if (I.op == TDG_X_AND)
        return collect_terms(e, I.a, p) && collect_terms(e, I.b, p);
    if (I.op < TDG_X_EQ || I.op > TDG_X_GE) return false;
    const tdg_ins& A = e->ins[I.a];
    const tdg_ins& B = e->ins[I.b];
    int32_t op = I.op;
    const tdg_ins *col, *cst;
    if (A.op == TDG_X_COL && B.op == TDG_X_CONST) { col = &A; cst = &B; }
    else if (A.op == TDG_X_CONST && B.op == TDG_X_COL) {
        col = &B; cst = &A;    // k OP c  ->  c OP' k
        op = op == TDG_X_LT ? TDG_X_GT : op == TDG_X_GT ? TDG_X_LT :
             op == TDG_X_LE ? TDG_X_GE : op == TDG_X_GE ? TDG_X_LE : op;
    } else {
        return false;
    }
    if (col->kind != cst->kind || p->n >= kMaxTerms) return false;
    Term& t = p->t[p->n++];
    t.col = e->cols[col->imm];
    t.op = op;
    t.f = col->kind == 1;
    t.k = cst->imm;
    t.neg = op == TDG_X_NE;
    if (t.f) {
        double k;
        memcpy(&k, &cst->imm, 8);
        double lo = -INFINITY, hi = INFINITY;
        switch (op) {
            case TDG_X_EQ: case TDG_X_NE: lo = hi = k; break;
            case TDG_X_LT: hi = nextafter(k, -INFINITY); break;
            case TDG_X_LE: hi = k; break;
            case TDG_X_GT: lo = nextafter(k, INFINITY); break;
            default: lo = k; break;
        }
        if (k != k) { lo = INFINITY; hi = -INFINITY; }   // comparisons with NaN are false
        if (k != k && op == TDG_X_NE) { lo = INFINITY; hi = -INFINITY; }
        memcpy(&t.lo, &lo, 8);
        memcpy(&t.hi, &hi, 8);
    } else {
        const int64_t k = cst->imm;
        int64_t lo = INT64_MIN, hi = INT64_MAX;
        switch (op) {
            case TDG_X_EQ: case TDG_X_NE: lo = hi = k; break;
            case TDG_X_LT: if (k == INT64_MIN) { lo = 1; hi = 0; } else hi = k - 1; break;
            case TDG_X_LE: hi = k; break;
            case TDG_X_GT: if (k == INT64_MAX) { lo = 1; hi = 0; } else lo = k + 1; break;
            default: lo = k; break;
        }
        t.lo = lo;
        t.hi = hi;
    }
    return true;
}

Pred make_pred(const tdg_expr* prog, const uint64_t* sel, int* pk) {
    Pred p;
    memset(&p, 0, sizeof(p));
    p.sel = sel;
    p.w8 = 1;
    if (!prog || prog->n_ins <= 0) { *pk = 0; return p; }
    if (collect_terms(prog, prog->out, &p)) {
        for (int i = 0; i < p.n; i++) p.w8 = p.w8 && elem_size(p.t[i].col.type, p.t[i].col.attrs) == 8;
        p.kind = 1;
        *pk = 1;
        return p;
    }
    p.w8 = 0;
    memset(p.t, 0, sizeof(p.t));
    p.n = 0;
    p.kind = 2;
    *pk = 2;
    return p;
}

// ---- column min/max --------------------------------------------------------------

__global__ void k_minmax_init(int64_t* out) { out[0] = INT64_MAX; out[1] = INT64_MIN; }

__global__ void __launch_bounds__(kThreads) k_minmax(tdg_col c, int64_t n, int64_t* out) {
    long long lo = INT64_MAX, hi = INT64_MIN;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
         r += (int64_t)gridDim.x * blockDim.x) {
        long long v = ld_i(c, r);
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        long long a = __shfl_xor_sync(0xffffffffu, lo, o);
        long long b = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin((long long*)out, lo);
        atomicMax((long long*)out + 1, hi);
    }
}

// ---- expression -> column ------------------------------------------------------------

__global__ void __launch_bounds__(kThreads) k_eval(const tdg_expr e, int64_t n, void* out, int kind) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n;
         r += (int64_t)gridDim.x * blockDim.x) {
        uint64_t v = x_eval(e, r);
        const bool vf = e.ins[e.out].kind == 1;
        if (kind == 2) {
            ((uint8_t*)out)[r] = v != 0;
        } else if (kind == 1) {
            ((double*)out)[r] = vf ? __longlong_as_double((long long)v) : (double)(int64_t)v;
        } else {
            ((int64_t*)out)[r] = vf ? (int64_t)__longlong_as_double((long long)v) : (int64_t)v;
        }
    }
}

// ---- TD_SEL bitmap ----------------------------------------------------------------
// One warp per 1024-row segment: 32 ballots of 32 rows give the segment's
// 16 words, its popcount and its NONE/ALL/MIX flag.
template <int PK>
__global__ void __launch_bounds__(kThreads) k_sel_bitmap(const Pred p, const tdg_expr prog, int64_t n,
                                                         uint64_t* bits, uint8_t* flags, uint16_t* pop,
                                                         unsigned long long* total) {
    const int lane = threadIdx.x & 31;
    const int64_t nseg = (n + 1023) >> 10;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    unsigned long long my_total = 0;
    for (int64_t s = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5); s < nseg; s += warps) {
        const int64_t base = s << 10;
        uint32_t lo = 0;
        int cnt = 0;
        for (int i = 0; i < 32; i++) {
            const int64_t r = base + i * 32 + lane;
            const bool pass = r < n && row_pass<PK>(p, prog, r);
            const uint32_t m = __ballot_sync(0xffffffffu, pass);
            cnt += __popc(m);
            if (i & 1) {
                const uint64_t w = (uint64_t)lo | ((uint64_t)m << 32);
                const int64_t wi = (base >> 6) + (i >> 1);
                if (lane == 0 && wi < ((n + 63) >> 6)) bits[wi] = w;
            } else {
                lo = m;
            }
        }
        if (lane == 0) {
            const int64_t rows = n - base < 1024 ? n - base : 1024;
            pop[s] = (uint16_t)cnt;
            flags[s] = cnt == 0 ? 0 : (cnt == rows ? 1 : 2);
            my_total += cnt;
        }
    }
    if (lane == 0 && my_total) atomicAdd(total, my_total);
}

// ---- stable compaction -------------------------------------------------------------
// Rows are cut into chunks of kChunk; pass 1 counts the selected rows of
// each chunk, a single-block pass turns the counts into offsets, pass 2
// writes the selected rows of each chunk in row order.
constexpr int kChunk = kThreads * 32;

template <int PK>
__global__ void __launch_bounds__(kThreads) k_sel_count(const Pred p, const tdg_expr prog, int64_t n,
                                                        int64_t* counts) {
    __shared__ int red[32];
    const int64_t base = (int64_t)blockIdx.x * kChunk;
    int c = 0;
    for (int i = 0; i < kChunk / kThreads; i++) {
        const int64_t r = base + i * kThreads + threadIdx.x;
        c += (r < n && row_pass<PK>(p, prog, r)) ? 1 : 0;
    }
    int tot;
    block_excl_scan(c, &tot, red);
    if (threadIdx.x == 0) counts[blockIdx.x] = tot;
}

// Exclusive scan of m int64 counts in place by one block; total to *d_total.
__global__ void __launch_bounds__(1024) k_scan_counts(int64_t* counts, int64_t m, int64_t* d_total) {
    __shared__ long long part[1024];
    const int64_t per = (m + blockDim.x - 1) / blockDim.x;
    const int64_t b = threadIdx.x * per, e = b + per < m ? b + per : m;
    long long s = 0;
    for (int64_t i = b; i < e; i++) s += counts[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {
        long long v = threadIdx.x >= (unsigned)o ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    long long run = threadIdx.x ? part[threadIdx.x - 1] : 0;
    for (int64_t i = b; i < e; i++) { long long c = counts[i]; counts[i] = run; run += c; }
    if (threadIdx.x == blockDim.x - 1 && d_total) *d_total = part[blockDim.x - 1];
}

constexpr int kMaxGatherCols = 16;
struct GatherCols {
    int32_t n;
    int32_t esz[kMaxGatherCols];
    const void* src[kMaxGatherCols];
    void* dst[kMaxGatherCols];
};

__device__ __forceinline__ void copy_elem(void* dst, int64_t di, const void* src, int64_t si, int esz) {
    switch (esz) {
        case 8: ((uint64_t*)dst)[di] = ld_stream((const unsigned long long*)src + si); break;
        case 4: ((uint32_t*)dst)[di] = ld_stream((const unsigned int*)src + si); break;
        case 2: ((uint16_t*)dst)[di] = ld_stream((const unsigned short*)src + si); break;
        case 1: ((uint8_t*)dst)[di] = ld_stream((const unsigned char*)src + si); break;
        default:
            for (int b = 0; b < esz; b++) ((uint8_t*)dst)[di * esz + b] = ((const uint8_t*)src)[si * esz + b];
    }
}

template <int PK>
__global__ void __launch_bounds__(kThreads) k_sel_gather(const Pred p, const tdg_expr prog, int64_t n,
                                                         const int64_t* offsets, const GatherCols g) {
    __shared__ int red[32];
    const int64_t base = (int64_t)blockIdx.x * kChunk;
    int64_t out = offsets[blockIdx.x];
    for (int i = 0; i < kChunk / kThreads; i++) {
        const int64_t r = base + i * kThreads + threadIdx.x;
        const bool pass = r < n && row_pass<PK>(p, prog, r);
        int tot;
        const int pre = block_excl_scan(pass ? 1 : 0, &tot, red);
        if (pass)
            for (int c = 0; c < g.n; c++) copy_elem(g.dst[c], out + pre, g.src[c], r, g.esz[c]);
        out += tot;
        if (base + (i + 1) * kThreads >= n) break;
    }
}

}  // namespace tdg

using namespace tdg;

// ---- C ABI ------------------------------------------------------------------------

extern "C" int32_t tdg_device_sm_count(void) { return sm_count(); }

extern "C" tdg_status tdg_minmax(tdg_col col, int64_t n, int64_t* d_out, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (!is_int_class(col.type)) return E_TYPE;
    (note_launch(), k_minmax_init<<<1, 1, 0, s>>>(d_out));
    if (n > 0) {
        int g = grid_for((const void*)k_minmax, kThreads, 0, n);
        (note_launch(), k_minmax<<<g, kThreads, 0, s>>>(col, n, d_out));
    }
    return launch_status();
}

extern "C" tdg_status tdg_eval(const tdg_expr* e, int64_t n, void* out, int32_t out_kind, void* stream) {
    if (!e || e->n_ins <= 0 || e->n_ins > TDG_MAX_INS) return E_TYPE;
    if (n <= 0) return E_OK;
    int g = grid_for((const void*)k_eval, kThreads, 0, n);
    (note_launch(), k_eval<<<g, kThreads, 0, (cudaStream_t)stream>>>(*e, n, out, out_kind));
    return launch_status();
}

static const tdg_expr& prog_or_empty(const tdg_expr* e) {
    static tdg_expr empty;
    return e ? *e : empty;
}

extern "C" tdg_status tdg_select_bitmap(int64_t n, const tdg_expr* pred, const uint64_t* sel_in,
                                        uint64_t* bits, uint8_t* seg_flags, uint16_t* seg_popcnt,
                                        int64_t* d_total, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(d_total, 0, sizeof(int64_t), s);
    if (n <= 0) return launch_status();
    int pk;
    Pred p = make_pred(pred, sel_in, &pk);
    const tdg_expr& pr = prog_or_empty(pred);
    const int64_t nseg = (n + 1023) >> 10;
    const int64_t threads_needed = nseg * 32;
#define LAUNCH(PKV)                                                                                  \
    {                                                                                                \
        int g = grid_for((const void*)k_sel_bitmap<PKV>, kThreads, 0, threads_needed);               \
        (note_launch(), k_sel_bitmap<PKV><<<g, kThreads, 0, s>>>(p, pr, n, bits, seg_flags, seg_popcnt,              \
                                                 (unsigned long long*)d_total));                      \
    }
    if (pk == 0) LAUNCH(0) else if (pk == 1) LAUNCH(1) else LAUNCH(2)
#undef LAUNCH
    return launch_status();
}

extern "C" size_t tdg_select_ws_bytes(int64_t n) {
    int64_t chunks = (n + kChunk - 1) / kChunk;
    return (size_t)(chunks + 1) * sizeof(int64_t);
}

extern "C" tdg_status tdg_select_count(int64_t n, const tdg_expr* pred, const uint64_t* sel_in,
                                       void* ws, int64_t* d_count, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (n <= 0) { cudaMemsetAsync(d_count, 0, sizeof(int64_t), s); return launch_status(); }
    int pk;
    Pred p = make_pred(pred, sel_in, &pk);
    const tdg_expr& pr = prog_or_empty(pred);
    const int64_t chunks = (n + kChunk - 1) / kChunk;
    int64_t* counts = (int64_t*)ws;
    if (pk == 0) (note_launch(), k_sel_count<0><<<(unsigned)chunks, kThreads, 0, s>>>(p, pr, n, counts));
    else if (pk == 1) (note_launch(), k_sel_count<1><<<(unsigned)chunks, kThreads, 0, s>>>(p, pr, n, counts));
    else (note_launch(), k_sel_count<2><<<(unsigned)chunks, kThreads, 0, s>>>(p, pr, n, counts));
    (note_launch(), k_scan_counts<<<1, 1024, 0, s>>>(counts, chunks, d_count));
    return launch_status();
}

extern "C" tdg_status tdg_select_gather(int64_t n, const tdg_expr* pred, const uint64_t* sel_in,
                                        const void* ws, int32_t n_cols, const tdg_col* src,
                                        void* const* dst, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    if (n <= 0 || n_cols <= 0) return E_OK;
    int pk;
    Pred p = make_pred(pred, sel_in, &pk);
    const tdg_expr& pr = prog_or_empty(pred);
    const int64_t chunks = (n + kChunk - 1) / kChunk;
    for (int c0 = 0; c0 < n_cols; c0 += kMaxGatherCols) {
        GatherCols g;
        memset(&g, 0, sizeof(g));
        g.n = n_cols - c0 < kMaxGatherCols ? n_cols - c0 : kMaxGatherCols;
        for (int c = 0; c < g.n; c++) {
            g.esz[c] = elem_size(src[c0 + c].type, src[c0 + c].attrs);
            if (!g.esz[c]) return E_TYPE;
            g.src[c] = src[c0 + c].data;
            g.dst[c] = dst[c0 + c];
        }
        const int64_t* off = (const int64_t*)ws;
        if (pk == 0) (note_launch(), k_sel_gather<0><<<(unsigned)chunks, kThreads, 0, s>>>(p, pr, n, off, g));
        else if (pk == 1) (note_launch(), k_sel_gather<1><<<(unsigned)chunks, kThreads, 0, s>>>(p, pr, n, off, g));
        else (note_launch(), k_sel_gather<2><<<(unsigned)chunks, kThreads, 0, s>>>(p, pr, n, off, g));
    }
    return launch_status();
}

// ---- run-length expansion -----------------------------------------------------------
// out[r] = vals[p] for starts[p] <= r < starts[p + 1]: a column given as runs
// (a partitioned table's MAPCOMMON partition key, one value per partition)
// written out row by row.  Each thread finds its row's run by binary search.
__global__ void __launch_bounds__(kThreads) k_expand_runs(const char* vals, int esz, const int64_t* starts,
                                                          int64_t n_runs, char* out, int64_t n) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        int64_t a = 0, b = n_runs - 1;
        while (a < b) {
            const int64_t m = (a + b + 1) >> 1;
            if (__ldg(starts + m) <= r) a = m; else b = m - 1;
        }
        switch (esz) {
            case 8: ((int64_t*)out)[r] = ((const int64_t*)vals)[a]; break;
            case 4: ((int32_t*)out)[r] = ((const int32_t*)vals)[a]; break;
            case 2: ((int16_t*)out)[r] = ((const int16_t*)vals)[a]; break;
            default: out[r] = vals[a]; break;
        }
    }
}

extern "C" tdg_status tdg_expand_runs(const void* vals, int32_t esz, const int64_t* starts, int64_t n_runs,
                                      void* out, int64_t n, void* stream) {
    if (n <= 0) return E_OK;
    if (n_runs <= 0 || (esz != 1 && esz != 2 && esz != 4 && esz != 8)) return E_RANGE;
    const int g = grid_for((const void*)k_expand_runs, kThreads, 0, n);
    (note_launch(), k_expand_runs<<<g, kThreads, 0, (cudaStream_t)stream>>>((const char*)vals, esz, starts, n_runs,
                                                                          (char*)out, n));
    return launch_status();
}

extern "C" void tdg_set_timing(int32_t on) { g_timing.store(on ? 1 : 0); }
extern "C" int32_t tdg_timing_enabled(void) { return g_timing.load(); }
extern "C" void tdg_count_launches(uint64_t n) { note_launch((int)n); }
extern "C" float tdg_last_main_ms(void) { return g_main_ms.load(); }
extern "C" float tdg_last_build_ms(void) { return g_build_ms.load(); }
extern "C" float tdg_last_sort_ms(void) { return g_sort_ms.load(); }
extern "C" uint64_t tdg_launch_count(void) { return g_launches.load(); }
