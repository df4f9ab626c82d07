// Equi-join: build, probe and either materialize (count + emit) or aggregate
// in place (fused probe + group-by).
//
// Replaces exec_join (Teide src/ops/exec.c:8130-8741).  The CPU engine radix
// partitions both sides into 2^2..2^14 parts sized for a core's L2
// (radix_join_bits 7456-7471, join_radix_partition 7626-7742), builds and
// probes one open-addressing table per part (7824-7950), consolidates int32
// pair buffers into l_idx/r_idx (8357-8368) and gathers every output column
// (8607-8728).  Here:
//   - a build side whose single integer key spans a range no wider than
//     4x its row count gets a direct map: head[key - min] (TDG_JOIN_DIRECT);
//     anything else gets a global open-addressing table (TDG_JOIN_HASH);
//   - duplicate build keys chain through next[row];
//   - probing writes output columns directly at their final offsets (a
//     stable two-pass scheme, no pair buffers), or feeds the group-by.
#include "tdg_hash.cuh"
#include <string.h>

namespace tdg {

tdg_status group_run_joined(const tdg_group_desc* d, const tdg_group_plan* p, void* ws,
                            const tdg_expr* pred, const uint64_t* sel, const JoinK* J, int64_t n_left,
                            int64_t n_right, const tdg_group_out* out, cudaStream_t s);
tdg_status group_run_payload(const tdg_group_desc* d, const tdg_group_plan* p, void* ws,
                             const tdg_expr* pred, const uint64_t* sel, const JoinK* J, int64_t n_left,
                             int64_t n_right, const tdg_group_out* out, cudaStream_t s, bool* used,
                             bool prebuilt);
tdg_status join_payload_build(const tdg_group_desc* d, const tdg_group_plan* p, const JoinK* J, int32_t* err,
                              int64_t n_right, cudaStream_t s, int32_t* used);

constexpr int kJChunk = kThreads * 16;
constexpr int kMaxJCols = 16;

struct JLayout { size_t err, head, next, matched, state, keys, counts, total; };

static size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

static JLayout jlayout(const tdg_join_desc* d, const tdg_join_plan* p) {
    JLayout L;
    size_t o = 0;
    L.err = o; o += 256;
    L.head = o; o += al((size_t)p->n_slots * 4);
    L.next = o; o += al((size_t)(d->n_right > 0 ? d->n_right : 1) * 4);
    L.matched = o; o += al((size_t)(d->n_right > 0 ? d->n_right : 1));
    L.state = o; o += p->method == TDG_JOIN_HASH ? al((size_t)p->n_slots * 4) : 0;
    L.keys = o; o += p->method == TDG_JOIN_HASH ? al((size_t)p->n_slots * 8 * d->n_keys) : 0;
    L.counts = o; o += al((size_t)((d->n_left + kJChunk - 1) / kJChunk + 2) * 8);
    L.total = o;
    return L;
}

static JoinK make_jk(const tdg_join_desc* d, const tdg_join_plan* p, void* ws) {
    JoinK J;
    memset(&J, 0, sizeof(J));
    const JLayout L = jlayout(d, p);
    char* w = (char*)ws;
    J.method = p->method;
    J.nk = d->n_keys;
    J.join_type = d->join_type;
    for (int k = 0; k < d->n_keys; k++) {
        J.lkeys[k] = d->lkeys[k]; J.lkeys[k].side = 0;
        J.rkeys[k] = d->rkeys[k]; J.rkeys[k].side = 1;
    }
    J.key_f64 = d->n_keys == 1 && d->lkeys[0].type == T_F64;
    J.kmin = d->rkey_min;
    J.n_slots = p->n_slots;
    J.head = (int32_t*)(w + L.head);
    J.next = (int32_t*)(w + L.next);
    J.matched = d->join_type == 2 ? (uint8_t*)(w + L.matched) : nullptr;
    J.ht.state = (uint32_t*)(w + L.state);
    J.ht.keys = (int64_t*)(w + L.keys);
    J.ht.mask = (uint64_t)p->n_slots - 1;
    J.ht.nk = d->n_keys;
    J.ht.err = (int32_t*)(w + L.err);
    return J;
}

__global__ void k_join_init(int32_t* head, uint32_t* state, int64_t n_slots) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_slots; i += (int64_t)gridDim.x * blockDim.x) {
        head[i] = -1;
        if (state) state[i] = 0;
    }
}

__global__ void __launch_bounds__(kThreads) k_join_build(const JoinK J, int64_t n_right) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n_right;
         r += (int64_t)gridDim.x * blockDim.x) {
        int64_t slot;
        if (J.method == TDG_JOIN_DIRECT) {
            slot = ld_i(J.rkeys[0], r) - J.kmin;
            if (slot < 0 || slot >= J.n_slots) { set_err(J.ht.err, E_DOMAIN); continue; }
        } else {
            int64_t kv[TDG_MAX_KEYS];
            bool nan = false;
            for (int k = 0; k < J.nk; k++) {
                kv[k] = ld_keybits(J.rkeys[k], r);
                nan = nan || (J.rkeys[k].type == T_F64 && nan_bits(kv[k]));
            }
            if (nan) { J.next[r] = -1; continue; }   // NaN keys never match
            slot = ht_upsert(J.ht, kv, hash_keys(kv, J.nk));
            if (slot < 0) continue;
        }
        J.next[r] = atomicExch(&J.head[slot], (int32_t)r);
    }
}

template <int PK>
__device__ __forceinline__ int join_rows_of(const JoinK& J, const Pred& P, const tdg_expr& prog, int64_t r,
                                            int64_t n, int32_t* first) {
    *first = -1;
    if (r >= n || !row_pass<PK>(P, prog, r)) return 0;
    int32_t b = join_first(J, r);
    *first = b;
    int c = 0;
    while (b >= 0) { c++; b = __ldg(&J.next[b]); }
    return (c == 0 && J.join_type != 0) ? 1 : c;
}

template <int PK>
__global__ void __launch_bounds__(kThreads) k_join_count(const JoinK J, const Pred P, const tdg_expr prog,
                                                         int64_t n, int64_t* counts) {
    __shared__ int red[32];
    const int64_t base = (int64_t)blockIdx.x * kJChunk;
    long long c = 0;
    for (int i = 0; i < kJChunk / kThreads; i++) {
        int32_t f;
        const int64_t r = base + i * kThreads + threadIdx.x;
        const int m = join_rows_of<PK>(J, P, prog, r, n, &f);
        if (J.matched)
            for (int32_t b = f; b >= 0; b = __ldg(&J.next[b])) J.matched[b] = 1;
        c += m;
    }
    (void)red;
    __shared__ long long part[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += part[w];
        counts[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(kThreads) k_unmatched_count(const uint8_t* matched, int64_t n_right, int64_t* counts) {
    __shared__ int red[32];
    int c = 0;
    for (int64_t b = threadIdx.x; b < n_right; b += blockDim.x) c += matched[b] == 0;
    int tot;
    block_excl_scan(c, &tot, red);
    if (threadIdx.x == 0) *counts = tot;
}

struct JCols {
    int32_t nl, nr;
    int32_t lesz[kMaxJCols], resz[kMaxJCols];
    const void* lsrc[kMaxJCols];
    const void* rsrc[kMaxJCols];
    void* ldst[kMaxJCols];
    void* rdst[kMaxJCols];
};

__device__ __forceinline__ void put_elem(void* dst, int64_t di, const void* src, int64_t si, int esz) {
    if (si < 0) {
        for (int b = 0; b < esz; b++) ((uint8_t*)dst)[di * esz + b] = 0;
        return;
    }
    switch (esz) {
        case 8: ((uint64_t*)dst)[di] = __ldg((const unsigned long long*)src + si); break;
        case 4: ((uint32_t*)dst)[di] = __ldg((const unsigned int*)src + si); break;
        case 2: ((uint16_t*)dst)[di] = __ldg((const unsigned short*)src + si); break;
        case 1: ((uint8_t*)dst)[di] = __ldg((const unsigned char*)src + si); break;
        default: for (int b = 0; b < esz; b++) ((uint8_t*)dst)[di * esz + b] = ((const uint8_t*)src)[si * esz + b];
    }
}

__device__ __forceinline__ void emit_pair(const JCols& C, int64_t o, int64_t l, int64_t r) {
    for (int c = 0; c < C.nl; c++) put_elem(C.ldst[c], o, C.lsrc[c], l, C.lesz[c]);
    for (int c = 0; c < C.nr; c++) put_elem(C.rdst[c], o, C.rsrc[c], r, C.resz[c]);
}

template <int PK>
__global__ void __launch_bounds__(kThreads) k_join_emit(const JoinK J, const Pred P, const tdg_expr prog,
                                                        int64_t n, const int64_t* offsets, const JCols C) {
    __shared__ int red[32];
    const int64_t base = (int64_t)blockIdx.x * kJChunk;
    int64_t out = offsets[blockIdx.x];
    for (int i = 0; i < kJChunk / kThreads; i++) {
        int32_t f;
        const int64_t r = base + i * kThreads + threadIdx.x;
        const int m = join_rows_of<PK>(J, P, prog, r, n, &f);
        int tot;
        const int pre = block_excl_scan(m, &tot, red);
        int64_t o = out + pre;
        if (m > 0) {
            if (f < 0) {
                emit_pair(C, o, r, -1);                 // outer join: unmatched probe row
            } else {
                for (int32_t b = f; b >= 0; b = __ldg(&J.next[b])) emit_pair(C, o++, r, b);
            }
        }
        out += tot;
        if (base + (i + 1) * kThreads >= n) break;
    }
}

// Full outer join tail: build rows no probe row matched, in build-row order.
__global__ void __launch_bounds__(kThreads) k_unmatched_emit(const uint8_t* matched, int64_t n_right, int64_t out0,
                                                              const JCols C) {
    __shared__ int red[32];
    int64_t out = out0;
    for (int64_t b0 = 0; b0 < n_right; b0 += blockDim.x) {
        const int64_t b = b0 + threadIdx.x;
        const bool u = b < n_right && matched[b] == 0;
        int tot;
        const int pre = block_excl_scan(u ? 1 : 0, &tot, red);
        if (u) emit_pair(C, out + pre, -1, b);
        out += tot;
    }
}

__global__ void k_join_total(const int64_t* counts, int64_t chunks, int64_t* d_count) {
    // counts[] holds exclusive offsets after the scan; counts[chunks] is the
    // probe total and counts[chunks + 1] the unmatched build rows.
    *d_count = counts[chunks] + counts[chunks + 1];
}

__global__ void k_scan_counts_g(int64_t* counts, int64_t m, int64_t* d_total, const int32_t* err,
                                int32_t* herr);   // tdg_group.cu

static tdg_status jstatus(const JoinK& J, cudaStream_t s) {
    int32_t err = 0;
    if (cudaMemcpyAsync(&err, J.ht.err, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return E_IO;
    if (cudaStreamSynchronize(s) != cudaSuccess) return E_IO;
    return err;
}

static tdg_status check_desc(const tdg_join_desc* d) {
    if (d->n_keys < 1 || d->n_keys > TDG_MAX_KEYS) return E_NYI;
    if (d->join_type < 0 || d->join_type > 2) return E_NYI;
    if (d->n_left > INT32_MAX || d->n_right > INT32_MAX) return E_NYI;
    for (int k = 0; k < d->n_keys; k++) {
        const bool lf = d->lkeys[k].type == T_F64, rf = d->rkeys[k].type == T_F64;
        if (lf != rf) return E_TYPE;
        if (!elem_size(d->lkeys[k].type, d->lkeys[k].attrs) || !elem_size(d->rkeys[k].type, d->rkeys[k].attrs))
            return E_TYPE;
    }
    return E_OK;
}

}  // namespace tdg

using namespace tdg;

static int64_t pow2_at_least(int64_t x) {
    int64_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

extern "C" tdg_status tdg_join_plan_make(const tdg_join_desc* d, tdg_join_plan* p) {
    if (!d || !p) return E_TYPE;
    tdg_status st = check_desc(d);
    if (st) return st;
    memset(p, 0, sizeof(*p));
    const int64_t nr = d->n_right > 0 ? d->n_right : 1;
    bool direct = d->n_keys == 1 && d->have_range && is_int_class(d->rkeys[0].type) &&
                  is_int_class(d->lkeys[0].type) && d->rkey_max >= d->rkey_min;
    if (direct) {
        const uint64_t range = (uint64_t)d->rkey_max - (uint64_t)d->rkey_min + 1;
        direct = range != 0 && range <= (uint64_t)(4 * nr + 1024) && range <= ((uint64_t)1 << 31);
        if (direct) { p->method = TDG_JOIN_DIRECT; p->n_slots = (int64_t)range; }
    }
    if (!direct) {
        p->method = TDG_JOIN_HASH;
        p->n_slots = pow2_at_least(2 * nr > 1024 ? 2 * nr : 1024);
    }
    p->ws_bytes = jlayout(d, p).total;
    return E_OK;
}

extern "C" tdg_status tdg_join_build(const tdg_join_desc* d, const tdg_join_plan* p, void* ws, void* stream) {
    if (!d || !p || !ws) return E_TYPE;
    tdg_status st = check_desc(d);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    JoinK J = make_jk(d, p, ws);
    cudaMemsetAsync(J.ht.err, 0, 256, s);
    EventTimer tm;
    tm.start(s);
    int g = grid_for((const void*)k_join_init, kThreads, 0, p->n_slots);
    (note_launch(), k_join_init<<<g, kThreads, 0, s>>>(J.head, p->method == TDG_JOIN_HASH ? J.ht.state : nullptr, p->n_slots));
    if (d->join_type == 2 && d->n_right > 0) cudaMemsetAsync(J.matched, 0, (size_t)d->n_right, s);
    if (d->n_right > 0) {
        g = grid_for((const void*)k_join_build, kThreads, 0, d->n_right);
        (note_launch(), k_join_build<<<g, kThreads, 0, s>>>(J, d->n_right));
    }
    tm.stop(s);
    st = launch_status();
    if (st) { tm.ms(); return st; }
    st = jstatus(J, s);                  // synchronizes the stream
    const float ms = tm.ms();
    if (tm.on) set_last_build_ms(ms);
    return st;
}

static const tdg_expr& prog_ref(const tdg_expr* e) {
    static tdg_expr empty;
    return e ? *e : empty;
}

extern "C" tdg_status tdg_join_count(const tdg_join_desc* d, const tdg_join_plan* p, void* ws,
                                     const tdg_expr* lpred, const uint64_t* lsel, int64_t* d_count,
                                     void* stream) {
    if (!d || !p || !ws || !d_count) return E_TYPE;
    cudaStream_t s = (cudaStream_t)stream;
    JoinK J = make_jk(d, p, ws);
    const JLayout L = jlayout(d, p);
    int64_t* counts = (int64_t*)((char*)ws + L.counts);
    const int64_t chunks = (d->n_left + kJChunk - 1) / kJChunk;
    cudaMemsetAsync(counts, 0, (size_t)(chunks + 2) * 8, s);
    if (d->join_type == 2 && d->n_right > 0) cudaMemsetAsync(J.matched, 0, (size_t)d->n_right, s);
    int pk;
    Pred P = make_pred(lpred, lsel, &pk);
    const tdg_expr& pr = prog_ref(lpred);
    if (chunks > 0) {
        if (pk == 0) (note_launch(), k_join_count<0><<<(unsigned)chunks, kThreads, 0, s>>>(J, P, pr, d->n_left, counts));
        else if (pk == 1) (note_launch(), k_join_count<1><<<(unsigned)chunks, kThreads, 0, s>>>(J, P, pr, d->n_left, counts));
        else (note_launch(), k_join_count<2><<<(unsigned)chunks, kThreads, 0, s>>>(J, P, pr, d->n_left, counts));
    }
    (note_launch(), k_scan_counts_g<<<1, 1024, 0, s>>>(counts, chunks, counts + chunks, nullptr, nullptr));
    if (d->join_type == 2 && d->n_right > 0)
        (note_launch(), k_unmatched_count<<<1, kThreads, 0, s>>>(J.matched, d->n_right, counts + chunks + 1));
    (note_launch(), k_join_total<<<1, 1, 0, s>>>(counts, chunks, d_count));
    tdg_status st = launch_status();
    if (st) return st;
    return jstatus(J, s);
}

extern "C" tdg_status tdg_join_emit(const tdg_join_desc* d, const tdg_join_plan* p, void* ws,
                                    const tdg_expr* lpred, const uint64_t* lsel,
                                    int32_t n_lcols, const tdg_col* lsrc, void* const* ldst,
                                    int32_t n_rcols, const tdg_col* rsrc, void* const* rdst,
                                    void* stream) {
    if (!d || !p || !ws) return E_TYPE;
    if (n_lcols > kMaxJCols || n_rcols > kMaxJCols || n_lcols < 0 || n_rcols < 0) return E_NYI;
    cudaStream_t s = (cudaStream_t)stream;
    JoinK J = make_jk(d, p, ws);
    J.matched = nullptr;     // already marked by tdg_join_count
    const JLayout L = jlayout(d, p);
    int64_t* counts = (int64_t*)((char*)ws + L.counts);
    const int64_t chunks = (d->n_left + kJChunk - 1) / kJChunk;
    JCols C;
    memset(&C, 0, sizeof(C));
    C.nl = n_lcols;
    C.nr = n_rcols;
    for (int c = 0; c < n_lcols; c++) {
        C.lesz[c] = elem_size(lsrc[c].type, lsrc[c].attrs);
        C.lsrc[c] = lsrc[c].data;
        C.ldst[c] = ldst[c];
        if (!C.lesz[c]) return E_TYPE;
    }
    for (int c = 0; c < n_rcols; c++) {
        C.resz[c] = elem_size(rsrc[c].type, rsrc[c].attrs);
        C.rsrc[c] = rsrc[c].data;
        C.rdst[c] = rdst[c];
        if (!C.resz[c]) return E_TYPE;
    }
    int pk;
    Pred P = make_pred(lpred, lsel, &pk);
    const tdg_expr& pr = prog_ref(lpred);
    if (chunks > 0) {
        if (pk == 0) (note_launch(), k_join_emit<0><<<(unsigned)chunks, kThreads, 0, s>>>(J, P, pr, d->n_left, counts, C));
        else if (pk == 1) (note_launch(), k_join_emit<1><<<(unsigned)chunks, kThreads, 0, s>>>(J, P, pr, d->n_left, counts, C));
        else (note_launch(), k_join_emit<2><<<(unsigned)chunks, kThreads, 0, s>>>(J, P, pr, d->n_left, counts, C));
    }
    if (d->join_type == 2 && d->n_right > 0) {
        int64_t probe_total = 0;
        if (cudaMemcpyAsync(&probe_total, counts + chunks, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess) return E_IO;
        if (cudaStreamSynchronize(s) != cudaSuccess) return E_IO;
        const uint8_t* matched = (const uint8_t*)((char*)ws + L.matched);
        (note_launch(), k_unmatched_emit<<<1, kThreads, 0, s>>>(matched, d->n_right, probe_total, C));
    }
    return launch_status();
}

extern "C" tdg_status tdg_join_group_run(const tdg_join_desc* d, const tdg_join_plan* jp, void* jws,
                                         const tdg_expr* lpred, const uint64_t* lsel,
                                         const tdg_group_desc* g, const tdg_group_plan* gp, void* gws,
                                         const tdg_group_out* out, void* stream) {
    if (!d || !jp || !jws || !g || !gp || !gws || !out) return E_TYPE;
    tdg_status st = check_desc(d);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    JoinK J = make_jk(d, jp, jws);
    bool used = false;
    if (d->flags & TDG_JOIN_PREBUILT)    // the map is in jws; nothing here writes to it
        return group_run_payload(g, gp, gws, lpred, lsel, &J, d->n_left, d->n_right, out, s, &used, true);
    cudaMemsetAsync(J.ht.err, 0, 256, s);
    st = group_run_payload(g, gp, gws, lpred, lsel, &J, d->n_left, d->n_right, out, s, &used, false);
    if (st || used) return st;
    st = tdg_join_build(d, jp, jws, stream);
    if (st) return st;
    if (d->join_type == 2 && d->n_right > 0) cudaMemsetAsync(J.matched, 0, (size_t)d->n_right, s);
    return group_run_joined(g, gp, gws, lpred, lsel, &J, d->n_left, d->n_right, out, s);
}

extern "C" tdg_status tdg_join_payload_build(const tdg_join_desc* d, const tdg_join_plan* jp, void* jws,
                                             const tdg_group_desc* g, const tdg_group_plan* gp, int32_t* used,
                                             void* stream) {
    if (!d || !jp || !jws || !g || !gp || !used) return E_TYPE;
    *used = 0;
    tdg_status st = check_desc(d);
    if (st) return st;
    JoinK J = make_jk(d, jp, jws);
    return join_payload_build(g, gp, &J, J.ht.err, d->n_right, (cudaStream_t)stream, used);
}

// ---- the hash-table upsert as an entry point --------------------------------------
// One thread per key tuple; each one finds or claims its slot with ht_upsert.
__global__ void k_ht_upsert(tdg::HtRef H, const int64_t* kv, int64_t n, int64_t* slot) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int64_t t[TDG_MAX_KEYS];
    for (int k = 0; k < H.nk; k++) t[k] = kv[(int64_t)k * n + i];
    slot[i] = tdg::ht_upsert(H, t, tdg::hash_keys(t, H.nk));
}

extern "C" tdg_status tdg_hash_upsert(uint32_t* state, int64_t* keys, uint64_t cap, int32_t n_keys,
                                      const int64_t* kv, int64_t n, int32_t spin_limit, int64_t* d_slot,
                                      int32_t* d_err, void* stream) {
    using namespace tdg;
    if (cap == 0 || (cap & (cap - 1)) || n_keys < 1 || n_keys > TDG_MAX_KEYS || n < 0 || spin_limit < 0)
        return E_RANGE;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(d_err, 0, 4, s) != cudaSuccess) return launch_status();
    if (n > 0) {
        HtRef H;
        memset(&H, 0, sizeof(H));
        H.state = state;
        H.keys = keys;
        H.mask = cap - 1;
        H.nk = n_keys;
        H.spin_limit = spin_limit;
        H.err = d_err;
        const int threads = 256;
        (note_launch(), k_ht_upsert<<<(unsigned)((n + threads - 1) / threads), threads, 0, s>>>(H, kv, n, d_slot));
    }
    int32_t err = 0;
    if (cudaMemcpyAsync(&err, d_err, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        const tdg_status e = launch_status();
        return e ? e : E_IO;
    }
    return err ? err : launch_status();
}

