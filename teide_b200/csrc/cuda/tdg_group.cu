// Group-by: fused selection + aggregation + emit.
//
// Replaces exec_group (Teide src/ops/exec.c:5542-6879).  The CPU engine picks
// a direct array for dense integer keys of at most 262,144 composite slots
// (exec.c:5948-6404) and otherwise a 256-way radix-partitioned hash table
// built in three phases (exec.c:6406-6667).  Here:
//
//   direct array (TDG_GROUP_DIRECT) -- slot = sum_k (key_k - min_k) * stride_k.
//     When the accumulators fit in 48 KB they are privatized per CTA in
//     shared memory and merged into global memory once per CTA; larger
//     arrays (up to 2^26 slots) are updated in place with global atomics,
//     whose hot lines stay in L2.
//   hash table (TDG_GROUP_HASH) -- open addressing in HBM (tdg_hash.cuh),
//     one pass, no partitioning.
//
// Both keep the same accumulator layout -- count[S] plus one 8-byte array
// per non-COUNT aggregate -- and share one emit pass that writes the groups
// whose count is non-zero in slot order (ascending key order for the direct
// array, like Teide's DA emit at exec.c:6330-6391).
//
// Arithmetic matches the CPU loops: integer SUM wraps, AVG = sum / count in
// double (exec.c:4430-4432, emit_agg_columns 4632-4773), MIN/MAX of F64 skip
// NaN.  F64 SUM is accumulated with atomics, so its summation order differs
// from the CPU's per-worker order; results agree to ~1e-15 relative.
#include "tdg_hash.cuh"
#include <string.h>

namespace tdg {

constexpr int kItems = 4;
constexpr int kEmitChunk = kThreads * 32;
constexpr size_t kSmemAccMax = 48 * 1024;
constexpr int64_t kDirectMaxSlots = (int64_t)1 << 26;

struct GroupK {
    int32_t nk, na, method, n_acc;
    tdg_col key[TDG_MAX_KEYS];
    int64_t kmin[TDG_MAX_KEYS], krange[TDG_MAX_KEYS], stride[TDG_MAX_KEYS];
    int32_t op[TDG_MAX_AGGS];
    int32_t f[TDG_MAX_AGGS];      // aggregate input is F64
    int32_t ai[TDG_MAX_AGGS];     // accumulator index, -1 for COUNT
    tdg_col in[TDG_MAX_AGGS];
    int64_t S;
    unsigned long long* cnt;
    unsigned long long* acc;      // n_acc * S
    HtRef ht;
    int32_t* err;
};

struct OutK {
    void* keys[TDG_MAX_KEYS];
    int32_t kesz[TDG_MAX_KEYS];
    void* aggs[TDG_MAX_AGGS];
};

// ---- typed multi-row loads --------------------------------------------------
// Loads N rows of one column (row < 0 or masked off gives 0).  The type switch
// runs once per column, so the N loads issue back to back.  Probe-side
// columns stream (evict-first); build-side columns are gathered at random and
// use the read-only path so they stay cached.
template <int N>
__device__ __forceinline__ void ld_items_i(const tdg_col& c, const int64_t (&r)[N], const bool (&m)[N],
                                           int64_t (&v)[N]) {
#define TDG_LD(T)                                                                        \
    {                                                                                    \
        const T* p = (const T*)c.data;                                                   \
        _Pragma("unroll") for (int i = 0; i < N; i++)                                    \
            v[i] = (m[i] && r[i] >= 0) ? (int64_t)(c.side ? __ldg(p + r[i]) : ld_stream(p + r[i])) : 0; \
    }
    switch (c.type) {
        case T_I64: case T_TIMESTAMP: TDG_LD(long long) break;
        case T_I32: case T_DATE: case T_TIME: TDG_LD(int) break;
        case T_I16: TDG_LD(short) break;
        case T_BOOL: case T_U8: case T_CHAR: TDG_LD(unsigned char) break;
        case T_SYM:
            switch (c.attrs & 3) {
                case 0: TDG_LD(unsigned char) break;
                case 1: TDG_LD(unsigned short) break;
                case 2: TDG_LD(unsigned int) break;
                default: TDG_LD(long long) break;
            }
            break;
        case T_F64: {
            const double* p = (const double*)c.data;
#pragma unroll
            for (int i = 0; i < N; i++)
                v[i] = (m[i] && r[i] >= 0) ? (int64_t)(c.side ? __ldg(p + r[i]) : ld_stream(p + r[i])) : 0;
            break;
        }
        default:
#pragma unroll
            for (int i = 0; i < N; i++) v[i] = 0;
    }
#undef TDG_LD
}

template <int N>
__device__ __forceinline__ void ld_items_f(const tdg_col& c, const int64_t (&r)[N], const bool (&m)[N],
                                           double (&v)[N]) {
    if (c.type == T_F64) {
        const double* p = (const double*)c.data;
#pragma unroll
        for (int i = 0; i < N; i++)
            v[i] = (m[i] && r[i] >= 0) ? (c.side ? __ldg(p + r[i]) : ld_stream(p + r[i])) : 0.0;
    } else {
        int64_t t[N];
        ld_items_i<N>(c, r, m, t);
#pragma unroll
        for (int i = 0; i < N; i++) v[i] = (double)t[i];
    }
}

__device__ __forceinline__ unsigned long long acc_init(int op) {
    return op == A_MIN ? (unsigned long long)INT64_MAX : op == A_MAX ? (unsigned long long)INT64_MIN : 0ULL;
}

template <bool GLOBAL>
__device__ __forceinline__ void upd_i(unsigned long long* a, int op, int64_t v) {
    if (op == A_MIN) {
        if (!GLOBAL || v < *(volatile long long*)a) atomicMin((long long*)a, (long long)v);
    } else if (op == A_MAX) {
        if (!GLOBAL || v > *(volatile long long*)a) atomicMax((long long*)a, (long long)v);
    } else {
        atomicAdd(a, (unsigned long long)v);
    }
}

template <bool GLOBAL>
__device__ __forceinline__ void upd_f(unsigned long long* a, int op, double v) {
    if (op == A_MIN || op == A_MAX) {
        if (v != v) return;                       // NaN never becomes a MIN/MAX
        const long long o = f2ord(v);
        if (op == A_MIN) {
            if (!GLOBAL || o < *(volatile long long*)a) atomicMin((long long*)a, o);
        } else {
            if (!GLOBAL || o > *(volatile long long*)a) atomicMax((long long*)a, o);
        }
    } else {
        atomicAdd((double*)a, v);
    }
}

// Slot of each (probe row, build row) pair; -1 when masked off or on error.
template <int MODE, int N>
__device__ __forceinline__ void slots_of(const GroupK& G, const int64_t (&rp)[N], const int64_t (&rb)[N],
                                         const bool (&m)[N], int64_t (&slot)[N]) {
    if (MODE != 2) {
        bool ok[N];
#pragma unroll
        for (int i = 0; i < N; i++) { slot[i] = 0; ok[i] = m[i]; }
        for (int k = 0; k < G.nk; k++) {
            int64_t v[N];
            ld_items_i<N>(G.key[k], G.key[k].side ? rb : rp, m, v);
#pragma unroll
            for (int i = 0; i < N; i++) {
                const int64_t d = v[i] - G.kmin[k];
                if (ok[i] && (d < 0 || d >= G.krange[k])) { set_err(G.err, E_DOMAIN); ok[i] = false; }
                slot[i] += d * G.stride[k];
            }
        }
#pragma unroll
        for (int i = 0; i < N; i++) if (!ok[i]) slot[i] = -1;
    } else {
#pragma unroll
        for (int i = 0; i < N; i++) {
            slot[i] = -1;
            if (!m[i]) continue;
            int64_t kv[TDG_MAX_KEYS];
            for (int k = 0; k < G.nk; k++) {
                const tdg_col& c = G.key[k];
                const int64_t row = c.side ? rb[i] : rp[i];
                kv[k] = row < 0 ? 0 : ld_keybits(c, row);
            }
            slot[i] = ht_upsert(G.ht, kv, hash_keys(kv, G.nk));
        }
    }
}

template <int MODE, int N>
__device__ __forceinline__ void accumulate(const GroupK& G, unsigned long long* cnt, unsigned long long* acc,
                                           int64_t S, const int64_t (&rp)[N], const int64_t (&rb)[N],
                                           const bool (&m)[N]) {
    constexpr bool GL = MODE != 0;
    int64_t slot[N];
    slots_of<MODE, N>(G, rp, rb, m, slot);
    bool ok[N];
#pragma unroll
    for (int i = 0; i < N; i++) {
        ok[i] = m[i] && slot[i] >= 0;
        if (ok[i]) atomicAdd(&cnt[slot[i]], 1ULL);
    }
    for (int a = 0; a < G.na; a++) {
        const int op = G.op[a];
        if (op == A_COUNT) continue;
        unsigned long long* base = acc + (int64_t)G.ai[a] * S;
        const tdg_col& c = G.in[a];
        const int64_t (&rr)[N] = c.side ? rb : rp;
        if (G.f[a]) {
            double v[N];
            ld_items_f<N>(c, rr, ok, v);
#pragma unroll
            for (int i = 0; i < N; i++) if (ok[i]) upd_f<GL>(base + slot[i], op, v[i]);
        } else {
            int64_t v[N];
            ld_items_i<N>(c, rr, ok, v);
#pragma unroll
            for (int i = 0; i < N; i++) if (ok[i]) upd_i<GL>(base + slot[i], op, v[i]);
        }
    }
}

// MODE 0: direct array in shared memory; 1: direct array in global memory;
// 2: hash table.  JOIN: probe rows are joined through J first and every
// (probe, build) match is one input row of the group-by.
template <int PK, int MODE, bool JOIN>
__global__ void __launch_bounds__(kThreads) k_group(const GroupK G, const Pred P, const tdg_expr prog,
                                                    const JoinK J, int64_t n) {
    extern __shared__ unsigned long long sm[];
    const int64_t S = G.S;
    unsigned long long* cnt = MODE == 0 ? sm : G.cnt;
    unsigned long long* acc = MODE == 0 ? sm + S : G.acc;
    if (MODE == 0) {
        for (int64_t s = threadIdx.x; s < S; s += blockDim.x) cnt[s] = 0;
        for (int a = 0; a < G.na; a++) {
            if (G.ai[a] < 0) continue;
            const unsigned long long init = acc_init(G.op[a]);
            for (int64_t s = threadIdx.x; s < S; s += blockDim.x) acc[(int64_t)G.ai[a] * S + s] = init;
        }
        __syncthreads();
    }
    const int64_t tile = (int64_t)kThreads * kItems;
    for (int64_t base = (int64_t)blockIdx.x * tile; base < n; base += (int64_t)gridDim.x * tile) {
        int64_t rp[kItems], rb[kItems];
        bool m[kItems];
#pragma unroll
        for (int i = 0; i < kItems; i++) {
            rp[i] = base + i * kThreads + threadIdx.x;
            rb[i] = -1;
            m[i] = rp[i] < n && row_pass<PK>(P, prog, rp[i]);
        }
        if (JOIN) {
#pragma unroll
            for (int i = 0; i < kItems; i++) {
                if (m[i]) rb[i] = join_first(J, rp[i]);
                if (J.join_type == 0) m[i] = m[i] && rb[i] >= 0;
                if (J.matched && rb[i] >= 0) J.matched[rb[i]] = 1;
            }
        }
        accumulate<MODE, kItems>(G, cnt, acc, S, rp, rb, m);
        if (JOIN) {
            // further matches of duplicate build keys
            for (int i = 0; i < kItems; i++) {
                if (!m[i] || rb[i] < 0) continue;
                int32_t nb = __ldg(&J.next[rb[i]]);
                while (nb >= 0) {
                    int64_t p1[1] = {rp[i]}, b1[1] = {nb};
                    bool m1[1] = {true};
                    if (J.matched) J.matched[nb] = 1;
                    accumulate<MODE, 1>(G, cnt, acc, S, p1, b1, m1);
                    nb = __ldg(&J.next[nb]);
                }
            }
        }
    }
    if (MODE == 0) {
        __syncthreads();
        for (int64_t s = threadIdx.x; s < S; s += blockDim.x) {
            const unsigned long long c = cnt[s];
            if (!c) continue;
            atomicAdd(&G.cnt[s], c);
            for (int a = 0; a < G.na; a++) {
                const int op = G.op[a];
                if (op == A_COUNT) continue;
                const int64_t o = (int64_t)G.ai[a] * S + s;
                const unsigned long long v = acc[o];
                if (op == A_MIN) atomicMin((long long*)&G.acc[o], (long long)v);
                else if (op == A_MAX) atomicMax((long long*)&G.acc[o], (long long)v);
                else if (G.f[a]) atomicAdd((double*)&G.acc[o], __longlong_as_double((long long)v));
                else atomicAdd(&G.acc[o], v);
            }
        }
    }
}

// Full outer join: build rows that no probe row matched enter the group-by
// with zero-filled probe-side values.
template <int MODE>
__global__ void __launch_bounds__(kThreads) k_group_unmatched(const GroupK G, const JoinK J, int64_t n_right) {
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < n_right;
         b += (int64_t)gridDim.x * blockDim.x) {
        if (J.matched[b]) continue;
        int64_t p1[1] = {-1}, b1[1] = {b};
        bool m1[1] = {true};
        accumulate<MODE == 0 ? 1 : MODE, 1>(G, G.cnt, G.acc, G.S, p1, b1, m1);
    }
}

__global__ void k_group_init(const GroupK G) {
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < G.S; s += (int64_t)gridDim.x * blockDim.x) {
        G.cnt[s] = 0;
        for (int a = 0; a < G.na; a++)
            if (G.ai[a] >= 0) G.acc[(int64_t)G.ai[a] * G.S + s] = acc_init(G.op[a]);
        if (G.method == TDG_GROUP_HASH) G.ht.state[s] = 0;
    }
}

// ---- emit ------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_emit_count(const unsigned long long* cnt, int64_t S, int64_t* counts) {
    __shared__ int red[32];
    const int64_t base = (int64_t)blockIdx.x * kEmitChunk;
    int c = 0;
    for (int i = 0; i < kEmitChunk / kThreads; i++) {
        const int64_t s = base + i * kThreads + threadIdx.x;
        c += (s < S && cnt[s] != 0) ? 1 : 0;
    }
    int tot;
    block_excl_scan(c, &tot, red);
    if (threadIdx.x == 0) counts[blockIdx.x] = tot;
}

__device__ __forceinline__ void put_key(void* dst, int esz, int64_t i, int64_t v) {
    switch (esz) {
        case 8: ((int64_t*)dst)[i] = v; break;
        case 4: ((int32_t*)dst)[i] = (int32_t)v; break;
        case 2: ((int16_t*)dst)[i] = (int16_t)v; break;
        default: ((int8_t*)dst)[i] = (int8_t)v; break;
    }
}

__global__ void __launch_bounds__(kThreads) k_emit(const GroupK G, const OutK O, const int64_t* offsets) {
    __shared__ int red[32];
    const int64_t base = (int64_t)blockIdx.x * kEmitChunk;
    int64_t out = offsets[blockIdx.x];
    const int64_t S = G.S;
    for (int i = 0; i < kEmitChunk / kThreads; i++) {
        const int64_t s = base + i * kThreads + threadIdx.x;
        const unsigned long long c = s < S ? G.cnt[s] : 0;
        int tot;
        const int pre = block_excl_scan(c ? 1 : 0, &tot, red);
        if (c) {
            const int64_t o = out + pre;
            for (int k = 0; k < G.nk; k++) {
                int64_t v;
                if (G.method == TDG_GROUP_DIRECT) v = G.kmin[k] + (s / G.stride[k]) % G.krange[k];
                else v = G.ht.keys[(int64_t)k * S + s];
                put_key(O.keys[k], O.kesz[k], o, v);
            }
            for (int a = 0; a < G.na; a++) {
                const int op = G.op[a];
                uint64_t r;
                if (op == A_COUNT) {
                    r = c;
                } else {
                    const unsigned long long v = G.acc[(int64_t)G.ai[a] * S + s];
                    if (op == A_AVG) {
                        const double sum = G.f[a] ? __longlong_as_double((long long)v) : (double)(long long)v;
                        r = (uint64_t)__double_as_longlong(sum / (double)c);
                    } else if ((op == A_MIN || op == A_MAX) && G.f[a]) {
                        r = (uint64_t)__double_as_longlong(ord2f((long long)v));
                    } else {
                        r = v;
                    }
                }
                ((uint64_t*)O.aggs[a])[o] = r;
            }
        }
        out += tot;
        if (base + (i + 1) * kThreads >= S) break;
    }
}

__global__ void k_scan_counts_g(int64_t* counts, int64_t m, int64_t* d_total);

// ---- workspace layout -----------------------------------------------------------------
struct Layout {
    size_t err, cnt, acc, state, keys, emit, total;
};

static size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

static Layout layout_of(int64_t S, int n_acc, int nk, int method) {
    Layout L;
    size_t o = 0;
    L.err = o; o += 256;
    L.cnt = o; o += al((size_t)S * 8);
    L.acc = o; o += al((size_t)S * 8 * n_acc);
    L.state = o; o += method == TDG_GROUP_HASH ? al((size_t)S * 4) : 0;
    L.keys = o; o += method == TDG_GROUP_HASH ? al((size_t)S * 8 * nk) : 0;
    L.emit = o; o += al((size_t)((S + kEmitChunk - 1) / kEmitChunk + 1) * 8);
    L.total = o;
    return L;
}

static int count_acc(const tdg_group_desc* d) {
    int n = 0;
    for (int a = 0; a < d->n_aggs; a++) n += d->aggs[a].op != A_COUNT;
    return n;
}

static int64_t next_pow2(int64_t x) {
    int64_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

static tdg_status validate(const tdg_group_desc* d) {
    if (d->n_keys < 0 || d->n_keys > TDG_MAX_KEYS || d->n_aggs < 0 || d->n_aggs > TDG_MAX_AGGS) return E_NYI;
    for (int k = 0; k < d->n_keys; k++)
        if (!elem_size(d->keys[k].type, d->keys[k].attrs) || elem_size(d->keys[k].type, d->keys[k].attrs) > 8)
            return E_TYPE;
    for (int a = 0; a < d->n_aggs; a++) {
        const int op = d->aggs[a].op;
        if (op != A_SUM && op != A_COUNT && op != A_MIN && op != A_MAX && op != A_AVG) return E_NYI;
        if (op != A_COUNT && !elem_size(d->aggs[a].in.type, d->aggs[a].in.attrs)) return E_TYPE;
    }
    return E_OK;
}

static tdg_status plan_group(const tdg_group_desc* d, int64_t nrows_bound, int64_t hint, tdg_group_plan* p) {
    tdg_status st = validate(d);
    if (st) return st;
    memset(p, 0, sizeof(*p));
    const int n_acc = count_acc(d);
    bool direct = d->have_range != 0;
    int64_t slots = 1;
    for (int k = 0; k < d->n_keys && direct; k++) {
        if (!is_int_class(d->keys[k].type)) { direct = false; break; }
        const int64_t lo = d->key_min[k], hi = d->key_max[k];
        if (hi < lo) { direct = false; break; }
        const uint64_t range = (uint64_t)hi - (uint64_t)lo + 1;
        if (range == 0 || range > (uint64_t)kDirectMaxSlots || slots > kDirectMaxSlots / (int64_t)range) {
            direct = false;
            break;
        }
        slots *= (int64_t)range;
    }
    const int64_t dense_cap = nrows_bound * 2 > 65536 ? nrows_bound * 2 : 65536;
    if (direct && slots > dense_cap) direct = false;
    if (direct) {
        p->method = TDG_GROUP_DIRECT;
        p->n_slots = slots;
        p->smem = (size_t)slots * 8 * (1 + n_acc) <= kSmemAccMax ? 1 : 0;
    } else {
        int64_t bound = nrows_bound > 0 ? nrows_bound : 1;
        if (hint > 0 && hint < bound) bound = hint;
        if (d->have_range) {
            uint64_t prod = 1;
            bool fits = true;
            for (int k = 0; k < d->n_keys; k++) {
                if (!is_int_class(d->keys[k].type)) { fits = false; break; }
                const uint64_t range = (uint64_t)d->key_max[k] - (uint64_t)d->key_min[k] + 1;
                if (range == 0 || prod > (uint64_t)INT64_MAX / range) { fits = false; break; }
                prod *= range;
            }
            if (fits && (int64_t)prod < bound) bound = (int64_t)prod;
        }
        p->method = TDG_GROUP_HASH;
        p->n_slots = next_pow2(bound * 2 > 1024 ? bound * 2 : 1024);
    }
    p->max_groups = p->n_slots;
    p->ws_bytes = layout_of(p->n_slots, n_acc, d->n_keys, p->method).total;
    return E_OK;
}

static GroupK make_gk(const tdg_group_desc* d, const tdg_group_plan* p, void* ws) {
    GroupK G;
    memset(&G, 0, sizeof(G));
    const int n_acc = count_acc(d);
    const Layout L = layout_of(p->n_slots, n_acc, d->n_keys, p->method);
    char* w = (char*)ws;
    G.nk = d->n_keys;
    G.na = d->n_aggs;
    G.method = p->method;
    G.n_acc = n_acc;
    G.S = p->n_slots;
    G.err = (int32_t*)(w + L.err);
    G.cnt = (unsigned long long*)(w + L.cnt);
    G.acc = (unsigned long long*)(w + L.acc);
    int64_t stride = 1;
    for (int k = d->n_keys - 1; k >= 0; k--) {
        G.key[k] = d->keys[k];
        if (p->method == TDG_GROUP_DIRECT) {
            G.kmin[k] = d->key_min[k];
            G.krange[k] = d->key_max[k] - d->key_min[k] + 1;
            G.stride[k] = stride;
            stride *= G.krange[k];
        }
    }
    int ai = 0;
    for (int a = 0; a < d->n_aggs; a++) {
        G.op[a] = d->aggs[a].op;
        G.in[a] = d->aggs[a].in;
        G.f[a] = d->aggs[a].in.type == T_F64;
        G.ai[a] = G.op[a] == A_COUNT ? -1 : ai++;
    }
    if (p->method == TDG_GROUP_HASH) {
        G.ht.state = (uint32_t*)(w + L.state);
        G.ht.keys = (int64_t*)(w + L.keys);
        G.ht.mask = (uint64_t)p->n_slots - 1;
        G.ht.nk = d->n_keys;
        G.ht.err = G.err;
    }
    return G;
}

static tdg_status prepare(const GroupK& G, const tdg_group_plan* p, cudaStream_t s) {
    cudaMemsetAsync(G.err, 0, 256, s);
    const int g = grid_for((const void*)k_group_init, kThreads, 0, G.S);
    (note_launch(), k_group_init<<<g, kThreads, 0, s>>>(G));
    (void)p;
    return launch_status();
}

static tdg_status finish(const GroupK& G, const tdg_group_desc* d, void* ws, const tdg_group_out* out,
                         cudaStream_t s) {
    const Layout L = layout_of(G.S, G.n_acc, G.nk, G.method);
    int64_t* counts = (int64_t*)((char*)ws + L.emit);
    const int64_t chunks = (G.S + kEmitChunk - 1) / kEmitChunk;
    (note_launch(), k_emit_count<<<(unsigned)chunks, kThreads, 0, s>>>(G.cnt, G.S, counts));
    (note_launch(), k_scan_counts_g<<<1, 1024, 0, s>>>(counts, chunks, out->d_n_groups));
    OutK O;
    memset(&O, 0, sizeof(O));
    for (int k = 0; k < G.nk; k++) {
        O.keys[k] = out->keys[k];
        O.kesz[k] = elem_size(d->keys[k].type, d->keys[k].attrs);
    }
    for (int a = 0; a < G.na; a++) O.aggs[a] = out->aggs[a];
    (note_launch(), k_emit<<<(unsigned)chunks, kThreads, 0, s>>>(G, O, counts));
    tdg_status st = launch_status();
    if (st) return st;
    int32_t err = 0;
    if (cudaMemcpyAsync(&err, G.err, sizeof(err), cudaMemcpyDeviceToHost, s) != cudaSuccess) return E_IO;
    if (cudaStreamSynchronize(s) != cudaSuccess) return E_IO;
    return err;
}

template <int PK, int MODE, bool JOIN>
static tdg_status launch_main(const GroupK& G, const Pred& P, const tdg_expr& prog, const JoinK& J, int64_t n,
                              cudaStream_t s) {
    const size_t smem = MODE == 0 ? (size_t)G.S * 8 * (1 + G.n_acc) : 0;
    const void* fn = (const void*)k_group<PK, MODE, JOIN>;
    const int g = grid_for(fn, kThreads, smem, (n + kItems - 1) / kItems);
    (note_launch(), k_group<PK, MODE, JOIN><<<g, kThreads, smem, s>>>(G, P, prog, J, n));
    return launch_status();
}

template <bool JOIN>
static tdg_status dispatch(int pk, const GroupK& G, bool smem, const Pred& P, const tdg_expr& prog,
                           const JoinK& J, int64_t n, cudaStream_t s) {
    const int mode = G.method == TDG_GROUP_HASH ? 2 : (smem ? 0 : 1);
#define TDG_CASE(PKV, MV) if (pk == PKV && mode == MV) return launch_main<PKV, MV, JOIN>(G, P, prog, J, n, s);
    TDG_CASE(0, 0) TDG_CASE(0, 1) TDG_CASE(0, 2)
    TDG_CASE(1, 0) TDG_CASE(1, 1) TDG_CASE(1, 2)
    TDG_CASE(2, 0) TDG_CASE(2, 1) TDG_CASE(2, 2)
#undef TDG_CASE
    return E_NYI;
}

__global__ void __launch_bounds__(1024) k_scan_counts_g(int64_t* counts, int64_t m, int64_t* d_total) {
    __shared__ long long part[1024];
    const int64_t per = (m + blockDim.x - 1) / blockDim.x;
    const int64_t b = threadIdx.x * per, e = b + per < m ? b + per : m;
    long long sum = 0;
    for (int64_t i = b; i < e; i++) sum += counts[i];
    part[threadIdx.x] = sum;
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

// ---- shared with tdg_join.cu ------------------------------------------------------
tdg_status group_run_joined(const tdg_group_desc* d, const tdg_group_plan* p, void* ws,
                            const tdg_expr* pred, const uint64_t* sel, const JoinK* J, int64_t n_left,
                            int64_t n_right, const tdg_group_out* out, cudaStream_t s) {
    if (p->method != TDG_GROUP_DIRECT && p->method != TDG_GROUP_HASH) return E_RANGE;
    GroupK G = make_gk(d, p, ws);
    tdg_status st = prepare(G, p, s);
    if (st) return st;
    int pk;
    Pred P = make_pred(pred, sel, &pk);
    static tdg_expr empty;
    const tdg_expr& prog = pred ? *pred : empty;
    EventTimer tm;
    if (J) {
        tm.start(s);
        st = dispatch<true>(pk, G, p->smem != 0, P, prog, *J, n_left, s);
        tm.stop(s);
        if (!st && J->join_type == 2 && n_right > 0) {
            const int mode = G.method == TDG_GROUP_HASH ? 2 : 1;
            const int g = grid_for((const void*)k_group_unmatched<1>, kThreads, 0, n_right);
            if (mode == 2) (note_launch(), k_group_unmatched<2><<<g, kThreads, 0, s>>>(G, *J, n_right));
            else (note_launch(), k_group_unmatched<1><<<g, kThreads, 0, s>>>(G, *J, n_right));
            st = launch_status();
        }
    } else {
        JoinK none;
        memset(&none, 0, sizeof(none));
        tm.start(s);
        st = dispatch<false>(pk, G, p->smem != 0, P, prog, none, d->nrows, s);
        tm.stop(s);
    }
    if (st) { tm.ms(); return st; }
    st = finish(G, d, ws, out, s);       // synchronizes the stream
    const float ms = tm.ms();
    if (tm.on) set_last_main_ms(ms);
    return st;
}

}  // namespace tdg

using namespace tdg;

extern "C" tdg_status tdg_group_plan_make(const tdg_group_desc* d, int64_t hint_groups, tdg_group_plan* plan) {
    if (!d || !plan) return E_TYPE;
    return plan_group(d, d->nrows, hint_groups, plan);
}

extern "C" tdg_status tdg_group_run(const tdg_group_desc* d, const tdg_expr* pred, const uint64_t* sel_in,
                                    const tdg_group_plan* plan, void* ws, const tdg_group_out* out,
                                    void* stream) {
    if (!d || !plan || !ws || !out) return E_TYPE;
    tdg_status st = validate(d);
    if (st) return st;
    return group_run_joined(d, plan, ws, pred, sel_in, nullptr, 0, 0, out, (cudaStream_t)stream);
}
