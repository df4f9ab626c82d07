// Group-by: fused selection + aggregation + emit.
//
// Replaces exec_group (Teide src/ops/exec.c:5542-6879).  The CPU engine picks
// a direct array for dense integer keys of at most 262,144 composite slots
// (exec.c:5948-6404) and otherwise a 256-way radix-partitioned hash table
// built in three phases (exec.c:6406-6667).  Here:
//
//   direct array (TDG_GROUP_DIRECT) -- slot = sum_k (key_k - min_k) * stride_k,
//     up to 2^26 slots.
//   hash table (TDG_GROUP_HASH) -- open addressing in HBM (tdg_hash.cuh), one
//     pass, no partitioning: the hot part of the table stays in the 126 MB L2.
//
// Accumulators live in three places:
//   MODE 0  every slot privatized per CTA in shared memory (32-bit counts,
//           8-byte accumulators), merged into the global records once per CTA;
//   MODE 1  direct array in global memory;
//   MODE 2  hash table in global memory;
//   MODE 3  direct array in global memory, one key, partitioned: hot slots
//           aggregate in shared memory as in MODE 1, every other row becomes
//           an entry (slot, values) of its slot range's partition, and a
//           second pass aggregates each partition in shared memory and merges
//           it into the records -- the partitioned aggregation of
//           exec.c:6406-6667 with shared memory as the per-partition table,
//           so cold rows cost streaming writes and reads instead of random or
//           contended global atomics.
// Global accumulators are slot-major records [count, acc_0, acc_1, ...] so
// one row's updates touch at most two 32-byte sectors.  In MODES 1 and 2 a
// sampling pass finds the slots that take a large share of the rows (Zipf
// heads) and every CTA caches those "hot" slots in shared memory; only cold
// slots are updated with global atomics, so a key that holds 11% of the rows
// no longer serializes on one L2 address.
//
// Every aggregate reads its input once per row; the emit pass writes the
// groups whose count is non-zero in slot order (ascending key order for the
// direct array, like Teide's DA emit at exec.c:6330-6391).  Arithmetic
// follows the CPU loops: integer SUM wraps, AVG = sum / count in double
// (exec.c:4430-4432, emit_agg_columns 4632-4773), MIN/MAX of F64 skip NaN.
// F64 SUM uses atomics, so its summation order differs from the CPU's
// per-worker order (results agree to ~1e-15 relative).
#include "tdg_hash.cuh"
#include <string.h>

namespace tdg {

// Minimum resident CTAs per SM the streaming kernels are compiled for
// (bounds their registers): 6 keeps every hot variant spill-free.
#ifndef TDG_MINB
#define TDG_MINB 6
#endif
#ifndef TDG_ITEMS
#define TDG_ITEMS 4
#endif
constexpr int kItems = TDG_ITEMS;
constexpr int kEmitChunk = kThreads * 32;
constexpr size_t kSmemMax = 48 * 1024;
constexpr int64_t kDirectMaxSlots = (int64_t)1 << 26;
constexpr int kHotMap = 2048;                 // shared hot-slot map entries (power of 2)
constexpr int kHotBuckets = kHotMap / 4;       // the map is probed four entries (16 bytes) at a time
constexpr int kHotMax = 1024;                 // at most this many hot slots
constexpr int64_t kSampleRows = (int64_t)1 << 18;
constexpr int64_t kSampleCap = (int64_t)1 << 19;
constexpr uint32_t kHotMin = 8;               // sampled hits that make a slot hot
constexpr int64_t kSampleMinRows = (int64_t)1 << 22;
constexpr int kHotHist = 1024;                // sampled-count histogram buckets (hot threshold)
// MODE 3 (partitioned cold rows)
constexpr int64_t kPartMinRows = (int64_t)1 << 20;   // smaller inputs keep MODE 1
// A partition's shared-memory table: 96 KB (2048 slots at 5 words), or 192 KB
// from kPartWideSlots slots on.  Measured on 200M Zipf rows: with 2^14 and
// 2^20 keys the partition pass aggregates dense items in the table, and the
// larger table's one CTA per SM took 3.7 -> 6.3 ms and 4.4 -> 4.5 ms; with
// 2^24 keys the items are sparse, and half as many partitions took
// 5.7 -> 5.4 ms.
constexpr size_t kPartSmem = 96 * 1024;
constexpr size_t kPartSmemWide = 192 * 1024;
constexpr int64_t kPartWideSlots = (int64_t)1 << 23;
constexpr int kPartThreads = 512;
constexpr int64_t kPartItem = 16384;          // entries per aggregation work item
constexpr int kPartRegions = 1024;            // partitions below this are split into stripes
constexpr int kPartMaxStripes = 64;
constexpr uint32_t kPartMargin = 32;          // entries every region holds beyond its estimate
constexpr int64_t kPartDense = 4;             // entries per slot below which an item skips the table

enum : int32_t { K_COUNT = 0, K_SUM_I, K_SUM_F, K_MIN_I, K_MAX_I, K_MIN_F, K_MAX_F };

// MODE 3: partition p holds slots [p << shift, (p + 1) << shift); its rows go
// to `stripes` regions (region r = p * stripes + stripe, the stripe chosen by
// the CTA) so that small partition counts do not serialize on one counter.
// Region r holds cap[r] entries from base[r]: e_slot[e] and the values
// e_val[j][e].  fill[r] counts reservations and may pass cap[r]; rows beyond
// it update the global records directly.
struct PartK {
    int32_t shift, stripes;
    int32_t ne, pad;              // values per entry
    int64_t P, R;                 // partitions, regions
    int64_t cap_total;            // entries the buffers hold
    uint32_t* est;                // [P] sampled cold rows per partition
    uint32_t* fill;               // [R]
    uint32_t* cap;                // [R]
    int64_t* base;                // [R]
    int64_t* item_start;          // [R + 1] aggregation work items per region, prefix
    int32_t* item_region;         // [R + cap_total / kPartItem + 1] region of each work item
    uint32_t* item_next;          // work-item counter
    uint32_t* e_slot;
    unsigned long long* e_val[2];
};

struct GroupK {
    int32_t nk, na, method, n_acc;
    int32_t W;                    // 8-byte words per global slot record
    int32_t hot_cap;              // hot slots a CTA caches (0: no cache)
    int32_t cps;                  // persistent CTAs per SM of the streaming kernel (0: all that fit)
    int32_t rep0;                 // MODE 0: copies of the shared table, one per warp (kThreads / 32) or 1
    tdg_col key[TDG_MAX_KEYS];
    int64_t kmin[TDG_MAX_KEYS], krange[TDG_MAX_KEYS], stride[TDG_MAX_KEYS];
    int32_t op[TDG_MAX_AGGS];
    int32_t kind[TDG_MAX_AGGS];   // K_*
    int32_t ai[TDG_MAX_AGGS];     // accumulator index, -1 for COUNT
    int32_t akind[TDG_MAX_AGGS];  // K_* of each accumulator
    tdg_col in[TDG_MAX_AGGS];
    int64_t S;
    unsigned long long* rec;      // S * W words
    unsigned long long finit[TDG_MAX_AGGS + 2];   // initial value of each record word
    HtRef ht;
    int32_t* err;                 // [0] error code, [1] duplicate build key (payload join)
    int64_t* sample_keys;
    uint32_t* sample_cnt;
    int64_t* hot;                 // hot slot list
    int32_t* hot_n;               // [0] hot slots, [1] sampled-count threshold; hot_hist follows
    uint32_t* hot_hist;           // [kHotHist] sampled slots per count
    int64_t sample_rows;          // rows the sample drew
    PartK pk;                     // MODE 3 buffers (pk.P == 0: not planned)
    PfCols pf;                    // streamed columns the main kernels prefetch into L2
};

struct OutK {
    void* keys[TDG_MAX_KEYS];
    int32_t kesz[TDG_MAX_KEYS];
    void* aggs[TDG_MAX_AGGS];
    const int32_t* err;           // the run's error word and repeated-key flag ...
    int32_t* herr;                // ... copied here (device-mapped host words) by the emit, if set
};

__device__ __forceinline__ unsigned long long* grec(const GroupK& G, int64_t s) { return G.rec + s * G.W; }

__host__ __device__ __forceinline__ unsigned long long acc_init_kind(int kind) {
    return (kind == K_MIN_I || kind == K_MIN_F) ? (unsigned long long)INT64_MAX
         : (kind == K_MAX_I || kind == K_MAX_F) ? (unsigned long long)INT64_MIN : 0ULL;
}

// ---- typed multi-row loads --------------------------------------------------
// N rows of one column (row < 0 or masked off gives 0).  The type switch runs
// once per column, so the N loads issue back to back; with W8 every column is
// 8 bytes and there is no switch at all.  Probe-side columns stream
// (evict-first); build-side columns are gathered at random and use the
// read-only path so they stay cached.
template <bool W8, int N>
__device__ __forceinline__ void ld_items_i(const tdg_col& c, const int64_t (&r)[N], const bool (&m)[N],
                                           int64_t (&v)[N]) {
#define TDG_LD(T, CONV)                                                                                   \
    {                                                                                                     \
        const T* p = (const T*)c.data;                                                                    \
        _Pragma("unroll") for (int i = 0; i < N; i++)                                                    \
            v[i] = (m[i] && r[i] >= 0) ? (int64_t)CONV(c.side ? __ldg(p + r[i]) : ld_stream(p + r[i])) : 0; \
    }
#define TDG_ID(x) (x)
    if (W8) {
        if (c.type == T_F64) TDG_LD(double, TDG_ID) else TDG_LD(long long, TDG_ID)
        return;
    }
    switch (c.type) {
        case T_I64: case T_TIMESTAMP: TDG_LD(long long, TDG_ID) break;
        case T_I32: case T_DATE: case T_TIME: TDG_LD(int, TDG_ID) break;
        case T_I16: TDG_LD(short, TDG_ID) break;
        case T_BOOL: case T_U8: case T_CHAR: TDG_LD(unsigned char, TDG_ID) break;
        case T_SYM:
            switch (c.attrs & 3) {
                case 0: TDG_LD(unsigned char, TDG_ID) break;
                case 1: TDG_LD(unsigned short, TDG_ID) break;
                case 2: TDG_LD(unsigned int, TDG_ID) break;
                default: TDG_LD(long long, TDG_ID) break;
            }
            break;
        case T_F64: TDG_LD(double, TDG_ID) break;
        default:
#pragma unroll
            for (int i = 0; i < N; i++) v[i] = 0;
    }
#undef TDG_ID
#undef TDG_LD
}

template <bool W8, int N>
__device__ __forceinline__ void ld_items_f(const tdg_col& c, const int64_t (&r)[N], const bool (&m)[N],
                                           double (&v)[N]) {
    if (c.type == T_F64) {
        const double* p = (const double*)c.data;
#pragma unroll
        for (int i = 0; i < N; i++)
            v[i] = (m[i] && r[i] >= 0) ? (c.side ? __ldg(p + r[i]) : ld_stream(p + r[i])) : 0.0;
    } else {
        int64_t t[N];
        ld_items_i<W8, N>(c, r, m, t);
#pragma unroll
        for (int i = 0; i < N; i++) v[i] = (double)t[i];
    }
}

// Accumulator updates.  Sums are fire-and-forget reductions; a global MIN/MAX
// first reads the current value and skips the atomic when it cannot change,
// which after the first rows of a group is almost always.
template <bool GL>
__device__ __forceinline__ void upd_min(unsigned long long* a, long long v) {
    // the L2 read (ld.global.cg) is only a filter: the stored extreme only
    // moves toward v, so a stale read can cost an extra atomic, never a lost one
    if (!GL || v < __ldcg((const long long*)a)) atomicMin((long long*)a, v);
}
template <bool GL>
__device__ __forceinline__ void upd_max(unsigned long long* a, long long v) {
    if (!GL || v > __ldcg((const long long*)a)) atomicMax((long long*)a, v);
}

// Merge one accumulator value (already in accumulator form) into another.
__device__ __forceinline__ void merge(unsigned long long* a, int kind, unsigned long long v) {
    switch (kind) {
        case K_SUM_I: atomicAdd(a, v); break;
        case K_SUM_F: atomicAdd((double*)a, __longlong_as_double((long long)v)); break;
        case K_MIN_I: case K_MIN_F:
            if ((long long)v != INT64_MAX) atomicMin((long long*)a, (long long)v);
            break;
        case K_MAX_I: case K_MAX_F:
            if ((long long)v != INT64_MIN) atomicMax((long long*)a, (long long)v);
            break;
        default: break;
    }
}

// Slot of each (probe row, build row) pair; -1 when masked off or on error.
template <int MODE, bool W8, int N>
__device__ __forceinline__ void slots_of(const GroupK& G, const int64_t (&rp)[N], const int64_t (&rb)[N],
                                         const bool (&m)[N], int64_t (&slot)[N]) {
    if (MODE != 2) {
        bool ok[N];
#pragma unroll
        for (int i = 0; i < N; i++) { slot[i] = 0; ok[i] = m[i]; }
        for (int k = 0; k < G.nk; k++) {
            int64_t v[N];
            ld_items_i<W8, N>(G.key[k], G.key[k].side ? rb : rp, m, v);
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

// ---- shared-memory accumulators -----------------------------------------------------
// MODE 0: cnt[S] (32-bit) then acc[n_acc][S].
// MODES 1/2: a map from hot slot to cache index, then cnt[hot_cap] and
// acc[n_acc][hot_cap].
struct SmemView {
    uint32_t* cnt;
    unsigned long long* acc;
    int64_t cap;        // entries per array
    int32_t* map_key;   // hot slot, -1 empty
    int16_t* map_idx;
    int n_hot;
};

__host__ __device__ inline size_t smem_full_bytes(int64_t S, int n_acc) {
    return (((size_t)S * 4 + 7) & ~(size_t)7) + (size_t)S * 8 * n_acc;
}
__host__ __device__ inline size_t smem_hot_bytes(int hot_cap, int n_acc) {
    return (size_t)kHotMap * 4 + (size_t)kHotMap * 2 + (((size_t)hot_cap * 4 + 7) & ~(size_t)7) +
           (size_t)hot_cap * 8 * n_acc;
}

// Bucket of a hot slot: the MurmurHash3 32-bit finalizer, so structured key
// sets (strided or multiplicative ones) spread evenly -- a warp waits for its
// longest probe, so clustering costs far more than its average suggests.
__host__ __device__ __forceinline__ uint32_t hot_bucket(int64_t slot) {
    uint32_t x = (uint32_t)slot;
    x ^= x >> 16;
    x *= 0x85ebca6bu;
    x ^= x >> 13;
    x *= 0xc2b2ae35u;
    x ^= x >> 16;
    return x & (kHotBuckets - 1);
}

// Linear probing over the map in bucket order, a key inserted from the start
// of its bucket: one 16-byte load answers a lookup unless the bucket is full.
__device__ __forceinline__ int hot_find(const SmemView& V, int64_t slot) {
    const int32_t key = (int32_t)slot;
    uint32_t b = hot_bucket(slot);
    for (int t = 0; t < kHotBuckets; t++) {
        const int4 k = *reinterpret_cast<const int4*>(V.map_key + 4 * b);
        if (k.x == key) return V.map_idx[4 * b];
        if (k.y == key) return V.map_idx[4 * b + 1];
        if (k.z == key) return V.map_idx[4 * b + 2];
        if (k.w == key) return V.map_idx[4 * b + 3];
        if ((k.x == -1) | (k.y == -1) | (k.z == -1) | (k.w == -1)) return -1;
        b = (b + 1) & (kHotBuckets - 1);
    }
    return -1;
}

template <int MODE>
__device__ SmemView smem_setup(const GroupK& G, unsigned long long* sm) {
    SmemView V;
    V.cnt = nullptr;
    V.acc = nullptr;
    V.cap = 0;
    V.map_key = nullptr;
    V.map_idx = nullptr;
    V.n_hot = 0;
    if (MODE == 0) {
        // one copy of the table per warp when rep0 > 1: a few dozen slots
        // updated by all 256 threads of a CTA otherwise serialize on the same
        // shared addresses; the copies are summed at the flush
        V.cap = G.S;
        const size_t words = smem_full_bytes(G.S, G.n_acc) >> 3;
        unsigned long long* base = sm + (G.rep0 > 1 ? (size_t)(threadIdx.x >> 5) * words : 0);
        V.cnt = (uint32_t*)base;
        V.acc = base + ((G.S * 4 + 7) >> 3);
        if (G.rep0 > 1) {
            for (int64_t i = threadIdx.x; i < (int64_t)G.rep0 * G.S; i += blockDim.x) {
                unsigned long long* cb = sm + (size_t)(i / G.S) * words;
                const int64_t k = i % G.S;
                ((uint32_t*)cb)[k] = 0;
                for (int a = 0; a < G.na; a++)
                    if (G.ai[a] >= 0) (cb + ((G.S * 4 + 7) >> 3))[(int64_t)G.ai[a] * G.S + k] = acc_init_kind(G.kind[a]);
            }
            __syncthreads();
            return V;
        }
    } else {
        V.cap = G.hot_cap;
        if (!G.hot_cap) return V;
        V.map_key = (int32_t*)sm;
        V.map_idx = (int16_t*)(V.map_key + kHotMap);
        V.cnt = (uint32_t*)(V.map_idx + kHotMap);
        V.acc = (unsigned long long*)((char*)V.cnt + (((size_t)G.hot_cap * 4 + 7) & ~(size_t)7));
        const int nh = *G.hot_n;
        V.n_hot = nh < G.hot_cap ? nh : G.hot_cap;
        for (int i = threadIdx.x; i < kHotMap; i += blockDim.x) V.map_key[i] = -1;
        __syncthreads();
        for (int h = threadIdx.x; h < V.n_hot; h += blockDim.x) {
            const int32_t slot = (int32_t)G.hot[h];
            uint32_t p = 4 * hot_bucket(slot);
            for (int t = 0; t < kHotMap; t++) {
                if (atomicCAS(&V.map_key[p], -1, slot) == -1) { V.map_idx[p] = (int16_t)h; break; }
                p = (p + 1) & (kHotMap - 1);
            }
        }
    }
    const int64_t n = MODE == 0 ? G.S : V.n_hot;
    for (int64_t s = threadIdx.x; s < n; s += blockDim.x) V.cnt[s] = 0;
    for (int a = 0; a < G.na; a++) {
        if (G.ai[a] < 0) continue;
        const unsigned long long init = acc_init_kind(G.kind[a]);
        for (int64_t s = threadIdx.x; s < n; s += blockDim.x) V.acc[(int64_t)G.ai[a] * V.cap + s] = init;
    }
    __syncthreads();
    return V;
}

template <int MODE>
__device__ void smem_flush(const GroupK& G, const SmemView& V) {
    __syncthreads();
    if (MODE == 0 && G.rep0 > 1) {
        // the warps' copies summed per slot, then one merge into the record
        extern __shared__ unsigned long long sm_base[];
        const size_t words = smem_full_bytes(G.S, G.n_acc) >> 3;
        for (int64_t s = threadIdx.x; s < G.S; s += blockDim.x) {
            uint32_t c = 0;
            for (int w = 0; w < G.rep0; w++) c += ((const uint32_t*)(sm_base + (size_t)w * words))[s];
            if (!c) continue;
            unsigned long long* r = grec(G, s);
            atomicAdd(r, (unsigned long long)c);
            for (int a = 0; a < G.na; a++) {
                if (G.ai[a] < 0) continue;
                const int kind = G.kind[a];
                unsigned long long x = acc_init_kind(kind);
                for (int w = 0; w < G.rep0; w++) {
                    const unsigned long long y =
                        (sm_base + (size_t)w * words + ((G.S * 4 + 7) >> 3))[(int64_t)G.ai[a] * G.S + s];
                    switch (kind) {
                        case K_SUM_F:
                            x = (unsigned long long)__double_as_longlong(__longlong_as_double((long long)x) +
                                                                         __longlong_as_double((long long)y));
                            break;
                        case K_SUM_I: x += y; break;
                        case K_MIN_I: case K_MIN_F: if ((long long)y < (long long)x) x = y; break;
                        case K_MAX_I: case K_MAX_F: if ((long long)y > (long long)x) x = y; break;
                        default: break;
                    }
                }
                merge(r + 1 + G.ai[a], kind, x);
            }
        }
        return;
    }
    const int64_t n = MODE == 0 ? G.S : V.n_hot;
    for (int64_t s = threadIdx.x; s < n; s += blockDim.x) {
        const uint32_t c = V.cnt[s];
        if (!c) continue;
        const int64_t slot = MODE == 0 ? s : G.hot[s];
        unsigned long long* r = grec(G, slot);
        atomicAdd(r, (unsigned long long)c);
        for (int a = 0; a < G.na; a++)
            if (G.ai[a] >= 0) merge(r + 1 + G.ai[a], G.kind[a], V.acc[(int64_t)G.ai[a] * V.cap + s]);
    }
}

// Aggregate N rows whose slots are known (slot < 0 or !m[i]: skipped).
template <int MODE, bool W8, int N>
__device__ __forceinline__ void accumulate_at(const GroupK& G, const SmemView& V, const int64_t (&rp)[N],
                                              const int64_t (&rb)[N], const int64_t (&slot)[N], const bool (&m)[N]) {
    bool ok[N];
    int hidx[N];
#pragma unroll
    for (int i = 0; i < N; i++) {
        ok[i] = m[i] && slot[i] >= 0;
        hidx[i] = -1;
        if (MODE == 0) hidx[i] = ok[i] ? (int)slot[i] : -1;
        else if (V.n_hot && ok[i]) hidx[i] = hot_find(V, slot[i]);
        // a cold record's line is fetched now, so the N rows' DRAM round trips
        // overlap instead of queueing behind the MIN/MAX filter reads below
        if (MODE != 0 && ok[i] && hidx[i] < 0)
            asm volatile("{\n\t.reg .u64 g;\n\tcvta.to.global.u64 g, %0;\n\tprefetch.global.L2 [g];\n\t}"
                         :: "l"(grec(G, slot[i])));
        if (ok[i]) {
            if (hidx[i] >= 0) atomicAdd(&V.cnt[hidx[i]], 1u);
            else atomicAdd(grec(G, slot[i]), 1ULL);
        }
    }
    // one dispatch per aggregate, then a straight loop over the N rows
#define TDG_TARGET(i) (hidx[i] >= 0 ? V.acc + (int64_t)ai * V.cap + hidx[i] : grec(G, slot[i]) + 1 + ai)
    for (int a = 0; a < G.na; a++) {
        const int kind = G.kind[a];
        if (kind == K_COUNT) continue;
        const int ai = G.ai[a];
        const tdg_col& c = G.in[a];
        const int64_t (&rr)[N] = c.side ? rb : rp;
        if (kind == K_SUM_F || kind == K_MIN_F || kind == K_MAX_F) {
            double v[N];
            ld_items_f<W8, N>(c, rr, ok, v);
            if (kind == K_SUM_F) {
#pragma unroll
                for (int i = 0; i < N; i++) if (ok[i]) atomicAdd((double*)TDG_TARGET(i), v[i]);
            } else if (kind == K_MIN_F) {
#pragma unroll
                for (int i = 0; i < N; i++)
                    if (ok[i] && v[i] == v[i]) {
                        if (hidx[i] >= 0) upd_min<false>(TDG_TARGET(i), f2ord(v[i]));
                        else upd_min<true>(TDG_TARGET(i), f2ord(v[i]));
                    }
            } else {
#pragma unroll
                for (int i = 0; i < N; i++)
                    if (ok[i] && v[i] == v[i]) {
                        if (hidx[i] >= 0) upd_max<false>(TDG_TARGET(i), f2ord(v[i]));
                        else upd_max<true>(TDG_TARGET(i), f2ord(v[i]));
                    }
            }
        } else {
            int64_t v[N];
            ld_items_i<W8, N>(c, rr, ok, v);
            if (kind == K_SUM_I) {
#pragma unroll
                for (int i = 0; i < N; i++) if (ok[i]) atomicAdd(TDG_TARGET(i), (unsigned long long)v[i]);
            } else if (kind == K_MIN_I) {
#pragma unroll
                for (int i = 0; i < N; i++)
                    if (ok[i]) {
                        if (hidx[i] >= 0) upd_min<false>(TDG_TARGET(i), v[i]);
                        else upd_min<true>(TDG_TARGET(i), v[i]);
                    }
            } else {
#pragma unroll
                for (int i = 0; i < N; i++)
                    if (ok[i]) {
                        if (hidx[i] >= 0) upd_max<false>(TDG_TARGET(i), v[i]);
                        else upd_max<true>(TDG_TARGET(i), v[i]);
                    }
            }
        }
    }
#undef TDG_TARGET
}

template <int MODE, bool W8, int N>
__device__ __forceinline__ void accumulate(const GroupK& G, const SmemView& V, const int64_t (&rp)[N],
                                           const int64_t (&rb)[N], const bool (&m)[N]) {
    int64_t slot[N];
    slots_of<MODE, W8, N>(G, rp, rb, m, slot);
    accumulate_at<MODE, W8, N>(G, V, rp, rb, slot, m);
}

// The main kernel.  JOIN: probe rows are joined through J first and every
// (probe, build) match is one input row of the group-by.
template <int PK, int MODE, bool JOIN, bool W8>
__global__ void __launch_bounds__(kThreads, TDG_MINB) k_group(const GroupK G, const Pred P, const tdg_expr prog,
                                                    const JoinK J, int64_t n) {
    extern __shared__ unsigned long long sm[];
    const SmemView V = smem_setup<MODE>(G, sm);
    const int64_t tile = (int64_t)kThreads * kItems;
    for (int64_t base = (int64_t)blockIdx.x * tile; base < n; base += (int64_t)gridDim.x * tile) {
        const int64_t nb = base + (int64_t)gridDim.x * tile;        // this CTA's next tile
        prefetch_rows(G.pf, nb, nb + tile < n ? nb + tile : n);
        int64_t rp[kItems], rb[kItems];
        bool m[kItems];
#pragma unroll
        for (int i = 0; i < kItems; i++) {
            rp[i] = base + i * kThreads + threadIdx.x;
            rb[i] = -1;
            m[i] = rp[i] < n && row_pass<PK, W8>(P, prog, rp[i]);
        }
        if (JOIN) {
#pragma unroll
            for (int i = 0; i < kItems; i++) {
                if (m[i]) rb[i] = join_first(J, rp[i]);
                if (J.join_type == 0) m[i] = m[i] && rb[i] >= 0;
                if (J.matched && rb[i] >= 0) J.matched[rb[i]] = 1;
            }
        }
        accumulate<MODE, W8, kItems>(G, V, rp, rb, m);
        if (JOIN) {
            // further matches of duplicate build keys
            for (int i = 0; i < kItems; i++) {
                if (!m[i] || rb[i] < 0) continue;
                int32_t nb = __ldg(&J.next[rb[i]]);
                while (nb >= 0) {
                    int64_t p1[1] = {rp[i]}, b1[1] = {nb};
                    bool m1[1] = {true};
                    if (J.matched) J.matched[nb] = 1;
                    accumulate<MODE, W8, 1>(G, V, p1, b1, m1);
                    nb = __ldg(&J.next[nb]);
                }
            }
        }
    }
    if (MODE == 0 || V.n_hot) smem_flush<MODE>(G, V);
}

// ---- hot-slot sampling (MODES 1 and 2) ---------------------------------------------
// Rows at a fixed stride go through the same selection, join and slot
// computation as the main kernel; their slots are counted in a small hash
// table, and slots seen at least kHotMin times become the hot list.
template <int PK, int MODE, bool JOIN>
__global__ void __launch_bounds__(kThreads) k_sample(const GroupK G, const Pred P, const tdg_expr prog,
                                                     const JoinK J, int64_t n, int64_t step, int64_t m_rows) {
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m_rows; j += (int64_t)gridDim.x * blockDim.x) {
        int64_t rp[1] = {j * step}, rb[1] = {-1}, slot[1];
        bool m[1] = {rp[0] < n && row_pass<PK>(P, prog, rp[0])};
        if (JOIN && m[0]) {
            rb[0] = join_first(J, rp[0]);
            if (J.join_type == 0) m[0] = rb[0] >= 0;
        }
        slots_of<MODE, false, 1>(G, rp, rb, m, slot);
        if (!m[0] || slot[0] < 0) continue;
        uint64_t h = mix64((uint64_t)slot[0]) & (uint64_t)(kSampleCap - 1);
        for (int64_t t = 0; t < kSampleCap; t++) {
            const unsigned long long prev = atomicCAS((unsigned long long*)&G.sample_keys[h], ~0ULL,
                                                      (unsigned long long)slot[0]);
            if (prev == ~0ULL || prev == (unsigned long long)slot[0]) { atomicAdd(&G.sample_cnt[h], 1u); break; }
            h = (h + 1) & (uint64_t)(kSampleCap - 1);
        }
    }
}

// Histogram of the sampled slots by how often they were drawn.
__global__ void __launch_bounds__(kThreads) k_hot_hist(const GroupK G) {
    __shared__ uint32_t h[kHotHist];
    for (int i = threadIdx.x; i < kHotHist; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < kSampleCap; e += (int64_t)gridDim.x * blockDim.x) {
        if (G.sample_keys[e] == -1) continue;
        const uint32_t c = G.sample_cnt[e];
        atomicAdd(&h[c < (uint32_t)kHotHist ? c : kHotHist - 1], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kHotHist; i += blockDim.x) if (h[i]) atomicAdd(&G.hot_hist[i], h[i]);
}

// The hot threshold: the smallest count (at least kHotMin) whose slots --
// every slot drawn at least that often -- fit one CTA's cache, so the cache
// holds the most frequent slots.  hot_n[1] = kHotHist: no slot is hot.
__global__ void __launch_bounds__(kHotHist) k_hot_threshold(const GroupK G) {
    __shared__ uint32_t sfx[kHotHist];                 // slots drawn at least c times
    const int c = threadIdx.x;
    sfx[c] = G.hot_hist[c];
    __syncthreads();
    for (int off = 1; off < kHotHist; off <<= 1) {
        const uint32_t v = c + off < kHotHist ? sfx[c + off] : 0u;
        __syncthreads();
        sfx[c] += v;
        __syncthreads();
    }
    if (c == 0) G.hot_n[1] = kHotHist;
    __syncthreads();
    const uint32_t cap = (uint32_t)G.hot_cap;
    if (c >= (int)kHotMin && sfx[c] <= cap && (c == (int)kHotMin || sfx[c - 1] > cap)) G.hot_n[1] = c;
}

// Slots at or above the threshold become the hot list; with MODE 3 planned,
// every other sampled slot's draws count toward its partition's estimate.
__global__ void __launch_bounds__(kThreads) k_select_hot(const GroupK G) {
    const uint32_t t = (uint32_t)G.hot_n[1];
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < kSampleCap; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = G.sample_keys[e];
        if (k == -1) continue;
        const uint32_t c = G.sample_cnt[e] < (uint32_t)kHotHist ? G.sample_cnt[e] : kHotHist - 1;
        if (c >= t) {
            const int i = atomicAdd(G.hot_n, 1);
            if (i < kHotMax) G.hot[i] = k;
        } else if (G.pk.P) {
            atomicAdd(&G.pk.est[k >> G.pk.shift], G.sample_cnt[e]);
        }
    }
}

// ---- payload join -> group ---------------------------------------------------------
// When the build side has unique, dense integer join keys and the group-by
// is a direct array whose aggregate inputs all come from the probe side, the
// build pass stores in map[key - kmin] the build row's share of the group
// slot (sum over build-side group keys of (key - min) * stride), or EMPTY.
// The probe then needs one 4-byte random read per row -- a 10M-row build side
// is a 40 MB map that stays in L2 -- instead of the head[] lookup plus the
// build-column gather.
template <typename PT> struct Empty;
template <> struct Empty<uint32_t> { static constexpr uint32_t v = 0xFFFFFFFFu; };

template <typename PT>
__global__ void __launch_bounds__(kThreads) k_payload_build(const GroupK G, const JoinK J, PT* map,
                                                            int64_t n_right, int32_t* dup) {
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n_right;
         r += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = ld_i(J.rkeys[0], r) - J.kmin;
        if (k < 0 || k >= J.n_slots) { set_err(G.err, E_DOMAIN); continue; }
        int64_t s = 0;
        bool ok = true;
        for (int kk = 0; kk < G.nk; kk++) {
            if (!G.key[kk].side) continue;
            const int64_t d = ld_i(G.key[kk], r) - G.kmin[kk];
            ok = ok && d >= 0 && d < G.krange[kk];
            s += d * G.stride[kk];
        }
        if (!ok) { set_err(G.err, E_DOMAIN); continue; }
        const PT old = atomicCAS(map + k, Empty<PT>::v, (PT)s);
        if (old != Empty<PT>::v) atomicExch(dup, 1);
    }
}

// The common build shape -- an 8-byte join key and one 8-byte group key on
// the build side, both 16-byte aligned -- four rows per thread: two 16-byte
// loads per column, then four independent map writes in flight at once.
// STORE (the key range holds exactly as many slots as there are build rows):
// plain stores, since then the keys are distinct exactly when every slot is
// written, which k_map_holes checks afterwards; otherwise a CAS per key both
// stores the slot and detects a repeated key.
template <bool STORE>
__global__ void __launch_bounds__(kThreads) k_payload_build_vec(const long long* __restrict__ jk,
                                                                const long long* __restrict__ gk, int64_t jmin,
                                                                int64_t n_slots, int64_t gmin, int64_t grange,
                                                                int64_t gstride, uint32_t* map, int64_t n,
                                                                int32_t* err, int32_t* dup) {
    const int64_t step = (int64_t)gridDim.x * blockDim.x * 4;
    for (int64_t r0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4; r0 < n; r0 += step) {
        long long k[4], g[4];
        if (r0 + 3 < n) {
            const longlong2 a = __ldcs((const longlong2*)(jk + r0)), b = __ldcs((const longlong2*)(jk + r0 + 2));
            const longlong2 c = __ldcs((const longlong2*)(gk + r0)), d = __ldcs((const longlong2*)(gk + r0 + 2));
            k[0] = a.x; k[1] = a.y; k[2] = b.x; k[3] = b.y;
            g[0] = c.x; g[1] = c.y; g[2] = d.x; g[3] = d.y;
        } else {
#pragma unroll
            for (int i = 0; i < 4; i++) {
                k[i] = r0 + i < n ? jk[r0 + i] : 0;
                g[i] = r0 + i < n ? gk[r0 + i] : 0;
            }
        }
        uint32_t old[4];
        bool on[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int64_t kk = k[i] - jmin, d = g[i] - gmin;
            on[i] = r0 + i < n;
            if (on[i] && (kk < 0 || kk >= n_slots || d < 0 || d >= grange)) { set_err(err, E_DOMAIN); on[i] = false; }
            if (STORE) {
                if (on[i]) map[kk] = (uint32_t)(d * gstride);
                old[i] = 0xFFFFFFFFu;
            } else {
                old[i] = on[i] ? atomicCAS(map + kk, 0xFFFFFFFFu, (uint32_t)(d * gstride)) : 0xFFFFFFFFu;
            }
        }
        if (!STORE && (old[0] & old[1] & old[2] & old[3]) != 0xFFFFFFFFu) atomicExch(dup, 1);
    }
}

// After a STORE build: an empty entry means some key was written twice (n
// keys into n slots), so the repeated-key flag is raised.  16-byte loads; the
// map was just written and is read from L2.
__global__ void __launch_bounds__(kThreads) k_map_holes(const uint32_t* __restrict__ map, int64_t n, int32_t* dup) {
    bool hole = false;
    const int64_t n4 = n >> 2;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n4; i += (int64_t)gridDim.x * blockDim.x) {
        const uint4 v = ((const uint4*)map)[i];
        hole |= v.x == 0xFFFFFFFFu || v.y == 0xFFFFFFFFu ||
                v.z == 0xFFFFFFFFu || v.w == 0xFFFFFFFFu;
    }
    if (blockIdx.x == 0 && (int64_t)threadIdx.x < (n & 3)) hole |= map[(n4 << 2) + threadIdx.x] == 0xFFFFFFFFu;
    if (__syncthreads_or(hole) && threadIdx.x == 0) atomicExch(dup, 1);
}

// Returns 1 when a plain-store build left its empty-entry check to the
// caller (defer_holes: the vector probe scans the map as it starts), else 0.
static int launch_payload_build(const GroupK& G, const JoinK& J, uint32_t* map, int64_t n_right, cudaStream_t s,
                                bool defer_holes = false) {
    int gi = -1, nb = 0;
    for (int k = 0; k < G.nk; k++)
        if (G.key[k].side) { gi = k; nb++; }
    const bool vec = nb == 1 && J.nk == 1 && elem_size(J.rkeys[0].type, J.rkeys[0].attrs) == 8 &&
                     J.rkeys[0].type != T_F64 && elem_size(G.key[gi].type, G.key[gi].attrs) == 8 &&
                     (((uintptr_t)J.rkeys[0].data | (uintptr_t)G.key[gi].data) & 15) == 0;
    if (vec) {
        const bool store = J.n_slots == n_right && ((uintptr_t)map & 15) == 0;
        const void* k = store ? (const void*)k_payload_build_vec<true> : (const void*)k_payload_build_vec<false>;
        const int g = grid_for(k, kThreads, 0, (n_right + 3) / 4);
        if (store)
            (note_launch(), k_payload_build_vec<true><<<g, kThreads, 0, s>>>(
                (const long long*)J.rkeys[0].data, (const long long*)G.key[gi].data, J.kmin, J.n_slots, G.kmin[gi],
                G.krange[gi], G.stride[gi], map, n_right, G.err, G.err + 1));
        else
            (note_launch(), k_payload_build_vec<false><<<g, kThreads, 0, s>>>(
                (const long long*)J.rkeys[0].data, (const long long*)G.key[gi].data, J.kmin, J.n_slots, G.kmin[gi],
                G.krange[gi], G.stride[gi], map, n_right, G.err, G.err + 1));
        if (store && defer_holes) return 1;
        if (store) {
            const int gh = grid_for((const void*)k_map_holes, kThreads, 0, (J.n_slots + 3) / 4);
            (note_launch(), k_map_holes<<<gh, kThreads, 0, s>>>(map, J.n_slots, G.err + 1));
        }
    } else {
        const int g = grid_for((const void*)k_payload_build<uint32_t>, kThreads, 0, n_right);
        (note_launch(), k_payload_build<uint32_t><<<g, kThreads, 0, s>>>(G, J, map, n_right, G.err + 1));
    }
    return 0;
}

static void launch_map_holes(const GroupK& G, const uint32_t* map, int64_t n_slots, cudaStream_t s) {
    const int gh = grid_for((const void*)k_map_holes, kThreads, 0, (n_slots + 3) / 4);
    (note_launch(), k_map_holes<<<gh, kThreads, 0, s>>>(map, n_slots, G.err + 1));
}

template <int PK, bool SMEM, typename PT, bool W8>
__global__ void __launch_bounds__(kThreads, TDG_MINB) k_payload_probe(const GroupK G, const Pred P, const tdg_expr prog,
                                                            const tdg_col lkey, int64_t kmin, int64_t n_map,
                                                            const PT* __restrict__ map, int64_t n) {
    extern __shared__ unsigned long long sm[];
    constexpr int MODE = SMEM ? 0 : 1;
    const SmemView V = smem_setup<MODE>(G, sm);
    const int64_t tile = (int64_t)kThreads * kItems;
    for (int64_t base = (int64_t)blockIdx.x * tile; base < n; base += (int64_t)gridDim.x * tile) {
        const int64_t nb = base + (int64_t)gridDim.x * tile;        // this CTA's next tile
        prefetch_rows(G.pf, nb, nb + tile < n ? nb + tile : n);
        int64_t rp[kItems], rb[kItems], kv[kItems], slot[kItems];
        bool m[kItems];
#pragma unroll
        for (int i = 0; i < kItems; i++) {
            rp[i] = base + i * kThreads + threadIdx.x;
            rb[i] = -1;
            m[i] = rp[i] < n && row_pass<PK, W8>(P, prog, rp[i]);
        }
        ld_items_i<W8, kItems>(lkey, rp, m, kv);
#pragma unroll
        for (int i = 0; i < kItems; i++) {
            const int64_t k = kv[i] - kmin;
            const bool in = m[i] && k >= 0 && k < n_map;
            const PT pl = in ? __ldg(map + k) : Empty<PT>::v;
            m[i] = pl != Empty<PT>::v;
            slot[i] = m[i] ? (int64_t)pl : -1;
        }
        for (int kk = 0; kk < G.nk; kk++) {       // probe-side share of the slot
            if (G.key[kk].side) continue;
            int64_t v[kItems];
            ld_items_i<W8, kItems>(G.key[kk], rp, m, v);
#pragma unroll
            for (int i = 0; i < kItems; i++) {
                const int64_t d = v[i] - G.kmin[kk];
                if (m[i] && (d < 0 || d >= G.krange[kk])) { set_err(G.err, E_DOMAIN); m[i] = false; }
                slot[i] += d * G.stride[kk];
            }
        }
        accumulate_at<MODE, W8, kItems>(G, V, rp, rb, slot, m);
    }
    if (MODE == 0 || V.n_hot) smem_flush<MODE>(G, V);
}

// The vector form.  For the common shapes (8-byte columns aligned to 16
// bytes, at most two predicate terms, at most two distinct columns read
// besides the key -- a column that is both filtered and aggregated is read
// once) each thread owns two pairs of adjacent rows and loads every column it
// needs for them up front with 16-byte loads: nothing waits for the
// predicate, so a tile costs one memory round trip (two for the join probe,
// whose map gather depends on the key).  It serves
//   k_probe_vec        the fused join probe (slot from the payload map);
//   k_group_vec<0>     a one-key group-by with shared-memory accumulators;
//   k_group_vec<1>     a one-key group-by over the global record array, with
//                      the CTA's cache of sampled hot slots in shared memory.
// Column choices are bit masks (bit k set: the second column), so kernels
// never index a parameter array at run time -- that would copy the struct
// to local memory.
struct VecAgg {
    uint32_t vsel;               // bit a: aggregate a reads the second loaded column
    uint32_t tsel;               // bit t: predicate term t reads the second loaded column
    uint32_t esel;               // bit j: MODE 3 entry value j is the second loaded column
    uint32_t asel;               // bit a: aggregate a reads MODE 3 entry value 1
    int32_t ne, pad;             // MODE 3 values per entry
    tdg_col vc[2];               // the distinct columns read besides the key
};

__device__ __forceinline__ void ld_pair(const tdg_col& c, int64_t r, int64_t n, long long& a, long long& b) {
    const long long* p = (const long long*)c.data;
    if (r + 1 < n) {
        const longlong2 v = __ldcs((const longlong2*)p + (r >> 1));
        a = v.x;
        b = v.y;
    } else {
        a = r < n ? __ldcs(p + r) : 0;
        b = 0;
    }
}

// Reductions on the shared window by address: always the shared-memory
// atomic unit, whatever the compiler can prove about a pointer.
__device__ __forceinline__ void sh_add_u32(uint32_t a, uint32_t v) {
    asm volatile("red.shared.add.u32 [%0], %1;" :: "r"(a), "r"(v) : "memory");
}
__device__ __forceinline__ void sh_add_u64(uint32_t a, unsigned long long v) {
    asm volatile("red.shared.add.u64 [%0], %1;" :: "r"(a), "l"(v) : "memory");
}
__device__ __forceinline__ void sh_add_f64(uint32_t a, double v) {
    asm volatile("red.shared.add.f64 [%0], %1;" :: "r"(a), "d"(v) : "memory");
}
__device__ __forceinline__ void sh_min_s64(uint32_t a, long long v) {
    asm volatile("red.shared.min.s64 [%0], %1;" :: "r"(a), "l"(v) : "memory");
}
__device__ __forceinline__ void sh_max_s64(uint32_t a, long long v) {
    asm volatile("red.shared.max.s64 [%0], %1;" :: "r"(a), "l"(v) : "memory");
}
__device__ __forceinline__ long long sh_ld_s64(uint32_t a) {
    long long v;
    asm volatile("ld.shared.s64 %0, [%1];" : "=l"(v) : "r"(a) : "memory");
    return v;
}

// Column c of row i.  The two candidates pass through an empty asm first, so
// the choice is a register select: folded into an indexed load it would put
// the whole column array in local memory.
template <int NC>
__device__ __forceinline__ long long vec_pick(const long long (&cv)[NC > 0 ? NC : 1][4], int c, int i) {
    if (NC < 2) return cv[0][i];
    long long a = cv[0][i], b = cv[NC > 1 ? 1 : 0][i];
    asm("" : "+l"(a), "+l"(b));
    return c == 1 ? b : a;
}

// One tile of 4 * kThreads rows.  MAP: the key indexes the join's payload
// map, whose entry is the slot; otherwise slot = key - key_min.  MODE 0:
// every slot has shared-memory accumulators; MODE 1: hot slots do, the rest
// update the global records.
// A payload-map entry, read through L2 with the evict-last policy `pol`:
// the map is the one structure the probe re-reads, so the streamed columns
// (evict-first) should leave before it does.
__device__ __forceinline__ uint32_t ld_map(const uint32_t* p, uint64_t pol) {
    uint32_t v;
    asm volatile("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ uint64_t evict_last_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// The four rows of a thread once their key (fk) and value columns (cv) are
// in registers (vec_stream loads them): predicate, slot, and the aggregate
// updates.
template <int NT, int NC, int MODE, bool MAP, typename PT>
__device__ __forceinline__ void vec_rows(const GroupK& G, const SmemView& V, const Pred& P, const VecAgg& A,
                                         const int64_t (&row)[4], const long long (&fk)[4],
                                         const long long (&cv)[NC > 0 ? NC : 1][4], int64_t kmin, int64_t n_map,
                                         const PT* __restrict__ map, int64_t n, uint64_t pol) {
    int64_t slot[4];
    int hidx[4];
    bool ok[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        bool m = row[i] < n;
#pragma unroll
        for (int t = 0; t < NT; t++) {
            const Term& T = P.t[t];
            const long long x = vec_pick<NC>(cv, (A.tsel >> t) & 1, i);
            bool b;
            if (T.f) {
                const double v = __longlong_as_double(x);
                b = (v >= __longlong_as_double(T.lo)) & (v <= __longlong_as_double(T.hi));
            } else {
                b = (x >= T.lo) & (x <= T.hi);
            }
            m = m && (b != (bool)T.neg);
        }
        const int64_t k = fk[i] - kmin;
        if (MAP) {
            const bool in = m && k >= 0 && k < n_map;
            const uint32_t pl = in ? ld_map(map + k, pol) : (uint32_t)Empty<PT>::v;
            ok[i] = pl != (uint32_t)Empty<PT>::v;
            slot[i] = pl;
        } else {
            const bool in = k >= 0 && k < n_map;
            if (m && !in) set_err(G.err, E_DOMAIN);
            ok[i] = m && in;
            slot[i] = k;
        }
        hidx[i] = MODE == 0 ? (int)slot[i] : -1;
        if (MODE != 0 && ok[i]) {
            if (V.n_hot) hidx[i] = hot_find(V, slot[i]);
            // a cold record's line is fetched now, so the four rows' DRAM
            // round trips overlap
            if (MODE == 1 && hidx[i] < 0)
                asm volatile("{\n\t.reg .u64 g;\n\tcvta.to.global.u64 g, %0;\n\tprefetch.global.L2 [g];\n\t}"
                             :: "l"(grec(G, slot[i])));
        }
    }
    if (MODE == 3) {
        // cold rows become entries of their region; the lanes of a warp that
        // share a region reserve their places with one atomic.  (One atomic
        // per row, all four in flight at once, measured slower at 2^24 keys.)
        const PartK& K = G.pk;
        const unsigned lane = threadIdx.x & 31;
        const uint32_t stripe = blockIdx.x & (uint32_t)(K.stripes - 1);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const bool cold = ok[i] && hidx[i] < 0;
            const unsigned act = __ballot_sync(0xffffffffu, cold);
            if (!cold) continue;
            const uint32_t r = (uint32_t)(slot[i] >> K.shift) * (uint32_t)K.stripes + stripe;
            const unsigned peers = __match_any_sync(act, r);
            const int leader = __ffs(peers) - 1;
            uint32_t pos = 0, cap = 0;
            long long base = 0;
            if ((int)lane == leader) {
                pos = atomicAdd(&K.fill[r], (uint32_t)__popc(peers));
                cap = K.cap[r];
                base = K.base[r];
            }
            pos = __shfl_sync(peers, pos, leader) + (uint32_t)__popc(peers & ((1u << lane) - 1u));
            cap = __shfl_sync(peers, cap, leader);
            base = __shfl_sync(peers, base, leader);
            if (pos < cap) {
                const int64_t e = base + pos;
                K.e_slot[e] = (uint32_t)slot[i];
#pragma unroll
                for (int j = 0; j < 2; j++)
                    if (j < K.ne) K.e_val[j][e] = (unsigned long long)vec_pick<NC>(cv, (A.esel >> j) & 1, i);
                ok[i] = false;              // the partition pass aggregates it
            }
        }
    }
    // hot (shared-memory) and cold (global-record) updates are separate call
    // sites; a MIN/MAX reads the shared extreme first, which stops moving
    // after a slot's first rows, so most of those atomics are skipped
    const uint32_t scnt = sh_addr(V.cnt);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        if (!ok[i]) continue;
        if (MODE == 0 || hidx[i] >= 0) sh_add_u32(scnt + 4u * (uint32_t)hidx[i], 1u);
        else atomicAdd(grec(G, slot[i]), 1ULL);
    }
    for (int a = 0; a < G.na; a++) {
        const int kind = G.kind[a];
        if (kind == K_COUNT || NC == 0) continue;
        const int ai = G.ai[a];
        const uint32_t sacc = sh_addr(V.acc + (int64_t)ai * V.cap);
        const int c = (A.vsel >> a) & 1;
        long long w[4];
        bool on[4];
        const bool fl = kind == K_MIN_F || kind == K_MAX_F;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            w[i] = vec_pick<NC>(cv, c, i);
            on[i] = ok[i];
            if (fl) {
                const double d = __longlong_as_double(w[i]);
                on[i] = ok[i] && d == d;               // MIN/MAX of F64 skip NaN
                w[i] = f2ord(d);
            }
        }
#define TDG_HOT(i) (MODE == 0 || hidx[i] >= 0)
#define TDG_SA(i) (sacc + 8u * (uint32_t)hidx[i])
#define TDG_GA(i) (grec(G, slot[i]) + 1 + ai)
        switch (kind) {
            case K_SUM_F:
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    if (!on[i]) continue;
                    if (TDG_HOT(i)) sh_add_f64(TDG_SA(i), __longlong_as_double(w[i]));
                    else atomicAdd((double*)TDG_GA(i), __longlong_as_double(w[i]));
                }
                break;
            case K_SUM_I:
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    if (!on[i]) continue;
                    if (TDG_HOT(i)) sh_add_u64(TDG_SA(i), (unsigned long long)w[i]);
                    else atomicAdd(TDG_GA(i), (unsigned long long)w[i]);
                }
                break;
            case K_MIN_I: case K_MIN_F:
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    if (!on[i]) continue;
                    if (TDG_HOT(i)) { if (w[i] < sh_ld_s64(TDG_SA(i))) sh_min_s64(TDG_SA(i), w[i]); }
                    else upd_min<true>(TDG_GA(i), w[i]);
                }
                break;
            case K_MAX_I: case K_MAX_F:
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    if (!on[i]) continue;
                    if (TDG_HOT(i)) { if (w[i] > sh_ld_s64(TDG_SA(i))) sh_max_s64(TDG_SA(i), w[i]); }
                    else upd_max<true>(TDG_GA(i), w[i]);
                }
                break;
            default: break;
        }
#undef TDG_HOT
#undef TDG_SA
#undef TDG_GA
    }
}

// The rows a thread owns in the 4 * kThreads-row tile at base: two pairs of
// adjacent rows, each pair one 16-byte load per column.
__device__ __forceinline__ void tile_rows(int64_t base, int64_t (&row)[4]) {
#pragma unroll
    for (int j = 0; j < 2; j++) {
        row[2 * j] = base + (int64_t)j * 2 * kThreads + 2 * threadIdx.x;
        row[2 * j + 1] = row[2 * j] + 1;
    }
}

template <int NC>
__device__ __forceinline__ void vec_load(const VecAgg& A, const tdg_col& kcol, int64_t n, int64_t base,
                                         long long (&fk)[4], long long (&cv)[NC > 0 ? NC : 1][4]) {
#pragma unroll
    for (int j = 0; j < 2; j++) {
        const int64_t r = base + (int64_t)j * 2 * kThreads + 2 * threadIdx.x;
        ld_pair(kcol, r, n, fk[2 * j], fk[2 * j + 1]);
#pragma unroll
        for (int c = 0; c < NC; c++) ld_pair(A.vc[c], r, n, cv[c][2 * j], cv[c][2 * j + 1]);
    }
}

// The grid-stride loop of the vector kernels.  Registers double-buffer the
// columns: the next tile's loads are issued before this tile's map reads and
// shared-memory updates wait on theirs.  (An L2 bulk prefetch of the next
// tile instead re-read about 16% of the streamed bytes from DRAM in the join
// probe: prefetched lines left L2 before their loads.)
template <int NT, int NC, int MODE, bool MAP, typename PT>
__device__ __forceinline__ void vec_stream(const GroupK& G, const SmemView& V, const Pred& P, const VecAgg& A,
                                           const tdg_col& kcol, int64_t kmin, int64_t n_map,
                                           const PT* __restrict__ map, int64_t n, uint64_t pol) {
    const int64_t tile = (int64_t)kThreads * 4, stride = (int64_t)gridDim.x * tile;
    long long fk[4], cv[NC > 0 ? NC : 1][4];
    int64_t base = (int64_t)blockIdx.x * tile;
    if (base < n) vec_load<NC>(A, kcol, n, base, fk, cv);
    for (; base < n; base += stride) {
        long long fk2[4] = {0, 0, 0, 0}, cv2[NC > 0 ? NC : 1][4] = {};
        if (base + stride < n) vec_load<NC>(A, kcol, n, base + stride, fk2, cv2);
        int64_t row[4];
        tile_rows(base, row);
        vec_rows<NT, NC, MODE, MAP, PT>(G, V, P, A, row, fk, cv, kmin, n_map, map, n, pol);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            fk[i] = fk2[i];
#pragma unroll
            for (int c = 0; c < NC; c++) cv[c][i] = cv2[c][i];
        }
    }
}

// The double buffer holds a second tile of columns in registers, so the
// probe is bounded for 4 resident CTAs (64 registers) where the others use
// TDG_MINB.
constexpr int kVecMinBlocks = 4;

template <int NT, int NC, typename PT>
__global__ void __launch_bounds__(kThreads, kVecMinBlocks) k_probe_vec(const GroupK G, const Pred P, const VecAgg A,
                                                                       const tdg_col lkey, int64_t kmin, int64_t n_map,
                                                                       const PT* __restrict__ map, int64_t n,
                                                                       int64_t holes) {
    extern __shared__ unsigned long long sm[];
    if (holes) {
        // a plain-store build's empty-entry check (k_map_holes' work) as the
        // probe starts: the CTAs share the map (from L2) before streaming
        bool hole = false;
        const uint4* m4 = (const uint4*)map;
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (holes >> 2);
             i += (int64_t)gridDim.x * blockDim.x) {
            const uint4 v = m4[i];
            hole |= v.x == 0xFFFFFFFFu || v.y == 0xFFFFFFFFu || v.z == 0xFFFFFFFFu || v.w == 0xFFFFFFFFu;
        }
        if (blockIdx.x == 0 && (int64_t)threadIdx.x < (holes & 3))
            hole |= (uint32_t)map[((holes >> 2) << 2) + threadIdx.x] == 0xFFFFFFFFu;
        if (__syncthreads_or(hole) && threadIdx.x == 0) atomicExch(G.err + 1, 1);
    }
    const SmemView V = smem_setup<0>(G, sm);
    vec_stream<NT, NC, 0, true, PT>(G, V, P, A, lkey, kmin, n_map, map, n, evict_last_policy());
    smem_flush<0>(G, V);
}

// MODE 1 holds fewer CTAs per SM (the hot cache's shared memory), so it may
// use more registers.
constexpr int kVecHotMinBlocks = 3;

// The plain group-by keeps single-buffered tiles with an L2 bulk prefetch of
// the CTA's next tile: the double buffer of the probe measured no faster for
// MODE 0 and 13% slower for MODE 3, which is issue-bound and loses occupancy
// to the extra registers.
template <int NT, int NC, int MODE>
__global__ void __launch_bounds__(kThreads, MODE == 0 ? TDG_MINB : kVecHotMinBlocks)
k_group_vec(const GroupK G, const Pred P, const VecAgg A, int64_t n) {
    extern __shared__ unsigned long long sm[];
    const SmemView V = smem_setup<MODE>(G, sm);
    const int64_t tile = (int64_t)kThreads * 4;
    for (int64_t base = (int64_t)blockIdx.x * tile; base < n; base += (int64_t)gridDim.x * tile) {
        const int64_t nb = base + (int64_t)gridDim.x * tile;
        prefetch_rows(G.pf, nb, nb + tile < n ? nb + tile : n);
        long long fk[4], cv[NC > 0 ? NC : 1][4];
        int64_t row[4];
        vec_load<NC>(A, G.key[0], n, base, fk, cv);
        tile_rows(base, row);
        vec_rows<NT, NC, MODE, false, uint32_t>(G, V, P, A, row, fk, cv, G.kmin[0], G.krange[0], nullptr, n, 0);
    }
    if (MODE == 0 || V.n_hot) smem_flush<MODE>(G, V);
}

// ---- MODE 3: partitioned cold rows -----------------------------------------------

__device__ __forceinline__ double block_sum(double v, double* sh) {
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        double w = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        if (threadIdx.x == 0) sh[32] = w;
    }
    __syncthreads();
    const double r = sh[32];
    __syncthreads();
    return r;
}

// Exclusive prefix of v[0, m) into out[0, m] (out[m] = total), one CTA.
__device__ void block_scan_i64(const uint32_t* v, int64_t m, int64_t* out, long long* part) {
    const int64_t per = (m + blockDim.x - 1) / blockDim.x;
    const int64_t b = threadIdx.x * per, e = b + per < m ? b + per : m;
    long long sum = 0;
    for (int64_t i = b; i < e; i++) sum += v[i];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < (int)blockDim.x; off <<= 1) {
        const long long add = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += add;
        __syncthreads();
    }
    long long run = threadIdx.x ? part[threadIdx.x - 1] : 0;
    for (int64_t i = b; i < e; i++) { out[i] = run; run += v[i]; }
    if (threadIdx.x == blockDim.x - 1) out[m] = part[blockDim.x - 1];
    __syncthreads();
}

// Region capacities from the sampled estimates: 1.5x the partition's own
// estimate plus half the mean (so a partition the sample under-counted still
// gets room), scaled from the sampled rows to the input, shared by its
// stripes, plus a margin -- shrunk to the entry buffers when they would not
// fit.  Bases are the prefix of the capacities; fills and the work counter
// start at zero.
__global__ void __launch_bounds__(1024) k_part_plan(const GroupK G, int64_t n, int64_t m_rows) {
    const PartK& K = G.pk;
    __shared__ double sh[33];
    __shared__ long long part[1024];
    double s = 0;
    for (int64_t p = threadIdx.x; p < K.P; p += blockDim.x) s += K.est[p];
    const double mean = block_sum(s, sh) / (double)K.P;
    const double scale = (double)n / (double)(m_rows > 0 ? m_rows : 1) / (double)K.stripes;
    double tot = 0;
    for (int64_t r = threadIdx.x; r < K.R; r += blockDim.x) {
        double c = (1.5 * K.est[r / K.stripes] + 0.5 * mean) * scale + kPartMargin;
        if (c > 2.0e9) c = 2.0e9;
        K.cap[r] = (uint32_t)c;
        tot += (double)(uint32_t)c;
    }
    const double total = block_sum(tot, sh);
    if (total > (double)K.cap_total) {
        // R entries of slack: the truncations can never round the sum past the buffers
        const double room = (double)K.cap_total - (double)K.R;
        const double f = room > 0 ? room / total : 0.0;
        for (int64_t r = threadIdx.x; r < K.R; r += blockDim.x) K.cap[r] = (uint32_t)((double)K.cap[r] * f);
    }
    __syncthreads();
    block_scan_i64(K.cap, K.R, K.base, part);
    for (int64_t r = threadIdx.x; r < K.R; r += blockDim.x) K.fill[r] = 0;
    if (threadIdx.x == 0) *K.item_next = 0;
}

// Work items of the partition pass: ceil(entries / kPartItem) per region.
__global__ void __launch_bounds__(1024) k_part_items(const GroupK G) {
    const PartK& K = G.pk;
    __shared__ long long part[1024];
    // the capacities are no longer needed: reuse them for the item counts
    // after the fills are clamped
    for (int64_t r = threadIdx.x; r < K.R; r += blockDim.x) {
        const uint32_t f = K.fill[r] < K.cap[r] ? K.fill[r] : K.cap[r];
        K.fill[r] = f;
        K.cap[r] = (uint32_t)((f + kPartItem - 1) / kPartItem);
    }
    __syncthreads();
    block_scan_i64(K.cap, K.R, K.item_start, part);
    for (int64_t r = threadIdx.x; r < K.R; r += blockDim.x)
        for (int64_t i = K.item_start[r]; i < K.item_start[r + 1]; i++) K.item_region[i] = (int32_t)r;
}

// The partition pass: each work item aggregates up to kPartItem entries of
// one region in a shared-memory table of the partition's slots, then merges
// the table into the global records -- with plain read-modify-writes when
// the item is its partition's only one, with atomics otherwise.  Every
// thread loads four entries before it aggregates them.
__global__ void __launch_bounds__(kPartThreads) k_part_agg(const GroupK G, const VecAgg A) {
    extern __shared__ unsigned long long sm[];
    __shared__ long long s_item;
    const PartK& K = G.pk;
    const int64_t PS = (int64_t)1 << K.shift;
    uint32_t* cnt = (uint32_t*)sm;
    unsigned long long* acc = sm + ((PS * 4 + 7) >> 3);
    const uint32_t scnt = sh_addr(cnt), sacc = sh_addr(acc);
    const int64_t n_items = K.item_start[K.R];
    if (threadIdx.x == 0) s_item = (long long)atomicAdd(K.item_next, 1u);
    __syncthreads();
    for (;;) {
        const int64_t item = s_item;
        if (item >= n_items) break;
        // the next item is claimed now; its index is published after this one
        long long next = 0;
        if (threadIdx.x == 0) next = (long long)atomicAdd(K.item_next, 1u);
        const int64_t r = K.item_region[item], k = item - K.item_start[r];
        const int64_t p = r / K.stripes, slot0 = p << K.shift;
        const int64_t f = K.fill[r];
        const int64_t e0 = K.base[r] + k * kPartItem;
        const int64_t e1 = K.base[r] + ((k + 1) * kPartItem < f ? (k + 1) * kPartItem : f);
        const bool sole = K.stripes == 1 && K.item_start[r + 1] - K.item_start[r] == 1;
        if (threadIdx.x == 0) {
            // the records of this item's partition and of the next claimed
            // item's are brought into L2 with bulk prefetches, so the record
            // updates below find their lines there instead of each waiting
            // on DRAM
            const int64_t n_ls = G.S - slot0 < PS ? G.S - slot0 : PS;
            if (k == 0) l2_prefetch(grec(G, slot0), n_ls * G.W * 8);
            if (next < n_items) {
                const int64_t r2 = K.item_region[next], p2 = r2 / K.stripes, s2 = p2 << K.shift;
                if (r2 != r) l2_prefetch(grec(G, s2), (G.S - s2 < PS ? G.S - s2 : PS) * G.W * 8);
            }
        }
        if (e1 - e0 < PS * kPartDense) {
            // sparse: a table would cost more to clear and merge than the
            // entries themselves; they update the records directly, which
            // this item's partition keeps in L2 meanwhile
            for (int64_t eb = e0; eb < e1; eb += 4 * (int64_t)blockDim.x) {
                int64_t sl[4];
                long long v0[4], v1[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {           // four entries' loads in flight together
                    const int64_t e = eb + u * (int64_t)blockDim.x + threadIdx.x;
                    sl[u] = e < e1 ? (int64_t)__ldcs(K.e_slot + e) : -1;
                    v0[u] = e < e1 && K.ne > 0 ? (long long)__ldcs(K.e_val[0] + e) : 0;
                    v1[u] = e < e1 && K.ne > 1 ? (long long)__ldcs(K.e_val[1] + e) : 0;
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    if (sl[u] < 0) continue;
                    unsigned long long* rec = grec(G, sl[u]);
                    atomicAdd(rec, 1ULL);
                    for (int a = 0; a < G.na; a++) {
                        const int kind = G.kind[a];
                        if (kind == K_COUNT) continue;
                        long long w0 = v0[u], w1 = v1[u];
                        asm("" : "+l"(w0), "+l"(w1));     // a register select, not an indexed load
                        long long w = ((A.asel >> a) & 1) ? w1 : w0;
                        if (kind == K_MIN_F || kind == K_MAX_F) {
                            const double d = __longlong_as_double(w);
                            if (d != d) continue;
                            w = f2ord(d);
                        }
                        merge(rec + 1 + G.ai[a], kind, (unsigned long long)w);
                    }
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) s_item = next;
            __syncthreads();
            continue;
        }
        for (int64_t i = threadIdx.x; i < PS; i += blockDim.x) cnt[i] = 0;
        for (int a = 0; a < G.na; a++) {
            if (G.ai[a] < 0) continue;
            const unsigned long long init = acc_init_kind(G.kind[a]);
            for (int64_t i = threadIdx.x; i < PS; i += blockDim.x) acc[(int64_t)G.ai[a] * PS + i] = init;
        }
        __syncthreads();
        for (int64_t eb = e0; eb < e1; eb += 4 * (int64_t)blockDim.x) {
            uint32_t ls[4];
            long long v[2][4];
            bool in[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int64_t e = eb + u * (int64_t)blockDim.x + threadIdx.x;
                in[u] = e < e1;
                ls[u] = in[u] ? (uint32_t)((int64_t)__ldcs(K.e_slot + e) - slot0) : 0u;
                v[0][u] = in[u] && K.ne > 0 ? (long long)__ldcs(K.e_val[0] + e) : 0;
                v[1][u] = in[u] && K.ne > 1 ? (long long)__ldcs(K.e_val[1] + e) : 0;
            }
#pragma unroll
            for (int u = 0; u < 4; u++) if (in[u]) sh_add_u32(scnt + 4u * ls[u], 1u);
            for (int a = 0; a < G.na; a++) {
                const int kind = G.kind[a];
                if (kind == K_COUNT) continue;
                const uint32_t sa = sacc + 8u * (uint32_t)(G.ai[a] * PS);
                const bool second = (A.asel >> a) & 1;
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    if (!in[u]) continue;
                    long long w0 = v[0][u], w1 = v[1][u];
                    asm("" : "+l"(w0), "+l"(w1));     // a register select, not an indexed load
                    long long w = second ? w1 : w0;
                    const uint32_t t = sa + 8u * ls[u];
                    switch (kind) {
                        case K_SUM_F: sh_add_f64(t, __longlong_as_double(w)); break;
                        case K_SUM_I: sh_add_u64(t, (unsigned long long)w); break;
                        case K_MIN_I: if (w < sh_ld_s64(t)) sh_min_s64(t, w); break;
                        case K_MAX_I: if (w > sh_ld_s64(t)) sh_max_s64(t, w); break;
                        case K_MIN_F: {
                            const double d = __longlong_as_double(w);
                            w = f2ord(d);
                            if (d == d && w < sh_ld_s64(t)) sh_min_s64(t, w);
                            break;
                        }
                        case K_MAX_F: {
                            const double d = __longlong_as_double(w);
                            w = f2ord(d);
                            if (d == d && w > sh_ld_s64(t)) sh_max_s64(t, w);
                            break;
                        }
                        default: break;
                    }
                }
            }
        }
        __syncthreads();
        const int64_t n_ls = G.S - slot0 < PS ? G.S - slot0 : PS;
        for (int64_t i = threadIdx.x; i < n_ls; i += blockDim.x) {
            const uint32_t c = cnt[i];
            if (!c) continue;
            unsigned long long* rec = grec(G, slot0 + i);
            if (sole) {
                // every word of the record is read before any is combined, so
                // a record costs one memory round trip
                unsigned long long y[TDG_MAX_AGGS + 1];
#pragma unroll
                for (int w = 0; w <= TDG_MAX_AGGS; w++) if (w <= G.n_acc) y[w] = rec[w];
                y[0] += c;
#pragma unroll
                for (int w = 1; w <= TDG_MAX_AGGS; w++) {
                    if (w > G.n_acc) break;
                    const unsigned long long x = acc[(int64_t)(w - 1) * PS + i];
                    switch (G.akind[w - 1]) {
                        case K_SUM_I: y[w] += x; break;
                        case K_SUM_F: y[w] = (unsigned long long)__double_as_longlong(
                                          __longlong_as_double((long long)y[w]) + __longlong_as_double((long long)x));
                                      break;
                        case K_MIN_I: case K_MIN_F: if ((long long)x < (long long)y[w]) y[w] = x; break;
                        case K_MAX_I: case K_MAX_F: if ((long long)x > (long long)y[w]) y[w] = x; break;
                        default: break;
                    }
                }
#pragma unroll
                for (int w = 0; w <= TDG_MAX_AGGS; w++) if (w <= G.n_acc) rec[w] = y[w];
            } else {
                atomicAdd(rec, (unsigned long long)c);
                for (int a = 0; a < G.na; a++)
                    if (G.ai[a] >= 0) merge(rec + 1 + G.ai[a], G.kind[a], acc[(int64_t)G.ai[a] * PS + i]);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_item = next;
        __syncthreads();
    }
}

// Full outer join: build rows that no probe row matched enter the group-by
// with zero-filled probe-side values (global accumulators, no cache).
template <int MODE>
__global__ void __launch_bounds__(kThreads) k_group_unmatched(GroupK G, const JoinK J, int64_t n_right) {
    G.hot_cap = 0;
    SmemView V;
    memset(&V, 0, sizeof(V));
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < n_right;
         b += (int64_t)gridDim.x * blockDim.x) {
        if (J.matched[b]) continue;
        int64_t p1[1] = {-1}, b1[1] = {b};
        bool m1[1] = {true};
        accumulate<MODE, false, 1>(G, V, p1, b1, m1);
    }
}

// Initial values of the slot records.  Each warp fills 32 whole records as
// 32*W consecutive words, so every store instruction writes 256 contiguous
// bytes (no partial-sector read-modify-write in L2).
__global__ void k_group_init(const GroupK G) {
    if (blockIdx.x == 0 && threadIdx.x < 64) G.err[threadIdx.x] = 0;     // the 256-byte error area
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int W = G.W;
    const int step = 32 % W;
    const int64_t nchunks = (G.S + 31) >> 5;
    for (int64_t ch = warp; ch < nchunks; ch += nwarps) {
        const int64_t recs = G.S - ch * 32 < 32 ? G.S - ch * 32 : 32;
        const int words = (int)(recs * W);
        unsigned long long* base = G.rec + ch * 32 * W;
        int f = lane % W;
        for (int j = lane; j < words; j += 32) {
            base[j] = G.finit[f];
            f += step;
            if (f >= W) f -= W;
        }
    }
    if (G.method == TDG_GROUP_HASH)
        for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < G.S; s += (int64_t)gridDim.x * blockDim.x)
            G.ht.state[s] = 0;
}

// ---- emit ------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) k_emit_count(const GroupK G, int64_t* counts) {
    __shared__ int red[32];
    const int64_t base = (int64_t)blockIdx.x * kEmitChunk;
    int c = 0;
    for (int i = 0; i < kEmitChunk / kThreads; i++) {
        const int64_t s = base + i * kThreads + threadIdx.x;
        c += (s < G.S && grec(G, s)[0] != 0) ? 1 : 0;
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
        const unsigned long long* r = s < S ? grec(G, s) : nullptr;
        const unsigned long long c = r ? r[0] : 0;
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
                const int kind = G.kind[a];
                uint64_t res;
                if (kind == K_COUNT) {
                    res = c;
                } else {
                    const unsigned long long v = r[1 + G.ai[a]];
                    if (G.op[a] == A_AVG) {
                        const double sum = kind == K_SUM_F ? __longlong_as_double((long long)v) : (double)(long long)v;
                        res = (uint64_t)__double_as_longlong(sum / (double)c);
                    } else if (kind == K_MIN_F || kind == K_MAX_F) {
                        res = (uint64_t)__double_as_longlong(ord2f((long long)v));
                    } else {
                        res = v;
                    }
                }
                ((uint64_t*)O.aggs[a])[o] = res;
            }
        }
        out += tot;
        if (base + (i + 1) * kThreads >= S) break;
    }
}

// Small group-bys (S <= kSmallEmit slots): one CTA counts, scans and emits in
// slot order in a single launch.
constexpr int64_t kSmallEmit = 8192;

__device__ __forceinline__ void emit_one(const GroupK& G, const OutK& O, int64_t s, const unsigned long long* r,
                                         unsigned long long c, int64_t o) {
    for (int k = 0; k < G.nk; k++) {
        int64_t v;
        if (G.method == TDG_GROUP_DIRECT) v = G.kmin[k] + (s / G.stride[k]) % G.krange[k];
        else v = G.ht.keys[(int64_t)k * G.S + s];
        put_key(O.keys[k], O.kesz[k], o, v);
    }
    for (int a = 0; a < G.na; a++) {
        const int kind = G.kind[a];
        uint64_t res;
        if (kind == K_COUNT) {
            res = c;
        } else {
            const unsigned long long v = r[1 + G.ai[a]];
            if (G.op[a] == A_AVG) {
                const double sum = kind == K_SUM_F ? __longlong_as_double((long long)v) : (double)(long long)v;
                res = (uint64_t)__double_as_longlong(sum / (double)c);
            } else if (kind == K_MIN_F || kind == K_MAX_F) {
                res = (uint64_t)__double_as_longlong(ord2f((long long)v));
            } else {
                res = v;
            }
        }
        ((uint64_t*)O.aggs[a])[o] = res;
    }
}

__global__ void __launch_bounds__(1024) k_emit_small(const GroupK G, const OutK O, int64_t* d_total) {
    __shared__ int red[32];
    int64_t out = 0;
    for (int64_t s0 = 0; s0 < G.S; s0 += blockDim.x) {
        const int64_t s = s0 + threadIdx.x;
        const unsigned long long* r = s < G.S ? grec(G, s) : nullptr;
        const unsigned long long c = r ? r[0] : 0;
        int tot;
        const int pre = block_excl_scan(c ? 1 : 0, &tot, red);
        if (c) emit_one(G, O, s, r, c, out + pre);
        out += tot;
    }
    if (threadIdx.x == 0) {
        *d_total = out;
        if (O.herr) { O.herr[0] = O.err[0]; O.herr[1] = O.err[1]; }
    }
}

__global__ void __launch_bounds__(1024) k_scan_counts_g(int64_t* counts, int64_t m, int64_t* d_total,
                                                        const int32_t* err, int32_t* herr) {
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
    if (threadIdx.x == 0 && herr) { herr[0] = err[0]; herr[1] = err[1]; }
}

// ---- host side: layout, plan, launch ----------------------------------------------------
struct Layout {
    size_t err, rec, state, keys, emit, sample_keys, sample_cnt, hot, hot_n, total;
};

static size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

static int words_of(int n_acc) { return 1 + n_acc == 3 ? 4 : 1 + n_acc; }

static Layout layout_of(int64_t S, int n_acc, int nk, int method, bool sampled) {
    Layout L;
    size_t o = 0;
    L.err = o; o += 256;
    L.rec = o; o += al((size_t)S * 8 * words_of(n_acc));
    L.state = o; o += method == TDG_GROUP_HASH ? al((size_t)S * 4) : 0;
    L.keys = o; o += method == TDG_GROUP_HASH ? al((size_t)S * 8 * nk) : 0;
    L.emit = o; o += al((size_t)((S + kEmitChunk - 1) / kEmitChunk + 1) * 8);
    L.sample_keys = o; o += sampled ? al((size_t)kSampleCap * 8) : 0;
    L.sample_cnt = o; o += sampled ? al((size_t)kSampleCap * 4) : 0;
    L.hot = o; o += sampled ? al((size_t)kHotMax * 8) : 0;
    L.hot_n = o; o += sampled ? al(256 + (size_t)kHotHist * 4) : 0;   // hot_n, threshold, then hot_hist
    L.total = o;
    return L;
}

// ---- MODE 3 planning ----
// Distinct aggregate input columns (-1 when an input is not 8 bytes wide or
// there are more than two).
static int part_values(const tdg_group_desc* d) {
    const void* seen[2] = {nullptr, nullptr};
    int ne = 0;
    for (int a = 0; a < d->n_aggs; a++) {
        if (d->aggs[a].op == A_COUNT) continue;
        if (elem_size(d->aggs[a].in.type, d->aggs[a].in.attrs) != 8) return -1;
        int j = 0;
        while (j < ne && seen[j] != d->aggs[a].in.data) j++;
        if (j < ne) continue;
        if (ne == 2) return -1;
        seen[ne++] = d->aggs[a].in.data;
    }
    return ne;
}

static bool wants_partition(const tdg_group_desc* d, int method, bool smem, int64_t S, int64_t nrows) {
    return method == TDG_GROUP_DIRECT && !smem && nrows >= kPartMinRows && d->n_keys == 1 &&
           is_int_class(d->keys[0].type) && elem_size(d->keys[0].type, d->keys[0].attrs) == 8 &&
           S < ((int64_t)1 << 32) && part_values(d) >= 0;
}

static bool wants_sampling(int method, bool smem, int64_t S, int64_t nrows);

static bool group_sampled(const tdg_group_desc* d, int method, bool smem, int64_t S, int64_t nrows) {
    return wants_sampling(method, smem, S, nrows) || wants_partition(d, method, smem, S, nrows);
}

struct PartLayout {
    PartK k;                      // dimensions; pointers are offsets from the section start
    size_t est, fill, cap, base, item_start, item_region, item_next, e_slot, e_val[2], total;
};

// The MODE 3 section, placed after the rest of the workspace.  A partition
// spans the slots whose shared-memory table (32-bit count, 8-byte
// accumulators) fits kPartSmem (kPartSmemWide for wide key ranges); the entry buffers hold one entry per input row.
static PartLayout part_layout(const tdg_group_desc* d, int64_t S, int n_acc, int64_t nrows) {
    PartLayout L;
    memset(&L, 0, sizeof(L));
    const size_t per = 4 + 8 * (size_t)n_acc;
    int shift = 0;
    const size_t table = S >= kPartWideSlots ? kPartSmemWide : kPartSmem;
    while (((size_t)2 << shift) * per <= table) shift++;
    L.k.shift = shift;
    L.k.P = (S + ((int64_t)1 << shift) - 1) >> shift;
    int st = 1;
    while (st < kPartMaxStripes && L.k.P * st * 2 <= kPartRegions) st <<= 1;
    L.k.stripes = st;
    L.k.R = L.k.P * st;
    L.k.ne = part_values(d);
    L.k.cap_total = nrows;
    size_t o = 0;
    L.est = o; o += al((size_t)L.k.P * 4);
    L.fill = o; o += al((size_t)L.k.R * 4);
    L.cap = o; o += al((size_t)L.k.R * 4);
    L.base = o; o += al((size_t)L.k.R * 8);
    L.item_start = o; o += al((size_t)(L.k.R + 1) * 8);
    L.item_region = o; o += al((size_t)(L.k.R + nrows / kPartItem + 1) * 4);
    L.item_next = o; o += 256;
    L.e_slot = o; o += al((size_t)nrows * 4);
    for (int j = 0; j < L.k.ne; j++) { L.e_val[j] = o; o += al((size_t)nrows * 8); }
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

// The hot-slot cache pays off for large inputs aggregated in global memory.
static bool wants_sampling(int method, bool smem, int64_t S, int64_t nrows) {
    return !smem && nrows >= kSampleMinRows && S < ((int64_t)1 << 31) && (method == TDG_GROUP_DIRECT || method == TDG_GROUP_HASH);
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
        p->smem = smem_full_bytes(slots, n_acc) <= kSmemMax ? 1 : 0;
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
    const bool sampled = group_sampled(d, p->method, p->smem != 0, p->n_slots, nrows_bound);
    p->ws_bytes = layout_of(p->n_slots, n_acc, d->n_keys, p->method, sampled).total;
    if (wants_partition(d, p->method, p->smem != 0, p->n_slots, nrows_bound))
        p->ws_bytes += part_layout(d, p->n_slots, n_acc, nrows_bound).total;
    return E_OK;
}

static int kind_of(const tdg_agg& a) {
    const bool f = a.in.type == T_F64;
    switch (a.op) {
        case A_COUNT: return K_COUNT;
        case A_MIN: return f ? K_MIN_F : K_MIN_I;
        case A_MAX: return f ? K_MAX_F : K_MAX_I;
        default: return f ? K_SUM_F : K_SUM_I;     // SUM, AVG
    }
}

// Grid of a streaming kernel: all CTAs that fit, or cps per SM when the
// plan's launch shape asks for fewer; never more CTAs than work items.
static int stream_grid(const void* kernel, int threads, size_t smem, int64_t items, int cps) {
    int g = grid_for(kernel, threads, smem, items);
    if (cps > 0) {
        const int64_t cap = (int64_t)cps * sm_count();
        if (g > cap) g = (int)cap;
    }
    return g;
}

static GroupK make_gk(const tdg_group_desc* d, const tdg_group_plan* p, void* ws, int64_t nrows_bound) {
    GroupK G;
    memset(&G, 0, sizeof(G));
    G.cps = p->ctas_per_sm;
    G.rep0 = p->smem && smem_full_bytes(p->n_slots, count_acc(d)) * (kThreads / 32) <= kSmemMax ? kThreads / 32 : 1;
    const int n_acc = count_acc(d);
    const bool sampled = group_sampled(d, p->method, p->smem != 0, p->n_slots, nrows_bound);
    const Layout L = layout_of(p->n_slots, n_acc, d->n_keys, p->method, sampled);
    char* w = (char*)ws;
    G.nk = d->n_keys;
    G.na = d->n_aggs;
    G.method = p->method;
    G.n_acc = n_acc;
    G.W = words_of(n_acc);
    G.S = p->n_slots;
    G.err = (int32_t*)(w + L.err);
    G.rec = (unsigned long long*)(w + L.rec);
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
        G.kind[a] = kind_of(d->aggs[a]);
        G.ai[a] = G.op[a] == A_COUNT ? -1 : ai++;
        if (G.ai[a] >= 0) {
            G.finit[1 + G.ai[a]] = acc_init_kind(G.kind[a]);
            G.akind[G.ai[a]] = G.kind[a];
        }
    }
    if (p->method == TDG_GROUP_HASH) {
        G.ht.state = (uint32_t*)(w + L.state);
        G.ht.keys = (int64_t*)(w + L.keys);
        G.ht.mask = (uint64_t)p->n_slots - 1;
        G.ht.nk = d->n_keys;
        G.ht.err = G.err;
    }
    if (sampled) {
        G.sample_keys = (int64_t*)(w + L.sample_keys);
        G.sample_cnt = (uint32_t*)(w + L.sample_cnt);
        G.hot = (int64_t*)(w + L.hot);
        G.hot_n = (int32_t*)(w + L.hot_n);
        G.hot_hist = (uint32_t*)(w + L.hot_n + 256);
        int cap = (int)((kSmemMax - (size_t)kHotMap * 6 - 8) / (4 + 8 * (size_t)n_acc));
        G.hot_cap = cap < kHotMax ? cap : kHotMax;
    }
    if (wants_partition(d, p->method, p->smem != 0, p->n_slots, nrows_bound)) {
        const PartLayout PL = part_layout(d, p->n_slots, n_acc, nrows_bound);
        char* b = w + L.total;
        G.pk = PL.k;
        G.pk.est = (uint32_t*)(b + PL.est);
        G.pk.fill = (uint32_t*)(b + PL.fill);
        G.pk.cap = (uint32_t*)(b + PL.cap);
        G.pk.base = (int64_t*)(b + PL.base);
        G.pk.item_start = (int64_t*)(b + PL.item_start);
        G.pk.item_region = (int32_t*)(b + PL.item_region);
        G.pk.item_next = (uint32_t*)(b + PL.item_next);
        G.pk.e_slot = (uint32_t*)(b + PL.e_slot);
        for (int j = 0; j < PL.k.ne; j++) G.pk.e_val[j] = (unsigned long long*)(b + PL.e_val[j]);
    }
    return G;
}

static tdg_status prepare(const GroupK& G, cudaStream_t s) {
    const int g = grid_for((const void*)k_group_init, kThreads, 0, G.S);
    (note_launch(), k_group_init<<<g, kThreads, 0, s>>>(G));
    if (G.hot_cap) {
        cudaMemsetAsync(G.sample_keys, 0xFF, (size_t)kSampleCap * 8, s);
        cudaMemsetAsync(G.sample_cnt, 0, (size_t)kSampleCap * 4, s);
        cudaMemsetAsync(G.hot_n, 0, 256 + (size_t)kHotHist * 4, s);
    }
    if (G.pk.P) cudaMemsetAsync(G.pk.est, 0, (size_t)G.pk.P * 4, s);
    return launch_status();
}

// A few device-mapped page-locked words per host thread: kernels write
// status words there and the host reads them once the stream has
// synchronized, with no copy.  Freed when the thread exits.
namespace {
struct MappedWords {
    int32_t* h = nullptr;
    int32_t* d = nullptr;
    ~MappedWords() {
        if (h) cudaFreeHost(h);
    }
};
}  // namespace

static MappedWords* mapped_words() {
    static thread_local MappedWords w;
    if (no_alloc()) return nullptr;
    if (!w.h) {
        void *h = nullptr, *d = nullptr;
        if (cudaHostAlloc(&h, 64, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        if (cudaHostGetDevicePointer(&d, h, 0) != cudaSuccess) {
            cudaGetLastError();
            cudaFreeHost(h);
            return nullptr;
        }
        w.h = (int32_t*)h;
        w.d = (int32_t*)d;
    }
    return &w;
}

static int32_t* pinned_words() {
    MappedWords* m = mapped_words();
    return m ? m->h : nullptr;
}

static tdg_status finish(const GroupK& G, const tdg_group_desc* d, void* ws, const tdg_group_out* out,
                         cudaStream_t s, int32_t* flag1 = nullptr) {
    OutK O;
    memset(&O, 0, sizeof(O));
    for (int k = 0; k < G.nk; k++) {
        O.keys[k] = out->keys[k];
        O.kesz[k] = elem_size(d->keys[k].type, d->keys[k].attrs);
    }
    for (int a = 0; a < G.na; a++) O.aggs[a] = out->aggs[a];
    // the emit copies the error word and the repeated-key flag into mapped
    // host words; without them (no allocation allowed) they are copied
    MappedWords* mw = mapped_words();
    O.err = G.err;
    O.herr = mw ? mw->d : nullptr;
    if (G.S <= kSmallEmit) {
        (note_launch(), k_emit_small<<<1, 1024, 0, s>>>(G, O, out->d_n_groups));
    } else {
        const Layout L = layout_of(G.S, G.n_acc, G.nk, G.method, G.hot_cap != 0);
        int64_t* counts = (int64_t*)((char*)ws + L.emit);
        const int64_t chunks = (G.S + kEmitChunk - 1) / kEmitChunk;
        (note_launch(), k_emit_count<<<(unsigned)chunks, kThreads, 0, s>>>(G, counts));
        (note_launch(), k_scan_counts_g<<<1, 1024, 0, s>>>(counts, chunks, out->d_n_groups, O.err, O.herr));
        (note_launch(), k_emit<<<(unsigned)chunks, kThreads, 0, s>>>(G, O, counts));
    }
    tdg_status st = launch_status();
    if (st) return st;
    int32_t local[2] = {0, 0};
    if (!mw && cudaMemcpyAsync(local, G.err, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return E_IO;
    if (cudaStreamSynchronize(s) != cudaSuccess) return E_IO;
    const volatile int32_t* w = mw ? mw->h : local;
    if (flag1) *flag1 = w[1];
    return w[0];
}

static bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

static bool group_w8(const GroupK& G, const Pred& P, const JoinK* J) {
    if (!P.w8) return false;
    for (int k = 0; k < G.nk; k++) if (elem_size(G.key[k].type, G.key[k].attrs) != 8) return false;
    for (int a = 0; a < G.na; a++)
        if (G.kind[a] != K_COUNT && elem_size(G.in[a].type, G.in[a].attrs) != 8) return false;
    if (J) for (int k = 0; k < J->nk; k++) if (elem_size(J->lkeys[k].type, J->lkeys[k].attrs) != 8) return false;
    return true;
}

template <int PK, int MODE, bool JOIN, bool W8>
static tdg_status launch_main(const GroupK& G, const Pred& P, const tdg_expr& prog, const JoinK& J, int64_t n,
                              cudaStream_t s) {
    const size_t smem = MODE == 0 ? smem_full_bytes(G.S, G.n_acc) * G.rep0 : (G.hot_cap ? smem_hot_bytes(G.hot_cap, G.n_acc) : 0);
    const void* fn = (const void*)k_group<PK, MODE, JOIN, W8>;
    const int g = grid_for(fn, kThreads, smem, (n + kItems - 1) / kItems);
    (note_launch(), k_group<PK, MODE, JOIN, W8><<<g, kThreads, smem, s>>>(G, P, prog, J, n));
    return launch_status();
}

template <int PK, int MODE, bool JOIN>
static tdg_status launch_sample(const GroupK& G, const Pred& P, const tdg_expr& prog, const JoinK& J, int64_t n,
                                cudaStream_t s) {
    const int64_t m_rows = n < kSampleRows ? n : kSampleRows;
    const int64_t step = n / m_rows;
    const int g = grid_for((const void*)k_sample<PK, MODE, JOIN>, kThreads, 0, m_rows);
    (note_launch(), k_sample<PK, MODE, JOIN><<<g, kThreads, 0, s>>>(G, P, prog, J, n, step, m_rows));
    const int g2 = grid_for((const void*)k_select_hot, kThreads, 0, kSampleCap);
    (note_launch(), k_hot_hist<<<g2, kThreads, 0, s>>>(G));
    (note_launch(), k_hot_threshold<<<1, kHotHist, 0, s>>>(G));
    (note_launch(), k_select_hot<<<g2, kThreads, 0, s>>>(G));
    return launch_status();
}

// Streamed (row-indexed, probe-side) columns of a launch, for L2 prefetch.
static void set_prefetch(GroupK& G, const Pred& P, const tdg_expr& prog, int pk, const JoinK* J) {
    memset(&G.pf, 0, sizeof(G.pf));
    if (pk == 1)
        for (int i = 0; i < P.n; i++) pf_add(G.pf, P.t[i].col);
    if (pk == 2)
        for (int i = 0; i < prog.n_cols; i++) pf_add(G.pf, prog.cols[i]);
    if (J)
        for (int k = 0; k < J->nk; k++) pf_add(G.pf, J->lkeys[k]);
    for (int k = 0; k < G.nk; k++)
        if (!G.key[k].side) pf_add(G.pf, G.key[k]);
    for (int a = 0; a < G.na; a++)
        if (G.kind[a] != K_COUNT && !G.in[a].side) pf_add(G.pf, G.in[a]);
}

// Columns of the vector form: the predicate's terms (the range form, at most
// two) and the aggregates' inputs, at most two distinct columns between them,
// each 16-byte aligned.  False when the shape needs more.
static int vec_col(VecAgg& A, int& nc, const tdg_col& c) {
    for (int i = 0; i < nc; i++) if (A.vc[i].data == c.data) return i;
    if (nc == 2 || !aligned16(c.data)) return -1;
    A.vc[nc] = c;
    return nc++;
}

static bool vec_plan(const GroupK& G, int pk, const Pred& P, VecAgg& A, int* nt, int* nc) {
    memset(&A, 0, sizeof(A));
    *nt = 0;
    *nc = 0;
    if (P.sel || !(pk == 0 || (pk == 1 && P.n <= 2))) return false;
    *nt = pk == 1 ? P.n : 0;
    for (int t = 0; t < *nt; t++) {
        const int c = vec_col(A, *nc, P.t[t].col);
        if (c < 0) return false;
        A.tsel |= (uint32_t)c << t;
    }
    int ec[2] = {-1, -1};
    for (int a = 0; a < G.na; a++) {
        if (G.kind[a] == K_COUNT) continue;
        const int c = vec_col(A, *nc, G.in[a]);
        if (c < 0) return false;
        A.vsel |= (uint32_t)c << a;
        int j = 0;
        while (j < A.ne && ec[j] != c) j++;
        if (j == A.ne) {
            ec[j] = c;
            A.esel |= (uint32_t)c << j;
            A.ne++;
        }
        A.asel |= (uint32_t)j << a;
    }
    return true;
}

// Plain group-by with one 8-byte key in the vector form (MODE 0: shared-memory
// accumulators; MODE 1: global records and the hot cache; MODE 3 when its
// buffers are planned: MODE 1 with the cold rows partitioned); false when the
// shape does not qualify.
static bool launch_group_vec(const GroupK& G, const Pred& P, int pk, int mode, int64_t n, cudaStream_t s,
                             tdg_status* st) {
    if (G.nk != 1 || G.key[0].type == T_F64 || !aligned16(G.key[0].data)) return false;
    VecAgg A;
    int nt, nc;
    if (!vec_plan(G, pk, P, A, &nt, &nc)) return false;
    if (mode == 1 && G.pk.P && G.hot_cap && A.ne <= G.pk.ne) mode = 3;
    const size_t smem = mode == 0 ? smem_full_bytes(G.S, G.n_acc) * G.rep0 : (G.hot_cap ? smem_hot_bytes(G.hot_cap, G.n_acc) : 0);
    if (mode == 3) {
        const int64_t m_rows = n < kSampleRows ? n : kSampleRows;
        (note_launch(), k_part_plan<<<1, 1024, 0, s>>>(G, n, m_rows));
    }
    bool launched = false;
#define TDG_GV(NTV, NCV, MV)                                                                            \
    if (!launched && nt == NTV && nc == NCV && mode == MV) {                                            \
        const int g = stream_grid((const void*)k_group_vec<NTV, NCV, MV>, kThreads, smem, (n + 3) / 4, G.cps); \
        (note_launch(), k_group_vec<NTV, NCV, MV><<<g, kThreads, smem, s>>>(G, P, A, n));               \
        launched = true;                                                                                \
    }
    TDG_GV(0, 0, 0) TDG_GV(0, 1, 0) TDG_GV(0, 2, 0) TDG_GV(1, 1, 0) TDG_GV(1, 2, 0) TDG_GV(2, 1, 0) TDG_GV(2, 2, 0)
    TDG_GV(0, 0, 1) TDG_GV(0, 1, 1) TDG_GV(0, 2, 1) TDG_GV(1, 1, 1) TDG_GV(1, 2, 1) TDG_GV(2, 1, 1) TDG_GV(2, 2, 1)
    TDG_GV(0, 0, 3) TDG_GV(0, 1, 3) TDG_GV(0, 2, 3) TDG_GV(1, 1, 3) TDG_GV(1, 2, 3) TDG_GV(2, 1, 3) TDG_GV(2, 2, 3)
#undef TDG_GV
    if (!launched) {
        // k_part_plan ran for nothing: harmless, the fallback kernel does not read its buffers
        return false;
    }
    if (mode == 3) {
        (note_launch(), k_part_items<<<1, 1024, 0, s>>>(G));
        const int64_t PS = (int64_t)1 << G.pk.shift;
        const size_t smb = smem_full_bytes(PS, G.n_acc);
        if (cudaFuncSetAttribute((const void*)k_part_agg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smb) !=
            cudaSuccess) {
            *st = launch_status();
            return true;
        }
        const int g = grid_for((const void*)k_part_agg, kPartThreads, smb, (int64_t)1 << 40);
        (note_launch(), k_part_agg<<<g, kPartThreads, smb, s>>>(G, A));
    }
    *st = launch_status();
    return true;
}

template <bool JOIN>
static tdg_status dispatch(int pk, const GroupK& G0, bool smem, const Pred& P, const tdg_expr& prog,
                           const JoinK& J, int64_t n, cudaStream_t s, EventTimer& tm) {
    GroupK G = G0;
    set_prefetch(G, P, prog, pk, JOIN ? &J : nullptr);
    const int mode = G.method == TDG_GROUP_HASH ? 2 : (smem ? 0 : 1);
    tdg_status st = E_OK;
    if (G.hot_cap && n > 0) {
#define TDG_SMP(PKV, MV) if (pk == PKV && mode == MV) st = launch_sample<PKV, MV, JOIN>(G, P, prog, J, n, s);
        TDG_SMP(0, 1) TDG_SMP(0, 2) TDG_SMP(1, 1) TDG_SMP(1, 2) TDG_SMP(2, 1) TDG_SMP(2, 2)
#undef TDG_SMP
        if (st) return st;
    }
    const bool w8 = pk != 2 && group_w8(G, P, JOIN ? &J : nullptr);
    tm.start(s);
    if (!JOIN && mode != 2 && w8 && n > 0 && launch_group_vec(G, P, pk, mode, n, s, &st)) { tm.stop(s); return st; }
#define TDG_CASE(PKV, MV, W) \
    if (pk == PKV && mode == MV && w8 == W) { st = launch_main<PKV, MV, JOIN, W>(G, P, prog, J, n, s); tm.stop(s); return st; }
    TDG_CASE(0, 0, true) TDG_CASE(0, 1, true) TDG_CASE(0, 2, true)
    TDG_CASE(0, 0, false) TDG_CASE(0, 1, false) TDG_CASE(0, 2, false)
    TDG_CASE(1, 0, true) TDG_CASE(1, 1, true) TDG_CASE(1, 2, true)
    TDG_CASE(1, 0, false) TDG_CASE(1, 1, false) TDG_CASE(1, 2, false)
    TDG_CASE(2, 0, false) TDG_CASE(2, 1, false) TDG_CASE(2, 2, false)
#undef TDG_CASE
    tm.stop(s);
    return E_NYI;
}

// ---- shared with tdg_join.cu ------------------------------------------------------

// Payload join -> group (see k_payload_build).  Sets *used when it ran; when
// the shape does not qualify, or the build side turns out to hold duplicate
// keys, it returns with *used == false and the caller takes the general path.
// The shapes the payload map serves: a direct inner join on one integer key
// and a direct group-by whose aggregate inputs all come from the probe side.
static bool payload_ok(const tdg_group_desc* d, const tdg_group_plan* p, const JoinK* J) {
    if (J->method != TDG_JOIN_DIRECT || J->join_type != 0 || p->method != TDG_GROUP_DIRECT) return false;
    if (J->rkeys[0].type == T_F64 || p->n_slots >= 0xFFFFFFFFLL) return false;
    for (int a = 0; a < d->n_aggs; a++)
        if (d->aggs[a].op != A_COUNT && d->aggs[a].in.side != 0) return false;
    return true;
}

// The payload map's build pass into J->head: errors and the repeated-key
// flag land in err[0] and err[1] (zeroed here).
static tdg_status payload_build(const GroupK& G0, const JoinK* J, int32_t* err, int64_t n_right, cudaStream_t s) {
    GroupK G = G0;
    G.err = err;
    cudaMemsetAsync(err, 0, 8, s);
    cudaMemsetAsync(J->head, 0xFF, (size_t)J->n_slots * 4, s);
    if (n_right > 0) launch_payload_build(G, *J, (uint32_t*)J->head, n_right, s);
    return launch_status();
}

tdg_status join_payload_build(const tdg_group_desc* d, const tdg_group_plan* p, const JoinK* J, int32_t* err,
                              int64_t n_right, cudaStream_t s, int32_t* used) {
    *used = 0;
    if (!payload_ok(d, p, J)) return E_OK;
    GroupK G = make_gk(d, p, err, d->nrows);          // only the key fields are read
    tdg_status st = payload_build(G, J, err, n_right, s);
    if (st) return st;
    int32_t* w = pinned_words();
    int32_t local[2] = {0, 0};
    int32_t* dst = w ? w : local;
    if (cudaMemcpyAsync(dst, err, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return E_IO;
    }
    if (dst[0]) return dst[0];
    *used = dst[1] ? 0 : 1;
    return E_OK;
}

tdg_status group_run_payload(const tdg_group_desc* d, const tdg_group_plan* p, void* ws,
                             const tdg_expr* pred, const uint64_t* sel, const JoinK* J, int64_t n_left,
                             int64_t n_right, const tdg_group_out* out, cudaStream_t s, bool* used,
                             bool prebuilt) {
    *used = false;
    if (!payload_ok(d, p, J)) return prebuilt ? E_RANGE : E_OK;
    GroupK G = make_gk(d, p, ws, d->nrows);
    G.hot_cap = 0;
    tdg_status st = prepare(G, s);
    if (st) return st;
    // 32-bit entries: a native atomicCAS per build key both stores the slot
    // and detects a repeated key (or, for dense keys, a plain store and a
    // check for empty entries), and 4 bytes per key keeps a 10M-row build
    // side's map (40 MB) in L2.  (A 16-bit map with plain stores and a
    // duplicate bitmap measured slower on both passes.)  A prebuilt map was
    // checked for repeated keys when it was built.
    void* map = J->head;
    EventTimer tb;
    tb.start(s);
    int holes_pending = 0;
    if (!prebuilt) {
        cudaMemsetAsync(map, 0xFF, (size_t)J->n_slots * 4, s);
        if (n_right > 0) holes_pending = launch_payload_build(G, *J, (uint32_t*)map, n_right, s, true);
    }
    tb.stop(s);
    st = launch_status();
    if (st) { tb.ms(); return st; }
    // the probe runs without waiting for the build's duplicate-key flag; the
    // flag is read with the error word at the end, and if the build side had
    // duplicate keys the caller runs the general join instead
    int pk;
    Pred P = make_pred(pred, sel, &pk);
    static tdg_expr empty;
    const tdg_expr& prog = pred ? *pred : empty;
    const bool sm = p->smem != 0;
    const bool w8 = pk != 2 && group_w8(G, P, J);
    const size_t smem = sm ? smem_full_bytes(G.S, G.n_acc) * G.rep0 : 0;
    set_prefetch(G, P, prog, pk, J);
    EventTimer tm;
    tm.start(s);
    // the vector form, when the shape and the alignment allow it
    VecAgg A;
    int nc = 0, nt = 0;
    bool vec = sm && w8 && aligned16(J->lkeys[0].data);
    for (int k = 0; k < G.nk && vec; k++) vec = G.key[k].side == 1;
    vec = vec && vec_plan(G, pk, P, A, &nt, &nc);
    bool launched = false;
    if (holes_pending && !vec) launch_map_holes(G, (const uint32_t*)map, J->n_slots, s);
    const int64_t holes = holes_pending && vec ? J->n_slots : 0;
#define TDG_PV(NTV, NCV)                                                                                  \
    if (vec && !launched && nt == NTV && nc == NCV) {                                                     \
        const int g = stream_grid((const void*)k_probe_vec<NTV, NCV, uint32_t>, kThreads, smem, (n_left + 3) / 4, \
                                  G.cps);                                                                 \
        (note_launch(), k_probe_vec<NTV, NCV, uint32_t><<<g, kThreads, smem, s>>>(G, P, A, J->lkeys[0], J->kmin, \
                                                                                  J->n_slots, (const uint32_t*)map, n_left, holes)); \
        launched = true;                                                                                  \
    }
    TDG_PV(0, 0) TDG_PV(0, 1) TDG_PV(0, 2) TDG_PV(1, 1) TDG_PV(1, 2) TDG_PV(2, 1) TDG_PV(2, 2)
#undef TDG_PV
    if (!launched && holes) launch_map_holes(G, (const uint32_t*)map, J->n_slots, s);   // no vector form after all
#define TDG_PL(PKV, SMV, PT, W)                                                                         \
    if (!launched && pk == PKV && sm == SMV && w8 == W) {                                                \
        const int g = grid_for((const void*)k_payload_probe<PKV, SMV, PT, W>, kThreads, smem,            \
                               (n_left + kItems - 1) / kItems);                                          \
        (note_launch(), k_payload_probe<PKV, SMV, PT, W><<<g, kThreads, smem, s>>>(                      \
            G, P, prog, J->lkeys[0], J->kmin, J->n_slots, (const PT*)map, n_left));                      \
    }
    TDG_PL(0, true, uint32_t, true) TDG_PL(0, false, uint32_t, true)
    TDG_PL(1, true, uint32_t, true) TDG_PL(1, false, uint32_t, true)
    TDG_PL(0, true, uint32_t, false) TDG_PL(0, false, uint32_t, false)
    TDG_PL(1, true, uint32_t, false) TDG_PL(1, false, uint32_t, false)
    TDG_PL(2, true, uint32_t, false) TDG_PL(2, false, uint32_t, false)
#undef TDG_PL
    tm.stop(s);
    st = launch_status();
    if (st) { tm.ms(); tb.ms(); return st; }
    int32_t dup = 0;
    st = finish(G, d, ws, out, s, &dup);
    const float ms = tm.ms(), bms = tb.ms();
    if (st) return st;
    if (dup) return E_OK;                           // duplicate build keys: general path
    *used = true;
    if (tm.on) set_last_main_ms(ms);
    if (tb.on) set_last_build_ms(bms);
    return E_OK;
}

tdg_status group_run_joined(const tdg_group_desc* d, const tdg_group_plan* p, void* ws,
                            const tdg_expr* pred, const uint64_t* sel, const JoinK* J, int64_t n_left,
                            int64_t n_right, const tdg_group_out* out, cudaStream_t s) {
    if (p->method != TDG_GROUP_DIRECT && p->method != TDG_GROUP_HASH) return E_RANGE;
    GroupK G = make_gk(d, p, ws, d->nrows);
    tdg_status st = prepare(G, s);
    if (st) return st;
    int pk;
    Pred P = make_pred(pred, sel, &pk);
    static tdg_expr empty;
    const tdg_expr& prog = pred ? *pred : empty;
    EventTimer tm;
    if (J) {
        st = dispatch<true>(pk, G, p->smem != 0, P, prog, *J, n_left, s, tm);
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
        st = dispatch<false>(pk, G, p->smem != 0, P, prog, none, d->nrows, s, tm);
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
