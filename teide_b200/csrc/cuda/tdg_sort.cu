// Sort: the permutation that orders a table's rows by up to 16 keys, and the
// gather that applies it to a column.
//
// Replaces exec_sort (Teide src/ops/exec.c:3370-3862) for its radix-sortable
// key types.  Teide encodes every key as an order-preserving u64
// (radix_encode_fn, exec.c:2739-2840) and sorts the encoded keys with an
// 8-pass LSD radix sort carrying row indices (radix_sort_run, exec.c:2647-
// 2737); several keys are bit-packed into one composite when their ranges
// fit 64 bits.  Here each key is encoded the same way, the keys are applied
// from the last to the first with a stable LSD radix sort (8-bit digits), and
// the result -- stable, so equal keys keep their row order -- is the order
// Teide's radix path produces.  Only the digits that differ are sorted: the
// key range (max - min of the encoded keys) sets the number of passes.
//
// One pass over n keys: a per-tile digit histogram, a prefix over
// (digit, tile) in three coalesced steps, and a stable scatter in which every
// tile ranks its rows 1024 at a time (four 256-row sub-rounds, warp match
// masks), so rows of equal digit keep their order.  Keys move as 64 bits and
// row indices as 32 bits (n < 2^32); the permutation is widened to int64 last.
#include "tdg_common.cuh"
#include <string.h>

namespace tdg {

constexpr int kSortThreads = 256;
constexpr int kSortRounds = 16;                           // 256-row rounds per tile
constexpr int64_t kSortTile = (int64_t)kSortThreads * kSortRounds;
constexpr int kSortWarps = kSortThreads / 32;

// The order-preserving key of one row (radix_encode_fn, exec.c:2739-2800):
// integers flip the sign bit, F64 flips every bit of negatives and the sign
// of the rest (IEEE order, -0.0 before +0.0), NaN is the smallest or largest
// key by nulls_first, SYM reads the rank of its string, DESC complements.
// BOOL / U8 sort as unsigned bytes and I16 as signed (sort_cmp, exec.c:
// 2538-2547).  zero_eq encodes -0.0 as +0.0: the comparator Teide sorts
// with outside its radix path (sort_cmp, exec.c:2512-2521) finds them equal.
__device__ __forceinline__ uint64_t sort_encode(const tdg_sort_key& K, int64_t r, bool zero_eq) {
    const tdg_col& c = K.col;
    uint64_t e;
    switch (c.type) {
        case T_BOOL: case T_U8:
            e = ((const uint8_t*)c.data)[r];
            break;
        case T_I16:
            e = (uint64_t)((uint16_t)((const short*)c.data)[r] ^ 0x8000u);
            break;
        case T_I64: case T_TIMESTAMP:
            e = (uint64_t)((const long long*)c.data)[r] ^ (1ULL << 63);
            break;
        case T_I32: case T_DATE: case T_TIME:
            e = (uint64_t)((uint32_t)((const int*)c.data)[r] ^ (1u << 31));
            break;
        case T_F64: {
            uint64_t b = (uint64_t)__double_as_longlong(((const double*)c.data)[r]);
            if (zero_eq && b == (1ULL << 63)) b = 0;
            if ((b & 0x7FF0000000000000ULL) == 0x7FF0000000000000ULL && (b & 0x000FFFFFFFFFFFFFULL)) {
                const uint64_t nan_e = (K.nulls_first ^ K.desc) ? 0ULL : ~0ULL;
                return K.desc ? ~nan_e : nan_e;
            }
            e = b ^ ((0ULL - (b >> 63)) | (1ULL << 63));
            break;
        }
        case T_SYM: {
            const int w = elem_size(c.type, c.attrs);
            uint32_t id;
            if (w == 1) id = ((const uint8_t*)c.data)[r];
            else if (w == 2) id = ((const uint16_t*)c.data)[r];
            else if (w == 4) id = ((const uint32_t*)c.data)[r];
            else id = (uint32_t)((const long long*)c.data)[r];
            e = K.sym_rank[id];
            break;
        }
        default:
            e = 0;
            break;
    }
    return K.desc ? ~e : e;
}

// keys[i] = encoded key of row perm[i]; folds the min and max into mm[0..1].
__global__ void __launch_bounds__(kThreads) k_sort_encode(const tdg_sort_key K, const uint32_t* __restrict__ perm,
                                                          int64_t n, uint64_t* __restrict__ keys,
                                                          unsigned long long* mm, bool zero_eq) {
    unsigned long long lo = ~0ULL, hi = 0ULL;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t e = sort_encode(K, perm[i], zero_eq);
        keys[i] = e;
        lo = e < lo ? e : lo;
        hi = e > hi ? e : hi;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long a = __shfl_xor_sync(0xffffffffu, lo, o);
        const unsigned long long b = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(mm, lo);
        atomicMax(mm + 1, hi);
    }
}

// Row indices travel through the passes as 32 bits (n < 2^32); the result
// is widened to int64 once at the end.
__global__ void k_sort_iota(uint32_t* __restrict__ perm, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        perm[i] = (uint32_t)i;
}

__global__ void k_sort_widen(const uint32_t* __restrict__ in, int64_t n, int64_t* __restrict__ perm) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        perm[i] = in[i];
}

__global__ void k_sort_mm_init(unsigned long long* mm) { mm[0] = ~0ULL; mm[1] = 0ULL; }

// hist[d * n_tiles + tile]: rows of the tile whose digit ((key - kmin) >> shift) & 255 is d.
__global__ void __launch_bounds__(kSortThreads) k_sort_hist(const uint64_t* __restrict__ keys, int64_t n,
                                                             uint64_t kmin, int shift, uint32_t* __restrict__ hist,
                                                             int64_t n_tiles) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t t0 = blockIdx.x * kSortTile;
    for (int q = 0; q < kSortRounds; q++) {
        const int64_t i = t0 + (int64_t)q * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[((keys[i] - kmin) >> shift) & 255], 1u);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * n_tiles + blockIdx.x] = h[threadIdx.x];
}

// In-place exclusive prefix of a[0, m) in three steps: every CTA sums a
// segment of kScanSeg entries, one CTA scans those sums, and every CTA
// rescans its segment from its offset -- coalesced, and all SMs take part.
constexpr int kScanThreads = 1024;
constexpr int kScanPer = 4;
constexpr int64_t kScanSeg = (int64_t)kScanThreads * kScanPer;

__device__ __forceinline__ uint32_t block_incl_scan(uint32_t x, uint32_t* wsum) {
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (unsigned)o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < (blockDim.x >> 5) ? wsum[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (unsigned)o) w += y;
        }
        wsum[lane] = w;
    }
    __syncthreads();
    const uint32_t r = x + (warp ? wsum[warp - 1] : 0u);
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_sums(const uint32_t* __restrict__ a, int64_t m,
                                                            uint32_t* __restrict__ sums) {
    __shared__ uint32_t wsum[32];
    const int64_t b = blockIdx.x * kScanSeg + (int64_t)threadIdx.x * kScanPer;
    uint32_t t = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; k++) t += b + k < m ? a[b + k] : 0u;
    const uint32_t incl = block_incl_scan(t, wsum);
    if (threadIdx.x == blockDim.x - 1) sums[blockIdx.x] = incl;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_top(uint32_t* sums, int64_t nb) {
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    for (int64_t c = 0; c < nb; c += blockDim.x) {
        const int64_t i = c + threadIdx.x;
        const uint32_t v = i < nb ? sums[i] : 0u;
        const uint32_t incl = block_incl_scan(v, wsum);
        const uint32_t carry = s_carry;
        if (i < nb) sums[i] = carry + incl - v;
        __syncthreads();                                  // every thread has read the carry
        if (threadIdx.x == blockDim.x - 1) s_carry = carry + incl;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(uint32_t* __restrict__ a, int64_t m,
                                                             const uint32_t* __restrict__ offs) {
    __shared__ uint32_t wsum[32];
    const int64_t b = blockIdx.x * kScanSeg + (int64_t)threadIdx.x * kScanPer;
    uint32_t v[kScanPer], t = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
        v[k] = b + k < m ? a[b + k] : 0u;
        t += v[k];
    }
    uint32_t run = offs[blockIdx.x] + block_incl_scan(t, wsum) - t;
#pragma unroll
    for (int k = 0; k < kScanPer; k++) {
        if (b + k < m) a[b + k] = run;
        run += v[k];
    }
}

// The stable scatter of one pass.  A tile's rows go 1024 at a time, as four
// sub-rounds of 256 (row order = sub-round, then thread).  Every row's rank
// among the lanes of its warp and sub-round with the same digit comes from a
// warp match mask; after one barrier the thread that owns digit d turns the
// per-(sub-round, warp) counts into running offsets from the tile's base for
// d, and after a second every row writes at its offset plus its rank -- two
// barriers per 1024 rows, and rows of equal digit keep their order.
constexpr int kSortSub = 4;
static_assert(kSortRounds % kSortSub == 0, "a tile is a whole number of 1024-row rounds");

__global__ void __launch_bounds__(kSortThreads) k_sort_scatter(const uint64_t* __restrict__ kin,
                                                                const uint32_t* __restrict__ vin,
                                                                uint64_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                                int64_t n, uint64_t kmin, int shift,
                                                                const uint32_t* __restrict__ offs, int64_t n_tiles) {
    __shared__ uint32_t base[256];
    __shared__ uint8_t wc[kSortSub][kSortWarps][256];          // lanes of a warp per digit: at most 32
    __shared__ uint32_t pre[kSortSub][kSortWarps][256];
    base[threadIdx.x] = offs[(int64_t)threadIdx.x * n_tiles + blockIdx.x];
    for (int k = 0; k < kSortSub; k++)
        for (int w = 0; w < kSortWarps; w++) wc[k][w][threadIdx.x] = 0;
    __syncthreads();
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t t0 = blockIdx.x * kSortTile;
    for (int q = 0; q < kSortRounds; q += kSortSub) {
        uint64_t k[kSortSub];
        uint32_t v[kSortSub];
        uint32_t d[kSortSub], rank[kSortSub];
#pragma unroll
        for (int s = 0; s < kSortSub; s++) {
            const int64_t i = t0 + (int64_t)(q + s) * kSortThreads + threadIdx.x;
            const bool in = i < n;
            k[s] = in ? kin[i] : 0;
            v[s] = in ? vin[i] : 0;
            d[s] = in ? (uint32_t)(((k[s] - kmin) >> shift) & 255) : 256u;
        }
#pragma unroll
        for (int s = 0; s < kSortSub; s++) {
            const unsigned peers = __match_any_sync(0xffffffffu, d[s]);
            rank[s] = (uint32_t)__popc(peers & lt);
            if (d[s] < 256 && (peers & lt) == 0) wc[s][warp][d[s]] = (uint8_t)__popc(peers);
        }
        __syncthreads();
        {
            const unsigned dg = threadIdx.x;                     // this thread's digit
            uint32_t run = base[dg];
            for (int s = 0; s < kSortSub; s++)
                for (int w = 0; w < kSortWarps; w++) {
                    const uint32_t c = wc[s][w][dg];
                    pre[s][w][dg] = run;
                    run += c;
                    wc[s][w][dg] = 0;
                }
            base[dg] = run;
        }
        __syncthreads();
#pragma unroll
        for (int s = 0; s < kSortSub; s++) {
            if (d[s] >= 256) continue;
            const uint32_t pos = pre[s][warp][d[s]] + rank[s];
            kout[pos] = k[s];
            vout[pos] = v[s];
        }
    }
}

template <typename T>
__global__ void k_gather(const T* __restrict__ in, const int64_t* __restrict__ perm, int64_t n, T* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = in[perm[i]];
}

static bool sortable(const tdg_sort_key& k) {
    switch (k.col.type) {
        case T_I64: case T_TIMESTAMP: case T_I32: case T_DATE: case T_TIME: case T_F64:
        case T_BOOL: case T_U8: case T_I16: return true;
        case T_SYM: return k.sym_rank != nullptr;
        default: return false;
    }
}

struct SortWs {
    uint64_t* ka;
    uint64_t* kb;
    uint32_t* va;
    uint32_t* vb;
    uint32_t* hist;
    uint32_t* sums;
    unsigned long long* mm;
};

static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }
static int64_t scan_blocks(int64_t n_tiles) { return (n_tiles * 256 + kScanSeg - 1) / kScanSeg; }

// Two page-locked words per host thread for the key range read-back (the
// copy is asynchronous); pageable memory when allocation is not allowed.
static unsigned long long* pinned_pair() {
    static thread_local unsigned long long* w = nullptr;
    if (no_alloc()) return nullptr;
    if (!w && cudaMallocHost((void**)&w, 16) != cudaSuccess) { cudaGetLastError(); w = nullptr; }
    return w;
}

static SortWs sort_ws(void* ws, int64_t n) {
    SortWs W;
    char* p = (char*)ws;
    const size_t kb = al256((size_t)n * 8);
    const int64_t n_tiles = (n + kSortTile - 1) / kSortTile;
    W.ka = (uint64_t*)p; p += kb;
    W.kb = (uint64_t*)p; p += kb;
    W.va = (uint32_t*)p; p += kb;
    W.vb = (uint32_t*)p; p += kb;
    W.hist = (uint32_t*)p; p += al256((size_t)n_tiles * 256 * 4);
    W.sums = (uint32_t*)p; p += al256((size_t)scan_blocks(n_tiles) * 4);
    W.mm = (unsigned long long*)p;
    return W;
}

}  // namespace tdg

using namespace tdg;

extern "C" size_t tdg_sort_ws_bytes(int64_t n) {
    if (n < 0) n = 0;
    const int64_t n_tiles = (n + kSortTile - 1) / kSortTile;
    return 4 * al256((size_t)n * 8) + al256((size_t)n_tiles * 256 * 4) + al256((size_t)scan_blocks(n_tiles) * 4) + 256;
}

extern "C" tdg_status tdg_sort_perm(const tdg_sort_key* keys, int32_t n_keys, int64_t n, void* ws, int64_t* perm,
                                    void* stream) {
    if ((n_keys > 0 && !keys) || n_keys < 0 || n_keys > TDG_MAX_SORT_KEYS || n < 0) return E_RANGE;
    if (n > (int64_t)UINT32_MAX) return E_RANGE;                     // 32-bit positions in the scatter
    for (int k = 0; k < n_keys; k++) if (!sortable(keys[k])) return E_NYI;
    if (n == 0) return E_OK;
    if (!ws || !perm) return E_RANGE;
    cudaStream_t s = (cudaStream_t)stream;
    EventTimer tm;
    tm.start(s);
    SortWs W = sort_ws(ws, n);
    const int64_t n_tiles = (n + kSortTile - 1) / kSortTile;
    const int g = grid_for((const void*)k_sort_iota, kThreads, 0, n);
    (note_launch(), k_sort_iota<<<g, kThreads, 0, s>>>(W.va, n));
    uint32_t* cur = W.va;
    uint32_t* alt = W.vb;
    // Teide radix-sorts one key of a radix type over more than 64 rows
    // (exec.c:3426-3453); every other case goes through sort_cmp, where
    // -0.0 equals +0.0.  Several keys of radix types pack into one composite
    // only when their ranges fit 64 bits, which a key holding both zeros
    // (a 64-bit range) never does, so treating the zeros as equal there is
    // the composite's order as well.
    bool zero_eq = n <= 64 || n_keys > 1;
    for (int k = 0; k < n_keys; k++) {
        const int t = keys[k].col.type;
        if (t == T_BOOL || t == T_U8 || t == T_I16) zero_eq = true;
    }
    unsigned long long* mmh = pinned_pair();
    unsigned long long mm_local[2];
    tdg_status st = E_OK;
    // the last key first: a stable sort by each earlier key keeps the later ones' order within ties
    for (int k = n_keys - 1; k >= 0 && !st; k--) {
        (note_launch(), k_sort_mm_init<<<1, 1, 0, s>>>(W.mm));
        const int ge = grid_for((const void*)k_sort_encode, kThreads, 0, n);
        (note_launch(), k_sort_encode<<<ge, kThreads, 0, s>>>(keys[k], cur, n, W.ka, W.mm, zero_eq));
        unsigned long long* mm = mmh ? mmh : mm_local;
        if (cudaMemcpyAsync(mm, W.mm, 16, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) { st = launch_status(); if (!st) st = E_IO; break; }
        const uint64_t kmin = mm[0], range = mm[1] - mm[0];
        int bits = 0;
        while (bits < 64 && (range >> bits) != 0) bits++;
        uint64_t* kc = W.ka;
        uint64_t* kd = W.kb;
        for (int shift = 0; shift < bits; shift += 8) {
            (note_launch(), k_sort_hist<<<(unsigned)n_tiles, kSortThreads, 0, s>>>(kc, n, kmin, shift, W.hist, n_tiles));
            const int64_t m = n_tiles * 256, nb = (m + kScanSeg - 1) / kScanSeg;
            (note_launch(), k_scan_sums<<<(unsigned)nb, kScanThreads, 0, s>>>(W.hist, m, W.sums));
            (note_launch(), k_scan_top<<<1, kScanThreads, 0, s>>>(W.sums, nb));
            (note_launch(), k_scan_apply<<<(unsigned)nb, kScanThreads, 0, s>>>(W.hist, m, W.sums));
            (note_launch(), k_sort_scatter<<<(unsigned)n_tiles, kSortThreads, 0, s>>>(kc, cur, kd, alt, n, kmin, shift,
                                                                                     W.hist, n_tiles));
            uint64_t* tk = kc; kc = kd; kd = tk;
            uint32_t* tv = cur; cur = alt; alt = tv;
        }
        st = launch_status();
    }
    if (!st) (note_launch(), k_sort_widen<<<g, kThreads, 0, s>>>(cur, n, perm));
    if (!st) st = launch_status();
    tm.stop(s);
    if (tm.on) {
        if (!st && cudaStreamSynchronize(s) != cudaSuccess) st = E_IO;
        const float ms = tm.ms();
        if (!st) set_last_sort_ms(ms);
    }
    return st;
}

extern "C" tdg_status tdg_gather(const tdg_col* in, const int64_t* perm, int64_t n_out, void* out, void* stream) {
    if (!in || n_out < 0) return E_RANGE;
    if (n_out == 0) return E_OK;
    if (!in->data || !perm || !out) return E_RANGE;
    cudaStream_t s = (cudaStream_t)stream;
    const int w = elem_size(in->type, in->attrs);
    const int g = grid_for((const void*)k_gather<long long>, kThreads, 0, n_out);
    switch (w) {
        case 1: (note_launch(), k_gather<uint8_t><<<g, kThreads, 0, s>>>((const uint8_t*)in->data, perm, n_out, (uint8_t*)out)); break;
        case 2: (note_launch(), k_gather<uint16_t><<<g, kThreads, 0, s>>>((const uint16_t*)in->data, perm, n_out, (uint16_t*)out)); break;
        case 4: (note_launch(), k_gather<uint32_t><<<g, kThreads, 0, s>>>((const uint32_t*)in->data, perm, n_out, (uint32_t*)out)); break;
        case 8: (note_launch(), k_gather<unsigned long long><<<g, kThreads, 0, s>>>((const unsigned long long*)in->data, perm, n_out, (unsigned long long*)out)); break;
        default: return E_TYPE;
    }
    return launch_status();
}
