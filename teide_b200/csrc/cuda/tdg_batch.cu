// Batched group-by: many independent queries in one persistent launch.
//
// Teide runs each group-by as its own exec_group call (exec.c:5542-6879),
// with its own thread-pool dispatches.  For thousands of small or uneven
// queries the per-query launch and synchronization cost dominates on a GPU,
// so here all queries of one shape share one launch:
//
//   work items   each query is cut into tiles of tile_rows rows; a CTA takes
//                the next item from a global counter (atomicAdd), so long and
//                short queries balance across the 148 SMs;
//   accumulate   a query with at most smem_slots slots (and a tile at least
//                twice that long) aggregates its tile in shared memory and
//                merges once; a query with more slots but at least
//                kRowsPerSlot rows per slot is cut into at most
//                kMaxSlices key slices of at most smem_slots slots, and an
//                item is then a (tile, slice) pair that aggregates only its
//                slice's rows in shared memory (the slices of a tile are
//                consecutive items, so the tile's columns are read from DRAM
//                once and from L2 by the others); the remaining tiles update
//                the query's slot records in global memory (L2-resident per
//                query);
//   emit         one CTA per query writes its non-empty slots, keys ascending,
//                at the query's offset from an exclusive scan of group counts.
//
// tdg_batch_run issues only kernels and memsets on the given stream (no
// allocation, no host synchronization), so the host can capture it once in
// a CUDA graph and replay it; tdg_batch_prepare writes the work description
// (per-query descriptors and the item -> query map) into the workspace.
#include "tdg_common.cuh"
#include <string.h>
#include <vector>

namespace tdg {

constexpr int kBatchThreads = 256;
constexpr int kBatchMaxThreads = 1024;
constexpr int64_t kDefaultTile = 16384;
constexpr int kStaticSmemReserve = 256;   // the kernel's own __shared__ words
constexpr int64_t kRowsPerSlot = 8;       // shared-path tiles hold >= 8 rows per slot
constexpr int64_t kMaxSlices = 8;         // more key slices than this: global records instead
constexpr int kBR = 4;                    // rows per thread per chunk
constexpr int kEmitBlock = 256;
constexpr int64_t kMaxDenseSlots = 1 << 20;

enum : int32_t { BK_COUNT = 0, BK_SUM_I, BK_SUM_F, BK_MIN_I, BK_MAX_I, BK_MIN_F, BK_MAX_F };

struct BQ {
    tdg_col key, val;
    int64_t nrows, key_min, n_slots, acc_off, first_item, tile_rows;
    int64_t n_slices, slice_slots;    // key slices per tile (1: the whole key range)
};

struct BatchK {
    const BQ* q;
    const int32_t* item_q;
    int64_t n_items, total_slots;
    unsigned long long* rec;
    unsigned long long* counter;
    int32_t* err;
    const volatile int32_t* cancel;  // host-mapped cancel word (pool.c:485-489's per-task check)
    int32_t* stop;                   // device copy of a seen cancel, read per work item
    const int32_t* piece_q;       // emit piece -> query
    const int64_t* piece_s0;      // emit piece -> first slot within the query
    int64_t* pcount;              // groups per piece, then exclusive offsets
    int64_t n_pieces;
    int32_t n_queries, W, na, smem_slots, query_base;
    int32_t kind[TDG_MAX_AGGS];
    int32_t ai[TDG_MAX_AGGS];
    int32_t op[TDG_MAX_AGGS];
    unsigned long long finit[TDG_MAX_AGGS + 2];
};

struct BLayout { size_t hdr, q, item_q, piece_q, piece_s0, pcount, rec, total; };

static size_t al(size_t x) { return (x + 255) & ~(size_t)255; }

constexpr int64_t kPiece = 4096;          // slots one emit CTA handles

static BLayout blayout(int64_t n_queries, int64_t n_items, int64_t total_slots, int W, int64_t n_pieces) {
    BLayout L;
    size_t o = 0;
    L.hdr = o; o += 256;
    L.q = o; o += al((size_t)n_queries * sizeof(BQ));
    L.item_q = o; o += al((size_t)n_items * 4);
    L.piece_q = o; o += al((size_t)n_pieces * 4);
    L.piece_s0 = o; o += al((size_t)n_pieces * 8);
    L.pcount = o; o += al((size_t)(n_pieces + 1) * 8);
    L.rec = o; o += al((size_t)total_slots * 8 * W);
    L.total = o;
    return L;
}

__host__ __device__ inline unsigned long long binit(int kind) {
    return (kind == BK_MIN_I || kind == BK_MIN_F) ? (unsigned long long)INT64_MAX
         : (kind == BK_MAX_I || kind == BK_MAX_F) ? (unsigned long long)INT64_MIN : 0ULL;
}

static BatchK make_bk(const tdg_batch_plan* p, void* ws) {
    BatchK B;
    memset(&B, 0, sizeof(B));
    const BLayout L = blayout(p->n_queries, p->n_items, p->total_slots, p->words, p->n_pieces);
    char* w = (char*)ws;
    B.counter = (unsigned long long*)(w + L.hdr);
    B.err = (int32_t*)(w + L.hdr + 16);
    B.stop = (int32_t*)(w + L.hdr + 32);
    B.cancel = p->cancel;
    B.q = (const BQ*)(w + L.q);
    B.item_q = (const int32_t*)(w + L.item_q);
    B.piece_q = (const int32_t*)(w + L.piece_q);
    B.piece_s0 = (const int64_t*)(w + L.piece_s0);
    B.pcount = (int64_t*)(w + L.pcount);
    B.n_pieces = p->n_pieces;
    B.rec = (unsigned long long*)(w + L.rec);
    B.n_items = p->n_items;
    B.total_slots = p->total_slots;
    B.n_queries = p->n_queries;
    B.W = p->words;
    B.na = p->n_aggs;
    B.smem_slots = p->smem_slots;
    B.query_base = p->query_base;
    int ai = 0;
    for (int a = 0; a < p->n_aggs; a++) {
        const int op = p->agg_ops[a], f = p->val_f64;
        B.op[a] = op;
        B.kind[a] = op == A_COUNT ? BK_COUNT : op == A_MIN ? (f ? BK_MIN_F : BK_MIN_I)
                  : op == A_MAX ? (f ? BK_MAX_F : BK_MAX_I) : (f ? BK_SUM_F : BK_SUM_I);
        B.ai[a] = op == A_COUNT ? -1 : ai++;
        if (B.ai[a] >= 0) B.finit[1 + B.ai[a]] = binit(B.kind[a]);
    }
    return B;
}

__global__ void k_batch_init(const BatchK B) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int W = B.W;
    const int step = 32 % W;
    const int64_t nchunks = (B.total_slots + 31) >> 5;
    for (int64_t ch = warp; ch < nchunks; ch += nwarps) {
        const int64_t recs = B.total_slots - ch * 32 < 32 ? B.total_slots - ch * 32 : 32;
        const int words = (int)(recs * W);
        unsigned long long* base = B.rec + ch * 32 * W;
        int f = lane % W;
        for (int j = lane; j < words; j += 32) {
            base[j] = B.finit[f];
            f += step;
            if (f >= W) f -= W;
        }
    }
}

__device__ __forceinline__ void bupd(unsigned long long* a, int kind, int64_t iv, double fv, bool global) {
    // global MIN/MAX: an L2 read filters updates that cannot win; the stored
    // extreme only moves toward the row's value, so a stale read never loses one
    switch (kind) {
        case BK_SUM_I: atomicAdd(a, (unsigned long long)iv); break;
        case BK_SUM_F: atomicAdd((double*)a, fv); break;
        case BK_MIN_I:
            if (!global || iv < __ldcg((const long long*)a)) atomicMin((long long*)a, (long long)iv);
            break;
        case BK_MAX_I:
            if (!global || iv > __ldcg((const long long*)a)) atomicMax((long long*)a, (long long)iv);
            break;
        case BK_MIN_F:
            if (fv == fv) {
                const long long o = f2ord(fv);
                if (!global || o < __ldcg((const long long*)a)) atomicMin((long long*)a, o);
            }
            break;
        case BK_MAX_F:
            if (fv == fv) {
                const long long o = f2ord(fv);
                if (!global || o > __ldcg((const long long*)a)) atomicMax((long long*)a, o);
            }
            break;
        default: break;
    }
}

__device__ __forceinline__ void bmerge(unsigned long long* a, int kind, unsigned long long v) {
    switch (kind) {
        case BK_SUM_I: atomicAdd(a, v); break;
        case BK_SUM_F: atomicAdd((double*)a, __longlong_as_double((long long)v)); break;
        case BK_MIN_I: case BK_MIN_F: if ((long long)v != INT64_MAX) atomicMin((long long*)a, (long long)v); break;
        case BK_MAX_I: case BK_MAX_F: if ((long long)v != INT64_MIN) atomicMax((long long*)a, (long long)v); break;
        default: break;
    }
}

// The persistent kernel: CTAs pull (query, tile) items until the queue drains.
__global__ void __launch_bounds__(kBatchMaxThreads) k_batch_agg(const BatchK B) {
    extern __shared__ unsigned long long sm[];
    __shared__ long long s_item;
    uint32_t* scnt = (uint32_t*)sm;
    unsigned long long* sacc = sm + ((B.smem_slots * 4 + 7) >> 3);
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            long long it = (long long)atomicAdd(B.counter, 1ULL);
            if (B.cancel) {
                // the host word is read over the link by every 64th claim only
                // (one read per claim measured 2x slower on a 4096-query
                // batch); a cancel seen there stops every CTA at its next claim
                if ((it & 63) == 0 && *B.cancel) atomicExch(B.stop, 1);
                if (*(volatile int32_t*)B.stop) it = B.n_items;   // cancelled: take no further item
            }
            s_item = it;
        }
        __syncthreads();
        const int64_t item = s_item;
        if (item >= B.n_items) break;
        const int q = B.item_q[item];
        const BQ Q = B.q[q];
        const int64_t local = item - Q.first_item;
        const int64_t tix = local / Q.n_slices, six = local - tix * Q.n_slices;
        const int64_t r0 = tix * Q.tile_rows;
        const int64_t r1 = r0 + Q.tile_rows < Q.nrows ? r0 + Q.tile_rows : Q.nrows;
        const bool sliced = Q.n_slices > 1;
        const int64_t s_lo = six * Q.slice_slots;
        const bool use_smem = sliced || (Q.n_slots <= B.smem_slots && (r1 - r0) >= 2 * Q.n_slots);
        const int64_t S = sliced ? (Q.n_slots - s_lo < Q.slice_slots ? Q.n_slots - s_lo : Q.slice_slots) : Q.n_slots;
        if (use_smem) {
            for (int64_t s = threadIdx.x; s < S; s += blockDim.x) scnt[s] = 0;
            for (int a = 0; a < B.na; a++)
                if (B.ai[a] >= 0)
                    for (int64_t s = threadIdx.x; s < S; s += blockDim.x) sacc[B.ai[a] * S + s] = B.finit[1 + B.ai[a]];
            __syncthreads();
        }
        // rows in chunks of kBR per thread: the chunk's loads issue together,
        // and the CTA keeps the chunk two ahead in flight as an L2 prefetch
        const int64_t chunk = (int64_t)blockDim.x * kBR;
        const int vsz = elem_size(Q.val.type, Q.val.attrs), ksz = elem_size(Q.key.type, Q.key.attrs);
        if (threadIdx.x < 2) {
            const int64_t e = r0 + 2 * chunk < r1 ? r0 + 2 * chunk : r1;
            const tdg_col& c = threadIdx.x ? Q.val : Q.key;
            const int64_t z = threadIdx.x ? vsz : ksz;
            l2_prefetch((const char*)c.data + r0 * z, (e - r0) * z);
        }
        const bool vf = Q.val.type == T_F64;
        for (int64_t c0 = r0; c0 < r1; c0 += chunk) {
            if (threadIdx.x < 2) {
                const int64_t p0 = c0 + 2 * chunk, p1 = p0 + chunk < r1 ? p0 + chunk : r1;
                if (p0 < p1) {
                    const tdg_col& c = threadIdx.x ? Q.val : Q.key;
                    const int64_t z = threadIdx.x ? vsz : ksz;
                    l2_prefetch((const char*)c.data + p0 * z, (p1 - p0) * z);
                }
            }
            int64_t k[kBR], iv[kBR];
            double fv[kBR];
            bool ok[kBR];
#pragma unroll
            for (int j = 0; j < kBR; j++) {
                const int64_t r = c0 + j * (int64_t)blockDim.x + threadIdx.x;
                ok[j] = r < r1;
                k[j] = ok[j] ? ld_i(Q.key, r) - Q.key_min : 0;
                fv[j] = ok[j] && vf ? ld_f(Q.val, r) : 0.0;
                iv[j] = ok[j] && !vf ? ld_i(Q.val, r) : 0;
            }
#pragma unroll
            for (int j = 0; j < kBR; j++)
                if (ok[j] && (k[j] < 0 || k[j] >= Q.n_slots)) {
                    if (six == 0) atomicCAS(B.err, 0, E_DOMAIN);     // reported once, by the first slice
                    ok[j] = false;
                }
            if (sliced) {
#pragma unroll
                for (int j = 0; j < kBR; j++) {
                    k[j] -= s_lo;
                    ok[j] = ok[j] && k[j] >= 0 && k[j] < S;        // another slice's row
                }
            }
            if (use_smem) {
#pragma unroll
                for (int j = 0; j < kBR; j++) if (ok[j]) atomicAdd(&scnt[k[j]], 1u);
                for (int a = 0; a < B.na; a++)
                    if (B.ai[a] >= 0) {
#pragma unroll
                        for (int j = 0; j < kBR; j++)
                            if (ok[j]) bupd(&sacc[B.ai[a] * S + k[j]], B.kind[a], iv[j], fv[j], false);
                    }
            } else {
                unsigned long long* base = B.rec + Q.acc_off * B.W;
#pragma unroll
                for (int j = 0; j < kBR; j++) if (ok[j]) atomicAdd(base + k[j] * B.W, 1ULL);
                for (int a = 0; a < B.na; a++) {
                    const int kind = B.kind[a];
                    if (B.ai[a] < 0) continue;
                    const int w = 1 + B.ai[a];
                    if (kind == BK_SUM_I || kind == BK_SUM_F) {
#pragma unroll
                        for (int j = 0; j < kBR; j++)
                            if (ok[j]) bupd(base + k[j] * B.W + w, kind, iv[j], fv[j], true);
                        continue;
                    }
                    // MIN/MAX: the four rows' current values are read together (one
                    // L2 round trip, not four), then only the rows that can win update
                    const bool fk = kind == BK_MIN_F || kind == BK_MAX_F;
                    const bool mn = kind == BK_MIN_I || kind == BK_MIN_F;
                    long long cur[kBR], v[kBR];
#pragma unroll
                    for (int j = 0; j < kBR; j++) {
                        v[j] = fk ? f2ord(fv[j]) : iv[j];
                        cur[j] = ok[j] ? __ldcg((const long long*)(base + k[j] * B.W + w)) : 0;
                    }
#pragma unroll
                    for (int j = 0; j < kBR; j++) {
                        if (!ok[j] || (fk && fv[j] != fv[j])) continue;
                        long long* t = (long long*)(base + k[j] * B.W + w);
                        if (mn) { if (v[j] < cur[j]) atomicMin(t, v[j]); }
                        else if (v[j] > cur[j]) atomicMax(t, v[j]);
                    }
                }
            }
        }
        if (use_smem) {
            __syncthreads();
            for (int64_t s = threadIdx.x; s < S; s += blockDim.x) {
                const uint32_t c = scnt[s];
                if (!c) continue;
                unsigned long long* rec = B.rec + (Q.acc_off + s_lo + s) * B.W;
                atomicAdd(rec, (unsigned long long)c);
                for (int a = 0; a < B.na; a++)
                    if (B.ai[a] >= 0) bmerge(rec + 1 + B.ai[a], B.kind[a], sacc[B.ai[a] * S + s]);
            }
        }
    }
}

// Emit runs in pieces of kPiece slots (one CTA each), so a query with a wide
// key range is counted and written by many CTAs; pieces are ordered by query,
// then slot, so the scan of piece counts keeps queries in order and keys
// ascending within a query.
__global__ void __launch_bounds__(kEmitBlock) k_batch_count(const BatchK B) {
    __shared__ int red[32];
    const int64_t i = blockIdx.x;
    const BQ& Q = B.q[B.piece_q[i]];
    const int64_t s0 = B.piece_s0[i], s1 = s0 + kPiece < Q.n_slots ? s0 + kPiece : Q.n_slots;
    int c = 0;
    for (int64_t s = s0 + threadIdx.x; s < s1; s += blockDim.x) c += B.rec[(Q.acc_off + s) * B.W] != 0;
    int tot;
    block_excl_scan(c, &tot, red);
    if (threadIdx.x == 0) B.pcount[i] = tot;
}

__global__ void __launch_bounds__(1024) k_batch_scan(const BatchK B, int64_t* d_total) {
    __shared__ long long part[1024];
    const int64_t m = B.n_pieces;
    const int64_t per = (m + blockDim.x - 1) / blockDim.x;
    const int64_t b = threadIdx.x * per, e = b + per < m ? b + per : m;
    long long sum = 0;
    for (int64_t i = b; i < e; i++) sum += B.pcount[i];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int o = 1; o < (int)blockDim.x; o <<= 1) {
        long long v = threadIdx.x >= (unsigned)o ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    long long run = threadIdx.x ? part[threadIdx.x - 1] : 0;
    for (int64_t i = b; i < e; i++) { const long long c = B.pcount[i]; B.pcount[i] = run; run += c; }
    if (threadIdx.x == blockDim.x - 1) {
        B.pcount[m] = part[blockDim.x - 1];
        // a key outside its query's [key_min, key_min + n_slots) range is
        // reported as a negative row count (the host maps it to an error)
        *d_total = *(volatile int32_t*)B.err ? -1 : part[blockDim.x - 1];
    }
}

struct BOut {
    int64_t* query;
    int64_t* key;
    void* aggs[TDG_MAX_AGGS];
};

__global__ void __launch_bounds__(kEmitBlock) k_batch_emit(const BatchK B, const BOut O) {
    __shared__ int red[32];
    const int64_t i = blockIdx.x;
    const int q = B.piece_q[i];
    const BQ& Q = B.q[q];
    const int64_t p0 = B.piece_s0[i], p1 = p0 + kPiece < Q.n_slots ? p0 + kPiece : Q.n_slots;
    int64_t out = B.pcount[i];
    for (int64_t s0 = p0; s0 < p1; s0 += blockDim.x) {
        const int64_t s = s0 + threadIdx.x;
        const unsigned long long* rec = s < p1 ? B.rec + (Q.acc_off + s) * B.W : nullptr;
        const unsigned long long c = rec ? rec[0] : 0;
        int tot;
        const int pre = block_excl_scan(c ? 1 : 0, &tot, red);
        if (c) {
            const int64_t o = out + pre;
            O.query[o] = (int64_t)q + B.query_base;
            O.key[o] = Q.key_min + s;
            for (int a = 0; a < B.na; a++) {
                const int kind = B.kind[a];
                uint64_t r;
                if (kind == BK_COUNT) {
                    r = c;
                } else {
                    const unsigned long long v = rec[1 + B.ai[a]];
                    if (B.op[a] == A_AVG) {
                        const double sum = kind == BK_SUM_F ? __longlong_as_double((long long)v) : (double)(long long)v;
                        r = (uint64_t)__double_as_longlong(sum / (double)c);
                    } else if (kind == BK_MIN_F || kind == BK_MAX_F) {
                        r = (uint64_t)__double_as_longlong(ord2f((long long)v));
                    } else {
                        r = v;
                    }
                }
                ((uint64_t*)O.aggs[a])[o] = r;
            }
        }
        out += tot;
    }
}

}  // namespace tdg

using namespace tdg;

// Key slices per tile: more than one when the query's slots exceed shared
// memory but it has at least kRowsPerSlot rows per slot.  (Slicing from two
// rows per slot measured no faster on the 4096-query batch.)
static int64_t query_slices(const tdg_batch_query& q, const tdg_batch_plan* p) {
    if (q.n_slots <= p->smem_slots || p->smem_slots < 1 || q.nrows < kRowsPerSlot * q.n_slots) return 1;
    const int64_t n = (q.n_slots + p->smem_slots - 1) / p->smem_slots;
    return n <= kMaxSlices ? n : 1;
}

// Per-query tile: a query aggregated in shared memory (whole or by key slice)
// gets tiles of at least kRowsPerSlot rows per slot of its key range (fewer
// flushes of its shared aggregates).
static int64_t query_tile(const tdg_batch_query& q, const tdg_batch_plan* p) {
    if (q.n_slots <= p->smem_slots || query_slices(q, p) > 1) {
        const int64_t t = q.n_slots * kRowsPerSlot;
        return t > p->tile_rows ? t : p->tile_rows;
    }
    return p->tile_rows;
}

// Work items of a query: its tiles times its key slices.
static int64_t query_items(const tdg_batch_query& q, const tdg_batch_plan* p) {
    const int64_t t = query_tile(q, p);
    return (q.nrows + t - 1) / t * query_slices(q, p);
}

extern "C" tdg_status tdg_batch_plan_make(const tdg_batch_desc* d, int64_t tile_rows, int32_t ctas_per_sm,
                                          tdg_batch_plan* p) {
    if (!d || !p || (d->n_queries > 0 && !d->queries)) return E_TYPE;
    if (d->n_aggs < 1 || d->n_aggs > TDG_MAX_AGGS || d->n_queries < 0) return E_NYI;
    memset(p, 0, sizeof(*p));
    p->tile_rows = tile_rows > 0 ? tile_rows : kDefaultTile;
    p->ctas_per_sm = ctas_per_sm > 0 ? ctas_per_sm : 0;
    p->n_queries = d->n_queries;
    p->n_aggs = d->n_aggs;
    int n_acc = 0;
    for (int a = 0; a < d->n_aggs; a++) {
        const int op = d->agg_ops[a];
        if (op != A_SUM && op != A_COUNT && op != A_MIN && op != A_MAX && op != A_AVG) return E_NYI;
        p->agg_ops[a] = op;
        n_acc += op != A_COUNT;
    }
    p->words = 1 + n_acc == 3 ? 4 : 1 + n_acc;
    // 1 CTA per SM: 1024 threads and most of the SM's shared memory; 2: 512
    // threads and half of it; otherwise 256 threads in the default 48 KB.
    // The kernel's static __shared__ words come out of the same budget.
    size_t budget = 48 * 1024;
    p->threads = kBatchThreads;
    if (p->ctas_per_sm == 1 || p->ctas_per_sm == 2) {
        int optin = 0, dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess || optin <= 0) {
            cudaGetLastError();
            optin = 48 * 1024;
        }
        budget = p->ctas_per_sm == 1 ? (size_t)optin : (size_t)optin / 2;
        p->threads = p->ctas_per_sm == 1 ? 1024 : 512;
    }
    budget -= kStaticSmemReserve;
    // shared accumulators: 32-bit counts + n_acc 8-byte values per slot
    p->smem_slots = (int32_t)((budget - 8) / (4 + 8 * (size_t)n_acc));
    p->smem_bytes = (int32_t)(((((size_t)p->smem_slots * 4) + 7) & ~(size_t)7) + (size_t)p->smem_slots * 8 * n_acc);
    p->val_f64 = d->n_queries > 0 && d->queries[0].val.type == T_F64;
    int64_t pieces = 0;
    for (int i = 0; i < d->n_queries; i++) {
        const tdg_batch_query& q = d->queries[i];
        if (!is_int_class(q.key.type) || !elem_size(q.val.type, q.val.attrs)) return E_TYPE;
        if ((q.val.type == T_F64) != (p->val_f64 != 0)) return E_TYPE;
        if (q.n_slots < 1 || q.nrows < 0) return E_RANGE;
        // direct-indexed records only: a key range far wider than the query
        // (sparse keys) belongs to the hash-table group-by, not the batch
        if (q.n_slots > kMaxDenseSlots && q.n_slots > 4 * q.nrows) return E_NYI;
        p->n_items += query_items(q, p);
        p->total_slots += q.n_slots;
        pieces += (q.n_slots + kPiece - 1) / kPiece;
    }
    if (p->n_items > INT32_MAX || pieces > INT32_MAX) return E_RANGE;
    p->n_pieces = (int32_t)pieces;
    p->ws_bytes = blayout(p->n_queries, p->n_items, p->total_slots, p->words, p->n_pieces).total;
    return E_OK;
}

extern "C" tdg_status tdg_batch_prepare(const tdg_batch_desc* d, const tdg_batch_plan* p, void* ws, void* stream) {
    if (!d || !p || !ws) return E_TYPE;
    const BLayout L = blayout(p->n_queries, p->n_items, p->total_slots, p->words, p->n_pieces);
    std::vector<BQ> qs((size_t)p->n_queries);
    std::vector<int32_t> item_q((size_t)p->n_items);
    std::vector<int32_t> piece_q((size_t)p->n_pieces);
    std::vector<int64_t> piece_s0((size_t)p->n_pieces);
    int64_t piece = 0;
    int64_t acc = 0, item = 0;
    for (int i = 0; i < p->n_queries; i++) {
        const tdg_batch_query& q = d->queries[i];
        BQ& b = qs[i];
        b.key = q.key; b.val = q.val;
        b.nrows = q.nrows; b.key_min = q.key_min; b.n_slots = q.n_slots;
        b.acc_off = acc;
        b.first_item = item;
        b.tile_rows = query_tile(q, p);
        b.n_slices = query_slices(q, p);
        b.slice_slots = (q.n_slots + b.n_slices - 1) / b.n_slices;
        const int64_t items = query_items(q, p);
        if (item + items > p->n_items) return E_RANGE;
        for (int64_t t = 0; t < items; t++) item_q[(size_t)(item + t)] = i;
        item += items;
        acc += q.n_slots;
        for (int64_t s0 = 0; s0 < q.n_slots && piece < p->n_pieces; s0 += kPiece, piece++) {
            piece_q[(size_t)piece] = i;
            piece_s0[(size_t)piece] = s0;
        }
    }
    if (item != p->n_items || acc != p->total_slots || piece != p->n_pieces) return E_RANGE;
    if (p->smem_bytes > 48 * 1024 &&
        cudaFuncSetAttribute((const void*)k_batch_agg, cudaFuncAttributeMaxDynamicSharedMemorySize, p->smem_bytes) != cudaSuccess) {
        cudaGetLastError();
        return E_IO;
    }
    cudaStream_t s = (cudaStream_t)stream;
    char* w = (char*)ws;
    if (cudaMemsetAsync(w + L.hdr, 0, 256, s) != cudaSuccess ||
        (p->n_queries && cudaMemcpyAsync(w + L.q, qs.data(), qs.size() * sizeof(BQ), cudaMemcpyHostToDevice, s) != cudaSuccess) ||
        (p->n_items && cudaMemcpyAsync(w + L.item_q, item_q.data(), item_q.size() * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) ||
        (p->n_pieces && cudaMemcpyAsync(w + L.piece_q, piece_q.data(), piece_q.size() * 4, cudaMemcpyHostToDevice, s) != cudaSuccess) ||
        (p->n_pieces && cudaMemcpyAsync(w + L.piece_s0, piece_s0.data(), piece_s0.size() * 8, cudaMemcpyHostToDevice, s) != cudaSuccess) ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        return E_IO;
    }
    return E_OK;
}

extern "C" tdg_status tdg_batch_run(const tdg_batch_plan* p, void* ws, const tdg_batch_out* out, void* stream) {
    if (!p || !ws || !out) return E_TYPE;
    cudaStream_t s = (cudaStream_t)stream;
    BatchK B = make_bk(p, ws);
    cudaMemsetAsync(B.counter, 0, 256, s);   // work counter and error word
    if (p->total_slots > 0) {
        const int g = grid_for((const void*)k_batch_init, kThreads, 0, (p->total_slots * p->words + 31) / 32 * 32);
        (note_launch(), k_batch_init<<<g, kThreads, 0, s>>>(B));
    }
    const size_t smem = (size_t)p->smem_bytes;
    const int threads = p->threads > 0 ? p->threads : kBatchThreads;
    if (p->n_items > 0) {
        int per_sm = p->ctas_per_sm;
        if (per_sm <= 0) {
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)k_batch_agg, threads, smem) != cudaSuccess || per_sm < 1)
                per_sm = 1;
        }
        int64_t g = (int64_t)per_sm * sm_count();
        if (g > p->n_items) g = p->n_items;
        // instrumentation: time the aggregation kernel, never inside a capture
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) cs = cudaStreamCaptureStatusActive;
        EventTimer t;
        const bool timed = cs == cudaStreamCaptureStatusNone && timing_on();
        if (timed) t.start(s);
        (note_launch(), k_batch_agg<<<(unsigned)g, threads, smem, s>>>(B));
        if (timed) {
            t.stop(s);
            cudaEventSynchronize(t.b);
            set_last_main_ms(t.ms());
        }
    }
    BOut O;
    memset(&O, 0, sizeof(O));
    O.query = out->query;
    O.key = out->key;
    for (int a = 0; a < p->n_aggs; a++) O.aggs[a] = out->aggs[a];
    if (p->n_queries > 0) {
        (note_launch(), k_batch_count<<<(unsigned)p->n_pieces, kEmitBlock, 0, s>>>(B));
        (note_launch(), k_batch_scan<<<1, 1024, 0, s>>>(B, out->d_n_rows));
        (note_launch(), k_batch_emit<<<(unsigned)p->n_pieces, kEmitBlock, 0, s>>>(B, O));
    } else {
        cudaMemsetAsync(out->d_n_rows, 0, 8, s);
    }
    return launch_status();
}
