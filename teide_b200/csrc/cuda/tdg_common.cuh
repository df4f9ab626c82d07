// Device-side building blocks shared by the tdg kernels: typed column loads,
// the expression interpreter, the conjunctive-predicate fast path, block-wide
// scans and launch helpers.  Everything is written for sm_100a: 32-lane
// warps, 148 SMs, 228 KB shared memory per SM.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "tdg.h"

namespace tdg {

// Teide type tags and aggregate opcodes (include/teide/td.h; the values are
// part of the ABI and are checked against the header by tests/test_abi.py).
enum : int8_t {
    T_BOOL = 1, T_U8 = 2, T_CHAR = 3, T_I16 = 4, T_I32 = 5, T_I64 = 6, T_F64 = 7,
    T_DATE = 9, T_TIME = 10, T_TIMESTAMP = 11, T_SYM = 20
};
enum : int32_t { A_SUM = 50, A_MIN = 52, A_MAX = 53, A_COUNT = 54, A_AVG = 55 };
enum : int32_t {
    E_OK = 0, E_OOM = 1, E_TYPE = 2, E_RANGE = 3, E_LENGTH = 4, E_DOMAIN = 6,
    E_NYI = 7, E_IO = 8, E_CANCEL = 11
};

constexpr int kThreads = 256;

__host__ __device__ inline int elem_size(int8_t type, uint8_t attrs) {
    switch (type) {
        case T_BOOL: case T_U8: case T_CHAR: return 1;
        case T_I16: return 2;
        case T_I32: case T_DATE: case T_TIME: return 4;
        case T_I64: case T_F64: case T_TIMESTAMP: return 8;
        case T_SYM: return 1 << (attrs & 3);
        default: return 0;
    }
}

__host__ __device__ inline bool is_int_class(int8_t t) {
    return t == T_BOOL || t == T_U8 || t == T_CHAR || t == T_I16 || t == T_I32 ||
           t == T_I64 || t == T_DATE || t == T_TIME || t == T_TIMESTAMP || t == T_SYM;
}

// Streaming load: columns are read once per query, so they are marked
// evict-first in L2 to leave room for the hash tables and accumulators.
template <typename T>
__device__ __forceinline__ T ld_stream(const T* p) { return __ldcs(p); }

// Integer-class value of row r (F64 columns are truncated, as Teide's
// read_col_i64 would never be asked to do; callers use ld_f for them).
__device__ __forceinline__ int64_t ld_i(const tdg_col& c, int64_t r) {
    switch (c.type) {
        case T_I64: case T_TIMESTAMP: return ld_stream((const long long*)c.data + r);
        case T_F64: return (int64_t)ld_stream((const double*)c.data + r);
        case T_I32: case T_DATE: case T_TIME: return ld_stream((const int*)c.data + r);
        case T_I16: return ld_stream((const short*)c.data + r);
        case T_BOOL: case T_U8: case T_CHAR: return ld_stream((const unsigned char*)c.data + r);
        case T_SYM:
            switch (c.attrs & 3) {
                case 0: return ld_stream((const unsigned char*)c.data + r);
                case 1: return ld_stream((const unsigned short*)c.data + r);
                case 2: return ld_stream((const unsigned int*)c.data + r);
                default: return ld_stream((const long long*)c.data + r);
            }
        default: return 0;
    }
}

__device__ __forceinline__ double ld_f(const tdg_col& c, int64_t r) {
    if (c.type == T_F64) return ld_stream((const double*)c.data + r);
    return (double)ld_i(c, r);
}

// Raw 8-byte key bits of row r: integer value, or the F64 bit pattern with
// -0.0 folded into +0.0 (Teide's td_hash_f64 folds the same way).
__device__ __forceinline__ int64_t ld_keybits(const tdg_col& c, int64_t r) {
    if (c.type == T_F64) {
        double v = ld_stream((const double*)c.data + r);
        if (v == 0.0) v = 0.0;
        return __double_as_longlong(v);
    }
    return ld_i(c, r);
}

// Total order on doubles as signed 64-bit integers, for atomicMin/atomicMax.
__device__ __forceinline__ long long f2ord(double v) {
    long long b = __double_as_longlong(v);
    return b ^ ((b >> 63) & 0x7FFFFFFFFFFFFFFFLL);
}
__device__ __forceinline__ double ord2f(long long o) {
    return __longlong_as_double(o ^ ((o >> 63) & 0x7FFFFFFFFFFFFFFFLL));
}

// 64-bit mixer (splitmix64 finalizer) for hash tables.
__device__ __forceinline__ uint64_t mix64(uint64_t x) {
    x ^= x >> 30; x *= 0xbf58476d1ce4e5b9ULL;
    x ^= x >> 27; x *= 0x94d049bb133111ebULL;
    x ^= x >> 31;
    return x;
}

// ---- expression interpreter ------------------------------------------------
// Registers hold raw 64-bit patterns; ins[k].kind says whether register k is
// an int64 or a double.  Mirrors Teide's expr_exec_binary (exec.c:982-1051):
// integer ADD/SUB/MUL wrap, integer MOD by zero yields 0, DIV is F64.
__device__ inline uint64_t x_eval(const tdg_expr& e, int64_t row) {
    uint64_t R[TDG_MAX_INS];
    const int n = e.n_ins;
    for (int k = 0; k < n; k++) {
        const tdg_ins I = e.ins[k];
        uint64_t r = 0;
        const bool fk = I.kind == 1;
        switch (I.op) {
            case TDG_X_COL: {
                const tdg_col& c = e.cols[I.imm];
                r = fk ? (uint64_t)__double_as_longlong(ld_f(c, row)) : (uint64_t)ld_i(c, row);
                break;
            }
            case TDG_X_CONST: r = (uint64_t)I.imm; break;
            case TDG_X_EQ: case TDG_X_NE: case TDG_X_LT:
            case TDG_X_LE: case TDG_X_GT: case TDG_X_GE: {
                bool res;
                if (e.ins[I.a].kind == 1) {
                    double x = __longlong_as_double((long long)R[I.a]);
                    double y = __longlong_as_double((long long)R[I.b]);
                    res = I.op == TDG_X_EQ ? x == y : I.op == TDG_X_NE ? x != y :
                          I.op == TDG_X_LT ? x < y  : I.op == TDG_X_LE ? x <= y :
                          I.op == TDG_X_GT ? x > y  : x >= y;
                } else {
                    int64_t x = (int64_t)R[I.a], y = (int64_t)R[I.b];
                    res = I.op == TDG_X_EQ ? x == y : I.op == TDG_X_NE ? x != y :
                          I.op == TDG_X_LT ? x < y  : I.op == TDG_X_LE ? x <= y :
                          I.op == TDG_X_GT ? x > y  : x >= y;
                }
                r = res ? 1 : 0;
                break;
            }
            case TDG_X_AND: r = (R[I.a] != 0 && R[I.b] != 0) ? 1 : 0; break;
            case TDG_X_OR:  r = (R[I.a] != 0 || R[I.b] != 0) ? 1 : 0; break;
            case TDG_X_NOT: r = R[I.a] == 0 ? 1 : 0; break;
            case TDG_X_TOF64: r = (uint64_t)__double_as_longlong((double)(int64_t)R[I.a]); break;
            case TDG_X_TOI64: r = (uint64_t)(int64_t)__longlong_as_double((long long)R[I.a]); break;
            case TDG_X_NEG: case TDG_X_ABS: {
                if (fk) {
                    double x = __longlong_as_double((long long)R[I.a]);
                    x = I.op == TDG_X_NEG ? -x : fabs(x);
                    r = (uint64_t)__double_as_longlong(x);
                } else {
                    int64_t x = (int64_t)R[I.a];
                    r = I.op == TDG_X_NEG ? (uint64_t)0 - (uint64_t)x
                                          : (x < 0 ? (uint64_t)0 - (uint64_t)x : (uint64_t)x);
                }
                break;
            }
            default: {   // binary arithmetic
                if (fk) {
                    double x = __longlong_as_double((long long)R[I.a]);
                    double y = __longlong_as_double((long long)R[I.b]);
                    double z;
                    switch (I.op) {
                        case TDG_X_ADD: z = x + y; break;
                        case TDG_X_SUB: z = x - y; break;
                        case TDG_X_MUL: z = x * y; break;
                        case TDG_X_DIV: z = x / y; break;
                        case TDG_X_MOD: z = fmod(x, y); break;
                        case TDG_X_MIN2: z = x < y ? x : y; break;
                        case TDG_X_MAX2: z = x > y ? x : y; break;
                        default: z = 0; break;
                    }
                    r = (uint64_t)__double_as_longlong(z);
                } else {
                    uint64_t x = R[I.a], y = R[I.b];
                    int64_t sx = (int64_t)x, sy = (int64_t)y;
                    switch (I.op) {
                        case TDG_X_ADD: r = x + y; break;
                        case TDG_X_SUB: r = x - y; break;
                        case TDG_X_MUL: r = x * y; break;
                        case TDG_X_MOD: r = sy == 0 ? 0 : (uint64_t)(sx % sy); break;
                        case TDG_X_MIN2: r = sx < sy ? x : y; break;
                        case TDG_X_MAX2: r = sx > sy ? x : y; break;
                        default: r = 0; break;
                    }
                }
                break;
            }
        }
        R[k] = r;
    }
    return n > 0 ? R[e.out] : 1;
}

// ---- predicate ----------------------------------------------------------------
// Fast path for the common shape "c1 OP k1 AND c2 OP k2 AND ..." (at most
// kMaxTerms column-vs-constant comparisons); anything else runs through the
// interpreter.  The launcher analyses the program on the host.
constexpr int kMaxTerms = 4;
// A term is evaluated branch-free as (lo <= v && v <= hi) != neg: EQ is
// [k, k], LT/LE/GT/GE are half-open ranges (strict bounds on doubles move to
// the adjacent representable value, so NaN still fails), NE is EQ negated.
struct Term {
    tdg_col col;
    int32_t op;      // TDG_X_EQ .. TDG_X_GE (for the interpreter fallback)
    int32_t f;       // compare as double
    int64_t k;       // constant bits (int64 or double)
    int64_t lo, hi;  // inclusive bounds (double bits when f)
    int32_t neg;
    int32_t pad;
};
struct Pred {
    int32_t kind;    // 0 = every row, 1 = conjunction of terms, 2 = program
    int32_t n;
    Term t[kMaxTerms];
    const uint64_t* sel;   // optional TD_SEL bit array
    int32_t w8;            // every term column is 8 bytes wide (kind 0 or 1)
    int32_t pad;
};

template <typename T>
__device__ __forceinline__ bool cmp(int32_t op, T x, T y) {
    switch (op) {
        case TDG_X_EQ: return x == y;
        case TDG_X_NE: return x != y;
        case TDG_X_LT: return x < y;
        case TDG_X_LE: return x <= y;
        case TDG_X_GT: return x > y;
        default:       return x >= y;
    }
}

// 8-byte columns (I64, F64, TIMESTAMP, SYM W64) read without a type switch:
// the raw word is an integer unless the column is F64.
__device__ __forceinline__ int64_t ld_i8(const tdg_col& c, int64_t r) {
    const long long x = ld_stream((const long long*)c.data + r);
    return c.type == T_F64 ? (int64_t)__longlong_as_double(x) : (int64_t)x;
}
__device__ __forceinline__ double ld_f8(const tdg_col& c, int64_t r) {
    const long long x = ld_stream((const long long*)c.data + r);
    return c.type == T_F64 ? __longlong_as_double(x) : (double)x;
}

// PK: 0 = none, 1 = conjunction, 2 = interpreter.  `prog` is only read for PK 2.
// W8: every column the predicate reads is 8 bytes wide.
template <int PK, bool W8 = false>
__device__ __forceinline__ bool row_pass(const Pred& p, const tdg_expr& prog, int64_t r) {
    bool ok = true;
    if (p.sel) ok = (__ldg(p.sel + (r >> 6)) >> (r & 63)) & 1;
    if (PK == 1) {
#pragma unroll
        for (int i = 0; i < kMaxTerms; i++) {
            if (i < p.n) {
                const Term& t = p.t[i];
                bool b;
                if (t.f) {
                    const double v = W8 ? ld_f8(t.col, r) : ld_f(t.col, r);
                    b = (v >= __longlong_as_double(t.lo)) & (v <= __longlong_as_double(t.hi));
                } else {
                    const int64_t v = W8 ? ld_i8(t.col, r) : ld_i(t.col, r);
                    b = (v >= t.lo) & (v <= t.hi);
                }
                ok = ok && (b != (bool)t.neg);
            }
        }
    } else if (PK == 2) {
        ok = ok && x_eval(prog, r) != 0;
    }
    return ok;
}

// ---- block-wide exclusive scan of one int per thread ------------------------------
// Returns the exclusive prefix; *total receives the block sum.  `scratch`
// holds 32 ints.  Every thread of the block must call it.
__device__ inline int block_excl_scan(int v, int* total, int* scratch) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) scratch[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int w = lane < nw ? scratch[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        scratch[lane] = w;   // inclusive over warps
    }
    __syncthreads();
    int warp_off = wid > 0 ? scratch[wid - 1] : 0;
    *total = scratch[nw - 1];
    __syncthreads();
    return warp_off + x - v;
}

// ---- shared-memory rings fed by bulk copies ----------------------------------------
// A producer thread copies column chunks from global memory into a ring of
// shared-memory stages with cp.async.bulk (the copy engine moves the bytes;
// no registers, no thread waits on DRAM), each stage guarded by two
// mbarriers: `full` completes when the stage's bytes have landed (the
// producer's arrive.expect_tx plus the copies' complete_tx), `empty` when
// every consumer warp has finished reading it.  Every wait is bounded: a
// wait that runs out returns false and the kernel records an error instead
// of hanging.  Plain (non-multicast) copies from this GPU's own memory only.
__device__ __forceinline__ uint32_t sh_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(sh_addr(bar)), "r"(count) : "memory");
}
// Makes the initialized barriers visible to the copy engine (async proxy).
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(sh_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(sh_addr(bar)), "r"(bytes) : "memory");
}
// Waits for the phase of parity `parity` to complete; false after `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    const uint32_t a = sh_addr(bar);
    for (uint32_t i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}" : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}
// bytes from global `src` to this CTA's shared `dst`, completing on `bar`.
// src, dst and bytes must be multiples of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(sh_addr(dst)), "l"(src), "r"(bytes), "r"(sh_addr(bar)) : "memory");
}
constexpr uint32_t kWaitLimit = 1u << 22;    // polls of one bounded mbarrier wait

// ---- L2 prefetch of streamed column ranges ------------------------------------------
// cp.async.bulk.prefetch.L2 asks the copy engine to pull a contiguous range
// into L2 without registers, shared memory or a completion wait, so a CTA can
// keep the next tile's DRAM reads in flight while its threads work on the
// current tile.  The range is shrunk inward to 16-byte boundaries (the
// instruction's alignment rule), so it never touches bytes outside
// [p, p + bytes); the few edge bytes are simply loaded without a prefetch.
__device__ __forceinline__ void l2_prefetch(const void* p, int64_t bytes) {
    if (bytes <= 0) return;
    const unsigned long long a = (unsigned long long)p;
    unsigned long long lo = (a + 15ull) & ~15ull;
    const unsigned long long hi = (a + (unsigned long long)bytes) & ~15ull;
    while (lo < hi) {
        const unsigned long long left = hi - lo;
        const unsigned sz = (unsigned)(left < (1ull << 20) ? left : (1ull << 20));
        asm volatile("{\n\t.reg .u64 g;\n\tcvta.to.global.u64 g, %0;\n\t"
                     "cp.async.bulk.prefetch.L2.global [g], %1;\n\t}" :: "l"(lo), "r"(sz) : "memory");
        lo += sz;
    }
}

// Columns a kernel streams row by row (probe side / plain table side).
constexpr int kMaxPf = 16;
struct PfCols {
    const char* p[kMaxPf];
    int32_t esz[kMaxPf];
    int32_t n;
    int32_t pad;
};

// Threads 0..n-1 of a CTA each prefetch rows [r0, r1) of one column.
__device__ __forceinline__ void prefetch_rows(const PfCols& F, int64_t r0, int64_t r1) {
    if ((int)threadIdx.x < F.n && r0 < r1) {
        const int64_t e = F.esz[threadIdx.x];
        l2_prefetch(F.p[threadIdx.x] + r0 * e, (r1 - r0) * e);
    }
}

inline void pf_add(PfCols& F, const tdg_col& c) {
    if (!c.data || F.n >= kMaxPf) return;
    for (int i = 0; i < F.n; i++) if (F.p[i] == (const char*)c.data) return;
    const int e = elem_size(c.type, c.attrs);
    if (e <= 0) return;
    F.p[F.n] = (const char*)c.data;
    F.esz[F.n] = e;
    F.n++;
}

// ---- host-side helpers ------------------------------------------------------------
Pred make_pred(const tdg_expr* prog, const uint64_t* sel, int* pk);
int sm_count();
int grid_for(const void* kernel, int threads, size_t smem, int64_t work_items);
tdg_status launch_status();
void note_launch(int n = 1);          // counts kernel launches (tdg_launch_count)

// CUDA-event timer around one launch on a stream (active when timing is on).
struct EventTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    bool on = false;
    void start(cudaStream_t s);
    void stop(cudaStream_t s);
    float ms();                        // valid after the stream has synchronized
    ~EventTimer();                     // returns the events if ms() was not called
};
bool timing_on();
void set_last_main_ms(float ms);
void set_last_build_ms(float ms);
void set_last_sort_ms(float ms);

// While alive, this thread's tdg calls make no allocating CUDA call (no
// page-locked status buffers either): the entry points that allocate nothing.
struct ThreadNoAlloc {
    ThreadNoAlloc();
    ~ThreadNoAlloc();
};
bool no_alloc();

// While alive, this thread's tdg calls record no timing events.
struct ThreadTimingOff {
    ThreadTimingOff();
    ~ThreadTimingOff();
};

}  // namespace tdg
