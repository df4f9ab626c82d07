// Device hash tables shared by the group-by and join kernels.
//
// Open addressing with linear probing over a power-of-two capacity.  Slot i
// has a 32-bit state (0 empty, 1 being written, 2 ready) and the key tuple
// stored column-wise (keys[k * cap + i], raw 8-byte key bits).  A thread
// claims an empty slot with a CAS 0 -> 1, writes the key, fences and
// publishes 2; readers that meet state 1 wait -- with an iteration limit,
// after which the kernel records TD_ERR_IO in the error word and gives up on
// the row -- for the writer to publish.
//
// Teide's CPU tables (group: exec.c:3917-4170 with 4-byte salt|gid slots;
// join: exec.c:7824-7950 with 8-byte hash|row slots) partition first so each
// table fits a core's cache.  On the GPU the table lives in HBM and the hot
// part of it stays in the 126 MB L2; no partitioning pass is needed.
#pragma once
#include "tdg_common.cuh"

namespace tdg {

constexpr int kSpinLimit = 1 << 20;

struct HtRef {
    uint32_t* state;
    int64_t*  keys;        // n_keys * cap
    uint64_t  mask;        // cap - 1
    int32_t   nk;
    int32_t   spin_limit;  // polls of a state-1 slot before giving up (0: kSpinLimit)
    int32_t*  err;
};

__device__ __forceinline__ uint64_t hash_keys(const int64_t* kv, int nk) {
    uint64_t h = 0x9E3779B97F4A7C15ULL;
    for (int k = 0; k < nk; k++) h = mix64(h ^ (uint64_t)kv[k]) + (uint64_t)k;
    return h;
}

__device__ __forceinline__ void set_err(int32_t* err, int32_t code) {
    if (err) atomicCAS(err, 0, code);
}

// Find the slot of key tuple kv, inserting it when absent.  -1 on failure
// (table full or a writer that never published), with the error recorded.
__device__ inline int64_t ht_upsert(const HtRef& H, const int64_t* kv, uint64_t h) {
    const uint64_t cap = H.mask + 1;
    uint64_t i = h & H.mask;
    for (uint64_t probe = 0; probe < cap; probe++) {
        uint32_t s = *(volatile uint32_t*)&H.state[i];
        if (s == 0) {
            const uint32_t prev = atomicCAS(&H.state[i], 0u, 1u);
            if (prev == 0) {
                for (int k = 0; k < H.nk; k++) H.keys[(uint64_t)k * cap + i] = kv[k];
                __threadfence();
                atomicExch(&H.state[i], 2u);
                return (int64_t)i;
            }
            s = prev;
        }
        if (s == 1) {
            const int limit = H.spin_limit > 0 ? H.spin_limit : kSpinLimit;
            int spins = 0;
            do {
                s = *(volatile uint32_t*)&H.state[i];
                if (++spins > limit) { set_err(H.err, E_IO); return -1; }
            } while (s == 1);
        }
        __threadfence();
        bool eq = true;
        for (int k = 0; k < H.nk; k++)
            eq = eq && (*(volatile int64_t*)&H.keys[(uint64_t)k * cap + i] == kv[k]);
        if (eq) return (int64_t)i;
        i = (i + 1) & H.mask;
    }
    set_err(H.err, E_RANGE);
    return -1;
}

// Lookup only (the table is complete: no state-1 slots remain).
__device__ inline int64_t ht_find(const HtRef& H, const int64_t* kv, uint64_t h) {
    const uint64_t cap = H.mask + 1;
    uint64_t i = h & H.mask;
    for (uint64_t probe = 0; probe < cap; probe++) {
        const uint32_t s = __ldg(&H.state[i]);
        if (s == 0) return -1;
        bool eq = true;
        for (int k = 0; k < H.nk; k++) eq = eq && (__ldg(&H.keys[(uint64_t)k * cap + i]) == kv[k]);
        if (eq) return (int64_t)i;
        i = (i + 1) & H.mask;
    }
    return -1;
}

// ---- join table -------------------------------------------------------------------
// head[slot] is the most recently inserted build row with that key, next[row]
// the previous one (-1 ends the chain): every build row is reachable, so
// duplicate build keys produce one output row per match.
struct JoinK {
    int32_t method;        // TDG_JOIN_DIRECT or TDG_JOIN_HASH
    int32_t nk;
    int32_t join_type;     // 0 inner, 1 left, 2 full
    int32_t key_f64;       // single F64 key: NaN never matches
    tdg_col lkeys[TDG_MAX_KEYS];
    tdg_col rkeys[TDG_MAX_KEYS];
    int64_t kmin;          // direct map: key - kmin indexes head[]
    int64_t n_slots;
    int32_t* head;
    int32_t* next;
    uint8_t* matched;      // full join: build rows that found a partner
    HtRef    ht;
};

__device__ __forceinline__ bool nan_bits(int64_t b) {
    return ((b >> 52) & 0x7FF) == 0x7FF && (b & 0xFFFFFFFFFFFFFLL) != 0;
}

// First build row matching probe row r, or -1.
__device__ __forceinline__ int32_t join_first(const JoinK& J, int64_t r) {
    if (J.method == TDG_JOIN_DIRECT) {
        const int64_t k = ld_i(J.lkeys[0], r) - J.kmin;
        if (k < 0 || k >= J.n_slots) return -1;
        return __ldg(&J.head[k]);
    }
    int64_t kv[TDG_MAX_KEYS];
    for (int k = 0; k < J.nk; k++) {
        kv[k] = ld_keybits(J.lkeys[k], r);
        if (J.lkeys[k].type == T_F64 && nan_bits(kv[k])) return -1;
    }
    const int64_t s = ht_find(J.ht, kv, hash_keys(kv, J.nk));
    return s < 0 ? -1 : __ldg(&J.head[s]);
}

}  // namespace tdg
