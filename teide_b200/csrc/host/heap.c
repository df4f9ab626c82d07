/*
 * Host heap for td_t blocks.
 *
 * Contract kept from Teide (src/mem/heap.c:61-67, 468-553, 559-633;
 * src/mem/cow.c:31-65): a block is 2^order bytes, order = ceil(log2(32 +
 * data_size)) clamped to >= TD_ORDER_MIN; the 32-byte header is zeroed with
 * rc = 1, mmod = 0 and `order` set; td_free releases the references a block
 * owns (table schema and columns, slice parent, external null map, string
 * payload) before returning the memory; td_cow copies when rc > 1.
 *
 * What is different: instead of a per-thread buddy allocator this heap takes
 * small blocks from malloc and blocks of 2 MB and more from mmap, whose pages
 * are committed on first touch.  Large blocks are what columns live in; the
 * GPU layer page-locks them on first upload (cudaHostRegister) so that
 * host->device copies reach link bandwidth, and unregisters them here on
 * free.  Blocks are thread-agnostic: any thread may free any block.
 */

#include "internal.h"
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>

#define TDB_MMAP_MIN ((size_t)2 << 20)

static _Atomic(size_t) st_alloc, st_free, st_bytes, st_peak, st_direct, st_direct_bytes;
static _Atomic(uint64_t) st_serial;

void tdb_gpu_on_free(td_t* v, tdb_block_prefix* p);   /* gpu.c */
void tdb_gpu_unpin_raw(void* raw);                    /* gpu.c */

/* Freed mmap blocks are kept (up to TDB_CACHE_MAX bytes) and handed out again
 * for the same block size: their pages are already committed and, once a
 * block has been page-locked for a transfer, it stays page-locked, so
 * query results reuse fast DMA destinations instead of faulting in fresh
 * pages every time. */
#define TDB_CACHE_MAX ((size_t)16 << 30)
#define TDB_CACHE_SLOTS 256
static pthread_mutex_t cache_mu = PTHREAD_MUTEX_INITIALIZER;
static void* cache_raw[TDB_CACHE_SLOTS];
static size_t cache_size[TDB_CACHE_SLOTS];
static size_t cache_pinned[TDB_CACHE_SLOTS];
static int cache_n;
static size_t cache_bytes;

/* The smallest cached block of at least raw_size bytes and at most four
 * times that (page-locked blocks preferred): query results vary in size from
 * call to call, and a block one or two size classes up is still far cheaper
 * than fresh pages that must be faulted in and page-locked again.  *got
 * receives the block's actual size. */
static void* cache_take(size_t raw_size, size_t* pinned, size_t* got) {
    void* r = NULL;
    pthread_mutex_lock(&cache_mu);
    int best = -1;
    for (int i = 0; i < cache_n; i++) {
        if (cache_size[i] < raw_size || cache_size[i] / 4 > raw_size) continue;
        if (best < 0 || (cache_pinned[i] != 0) > (cache_pinned[best] != 0) ||
            ((cache_pinned[i] != 0) == (cache_pinned[best] != 0) && cache_size[i] < cache_size[best]))
            best = i;
    }
    if (best >= 0) {
        r = cache_raw[best];
        *pinned = cache_pinned[best];
        *got = cache_size[best];
        cache_bytes -= cache_size[best];
        cache_n--;
        cache_raw[best] = cache_raw[cache_n];
        cache_size[best] = cache_size[cache_n];
        cache_pinned[best] = cache_pinned[cache_n];
    }
    pthread_mutex_unlock(&cache_mu);
    return r;
}

static int cache_put(void* raw, size_t raw_size, size_t pinned) {
    int ok = 0;
    pthread_mutex_lock(&cache_mu);
    if (cache_n < TDB_CACHE_SLOTS && cache_bytes + raw_size <= TDB_CACHE_MAX) {
        cache_raw[cache_n] = raw;
        cache_size[cache_n] = raw_size;
        cache_pinned[cache_n] = pinned;
        cache_n++;
        cache_bytes += raw_size;
        ok = 1;
    }
    pthread_mutex_unlock(&cache_mu);
    return ok;
}

static uint8_t ceil_log2(size_t x) {
    uint8_t k = 0;
    size_t p = 1;
    while (p < x) { p <<= 1; k++; }
    return k;
}

uint8_t td_order_for_size(size_t data_size) {
    if (data_size > SIZE_MAX / 2) return 64;
    uint8_t k = ceil_log2(data_size + 32);
    return k < TD_ORDER_MIN ? TD_ORDER_MIN : k;
}

void td_heap_init(void) {}
void td_heap_destroy(void) {}
void td_heap_gc(void) {}

void td_mem_stats(td_mem_stats_t* out) {
    if (!out) return;
    memset(out, 0, sizeof(*out));
    out->alloc_count = atomic_load(&st_alloc);
    out->free_count = atomic_load(&st_free);
    out->bytes_allocated = atomic_load(&st_bytes);
    out->peak_bytes = atomic_load(&st_peak);
    out->direct_count = atomic_load(&st_direct);
    out->direct_bytes = atomic_load(&st_direct_bytes);
    out->sys_current = out->bytes_allocated;
    out->sys_peak = out->peak_bytes;
}

/* Freed small blocks are kept per order (up to TDB_SMALL_KEEP bytes in all)
 * and handed out again: a block taken back from the C allocator is often
 * fresh memory whose pages fault on first touch, which costs more than the
 * copy that fills it (measured: 4000 blocks of 32 KB filled at about 2 GB/s
 * when every round allocated anew). */
#define TDB_SMALL_KEEP ((size_t)256 << 20)
#define TDB_SMALL_ORDERS 32
static pthread_mutex_t small_mu = PTHREAD_MUTEX_INITIALIZER;
static void* small_free[TDB_SMALL_ORDERS];      /* singly linked through each block's first word */
static size_t small_bytes;

static void* small_take(uint8_t order) {
    if (order >= TDB_SMALL_ORDERS) return NULL;
    pthread_mutex_lock(&small_mu);
    void* r = small_free[order];
    if (r) {
        small_free[order] = *(void**)r;
        small_bytes -= (size_t)1 << order;
    }
    pthread_mutex_unlock(&small_mu);
    return r;
}

static int small_put(void* raw, uint8_t order) {
    if (order >= TDB_SMALL_ORDERS) return 0;
    int ok = 0;
    pthread_mutex_lock(&small_mu);
    if (small_bytes + ((size_t)1 << order) <= TDB_SMALL_KEEP) {
        *(void**)raw = small_free[order];
        small_free[order] = raw;
        small_bytes += (size_t)1 << order;
        ok = 1;
    }
    pthread_mutex_unlock(&small_mu);
    return ok;
}

td_t* td_alloc(size_t data_size) {
    uint8_t order = td_order_for_size(data_size);
    if (order > 48) return NULL;
    size_t block = (size_t)1 << order;
    size_t raw_size = block + sizeof(tdb_block_prefix);
    void* raw;
    uint32_t kind;
    size_t pinned = 0;
    if (block >= TDB_MMAP_MIN) {
        raw_size = (raw_size + 4095) & ~(size_t)4095;
        size_t got = 0;
        raw = cache_take(raw_size, &pinned, &got);
        if (raw) raw_size = got;
        else {
            raw = mmap(NULL, raw_size, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
            if (raw == MAP_FAILED) return NULL;
        }
        kind = TDB_BLK_MMAP;
        atomic_fetch_add(&st_direct, 1);
        atomic_fetch_add(&st_direct_bytes, raw_size);
    } else {
        raw = small_take(order);
        if (!raw) raw = aligned_alloc(64, (raw_size + 63) & ~(size_t)63);
        if (!raw) return NULL;
        kind = TDB_BLK_MALLOC;
    }
    tdb_block_prefix* p = (tdb_block_prefix*)raw;
    memset(p, 0, sizeof(*p));
    p->magic = TDB_BLK_MAGIC;
    p->kind = kind;
    p->raw = raw;
    p->raw_size = raw_size;
    atomic_store(&p->pinned, pinned);
    p->serial = atomic_fetch_add(&st_serial, 1) + 1;
    td_t* v = (td_t*)(p + 1);
    memset(v, 0, 32);
    v->order = order;
    atomic_store_explicit(&v->rc, 1, memory_order_relaxed);
    atomic_fetch_add(&st_alloc, 1);
    size_t now = atomic_fetch_add(&st_bytes, block) + block;
    size_t pk = atomic_load(&st_peak);
    while (now > pk && !atomic_compare_exchange_weak(&st_peak, &pk, now)) {}
    return v;
}

int tdb_is_heap_block(td_t* v) {
    return v && !TD_IS_ERR(v) && tdb_prefix(v)->magic == TDB_BLK_MAGIC;
}

uint64_t tdb_block_serial(td_t* v) {
    return tdb_is_heap_block(v) ? tdb_prefix(v)->serial : 0;
}

static int atom_owns_obj(td_t* v) {
    /* long string atoms point at a CHAR vector (see vec.c: td_str) */
    if (v->type == TD_ATOM_STR) return !(v->slen >= 1 && v->slen <= 7) && v->obj != NULL;
    if (v->type == TD_ATOM_GUID) return v->obj != NULL;
    return 0;
}

static void for_each_owned(td_t* v, void (*fn)(td_t*)) {
    if (td_is_atom(v)) {
        if (atom_owns_obj(v) && !TD_IS_ERR(v->obj)) fn(v->obj);
        return;
    }
    if (v->attrs & TD_ATTR_SLICE) {
        if (v->slice_parent && !TD_IS_ERR(v->slice_parent)) fn(v->slice_parent);
        return;
    }
    if ((v->attrs & TD_ATTR_NULLMAP_EXT) && v->ext_nullmap && !TD_IS_ERR(v->ext_nullmap))
        fn(v->ext_nullmap);
    if (v->type == TD_TABLE) {
        if (v->len < 0) return;
        td_t** slots = (td_t**)td_data(v);
        if (slots[0] && !TD_IS_ERR(slots[0])) fn(slots[0]);
        for (int64_t i = 0; i < v->len; i++)
            if (slots[1 + i] && !TD_IS_ERR(slots[1 + i])) fn(slots[1 + i]);
        return;
    }
    if (v->type == TD_LIST || TD_IS_PARTED(v->type) || v->type == TD_MAPCOMMON) {
        /* a list's items, a parted column's segments, a MAPCOMMON's key values and counts */
        td_t** items = (td_t**)td_data(v);
        for (int64_t i = 0; i < v->len; i++)
            if (items[i] && !TD_IS_ERR(items[i])) fn(items[i]);
    }
}

void tdb_retain_owned_refs(td_t* v) { if (v && !TD_IS_ERR(v)) for_each_owned(v, td_retain); }

/* Return a block's memory: large blocks go back to the cache (still
 * page-locked) when there is room, else to the OS. */
static void release_block(td_t* v) {
    tdb_block_prefix* p = tdb_prefix(v);
    tdb_gpu_on_free(v, p);
    size_t block = (size_t)1 << v->order;
    p->magic = 0;
    atomic_fetch_add(&st_free, 1);
    atomic_fetch_sub(&st_bytes, block);
    if (p->kind == TDB_BLK_FILE) {
        munmap(p->raw, p->raw_size);          /* the prefix page and the file mapping */
    } else if (p->kind == TDB_BLK_MMAP) {
        void* raw = p->raw;
        size_t raw_size = p->raw_size, pinned = atomic_load(&p->pinned);
        atomic_fetch_sub(&st_direct, 1);
        atomic_fetch_sub(&st_direct_bytes, raw_size);
        if (!cache_put(raw, raw_size, pinned)) {
            if (pinned) tdb_gpu_unpin_raw(raw);
            munmap(raw, raw_size);
        }
    } else if (!small_put(p->raw, v->order)) {
        free(p->raw);
    }
}

td_t* tdb_file_block(void* base, size_t total) {
    tdb_block_prefix* p = (tdb_block_prefix*)((char*)base + 4096 - sizeof(tdb_block_prefix));
    memset(p, 0, sizeof(*p));
    p->magic = TDB_BLK_MAGIC;
    p->kind = TDB_BLK_FILE;
    p->raw = base;
    p->raw_size = total;
    p->serial = atomic_fetch_add(&st_serial, 1) + 1;
    td_t* v = (td_t*)(p + 1);
    /* the block's capacity: the largest power of two the mapping holds, so
     * code that writes within a block's capacity stays inside it */
    uint8_t order = 5;
    while (((size_t)2 << order) <= total - 4096) order++;
    v->order = order;
    atomic_fetch_add(&st_alloc, 1);
    atomic_fetch_add(&st_bytes, (size_t)1 << order);
    return v;
}

void td_free(td_t* v) {
    if (!v || TD_IS_ERR(v)) return;
    atomic_store_explicit(&v->rc, 1, memory_order_relaxed);
    for_each_owned(v, td_release);
    if (!tdb_is_heap_block(v)) return;          /* not ours: leave it alone */
    release_block(v);
}

td_t* td_alloc_copy(td_t* v) {
    if (!v || TD_IS_ERR(v)) return NULL;
    size_t data_size = ((size_t)1 << v->order) - 32;
    size_t used = data_size;
    if (v->type > 0 && v->type < TD_TYPE_COUNT && v->type != TD_TABLE && v->type != TD_LIST
        && v->type != TD_SEL) {
        size_t esz = td_sym_elem_size(v->type, v->attrs);
        if (esz && (size_t)v->len * esz < used) used = (size_t)v->len * esz;
    }
    td_t* c = td_alloc(data_size);
    if (!c) return NULL;
    uint8_t order = c->order;
    memcpy(c, v, 32);
    memcpy(td_data(c), td_data(v), used);
    c->order = order;
    c->mmod = 0;
    atomic_store_explicit(&c->rc, 1, memory_order_relaxed);
    tdb_retain_owned_refs(c);
    return c;
}

td_t* td_scratch_alloc(size_t data_size) { return td_alloc(data_size); }

td_t* td_scratch_realloc(td_t* v, size_t new_data_size) {
    if (!v || TD_IS_ERR(v)) return td_alloc(new_data_size);
    size_t old = ((size_t)1 << v->order) - 32;
    if (new_data_size <= old) return v;
    td_t* n = td_alloc(new_data_size);
    if (!n) return TD_ERR_PTR(TD_ERR_OOM);
    uint8_t order = n->order;
    memcpy(n, v, 32);
    memcpy(td_data(n), td_data(v), old);
    n->order = order;
    atomic_store_explicit(&n->rc, 1, memory_order_relaxed);
    /* ownership of children moves to the new block: free the old one without
     * releasing them */
    if (tdb_is_heap_block(v)) release_block(v);
    return n;
}

void td_retain(td_t* v) {
    if (!v || TD_IS_ERR(v)) return;
    atomic_fetch_add_explicit(&v->rc, 1, memory_order_relaxed);
}

void td_release(td_t* v) {
    if (!v || TD_IS_ERR(v)) return;
    if (atomic_fetch_sub_explicit(&v->rc, 1, memory_order_acq_rel) == 1) td_free(v);
}

td_t* td_cow(td_t* v) {
    if (!v || TD_IS_ERR(v)) return v;
    if (atomic_load_explicit(&v->rc, memory_order_acquire) == 1) {
        tdb_mirror_forget(v);       /* about to be mutated in place */
        return v;
    }
    td_t* c = td_alloc_copy(v);
    if (!c) return TD_ERR_PTR(TD_ERR_OOM);
    td_release(v);
    return c;
}
