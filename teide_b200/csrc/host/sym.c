/*
 * Global symbol table: interned strings with dense ids 0, 1, 2, ... in
 * intern order (Teide src/table/sym.c:81-200 assigns ids the same way, so
 * column-name ids agree with a caller that interns names in the same order).
 * Ids are stable for the life of the table; lookups are open addressing on an
 * FNV-1a hash under a mutex.
 */
#include "internal.h"
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

static pthread_mutex_t sym_mu = PTHREAD_MUTEX_INITIALIZER;
static td_t**   sym_strs;      /* id -> string atom */
static uint32_t sym_n, sym_cap;
static uint32_t* sym_slots;    /* id + 1, 0 = empty */
static uint32_t sym_nslots;
static int      sym_ready;

static uint32_t fnv1a(const char* s, size_t n) {
    uint32_t h = 2166136261u;
    for (size_t i = 0; i < n; i++) { h ^= (uint8_t)s[i]; h *= 16777619u; }
    return h;
}

void td_sym_init(void) {
    pthread_mutex_lock(&sym_mu);
    if (!sym_ready) {
        sym_cap = 1024;
        sym_strs = calloc(sym_cap, sizeof(td_t*));
        sym_nslots = 4096;
        sym_slots = calloc(sym_nslots, sizeof(uint32_t));
        sym_n = 0;
        sym_ready = sym_strs && sym_slots;
    }
    pthread_mutex_unlock(&sym_mu);
}

void td_sym_destroy(void) {
    pthread_mutex_lock(&sym_mu);
    if (sym_ready) {
        for (uint32_t i = 0; i < sym_n; i++) td_release(sym_strs[i]);
        free(sym_strs);
        free(sym_slots);
        sym_strs = NULL; sym_slots = NULL;
        sym_n = sym_cap = sym_nslots = 0;
        sym_ready = 0;
    }
    pthread_mutex_unlock(&sym_mu);
}

static int64_t lookup_locked(const char* s, size_t n, uint32_t h, uint32_t* slot_out) {
    uint32_t mask = sym_nslots - 1, i = h & mask;
    for (;;) {
        uint32_t e = sym_slots[i];
        if (!e) { *slot_out = i; return -1; }
        td_t* a = sym_strs[e - 1];
        if (td_str_len(a) == n && memcmp(td_str_ptr(a), s, n) == 0) return (int64_t)(e - 1);
        i = (i + 1) & mask;
    }
}

static int grow_locked(void) {
    uint32_t ns = sym_nslots * 2;
    uint32_t* nsl = calloc(ns, sizeof(uint32_t));
    if (!nsl) return 0;
    for (uint32_t id = 0; id < sym_n; id++) {
        td_t* a = sym_strs[id];
        uint32_t i = fnv1a(td_str_ptr(a), td_str_len(a)) & (ns - 1);
        while (nsl[i]) i = (i + 1) & (ns - 1);
        nsl[i] = id + 1;
    }
    free(sym_slots);
    sym_slots = nsl;
    sym_nslots = ns;
    return 1;
}

int64_t td_sym_intern(const char* s, size_t n) {
    if (!sym_ready) td_sym_init();
    pthread_mutex_lock(&sym_mu);
    uint32_t h = fnv1a(s, n), slot;
    int64_t id = lookup_locked(s, n, h, &slot);
    if (id < 0) {
        if ((uint64_t)(sym_n + 1) * 2 > sym_nslots) {
            if (!grow_locked()) { pthread_mutex_unlock(&sym_mu); return -1; }
            lookup_locked(s, n, h, &slot);
        }
        if (sym_n == sym_cap) {
            td_t** ns = realloc(sym_strs, sizeof(td_t*) * sym_cap * 2);
            if (!ns) { pthread_mutex_unlock(&sym_mu); return -1; }
            sym_strs = ns;
            sym_cap *= 2;
        }
        td_t* a = td_str(s, n);
        if (TD_IS_ERR(a)) { pthread_mutex_unlock(&sym_mu); return -1; }
        sym_strs[sym_n] = a;
        sym_slots[slot] = sym_n + 1;
        id = sym_n++;
    }
    pthread_mutex_unlock(&sym_mu);
    return id;
}

int64_t td_sym_find(const char* s, size_t n) {
    if (!sym_ready) return -1;
    pthread_mutex_lock(&sym_mu);
    uint32_t slot;
    int64_t id = lookup_locked(s, n, fnv1a(s, n), &slot);
    pthread_mutex_unlock(&sym_mu);
    return id;
}

td_t* td_sym_str(int64_t id) {
    if (!sym_ready || id < 0) return NULL;
    pthread_mutex_lock(&sym_mu);
    td_t* a = (uint64_t)id < sym_n ? sym_strs[id] : NULL;
    pthread_mutex_unlock(&sym_mu);
    return a;
}

uint32_t td_sym_count(void) { return sym_n; }
