/*
 * Atoms, strings, vectors, null bitmaps, selections, type sizes and error
 * strings.
 *
 * Behaviour kept from Teide:
 *   - type sizes (src/core/types.c:27-49) and error strings (src/core/err.c);
 *   - atoms are 0-data blocks with the value in the header union
 *     (src/vec/atom.c); strings of <= 7 bytes are stored inline (slen/sdata),
 *     longer ones point at a CHAR vector (src/vec/str.c:36-60);
 *   - vector capacity = (2^order - 32) / element size, growth by realloc to
 *     the next power of two (src/vec/vec.c:30-160, 284-318);
 *   - null bits inline for <= 128 rows, else an external U8 bitmap vector;
 *   - TD_SEL construction and segment summaries (src/vec/sel.c:36-189).
 */
#include "internal.h"
#include <string.h>
#include <stdlib.h>

const uint8_t td_type_sizes[TD_TYPE_COUNT] = {
    [TD_LIST] = 8, [TD_BOOL] = 1, [TD_U8] = 1, [TD_CHAR] = 1, [TD_I16] = 2,
    [TD_I32] = 4, [TD_I64] = 8, [TD_F64] = 8, [TD_DATE] = 4, [TD_TIME] = 4,
    [TD_TIMESTAMP] = 8, [TD_GUID] = 16, [TD_TABLE] = 8, [TD_SYM] = 8,
    /* 8, 14, 15, 17-19 are unused tags; TD_SEL has no element size */
};

const char* td_err_str(td_err_t e) {
    switch (e) {
        case TD_OK:          return "ok";
        case TD_ERR_OOM:     return "out of memory";
        case TD_ERR_TYPE:    return "type error";
        case TD_ERR_RANGE:   return "range error";
        case TD_ERR_LENGTH:  return "length mismatch";
        case TD_ERR_RANK:    return "rank error";
        case TD_ERR_DOMAIN:  return "domain error";
        case TD_ERR_NYI:     return "not yet implemented";
        case TD_ERR_IO:      return "I/O error";
        case TD_ERR_SCHEMA:  return "schema error";
        case TD_ERR_CORRUPT: return "corrupt data";
        case TD_ERR_CANCEL:  return "query cancelled";
    }
    return "unknown error";
}

/* ---- atoms ---------------------------------------------------------------- */
static td_t* atom(int8_t t) {
    td_t* v = td_alloc(0);
    if (!v) return TD_ERR_PTR(TD_ERR_OOM);
    v->type = t;
    return v;
}
td_t* td_bool(bool x)   { td_t* v = atom(TD_ATOM_BOOL); if (!TD_IS_ERR(v)) v->b8 = x ? 1 : 0; return v; }
td_t* td_u8(uint8_t x)  { td_t* v = atom(TD_ATOM_U8);   if (!TD_IS_ERR(v)) v->u8 = x; return v; }
td_t* td_char(char x)   { td_t* v = atom(TD_ATOM_CHAR); if (!TD_IS_ERR(v)) v->c8 = x; return v; }
td_t* td_i16(int16_t x) { td_t* v = atom(TD_ATOM_I16);  if (!TD_IS_ERR(v)) v->i16 = x; return v; }
td_t* td_i32(int32_t x) { td_t* v = atom(TD_ATOM_I32);  if (!TD_IS_ERR(v)) v->i32 = x; return v; }
td_t* td_i64(int64_t x) { td_t* v = atom(TD_ATOM_I64);  if (!TD_IS_ERR(v)) v->i64 = x; return v; }
td_t* td_f64(double x)  { td_t* v = atom(TD_ATOM_F64);  if (!TD_IS_ERR(v)) v->f64 = x; return v; }
td_t* td_sym(int64_t x) { td_t* v = atom(TD_ATOM_SYM);  if (!TD_IS_ERR(v)) v->i64 = x; return v; }
td_t* td_date(int64_t x){ td_t* v = atom(TD_ATOM_DATE); if (!TD_IS_ERR(v)) v->i64 = x; return v; }
td_t* td_time(int64_t x){ td_t* v = atom(TD_ATOM_TIME); if (!TD_IS_ERR(v)) v->i64 = x; return v; }
td_t* td_timestamp(int64_t x) { td_t* v = atom(TD_ATOM_TIMESTAMP); if (!TD_IS_ERR(v)) v->i64 = x; return v; }

/* numeric value of an atom; returns 0 for non-numeric atoms */
int tdb_atom_numeric(td_t* a, double* f, int64_t* i, int* is_f64) {
    if (!a || TD_IS_ERR(a) || !td_is_atom(a)) return 0;
    switch (a->type) {
        case TD_ATOM_F64:  *f = a->f64; *i = (int64_t)a->f64; *is_f64 = 1; return 1;
        case TD_ATOM_BOOL: *i = a->b8; break;
        case TD_ATOM_U8:   *i = a->u8; break;
        case TD_ATOM_I16:  *i = a->i16; break;
        case TD_ATOM_I32:  *i = a->i32; break;
        case TD_ATOM_I64: case TD_ATOM_SYM: case TD_ATOM_DATE:
        case TD_ATOM_TIME: case TD_ATOM_TIMESTAMP: *i = a->i64; break;
        default: return 0;
    }
    *f = (double)*i;
    *is_f64 = 0;
    return 1;
}

/* ---- strings ------------------------------------------------------------------ */
static int str_inline(td_t* s) {
    return (s->slen >= 1 && s->slen <= 7) || (s->slen == 0 && s->obj == NULL);
}

td_t* td_str(const char* s, size_t len) {
    td_t* v = atom(TD_ATOM_STR);
    if (TD_IS_ERR(v)) return v;
    if (len <= 7) {
        v->slen = (uint8_t)len;
        if (len) memcpy(v->sdata, s, len);
        return v;
    }
    td_t* chars = td_vec_new(TD_CHAR, (int64_t)len);
    if (!chars || TD_IS_ERR(chars)) { td_free(v); return TD_ERR_PTR(TD_ERR_OOM); }
    memcpy(td_data(chars), s, len);
    chars->len = (int64_t)len;
    v->obj = chars;
    return v;
}
const char* td_str_ptr(td_t* s) {
    if (!s || TD_IS_ERR(s)) return NULL;
    return str_inline(s) ? (const char*)s->sdata : (const char*)td_data(s->obj);
}
size_t td_str_len(td_t* s) {
    if (!s || TD_IS_ERR(s)) return 0;
    return str_inline(s) ? (size_t)s->slen : (size_t)s->obj->len;
}
int td_str_cmp(td_t* a, td_t* b) {
    if (!a || TD_IS_ERR(a) || !b || TD_IS_ERR(b)) return 0;
    size_t la = td_str_len(a), lb = td_str_len(b);
    int c = memcmp(td_str_ptr(a), td_str_ptr(b), la < lb ? la : lb);
    if (c) return c;
    return la < lb ? -1 : la > lb ? 1 : 0;
}

/* ---- vectors ------------------------------------------------------------------ */
int64_t tdb_vec_capacity(td_t* v) {
    size_t esz = td_sym_elem_size(v->type, v->attrs);
    if (!esz) return 0;
    return (int64_t)((((size_t)1 << v->order) - 32) / esz);
}

td_t* td_sym_vec_new(uint8_t w, int64_t capacity) {
    if (w & ~TD_SYM_W_MASK) return TD_ERR_PTR(TD_ERR_TYPE);
    if (capacity < 0) return TD_ERR_PTR(TD_ERR_RANGE);
    td_t* v = td_alloc((size_t)capacity * TD_SYM_ELEM(w));
    if (!v) return TD_ERR_PTR(TD_ERR_OOM);
    v->type = TD_SYM;
    v->attrs = w;
    return v;
}

td_t* td_vec_new(int8_t type, int64_t capacity) {
    if (type <= 0 || type >= TD_TYPE_COUNT) return TD_ERR_PTR(TD_ERR_TYPE);
    if (type == TD_SYM) return td_sym_vec_new(TD_SYM_W64, capacity);
    if (capacity < 0) return TD_ERR_PTR(TD_ERR_RANGE);
    size_t esz = td_elem_size(type);
    if (esz > 1 && (size_t)capacity > SIZE_MAX / esz) return TD_ERR_PTR(TD_ERR_OOM);
    td_t* v = td_alloc((size_t)capacity * esz);
    if (!v) return TD_ERR_PTR(TD_ERR_OOM);
    v->type = type;
    return v;
}

td_t* td_vec_from_raw(int8_t type, const void* data, int64_t count) {
    if (type <= 0 || type >= TD_TYPE_COUNT) return TD_ERR_PTR(TD_ERR_TYPE);
    if (count < 0) return TD_ERR_PTR(TD_ERR_RANGE);
    uint8_t w = type == TD_SYM ? TD_SYM_W64 : 0;
    size_t bytes = (size_t)count * td_sym_elem_size(type, w);
    td_t* v = td_alloc(bytes);
    if (!v) return TD_ERR_PTR(TD_ERR_OOM);
    v->type = type;
    v->attrs = w;
    v->len = count;
    if (bytes) memcpy(td_data(v), data, bytes);
    if (type == TD_LIST || type == TD_TABLE) {
        td_t** p = (td_t**)td_data(v);
        for (int64_t i = 0; i < count; i++) if (p[i]) td_retain(p[i]);
    }
    return v;
}

td_t* td_vec_append(td_t* vec, const void* elem) {
    if (!vec || TD_IS_ERR(vec)) return vec;
    if (vec->type <= 0 || vec->type >= TD_TYPE_COUNT) return TD_ERR_PTR(TD_ERR_TYPE);
    vec = td_cow(vec);
    if (!vec || TD_IS_ERR(vec)) return vec;
    size_t esz = td_sym_elem_size(vec->type, vec->attrs);
    if (vec->len >= tdb_vec_capacity(vec)) {
        size_t want = (size_t)(vec->len + 1) * esz, s = 32;
        while (s < want) s <<= 1;
        td_t* n = td_scratch_realloc(vec, s);
        if (!n || TD_IS_ERR(n)) return n ? n : TD_ERR_PTR(TD_ERR_OOM);
        vec = n;
    }
    memcpy((char*)td_data(vec) + (size_t)vec->len * esz, elem, esz);
    vec->len++;
    return vec;
}

td_t* td_vec_set(td_t* vec, int64_t idx, const void* elem) {
    if (!vec || TD_IS_ERR(vec)) return vec;
    if (idx < 0 || idx >= vec->len) return TD_ERR_PTR(TD_ERR_RANGE);
    vec = td_cow(vec);
    if (!vec || TD_IS_ERR(vec)) return vec;
    size_t esz = td_sym_elem_size(vec->type, vec->attrs);
    memcpy((char*)td_data(vec) + (size_t)idx * esz, elem, esz);
    return vec;
}

void* td_vec_get(td_t* vec, int64_t idx) {
    if (!vec || TD_IS_ERR(vec) || idx < 0 || idx >= vec->len) return NULL;
    if (vec->attrs & TD_ATTR_SLICE)
        return td_vec_get(vec->slice_parent, vec->slice_offset + idx);
    return (char*)td_data(vec) + (size_t)idx * td_sym_elem_size(vec->type, vec->attrs);
}

/* A slice is a header-only view [offset, offset + len) of its parent vector
 * (src/vec/vec.c:185-212 in Teide): TD_ATTR_SLICE, slice_parent retained,
 * slice_offset.  Slices of slices resolve to the ultimate parent.  On the
 * GPU a slice of a resident column is read in place (no copy). */
td_t* td_vec_slice(td_t* vec, int64_t offset, int64_t len) {
    if (!vec || TD_IS_ERR(vec)) return vec;
    if (offset < 0 || len < 0 || offset > vec->len || len > vec->len - offset) return TD_ERR_PTR(TD_ERR_RANGE);
    td_t* parent = vec;
    int64_t off = offset;
    if (vec->attrs & TD_ATTR_SLICE) { parent = vec->slice_parent; off += vec->slice_offset; }
    td_t* s = td_alloc(0);
    if (!s) return TD_ERR_PTR(TD_ERR_OOM);
    s->type = parent->type;
    s->attrs = TD_ATTR_SLICE | (parent->attrs & TD_SYM_W_MASK);
    s->len = len;
    s->slice_parent = parent;
    s->slice_offset = off;
    td_retain(parent);
    return s;
}

td_t* td_vec_concat(td_t* a, td_t* b) {
    if (!a || TD_IS_ERR(a)) return a;
    if (!b || TD_IS_ERR(b)) return b;
    if (a->type != b->type) return TD_ERR_PTR(TD_ERR_TYPE);
    size_t esz = td_sym_elem_size(a->type, a->attrs);
    if (esz != td_sym_elem_size(b->type, b->attrs)) return TD_ERR_PTR(TD_ERR_TYPE);
    int64_t n = a->len + b->len;
    td_t* v = a->type == TD_SYM ? td_sym_vec_new(a->attrs & TD_SYM_W_MASK, n) : td_vec_new(a->type, n);
    if (!v || TD_IS_ERR(v)) return v;
    memcpy(td_data(v), td_data(a), (size_t)a->len * esz);
    memcpy((char*)td_data(v) + (size_t)a->len * esz, td_data(b), (size_t)b->len * esz);
    v->len = n;
    if (a->type == TD_LIST || a->type == TD_TABLE) {
        td_t** p = (td_t**)td_data(v);
        for (int64_t i = 0; i < n; i++) if (p[i]) td_retain(p[i]);
    }
    return v;
}

void td_vec_set_null(td_t* vec, int64_t idx, bool is_null) {
    if (!vec || TD_IS_ERR(vec) || (vec->attrs & TD_ATTR_SLICE)) return;
    if (idx < 0 || idx >= vec->len) return;
    tdb_mirror_forget(vec);
    if (is_null) vec->attrs |= TD_ATTR_HAS_NULLS;
    uint8_t* bits;
    if (!(vec->attrs & TD_ATTR_NULLMAP_EXT)) {
        if (vec->len <= 128) {
            bits = vec->nullmap;
        } else {
            td_t* ext = td_vec_new(TD_U8, (vec->len + 7) / 8);
            if (!ext || TD_IS_ERR(ext)) return;
            ext->len = (vec->len + 7) / 8;
            memset(td_data(ext), 0, (size_t)ext->len);
            memcpy(td_data(ext), vec->nullmap, 16);
            vec->ext_nullmap = ext;
            vec->attrs |= TD_ATTR_NULLMAP_EXT;
            bits = (uint8_t*)td_data(ext);
        }
    } else {
        bits = (uint8_t*)td_data(vec->ext_nullmap);
    }
    if (is_null) bits[idx >> 3] |= (uint8_t)(1u << (idx & 7));
    else bits[idx >> 3] &= (uint8_t)~(1u << (idx & 7));
}

bool td_vec_is_null(td_t* vec, int64_t idx) {
    if (!vec || TD_IS_ERR(vec) || idx < 0 || idx >= vec->len) return false;
    if (!(vec->attrs & TD_ATTR_HAS_NULLS)) return false;
    const uint8_t* bits = (vec->attrs & TD_ATTR_NULLMAP_EXT)
                        ? (const uint8_t*)td_data(vec->ext_nullmap) : vec->nullmap;
    return (bits[idx >> 3] >> (idx & 7)) & 1;
}

/* ---- TD_SEL ------------------------------------------------------------------- */
static size_t sel_bytes(int64_t nrows, uint32_t* n_segs_out) {
    uint32_t n_segs = (uint32_t)((nrows + TD_MORSEL_ELEMS - 1) / TD_MORSEL_ELEMS);
    size_t n_words = (size_t)((nrows + 63) / 64);
    *n_segs_out = n_segs;
    return sizeof(td_sel_meta_t) + ((n_segs + 7u) & ~(size_t)7)
         + (((size_t)n_segs * 2 + 7u) & ~(size_t)7) + n_words * 8;
}

td_t* td_sel_new(int64_t nrows) {
    if (nrows < 0) return TD_ERR_PTR(TD_ERR_RANGE);
    uint32_t n_segs;
    size_t sz = sel_bytes(nrows, &n_segs);
    td_t* s = td_alloc(sz);
    if (!s) return TD_ERR_PTR(TD_ERR_OOM);
    s->type = TD_SEL;
    s->len = nrows;
    memset(td_data(s), 0, sz);
    td_sel_meta(s)->n_segs = n_segs;
    return s;
}

void td_sel_recompute(td_t* sel) {
    if (!sel || TD_IS_ERR(sel) || sel->type != TD_SEL) return;
    td_sel_meta_t* m = td_sel_meta(sel);
    uint8_t* flags = td_sel_flags(sel);
    uint16_t* pc = td_sel_popcnt(sel);
    uint64_t* bits = td_sel_bits(sel);
    int64_t n = sel->len, total = 0;
    if (n & 63) bits[n >> 6] &= (1ULL << (n & 63)) - 1;   /* bits past the end never count */
    for (uint32_t s = 0; s < m->n_segs; s++) {
        int64_t r0 = (int64_t)s * TD_MORSEL_ELEMS;
        int64_t rows = n - r0 < TD_MORSEL_ELEMS ? n - r0 : TD_MORSEL_ELEMS;
        int64_t w0 = r0 >> 6, w1 = (r0 + rows + 63) >> 6, cnt = 0;
        for (int64_t w = w0; w < w1; w++) cnt += __builtin_popcountll(bits[w]);
        pc[s] = (uint16_t)cnt;
        total += cnt;
        flags[s] = cnt == 0 ? TD_SEL_NONE : cnt == rows ? TD_SEL_ALL : TD_SEL_MIX;
    }
    m->total_pass = total;
}

/* BOOL vector -> TD_SEL (sel.c:128-161 packs bytes into bits in one
 * thread, then td_sel_recompute counts every segment).  Here the device
 * does both in one pass: tdg_select_bitmap evaluates `pred != 0` over the
 * vector's device copy (uploaded unless resident), packs each warp's 32
 * rows with a ballot and writes every 1024-row segment's flag and popcount;
 * the bits, flags, popcounts and total come back into the block. */
td_t* td_sel_from_pred(td_t* pred) {
    if (!pred || TD_IS_ERR(pred)) return pred;
    if (pred->type != TD_BOOL) return TD_ERR_PTR(TD_ERR_TYPE);
    td_t* s = td_sel_new(pred->len);
    if (!s || TD_IS_ERR(s) || pred->len == 0) return s;
    const int64_t n = pred->len;
    const int64_t words = (n + 63) >> 6;
    const uint32_t n_segs = td_sel_meta(s)->n_segs;
    tdb_ctx c;
    int st = tdb_ctx_begin(&c);
    tdb_devcol dc;
    if (!st) st = tdb_col_device(&c, pred, 0, &dc);
    uint64_t* dbits = NULL;
    uint8_t* dflags = NULL;
    uint16_t* dpop = NULL;
    int64_t* dtotal = NULL;
    if (!st) {
        dbits = tdb_dev_alloc(&c, (size_t)words * 8);
        dflags = tdb_dev_alloc(&c, n_segs);
        dpop = tdb_dev_alloc(&c, (size_t)n_segs * 2);
        dtotal = tdb_dev_alloc(&c, 8);
        if (!dbits || !dflags || !dpop || !dtotal) st = TD_ERR_OOM;
    }
    if (!st) {
        tdg_expr e;
        memset(&e, 0, sizeof(e));
        e.n_cols = 1;
        e.cols[0].data = dc.dptr;
        e.cols[0].type = TD_BOOL;
        e.n_ins = 3;
        e.ins[0].op = TDG_X_COL;
        e.ins[1].op = TDG_X_CONST;
        e.ins[2].op = TDG_X_NE; e.ins[2].a = 0; e.ins[2].b = 1;
        e.out = 2;
        st = tdg_select_bitmap(n, &e, NULL, dbits, dflags, dpop, dtotal, c.stream);
    }
    int64_t total = 0;
    if (!st) st = tdb_d2h(&c, td_sel_bits(s), dbits, (size_t)words * 8);
    if (!st) st = tdb_d2h(&c, td_sel_flags(s), dflags, n_segs);
    if (!st) st = tdb_d2h(&c, td_sel_popcnt(s), dpop, (size_t)n_segs * 2);
    if (!st) st = tdb_d2h(&c, &total, dtotal, 8);
    if (!st) st = tdb_ctx_sync(&c);
    tdb_ctx_end(&c);
    if (st) { td_release(s); return TD_ERR_PTR(st); }
    td_sel_meta(s)->total_pass = total;
    return s;
}

td_t* td_sel_and(td_t* a, td_t* b) {
    if (!a || TD_IS_ERR(a)) return a;
    if (!b || TD_IS_ERR(b)) return b;
    if (a->type != TD_SEL || b->type != TD_SEL) return TD_ERR_PTR(TD_ERR_TYPE);
    if (a->len != b->len) return TD_ERR_PTR(TD_ERR_RANGE);
    td_t* s = td_sel_new(a->len);
    if (!s || TD_IS_ERR(s)) return s;
    uint64_t *d = td_sel_bits(s), *x = td_sel_bits(a), *y = td_sel_bits(b);
    for (int64_t w = 0; w < (a->len + 63) / 64; w++) d[w] = x[w] & y[w];
    td_sel_recompute(s);
    return s;
}
