/*
 * td_execute: walks a Teide DAG and runs its relational operators on the GPU.
 *
 * The walk mirrors exec_node (Teide src/ops/exec.c:11561-12321), with every
 * compute step lowered to the kernels behind tdg.h and no CPU execution path:
 *
 *   OP_SCAN / OP_CONST     host objects, uploaded on first use (or resident)
 *   element-wise ops       compiled to a tdg_expr program (exec.c:760-918);
 *                          evaluated on the device when a value is needed
 *   OP_FILTER on a table   lazy: the table plus a predicate program, like
 *                          Teide's g->selection (exec.c:11674-11739); the
 *                          consumer fuses it, or the final step compacts it
 *   OP_FILTER on a vector  lazy filtered vector; consumed by OP_GROUP it
 *                          defines the README pipeline (below), otherwise
 *                          compacted
 *   OP_GROUP               fused select + group-by (exec_group 5542-6879)
 *   OP_JOIN                build + probe + gather (exec_join 8130-8741)
 *   OP_COUNT/SUM/MIN/MAX/AVG  scalar reductions on the device
 *
 * Two DAG shapes get defined semantics here that Teide's CPU executor does
 * not give them:
 *   1. The README pipeline -- OP_GROUP whose key and aggregate inputs are
 *      td_filter(td_scan(col), pred) vectors sharing one predicate -- groups
 *      the rows that pass the predicate.  (Teide's exec_group reads such
 *      vectors past their end, exec.c:5560 with 5654-5663.)  Columns are
 *      named after the scanned column, as the filter-then-group pipeline
 *      names them.
 *   2. Filter -> join -> group in one graph: when OP_GROUP runs in a graph
 *      bound to no table (td_graph_new(NULL)) that holds exactly one OP_JOIN,
 *      the group reads the join's output -- the same hookup Teide makes for
 *      a factorized OP_EXPAND (exec.c:11768-11800).  Its scans name columns
 *      of the join output (left columns, then right non-key columns) and the
 *      join is never materialized.  In Teide this graph fails with
 *      TD_ERR_SCHEMA.
 *
 * Results are host td_t objects.  Device copies of result columns stay
 * resident until the host column is freed, so a second graph over a result
 * (the two-call join -> group chain) uploads nothing.
 */

#include "internal.h"
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    td_t*           obj;       /* retained host table, vector or atom */
    int             lazy;      /* rows of obj are filtered by pred / dsel */
    int             has_pred;
    tdg_expr        pred;      /* over the rows of obj (vectors: rows of rows_tbl) */
    const uint64_t* dsel;      /* device TD_SEL bits */
} val_t;

typedef struct {
    td_graph_t* g;
    tdb_ctx     c;
    int         dev_only;      /* a group result that only a sort reads stays on the device */
} ex_t;

static val_t vnone(void) { val_t v; memset(&v, 0, sizeof(v)); return v; }
static void vfree(val_t* v) { if (v->obj && !TD_IS_ERR(v->obj)) td_release(v->obj); v->obj = NULL; }
#define CALL(expr) (tdb_note_kernel(), (expr))

/* ---- expression compilation ----------------------------------------------------- */
typedef struct {
    ex_t*     x;
    td_t*     tbl;             /* table scans resolve against */
    tdg_expr* e;
    uint32_t  ids[TDG_MAX_INS];
    int       regs[TDG_MAX_INS];
    int       n_memo;
    int       err;
} xc_t;

static td_t* scan_table_of(ex_t* x, td_op_ext_t* ext, td_t* dflt) {
    uint16_t tid = 0;
    memcpy(&tid, ext->base.pad, sizeof(tid));
    if (tid > 0 && x->g->tables && tid - 1 < x->g->n_tables) return x->g->tables[tid - 1];
    return dflt;
}

static int emit_ins(xc_t* xc, uint8_t op, int a, int b, int kind, int64_t imm) {
    tdg_expr* e = xc->e;
    if (e->n_ins >= TDG_MAX_INS) { xc->err = TD_ERR_NYI; return -1; }
    tdg_ins* I = &e->ins[e->n_ins];
    memset(I, 0, sizeof(*I));
    I->op = op; I->a = (uint8_t)(a < 0 ? 0 : a); I->b = (uint8_t)(b < 0 ? 0 : b);
    I->kind = (uint8_t)kind; I->imm = imm;
    return e->n_ins++;
}

static int add_col(xc_t* xc, const tdb_devcol* d) {
    tdg_expr* e = xc->e;
    for (int i = 0; i < e->n_cols; i++) if (e->cols[i].data == d->dptr) return i;
    if (e->n_cols >= TDG_MAX_XCOLS) { xc->err = TD_ERR_NYI; return -1; }
    tdg_col* c = &e->cols[e->n_cols];
    memset(c, 0, sizeof(*c));
    c->data = d->dptr; c->type = d->type; c->attrs = d->attrs;
    return e->n_cols++;
}

static int to_kind(xc_t* xc, int r, int kind) {
    if (r < 0) return r;
    int k = xc->e->ins[r].kind;
    if (k == kind) return r;
    return emit_ins(xc, kind == 1 ? TDG_X_TOF64 : TDG_X_TOI64, r, 0, kind, 0);
}

static int xc_node(xc_t* xc, td_op_t* op) {
    if (!op || xc->err) { if (!xc->err) xc->err = TD_ERR_NYI; return -1; }
    for (int i = 0; i < xc->n_memo; i++) if (xc->ids[i] == op->id) return xc->regs[i];
    int r = -1;
    td_graph_t* g = xc->x->g;
    switch (op->opcode) {
        case OP_SCAN: {
            td_op_ext_t* ext = tdb_find_ext(g, op->id);
            td_t* tbl = ext ? scan_table_of(xc->x, ext, xc->tbl) : NULL;
            td_t* col = tbl ? td_table_get_col(tbl, ext->sym) : NULL;
            if (!col) { xc->err = TD_ERR_SCHEMA; return -1; }
            if (td_parted_nrows(col) != td_table_nrows(xc->tbl)) { xc->err = TD_ERR_LENGTH; return -1; }
            tdb_devcol d;
            int st = tdb_col_device(&xc->x->c, col, 0, &d);
            if (st) { xc->err = st; return -1; }
            int ci = add_col(xc, &d);
            if (ci < 0) return -1;
            r = emit_ins(xc, TDG_X_COL, 0, 0, d.type == TD_F64 ? 1 : 0, ci);
            break;
        }
        case OP_CONST: {
            td_op_ext_t* ext = tdb_find_ext(g, op->id);
            td_t* lit = ext ? ext->literal : NULL;
            double f; int64_t i; int isf;
            if (lit && tdb_atom_numeric(lit, &f, &i, &isf)) {
                int64_t bits;
                if (isf) memcpy(&bits, &f, 8); else bits = i;
                r = emit_ins(xc, TDG_X_CONST, 0, 0, isf, bits);
            } else if (lit && lit->type == TD_ATOM_STR) {
                /* string constant compares as its symbol id (exec.c:829-839);
                 * an unknown string matches no symbol, whose ids are >= 0 */
                int64_t sid = td_sym_find(td_str_ptr(lit), td_str_len(lit));
                r = emit_ins(xc, TDG_X_CONST, 0, 0, 0, sid < 0 ? -1 : sid);
            } else {
                xc->err = TD_ERR_NYI;
                return -1;
            }
            break;
        }
        case OP_ALIAS: case OP_MATERIALIZE:
            r = xc_node(xc, op->inputs[0]);
            break;
        case OP_EQ: case OP_NE: case OP_LT: case OP_LE: case OP_GT: case OP_GE: {
            int a = xc_node(xc, op->inputs[0]), b = xc_node(xc, op->inputs[1]);
            if (a < 0 || b < 0) return -1;
            int kind = (xc->e->ins[a].kind || xc->e->ins[b].kind) ? 1 : 0;
            a = to_kind(xc, a, kind); b = to_kind(xc, b, kind);
            if (a < 0 || b < 0) return -1;
            r = emit_ins(xc, (uint8_t)(TDG_X_EQ + (op->opcode - OP_EQ)), a, b, 0, 0);
            break;
        }
        case OP_AND: case OP_OR: {
            int a = xc_node(xc, op->inputs[0]), b = xc_node(xc, op->inputs[1]);
            if (a < 0 || b < 0) return -1;
            r = emit_ins(xc, op->opcode == OP_AND ? TDG_X_AND : TDG_X_OR, a, b, 0, 0);
            break;
        }
        case OP_NOT: {
            int a = xc_node(xc, op->inputs[0]);
            if (a < 0) return -1;
            r = emit_ins(xc, TDG_X_NOT, a, 0, 0, 0);
            break;
        }
        case OP_NEG: case OP_ABS: {
            int a = xc_node(xc, op->inputs[0]);
            if (a < 0) return -1;
            r = emit_ins(xc, op->opcode == OP_NEG ? TDG_X_NEG : TDG_X_ABS, a, 0, xc->e->ins[a].kind, 0);
            break;
        }
        case OP_CAST: {
            int a = xc_node(xc, op->inputs[0]);
            if (a < 0) return -1;
            r = to_kind(xc, a, op->out_type == TD_F64 ? 1 : 0);
            break;
        }
        case OP_ADD: case OP_SUB: case OP_MUL: case OP_DIV: case OP_MOD:
        case OP_MIN2: case OP_MAX2: {
            int a = xc_node(xc, op->inputs[0]), b = xc_node(xc, op->inputs[1]);
            if (a < 0 || b < 0) return -1;
            int kind = (op->opcode == OP_DIV || xc->e->ins[a].kind || xc->e->ins[b].kind) ? 1 : 0;
            a = to_kind(xc, a, kind); b = to_kind(xc, b, kind);
            if (a < 0 || b < 0) return -1;
            static const uint8_t map[] = {
                [OP_ADD] = TDG_X_ADD, [OP_SUB] = TDG_X_SUB, [OP_MUL] = TDG_X_MUL, [OP_DIV] = TDG_X_DIV,
                [OP_MOD] = TDG_X_MOD, [OP_MIN2] = TDG_X_MIN2, [OP_MAX2] = TDG_X_MAX2 };
            r = emit_ins(xc, map[op->opcode], a, b, kind, 0);
            break;
        }
        default:
            xc->err = TD_ERR_NYI;
            return -1;
    }
    if (r >= 0 && xc->n_memo < TDG_MAX_INS) {
        xc->ids[xc->n_memo] = op->id;
        xc->regs[xc->n_memo++] = r;
    }
    return r;
}

static int compile_expr(ex_t* x, td_t* tbl, td_op_t* op, tdg_expr* e) {
    memset(e, 0, sizeof(*e));
    if (!tbl || tbl->type != TD_TABLE) return TD_ERR_SCHEMA;
    xc_t xc;
    memset(&xc, 0, sizeof(xc));
    xc.x = x; xc.tbl = tbl; xc.e = e;
    int r = xc_node(&xc, op);
    if (xc.err) return xc.err;
    if (r < 0) return TD_ERR_NYI;
    e->out = r;
    return TD_OK;
}

/* p = p AND q */
static int expr_and(tdg_expr* p, const tdg_expr* q) {
    if (p->n_ins == 0) { *p = *q; return TD_OK; }
    if (q->n_ins == 0) return TD_OK;
    if (p->n_ins + q->n_ins + 1 > TDG_MAX_INS) return TD_ERR_NYI;
    int colmap[TDG_MAX_XCOLS];
    for (int i = 0; i < q->n_cols; i++) {
        int found = -1;
        for (int j = 0; j < p->n_cols; j++) if (p->cols[j].data == q->cols[i].data) found = j;
        if (found < 0) {
            if (p->n_cols >= TDG_MAX_XCOLS) return TD_ERR_NYI;
            p->cols[p->n_cols] = q->cols[i];
            found = p->n_cols++;
        }
        colmap[i] = found;
    }
    int base = p->n_ins;
    for (int k = 0; k < q->n_ins; k++) {
        tdg_ins I = q->ins[k];
        if (I.op == TDG_X_COL) I.imm = colmap[I.imm];
        else if (I.op != TDG_X_CONST) { I.a = (uint8_t)(I.a + base); I.b = (uint8_t)(I.b + base); }
        p->ins[p->n_ins++] = I;
    }
    tdg_ins* A = &p->ins[p->n_ins];
    memset(A, 0, sizeof(*A));
    A->op = TDG_X_AND; A->a = (uint8_t)p->out; A->b = (uint8_t)(base + q->out);
    p->out = p->n_ins++;
    return TD_OK;
}

/* ---- host result construction ------------------------------------------------------ */

/* New host vector of n elements with the element type of `like`. */
static td_t* vec_like(int8_t type, uint8_t attrs, int64_t n) {
    td_t* v = type == TD_SYM ? td_sym_vec_new(attrs & TD_SYM_W_MASK, n) : td_vec_new(type, n);
    if (v && !TD_IS_ERR(v)) v->len = n;
    return v;
}

/* Copy n elements from the device into a new host vector.  With `deferred`
 * the copy is only queued: the caller synchronizes the stream (once for all
 * the columns of a result) before reading the vector.  deferred == 2 marks a
 * column the executor may leave on the device: while x->dev_only is set the
 * vector is only the handle of its device copy (its host bytes are never
 * written, and it does not outlive the query). */
static td_t* fetch_vec_q(ex_t* x, const void* dptr, int8_t type, uint8_t attrs, int64_t n, int deferred) {
    td_t* v = vec_like(type, attrs, n);
    if (!v || TD_IS_ERR(v)) return v ? v : TD_ERR_PTR(TD_ERR_OOM);
    if (deferred == 2 && x->dev_only && tdb_adopt_mirror(&x->c, v, (void*)dptr)) return v;
    size_t bytes = (size_t)n * td_sym_elem_size(type, attrs);
    if (bytes >= ((size_t)2 << 20)) tdb_pin_host(v);     /* heap-mapped block: DMA straight into it */
    int st = deferred ? tdb_d2h_async(&x->c, td_data(v), dptr, bytes) : tdb_d2h(&x->c, td_data(v), dptr, bytes);
    if (st) { td_release(v); return TD_ERR_PTR(st); }
    tdb_adopt_mirror(&x->c, v, (void*)dptr);
    return v;
}

/* A new host vector holding n elements of a result the kernels wrote into
 * mapped host memory (read after the stream synchronized). */
static td_t* host_vec(const void* hptr, int8_t type, uint8_t attrs, int64_t n) {
    td_t* v = vec_like(type, attrs, n);
    if (!v || TD_IS_ERR(v)) return v ? v : TD_ERR_PTR(TD_ERR_OOM);
    const size_t bytes = (size_t)n * td_sym_elem_size(type, attrs);
    if (bytes) memcpy(td_data(v), hptr, bytes);
    return v;
}

static td_t* fetch_vec(ex_t* x, const void* dptr, int8_t type, uint8_t attrs, int64_t n) {
    return fetch_vec_q(x, dptr, type, attrs, n, 0);
}

/* ---- values ------------------------------------------------------------------------------- */
static td_t* exec_value(ex_t* x, td_op_t* op, val_t* out);

/* Device columns of a whole table, in column order. */
static int table_dev_cols(ex_t* x, td_t* t, tdg_col* cols, int max) {
    int64_t nc = td_table_ncols(t);
    if (nc > max) return -TD_ERR_NYI;
    for (int64_t j = 0; j < nc; j++) {
        tdb_devcol d;
        int st = tdb_col_device(&x->c, td_table_get_col_idx(t, j), 0, &d);
        if (st) return -st;
        memset(&cols[j], 0, sizeof(tdg_col));
        cols[j].data = d.dptr; cols[j].type = d.type; cols[j].attrs = d.attrs;
    }
    return (int)nc;
}

#define MAX_TCOLS 256

/* Compact a lazy table or vector on the device and bring it to the host. */
static td_t* materialize(ex_t* x, val_t* v) {
    if (!v->lazy) { td_t* o = v->obj; td_retain(o); return o; }
    td_t* src = v->obj;
    int is_tbl = src->type == TD_TABLE;
    int64_t n = is_tbl ? td_table_nrows(src) : src->len;
    const tdg_expr* pred = v->has_pred ? &v->pred : NULL;
    void* ws = tdb_dev_alloc(&x->c, tdg_select_ws_bytes(n));
    int64_t* dcount = tdb_dev_alloc(&x->c, 8);
    if (!ws || !dcount) return TD_ERR_PTR(TD_ERR_OOM);
    int st = CALL(tdg_select_count(n, pred, v->dsel, ws, dcount, x->c.stream));
    if (st) return TD_ERR_PTR(st);
    int64_t m = 0;
    st = tdb_d2h(&x->c, &m, dcount, 8);
    if (st) return TD_ERR_PTR(st);
    tdg_col cols[MAX_TCOLS];
    void* dst[MAX_TCOLS];
    int nc;
    if (is_tbl) {
        nc = table_dev_cols(x, src, cols, MAX_TCOLS);
        if (nc < 0) return TD_ERR_PTR(-nc);
    } else {
        tdb_devcol d;
        st = tdb_col_device(&x->c, src, 0, &d);
        if (st) return TD_ERR_PTR(st);
        memset(&cols[0], 0, sizeof(tdg_col));
        cols[0].data = d.dptr; cols[0].type = d.type; cols[0].attrs = d.attrs;
        nc = 1;
    }
    for (int j = 0; j < nc; j++) {
        dst[j] = tdb_dev_alloc(&x->c, (size_t)(m ? m : 1) * td_sym_elem_size(cols[j].type, cols[j].attrs));
        if (!dst[j]) return TD_ERR_PTR(TD_ERR_OOM);
    }
    st = CALL(tdg_select_gather(n, pred, v->dsel, ws, nc, cols, dst, x->c.stream));
    if (st) return TD_ERR_PTR(st);
    if (!is_tbl) return fetch_vec(x, dst[0], cols[0].type, cols[0].attrs, m);
    td_t* out = td_table_new(nc);
    if (!out || TD_IS_ERR(out)) return out;
    for (int j = 0; j < nc; j++) {
        td_t* col = fetch_vec(x, dst[j], cols[j].type, cols[j].attrs, m);
        if (TD_IS_ERR(col)) { td_release(out); return col; }
        out = td_table_add_col(out, td_table_col_name(src, j), col);
        td_release(col);
        if (TD_IS_ERR(out)) return out;
    }
    return out;
}

/* ---- group-by --------------------------------------------------------------------------- */

/* One key or aggregate input of a group-by, resolved to a device column. */
typedef struct {
    tdg_col  col;
    int64_t  name;      /* output base name: column symbol, or -1 for expressions */
    int      filtered;  /* came through td_filter(vector, pred) */
    td_op_t* pred_op;
    td_t*    src;       /* host column (for output type), may be NULL for expressions */
    int8_t   type;
    uint8_t  attrs;
    int      has_stats;
    int64_t  kmin, kmax;
} gin_t;

/* Join output as a group-by input: where each named column comes from. */
typedef struct {
    td_t* left;
    td_t* right;
    td_op_ext_t* jext;
} jsrc_t;

static int col_of_join(ex_t* x, jsrc_t* js, int64_t sym, td_t** col, int* side) {
    td_t* c = td_table_get_col(js->left, sym);
    if (c) { *col = c; *side = 0; return TD_OK; }
    for (int k = 0; k < js->jext->join.n_join_keys; k++) {
        td_op_ext_t* rk = tdb_find_ext(x->g, js->jext->join.right_keys[k]->id);
        if (rk && rk->base.opcode == OP_SCAN && rk->sym == sym) return TD_ERR_SCHEMA;
    }
    c = td_table_get_col(js->right, sym);
    if (!c) return TD_ERR_SCHEMA;
    *col = c; *side = 1;
    return TD_OK;
}

static int resolve_gin(ex_t* x, td_op_t* op, td_t* tbl, jsrc_t* js, int want_stats, gin_t* gi) {
    memset(gi, 0, sizeof(*gi));
    gi->name = -1;
    td_op_t* o = op;
    while (o && (o->opcode == OP_ALIAS || o->opcode == OP_MATERIALIZE)) o = o->inputs[0];
    if (o && o->opcode == OP_FILTER && o->inputs[0] &&
        (o->inputs[0]->opcode == OP_SCAN || o->inputs[0]->opcode == OP_ALIAS)) {
        gi->filtered = 1;
        gi->pred_op = o->inputs[1];
        o = o->inputs[0];
        while (o && o->opcode == OP_ALIAS) o = o->inputs[0];
    }
    if (!o) return TD_ERR_NYI;
    if (o->opcode == OP_SCAN) {
        td_op_ext_t* ext = tdb_find_ext(x->g, o->id);
        if (!ext) return TD_ERR_NYI;
        td_t* col = NULL;
        int side = 0;
        if (js) {
            int st = col_of_join(x, js, ext->sym, &col, &side);
            if (st) return st;
        } else {
            td_t* t = scan_table_of(x, ext, tbl);
            col = t ? td_table_get_col(t, ext->sym) : NULL;
            if (!col) return TD_ERR_SCHEMA;
            if (td_parted_nrows(col) != td_table_nrows(tbl)) return TD_ERR_LENGTH;
        }
        tdb_devcol d;
        int st = tdb_col_device(&x->c, col, want_stats, &d);
        if (st) return st;
        gi->col.data = d.dptr; gi->col.type = d.type; gi->col.attrs = d.attrs; gi->col.side = (uint8_t)side;
        gi->name = ext->sym;
        gi->src = col;
        gi->type = d.type;                      /* a parted column's segments' type */
        gi->attrs = d.attrs;
        gi->has_stats = d.has_stats;
        gi->kmin = d.kmin; gi->kmax = d.kmax;
        return TD_OK;
    }
    if (js) return TD_ERR_NYI;     /* expressions over a join output are not lowered */
    /* expression input: evaluate on the device into a temporary column */
    tdg_expr e;
    int st = compile_expr(x, tbl, o, &e);
    if (st) return st;
    int kind = e.ins[e.out].kind;
    int64_t n = td_table_nrows(tbl);
    void* d = tdb_dev_alloc(&x->c, (size_t)(n ? n : 1) * 8);
    if (!d) return TD_ERR_OOM;
    st = CALL(tdg_eval(&e, n, d, kind, x->c.stream));
    if (st) return st;
    gi->col.data = d; gi->col.type = kind ? TD_F64 : TD_I64;
    gi->type = gi->col.type;
    if (want_stats && !kind) {
        int64_t* mm = tdb_dev_alloc(&x->c, 16);
        int64_t h[2];
        if (!mm) return TD_ERR_OOM;
        st = CALL(tdg_minmax(gi->col, n, mm, x->c.stream));
        if (!st) st = tdb_d2h(&x->c, h, mm, 16);
        if (st) return st;
        gi->has_stats = 1; gi->kmin = h[0]; gi->kmax = h[1];
    }
    return TD_OK;
}

static int64_t agg_name(uint16_t op, int64_t base, int a) {
    const char* sfx = op == OP_SUM ? "_sum" : op == OP_COUNT ? "_count" : op == OP_AVG ? "_mean"
                    : op == OP_MIN ? "_min" : op == OP_MAX ? "_max" : "";
    char buf[300];
    int n;
    td_t* s = base >= 0 ? td_sym_str(base) : NULL;
    if (s && td_str_len(s) + strlen(sfx) < sizeof(buf)) {
        n = (int)td_str_len(s);
        memcpy(buf, td_str_ptr(s), (size_t)n);
        memcpy(buf + n, sfx, strlen(sfx));
        n += (int)strlen(sfx);
    } else {
        n = snprintf(buf, sizeof(buf), "_e%d%s", a, sfx);
    }
    return td_sym_intern(buf, (size_t)n);
}

typedef struct {
    const tdg_join_desc* jd;
    const tdg_join_plan* jp;
    void*                jws;
    td_t*                rkey;     /* host build key column (one key), or NULL */
} jrun_t;

/* ---- shared join builds -------------------------------------------------------------------
 * A server answers many join queries over the same resident build table; the
 * payload map of that build side (each build key's group slot) is the same
 * for all of them.  While this thread's flag is set (td_server's workers set
 * it), the map is built once by tdg_join_payload_build into a kept workspace
 * and every later query with the same build key column, key range and group
 * keys probes it with TDG_JOIN_PREBUILT, concurrently with the others.  An
 * entry matches only the same resident device copies (tdb_col_stamp: a
 * column freed, modified or unpinned since gets a new stamp), so a stale map
 * is never read. */
#define TDB_BCACHE 8
typedef struct {
    int           ready;
    int           users;                       /* probes in flight */
    uint64_t      tick;
    uint64_t      rstamp, gstamp[TDG_MAX_KEYS];
    int64_t       gmin[TDG_MAX_KEYS], gmax[TDG_MAX_KEYS];
    int32_t       nk;
    tdg_join_desc jd;
    tdg_join_plan jp;
    void*         jws;
} bentry_t;

static pthread_mutex_t bc_mu = PTHREAD_MUTEX_INITIALIZER;
static bentry_t bc[TDB_BCACHE];
static uint64_t bc_tick;
static _Thread_local int tls_share_builds;

void tdb_share_builds(int on) { tls_share_builds = on; }

void tdb_build_cache_clear(void) {
    pthread_mutex_lock(&bc_mu);
    for (int i = 0; i < TDB_BCACHE; i++) {
        if (!bc[i].ready || bc[i].users) continue;
        tdb_dev_free_persistent(bc[i].jws);
        memset(&bc[i], 0, sizeof(bc[i]));
    }
    pthread_mutex_unlock(&bc_mu);
}

static int bc_match(const bentry_t* e, const jrun_t* jr, const tdg_group_desc* d, const uint64_t* gst,
                    uint64_t rst) {
    if (!e->ready || e->rstamp != rst || e->nk != d->n_keys) return 0;
    if (e->jd.n_right != jr->jd->n_right || e->jd.rkey_min != jr->jd->rkey_min ||
        e->jd.rkey_max != jr->jd->rkey_max || e->jp.n_slots != jr->jp->n_slots || e->jp.method != jr->jp->method)
        return 0;
    for (int k = 0; k < d->n_keys; k++)
        if (e->gstamp[k] != gst[k] || e->gmin[k] != d->key_min[k] || e->gmax[k] != d->key_max[k]) return 0;
    return 1;
}

/* A kept map for this join -> group-by (users counted), building it on a
 * miss; NULL when sharing does not apply. */
static bentry_t* bc_acquire(ex_t* x, const jrun_t* jr, const tdg_group_desc* d, const tdg_group_plan* gp,
                            const gin_t* keys) {
    if (!tls_share_builds || !jr->rkey || jr->jd->n_keys != 1 || jr->jd->join_type != 0 || !d->have_range) return NULL;
    const uint64_t rst = tdb_col_stamp(jr->rkey);
    if (!rst) return NULL;
    uint64_t gst[TDG_MAX_KEYS];
    for (int k = 0; k < d->n_keys; k++) {
        if (d->keys[k].side != 1 || !keys[k].src) return NULL;      /* every group key from the build side */
        if (!(gst[k] = tdb_col_stamp(keys[k].src))) return NULL;
    }
    pthread_mutex_lock(&bc_mu);
    for (int i = 0; i < TDB_BCACHE; i++) {
        if (bc_match(&bc[i], jr, d, gst, rst)) {
            bc[i].users++;
            bc[i].tick = ++bc_tick;
            pthread_mutex_unlock(&bc_mu);
            return &bc[i];
        }
    }
    pthread_mutex_unlock(&bc_mu);
    void* jws = tdb_dev_alloc_persistent(jr->jp->ws_bytes);
    if (!jws) return NULL;
    int32_t used = 0;
    int st = CALL(tdg_join_payload_build(jr->jd, jr->jp, jws, d, gp, &used, x->c.stream));
    if (st || !used) { tdb_dev_free_persistent(jws); return NULL; }
    pthread_mutex_lock(&bc_mu);
    int slot = -1;
    for (int i = 0; i < TDB_BCACHE; i++) {
        if (!bc[i].ready) { slot = i; break; }
        if (!bc[i].users && (slot < 0 || bc[i].tick < bc[slot].tick)) slot = i;
    }
    bentry_t* e = NULL;
    if (slot >= 0) {
        e = &bc[slot];
        if (e->ready) tdb_dev_free_persistent(e->jws);
        memset(e, 0, sizeof(*e));
        e->ready = 1;
        e->users = 1;
        e->tick = ++bc_tick;
        e->rstamp = rst;
        e->nk = d->n_keys;
        for (int k = 0; k < d->n_keys; k++) { e->gstamp[k] = gst[k]; e->gmin[k] = d->key_min[k]; e->gmax[k] = d->key_max[k]; }
        e->jd = *jr->jd;
        e->jp = *jr->jp;
        e->jws = jws;
    }
    pthread_mutex_unlock(&bc_mu);
    if (!e) tdb_dev_free_persistent(jws);          /* every entry busy: this query builds its own */
    return e;
}

/* ---- launch-shape autotuner of the streaming kernels ------------------------------------
 * The vector kernels of the group-by and of the fused join probe run as many
 * persistent CTAs per SM as fit unless the plan says otherwise.  The first
 * time a shape class -- method, log2 of the rows and of the slots, the
 * number of aggregates, join or not -- of at least 2^22 rows is met, the
 * query runs once per candidate CTAs-per-SM value with CUDA events around
 * the call; the fastest is kept in memory and in the tuner's JSON file
 * ($TD_TUNE_CACHE), so later queries of that class, in this process or a
 * later one, launch with it.  Every candidate run computes the whole
 * result, so the query's answer is the last run's.  Teide's counterparts
 * are fixed constants (td.h:190-197 morsel sizes, exec.c:4230-4233 radix
 * fan-out).  TD_NO_AUTOTUNE in the environment keeps the defaults. */
#define TDB_TUNE_MIN_ROWS ((int64_t)1 << 22)
#define TDB_TUNE_MEM 64
static pthread_mutex_t tn_mu = PTHREAD_MUTEX_INITIALIZER;
static struct { char key[64]; int32_t cps; } tn_mem[TDB_TUNE_MEM];
static int tn_n;

static int ilog2(int64_t x) { int k = 0; while (x > 1) { x >>= 1; k++; } return k; }

static void tune_key(const tdg_group_desc* d, const tdg_group_plan* p, int join, char* key, size_t n) {
    snprintf(key, n, "stream:m%d:s%d:r%d:g%d:k%d:a%d:j%d", p->method, p->smem, ilog2(d->nrows), ilog2(p->n_slots),
             d->n_keys, d->n_aggs, join);
}

/* 1 and *cps when the class is known (in memory, else in the JSON file). */
static int tune_lookup(const char* key, int32_t* cps) {
    int found = 0;
    pthread_mutex_lock(&tn_mu);
    for (int i = 0; i < tn_n && !found; i++)
        if (!strcmp(tn_mem[i].key, key)) { *cps = tn_mem[i].cps; found = 1; }
    pthread_mutex_unlock(&tn_mu);
    if (found) return 1;
    int64_t tile = 0;
    if (!tdb_tune_load(key, &tile, cps)) return 0;
    pthread_mutex_lock(&tn_mu);
    if (tn_n < TDB_TUNE_MEM) { snprintf(tn_mem[tn_n].key, sizeof(tn_mem[0].key), "%s", key); tn_mem[tn_n++].cps = *cps; }
    pthread_mutex_unlock(&tn_mu);
    return 1;
}

static void tune_remember(const char* key, int32_t cps) {
    pthread_mutex_lock(&tn_mu);
    if (tn_n < TDB_TUNE_MEM) { snprintf(tn_mem[tn_n].key, sizeof(tn_mem[0].key), "%s", key); tn_mem[tn_n++].cps = cps; }
    pthread_mutex_unlock(&tn_mu);
    tdb_tune_store(key, 0, cps);
}

typedef struct {
    const jrun_t* jr;
    const tdg_expr* pp;
    const uint64_t* dsel;
    const tdg_group_desc* d;
    tdg_group_plan* plan;
    void* ws;
    const tdg_group_out* out;
    void* stream;
} grun_t;

static int grun(void* a) {
    grun_t* r = a;
    if (r->jr)
        return tdg_join_group_run(r->jr->jd, r->jr->jp, r->jr->jws, r->pp, r->dsel, r->d, r->plan, r->ws, r->out,
                                  r->stream);
    return tdg_group_run(r->d, r->pp, r->dsel, r->plan, r->ws, r->out, r->stream);
}

/* Runs the query, first choosing the plan's launch shape for its class. */
static int run_tuned(ex_t* x, grun_t* r) {
    if (r->d->nrows < TDB_TUNE_MIN_ROWS || getenv("TD_NO_AUTOTUNE")) return grun(r);
    char key[64];
    tune_key(r->d, r->plan, r->jr != NULL, key, sizeof(key));
    int32_t cps = 0;
    if (tune_lookup(key, &cps)) {
        r->plan->ctas_per_sm = cps;
        return grun(r);
    }
    static const int32_t cand[] = {1, 2, 4, 0};      /* 0 (all that fit) last: its result is kept */
    float best = -1.f;
    int32_t best_cps = 0;
    int st = TD_OK;
    for (int i = 0; i < 4; i++) {
        r->plan->ctas_per_sm = cand[i];
        const float ms = tdb_time_call(&x->c, grun, r, &st);
        if (st) return st;
        if (ms > 0 && (best < 0 || ms < best)) { best = ms; best_cps = cand[i]; }
    }
    if (best > 0) tune_remember(key, best_cps);
    r->plan->ctas_per_sm = best_cps;
    return TD_OK;
}

static void bc_release(bentry_t* e) {
    pthread_mutex_lock(&bc_mu);
    e->users--;
    pthread_mutex_unlock(&bc_mu);
}

/* Group-by over `tbl` rows (or over a join's output when js/jr are given). */
static td_t* run_group(ex_t* x, td_op_ext_t* ext, td_t* tbl, const tdg_expr* pred_in,
                       const uint64_t* dsel, jsrc_t* js, jrun_t* jr) {
    int nk = ext->n_keys, na = ext->n_aggs;
    if (nk > TDG_MAX_KEYS || na > TDG_MAX_AGGS) return TD_ERR_PTR(TD_ERR_NYI);
    gin_t keys[TDG_MAX_KEYS], ins[TDG_MAX_AGGS];
    td_op_t* pred_op = NULL;
    int st;
    for (int k = 0; k < nk; k++) {
        st = resolve_gin(x, ext->keys[k], tbl, js, 1, &keys[k]);
        if (st) return TD_ERR_PTR(st);
        if (keys[k].filtered) {
            if (pred_op && pred_op != keys[k].pred_op) return TD_ERR_PTR(TD_ERR_NYI);
            pred_op = keys[k].pred_op;
        }
    }
    for (int a = 0; a < na; a++) {
        memset(&ins[a], 0, sizeof(gin_t));
        ins[a].name = -1;
        td_op_t* in = ext->agg_ins[a];
        if (ext->agg_ops[a] == OP_COUNT && in && in->opcode == OP_CONST) continue;
        st = resolve_gin(x, in, tbl, js, 0, &ins[a]);
        if (st == TD_ERR_NYI && ext->agg_ops[a] == OP_COUNT) { st = TD_OK; continue; }
        if (st) return TD_ERR_PTR(st);
        if (ins[a].filtered) {
            if (pred_op && pred_op != ins[a].pred_op) return TD_ERR_PTR(TD_ERR_NYI);
            pred_op = ins[a].pred_op;
        }
    }
    /* selection: caller's lazy filter AND the README-style shared predicate */
    tdg_expr pred;
    memset(&pred, 0, sizeof(pred));
    if (pred_in) pred = *pred_in;
    if (pred_op) {
        if (js) return TD_ERR_PTR(TD_ERR_NYI);
        tdg_expr p2;
        st = compile_expr(x, tbl, pred_op, &p2);
        if (st) return TD_ERR_PTR(st);
        st = expr_and(&pred, &p2);
        if (st) return TD_ERR_PTR(st);
    }
    const tdg_expr* pp = pred.n_ins ? &pred : NULL;

    tdg_group_desc d;
    memset(&d, 0, sizeof(d));
    d.nrows = js ? 0 : td_table_nrows(tbl);
    d.n_keys = nk;
    d.n_aggs = na;
    d.have_range = 1;
    int jtype = jr ? jr->jd->join_type : 0;
    for (int k = 0; k < nk; k++) {
        d.keys[k] = keys[k].col;
        if (!keys[k].has_stats) { d.have_range = 0; continue; }
        d.key_min[k] = keys[k].kmin;
        d.key_max[k] = keys[k].kmax;
        /* outer joins zero-fill the unmatched side: 0 must be a valid key */
        int nullable = (jtype >= 1 && keys[k].col.side == 1) || (jtype == 2 && keys[k].col.side == 0);
        if (nullable) {
            if (d.key_min[k] > 0) d.key_min[k] = 0;
            if (d.key_max[k] < 0) d.key_max[k] = 0;
        }
    }
    for (int a = 0; a < na; a++) {
        d.aggs[a].op = ext->agg_ops[a];
        d.aggs[a].in = ins[a].col;
        if (d.aggs[a].op != OP_COUNT && !ins[a].col.data) return TD_ERR_PTR(TD_ERR_NYI);
    }
    int64_t rows_bound = js ? (jr->jd->n_left + jr->jd->n_right) : d.nrows;
    if (js) d.nrows = rows_bound;
    tdg_group_plan plan;
    st = tdg_group_plan_make(&d, 0, &plan);
    if (st) return TD_ERR_PTR(st);
    tdb_trace("group planned");
    void* ws = tdb_dev_alloc(&x->c, plan.ws_bytes);
    tdg_group_out out;
    memset(&out, 0, sizeof(out));
    /* the group count lands in mapped host memory: readable once the group-by
     * (which ends with a stream synchronization) returns, without a copy */
    void* dng = NULL;
    volatile int64_t* hng = tdb_host_scalar(&x->c, &dng);
    out.d_n_groups = hng ? dng : tdb_dev_alloc(&x->c, 8);
    if (!ws || !out.d_n_groups) return TD_ERR_PTR(TD_ERR_OOM);
    /* a small result is emitted straight into mapped host memory: the host
     * reads it once the group-by's synchronization returns, with no copy */
    void* hout[TDG_MAX_KEYS + TDG_MAX_AGGS];
    memset(hout, 0, sizeof(hout));
    size_t obytes = 0;
    for (int k = 0; k < nk; k++) obytes += 256 + (size_t)plan.max_groups * td_sym_elem_size(keys[k].type, keys[k].attrs);
    obytes += (size_t)na * (256 + (size_t)plan.max_groups * 8);
    const int mapped = !x->dev_only && obytes <= TDB_OUT_BYTES - x->c.out_used;
    for (int k = 0; k < nk; k++) {
        const size_t b = (size_t)plan.max_groups * td_sym_elem_size(keys[k].type, keys[k].attrs);
        if (mapped) hout[k] = tdb_host_out(&x->c, b ? b : 1, &out.keys[k]);
        if (!hout[k]) out.keys[k] = tdb_dev_alloc(&x->c, b);
        if (!out.keys[k]) return TD_ERR_PTR(TD_ERR_OOM);
    }
    for (int a = 0; a < na; a++) {
        const size_t b = (size_t)plan.max_groups * 8;
        if (mapped) hout[nk + a] = tdb_host_out(&x->c, b ? b : 1, &out.aggs[a]);
        if (!hout[nk + a]) out.aggs[a] = tdb_dev_alloc(&x->c, b);
        if (!out.aggs[a]) return TD_ERR_PTR(TD_ERR_OOM);
    }
    if ((st = tdb_check_cancel())) return TD_ERR_PTR(st);
    if (jr) {
        bentry_t* be = bc_acquire(x, jr, &d, &plan, keys);
        if (be) {
            tdg_join_desc jd = *jr->jd;
            jd.flags |= TDG_JOIN_PREBUILT;
            st = CALL(tdg_join_group_run(&jd, &be->jp, be->jws, pp, dsel, &d, &plan, ws, &out, x->c.stream));
            bc_release(be);
        }
        if (!be || st == TD_ERR_RANGE) {    /* no kept map, or this plan cannot use it */
            grun_t r = { jr, pp, dsel, &d, &plan, ws, &out, x->c.stream };
            st = CALL(run_tuned(x, &r));
        }
        tdb_note_methods(plan.method, jr->jp->method, 1);
    } else {
        grun_t r = { NULL, pp, dsel, &d, &plan, ws, &out, x->c.stream };
        st = CALL(run_tuned(x, &r));
        tdb_note_methods(plan.method, 0, pp != NULL);
    }
    if (st) return TD_ERR_PTR(st);
    tdb_trace("group kernels done");
    int64_t ng = 0;
    if (hng) { ng = *hng; x->c.d2h_bytes += 8; }          /* written over the link by the kernel */
    else if ((st = tdb_d2h(&x->c, &ng, out.d_n_groups, 8))) return TD_ERR_PTR(st);
    tdb_trace("group count read");
    /* rows the kernels wrote into mapped host memory crossed the link too */
    for (int k = 0; k < nk; k++)
        if (hout[k]) x->c.d2h_bytes += (uint64_t)ng * td_sym_elem_size(keys[k].type, keys[k].attrs);
    for (int a = 0; a < na; a++)
        if (hout[nk + a]) x->c.d2h_bytes += (uint64_t)ng * 8;

    /* every result column is copied with one stream synchronization */
    td_t* cols[TDG_MAX_KEYS + TDG_MAX_AGGS];
    td_t* wide[TDG_MAX_AGGS];
    int8_t otype[TDG_MAX_AGGS];
    memset(cols, 0, sizeof(cols));
    memset(wide, 0, sizeof(wide));
    td_t* err = NULL;
    for (int k = 0; k < nk && !err; k++) {
        cols[k] = hout[k] ? host_vec(hout[k], keys[k].type, keys[k].attrs, ng)
                          : fetch_vec_q(x, out.keys[k], keys[k].type, keys[k].attrs, ng, 2);
        if (TD_IS_ERR(cols[k])) { err = cols[k]; cols[k] = NULL; }
    }
    for (int a = 0; a < na && !err; a++) {
        uint16_t op = ext->agg_ops[a];
        int is_f = ins[a].col.data && ins[a].col.type == TD_F64;
        int8_t ot = op == OP_AVG ? TD_F64 : op == OP_COUNT ? TD_I64
                  : op == OP_SUM ? (is_f ? TD_F64 : TD_I64)
                  : (ins[a].type ? ins[a].type : TD_I64);
        otype[a] = ot;
        td_t* v;
        if (td_sym_elem_size(ot, ins[a].attrs) == 8 || op == OP_AVG || op == OP_COUNT || op == OP_SUM) {
            int8_t vt = (ot == TD_F64 || op == OP_AVG) ? TD_F64 : (td_sym_elem_size(ot, ins[a].attrs) == 8 ? ot : TD_I64);
            v = hout[nk + a] ? host_vec(hout[nk + a], vt, vt == TD_SYM ? ins[a].attrs : 0, ng)
                             : fetch_vec_q(x, out.aggs[a], vt, vt == TD_SYM ? ins[a].attrs : 0, ng, 2);
            if (!TD_IS_ERR(v)) cols[nk + a] = v;
        } else {
            /* MIN/MAX of a narrow integer column: int64 results, narrowed below */
            v = hout[nk + a] ? host_vec(hout[nk + a], TD_I64, 0, ng) : fetch_vec_q(x, out.aggs[a], TD_I64, 0, ng, 1);
            if (!TD_IS_ERR(v)) wide[a] = v;
        }
        if (TD_IS_ERR(v)) err = v;
    }
    if (!err && (st = tdb_ctx_sync(&x->c))) err = TD_ERR_PTR(st);
    for (int a = 0; a < na && !err; a++) {
        if (!wide[a]) continue;
        const int8_t ot = otype[a];
        td_t* col = vec_like(ot, ins[a].attrs, ng);
        if (TD_IS_ERR(col)) { err = col; break; }
        const int64_t* w = (const int64_t*)td_data(wide[a]);
        for (int64_t i = 0; i < ng; i++) {
            if (ot == TD_SYM) td_write_sym(td_data(col), i, (uint64_t)w[i], TD_SYM, ins[a].attrs);
            else switch (td_elem_size(ot)) {
                case 4: ((int32_t*)td_data(col))[i] = (int32_t)w[i]; break;
                case 2: ((int16_t*)td_data(col))[i] = (int16_t)w[i]; break;
                default: ((uint8_t*)td_data(col))[i] = (uint8_t)w[i]; break;
            }
        }
        cols[nk + a] = col;
    }
    td_t* res = err ? NULL : td_table_new(nk + na);
    if (!err && (!res || TD_IS_ERR(res))) { err = res ? res : TD_ERR_PTR(TD_ERR_OOM); res = NULL; }
    for (int j = 0; j < nk + na && !err; j++) {
        int64_t nm = j < nk ? (keys[j].name >= 0 ? keys[j].name : (int64_t)j)
                            : agg_name(ext->agg_ops[j - nk], ins[j - nk].name, j - nk);
        td_t* r2 = td_table_add_col(res, nm, cols[j]);
        if (TD_IS_ERR(r2)) { err = r2; break; }
        res = r2;
    }
    if (err) tdb_ctx_sync(&x->c);          /* no queued copy may still target a vector freed here */
    for (int j = 0; j < nk + na; j++) if (cols[j]) td_release(cols[j]);
    for (int a = 0; a < na; a++) if (wide[a]) td_release(wide[a]);
    if (err) {
        if (res) td_release(res);
        return err;
    }
    tdb_trace("group result copied");
    return res;
}

/* ---- join ---------------------------------------------------------------------------------- */
typedef struct {
    tdg_join_desc d;
    tdg_join_plan p;
    void* ws;
    td_t* left;      /* host tables (retained by the caller's val_t) */
    td_t* right;
    td_t* rkey;      /* the build side's (single) key column */
} jbuilt_t;

/* Right side with a pending filter: compact it on the device first. */
static td_t* dense_side(ex_t* x, val_t* v) {
    if (!v->lazy) { td_retain(v->obj); return v->obj; }
    return materialize(x, v);
}

/* Plan the join and allocate its scratch; build the table unless the caller
 * hands it to tdg_join_group_run, which builds it itself. */
static int prepare_join(ex_t* x, td_op_ext_t* ext, val_t* lv, td_t* right, jbuilt_t* jb, int build) {
    memset(jb, 0, sizeof(*jb));
    td_t* left = lv->obj;
    if (!left || left->type != TD_TABLE || !right || right->type != TD_TABLE) return TD_ERR_TYPE;
    int nk = ext->join.n_join_keys;
    if (nk < 1 || nk > TDG_MAX_KEYS) return TD_ERR_NYI;
    jb->left = left; jb->right = right;
    tdg_join_desc* d = &jb->d;
    d->n_left = td_table_nrows(left);
    d->n_right = td_table_nrows(right);
    if (d->n_left > INT32_MAX || d->n_right > INT32_MAX) return TD_ERR_NYI;
    d->n_keys = nk;
    d->join_type = ext->join.join_type;
    for (int k = 0; k < nk; k++) {
        td_op_ext_t* lk = tdb_find_ext(x->g, ext->join.left_keys[k]->id);
        td_op_ext_t* rk = tdb_find_ext(x->g, ext->join.right_keys[k]->id);
        td_t* lc = (lk && lk->base.opcode == OP_SCAN) ? td_table_get_col(left, lk->sym) : NULL;
        td_t* rc = NULL;
        if (rk && rk->base.opcode == OP_SCAN) rc = td_table_get_col(right, rk->sym);
        else if (rk && rk->base.opcode == OP_CONST && rk->literal && td_is_vec(rk->literal)) rc = rk->literal;
        if (!lc || !rc) return TD_ERR_SCHEMA;
        tdb_devcol dl, dr;
        int st = tdb_col_device(&x->c, lc, 0, &dl);
        if (!st) st = tdb_col_device(&x->c, rc, nk == 1, &dr);
        if (st) return st;
        d->lkeys[k] = (tdg_col){ dl.dptr, dl.type, dl.attrs, 0, {0} };
        d->rkeys[k] = (tdg_col){ dr.dptr, dr.type, dr.attrs, 1, {0} };
        if (nk == 1) jb->rkey = rc;
        if (nk == 1 && dr.has_stats && dr.len > 0) {
            d->have_range = 1;
            d->rkey_min = dr.kmin;
            d->rkey_max = dr.kmax;
        }
    }
    int st = tdg_join_plan_make(d, &jb->p);
    if (st) return st;
    jb->ws = tdb_dev_alloc(&x->c, jb->p.ws_bytes);
    if (!jb->ws) return TD_ERR_OOM;
    if ((st = tdb_check_cancel())) return st;
    return build ? CALL(tdg_join_build(d, &jb->p, jb->ws, x->c.stream)) : TD_OK;
}

static int is_right_key(ex_t* x, td_op_ext_t* ext, int64_t name) {
    for (int k = 0; k < ext->join.n_join_keys; k++) {
        td_op_ext_t* rk = tdb_find_ext(x->g, ext->join.right_keys[k]->id);
        if (rk && rk->base.opcode == OP_SCAN && rk->sym == name) return 1;
    }
    return 0;
}

static td_t* join_materialize(ex_t* x, td_op_ext_t* ext, val_t* lv, jbuilt_t* jb) {
    const tdg_expr* lp = lv->has_pred ? &lv->pred : NULL;
    int64_t* dcount = tdb_dev_alloc(&x->c, 8);
    if (!dcount) return TD_ERR_PTR(TD_ERR_OOM);
    int st = CALL(tdg_join_count(&jb->d, &jb->p, jb->ws, lp, lv->dsel, dcount, x->c.stream));
    if (st) return TD_ERR_PTR(st);
    int64_t m = 0;
    st = tdb_d2h(&x->c, &m, dcount, 8);
    if (st) return TD_ERR_PTR(st);
    tdg_col lsrc[MAX_TCOLS], rsrc[MAX_TCOLS];
    void *ldst[MAX_TCOLS], *rdst[MAX_TCOLS];
    int64_t rname[MAX_TCOLS];
    int nl = table_dev_cols(x, jb->left, lsrc, 16);
    if (nl < 0) return TD_ERR_PTR(-nl);
    int nr = 0;
    for (int64_t j = 0; j < td_table_ncols(jb->right); j++) {
        int64_t nm = td_table_col_name(jb->right, j);
        if (is_right_key(x, ext, nm)) continue;
        if (nr >= 16) return TD_ERR_PTR(TD_ERR_NYI);
        tdb_devcol dd;
        st = tdb_col_device(&x->c, td_table_get_col_idx(jb->right, j), 0, &dd);
        if (st) return TD_ERR_PTR(st);
        rsrc[nr] = (tdg_col){ dd.dptr, dd.type, dd.attrs, 1, {0} };
        rname[nr++] = nm;
    }
    size_t cnt = (size_t)(m ? m : 1);
    for (int j = 0; j < nl; j++)
        if (!(ldst[j] = tdb_dev_alloc(&x->c, cnt * td_sym_elem_size(lsrc[j].type, lsrc[j].attrs))))
            return TD_ERR_PTR(TD_ERR_OOM);
    for (int j = 0; j < nr; j++)
        if (!(rdst[j] = tdb_dev_alloc(&x->c, cnt * td_sym_elem_size(rsrc[j].type, rsrc[j].attrs))))
            return TD_ERR_PTR(TD_ERR_OOM);
    st = CALL(tdg_join_emit(&jb->d, &jb->p, jb->ws, lp, lv->dsel, nl, lsrc, ldst, nr, rsrc, rdst, x->c.stream));
    if (st) return TD_ERR_PTR(st);
    tdb_note_methods(0, jb->p.method, 0);
    td_t* res = td_table_new(nl + nr);
    if (!res || TD_IS_ERR(res)) return res;
    for (int j = 0; j < nl + nr; j++) {
        const tdg_col* sc = j < nl ? &lsrc[j] : &rsrc[j - nl];
        void* dp = j < nl ? ldst[j] : rdst[j - nl];
        td_t* col = fetch_vec(x, dp, sc->type, sc->attrs, m);
        if (TD_IS_ERR(col)) { td_release(res); return col; }
        int64_t nm = j < nl ? td_table_col_name(jb->left, j) : rname[j - nl];
        res = td_table_add_col(res, nm, col);
        td_release(col);
        if (TD_IS_ERR(res)) return res;
    }
    return res;
}

/* ---- scalar reductions ------------------------------------------------------------------------ */
static td_t* reduce(ex_t* x, uint16_t opc, val_t* v) {
    td_t* o = v->obj;
    if (td_is_atom(o)) {
        if (opc == OP_COUNT) return td_i64(1);
        td_retain(o);
        return o;
    }
    if (o->type == TD_TABLE) {
        /* COUNT of a table counts its (selected) rows */
        if (opc != OP_COUNT) return TD_ERR_PTR(TD_ERR_TYPE);
        if (!v->lazy) return td_i64(td_table_nrows(o));
        int64_t n = td_table_nrows(o);
        void* ws = tdb_dev_alloc(&x->c, tdg_select_ws_bytes(n));
        int64_t* dc = tdb_dev_alloc(&x->c, 8);
        if (!ws || !dc) return TD_ERR_PTR(TD_ERR_OOM);
        int st = CALL(tdg_select_count(n, v->has_pred ? &v->pred : NULL, v->dsel, ws, dc, x->c.stream));
        int64_t m = 0;
        if (!st) st = tdb_d2h(&x->c, &m, dc, 8);
        return st ? TD_ERR_PTR(st) : td_i64(m);
    }
    if (!v->lazy && opc == OP_COUNT) return td_i64(o->len);
    if (o->type == TD_BOOL || o->type == TD_SEL || o->type == TD_LIST) {
        if (opc == OP_COUNT) return td_i64(o->len);
    }
    /* one-slot group-by over the vector's (selected) rows */
    tdb_devcol dc;
    int st = tdb_col_device(&x->c, o, 0, &dc);
    if (st) return TD_ERR_PTR(st);
    tdg_group_desc d;
    memset(&d, 0, sizeof(d));
    d.nrows = o->len;
    d.n_aggs = 2;
    d.aggs[0].op = opc == OP_AVG ? OP_SUM : opc;
    d.aggs[0].in = (tdg_col){ dc.dptr, dc.type, dc.attrs, 0, {0} };
    d.aggs[1].op = OP_COUNT;
    d.have_range = 1;
    tdg_group_plan plan;
    st = tdg_group_plan_make(&d, 1, &plan);
    if (st) return TD_ERR_PTR(st);
    void* ws = tdb_dev_alloc(&x->c, plan.ws_bytes);
    tdg_group_out out;
    memset(&out, 0, sizeof(out));
    /* the count and both aggregates land in mapped host memory when it has room */
    const size_t ab = 8 * (size_t)plan.max_groups;
    int64_t* h[3] = {0, 0, 0};
    void* dng = NULL;
    h[0] = tdb_host_out(&x->c, 8, &dng);
    out.d_n_groups = dng;
    if (h[0]) h[1] = tdb_host_out(&x->c, ab, &out.aggs[0]);
    if (h[1]) h[2] = tdb_host_out(&x->c, ab, &out.aggs[1]);
    if (!h[2]) {
        h[0] = h[1] = NULL;
        out.d_n_groups = tdb_dev_alloc(&x->c, 8);
        out.aggs[0] = tdb_dev_alloc(&x->c, ab);
        out.aggs[1] = tdb_dev_alloc(&x->c, ab);
    }
    if (!ws || !out.d_n_groups || !out.aggs[0] || !out.aggs[1]) return TD_ERR_PTR(TD_ERR_OOM);
    st = CALL(tdg_group_run(&d, v->has_pred ? &v->pred : NULL, v->dsel, &plan, ws, &out, x->c.stream));
    if (st) return TD_ERR_PTR(st);
    int64_t ng = 0;
    uint64_t val = 0;
    int64_t cnt = 0;
    if (h[2]) {   /* tdg_group_run synchronized its stream */
        ng = h[0][0];
        if (ng > 0) { memcpy(&val, h[1], 8); cnt = h[2][0]; }
        x->c.d2h_bytes += 8 + 16 * (uint64_t)ng;        /* the kernel wrote them over the link */
    } else {
        st = tdb_d2h(&x->c, &ng, out.d_n_groups, 8);
        if (!st && ng > 0) st = tdb_d2h(&x->c, &val, out.aggs[0], 8);
        if (!st && ng > 0) st = tdb_d2h(&x->c, &cnt, out.aggs[1], 8);
    }
    if (st) return TD_ERR_PTR(st);
    int isf = dc.type == TD_F64;
    double f; int64_t i;
    memcpy(&f, &val, 8);
    i = (int64_t)val;
    switch (opc) {
        case OP_COUNT: return td_i64(cnt);
        case OP_SUM:   return isf ? td_f64(ng ? f : 0.0) : td_i64(ng ? i : 0);
        case OP_MIN: case OP_MAX:
            return isf ? td_f64(cnt ? f : 0.0) : td_i64(cnt ? i : 0);
        case OP_AVG:
            if (!cnt) return td_f64(0.0);
            return td_f64(isf ? f / (double)cnt : (double)i / (double)cnt);
    }
    return TD_ERR_PTR(TD_ERR_NYI);
}

/* ---- the walk -------------------------------------------------------------------------------------- */
static int is_elementwise(uint16_t o) {
    return (o >= OP_NEG && o <= OP_CAST && o != OP_SQRT && o != OP_LOG && o != OP_EXP &&
            o != OP_CEIL && o != OP_FLOOR && o != OP_ISNULL) ||
           (o >= OP_ADD && o <= OP_MAX2);
}

static td_op_ext_t* single_join(td_graph_t* g) {
    td_op_ext_t* found = NULL;
    for (uint32_t i = 0; i < g->ext_count; i++) {
        td_op_ext_t* e = g->ext_nodes[i];
        if (e && g->nodes[e->base.id].opcode == OP_JOIN) {
            if (found) return NULL;
            found = e;
        }
    }
    return found;
}

static td_t* exec_group_node(ex_t* x, td_op_t* op) {
    td_op_ext_t* ext = tdb_find_ext(x->g, op->id);
    if (!ext) return TD_ERR_PTR(TD_ERR_NYI);
    td_graph_t* g = x->g;
    if (!g->table) {
        td_op_ext_t* jext = single_join(g);
        if (!jext) return TD_ERR_PTR(TD_ERR_SCHEMA);
        /* fused filter -> join -> group: the join is probed, never materialized */
        val_t lv = vnone(), rv = vnone();
        td_t* r = exec_value(x, jext->base.inputs[0], &lv);
        if (TD_IS_ERR(r)) return r;
        r = exec_value(x, jext->base.inputs[1], &rv);
        if (TD_IS_ERR(r)) { vfree(&lv); return r; }
        td_t* right = dense_side(x, &rv);
        td_t* res;
        if (TD_IS_ERR(right)) {
            res = right;
        } else {
            jbuilt_t jb;
            tdb_trace("join lowering");
            int st = prepare_join(x, jext, &lv, right, &jb, 0);
            tdb_trace("join prepared");
            if (st) {
                res = TD_ERR_PTR(st);
            } else {
                jsrc_t js = { lv.obj, right, jext };
                jrun_t jr = { &jb.d, &jb.p, jb.ws, jb.rkey };
                res = run_group(x, ext, NULL, lv.has_pred ? &lv.pred : NULL, lv.dsel, &js, &jr);
            }
            td_release(right);
        }
        vfree(&lv);
        vfree(&rv);
        return res;
    }
    /* the caller's TD_SEL (if any) restricts the rows */
    const uint64_t* dsel = NULL;
    if (g->selection && g->selection->type == TD_SEL && g->selection->len == td_table_nrows(g->table)) {
        size_t bytes = (size_t)((g->selection->len + 63) / 64) * 8;
        void* d = tdb_dev_alloc(&x->c, bytes ? bytes : 8);
        if (!d) return TD_ERR_PTR(TD_ERR_OOM);
        int st = tdb_h2d(&x->c, d, td_sel_bits(g->selection), bytes);
        if (st) return TD_ERR_PTR(st);
        dsel = d;
    }
    return run_group(x, ext, g->table, NULL, dsel, NULL, NULL);
}

/* Evaluate op; sets *out (retained value) and returns its obj or an error. */
/* ---- sort ------------------------------------------------------------------------------- */

typedef struct { const char* p; uint32_t len; uint32_t id; } symstr_t;

static int symstr_cmp(const void* a, const void* b) {
    const symstr_t* x = a;
    const symstr_t* y = b;
    const uint32_t ml = x->len < y->len ? x->len : y->len;
    int c = ml ? memcmp(x->p, y->p, ml) : 0;
    if (!c) c = (x->len > y->len) - (x->len < y->len);
    if (!c) c = (x->id > y->id) - (x->id < y->id);
    return c;
}

static uint32_t sym_id_at(td_t* col, int64_t i) {
    const void* d = td_data(col);
    switch (td_sym_elem_size(col->type, col->attrs)) {
        case 1: return ((const uint8_t*)d)[i];
        case 2: return ((const uint16_t*)d)[i];
        case 4: return ((const uint32_t*)d)[i];
        default: return (uint32_t)((const int64_t*)d)[i];
    }
}

/* Rank of every intern id up to the column's largest, by its string: the
 * bytes of the shorter length, then the length (build_enum_rank,
 * exec.c:2876-2975); returned as a device array. */
static const uint32_t* sym_rank_dev(ex_t* x, td_t* col) {
    uint32_t max_id = 0;
    for (int64_t i = 0; i < col->len; i++) {
        const uint32_t v = sym_id_at(col, i);
        if (v > max_id) max_id = v;
    }
    if (max_id >= UINT32_MAX - 1) return NULL;
    const uint32_t n_ids = max_id + 1;
    symstr_t* s = malloc((size_t)n_ids * sizeof(symstr_t));
    uint32_t* rank = malloc((size_t)n_ids * sizeof(uint32_t));
    uint32_t* d = rank ? tdb_dev_alloc(&x->c, (size_t)n_ids * sizeof(uint32_t)) : NULL;
    if (!s || !rank || !d) { free(s); free(rank); return NULL; }
    for (uint32_t i = 0; i < n_ids; i++) {
        td_t* str = td_sym_str((int64_t)i);
        s[i].p = str ? td_str_ptr(str) : NULL;
        s[i].len = str ? (uint32_t)td_str_len(str) : 0;
        s[i].id = i;
    }
    qsort(s, n_ids, sizeof(symstr_t), symstr_cmp);
    for (uint32_t i = 0; i < n_ids; i++) rank[s[i].id] = i;
    int st = tdb_h2d(&x->c, d, rank, (size_t)n_ids * sizeof(uint32_t));
    free(s);
    free(rank);
    return st ? NULL : d;
}

/* Sort a table by the node's key columns on the device and keep the first
 * `limit` rows (all when limit < 0): exec_sort (exec.c:3370-3862), with
 * HEAD(SORT) as in exec.c:11895-11917.  Keys are column scans of the sorted
 * table; the table's columns that came from an earlier step of this query
 * are still on the device, so only host-born columns are uploaded. */
static td_t* exec_sort_node(ex_t* x, td_op_t* sop, int64_t limit) {
    td_graph_t* g = x->g;
    td_op_ext_t* ext = tdb_find_ext(g, sop->id);
    if (!ext || ext->sort.n_cols > TDG_MAX_SORT_KEYS) return TD_ERR_PTR(TD_ERR_NYI);
    val_t in;
    const int dev_only = x->dev_only;
    x->dev_only = sop->inputs[0] && sop->inputs[0]->opcode == OP_GROUP;   /* read only through its device copy */
    td_t* r = exec_value(x, sop->inputs[0], &in);
    x->dev_only = dev_only;
    if (TD_IS_ERR(r)) return r;
    td_t* tbl = materialize(x, &in);
    vfree(&in);
    if (TD_IS_ERR(tbl)) return tbl;
    if (tbl->type != TD_TABLE) { td_release(tbl); return TD_ERR_PTR(TD_ERR_TYPE); }
    const int64_t n = td_table_nrows(tbl);
    const int64_t n_out = limit >= 0 && limit < n ? limit : n;
    const int nk = ext->sort.n_cols;
    tdg_sort_key keys[TDG_MAX_SORT_KEYS];
    td_t* kexpr[TDG_MAX_SORT_KEYS];
    memset(kexpr, 0, sizeof(kexpr));
    td_t* res = NULL;
    int st = 0;
    for (int k = 0; k < nk && !st; k++) {
        td_op_ext_t* ke = tdb_find_ext(g, ext->sort.columns[k]->id);
        td_t* col;
        if (ke && ke->base.opcode == OP_SCAN) {
            col = td_table_get_col(tbl, ke->sym);
        } else {
            /* a key expression is evaluated over the sort's input table, as
             * exec_sort does (exec.c:3393-3401) */
            td_t* saved = g->table;
            g->table = tbl;
            val_t kv;
            td_t* r = exec_value(x, ext->sort.columns[k], &kv);
            g->table = saved;
            if (TD_IS_ERR(r)) { st = TD_ERR_CODE(r); break; }
            col = materialize(x, &kv);
            vfree(&kv);
            if (TD_IS_ERR(col)) { st = TD_ERR_CODE(col); break; }
            kexpr[k] = col;
            if (col->type <= 0 || col->type == TD_TABLE || col->type >= TD_PARTED_BASE) { st = TD_ERR_NYI; break; }
            if (col->len != n) { st = TD_ERR_LENGTH; break; }
        }
        if (!col) { st = TD_ERR_SCHEMA; break; }
        tdb_devcol d;
        st = tdb_col_device(&x->c, col, 0, &d);
        if (st) break;
        memset(&keys[k], 0, sizeof(keys[k]));
        keys[k].col.data = d.dptr;
        keys[k].col.type = d.type;
        keys[k].col.attrs = d.attrs;
        keys[k].desc = ext->sort.desc ? ext->sort.desc[k] : 0;
        keys[k].nulls_first = ext->sort.nulls_first ? ext->sort.nulls_first[k] : keys[k].desc;
        if (d.type == TD_SYM && !(keys[k].sym_rank = sym_rank_dev(x, col))) st = TD_ERR_OOM;
    }
    void* ws = st ? NULL : tdb_dev_alloc(&x->c, tdg_sort_ws_bytes(n));
    int64_t* perm = st ? NULL : tdb_dev_alloc(&x->c, (size_t)(n ? n : 1) * 8);
    if (!st && (!ws || !perm)) st = TD_ERR_OOM;
    if (!st) st = CALL(tdg_sort_perm(keys, nk, n, ws, perm, x->c.stream));
    tdg_col cols[MAX_TCOLS];
    int nc = 0;
    if (!st) {
        nc = table_dev_cols(x, tbl, cols, MAX_TCOLS);
        if (nc < 0) st = -nc;
    }
    if (!st) {
        res = td_table_new(nc);
        if (!res || TD_IS_ERR(res)) { st = res ? TD_ERR_CODE(res) : TD_ERR_OOM; res = NULL; }
    }
    for (int j = 0; j < nc && !st; j++) {
        void* out = tdb_dev_alloc(&x->c, (size_t)(n_out ? n_out : 1) * td_sym_elem_size(cols[j].type, cols[j].attrs));
        if (!out) { st = TD_ERR_OOM; break; }
        st = CALL(tdg_gather(&cols[j], perm, n_out, out, x->c.stream));
        if (st) break;
        td_t* col = fetch_vec_q(x, out, cols[j].type, cols[j].attrs, n_out, 1);
        if (TD_IS_ERR(col)) { st = TD_ERR_CODE(col); break; }
        td_t* t2 = td_table_add_col(res, td_table_col_name(tbl, j), col);
        td_release(col);
        if (TD_IS_ERR(t2)) { st = TD_ERR_CODE(t2); break; }
        res = t2;
    }
    int st2 = tdb_ctx_sync(&x->c);                 /* the queued copies land before anything is returned or freed */
    if (!st) st = st2;
    for (int k = 0; k < nk; k++) if (kexpr[k]) td_release(kexpr[k]);
    td_release(tbl);
    if (st) {
        if (res) td_release(res);
        return TD_ERR_PTR(st);
    }
    return res;
}

/* The first m elements of a vector, as a new vector with inline data. */
static td_t* vec_prefix(td_t* v, int64_t m) {
    td_t* c = vec_like(v->type, v->attrs, m);
    if (!c || TD_IS_ERR(c)) return c ? c : TD_ERR_PTR(TD_ERR_OOM);
    if (m) memcpy(td_data(c), td_data(v), (size_t)m * td_sym_elem_size(v->type, v->attrs));
    return c;
}

/* HEAD of anything but a sort: the first n rows, copied. */
static td_t* head_rows(td_t* v, int64_t limit) {
    if (v->type != TD_TABLE) return vec_prefix(v, limit < v->len ? limit : v->len);
    const int64_t n = td_table_nrows(v), m = limit < n ? limit : n;
    td_t* out = td_table_new(td_table_ncols(v));
    for (int64_t j = 0; j < td_table_ncols(v) && out && !TD_IS_ERR(out); j++) {
        td_t* s = vec_prefix(td_table_get_col_idx(v, j), m);
        if (TD_IS_ERR(s)) { td_release(out); return s; }
        out = td_table_add_col(out, td_table_col_name(v, j), s);
        td_release(s);
    }
    return out ? out : TD_ERR_PTR(TD_ERR_OOM);
}

static td_t* exec_value(ex_t* x, td_op_t* op, val_t* out) {
    *out = vnone();
    if (!op) return TD_ERR_PTR(TD_ERR_NYI);
    int st = tdb_check_cancel();
    if (st) return TD_ERR_PTR(st);
    td_graph_t* g = x->g;
    switch (op->opcode) {
        case OP_SCAN: {
            td_op_ext_t* ext = tdb_find_ext(g, op->id);
            if (!ext) return TD_ERR_PTR(TD_ERR_NYI);
            td_t* t = scan_table_of(x, ext, g->table);
            td_t* col = t ? td_table_get_col(t, ext->sym) : NULL;
            if (!col) return TD_ERR_PTR(TD_ERR_SCHEMA);
            td_retain(col);
            out->obj = col;
            return col;
        }
        case OP_CONST: {
            td_op_ext_t* ext = tdb_find_ext(g, op->id);
            if (!ext || !ext->literal) return TD_ERR_PTR(TD_ERR_NYI);
            td_retain(ext->literal);
            out->obj = ext->literal;
            return out->obj;
        }
        case OP_ALIAS: case OP_MATERIALIZE:
            return exec_value(x, op->inputs[0], out);
        case OP_FILTER: {
            td_op_t* child = op->inputs[0];
            if (child && child->opcode == OP_GROUP) {
                /* HAVING: the predicate reads the group-by result */
                td_t* grp = exec_group_node(x, child);
                if (TD_IS_ERR(grp)) return grp;
                tdg_expr p;
                st = compile_expr(x, grp, op->inputs[1], &p);
                if (st) { td_release(grp); return TD_ERR_PTR(st); }
                out->obj = grp;
                out->lazy = 1;
                out->has_pred = 1;
                out->pred = p;
                return grp;
            }
            val_t in;
            td_t* r = exec_value(x, child, &in);
            if (TD_IS_ERR(r)) return r;
            td_t* rows_tbl = in.obj->type == TD_TABLE ? in.obj : g->table;
            if (!rows_tbl) { vfree(&in); return TD_ERR_PTR(TD_ERR_SCHEMA); }
            if (in.obj->type != TD_TABLE && in.obj->len != td_table_nrows(rows_tbl)) {
                vfree(&in);
                return TD_ERR_PTR(TD_ERR_LENGTH);
            }
            tdg_expr p;
            st = compile_expr(x, rows_tbl, op->inputs[1], &p);
            if (!st) {
                if (!in.has_pred) { memset(&in.pred, 0, sizeof(in.pred)); }
                st = expr_and(&in.pred, &p);
            }
            if (st) { vfree(&in); return TD_ERR_PTR(st); }
            in.lazy = 1;
            in.has_pred = 1;
            *out = in;
            return out->obj;
        }
        case OP_GROUP: {
            td_t* r = exec_group_node(x, op);
            if (TD_IS_ERR(r)) return r;
            out->obj = r;
            return r;
        }
        case OP_JOIN: {
            val_t lv, rv;
            td_t* r = exec_value(x, op->inputs[0], &lv);
            if (TD_IS_ERR(r)) return r;
            r = exec_value(x, op->inputs[1], &rv);
            if (TD_IS_ERR(r)) { vfree(&lv); return r; }
            td_op_ext_t* ext = tdb_find_ext(g, op->id);
            td_t* right = ext ? dense_side(x, &rv) : TD_ERR_PTR(TD_ERR_NYI);
            td_t* res = right;
            if (!TD_IS_ERR(right)) {
                jbuilt_t jb;
                st = prepare_join(x, ext, &lv, right, &jb, 1);
                res = st ? TD_ERR_PTR(st) : join_materialize(x, ext, &lv, &jb);
                td_release(right);
            }
            vfree(&lv);
            vfree(&rv);
            if (TD_IS_ERR(res)) return res;
            out->obj = res;
            return res;
        }
        case OP_SORT: {
            td_t* res = exec_sort_node(x, op, -1);
            if (TD_IS_ERR(res)) return res;
            out->obj = res;
            return res;
        }
        case OP_HEAD: {
            td_op_ext_t* he = tdb_find_ext(g, op->id);
            int64_t limit = he ? he->sym : 10;
            if (limit < 0) limit = 0;
            td_op_t* child = op->inputs[0];
            td_t* res;
            if (child && child->opcode == OP_SORT) {
                res = exec_sort_node(x, child, limit);
            } else {
                val_t in;
                td_t* r = exec_value(x, child, &in);
                if (TD_IS_ERR(r)) return r;
                td_t* v = materialize(x, &in);
                vfree(&in);
                if (TD_IS_ERR(v)) return v;
                res = head_rows(v, limit);
                td_release(v);
            }
            if (TD_IS_ERR(res)) return res;
            out->obj = res;
            return res;
        }
        case OP_COUNT: case OP_SUM: case OP_MIN: case OP_MAX: case OP_AVG: {
            val_t in;
            td_t* r = exec_value(x, op->inputs[0], &in);
            if (TD_IS_ERR(r)) return r;
            td_t* res = reduce(x, op->opcode, &in);
            vfree(&in);
            if (TD_IS_ERR(res)) return res;
            out->obj = res;
            return res;
        }
        default:
            break;
    }
    if (is_elementwise(op->opcode)) {
        if (!g->table) return TD_ERR_PTR(TD_ERR_SCHEMA);
        tdg_expr e;
        st = compile_expr(x, g->table, op, &e);
        if (st) return TD_ERR_PTR(st);
        int64_t n = td_table_nrows(g->table);
        int kind = e.ins[e.out].kind;
        int is_bool = op->out_type == TD_BOOL || (op->opcode >= OP_EQ && op->opcode <= OP_OR) || op->opcode == OP_NOT;
        int out_kind = is_bool ? 2 : kind;
        void* d = tdb_dev_alloc(&x->c, (size_t)(n ? n : 1) * 8);
        if (!d) return TD_ERR_PTR(TD_ERR_OOM);
        st = CALL(tdg_eval(&e, n, d, out_kind, x->c.stream));
        if (st) return TD_ERR_PTR(st);
        td_t* v = fetch_vec(x, d, is_bool ? TD_BOOL : (kind ? TD_F64 : TD_I64), 0, n);
        if (TD_IS_ERR(v)) return v;
        out->obj = v;
        return v;
    }
    return TD_ERR_PTR(TD_ERR_NYI);
}

td_t* tdb_exec(td_graph_t* g, td_op_t* root, int dev_only) {
    ex_t x;
    memset(&x, 0, sizeof(x));
    x.g = g;
    x.dev_only = dev_only;
    tdb_reset_methods();
    int st = tdb_ctx_begin(&x.c);
    if (st) return TD_ERR_PTR(st);
    val_t v;
    td_t* r = exec_value(&x, root, &v);
    td_t* res;
    if (TD_IS_ERR(r)) {
        res = r;
    } else {
        res = materialize(&x, &v);
        vfree(&v);
    }
    tdb_ctx_end(&x.c);
    if (g->selection) { td_release(g->selection); g->selection = NULL; }
    return res;
}

td_t* td_execute(td_graph_t* g, td_op_t* root) {
    if (!g || !root) return TD_ERR_PTR(TD_ERR_NYI);
    tdb_cancel_reset();
    tdb_trace_begin();
    td_t* r = tdb_exec(g, root, 0);
    tdb_trace("td_execute returns");
    return r;
}

td_t* td_execute_device(td_graph_t* g, td_op_t* root) {
    if (!g || !root) return TD_ERR_PTR(TD_ERR_NYI);
    if (root->opcode != OP_GROUP) return TD_ERR_PTR(TD_ERR_NYI);
    tdb_cancel_reset();
    tdb_trace_begin();
    td_t* r = tdb_exec(g, root, 1);
    tdb_trace("td_execute_device returns");
    return r;
}
