/*
 * DAG construction.  Node layout and builder semantics are the ones callers
 * of Teide's td.h rely on (src/ops/graph.c:182-749, 942-1063):
 *   - g->nodes is a growable array of 32-byte td_op_t; builders return
 *     &g->nodes[id], and every input pointer points into that array, so when
 *     the array moves all stored pointers are rebased;
 *   - nodes with a payload (scan, const, group, join, alias) also own a
 *     td_op_ext_t kept in g->ext_nodes; its base is copied into g->nodes[id]
 *     once filled in, and executors find it by id;
 *   - output types: comparisons/AND/OR/NOT give BOOL, arithmetic promotes
 *     BOOL < U8 < I16 < I32 < I64 < F64 (SYM/TIMESTAMP count as I64,
 *     DATE/TIME as I32), DIV gives F64, SUM keeps F64 else I64, COUNT I64,
 *     AVG F64, MIN/MAX the input type;
 *   - the graph retains its bound table, registered tables and every const
 *     literal, and releases them in td_graph_free.
 */
#include "internal.h"
#include <stdlib.h>
#include <string.h>

#define NODES_INIT 4096

static void rebase(td_op_t** p, uintptr_t old_base, uintptr_t new_base, uint32_t n) {
    if (!*p) return;
    uintptr_t a = (uintptr_t)*p;
    if (a >= old_base && a < old_base + (uintptr_t)n * sizeof(td_op_t))
        *p = (td_op_t*)(new_base + (a - old_base));
}

static void rebase_all(td_graph_t* g, uintptr_t ob) {
    uintptr_t nb = (uintptr_t)g->nodes;
    uint32_t n = g->node_count;
    if (ob == nb) return;
    for (uint32_t i = 0; i < n; i++) {
        rebase(&g->nodes[i].inputs[0], ob, nb, n);
        rebase(&g->nodes[i].inputs[1], ob, nb, n);
    }
    for (uint32_t i = 0; i < g->ext_count; i++) {
        td_op_ext_t* e = g->ext_nodes[i];
        if (!e) continue;
        rebase(&e->base.inputs[0], ob, nb, n);
        rebase(&e->base.inputs[1], ob, nb, n);
        switch (e->base.opcode) {
            case OP_GROUP:
                for (int k = 0; k < e->n_keys; k++) rebase(&e->keys[k], ob, nb, n);
                for (int a = 0; a < e->n_aggs; a++) rebase(&e->agg_ins[a], ob, nb, n);
                break;
            case OP_JOIN:
                for (int k = 0; k < e->join.n_join_keys; k++) {
                    rebase(&e->join.left_keys[k], ob, nb, n);
                    rebase(&e->join.right_keys[k], ob, nb, n);
                }
                break;
            case OP_SORT: case OP_SELECT:
                for (int k = 0; k < e->sort.n_cols; k++) rebase(&e->sort.columns[k], ob, nb, n);
                break;
            default: break;
        }
    }
}

static int grow_nodes(td_graph_t* g) {
    if (g->node_count < g->node_cap) return 1;
    if (g->node_cap > UINT32_MAX / 2) return 0;
    uintptr_t ob = (uintptr_t)g->nodes;
    td_op_t* nn = realloc(g->nodes, (size_t)g->node_cap * 2 * sizeof(td_op_t));
    if (!nn) return 0;
    g->nodes = nn;
    g->node_cap *= 2;
    rebase_all(g, ob);
    return 1;
}

static td_op_t* new_node(td_graph_t* g) {
    if (!grow_nodes(g)) return NULL;
    td_op_t* n = &g->nodes[g->node_count];
    memset(n, 0, sizeof(*n));
    n->id = g->node_count++;
    return n;
}

/* ext node with `extra` trailing bytes; reserves its id in g->nodes */
static td_op_ext_t* new_ext(td_graph_t* g, size_t extra) {
    td_op_ext_t* e = calloc(1, sizeof(td_op_ext_t) + extra);
    if (!e) return NULL;
    if (g->ext_count == g->ext_cap) {
        uint32_t nc = g->ext_cap ? g->ext_cap * 2 : 16;
        td_op_ext_t** ne = realloc(g->ext_nodes, nc * sizeof(*ne));
        if (!ne) { free(e); return NULL; }
        g->ext_nodes = ne;
        g->ext_cap = nc;
    }
    td_op_t* slot = new_node(g);
    if (!slot) { free(e); return NULL; }
    e->base.id = slot->id;
    g->ext_nodes[g->ext_count++] = e;
    return e;
}

static td_op_t* publish(td_graph_t* g, td_op_ext_t* e) {
    g->nodes[e->base.id] = e->base;
    return &g->nodes[e->base.id];
}

td_op_ext_t* tdb_find_ext(td_graph_t* g, uint32_t id) {
    for (uint32_t i = 0; i < g->ext_count; i++)
        if (g->ext_nodes[i] && g->ext_nodes[i]->base.id == id) return g->ext_nodes[i];
    return NULL;
}

td_graph_t* td_graph_new(td_t* tbl) {
    td_graph_t* g = calloc(1, sizeof(td_graph_t));
    if (!g) return NULL;
    g->nodes = malloc(NODES_INIT * sizeof(td_op_t));
    if (!g->nodes) { free(g); return NULL; }
    g->node_cap = NODES_INIT;
    g->table = tbl;
    if (tbl) td_retain(tbl);
    return g;
}

void td_graph_free(td_graph_t* g) {
    if (!g) return;
    for (uint32_t i = 0; i < g->ext_count; i++) {
        td_op_ext_t* e = g->ext_nodes[i];
        if (e && g->nodes[e->base.id].opcode == OP_CONST && e->literal) td_release(e->literal);
        free(e);
    }
    free(g->ext_nodes);
    free(g->nodes);
    if (g->table) td_release(g->table);
    for (uint16_t i = 0; i < g->n_tables; i++) td_release(g->tables[i]);
    free(g->tables);
    if (g->selection) td_release(g->selection);
    free(g);
}

uint16_t td_graph_add_table(td_graph_t* g, td_t* table) {
    td_t** nt = realloc(g->tables, (size_t)(g->n_tables + 1) * sizeof(td_t*));
    if (!nt) return UINT16_MAX;
    g->tables = nt;
    g->tables[g->n_tables] = table;
    td_retain(table);
    return g->n_tables++;
}

static td_op_t* scan_in(td_graph_t* g, td_t* tbl, uint16_t stored_id, const char* name) {
    td_op_ext_t* e = new_ext(g, 0);
    if (!e) return NULL;
    e->base.opcode = OP_SCAN;
    e->sym = td_sym_intern(name, strlen(name));
    memcpy(e->base.pad, &stored_id, sizeof(stored_id));
    td_t* col = tbl ? td_table_get_col(tbl, e->sym) : NULL;
    if (col) { e->base.out_type = col->type; e->base.est_rows = (uint32_t)col->len; }
    return publish(g, e);
}

td_op_t* td_scan(td_graph_t* g, const char* name) { return scan_in(g, g->table, 0, name); }

td_op_t* td_scan_table(td_graph_t* g, uint16_t tid, const char* name) {
    if (tid >= g->n_tables || !g->tables[tid]) return NULL;
    return scan_in(g, g->tables[tid], (uint16_t)(tid + 1), name);
}

static td_op_t* const_lit(td_graph_t* g, td_t* lit, int8_t out_type, uint32_t est, int retain) {
    td_op_ext_t* e = new_ext(g, 0);
    if (!e) { if (!retain && lit && !TD_IS_ERR(lit)) td_release(lit); return NULL; }
    e->base.opcode = OP_CONST;
    e->base.out_type = out_type;
    e->base.est_rows = est;
    e->literal = (lit && !TD_IS_ERR(lit)) ? lit : NULL;
    if (retain && e->literal) td_retain(e->literal);
    return publish(g, e);
}

td_op_t* td_const_f64(td_graph_t* g, double v)  { return const_lit(g, td_f64(v), TD_F64, 0, 0); }
td_op_t* td_const_i64(td_graph_t* g, int64_t v) { return const_lit(g, td_i64(v), TD_I64, 0, 0); }
td_op_t* td_const_bool(td_graph_t* g, bool v)   { return const_lit(g, td_bool(v), TD_BOOL, 0, 0); }
td_op_t* td_const_str(td_graph_t* g, const char* s) {
    return const_lit(g, td_str(s, strlen(s)), TD_SYM, 0, 0);
}
td_op_t* td_const_vec(td_graph_t* g, td_t* v) {
    return const_lit(g, v, v->type, (uint32_t)v->len, 1);
}
td_op_t* td_const_table(td_graph_t* g, td_t* t) { return const_lit(g, t, TD_TABLE, 0, 1); }

static td_op_t* unary(td_graph_t* g, uint16_t op, td_op_t* a, int8_t ot) {
    uint32_t ai = a->id, est = a->est_rows;
    td_op_t* n = new_node(g);
    if (!n) return NULL;
    n->opcode = op; n->arity = 1; n->inputs[0] = &g->nodes[ai];
    n->out_type = ot; n->est_rows = est;
    return n;
}

static td_op_t* binary(td_graph_t* g, uint16_t op, td_op_t* a, td_op_t* b, int8_t ot) {
    uint32_t ai = a->id, bi = b->id;
    uint32_t est = a->est_rows > b->est_rows ? a->est_rows : b->est_rows;
    td_op_t* n = new_node(g);
    if (!n) return NULL;
    n->opcode = op; n->arity = 2;
    n->inputs[0] = &g->nodes[ai]; n->inputs[1] = &g->nodes[bi];
    n->out_type = ot; n->est_rows = est;
    return n;
}

static int8_t promote(int8_t a, int8_t b) {
#define ANY(t) (a == (t) || b == (t))
    if (ANY(TD_F64)) return TD_F64;
    if (ANY(TD_I64) || ANY(TD_SYM) || ANY(TD_TIMESTAMP)) return TD_I64;
    if (ANY(TD_I32) || ANY(TD_DATE) || ANY(TD_TIME)) return TD_I32;
    if (ANY(TD_I16)) return TD_I16;
    if (ANY(TD_U8)) return TD_U8;
    return TD_BOOL;
#undef ANY
}

td_op_t* td_neg(td_graph_t* g, td_op_t* a) { return unary(g, OP_NEG, a, a->out_type); }
td_op_t* td_abs(td_graph_t* g, td_op_t* a) { return unary(g, OP_ABS, a, a->out_type); }
td_op_t* td_not(td_graph_t* g, td_op_t* a) { return unary(g, OP_NOT, a, TD_BOOL); }
td_op_t* td_cast(td_graph_t* g, td_op_t* a, int8_t t) { return unary(g, OP_CAST, a, t); }

#define ARITH(name, OPC) \
    td_op_t* name(td_graph_t* g, td_op_t* a, td_op_t* b) { \
        return binary(g, OPC, a, b, promote(a->out_type, b->out_type)); }
#define PRED(name, OPC) \
    td_op_t* name(td_graph_t* g, td_op_t* a, td_op_t* b) { return binary(g, OPC, a, b, TD_BOOL); }
ARITH(td_add, OP_ADD)
ARITH(td_sub, OP_SUB)
ARITH(td_mul, OP_MUL)
ARITH(td_mod, OP_MOD)
ARITH(td_min2, OP_MIN2)
ARITH(td_max2, OP_MAX2)
td_op_t* td_div(td_graph_t* g, td_op_t* a, td_op_t* b) { return binary(g, OP_DIV, a, b, TD_F64); }
PRED(td_eq, OP_EQ)
PRED(td_ne, OP_NE)
PRED(td_lt, OP_LT)
PRED(td_le, OP_LE)
PRED(td_gt, OP_GT)
PRED(td_ge, OP_GE)
PRED(td_and, OP_AND)
PRED(td_or, OP_OR)

td_op_t* td_sum(td_graph_t* g, td_op_t* a)    { return unary(g, OP_SUM, a, a->out_type == TD_F64 ? TD_F64 : TD_I64); }
td_op_t* td_min_op(td_graph_t* g, td_op_t* a) { return unary(g, OP_MIN, a, a->out_type); }
td_op_t* td_max_op(td_graph_t* g, td_op_t* a) { return unary(g, OP_MAX, a, a->out_type); }
td_op_t* td_count(td_graph_t* g, td_op_t* a)  { return unary(g, OP_COUNT, a, TD_I64); }
td_op_t* td_avg(td_graph_t* g, td_op_t* a)    { return unary(g, OP_AVG, a, TD_F64); }

td_op_t* td_filter(td_graph_t* g, td_op_t* input, td_op_t* pred) {
    uint32_t ii = input->id, pi = pred->id, est = input->est_rows / 2;
    td_op_t* n = new_node(g);
    if (!n) return NULL;
    n->opcode = OP_FILTER; n->arity = 2;
    n->inputs[0] = &g->nodes[ii]; n->inputs[1] = &g->nodes[pi];
    n->out_type = g->nodes[ii].out_type; n->est_rows = est;
    return n;
}

td_op_t* td_group(td_graph_t* g, td_op_t** keys, uint8_t n_keys,
                  uint16_t* agg_ops, td_op_t** agg_ins, uint8_t n_aggs) {
    uint32_t kid[256], aid[256];
    for (int i = 0; i < n_keys; i++) kid[i] = keys[i]->id;
    for (int i = 0; i < n_aggs; i++) aid[i] = agg_ins[i]->id;
    size_t ksz = (size_t)n_keys * sizeof(td_op_t*);
    size_t osz = (size_t)n_aggs * sizeof(uint16_t);
    size_t ioff = (ksz + osz + sizeof(td_op_t*) - 1) & ~(sizeof(td_op_t*) - 1);
    td_op_ext_t* e = new_ext(g, ioff + (size_t)n_aggs * sizeof(td_op_t*));
    if (!e) return NULL;
    char* trail = (char*)(e + 1);
    e->base.opcode = OP_GROUP;
    e->base.out_type = TD_TABLE;
    if (n_keys > 0) {
        e->base.est_rows = g->nodes[kid[0]].est_rows / 10;
        e->base.inputs[0] = &g->nodes[kid[0]];
    }
    e->keys = (td_op_t**)trail;
    for (int i = 0; i < n_keys; i++) e->keys[i] = &g->nodes[kid[i]];
    e->agg_ops = (uint16_t*)(trail + ksz);
    if (osz) memcpy(e->agg_ops, agg_ops, osz);
    e->agg_ins = (td_op_t**)(trail + ioff);
    for (int i = 0; i < n_aggs; i++) e->agg_ins[i] = &g->nodes[aid[i]];
    e->n_keys = n_keys;
    e->n_aggs = n_aggs;
    return publish(g, e);
}

/* Sort node (graph.c:620-663 of Teide): key columns, DESC flags and
 * nulls-first flags stored after the ext node; nulls_first defaults to DESC
 * (NULLS LAST ascending, NULLS FIRST descending). */
td_op_t* td_sort_op(td_graph_t* g, td_op_t* table_node, td_op_t** keys, uint8_t* descs, uint8_t* nulls_first,
                    uint8_t n_cols) {
    uint32_t ti = table_node->id, kid[256];
    for (int i = 0; i < n_cols; i++) kid[i] = keys[i]->id;
    size_t ksz = (size_t)n_cols * sizeof(td_op_t*);
    td_op_ext_t* e = new_ext(g, ksz + 2 * (size_t)n_cols);
    if (!e) return NULL;
    char* trail = (char*)(e + 1);
    e->base.opcode = OP_SORT;
    e->base.arity = 1;
    e->base.inputs[0] = &g->nodes[ti];
    e->base.out_type = TD_TABLE;
    e->base.est_rows = g->nodes[ti].est_rows;
    e->sort.columns = (td_op_t**)trail;
    for (int i = 0; i < n_cols; i++) e->sort.columns[i] = &g->nodes[kid[i]];
    e->sort.desc = (uint8_t*)(trail + ksz);
    e->sort.nulls_first = (uint8_t*)(trail + ksz + n_cols);
    for (int i = 0; i < n_cols; i++) {
        e->sort.desc[i] = descs ? descs[i] : 0;
        e->sort.nulls_first[i] = nulls_first ? nulls_first[i] : e->sort.desc[i];
    }
    e->sort.n_cols = n_cols;
    return publish(g, e);
}

/* First n rows (graph.c:906-922 of Teide): n is kept in the ext node's sym. */
td_op_t* td_head(td_graph_t* g, td_op_t* input, int64_t n) {
    uint32_t ii = input->id;
    td_op_ext_t* e = new_ext(g, 0);
    if (!e) return NULL;
    e->base.opcode = OP_HEAD;
    e->base.arity = 1;
    e->base.inputs[0] = &g->nodes[ii];
    e->base.out_type = g->nodes[ii].out_type;
    e->base.est_rows = (uint32_t)n;
    e->sym = n;
    return publish(g, e);
}

td_op_t* td_distinct(td_graph_t* g, td_op_t** keys, uint8_t n_keys) {
    return td_group(g, keys, n_keys, NULL, NULL, 0);
}

td_op_t* td_join(td_graph_t* g, td_op_t* lt, td_op_t** lkeys,
                 td_op_t* rt, td_op_t** rkeys, uint8_t n_keys, uint8_t join_type) {
    uint32_t li = lt->id, ri = rt->id, lk[256], rk[256];
    for (int i = 0; i < n_keys; i++) { lk[i] = lkeys[i]->id; rk[i] = rkeys[i]->id; }
    size_t ksz = (size_t)n_keys * sizeof(td_op_t*);
    td_op_ext_t* e = new_ext(g, 2 * ksz);
    if (!e) return NULL;
    char* trail = (char*)(e + 1);
    e->base.opcode = OP_JOIN;
    e->base.arity = 2;
    e->base.inputs[0] = &g->nodes[li];
    e->base.inputs[1] = &g->nodes[ri];
    e->base.out_type = TD_TABLE;
    e->base.est_rows = g->nodes[li].est_rows;
    e->join.left_keys = (td_op_t**)trail;
    e->join.right_keys = (td_op_t**)(trail + ksz);
    for (int i = 0; i < n_keys; i++) {
        e->join.left_keys[i] = &g->nodes[lk[i]];
        e->join.right_keys[i] = &g->nodes[rk[i]];
    }
    e->join.n_join_keys = n_keys;
    e->join.join_type = join_type;
    return publish(g, e);
}

td_op_t* td_alias(td_graph_t* g, td_op_t* input, const char* name) {
    uint32_t ii = input->id;
    td_op_ext_t* e = new_ext(g, 0);
    if (!e) return NULL;
    e->base.opcode = OP_ALIAS;
    e->base.arity = 1;
    e->base.inputs[0] = &g->nodes[ii];
    e->base.out_type = g->nodes[ii].out_type;
    e->base.est_rows = g->nodes[ii].est_rows;
    e->sym = td_sym_intern(name, strlen(name));
    return publish(g, e);
}

td_op_t* td_materialize(td_graph_t* g, td_op_t* input) {
    uint32_t ii = input->id;
    td_op_t* n = new_node(g);
    if (!n) return NULL;
    n->opcode = OP_MATERIALIZE; n->arity = 1;
    n->inputs[0] = &g->nodes[ii];
    n->out_type = g->nodes[ii].out_type;
    n->est_rows = g->nodes[ii].est_rows;
    return n;
}

/* The optimizer passes Teide runs for these DAGs (src/ops/opt.c:1641-1675)
 * only rewrite shapes that the GPU lowering recognizes either way
 * (filter chains, predicate order); the DAG is executed as built. */
td_op_t* td_optimize(td_graph_t* g, td_op_t* root) { (void)g; return root; }
void td_fuse_pass(td_graph_t* g, td_op_t* root) { (void)g; (void)root; }
