/*
 * Tables.  Layout kept from Teide (src/table/table.c:40-127): a TD_TABLE
 * block whose data is [schema, col_0, col_1, ...] -- schema an I64 vector of
 * column-name symbol ids -- and whose len is the column count.  Columns are
 * retained by the table; nrows is the first column's length.
 */
#include "internal.h"
#include <string.h>

static td_t** schema_slot(td_t* t) { return (td_t**)td_data(t); }
static td_t** col_slots(td_t* t)   { return (td_t**)td_data(t) + 1; }

td_t* td_table_new(int64_t ncols) {
    if (ncols < 0) return TD_ERR_PTR(TD_ERR_RANGE);
    size_t bytes = (size_t)(ncols + 1) * sizeof(td_t*);
    td_t* t = td_alloc(bytes);
    if (!t) return TD_ERR_PTR(TD_ERR_OOM);
    t->type = TD_TABLE;
    memset(td_data(t), 0, bytes);
    td_t* schema = td_vec_new(TD_I64, ncols);
    if (!schema || TD_IS_ERR(schema)) { td_free(t); return schema; }
    *schema_slot(t) = schema;
    return t;
}

td_t* td_table_add_col(td_t* t, int64_t name_id, td_t* col) {
    if (!t || TD_IS_ERR(t)) return t;
    if (!col || TD_IS_ERR(col)) return TD_ERR_PTR(TD_ERR_TYPE);
    t = td_cow(t);
    if (!t || TD_IS_ERR(t)) return t;
    int64_t idx = t->len;
    int64_t max_cols = (int64_t)((((size_t)1 << t->order) - 32) / sizeof(td_t*)) - 1;
    if (idx >= max_cols) {
        td_t* n = td_scratch_realloc(t, (size_t)(1 + (idx + 1) * 2) * sizeof(td_t*));
        if (!n || TD_IS_ERR(n)) return n ? n : TD_ERR_PTR(TD_ERR_OOM);
        t = n;
    }
    td_t* schema = td_vec_append(*schema_slot(t), &name_id);
    if (!schema || TD_IS_ERR(schema)) return TD_ERR_PTR(TD_ERR_OOM);
    *schema_slot(t) = schema;
    col_slots(t)[idx] = col;
    td_retain(col);
    t->len = idx + 1;
    return t;
}

td_t* td_table_get_col(td_t* t, int64_t name_id) {
    if (!t || TD_IS_ERR(t) || t->type != TD_TABLE) return NULL;
    td_t* schema = *schema_slot(t);
    if (!schema || TD_IS_ERR(schema)) return NULL;
    const int64_t* ids = (const int64_t*)td_data(schema);
    for (int64_t i = 0; i < t->len; i++)
        if (ids[i] == name_id) return col_slots(t)[i];
    return NULL;
}

td_t* td_table_get_col_idx(td_t* t, int64_t idx) {
    if (!t || TD_IS_ERR(t) || idx < 0 || idx >= t->len) return NULL;
    return col_slots(t)[idx];
}

int64_t td_table_col_name(td_t* t, int64_t idx) {
    if (!t || TD_IS_ERR(t) || idx < 0 || idx >= t->len) return -1;
    td_t* schema = *schema_slot(t);
    if (!schema || TD_IS_ERR(schema)) return -1;
    return ((const int64_t*)td_data(schema))[idx];
}

void td_table_set_col_name(td_t* t, int64_t idx, int64_t name_id) {
    if (!t || TD_IS_ERR(t) || idx < 0 || idx >= t->len) return;
    td_t* schema = td_cow(*schema_slot(t));
    if (!schema || TD_IS_ERR(schema)) return;
    *schema_slot(t) = schema;
    ((int64_t*)td_data(schema))[idx] = name_id;
}

int64_t td_table_ncols(td_t* t) { return (!t || TD_IS_ERR(t)) ? 0 : t->len; }

int64_t td_table_nrows(td_t* t) {
    if (!t || TD_IS_ERR(t) || t->len <= 0) return 0;
    td_t* c = col_slots(t)[0];
    return (!c || TD_IS_ERR(c)) ? 0 : td_parted_nrows(c);
}

/* Rows of a column: its length, or for a parted column the sum of its
 * segments' lengths and for a MAPCOMMON column the sum of its row counts
 * (table.c:226-250). */
int64_t td_parted_nrows(td_t* v) {
    if (!v || TD_IS_ERR(v)) return 0;
    if (v->type == TD_MAPCOMMON) {
        td_t* counts = ((td_t**)td_data(v))[1];
        if (!counts || TD_IS_ERR(counts)) return 0;
        int64_t total = 0;
        for (int64_t i = 0; i < counts->len; i++) total += ((const int64_t*)td_data(counts))[i];
        return total;
    }
    if (!TD_IS_PARTED(v->type)) return v->len;
    int64_t total = 0;
    for (int64_t i = 0; i < v->len; i++) {
        td_t* seg = ((td_t**)td_data(v))[i];
        if (seg && !TD_IS_ERR(seg)) total += seg->len;
    }
    return total;
}

td_t* td_table_schema(td_t* t) {
    return (!t || TD_IS_ERR(t)) ? NULL : *schema_slot(t);
}
