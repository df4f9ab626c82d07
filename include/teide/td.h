/*
 * teide/td.h -- public C17 API of the B200 executor.
 *
 * This header is a drop-in for Teide's public header (include/teide/td.h in
 * TeideDB/teide).  A caller that builds a DAG with td_graph_new / td_scan /
 * td_filter / td_group / td_join and runs it with td_optimize + td_execute
 * compiles against this file unchanged and links against libteide_b200.so.
 *
 * What must be identical, and is:
 *   - the td_t object header (32 bytes, element data inline after it), because
 *     callers read columns through the inline accessors below (td.h:224-311);
 *   - td_op_t / td_op_ext_t / td_graph_t field layout (td.h:443-530), because
 *     callers and the optimizer walk g->nodes and ext->keys directly;
 *   - the TD_SEL selection block layout (td.h:546-589);
 *   - type tags, opcodes, error codes and constants (td.h:104-214, 315-440).
 * The layouts are restated here field by field; tests/test_abi.py checks every
 * offset against the reference's compiled header.
 *
 * What is different: td_execute runs filter / group-by / join on the GPU
 * (hand-written sm_100a kernels behind include/tdg.h).  There is no CPU
 * execution path.  Opcodes outside that relational path return TD_ERR_NYI.
 * The B200-only extensions (device residency, statistics) are declared in
 * teide/td_b200.h.
 */
#ifndef TD_H
#define TD_H

#include <stdint.h>
#include <stdbool.h>
#include <stddef.h>
#include <stdatomic.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef TD_LIKELY
#  define TD_LIKELY(x)   __builtin_expect(!!(x), 1)
#  define TD_UNLIKELY(x) __builtin_expect(!!(x), 0)
#  define TD_ALIGN(n)    __attribute__((aligned(n)))
#  define TD_INLINE      static inline __attribute__((always_inline))
#endif
#ifndef TD_ASSUME_ALIGNED
#  define TD_ASSUME_ALIGNED(p, n) __builtin_assume_aligned((p), (n))
#endif
#define TD_TLS _Thread_local

#define td_atomic_inc(p)   atomic_fetch_add_explicit(p, 1, memory_order_relaxed)
#define td_atomic_dec(p)   atomic_fetch_sub_explicit(p, 1, memory_order_acq_rel)
#define td_atomic_load(p)  atomic_load_explicit(p, memory_order_acquire)

/* ---- type tags (positive = vector, negative = atom) ---------------------- */
#define TD_LIST       0
#define TD_BOOL       1
#define TD_U8         2
#define TD_CHAR       3
#define TD_I16        4
#define TD_I32        5
#define TD_I64        6
#define TD_F64        7
#define TD_DATE       9
#define TD_TIME      10
#define TD_TIMESTAMP 11
#define TD_GUID      12
#define TD_TABLE     13
#define TD_SEL       16
#define TD_SYM       20

/* Partitioned tables (src/store/part.c): a parted column is a vector of
 * segment pointers, one per partition, typed TD_PARTED_BASE + the segments'
 * type; the MAPCOMMON column holds the partition keys -- its two elements
 * are the key values (DATE, I64 or SYM by the directory names, attrs
 * TD_MC_*) and the partitions' row counts (I64). */
#define TD_PARTED_BASE   32
#define TD_MAPCOMMON     64
#define TD_MC_SYM    0
#define TD_MC_DATE   1
#define TD_MC_I64    2
#define TD_IS_PARTED(t)       ((t) >= TD_PARTED_BASE && (t) < TD_MAPCOMMON)
#define TD_PARTED_BASETYPE(t) ((t) - TD_PARTED_BASE)

/* dictionary-index width of a TD_SYM column: low two bits of attrs */
#define TD_SYM_W_MASK   0x03
#define TD_SYM_W8       0x00
#define TD_SYM_W16      0x01
#define TD_SYM_W32      0x02
#define TD_SYM_W64      0x03
#define TD_IS_SYM(t)         ((t) == TD_SYM)
#define TD_SYM_ELEM(attrs)   (1u << ((attrs) & TD_SYM_W_MASK))
#define TD_META_DICT  0x4449

#define TD_PARTED_BASE   32
#define TD_MAPCOMMON     64
#define TD_MC_SYM    0
#define TD_MC_DATE   1
#define TD_MC_I64    2
#define TD_IS_PARTED(t)       ((t) >= TD_PARTED_BASE && (t) < TD_MAPCOMMON)
#define TD_PARTED_BASETYPE(t) ((t) - TD_PARTED_BASE)

#define TD_ATOM_BOOL       (-TD_BOOL)
#define TD_ATOM_U8         (-TD_U8)
#define TD_ATOM_CHAR       (-TD_CHAR)
#define TD_ATOM_I16        (-TD_I16)
#define TD_ATOM_I32        (-TD_I32)
#define TD_ATOM_I64        (-TD_I64)
#define TD_ATOM_F64        (-TD_F64)
#define TD_ATOM_STR        (-8)
#define TD_ATOM_DATE       (-TD_DATE)
#define TD_ATOM_TIME       (-TD_TIME)
#define TD_ATOM_TIMESTAMP  (-TD_TIMESTAMP)
#define TD_ATOM_GUID       (-TD_GUID)
#define TD_ATOM_SYM        (-TD_SYM)
#define TD_TYPE_COUNT 21

#define TD_ATTR_SLICE        0x10
#define TD_ATTR_NULLMAP_EXT  0x20
#define TD_ATTR_HAS_NULLS    0x40

/* ---- tuning constants (kept for source compatibility) -------------------- */
#define TD_MORSEL_ELEMS        1024
#define TD_SLAB_CACHE_SIZE     64
#define TD_SLAB_ORDERS         5
#define TD_ORDER_MIN           6
#define TD_ORDER_MAX           30
#define TD_PARALLEL_THRESHOLD  (64 * TD_MORSEL_ELEMS)
#define TD_DISPATCH_MORSELS    8
#define TD_JOIN_L2_TARGET      (256 * 1024)
#define TD_JOIN_MIN_RADIX      2
#define TD_JOIN_MAX_RADIX      14

/* ---- errors: td_t* results carry a code in the pointer value ------------- */
typedef enum {
    TD_OK = 0,
    TD_ERR_OOM,
    TD_ERR_TYPE,
    TD_ERR_RANGE,
    TD_ERR_LENGTH,
    TD_ERR_RANK,
    TD_ERR_DOMAIN,
    TD_ERR_NYI,
    TD_ERR_IO,
    TD_ERR_SCHEMA,
    TD_ERR_CORRUPT,
    TD_ERR_CANCEL
} td_err_t;

#define TD_ERR_PTR(e)   ((td_t*)(uintptr_t)(e))
#define TD_IS_ERR(p)    ((uintptr_t)(p) < 32)
#define TD_ERR_CODE(p)  ((td_err_t)(uintptr_t)(p))

const char* td_err_str(td_err_t e);

/* ---- td_t: 32-byte header, element data follows inline ------------------- */
typedef union TD_ALIGN(32) td_t {
    struct {
        union {                                   /* bytes 0-15 */
            uint8_t nullmap[16];
            struct { union td_t* slice_parent; int64_t slice_offset; };
            struct { union td_t* ext_nullmap;  union td_t* sym_dict; };
        };
        uint8_t  mmod;                            /* 16: 0 heap, 1 file map */
        uint8_t  order;                           /* 17: block = 2^order bytes */
        int8_t   type;                            /* 18 */
        uint8_t  attrs;                           /* 19 */
        _Atomic(uint32_t) rc;                     /* 20: 0 = free */
        union {                                   /* 24: atom value or length */
            uint8_t  b8;
            uint8_t  u8;
            char     c8;
            int16_t  i16;
            int32_t  i32;
            uint32_t u32;
            int64_t  i64;
            double   f64;
            union td_t* obj;
            struct { uint8_t slen; char sdata[7]; };
            int64_t  len;
        };
        uint8_t data[];                           /* 32: elements */
    };
    struct { union td_t* fl_prev; union td_t* fl_next; };
} td_t;

extern const uint8_t td_type_sizes[TD_TYPE_COUNT];

#define td_type(v)       ((v)->type)
#define td_is_atom(v)    ((v)->type < 0)
#define td_is_vec(v)     ((v)->type > 0)
#define td_len(v)        ((v)->len)
static inline void* td_data_fn(td_t* v) { return TD_ASSUME_ALIGNED((void*)v->data, 32); }
#define td_data(v)       td_data_fn(v)
#define td_elem_size(t)  (td_type_sizes[(t)])

static inline uint8_t td_sym_elem_size(int8_t type, uint8_t attrs) {
    return type == TD_SYM ? (uint8_t)TD_SYM_ELEM(attrs) : td_elem_size(type);
}
static inline int64_t td_read_sym(const void* data, int64_t row, int8_t type, uint8_t attrs) {
    (void)type;
    switch (attrs & TD_SYM_W_MASK) {
        case TD_SYM_W8:  return ((const uint8_t*)data)[row];
        case TD_SYM_W16: return ((const uint16_t*)data)[row];
        case TD_SYM_W32: return ((const uint32_t*)data)[row];
        default:         return ((const int64_t*)data)[row];
    }
}
static inline void td_write_sym(void* data, int64_t row, uint64_t val, int8_t type, uint8_t attrs) {
    (void)type;
    switch (attrs & TD_SYM_W_MASK) {
        case TD_SYM_W8:  ((uint8_t*)data)[row]  = (uint8_t)val;  break;
        case TD_SYM_W16: ((uint16_t*)data)[row] = (uint16_t)val; break;
        case TD_SYM_W32: ((uint32_t*)data)[row] = (uint32_t)val; break;
        default:         ((int64_t*)data)[row]  = (int64_t)val;  break;
    }
}
static inline uint8_t td_sym_dict_width(int64_t dict_size) {
    return dict_size <= 255 ? TD_SYM_W8 : dict_size <= 65535 ? TD_SYM_W16
         : dict_size <= 4294967295LL ? TD_SYM_W32 : TD_SYM_W64;
}

/* ---- opcodes -------------------------------------------------------------- */
#define OP_SCAN          1
#define OP_CONST         2
#define OP_NEG          10
#define OP_ABS          11
#define OP_NOT          12
#define OP_SQRT         13
#define OP_LOG          14
#define OP_EXP          15
#define OP_CEIL         16
#define OP_FLOOR        17
#define OP_ISNULL       18
#define OP_CAST         19
#define OP_ADD          20
#define OP_SUB          21
#define OP_MUL          22
#define OP_DIV          23
#define OP_MOD          24
#define OP_EQ           25
#define OP_NE           26
#define OP_LT           27
#define OP_LE           28
#define OP_GT           29
#define OP_GE           30
#define OP_AND          31
#define OP_OR           32
#define OP_MIN2         33
#define OP_MAX2         34
#define OP_IF           35
#define OP_LIKE         36
#define OP_UPPER        37
#define OP_LOWER        38
#define OP_STRLEN       39
#define OP_SUBSTR       40
#define OP_REPLACE      41
#define OP_TRIM         42
#define OP_CONCAT       43
#define OP_EXTRACT      45
#define OP_DATE_TRUNC   46
#define OP_SUM          50
#define OP_PROD         51
#define OP_MIN          52
#define OP_MAX          53
#define OP_COUNT        54
#define OP_AVG          55
#define OP_FIRST        56
#define OP_LAST         57
#define OP_COUNT_DISTINCT 58
#define OP_STDDEV       59
#define OP_FILTER       60
#define OP_SORT         61
#define OP_GROUP        62
#define OP_JOIN         63
#define OP_WINDOW_JOIN  64
#define OP_SELECT       66
#define OP_HEAD         67
#define OP_TAIL         68
#define OP_ALIAS        70
#define OP_MATERIALIZE  71
#define OP_WINDOW       72
#define OP_STDDEV_POP   73
#define OP_VAR          74
#define OP_VAR_POP      75
#define OP_ILIKE        76
#define OP_EXPAND        80
#define OP_VAR_EXPAND    81
#define OP_SHORTEST_PATH 82
#define OP_WCO_JOIN      83

#define OP_FLAG_FUSED   0x01
#define OP_FLAG_DEAD    0x02

/* 32-byte DAG node */
typedef struct td_op {
    uint16_t       opcode;
    uint8_t        arity;
    uint8_t        flags;
    int8_t         out_type;
    uint8_t        pad[3];      /* OP_SCAN: pad[0..1] = table id + 1 (0 = g->table) */
    uint32_t       id;
    uint32_t       est_rows;
    struct td_op*  inputs[2];
} td_op_t;

/* N-ary node: the 32-byte base plus an opcode-specific payload.  Arrays the
 * payload points to live in the same allocation, after the struct. */
typedef struct td_op_ext {
    td_op_t base;
    union {
        td_t*   literal;                          /* OP_CONST */
        int64_t sym;                              /* OP_SCAN column name */
        struct {                                  /* OP_GROUP */
            td_op_t**  keys;
            uint8_t    n_keys;
            uint8_t    n_aggs;
            uint16_t*  agg_ops;
            td_op_t**  agg_ins;
        };
        struct {                                  /* OP_SORT / OP_SELECT */
            td_op_t**  columns;
            uint8_t*   desc;
            uint8_t*   nulls_first;
            uint8_t    n_cols;
        } sort;
        struct {                                  /* OP_JOIN */
            td_op_t**  left_keys;
            td_op_t**  right_keys;
            uint8_t    n_join_keys;
            uint8_t    join_type;                 /* 0 inner, 1 left, 2 full */
        } join;
        struct {
            td_op_t*   time_key;
            td_op_t**  eq_keys;
            uint8_t    n_eq_keys;
            uint8_t    join_type;
        } asof;
        struct {
            td_op_t**  part_keys;
            td_op_t**  order_keys;
            uint8_t*   order_descs;
            td_op_t**  func_inputs;
            uint8_t*   func_kinds;
            int64_t*   func_params;
            uint8_t    n_part_keys;
            uint8_t    n_order_keys;
            uint8_t    n_funcs;
            uint8_t    frame_type;
            uint8_t    frame_start;
            uint8_t    frame_end;
            int64_t    frame_start_n;
            int64_t    frame_end_n;
        } window;
        struct {
            void*     rel;
            void*     sip_sel;
            uint8_t   direction;
            uint8_t   min_depth;
            uint8_t   max_depth;
            uint8_t   path_tracking;
            uint8_t   factorized;
        } graph;
        struct {
            void**    rels;
            uint8_t   n_rels;
            uint8_t   n_vars;
        } wco;
    };
} td_op_ext_t;

typedef struct td_graph {
    td_op_t*       nodes;
    uint32_t       node_count;
    uint32_t       node_cap;
    td_t*          table;
    td_t**         tables;
    uint16_t       n_tables;
    td_op_ext_t**  ext_nodes;
    uint32_t       ext_count;
    uint32_t       ext_cap;
    td_t*          selection;   /* TD_SEL lazy filter, NULL = every row */
} td_graph_t;

typedef struct {
    td_t*    vec;
    int64_t  offset;
    int64_t  len;
    uint32_t elem_size;
    int64_t  morsel_len;
    void*    morsel_ptr;
    uint8_t* null_bits;
} td_morsel_t;

/* ---- TD_SEL: per-1024-row segment summary + one bit per row --------------
 *   td_sel_meta_t meta            16 B
 *   uint8_t  seg_flags[n_segs]    padded to 8 B
 *   uint16_t seg_popcnt[n_segs]   padded to 8 B
 *   uint64_t bits[ceil(n/64)]                                               */
#define TD_SEL_NONE  0
#define TD_SEL_ALL   1
#define TD_SEL_MIX   2
#define TD_SEL_WORDS_PER_SEG  (TD_MORSEL_ELEMS / 64)

typedef struct {
    int64_t   total_pass;
    uint32_t  n_segs;
    uint32_t  _pad;
} td_sel_meta_t;

static inline td_sel_meta_t* td_sel_meta(td_t* s) { return (td_sel_meta_t*)td_data(s); }
static inline uint8_t* td_sel_flags(td_t* s) { return (uint8_t*)td_data(s) + sizeof(td_sel_meta_t); }
static inline uint16_t* td_sel_popcnt(td_t* s) {
    uint32_t n = td_sel_meta(s)->n_segs;
    return (uint16_t*)(td_sel_flags(s) + ((n + 7u) & ~7u));
}
static inline uint64_t* td_sel_bits(td_t* s) {
    uint32_t n = td_sel_meta(s)->n_segs;
    return (uint64_t*)(td_sel_popcnt(s) + ((n + 3u) & ~3u));
}
#define TD_SEL_BIT_TEST(bits, r)  ((bits)[(r) >> 6] & (1ULL << ((r) & 63)))
#define TD_SEL_BIT_SET(bits, r)   ((bits)[(r) >> 6] |= (1ULL << ((r) & 63)))
#define TD_SEL_BIT_CLR(bits, r)   ((bits)[(r) >> 6] &= ~(1ULL << ((r) & 63)))

typedef struct td_pipe {
    td_op_t*          op;
    struct td_pipe*   inputs[2];
    td_morsel_t       state;
    td_t*             materialized;
    int               spill_fd;
} td_pipe_t;

typedef struct {
    size_t alloc_count;
    size_t free_count;
    size_t bytes_allocated;
    size_t peak_bytes;
    size_t slab_hits;
    size_t direct_count;
    size_t direct_bytes;
    size_t sys_current;
    size_t sys_peak;
} td_mem_stats_t;

typedef struct td_heap      td_heap_t;
typedef struct td_sym_table td_sym_table_t;
typedef struct td_pool      td_pool_t;
typedef struct td_rel       td_rel_t;

/* ==== API provided by libteide_b200.so ==================================== */

uint32_t td_thread_count(void);

/* memory (host heap; large blocks are page-locked so uploads run at link speed) */
td_t*    td_alloc(size_t data_size);
void     td_free(td_t* v);
td_t*    td_alloc_copy(td_t* v);
td_t*    td_scratch_alloc(size_t data_size);
td_t*    td_scratch_realloc(td_t* v, size_t new_data_size);
void     td_heap_init(void);
void     td_heap_destroy(void);
void     td_heap_gc(void);
uint8_t  td_order_for_size(size_t data_size);
void     td_mem_stats(td_mem_stats_t* out);

void     td_retain(td_t* v);
void     td_release(td_t* v);
td_t*    td_cow(td_t* v);

/* atoms */
td_t* td_bool(bool val);
td_t* td_u8(uint8_t val);
td_t* td_char(char val);
td_t* td_i16(int16_t val);
td_t* td_i32(int32_t val);
td_t* td_i64(int64_t val);
td_t* td_f64(double val);
td_t* td_str(const char* s, size_t len);
td_t* td_sym(int64_t id);
td_t* td_date(int64_t val);
td_t* td_time(int64_t val);
td_t* td_timestamp(int64_t val);

/* selections */
td_t* td_sel_new(int64_t nrows);
td_t* td_sel_from_pred(td_t* bool_vec);
td_t* td_sel_and(td_t* a, td_t* b);
void  td_sel_recompute(td_t* sel);

/* vectors */
td_t* td_vec_new(int8_t type, int64_t capacity);
td_t* td_sym_vec_new(uint8_t sym_width, int64_t capacity);
td_t* td_vec_append(td_t* vec, const void* elem);
td_t* td_vec_set(td_t* vec, int64_t idx, const void* elem);
void* td_vec_get(td_t* vec, int64_t idx);
td_t* td_vec_slice(td_t* vec, int64_t offset, int64_t len);
td_t* td_vec_concat(td_t* a, td_t* b);
td_t* td_vec_from_raw(int8_t type, const void* data, int64_t count);
void  td_vec_set_null(td_t* vec, int64_t idx, bool is_null);
bool  td_vec_is_null(td_t* vec, int64_t idx);

/* strings */
const char* td_str_ptr(td_t* s);
size_t      td_str_len(td_t* s);
int         td_str_cmp(td_t* a, td_t* b);

/* symbols */
void     td_sym_init(void);
void     td_sym_destroy(void);
int64_t  td_sym_intern(const char* str, size_t len);
int64_t  td_sym_find(const char* str, size_t len);
td_t*    td_sym_str(int64_t id);
uint32_t td_sym_count(void);

/* tables */
td_t*   td_table_new(int64_t ncols);
td_t*   td_table_add_col(td_t* tbl, int64_t name_id, td_t* col_vec);
td_t*   td_table_get_col(td_t* tbl, int64_t name_id);
td_t*   td_table_get_col_idx(td_t* tbl, int64_t idx);
int64_t td_table_col_name(td_t* tbl, int64_t idx);
void    td_table_set_col_name(td_t* tbl, int64_t idx, int64_t name_id);
int64_t td_table_ncols(td_t* tbl);
int64_t td_table_nrows(td_t* tbl);
td_t*   td_table_schema(td_t* tbl);

/* Column files and splayed tables (src/store/col.c, splay.c): scalar
 * columns as the 32-byte header plus raw data; a splayed table is a
 * directory of column files and a ".d" file of column-name symbol ids. */
td_err_t td_col_save(td_t* vec, const char* path);
td_t*    td_col_load(const char* path);
/* Zero-copy: the vector's data is the file's own pages, mapped copy-on-write
 * (mmod = 1); td_release unmaps it. */
td_t*    td_col_mmap(const char* path);
td_err_t td_splay_save(td_t* tbl, const char* dir, const char* sym_path);
td_t*    td_splay_load(const char* dir);
/* td_splay_load with every column mapped by td_col_mmap; sym_path (or NULL)
 * is a symbol file loaded first. */
td_t*    td_read_splayed(const char* dir, const char* sym_path);
/* The symbol table file ("TSYM", count, then length-prefixed strings). */
td_err_t td_sym_save(const char* path);
td_err_t td_sym_load(const char* path);
/* A partitioned database: every partition directory of db_root (a name of
 * digits and dots, in name order) holds the splayed table `table_name`; the
 * partitions' columns are concatenated (src/store/part.c). */
td_t*    td_part_load(const char* db_root, const char* table_name);
/* The same database as a partitioned table: the MAPCOMMON column first
 * (named "date" for YYYY.MM.DD directories, else "part"), then one parted
 * column per column of the partitions, segments in partition-name order;
 * db_root/sym is loaded first when present.  Rows = td_parted_nrows. */
td_t*    td_read_parted(const char* db_root, const char* table_name);
int64_t  td_parted_nrows(td_t* parted_col);

/* DAG construction */
td_graph_t* td_graph_new(td_t* tbl);
void        td_graph_free(td_graph_t* g);
uint16_t    td_graph_add_table(td_graph_t* g, td_t* table);

td_op_t* td_scan(td_graph_t* g, const char* col_name);
td_op_t* td_scan_table(td_graph_t* g, uint16_t table_id, const char* col_name);
td_op_t* td_const_f64(td_graph_t* g, double val);
td_op_t* td_const_i64(td_graph_t* g, int64_t val);
td_op_t* td_const_bool(td_graph_t* g, bool val);
td_op_t* td_const_str(td_graph_t* g, const char* s);
td_op_t* td_const_vec(td_graph_t* g, td_t* vec);
td_op_t* td_const_table(td_graph_t* g, td_t* table);

td_op_t* td_neg(td_graph_t* g, td_op_t* a);
td_op_t* td_abs(td_graph_t* g, td_op_t* a);
td_op_t* td_not(td_graph_t* g, td_op_t* a);
td_op_t* td_cast(td_graph_t* g, td_op_t* a, int8_t target_type);

td_op_t* td_add(td_graph_t* g, td_op_t* a, td_op_t* b);
td_op_t* td_sub(td_graph_t* g, td_op_t* a, td_op_t* b);
td_op_t* td_mul(td_graph_t* g, td_op_t* a, td_op_t* b);
td_op_t* td_div(td_graph_t* g, td_op_t* a, td_op_t* b);
td_op_t* td_mod(td_graph_t* g, td_op_t* a, td_op_t* b);
td_op_t* td_eq(td_graph_t* g, td_op_t* a, td_op_t* b);
td_op_t* td_ne(td_graph_t* g, td_op_t* a, td_op_t* b);
td_op_t* td_lt(td_graph_t* g, td_op_t* a, td_op_t* b);
td_op_t* td_le(td_graph_t* g, td_op_t* a, td_op_t* b);
td_op_t* td_gt(td_graph_t* g, td_op_t* a, td_op_t* b);
td_op_t* td_ge(td_graph_t* g, td_op_t* a, td_op_t* b);
td_op_t* td_and(td_graph_t* g, td_op_t* a, td_op_t* b);
td_op_t* td_or(td_graph_t* g, td_op_t* a, td_op_t* b);
td_op_t* td_min2(td_graph_t* g, td_op_t* a, td_op_t* b);
td_op_t* td_max2(td_graph_t* g, td_op_t* a, td_op_t* b);

td_op_t* td_sum(td_graph_t* g, td_op_t* a);
td_op_t* td_min_op(td_graph_t* g, td_op_t* a);
td_op_t* td_max_op(td_graph_t* g, td_op_t* a);
td_op_t* td_count(td_graph_t* g, td_op_t* a);
td_op_t* td_avg(td_graph_t* g, td_op_t* a);

td_op_t* td_filter(td_graph_t* g, td_op_t* input, td_op_t* predicate);
td_op_t* td_group(td_graph_t* g, td_op_t** keys, uint8_t n_keys,
                  uint16_t* agg_ops, td_op_t** agg_ins, uint8_t n_aggs);
td_op_t* td_distinct(td_graph_t* g, td_op_t** keys, uint8_t n_keys);
td_op_t* td_sort_op(td_graph_t* g, td_op_t* table_node,
                    td_op_t** keys, uint8_t* descs, uint8_t* nulls_first,
                    uint8_t n_cols);
td_op_t* td_head(td_graph_t* g, td_op_t* input, int64_t n);
td_op_t* td_join(td_graph_t* g,
                 td_op_t* left_table, td_op_t** left_keys,
                 td_op_t* right_table, td_op_t** right_keys,
                 uint8_t n_keys, uint8_t join_type);
td_op_t* td_alias(td_graph_t* g, td_op_t* input, const char* name);
td_op_t* td_materialize(td_graph_t* g, td_op_t* input);

/* optimizer and executor */
td_op_t* td_optimize(td_graph_t* g, td_op_t* root);
void     td_fuse_pass(td_graph_t* g, td_op_t* root);
td_t*    td_execute(td_graph_t* g, td_op_t* root);

/* execution control */
td_err_t td_pool_init(uint32_t n_workers);
void     td_pool_destroy(void);
void     td_cancel(void);

#ifdef __cplusplus
}
#endif

#endif /* TD_H */
