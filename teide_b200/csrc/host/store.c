/*
 * Column files, splayed tables and the symbol file, in Teide's on-disk
 * formats (src/store/col.c, src/store/splay.c, src/table/sym.c of
 * TeideDB/teide), so files written by either library load in the other.
 *
 *   column file   the 32-byte td_t header (nullmap bytes kept only when the
 *                 column has inline nulls; mmod, order, rc and the slice
 *                 flag cleared) followed by len * element-size data bytes
 *                 (col.c:34-41, td_col_save 344-444, td_col_load 449-561).
 *                 Scalar types only: BOOL, U8, CHAR, I16, I32, I64, F64,
 *                 DATE, TIME, TIMESTAMP, GUID, SYM.
 *   splayed table a directory: ".d", an I64 column of the column-name symbol
 *                 ids, and one column file per column named by its column
 *                 (splay.c:46-176).
 *   symbol file   "TSYM", a u32 count, then per symbol a u32 length and its
 *                 bytes; loading interns them in order (sym.c:314-437).
 *
 * td_gpu_splay_load is the device form: the splayed table is read and its
 * columns are made resident in HBM (td_gpu_pin), each file read straight
 * into its final host block -- large blocks are heap-mapped and page-locked
 * before the upload, so the data crosses PCIe at DMA speed.
 */
#include "internal.h"
#include <dirent.h>
#include <errno.h>
#include <pthread.h>
#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#define TD_SYM_FILE_MAGIC 0x4D595354u            /* "TSYM" */

static int serializable(int8_t t) {
    switch (t) {
        case TD_BOOL: case TD_U8: case TD_CHAR: case TD_I16: case TD_I32: case TD_I64: case TD_F64:
        case TD_DATE: case TD_TIME: case TD_TIMESTAMP: case TD_GUID: case TD_SYM:
            return 1;
        default:
            return 0;
    }
}

static int write_all(int fd, const void* p, size_t n) {
    const char* c = p;
    while (n) {
        ssize_t w = write(fd, c, n);
        if (w < 0) { if (errno == EINTR) continue; return -1; }
        c += w;
        n -= (size_t)w;
    }
    return 0;
}

static int read_at(int fd, void* p, size_t n, off_t off) {
    char* c = p;
    while (n) {
        ssize_t r = pread(fd, c, n, off);
        if (r < 0) { if (errno == EINTR) continue; return -1; }
        if (r == 0) return -1;
        c += r;
        n -= (size_t)r;
        off += r;
    }
    return 0;
}

/* Large column files are read by several threads, each a contiguous range
 * of the file, straight into the column's block: one copy out of the page
 * cache, at the bandwidth of several cores. */
#define STORE_PAR_MIN ((size_t)64 << 20)
#define STORE_PAR_MAX 8

typedef struct { int fd; char* dst; size_t n; off_t off; int bad; } rd_part_t;

static void* rd_part_main(void* a) {
    rd_part_t* r = a;
    r->bad = read_at(r->fd, r->dst, r->n, r->off);
    return NULL;
}

static int read_big(int fd, void* dst, size_t n, off_t off) {
    if (n < STORE_PAR_MIN) return read_at(fd, dst, n, off);
    long cores = sysconf(_SC_NPROCESSORS_ONLN);
    int k = (int)(n / (STORE_PAR_MIN / 2));
    if (k > STORE_PAR_MAX) k = STORE_PAR_MAX;
    if (cores > 0 && k > cores) k = (int)cores;
    if (k < 2) return read_at(fd, dst, n, off);
    rd_part_t parts[STORE_PAR_MAX];
    pthread_t th[STORE_PAR_MAX];
    const size_t step = (n / (size_t)k + 4095) & ~(size_t)4095;
    int started = 0, bad = 0;
    for (int i = 0; i < k; i++) {
        const size_t b = (size_t)i * step;
        if (b >= n) break;
        parts[i] = (rd_part_t){ fd, (char*)dst + b, b + step < n ? step : n - b, off + (off_t)b, 0 };
        if (pthread_create(&th[i], NULL, rd_part_main, &parts[i]) != 0) { parts[i].bad = read_at(fd, parts[i].dst, parts[i].n, parts[i].off); bad |= parts[i].bad; continue; }
        started |= 1 << i;
    }
    for (int i = 0; i < k; i++)
        if (started & (1 << i)) { pthread_join(th[i], NULL); bad |= parts[i].bad; }
    return bad ? -1 : 0;
}

td_err_t td_col_save(td_t* vec, const char* path) {
    if (!vec || TD_IS_ERR(vec)) return TD_ERR_TYPE;
    if (!path) return TD_ERR_IO;
    if (!serializable(vec->type)) return TD_ERR_NYI;
    if (vec->len < 0) return TD_ERR_CORRUPT;
    if ((vec->attrs & TD_ATTR_HAS_NULLS) && (vec->attrs & TD_ATTR_NULLMAP_EXT)) return TD_ERR_NYI;
    const size_t esz = td_sym_elem_size(vec->type, vec->attrs);
    const size_t bytes = (size_t)vec->len * esz;
    td_t h;
    memcpy(&h, vec, 32);
    h.mmod = 0;
    h.order = 0;
    atomic_store_explicit(&h.rc, 0, memory_order_relaxed);
    h.attrs &= (uint8_t)~TD_ATTR_SLICE;
    if (!(h.attrs & TD_ATTR_HAS_NULLS)) memset(h.nullmap, 0, 16);
    const char* data = (vec->attrs & TD_ATTR_SLICE)
        ? (const char*)td_data(vec->slice_parent) + (size_t)vec->slice_offset * esz
        : (const char*)td_data(vec);
    int fd = open(path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (fd < 0) return TD_ERR_IO;
    int bad = write_all(fd, &h, 32) || (bytes && write_all(fd, data, bytes));
    if (close(fd) != 0) bad = 1;
    return bad ? TD_ERR_IO : TD_OK;
}

td_t* td_col_load(const char* path) {
    if (!path) return TD_ERR_PTR(TD_ERR_IO);
    int fd = open(path, O_RDONLY);
    if (fd < 0) return TD_ERR_PTR(TD_ERR_IO);
    struct stat sb;
    td_t h;
    if (fstat(fd, &sb) != 0 || sb.st_size < 32 || read_at(fd, &h, 32, 0)) { close(fd); return TD_ERR_PTR(TD_ERR_CORRUPT); }
    if (!serializable(h.type)) { close(fd); return TD_ERR_PTR(TD_ERR_NYI); }
    if (h.len < 0) { close(fd); return TD_ERR_PTR(TD_ERR_CORRUPT); }
    if ((h.attrs & TD_ATTR_HAS_NULLS) && (h.attrs & TD_ATTR_NULLMAP_EXT)) { close(fd); return TD_ERR_PTR(TD_ERR_NYI); }
    const size_t esz = td_sym_elem_size(h.type, h.attrs);
    if (esz && (uint64_t)h.len > (SIZE_MAX - 32) / esz) { close(fd); return TD_ERR_PTR(TD_ERR_IO); }
    const size_t bytes = (size_t)h.len * esz;
    if ((uint64_t)sb.st_size < 32 + (uint64_t)bytes) { close(fd); return TD_ERR_PTR(TD_ERR_CORRUPT); }
    td_t* v = td_alloc(bytes);
    if (!v || TD_IS_ERR(v)) { close(fd); return v ? v : TD_ERR_PTR(TD_ERR_OOM); }
    const uint8_t order = v->order;
    if (bytes && read_big(fd, td_data(v), bytes, 32)) { close(fd); td_free(v); return TD_ERR_PTR(TD_ERR_IO); }
    close(fd);
    memcpy(v, &h, 32);                            /* the header as saved, then this block's own fields */
    v->mmod = 0;
    v->order = order;
    v->attrs &= (uint8_t)~(TD_ATTR_SLICE | TD_ATTR_NULLMAP_EXT);
    atomic_store_explicit(&v->rc, 1, memory_order_relaxed);
    return v;
}

/* Zero-copy column load (col.c:555-632's td_col_mmap): the file is mapped
 * copy-on-write one page into a reserved range whose first page holds the
 * heap prefix, so the vector is an ordinary heap block whose data are the
 * file's own pages; writing the header (mmod, rc, order) copies only its
 * page.  The file must be exactly the header plus its elements, as
 * td_col_save writes it. */
td_t* td_col_mmap(const char* path) {
    if (!path) return TD_ERR_PTR(TD_ERR_IO);
    int fd = open(path, O_RDONLY);
    if (fd < 0) return TD_ERR_PTR(TD_ERR_IO);
    struct stat sb;
    td_t h;
    if (fstat(fd, &sb) != 0 || sb.st_size < 32 || read_at(fd, &h, 32, 0)) { close(fd); return TD_ERR_PTR(TD_ERR_CORRUPT); }
    if (!serializable(h.type)) { close(fd); return TD_ERR_PTR(TD_ERR_NYI); }
    if (h.len < 0) { close(fd); return TD_ERR_PTR(TD_ERR_CORRUPT); }
    if ((h.attrs & TD_ATTR_HAS_NULLS) && (h.attrs & TD_ATTR_NULLMAP_EXT)) { close(fd); return TD_ERR_PTR(TD_ERR_NYI); }
    const size_t esz = td_sym_elem_size(h.type, h.attrs);
    if (esz && (uint64_t)h.len > (SIZE_MAX - 32 - 8192) / esz) { close(fd); return TD_ERR_PTR(TD_ERR_IO); }
    const size_t bytes = 32 + (size_t)h.len * esz;
    if ((uint64_t)sb.st_size != (uint64_t)bytes) { close(fd); return TD_ERR_PTR(TD_ERR_CORRUPT); }
    const size_t total = 4096 + ((bytes + 4095) & ~(size_t)4095);
    char* base = mmap(NULL, total, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
    if (base == MAP_FAILED) { close(fd); return TD_ERR_PTR(TD_ERR_OOM); }
    if (mmap(base + 4096, bytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_FIXED, fd, 0) == MAP_FAILED) {
        munmap(base, total);
        close(fd);
        return TD_ERR_PTR(TD_ERR_IO);
    }
    close(fd);
    td_t* v = tdb_file_block(base, total);
    v->mmod = 1;
    v->attrs &= (uint8_t)~(TD_ATTR_SLICE | TD_ATTR_NULLMAP_EXT);
    atomic_store_explicit(&v->rc, 1, memory_order_relaxed);
    return v;
}

/* A column name usable as a file name (splay.c:79-85). */
static int plain_name(const char* s, size_t n) {
    return n && s[0] != '.' && !memchr(s, '/', n) && !memchr(s, '\\', n) && !memchr(s, '\0', n);
}

td_err_t td_sym_save(const char* path) {
    if (!path) return TD_ERR_IO;
    FILE* f = fopen(path, "wb");
    if (!f) return TD_ERR_IO;
    const uint32_t magic = TD_SYM_FILE_MAGIC;
    const uint32_t count = td_sym_count();
    int bad = fwrite(&magic, 4, 1, f) != 1 || fwrite(&count, 4, 1, f) != 1;
    for (uint32_t i = 0; i < count && !bad; i++) {
        td_t* s = td_sym_str((int64_t)i);
        const uint32_t len = s ? (uint32_t)td_str_len(s) : 0;
        bad = fwrite(&len, 4, 1, f) != 1 || (len && fwrite(td_str_ptr(s), 1, len, f) != len);
    }
    if (fclose(f) != 0) bad = 1;
    return bad ? TD_ERR_IO : TD_OK;
}

td_err_t td_sym_load(const char* path) {
    if (!path) return TD_ERR_IO;
    FILE* f = fopen(path, "rb");
    if (!f) return TD_ERR_IO;
    uint32_t magic, count;
    if (fread(&magic, 4, 1, f) != 1 || fread(&count, 4, 1, f) != 1 || magic != TD_SYM_FILE_MAGIC ||
        count > 100000000u) {
        fclose(f);
        return TD_ERR_CORRUPT;
    }
    char* buf = NULL;
    size_t cap = 0;
    td_err_t err = TD_OK;
    for (uint32_t i = 0; i < count && !err; i++) {
        uint32_t len;
        if (fread(&len, 4, 1, f) != 1 || len > (16u << 20)) { err = TD_ERR_CORRUPT; break; }
        if (len > cap) {
            char* nb = realloc(buf, len);
            if (!nb) { err = TD_ERR_OOM; break; }
            buf = nb;
            cap = len;
        }
        if (len && fread(buf, 1, len, f) != len) { err = TD_ERR_CORRUPT; break; }
        if (td_sym_intern(len ? buf : "", len) < 0) err = TD_ERR_OOM;
    }
    free(buf);
    fclose(f);
    return err;
}

td_err_t td_splay_save(td_t* tbl, const char* dir, const char* sym_path) {
    if (!tbl || TD_IS_ERR(tbl) || tbl->type != TD_TABLE) return TD_ERR_TYPE;
    if (!dir) return TD_ERR_IO;
    if (sym_path) {
        td_err_t e = td_sym_save(sym_path);
        if (e != TD_OK) return e;
    }
    if (mkdir(dir, 0755) != 0 && errno != EEXIST) return TD_ERR_IO;
    char path[1024];
    td_t* schema = td_table_schema(tbl);
    if (schema && !TD_IS_ERR(schema)) {
        if (snprintf(path, sizeof(path), "%s/.d", dir) >= (int)sizeof(path)) return TD_ERR_RANGE;
        td_err_t e = td_col_save(schema, path);
        if (e != TD_OK) return e;
    }
    for (int64_t j = 0; j < td_table_ncols(tbl); j++) {
        td_t* col = td_table_get_col_idx(tbl, j);
        td_t* name = td_sym_str(td_table_col_name(tbl, j));
        if (!col || !name) continue;
        const char* s = td_str_ptr(name);
        const size_t n = td_str_len(name);
        if (!plain_name(s, n)) continue;
        if (snprintf(path, sizeof(path), "%s/%.*s", dir, (int)n, s) >= (int)sizeof(path)) return TD_ERR_RANGE;
        td_err_t e = td_col_save(col, path);
        if (e != TD_OK) return e;
    }
    return TD_OK;
}

static td_t* splay_read(const char* dir, td_t* (*load)(const char*));

td_t* td_splay_load(const char* dir) { return splay_read(dir, td_col_load); }

/* splay.c's td_read_splayed: the columns mapped rather than read. */
td_t* td_read_splayed(const char* dir, const char* sym_path) {
    if (!dir) return TD_ERR_PTR(TD_ERR_IO);
    if (sym_path) {
        const td_err_t e = td_sym_load(sym_path);
        if (e != TD_OK) return TD_ERR_PTR(e);
    }
    return splay_read(dir, td_col_mmap);
}

static td_t* splay_read(const char* dir, td_t* (*load)(const char*)) {
    if (!dir) return TD_ERR_PTR(TD_ERR_IO);
    char path[1024];
    if (snprintf(path, sizeof(path), "%s/.d", dir) >= (int)sizeof(path)) return TD_ERR_PTR(TD_ERR_RANGE);
    td_t* schema = td_col_load(path);
    if (!schema || TD_IS_ERR(schema)) return schema;
    if (schema->type != TD_I64) { td_release(schema); return TD_ERR_PTR(TD_ERR_CORRUPT); }
    const int64_t nc = schema->len;
    const int64_t* ids = (const int64_t*)td_data(schema);
    td_t* tbl = td_table_new(nc);
    for (int64_t j = 0; j < nc && tbl && !TD_IS_ERR(tbl); j++) {
        td_t* name = td_sym_str(ids[j]);
        if (!name) continue;
        const char* s = td_str_ptr(name);
        const size_t n = td_str_len(name);
        if (!plain_name(s, n)) continue;
        if (snprintf(path, sizeof(path), "%s/%.*s", dir, (int)n, s) >= (int)sizeof(path)) {
            td_release(tbl);
            tbl = TD_ERR_PTR(TD_ERR_RANGE);
            break;
        }
        td_t* col = load(path);
        if (!col || TD_IS_ERR(col)) {
            td_release(tbl);
            tbl = col ? col : TD_ERR_PTR(TD_ERR_IO);
            break;
        }
        td_t* t2 = td_table_add_col(tbl, ids[j], col);
        td_release(col);
        if (!t2 || TD_IS_ERR(t2)) { td_release(tbl); tbl = t2 ? t2 : TD_ERR_PTR(TD_ERR_OOM); break; }
        tbl = t2;
    }
    td_release(schema);
    return tbl ? tbl : TD_ERR_PTR(TD_ERR_OOM);
}

td_t* td_gpu_splay_load(const char* dir) {
    td_t* tbl = td_splay_load(dir);
    if (!tbl || TD_IS_ERR(tbl)) return tbl;
    td_err_t e = td_gpu_pin(tbl);
    if (e != TD_OK) {
        td_release(tbl);
        return TD_ERR_PTR(e);
    }
    return tbl;
}

/* ---- partitioned databases (part.c:111-279) ------------------------------------
 * db_root holds one directory per partition (a name of digits and dots, such as
 * "2024.01.15"), each holding the splayed table `table_name`.  td_part_load
 * loads the partitions in name order and concatenates every column: one
 * allocation per column, each partition copied in once. */

static int part_dir_name(const char* s) {
    int dot = 0;
    for (const char* c = s; *c; c++) {
        if (*c == '.') { dot = 1; continue; }
        if (*c < '0' || *c > '9') return 0;
    }
    return dot;
}

static int cmp_str(const void* a, const void* b) { return strcmp(*(char* const*)a, *(char* const*)b); }

static td_t* concat_cols(td_t** parts, int64_t np) {
    int64_t total = 0;
    int same = 1;
    for (int64_t p = 0; p < np; p++) {
        if (parts[p]->type != parts[0]->type) return TD_ERR_PTR(TD_ERR_TYPE);
        same = same && td_sym_elem_size(parts[p]->type, parts[p]->attrs) ==
                       td_sym_elem_size(parts[0]->type, parts[0]->attrs);
        total += parts[p]->len;
    }
    if (!same) {                                  /* SYM columns of different widths: widen pairwise */
        td_t* acc = parts[0];
        td_retain(acc);
        for (int64_t p = 1; p < np; p++) {
            td_t* n = td_vec_concat(acc, parts[p]);
            td_release(acc);
            if (!n || TD_IS_ERR(n)) return n ? n : TD_ERR_PTR(TD_ERR_OOM);
            acc = n;
        }
        return acc;
    }
    const size_t esz = td_sym_elem_size(parts[0]->type, parts[0]->attrs);
    td_t* v = td_alloc((size_t)total * esz);
    if (!v || TD_IS_ERR(v)) return v ? v : TD_ERR_PTR(TD_ERR_OOM);
    v->type = parts[0]->type;
    v->attrs = parts[0]->attrs & (uint8_t)~(TD_ATTR_SLICE | TD_ATTR_NULLMAP_EXT | TD_ATTR_HAS_NULLS);
    v->len = total;
    char* dst = td_data(v);
    for (int64_t p = 0; p < np; p++) {
        const size_t b = (size_t)parts[p]->len * esz;
        if (b) memcpy(dst, td_data(parts[p]), b);
        dst += b;
    }
    return v;
}

td_t* td_part_load(const char* db_root, const char* table_name) {
    if (!db_root || !table_name) return TD_ERR_PTR(TD_ERR_IO);
    if (strchr(table_name, '/') || strchr(table_name, '\\') || strstr(table_name, "..") || table_name[0] == '.')
        return TD_ERR_PTR(TD_ERR_IO);
    DIR* d = opendir(db_root);
    if (!d) return TD_ERR_PTR(TD_ERR_IO);
    char** names = NULL;
    int64_t np = 0, cap = 0;
    struct dirent* e;
    while ((e = readdir(d))) {
        if (e->d_name[0] == '.' || !part_dir_name(e->d_name)) continue;
        if (np == cap) {
            cap = cap ? cap * 2 : 16;
            char** nn = realloc(names, (size_t)cap * sizeof(char*));
            if (!nn) break;
            names = nn;
        }
        if (!(names[np] = strdup(e->d_name))) break;
        np++;
    }
    closedir(d);
    td_t* res = NULL;
    td_t** tabs = np ? calloc((size_t)np, sizeof(td_t*)) : NULL;
    if (!np) res = TD_ERR_PTR(TD_ERR_IO);
    else if (!tabs) res = TD_ERR_PTR(TD_ERR_OOM);
    else {
        qsort(names, (size_t)np, sizeof(char*), cmp_str);
        char path[1024];
        for (int64_t p = 0; p < np && !res; p++) {
            if (snprintf(path, sizeof(path), "%s/%s/%s", db_root, names[p], table_name) >= (int)sizeof(path)) {
                res = TD_ERR_PTR(TD_ERR_IO);
                break;
            }
            tabs[p] = td_splay_load(path);
            if (!tabs[p] || TD_IS_ERR(tabs[p])) { tabs[p] = NULL; res = TD_ERR_PTR(TD_ERR_IO); }
        }
        if (!res && np == 1) { res = tabs[0]; tabs[0] = NULL; }
        else if (!res) {
            const int64_t nc = td_table_ncols(tabs[0]);
            td_t** cols = malloc((size_t)np * sizeof(td_t*));
            res = cols ? td_table_new(nc) : TD_ERR_PTR(TD_ERR_OOM);
            for (int64_t c = 0; c < nc && res && !TD_IS_ERR(res); c++) {
                int ok = 1;
                for (int64_t p = 0; p < np; p++) {
                    cols[p] = td_table_get_col_idx(tabs[p], c);
                    if (!cols[p]) ok = 0;
                }
                if (!ok) continue;
                td_t* v = concat_cols(cols, np);
                if (!v || TD_IS_ERR(v)) { td_release(res); res = v ? v : TD_ERR_PTR(TD_ERR_OOM); break; }
                td_t* t2 = td_table_add_col(res, td_table_col_name(tabs[0], c), v);
                td_release(v);
                if (!t2 || TD_IS_ERR(t2)) { td_release(res); res = t2 ? t2 : TD_ERR_PTR(TD_ERR_OOM); break; }
                res = t2;
            }
            free(cols);
        }
    }
    for (int64_t p = 0; p < np; p++) {
        if (tabs && tabs[p]) td_release(tabs[p]);
        free(names[p]);
    }
    free(tabs);
    free(names);
    return res ? res : TD_ERR_PTR(TD_ERR_OOM);
}

/* ---- partitioned tables (part.c:284-520) ----------------------------------------- */

static int is_date_dir(const char* s) {
    if (strlen(s) != 10 || s[4] != '.' || s[7] != '.') return 0;
    for (int i = 0; i < 10; i++)
        if (i != 4 && i != 7 && (s[i] < '0' || s[i] > '9')) return 0;
    const int m = (s[5] - '0') * 10 + (s[6] - '0'), d = (s[8] - '0') * 10 + (s[9] - '0');
    return m >= 1 && m <= 12 && d >= 1 && d <= 31;
}

static int is_int_str(const char* s) {
    if (*s == '-') s++;
    if (!*s) return 0;
    for (; *s; s++) if (*s < '0' || *s > '9') return 0;
    return 1;
}

/* Days from 2000-01-01 to y-m-d in the proleptic Gregorian calendar: the
 * count of days in whole 400-year eras (146097 each), then in the years of
 * the era and in the months from March (so the leap day falls last). */
static int32_t days_since_2000(int64_t y, int64_t m, int64_t d) {
    y -= m <= 2;
    const int64_t era = (y >= 0 ? y : y - 399) / 400;
    const int64_t yoe = y - era * 400;
    const int64_t doy = (153 * (m > 2 ? m - 3 : m + 9) + 2) / 5 + d - 1;
    const int64_t doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
    return (int32_t)(era * 146097 + doe - 719468 - 10957);
}

/* Partition directory names of db_root, in name order. */
static int64_t list_parts(const char* db_root, char*** out) {
    *out = NULL;
    DIR* d = opendir(db_root);
    if (!d) return -TD_ERR_IO;
    char** names = NULL;
    int64_t np = 0, cap = 0;
    struct dirent* e;
    while ((e = readdir(d))) {
        if (e->d_name[0] == '.' || !part_dir_name(e->d_name)) continue;
        if (np == cap) {
            cap = cap ? cap * 2 : 16;
            char** nn = realloc(names, (size_t)cap * sizeof(char*));
            if (!nn) break;
            names = nn;
        }
        if (!(names[np] = strdup(e->d_name))) break;
        np++;
    }
    closedir(d);
    if (np) qsort(names, (size_t)np, sizeof(char*), cmp_str);
    *out = names;
    return np;
}

static td_t* ptr_block(int8_t type, int64_t n) {
    td_t* v = td_alloc((size_t)(n ? n : 1) * sizeof(td_t*));
    if (!v) return TD_ERR_PTR(TD_ERR_OOM);
    v->type = type;
    v->len = n;
    memset(td_data(v), 0, (size_t)(n ? n : 1) * sizeof(td_t*));
    return v;
}

td_t* td_read_parted(const char* db_root, const char* table_name) {
    if (!db_root || !table_name) return TD_ERR_PTR(TD_ERR_IO);
    if (strchr(table_name, '/') || strchr(table_name, '\\') || strstr(table_name, "..") || table_name[0] == '.')
        return TD_ERR_PTR(TD_ERR_IO);
    char path[1024];
    if (snprintf(path, sizeof(path), "%s/sym", db_root) >= (int)sizeof(path)) return TD_ERR_PTR(TD_ERR_IO);
    struct stat sb;
    if (stat(path, &sb) == 0) {
        td_err_t e = td_sym_load(path);
        if (e != TD_OK) return TD_ERR_PTR(e);
    }
    char** names = NULL;
    const int64_t np = list_parts(db_root, &names);
    if (np <= 0) { free(names); return TD_ERR_PTR(np < 0 ? (td_err_t)-np : TD_ERR_IO); }
    td_t* res = NULL;
    td_t** tabs = calloc((size_t)np, sizeof(td_t*));
    if (!tabs) res = TD_ERR_PTR(TD_ERR_OOM);
    for (int64_t p = 0; p < np && !res; p++) {
        if (snprintf(path, sizeof(path), "%s/%s/%s", db_root, names[p], table_name) >= (int)sizeof(path)) {
            res = TD_ERR_PTR(TD_ERR_IO);
            break;
        }
        tabs[p] = td_splay_load(path);
        if (!tabs[p] || TD_IS_ERR(tabs[p])) { tabs[p] = NULL; res = TD_ERR_PTR(TD_ERR_IO); }
    }
    if (!res) {
        /* the partition keys: dates, integers or symbols by the directory names */
        int all_date = 1, all_int = 1;
        for (int64_t p = 0; p < np; p++) {
            all_date = all_date && is_date_dir(names[p]);
            all_int = all_int && is_int_str(names[p]);
        }
        const uint8_t mc = all_date ? TD_MC_DATE : all_int ? TD_MC_I64 : TD_MC_SYM;
        td_t* kv = td_vec_new(mc == TD_MC_DATE ? TD_DATE : mc == TD_MC_I64 ? TD_I64 : TD_SYM, np);
        td_t* rc = td_vec_new(TD_I64, np);
        td_t* mcol = ptr_block(TD_MAPCOMMON, 2);
        const int64_t nc = td_table_ncols(tabs[0]);
        res = td_table_new(nc + 2);
        if (!kv || TD_IS_ERR(kv) || !rc || TD_IS_ERR(rc) || TD_IS_ERR(mcol) || !res || TD_IS_ERR(res)) {
            if (kv && !TD_IS_ERR(kv)) td_release(kv);
            if (rc && !TD_IS_ERR(rc)) td_release(rc);
            if (!TD_IS_ERR(mcol)) td_release(mcol);
            if (res && !TD_IS_ERR(res)) td_release(res);
            res = TD_ERR_PTR(TD_ERR_OOM);
        } else {
            for (int64_t p = 0; p < np; p++) {
                const char* nm = names[p];
                if (mc == TD_MC_DATE)
                    ((int32_t*)td_data(kv))[p] = days_since_2000((nm[0] - '0') * 1000 + (nm[1] - '0') * 100 +
                                                                 (nm[2] - '0') * 10 + (nm[3] - '0'),
                                                                 (nm[5] - '0') * 10 + (nm[6] - '0'),
                                                                 (nm[8] - '0') * 10 + (nm[9] - '0'));
                else if (mc == TD_MC_I64)
                    ((int64_t*)td_data(kv))[p] = strtoll(nm, NULL, 10);
                else
                    ((int64_t*)td_data(kv))[p] = td_sym_intern(nm, strlen(nm));
                ((int64_t*)td_data(rc))[p] = td_table_nrows(tabs[p]);
            }
            kv->len = np;
            rc->len = np;
            mcol->attrs = mc;
            ((td_t**)td_data(mcol))[0] = kv;             /* the block owns both */
            ((td_t**)td_data(mcol))[1] = rc;
            const char* mname = mc == TD_MC_DATE ? "date" : "part";
            td_t* t2 = td_table_add_col(res, td_sym_intern(mname, strlen(mname)), mcol);
            td_release(mcol);
            res = t2;
            for (int64_t c = 0; c < nc && res && !TD_IS_ERR(res); c++) {
                td_t* first = td_table_get_col_idx(tabs[0], c);
                if (!first) continue;
                td_t* pc = ptr_block((int8_t)(TD_PARTED_BASE + first->type), np);
                if (TD_IS_ERR(pc)) { td_release(res); res = pc; break; }
                for (int64_t p = 0; p < np; p++) {
                    td_t* seg = td_table_get_col_idx(tabs[p], c);
                    if (seg) td_retain(seg);
                    ((td_t**)td_data(pc))[p] = seg;
                }
                t2 = td_table_add_col(res, td_table_col_name(tabs[0], c), pc);
                td_release(pc);
                res = t2;
            }
        }
    }
    for (int64_t p = 0; p < np; p++) {
        if (tabs && tabs[p]) td_release(tabs[p]);
        free(names[p]);
    }
    free(tabs);
    free(names);
    return res ? res : TD_ERR_PTR(TD_ERR_OOM);
}

td_t* td_gpu_part_load(const char* db_root, const char* table_name) {
    td_t* tbl = td_part_load(db_root, table_name);
    if (!tbl || TD_IS_ERR(tbl)) return tbl;
    td_err_t e = td_gpu_pin(tbl);
    if (e != TD_OK) {
        td_release(tbl);
        return TD_ERR_PTR(e);
    }
    return tbl;
}
