/* gbref_hook.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Builds the unmodified reference gb library (ederc/gb v0.16) from its own
 * sources as a shared object, oracle/_ref/libgbref.so, so that tests and the
 * CPU-baseline leg of bench.py can run the reference's own finite-field linear
 * algebra.  Nothing in the product links or loads this file.
 *
 * The Makefile next to this file compiles it with
 *   -D'linear_algebra(m,b,s)=gbref_hook_linear_algebra(m,b,s)'
 *   -D'interreduce_matrix_rows(m,b,s)=gbref_hook_interreduce(m,b,s)'
 * which re-routes exactly the two call sites src/f4.c:306 and src/f4.c:137 (the
 * function-pointer declarations in src/data.h:269-279 and the assignments in
 * src/io.c:612-750 are not followed by '(' and stay untouched).  The hooks
 * below can
 *   - capture every matrix handed to the linear algebra, with the reference's
 *     answer, into a binary .gbm file (format documented at gbref_write_gbm);
 *   - forward the call to an external implementation with the same signature
 *     (the GPU library's gbgpu_linear_algebra, or the C oracle) instead of the
 *     reference's own function pointer.
 * It also exports flat-CSR entry points that run the reference's own la on a
 * standalone matrix (gbref_la_csr, gbref_interreduce_csr), used to pin the C
 * oracle and as the timed CPU baseline.
 */
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#include <unistd.h>

struct mat_t;
struct bs_t;
struct stat_t;
void gbref_hook_linear_algebra(struct mat_t *mat, const struct bs_t *bs,
                               struct stat_t *st);
void gbref_hook_interreduce(struct mat_t *mat, struct bs_t *bs,
                            const struct stat_t *st);

#include "gb.c" /* the reference's unity build, src/gb.c:27-42 */

typedef void (*gbref_la_fn)(mat_t *, const bs_t *, stat_t *);
typedef void (*gbref_ir_fn)(mat_t *, bs_t *, const stat_t *);

static gbref_la_fn gbref_ext_la = NULL;
static gbref_ir_fn gbref_ext_ir = NULL;
static char gbref_capture_dir[4096];
static int gbref_capture_on = 0;
static int gbref_capture_seq = 0;
static int64_t gbref_la_calls = 0;
static double gbref_la_seconds = 0.0;

/* Route the hooked call sites: ext_la / ext_ir == NULL selects the
 * reference's own function pointers. */
void gbref_set_la(void *ext_la, void *ext_ir)
{
    gbref_ext_la = (gbref_la_fn)ext_la;
    gbref_ext_ir = (gbref_ir_fn)ext_ir;
}

void gbref_set_capture(const char *dir)
{
    if (dir == NULL || dir[0] == '\0') {
        gbref_capture_on = 0;
        return;
    }
    snprintf(gbref_capture_dir, sizeof(gbref_capture_dir), "%s", dir);
    gbref_capture_on = 1;
    gbref_capture_seq = 0;
}

int64_t gbref_hook_calls(void) { return gbref_la_calls; }
double gbref_hook_seconds(void) { return gbref_la_seconds; }

/* Coefficient i of the array at index `idx` of a cf_8/16/32 table. */
static int32_t gbref_cf(void *const *tab, int ff_bits, int32_t idx, int32_t i)
{
    if (ff_bits == 8) {
        return (int32_t)((cf8_t *const *)tab)[idx][i];
    }
    if (ff_bits == 16) {
        return (int32_t)((cf16_t *const *)tab)[idx][i];
    }
    return (int32_t)((cf32_t *const *)tab)[idx][i];
}

static void *const *gbref_bs_table(const bs_t *bs, int ff_bits)
{
    if (ff_bits == 8) return (void *const *)bs->cf_8;
    if (ff_bits == 16) return (void *const *)bs->cf_16;
    return (void *const *)bs->cf_32;
}

static void *const *gbref_mat_table(const mat_t *mat, int ff_bits)
{
    if (ff_bits == 8) return (void *const *)mat->cf_8;
    if (ff_bits == 16) return (void *const *)mat->cf_16;
    return (void *const *)mat->cf_32;
}

/* .gbm layout (little endian):
 *   char[4] "GBM1"; int32 kind (0 linear_algebra, 1 interreduce), p, laopt,
 *   nr, nru, nrl, ncl, ncr; int64 nnz; int64 row_ptr[nr+1]; int32 cols[nnz];
 *   int32 vals[nnz];
 * followed, once the call returned, by the answer:
 *   int32 np; int64 onnz; int64 optr[np+1]; int32 ocols[onnz]; int32 ovals[onnz]
 * Rows are stored in the order of mat->r. */
static void gbref_write_rows(FILE *f, hm_t *const *rows, int32_t nr,
                             void *const *tab, int ff_bits)
{
    int64_t nnz = 0;
    int32_t i, j;
    for (i = 0; i < nr; ++i) nnz += rows[i][2];
    fwrite(&nnz, sizeof(int64_t), 1, f);
    int64_t off = 0;
    fwrite(&off, sizeof(int64_t), 1, f);
    for (i = 0; i < nr; ++i) {
        off += rows[i][2];
        fwrite(&off, sizeof(int64_t), 1, f);
    }
    for (i = 0; i < nr; ++i) {
        fwrite(rows[i] + 3, sizeof(int32_t), (size_t)rows[i][2], f);
    }
    for (i = 0; i < nr; ++i) {
        for (j = 0; j < rows[i][2]; ++j) {
            int32_t v = gbref_cf(tab, ff_bits, rows[i][0], j);
            fwrite(&v, sizeof(int32_t), 1, f);
        }
    }
}

static FILE *gbref_capture_open(void)
{
    char path[4200];
    snprintf(path, sizeof(path), "%s/%04d.gbm", gbref_capture_dir,
             gbref_capture_seq++);
    return fopen(path, "wb");
}

static void gbref_write_header(FILE *f, int32_t kind, const mat_t *mat,
                               int32_t p, int32_t laopt)
{
    int32_t hdr[8] = {kind, p, laopt, mat->nr, mat->nru, mat->nrl, mat->ncl,
                      mat->ncr};
    fwrite("GBM1", 1, 4, f);
    fwrite(hdr, sizeof(int32_t), 8, f);
}

static void gbref_write_answer(FILE *f, const mat_t *mat, int ff_bits)
{
    int32_t np = mat->np;
    fwrite(&np, sizeof(int32_t), 1, f);
    gbref_write_rows(f, mat->r, np, gbref_mat_table(mat, ff_bits), ff_bits);
}

/* Comparison mode: every la call of an F4 run goes to an implementation
 * under test (cmp_la, e.g. the GPU library's gbgpu_linear_algebra; NULL: the
 * reference's own function again) AND, on a deep copy of the matrix, to the
 * reference's own linear_algebra; the two answers are compared row by row
 * (np, lengths, columns, coefficients) and one line per call goes to the log:
 *   call K nr NR nc NC ncl NCL ncr NCR nrl NRL np NP ref_np RNP ref_s T gpu_s T equal E
 * Once the reference calls have taken more than `budget_s` seconds in total
 * the process ends (_exit(0)) right after logging, so that a large F4 run is
 * compared round by round up to a fixed CPU budget. */
static void gbref_free_mat_output(mat_t *mat, int ff_bits, int32_t np);
static int gbref_cmp_on = 0;
static gbref_la_fn gbref_cmp_la = NULL;
static double gbref_cmp_budget = 0.0;
static double gbref_cmp_spent = 0.0;
static int64_t gbref_cmp_calls = 0;
static FILE *gbref_cmp_log = NULL;

int gbref_set_compare(void *cmp_la, double budget_s, const char *log_path)
{
    if (gbref_cmp_log) {
        fclose(gbref_cmp_log);
        gbref_cmp_log = NULL;
    }
    gbref_cmp_on = 0;
    if (log_path == NULL || log_path[0] == '\0') return 0;
    gbref_cmp_log = fopen(log_path, "w");
    if (!gbref_cmp_log) return -1;
    gbref_cmp_la = (gbref_la_fn)cmp_la;
    gbref_cmp_budget = budget_s;
    gbref_cmp_spent = 0.0;
    gbref_cmp_calls = 0;
    gbref_cmp_on = 1;
    return 0;
}

static mat_t *gbref_copy_mat(const mat_t *mat)
{
    int32_t i;
    mat_t *c = (mat_t *)malloc(sizeof(mat_t));
    *c = *mat;
    c->r = (hm_t **)malloc((size_t)(mat->nr > 0 ? mat->nr : 1) * sizeof(hm_t *));
    for (i = 0; i < mat->nr; ++i) {
        const size_t n = (size_t)mat->r[i][2] + 3;
        c->r[i] = (hm_t *)malloc(n * sizeof(hm_t));
        memcpy(c->r[i], mat->r[i], n * sizeof(hm_t));
    }
    c->cf_8 = NULL;
    c->cf_16 = NULL;
    c->cf_32 = NULL;
    c->cf_qq = NULL;
    c->cf_ab_qq = NULL;
    return c;
}

static int gbref_same_answer(const mat_t *a, const mat_t *b, int ff_bits)
{
    int32_t i, j;
    void *const *ta = gbref_mat_table(a, ff_bits);
    void *const *tb = gbref_mat_table(b, ff_bits);
    if (a->np != b->np) return 0;
    for (i = 0; i < a->np; ++i) {
        const hm_t *ra = a->r[i], *rb = b->r[i];
        if (ra[2] != rb[2]) return 0;
        for (j = 0; j < ra[2]; ++j) {
            if (ra[3 + j] != rb[3 + j]) return 0;
            if (gbref_cf(ta, ff_bits, ra[0], j) != gbref_cf(tb, ff_bits, rb[0], j)) return 0;
        }
    }
    return 1;
}

static void gbref_compare_call(mat_t *mat, const bs_t *bs, stat_t *st)
{
    mat_t *ref = gbref_copy_mat(mat);
    stat_t st_ref = *st;
    const int32_t nr = mat->nr, nc = mat->nc, ncl = mat->ncl, ncr = mat->ncr,
                  nrl = mat->nrl;
    double t0 = realtime();
    (linear_algebra)(ref, bs, &st_ref);
    double t1 = realtime();
    if (gbref_cmp_la) {
        gbref_cmp_la(mat, bs, st);
    } else {
        (linear_algebra)(mat, bs, st);
    }
    double t2 = realtime();
    const int eq = gbref_same_answer(mat, ref, st->ff_bits);
    gbref_cmp_spent += t1 - t0;
    fprintf(gbref_cmp_log,
            "call %lld nr %d nc %d ncl %d ncr %d nrl %d np %d ref_np %d ref_s %.6f "
            "gpu_s %.6f equal %d\n",
            (long long)gbref_cmp_calls++, nr, nc, ncl, ncr, nrl, mat->np, ref->np, t1 - t0,
            t2 - t1, eq);
    fflush(gbref_cmp_log);
    gbref_free_mat_output(ref, st->ff_bits, ref->np);
    free(ref);
    if (gbref_cmp_budget > 0.0 && gbref_cmp_spent > gbref_cmp_budget) {
        fprintf(gbref_cmp_log, "stop budget %.3f\n", gbref_cmp_spent);
        fclose(gbref_cmp_log);
        _exit(0);
    }
}

void gbref_hook_linear_algebra(struct mat_t *mat, const struct bs_t *bs,
                               struct stat_t *st)
{
    FILE *f = NULL;
    if (gbref_capture_on) {
        f = gbref_capture_open();
        if (f) {
            gbref_write_header(f, 0, mat, st->fc, st->laopt);
            gbref_write_rows(f, mat->r, mat->nr, gbref_bs_table(bs, st->ff_bits),
                             st->ff_bits);
        }
    }
    double t0 = realtime();
    if (gbref_cmp_on) {
        gbref_compare_call(mat, bs, st);
    } else if (gbref_ext_la) {
        gbref_ext_la(mat, bs, st);
    } else {
        (linear_algebra)(mat, bs, st);
    }
    gbref_la_seconds += realtime() - t0;
    gbref_la_calls++;
    if (f) {
        gbref_write_answer(f, mat, st->ff_bits);
        fclose(f);
    }
}

void gbref_hook_interreduce(struct mat_t *mat, struct bs_t *bs,
                            const struct stat_t *st)
{
    FILE *f = NULL;
    if (gbref_capture_on) {
        f = gbref_capture_open();
        if (f) {
            gbref_write_header(f, 1, mat, st->fc, st->laopt);
            gbref_write_rows(f, mat->r, mat->nr, gbref_bs_table(bs, st->ff_bits),
                             st->ff_bits);
        }
    }
    double t0 = realtime();
    if (gbref_ext_ir) {
        gbref_ext_ir(mat, bs, st);
    } else {
        (interreduce_matrix_rows)(mat, bs, st);
    }
    gbref_la_seconds += realtime() - t0;
    gbref_la_calls++;
    if (f) {
        gbref_write_answer(f, mat, st->ff_bits);
        fclose(f);
    }
}

/* Byte layout of the structs the linear-algebra boundary passes, so the GPU
 * library's mirrored declarations can be checked against the real ones.
 * Writes up to n values and returns how many it knows. */
int gbref_layout(int64_t *out, int n)
{
    int64_t v[] = {
        (int64_t)sizeof(mat_t),
        (int64_t)offsetof(mat_t, r), (int64_t)offsetof(mat_t, cf_8),
        (int64_t)offsetof(mat_t, cf_16), (int64_t)offsetof(mat_t, cf_32),
        (int64_t)offsetof(mat_t, sz), (int64_t)offsetof(mat_t, np),
        (int64_t)offsetof(mat_t, nr), (int64_t)offsetof(mat_t, nc),
        (int64_t)offsetof(mat_t, nru), (int64_t)offsetof(mat_t, nrl),
        (int64_t)offsetof(mat_t, ncl), (int64_t)offsetof(mat_t, ncr),
        (int64_t)sizeof(bs_t),
        (int64_t)offsetof(bs_t, ld), (int64_t)offsetof(bs_t, hm),
        (int64_t)offsetof(bs_t, cf_8), (int64_t)offsetof(bs_t, cf_16),
        (int64_t)offsetof(bs_t, cf_32),
        (int64_t)sizeof(stat_t),
        (int64_t)offsetof(stat_t, la_ctime), (int64_t)offsetof(stat_t, la_rtime),
        (int64_t)offsetof(stat_t, num_zerored), (int64_t)offsetof(stat_t, fc),
        (int64_t)offsetof(stat_t, laopt), (int64_t)offsetof(stat_t, nthrds),
        (int64_t)offsetof(stat_t, ff_bits), (int64_t)offsetof(stat_t, info_level),
        (int64_t)offsetof(stat_t, mo), (int64_t)offsetof(stat_t, num_rowsred),
        (int64_t)offsetof(stat_t, convert_ctime), (int64_t)offsetof(stat_t, convert_rtime),
        (int64_t)sizeof(hd_t), (int64_t)offsetof(hd_t, deg), (int64_t)offsetof(hd_t, idx),
        (int64_t)sizeof(ht_t), (int64_t)offsetof(ht_t, ev), (int64_t)offsetof(ht_t, hd),
        (int64_t)offsetof(ht_t, eld), (int64_t)offsetof(ht_t, nv),
    };
    int k = (int)(sizeof(v) / sizeof(v[0]));
    int i;
    for (i = 0; i < k && i < n; ++i) out[i] = v[i];
    return k;
}

/* ff_bits exactly as src/io.c:815-828 derives it from the prime. */
static int gbref_ff_bits(int32_t p)
{
    if (p < 128) return 8;
    if (p < 32768) return 16;
    return 32;
}

static void *gbref_alloc_cf(int ff_bits, const int32_t *src, int64_t len)
{
    int64_t j;
    if (ff_bits == 8) {
        cf8_t *c = (cf8_t *)malloc((size_t)(len > 0 ? len : 1) * sizeof(cf8_t));
        for (j = 0; j < len; ++j) c[j] = (cf8_t)src[j];
        return c;
    }
    if (ff_bits == 16) {
        cf16_t *c = (cf16_t *)malloc((size_t)(len > 0 ? len : 1) * sizeof(cf16_t));
        for (j = 0; j < len; ++j) c[j] = (cf16_t)src[j];
        return c;
    }
    cf32_t *c = (cf32_t *)malloc((size_t)(len > 0 ? len : 1) * sizeof(cf32_t));
    for (j = 0; j < len; ++j) c[j] = (cf32_t)src[j];
    return c;
}

static void gbref_export_rows(const mat_t *mat, int ff_bits, int32_t np,
                              int64_t **optr, int32_t **ocols, int32_t **ovals)
{
    void *const *tab = gbref_mat_table(mat, ff_bits);
    int64_t nnz = 0;
    int32_t i, j;
    for (i = 0; i < np; ++i) nnz += mat->r[i][2];
    int64_t *ptr = (int64_t *)malloc((size_t)(np + 1) * sizeof(int64_t));
    int32_t *c = (int32_t *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int32_t));
    int32_t *v = (int32_t *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int32_t));
    int64_t off = 0;
    ptr[0] = 0;
    for (i = 0; i < np; ++i) {
        const hm_t *row = mat->r[i];
        for (j = 0; j < row[2]; ++j) {
            c[off + j] = row[3 + j];
            v[off + j] = gbref_cf(tab, ff_bits, row[0], j);
        }
        off += row[2];
        ptr[i + 1] = off;
    }
    *optr = ptr;
    *ocols = c;
    *ovals = v;
}

static void gbref_free_mat_output(mat_t *mat, int ff_bits, int32_t np)
{
    void *const *tab = gbref_mat_table(mat, ff_bits);
    int32_t i;
    for (i = 0; i < np; ++i) {
        if (tab) free(tab[mat->r[i][0]]);
        free(mat->r[i]);
    }
    free(mat->r);
    free(mat->cf_8);
    free(mat->cf_16);
    free(mat->cf_32);
}

/* Run the reference's linear_algebra (la option `laopt`, `nthreads` OpenMP
 * threads) on one Macaulay matrix given as CSR.  Rows must satisfy the mat_t
 * contract of src/data.h:137-155: every lead (first column of a row) is below
 * ncl, the first row of each lead is the known pivot, nrl = nr - ncl.
 * Returns the new pivots in the reference's output order through malloc'ed
 * arrays (release with gbref_free) and the time of the la call alone. */
int gbref_la_csr(int32_t p, int32_t laopt, int32_t nthreads, int32_t nr,
                 int32_t nru, int32_t nrl, int32_t ncl, int32_t ncr,
                 const int64_t *row_ptr, const int32_t *cols, const int32_t *vals,
                 int32_t *out_np, int64_t **optr, int32_t **ocols,
                 int32_t **ovals, double *seconds)
{
    int32_t i;
    const int ff_bits = gbref_ff_bits(p);
    stat_t *st = (stat_t *)calloc(1, sizeof(stat_t));
    bs_t *bs = (bs_t *)calloc(1, sizeof(bs_t));
    mat_t *mat = (mat_t *)calloc(1, sizeof(mat_t));
    void **tab = (void **)calloc((size_t)(nr > 0 ? nr : 1), sizeof(void *));

    st->fc = p;
    st->ff_bits = ff_bits;
    st->laopt = laopt;
    st->nthrds = nthreads > 0 ? nthreads : 1;
    st->info_level = 0;
    st->mo = 0;
    set_function_pointers(st);

    if (ff_bits == 8) bs->cf_8 = (cf8_t **)tab;
    else if (ff_bits == 16) bs->cf_16 = (cf16_t **)tab;
    else bs->cf_32 = (cf32_t **)tab;

    mat->r = (hm_t **)malloc((size_t)(nr > 0 ? nr : 1) * sizeof(hm_t *));
    for (i = 0; i < nr; ++i) {
        const int64_t len = row_ptr[i + 1] - row_ptr[i];
        hm_t *row = (hm_t *)malloc((size_t)(len + 3) * sizeof(hm_t));
        row[0] = i;
        row[1] = (hm_t)(len % UNROLL);
        row[2] = (hm_t)len;
        memcpy(row + 3, cols + row_ptr[i], (size_t)len * sizeof(int32_t));
        mat->r[i] = row;
        tab[i] = gbref_alloc_cf(ff_bits, vals + row_ptr[i], len);
    }
    mat->nr = nr;
    mat->sz = nr;
    mat->nru = nru;
    mat->nrl = nrl;
    mat->ncl = ncl;
    mat->ncr = ncr;
    mat->nc = ncl + ncr;

    double t0 = realtime();
    (linear_algebra)(mat, bs, st);
    double t1 = realtime();
    if (seconds) *seconds = t1 - t0;

    *out_np = mat->np;
    gbref_export_rows(mat, ff_bits, mat->np, optr, ocols, ovals);
    gbref_free_mat_output(mat, ff_bits, mat->np);
    for (i = 0; i < nr; ++i) free(tab[i]);
    free(tab);
    free(bs);
    free(mat);
    free(st);
    return 0;
}

/* Run the reference's interreduce_matrix_rows (src/la_ff_16.c:1605-1673 and
 * its 8/32-bit twins) on nr rows with pairwise distinct leads over nc
 * columns.  Output rows come in the reference's order (ascending lead). */
int gbref_interreduce_csr(int32_t p, int32_t nr, int32_t nc,
                          const int64_t *row_ptr, const int32_t *cols,
                          const int32_t *vals, int64_t **optr, int32_t **ocols,
                          int32_t **ovals, double *seconds)
{
    int32_t i;
    const int ff_bits = gbref_ff_bits(p);
    stat_t *st = (stat_t *)calloc(1, sizeof(stat_t));
    bs_t *bs = (bs_t *)calloc(1, sizeof(bs_t));
    mat_t *mat = (mat_t *)calloc(1, sizeof(mat_t));
    void **tab = (void **)calloc((size_t)(nr > 0 ? nr : 1), sizeof(void *));

    st->fc = p;
    st->ff_bits = ff_bits;
    st->laopt = 2;
    st->nthrds = 1;
    st->info_level = 0;
    set_function_pointers(st);

    if (ff_bits == 8) bs->cf_8 = (cf8_t **)tab;
    else if (ff_bits == 16) bs->cf_16 = (cf16_t **)tab;
    else bs->cf_32 = (cf32_t **)tab;
    bs->hm = (hm_t **)calloc((size_t)(nr > 0 ? nr : 1), sizeof(hm_t *));
    bs->ld = nr;

    mat->r = (hm_t **)malloc((size_t)(nr > 0 ? nr : 1) * sizeof(hm_t *));
    for (i = 0; i < nr; ++i) {
        const int64_t len = row_ptr[i + 1] - row_ptr[i];
        hm_t *row = (hm_t *)malloc((size_t)(len + 3) * sizeof(hm_t));
        row[0] = i;
        row[1] = (hm_t)(len % UNROLL);
        row[2] = (hm_t)len;
        memcpy(row + 3, cols + row_ptr[i], (size_t)len * sizeof(int32_t));
        mat->r[i] = row;
        tab[i] = gbref_alloc_cf(ff_bits, vals + row_ptr[i], len);
        bs->hm[i] = (hm_t *)malloc(sizeof(hm_t));
    }
    mat->nr = nr;
    mat->sz = nr;
    mat->nru = 0;
    mat->nrl = nr;
    mat->ncl = 0;
    mat->ncr = nc;
    mat->nc = nc;

    double t0 = realtime();
    (interreduce_matrix_rows)(mat, bs, st);
    double t1 = realtime();
    if (seconds) *seconds = t1 - t0;

    gbref_export_rows(mat, ff_bits, mat->np, optr, ocols, ovals);
    gbref_free_mat_output(mat, ff_bits, mat->np);
    free(tab);      /* entries were released by free_basis_elements */
    free(bs->hm);
    free(bs);
    free(mat);
    free(st);
    return 0;
}

void gbref_free(void *ptr) { free(ptr); }

/* The reference's convert_hashes_to_columns (src/convert.c:30-135) followed
 * by sort_matrix_rows (src/order.c:125-131) on a flat description of one F4
 * round: the secondary hash table's monomials 1..n (exponents exps[n][nv],
 * total degrees deg[n], idx[n] = 2 for the lead monomials of known pivots,
 * 1 otherwise) and nr rows of hash indices (row_ptr, hashes; the first entry
 * of a row is its lead term).  Outputs: hcm[n] (the hash of every column, in
 * column order), *ncl, row_order[nr] (input row of every row after the sort)
 * and out_cols (the rows' column indices, rows in the sorted order, entries
 * in their input order).  mo: 0 DRL, 1 LEX. */
int gbref_convert_csr(int32_t nv, int32_t n, const int16_t *exps, const int32_t *deg,
                      const int32_t *idx, int32_t mo, int32_t nr, const int64_t *row_ptr,
                      const int32_t *hashes, int32_t *hcm_out, int32_t *ncl_out,
                      int32_t *row_order, int32_t *out_cols, double *seconds)
{
    int32_t i, j;
    stat_t *st = (stat_t *)calloc(1, sizeof(stat_t));
    st->mo = mo;
    st->nthrds = 1;
    st->fc = 65521;
    st->ff_bits = 32;
    st->laopt = 2;
    set_function_pointers(st);
    ht_t *sht = (ht_t *)calloc(1, sizeof(ht_t));
    sht->nv = nv;
    sht->eld = n + 1;
    sht->esz = n + 1;
    sht->hd = (hd_t *)calloc((size_t)n + 1, sizeof(hd_t));
    sht->ev = (exp_t **)calloc((size_t)n + 1, sizeof(exp_t *));
    exp_t *block = (exp_t *)calloc((size_t)(n + 1) * (size_t)(nv > 0 ? nv : 1), sizeof(exp_t));
    for (i = 0; i <= n; ++i) sht->ev[i] = block + (size_t)i * nv;
    for (i = 0; i < n; ++i) {
        for (j = 0; j < nv; ++j) sht->ev[i + 1][j] = exps[(size_t)i * nv + j];
        sht->hd[i + 1].deg = deg[i];
        sht->hd[i + 1].idx = idx[i];
    }
    mat_t *mat = (mat_t *)calloc(1, sizeof(mat_t));
    mat->r = (hm_t **)malloc((size_t)(nr > 0 ? nr : 1) * sizeof(hm_t *));
    for (i = 0; i < nr; ++i) {
        const int64_t len = row_ptr[i + 1] - row_ptr[i];
        hm_t *row = (hm_t *)malloc((size_t)(len + 3) * sizeof(hm_t));
        row[0] = i; /* tags the input row through the sort */
        row[1] = (hm_t)(len % UNROLL);
        row[2] = (hm_t)len;
        memcpy(row + 3, hashes + row_ptr[i], (size_t)len * sizeof(int32_t));
        mat->r[i] = row;
    }
    mat->nr = nr;
    mat->sz = nr;
    mat->nc = n;
    hl_t *hcm = NULL;
    double t0 = realtime();
    convert_hashes_to_columns(&hcm, mat, st, sht);
    sort_matrix_rows(mat);
    double t1 = realtime();
    if (seconds) *seconds = t1 - t0;
    for (i = 0; i < n; ++i) hcm_out[i] = hcm[i];
    *ncl_out = mat->ncl;
    int64_t off = 0;
    for (i = 0; i < nr; ++i) {
        const hm_t *row = mat->r[i];
        row_order[i] = row[0];
        memcpy(out_cols + off, row + 3, (size_t)row[2] * sizeof(int32_t));
        off += row[2];
        free(mat->r[i]);
    }
    free(mat->r);
    free(mat);
    free(hcm);
    free(block);
    free(sht->ev);
    free(sht->hd);
    free(sht);
    free(st);
    return 0;
}

/* ---- the step after the linear algebra, timed and digested --------------
 * One matrix through the la and then convert_sparse_matrix_rows_to_basis_
 * elements (src/f4.c:306-311, src/convert.c:137-280) with a fresh basis and a
 * fresh basis hash table: the reference's own functions, or ext_keep /
 * ext_convert (gbgpu_linear_algebra_keep and
 * gbgpu_convert_sparse_matrix_rows_to_basis_elements) when given.  The nc
 * column monomials (exps, nc x nv, distinct) go into a secondary table in
 * column order; hcm maps columns to them.  Returns the conversion's seconds,
 * the new elements' count, bht->eld, a digest of the new basis elements
 * (every entry's table index, its monomial's exponents and its coefficient,
 * FNV-1a) and a digest of the table's hash map (every occupied slot). */
typedef void (*gbref_conv_fn)(mat_t *, bs_t *, ht_t *, const ht_t *, const hl_t *, stat_t *);

static uint64_t gbref_fnv(uint64_t h, uint64_t v)
{
    for (int b = 0; b < 8; ++b) {
        h ^= (v >> (8 * b)) & 0xFFu;
        h *= 1099511628211ull;
    }
    return h;
}

int gbref_basis_bench(int32_t p, int32_t nv, int32_t nthreads, int32_t nr, int32_t nru,
                      int32_t nrl, int32_t ncl, int32_t ncr, const int64_t *row_ptr,
                      const int32_t *cols, const int32_t *vals, const int16_t *exps,
                      void *ext_keep, void *ext_convert, double *seconds, int32_t *out_np,
                      int32_t *out_eld, uint64_t *digest, uint64_t *map_digest)
{
    int32_t i;
    const int32_t nc = ncl + ncr;
    const int ff_bits = gbref_ff_bits(p);
    stat_t *st = (stat_t *)calloc(1, sizeof(stat_t));
    bs_t *bs = (bs_t *)calloc(1, sizeof(bs_t));
    mat_t *mat = (mat_t *)calloc(1, sizeof(mat_t));
    void **tab = (void **)calloc((size_t)(nr > 0 ? nr : 1), sizeof(void *));
    void **inputs = (void **)calloc((size_t)(nr > 0 ? nr : 1), sizeof(void *));
    int hts = 17;
    while ((1 << (hts - 6)) < nc + 2) ++hts;

    st->fc = p;
    st->ff_bits = ff_bits;
    st->laopt = 1;
    st->nthrds = nthreads > 0 ? nthreads : 1;
    st->info_level = 0;
    st->mo = 0;
    st->nvars = nv;
    st->init_hts = hts;
    set_function_pointers(st);

    ht_t *bht = initialize_basis_hash_table(st);
    ht_t *sht = initialize_secondary_hash_table(bht, st);
    hl_t *hcm = (hl_t *)malloc((size_t)(nc > 0 ? nc : 1) * sizeof(hl_t));
    for (i = 0; i < nc; ++i) hcm[i] = insert_in_hash_table(exps + (size_t)i * nv, sht);

    if (ff_bits == 8) bs->cf_8 = (cf8_t **)tab;
    else if (ff_bits == 16) bs->cf_16 = (cf16_t **)tab;
    else bs->cf_32 = (cf32_t **)tab;
    mat->r = (hm_t **)malloc((size_t)(nr > 0 ? nr : 1) * sizeof(hm_t *));
    for (i = 0; i < nr; ++i) {
        const int64_t len = row_ptr[i + 1] - row_ptr[i];
        hm_t *row = (hm_t *)malloc((size_t)(len + 3) * sizeof(hm_t));
        row[0] = i;
        row[1] = (hm_t)(len % UNROLL);
        row[2] = (hm_t)len;
        memcpy(row + 3, cols + row_ptr[i], (size_t)len * sizeof(int32_t));
        mat->r[i] = row;
        tab[i] = gbref_alloc_cf(ff_bits, vals + row_ptr[i], len);
        inputs[i] = tab[i];
    }
    mat->nr = nr;
    mat->sz = nr;
    mat->nru = nru;
    mat->nrl = nrl;
    mat->ncl = ncl;
    mat->ncr = ncr;
    mat->nc = nc;

    if (ext_keep) ((gbref_la_fn)ext_keep)(mat, bs, st);
    else (linear_algebra)(mat, bs, st);
    /* the basis' coefficient table is the input table until it grows */
    const int32_t np = mat->np;
    double t0 = realtime();
    if (np > 0) {
        if (ext_convert) ((gbref_conv_fn)ext_convert)(mat, bs, bht, sht, hcm, st);
        else convert_sparse_matrix_rows_to_basis_elements(mat, bs, bht, sht, hcm, st);
    }
    double t1 = realtime();
    if (seconds) *seconds = t1 - t0;

    uint64_t h = 1469598103934665603ull;
    void *const *btab = gbref_bs_table(bs, ff_bits);
    for (i = 0; i < np; ++i) {
        const hm_t *row = bs->hm[bs->ld + i];
        h = gbref_fnv(h, (uint64_t)row[2]);
        for (int32_t l = 0; l < row[2]; ++l) {
            const hl_t ix = row[3 + l];
            h = gbref_fnv(h, (uint64_t)(uint32_t)ix);
            for (int32_t v = 0; v < nv; ++v) h = gbref_fnv(h, (uint64_t)(uint16_t)bht->ev[ix][v]);
            h = gbref_fnv(h, (uint64_t)(uint32_t)gbref_cf(btab, ff_bits, row[0], l));
        }
    }
    uint64_t hm = 1469598103934665603ull;
    for (hl_t k = 0; k < bht->hsz; ++k)
        if (bht->hmap[k]) {
            hm = gbref_fnv(hm, (uint64_t)(uint32_t)k);
            hm = gbref_fnv(hm, (uint64_t)(uint32_t)bht->hmap[k]);
        }
    *out_np = np;
    *out_eld = bht->eld;
    *digest = h;
    *map_digest = hm;

    for (i = 0; i < np; ++i) {
        free(bs->hm[bs->ld + i]);
        free(((void **)btab)[bs->ld + i]);
    }
    for (i = 0; i < nr; ++i)
        if (i >= np || inputs[i] != ((void **)btab)[i]) free(inputs[i]);
    free(inputs);
    free((void *)btab);
    free(bs->hm);
    free(bs->lm);
    free(bs->lmps);
    free(bs->red);
    free(bs);
    free(mat->r);
    free(mat->cf_8);
    free(mat->cf_16);
    free(mat->cf_32);
    free(mat);
    free(hcm);
    free(sht->ev[0]);
    free(sht->ev);
    free(sht->hd);
    free(sht->hmap);
    free(sht);
    free(bht->ev[0]);
    free(bht->ev);
    free(bht->hd);
    free(bht->hmap);
    free(bht->dm);
    free(bht->rn);
    free(bht);
    free(st);
    return 0;
}
