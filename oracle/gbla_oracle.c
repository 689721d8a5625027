/* gbla_oracle.c -- TEST INFRASTRUCTURE ONLY: the CPU oracle.
 *
 * A plain-C, single-threaded restatement of the reference's exact finite-field
 * linear algebra (ederc/gb v0.16, src/la_ff_8.c, src/la_ff_16.c,
 * src/la_ff_32.c).  It is the checker the GPU library is compared against; it
 * is never linked into, loaded by, or called from the product.
 *
 * Pinning: tests/test_oracle.py checks this code against
 *   - every matrix the reference's own F4 golden tests (test/<name>.c) hand
 *     to the linear algebra, captured together with the reference's answer
 *     (tests/golden/mats/<name>.npz, made by tests/golden/make_golden.py),
 *   - the reference compiled from its own sources (oracle/_ref/libgbref.so) on
 *     seeded synthetic matrices, and
 *   - the known-answer test of test/normalize_row.c.
 *
 * Input format (flat CSR): nr rows over nc = ncl + ncr columns, row i holds
 * cols[row_ptr[i] .. row_ptr[i+1]) with residues vals[...] in [0, p).  The
 * first entry of a row is its lead (smallest column); the remaining entries
 * may come in any order (src/convert.c:111-120).  Output rows are CSR with
 * ascending columns and lead coefficient 1.
 *
 * Arithmetic follows the two kernel families of the reference:
 *   p <  2^17: lazy accumulation  dr[c] += (p - m) * cf   (la_ff_32.c:100-189,
 *              la_ff_16.c:102-190: the 8/16-bit files compute the same sums)
 *   p >= 2^17: bounded form  dr[c] -= m * cf; if (dr[c] < 0) dr[c] += p^2
 *              (la_ff_32.c:191-288)
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "gbla_oracle.h"

/* ---------------------------------------------------------------------- */
/* Modular inverse by the extended Euclidean algorithm (src/tools.c:83-110). */
int32_t oracle_inverse(int32_t val, int32_t p)
{
    int64_t a = p, b = val % p, c = 1, d = 0, e, f;
    if (b < 0) b += p;
    while (b != 0) {
        f = b;
        e = a / f;
        b = a - e * f;
        a = f;
        f = c;
        c = d - e * f;
        d = f;
    }
    if (d < 0) d += p;
    return (int32_t)d;
}

/* Multiply row[0..len) by row[0]^-1 mod p and set row[0] = 1
 * (normalize_dense_matrix_row_ff_32, src/la_ff_32.c:24-59).  Entries may be
 * unreduced non-negative integers, as in test/normalize_row.c. */
void oracle_normalize_row(int32_t *row, int64_t len, int32_t p)
{
    int64_t i;
    if (len <= 0) return;
    const int64_t inv = oracle_inverse(row[0], p);
    for (i = 1; i < len; ++i) {
        int64_t t = ((int64_t)row[i] * inv) % p;
        if (t < 0) t += p;
        row[i] = (int32_t)t;
    }
    row[0] = 1;
}

/* ---------------------------------------------------------------------- */
/* Sparse rows as the reference keeps them: column list + coefficient list. */
typedef struct {
    int64_t len;
    int32_t *cols;
    int32_t *cfs;
} orow_t;

typedef struct {
    int64_t p;
    int64_t p2;
    int lazy; /* p < 2^17: lazy-add family */
    int32_t ncl;     /* pivots of columns below ncl are the known ones */
    int64_t work[2]; /* entries applied: [0] known pivots, [1] new pivots */
} ofield_t;

static void ofield_init(ofield_t *f, int32_t p)
{
    f->p = p;
    f->p2 = (int64_t)p * p;
    f->lazy = p < (1 << 17);
    f->ncl = 0;
    f->work[0] = f->work[1] = 0;
}

/* dr[c] += mul * cf, with mul the multiplier that cancels a residue `m`. */
static inline void oaxpy(const ofield_t *f, int64_t *dr, int32_t c, int64_t m,
                         int64_t cf)
{
    if (f->lazy) {
        dr[c] += (f->p - m) * cf;
    } else {
        dr[c] -= m * cf;
        if (dr[c] < 0) dr[c] += f->p2;
    }
}

static inline int64_t ored(const ofield_t *f, int64_t v)
{
    return v % f->p;
}

/* Load a sparse row into a zeroed dense int64 row. */
static void oscatter(int64_t *dr, const orow_t *r)
{
    int64_t j;
    for (j = 0; j < r->len; ++j) dr[r->cols[j]] = r->cfs[j];
}

/* Reduce the dense row dr over columns [dpiv, ncols) by the pivot table pivs
 * (known pivots below ncl, new pivots at or above).  Returns the remaining
 * row restricted to columns >= emit_from, unnormalised, or len == 0 when the
 * row reduced to zero in all columns (reduce_dense_row_by_known_pivots_sparse,
 * src/la_ff_16.c:102-190, src/la_ff_32.c:100-288). */
static orow_t oreduce_sparse(ofield_t *f, int64_t *dr, orow_t *const *pivs,
                             int32_t dpiv, int32_t ncols, int32_t emit_from)
{
    orow_t out = {0, NULL, NULL};
    int32_t i;
    int64_t j, k = 0;
    for (i = dpiv; i < ncols; ++i) {
        if (dr[i] != 0) dr[i] = ored(f, dr[i]);
        if (dr[i] == 0) continue;
        if (pivs[i] == NULL) {
            k++;
            continue;
        }
        const orow_t *pr = pivs[i];
        const int64_t m = dr[i];
        for (j = 0; j < pr->len; ++j) oaxpy(f, dr, pr->cols[j], m, pr->cfs[j]);
        f->work[i < f->ncl ? 0 : 1] += pr->len;
        dr[i] = 0;
    }
    if (k == 0) return out;
    out.cols = (int32_t *)malloc((size_t)(ncols - emit_from + 1) * sizeof(int32_t));
    out.cfs = (int32_t *)malloc((size_t)(ncols - emit_from + 1) * sizeof(int32_t));
    for (i = emit_from; i < ncols; ++i) {
        if (dr[i] != 0) {
            dr[i] = ored(f, dr[i]);
            if (dr[i] != 0) {
                out.cols[out.len] = i;
                out.cfs[out.len] = (int32_t)dr[i];
                out.len++;
            }
        }
    }
    if (out.len == 0) {
        free(out.cols);
        free(out.cfs);
        out.cols = out.cfs = NULL;
    }
    return out;
}

static orow_t *orow_box(orow_t r)
{
    orow_t *b = (orow_t *)malloc(sizeof(orow_t));
    *b = r;
    return b;
}

static void orow_free(orow_t *r)
{
    if (!r) return;
    free(r->cols);
    free(r->cfs);
    free(r);
}

/* Collect output rows into malloc'ed CSR arrays. */
static void oexport(orow_t *const *rows, int32_t n, int64_t **optr,
                    int32_t **ocols, int32_t **ovals)
{
    int64_t nnz = 0, off = 0;
    int32_t i;
    for (i = 0; i < n; ++i) nnz += rows[i]->len;
    int64_t *ptr = (int64_t *)malloc((size_t)(n + 1) * sizeof(int64_t));
    int32_t *c = (int32_t *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int32_t));
    int32_t *v = (int32_t *)malloc((size_t)(nnz > 0 ? nnz : 1) * sizeof(int32_t));
    ptr[0] = 0;
    for (i = 0; i < n; ++i) {
        memcpy(c + off, rows[i]->cols, (size_t)rows[i]->len * sizeof(int32_t));
        memcpy(v + off, rows[i]->cfs, (size_t)rows[i]->len * sizeof(int32_t));
        off += rows[i]->len;
        ptr[i + 1] = off;
    }
    *optr = ptr;
    *ocols = c;
    *ovals = v;
}

/* Split the input rows into the known pivot per lead (the first row with
 * that lead, src/la_ff_16.c:630-639) and the rows still to reduce. */
static int osplit(int32_t p, int32_t nr, int32_t ncols, int32_t lead_bound,
                  const int64_t *row_ptr, const int32_t *cols,
                  const int32_t *vals, orow_t **pivs, orow_t **upivs,
                  int32_t *nup)
{
    int32_t i, n = 0;
    int64_t j;
    for (i = 0; i < nr; ++i) {
        orow_t r;
        r.len = row_ptr[i + 1] - row_ptr[i];
        if (r.len <= 0) {
            *nup = n;
            return ORACLE_EINVAL;
        }
        r.cols = (int32_t *)malloc((size_t)r.len * sizeof(int32_t));
        r.cfs = (int32_t *)malloc((size_t)r.len * sizeof(int32_t));
        memcpy(r.cols, cols + row_ptr[i], (size_t)r.len * sizeof(int32_t));
        memcpy(r.cfs, vals + row_ptr[i], (size_t)r.len * sizeof(int32_t));
        const int32_t lead = r.cols[0];
        int bad = lead < 0 || lead >= lead_bound;
        for (j = 1; j < r.len; ++j) {
            bad |= r.cols[j] <= lead || r.cols[j] >= ncols;
        }
        for (j = 0; j < r.len; ++j) bad |= r.cfs[j] <= 0 || r.cfs[j] >= p;
        bad |= r.cfs[0] != 1; /* F4 rows are monic (src/basis.c:252) */
        if (bad) {
            free(r.cols);
            free(r.cfs);
            *nup = n;
            return ORACLE_EINVAL;
        }
        if (pivs[lead] == NULL) {
            pivs[lead] = orow_box(r);
        } else {
            upivs[n++] = orow_box(r);
        }
    }
    *nup = n;
    /* every column left of lead_bound needs its known pivot: the reference
     * silently drops such a column otherwise, which no F4 matrix produces */
    for (i = 0; i < lead_bound; ++i) {
        if (pivs[i] == NULL && lead_bound < ncols) return ORACLE_EINVAL;
    }
    return 0;
}

/* ---------------------------------------------------------------------- */
/* la option 2: exact_sparse_reduced_echelon_form (src/la_ff_16.c:601-735,
 * src/la_ff_32.c:945-1079) run with one thread. */
static int oracle_sparse_echelon(ofield_t *f, int32_t nr, int32_t ncl,
                                 int32_t ncr, const int64_t *row_ptr,
                                 const int32_t *cols, const int32_t *vals,
                                 int32_t *out_np, int64_t **optr,
                                 int32_t **ocols, int32_t **ovals)
{
    const int32_t ncols = ncl + ncr;
    int32_t i, nup = 0, np = 0;
    orow_t **pivs = (orow_t **)calloc((size_t)ncols + 1, sizeof(orow_t *));
    orow_t **upivs = (orow_t **)calloc((size_t)nr + 1, sizeof(orow_t *));
    int64_t *dr = (int64_t *)malloc((size_t)(ncols + 1) * sizeof(int64_t));
    int rc = osplit((int32_t)f->p, nr, ncols, ncl, row_ptr, cols, vals, pivs,
                    upivs, &nup);
    if (rc) goto done;

    /* reduce each remaining row by all pivots known so far; a surviving row
     * is normalised and becomes the pivot of its lead */
    for (i = 0; i < nup; ++i) {
        memset(dr, 0, (size_t)ncols * sizeof(int64_t));
        oscatter(dr, upivs[i]);
        orow_t r = oreduce_sparse(f, dr, pivs, upivs[i]->cols[0], ncols, ncl);
        if (r.len == 0) continue;
        oracle_normalize_row(r.cfs, r.len, (int32_t)f->p);
        pivs[r.cols[0]] = orow_box(r);
    }
    /* known pivots are not needed any more (src/la_ff_16.c:688-691) */
    for (i = 0; i < ncl; ++i) {
        orow_free(pivs[i]);
        pivs[i] = NULL;
    }
    /* interreduce the new pivots from the last column down
     * (src/la_ff_16.c:702-727) */
    orow_t **rows = (orow_t **)calloc((size_t)ncr + 1, sizeof(orow_t *));
    for (i = ncols - 1; i >= ncl; --i) {
        if (pivs[i] == NULL) continue;
        memset(dr, 0, (size_t)ncols * sizeof(int64_t));
        oscatter(dr, pivs[i]);
        orow_free(pivs[i]);
        pivs[i] = NULL;
        orow_t r = oreduce_sparse(f, dr, pivs, i, ncols, ncl);
        pivs[i] = rows[np++] = orow_box(r);
    }
    *out_np = np;
    oexport(rows, np, optr, ocols, ovals);
    for (i = 0; i < np; ++i) orow_free(rows[i]);
    free(rows);
done:
    for (i = 0; i < nup; ++i) orow_free(upivs[i]);
    if (rc) {
        for (i = 0; i < ncols; ++i) orow_free(pivs[i]);
    }
    free(upivs);
    free(pivs);
    free(dr);
    return rc;
}

/* ---------------------------------------------------------------------- */
/* la option 1: sparse A|B / C|D step, dense echelon of D, dense
 * interreduction, conversion back to sparse rows
 * (exact_sparse_dense_linear_algebra_ff_16, src/la_ff_16.c:1460-1507). */

/* Dense row stored from its first column `start` to ncr-1. */
typedef struct {
    int32_t start;
    int32_t *v; /* length ncr - start */
} odrow_t;

/* reduce_dense_row_by_dense_new_pivots (src/la_ff_16.c:353-409,
 * src/la_ff_32.c:632-748): reduce dr[pc..ncr) by the dense pivots nps; return
 * the normalised remainder starting at its lead, or v == NULL if zero. */
static odrow_t oreduce_dense(ofield_t *f, int64_t *dr, int32_t pc,
                             odrow_t *const *nps, int32_t ncr)
{
    odrow_t out = {-1, NULL};
    int32_t i, j, np = -1;
    for (i = pc; i < ncr; ++i) {
        if (dr[i] != 0) dr[i] = ored(f, dr[i]);
        if (dr[i] == 0) continue;
        if (nps[i] == NULL) {
            if (np == -1) np = i;
            continue;
        }
        const int64_t m = dr[i];
        const int32_t *pv = nps[i]->v;
        for (j = i; j < ncr; ++j) oaxpy(f, dr, j, m, pv[j - i]);
        f->work[1] += ncr - i;
    }
    if (np == -1) return out;
    out.start = np;
    out.v = (int32_t *)malloc((size_t)(ncr - np) * sizeof(int32_t));
    for (i = np; i < ncr; ++i) {
        if (dr[i] != 0) dr[i] = ored(f, dr[i]);
        out.v[i - np] = (int32_t)dr[i];
    }
    if (out.v[0] != 1) oracle_normalize_row(out.v, ncr - np, (int32_t)f->p);
    return out;
}

static int oracle_sparse_dense(ofield_t *f, int32_t nr, int32_t ncl,
                               int32_t ncr, const int64_t *row_ptr,
                               const int32_t *cols, const int32_t *vals,
                               int32_t *out_np, int64_t **optr,
                               int32_t **ocols, int32_t **ovals)
{
    const int32_t ncols = ncl + ncr;
    int32_t i, j, nup = 0, nd = 0, np = 0;
    orow_t **pivs = (orow_t **)calloc((size_t)ncols + 1, sizeof(orow_t *));
    orow_t **upivs = (orow_t **)calloc((size_t)nr + 1, sizeof(orow_t *));
    int64_t *dr = (int64_t *)malloc((size_t)(ncols + 1) * sizeof(int64_t));
    int32_t **dm = NULL;
    odrow_t **nps = NULL;
    int rc = osplit((int32_t)f->p, nr, ncols, ncl, row_ptr, cols, vals, pivs,
                    upivs, &nup);
    if (rc) goto done;

    /* sparse_AB_CD_linear_algebra (src/la_ff_16.c:737-835): reduce each C|D
     * row by the known A|B pivots on columns [lead, ncl) and keep the dense D
     * part (reduce_dense_row_by_old_pivots, src/la_ff_16.c:289-351) */
    dm = (int32_t **)calloc((size_t)nup + 1, sizeof(int32_t *));
    for (i = 0; i < nup; ++i) {
        memset(dr, 0, (size_t)ncols * sizeof(int64_t));
        oscatter(dr, upivs[i]);
        int32_t c;
        for (c = upivs[i]->cols[0]; c < ncl; ++c) {
            if (dr[c] != 0) dr[c] = ored(f, dr[c]);
            if (dr[c] == 0 || pivs[c] == NULL) continue;
            const orow_t *pr = pivs[c];
            const int64_t m = dr[c];
            int64_t k;
            for (k = 0; k < pr->len; ++k) oaxpy(f, dr, pr->cols[k], m, pr->cfs[k]);
            f->work[0] += pr->len;
            dr[c] = 0;
        }
        int32_t *row = (int32_t *)calloc((size_t)ncr + 1, sizeof(int32_t));
        int32_t nz = 0;
        for (c = ncl; c < ncols; ++c) {
            if (dr[c] != 0) {
                dr[c] = ored(f, dr[c]);
                if (dr[c] != 0) {
                    row[c - ncl] = (int32_t)dr[c];
                    nz++;
                }
            }
        }
        if (nz == 0) {
            free(row);
            continue;
        }
        dm[nd++] = row;
    }

    /* exact_dense_linear_algebra (src/la_ff_16.c:873-989): rows whose first
     * nonzero column is still free become pivots, the others are reduced by
     * the dense pivots and published */
    nps = (odrow_t **)calloc((size_t)ncr + 1, sizeof(odrow_t *));
    int32_t ntr = 0;
    int32_t **tbr = (int32_t **)calloc((size_t)nd + 1, sizeof(int32_t *));
    for (i = 0; i < nd; ++i) {
        int32_t k = 0;
        while (dm[i][k] == 0) ++k;
        if (nps[k] == NULL) {
            odrow_t *pr = (odrow_t *)malloc(sizeof(odrow_t));
            pr->start = k;
            pr->v = (int32_t *)malloc((size_t)(ncr - k) * sizeof(int32_t));
            memcpy(pr->v, dm[i] + k, (size_t)(ncr - k) * sizeof(int32_t));
            if (pr->v[0] != 1) oracle_normalize_row(pr->v, ncr - k, (int32_t)f->p);
            nps[k] = pr;
            free(dm[i]);
        } else {
            tbr[ntr++] = dm[i];
        }
        dm[i] = NULL;
    }
    for (i = 0; i < ntr; ++i) {
        memset(dr, 0, (size_t)ncr * sizeof(int64_t));
        for (j = 0; j < ncr; ++j) dr[j] = tbr[i][j];
        free(tbr[i]);
        odrow_t r = oreduce_dense(f, dr, 0, nps, ncr);
        if (r.v == NULL) continue;
        odrow_t *pr = (odrow_t *)malloc(sizeof(odrow_t));
        *pr = r;
        nps[r.start] = pr;
    }
    free(tbr);

    /* interreduce_dense_matrix (src/la_ff_16.c:837-871) */
    for (i = ncr - 1; i >= 0; --i) {
        if (nps[i] == NULL) continue;
        memset(dr, 0, (size_t)ncr * sizeof(int64_t));
        for (j = i; j < ncr; ++j) dr[j] = nps[i]->v[j - i];
        free(nps[i]->v);
        free(nps[i]);
        nps[i] = NULL;
        odrow_t r = oreduce_dense(f, dr, i, nps, ncr);
        odrow_t *pr = (odrow_t *)malloc(sizeof(odrow_t));
        *pr = r;
        nps[i] = pr;
    }

    /* convert_to_sparse_matrix_rows (src/la_ff_16.c:1322-1392): descending
     * lead, columns shifted by ncl, zeros dropped */
    orow_t **rows = (orow_t **)calloc((size_t)ncr + 1, sizeof(orow_t *));
    for (i = ncr - 1; i >= 0; --i) {
        if (nps[i] == NULL) continue;
        orow_t r;
        r.len = 0;
        r.cols = (int32_t *)malloc((size_t)(ncr - i) * sizeof(int32_t));
        r.cfs = (int32_t *)malloc((size_t)(ncr - i) * sizeof(int32_t));
        for (j = i; j < ncr; ++j) {
            const int32_t v = nps[i]->v[j - i];
            if (v != 0) {
                r.cols[r.len] = j + ncl;
                r.cfs[r.len] = v;
                r.len++;
            }
        }
        rows[np++] = orow_box(r);
    }
    *out_np = np;
    oexport(rows, np, optr, ocols, ovals);
    for (i = 0; i < np; ++i) orow_free(rows[i]);
    free(rows);
done:
    if (nps) {
        for (i = 0; i < ncr; ++i) {
            if (nps[i]) {
                free(nps[i]->v);
                free(nps[i]);
            }
        }
        free(nps);
    }
    if (dm) {
        for (i = 0; i < nd; ++i) free(dm[i]);
        free(dm);
    }
    for (i = 0; i < ncols; ++i) orow_free(pivs[i]);
    for (i = 0; i < nup; ++i) orow_free(upivs[i]);
    free(upivs);
    free(pivs);
    free(dr);
    return rc;
}

/* ---------------------------------------------------------------------- */
int oracle_la_csr(int32_t p, int32_t laopt, int32_t nr, int32_t ncl,
                  int32_t ncr, const int64_t *row_ptr, const int32_t *cols,
                  const int32_t *vals, int32_t *out_np, int64_t **optr,
                  int32_t **ocols, int32_t **ovals, int64_t *work)
{
    ofield_t f;
    int rc;
    if (p < 2 || nr < 0 || ncl < 0 || ncr < 0) return ORACLE_EINVAL;
    ofield_init(&f, p);
    f.ncl = ncl;
    /* option 1 is the sparse/dense split; every other option is answered by
     * the exact sparse echelon (the probabilistic options 42/43/44 return the
     * same reduced rows, src/io.c:630-650 maps unknown options to 2) */
    if (laopt == 1 || laopt <= 0) {
        rc = oracle_sparse_dense(&f, nr, ncl, ncr, row_ptr, cols, vals, out_np,
                                 optr, ocols, ovals);
    } else {
        rc = oracle_sparse_echelon(&f, nr, ncl, ncr, row_ptr, cols, vals,
                                   out_np, optr, ocols, ovals);
    }
    if (work) {
        work[0] = f.work[0];
        work[1] = f.work[1];
    }
    return rc;
}

/* interreduce_matrix_rows (src/la_ff_16.c:1605-1673): every row is a pivot
 * (distinct leads); reduce each by the already interreduced rows of higher
 * columns, from the last column down.  Output in ascending lead order, the
 * order the reference stores them (mat->r[k--]). */
int oracle_interreduce_csr(int32_t p, int32_t nr, int32_t nc,
                           const int64_t *row_ptr, const int32_t *cols,
                           const int32_t *vals, int64_t **optr,
                           int32_t **ocols, int32_t **ovals, int64_t *work)
{
    ofield_t f;
    int32_t i, nup = 0, k;
    ofield_init(&f, p);
    orow_t **pivs = (orow_t **)calloc((size_t)nc + 1, sizeof(orow_t *));
    orow_t **dup = (orow_t **)calloc((size_t)nr + 1, sizeof(orow_t *));
    int64_t *dr = (int64_t *)malloc((size_t)(nc + 1) * sizeof(int64_t));
    int rc = osplit(p, nr, nc, nc, row_ptr, cols, vals, pivs, dup, &nup);
    if (rc == 0 && nup != 0) rc = ORACLE_EINVAL; /* leads must be distinct */
    orow_t **rows = (orow_t **)calloc((size_t)nr + 1, sizeof(orow_t *));
    if (rc == 0) {
        k = nr - 1;
        for (i = nc - 1; i >= 0; --i) {
            if (pivs[i] == NULL) continue;
            memset(dr, 0, (size_t)nc * sizeof(int64_t));
            oscatter(dr, pivs[i]);
            orow_free(pivs[i]);
            pivs[i] = NULL;
            orow_t r = oreduce_sparse(&f, dr, pivs, i, nc, 0);
            pivs[i] = rows[k--] = orow_box(r);
        }
        oexport(rows, nr, optr, ocols, ovals);
        for (i = 0; i < nc; ++i) pivs[i] = NULL;
        for (i = 0; i < nr; ++i) orow_free(rows[i]);
    } else {
        for (i = 0; i < nc; ++i) orow_free(pivs[i]);
    }
    for (i = 0; i < nup; ++i) orow_free(dup[i]);
    free(rows);
    free(dup);
    free(pivs);
    free(dr);
    if (work) {
        work[0] = f.work[0];
        work[1] = f.work[1];
    }
    return rc;
}

void oracle_free(void *ptr) { free(ptr); }
