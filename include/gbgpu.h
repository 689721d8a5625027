/* gbgpu.h -- C ABI of the B200 GF(p) linear-algebra library (libgbgpu.so).
 *
 * The library performs the linear-algebra step of gb's F4 (ederc/gb v0.16):
 * the exact reduction over GF(p) of one Macaulay matrix, for primes below
 * 2^31 (the 8-, 16-, 17- and 31-bit paths of src/la_ff_8.c, src/la_ff_16.c,
 * src/la_ff_32.c), on one NVIDIA B200.  There is no CPU fallback: every entry
 * point fails with GBGPU_ENODEV when no usable sm_100 device is present.
 *
 * Two layers:
 *   1. Drop-in replacements for the reference's function pointers
 *      linear_algebra / interreduce_matrix_rows (src/data.h:269-279), over
 *      layout-compatible mirrors of mat_t, bs_t and stat_t.
 *   2. A flat CSR interface (plain pointers and sizes) for standalone and
 *      batched matrices, with a device-resident plan for repeated runs.
 *
 * Answer of one reduction: the rows of the reduced row echelon form of the
 * matrix's row space restricted to {x : x vanishes on the left block}, i.e.
 * the new pivots of src/la_ff_16.c:702-727 / :1343-1390: lead coefficient 1,
 * columns ascending (all >= ncl), rows in descending lead order.  The answer
 * does not depend on the la option; options 1, 2, 42, 43 and 44 return the
 * same rows in the reference too.
 */
#ifndef GBGPU_H
#define GBGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------- */
#define GBGPU_OK 0
#define GBGPU_EINVAL (-22)  /* input breaks the mat_t contract          */
#define GBGPU_ENOMEM (-12)  /* host or device allocation failed         */
#define GBGPU_ENODEV (-19)  /* no sm_100 device / CUDA error at init    */
#define GBGPU_ECUDA (-5)    /* a CUDA call failed                       */
#define GBGPU_ETIMEDOUT (-110) /* a device-side bounded wait gave up     */
#define GBGPU_ERANGE (-34)  /* size beyond a documented limit           */

/* ---- 1. drop-in boundary -------------------------------------------- */
/* Layout mirrors of the reference structs (src/data.h:117-211).  Only the
 * members the linear algebra reads or writes are named; the byte layout is
 * identical (checked by the test-suite against the reference build). */
typedef int32_t gbgpu_hm_t;   /* hm_t  (src/data.h:59-60) */
typedef int32_t gbgpu_len_t;  /* len_t (src/data.h:64)    */

typedef struct gbgpu_bs_t {   /* bs_t, src/data.h:117-135 */
    int32_t ld, sz, lo, mltdeg;
    int32_t *lmps;
    int32_t *lm;
    int32_t lml;
    int8_t *red;
    gbgpu_hm_t **hm;
    int8_t **cf_8;
    int16_t **cf_16;
    int32_t **cf_32;
    void **cf_qq;
} gbgpu_bs_t;

typedef struct gbgpu_mat_t {  /* mat_t, src/data.h:137-155 */
    gbgpu_hm_t **r;
    int8_t **cf_8;
    int16_t **cf_16;
    int32_t **cf_32;
    void **cf_qq;
    void **cf_ab_qq;
    gbgpu_len_t sz, np, nr, nc, nru, nrl, ncl, ncr;
} gbgpu_mat_t;

typedef struct gbgpu_stat_t { /* stat_t, src/data.h:157-211 */
    double round_ctime, select_ctime, symbol_ctime, la_ctime, update_ctime,
        convert_ctime, overall_ctime, reduce_gb_ctime, rht_ctime;
    double round_rtime, select_rtime, symbol_rtime, la_rtime, update_rtime,
        convert_rtime, overall_rtime, reduce_gb_rtime, rht_rtime;
    int64_t num_pairsred, num_gb_crit, num_redundant_old, num_redundant,
        num_rht, num_rowsred, num_zerored;
    int32_t ngens, nvars, mnsel, homogeneous, fc, mo, laopt, init_hts,
        nthrds, reset_ht, current_rd, current_deg;
    int64_t max_bht_size, max_sht_size, max_uht_size, nterms_basis;
    int32_t size_basis, ff_bits, reduce_gb;
    int32_t info_level, gen_pbm_file;
} gbgpu_stat_t;

/* hd_t and ht_t, src/data.h:69-97 (the hash data and the hash table) */
typedef struct gbgpu_hd_t {
    int32_t val, sdm, deg, idx;
} gbgpu_hd_t;

typedef struct gbgpu_ht_t {
    int16_t **ev;        /* exponent vectors, exp_t = int16_t */
    gbgpu_hd_t *hd;
    int32_t *hmap;
    int32_t eld, esz, hsz, nv;
    int32_t *dm;
    int32_t ndv, bpv;
    int32_t *rn;
    uint32_t rsd;
} gbgpu_ht_t;

/* Replaces `linear_algebra(mat, bs, st)` at src/f4.c:306 for every la option
 * (the function-pointer table of src/io.c:581-780).  Same contract as the
 * reference (src/la_ff_16.c:1430-1507): reads mat->r rows and bs->cf_X
 * coefficient arrays, frees the input rows, sets mat->np / mat->r /
 * mat->cf_X with malloc'ed output rows (row[0] = index into mat->cf_X,
 * row[1] = len % 4, row[2] = len), updates st->la_ctime / la_rtime /
 * num_zerored.  The reference's function returns void and cannot fail; this
 * one prints the GBGPU_* status and exits on error, since it has no CPU
 * fallback. */
void gbgpu_linear_algebra(gbgpu_mat_t *mat, const gbgpu_bs_t *bs,
                          gbgpu_stat_t *st);

/* Replaces `interreduce_matrix_rows(mat, bs, st)` at src/f4.c:137
 * (src/la_ff_16.c:1605-1673 and twins): fully interreduces rows with
 * distinct leads, frees the basis elements like free_basis_elements
 * (src/basis.c:25-57), stores the reduced rows in mat->r in ascending lead
 * order and sets mat->np = mat->nr. */
void gbgpu_interreduce_matrix_rows(gbgpu_mat_t *mat, gbgpu_bs_t *bs,
                                   const gbgpu_stat_t *st);

/* Replaces `convert_hashes_to_columns(&hcm, mat, st, sht)` at src/f4.c:299
 * (src/convert.c:30-135): the columns of the round are the monomials
 * 1 .. sht->eld-1 of the secondary hash table, ordered as the reference's
 * hcm_cmp orders them (src/order.c:153-235; st->mo 0 DRL, 1 LEX) on the
 * device; *hcmp (realloc'ed) receives the hash of every column, sht->hd[h].idx
 * the column of hash h, every row's entries their columns, and mat->nru /
 * ncl / nrl / ncr and st->num_rowsred are set as the reference sets them.
 * The rows of mat->r also come back in the order of sort_matrix_rows
 * (lead column, then length), so that the reference's sort which follows
 * finds them sorted.  Prints the status and exits on error. */
void gbgpu_convert_hashes_to_columns(int32_t **hcmp, gbgpu_mat_t *mat, gbgpu_stat_t *st,
                                     gbgpu_ht_t *sht);
/* Replaces `sort_matrix_rows(mat)` at src/f4.c:300 (src/order.c:125-131):
 * rows by (lead column, length) on the device; rows that tie keep their
 * order. */
void gbgpu_sort_matrix_rows(gbgpu_mat_t *mat);

/* Replaces `symbolic_preprocessing(mat, bs, st, sht, bht)` at src/f4.c:298
 * and :121 (src/symbol.c:202-272): walks the secondary table's monomials in
 * index order, marks every one as a column, and for each the first basis
 * element of the lead-monomial list whose lead divides it becomes a matrix
 * row (multiplied by the quotient, its terms inserted into sht as
 * src/hash.c:672-746 inserts them).  The reducer search runs on the device
 * for a wave of monomials at a time; the walk itself, the rows and the
 * insertions follow the reference step by step, so sht and mat end as the
 * reference leaves them.  Grows sht and mat->r as the reference does.
 * Prints the status and exits on error. */
void gbgpu_symbolic_preprocessing(gbgpu_mat_t *mat, const gbgpu_bs_t *bs, gbgpu_stat_t *st,
                                  gbgpu_ht_t *sht, const gbgpu_ht_t *bht);
int gbgpu_symbolic_preprocessing_status(gbgpu_mat_t *mat, const gbgpu_bs_t *bs,
                                        gbgpu_stat_t *st, gbgpu_ht_t *sht,
                                        const gbgpu_ht_t *bht);

/* The linear algebra and the step after it with the answer kept on the
 * device in between (src/f4.c:306-311).
 *
 * gbgpu_linear_algebra_keep replaces `linear_algebra(mat, bs, st)` at
 * src/f4.c:306 like gbgpu_linear_algebra (input rows freed, mat->np and, for
 * the sparse options, mat->nr / mat->sz set, statistics updated), but keeps
 * the answer on the device, in a slot of the calling thread, instead of
 * building mat->r; the next call of either function below on this thread
 * takes it (a new gbgpu_linear_algebra_keep drops an answer nobody took).
 *
 * gbgpu_convert_sparse_matrix_rows_to_basis_elements replaces
 * `convert_sparse_matrix_rows_to_basis_elements(mat, bs, bht, sht, hcm, st)`
 * at src/f4.c:309 (src/convert.c:137-280): the kept answer becomes basis
 * elements bs->hm[bs->ld + i] / bs->cf_X[bs->ld + i] (mat->r and mat->cf_X
 * point to the same rows, as after the reference), every entry holding the
 * index of its monomial in the basis hash table bht.  The reference looks up
 * every entry in bht and inserts the monomials it does not find
 * (src/hash.c:604-669); here each right column is looked up once, in the
 * order of its first entry in the answer (found on the device), which gives
 * bht exactly the indices and the layout the reference gives it, and the
 * entries are rewritten on the device through the column -> index map.
 * Grows bs (src/basis.c:149-165) and bht (src/hash.c:185-240) as the
 * reference does.  GBGPU_EINVAL without a kept answer for mat.  The call at
 * src/f4.c:140 (after the final interreduction) has no kept answer and stays
 * the reference's. */
void gbgpu_linear_algebra_keep(gbgpu_mat_t *mat, const gbgpu_bs_t *bs,
                               gbgpu_stat_t *st);
int gbgpu_linear_algebra_keep_status(gbgpu_mat_t *mat, const gbgpu_bs_t *bs,
                                     gbgpu_stat_t *st);
/* 1 when the calling thread holds the kept answer of mat, else 0 */
int gbgpu_kept_answer(const gbgpu_mat_t *mat);
void gbgpu_convert_sparse_matrix_rows_to_basis_elements(gbgpu_mat_t *mat, gbgpu_bs_t *bs,
                                                        gbgpu_ht_t *bht, const gbgpu_ht_t *sht,
                                                        const int32_t *hcm, gbgpu_stat_t *st);
int gbgpu_convert_sparse_matrix_rows_to_basis_elements_status(
    gbgpu_mat_t *mat, gbgpu_bs_t *bs, gbgpu_ht_t *bht, const gbgpu_ht_t *sht,
    const int32_t *hcm, gbgpu_stat_t *st);

/* Same as the two above but returning a status instead of exiting. */
int gbgpu_linear_algebra_status(gbgpu_mat_t *mat, const gbgpu_bs_t *bs,
                                gbgpu_stat_t *st);
int gbgpu_interreduce_matrix_rows_status(gbgpu_mat_t *mat, gbgpu_bs_t *bs,
                                         const gbgpu_stat_t *st);

/* ---- 2. flat CSR interface ------------------------------------------ */
typedef struct gbgpu_csr {
    int32_t p;        /* prime, 2 <= p < 2^31                           */
    int32_t laopt;    /* reference la option (1, 2, 42, 43, 44); informational */
    int32_t nr;       /* rows                                           */
    int32_t ncl;      /* left-block columns (= number of known pivots)  */
    int32_t ncr;      /* right-block columns                            */
    const int64_t *row_ptr; /* [nr + 1], host or device (see flags)      */
    const int32_t *cols;    /* [nnz]; first entry of a row = its lead     */
    const int32_t *vals;    /* [nnz]; residues in [1, p), lead = 1        */
    /* Width of one entry of vals in bytes: 4 (int32, also when 0), 2 (uint16,
     * p < 2^16) or 1 (uint8, p < 2^8) -- the coefficient widths of the
     * reference's cf_32 / cf_16 / cf_8 arrays (src/data.h), which halve or
     * quarter the host-to-device traffic of the values. */
    int32_t val_bytes;
} gbgpu_csr;

/* Reduced rows in host memory allocated by the library with malloc. */
typedef struct gbgpu_rows {
    int32_t np;
    int64_t nnz;
    int64_t *row_ptr; /* [np + 1] */
    int32_t *cols;    /* [nnz]    */
    int32_t *vals;    /* [nnz]    */
} gbgpu_rows;

/* Algorithm selection. */
#define GBGPU_FORM_AUTO 0
#define GBGPU_FORM_PLAIN 1  /* sparse rows on CUDA cores                */
#define GBGPU_FORM_TENSOR 2 /* blocked, int8 tensor-core modular GEMMs  */
#define GBGPU_FORM_BLOCKED_PLAIN 3 /* blocked, CUDA-core modular GEMMs    */

typedef struct gbgpu_options {
    int32_t form;       /* GBGPU_FORM_*                                  */
    int32_t device;     /* CUDA device ordinal                           */
    int32_t check;      /* 1: validate the input contract on the device  */
    int32_t profile;    /* 1: time every tensor-core GEMM launch (events)  */
    void *stream;       /* cudaStream_t to run on; NULL = library stream */
} gbgpu_options;

/* Work counters and timings of the last run of a plan. */
typedef struct gbgpu_stats {
    double ms_total;        /* device time of the whole reduction (events)   */
    double ms_schur;        /* known-pivot reduction of the C|D rows         */
    double ms_echelon;      /* echelon of the reduced right block            */
    double ms_rref;         /* back substitution to reduced echelon form     */
    double ms_compact;      /* output compaction                             */
    int64_t rows_reduced;   /* C|D rows                                      */
    int64_t dense_rows;     /* nonzero rows after the known-pivot step       */
    int64_t rank;           /* np                                            */
    int64_t echelon_rounds; /* pivot-claiming rounds of the echelon          */
    int64_t kernel_launches;/* kernels launched by the last run              */
    int64_t work_schur;     /* known-pivot entries applied (sum of pivot row
                               lengths over every pivot application)        */
    int64_t work_dense;     /* dense-pivot entries applied in the echelon and
                               back substitution                            */
    int64_t gemm_launches;  /* tensor-core GEMM kernels (k_tc_submul) run    */
    double gemm_ms;         /* their summed device time (profile = 1 only)   */
    double gemm_int8_ops;   /* int8 tensor ops they executed (2 per MAC, all
                               limb products, zero tiles skipped)           */
    int64_t form_used;      /* GBGPU_FORM_PLAIN / _TENSOR / _BLOCKED_PLAIN   */
    double ms_classify;     /* input checks, known pivots, C|D row list      */
    double ms_check;        /* the device-side input checks alone            */
} gbgpu_stats;

/* One-shot: host CSR in, host rows out (H2D, reduction, D2H). */
int gbgpu_reduce(const gbgpu_csr *m, const gbgpu_options *opt,
                 gbgpu_rows *out);

/* Full interreduction of rows with distinct leads over nc columns (the
 * reference's interreduce_matrix_rows on a flat matrix); ascending leads. */
int gbgpu_interreduce(int32_t p, int32_t nr, int32_t nc,
                      const int64_t *row_ptr, const int32_t *cols,
                      const int32_t *vals, const gbgpu_options *opt,
                      gbgpu_rows *out);

void gbgpu_rows_free(gbgpu_rows *rows);

/* Device-resident plan: the matrix is uploaded once; each run reduces it
 * again from the uploaded copy (inputs are never modified). */
typedef struct gbgpu_plan gbgpu_plan;

int gbgpu_plan_create(const gbgpu_csr *m, const gbgpu_options *opt,
                      gbgpu_plan **plan);
/* Enqueue one reduction on the plan's stream; returns after enqueueing
 * (the echelon's claiming rounds read one counter back per round). */
int gbgpu_plan_run(gbgpu_plan *plan);
/* Block until the last run finished and copy its answer to host memory. */
int gbgpu_plan_result(gbgpu_plan *plan, gbgpu_rows *out);
/* Same into caller-provided host arrays (pinned memory makes the copy run at
 * full PCIe speed): cap_rows >= np + 1 and cap_nnz >= nnz entries, else
 * GBGPU_ERANGE with *np / *nnz set to the sizes needed (NULL arrays with zero
 * capacities just query the sizes). */
int gbgpu_plan_result_into(gbgpu_plan *plan, int64_t *row_ptr, int32_t *cols,
                           int32_t *vals, int64_t cap_rows, int64_t cap_nnz,
                           int32_t *np, int64_t *nnz);
/* gbgpu_plan_result_into with values of val_bytes bytes each (4: int32,
 * 2: uint16 for p < 2^16, 1: uint8 for p < 2^8), the widths the reference
 * keeps in mat->cf_32 / cf_16 / cf_8; narrower values shorten the copy. */
int gbgpu_plan_result_into_v(gbgpu_plan *plan, int64_t *row_ptr, int32_t *cols,
                             void *vals, int32_t val_bytes, int64_t cap_rows,
                             int64_t cap_nnz, int32_t *np, int64_t *nnz);
/* Run and deliver the answer into caller host arrays (values of val_bytes
 * bytes, as gbgpu_plan_result_into_v).  On the blocked forms the finished
 * blocks of the back substitution are compacted and copied while the rest is
 * still computed, so most of the device-to-host copy overlaps the reduction.
 * Arrays too small: GBGPU_ERANGE with *np / *nnz set (run again with larger
 * arrays).  After a streamed run the gbgpu_plan_result* calls return
 * GBGPU_EINVAL until the next gbgpu_plan_run. */
int gbgpu_plan_run_into_v(gbgpu_plan *plan, int64_t *row_ptr, int32_t *cols,
                          void *vals, int32_t val_bytes, int64_t cap_rows,
                          int64_t cap_nnz, int32_t *np, int64_t *nnz);
int gbgpu_plan_stats(const gbgpu_plan *plan, gbgpu_stats *stats);
/* After gbgpu_plan_run of a linear_algebra plan (not streamed): first[j]
 * (n = ncr entries) = the position, in the answer's entry array, of the
 * first entry in right column j (column ncl + j), -1 when no row has one.
 * The basis conversion's insertion order (src/hash.c:604-669). */
int gbgpu_plan_first_entry(gbgpu_plan *plan, int64_t *first, int32_t n);
/* Rewrites every entry of the plan's answer on the device: column ncl + j
 * becomes map[j] (n = ncr entries; the basis hash table's indices for the
 * conversion of src/convert.c:137-280).  The gbgpu_plan_result* calls then
 * return the mapped entries.  Once mapped, the answer's columns no longer
 * count from ncl: a second map or a gbgpu_plan_first_entry call returns
 * GBGPU_EINVAL until the plan runs again. */
int gbgpu_plan_map_columns(gbgpu_plan *plan, const int32_t *map, int32_t n);
void gbgpu_plan_destroy(gbgpu_plan *plan);

/* Batched reduction of n independent matrices (different sizes and primes)
 * in one pass: status[i] receives each matrix's own status, so one bad
 * matrix does not fail the others.  Returns GBGPU_OK if the batch ran;
 * without a usable device none runs and the call and every status[i]
 * return the device error (GBGPU_ENODEV).
 * GBGPU_BATCH_WORKERS (default 4) matrices are in flight at once, each on a
 * stream of its own (opt->stream is not used). */
int gbgpu_reduce_batch(int32_t n, const gbgpu_csr *ms,
                       const gbgpu_options *opt, gbgpu_rows *outs,
                       int32_t *status);

/* ---- 3. dense exact modular GEMM -------------------------------------- */
/* D <- (D - A B) mod p for residue matrices (uint32 in [0, p), row-major,
 * leading dimensions in elements): A is M x K, B is K x N, D is M x N.  The
 * Schur update D - C A^-1 B of the A|B/C|D split and the trailing updates of
 * the dense echelon are this operation (the dense steps of
 * src/la_ff_16.c:353-409 / :837-989 done blockwise).  GBGPU_FORM_TENSOR (the
 * AUTO choice for odd p) runs it on the int8 tensor cores with the residues
 * split into 8-bit limbs, GBGPU_FORM_PLAIN on CUDA cores; both are exact.
 * Pointers are device memory; runs on opt->stream (NULL: the legacy default
 * stream) and returns when the result is complete. */
int gbgpu_dense_submul(int32_t p, int32_t M, int32_t N, int32_t K,
                       const uint32_t *A, int64_t lda, const uint32_t *B,
                       int64_t ldb, uint32_t *D, int64_t ldd,
                       const gbgpu_options *opt);
/* Same with host arrays (copied in and out). */
int gbgpu_dense_submul_host(int32_t p, int32_t M, int32_t N, int32_t K,
                            const uint32_t *A, int64_t lda, const uint32_t *B,
                            int64_t ldb, uint32_t *D, int64_t ldd,
                            const gbgpu_options *opt);

/* Reduced row echelon form of a dense residue matrix (rows x cols, row-major,
 * device memory, leading dimension ld >= cols), in place: on return the
 * first *rank rows are the reduced rows in ascending pivot-column order
 * (lead 1, zero at every other pivot column), the remaining rows are zero,
 * and piv_cols[0 .. *rank) (device memory, min(rows, cols) entries) holds the
 * pivot columns.  This is the dense echelon + interreduction of the D block
 * (src/la_ff_16.c:873-989 and :837-871) run blockwise: claiming rounds,
 * shared-memory panel factorizations and tensor-core GEMMs for the updates
 * (GBGPU_FORM_PLAIN: CUDA-core GEMMs). */
int gbgpu_dense_rref(int32_t p, int32_t rows, int32_t cols, uint32_t *D,
                     int64_t ld, int32_t *rank, int32_t *piv_cols,
                     const gbgpu_options *opt);

/* Allocation-free variant of gbgpu_dense_submul (tensor-core form, odd p),
 * for callers that must not allocate device memory once they run: a service
 * whose device-memory budget is reserved up front, or a host program whose
 * own allocator owns all device memory and forbids other cudaMalloc /
 * cudaFree calls.  No counterpart in the reference.  Its scratch (the 8-bit
 * limb planes of A and B and a status word) is one fixed 32 MiB device array
 * inside the library, present on every GPU that loads it until the process
 * exits; requests whose limb planes need more than 32 MiB - 256 bytes are
 * rejected with GBGPU_ERANGE.  The first call on a device looks the array's
 * address up (cudaGetSymbolAddress) and caches it for the life of the
 * process, so calls may not follow a cudaDeviceReset of that device.  Calls
 * share the array: calls that overlap on the GPU race and must be serialised
 * by the caller.  Device pointers; runs on `stream` (NULL: legacy default
 * stream), waits for it and returns when the result is complete. */
int gbgpu_dense_submul_noalloc(int32_t p, int32_t M, int32_t N, int32_t K,
                               const uint32_t *A, int64_t lda,
                               const uint32_t *B, int64_t ldb, uint32_t *D,
                               int64_t ldd, int32_t device, void *stream);

/* ---- the step before the linear algebra -------------------------------- */
/* convert_hashes_to_columns + sort_matrix_rows (src/convert.c:30-135,
 * src/order.c:98-131) on flat host arrays: the n monomials of one round
 * (exps[n][nv], total degrees deg[n], idx[n] = 2 for the lead monomials of
 * known pivots, 1 otherwise; monomial i has hash index i + 1) and nr rows of
 * hash indices (row_ptr[nr + 1], hashes[nnz], first entry = lead term); mo 0
 * DRL, 1 LEX.  Outputs: hcm[n] (hash index of every column, in column order),
 * *ncl (columns of known pivots), row_order[nr] (input row of every output
 * row), out_row_ptr[nr + 1] and out_cols[nnz] (the rows in that order, every
 * entry's column, entries in input order).  Rows tie-broken by input order. */
int gbgpu_convert_hashes_to_columns_flat(int32_t nv, int32_t n, const int16_t *exps,
                                         const int32_t *deg, const int32_t *idx, int32_t mo,
                                         int32_t nr, const int64_t *row_ptr,
                                         const int32_t *hashes, int32_t *hcm, int32_t *ncl,
                                         int32_t *row_order, int64_t *out_row_ptr,
                                         int32_t *out_cols, int32_t device);

/* ---- autotuning -------------------------------------------------------- */
/* Times every tile shape of the tensor-core GEMM for every limb count the
 * shapes differ in (1 and 2) and every band of reduction depths K on this
 * device, and writes the fastest shape per (limbs, K band) to the cache file
 * `path` (NULL: $GBGPU_TUNE_FILE, else $HOME/.cache/gbgpu/gemm_shapes.txt),
 * which every later process reads at its first GEMM; this process uses the
 * result at once.  No counterpart in the reference (it has no GPU code); the
 * tuned choice never changes a result, only its speed.  About 2 s. */
int gbgpu_autotune(int32_t device, const char *path);

/* ---- misc ------------------------------------------------------------ */
/* Fills out[0..n) with sizeof/offsetof values of the mirrored structs in
 * the order the test-suite compares; returns how many it knows. */
int gbgpu_layout(int64_t *out, int32_t n);
/* Short description of the last error on this thread. */
const char *gbgpu_last_error(void);
/* Kernels launched since load (all entry points), for accounting. */
int64_t gbgpu_kernel_launches(void);

#ifdef __cplusplus
}
#endif
#endif /* GBGPU_H */
