/* gbla_oracle.h -- TEST INFRASTRUCTURE ONLY: CPU oracle for the GF(p)
 * Macaulay-matrix reduction.  See gbla_oracle.c for what it restates and how
 * it is pinned against the reference. */
#ifndef GBLA_ORACLE_H
#define GBLA_ORACLE_H
#include <stdint.h>

#define ORACLE_EINVAL (-22)

int32_t oracle_inverse(int32_t val, int32_t p);
void oracle_normalize_row(int32_t *row, int64_t len, int32_t p);

/* Reduced new pivots of one Macaulay matrix (the reference's linear_algebra),
 * descending lead order, columns >= ncl, lead coefficient 1.  work[0] counts
 * the known-pivot row entries applied, work[1] the new-pivot entries, in this
 * single-threaded order (work may be NULL, else points to 2 counters). */
int oracle_la_csr(int32_t p, int32_t laopt, int32_t nr, int32_t ncl,
                  int32_t ncr, const int64_t *row_ptr, const int32_t *cols,
                  const int32_t *vals, int32_t *out_np, int64_t **optr,
                  int32_t **ocols, int32_t **ovals, int64_t *work);

/* Full interreduction of rows with distinct leads (the reference's
 * interreduce_matrix_rows); output in ascending lead order; work as above
 * (all applications count as new pivots). */
int oracle_interreduce_csr(int32_t p, int32_t nr, int32_t nc,
                           const int64_t *row_ptr, const int32_t *cols,
                           const int32_t *vals, int64_t **optr,
                           int32_t **ocols, int32_t **ovals, int64_t *work);

void oracle_free(void *ptr);
#endif
