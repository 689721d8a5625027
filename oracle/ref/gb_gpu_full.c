/* gb_gpu_full.c -- TEST INFRASTRUCTURE ONLY (and the recipe a user follows).
 *
 * gb (ederc/gb v0.16) with the steps before the linear algebra on the GPU as
 * well: its unity build (the include list of src/gb.c) with function-like
 * macros defined just before f4.c, so that only f4.c's calls of
 * symbolic_preprocessing, convert_hashes_to_columns and sort_matrix_rows
 * (src/f4.c:121, :132-135, :298-300) go to libgbgpu.so; their definitions in
 * symbol.c, convert.c and order.c, compiled earlier, keep their names.  The Makefile adds the two -D macros
 * that reroute the linear algebra (src/f4.c:137, :306), as for libgb_gpu.so;
 * below, the round's linear algebra and the conversion of its answer into
 * basis elements (src/f4.c:306-311) are rerouted together. */
#include <stdio.h>
#include <stdlib.h>
#include <gmp.h>

#include "stat.c"
#include "time.c"
#include "tools.c"
#include "sort_r.h"
#include "hash.c"
#include "order.c"
#include "basis.c"
#include "la_ff_8.c"
#include "la_ff_16.c"
#include "la_ff_32.c"
#include "la_qq.c"
#include "update.c"
#include "convert.c"
#include "symbol.c"
#include "io.c"

#define convert_hashes_to_columns(a, b, c, d) \
    gbgpu_convert_hashes_to_columns((void *)(a), (void *)(b), (void *)(c), (void *)(d))
#define sort_matrix_rows(m) gbgpu_sort_matrix_rows((void *)(m))
#define symbolic_preprocessing(m, b, s, sh, bh) \
    gbgpu_symbolic_preprocessing((void *)(m), (const void *)(b), (void *)(s), (void *)(sh), \
                                 (const void *)(bh))

/* The linear algebra of every round keeps its answer on the device, and the
 * step after it (src/f4.c:309) turns that answer into basis elements there.
 * The same function's other call (src/f4.c:140, after the final
 * interreduction) has no kept answer and stays gb's own. */
static void gbgpu_rows_to_basis(mat_t *mat, bs_t *bs, ht_t *bht, const ht_t *sht,
                                const hl_t *hcm, stat_t *st)
{
    if (gbgpu_kept_answer(mat))
        gbgpu_convert_sparse_matrix_rows_to_basis_elements(mat, bs, bht, sht, hcm, st);
    else
        (convert_sparse_matrix_rows_to_basis_elements)(mat, bs, bht, sht, hcm, st);
}
#undef linear_algebra
#define linear_algebra(m, b, s) \
    gbgpu_linear_algebra_keep((void *)(m), (const void *)(b), (void *)(s))
#define convert_sparse_matrix_rows_to_basis_elements(m, b, bh, sh, hc, s) \
    gbgpu_rows_to_basis(m, b, bh, sh, hc, s)

#include "f4.c"
