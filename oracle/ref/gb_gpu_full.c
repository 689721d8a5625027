/* gb_gpu_full.c -- TEST INFRASTRUCTURE ONLY (and the recipe a user follows).
 *
 * gb (ederc/gb v0.16) with the step before the linear algebra on the GPU as
 * well: its unity build (the include list of src/gb.c) with two function-like
 * macros defined just before f4.c, so that only f4.c's calls of
 * convert_hashes_to_columns and sort_matrix_rows (src/f4.c:132-135 and
 * :299-300) go to libgbgpu.so; their definitions in convert.c and order.c,
 * compiled earlier, keep their names.  The Makefile adds the two -D macros
 * that reroute the linear algebra (src/f4.c:137, :306), as for libgb_gpu.so. */
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

#include "f4.c"
