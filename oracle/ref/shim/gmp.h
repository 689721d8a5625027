/* Placeholder for <gmp.h>, used only to compile the reference gb sources as a
 * test oracle.  The finite-field linear algebra never touches GMP; the rational
 * code paths (la_qq.c, the qq import/export in io.c) still have to compile, so
 * mpz_t is an opaque type and every mpz_* / gmp_* entry point aborts if it is
 * ever reached.  Struct layouts that hold mpz_t only hold pointers to it. */
#ifndef GBREF_GMP_SHIM_H
#define GBREF_GMP_SHIM_H
#include <stdio.h>
#include <stdlib.h>

typedef struct { int alloc_; int size_; void *limbs_; } gbref_mpz_struct;
typedef gbref_mpz_struct mpz_t[1];

static inline int gbref_gmp_unavailable(void)
{
    fprintf(stderr, "gbref: rational (GMP) path reached in an FF-only build\n");
    abort();
    return 0;
}

#define GBREF_GMP_VOID(...) ((void)gbref_gmp_unavailable())
#define GBREF_GMP_INT(...)  (gbref_gmp_unavailable())

#define mpz_init        GBREF_GMP_VOID
#define mpz_inits       GBREF_GMP_VOID
#define mpz_init_set    GBREF_GMP_VOID
#define mpz_clear       GBREF_GMP_VOID
#define mpz_clears      GBREF_GMP_VOID
#define mpz_set         GBREF_GMP_VOID
#define mpz_set_si      GBREF_GMP_VOID
#define mpz_swap        GBREF_GMP_VOID
#define mpz_neg         GBREF_GMP_VOID
#define mpz_mul         GBREF_GMP_VOID
#define mpz_submul      GBREF_GMP_VOID
#define mpz_divexact    GBREF_GMP_VOID
#define mpz_gcd         GBREF_GMP_VOID
#define mpz_lcm         GBREF_GMP_VOID
#define mpz_sgn         GBREF_GMP_INT
#define mpz_cmp_si      GBREF_GMP_INT
#define mpz_divisible_p GBREF_GMP_INT
#define gmp_printf      GBREF_GMP_INT
#endif
