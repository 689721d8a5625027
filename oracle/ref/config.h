/* Build-time configuration for compiling the reference gb sources as a test
 * oracle.  The reference's autotools step would generate this file; only the
 * OpenMP switch is consulted by its finite-field code. */
#ifndef GBREF_CONFIG_H
#define GBREF_CONFIG_H
#define HAVE_OPENMP 1
#endif
