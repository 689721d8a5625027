/* Declarations force-included into gb's unity build when its two
 * linear-algebra call sites are rerouted to libgbgpu.so by two -D macros:
 * gb's own headers define mat_t / bs_t / stat_t, so
 * the GPU entry points are declared here with void pointers. */
void gbgpu_linear_algebra(void *mat, const void *bs, void *st);
void gbgpu_interreduce_matrix_rows(void *mat, void *bs, const void *st);
void gbgpu_convert_hashes_to_columns(void *hcmp, void *mat, void *st, void *sht);
void gbgpu_sort_matrix_rows(void *mat);
void gbgpu_linear_algebra_keep(void *mat, const void *bs, void *st);
int gbgpu_kept_answer(const void *mat);
void gbgpu_convert_sparse_matrix_rows_to_basis_elements(void *mat, void *bs, void *bht,
                                                        const void *sht, const void *hcm,
                                                        void *st);
void gbgpu_symbolic_preprocessing(void *mat, const void *bs, void *st, void *sht,
                                  const void *bht);
