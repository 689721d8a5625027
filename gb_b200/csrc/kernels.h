// kernels.h -- argument blocks and declarations of the device kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "field.cuh"

namespace gbgpu {

constexpr int kReduceThreads = 512;
enum DenseMode : int32_t { kUntilFree = 0, kFull = 1 };

struct SparseReduceArgs {
    const int64_t* row_ptr;
    const int32_t* cols;
    const uint32_t* vals;
    const int32_t* piv_row;  // [piv_limit]: pivot row of a column, INT_MAX if none
    int32_t piv_limit;       // only columns < piv_limit are reduced
    int32_t skip_lead;       // 1: a row is itself the pivot of its lead
    const int32_t* work;     // rows to reduce
    int32_t n_work;
    int32_t nc;              // accumulator width
    int32_t emit_from;       // first column written out
    int32_t emit_width;      // number of columns written out
    int64_t out_ld;          // row stride of `out`
    int64_t acc_stride;      // per-CTA stride of gacc
    uint32_t* out;           // [n_work][out_ld]
    int32_t* out_lead;       // [n_work]: first nonzero column - emit_from, or -1
    uint32_t* gacc;          // [grid][acc_stride] when the accumulator is global
    int32_t* queue;          // work counter, zero before the launch
    int64_t* work_count;     // pivot entries applied (statistics)
    const uint32_t* err = nullptr;  // optional: the input checks' flags (nonzero: skip)
};

struct DenseReduceArgs {
    const uint32_t* src;     // rows read (pivot rows and the rows' start values)
    uint32_t* dst;           // rows written (== src for kUntilFree)
    int64_t ld;
    int32_t ncr;
    int32_t mode;            // DenseMode
    const int32_t* piv_of_col;  // [ncr]: pivot row of a column or -1
    const int32_t* work;
    const int32_t* n_work;   // device count
    int32_t* lead;           // [rows] lead per row (kUntilFree updates it)
    int32_t* next;           // kUntilFree: survivors
    int32_t* n_next;
    int32_t* queue;
    int64_t* work_count;
};

__global__ void k_check_rows(int32_t nr, const int64_t* row_ptr, const int32_t* cols,
                             const uint32_t* vals, int32_t lead_bound, int32_t nc, uint32_t p,
                             uint32_t* err);
__global__ void k_fill_i32(int32_t* a, int64_t n, int32_t v);
__global__ void k_classify(int32_t nr, const int64_t* row_ptr, const int32_t* cols,
                           int32_t table_size, int32_t* piv_row);
__global__ void k_mark_lower(int32_t nr, const int64_t* row_ptr, const int32_t* cols,
                             int32_t table_size, const int32_t* piv_row, uint8_t* flag,
                             uint32_t* err, int32_t dup_is_error);
__global__ void k_check_pivots(int32_t ncl, const int32_t* piv_row, uint32_t* err);
__global__ void k_iota(int32_t* a, int32_t n);
__global__ void k_pivtab(int32_t n, const int32_t* piv_row, int32_t* piv_of_col);
__global__ void k_gather_rows(int32_t n, const int32_t* pivcol, const int32_t* piv_of_col,
                              int32_t* out, int32_t* n_out);

// templated kernels are launched through these host functions, defined in
// the translation unit that defines the kernels
template <class F>
cudaError_t launch_reduce_sparse(const SparseReduceArgs& a, const F& f, int grid, bool smem,
                                 int smem_bytes, cudaStream_t s);
// the team-per-row form of the known-pivot reduction (pivot rows staged in
// shared memory ahead of use); pext from k_pivot_extents
__global__ void k_pivot_extents(int32_t n, const int32_t* piv_row, const int64_t* row_ptr,
                                longlong2* ext);
int team_smem_bytes(int32_t nc, int smem_optin);
template <class F>
cudaError_t launch_reduce_team(const SparseReduceArgs& a, const longlong2* pext, const F& f,
                               int grid, int smem_bytes, cudaStream_t s);
template <class F>
cudaError_t launch_reduce_dense(const DenseReduceArgs& a, const F& f, int grid, bool smem,
                                int smem_bytes, cudaStream_t s);
template <class F>
cudaError_t launch_promote(int grid, int threads, cudaStream_t s, const int32_t* cand,
                           const int32_t* n_cand, const int32_t* lead, int32_t* claim,
                           int32_t* piv_of_col, uint32_t* rows, int64_t ld, int32_t ncr,
                           int32_t* losers, int32_t* n_losers, const F& f);

// one-CTA reduced row echelon form of a small dense block (see plain.cu)
int tiny_rref_bytes(int32_t n, int32_t m, int smem_optin);
template <class F>
cudaError_t launch_tiny_rref(int32_t n, int32_t m, const uint32_t* D, int64_t ld,
                             const int32_t* lead, const uint32_t* err, int32_t col_shift,
                             int64_t* offs, int32_t* cols, int32_t* vals, int32_t* piv_of_col,
                             int64_t* counts, int bytes, cudaStream_t s, const F& f);

__global__ void k_claim(const int32_t* cand, const int32_t* n_cand, const int32_t* lead,
                        int32_t* claim);
__global__ void k_collect_nonzero(int32_t n, const int32_t* lead, int32_t* out, int32_t* n_out);
__global__ void k_pivot_flags(int32_t ncr, const int32_t* piv_of_col, int32_t desc,
                              int32_t* flag);
__global__ void k_pivot_list(int32_t ncr, const int32_t* flag, const int32_t* pos, int32_t desc,
                             int32_t* pivcol);
__global__ void k_row_nnz(int32_t np, const int32_t* pivcol, const int32_t* piv_of_col,
                          const uint32_t* rows, int64_t ld, int32_t ncr, int64_t* counts);
__global__ void k_row_write(int32_t np, const int32_t* pivcol, const int32_t* piv_of_col,
                            const uint32_t* rows, int64_t ld, int32_t ncr, const int64_t* offs,
                            int32_t col_shift, int32_t* out_cols, void* out_vals, int32_t vb);

}  // namespace gbgpu
