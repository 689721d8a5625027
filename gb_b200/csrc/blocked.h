// blocked.h -- the blocked (tensor-core) form of the Macaulay reduction.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace gbgpu {

struct BlockedInput {
    uint32_t p;
    int32_t ncl, ncr;
    int32_t n_work;           // C|D rows
    const int32_t* work;      // their CSR row indices (device)
    const int64_t* row_ptr;   // device CSR of the whole matrix
    const int32_t* cols;
    const uint32_t* vals;
    const int32_t* piv_row;   // [ncl]: known pivot row of each left column
    cudaStream_t stream;
    int form;                 // GBGPU_FORM_TENSOR: int8 tensor-core GEMMs, else CUDA cores
    int32_t* err;             // device status word of the tensor-core kernels
};

struct BlockedOutput {
    int32_t* piv_of_col = nullptr;  // [ncr], filled: reduced row of each pivot column or -1
    uint32_t* rows = nullptr;       // reduced rows (row piv_of_col[c] of `rows`), ld below
    int64_t ld = 0;
    int64_t rank = 0, dense_rows = 0, echelon_rounds = 0;
    cudaEvent_t ms_event_schur = nullptr, ms_event_echelon = nullptr;
    std::vector<void*>* keep = nullptr;  // device buffers alive until blocked_release
};

int blocked_reduce(const BlockedInput& in, BlockedOutput* out, long long* launches);

// reduced row echelon form of a dense residue matrix, in place (device memory)
struct DenseRrefInput {
    uint32_t p;
    int32_t rows, cols;
    uint32_t* D;        // rows x cols, leading dimension ld
    int64_t ld;
    int32_t* piv_cols;  // device, >= min(rows, cols) entries: the pivot columns
    cudaStream_t stream;
    int form;
    int32_t* err;
};
int dense_rref(const DenseRrefInput& in, int32_t* rank, long long* launches);
void blocked_release(BlockedOutput* out, cudaStream_t s);

}  // namespace gbgpu
