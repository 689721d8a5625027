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

// Streaming of the answer while the back substitution runs: each finished
// block of pivot rows (the output is in descending pivot order, so the last
// block comes first) is compacted into CSR and copied to host memory on a
// second stream, overlapping the copies with the remaining blocks.
struct StreamOut {
    int32_t col_shift = 0;
    int64_t* offs = nullptr;     // device [rank + 1]: row offsets of the answer (filled)
    int32_t* h_cols = nullptr;   // host destinations (pinned for full speed)
    void* h_vals = nullptr;
    int32_t val_bytes = 4;       // 4, 2 or 1 bytes per host value
    int64_t cap_nnz = 0;
    cudaStream_t s_out = nullptr;
    // results
    int64_t nnz = 0;             // entries of the answer
    bool overflow = false;       // host arrays too small: nothing was copied
};

struct BlockedOutput {
    StreamOut* stream_out = nullptr;  // optional (see StreamOut)
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
