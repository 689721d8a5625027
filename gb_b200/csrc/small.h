// small.h -- one-pass reduction of small Macaulay matrices (small.cu).
#pragma once
#include <stdint.h>

#include "../../include/gbgpu.h"

namespace gbgpu {

// One matrix for the small path.  The rows are written by `fill` straight
// into the session's pinned staging (row_ptr[nr + 1], cols[nnz], vals[nnz] as
// residues in [0, p)), so the caller's row format is converted once.
struct SmallInput {
    int32_t p, nr, ncl, ncr;
    int64_t nnz;
    int device;
    void (*fill)(void* ctx, int64_t* row_ptr, int32_t* cols, uint32_t* vals);
    void* ctx;
};

// The answer, valid until the next small call of this thread on this device:
// np rows in descending lead order, offs[np + 1], cols (shifted by ncl) and
// vals in host memory.
struct SmallAnswer {
    int32_t np = 0;
    int64_t nnz = 0;
    const int64_t* offs = nullptr;
    const int32_t* cols = nullptr;
    const int32_t* vals = nullptr;
};

// True when the small path takes a matrix of this shape on `device`.
bool small_eligible(int32_t nr, int32_t ncl, int32_t ncr, int device);
int small_reduce(const SmallInput& in, SmallAnswer* ans);

// Batches: shared memory the one-launch batch kernel needs for a matrix of
// this shape (0: not a batch-small matrix), and the batch itself -- every
// matrix in one persistent launch, one status each (outs[i] malloc'ed rows).
int small_batch_bytes(int32_t nr, int32_t ncl, int32_t ncr, int device);
int small_batch(int32_t n, const gbgpu_csr* const* ms, int device, gbgpu_rows* outs,
                int32_t* status);
// host CSR of a gbgpu_csr (values widened to u32) into three arrays
void fill_from_csr_vals(void* csr, int64_t* row_ptr, int32_t* cols, uint32_t* vals);

}  // namespace gbgpu
