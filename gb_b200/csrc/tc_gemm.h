// tc_gemm.h -- exact modular GEMM D <- (D - A B) mod p (device pointers).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <utility>
#include <vector>

namespace gbgpu {

struct TcGemmArgs {
    uint32_t p;
    int32_t M, N, K;
    const uint32_t* A;  // M x K, row-major, residues
    int64_t lda;
    const uint32_t* B;  // K x N, row-major, residues
    int64_t ldb;
    uint32_t* D;        // M x N, row-major, residues, updated in place
    int64_t ldd;
    // batched form: `batch` independent products, item z at A + z sA,
    // B + z sB, D + z sD (element strides)
    int32_t batch = 1;
    int64_t sA = 0, sB = 0, sD = 0;
    // optional row indirection: row m of A is A + a_rows[m] lda (row k of B
    // is B + b_rows[k] ldb, row m of D is D + d_rows[m] ldd); a negative index
    // is a zero row of A or B and a row of D that is left untouched.  Batch
    // item z reads its indices at a_rows + z sAr (b_rows + z sBr, d_rows + z sDr).
    const int32_t* a_rows = nullptr;
    const int32_t* b_rows = nullptr;
    const int32_t* d_rows = nullptr;
    int64_t sAr = 0, sBr = 0, sDr = 0;
    // optional (unbatched, no b_rows): for every group of 128 rows of B
    // (rows [128 g, 128 g + 128)) the first and last column that may be
    // nonzero (.x > .y: the group is zero).  B is zero outside, and its
    // memory there is never read; between the two columns widened to
    // 64-column boundaries every entry must be valid.
    const int2* b_nrange = nullptr;
};

// Optional per-thread profiling of the tensor-core GEMM launches: CUDA events
// around every k_tc_submul launch and a device counter of executed K steps.
struct GemmProfile {
    unsigned long long* d_steps = nullptr;  // device counters, one per launch
    int capacity = 0;                       // counters in d_steps
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
    std::vector<cudaEvent_t> split_events;  // per launch: before its limb splits
    std::vector<double> macs_per_step;      // per launch
    std::vector<int> shape;                 // per launch: M, N, K, batch
};
GemmProfile* gemm_profile();
void set_gemm_profile(GemmProfile* p);

int limbs_for(uint32_t p);
// bytes of device workspace the tensor-core path needs for the limb planes
size_t tc_workspace_bytes(uint32_t p, int32_t M, int32_t N, int32_t K, int32_t batch = 1);
// tensor-core path (odd p); enqueues on s, *err receives GBGPU_ETIMEDOUT if a
// bounded wait expired
int tc_submul(const TcGemmArgs& g, void* workspace, cudaStream_t s, int32_t* err,
              long long* launches);
// the same with an explicit tile shape (0 big, 1 small, 2 mid; tune.cu)
int tc_submul_shape(const TcGemmArgs& g, void* workspace, cudaStream_t s, int32_t* err,
                    long long* launches, int shape);
// the tile shape the autotuner's cache (or the built-in rule) picks for L, K
int tc_shape_for(int L, int K);
// CUDA-core path (any p)
int plain_submul(const TcGemmArgs& g, cudaStream_t s, long long* launches);

}  // namespace gbgpu
