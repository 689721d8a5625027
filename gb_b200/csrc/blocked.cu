// blocked.cu -- the tensor-core (blocked) form of the Macaulay reduction.
//
// The answer is the reduced row echelon form of the Schur complement
//   D' = D - C A^-1 B
// of the A|B / C|D split (A: the known pivots restricted to the left block,
// unit upper triangular; the reference reaches the same rows by reducing one
// C|D row at a time, src/la_ff_16.c:737-835 and :601-735).  Here every step is
// a dense block operation on residue matrices, and every O(n^3) step is the
// exact modular GEMM of tc_gemm.cu (int8 tensor cores):
//
//   1. Schur complement, right-looking over 128-column blocks k of A:
//        X_k  = W[:, k] A_kk^-1                  (GEMM with a precomputed
//                                                  block inverse)
//        W[:, >k] -= X_k P_k[:, >k]              (GEMM)
//      where W = [C | D] holds the C|D rows (sorted by lead, so only a prefix
//      of rows is active for block k) and P = [A | B] the known pivots.
//   2. Echelon of D' by claiming rounds: the first row of every lead column
//      becomes a normalised pivot; the other rows are reduced by the round's
//      new pivots with the same block elimination (gathered pivot columns),
//      which leaves them zero at every pivot column, and the nonzero ones
//      claim again.
//   3. Back substitution to reduced echelon form, blocks of 128 pivots from
//      the last to the first: U_k -= U_k[:, piv(>k)] R_(>k) (GEMM against the
//      already reduced later rows), then U_k = (U_k[:, piv(k)])^-1 U_k.
//   4. Compaction into CSR rows in descending lead order (plain.cu kernels).
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gbgpu.h"
#include "blocked.h"
#include "field.cuh"
#include "internal.h"
#include "kernels.h"
#include "tc_gemm.h"

namespace gbgpu {

constexpr int KB = 128;  // pivots per elimination block

// ---------------------------------------------------------------------------
// kernels

// scatter CSR rows rows[i] (i < n) into dense row i of out (columns
// [col0, col0 + width) only), out already zeroed
__global__ void k_densify(int32_t n, const int32_t* __restrict__ rows,
                          const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ cols,
                          const uint32_t* __restrict__ vals, int32_t col0, int32_t width,
                          uint32_t* out, int64_t ld) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < n; i += nwarps) {
        const int32_t r = rows ? rows[i] : i;
        uint32_t* o = out + (size_t)i * ld;
        for (int64_t k = row_ptr[r] + lane; k < row_ptr[r + 1]; k += 32) {
            const int32_t c = cols[k] - col0;
            if (c >= 0 && c < width) o[c] = vals[k];
        }
    }
}

// dense known-pivot matrix: row c of out = the pivot row of lead c
__global__ void k_densify_pivots(int32_t ncl, const int32_t* __restrict__ piv_row,
                                 const int64_t* __restrict__ row_ptr,
                                 const int32_t* __restrict__ cols,
                                 const uint32_t* __restrict__ vals, uint32_t* out, int64_t ld) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int c = warp; c < ncl; c += nwarps) {
        const int32_t r = piv_row[c];
        uint32_t* o = out + (size_t)c * ld;
        for (int64_t k = row_ptr[r] + lane; k < row_ptr[r + 1]; k += 32) o[cols[k]] = vals[k];
    }
}

// lead (first column) of each listed CSR row
__global__ void k_csr_leads(int32_t n, const int32_t* __restrict__ rows,
                            const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ cols,
                            int32_t* lead) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        lead[i] = cols[row_ptr[rows[i]]];
}

// number of entries of the sorted array `v` that are < bound[j], per j
__global__ void k_count_below(int32_t n, const int32_t* __restrict__ v, int32_t nb,
                              int32_t step, int32_t* out) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < nb; j += gridDim.x * blockDim.x) {
        const int32_t bound = (j + 1) * step;
        int lo = 0, hi = n;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (v[mid] < bound) lo = mid + 1;
            else hi = mid;
        }
        out[j] = lo;
    }
}

// -U^-1 mod p for unit upper triangular blocks.  Block b is read from
// src + b * stride_b with leading dimension ld (kb x kb, kb <= KB); the result
// goes to out + b * KB * KB (KB x KB, identity-padded).  One CTA per block,
// thread j solves column j by back substitution.
template <class F>
__global__ void __launch_bounds__(KB)
k_neg_inverse(const uint32_t* __restrict__ src, int64_t ld, int64_t stride_b, int32_t n_blocks,
              int32_t last_kb, uint32_t* out, F f) {
    extern __shared__ uint32_t inv_smem[];
    uint32_t(*U)[KB + 1] = (uint32_t(*)[KB + 1])inv_smem;
    uint32_t(*V)[KB + 1] = (uint32_t(*)[KB + 1])(inv_smem + KB * (KB + 1));
    const int b = blockIdx.x;
    const int kb = b == n_blocks - 1 ? last_kb : KB;
    const uint32_t* s = src + (size_t)b * stride_b;
    for (int t = threadIdx.x; t < KB * KB; t += blockDim.x) {
        const int i = t / KB, j = t % KB;
        uint32_t v;
        if (i < kb && j < kb) v = s[(size_t)i * ld + j];
        else v = i == j ? 1u : 0u;
        U[i][j] = v;
    }
    __syncthreads();
    const int j = threadIdx.x;
    // V[., j] solves U x = e_j; V[i][j] = -sum_{i<k<=j} U[i][k] V[k][j]
    V[j][j] = 1u;
    for (int i = KB - 1; i > j; --i) V[i][j] = 0u;
    for (int i = j - 1; i >= 0; --i) {
        uint32_t acc = 0;
        for (int k = i + 1; k <= j; ++k) {
            const uint32_t u = U[i][k];
            if (u) {
                const uint32_t t = f.mulmod(u, V[k][j]);
                acc = acc + t >= f.p ? acc + t - f.p : acc + t;
            }
        }
        V[i][j] = acc ? f.p - acc : 0u;
    }
    __syncthreads();
    uint32_t* o = out + (size_t)b * KB * KB;
    for (int t = threadIdx.x; t < KB * KB; t += blockDim.x) {
        const int i = t / KB, jj = t % KB;
        const uint32_t v = V[i][jj];
        o[t] = v ? f.p - v : 0u;  // -V
    }
}

// dst[i][j] = src[i][cols[j]]
__global__ void k_gather_cols(int32_t rows, int32_t n, const uint32_t* __restrict__ src,
                              int64_t lds, const int32_t* __restrict__ cols, uint32_t* dst,
                              int64_t ldd) {
    const int64_t total = (int64_t)rows * n;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / n;
        const int j = (int)(t % n);
        dst[i * ldd + j] = src[i * lds + cols[j]];
    }
}

// dst row i = src row rows[i] (n columns)
__global__ void k_gather_rows_dense(int32_t nrows, const int32_t* __restrict__ rows, int32_t n,
                                    const uint32_t* __restrict__ src, int64_t lds, uint32_t* dst,
                                    int64_t ldd) {
    const int64_t total = (int64_t)nrows * n;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / n;
        const int j = (int)(t % n);
        dst[i * ldd + j] = src[(int64_t)rows[i] * lds + j];
    }
}

// dst row rows[i] = src row i
__global__ void k_scatter_rows_dense(int32_t nrows, const int32_t* __restrict__ rows, int32_t n,
                                     const uint32_t* __restrict__ src, int64_t lds,
                                     uint32_t* dst, int64_t ldd) {
    const int64_t total = (int64_t)nrows * n;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / n;
        const int j = (int)(t % n);
        dst[(int64_t)rows[i] * ldd + j] = src[i * lds + j];
    }
}

// first nonzero column of every row (-1 for zero rows), one warp per row
__global__ void k_row_leads(int32_t rows, const int32_t* __restrict__ list, int32_t ncols,
                            const uint32_t* __restrict__ M, int64_t ld, int32_t* lead) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < rows; i += nwarps) {
        const int32_t r = list ? list[i] : i;
        const uint32_t* row = M + (size_t)r * ld;
        int found = -1;
        for (int base = 0; base < ncols; base += 32) {
            const int c = base + lane;
            const unsigned bal = __ballot_sync(0xffffffffu, c < ncols && row[c] != 0u);
            if (bal) {
                found = base + __ffs(bal) - 1;
                break;
            }
        }
        if (lane == 0) lead[r] = found;
    }
}

// scale each listed row by the inverse of its lead entry (warp per row)
template <class F>
__global__ void k_normalize_rows(int32_t n, const int32_t* __restrict__ list,
                                 const int32_t* __restrict__ lead, int32_t ncols, uint32_t* M,
                                 int64_t ld, F f) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < n; i += nwarps) {
        const int32_t r = list[i];
        const int32_t c0 = lead[r];
        uint32_t* row = M + (size_t)r * ld;
        const uint32_t inv = inverse_mod(row[c0], f.p);
        __syncwarp();
        for (int c = c0 + 1 + lane; c < ncols; c += 32) {
            const uint32_t v = row[c];
            if (v) row[c] = f.mulmod(v, inv);
        }
        __syncwarp();
        if (lane == 0) row[c0] = 1u;
    }
}

// claim[lead[r]] = min r over candidate rows
__global__ void k_claim_dense(int32_t n, const int32_t* __restrict__ cand,
                              const int32_t* __restrict__ lead, int32_t* claim) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        atomicMin(&claim[lead[cand[i]]], cand[i]);
}

// winners -> piv_of_col and flags; losers -> list
__global__ void k_split_claims(int32_t n, const int32_t* __restrict__ cand,
                               const int32_t* __restrict__ lead, const int32_t* __restrict__ claim,
                               int32_t* piv_of_col, int32_t* winner_flag, int32_t* losers,
                               int32_t* n_losers) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t r = cand[i];
        const int32_t c = lead[r];
        if (claim[c] == r) {
            piv_of_col[c] = r;
            winner_flag[c] = 1;
        } else {
            losers[atomicAdd(n_losers, 1)] = r;
        }
    }
}

// rows of `list` with lead >= 0 -> out
__global__ void k_keep_nonzero(int32_t n, const int32_t* __restrict__ list,
                               const int32_t* __restrict__ lead, int32_t* out, int32_t* n_out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (lead[list[i]] >= 0) out[atomicAdd(n_out, 1)] = list[i];
}

// columns with flag set, ascending, via a precomputed exclusive scan
__global__ void k_compact_cols(int32_t n, const int32_t* __restrict__ flag,
                               const int32_t* __restrict__ pos, int32_t* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flag[i]) out[pos[i]] = i;
}

// ---------------------------------------------------------------------------
// host helpers

struct Ctx {
    cudaStream_t s;
    uint32_t p;
    int form;
    int32_t* err;
    long long launches = 0;
    std::vector<void*> tmp;
    void* ws = nullptr;  // GEMM limb planes
    size_t ws_bytes = 0;

    template <class T>
    T* alloc(size_t n) {
        void* q = nullptr;
        if (cudaMallocAsync(&q, std::max<size_t>(n, 1) * sizeof(T), s) != cudaSuccess)
            return nullptr;
        tmp.push_back(q);
        return (T*)q;
    }
    void release() {
        for (void* q : tmp) cudaFreeAsync(q, s);
        tmp.clear();
        if (ws) cudaFreeAsync(ws, s);
        ws = nullptr;
        ws_bytes = 0;
    }
};

#define BL_CHECK(expr)                                                   \
    do {                                                                 \
        int rc_ = (expr);                                                \
        if (rc_) return rc_;                                             \
    } while (0)
#define BL_CUDA(expr)                                                    \
    do {                                                                 \
        cudaError_t e_ = (expr);                                         \
        if (e_ != cudaSuccess) {                                         \
            set_error(std::string(#expr) + ": " + cudaGetErrorString(e_)); \
            return GBGPU_ECUDA;                                          \
        }                                                                \
    } while (0)
#define BL_LAUNCH(...)                                                   \
    do {                                                                 \
        __VA_ARGS__;                                                     \
        ++c.launches;                                                    \
        BL_CUDA(cudaGetLastError());                                     \
    } while (0)

static int grid_of(int64_t n, int t = 256) {
    int64_t g = (n + t - 1) / t;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 16));
}

// D (M x N) -= A (M x K) B (K x N), exact mod p
static int gemm(Ctx& c, uint32_t* D, int64_t ldd, const uint32_t* A, int64_t lda,
                const uint32_t* B, int64_t ldb, int32_t M, int32_t N, int32_t K) {
    if (M <= 0 || N <= 0 || K <= 0) return GBGPU_OK;
    TcGemmArgs g{c.p, M, N, K, A, lda, B, ldb, D, ldd};
    if (c.form == GBGPU_FORM_PLAIN) return plain_submul(g, c.s, &c.launches);
    const size_t need = tc_workspace_bytes(c.p, M, N, K);
    if (need > c.ws_bytes) {
        if (c.ws) cudaFreeAsync(c.ws, c.s);
        c.ws = nullptr;
        const size_t bytes = std::max(need, c.ws_bytes * 2);
        if (cudaMallocAsync(&c.ws, bytes, c.s) != cudaSuccess) {
            set_error("GEMM workspace allocation failed");
            return GBGPU_ENOMEM;
        }
        c.ws_bytes = bytes;
    }
    return tc_submul(g, c.ws, c.s, c.err, &c.launches);
}

template <class F>
static int neg_inverse(Ctx& c, const F& f, const uint32_t* src, int64_t ld, int64_t stride_b,
                       int32_t n_blocks, int32_t last_kb, uint32_t* out) {
    if (n_blocks <= 0) return GBGPU_OK;
    const int bytes = 2 * KB * (KB + 1) * (int)sizeof(uint32_t);
    BL_CUDA(cudaFuncSetAttribute(k_neg_inverse<F>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    BL_LAUNCH(k_neg_inverse<F><<<n_blocks, KB, bytes, c.s>>>(src, ld, stride_b, n_blocks, last_kb, out, f));
    return GBGPU_OK;
}

// T (rows x ncols, ld) <- T - T[:, pc] (U[:, pc])^-1 U for pivot rows U
// (n_p x ncols, ld_u, sorted by lead, monic, zero left of their leads) with
// pivot columns pc (ascending): afterwards T is zero at every pivot column.
// Blocks of KB pivots, left to right.
template <class F>
static int eliminate(Ctx& c, const F& f, uint32_t* T, int64_t ldt, int32_t rows, int32_t ncols,
                     const uint32_t* U, int64_t ldu, int32_t n_p, const int32_t* d_pc,
                     const std::vector<int32_t>& pc) {
    if (rows <= 0 || n_p <= 0) return GBGPU_OK;
    const int32_t nb = (n_p + KB - 1) / KB;
    uint32_t* Ublk = c.alloc<uint32_t>((size_t)nb * KB * KB);   // U[:, pc] diagonal blocks
    uint32_t* Ninv = c.alloc<uint32_t>((size_t)nb * KB * KB);
    uint32_t* G = c.alloc<uint32_t>((size_t)rows * KB);         // T[:, pc_k]
    uint32_t* X = c.alloc<uint32_t>((size_t)rows * KB);
    if (!Ublk || !Ninv || !G || !X) return GBGPU_ENOMEM;
    for (int b = 0; b < nb; ++b) {
        const int kb = std::min(KB, n_p - b * KB);
        BL_LAUNCH(k_gather_cols<<<grid_of((int64_t)kb * kb), 256, 0, c.s>>>(
            kb, kb, U + (size_t)b * KB * ldu, ldu, d_pc + b * KB, Ublk + (size_t)b * KB * KB, KB));
    }
    BL_CHECK(neg_inverse(c, f, Ublk, KB, (int64_t)KB * KB, nb, n_p - (nb - 1) * KB, Ninv));
    for (int b = 0; b < nb; ++b) {
        const int kb = std::min(KB, n_p - b * KB);
        const int32_t first_col = pc[b * KB];
        BL_LAUNCH(k_gather_cols<<<grid_of((int64_t)rows * kb), 256, 0, c.s>>>(
            rows, kb, T, ldt, d_pc + b * KB, G, KB));
        BL_CUDA(cudaMemsetAsync(X, 0, sizeof(uint32_t) * (size_t)rows * KB, c.s));
        // X = G * (U_kk)^-1 = 0 - G * (-(U_kk)^-1)
        BL_CHECK(gemm(c, X, KB, G, KB, Ninv + (size_t)b * KB * KB, KB, rows, kb, kb));
        // T[:, first_col:] -= X * U_k[:, first_col:]
        BL_CHECK(gemm(c, T + first_col, ldt, X, KB, U + (size_t)b * KB * ldu + first_col, ldu, rows,
                      ncols - first_col, kb));
    }
    return GBGPU_OK;
}

// ---------------------------------------------------------------------------
template <class F>
static int blocked_run(const BlockedInput& in, BlockedOutput* out, Ctx& c, const F& f) {
    const int32_t ncl = in.ncl, ncr = in.ncr, nc = ncl + ncr, t = in.n_work;
    const int64_t ld = ((int64_t)nc + 3) & ~(int64_t)3;
    cudaStream_t s = c.s;

    // ---- 1. Schur complement ---------------------------------------------------
    // C|D rows sorted by lead (stable), dense
    int32_t* lead_in = c.alloc<int32_t>(t);
    int32_t* lead_sorted = c.alloc<int32_t>(t);
    int32_t* work_sorted = c.alloc<int32_t>(t);
    uint32_t* W = c.alloc<uint32_t>((size_t)t * ld);
    if (!lead_in || !lead_sorted || !work_sorted || !W) return GBGPU_ENOMEM;
    if (t > 0) {
        BL_LAUNCH(k_csr_leads<<<grid_of(t), 256, 0, s>>>(t, in.work, in.row_ptr, in.cols, lead_in));
        size_t bytes = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, bytes, lead_in, lead_sorted, in.work, work_sorted,
                                        t, 0, 32, s);
        void* tmp = c.alloc<uint8_t>(bytes);
        if (!tmp) return GBGPU_ENOMEM;
        BL_CUDA(cub::DeviceRadixSort::SortPairs(tmp, bytes, lead_in, lead_sorted, in.work,
                                                work_sorted, t, 0, 32, s));
        ++c.launches;
        BL_CUDA(cudaMemsetAsync(W, 0, sizeof(uint32_t) * (size_t)t * ld, s));
        BL_LAUNCH(k_densify<<<grid_of((int64_t)t * 32), 256, 0, s>>>(
            t, work_sorted, in.row_ptr, in.cols, in.vals, 0, nc, W, ld));
    }
    if (t > 0 && ncl > 0) {
        uint32_t* P = c.alloc<uint32_t>((size_t)ncl * ld);
        const int32_t nbk = (ncl + KB - 1) / KB;
        uint32_t* Ninv = c.alloc<uint32_t>((size_t)nbk * KB * KB);
        uint32_t* X = c.alloc<uint32_t>((size_t)t * KB);
        int32_t* act = c.alloc<int32_t>(nbk);
        if (!P || !Ninv || !X || !act) return GBGPU_ENOMEM;
        BL_CUDA(cudaMemsetAsync(P, 0, sizeof(uint32_t) * (size_t)ncl * ld, s));
        BL_LAUNCH(k_densify_pivots<<<grid_of((int64_t)ncl * 32), 256, 0, s>>>(
            ncl, in.piv_row, in.row_ptr, in.cols, in.vals, P, ld));
        // -A_kk^-1 of every diagonal block of A (read in place from P)
        BL_CHECK(neg_inverse(c, f, P, ld, (int64_t)KB * ld + KB, nbk, ncl - (nbk - 1) * KB, Ninv));
        BL_LAUNCH(k_count_below<<<grid_of(nbk), 256, 0, s>>>(t, lead_sorted, nbk, KB, act));
        std::vector<int32_t> h_act(nbk);
        BL_CUDA(cudaMemcpyAsync(h_act.data(), act, sizeof(int32_t) * nbk, cudaMemcpyDeviceToHost, s));
        BL_CUDA(cudaStreamSynchronize(s));
        for (int k = 0; k < nbk; ++k) {
            const int32_t c0 = k * KB, kb = std::min(KB, ncl - c0), c1 = c0 + kb;
            const int32_t rows = h_act[k];
            if (rows <= 0) continue;
            BL_CUDA(cudaMemsetAsync(X, 0, sizeof(uint32_t) * (size_t)rows * KB, s));
            // X = W[:, block] A_kk^-1
            BL_CHECK(gemm(c, X, KB, W + c0, ld, Ninv + (size_t)k * KB * KB, KB, rows, kb, kb));
            // W[:, c1:] -= X P[block rows, c1:]
            BL_CHECK(gemm(c, W + c1, ld, X, KB, P + (size_t)c0 * ld + c1, ld, rows, nc - c1, kb));
        }
        c.launches += 0;
    }
    if (out->ms_event_schur) BL_CUDA(cudaEventRecord(out->ms_event_schur, s));

    // ---- 2. echelon of D' = W[:, ncl:] by claiming rounds ----------------------
    uint32_t* Dp = W + ncl;  // t x ncr, leading dimension ld
    int32_t* lead = c.alloc<int32_t>(t);
    int32_t* claim = c.alloc<int32_t>(ncr);
    int32_t* piv_of_col = out->piv_of_col;  // [ncr], -1 if none
    int32_t* wflag = c.alloc<int32_t>(ncr);
    int32_t* wpos = c.alloc<int32_t>(ncr);
    int32_t* cand = c.alloc<int32_t>(t);
    int32_t* losers = c.alloc<int32_t>(t);
    int32_t* counters = c.alloc<int32_t>(4);
    int32_t* pc = c.alloc<int32_t>(ncr);      // pivot columns of the round
    int32_t* prow = c.alloc<int32_t>(ncr);    // their rows
    if (!lead || !claim || !wflag || !wpos || !cand || !losers || !counters || !pc || !prow)
        return GBGPU_ENOMEM;
    size_t scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, wflag, wpos, ncr, s);
    void* scan_tmp = c.alloc<uint8_t>(scan_bytes);
    if (!scan_tmp) return GBGPU_ENOMEM;
    BL_LAUNCH(k_fill_i32<<<grid_of(ncr), 256, 0, s>>>(piv_of_col, ncr, -1));
    int32_t n_cand = 0;
    if (t > 0 && ncr > 0) {
        BL_LAUNCH(k_row_leads<<<grid_of((int64_t)t * 32), 256, 0, s>>>(t, nullptr, ncr, Dp, ld, lead));
        BL_CUDA(cudaMemsetAsync(counters, 0, 4 * sizeof(int32_t), s));
        BL_LAUNCH(k_collect_nonzero<<<grid_of(t), 256, 0, s>>>(t, lead, cand, counters));
        BL_CUDA(cudaMemcpyAsync(&n_cand, counters, 4, cudaMemcpyDeviceToHost, s));
        BL_CUDA(cudaStreamSynchronize(s));
    }
    out->dense_rows = n_cand;
    int rounds = 0;
    uint32_t* Ubuf = nullptr;
    size_t ubuf_rows = 0;
    while (n_cand > 0) {
        ++rounds;
        BL_LAUNCH(k_fill_i32<<<grid_of(ncr), 256, 0, s>>>(claim, ncr, INT_MAX));
        BL_CUDA(cudaMemsetAsync(wflag, 0, sizeof(int32_t) * ncr, s));
        BL_CUDA(cudaMemsetAsync(counters, 0, 4 * sizeof(int32_t), s));
        BL_LAUNCH(k_claim_dense<<<grid_of(n_cand), 256, 0, s>>>(n_cand, cand, lead, claim));
        BL_LAUNCH(k_split_claims<<<grid_of(n_cand), 256, 0, s>>>(n_cand, cand, lead, claim,
                                                                piv_of_col, wflag, losers,
                                                                counters + 1));
        // new pivots, ascending columns
        BL_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, wflag, wpos, ncr, s));
        ++c.launches;
        BL_LAUNCH(k_compact_cols<<<grid_of(ncr), 256, 0, s>>>(ncr, wflag, wpos, pc));
        int32_t h[2] = {0, 0};
        BL_CUDA(cudaMemcpyAsync(&h[1], counters + 1, 4, cudaMemcpyDeviceToHost, s));
        int32_t last_pos = 0, last_flag = 0;
        BL_CUDA(cudaMemcpyAsync(&last_pos, wpos + ncr - 1, 4, cudaMemcpyDeviceToHost, s));
        BL_CUDA(cudaMemcpyAsync(&last_flag, wflag + ncr - 1, 4, cudaMemcpyDeviceToHost, s));
        BL_CUDA(cudaStreamSynchronize(s));
        const int32_t n_new = last_pos + last_flag, n_lost = h[1];
        // normalise the new pivots
        BL_LAUNCH(k_gather_rows<<<grid_of(n_new), 256, 0, s>>>(n_new, pc, piv_of_col, prow,
                                                               counters + 2));
        BL_LAUNCH(k_normalize_rows<F><<<grid_of((int64_t)n_new * 32), 256, 0, s>>>(
            n_new, prow, lead, ncr, Dp, ld, f));
        if (n_lost == 0) break;
        // losers -= (losers at pivot columns) (pivots at pivot columns)^-1 pivots
        std::vector<int32_t> h_pc(n_new);
        BL_CUDA(cudaMemcpyAsync(h_pc.data(), pc, sizeof(int32_t) * n_new, cudaMemcpyDeviceToHost, s));
        if ((size_t)n_new > ubuf_rows || (size_t)n_lost > ubuf_rows) {
            ubuf_rows = std::max<size_t>(std::max(n_new, n_lost), ubuf_rows * 2);
            Ubuf = c.alloc<uint32_t>(ubuf_rows * ld * 2);
            if (!Ubuf) return GBGPU_ENOMEM;
        }
        uint32_t* Ucmp = Ubuf;                        // pivot rows, compact
        uint32_t* Tcmp = Ubuf + ubuf_rows * ld;       // loser rows, compact
        BL_LAUNCH(k_gather_rows_dense<<<grid_of((int64_t)n_new * ncr), 256, 0, s>>>(
            n_new, prow, ncr, Dp, ld, Ucmp, ld));
        BL_LAUNCH(k_gather_rows_dense<<<grid_of((int64_t)n_lost * ncr), 256, 0, s>>>(
            n_lost, losers, ncr, Dp, ld, Tcmp, ld));
        BL_CUDA(cudaStreamSynchronize(s));
        BL_CHECK(eliminate(c, f, Tcmp, ld, n_lost, ncr, Ucmp, ld, n_new, pc, h_pc));
        BL_LAUNCH(k_scatter_rows_dense<<<grid_of((int64_t)n_lost * ncr), 256, 0, s>>>(
            n_lost, losers, ncr, Tcmp, ld, Dp, ld));
        // nonzero losers claim again
        BL_LAUNCH(k_row_leads<<<grid_of((int64_t)n_lost * 32), 256, 0, s>>>(n_lost, losers, ncr,
                                                                             Dp, ld, lead));
        BL_CUDA(cudaMemsetAsync(counters + 3, 0, sizeof(int32_t), s));
        BL_LAUNCH(k_keep_nonzero<<<grid_of(n_lost), 256, 0, s>>>(n_lost, losers, lead, cand,
                                                                 counters + 3));
        BL_CUDA(cudaMemcpyAsync(&n_cand, counters + 3, 4, cudaMemcpyDeviceToHost, s));
        BL_CUDA(cudaStreamSynchronize(s));
    }
    out->echelon_rounds = rounds;
    if (out->ms_event_echelon) BL_CUDA(cudaEventRecord(out->ms_event_echelon, s));

    // ---- 3. back substitution --------------------------------------------------
    // all pivots in ascending column order
    BL_LAUNCH(k_pivot_flags<<<grid_of(ncr), 256, 0, s>>>(ncr, piv_of_col, 0, wflag));
    BL_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, wflag, wpos, ncr, s));
    ++c.launches;
    BL_LAUNCH(k_compact_cols<<<grid_of(ncr), 256, 0, s>>>(ncr, wflag, wpos, pc));
    int32_t r = 0;
    if (ncr > 0) {
        int32_t last_pos = 0, last_flag = 0;
        BL_CUDA(cudaMemcpyAsync(&last_pos, wpos + ncr - 1, 4, cudaMemcpyDeviceToHost, s));
        BL_CUDA(cudaMemcpyAsync(&last_flag, wflag + ncr - 1, 4, cudaMemcpyDeviceToHost, s));
        BL_CUDA(cudaStreamSynchronize(s));
        r = last_pos + last_flag;
    }
    out->rank = r;
    if (r > 0) {
        std::vector<int32_t> h_pc(r);
        BL_CUDA(cudaMemcpyAsync(h_pc.data(), pc, sizeof(int32_t) * r, cudaMemcpyDeviceToHost, s));
        BL_CUDA(cudaStreamSynchronize(s));
        BL_LAUNCH(k_gather_rows<<<grid_of(r), 256, 0, s>>>(r, pc, piv_of_col, prow, counters + 2));
        // compact echelon rows E (r x ncr), ascending lead
        uint32_t* E = c.alloc<uint32_t>((size_t)r * ld);
        const int32_t nb = (r + KB - 1) / KB;
        uint32_t* Ublk = c.alloc<uint32_t>((size_t)nb * KB * KB);
        uint32_t* Ninv = c.alloc<uint32_t>((size_t)nb * KB * KB);
        uint32_t* G = c.alloc<uint32_t>((size_t)KB * std::max(r, 1));
        uint32_t* Y = c.alloc<uint32_t>((size_t)KB * ld);
        if (!E || !Ublk || !Ninv || !G || !Y) return GBGPU_ENOMEM;
        BL_LAUNCH(k_gather_rows_dense<<<grid_of((int64_t)r * ncr), 256, 0, s>>>(r, prow, ncr, Dp,
                                                                                ld, E, ld));
        for (int b = 0; b < nb; ++b) {
            const int kb = std::min(KB, r - b * KB);
            BL_LAUNCH(k_gather_cols<<<grid_of((int64_t)kb * kb), 256, 0, s>>>(
                kb, kb, E + (size_t)b * KB * ld, ld, pc + b * KB, Ublk + (size_t)b * KB * KB, KB));
        }
        BL_CHECK(neg_inverse(c, f, Ublk, KB, (int64_t)KB * KB, nb, r - (nb - 1) * KB, Ninv));
        for (int b = nb - 1; b >= 0; --b) {
            const int kb = std::min(KB, r - b * KB);
            const int32_t later = r - (b * KB + kb);
            uint32_t* Ek = E + (size_t)b * KB * ld;
            const int32_t c0 = h_pc[b * KB];
            if (later > 0) {
                // Ek -= Ek[:, pc(>k)] R(>k)
                BL_LAUNCH(k_gather_cols<<<grid_of((int64_t)kb * later), 256, 0, s>>>(
                    kb, later, Ek, ld, pc + b * KB + kb, G, later));
                const int32_t c_later = h_pc[b * KB + kb];
                BL_CHECK(gemm(c, Ek + c_later, ld, G, later, E + (size_t)(b * KB + kb) * ld + c_later,
                              ld, kb, ncr - c_later, later));
            }
            // Ek = (Ek[:, pc(k)])^-1 Ek = Ek - (-(U_kk)^-1 - I) ... computed as
            // Y = 0 - (-(U_kk)^-1) Ek, then Ek = Y
            BL_CUDA(cudaMemsetAsync(Y, 0, sizeof(uint32_t) * (size_t)KB * ld, s));
            BL_CHECK(gemm(c, Y + c0, ld, Ninv + (size_t)b * KB * KB, KB, Ek + c0, ld, kb, ncr - c0, kb));
            BL_CUDA(cudaMemcpy2DAsync(Ek + c0, ld * 4, Y + c0, ld * 4, (size_t)(ncr - c0) * 4, kb,
                                      cudaMemcpyDeviceToDevice, s));
        }
        // reduced rows back to their D' slots for the compaction
        BL_LAUNCH(k_scatter_rows_dense<<<grid_of((int64_t)r * ncr), 256, 0, s>>>(r, prow, ncr, E,
                                                                                 ld, Dp, ld));
    }
    out->rows = Dp;
    out->ld = ld;
    return GBGPU_OK;
}

int blocked_reduce(const BlockedInput& in, BlockedOutput* out, long long* launches) {
    Ctx c;
    c.s = in.stream;
    c.p = in.p;
    c.form = in.form;
    c.err = in.err;
    int rc;
    if (in.p < 65536u)
        rc = blocked_run(in, out, c, FieldSmall::make(in.p));
    else
        rc = blocked_run(in, out, c, FieldMont::make(in.p));
    *launches += c.launches;
    out->keep = new std::vector<void*>(c.tmp);
    if (c.ws) out->keep->push_back(c.ws);
    return rc;
}

void blocked_release(BlockedOutput* out, cudaStream_t s) {
    if (!out->keep) return;
    for (void* q : *out->keep) cudaFreeAsync(q, s);
    delete out->keep;
    out->keep = nullptr;
}

}  // namespace gbgpu
