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
//   1. Schur complement.  W = [C | D] holds the C|D rows sorted by lead (so
//      only a prefix of rows is active for a block of A), P = [A | B] the known
//      pivots.  (a) X = C A^-1, right-looking over 128-column blocks k of A:
//        X_k = W[:, k] A_kk^-1                   (GEMM, precomputed block inverse)
//        W[:, k+1 .. e_k] -= X_k A[k, k+1 .. e_k] (GEMM; e_k = last left column the
//                                                  pivots of block k touch)
//      with X_k stored over W[:, k]; (b) D' = D - X B as one GEMM whose zero
//      tiles (staircase X, banded B) are skipped.
//   2. Echelon of D': one claim round first (the first row of every distinct
//      lead becomes a pivot, all other rows are eliminated against these at
//      once), then 128-column panels, left to right, for the rows that remain:
//      the pending rows whose lead lies in the panel (128 at a time) are brought to echelon form
//      inside the panel in shared memory (k_panel_factor), the recorded row
//      transformation is applied to their trailing columns with one GEMM, the
//      pivots found are registered, and the panel's other pending rows are
//      eliminated against them (eliminate: gathered pivot columns, block
//      inverses, GEMMs).
//   3. Back substitution to reduced echelon form, blocks of 128 pivots from
//      the last to the first: U_k -= U_k[:, piv(>k)] R_(>k) (GEMM against the
//      already reduced later rows), then U_k = (U_k[:, piv(k)])^-1 U_k.
//   4. Compaction into CSR rows in descending lead order (plain.cu kernels).
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <cub/iterator/counting_input_iterator.cuh>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gbgpu.h"
#include "blocked.h"
#include "common.cuh"
#include "field.cuh"
#include "internal.h"
#include "kernels.h"
#include "tc_gemm.h"

namespace gbgpu {

constexpr int KB = 128;  // pivots per elimination block

// per-round statistics of the echelon on stderr when GBGPU_DEBUG is set
static bool trace_rounds() {
    static const bool on = getenv("GBGPU_DEBUG") != nullptr;
    return on;
}

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

// Dense rows from CSR without a separate clear: row i of out (i < n) receives
// CSR row rows[i], columns [from_i, nc), from_i = (i / stride) stride (0 when
// stride is 0); columns left of from_i are not written.  Each CTA assembles
// DS_COLS-column segments of a row in shared memory and writes them whole
// with 16-byte stores (ld a multiple of 4, out 16-byte aligned).
constexpr int DS_COLS = 16384;
__global__ void __launch_bounds__(512)
k_densify_seg(int32_t n, const int32_t* __restrict__ rows, const int64_t* __restrict__ row_ptr,
              const int32_t* __restrict__ cols, const uint32_t* __restrict__ vals, int32_t nc,
              int32_t stride, uint32_t* out, int64_t ld) {
    extern __shared__ uint4 ds_smem[];
    uint32_t* seg = (uint32_t*)ds_smem;
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const int32_t r = rows ? rows[i] : i;
        const int64_t b = row_ptr[r], e = row_ptr[r + 1];
        const int32_t from = stride ? (i / stride) * stride : 0;
        uint32_t* o = out + (size_t)i * ld;
        for (int32_t s0 = from; s0 < nc; s0 += DS_COLS) {
            const int32_t w = min(DS_COLS, nc - s0);
            for (int j = threadIdx.x; j < (w + 3) / 4; j += blockDim.x)
                ds_smem[j] = make_uint4(0u, 0u, 0u, 0u);
            __syncthreads();
            for (int64_t k = b + threadIdx.x; k < e; k += blockDim.x) {
                const int32_t c = cols[k] - s0;
                if (c >= 0 && c < w) seg[c] = vals[k];
            }
            __syncthreads();
            uint4* o4 = (uint4*)(o + s0);
            for (int j = threadIdx.x; j < w / 4; j += blockDim.x) o4[j] = ds_smem[j];
            for (int j = (w / 4) * 4 + threadIdx.x; j < w; j += blockDim.x) o[s0 + j] = seg[j];
            __syncthreads();
        }
    }
}

// The same rows without shared memory, for the known pivots (whose written
// intervals are short): a CTA takes a row:
// it fills each interval with zeros (16-byte stores; ld a multiple of 4, out
// 16-byte aligned), waits at a barrier (the zeros are then ordered before any
// later store of the CTA) and scatters the row's entries of the interval
// straight into place.  Every entry is read once per interval.
//
// With split > 0 (the known pivots P = [A | B] of the tensor form, whose
// readers need less) only two column intervals of row i are written:
//   [from_i, e1), e1 = min(split, max(from_i + stride, span[i / stride] + 1)):
//       the diagonal block and the left columns the block's rows reach;
//   [split + lo, split + hi): the right columns of row group i / 128, from
//       brange[i / 128] = (first, last) nonzero right column of the group,
//       widened to 64-column boundaries (the limb split reads whole
//       64-column blocks); nothing when the group's right part is zero.
// Everything else in the row is left as it was: its readers (the block
// inverses, the block solves and the limb split of the Schur product's B)
// never look there.
constexpr int DS_THREADS = 256;
__global__ void __launch_bounds__(DS_THREADS)
k_densify_direct(int32_t n, const int32_t* __restrict__ rows, const int64_t* __restrict__ row_ptr,
              const int32_t* __restrict__ cols, const uint32_t* __restrict__ vals, int32_t nc,
              int32_t stride, uint32_t* out, int64_t ld, int32_t split = 0,
              const int32_t* __restrict__ span = nullptr,
              const int2* __restrict__ brange = nullptr) {
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const int32_t r = rows ? rows[i] : i;
        const int64_t b = row_ptr[r], e = row_ptr[r + 1];
        const int32_t from = stride ? (i / stride) * stride : 0;
        uint32_t* o = out + (size_t)i * ld;
        // the (one or two) intervals of this row
        int32_t iv[2][2] = {{from, nc}, {0, 0}};
        int n_iv = 1;
        if (split > 0) {
            int32_t e1 = split;
            if (span && stride) e1 = min(split, max(from + stride, span[i / stride] + 1));
            iv[0][1] = e1;
            const int2 br = brange[i / 128];
            if (br.y >= br.x) {
                const int32_t lo = split + (br.x / 64) * 64;
                const int32_t hi = min(nc, split + (br.y / 64 + 1) * 64);
                const int32_t s = lo & ~3;
                if (s <= e1) {
                    iv[0][1] = max(e1, hi);
                } else {
                    iv[1][0] = s;
                    iv[1][1] = hi;
                    n_iv = 2;
                }
            }
        }
        for (int q = 0; q < n_iv; ++q) {
            const int32_t a0 = iv[q][0], a1 = iv[q][1];  // a0 is a multiple of 4
            const int32_t w4 = (a1 - a0) / 4;
            uint4* o4 = (uint4*)(o + a0);
            for (int j = threadIdx.x; j < w4; j += blockDim.x) o4[j] = make_uint4(0u, 0u, 0u, 0u);
            for (int32_t j = a0 + 4 * w4 + threadIdx.x; j < a1; j += blockDim.x) o[j] = 0u;
            __syncthreads();
            for (int64_t k = b + threadIdx.x; k < e; k += blockDim.x) {
                const int32_t c = cols[k];
                if (c >= a0 && c < a1) o[c] = vals[k];
            }
        }
        __syncthreads();  // this row's stores are done before the CTA's next row
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

// span[b] = largest column < limit of the known pivots of rows [bs b, bs b + bs);
// with brange, also the first and last column >= limit (as column - limit)
// of every group of 128 rows, (INT_MAX, -1) filled in before
__global__ void k_block_span(int32_t ncl, const int32_t* __restrict__ piv_row,
                             const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ cols,
                             int32_t limit, int32_t bs, int32_t* span, int2* brange = nullptr) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int c = warp; c < ncl; c += nwarps) {
        const int32_t r = piv_row[c];
        int32_t mx = -1, blo = INT_MAX, bhi = -1;
        for (int64_t k = row_ptr[r] + lane; k < row_ptr[r + 1]; k += 32) {
            const int32_t col = cols[k];
            if (col < limit) {
                mx = max(mx, col);
            } else {
                blo = min(blo, col - limit);
                bhi = max(bhi, col - limit);
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            blo = min(blo, __shfl_xor_sync(0xffffffffu, blo, o));
            bhi = max(bhi, __shfl_xor_sync(0xffffffffu, bhi, o));
        }
        if (lane == 0 && mx >= 0) atomicMax(&span[c / bs], mx);
        if (lane == 0 && brange && bhi >= 0) {
            atomicMin(&brange[c / 128].x, blo);
            atomicMax(&brange[c / 128].y, bhi);
        }
    }
}

// every range empty: (INT_MAX, -1)
__global__ void k_clear_ranges(int32_t n, int2* r) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        r[i] = make_int2(INT_MAX, -1);
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

// x mod p for any 64-bit x (p < 2^31) by Barrett reduction with
// m = floor((2^64 - 1) / p): the estimated quotient is at most 2 short.
__device__ __forceinline__ uint32_t mod64(uint64_t x, uint32_t p, uint64_t m) {
    const uint64_t q = __umul64hi(x, m);
    uint64_t r = x - q * p;
    r = r >= p ? r - p : r;
    r = r >= p ? r - p : r;
    return (uint32_t)r;
}

constexpr int INV_THREADS = 1024;  // threads of k_neg_inverse

// sum of u_k v_k mod p for u_k, v_k < p < 2^31, from 16-bit halves of v
// accumulated without reduction (each product < 2^47, at most 128 terms)
__device__ __forceinline__ uint32_t fold_lohi(uint64_t lo, uint64_t hi, uint32_t p, uint64_t m) {
    const uint32_t hr = mod64(hi, p, m);
    return mod64((uint64_t)mod64(lo, p, m) + ((uint64_t)hr << 16), p, m);
}

// sum_{k in [k0, k1)} a[k sa] b[k sb] mod p (residues < p < 2^31), two
// independent 16-bit-split accumulator pairs
__device__ __forceinline__ uint32_t dot_lohi(const uint32_t* a, int sa, const uint32_t* b, int sb,
                                             int k0, int k1, uint32_t p, uint64_t m) {
    uint64_t lo0 = 0, hi0 = 0, lo1 = 0, hi1 = 0;
    int k = k0;
    for (; k + 1 < k1; k += 2) {
        const uint32_t u0 = a[k * sa], v0 = b[k * sb];
        const uint32_t u1 = a[(k + 1) * sa], v1 = b[(k + 1) * sb];
        lo0 += (uint64_t)u0 * (v0 & 0xFFFFu);
        hi0 += (uint64_t)u0 * (v0 >> 16);
        lo1 += (uint64_t)u1 * (v1 & 0xFFFFu);
        hi1 += (uint64_t)u1 * (v1 >> 16);
    }
    if (k < k1) {
        const uint32_t u0 = a[k * sa], v0 = b[k * sb];
        lo0 += (uint64_t)u0 * (v0 & 0xFFFFu);
        hi0 += (uint64_t)u0 * (v0 >> 16);
    }
    return fold_lohi(lo0 + lo1, hi0 + hi1, p, m);
}

// -U^-1 mod p for unit upper triangular blocks.  Block b is read from
// src + b * stride_b with leading dimension ld (kb x kb, kb <= KB); the result
// (KB x KB, identity-padded) goes to out + b * ostride with leading dimension
// old.  One CTA per block, V = U^-1 built by doubling in shared memory: the
// 8 x 8 diagonal blocks by back substitution, then for sz = 8, 16, 32, 64
// every 2sz x 2sz diagonal block [[A, B], [0, C]] gets its top-right part
// -A^-1 B C^-1 as two small products (T = B C^-1, then -A^-1 T).
template <class F>
__global__ void __launch_bounds__(INV_THREADS)
k_neg_inverse(const uint32_t* __restrict__ src, int64_t ld, int64_t stride_b, int32_t n_blocks,
              int32_t last_kb, uint32_t* out, int64_t ostride, int64_t old, F f) {
    extern __shared__ uint32_t inv_smem[];
    uint32_t(*U)[KB + 1] = (uint32_t(*)[KB + 1])inv_smem;
    uint32_t(*V)[KB + 1] = (uint32_t(*)[KB + 1])(inv_smem + KB * (KB + 1));
    uint32_t* T = inv_smem + 2 * KB * (KB + 1);  // KB * KB / 4 entries
    const int b = blockIdx.x;
    const int kb = b == n_blocks - 1 ? last_kb : KB;
    const uint32_t* s = src + (size_t)b * stride_b;
    const int tid = threadIdx.x;
    // the block: KB * KB / blockDim.x entries per thread, all loads in flight
    constexpr int PER = KB * KB / INV_THREADS;
    {
        uint32_t v[PER];
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const int t = tid + q * INV_THREADS;
            const int i = t / KB, j = t % KB;
            v[q] = (i < kb && j < kb) ? s[(size_t)i * ld + j] : (i == j ? 1u : 0u);
        }
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const int t = tid + q * INV_THREADS;
            const int i = t / KB, j = t % KB;
            U[i][j] = v[q];
            V[i][j] = i == j ? 1u : 0u;
        }
    }
    __syncthreads();
    const uint32_t p = f.p;
    const uint64_t m = ~0ull / p;
    if (tid < KB) {
        // 8 x 8 diagonal blocks: V[i][j] = -sum_{i<k<=j} U[i][k] V[k][j]
        const int b0 = tid & ~7, j = b0 + (tid & 7);
        for (int i = j - 1; i >= b0; --i) {
            uint64_t lo = 0, hi = 0;
            for (int k = i + 1; k <= j; ++k) {
                const uint32_t u = U[i][k];
                const uint32_t v = V[k][j];
                lo += (uint64_t)u * (v & 0xFFFFu);
                hi += (uint64_t)u * (v >> 16);
            }
            const uint32_t acc = fold_lohi(lo, hi, p, m);
            V[i][j] = acc ? p - acc : 0u;
        }
    }
    __syncthreads();
    for (int sz = 8; sz < KB; sz *= 2) {
        const int per = sz * sz, total = (KB / (2 * sz)) * per;
        // T = B C^-1 (C^-1 upper triangular: k <= j)
        for (int e = tid; e < total; e += blockDim.x) {
            const int b0 = (e / per) * 2 * sz, i = (e % per) / sz, j = e % sz;
            const uint32_t* urow = &U[b0 + i][b0 + sz];
            const uint32_t* vcol = &V[b0 + sz][b0 + sz + j];
            T[e] = dot_lohi(urow, 1, vcol, KB + 1, 0, j + 1, p, m);
        }
        __syncthreads();
        // top-right of V = -A^-1 T (A^-1 upper triangular: k >= i)
        for (int e = tid; e < total; e += blockDim.x) {
            const int pr = e / per, b0 = pr * 2 * sz, i = (e % per) / sz, j = e % sz;
            const uint32_t* Tp = T + pr * per;
            const uint32_t acc =
                dot_lohi(&V[b0 + i][b0], 1, Tp + j, sz, i, sz, p, m);
            V[b0 + i][b0 + sz + j] = acc ? p - acc : 0u;
        }
        __syncthreads();
    }
    uint32_t* o = out + (size_t)b * ostride;
    for (int t = tid; t < KB * KB; t += blockDim.x) {
        const int i = t / KB, jj = t % KB;
        const uint32_t v = V[i][jj];
        o[(size_t)i * old + jj] = v ? f.p - v : 0u;  // -V
    }
}

// The row copies below give every piece of GB_PIECE columns of a row to one
// warp (32-bit index arithmetic, four independent loads per lane in flight);
// the loop body sees the row i and its columns [jb, je).
constexpr int GB_PIECE = 512;
#define GB_WARP_ROWS(rows, ncols)                                                    \
    const int lane = threadIdx.x & 31;                                               \
    const int warp_ = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;                  \
    const int nwarps_ = (gridDim.x * blockDim.x) >> 5;                               \
    const int npc_ = ((ncols) + GB_PIECE - 1) / GB_PIECE;                            \
    for (int it_ = warp_, i = it_ / max(npc_, 1), jb = (it_ % max(npc_, 1)) * GB_PIECE, \
             je = min((int)(ncols), jb + GB_PIECE);                                  \
         it_ < (rows) * npc_;                                                        \
         it_ += nwarps_, i = it_ / max(npc_, 1), jb = (it_ % max(npc_, 1)) * GB_PIECE, \
             je = min((int)(ncols), jb + GB_PIECE))

// dst[i][j] = src[r_i][cols[j]], r_i = rlist[i] (i without a list)
__global__ void k_gather_cols(int32_t rows, int32_t n, const uint32_t* __restrict__ src,
                              int64_t lds, const int32_t* __restrict__ cols, uint32_t* dst,
                              int64_t ldd, const int32_t* __restrict__ rlist = nullptr) {
    GB_WARP_ROWS(rows, n) {
        const uint32_t* s = src + (size_t)(rlist ? rlist[i] : i) * lds;
        uint32_t* o = dst + (size_t)i * ldd;
        for (int j0 = jb + lane; j0 < je; j0 += 128) {
            uint32_t v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int jj = j0 + 32 * u;
                v[u] = jj < je ? s[cols[jj]] : 0u;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (j0 + 32 * u < je) o[j0 + 32 * u] = v[u];
        }
    }
}

// dst row i = src row rows[i] (n columns; a negative index: a zero row)
__global__ void k_gather_rows_dense(int32_t nrows, const int32_t* __restrict__ rows, int32_t n,
                                    const uint32_t* __restrict__ src, int64_t lds, uint32_t* dst,
                                    int64_t ldd) {
    GB_WARP_ROWS(nrows, n) {
        const int32_t r = rows[i];
        const uint32_t* s = r >= 0 ? src + (size_t)r * lds : nullptr;
        uint32_t* o = dst + (size_t)i * ldd;
        for (int j0 = jb + lane; j0 < je; j0 += 128) {
            uint32_t v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int jj = j0 + 32 * u;
                v[u] = (s && jj < je) ? s[jj] : 0u;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (j0 + 32 * u < je) o[j0 + 32 * u] = v[u];
        }
    }
}

// dst row rows[i] = src row i
__global__ void k_scatter_rows_dense(int32_t nrows, const int32_t* __restrict__ rows, int32_t n,
                                     const uint32_t* __restrict__ src, int64_t lds,
                                     uint32_t* dst, int64_t ldd) {
    GB_WARP_ROWS(nrows, n) {
        const uint32_t* s = src + (size_t)i * lds;
        uint32_t* o = dst + (size_t)rows[i] * ldd;
        for (int j0 = jb + lane; j0 < je; j0 += 128) {
            uint32_t v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int jj = j0 + 32 * u;
                v[u] = jj < je ? s[jj] : 0u;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (j0 + 32 * u < je) o[j0 + 32 * u] = v[u];
        }
    }
}

// first nonzero column of every row (-1 for zero rows), one warp per row;
// with from_prev the scan starts at the row's current lead (leads only move
// right under elimination).  A pass covers LEAD_U chunks of 32 columns whose
// loads are in flight together.
constexpr int LEAD_U = 8;
__global__ void k_row_leads(int32_t rows, const int32_t* __restrict__ list, int32_t ncols,
                            const uint32_t* __restrict__ M, int64_t ld, int32_t* lead,
                            int32_t from_prev = 0) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < rows; i += nwarps) {
        const int32_t r = list ? list[i] : i;
        const uint32_t* row = M + (size_t)r * ld;
        int found = -1;
        const int start = from_prev && lead[r] > 0 ? lead[r] : 0;
        for (int base = start; base < ncols && found < 0; base += 32 * LEAD_U) {
            uint32_t v[LEAD_U];
#pragma unroll
            for (int u = 0; u < LEAD_U; ++u) {
                const int c = base + 32 * u + lane;
                v[u] = c < ncols ? row[c] : 0u;
            }
#pragma unroll
            for (int u = 0; u < LEAD_U; ++u) {
                const unsigned bal = __ballot_sync(0xffffffffu, v[u] != 0u);
                if (bal && found < 0) found = base + 32 * u + __ffs(bal) - 1;
            }
        }
        if (lane == 0) lead[r] = found;
    }
}

// columns with flag set, ascending, via a precomputed exclusive scan
__global__ void k_compact_cols(int32_t n, const int32_t* __restrict__ flag,
                               const int32_t* __restrict__ pos, int32_t* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (flag[i]) out[pos[i]] = i;
}


// ---------------------------------------------------------------------------
// panel echelon

// pending rows: nonzero and not yet pivots
__global__ void k_collect_pending(int32_t t, const int32_t* __restrict__ lead,
                                  const uint8_t* __restrict__ is_piv, int32_t* pend,
                                  int32_t* n_pend) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < t; r += gridDim.x * blockDim.x)
        if (lead[r] >= 0 && !is_piv[r]) pend[atomicAdd(n_pend, 1)] = r;
}

// the round's new pivots: count = last exclusive-scan position + last flag,
// and their rows in ascending pivot-column order
__global__ void k_new_pivots(int32_t ncr, const int32_t* __restrict__ wflag,
                             const int32_t* __restrict__ wpos, const int32_t* __restrict__ pc,
                             const int32_t* __restrict__ piv_of_col, int32_t* n_new,
                             int32_t* prow) {
    const int32_t n = ncr > 0 ? wpos[ncr - 1] + wflag[ncr - 1] : 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        prow[i] = piv_of_col[pc[i]];
    if (blockIdx.x == 0 && threadIdx.x == 0) *n_new = n;
}

// pending flags for an ordered compaction (rows in ascending order)
__global__ void k_pending_flags(int32_t t, const int32_t* __restrict__ lead,
                                const uint8_t* __restrict__ is_piv, uint8_t* flag) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < t; r += gridDim.x * blockDim.x)
        flag[r] = (lead[r] >= 0 && !is_piv[r]) ? 1 : 0;
}

// chunk slot key of every pending row: its panel's slot, n_dirty for rows of
// panels not factorized this round
__global__ void k_panel_keys(int32_t n, const int32_t* __restrict__ pend,
                             const int32_t* __restrict__ lead, const int32_t* __restrict__ dslot,
                             int32_t n_dirty, int32_t* key) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t d = dslot[lead[pend[i]] / KB];
        key[i] = d >= 0 ? d : n_dirty;
    }
}

// rows sorted by (chunk slot, row): the first KB rows of every selected panel
// fill its chunk in ascending row order; cursor = the panel's pending rows
__global__ void k_bucket_sorted(int32_t n, const int32_t* __restrict__ key,
                                const int32_t* __restrict__ rows, int32_t n_dirty,
                                int32_t* chunk_rows, int32_t* cursor) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
        const int32_t d = key[q];
        if (d >= n_dirty) continue;
        int lo = 0, hi = q;  // first position of this run
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (key[mid] < d) lo = mid + 1;
            else hi = mid;
        }
        const int slot = q - lo;
        if (slot < KB) chunk_rows[d * KB + slot] = rows[q];
        if (q == n - 1 || key[q + 1] != d) cursor[d] = q - lo + 1;
    }
}

// rows per lead column and per 128-column panel; a panel is "dirty" when
// two pending rows share a lead in it
__global__ void k_lead_hist(const int32_t* __restrict__ n_dev, const int32_t* __restrict__ pend,
                            const int32_t* __restrict__ lead, int32_t* hist, int32_t* pcnt) {
    const int32_t n = *n_dev;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t l = lead[pend[i]];
        atomicAdd(&hist[l], 1);
        atomicAdd(&pcnt[l / KB], 1);
    }
}
__global__ void k_dirty_panels(const int32_t* __restrict__ n_dev, const int32_t* __restrict__ pend,
                               const int32_t* __restrict__ lead, const int32_t* __restrict__ hist,
                               int32_t* pdirty) {
    const int32_t n = *n_dev;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t l = lead[pend[i]];
        if (hist[l] > 1) pdirty[l / KB] = 1;
    }
}

// rows of collision-free panels have leads of their own: they are pivots
__global__ void k_claim_clean(const int32_t* __restrict__ n_dev, const int32_t* __restrict__ pend,
                              const int32_t* __restrict__ lead, const int32_t* __restrict__ pdirty,
                              int32_t* piv_of_col, uint8_t* is_piv, int32_t* wflag) {
    const int32_t n = *n_dev;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t r = pend[i], l = lead[r];
        if (!pdirty[l / KB]) {
            piv_of_col[l] = r;
            is_piv[r] = 1;
            wflag[l] = 1;
        }
    }
}

// pending rows of the selected dirty panels (dslot[p] >= 0) into their
// panel's chunk (at most KB rows; the others stay pending)
__global__ void k_bucket_dirty(int32_t n, const int32_t* __restrict__ pend,
                               const int32_t* __restrict__ lead, const int32_t* __restrict__ dslot,
                               int32_t* cursor, int32_t* chunk_rows) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t r = pend[i];
        const int32_t d = dslot[lead[r] / KB];
        if (d < 0) continue;
        const int32_t slot = atomicAdd(&cursor[d], 1);
        if (slot < KB) chunk_rows[d * KB + slot] = r;
    }
}

// row lists of the pivot rows of every chunk, packed to the front (the rest
// -1): only the pivot rows take the panel transformation, as rows 0..n_piv of
// the product -- D row k is the chunk row of pivot k, A row k the row of I - E
// at that row's chunk position -- so that the GEMM's row quarters past n_piv
// hold no row and skip their epilogue.  The other chunk rows are cleared later
// by the round's elimination against all new pivots.
__global__ void k_pivot_rowlist(const int32_t* __restrict__ n_piv, const int32_t* __restrict__ piv_pos,
                                const int32_t* __restrict__ chunk_rows, int32_t* drows,
                                int32_t* arows) {
    const int d = blockIdx.x;
    for (int k = threadIdx.x; k < n_piv[d]; k += blockDim.x) {
        const int32_t pos = piv_pos[d * KB + k];
        drows[d * KB + k] = chunk_rows[d * KB + pos];
        arows[d * KB + k] = pos;
    }
}

// the factorized pivots of every chunk
__global__ void k_register_chunks(const int32_t* __restrict__ n_piv,
                                  const int32_t* __restrict__ piv_pos,
                                  const int32_t* __restrict__ piv_col,
                                  const int32_t* __restrict__ chunk_rows, int32_t* piv_of_col,
                                  uint8_t* is_piv, int32_t* wflag) {
    const int d = blockIdx.x;
    for (int k = threadIdx.x; k < n_piv[d]; k += blockDim.x) {
        const int32_t row = chunk_rows[d * KB + piv_pos[d * KB + k]];
        const int32_t col = piv_col[d * KB + k];
        piv_of_col[col] = row;
        is_piv[row] = 1;
        wflag[col] = 1;
    }
}

// scale row rows[i] by the inverse of its entry at column cols[i] (one CTA
// per row; NORM_U independent loads per thread and pass)
constexpr int NORM_U = 8;
template <class F>
__global__ void k_normalize_at(const int32_t* __restrict__ n_dev, const int32_t* __restrict__ rows,
                               const int32_t* __restrict__ cols, int32_t ncols, uint32_t* M,
                               int64_t ld, F f) {
    __shared__ uint32_t s_inv;
    const int32_t n = *n_dev;
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        uint32_t* row = M + (size_t)rows[i] * ld;
        const int32_t c0 = cols[i];
        const uint32_t lv = row[c0];
        if (lv == 1u) continue;  // uniform over the CTA
        __syncthreads();  // the previous row's readers of s_inv are done
        if (threadIdx.x == 0) s_inv = f.prep(inverse_mod(lv, f.p));
        __syncthreads();
        const uint32_t inv = s_inv;
        for (int c = c0 + 1 + threadIdx.x; c < ncols; c += blockDim.x * NORM_U) {
            uint32_t v[NORM_U];
#pragma unroll
            for (int u = 0; u < NORM_U; ++u) {
                const int cc = c + u * (int)blockDim.x;
                v[u] = cc < ncols ? row[cc] : 0u;
            }
#pragma unroll
            for (int u = 0; u < NORM_U; ++u) {
                const int cc = c + u * (int)blockDim.x;
                if (v[u]) row[cc] = f.mulp(v[u], inv);
            }
        }
        if (threadIdx.x == 0) row[c0] = 1u;
    }
}

// Row echelon of one panel (the 128 columns of panel dpanel[d], on the n <= KB
// rows chunk_rows[d KB + i] of Dp) in shared memory, recording the
// transformation E (E * old = rows whose panel part is in echelon form; the
// rows that are not pivots become zero in the panel).  Writes I - E (KB x KB,
// zero outside the leading n x n block), so that old - (I - E) old = E old is
// one in-place GEMM update of the chunk rows, and the panel-local index and
// column of every pivot, in increasing column order, and their count.
//
// Every row keeps its lead (first nonzero panel column) in registers of its
// eight threads (adjacent lanes).  A step takes the non-pivot row with the
// smallest (lead, index) as the next pivot -- the same pivot the column-by-
// column search finds -- and updates exactly the other non-pivot rows with that
// lead, fraction-free: row_r <- P[i][c] row_r - P[r][c] row_i on the columns
// after c and on E (a nonzero multiple of the usual update: the same zero
// pattern, hence the same leads and pivots, and no inverse on the sequential
// path; each entry takes one reduction, f.ffsub).  On E only the columns in
// the union of the two rows' supports are touched: every E row keeps its
// support as a 128-bit mask (the chunk rows combined into it so far).
// Pivot rows are not scaled (they are normalised after the round).
// Column c is never read again, so it is not written; the pivot row is not
// written in the step that chooses it, so the updates need no barrier of their
// own.  The updated rows recompute their leads from the values they wrote and
// publish their keys for the next step: one barrier per pivot.
constexpr int PF_GROUPS = 8;     // threads (adjacent lanes) per row in k_panel_factor
constexpr int PF_LD = KB + 8;    // row stride of P and E: conflict-free for 8 lanes per row

template <class F>
__global__ void __launch_bounds__(KB * PF_GROUPS)
k_panel_factor(const uint32_t* __restrict__ Dp, int64_t ld, const int32_t* __restrict__ chunk_rows,
               const int32_t* __restrict__ dpanel, const int32_t* __restrict__ cursor, int32_t ncr,
               uint32_t* ime_b, int32_t* piv_pos_b, int32_t* piv_col_b, int32_t* n_piv_b, F f) {
    // chunk blockIdx.x: panel dpanel[d]
    const int d = blockIdx.x;
    const int32_t pj = dpanel[d] * KB;
    const int32_t n = min(cursor[d], KB), bw = min(KB, ncr - pj), col0 = pj;
    const int32_t* rows = chunk_rows + (size_t)d * KB;
    uint32_t* ime = ime_b + (size_t)d * KB * KB;
    int32_t* piv_pos = piv_pos_b + d * KB;
    int32_t* piv_col = piv_col_b + d * KB;
    int32_t* n_piv = n_piv_b + d;
    extern __shared__ __align__(16) uint32_t pf_smem[];
    uint32_t(*P)[PF_LD] = (uint32_t(*)[PF_LD])pf_smem;
    uint32_t(*E)[PF_LD] = (uint32_t(*)[PF_LD])(pf_smem + KB * PF_LD);
    __shared__ int s_min[2][KB * PF_GROUPS / 32];  // double-buffered block minimum
    __shared__ uint32_t s_emask[KB][4];             // support of every E row
    const int tid = threadIdx.x, nt = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int r = tid / PF_GROUPS, g = tid % PF_GROUPS;  // row and column group of this thread
    const unsigned grp = 0xFFu << (lane & ~7);           // the row's eight lanes
    for (int t = tid; t < KB * KB; t += nt) {
        const int i = t / KB, c = t % KB;
        P[i][c] = (i < n && c < bw) ? Dp[(size_t)rows[i] * ld + pj + c] : 0u;
        E[i][c] = i == c ? 1u : 0u;
    }
    for (int t = tid; t < KB * 4; t += nt) {
        const int i = t / 4, w = t % 4;
        s_emask[i][w] = (i / 32 == w) ? 1u << (i % 32) : 0u;
    }
    __syncthreads();
    int my_lead = INT_MAX;  // this row's lead (INT_MAX: zero in the panel or not a row)
    bool my_piv = false;
    if (r < n)
        for (int cc = g; cc < bw; cc += PF_GROUPS)
            if (P[r][cc] != 0u) {
                my_lead = cc;
                break;
            }
    my_lead = min(my_lead, __shfl_xor_sync(0xffffffffu, my_lead, 1));
    my_lead = min(my_lead, __shfl_xor_sync(0xffffffffu, my_lead, 2));
    my_lead = min(my_lead, __shfl_xor_sync(0xffffffffu, my_lead, 4));
    int k = 0;
    for (int step = 0; step < KB; ++step) {
        // warp minima by the warp-wide integer reduction (one redux.sync each)
        const int key = __reduce_min_sync(
            0xffffffffu, (g == 0 && !my_piv && my_lead != INT_MAX) ? my_lead * KB + r : INT_MAX);
        int* sm = s_min[step & 1];
        if (lane == 0) sm[warp] = key;
        __syncthreads();  // also: the previous step's updates are visible
        // the 32 warp minima: one read per lane, then a warp reduction
        static_assert(KB * PF_GROUPS / 32 == 32, "one warp minimum per lane");
        const int best = __reduce_min_sync(0xffffffffu, sm[lane]);
        if (best == INT_MAX) break;  // uniform: no pivot left in the panel
        const int c = best / KB, i = best % KB;
        if (tid == 0) {
            piv_pos[k] = i;
            piv_col[k] = col0 + c;
        }
        if (r == i) my_piv = true;
        if (!my_piv && my_lead == c) {
            // row_r <- a row_r - m row_i, a = P[i][c], m = P[r][c], one
            // reduction per entry (f.ffsub).  Lane g takes the 4-column groups
            // 4 g + 32 t (16-byte shared-memory accesses).  Left of c both rows
            // are zero and at c the result is zero, so whole groups are
            // computed; groups entirely left of c are skipped.
            const uint32_t ap = f.prep(P[i][c]);
            const uint32_t mn = f.prep(f.p - P[r][c]);
            int nl = INT_MAX;
#pragma unroll
            for (int t4 = 0; t4 < 4; ++t4) {
                const int base = 32 * t4 + 4 * g;
                if (base + 3 <= c || base >= bw) continue;
                const uint4 x4 = *(const uint4*)&P[r][base];
                const uint4 v4 = *(const uint4*)&P[i][base];
                uint4 y;
                y.x = f.ffsub(x4.x, ap, v4.x, mn);
                y.y = f.ffsub(x4.y, ap, v4.y, mn);
                y.z = f.ffsub(x4.z, ap, v4.z, mn);
                y.w = f.ffsub(x4.w, ap, v4.w, mn);
                *(uint4*)&P[r][base] = y;
                const int first = y.x ? 0 : y.y ? 1 : y.z ? 2 : y.w ? 3 : 4;
                if (first < 4) nl = min(nl, base + first);
            }
            // E: only the 4-column groups that meet the union of the two
            // rows' supports (every E row keeps its support as a mask of the
            // chunk rows combined into it so far)
            uint32_t U[4];
#pragma unroll
            for (int w = 0; w < 4; ++w) U[w] = s_emask[r][w] | s_emask[i][w];
#pragma unroll
            for (int t4 = 0; t4 < 4; ++t4) {
                const int base = 32 * t4 + 4 * g;
                if (base >= n || ((U[t4] >> (4 * g)) & 0xFu) == 0u) continue;
                const uint4 x4 = *(const uint4*)&E[r][base];
                const uint4 v4 = *(const uint4*)&E[i][base];
                uint4 y;
                y.x = f.ffsub(x4.x, ap, v4.x, mn);
                y.y = f.ffsub(x4.y, ap, v4.y, mn);
                y.z = f.ffsub(x4.z, ap, v4.z, mn);
                y.w = f.ffsub(x4.w, ap, v4.w, mn);
                *(uint4*)&E[r][base] = y;
            }
            __syncwarp(grp);  // the row's lanes have read its old support
            if (g < 4) s_emask[r][g] = g == 0 ? U[0] : g == 1 ? U[1] : g == 2 ? U[2] : U[3];
            // the row's eight lanes (all of them take this branch together)
            my_lead = __reduce_min_sync(grp, nl);
        }
        ++k;
    }
    for (int t = tid; t < KB * KB; t += nt) {
        const int ii = t / KB, cc = t % KB;
        uint32_t v = 0u;
        if (ii < n && cc < n) {
            const uint32_t e = E[ii][cc];
            const uint32_t one = ii == cc ? 1u : 0u;
            v = one >= e ? one - e : one + (f.p - e);
        }
        ime[t] = v;
    }
    if (tid == 0) *n_piv = k;
}




// The panel transformation of every factorized chunk on CUDA cores: the pivot
// rows of chunk d become E_d old over the columns from the first dirty panel
// on, as  D[row of pivot k] = old[pos_k] - sum_j (I - E_d)[pos_k][j] old[j]
// (ime = I - E_d from k_panel_factor; pos_k = the pivot's chunk position).
// It is a small GEMM per chunk (np x n times n x width), done with register
// tiles: a block owns tiles of 64 columns of one chunk; it stages the (I - E)
// rows of its pivots transposed (A^T, n x 16 QC) once and, per tile, the old
// values of the chunk's n rows (T, n x 64).  Every thread forms 4 pivots x QC
// columns, one 16-byte read of A^T and QC reads of T per step of the sum; QC
// (1, 2 or 4) is the smallest that covers the chunk's pivots in one pass
// (16 QC pivots), so that every thread has work; chunks of more than 64
// pivots take several passes.  64-bit sums without reduction (p < 2^16: each
// product < 2^32, at most 128 of them; otherwise the column value in 16-bit
// halves), one reduction per result.  A block reads all of a tile's columns
// before it writes any (it owns them), so the update is in place.  Only pivot
// rows are written.
constexpr int PA_COLS = 64;
constexpr int PA_THREADS = 256;
constexpr int PA_PB = 64;            // most pivots per pass (QC = 4)
constexpr int PA_SMALL_ROWS = 32;    // chunks up to this many rows: k_panel_apply_small
constexpr int PA_ALD = PA_PB + 4;    // row stride of A^T (16-byte aligned rows)
constexpr int PA_SMEM = (KB * PA_COLS + KB * PA_ALD) * (int)sizeof(uint32_t);

// the sums of one pass: pivots kp + 4 pg + q (q < 4, below kp + kn) times
// columns cg + (64 / QC) u (u < QC) of the tile at c0, written to the pivots'
// rows
template <bool WIDE, int QC>
__device__ __forceinline__ void pa_pass(uint32_t* Dp, int64_t ld, int32_t ncr, int c0, int n,
                                        int kp, int kn, const uint32_t (*T)[PA_COLS],
                                        const uint32_t (*At)[PA_ALD], const int32_t* s_pos,
                                        const int32_t* s_drow, uint32_t p, uint64_t m) {
    constexpr int CG = PA_COLS / QC;  // column groups
    const int cg = threadIdx.x % CG, pg = threadIdx.x / CG;
    if (4 * pg >= kn) return;
    uint64_t lo[4][QC], hi[4][QC];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int u = 0; u < QC; ++u) lo[q][u] = hi[q][u] = 0;
    const bool full = 4 * pg + 4 <= kn;
#pragma unroll 2
    for (int j = 0; j < n; ++j) {
        uint4 a4 = *(const uint4*)&At[j][4 * pg];
        if (!full) {  // entries past kn are not this pass's pivots
            const int r = kn - 4 * pg;
            if (r < 4) a4.w = 0u;
            if (r < 3) a4.z = 0u;
            if (r < 2) a4.y = 0u;
        }
        const uint32_t a[4] = {a4.x, a4.y, a4.z, a4.w};
        uint32_t v[QC];
#pragma unroll
        for (int u = 0; u < QC; ++u) v[u] = T[j][cg + CG * u];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int u = 0; u < QC; ++u) {
                if (WIDE) {
                    lo[q][u] += (uint64_t)a[q] * (v[u] & 0xFFFFu);
                    hi[q][u] += (uint64_t)a[q] * (v[u] >> 16);
                } else {
                    lo[q][u] += (uint64_t)a[q] * v[u];
                }
            }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int k = kp + 4 * pg + q;
        if (k >= kp + kn) break;
        const int pos = s_pos[k];
        uint32_t* out = Dp + (size_t)s_drow[k] * ld;
#pragma unroll
        for (int u = 0; u < QC; ++u) {
            const int cc = cg + CG * u, col = c0 + cc;
            if (col < ncr) {
                const uint32_t s = WIDE ? fold_lohi(lo[q][u], hi[q][u], p, m) : mod64(lo[q][u], p, m);
                const uint32_t old = T[pos][cc];
                out[col] = old >= s ? old - s : old + (p - s);
            }
        }
    }
}

// Chunks of at most 32 rows: a warp per 32-column strip, the strip's old
// values of the chunk's n rows in registers (one independent load each), the
// chunk's transformation rows E (np x n, E = I - (I - E), so the pivot's own
// old value is part of the sum) broadcast from shared memory.  No barrier
// after the staging.  NJ >= n is the unrolled row count.
template <bool WIDE, int NJ>
__device__ __forceinline__ void pa_small(uint32_t* Dp, int64_t ld, int32_t ncr, int c_lo,
                                         int c_hi, int n, int np, const uint32_t* Es,
                                         const int32_t* s_rows, const int32_t* s_drow,
                                         uint32_t p, uint64_t m) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int s0 = c_lo + 32 * warp; s0 < c_hi; s0 += 32 * (PA_THREADS / 32)) {
        const int col = s0 + lane;
        const bool ok = col < c_hi && col < ncr;
        uint32_t v[NJ];
#pragma unroll
        for (int j = 0; j < NJ; ++j) v[j] = (ok && j < n) ? Dp[(size_t)s_rows[j] * ld + col] : 0u;
        for (int k = 0; k < np; ++k) {
            const uint32_t* e = Es + k * 32;
            uint64_t lo = 0, hi = 0;
#pragma unroll
            for (int j = 0; j < NJ; ++j) {
                const uint32_t a = e[j];  // zero for j >= n
                if (WIDE) {
                    lo += (uint64_t)a * (v[j] & 0xFFFFu);
                    hi += (uint64_t)a * (v[j] >> 16);
                } else {
                    lo += (uint64_t)a * v[j];
                }
            }
            if (ok) Dp[(size_t)s_drow[k] * ld + col] = WIDE ? fold_lohi(lo, hi, p, m) : mod64(lo, p, m);
        }
    }
}

template <bool WIDE>
__global__ void __launch_bounds__(PA_THREADS)
k_panel_apply(uint32_t* Dp, int64_t ld, int32_t ncr, int32_t j0, int32_t tiles_per_block,
              const int32_t* __restrict__ chunk_rows, const int32_t* __restrict__ dpanel,
              const int32_t* __restrict__ cursor, const uint32_t* __restrict__ ime_b,
              const int32_t* __restrict__ n_piv_b, const int32_t* __restrict__ arows_b,
              const int32_t* __restrict__ drows_b, uint32_t p) {
    extern __shared__ __align__(16) uint32_t pa_smem[];
    uint32_t(*T)[PA_COLS] = (uint32_t(*)[PA_COLS])pa_smem;
    uint32_t(*At)[PA_ALD] = (uint32_t(*)[PA_ALD])(pa_smem + KB * PA_COLS);
    __shared__ int32_t s_rows[KB], s_pos[KB], s_drow[KB];
    const int d = blockIdx.y;
    const int n = min(cursor[d], KB), np = n_piv_b[d];
    const int pj = dpanel[d] * KB;
    // the block's tiles: [tile0, tile1), the first one right of the chunk's
    // panel start (the chunk rows are zero left of it)
    const int ntiles = (ncr - j0 + PA_COLS - 1) / PA_COLS;
    int tile0 = blockIdx.x * tiles_per_block;
    const int tile1 = min(ntiles, tile0 + tiles_per_block);
    tile0 = max(tile0, pj > j0 ? (pj - j0) / PA_COLS : 0);
    // uniform: nothing to do, or a chunk for k_panel_apply_small
    if (np == 0 || tile0 >= tile1 || n <= PA_SMALL_ROWS) return;
    for (int t = threadIdx.x; t < KB; t += PA_THREADS) {
        s_rows[t] = t < n ? chunk_rows[(size_t)d * KB + t] : 0;
        s_pos[t] = t < np ? arows_b[(size_t)d * KB + t] : 0;
        s_drow[t] = t < np ? drows_b[(size_t)d * KB + t] : 0;
    }
    __syncthreads();
    const uint32_t* ime = ime_b + (size_t)d * KB * KB;
    const uint64_t m = ~0ull / p;
    // columns per thread and pivots per pass (uniform over the block)
    const int qc = np <= 16 ? 1 : (np <= 32 ? 2 : 4);
    const int pb = 16 * qc;
    // A^T of pivots [kp, kp + kn)
    auto stage_a = [&](int kp, int kn) {
        for (int t = threadIdx.x; t < kn * n; t += PA_THREADS) {
            const int k = t / n, j = t % n;
            At[j][k] = ime[(size_t)s_pos[kp + k] * KB + j];
        }
    };
    const bool one_pass = np <= pb;
    if (one_pass) stage_a(0, np);  // once for all tiles
    for (int tile = tile0; tile < tile1; ++tile) {
        const int c0 = j0 + tile * PA_COLS;
        __syncthreads();  // the last tile's readers of T are done
        {
            // n x 64 old values, eight independent loads per thread at a time
            const int total = n * PA_COLS;
            for (int t0 = threadIdx.x; t0 < total; t0 += 8 * PA_THREADS) {
                uint32_t v[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int t = t0 + q * PA_THREADS;
                    const int j = t / PA_COLS, col = c0 + t % PA_COLS;
                    v[q] = (t < total && col < ncr) ? Dp[(size_t)s_rows[j] * ld + col] : 0u;
                }
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int t = t0 + q * PA_THREADS;
                    if (t < total) T[t / PA_COLS][t % PA_COLS] = v[q];
                }
            }
        }
        for (int kp = 0; kp < np; kp += pb) {
            const int kn = min(pb, np - kp);
            if (!one_pass) {
                __syncthreads();  // the last pass's readers of A^T are done
                stage_a(kp, kn);
            }
            __syncthreads();  // T and A^T are in place
            if (qc == 1)
                pa_pass<WIDE, 1>(Dp, ld, ncr, c0, n, kp, kn, T, At, s_pos, s_drow, p, m);
            else if (qc == 2)
                pa_pass<WIDE, 2>(Dp, ld, ncr, c0, n, kp, kn, T, At, s_pos, s_drow, p, m);
            else
                pa_pass<WIDE, 4>(Dp, ld, ncr, c0, n, kp, kn, T, At, s_pos, s_drow, p, m);
        }
    }
}

// the chunks of k_panel_apply with at most PA_SMALL_ROWS rows (same grid)
template <bool WIDE>
__global__ void __launch_bounds__(PA_THREADS)
k_panel_apply_small(uint32_t* Dp, int64_t ld, int32_t ncr, int32_t j0, int32_t tiles_per_block,
                    const int32_t* __restrict__ chunk_rows, const int32_t* __restrict__ dpanel,
                    const int32_t* __restrict__ cursor, const uint32_t* __restrict__ ime_b,
                    const int32_t* __restrict__ n_piv_b, const int32_t* __restrict__ arows_b,
                    const int32_t* __restrict__ drows_b, uint32_t p) {
    __shared__ uint32_t Es[PA_SMALL_ROWS * 32];
    __shared__ int32_t s_rows[PA_SMALL_ROWS], s_drow[PA_SMALL_ROWS];
    const int d = blockIdx.y;
    const int n = min(cursor[d], KB), np = n_piv_b[d];
    const int pj = dpanel[d] * KB;
    const int ntiles = (ncr - j0 + PA_COLS - 1) / PA_COLS;
    int tile0 = blockIdx.x * tiles_per_block;
    const int tile1 = min(ntiles, tile0 + tiles_per_block);
    tile0 = max(tile0, pj > j0 ? (pj - j0) / PA_COLS : 0);
    if (np == 0 || tile0 >= tile1 || n > PA_SMALL_ROWS) return;  // uniform
    for (int t = threadIdx.x; t < PA_SMALL_ROWS; t += PA_THREADS) {
        s_rows[t] = t < n ? chunk_rows[(size_t)d * KB + t] : 0;
        s_drow[t] = t < np ? drows_b[(size_t)d * KB + t] : 0;
    }
    // E rows of the pivots, 32 entries each (zero past n):
    // E[k][j] = [j = pos_k] - (I - E)[pos_k][j] mod p
    const uint32_t* ime = ime_b + (size_t)d * KB * KB;
    for (int t = threadIdx.x; t < np * 32; t += PA_THREADS) {
        const int k = t / 32, j = t % 32;
        uint32_t e = 0u;
        if (j < n) {
            const int pos = arows_b[(size_t)d * KB + k];
            const uint32_t a = ime[(size_t)pos * KB + j];
            e = (j == pos) ? (a == 0u ? 1u : (1u + p - a) % p) : (a ? p - a : 0u);
        }
        Es[t] = e;
    }
    __syncthreads();
    const uint64_t m = ~0ull / p;
    const int c_lo = j0 + tile0 * PA_COLS, c_hi = min(ncr, j0 + tile1 * PA_COLS);
    if (n <= 8)
        pa_small<WIDE, 8>(Dp, ld, ncr, c_lo, c_hi, n, np, Es, s_rows, s_drow, p, m);
    else if (n <= 16)
        pa_small<WIDE, 16>(Dp, ld, ncr, c_lo, c_hi, n, np, Es, s_rows, s_drow, p, m);
    else
        pa_small<WIDE, 32>(Dp, ld, ncr, c_lo, c_hi, n, np, Es, s_rows, s_drow, p, m);
}

// dst block b (NB x NB, leading dimension NB, block stride NB (NB + 1)) =
// src block b (nb_b x nb_b at src + b stride_src, leading dimension lds),
// identity-padded; nb_b = NB except for the last block
__global__ void k_copy_blocks(const uint32_t* __restrict__ src, int64_t lds, int64_t stride_src,
                              int32_t n_blocks, int32_t last_nb, int32_t NB, uint32_t* dst) {
    GB_WARP_ROWS(n_blocks * NB, NB) {
        const int32_t b = i / NB, r = i % NB;
        const int32_t nb = b == n_blocks - 1 ? last_nb : NB;
        const uint32_t* s = src + (size_t)b * stride_src + (size_t)r * lds;
        uint32_t* o = dst + (size_t)b * NB * (NB + 1) + (size_t)r * NB;
        for (int j0 = jb + lane; j0 < je; j0 += 128) {
            uint32_t v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int jj = j0 + 32 * u;
                v[u] = (r < nb && jj < nb) ? s[jj] : (r == jj ? 1u : 0u);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (j0 + 32 * u < je) o[j0 + 32 * u] = v[u];
        }
    }
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

// D (M x N) -= A (M x K) B (K x N), exact mod p, for any TcGemmArgs (batch,
// row lists); the tensor-core workspace grows on demand
static int gemm_args(Ctx& c, TcGemmArgs g) {
    if (g.M <= 0 || g.N <= 0 || g.K <= 0 || g.batch <= 0) return GBGPU_OK;
    g.p = c.p;
    if (c.form == GBGPU_FORM_PLAIN) return plain_submul(g, c.s, &c.launches);
    const size_t need = tc_workspace_bytes(c.p, g.M, g.N, g.K, g.batch);
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

static int gemm(Ctx& c, uint32_t* D, int64_t ldd, const uint32_t* A, int64_t lda,
                const uint32_t* B, int64_t ldb, int32_t M, int32_t N, int32_t K) {
    TcGemmArgs g{c.p, M, N, K, A, lda, B, ldb, D, ldd};
    return gemm_args(c, g);
}

// batch of `batch` products D_z -= A_z B_z (element strides sA, sB, sD)
static int gemm_batched(Ctx& c, uint32_t* D, int64_t ldd, int64_t sD, const uint32_t* A,
                        int64_t lda, int64_t sA, const uint32_t* B, int64_t ldb, int64_t sB,
                        int32_t M, int32_t N, int32_t K, int32_t batch) {
    TcGemmArgs g{c.p, M, N, K, A, lda, B, ldb, D, ldd};
    g.batch = batch;
    g.sA = sA;
    g.sB = sB;
    g.sD = sD;
    return gemm_args(c, g);
}

// elimination block size: powers of two from 128 to `cap` (1024 by default)
static int32_t nb_for(int64_t n, int32_t cap = 8 * KB) {
    int32_t nb = KB;
    while (nb < n && nb < cap) nb *= 2;
    return nb;
}

// -U^-1 for n_blocks unit upper triangular blocks of size NB (block b at
// src + b * stride_src, leading dimension lds; the last one last_nb x last_nb,
// identity-padded).  Result: out + b NB (NB + 1), leading dimension NB.  The
// 128 x 128 diagonal blocks are inverted by k_neg_inverse; blocks are then
// merged by doubling,  -[[A, B], [0, C]]^-1 = [[-A^-1, A^-1 B C^-1], [0, -C^-1]],
// with two batched GEMMs per level (the NB + 1 block stride makes the
// diagonal blocks of one level equally spaced across all big blocks).
template <class F>
static int neg_inverse_big(Ctx& c, const F& f, const uint32_t* src, int64_t lds,
                           int64_t stride_src, int32_t n_blocks, int32_t last_nb, int32_t NB,
                           uint32_t* out) {
    if (n_blocks <= 0) return GBGPU_OK;
    const int64_t bstride = (int64_t)NB * (NB + 1);
    uint32_t* U = c.alloc<uint32_t>((size_t)n_blocks * bstride);
    uint32_t* T = c.alloc<uint32_t>((size_t)n_blocks * NB * NB / 4 + 1);
    if (!U || !T) return GBGPU_ENOMEM;
    BL_LAUNCH(k_copy_blocks<<<grid_of((int64_t)n_blocks * NB * NB), 256, 0, c.s>>>(
        src, lds, stride_src, n_blocks, last_nb, NB, U));
    BL_CUDA(cudaMemsetAsync(out, 0, sizeof(uint32_t) * (size_t)n_blocks * bstride, c.s));
    const int bytes = (2 * KB * (KB + 1) + KB * KB / 4) * (int)sizeof(uint32_t);
    BL_CUDA(ensure_smem_limit((const void*)k_neg_inverse<F>, bytes));
    const int32_t n_sub = n_blocks * (NB / KB);
    const int64_t dstep = (int64_t)KB * (NB + 1);  // between 128-blocks on the diagonal
    BL_LAUNCH(k_neg_inverse<F><<<n_sub, INV_THREADS, bytes, c.s>>>(U, NB, dstep, n_sub, KB, out,
                                                                   dstep, NB, f));
    for (int32_t sz = KB; sz < NB; sz *= 2) {
        const int32_t items = n_blocks * (NB / (2 * sz));
        const int64_t istep = (int64_t)2 * sz * (NB + 1);
        const int64_t half = (int64_t)sz * (NB + 1);
        BL_CUDA(cudaMemsetAsync(T, 0, sizeof(uint32_t) * (size_t)items * sz * sz, c.s));
        // T = B C^-1 = 0 - B (-C^-1)
        BL_CHECK(gemm_batched(c, T, sz, (int64_t)sz * sz, U + sz, NB, istep, out + half, NB, istep,
                              sz, sz, sz, items));
        // top right of -U^-1 = A^-1 B C^-1 = 0 - (-A^-1) T
        BL_CHECK(gemm_batched(c, out + sz, NB, istep, out, NB, istep, T, sz, (int64_t)sz * sz, sz,
                              sz, sz, items));
    }
    return GBGPU_OK;
}

// out[k] = in[n - 1 - k]
__global__ void k_reverse_i32(int32_t n, const int32_t* __restrict__ in, int32_t* out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        out[k] = in[n - 1 - k];
}

// offs[k] = base + loc[k]
__global__ void k_offs_write(int32_t n, const int64_t* __restrict__ loc, int64_t base,
                             int64_t* offs) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        offs[k] = base + loc[k];
}

// Rows t_rows[0 .. rows) of M (leading dimension ld, ncols columns) are
// reduced by the pivot rows u_rows[0 .. n_p) of M (sorted by lead, monic,
// zero left of their leads, pivot columns pc ascending):
//   T <- T - T[:, pc] (U[:, pc])^-1 U,
// after which every T row is zero at every pivot column.  Blocks of NB
// pivots, left to right; the rows are read and written in place through the
// row lists (T and U rows are distinct).
template <class F>
static int eliminate(Ctx& c, const F& f, uint32_t* M, int64_t ld, const int32_t* t_rows,
                     int32_t rows, int32_t ncols, const int32_t* u_rows, int32_t n_p,
                     const int32_t* d_pc, const std::vector<int32_t>& pc) {
    if (rows <= 0 || n_p <= 0) return GBGPU_OK;
    const int32_t NB = nb_for(n_p);
    const int32_t nb = (n_p + NB - 1) / NB;
    const int64_t bstride = (int64_t)NB * (NB + 1);
    uint32_t* Ublk = c.alloc<uint32_t>((size_t)nb * NB * NB);   // U[:, pc] diagonal blocks
    uint32_t* Ninv = c.alloc<uint32_t>((size_t)nb * bstride);
    uint32_t* G = c.alloc<uint32_t>((size_t)rows * NB);         // T[:, pc_k]
    uint32_t* X = c.alloc<uint32_t>((size_t)rows * NB);
    if (!Ublk || !Ninv || !G || !X) return GBGPU_ENOMEM;
    for (int b = 0; b < nb; ++b) {
        const int kb = std::min(NB, n_p - b * NB);
        BL_LAUNCH(k_gather_cols<<<grid_of((int64_t)kb * kb), 256, 0, c.s>>>(
            kb, kb, M, ld, d_pc + b * NB, Ublk + (size_t)b * NB * NB, NB, u_rows + b * NB));
    }
    BL_CHECK(neg_inverse_big(c, f, Ublk, NB, (int64_t)NB * NB, nb, n_p - (nb - 1) * NB, NB, Ninv));
    for (int b = 0; b < nb; ++b) {
        const int kb = std::min(NB, n_p - b * NB);
        const int32_t first_col = pc[b * NB];
        BL_LAUNCH(k_gather_cols<<<grid_of((int64_t)rows * kb), 256, 0, c.s>>>(
            rows, kb, M, ld, d_pc + b * NB, G, NB, t_rows));
        BL_CUDA(cudaMemsetAsync(X, 0, sizeof(uint32_t) * (size_t)rows * NB, c.s));
        // X = G * (U_kk)^-1 = 0 - G * (-(U_kk)^-1)
        BL_CHECK(gemm(c, X, NB, G, NB, Ninv + (size_t)b * bstride, NB, rows, kb, kb));
        // T[:, first_col:] -= X * U_k[:, first_col:]
        TcGemmArgs g{c.p, rows, ncols - first_col, kb, X, NB, M + first_col, ld, M + first_col, ld};
        g.b_rows = u_rows + b * NB;
        g.d_rows = t_rows;
        BL_CHECK(gemm_args(c, g));
    }
    return GBGPU_OK;
}

// ---------------------------------------------------------------------------
template <class F>
static int echelon_rref(Ctx& c, const F& f, uint32_t* Dp, int64_t ld, int32_t t, int32_t ncr,
                        BlockedOutput* out);

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
        BL_CUDA(ensure_smem_limit((const void*)k_densify_seg, DS_COLS * 4));
        BL_LAUNCH(k_densify_seg<<<std::min(t, 148 * 3), 512, DS_COLS * 4, s>>>(
            t, work_sorted, in.row_ptr, in.cols, in.vals, nc, 0, W, ld));
    }
    if (t > 0 && ncl > 0) {
        const int32_t NB = nb_for(ncl, 16 * KB);
        const int64_t bstride = (int64_t)NB * (NB + 1);
        uint32_t* P = c.alloc<uint32_t>((size_t)ncl * ld);
        const int32_t nbk = (ncl + NB - 1) / NB;
        uint32_t* Ninv = c.alloc<uint32_t>((size_t)nbk * bstride);
        uint32_t* X = c.alloc<uint32_t>((size_t)t * NB);
        int32_t* act = c.alloc<int32_t>(nbk);
        int32_t* span = c.alloc<int32_t>(nbk);
        const int32_t ngrp = (ncl + 127) / 128;
        int2* brange = c.alloc<int2>(ngrp);
        if (!P || !Ninv || !X || !act || !span || !brange) return GBGPU_ENOMEM;
        // active rows of each block (rows sorted by lead), the last left
        // column the known pivots of each block touch, and the right columns
        // every 128 known pivots reach
        BL_LAUNCH(k_count_below<<<grid_of(nbk), 256, 0, s>>>(t, lead_sorted, nbk, NB, act));
        BL_LAUNCH(k_fill_i32<<<grid_of(nbk), 256, 0, s>>>(span, nbk, -1));
        BL_LAUNCH(k_clear_ranges<<<grid_of(ngrp), 256, 0, s>>>(ngrp, brange));
        BL_LAUNCH(k_block_span<<<grid_of((int64_t)ncl * 32), 256, 0, s>>>(
            ncl, in.piv_row, in.row_ptr, in.cols, ncl, NB, span, brange));
        // pivot row of lead c into row c of P: on the tensor cores only the
        // parts a later step reads (its diagonal block, the left columns its
        // block reaches, the right columns its group of 128 reaches); the
        // CUDA-core GEMM reads B whole, so there P gets everything from the
        // diagonal block on
        const bool banded = c.form != GBGPU_FORM_PLAIN;
        BL_LAUNCH(k_densify_direct<<<std::min(ncl, 148 * 8), DS_THREADS, 0, s>>>(
            ncl, in.piv_row, in.row_ptr, in.cols, in.vals, nc, NB, P, ld, banded ? ncl : 0, span,
            brange));
        // -A_kk^-1 of every NB x NB diagonal block of A (read in place from P)
        BL_CHECK(neg_inverse_big(c, f, P, ld, (int64_t)NB * ld + NB, nbk, ncl - (nbk - 1) * NB, NB,
                                 Ninv));
        std::vector<int32_t> h_act(nbk), h_span(nbk);
        BL_CUDA(cudaMemcpyAsync(h_act.data(), act, sizeof(int32_t) * nbk, cudaMemcpyDeviceToHost, s));
        BL_CUDA(cudaMemcpyAsync(h_span.data(), span, sizeof(int32_t) * nbk, cudaMemcpyDeviceToHost, s));
        BL_CUDA(cudaStreamSynchronize(s));
        // (a) X = C A^-1, in place in W[:, 0:ncl], block by block; the update of
        //     the later left columns stops at the last column block k touches
        for (int k = 0; k < nbk; ++k) {
            const int32_t c0 = k * NB, kb = std::min(NB, ncl - c0), c1 = c0 + kb;
            const int32_t rows = h_act[k];
            if (rows <= 0) continue;
            BL_CUDA(cudaMemsetAsync(X, 0, sizeof(uint32_t) * (size_t)rows * NB, s));
            // X_k = W[:, block] A_kk^-1
            BL_CHECK(gemm(c, X, NB, W + c0, ld, Ninv + (size_t)k * bstride, NB, rows, kb, kb));
            BL_CUDA(cudaMemcpy2DAsync(W + c0, ld * 4, X, NB * 4, (size_t)kb * 4, rows,
                                      cudaMemcpyDeviceToDevice, s));
            // W[:, c1:e) -= X_k A[block rows, c1:e)
            const int32_t e = std::min(ncl, h_span[k] + 1);
            if (e > c1)
                BL_CHECK(gemm(c, W + c1, ld, X, NB, P + (size_t)c0 * ld + c1, ld, rows, e - c1, kb));
        }
        // (b) D' = D - X B: one GEMM over the whole left block; the tile flags of
        //     the GEMM skip the zero tiles of the staircase X and of B
        {
            TcGemmArgs g{c.p, t, ncr, ncl, W, ld, P + ncl, ld, W + ncl, ld};
            if (banded) g.b_nrange = brange;  // B is zero outside these columns
            BL_CHECK(gemm_args(c, g));
        }
    }
    if (out->ms_event_schur) BL_CUDA(cudaEventRecord(out->ms_event_schur, s));
    BL_CHECK(echelon_rref(c, f, W + ncl, ld, t, ncr, out));
    out->rows = W + ncl;
    out->ld = ld;
    return GBGPU_OK;
}

// Steps 2 and 3 on the dense t x ncr residue matrix Dp (leading dimension
// ld), in place: afterwards out->piv_of_col[c] is the row of Dp holding the
// reduced pivot row of column c (-1 for non-pivot columns), out->rank is the
// rank, and every other row's content is unspecified.
template <class F>
static int echelon_rref(Ctx& c, const F& f, uint32_t* Dp, int64_t ld, int32_t t, int32_t ncr,
                        BlockedOutput* out) {
    cudaStream_t s = c.s;
    // ---- 2. echelon of D' = W[:, ncl:] by rounds ----------------------------------
    // Every round looks at all pending rows (nonzero, not yet pivots) at once:
    //  * a 128-column panel in which no two pending rows share a lead is
    //    "clean": each of its rows has a lead of its own and becomes a pivot;
    //  * every other ("dirty") panel gets up to KB of its pending rows
    //    factorized in shared memory (k_panel_factor, one CTA per panel); the
    //    recorded row transformation E is applied to their trailing columns
    //    by one batched GEMM over all dirty panels;
    //  * the pending rows that did not become pivots are eliminated against
    //    all pivots of the round (eliminate), which leaves them zero at every
    //    pivot column, and the next round starts from their new leads.
    const int32_t npan = (ncr + KB - 1) / KB;
    int32_t* lead = c.alloc<int32_t>(t);
    uint8_t* is_piv = c.alloc<uint8_t>(t);
    int32_t* piv_of_col = out->piv_of_col;  // [ncr], -1 if none
    int32_t* wflag = c.alloc<int32_t>(ncr);
    int32_t* wpos = c.alloc<int32_t>(ncr);
    int32_t* pend = c.alloc<int32_t>(t);
    int32_t* counters = c.alloc<int32_t>(8);
    int32_t* pc = c.alloc<int32_t>(ncr);      // pivot columns
    int32_t* prow = c.alloc<int32_t>(ncr);    // their rows
    int32_t* hist = c.alloc<int32_t>(ncr);
    int32_t* pcnt = c.alloc<int32_t>(npan);
    int32_t* pdirty = c.alloc<int32_t>(npan);
    int32_t* dslot = c.alloc<int32_t>(npan);
    int32_t* dpanel = c.alloc<int32_t>(npan);
    if (!lead || !is_piv || !wflag || !wpos || !pend || !counters || !pc || !prow || !hist ||
        !pcnt || !pdirty || !dslot || !dpanel)
        return GBGPU_ENOMEM;
    size_t scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, wflag, wpos, ncr, s);
    void* scan_tmp = c.alloc<uint8_t>(scan_bytes);
    if (!scan_tmp) return GBGPU_ENOMEM;
    BL_LAUNCH(k_fill_i32<<<grid_of(ncr), 256, 0, s>>>(piv_of_col, ncr, -1));
    if (t > 0 && ncr > 0) {
        BL_CUDA(cudaMemsetAsync(is_piv, 0, t, s));
        BL_LAUNCH(k_row_leads<<<grid_of((int64_t)t * 32), 256, 0, s>>>(t, nullptr, ncr, Dp, ld, lead));
    }
    const int pf_bytes = 2 * KB * PF_LD * (int)sizeof(uint32_t);
    BL_CUDA(ensure_smem_limit((const void*)k_panel_factor<F>, pf_bytes));
    // every dirty panel is factorized in the round that finds it (batch <= 4096)
    const int32_t max_dirty = std::max<int32_t>(1, std::min<int32_t>(npan, 4096));
    int32_t* chunk_rows = c.alloc<int32_t>((size_t)max_dirty * KB);
    int32_t* cursor = c.alloc<int32_t>(max_dirty);
    uint32_t* imeB = c.alloc<uint32_t>((size_t)max_dirty * KB * KB);
    int32_t* piv_pos = c.alloc<int32_t>((size_t)max_dirty * KB);
    int32_t* piv_colb = c.alloc<int32_t>((size_t)max_dirty * KB);
    int32_t* n_piv = c.alloc<int32_t>(max_dirty);
    int32_t* piv_rows = c.alloc<int32_t>((size_t)max_dirty * KB);
    int32_t* piv_arows = c.alloc<int32_t>((size_t)max_dirty * KB);
    // ordered compaction of the pending rows and the stable (panel, row) sort
    // that fills the chunks: the same rows, in the same order, on every run
    uint8_t* pflag = c.alloc<uint8_t>(t);
    int32_t* pkey = c.alloc<int32_t>(t);
    int32_t* pkey_sorted = c.alloc<int32_t>(t);
    int32_t* prow_sorted = c.alloc<int32_t>(t);
    size_t sel_bytes = 0, sort_bytes = 0;
    cub::CountingInputIterator<int32_t> row_ids(0);
    cub::DeviceSelect::Flagged(nullptr, sel_bytes, row_ids, pflag, pend, counters, t, s);
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, pkey, pkey_sorted, pend, prow_sorted, t,
                                    0, 32, s);
    void* sel_tmp = c.alloc<uint8_t>(sel_bytes);
    void* sort_tmp = c.alloc<uint8_t>(sort_bytes);
    if (!chunk_rows || !cursor || !imeB || !piv_pos || !piv_colb || !n_piv || !piv_rows ||
        !piv_arows || !pflag || !pkey || !pkey_sorted || !prow_sorted || !sel_tmp || !sort_tmp)
        return GBGPU_ENOMEM;
    // pending rows (nonzero, not pivots) into pend[0 .. *count), ascending
    auto collect_pending = [&](int32_t* count) -> int {
        BL_LAUNCH(k_pending_flags<<<grid_of(t), 256, 0, s>>>(t, lead, is_piv, pflag));
        size_t bytes = sel_bytes;
        BL_CUDA(cub::DeviceSelect::Flagged(sel_tmp, bytes, row_ids, pflag, pend, count, t, s));
        ++c.launches;
        return GBGPU_OK;
    };
    int rounds = 0;
    bool first = true;
    while (t > 0 && ncr > 0) {
        // pending rows, lead histogram, clean panels claimed, dirty panels
        // flagged -- all sized on the device; one host round trip reads the
        // count and the dirty flags
        int32_t n_pend = 0;
        BL_CUDA(cudaMemsetAsync(counters, 0, 8 * sizeof(int32_t), s));
        BL_CHECK(collect_pending(counters));
        BL_CUDA(cudaMemsetAsync(hist, 0, sizeof(int32_t) * ncr, s));
        BL_CUDA(cudaMemsetAsync(pcnt, 0, sizeof(int32_t) * npan, s));
        BL_CUDA(cudaMemsetAsync(pdirty, 0, sizeof(int32_t) * npan, s));
        BL_CUDA(cudaMemsetAsync(wflag, 0, sizeof(int32_t) * ncr, s));
        BL_LAUNCH(k_lead_hist<<<grid_of(t), 256, 0, s>>>(counters, pend, lead, hist, pcnt));
        BL_LAUNCH(k_dirty_panels<<<grid_of(t), 256, 0, s>>>(counters, pend, lead, hist, pdirty));
        BL_LAUNCH(k_claim_clean<<<grid_of(t), 256, 0, s>>>(counters, pend, lead, pdirty,
                                                            piv_of_col, is_piv, wflag));
        // dirty panels, leftmost first, at most max_dirty of them this round
        std::vector<int32_t> h_dirty(npan);
        BL_CUDA(cudaMemcpyAsync(&n_pend, counters, 4, cudaMemcpyDeviceToHost, s));
        BL_CUDA(cudaMemcpyAsync(h_dirty.data(), pdirty, sizeof(int32_t) * npan,
                                cudaMemcpyDeviceToHost, s));
        BL_CUDA(cudaStreamSynchronize(s));
        if (first) out->dense_rows = n_pend;
        first = false;
        if (n_pend == 0) break;
        ++rounds;
        std::vector<int32_t> h_dpanel, h_dslot(npan, -1);
        for (int32_t p = 0; p < npan && (int32_t)h_dpanel.size() < max_dirty; ++p) {
            if (h_dirty[p]) {
                h_dslot[p] = (int32_t)h_dpanel.size();
                h_dpanel.push_back(p);
            }
        }
        const int32_t n_dirty = (int32_t)h_dpanel.size();
        if (n_dirty > 0) {
            const int32_t j0 = h_dpanel[0] * KB, width = ncr - j0;
            BL_CUDA(cudaMemcpyAsync(dslot, h_dslot.data(), sizeof(int32_t) * npan,
                                    cudaMemcpyHostToDevice, s));
            BL_CUDA(cudaMemcpyAsync(dpanel, h_dpanel.data(), sizeof(int32_t) * n_dirty,
                                    cudaMemcpyHostToDevice, s));
            BL_CUDA(cudaMemsetAsync(cursor, 0, sizeof(int32_t) * n_dirty, s));
            BL_LAUNCH(k_fill_i32<<<grid_of((int64_t)n_dirty * KB), 256, 0, s>>>(
                chunk_rows, n_dirty * KB, -1));
            BL_LAUNCH(k_panel_keys<<<grid_of(n_pend), 256, 0, s>>>(n_pend, pend, lead, dslot,
                                                                    n_dirty, pkey));
            {
                int bits = 1;
                while ((1 << bits) <= n_dirty) ++bits;
                size_t bytes = sort_bytes;
                BL_CUDA(cub::DeviceRadixSort::SortPairs(sort_tmp, bytes, pkey, pkey_sorted, pend,
                                                        prow_sorted, n_pend, 0, bits, s));
                ++c.launches;
            }
            BL_LAUNCH(k_bucket_sorted<<<grid_of(n_pend), 256, 0, s>>>(
                n_pend, pkey_sorted, prow_sorted, n_dirty, chunk_rows, cursor));
            BL_LAUNCH(k_panel_factor<F><<<n_dirty, KB * PF_GROUPS, pf_bytes, s>>>(
                Dp, ld, chunk_rows, dpanel, cursor, ncr, imeB, piv_pos, piv_colb, n_piv, f));
            // pivot rows of every chunk (columns j0..) <- old - (I - E_d) old =
            // E_d old, in place: the limb planes of `old` are cut before the
            // product writes the rows.  The non-pivot chunk rows keep their
            // values: their panel parts lie in the span of the pivot rows', so
            // the elimination against the round's pivots below clears them.
            BL_LAUNCH(k_fill_i32<<<grid_of((int64_t)n_dirty * KB), 256, 0, s>>>(
                piv_rows, n_dirty * KB, -1));
            BL_LAUNCH(k_fill_i32<<<grid_of((int64_t)n_dirty * KB), 256, 0, s>>>(
                piv_arows, n_dirty * KB, -1));
            BL_LAUNCH(k_pivot_rowlist<<<n_dirty, KB, 0, s>>>(n_piv, piv_pos, chunk_rows, piv_rows,
                                                             piv_arows));
            {
                // pivot rows of every chunk <- E_d old (CUDA cores, in place)
                const bool wide = c.p >= 65536u;
                // tiles per block: enough blocks for about six per SM, at most 8
                // tiles each (a block stages the (I - E) rows once for its tiles)
                const int tiles = (width + PA_COLS - 1) / PA_COLS;
                const int tpb = (int)std::max<int64_t>(
                    1, std::min<int64_t>(8, (int64_t)tiles * n_dirty / (148 * 6)));
                const dim3 grid((unsigned)((tiles + tpb - 1) / tpb), (unsigned)n_dirty);
                // the chunks of more than 32 rows are few and long: one tile per block
                const dim3 grid1((unsigned)tiles, (unsigned)n_dirty);
                if (wide) {
                    BL_CUDA(ensure_smem_limit((const void*)k_panel_apply<true>, PA_SMEM));
                    BL_LAUNCH(k_panel_apply_small<true><<<grid, PA_THREADS, 0, s>>>(
                        Dp, ld, ncr, j0, tpb, chunk_rows, dpanel, cursor, imeB, n_piv, piv_arows,
                        piv_rows, c.p));
                    BL_LAUNCH(k_panel_apply<true><<<grid1, PA_THREADS, PA_SMEM, s>>>(
                        Dp, ld, ncr, j0, 1, chunk_rows, dpanel, cursor, imeB, n_piv, piv_arows,
                        piv_rows, c.p));
                } else {
                    BL_CUDA(ensure_smem_limit((const void*)k_panel_apply<false>, PA_SMEM));
                    BL_LAUNCH(k_panel_apply_small<false><<<grid, PA_THREADS, 0, s>>>(
                        Dp, ld, ncr, j0, tpb, chunk_rows, dpanel, cursor, imeB, n_piv, piv_arows,
                        piv_rows, c.p));
                    BL_LAUNCH(k_panel_apply<false><<<grid1, PA_THREADS, PA_SMEM, s>>>(
                        Dp, ld, ncr, j0, 1, chunk_rows, dpanel, cursor, imeB, n_piv, piv_arows,
                        piv_rows, c.p));
                }
            }
            BL_LAUNCH(k_register_chunks<<<n_dirty, KB, 0, s>>>(n_piv, piv_pos, piv_colb, chunk_rows,
                                                                piv_of_col, is_piv, wflag));
            if (trace_rounds()) {
                std::vector<int32_t> h_cur(n_dirty), h_np(n_dirty);
                BL_CUDA(cudaMemcpyAsync(h_cur.data(), cursor, 4 * n_dirty, cudaMemcpyDeviceToHost, s));
                BL_CUDA(cudaMemcpyAsync(h_np.data(), n_piv, 4 * n_dirty, cudaMemcpyDeviceToHost, s));
                BL_CUDA(cudaStreamSynchronize(s));
                long long rows_in = 0, piv = 0;
                int mx = 0;
                for (int q = 0; q < n_dirty; ++q) {
                    rows_in += std::min(h_cur[q], KB);
                    piv += h_np[q];
                    mx = std::max(mx, h_cur[q]);
                }
                fprintf(stderr,
                        "gbgpu echelon round %d: pending %d, dirty panels %d (first %d), chunk rows "
                        "%lld (max %d), chunk pivots %lld\n",
                        rounds, n_pend, n_dirty, j0 / KB, rows_in, mx, piv);
            }
        }
        // all pivots of the round, ascending columns; normalise
        BL_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, wflag, wpos, ncr, s));
        ++c.launches;
        BL_LAUNCH(k_compact_cols<<<grid_of(ncr), 256, 0, s>>>(ncr, wflag, wpos, pc));
        BL_LAUNCH(k_new_pivots<<<grid_of(ncr), 256, 0, s>>>(ncr, wflag, wpos, pc, piv_of_col,
                                                           counters + 2, prow));
        BL_LAUNCH(k_normalize_at<F><<<std::min(t, 148 * 8), 256, 0, s>>>(counters + 2, prow, pc,
                                                                         ncr, Dp, ld, f));
        // the rest: eliminated against every pivot of the round; one host
        // round trip reads both counts and the pivot columns
        BL_CHECK(collect_pending(counters + 3));
        int32_t cnt[2] = {0, 0};
        std::vector<int32_t> h_pc((size_t)ncr);
        BL_CUDA(cudaMemcpyAsync(cnt, counters + 2, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        BL_CUDA(cudaMemcpyAsync(h_pc.data(), pc, sizeof(int32_t) * ncr, cudaMemcpyDeviceToHost, s));
        BL_CUDA(cudaStreamSynchronize(s));
        const int32_t n_new = cnt[0], n_rest = cnt[1];
        if (trace_rounds()) fprintf(stderr, "gbgpu echelon round %d: new pivots %d\n", rounds, n_new);
        if (n_rest == 0) break;
        h_pc.resize((size_t)n_new);
        BL_CHECK(eliminate(c, f, Dp, ld, pend, n_rest, ncr, prow, n_new, pc, h_pc));
        BL_LAUNCH(k_row_leads<<<grid_of((int64_t)n_rest * 32), 256, 0, s>>>(n_rest, pend, ncr, Dp,
                                                                             ld, lead, 1));
    }
    const int steps = rounds;
    out->echelon_rounds = steps;
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
        // echelon rows prow[0 .. r), ascending lead, reduced in place
        StreamOut* so = out->stream_out;
        int32_t* pcd = nullptr;          // pivot columns, descending (the answer's order)
        int64_t* cnt = nullptr;          // [NB + 1] entries per row of a block
        int64_t* loc = nullptr;          // [NB + 1] their exclusive scan
        void* cscan = nullptr;
        size_t cscan_bytes = 0;
        cudaEvent_t blk_ev = nullptr;
        if (so) {
            pcd = c.alloc<int32_t>(r);
            cnt = c.alloc<int64_t>(nb_for(r) + 1);
            loc = c.alloc<int64_t>(nb_for(r) + 1);
            cub::DeviceScan::ExclusiveSum(nullptr, cscan_bytes, cnt, loc, nb_for(r) + 1, s);
            cscan = c.alloc<uint8_t>(cscan_bytes);
            if (!pcd || !cnt || !loc || !cscan) return GBGPU_ENOMEM;
            BL_LAUNCH(k_reverse_i32<<<grid_of(r), 256, 0, s>>>(r, pc, pcd));
            BL_CUDA(cudaEventCreateWithFlags(&blk_ev, cudaEventDisableTiming));
            so->nnz = 0;
            so->overflow = false;
        }
        // block b's answer rows [r - b NB - kb, r - b NB): compacted and sent
        auto send_block = [&](int b, int kb) -> int {
            const int64_t out0 = (int64_t)r - ((int64_t)b * nb_for(r) + kb);
            BL_LAUNCH(k_row_nnz<<<grid_of((int64_t)kb * 32), 256, 0, s>>>(
                kb, pcd + out0, piv_of_col, Dp, ld, ncr, cnt));
            BL_CUDA(cudaMemsetAsync(cnt + kb, 0, sizeof(int64_t), s));
            size_t bytes = cscan_bytes;
            BL_CUDA(cub::DeviceScan::ExclusiveSum(cscan, bytes, cnt, loc, kb + 1, s));
            ++c.launches;
            int64_t blk = 0;
            BL_CUDA(cudaMemcpyAsync(&blk, loc + kb, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
            BL_CUDA(cudaStreamSynchronize(s));
            BL_LAUNCH(k_offs_write<<<grid_of(kb + 1), 256, 0, s>>>(kb + 1, loc, so->nnz,
                                                                   so->offs + out0));
            if (blk > 0) {
                int32_t* bc = nullptr;
                uint8_t* bw = nullptr;
                const int vb = so->val_bytes;
                if (cudaMallocAsync((void**)&bc, sizeof(int32_t) * blk, s) != cudaSuccess ||
                    cudaMallocAsync((void**)&bw, (size_t)vb * blk, s) != cudaSuccess) {
                    set_error("answer block allocation failed");
                    return GBGPU_ENOMEM;
                }
                BL_LAUNCH(k_row_write<<<grid_of((int64_t)kb * 32), 256, 0, s>>>(
                    kb, pcd + out0, piv_of_col, Dp, ld, ncr, loc, so->col_shift, bc, bw, vb));
                cudaStream_t fs = s;
                if (!so->overflow && so->nnz + blk <= so->cap_nnz) {
                    BL_CUDA(cudaEventRecord(blk_ev, s));
                    BL_CUDA(cudaStreamWaitEvent(so->s_out, blk_ev, 0));
                    BL_CUDA(cudaMemcpyAsync(so->h_cols + so->nnz, bc, sizeof(int32_t) * blk,
                                            cudaMemcpyDeviceToHost, so->s_out));
                    BL_CUDA(cudaMemcpyAsync((uint8_t*)so->h_vals + (size_t)so->nnz * vb, bw,
                                            (size_t)vb * blk, cudaMemcpyDeviceToHost, so->s_out));
                    fs = so->s_out;  // freed once copied
                } else {
                    so->overflow = true;
                }
                cudaFreeAsync(bc, fs);
                cudaFreeAsync(bw, fs);
            }
            so->nnz += blk;
            return GBGPU_OK;
        };
        const int32_t NB = nb_for(r);
        const int64_t bstride = (int64_t)NB * (NB + 1);
        const int32_t nb = (r + NB - 1) / NB;
        uint32_t* Ublk = c.alloc<uint32_t>((size_t)nb * NB * NB);
        uint32_t* Ninv = c.alloc<uint32_t>((size_t)nb * bstride);
        uint32_t* G = c.alloc<uint32_t>((size_t)NB * std::max(r, 1));
        uint32_t* Y = c.alloc<uint32_t>((size_t)NB * ld);
        if (!Ublk || !Ninv || !G || !Y) return GBGPU_ENOMEM;
        for (int b = 0; b < nb; ++b) {
            const int kb = std::min(NB, r - b * NB);
            BL_LAUNCH(k_gather_cols<<<grid_of((int64_t)kb * kb), 256, 0, s>>>(
                kb, kb, Dp, ld, pc + b * NB, Ublk + (size_t)b * NB * NB, NB, prow + b * NB));
        }
        BL_CHECK(neg_inverse_big(c, f, Ublk, NB, (int64_t)NB * NB, nb, r - (nb - 1) * NB, NB, Ninv));
        for (int b = nb - 1; b >= 0; --b) {
            const int kb = std::min(NB, r - b * NB);
            const int32_t later = r - (b * NB + kb);
            const int32_t* rows_k = prow + b * NB;
            const int32_t c0 = h_pc[b * NB];
            if (later > 0) {
                // E_k -= E_k[:, pc(>k)] R(>k)
                BL_LAUNCH(k_gather_cols<<<grid_of((int64_t)kb * later), 256, 0, s>>>(
                    kb, later, Dp, ld, pc + b * NB + kb, G, later, rows_k));
                const int32_t c_later = h_pc[b * NB + kb];
                TcGemmArgs g{c.p, kb, ncr - c_later, later, G, later, Dp + c_later, ld,
                             Dp + c_later, ld};
                g.b_rows = rows_k + kb;
                g.d_rows = rows_k;
                BL_CHECK(gemm_args(c, g));
            }
            // E_k = (E_k[:, pc(k)])^-1 E_k, as Y = 0 - (-(U_kk)^-1) E_k, E_k = Y
            BL_CUDA(cudaMemset2DAsync(Y + c0, ld * 4, 0, (size_t)(ncr - c0) * 4, kb, s));
            TcGemmArgs g{c.p, kb, ncr - c0, kb, Ninv + (size_t)b * bstride, NB, Dp + c0, ld, Y + c0,
                         ld};
            g.b_rows = rows_k;
            BL_CHECK(gemm_args(c, g));
            BL_LAUNCH(k_scatter_rows_dense<<<grid_of((int64_t)kb * (ncr - c0)), 256, 0, s>>>(
                kb, rows_k, ncr - c0, Y + c0, ld, Dp + c0, ld));
            if (so) BL_CHECK(send_block(b, kb));
        }
        if (blk_ev) cudaEventDestroy(blk_ev);
    } else if (out->stream_out) {
        out->stream_out->nnz = 0;
        BL_CUDA(cudaMemsetAsync(out->stream_out->offs, 0, sizeof(int64_t), s));
    }
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

// dst row i = src row order[i] (all ncols), rows >= n zeroed up to `rows`
__global__ void k_order_rows(int32_t n, int32_t rows, const int32_t* __restrict__ order,
                             int32_t ncols, const uint32_t* __restrict__ src, int64_t lds,
                             uint32_t* dst, int64_t ldd) {
    const int64_t total = (int64_t)rows * ncols;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = t / ncols;
        const int j = (int)(t % ncols);
        dst[i * ldd + j] = i < n ? src[(int64_t)order[i] * lds + j] : 0u;
    }
}

template <class F>
static int dense_rref_run(const DenseRrefInput& in, int32_t* rank, Ctx& c, const F& f) {
    BlockedOutput out{};
    int32_t* piv_of_col = c.alloc<int32_t>(in.cols);
    if (!piv_of_col) return GBGPU_ENOMEM;
    out.piv_of_col = piv_of_col;
    BL_CHECK(echelon_rref(c, f, in.D, in.ld, in.rows, in.cols, &out));
    const int32_t r = (int32_t)out.rank;
    *rank = r;
    // pivot rows in ascending pivot order into the first r rows, zeros after
    int32_t* flag = c.alloc<int32_t>(in.cols);
    int32_t* pos = c.alloc<int32_t>(in.cols);
    int32_t* order = c.alloc<int32_t>(std::max(r, 1));
    int32_t* cnt = c.alloc<int32_t>(1);
    uint32_t* tmp = c.alloc<uint32_t>((size_t)in.rows * in.ld);
    if (!flag || !pos || !order || !cnt || !tmp) return GBGPU_ENOMEM;
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, flag, pos, in.cols, c.s);
    void* scan_tmp = c.alloc<uint8_t>(bytes);
    if (!scan_tmp) return GBGPU_ENOMEM;
    BL_LAUNCH(k_pivot_flags<<<grid_of(in.cols), 256, 0, c.s>>>(in.cols, piv_of_col, 0, flag));
    BL_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, bytes, flag, pos, in.cols, c.s));
    BL_LAUNCH(k_compact_cols<<<grid_of(in.cols), 256, 0, c.s>>>(in.cols, flag, pos, in.piv_cols));
    if (r > 0)
        BL_LAUNCH(k_gather_rows<<<grid_of(r), 256, 0, c.s>>>(r, in.piv_cols, piv_of_col, order, cnt));
    BL_LAUNCH(k_order_rows<<<grid_of((int64_t)in.rows * in.cols), 256, 0, c.s>>>(
        r, in.rows, order, in.cols, in.D, in.ld, tmp, in.ld));
    BL_CUDA(cudaMemcpy2DAsync(in.D, in.ld * 4, tmp, in.ld * 4, (size_t)in.cols * 4, in.rows,
                              cudaMemcpyDeviceToDevice, c.s));
    return GBGPU_OK;
}

int dense_rref(const DenseRrefInput& in, int32_t* rank, long long* launches) {
    Ctx c;
    c.s = in.stream;
    c.p = in.p;
    c.form = in.form;
    c.err = in.err;
    int rc;
    if (in.p < 65536u)
        rc = dense_rref_run(in, rank, c, FieldSmall::make(in.p));
    else
        rc = dense_rref_run(in, rank, c, FieldMont::make(in.p));
    *launches += c.launches;
    c.release();
    return rc;
}

void blocked_release(BlockedOutput* out, cudaStream_t s) {
    if (!out->keep) return;
    for (void* q : *out->keep) cudaFreeAsync(q, s);
    delete out->keep;
    out->keep = nullptr;
}

}  // namespace gbgpu
