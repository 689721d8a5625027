// tiny.cuh -- the one-CTA reduced echelon form and compaction of a small
// dense block (the body of plain.cu's k_tiny_rref, also run per matrix by the
// batched small-matrix kernel of small.cu).  See plain.cu for the algorithm.
#pragma once
#include <climits>
#include <stdint.h>

#include "common.cuh"

namespace gbgpu {

constexpr int kTinyThreads = 1024;

// in-place exclusive prefix sum of a[0..n) in shared memory; returns the total
__device__ inline int tiny_exscan(int* a, int n, int* tmp) {
    for (int off = 1; off < n; off <<= 1) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) tmp[i] = a[i] + (i >= off ? a[i - off] : 0);
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] = tmp[i];
        __syncthreads();
    }
    const int total = n > 0 ? a[n - 1] : 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) tmp[i] = i > 0 ? a[i - 1] : 0;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) a[i] = tmp[i];
    __syncthreads();
    return total;
}

struct TinyOut {
    int32_t col_shift;
    int64_t* offs;      // [rank + 1]
    int32_t* cols;      // [entries]
    int32_t* vals;      // [entries]
    int32_t* piv_of_col;  // [m]
    int64_t* counts;    // rows, entries
};

template <class F>
__device__ void tiny_rref_body(int32_t n, int32_t m, const uint32_t* __restrict__ D, int64_t ld,
                               const int32_t* __restrict__ lead_in, const uint32_t* err,
                               TinyOut out, F f, uint32_t* tiny_smem) {
    const int tld = m + 1;
    uint32_t* T = tiny_smem;                                 // [n][m + 1]
    int32_t* lead = (int32_t*)(tiny_smem + (size_t)n * tld);  // [n]
    int32_t* pcol = lead + n;                                // [n] pivot column of a pivot row, -1
    int32_t* rcnt = pcol + n;                                // [n] entries of a pivot row
    int32_t* prow = rcnt + n;                                // [m] pivot row of a column, -1
    int32_t* rank = prow + m;                                // [max(n, m)] scan space
    int32_t* tmp = rank + max(n, m);                         // [max(n, m)]
    uint32_t* rinv = (uint32_t*)(tmp + max(n, m));           // [n] inverse of a row's lead entry
    __shared__ int s_min[2][kTinyThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = kTinyThreads / 32;
    static_assert(NW == 32, "one warp minimum per lane");
    if (*err) {  // invalid input: nothing is read, the answer is empty (uniform)
        for (int c = tid; c < m; c += blockDim.x) out.piv_of_col[c] = -1;
        if (tid == 0) {
            out.offs[0] = 0;
            out.counts[0] = 0;
            out.counts[1] = 0;
        }
        return;
    }
    for (int c = tid; c < m; c += blockDim.x) prow[c] = -1;
    for (int64_t t = tid; t < (int64_t)n * m; t += blockDim.x) {
        const int r = (int)(t / m), c = (int)(t % m);
        T[(size_t)r * tld + c] = D[(size_t)r * ld + c];
    }
    __syncthreads();  // the lead entries below were loaded by other threads
    for (int r = tid; r < n; r += blockDim.x) {
        const int l = lead_in[r] < 0 ? INT_MAX : lead_in[r];
        lead[r] = l;
        pcol[r] = -1;
        // inverse of the row's lead entry, ready for the step that picks it
        rinv[r] = l == INT_MAX ? 0u : f.inv(T[(size_t)r * tld + l]);
    }
    __syncthreads();
    // Pivot rows are normalised at the end (the entry at a pivot column never
    // changes afterwards, pivot columns only grow); a step clears the pivot
    // column with row_r -= (row_r[c] / a_i) row_i, the inverse of a_i being
    // ready since row i's lead was last set.  Every warp publishes the key of
    // its rows right after its own updates: one barrier per pivot.
    auto warp_key = [&]() {
        int key = INT_MAX;
        for (int r = warp + NW * lane; r < n; r += NW * 32)
            if (pcol[r] < 0 && lead[r] != INT_MAX) key = min(key, lead[r] * n + r);
        for (int o = 16; o > 0; o >>= 1) key = min(key, __shfl_xor_sync(0xffffffffu, key, o));
        return key;
    };
    {
        const int key = warp_key();
        if (lane == 0) s_min[0][warp] = key;
    }
    __syncthreads();
    for (int step = 0; step < n; ++step) {
        const int* sm = s_min[step & 1];
        // the NW (= 32) warp minima: one read per lane, then a warp reduction
        int best = sm[lane];
        for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
        if (best == INT_MAX) break;  // uniform: rank reached
        const int c = best / n, i = best % n;
        const uint32_t* pr = T + (size_t)i * tld;
        const uint32_t ainv = rinv[i];
        if (warp == (i % NW) && lane == 0) {
            pcol[i] = c;
            prow[c] = i;
        }
        __syncwarp();  // the owner warp's lanes see pcol[i]
        // clear column c from this warp's other rows, pivots included
        for (int r = warp; r < n; r += NW) {
            if (r == i) continue;
            uint32_t* row = T + (size_t)r * tld;
            const uint32_t mr = row[c];
            if (mr == 0u) continue;  // uniform over the warp
            const uint32_t mp = f.prep(f.mulmod(mr, ainv));
            const bool track = pcol[r] < 0;  // its lead was c: find the next one
            int nl = INT_MAX;
            for (int j0 = c + 1; j0 < m; j0 += 32) {
                const int j = j0 + lane;
                uint32_t y = 0u;
                if (j < m) {
                    const uint32_t v = pr[j];
                    y = row[j];
                    if (v) {
                        y = f.mulsub(y, mp, v);
                        row[j] = y;
                    }
                }
                if (track && nl == INT_MAX) {
                    const unsigned bal = __ballot_sync(0xffffffffu, y != 0u);
                    if (bal) nl = j0 + __ffs(bal) - 1;
                }
            }
            __syncwarp();
            if (lane == 0) {
                row[c] = 0u;
                if (track) {
                    lead[r] = nl;
                    rinv[r] = nl == INT_MAX ? 0u : f.inv(row[nl]);
                }
            }
            __syncwarp();
        }
        const int key = warp_key();
        if (lane == 0) s_min[(step + 1) & 1][warp] = key;
        __syncthreads();
    }
    // normalise the pivot rows
    for (int r = warp; r < n; r += NW) {
        const int c0 = pcol[r];
        if (c0 < 0) continue;
        uint32_t* row = T + (size_t)r * tld;
        const uint32_t ip = f.prep(rinv[r]);
        for (int j = c0 + 1 + lane; j < m; j += 32) {
            const uint32_t v = row[j];
            if (v) row[j] = f.mulp(v, ip);
        }
        __syncwarp();
        if (lane == 0) row[c0] = 1u;
    }
    __syncthreads();
    // ---- compaction: pivot rows in descending pivot-column order ----
    for (int r = warp; r < n; r += NW) {
        const int c0 = pcol[r];
        if (c0 < 0) continue;
        const uint32_t* row = T + (size_t)r * tld;
        int cnt = 0;
        for (int j0 = c0; j0 < m; j0 += 32) {
            const int j = j0 + lane;
            cnt += __popc(__ballot_sync(0xffffffffu, j < m && row[j] != 0u));
        }
        if (lane == 0) rcnt[r] = cnt;
    }
    // rank of a pivot column = pivot columns to its right
    for (int c = tid; c < m; c += blockDim.x) rank[c] = prow[m - 1 - c] >= 0 ? 1 : 0;
    __syncthreads();
    const int np = tiny_exscan(rank, m, tmp);  // rank[m-1-c] = pivots right of c
    // entries per output row (rank order) -> offsets
    for (int c = tid; c < m; c += blockDim.x) {
        const int r = prow[c];
        if (r >= 0) tmp[rank[m - 1 - c]] = rcnt[r];
    }
    __syncthreads();
    for (int k = tid; k < np; k += blockDim.x) rcnt[k] = tmp[k];  // rcnt reused: [np]
    __syncthreads();
    const int nnz = tiny_exscan(rcnt, np, tmp);
    for (int k = tid; k < np; k += blockDim.x) out.offs[k] = rcnt[k];
    for (int c = tid; c < m; c += blockDim.x) out.piv_of_col[c] = prow[c];
    if (tid == 0) {
        out.offs[np] = nnz;
        out.counts[0] = np;
        out.counts[1] = nnz;
    }
    for (int r = warp; r < n; r += NW) {
        const int c0 = pcol[r];
        if (c0 < 0) continue;
        const uint32_t* row = T + (size_t)r * tld;
        int64_t pos = rcnt[rank[m - 1 - c0]];
        for (int j0 = c0; j0 < m; j0 += 32) {
            const int j = j0 + lane;
            const uint32_t v = j < m ? row[j] : 0u;
            const unsigned bal = __ballot_sync(0xffffffffu, v != 0u);
            if (v) {
                const int64_t q = pos + __popc(bal & ((1u << lane) - 1u));
                out.cols[q] = j + out.col_shift;
                out.vals[q] = (int32_t)v;
            }
            pos += __popc(bal);
        }
    }
}

}  // namespace gbgpu
