// plain.cu -- the plain (CUDA-core) form of the GF(p) Macaulay reduction.
//
// Pipeline (host side in api.cu):
//   1. k_check / k_classify / k_mark_lower: input contract, the known pivot of
//      every lead (first row with that lead, src/la_ff_16.c:762-772) and the
//      list of C|D rows.
//   2. k_reduce_sparse: each C|D row is reduced by the known A|B pivots (the
//      sparse A^-1 step of src/la_ff_16.c:289-351 / :102-190) by one CTA with
//      a dense accumulator of the row in shared memory (global scratch when the
//      row does not fit); the D part is written out dense.
//   3. echelon rounds on the dense D' rows: every nonzero row claims its lead
//      column, one winner per column becomes a normalised pivot, the others
//      are reduced by the pivots until their lead is a free column
//      (src/la_ff_16.c:873-989 without the CAS retry loop).
//   4. k_reduce_dense in full mode: every pivot row is reduced by the echelon
//      pivots of all later columns, which gives the reduced row echelon form
//      (the result of interreduce_dense_matrix, src/la_ff_16.c:837-871).
//   5. compaction into CSR rows in descending lead order
//      (convert_to_sparse_matrix_rows, src/la_ff_16.c:1322-1392).
//
// Exactness: every value is a residue in [0, p) after every update (field.cuh).
#include <climits>

#include "common.cuh"
#include "internal.h"
#include "kernels.h"
#include "tiny.cuh"

namespace gbgpu {

// ---------------------------------------------------------------------------
// 1. classification and input checks
__global__ void k_check_rows(int32_t nr, const int64_t* __restrict__ row_ptr,
                             const int32_t* __restrict__ cols,
                             const uint32_t* __restrict__ vals, int32_t lead_bound,
                             int32_t nc, uint32_t p, uint32_t* err) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < nr; i += nwarps) {
        const int64_t b = row_ptr[i], e = row_ptr[i + 1];
        uint32_t bad = 0;
        if (e <= b) {
            bad |= kErrEmptyRow;
        } else {
            const int32_t lead = cols[b];
            if (lead < 0 || lead >= lead_bound) bad |= kErrLeadRange;
            if (vals[b] != 1u) bad |= kErrNotMonic;
            for (int64_t k = b + lane; k < e; k += 32) {
                const int32_t c = cols[k];
                const uint32_t v = vals[k];
                if (c < lead || c >= nc || (k > b && c == lead)) bad |= kErrColRange;
                if (v == 0u || v >= p) bad |= kErrCoefRange;
            }
        }
        for (int o = 16; o > 0; o >>= 1) bad |= __shfl_xor_sync(0xffffffffu, bad, o);
        if (lane == 0 && bad) atomicOr(err, bad);
    }
}

__global__ void k_fill_i32(int32_t* a, int64_t n, int32_t v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        a[i] = v;
}

// piv_row[c] = smallest row index whose lead is c (INT_MAX if none).
__global__ void k_classify(int32_t nr, const int64_t* __restrict__ row_ptr,
                           const int32_t* __restrict__ cols, int32_t table_size,
                           int32_t* piv_row) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nr; i += gridDim.x * blockDim.x) {
        const int64_t b = row_ptr[i];
        if (row_ptr[i + 1] <= b) continue;
        const int32_t lead = cols[b];
        if (lead >= 0 && lead < table_size) atomicMin(&piv_row[lead], i);
    }
}

// flag[i] = 1 for rows that are not the known pivot of their lead.
__global__ void k_mark_lower(int32_t nr, const int64_t* __restrict__ row_ptr,
                             const int32_t* __restrict__ cols, int32_t table_size,
                             const int32_t* __restrict__ piv_row, uint8_t* flag,
                             uint32_t* err, int32_t dup_is_error) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nr; i += gridDim.x * blockDim.x) {
        const int64_t b = row_ptr[i];
        uint8_t f = 0;
        if (row_ptr[i + 1] > b) {
            const int32_t lead = cols[b];
            if (lead >= 0 && lead < table_size) f = piv_row[lead] != i;
        }
        flag[i] = f;
        if (f && dup_is_error) atomicOr(err, kErrDupLead);
    }
}

__global__ void k_iota(int32_t* a, int32_t n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        a[i] = i;
}

// pivot table with -1 for columns that lead no row
__global__ void k_pivtab(int32_t n, const int32_t* __restrict__ piv_row, int32_t* piv_of_col) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        piv_of_col[i] = piv_row[i] == INT_MAX ? -1 : piv_row[i];
}

// out[i] = pivot row of the i-th pivot column; *n_out = n
__global__ void k_gather_rows(int32_t n, const int32_t* __restrict__ pivcol,
                              const int32_t* __restrict__ piv_of_col, int32_t* out,
                              int32_t* n_out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = piv_of_col[pivcol[i]];
    if (blockIdx.x == 0 && threadIdx.x == 0) *n_out = n;
}

// every column below ncl needs a known pivot
__global__ void k_check_pivots(int32_t ncl, const int32_t* __restrict__ piv_row, uint32_t* err) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncl; c += gridDim.x * blockDim.x)
        if (piv_row[c] == INT_MAX) atomicOr(err, kErrMissingPivot);
}

// ---------------------------------------------------------------------------
// 2. reduction of sparse rows by sparse pivot rows
//
// One CTA per row (persistent CTAs pull rows from a queue in order, so CTAs
// that run together sweep nearby pivot rows and share them in L2).  The row
// lives in a dense accumulator acc[0, nc).  Each step finds the first column
// after the last one handled whose value is nonzero and which has a pivot,
// then subtracts m * (pivot row) with m = acc[col] (pivot rows are monic).
// The lead entry of the pivot row is not applied; acc[col] is cleared.
template <class F, bool SMEM>
__global__ void __launch_bounds__(kReduceThreads)
k_reduce_sparse(SparseReduceArgs a, F f) {
    extern __shared__ __align__(16) uint32_t s_acc[];
    __shared__ int s_scratch[kReduceThreads / 32];
    __shared__ int s_work;
    uint32_t* acc = SMEM ? s_acc : a.gacc + (size_t)blockIdx.x * a.acc_stride;
    const int tid = threadIdx.x, nt = blockDim.x;
    if (a.err && *a.err) return;  // invalid input: nothing is read (uniform)

    for (;;) {
        if (tid == 0) s_work = atomicAdd(a.queue, 1);
        __syncthreads();
        const int w = s_work;
        __syncthreads();
        if (w >= a.n_work) break;
        const int32_t r = a.work[w];
        const int64_t rb = a.row_ptr[r], re = a.row_ptr[r + 1];
        const int32_t lead = a.cols[rb];

        for (int c = lead + tid; c < a.nc; c += nt) acc[c] = 0u;
        __syncthreads();
        for (int64_t k = rb + tid; k < re; k += nt) acc[a.cols[k]] = a.vals[k];
        __syncthreads();

        int last = lead - 1 + a.skip_lead;  // columns <= last are done
        for (;;) {
            // scan windows of nt columns after `last`
            int found = INT_MAX;
            uint32_t m = 0;
            for (int base = last + 1; base < a.piv_limit; base += nt) {
                const int c = base + tid;
                int cand = INT_MAX;
                if (c < a.piv_limit && acc[c] != 0u && a.piv_row[c] != INT_MAX) cand = c;
                found = block_min(cand, s_scratch);
                if (found != INT_MAX) break;
            }
            if (found == INT_MAX) break;
            m = f.prep(acc[found]);
            const int32_t pr = a.piv_row[found];
            const int64_t pb = a.row_ptr[pr] + 1, pe = a.row_ptr[pr + 1];
            __syncthreads();  // every thread read acc[found] before it is cleared
            for (int64_t k = pb + tid; k < pe; k += nt) {
                const int32_t c = a.cols[k];
                acc[c] = f.mulsub(acc[c], m, a.vals[k]);
            }
            if (tid == 0) acc[found] = 0u;
            if (tid == 0) atomicAdd((unsigned long long*)a.work_count,
                                    (unsigned long long)(pe - pb + 1));
            last = found;
            __syncthreads();
        }

        // write the window [emit_from, emit_from + emit_width) and its lead
        uint32_t* out = a.out + (size_t)w * a.out_ld;
        int first = INT_MAX;
        for (int k = tid; k < a.emit_width; k += nt) {
            const uint32_t v = acc[a.emit_from + k];
            out[k] = v;
            if (v != 0u && k < first) first = k;
        }
        first = block_min(first, s_scratch);
        if (tid == 0) a.out_lead[w] = first == INT_MAX ? -1 : first;
    }
}

// ---------------------------------------------------------------------------
// 2'. the same reduction by a team of warps per row with the pivot rows staged
// in shared memory ahead of use.
//
// One CTA (kTeamThreads) per row, the row's dense accumulator in shared
// memory.  The known pivots are applied in column order like the reference's
// reduce_dense_row_by_old_pivots (src/la_ff_16.c:289-351): the next pivot is
// the first nonzero column after the last one cleared.  Each step costs two
// barriers and no global round trip on its critical path: the cols/vals of the
// next two pivot rows the accumulator predicts (the next nonzero columns as it
// stands) are already being copied into a three-slot ring by cp.async while
// the current one is applied; a wrong prediction (an update created or
// cancelled a nonzero before the predicted column) drains the ring and
// restarts it at the true next pivot.  Pivot-row extents come from a window of
// 256 columns staged in shared memory.  The staged copies read whole 16-byte
// groups around each row, so cols/vals carry at least 4 elements of padding.
constexpr int kTeamThreads = 256;
constexpr int kStageLen = 2048;  // entries of one staged pivot row (longer rows: tail from global)
constexpr int kStages = 3;
constexpr int kExtWin = 256;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ext[c] = {first applied entry, end} of the pivot row of column c (its lead
// entry excluded), {-1, -1} when column c has no pivot
__global__ void k_pivot_extents(int32_t n, const int32_t* __restrict__ piv_row,
                                const int64_t* __restrict__ row_ptr, longlong2* ext) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int32_t r = piv_row[c];
        ext[c] = r == INT_MAX ? make_longlong2(-1, -1)
                              : make_longlong2(row_ptr[r] + 1, row_ptr[r + 1]);
    }
}

template <class F, bool CHECK>
__global__ void __launch_bounds__(kTeamThreads, 1)
k_reduce_team(SparseReduceArgs a, const longlong2* __restrict__ pext, F f) {
    extern __shared__ __align__(16) uint32_t t_smem[];
    uint32_t* st_cols = t_smem;                          // [kStages][kStageLen]
    uint32_t* st_vals = t_smem + kStages * kStageLen;    // [kStages][kStageLen]
    uint32_t* acc = t_smem + 2 * kStages * kStageLen;    // [nc]
    __shared__ longlong2 s_ext[kExtWin];
    __shared__ int s_scratch[kTeamThreads / 32];
    __shared__ int s_work;
    const int tid = threadIdx.x, lane = tid & 31;
    const int limit = a.piv_limit;
    if (a.err && *a.err) return;  // invalid input: nothing is read (uniform)
    int wb = -kExtWin;            // first column of the extents window

    // first column c >= from, c < limit, with acc[c] != 0 (and a pivot when
    // CHECK), -1 if none: every warp computes it from the same data
    auto scan = [&](int from) -> int {
        for (int base = from & ~3; base < limit; base += 128) {
            const int c0 = base + 4 * lane;
            uint32_t bits = 0;
            if (c0 < a.nc) {
                const uint4 v = *(const uint4*)(acc + c0);
                const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int c = c0 + j;
                    bool nz = w[j] != 0u && c >= from && c < limit;
                    if (CHECK && nz) nz = a.piv_row[c] != INT_MAX;
                    bits |= nz ? (1u << j) : 0u;
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, bits != 0u);
            if (bal) {
                const int l = __ffs(bal) - 1;
                const uint32_t b = __shfl_sync(0xffffffffu, bits, l);
                return base + 4 * l + __ffs(b) - 1;
            }
        }
        return -1;
    };
    // extents of column c through the shared window (uniform call: barriers)
    auto extent = [&](int c) -> longlong2 {
        if (c < wb || c >= wb + kExtWin) {
            __syncthreads();
            wb = c;
            if (wb + tid < limit) s_ext[tid] = pext[wb + tid];
            __syncthreads();
        }
        return s_ext[c - wb];
    };
    // copy the pivot row of column c into ring slot `slot`; one commit group
    // per call for every thread (empty for c < 0)
    int slot_off[kStages], slot_lim[kStages];
    long long slot_x[kStages], slot_len[kStages];
    auto issue = [&](int c, int slot) {
        if (c >= 0) {
            const longlong2 e = extent(c);
            const long long x0 = e.x & ~3ll, y0 = (e.y + 3) & ~3ll;
            const int n = (int)min(y0 - x0, (long long)kStageLen);
            slot_off[slot] = (int)(e.x - x0);
            slot_lim[slot] = n - (int)(e.x - x0);
            slot_x[slot] = e.x;
            slot_len[slot] = e.y - e.x;
            uint32_t* dc = st_cols + slot * kStageLen;
            uint32_t* dv = st_vals + slot * kStageLen;
            for (int i = 4 * tid; i < n; i += 4 * kTeamThreads) {
                cp_async16(dc + i, a.cols + x0 + i);
                cp_async16(dv + i, a.vals + x0 + i);
            }
        }
        cp_async_commit();
    };

    for (;;) {
        if (tid == 0) s_work = atomicAdd(a.queue, 1);
        __syncthreads();
        const int w = s_work;
        __syncthreads();
        if (w >= a.n_work) break;
        const int32_t r = a.work[w];
        const int64_t rb = a.row_ptr[r], re = a.row_ptr[r + 1];
        const int32_t lead = a.cols[rb];
        for (int c = (min(lead, a.emit_from) & ~3) + 4 * tid; c < a.nc; c += 4 * kTeamThreads)
            *(uint4*)(acc + c) = make_uint4(0u, 0u, 0u, 0u);
        __syncthreads();
        for (int64_t k = rb + tid; k < re; k += kTeamThreads) acc[a.cols[k]] = a.vals[k];
        __syncthreads();
        long long applied = 0;
        int cur = scan(lead + a.skip_lead);
        if (cur >= 0) {
            // ring: cur in slot s0, two predictions behind it
            int s0 = 0, q1 = scan(cur + 1), q2 = q1 >= 0 ? scan(q1 + 1) : -1;
            issue(cur, 0);
            issue(q1, 1);
            issue(q2, 2);
            for (;;) {
                cp_async_wait<2>();  // this thread's copies of `cur` have landed
                __syncthreads();     // ... and every thread's
                const uint32_t m = f.prep(acc[cur]);
                const uint32_t* sc = st_cols + s0 * kStageLen + slot_off[s0];
                const uint32_t* sv = st_vals + s0 * kStageLen + slot_off[s0];
                const int len = (int)slot_len[s0], lim = slot_lim[s0];
                const long long x = slot_x[s0];
                // four entries per thread at a time: their columns are distinct
                // (one pivot row), so all loads go before the stores
                int k = tid;
                const int lim4 = min(len, lim) - 3 * kTeamThreads;
                for (; k < lim4; k += 4 * kTeamThreads) {
                    uint32_t c[4], v[4], y[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        c[u] = sc[k + u * kTeamThreads];
                        v[u] = sv[k + u * kTeamThreads];
                    }
#pragma unroll
                    for (int u = 0; u < 4; ++u) y[u] = acc[c[u]];
#pragma unroll
                    for (int u = 0; u < 4; ++u) acc[c[u]] = f.mulsub(y[u], m, v[u]);
                }
                for (; k < len; k += kTeamThreads) {
                    uint32_t col, v;
                    if (k < lim) {
                        col = sc[k];
                        v = sv[k];
                    } else {
                        col = (uint32_t)a.cols[x + k];
                        v = a.vals[x + k];
                    }
                    acc[col] = f.mulsub(acc[col], m, v);
                }
                applied += len + 1;
                __syncthreads();  // the step's updates are complete
                if (tid == 0) acc[cur] = 0u;  // read by nobody before the row is emitted
                const int nxt = scan(cur + 1);
                if (nxt < 0) break;
                const int s1 = (s0 + 1) % kStages, s2 = (s0 + 2) % kStages;
                if (nxt == q1) {
                    // prediction held: slot s0 is free (its copies landed)
                    const int q3 = q2 >= 0 ? scan(q2 + 1) : scan(nxt + 1);
                    cur = nxt;
                    q1 = q2;
                    q2 = q3;
                    issue(q2, s0);
                    s0 = s1;
                    (void)s2;
                } else {
                    // mispredicted: let the copies in flight land, restart the ring
                    cp_async_wait<0>();
                    __syncthreads();
                    cur = nxt;
                    q1 = scan(cur + 1);
                    q2 = q1 >= 0 ? scan(q1 + 1) : -1;
                    s0 = 0;
                    issue(cur, 0);
                    issue(q1, 1);
                    issue(q2, 2);
                }
            }
            cp_async_wait<0>();
        }
        __syncthreads();
        if (tid == 0 && applied) atomicAdd((unsigned long long*)a.work_count,
                                           (unsigned long long)applied);
        // write the window [emit_from, emit_from + emit_width) and its lead
        uint32_t* out = a.out + (size_t)w * a.out_ld;
        int first = INT_MAX;
        for (int k = tid; k < a.emit_width; k += kTeamThreads) {
            const uint32_t v = acc[a.emit_from + k];
            out[k] = v;
            if (v != 0u && k < first) first = k;
        }
        first = block_min(first, s_scratch);
        if (tid == 0) a.out_lead[w] = first == INT_MAX ? -1 : first;
    }
}

// shared memory of k_reduce_team for nc columns (0: too large for one CTA)
int team_smem_bytes(int32_t nc, int smem_optin) {
    const int64_t b = (int64_t)2 * kStages * kStageLen * 4 + (((int64_t)nc + 3) & ~3ll) * 4;
    return b + 4096 <= smem_optin ? (int)b : 0;
}

// ---------------------------------------------------------------------------
// 3./4. reduction of dense rows by dense (echelon) pivot rows
//
// mode kUntilFree: reduce row r (in place in `rows`) by the pivots of its
//   nonzero columns, left to right, until its first nonzero column has no
//   pivot (its new lead) or the row is zero (lead -1).  Survivors are pushed
//   onto `next` for the next claiming round.
// mode kFull: reduce pivot row r of `src` by the pivots of every later
//   nonzero column and write the result to `dst` (reduced echelon form).
template <class F, bool SMEM>
__global__ void __launch_bounds__(kReduceThreads)
k_reduce_dense(DenseReduceArgs a, F f) {
    extern __shared__ __align__(16) uint32_t s_acc[];
    __shared__ int s_scratch[kReduceThreads / 32];
    __shared__ int s_work;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int ncr = a.ncr;

    for (;;) {
        if (tid == 0) s_work = atomicAdd(a.queue, 1);
        __syncthreads();
        const int w = s_work;
        __syncthreads();
        if (w >= *a.n_work) break;
        const int32_t r = a.work[w];
        const int32_t lead = a.lead[r];
        const uint32_t* src = a.src + (size_t)r * a.ld;
        uint32_t* dst = a.dst + (size_t)r * a.ld;
        uint32_t* acc = SMEM ? s_acc : dst;
        if (SMEM || src != dst) {
            for (int c = lead + tid; c < ncr; c += nt) acc[c] = src[c];
            __syncthreads();
        }
        int last = a.mode == kFull ? lead : lead - 1;
        int new_lead = -1;
        for (;;) {
            int found = INT_MAX;
            for (int base = last + 1; base < ncr; base += nt) {
                const int c = base + tid;
                int cand = INT_MAX;
                if (c < ncr && acc[c] != 0u) {
                    if (a.mode == kUntilFree || a.piv_of_col[c] >= 0) cand = c;
                }
                found = block_min(cand, s_scratch);
                if (found != INT_MAX) break;
            }
            if (found == INT_MAX) break;
            const int32_t pr = a.piv_of_col[found];
            if (pr < 0) {  // kUntilFree only: a free column is the new lead
                new_lead = found;
                break;
            }
            const uint32_t m = f.prep(acc[found]);
            const uint32_t* prow = a.src + (size_t)pr * a.ld;
            __syncthreads();
            for (int c = found + 1 + tid; c < ncr; c += nt) {
                const uint32_t v = prow[c];
                if (v != 0u) acc[c] = f.mulsub(acc[c], m, v);
            }
            if (tid == 0) acc[found] = 0u;
            if (tid == 0) atomicAdd((unsigned long long*)a.work_count,
                                    (unsigned long long)(ncr - found));
            last = found;
            __syncthreads();
        }
        if (SMEM) {
            for (int c = lead + tid; c < ncr; c += nt) dst[c] = acc[c];
        }
        if (a.mode == kUntilFree && tid == 0) {
            a.lead[r] = new_lead;
            if (new_lead >= 0) a.next[atomicAdd(a.n_next, 1)] = r;
        }
        __syncthreads();
    }
}

// claim[lead] = smallest candidate row with that lead
__global__ void k_claim(const int32_t* __restrict__ cand, const int32_t* n_cand,
                        const int32_t* __restrict__ lead, int32_t* claim) {
    const int n = *n_cand;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t r = cand[i];
        atomicMin(&claim[lead[r]], r);
    }
}

// winners become pivots (normalised by a warp each), losers are listed
template <class F>
__global__ void k_promote(const int32_t* __restrict__ cand, const int32_t* n_cand,
                          const int32_t* __restrict__ lead, int32_t* claim, int32_t* piv_of_col,
                          uint32_t* rows, int64_t ld, int32_t ncr, int32_t* losers,
                          int32_t* n_losers, F f) {
    const int n = *n_cand;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < n; i += nwarps) {
        const int32_t r = cand[i];
        const int32_t c = lead[r];
        if (claim[c] == r) {
            uint32_t* row = rows + (size_t)r * ld;
            const uint32_t inv = inverse_mod(row[c], f.p);
            for (int j = c + 1 + lane; j < ncr; j += 32) row[j] = f.mulmod(row[j], inv);
            __syncwarp();
            if (lane == 0) {
                row[c] = 1u;
                piv_of_col[c] = r;
            }
        } else if (lane == 0) {
            losers[atomicAdd(n_losers, 1)] = r;
        }
    }
}

// rows with lead >= 0 -> candidate list (first round)
__global__ void k_collect_nonzero(int32_t n, const int32_t* __restrict__ lead, int32_t* out,
                                  int32_t* n_out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (lead[i] >= 0) out[atomicAdd(n_out, 1)] = i;
}

// ---------------------------------------------------------------------------
// 5. compaction: output row k is the pivot of the k-th pivot column, in
// descending (linear_algebra) or ascending (interreduction) column order
__global__ void k_pivot_flags(int32_t ncr, const int32_t* __restrict__ piv_of_col,
                              int32_t desc, int32_t* flag) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncr; i += gridDim.x * blockDim.x)
        flag[i] = piv_of_col[desc ? ncr - 1 - i : i] >= 0;
}

// pos = exclusive scan of flag; writes the pivot column of output row k
__global__ void k_pivot_list(int32_t ncr, const int32_t* __restrict__ flag,
                             const int32_t* __restrict__ pos, int32_t desc, int32_t* pivcol) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncr; i += gridDim.x * blockDim.x)
        if (flag[i]) pivcol[pos[i]] = desc ? ncr - 1 - i : i;
}

// Both compaction kernels walk a row with one warp, ROW_U chunks of 32
// columns per pass: the ROW_U loads of a lane are independent and in flight
// together (a pass covers 256 columns), so a row costs a few load latencies
// instead of one per 32 columns.
constexpr int ROW_U = 8;

// nnz of each reduced pivot row (one warp per row)
__global__ void k_row_nnz(int32_t np, const int32_t* __restrict__ pivcol,
                          const int32_t* __restrict__ piv_of_col, const uint32_t* __restrict__ rows,
                          int64_t ld, int32_t ncr, int64_t* counts) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < np; i += nwarps) {
        const int32_t c0 = pivcol[i];
        const uint32_t* row = rows + (size_t)piv_of_col[c0] * ld;
        int cnt = 0;
        for (int base = c0; base < ncr; base += 32 * ROW_U) {
            uint32_t v[ROW_U];
#pragma unroll
            for (int u = 0; u < ROW_U; ++u) {
                const int j = base + 32 * u + lane;
                v[u] = j < ncr ? row[j] : 0u;
            }
#pragma unroll
            for (int u = 0; u < ROW_U; ++u) cnt += v[u] != 0u;
        }
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        if (lane == 0) counts[i] = cnt;
    }
}

// write CSR rows: columns shifted by col_shift, values at vb bytes (1, 2 or
// 4: the reference's cf_8 / cf_16 / cf_32 widths), order preserved by a warp
// ballot prefix over each 32-column chunk
__global__ void k_row_write(int32_t np, const int32_t* __restrict__ pivcol,
                            const int32_t* __restrict__ piv_of_col,
                            const uint32_t* __restrict__ rows, int64_t ld, int32_t ncr,
                            const int64_t* __restrict__ offs, int32_t col_shift,
                            int32_t* out_cols, void* out_vals, int32_t vb) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int i = warp; i < np; i += nwarps) {
        const int32_t c0 = pivcol[i];
        const uint32_t* row = rows + (size_t)piv_of_col[c0] * ld;
        int64_t o = offs[i];
        for (int base = c0; base < ncr; base += 32 * ROW_U) {
            uint32_t v[ROW_U];
#pragma unroll
            for (int u = 0; u < ROW_U; ++u) {
                const int j = base + 32 * u + lane;
                v[u] = j < ncr ? __ldcs(row + j) : 0u;
            }
#pragma unroll
            for (int u = 0; u < ROW_U; ++u) {
                const unsigned bal = __ballot_sync(0xffffffffu, v[u] != 0u);
                if (v[u] != 0u) {
                    const int64_t at = o + __popc(bal & ((1u << lane) - 1u));
                    out_cols[at] = base + 32 * u + lane + col_shift;
                    if (vb == 4) ((uint32_t*)out_vals)[at] = v[u];
                    else if (vb == 2) ((uint16_t*)out_vals)[at] = (uint16_t)v[u];
                    else ((uint8_t*)out_vals)[at] = (uint8_t)v[u];
                }
                o += __popc(bal);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// host launchers: every kernel is launched from this translation unit
template <class F>
cudaError_t launch_reduce_team(const SparseReduceArgs& a, const longlong2* pext, const F& f,
                               int grid, int smem_bytes, cudaStream_t s) {
    if (a.skip_lead) {
        cudaError_t e = ensure_smem_limit((const void*)k_reduce_team<F, true>, smem_bytes);
        if (e != cudaSuccess) return e;
        k_reduce_team<F, true><<<grid, kTeamThreads, smem_bytes, s>>>(a, pext, f);
    } else {
        cudaError_t e = ensure_smem_limit((const void*)k_reduce_team<F, false>, smem_bytes);
        if (e != cudaSuccess) return e;
        k_reduce_team<F, false><<<grid, kTeamThreads, smem_bytes, s>>>(a, pext, f);
    }
    return cudaGetLastError();
}

template <class F>
cudaError_t launch_reduce_sparse(const SparseReduceArgs& a, const F& f, int grid, bool smem,
                                 int smem_bytes, cudaStream_t s) {
    if (smem) {
        cudaError_t e = ensure_smem_limit((const void*)k_reduce_sparse<F, true>, smem_bytes);
        if (e != cudaSuccess) return e;
        k_reduce_sparse<F, true><<<grid, kReduceThreads, smem_bytes, s>>>(a, f);
    } else {
        k_reduce_sparse<F, false><<<grid, kReduceThreads, 0, s>>>(a, f);
    }
    return cudaGetLastError();
}

template <class F>
cudaError_t launch_reduce_dense(const DenseReduceArgs& a, const F& f, int grid, bool smem,
                                int smem_bytes, cudaStream_t s) {
    if (smem) {
        cudaError_t e = ensure_smem_limit((const void*)k_reduce_dense<F, true>, smem_bytes);
        if (e != cudaSuccess) return e;
        k_reduce_dense<F, true><<<grid, kReduceThreads, smem_bytes, s>>>(a, f);
    } else {
        k_reduce_dense<F, false><<<grid, kReduceThreads, 0, s>>>(a, f);
    }
    return cudaGetLastError();
}

template <class F>
cudaError_t launch_promote(int grid, int threads, cudaStream_t s, const int32_t* cand,
                           const int32_t* n_cand, const int32_t* lead, int32_t* claim,
                           int32_t* piv_of_col, uint32_t* rows, int64_t ld, int32_t ncr,
                           int32_t* losers, int32_t* n_losers, const F& f) {
    k_promote<F><<<grid, threads, 0, s>>>(cand, n_cand, lead, claim, piv_of_col, rows, ld, ncr,
                                          losers, n_losers, f);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Small matrices: the reduced row echelon form of the whole n x m block D'
// (rows with lead < 0 are zero) and its compaction to CSR in the shared
// memory of ONE CTA, in one launch instead of echelon rounds, back
// substitution and compaction (which cost a host round trip each).  Row r
// belongs to warp r % 32.  A step takes the non-pivot row with the smallest
// (lead, row) as the pivot (the pivots of the column-by-column search),
// normalises it (one inverse, lane 0 of its warp), and every warp clears the
// pivot column from its other rows, pivots included (Gauss-Jordan),
// recomputing the leads of the non-pivot rows it changed.  Output: the pivot
// rows in descending pivot-column order as CSR (columns + col_shift), their
// offsets, piv_of_col, and counts[0..1] = rows, entries.  When the input
// checks flagged an error nothing is read and the answer is empty.
template <class F>
__global__ void __launch_bounds__(kTinyThreads)
k_tiny_rref(int32_t n, int32_t m, const uint32_t* __restrict__ D, int64_t ld,
            const int32_t* __restrict__ lead_in, const uint32_t* err, TinyOut out, F f) {
    extern __shared__ uint32_t tiny_smem[];
    tiny_rref_body(n, m, D, ld, lead_in, err, out, f, tiny_smem);
}

// shared memory of k_tiny_rref for an n x m block (0: too large)
int tiny_rref_bytes(int32_t n, int32_t m, int smem_optin) {
    const int64_t mx = std::max(n, m);
    const int64_t bytes = (int64_t)n * (m + 1) * 4 + (int64_t)n * 16 + (int64_t)m * 4 + mx * 8 + 64;
    return bytes <= smem_optin - 4096 ? (int)bytes : 0;
}

template <class F>
cudaError_t launch_tiny_rref(int32_t n, int32_t m, const uint32_t* D, int64_t ld,
                             const int32_t* lead, const uint32_t* err, int32_t col_shift,
                             int64_t* offs, int32_t* cols, int32_t* vals, int32_t* piv_of_col,
                             int64_t* counts, int bytes, cudaStream_t s, const F& f) {
    cudaError_t e = ensure_smem_limit((const void*)k_tiny_rref<F>, bytes);
    if (e != cudaSuccess) return e;
    const TinyOut o{col_shift, offs, cols, vals, piv_of_col, counts};
    k_tiny_rref<F><<<1, kTinyThreads, bytes, s>>>(n, m, D, ld, lead, err, o, f);
    return cudaGetLastError();
}

#define GBGPU_INSTANTIATE(F)                                                                   \
    template cudaError_t launch_reduce_team<F>(const SparseReduceArgs&, const longlong2*,      \
                                               const F&, int, int, cudaStream_t);              \
    template cudaError_t launch_reduce_sparse<F>(const SparseReduceArgs&, const F&, int, bool, \
                                                 int, cudaStream_t);                            \
    template cudaError_t launch_reduce_dense<F>(const DenseReduceArgs&, const F&, int, bool,   \
                                                int, cudaStream_t);                             \
    template cudaError_t launch_promote<F>(int, int, cudaStream_t, const int32_t*,             \
                                           const int32_t*, const int32_t*, int32_t*, int32_t*, \
                                           uint32_t*, int64_t, int32_t, int32_t*, int32_t*,    \
                                           const F&);                                          \
    template cudaError_t launch_tiny_rref<F>(int32_t, int32_t, const uint32_t*, int64_t,       \
                                             const int32_t*, const uint32_t*, int32_t,         \
                                             int64_t*, int32_t*, int32_t*, int32_t*, int64_t*, \
                                             int, cudaStream_t, const F&);
GBGPU_INSTANTIATE(FieldSmall)
GBGPU_INSTANTIATE(FieldMont)
#undef GBGPU_INSTANTIATE

}  // namespace gbgpu
