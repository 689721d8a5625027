// small.cu -- one-pass reduction of small Macaulay matrices (the la calls of
// the early F4 rounds and of small systems), built for latency.
//
// A general plan (api.cu) creates a stream, allocates a dozen buffers, runs
// ten or more launches and copies in and out through pageable memory; for a
// matrix of a few hundred rows that overhead is most of the call.  Here every
// host thread keeps one session per device (a stream, a device arena, pinned
// input staging and mapped pinned output memory, all grown to a high-water
// mark and reused), and a call is
//
//   rows gathered into pinned staging  ->  one host-to-device copy
//   k_small_prep      (1 CTA)   input checks, known pivots, ordered C|D row list
//   k_reduce_rows_warp          one warp per C|D row, dense accumulator of the
//                               row in shared memory, known pivots applied in
//                               column order (src/la_ff_16.c:289-351 / :102-190)
//   k_tiny_rref       (1 CTA)   reduced echelon form of the right block and its
//                               compaction (plain.cu), written straight into
//                               mapped host memory
//   one 4-byte copy of the checks' verdict, one stream synchronisation.
//
// The answer is the canonical one of every other path (descending leads,
// monic, columns ascending).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gbgpu.h"
#include "common.cuh"
#include "internal.h"
#include "kernels.h"
#include "small.h"
#include "tiny.cuh"

namespace gbgpu {

constexpr int kPrepThreads = 1024;
constexpr int kSmallMaxLeft = 12288;  // left columns: the prep kernel's pivot table in smem
constexpr int kRowWarpsMax = 16;      // warps (rows) per CTA of k_reduce_rows_warp

// ---------------------------------------------------------------------------
// kernels

// Input checks (the contract k_check_rows enforces), the known pivot of every
// left column (first row with that lead, src/la_ff_16.c:762-772), the check
// that every left column has one, and the C|D rows in row order -- one CTA.
__device__ void small_prep_body(int32_t nr, int32_t ncl, int32_t nc, uint32_t p,
                                const int64_t* __restrict__ row_ptr,
                                const int32_t* __restrict__ cols,
                                const uint32_t* __restrict__ vals, int32_t* piv_row,
                                int2* pext, int32_t* work, int32_t* n_work, uint32_t* err,
                                int32_t* prep_tab /* smem [ncl] */) {
    __shared__ uint32_t s_err;
    __shared__ int s_warp[kPrepThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = kPrepThreads / 32;
    for (int c = tid; c < ncl; c += blockDim.x) prep_tab[c] = INT_MAX;
    if (tid == 0) s_err = 0;
    __syncthreads();
    for (int i = warp; i < nr; i += NW) {
        const int64_t b = row_ptr[i], e = row_ptr[i + 1];
        uint32_t bad = 0;
        if (e <= b) {
            bad |= kErrEmptyRow;
        } else {
            const int32_t lead = cols[b];
            if (lead < 0 || lead >= ncl) bad |= kErrLeadRange;
            if (vals[b] != 1u) bad |= kErrNotMonic;
            for (int64_t k = b + lane; k < e; k += 32) {
                const int32_t c = cols[k];
                const uint32_t v = vals[k];
                if (c < lead || c >= nc || (k > b && c == lead)) bad |= kErrColRange;
                if (v == 0u || v >= p) bad |= kErrCoefRange;
            }
            if (lane == 0 && lead >= 0 && lead < ncl) atomicMin(&prep_tab[lead], i);
        }
        for (int o = 16; o > 0; o >>= 1) bad |= __shfl_xor_sync(0xffffffffu, bad, o);
        if (lane == 0 && bad) atomicOr(&s_err, bad);
    }
    __syncthreads();
    for (int c = tid; c < ncl; c += blockDim.x) {
        const int32_t r = prep_tab[c];
        if (r == INT_MAX) atomicOr(&s_err, kErrMissingPivot);
        piv_row[c] = r;
        // the pivot row's applied entries (its lead excluded), as 32-bit offsets
        pext[c] = r == INT_MAX ? make_int2(0, 0)
                               : make_int2((int)row_ptr[r] + 1, (int)row_ptr[r + 1]);
    }
    // rows that are not the known pivot of their lead, in row order
    int base = 0;
    for (int r0 = 0; r0 < nr; r0 += kPrepThreads) {
        const int i = r0 + tid;
        int f = 0;
        if (i < nr) {
            const int64_t b = row_ptr[i];
            if (row_ptr[i + 1] > b) {
                const int32_t lead = cols[b];
                if (lead >= 0 && lead < ncl) f = prep_tab[lead] != i;
            }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, f);
        if (lane == 0) s_warp[warp] = __popc(bal);
        __syncthreads();
        int before = 0, total = 0;
        for (int w = 0; w < NW; ++w) {
            const int c = s_warp[w];
            before += w < warp ? c : 0;
            total += c;
        }
        if (f) work[base + before + __popc(bal & ((1u << lane) - 1u))] = i;
        base += total;
        __syncthreads();  // s_warp is rewritten by the next chunk
    }
    __syncthreads();
    if (tid == 0) {
        *n_work = base;
        *err = s_err;
    }
}

__global__ void __launch_bounds__(kPrepThreads)
k_small_prep(int32_t nr, int32_t ncl, int32_t nc, uint32_t p, const int64_t* __restrict__ row_ptr,
             const int32_t* __restrict__ cols, const uint32_t* __restrict__ vals,
             int32_t* piv_row, int2* pext, int32_t* work, int32_t* n_work, uint32_t* err) {
    extern __shared__ int32_t prep_smem[];  // [ncl]: first row of each lead
    small_prep_body(nr, ncl, nc, p, row_ptr, cols, vals, piv_row, pext, work, n_work, err,
                    prep_smem);
}

// One warp per C|D row: the row is scattered into a dense accumulator of nc
// residues in shared memory, then the known pivots are applied in column
// order -- the next column to clear is the first nonzero left column after
// the last one cleared (a warp ballot over 32 columns at a time); the pivot
// row (monic, its lead skipped) is applied by the 32 lanes in coalesced
// strides (distinct columns, no conflicts).  The right block is written out
// dense with its lead.  Nothing is read when the checks flagged the input.
// rows w = w0, w0 + step, ... (< n_rows) by the calling warp, whose
// accumulator is acc (stride entries, 16-byte aligned).  The pivot chain is
// software-pipelined: before the current pivot row is applied, the warp
// predicts the next pivot (the next nonzero column of the accumulator as it
// stands) and loads that pivot row's first 128 entries, so that when the
// prediction holds (the common case) the next step starts with its data in
// registers; the pivot rows' extents come from a window of 32 consecutive
// columns kept one per lane.
template <class F>
__device__ void rows_warp_body(int32_t n_rows, int w0, int step,
                               const int32_t* __restrict__ work,
                               const int64_t* __restrict__ row_ptr,
                               const int32_t* __restrict__ cols,
                               const uint32_t* __restrict__ vals,
                               const int2* __restrict__ pext, int32_t ncl, int32_t nc,
                               int32_t stride, uint32_t* out, int64_t ld, int32_t* out_lead,
                               F f, uint32_t* acc) {
    const int lane = threadIdx.x & 31;
    const int32_t ncr = nc - ncl;
    // first nonzero left column >= from (-1: none), the same for every lane
    auto scan = [&](int from) -> int {
        for (int base = from; base < ncl; base += 32) {
            const int c = base + lane;
            const unsigned bal = __ballot_sync(0xffffffffu, c < ncl && acc[c] != 0u);
            if (bal) return base + __ffs(bal) - 1;
        }
        return -1;
    };
    int wbase = INT_MIN;  // extents window: lane l holds pext[wbase + l]
    int2 wext = make_int2(0, 0);
    auto extent = [&](int c) -> int2 {
        if (c < wbase || c >= wbase + 32) {
            wbase = c;
            wext = c + lane < ncl ? pext[c + lane] : make_int2(0, 0);
        }
        const int l = c - wbase;
        return make_int2(__shfl_sync(0xffffffffu, wext.x, l), __shfl_sync(0xffffffffu, wext.y, l));
    };
    // the first 128 entries of a pivot row, four per lane
    auto fetch = [&](int2 e, int32_t (&c)[4], uint32_t (&v)[4]) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = e.x + lane + 32 * u;
            c[u] = k < e.y ? cols[k] : -1;
            v[u] = k < e.y ? vals[k] : 0u;
        }
    };
    for (int w = w0; w < n_rows; w += step) {
        const int32_t r = work[w];
        const int64_t rb = row_ptr[r], re = row_ptr[r + 1];
        const int32_t lead = cols[rb];
        for (int c = (lead & ~3) + 4 * lane; c < stride; c += 128)
            *(uint4*)(acc + c) = make_uint4(0u, 0u, 0u, 0u);
        __syncwarp();
        for (int64_t k = rb + lane; k < re; k += 32) acc[cols[k]] = vals[k];
        __syncwarp();
        int found = scan(lead);
        if (found >= 0) {
            int2 e = extent(found);
            int32_t pc[4];
            uint32_t pv[4];
            fetch(e, pc, pv);
            for (;;) {
                const uint32_t m = f.prep(acc[found]);
                // prediction: the next nonzero column before this update
                const int spec = scan(found + 1);
                int2 es = make_int2(0, 0);
                int32_t sc[4];
                uint32_t sv[4];
                if (spec >= 0) {
                    es = extent(spec);
                    fetch(es, sc, sv);
                }
                // this pivot row: the first 128 entries from registers (distinct
                // columns: all loads before the stores), the rest from memory
                uint32_t y[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) y[u] = pc[u] >= 0 ? acc[pc[u]] : 0u;
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (pc[u] >= 0) acc[pc[u]] = f.mulsub(y[u], m, pv[u]);
                for (int k = e.x + 128 + lane; k < e.y; k += 32) {
                    const int32_t c = cols[k];
                    acc[c] = f.mulsub(acc[c], m, vals[k]);
                }
                __syncwarp();
                const int nxt = scan(found + 1);
                if (nxt < 0) break;
                if (nxt == spec) {
                    e = es;
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        pc[u] = sc[u];
                        pv[u] = sv[u];
                    }
                } else {
                    e = extent(nxt);
                    fetch(e, pc, pv);
                }
                found = nxt;
            }
        }
        uint32_t* o = out + (size_t)w * ld;
        int first = -1;
        for (int j0 = 0; j0 < ncr; j0 += 32) {
            const int j = j0 + lane;
            const uint32_t v = j < ncr ? acc[ncl + j] : 0u;
            if (j < ncr) o[j] = v;
            const unsigned bal = __ballot_sync(0xffffffffu, v != 0u);
            if (first < 0 && bal) first = j0 + __ffs(bal) - 1;
        }
        if (lane == 0) out_lead[w] = first;
        __syncwarp();
    }
}

template <class F>
__global__ void __launch_bounds__(kRowWarpsMax * 32)
k_reduce_rows_warp(int32_t n_rows, const int32_t* __restrict__ work,
                   const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ cols,
                   const uint32_t* __restrict__ vals, const int2* __restrict__ pext,
                   int32_t ncl, int32_t nc, int32_t stride, uint32_t* out, int64_t ld,
                   int32_t* out_lead, const uint32_t* err, F f) {
    extern __shared__ __align__(16) uint32_t rw_acc[];
    if (*err) return;  // invalid input: nothing is read (uniform)
    const int warp = threadIdx.x >> 5, wpc = blockDim.x >> 5;
    rows_warp_body(n_rows, blockIdx.x * wpc + warp, gridDim.x * wpc, work, row_ptr, cols, vals,
                   pext, ncl, nc, stride, out, ld, out_lead, f,
                   rw_acc + (size_t)warp * stride);
}


// ---------------------------------------------------------------------------
// batches: every small matrix of a batch in ONE launch.  Each CTA takes the
// next matrix from a device work queue and runs the three phases above on it
// (checks and classification, warp-per-row known-pivot reduction into its
// scratch, one-CTA echelon and compaction into mapped host memory), so the
// uneven small matrices of a batch share one persistent launch.

struct BatchItem {
    int32_t p, nr, ncl, ncr;
    int64_t in_off, cols_off, vals_off;  // bytes into the input buffer
    int64_t scr_off;                     // bytes into the scratch buffer
    int64_t out_off;                     // bytes into the mapped output
    FieldSmall fs;
    FieldMont fm;
};

// scratch of one matrix: piv_row [ncl] | pivot extents [ncl] | work [nr] | n_work, err |
// D [n_work][ld] | lead [n_work] | piv_of_col [ncr]
struct ScrLayout {
    int64_t piv, pext, work, cnt, D, lead, poc, bytes, ld;
};
__host__ __device__ inline int64_t rup(int64_t x, int64_t a) { return (x + a - 1) / a * a; }
__host__ __device__ inline ScrLayout scr_layout(int32_t nr, int32_t ncl, int32_t ncr) {
    ScrLayout L;
    const int64_t nw = nr - ncl > 0 ? nr - ncl : 1;
    L.ld = rup(ncr > 0 ? ncr : 1, 4);
    L.piv = 0;
    L.pext = rup(4 * (int64_t)(ncl > 0 ? ncl : 1), 256);
    L.work = L.pext + rup(8 * (int64_t)(ncl > 0 ? ncl : 1), 256);
    L.cnt = L.work + rup(4 * (int64_t)nr, 256);
    L.D = L.cnt + 256;
    L.lead = L.D + rup(4 * nw * L.ld, 256);
    L.poc = L.lead + rup(4 * nw, 256);
    L.bytes = L.poc + rup(4 * (int64_t)(ncr > 0 ? ncr : 1), 256);
    return L;
}
// mapped output of one matrix: counts[2], err | offs [n_work + 1] | cols | vals
struct OutLayout {
    int64_t offs, cols, vals, bytes;
};
__host__ __device__ inline OutLayout out_layout(int32_t nr, int32_t ncl, int32_t ncr) {
    OutLayout L;
    const int64_t nw = nr - ncl > 0 ? nr - ncl : 0;
    const int64_t cap = nw * (ncr > 0 ? ncr : 0);
    L.offs = 32;
    L.cols = rup(L.offs + 8 * (nw + 1), 16);
    L.vals = rup(L.cols + 4 * (cap > 0 ? cap : 1), 16);
    L.bytes = rup(L.vals + 4 * (cap > 0 ? cap : 1), 256);
    return L;
}

__global__ void __launch_bounds__(kPrepThreads)
k_batch_small(int32_t n, const BatchItem* __restrict__ items, const uint8_t* __restrict__ in,
              uint8_t* scr, uint8_t* out, int32_t* queue, int32_t smem_bytes) {
    extern __shared__ __align__(16) uint8_t bt_smem[];
    __shared__ int s_item;
    const int tid = threadIdx.x, warp = tid >> 5;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(queue, 1);
        __syncthreads();
        const int i = s_item;
        __syncthreads();
        if (i >= n) break;
        const BatchItem it = items[i];
        const int32_t nr = it.nr, ncl = it.ncl, ncr = it.ncr, nc = ncl + ncr;
        const int64_t* row_ptr = (const int64_t*)(in + it.in_off);
        const int32_t* cols = (const int32_t*)(in + it.cols_off);
        const uint32_t* vals = (const uint32_t*)(in + it.vals_off);
        const ScrLayout S = scr_layout(nr, ncl, ncr);
        uint8_t* sb = scr + it.scr_off;
        int32_t* piv = (int32_t*)(sb + S.piv);
        int2* pext = (int2*)(sb + S.pext);
        int32_t* work = (int32_t*)(sb + S.work);
        int32_t* nwork = (int32_t*)(sb + S.cnt);
        uint32_t* err = (uint32_t*)(sb + S.cnt + 16);
        uint32_t* D = (uint32_t*)(sb + S.D);
        int32_t* lead = (int32_t*)(sb + S.lead);
        int32_t* poc = (int32_t*)(sb + S.poc);
        const OutLayout O = out_layout(nr, ncl, ncr);
        uint8_t* ob = out + it.out_off;
        int64_t* counts = (int64_t*)ob;
        small_prep_body(nr, ncl, nc, (uint32_t)it.p, row_ptr, cols, vals, piv, pext, work, nwork, err,
                        (int32_t*)bt_smem);
        __syncthreads();  // prep's global writes are visible to the block
        const uint32_t e = *err;
        const int32_t n_work = nr - ncl;
        if (e == 0 && n_work > 0) {
            const int32_t stride = (int32_t)rup(nc > 0 ? nc : 1, 4);
            const int wpc = min(kPrepThreads / 32, smem_bytes / (stride * 4));
            const TinyOut to{ncl, (int64_t*)(ob + O.offs), (int32_t*)(ob + O.cols),
                             (int32_t*)(ob + O.vals), poc, counts};
            uint32_t* acc = (uint32_t*)bt_smem + (size_t)warp * stride;
            if ((uint32_t)it.p < 65536u) {
                if (warp < wpc)
                    rows_warp_body(n_work, warp, wpc, work, row_ptr, cols, vals, pext, ncl, nc,
                                   stride, D, S.ld, lead, it.fs, acc);
                __syncthreads();
                tiny_rref_body(n_work, ncr, D, S.ld, lead, err, to, it.fs, (uint32_t*)bt_smem);
            } else {
                if (warp < wpc)
                    rows_warp_body(n_work, warp, wpc, work, row_ptr, cols, vals, pext, ncl, nc,
                                   stride, D, S.ld, lead, it.fm, acc);
                __syncthreads();
                tiny_rref_body(n_work, ncr, D, S.ld, lead, err, to, it.fm, (uint32_t*)bt_smem);
            }
        } else if (tid == 0) {
            counts[0] = 0;
            counts[1] = 0;
            ((int64_t*)(ob + O.offs))[0] = 0;
        }
        if (tid == 0) counts[2] = (int64_t)e;
        __syncthreads();  // the shared memory is reused by the next matrix
    }
}

// ---------------------------------------------------------------------------
// host side

namespace {

struct Session {
    DeviceInfo dev{};
    cudaStream_t s = nullptr;
    void* dmem = nullptr;  // device arena
    size_t dcap = 0;
    uint8_t* hin = nullptr;  // pinned input staging
    size_t hin_cap = 0;
    uint8_t* hout = nullptr;  // mapped pinned output
    size_t hout_cap = 0;
    uint32_t* herr = nullptr;  // pinned: the checks' verdict
    ~Session() {
        // runs at thread exit; at process exit the runtime may already be
        // gone, which these calls tolerate
        if (s) cudaStreamSynchronize(s);
        if (dmem) cudaFree(dmem);
        if (hin) cudaFreeHost(hin);
        if (hout) cudaFreeHost(hout);
        if (herr) cudaFreeHost(herr);
        if (s) cudaStreamDestroy(s);
    }
};

constexpr int kMaxDev = 64;
struct Sessions {
    Session* by_dev[kMaxDev] = {};
    ~Sessions() {
        for (auto*& x : by_dev) {
            delete x;
            x = nullptr;
        }
    }
};
thread_local Sessions t_sessions;

size_t round_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

int grow_device(Session& S, size_t need) {
    if (need <= S.dcap) return GBGPU_OK;
    const size_t cap = std::max(need, S.dcap * 2);
    if (S.dmem) {
        cudaStreamSynchronize(S.s);
        cudaFree(S.dmem);
        S.dmem = nullptr;
        S.dcap = 0;
    }
    if (cudaMalloc(&S.dmem, cap) != cudaSuccess) {
        set_error("small-matrix arena allocation failed");
        return GBGPU_ENOMEM;
    }
    S.dcap = cap;
    return GBGPU_OK;
}

int grow_host(uint8_t** buf, size_t* capv, size_t need, unsigned flags, cudaStream_t s) {
    if (need <= *capv) return GBGPU_OK;
    const size_t cap = std::max(need, *capv * 2);
    if (*buf) {
        cudaStreamSynchronize(s);
        cudaFreeHost(*buf);
        *buf = nullptr;
        *capv = 0;
    }
    if (cudaHostAlloc((void**)buf, cap, flags) != cudaSuccess) {
        set_error("small-matrix pinned staging allocation failed");
        return GBGPU_ENOMEM;
    }
    *capv = cap;
    return GBGPU_OK;
}

int session_for(int device, Session** out) {
    if (device < 0 || device >= kMaxDev) {
        set_error("device ordinal out of range");
        return GBGPU_ENODEV;
    }
    Session*& S = t_sessions.by_dev[device];
    if (!S) {
        Session* n = new Session();
        int rc = device_init(device, &n->dev);
        if (rc) {
            delete n;
            return rc;
        }
        if (cudaStreamCreateWithFlags(&n->s, cudaStreamNonBlocking) != cudaSuccess ||
            cudaHostAlloc((void**)&n->herr, 64, cudaHostAllocDefault) != cudaSuccess) {
            delete n;
            set_error("small-matrix session set-up failed");
            return GBGPU_ECUDA;
        }
        S = n;
    }
    *out = S;
    return GBGPU_OK;
}

// the device current on entry is made current again on return
struct DeviceGuard {
    int prev = -1;
    DeviceGuard() {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// rows (warps) per CTA of k_reduce_rows_warp and the accumulator stride
int rows_warps(int32_t nc, const DeviceInfo& dev, int32_t* stride) {
    *stride = (int32_t)round_up((size_t)std::max(nc, 1), 4);
    const int per = *stride * 4;
    const int fit = (dev.smem_optin - 2048) / per;
    return std::min(kRowWarpsMax, fit);
}

}  // namespace

bool small_eligible(int32_t nr, int32_t ncl, int32_t ncr, int device) {
    if (nr <= 0 || ncl < 0 || ncr <= 0 || nr < ncl || ncl > kSmallMaxLeft) return false;
    DeviceGuard guard;
    DeviceInfo dev{};
    if (device_init(device, &dev)) return false;
    int32_t stride = 0;
    if (rows_warps(ncl + ncr, dev, &stride) < 4) return false;
    const int32_t n_work = nr - ncl;
    return n_work == 0 || tiny_rref_bytes(n_work, ncr, dev.smem_optin) > 0;
}

int small_reduce(const SmallInput& in, SmallAnswer* ans) {
    DeviceGuard guard;
    Session* S = nullptr;
    int rc = session_for(in.device, &S);
    if (rc) return rc;
    const int32_t nr = in.nr, ncl = in.ncl, ncr = in.ncr, nc = ncl + ncr;
    const int32_t n_work = nr - ncl;
    const int64_t nnz = in.nnz;
    const int64_t ld = (int64_t)round_up((size_t)std::max(ncr, 1), 4);
    // pinned staging: row_ptr | cols | vals (copied to the arena's start)
    const size_t b_ptr = sizeof(int64_t) * (size_t)(nr + 1);
    const size_t o_cols = round_up(b_ptr, 16);
    const size_t o_vals = round_up(o_cols + 4 * (size_t)nnz, 16);
    const size_t in_bytes = round_up(o_vals + 4 * (size_t)nnz, 16);
    if ((rc = grow_host(&S->hin, &S->hin_cap, in_bytes, cudaHostAllocDefault, S->s))) return rc;
    // every call ends with a synchronisation, so the staging is free to refill
    in.fill(in.ctx, (int64_t*)S->hin, (int32_t*)(S->hin + o_cols), (uint32_t*)(S->hin + o_vals));
    // device arena
    const size_t o_piv = round_up(in_bytes, 256);
    const size_t o_pext = round_up(o_piv + 4 * (size_t)std::max(ncl, 1), 256);
    const size_t o_work = round_up(o_pext + 8 * (size_t)std::max(ncl, 1), 256);
    const size_t o_cnt = round_up(o_work + 4 * (size_t)nr, 256);  // n_work, err
    const size_t o_D = round_up(o_cnt + 64, 256);
    const size_t o_lead = round_up(o_D + 4 * (size_t)std::max(n_work, 1) * ld, 256);
    const size_t o_poc = round_up(o_lead + 4 * (size_t)std::max(n_work, 1), 256);
    const size_t d_bytes = round_up(o_poc + 4 * (size_t)ncr, 256);
    if ((rc = grow_device(*S, d_bytes))) return rc;
    uint8_t* d = (uint8_t*)S->dmem;
    const int64_t* d_ptr = (const int64_t*)d;
    const int32_t* d_cols = (const int32_t*)(d + o_cols);
    const uint32_t* d_vals = (const uint32_t*)(d + o_vals);
    int32_t* d_piv = (int32_t*)(d + o_piv);
    int2* d_pext = (int2*)(d + o_pext);
    int32_t* d_work = (int32_t*)(d + o_work);
    int32_t* d_nwork = (int32_t*)(d + o_cnt);
    uint32_t* d_err = (uint32_t*)(d + o_cnt + 16);
    uint32_t* d_D = (uint32_t*)(d + o_D);
    int32_t* d_lead = (int32_t*)(d + o_lead);
    int32_t* d_poc = (int32_t*)(d + o_poc);
    // mapped output: counts | offs | cols | vals
    const size_t cap = (size_t)std::max(n_work, 0) * ncr;
    const size_t h_offs = 64;
    const size_t h_cols = round_up(h_offs + 8 * (size_t)(std::max(n_work, 0) + 1), 16);
    const size_t h_vals = round_up(h_cols + 4 * std::max<size_t>(cap, 1), 16);
    const size_t out_bytes = round_up(h_vals + 4 * std::max<size_t>(cap, 1), 16);
    if ((rc = grow_host(&S->hout, &S->hout_cap, out_bytes, cudaHostAllocMapped, S->s))) return rc;
    uint8_t* hd = nullptr;
    if (cudaHostGetDevicePointer((void**)&hd, S->hout, 0) != cudaSuccess) {
        set_error("mapped output pointer unavailable");
        return GBGPU_ECUDA;
    }
    int64_t* h_counts = (int64_t*)S->hout;
    h_counts[0] = 0;
    h_counts[1] = 0;

    cudaStream_t s = S->s;
    long long launches = 0;
    if (cudaMemcpyAsync(d, S->hin, in_bytes, cudaMemcpyHostToDevice, s) != cudaSuccess) {
        set_error("small-matrix input copy failed");
        return GBGPU_ECUDA;
    }
    const int prep_bytes = 4 * std::max(ncl, 1);
    if (ensure_smem_limit((const void*)k_small_prep, prep_bytes) != cudaSuccess) {
        set_error("prep kernel shared memory");
        return GBGPU_ECUDA;
    }
    k_small_prep<<<1, kPrepThreads, prep_bytes, s>>>(nr, ncl, nc, (uint32_t)in.p, d_ptr, d_cols,
                                                     d_vals, d_piv, d_pext, d_work, d_nwork,
                                                     d_err);
    ++launches;
    if (n_work > 0) {
        int32_t stride = 0;
        const int wpc = rows_warps(nc, S->dev, &stride);
        const int bytes = wpc * stride * 4;
        const int grid = std::max(1, std::min((n_work + wpc - 1) / wpc, S->dev.sms * 4));
        const int tb = tiny_rref_bytes(n_work, ncr, S->dev.smem_optin);
        auto run = [&](auto f) -> int {
            using Fd = decltype(f);
            if (ensure_smem_limit((const void*)k_reduce_rows_warp<Fd>, bytes) != cudaSuccess) {
                set_error("row kernel shared memory");
                return GBGPU_ECUDA;
            }
            k_reduce_rows_warp<Fd><<<grid, wpc * 32, bytes, s>>>(
                n_work, d_work, d_ptr, d_cols, d_vals, d_pext, ncl, nc, stride, d_D, ld, d_lead,
                d_err, f);
            ++launches;
            cudaError_t e = launch_tiny_rref(n_work, ncr, d_D, ld, d_lead, d_err, ncl,
                                             (int64_t*)(hd + h_offs), (int32_t*)(hd + h_cols),
                                             (int32_t*)(hd + h_vals), d_poc, (int64_t*)hd, tb,
                                             s, f);
            ++launches;
            if (e != cudaSuccess) {
                set_error(std::string("small-matrix launch: ") + cudaGetErrorString(e));
                return GBGPU_ECUDA;
            }
            return GBGPU_OK;
        };
        rc = (uint32_t)in.p < 65536u ? run(FieldSmall::make((uint32_t)in.p))
                                     : run(FieldMont::make((uint32_t)in.p));
        if (rc) return rc;
    } else {
        ((int64_t*)(S->hout + h_offs))[0] = 0;
    }
    count_launch(launches);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(S->herr, d_err, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_error(std::string("small-matrix run: ") + cudaGetErrorString(e));
        return GBGPU_ECUDA;
    }
    if (*S->herr) {
        std::string msg;
        rc = err_to_status(*S->herr, &msg);
        set_error(msg);
        return rc;
    }
    ans->np = n_work > 0 ? (int32_t)h_counts[0] : 0;
    ans->nnz = n_work > 0 ? h_counts[1] : 0;
    ans->offs = (const int64_t*)(S->hout + h_offs);
    ans->cols = (const int32_t*)(S->hout + h_cols);
    ans->vals = (const int32_t*)(S->hout + h_vals);
    return GBGPU_OK;
}


int small_batch_bytes(int32_t nr, int32_t ncl, int32_t ncr, int device) {
    if (nr <= 0 || ncl < 0 || ncr <= 0 || nr < ncl || ncl > kSmallMaxLeft) return 0;
    DeviceGuard guard;
    DeviceInfo dev{};
    if (device_init(device, &dev)) return 0;
    const int64_t stride = rup(ncl + ncr, 4);
    const int64_t rows = 4 * 4 * stride;  // at least four row warps
    const int32_t n_work = nr - ncl;
    const int64_t tiny = n_work > 0 ? tiny_rref_bytes(n_work, ncr, dev.smem_optin) : 1;
    if (tiny <= 0) return 0;
    const int64_t need = std::max<int64_t>({4 * (int64_t)std::max(ncl, 1), rows, tiny});
    return need + 2048 <= dev.smem_optin ? (int)need : 0;
}

int small_batch(int32_t n, const gbgpu_csr* const* ms, int device, gbgpu_rows* outs,
                int32_t* status) {
    if (n <= 0) return GBGPU_OK;
    DeviceGuard guard;
    DeviceInfo dev{};
    int rc = device_init(device, &dev);
    if (rc) return rc;
    std::vector<BatchItem> items((size_t)n);
    int64_t in_bytes = 0, scr_bytes = 0, out_bytes = 0;
    int smem = 0;
    for (int32_t i = 0; i < n; ++i) {
        const gbgpu_csr* m = ms[i];
        BatchItem& it = items[i];
        it.p = m->p;
        it.nr = m->nr;
        it.ncl = m->ncl;
        it.ncr = m->ncr;
        const int64_t nnz = m->row_ptr[m->nr];
        it.in_off = in_bytes;
        it.cols_off = rup(it.in_off + 8 * (int64_t)(m->nr + 1), 16);
        it.vals_off = rup(it.cols_off + 4 * nnz, 16);
        in_bytes = rup(it.vals_off + 4 * nnz, 256);
        it.scr_off = scr_bytes;
        scr_bytes += scr_layout(m->nr, m->ncl, m->ncr).bytes;
        it.out_off = out_bytes;
        out_bytes += out_layout(m->nr, m->ncl, m->ncr).bytes;
        it.fs = FieldSmall::make((uint32_t)std::max(m->p, 2));
        it.fm = FieldMont::make((uint32_t)(m->p | 1));  // used only for odd p >= 2^16
        smem = std::max(smem, small_batch_bytes(m->nr, m->ncl, m->ncr, device));
    }
    smem = std::min(dev.smem_optin - 2048, std::max(smem, 4 * 4 * 1024));
    uint8_t *h_in = nullptr, *h_out = nullptr, *d_out = nullptr, *d_in = nullptr;
    BatchItem* d_items = nullptr;
    int32_t* d_queue = nullptr;
    cudaStream_t s = nullptr;
    auto cleanup = [&]() {
        if (s) cudaStreamSynchronize(s);
        if (d_in) cudaFree(d_in);
        if (h_in) cudaFreeHost(h_in);
        if (h_out) cudaFreeHost(h_out);
        if (s) cudaStreamDestroy(s);
    };
    // device: input | scratch | items | queue
    const int64_t o_scr = rup(in_bytes, 256), o_items = rup(o_scr + scr_bytes, 256);
    const int64_t o_queue = rup(o_items + (int64_t)sizeof(BatchItem) * n, 256);
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaHostAlloc((void**)&h_in, (size_t)std::max<int64_t>(in_bytes, 16), 0) != cudaSuccess ||
        cudaHostAlloc((void**)&h_out, (size_t)std::max<int64_t>(out_bytes, 256),
                      cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer((void**)&d_out, h_out, 0) != cudaSuccess ||
        cudaMalloc((void**)&d_in, (size_t)(o_queue + 256)) != cudaSuccess) {
        cleanup();
        set_error("small-matrix batch: allocation failed");
        return GBGPU_ENOMEM;
    }
    for (int32_t i = 0; i < n; ++i) {
        const gbgpu_csr* m = ms[i];
        fill_from_csr_vals((void*)m, (int64_t*)(h_in + items[i].in_off),
                           (int32_t*)(h_in + items[i].cols_off),
                           (uint32_t*)(h_in + items[i].vals_off));
    }
    d_items = (BatchItem*)(d_in + o_items);
    d_queue = (int32_t*)(d_in + o_queue);
    cudaError_t e = cudaMemcpyAsync(d_in, h_in, (size_t)in_bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_items, items.data(), sizeof(BatchItem) * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_queue, 0, sizeof(int32_t), s);
    if (e == cudaSuccess) e = ensure_smem_limit((const void*)k_batch_small, smem);
    if (e == cudaSuccess) {
        const int per_sm = std::max(1, std::min(2, (dev.smem_optin - 1024) / (smem + 1024)));
        const int grid = std::max(1, std::min(n, dev.sms * per_sm));
        k_batch_small<<<grid, kPrepThreads, smem, s>>>(n, d_items, d_in, d_in + o_scr, d_out,
                                                       d_queue, smem);
        count_launch(1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_error(std::string("small-matrix batch: ") + cudaGetErrorString(e));
        for (int32_t i = 0; i < n; ++i) status[i] = GBGPU_ECUDA;
        cleanup();
        return GBGPU_OK;
    }
    for (int32_t i = 0; i < n; ++i) {
        const uint8_t* ob = h_out + items[i].out_off;
        const OutLayout O = out_layout(items[i].nr, items[i].ncl, items[i].ncr);
        const int64_t* counts = (const int64_t*)ob;
        if (counts[2]) {
            std::string msg;
            status[i] = err_to_status((uint32_t)counts[2], &msg);
            continue;
        }
        gbgpu_rows& r = outs[i];
        r.np = (int32_t)counts[0];
        r.nnz = counts[1];
        r.row_ptr = (int64_t*)malloc(sizeof(int64_t) * (size_t)(r.np + 1));
        r.cols = (int32_t*)malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(r.nnz, 1));
        r.vals = (int32_t*)malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(r.nnz, 1));
        if (!r.row_ptr || !r.cols || !r.vals) {
            status[i] = GBGPU_ENOMEM;
            continue;
        }
        memcpy(r.row_ptr, ob + O.offs, sizeof(int64_t) * (size_t)(r.np + 1));
        memcpy(r.cols, ob + O.cols, sizeof(int32_t) * (size_t)r.nnz);
        memcpy(r.vals, ob + O.vals, sizeof(int32_t) * (size_t)r.nnz);
        status[i] = GBGPU_OK;
    }
    cleanup();
    return GBGPU_OK;
}

}  // namespace gbgpu
