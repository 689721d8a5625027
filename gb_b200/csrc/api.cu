// api.cu -- host orchestration and the C ABI declared in include/gbgpu.h.
//
// A plan owns the device copy of one matrix and every work buffer of one
// reduction (stream-ordered allocations from the device's default memory
// pool, which keeps freed blocks cached between F4 rounds).  Runs are
// enqueued on the plan's stream; the echelon's claiming rounds read one
// counter back per round, everything else stays on the device until the
// answer is copied out.
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <cub/iterator/counting_input_iterator.cuh>

#include <algorithm>
#include <atomic>
#include <map>
#include <mutex>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <sys/time.h>
#include <vector>

#include "../../include/gbgpu.h"
#include "blocked.h"
#include "common.cuh"
#include "internal.h"
#include "kernels.h"
#include "small.h"
#include "tc_gemm.h"

namespace gbgpu {

static thread_local std::string g_last_error;
static std::atomic<long long> g_launches{0};

void set_error(const std::string& s) { g_last_error = s; }
void count_launch(long long n) { g_launches += n; }

cudaError_t ensure_smem_limit(const void* kernel, int bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> limits;  // (kernel, device) -> bytes
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    int& cur = limits[{kernel, dev}];
    if (bytes <= cur) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

#define GB_CUDA(call)                                                              \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));         \
            return GBGPU_ECUDA;                                                    \
        }                                                                          \
    } while (0)

#define GB_LAUNCH(...)                                                             \
    do {                                                                           \
        __VA_ARGS__;                                                               \
        cudaError_t e_ = cudaGetLastError();                                       \
        if (debug_trace()) fprintf(stderr, "gbgpu launch %s: %s\n", #__VA_ARGS__,  \
                                   cudaGetErrorString(e_));                        \
        if (e_ != cudaSuccess) {                                                   \
            set_error(std::string("launch: ") + cudaGetErrorString(e_));           \
            return GBGPU_ECUDA;                                                    \
        }                                                                          \
        ++launches;                                                                \
    } while (0)

#define GB_CALL(expr)                                                              \
    do {                                                                           \
        cudaError_t e_ = (expr);                                                   \
        if (debug_trace()) fprintf(stderr, "gbgpu launch %s: %s\n", #expr,          \
                                   cudaGetErrorString(e_));                        \
        if (e_ != cudaSuccess) {                                                   \
            set_error(std::string("launch: ") + cudaGetErrorString(e_));           \
            return GBGPU_ECUDA;                                                    \
        }                                                                          \
        ++launches;                                                                \
    } while (0)

// per-launch executed-K-step counters of a profiled run
constexpr int kGemmProfileSlots = 4096;

static bool debug_trace() {
    static const bool on = getenv("GBGPU_DEBUG") != nullptr;
    return on;
}

static int grid_for(int64_t n, int threads, int cap = 148 * 16) {
    int64_t g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

int device_init(int device, DeviceInfo* info) {
    // properties are read once per device (cudaGetDeviceProperties is slow)
    static std::mutex mu;
    static DeviceInfo cache[64];
    static bool known[64] = {};
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
        set_error("no CUDA device");
        return GBGPU_ENODEV;
    }
    if (device < 0 || device >= n || device >= 64) {
        set_error("device ordinal out of range");
        return GBGPU_ENODEV;
    }
    GB_CUDA(cudaSetDevice(device));
    std::lock_guard<std::mutex> lock(mu);
    if (!known[device]) {
        cudaDeviceProp prop;
        GB_CUDA(cudaGetDeviceProperties(&prop, device));
        if (prop.major != 10) {
            set_error("libgbgpu is built for sm_100 (B200) only");
            return GBGPU_ENODEV;
        }
        cache[device].sms = prop.multiProcessorCount;
        cache[device].smem_optin = (int)prop.sharedMemPerBlockOptin;
        // keep freed blocks in the stream-ordered pool between reductions
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        known[device] = true;
    }
    *info = cache[device];
    return GBGPU_OK;
}

// ---------------------------------------------------------------------------
struct Plan {
    int device = 0;
    DeviceInfo dev{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int mode = 0;  // 0: linear_algebra, 1: interreduction
    int form = GBGPU_FORM_PLAIN;
    int requested_form = GBGPU_FORM_AUTO;
    int profile = 0;
    unsigned long long* gemm_steps = nullptr;
    bool blocked = false;  // blocked (dense block) algorithm instead of sparse rows
    int check = 1;
    int32_t p = 0, nr = 0, ncl = 0, ncr = 0, nc = 0, n_work = 0;
    int64_t nnz = 0;
    std::vector<void*> bufs;

    // inputs
    int64_t* row_ptr = nullptr;
    int32_t* cols = nullptr;
    uint32_t* vals = nullptr;
    // classification
    int32_t* piv_row = nullptr;
    uint8_t* flag = nullptr;
    int32_t* work = nullptr;
    int32_t* n_sel = nullptr;
    uint32_t* err = nullptr;
    int32_t* counters = nullptr;  // [0] queue, [1] n_cand, [2] n_losers, [3] n_next, [4] queue2
    int64_t* work_count = nullptr;
    // reduced rows
    int64_t ld = 0;
    uint32_t* D = nullptr;
    uint32_t* R = nullptr;
    int32_t* lead = nullptr;
    uint32_t* gacc = nullptr;
    int grid_sparse = 0;
    bool smem_sparse = true, smem_dense = true;
    // team-per-row known-pivot reduction (plain.cu k_reduce_team)
    int team_bytes = 0, grid_team = 0;
    longlong2* pext = nullptr;
    // echelon
    int32_t* piv_of_col = nullptr;
    int32_t* claim = nullptr;
    int32_t* cand = nullptr;
    int32_t* losers = nullptr;
    // compaction
    int32_t* pflag = nullptr;
    int32_t* ppos = nullptr;
    int32_t* pivcol = nullptr;
    int64_t* counts = nullptr;
    int64_t* offs = nullptr;
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    int32_t* out_cols = nullptr;
    int32_t* out_vals = nullptr;
    uint8_t* wire = nullptr;  // narrow values in transit (val_bytes 1 or 2)
    size_t wire_cap = 0;
    int64_t out_cap = 0;
    // answer
    int32_t np = 0;
    int64_t onnz = 0;
    uint32_t errbits = 0;
    // small matrices: one-CTA echelon + compaction, no host round trip in a
    // run; its checks, counts and timings are read when the answer is taken
    bool tiny = false;
    int tiny_bytes = 0;
    int64_t* tiny_counts = nullptr;  // [2]: rows, entries of the answer
    bool pending = false;            // a tiny run whose results are not read yet
    // answer streamed to host arrays during the run (gbgpu_plan_run_into_v)
    StreamOut* stream_req = nullptr;
    bool streamed = false;
    // the answer's columns were rewritten by plan_map_columns: they are the
    // caller's table indices and no longer count from ncl
    bool mapped = false;
    cudaStream_t s_out = nullptr;
    gbgpu_stats stats{};
    cudaEvent_t ev[8] = {};
    long long launches = 0;

    template <class T>
    int alloc(T** p, size_t count) {
        void* q = nullptr;
        const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
        cudaError_t e = cudaMallocAsync(&q, bytes, stream);
        if (e != cudaSuccess) {
            set_error(std::string("device allocation: ") + cudaGetErrorString(e));
            return GBGPU_ENOMEM;
        }
        bufs.push_back(q);
        *p = (T*)q;
        return GBGPU_OK;
    }
    ~Plan() {
        if (s_out) {
            cudaStreamSynchronize(s_out);
            cudaStreamDestroy(s_out);
        }
        for (void* q : bufs) cudaFreeAsync(q, stream);
        if (stream) cudaStreamSynchronize(stream);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }
};

int err_to_status(uint32_t bits, std::string* msg) {
    if (!bits) return GBGPU_OK;
    std::string s = "input breaks the mat_t contract:";
    if (bits & kErrEmptyRow) s += " empty row;";
    if (bits & kErrLeadRange) s += " lead outside the left block;";
    if (bits & kErrColRange) s += " column out of range or repeated lead;";
    if (bits & kErrCoefRange) s += " coefficient outside [1,p);";
    if (bits & kErrNotMonic) s += " row not monic;";
    if (bits & kErrMissingPivot) s += " left column without known pivot;";
    if (bits & kErrDupLead) s += " repeated lead in interreduction input;";
    *msg = s;
    return GBGPU_EINVAL;
}

static int plan_setup(Plan* P, const gbgpu_options* opt) {
    gbgpu_options o{};
    if (opt) o = *opt;
    P->device = o.device;
    int rc = device_init(P->device, &P->dev);
    if (rc) return rc;
    P->requested_form = o.form;
    P->profile = o.profile;
    P->check = 1;  // the contract check is cheap and guards every later index
    if (o.stream) {
        P->stream = (cudaStream_t)o.stream;
    } else {
        GB_CUDA(cudaStreamCreateWithFlags(&P->stream, cudaStreamNonBlocking));
        P->own_stream = true;
    }
    for (auto& e : P->ev) GB_CUDA(cudaEventCreate(&e));
    return GBGPU_OK;
}

static int plan_alloc(Plan* P) {
    int rc;
#define A(ptr, n) \
    if ((rc = P->alloc(&P->ptr, (size_t)(n)))) return rc
    A(row_ptr, P->nr + 1);
    // 16 entries of padding: the team kernel stages pivot rows in whole
    // 16-byte groups, reading up to 3 entries past a row's end
    A(cols, P->nnz + 16);
    A(vals, P->nnz + 16);
    A(piv_row, P->nc);
    A(flag, P->nr);
    A(work, P->nr);
    A(n_sel, 1);
    A(err, 1);
    A(counters, 8);
    A(work_count, 2);
    A(gemm_steps, kGemmProfileSlots);
    const int32_t width = P->mode == 0 ? P->ncr : P->nc;
    P->ld = ((int64_t)width + 3) & ~(int64_t)3;
    // algorithm: the blocked form runs its dense steps as exact modular GEMMs
    // (int8 tensor cores for odd p); AUTO picks it for matrices large enough
    // to feed them, the sparse-row form for the small ones
    const bool odd = (P->p & 1) && P->p >= 3;
    if (P->mode == 1) {
        P->blocked = false;
        P->form = GBGPU_FORM_PLAIN;
    } else if (P->requested_form == GBGPU_FORM_PLAIN) {
        P->blocked = false;
        P->form = GBGPU_FORM_PLAIN;
    } else if (P->requested_form == GBGPU_FORM_TENSOR) {
        P->blocked = true;
        P->form = odd ? GBGPU_FORM_TENSOR : GBGPU_FORM_PLAIN;
    } else if (P->requested_form == GBGPU_FORM_BLOCKED_PLAIN) {
        P->blocked = true;
        P->form = GBGPU_FORM_PLAIN;
    } else {
        P->blocked = odd && P->n_work >= 128 && P->ncr >= 128;
        P->form = P->blocked ? GBGPU_FORM_TENSOR : GBGPU_FORM_PLAIN;
    }
    if (!P->blocked) {
        A(D, (size_t)P->n_work * P->ld);
        A(lead, P->n_work);
        if (P->mode == 0) {
            A(R, (size_t)P->n_work * P->ld);
            A(claim, P->ncr);
            A(cand, P->n_work);
            A(losers, P->n_work);
        }
    }
    if (P->mode == 0 && !P->blocked && P->n_work > 0 && P->ncr > 0)
        P->tiny_bytes = tiny_rref_bytes(P->n_work, P->ncr, P->dev.smem_optin);
    P->tiny = P->tiny_bytes > 0;
    if (P->tiny) {
        // the answer has at most n_work rows of ncr entries
        const size_t cap = (size_t)P->n_work * P->ncr;
        A(tiny_counts, 2);
        A(out_cols, cap);
        A(out_vals, cap);
        P->out_cap = (int64_t)cap;
    }
    A(piv_of_col, width);
    A(pflag, width);
    A(ppos, width);
    A(pivcol, width);
    A(counts, width + 1);
    A(offs, width + 1);
    // shared memory budget for the dense accumulators
    const int64_t smem_cap = std::min<int64_t>(P->dev.smem_optin - 1024, 200 * 1024);
    P->smem_sparse = (int64_t)P->nc * 4 <= smem_cap;
    P->smem_dense = (int64_t)P->ncr * 4 <= smem_cap;
    P->team_bytes = team_smem_bytes(P->nc, P->dev.smem_optin);
    if (P->team_bytes > 0 && !P->blocked) {
        A(pext, P->mode == 0 ? std::max(P->ncl, 1) : std::max(P->nc, 1));
        const int per_sm = std::max(1, std::min(8, (P->dev.smem_optin - 1024) / (P->team_bytes + 3072)));
        P->grid_team = std::max(1, std::min<int>(P->n_work, P->dev.sms * per_sm));
    }
    P->grid_sparse = std::max(1, std::min<int>(P->n_work, P->dev.sms * (P->smem_sparse ? 1 : 2)));
    if (P->smem_sparse) {
        // two CTAs per SM when two accumulators fit
        if ((int64_t)P->nc * 4 * 2 <= P->dev.smem_optin - 4096)
            P->grid_sparse = std::max(1, std::min<int>(P->n_work, P->dev.sms * 2));
    } else if (!P->blocked) {
        A(gacc, (size_t)P->grid_sparse * (((size_t)P->nc + 31) & ~(size_t)31));
    }
    // cub temporaries: selection over rows, scans over columns
    size_t b1 = 0, b2 = 0, b3 = 0;
    cub::CountingInputIterator<int32_t> it(0);
    cub::DeviceSelect::Flagged(nullptr, b1, it, P->flag, P->work, P->n_sel, P->nr, P->stream);
    cub::DeviceScan::ExclusiveSum(nullptr, b2, P->pflag, P->ppos, width, P->stream);
    cub::DeviceScan::ExclusiveSum(nullptr, b3, P->counts, P->offs, width + 1, P->stream);
    P->cub_bytes = std::max(b1, std::max(b2, b3));
    A(cub_tmp, P->cub_bytes);
#undef A
    return GBGPU_OK;
}

template <class F>
static int run_form(Plan* P, const F& f) {
    cudaStream_t s = P->stream;
    long long& launches = P->launches;
    const int T = 256;
    const int32_t width = P->mode == 0 ? P->ncr : P->nc;

    {
        cudaError_t stale = cudaGetLastError();
        if (stale != cudaSuccess && debug_trace())
            fprintf(stderr, "gbgpu: stale error before run: %s\n", cudaGetErrorString(stale));
    }
    GB_CUDA(cudaEventRecord(P->ev[0], s));
    GB_CUDA(cudaMemsetAsync(P->err, 0, sizeof(uint32_t), s));
    GB_CUDA(cudaMemsetAsync(P->counters, 0, 8 * sizeof(int32_t), s));
    GB_CUDA(cudaMemsetAsync(P->work_count, 0, 2 * sizeof(int64_t), s));
    const int32_t lead_bound = P->mode == 0 ? P->ncl : P->nc;
    GB_LAUNCH(k_check_rows<<<grid_for((int64_t)P->nr * 32, T), T, 0, s>>>(
        P->nr, P->row_ptr, P->cols, P->vals, lead_bound, P->nc, (uint32_t)P->p, P->err));
    GB_LAUNCH(k_fill_i32<<<grid_for(P->nc, T), T, 0, s>>>(P->piv_row, P->nc, INT_MAX));
    GB_LAUNCH(k_classify<<<grid_for(P->nr, T), T, 0, s>>>(P->nr, P->row_ptr, P->cols, P->nc,
                                                          P->piv_row));
    GB_LAUNCH(k_mark_lower<<<grid_for(P->nr, T), T, 0, s>>>(P->nr, P->row_ptr, P->cols, P->nc,
                                                            P->piv_row, P->flag, P->err,
                                                            P->mode == 1));
    if (P->mode == 0)
        GB_LAUNCH(k_check_pivots<<<grid_for(P->ncl, T), T, 0, s>>>(P->ncl, P->piv_row, P->err));
    GB_CUDA(cudaEventRecord(P->ev[6], s));
    if (P->tiny) {
        // the checks' verdict is read with the answer; the kernels below skip
        // their work when it flags the input
        P->errbits = 0;
    } else {
        GB_CUDA(cudaMemcpyAsync(&P->errbits, P->err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        GB_CUDA(cudaStreamSynchronize(s));
    }
    GB_CUDA(cudaEventRecord(P->ev[7], s));
    if (P->errbits) {
        std::string msg;
        int rc = err_to_status(P->errbits, &msg);
        set_error(msg);
        return rc;
    }
    // rows to reduce: the C|D rows in row order (all rows for interreduction)
    if (P->mode == 0) {
        cub::CountingInputIterator<int32_t> it(0);
        size_t bytes = P->cub_bytes;
        GB_CUDA(cub::DeviceSelect::Flagged(P->cub_tmp, bytes, it, P->flag, P->work, P->n_sel,
                                           P->nr, s));
        ++launches;
    } else {
        // every row, in row order; row i of the output buffer is input row i,
        // so the pivot table of the compaction is the lead table itself
        GB_LAUNCH(k_iota<<<grid_for(P->nr, T), T, 0, s>>>(P->work, P->nr));
        GB_LAUNCH(k_pivtab<<<grid_for(P->nc, T), T, 0, s>>>(P->nc, P->piv_row, P->piv_of_col));
    }
    GB_CUDA(cudaEventRecord(P->ev[1], s));

    const uint32_t* final_rows = P->D;
    int64_t rows_ld = P->ld;
    BlockedOutput bo{};
    if (P->blocked) {
        BlockedInput bi{};
        bi.p = (uint32_t)P->p;
        bi.ncl = P->ncl;
        bi.ncr = P->ncr;
        bi.n_work = P->n_work;
        bi.work = P->work;
        bi.row_ptr = P->row_ptr;
        bi.cols = P->cols;
        bi.vals = P->vals;
        bi.piv_row = P->piv_row;
        bi.stream = s;
        bi.form = P->form;
        bi.err = P->counters + 6;
        bo.piv_of_col = P->piv_of_col;
        bo.ms_event_schur = P->ev[2];
        bo.ms_event_echelon = P->ev[3];
        bo.stream_out = P->stream_req;
        const int rc = blocked_reduce(bi, &bo, &launches);
        if (rc) {
            blocked_release(&bo, s);
            return rc;
        }
        final_rows = bo.rows;
        rows_ld = bo.ld;
        P->np = (int32_t)bo.rank;
        P->stats.dense_rows = bo.dense_rows;
        P->stats.echelon_rounds = bo.echelon_rounds;
        GB_CUDA(cudaEventRecord(P->ev[4], s));
        P->streamed = bo.stream_out != nullptr;
        if (P->streamed) {
            // the answer went to host memory block by block
            P->onnz = bo.stream_out->nnz;
        } else if (P->np > 0) {
            GB_LAUNCH(k_pivot_flags<<<grid_for(P->ncr, T), T, 0, s>>>(P->ncr, P->piv_of_col, 1,
                                                                       P->pflag));
            size_t bytes = P->cub_bytes;
            GB_CUDA(cub::DeviceScan::ExclusiveSum(P->cub_tmp, bytes, P->pflag, P->ppos, P->ncr, s));
            ++launches;
            GB_LAUNCH(k_pivot_list<<<grid_for(P->ncr, T), T, 0, s>>>(P->ncr, P->pflag, P->ppos, 1,
                                                                      P->pivcol));
        }
    } else {

    // ---- known-pivot reduction ----------------------------------------
    SparseReduceArgs sa{};
    sa.row_ptr = P->row_ptr;
    sa.cols = P->cols;
    sa.vals = P->vals;
    sa.piv_row = P->piv_row;
    sa.piv_limit = P->mode == 0 ? P->ncl : P->nc;
    sa.skip_lead = P->mode == 1;
    sa.work = P->work;
    sa.n_work = P->n_work;
    sa.nc = P->nc;
    sa.emit_from = P->mode == 0 ? P->ncl : 0;
    sa.emit_width = width;
    sa.out_ld = P->ld;
    sa.acc_stride = ((int64_t)P->nc + 31) & ~(int64_t)31;
    sa.out = P->D;
    sa.out_lead = P->lead;
    sa.gacc = P->gacc;
    sa.queue = P->counters + 0;
    sa.work_count = P->work_count + 0;
    sa.err = P->err;
    if (P->n_work > 0) {
        if (P->pext) {
            GB_LAUNCH(k_pivot_extents<<<grid_for(sa.piv_limit, T), T, 0, s>>>(
                sa.piv_limit, P->piv_row, P->row_ptr, P->pext));
            GB_CALL(launch_reduce_team(sa, P->pext, f, P->grid_team, P->team_bytes, s));
        } else {
            GB_CALL(launch_reduce_sparse(sa, f, P->grid_sparse, P->smem_sparse, P->nc * 4, s));
        }
    }
    GB_CUDA(cudaEventRecord(P->ev[2], s));

    if (P->tiny) {
        // ---- small right block: echelon form and compaction in one CTA ------
        GB_CALL(launch_tiny_rref(P->n_work, P->ncr, P->D, P->ld, P->lead, P->err, P->ncl,
                                 P->offs, P->out_cols, P->out_vals, P->piv_of_col,
                                 P->tiny_counts, P->tiny_bytes, s, f));
        P->stats.echelon_rounds = 0;
        GB_CUDA(cudaEventRecord(P->ev[3], s));
        GB_CUDA(cudaEventRecord(P->ev[4], s));
        GB_CUDA(cudaEventRecord(P->ev[5], s));
        P->pending = true;
        return GBGPU_OK;
    } else if (P->mode == 0) {
        // ---- echelon rounds on the dense right block ------------------------
        GB_LAUNCH(k_fill_i32<<<grid_for(P->ncr, T), T, 0, s>>>(P->piv_of_col, P->ncr, -1));
        GB_LAUNCH(k_collect_nonzero<<<grid_for(P->n_work, T), T, 0, s>>>(
            P->n_work, P->lead, P->cand, P->counters + 1));
        int32_t n_cand = 0;
        GB_CUDA(cudaMemcpyAsync(&n_cand, P->counters + 1, 4, cudaMemcpyDeviceToHost, s));
        GB_CUDA(cudaStreamSynchronize(s));
        P->stats.dense_rows = n_cand;
        const int dense_grid = std::max(1, P->dev.sms * (P->smem_dense && P->ncr * 8 <= P->dev.smem_optin - 4096 ? 2 : 1));
        const int dense_bytes = P->smem_dense ? P->ncr * 4 : 0;
        int rounds = 0;
        int32_t* cand = P->cand;
        int32_t* nxt = P->losers;
        while (n_cand > 0) {
            ++rounds;
            GB_LAUNCH(k_fill_i32<<<grid_for(P->ncr, T), T, 0, s>>>(P->claim, P->ncr, INT_MAX));
            GB_LAUNCH(k_claim<<<grid_for(n_cand, T), T, 0, s>>>(cand, P->counters + 1, P->lead,
                                                                P->claim));
            GB_CUDA(cudaMemsetAsync(P->counters + 2, 0, 3 * sizeof(int32_t), s));
            GB_CALL(launch_promote(grid_for((int64_t)n_cand * 32, T), T, s, cand, P->counters + 1,
                                   P->lead, P->claim, P->piv_of_col, P->D, P->ld, P->ncr, nxt,
                                   P->counters + 2, f));
            int32_t n_lost = 0;
            GB_CUDA(cudaMemcpyAsync(&n_lost, P->counters + 2, 4, cudaMemcpyDeviceToHost, s));
            GB_CUDA(cudaStreamSynchronize(s));
            if (n_lost == 0) break;
            DenseReduceArgs da{};
            da.src = P->D;
            da.dst = P->D;
            da.ld = P->ld;
            da.ncr = P->ncr;
            da.mode = kUntilFree;
            da.piv_of_col = P->piv_of_col;
            da.work = nxt;
            da.n_work = P->counters + 2;
            da.lead = P->lead;
            da.next = cand;
            da.n_next = P->counters + 3;
            da.queue = P->counters + 4;
            da.work_count = P->work_count + 1;
            const int g = std::min(dense_grid, n_lost);
            GB_CALL(launch_reduce_dense(da, f, g, P->smem_dense, dense_bytes, s));
            // survivors become the next candidates
            GB_CUDA(cudaMemcpyAsync(P->counters + 1, P->counters + 3, 4, cudaMemcpyDeviceToDevice, s));
            GB_CUDA(cudaMemcpyAsync(&n_cand, P->counters + 3, 4, cudaMemcpyDeviceToHost, s));
            GB_CUDA(cudaStreamSynchronize(s));
        }
        P->stats.echelon_rounds = rounds;
        GB_CUDA(cudaEventRecord(P->ev[3], s));

        // ---- back substitution: reduced row echelon form --------------------
        GB_LAUNCH(k_pivot_flags<<<grid_for(P->ncr, T), T, 0, s>>>(P->ncr, P->piv_of_col, 1,
                                                                   P->pflag));
        size_t bytes = P->cub_bytes;
        GB_CUDA(cub::DeviceScan::ExclusiveSum(P->cub_tmp, bytes, P->pflag, P->ppos, P->ncr, s));
        ++launches;
        GB_LAUNCH(k_pivot_list<<<grid_for(P->ncr, T), T, 0, s>>>(P->ncr, P->pflag, P->ppos, 1,
                                                                  P->pivcol));
        int32_t last_pos = 0, last_flag = 0;
        if (P->ncr > 0) {
            GB_CUDA(cudaMemcpyAsync(&last_pos, P->ppos + P->ncr - 1, 4, cudaMemcpyDeviceToHost, s));
            GB_CUDA(cudaMemcpyAsync(&last_flag, P->pflag + P->ncr - 1, 4, cudaMemcpyDeviceToHost, s));
        }
        GB_CUDA(cudaStreamSynchronize(s));
        P->np = last_pos + last_flag;
        if (P->np > 0) {
            // work list: the pivot rows (row index of each pivot column)
            GB_LAUNCH(k_gather_rows<<<grid_for(P->np, T), T, 0, s>>>(P->np, P->pivcol,
                                                                     P->piv_of_col, P->cand,
                                                                     P->counters + 1));
            GB_CUDA(cudaMemsetAsync(P->counters + 4, 0, sizeof(int32_t), s));
            DenseReduceArgs da{};
            da.src = P->D;
            da.dst = P->R;
            da.ld = P->ld;
            da.ncr = P->ncr;
            da.mode = kFull;
            da.piv_of_col = P->piv_of_col;
            da.work = P->cand;
            da.n_work = P->counters + 1;
            da.lead = P->lead;
            da.queue = P->counters + 4;
            da.work_count = P->work_count + 1;
            const int g = std::min(dense_grid, (int)P->np);
            GB_CALL(launch_reduce_dense(da, f, g, P->smem_dense, dense_bytes, s));
        }
        final_rows = P->R;
        GB_CUDA(cudaEventRecord(P->ev[4], s));
    } else {
        GB_LAUNCH(k_pivot_flags<<<grid_for(P->nc, T), T, 0, s>>>(P->nc, P->piv_of_col, 0, P->pflag));
        size_t bytes = P->cub_bytes;
        GB_CUDA(cub::DeviceScan::ExclusiveSum(P->cub_tmp, bytes, P->pflag, P->ppos, P->nc, s));
        ++launches;
        GB_LAUNCH(k_pivot_list<<<grid_for(P->nc, T), T, 0, s>>>(P->nc, P->pflag, P->ppos, 0,
                                                                 P->pivcol));
        P->np = P->nr;
        GB_CUDA(cudaEventRecord(P->ev[3], s));
        GB_CUDA(cudaEventRecord(P->ev[4], s));
    }
    }  // sparse-row form

    // ---- compaction -----------------------------------------------------------
    const int32_t shift = P->mode == 0 ? P->ncl : 0;
    if (!P->streamed) P->onnz = 0;
    if (P->np > 0 && !P->streamed) {
        GB_LAUNCH(k_row_nnz<<<grid_for((int64_t)P->np * 32, T), T, 0, s>>>(
            P->np, P->pivcol, P->piv_of_col, final_rows, rows_ld, width, P->counts));
        GB_CUDA(cudaMemsetAsync(P->counts + P->np, 0, sizeof(int64_t), s));
        size_t bytes = P->cub_bytes;
        GB_CUDA(cub::DeviceScan::ExclusiveSum(P->cub_tmp, bytes, P->counts, P->offs, P->np + 1, s));
        ++launches;
        GB_CUDA(cudaMemcpyAsync(&P->onnz, P->offs + P->np, 8, cudaMemcpyDeviceToHost, s));
        GB_CUDA(cudaStreamSynchronize(s));
        if (P->onnz > P->out_cap) {
            int rc;
            if ((rc = P->alloc(&P->out_cols, (size_t)P->onnz))) return rc;
            if ((rc = P->alloc(&P->out_vals, (size_t)P->onnz))) return rc;
            P->out_cap = P->onnz;
        }
        GB_LAUNCH(k_row_write<<<grid_for((int64_t)P->np * 32, T), T, 0, s>>>(
            P->np, P->pivcol, P->piv_of_col, final_rows, rows_ld, width, P->offs, shift,
            P->out_cols, P->out_vals, 4));
    }
    GB_CUDA(cudaEventRecord(P->ev[5], s));
    if (P->blocked) {
        blocked_release(&bo, s);
        int32_t tc_status = 0;
        GB_CUDA(cudaMemcpyAsync(&tc_status, P->counters + 6, 4, cudaMemcpyDeviceToHost, s));
        GB_CUDA(cudaStreamSynchronize(s));
        if (tc_status) {
            set_error("tensor-core kernel: a bounded wait expired");
            return tc_status;
        }
    }
    return GBGPU_OK;
}

int finish_stats(Plan* P);

// a small-matrix run enqueues everything without waiting; its input checks,
// answer size and statistics are read here, before the answer is used
int settle(Plan* P) {
    if (!P->pending) return GBGPU_OK;
    P->pending = false;
    int64_t counts[2] = {0, 0};
    GB_CUDA(cudaMemcpyAsync(&P->errbits, P->err, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                            P->stream));
    GB_CUDA(cudaMemcpyAsync(counts, P->tiny_counts, sizeof(counts), cudaMemcpyDeviceToHost,
                            P->stream));
    GB_CUDA(cudaStreamSynchronize(P->stream));
    if (P->errbits) {
        std::string msg;
        const int rc = err_to_status(P->errbits, &msg);
        set_error(msg);
        P->np = 0;
        P->onnz = 0;
        return rc;
    }
    P->np = (int32_t)counts[0];
    P->onnz = counts[1];
    return finish_stats(P);
}

int plan_run(Plan* P) {
    P->launches = 0;
    P->streamed = false;
    P->mapped = false;
    int rc;
    GemmProfile prof;
    if (P->profile) {
        prof.d_steps = P->gemm_steps;
        prof.capacity = kGemmProfileSlots;
        GB_CUDA(cudaMemsetAsync(P->gemm_steps, 0, sizeof(unsigned long long) * kGemmProfileSlots,
                                P->stream));
        set_gemm_profile(&prof);
    }
    if ((uint32_t)P->p < 65536u)
        rc = run_form(P, FieldSmall::make((uint32_t)P->p));
    else
        rc = run_form(P, FieldMont::make((uint32_t)P->p));
    set_gemm_profile(nullptr);
    count_launch(P->launches);
    P->stats.gemm_launches = (int64_t)prof.events.size();
    P->stats.gemm_ms = 0;
    P->stats.gemm_int8_ops = 0;
    if (P->profile && !prof.events.empty()) {
        std::vector<unsigned long long> steps(kGemmProfileSlots, 0);
        GB_CUDA(cudaMemcpyAsync(steps.data(), P->gemm_steps, sizeof(unsigned long long) * steps.size(),
                                cudaMemcpyDeviceToHost, P->stream));
        GB_CUDA(cudaStreamSynchronize(P->stream));
        for (size_t i = 0; i < prof.events.size(); ++i) {
            float ms = 0, split_ms = 0;
            cudaEventElapsedTime(&ms, prof.events[i].first, prof.events[i].second);
            if (i < prof.split_events.size()) {
                cudaEventElapsedTime(&split_ms, prof.split_events[i], prof.events[i].first);
                cudaEventDestroy(prof.split_events[i]);
            }
            cudaEventDestroy(prof.events[i].first);
            cudaEventDestroy(prof.events[i].second);
            const double ops =
                i < steps.size() ? 2.0 * (double)steps[i] * prof.macs_per_step[i] : 0.0;
            P->stats.gemm_ms += ms;
            P->stats.gemm_int8_ops += ops;
            if (debug_trace())
                fprintf(stderr,
                        "gbgpu gemm %3zu: M %6d N %6d K %6d batch %5d  %8.3f ms  %8.1f TOPS"
                        "  splits %8.3f ms\n",
                        i, prof.shape[4 * i], prof.shape[4 * i + 1], prof.shape[4 * i + 2],
                        prof.shape[4 * i + 3], ms, ms > 0 ? ops / (ms * 1e-3) / 1e12 : 0.0,
                        split_ms);
        }
    }
    if (rc) return rc;
    if (P->pending) return GBGPU_OK;  // small matrix: settled when the answer is read
    return finish_stats(P);
}

// statistics of the last run (waits for it)
int finish_stats(Plan* P) {
    GB_CUDA(cudaEventSynchronize(P->ev[5]));
    int64_t wc[2] = {0, 0};
    GB_CUDA(cudaMemcpyAsync(wc, P->work_count, sizeof(wc), cudaMemcpyDeviceToHost, P->stream));
    GB_CUDA(cudaStreamSynchronize(P->stream));
    P->stats.work_schur = wc[0];
    P->stats.work_dense = wc[1];
    float ms[5] = {0, 0, 0, 0, 0};
    cudaEventElapsedTime(&ms[0], P->ev[0], P->ev[5]);
    cudaEventElapsedTime(&ms[1], P->ev[1], P->ev[2]);
    cudaEventElapsedTime(&ms[2], P->ev[2], P->ev[3]);
    cudaEventElapsedTime(&ms[3], P->ev[3], P->ev[4]);
    cudaEventElapsedTime(&ms[4], P->ev[4], P->ev[5]);
    P->stats.ms_total = ms[0];
    P->stats.ms_schur = ms[1];
    P->stats.ms_echelon = ms[2];
    P->stats.ms_rref = ms[3];
    P->stats.ms_compact = ms[4];
    float mc = 0, mv = 0;
    cudaEventElapsedTime(&mc, P->ev[0], P->ev[1]);
    cudaEventElapsedTime(&mv, P->ev[0], P->ev[6]);
    P->stats.ms_classify = mc;
    P->stats.ms_check = mv;
    P->stats.rows_reduced = P->n_work;
    P->stats.rank = P->np;
    P->stats.kernel_launches = P->launches;
    P->stats.form_used = !P->blocked ? GBGPU_FORM_PLAIN
                         : (P->form == GBGPU_FORM_TENSOR ? GBGPU_FORM_TENSOR
                                                         : GBGPU_FORM_BLOCKED_PLAIN);
    return GBGPU_OK;
}

// residues of vb bytes (1 or 2) <-> uint32
__global__ void k_widen(const uint8_t* __restrict__ in, int32_t vb, int64_t n, uint32_t* out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = vb == 1 ? (uint32_t)in[i] : (uint32_t)((const uint16_t*)in)[i];
}
__global__ void k_narrow(const uint32_t* __restrict__ in, int32_t vb, int64_t n, uint8_t* out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (vb == 1) out[i] = (uint8_t)in[i];
        else ((uint16_t*)out)[i] = (uint16_t)in[i];
    }
}

static int val_bytes_of(const gbgpu_csr* m) { return m->val_bytes ? m->val_bytes : 4; }

// ---------------------------------------------------------------------------
// The step after the linear algebra (src/convert.c:137-280): the answer's
// columns become indices of the basis hash table.  The reference looks every
// entry up in that table (insert_in_basis_hash_table_pivots, src/hash.c:604),
// visiting the rows in answer order; a monomial that is not in the table yet
// is inserted when its first entry is met.  Here the answer stays on the
// device: k_first_entry gives every right column the position of its first
// entry in the answer (the order in which the reference inserts), the caller
// looks up or inserts each column's monomial once, and k_map_columns
// rewrites every entry through the resulting column -> index map.

// first[j] = smallest e with cols[e] = shift + j (INT64_MAX: no entry)
__global__ void k_first_entry(int64_t nnz, const int32_t* __restrict__ cols, int32_t shift,
                              unsigned long long* first) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t j = cols[e] - shift;
        // rows are visited roughly in order, so most later entries see a
        // smaller position already and skip the atomic
        if (first[j] > (unsigned long long)e) atomicMin(first + j, (unsigned long long)e);
    }
}

__global__ void k_fill_u64(int64_t n, unsigned long long v, unsigned long long* out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = v;
}

// cols[e] = map[cols[e] - shift]
__global__ void k_map_columns(int64_t nnz, int32_t* cols, int32_t shift,
                              const int32_t* __restrict__ map) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz;
         e += (int64_t)gridDim.x * blockDim.x)
        cols[e] = map[cols[e] - shift];
}

int plan_first_entry(Plan* P, int64_t* first, int32_t n) {
    if (int rc = settle(P)) return rc;
    if (P->mode != 0 || P->streamed || P->mapped || n != P->ncr) {
        set_error("first entries: a linear_algebra plan whose answer is on the device and "
                  "not mapped yet, n = ncr");
        return GBGPU_EINVAL;
    }
    if (n == 0) return GBGPU_OK;
    unsigned long long* d = nullptr;
    if (int rc = P->alloc(&d, (size_t)n)) return rc;
    cudaStream_t s = P->stream;
    k_fill_u64<<<grid_for(n, 256), 256, 0, s>>>(n, ~0ull >> 1, d);
    if (P->onnz > 0)
        k_first_entry<<<grid_for(P->onnz, 256), 256, 0, s>>>(P->onnz, P->out_cols, P->ncl, d);
    GB_CUDA(cudaGetLastError());
    count_launch(P->onnz > 0 ? 2 : 1);
    GB_CUDA(cudaMemcpyAsync(first, d, sizeof(int64_t) * (size_t)n, cudaMemcpyDeviceToHost, s));
    GB_CUDA(cudaStreamSynchronize(s));
    for (int32_t j = 0; j < n; ++j)
        if (first[j] == (int64_t)(~0ull >> 1)) first[j] = -1;
    return GBGPU_OK;
}

int plan_map_columns(Plan* P, const int32_t* map, int32_t n) {
    if (int rc = settle(P)) return rc;
    if (P->mode != 0 || P->streamed || P->mapped || n != P->ncr) {
        set_error("column map: a linear_algebra plan whose answer is on the device and not "
                  "mapped yet, n = ncr");
        return GBGPU_EINVAL;
    }
    if (P->onnz == 0) {
        P->mapped = true;
        return GBGPU_OK;
    }
    int32_t* d = nullptr;
    if (int rc = P->alloc(&d, (size_t)n)) return rc;
    cudaStream_t s = P->stream;
    GB_CUDA(cudaMemcpyAsync(d, map, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, s));
    k_map_columns<<<grid_for(P->onnz, 256), 256, 0, s>>>(P->onnz, P->out_cols, P->ncl, d);
    GB_CUDA(cudaGetLastError());
    count_launch(1);
    // the answer's columns are indices of the caller's table from now on:
    // they no longer count from ncl
    GB_CUDA(cudaStreamSynchronize(s));
    P->mapped = true;
    return GBGPU_OK;
}

int plan_create(const gbgpu_csr* m, const gbgpu_options* opt, int mode, Plan** out) {
    *out = nullptr;
    if (!m || m->p < 2 || m->nr < 0 || m->ncl < 0 || m->ncr < 0 ||
        (int64_t)m->ncl + m->ncr > INT_MAX / 2) {
        set_error("bad matrix header");
        return GBGPU_EINVAL;
    }
    if (m->nr > 0 && (!m->row_ptr || !m->cols || !m->vals)) {
        set_error("null CSR array");
        return GBGPU_EINVAL;
    }
    const int vb = val_bytes_of(m);
    if (!(vb == 1 || vb == 2 || vb == 4) || (vb < 4 && (int64_t)m->p >= ((int64_t)1 << (8 * vb)))) {
        set_error("val_bytes must be 4, 2 (p < 2^16) or 1 (p < 2^8)");
        return GBGPU_EINVAL;
    }
    Plan* P = new (std::nothrow) Plan();
    if (!P) return GBGPU_ENOMEM;
    int rc = plan_setup(P, opt);
    if (rc) {
        delete P;
        return rc;
    }
    P->mode = mode;
    P->p = m->p;
    P->nr = m->nr;
    P->ncl = m->ncl;
    P->ncr = m->ncr;
    P->nc = m->ncl + m->ncr;
    P->nnz = m->nr > 0 ? m->row_ptr[m->nr] : 0;
    if (m->nr > 0 && (m->row_ptr[0] != 0 || P->nnz < 0)) {
        delete P;
        set_error("row_ptr must start at 0");
        return GBGPU_EINVAL;
    }
    // rows to reduce: C|D rows (nr - ncl when the contract holds) or all rows
    P->n_work = mode == 0 ? std::max(0, m->nr - m->ncl) : m->nr;
    if ((rc = plan_alloc(P))) {
        delete P;
        return rc;
    }
    cudaError_t e1 = cudaMemcpyAsync(P->row_ptr, m->row_ptr, sizeof(int64_t) * (P->nr + 1),
                                     cudaMemcpyHostToDevice, P->stream);
    cudaError_t e2 = cudaMemcpyAsync(P->cols, m->cols, sizeof(int32_t) * P->nnz,
                                     cudaMemcpyHostToDevice, P->stream);
    cudaError_t e3 = cudaSuccess;
    if (vb == 4) {
        e3 = cudaMemcpyAsync(P->vals, m->vals, sizeof(int32_t) * P->nnz, cudaMemcpyHostToDevice,
                             P->stream);
    } else if (P->nnz > 0) {
        // narrow values on the wire, widened on the device
        if ((rc = P->alloc(&P->wire, (size_t)P->nnz * vb))) {
            delete P;
            return rc;
        }
        P->wire_cap = (size_t)P->nnz * vb;
        e3 = cudaMemcpyAsync(P->wire, m->vals, (size_t)P->nnz * vb, cudaMemcpyHostToDevice,
                             P->stream);
        if (e3 == cudaSuccess) {
            k_widen<<<grid_for(P->nnz, 256), 256, 0, P->stream>>>(P->wire, vb, P->nnz, P->vals);
            e3 = cudaGetLastError();
            count_launch(1);
        }
    }
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
        set_error("host to device copy failed");
        delete P;
        return GBGPU_ECUDA;
    }
    *out = P;
    return GBGPU_OK;
}

int plan_result(Plan* P, gbgpu_rows* out) {
    memset(out, 0, sizeof(*out));
    if (int rc = settle(P)) return rc;
    if (P->streamed) {
        set_error("the last run delivered its answer through gbgpu_plan_run_into_v");
        return GBGPU_EINVAL;
    }
    GB_CUDA(cudaStreamSynchronize(P->stream));
    out->np = P->np;
    out->nnz = P->onnz;
    out->row_ptr = (int64_t*)malloc(sizeof(int64_t) * (P->np + 1));
    out->cols = (int32_t*)malloc(sizeof(int32_t) * std::max<int64_t>(P->onnz, 1));
    out->vals = (int32_t*)malloc(sizeof(int32_t) * std::max<int64_t>(P->onnz, 1));
    if (!out->row_ptr || !out->cols || !out->vals) {
        gbgpu_rows_free(out);
        return GBGPU_ENOMEM;
    }
    out->row_ptr[0] = 0;
    if (P->np > 0) {
        GB_CUDA(cudaMemcpyAsync(out->row_ptr, P->offs, sizeof(int64_t) * (P->np + 1),
                                cudaMemcpyDeviceToHost, P->stream));
        if (P->onnz > 0) {
            GB_CUDA(cudaMemcpyAsync(out->cols, P->out_cols, sizeof(int32_t) * P->onnz,
                                    cudaMemcpyDeviceToHost, P->stream));
            GB_CUDA(cudaMemcpyAsync(out->vals, P->out_vals, sizeof(int32_t) * P->onnz,
                                    cudaMemcpyDeviceToHost, P->stream));
        }
        GB_CUDA(cudaStreamSynchronize(P->stream));
    }
    return GBGPU_OK;
}

// copy the answer into caller-provided host arrays (no allocation)
int plan_result_into(Plan* P, int64_t* row_ptr, int32_t* cols, int32_t* vals, int64_t cap_rows,
                     int64_t cap_nnz, int32_t* np, int64_t* nnz) {
    if (int rc = settle(P)) return rc;
    if (P->streamed) {
        set_error("the last run delivered its answer through gbgpu_plan_run_into_v");
        return GBGPU_EINVAL;
    }
    GB_CUDA(cudaStreamSynchronize(P->stream));
    *np = P->np;
    *nnz = P->onnz;
    if ((int64_t)P->np + 1 > cap_rows || P->onnz > cap_nnz) {
        set_error("result buffers too small");
        return GBGPU_ERANGE;
    }
    row_ptr[0] = 0;
    if (P->np > 0) {
        GB_CUDA(cudaMemcpyAsync(row_ptr, P->offs, sizeof(int64_t) * (P->np + 1),
                                cudaMemcpyDeviceToHost, P->stream));
        if (P->onnz > 0) {
            GB_CUDA(cudaMemcpyAsync(cols, P->out_cols, sizeof(int32_t) * P->onnz,
                                    cudaMemcpyDeviceToHost, P->stream));
            GB_CUDA(cudaMemcpyAsync(vals, P->out_vals, sizeof(int32_t) * P->onnz,
                                    cudaMemcpyDeviceToHost, P->stream));
        }
        GB_CUDA(cudaStreamSynchronize(P->stream));
    }
    return GBGPU_OK;
}

// the same with values of vb bytes (1, 2: narrowed on the device first)
int plan_result_into_v(Plan* P, int64_t* row_ptr, int32_t* cols, void* vals, int32_t vb,
                       int64_t cap_rows, int64_t cap_nnz, int32_t* np, int64_t* nnz) {
    if (vb == 4)
        return plan_result_into(P, row_ptr, cols, (int32_t*)vals, cap_rows, cap_nnz, np, nnz);
    if (!(vb == 1 || vb == 2) || (int64_t)P->p >= ((int64_t)1 << (8 * vb))) {
        set_error("val_bytes must be 4, 2 (p < 2^16) or 1 (p < 2^8)");
        return GBGPU_EINVAL;
    }
    if (int rc = settle(P)) return rc;
    if (P->streamed) {
        set_error("the last run delivered its answer through gbgpu_plan_run_into_v");
        return GBGPU_EINVAL;
    }
    GB_CUDA(cudaStreamSynchronize(P->stream));
    *np = P->np;
    *nnz = P->onnz;
    if ((int64_t)P->np + 1 > cap_rows || P->onnz > cap_nnz) {
        set_error("result buffers too small");
        return GBGPU_ERANGE;
    }
    row_ptr[0] = 0;
    if (P->np > 0) {
        GB_CUDA(cudaMemcpyAsync(row_ptr, P->offs, sizeof(int64_t) * (P->np + 1),
                                cudaMemcpyDeviceToHost, P->stream));
        if (P->onnz > 0) {
            const size_t need = (size_t)P->onnz * vb;
            if (need > P->wire_cap) {
                int rc = P->alloc(&P->wire, need);
                if (rc) return rc;
                P->wire_cap = need;
            }
            GB_CUDA(cudaMemcpyAsync(cols, P->out_cols, sizeof(int32_t) * P->onnz,
                                    cudaMemcpyDeviceToHost, P->stream));
            k_narrow<<<grid_for(P->onnz, 256), 256, 0, P->stream>>>((const uint32_t*)P->out_vals,
                                                                     vb, P->onnz, P->wire);
            GB_CUDA(cudaGetLastError());
            count_launch(1);
            GB_CUDA(cudaMemcpyAsync(vals, P->wire, need, cudaMemcpyDeviceToHost, P->stream));
        }
        GB_CUDA(cudaStreamSynchronize(P->stream));
    }
    return GBGPU_OK;
}

// run and deliver the answer into host arrays; on the blocked form the
// back substitution's finished blocks are copied while the rest is computed
int plan_run_into_v(Plan* P, int64_t* row_ptr, int32_t* cols, void* vals, int32_t vb,
                    int64_t cap_rows, int64_t cap_nnz, int32_t* np, int64_t* nnz) {
    if (!(vb == 1 || vb == 2 || vb == 4) || (vb < 4 && (int64_t)P->p >= ((int64_t)1 << (8 * vb)))) {
        set_error("val_bytes must be 4, 2 (p < 2^16) or 1 (p < 2^8)");
        return GBGPU_EINVAL;
    }
    if (!P->blocked || P->mode != 0 || !row_ptr || !cols || !vals) {
        int rc = plan_run(P);
        if (rc) return rc;
        return plan_result_into_v(P, row_ptr, cols, vals, vb, cap_rows, cap_nnz, np, nnz);
    }
    if (!P->s_out) GB_CUDA(cudaStreamCreateWithFlags(&P->s_out, cudaStreamNonBlocking));
    StreamOut so;
    so.col_shift = P->ncl;
    so.offs = P->offs;
    so.h_cols = cols;
    so.h_vals = vals;
    so.val_bytes = vb;
    so.cap_nnz = cap_nnz;
    so.s_out = P->s_out;
    P->stream_req = &so;
    int rc = plan_run(P);
    P->stream_req = nullptr;
    cudaError_t e = cudaStreamSynchronize(P->s_out);
    if (rc) return rc;
    if (e != cudaSuccess) {
        set_error(std::string("answer copy: ") + cudaGetErrorString(e));
        return GBGPU_ECUDA;
    }
    *np = P->np;
    *nnz = P->onnz;
    if ((int64_t)P->np + 1 > cap_rows || so.overflow) {
        set_error("result buffers too small");
        return GBGPU_ERANGE;
    }
    GB_CUDA(cudaMemcpyAsync(row_ptr, P->offs, sizeof(int64_t) * (P->np + 1),
                            cudaMemcpyDeviceToHost, P->stream));
    GB_CUDA(cudaStreamSynchronize(P->stream));
    return GBGPU_OK;
}

// host CSR of a gbgpu_csr into the small path's staging (values widened)
void fill_from_csr_vals(void* ctx, int64_t* row_ptr, int32_t* cols, uint32_t* vals) {
    const gbgpu_csr* m = (const gbgpu_csr*)ctx;
    const int64_t nnz = m->row_ptr[m->nr];
    memcpy(row_ptr, m->row_ptr, sizeof(int64_t) * (size_t)(m->nr + 1));
    memcpy(cols, m->cols, sizeof(int32_t) * (size_t)nnz);
    const int vb = m->val_bytes ? m->val_bytes : 4;
    if (vb == 4) {
        memcpy(vals, m->vals, sizeof(int32_t) * (size_t)nnz);
    } else if (vb == 2) {
        const uint16_t* v = (const uint16_t*)m->vals;
        for (int64_t k = 0; k < nnz; ++k) vals[k] = v[k];
    } else {
        const uint8_t* v = (const uint8_t*)m->vals;
        for (int64_t k = 0; k < nnz; ++k) vals[k] = v[k];
    }
}

void plan_destroy(Plan* P) { delete P; }
const gbgpu_stats& plan_stats(const Plan* P) { return P->stats; }

}  // namespace gbgpu

// ===========================================================================
// C ABI
using namespace gbgpu;

extern "C" {

struct gbgpu_plan {
    Plan* impl;
    int impl_device() const { return impl ? impl->device : -1; }
};

int gbgpu_plan_create(const gbgpu_csr* m, const gbgpu_options* opt, gbgpu_plan** plan) {
    DeviceScope scope;
    if (!plan) return GBGPU_EINVAL;
    Plan* P = nullptr;
    int rc = plan_create(m, opt, 0, &P);
    if (rc) return rc;
    *plan = new gbgpu_plan{P};
    return GBGPU_OK;
}

int gbgpu_plan_run(gbgpu_plan* plan) {
    DeviceScope scope(plan ? plan->impl_device() : -1);
    if (!plan) return GBGPU_EINVAL;
    return plan_run(plan->impl);
}

int gbgpu_plan_first_entry(gbgpu_plan* plan, int64_t* first, int32_t n) {
    DeviceScope scope(plan ? plan->impl_device() : -1);
    if (!plan || (!first && n > 0)) return GBGPU_EINVAL;
    return plan_first_entry(plan->impl, first, n);
}

int gbgpu_plan_map_columns(gbgpu_plan* plan, const int32_t* map, int32_t n) {
    DeviceScope scope(plan ? plan->impl_device() : -1);
    if (!plan || (!map && n > 0)) return GBGPU_EINVAL;
    return plan_map_columns(plan->impl, map, n);
}

int gbgpu_plan_result(gbgpu_plan* plan, gbgpu_rows* out) {
    DeviceScope scope(plan ? plan->impl_device() : -1);
    if (!plan || !out) return GBGPU_EINVAL;
    return plan_result(plan->impl, out);
}

int gbgpu_plan_result_into(gbgpu_plan* plan, int64_t* row_ptr, int32_t* cols, int32_t* vals,
                           int64_t cap_rows, int64_t cap_nnz, int32_t* np, int64_t* nnz) {
    DeviceScope scope(plan ? plan->impl_device() : -1);
    if (!plan || !np || !nnz) return GBGPU_EINVAL;
    if ((!row_ptr || !cols || !vals) && (cap_rows > 0 || cap_nnz > 0)) return GBGPU_EINVAL;
    // NULL buffers with zero capacities query the sizes (GBGPU_ERANGE)
    return plan_result_into(plan->impl, row_ptr, cols, vals, cap_rows, cap_nnz, np, nnz);
}

int gbgpu_plan_result_into_v(gbgpu_plan* plan, int64_t* row_ptr, int32_t* cols, void* vals,
                             int32_t val_bytes, int64_t cap_rows, int64_t cap_nnz, int32_t* np,
                             int64_t* nnz) {
    DeviceScope scope(plan ? plan->impl_device() : -1);
    if (!plan || !np || !nnz) return GBGPU_EINVAL;
    if ((!row_ptr || !cols || !vals) && (cap_rows > 0 || cap_nnz > 0)) return GBGPU_EINVAL;
    return plan_result_into_v(plan->impl, row_ptr, cols, vals, val_bytes, cap_rows, cap_nnz, np,
                              nnz);
}

int gbgpu_plan_run_into_v(gbgpu_plan* plan, int64_t* row_ptr, int32_t* cols, void* vals,
                          int32_t val_bytes, int64_t cap_rows, int64_t cap_nnz, int32_t* np,
                          int64_t* nnz) {
    DeviceScope scope(plan ? plan->impl_device() : -1);
    if (!plan || !np || !nnz) return GBGPU_EINVAL;
    if ((!row_ptr || !cols || !vals) && (cap_rows > 0 || cap_nnz > 0)) return GBGPU_EINVAL;
    return plan_run_into_v(plan->impl, row_ptr, cols, vals, val_bytes, cap_rows, cap_nnz, np,
                           nnz);
}

int gbgpu_plan_stats(const gbgpu_plan* plan, gbgpu_stats* stats) {
    DeviceScope scope(plan ? plan->impl_device() : -1);
    if (!plan || !stats) return GBGPU_EINVAL;
    // a pending small-matrix run is settled first (its timings, its checks)
    const int rc = settle(plan->impl);
    *stats = plan_stats(plan->impl);
    return rc;
}

void gbgpu_plan_destroy(gbgpu_plan* plan) {
    DeviceScope scope(plan ? plan->impl_device() : -1);
    if (!plan) return;
    plan_destroy(plan->impl);
    delete plan;
}

// small matrices take the one-pass path of small.cu (AUTO or the sparse-row
// form, library stream, no profiling); *handled tells whether it ran
static int reduce_small(const gbgpu_csr* m, const gbgpu_options* opt, gbgpu_rows* out,
                        bool* handled) {
    *handled = false;
    gbgpu_options o{};
    if (opt) o = *opt;
    if (!(o.form == GBGPU_FORM_AUTO || o.form == GBGPU_FORM_PLAIN) || o.stream || o.profile)
        return GBGPU_OK;
    if (!m || m->p < 2 || m->nr <= 0 || !m->row_ptr || !m->cols || !m->vals) return GBGPU_OK;
    const int vb = val_bytes_of(m);
    if (!(vb == 1 || vb == 2 || vb == 4) || (vb < 4 && (int64_t)m->p >= ((int64_t)1 << (8 * vb))))
        return GBGPU_OK;
    // 32-bit entry offsets on the small path
    if (m->row_ptr[0] != 0 || m->row_ptr[m->nr] < 0 || m->row_ptr[m->nr] > INT_MAX / 2)
        return GBGPU_OK;
    if (!small_eligible(m->nr, m->ncl, m->ncr, o.device)) return GBGPU_OK;
    *handled = true;
    SmallInput in{m->p, m->nr, m->ncl, m->ncr, m->row_ptr[m->nr], o.device, fill_from_csr_vals,
                  (void*)m};
    SmallAnswer a;
    int rc = small_reduce(in, &a);
    if (rc) return rc;
    out->np = a.np;
    out->nnz = a.nnz;
    out->row_ptr = (int64_t*)malloc(sizeof(int64_t) * (size_t)(a.np + 1));
    out->cols = (int32_t*)malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(a.nnz, 1));
    out->vals = (int32_t*)malloc(sizeof(int32_t) * (size_t)std::max<int64_t>(a.nnz, 1));
    if (!out->row_ptr || !out->cols || !out->vals) {
        gbgpu_rows_free(out);
        return GBGPU_ENOMEM;
    }
    memcpy(out->row_ptr, a.offs, sizeof(int64_t) * (size_t)(a.np + 1));
    memcpy(out->cols, a.cols, sizeof(int32_t) * (size_t)a.nnz);
    memcpy(out->vals, a.vals, sizeof(int32_t) * (size_t)a.nnz);
    return GBGPU_OK;
}

int gbgpu_reduce(const gbgpu_csr* m, const gbgpu_options* opt, gbgpu_rows* out) {
    DeviceScope scope;
    if (!out) return GBGPU_EINVAL;
    memset(out, 0, sizeof(*out));
    bool handled = false;
    int rs = reduce_small(m, opt, out, &handled);
    if (handled) return rs;
    Plan* P = nullptr;
    int rc = plan_create(m, opt, 0, &P);
    if (rc) return rc;
    rc = plan_run(P);
    if (!rc) rc = plan_result(P, out);
    plan_destroy(P);
    return rc;
}

int gbgpu_interreduce(int32_t p, int32_t nr, int32_t nc, const int64_t* row_ptr,
                      const int32_t* cols, const int32_t* vals, const gbgpu_options* opt,
                      gbgpu_rows* out) {
    DeviceScope scope;
    if (!out) return GBGPU_EINVAL;
    memset(out, 0, sizeof(*out));
    gbgpu_csr m{p, 2, nr, 0, nc, row_ptr, cols, vals};
    Plan* P = nullptr;
    int rc = plan_create(&m, opt, 1, &P);
    if (rc) return rc;
    rc = plan_run(P);
    if (!rc) rc = plan_result(P, out);
    plan_destroy(P);
    return rc;
}

void gbgpu_rows_free(gbgpu_rows* rows) {
    if (!rows) return;
    free(rows->row_ptr);
    free(rows->cols);
    free(rows->vals);
    memset(rows, 0, sizeof(*rows));
}

const char* gbgpu_last_error(void) { return g_last_error.c_str(); }
int64_t gbgpu_kernel_launches(void) { return g_launches.load(); }

}  // extern "C"
