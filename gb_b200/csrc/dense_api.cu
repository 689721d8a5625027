// dense_api.cu -- C ABI of the dense exact modular GEMM (include/gbgpu.h).
#include <cuda_runtime.h>

#include <cstring>
#include <string>

#include "../../include/gbgpu.h"
#include "blocked.h"
#include "internal.h"
#include "tc_gemm.h"

using namespace gbgpu;

namespace {

int check_args(int32_t p, int32_t M, int32_t N, int32_t K, int64_t lda, int64_t ldb,
               int64_t ldd) {
    if (p < 2 || M < 0 || N < 0 || K < 0 || lda < K || ldb < N || ldd < N) {
        set_error("bad dense GEMM arguments");
        return GBGPU_EINVAL;
    }
    return GBGPU_OK;
}

int run_dense(int32_t p, int32_t M, int32_t N, int32_t K, const uint32_t* A, int64_t lda,
              const uint32_t* B, int64_t ldb, uint32_t* D, int64_t ldd, const gbgpu_options* opt,
              cudaStream_t s) {
    const int form = opt ? opt->form : GBGPU_FORM_AUTO;
    long long launches = 0;
    TcGemmArgs g{(uint32_t)p, M, N, K, A, lda, B, ldb, D, ldd};
    int rc = GBGPU_OK;
    const bool tensor = form != GBGPU_FORM_PLAIN && (p & 1) && p >= 3;
    if (form == GBGPU_FORM_TENSOR && !tensor) {
        set_error("tensor-core form needs an odd prime");
        return GBGPU_EINVAL;
    }
    if (tensor) {
        void* ws = nullptr;
        int32_t* err = nullptr;
        const size_t bytes = tc_workspace_bytes((uint32_t)p, M, N, K);
        if (cudaMallocAsync(&ws, bytes > 0 ? bytes : 1, s) != cudaSuccess ||
            cudaMallocAsync((void**)&err, sizeof(int32_t), s) != cudaSuccess) {
            set_error("dense GEMM workspace allocation failed");
            return GBGPU_ENOMEM;
        }
        cudaMemsetAsync(err, 0, sizeof(int32_t), s);
        rc = tc_submul(g, ws, s, err, &launches);
        int32_t herr = 0;
        cudaMemcpyAsync(&herr, err, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
        cudaFreeAsync(ws, s);
        cudaFreeAsync(err, s);
        cudaError_t e = cudaStreamSynchronize(s);
        if (!rc && e != cudaSuccess) {
            set_error(std::string("dense GEMM: ") + cudaGetErrorString(e));
            rc = GBGPU_ECUDA;
        }
        if (!rc && herr) {
            set_error("tensor-core GEMM: a bounded wait expired");
            rc = herr;
        }
    } else {
        rc = plain_submul(g, s, &launches);
        cudaError_t e = cudaStreamSynchronize(s);
        if (!rc && e != cudaSuccess) {
            set_error(std::string("dense GEMM: ") + cudaGetErrorString(e));
            rc = GBGPU_ECUDA;
        }
    }
    count_launch(launches);
    return rc;
}

}  // namespace

extern "C" {

int gbgpu_dense_submul(int32_t p, int32_t M, int32_t N, int32_t K, const uint32_t* A,
                       int64_t lda, const uint32_t* B, int64_t ldb, uint32_t* D, int64_t ldd,
                       const gbgpu_options* opt) {
    DeviceScope scope;
    int rc = check_args(p, M, N, K, lda, ldb, ldd);
    if (rc) return rc;
    DeviceInfo dev;
    rc = device_init(opt ? opt->device : 0, &dev);
    if (rc) return rc;
    cudaStream_t s = opt ? (cudaStream_t)opt->stream : nullptr;
    return run_dense(p, M, N, K, A, lda, B, ldb, D, ldd, opt, s);
}

int gbgpu_dense_submul_host(int32_t p, int32_t M, int32_t N, int32_t K, const uint32_t* A,
                            int64_t lda, const uint32_t* B, int64_t ldb, uint32_t* D,
                            int64_t ldd, const gbgpu_options* opt) {
    DeviceScope scope;
    int rc = check_args(p, M, N, K, lda, ldb, ldd);
    if (rc) return rc;
    DeviceInfo dev;
    rc = device_init(opt ? opt->device : 0, &dev);
    if (rc) return rc;
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return GBGPU_ECUDA;
    uint32_t *dA = nullptr, *dB = nullptr, *dD = nullptr;
    const size_t na = (size_t)M * K, nb = (size_t)K * N, nd = (size_t)M * N;
    if (cudaMallocAsync((void**)&dA, na * 4 + 4, s) != cudaSuccess ||
        cudaMallocAsync((void**)&dB, nb * 4 + 4, s) != cudaSuccess ||
        cudaMallocAsync((void**)&dD, nd * 4 + 4, s) != cudaSuccess) {
        cudaStreamDestroy(s);
        set_error("dense GEMM allocation failed");
        return GBGPU_ENOMEM;
    }
    cudaMemcpy2DAsync(dA, (size_t)K * 4, A, (size_t)lda * 4, (size_t)K * 4, M,
                      cudaMemcpyHostToDevice, s);
    cudaMemcpy2DAsync(dB, (size_t)N * 4, B, (size_t)ldb * 4, (size_t)N * 4, K,
                      cudaMemcpyHostToDevice, s);
    cudaMemcpy2DAsync(dD, (size_t)N * 4, D, (size_t)ldd * 4, (size_t)N * 4, M,
                      cudaMemcpyHostToDevice, s);
    gbgpu_options o{};
    if (opt) o = *opt;
    rc = run_dense(p, M, N, K, dA, K, dB, N, dD, N, &o, s);
    if (!rc)
        cudaMemcpy2DAsync(D, (size_t)ldd * 4, dD, (size_t)N * 4, (size_t)N * 4, M,
                          cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(dA, s);
    cudaFreeAsync(dB, s);
    cudaFreeAsync(dD, s);
    cudaError_t e = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (!rc && e != cudaSuccess) {
        set_error(std::string("dense GEMM copy: ") + cudaGetErrorString(e));
        rc = GBGPU_ECUDA;
    }
    return rc;
}

int gbgpu_dense_rref(int32_t p, int32_t rows, int32_t cols, uint32_t* D, int64_t ld,
                     int32_t* rank, int32_t* piv_cols, const gbgpu_options* opt) {
    DeviceScope scope;
    if (p < 2 || rows < 0 || cols < 0 || ld < cols || !rank || (rows > 0 && cols > 0 && (!D || !piv_cols))) {
        set_error("bad dense RREF arguments");
        return GBGPU_EINVAL;
    }
    *rank = 0;
    DeviceInfo dev;
    int rc = device_init(opt ? opt->device : 0, &dev);
    if (rc) return rc;
    if (rows == 0 || cols == 0) return GBGPU_OK;
    cudaStream_t s = opt ? (cudaStream_t)opt->stream : nullptr;
    int32_t* err = nullptr;
    if (cudaMallocAsync((void**)&err, sizeof(int32_t), s) != cudaSuccess) return GBGPU_ENOMEM;
    cudaMemsetAsync(err, 0, sizeof(int32_t), s);
    const int form = opt ? opt->form : GBGPU_FORM_AUTO;
    DenseRrefInput in{(uint32_t)p, rows, cols, D, ld, piv_cols, s,
                      (form == GBGPU_FORM_PLAIN || form == GBGPU_FORM_BLOCKED_PLAIN || !(p & 1) || p < 3)
                          ? GBGPU_FORM_PLAIN
                          : GBGPU_FORM_TENSOR,
                      err};
    long long launches = 0;
    rc = dense_rref(in, rank, &launches);
    count_launch(launches);
    int32_t herr = 0;
    cudaMemcpyAsync(&herr, err, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(err, s);
    cudaError_t e = cudaStreamSynchronize(s);
    if (!rc && e != cudaSuccess) {
        set_error(std::string("dense RREF: ") + cudaGetErrorString(e));
        rc = GBGPU_ECUDA;
    }
    if (!rc && herr) {
        set_error("dense RREF: a bounded wait expired");
        rc = herr;
    }
    return rc;
}

}  // extern "C"
