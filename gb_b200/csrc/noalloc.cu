// noalloc.cu -- the one entry point of libgbgpu.so that allocates nothing.
//
// Some callers cannot allocate device memory once they are running: a
// service that reserves its whole device-memory budget at start-up and must
// not exceed it later, or a host program that hands the library pointers
// into a pool it manages itself and forbids any other cudaMalloc / cudaFree
// (a second allocator in the process would fragment or overrun its pool).
// For them, gbgpu_dense_submul_noalloc performs the same exact modular GEMM
// as gbgpu_dense_submul (tensor-core form) but takes its scratch memory --
// the 8-bit limb planes of A and B and the kernel's status word -- from one
// file-scope device array of kNoAllocScratchBytes bytes instead of
// allocating it.
//
// The array lives on every GPU that loads the library, from load until the
// process exits; the CUDA driver sets its memory aside when it loads the
// library's device code on that GPU (with lazy module loading, during the
// first call that needs it), not this entry point.  In host code its name is only a host-side stand-in, never
// a device address, so its device address is looked up with
// cudaGetSymbolAddress (with that device current) by the first call on each
// device, and cached for the life of the process; calls on a device after a
// cudaDeviceReset of it are therefore not supported.  All calls share the
// one array and it keeps the last call's contents: the status word is
// cleared by every call, the limb planes are fully rewritten (zero padding
// included).  Calls that overlap on the GPU (different streams or threads)
// race on it and must be serialised by the caller.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/gbgpu.h"
#include "internal.h"
#include "tc_gemm.h"

namespace {

// 32 MiB: 256 bytes of status, the rest for limb planes
constexpr size_t kNoAllocScratchBytes = (size_t)32 << 20;
constexpr size_t kStatusBytes = 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// device address of the scratch array on `device` (current device)
int scratch_address(int device, void** out) {
    if (device < 0 || device >= kMaxDevices) {
        gbgpu::set_error("device ordinal out of range");
        return GBGPU_ENODEV;
    }
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            gbgpu::set_error(std::string("cudaGetSymbolAddress(scratch): ") +
                             cudaGetErrorString(e));
            return GBGPU_ECUDA;
        }
        g_scratch_ptr[device] = p;
    }
    *out = g_scratch_ptr[device];
    return GBGPU_OK;
}

}  // namespace

extern "C" int gbgpu_dense_submul_noalloc(int32_t p, int32_t M, int32_t N, int32_t K,
                                          const uint32_t* A, int64_t lda, const uint32_t* B,
                                          int64_t ldb, uint32_t* D, int64_t ldd,
                                          int32_t device, void* stream) {
    using namespace gbgpu;
    if (p < 3 || (p & 1) == 0 || M < 0 || N < 0 || K < 0 || lda < K || ldb < N || ldd < N) {
        set_error("gbgpu_dense_submul_noalloc: bad arguments (needs an odd prime >= 3)");
        return GBGPU_EINVAL;
    }
    const size_t need = tc_workspace_bytes((uint32_t)p, M, N, K);
    if (need > kNoAllocScratchBytes - kStatusBytes) {
        set_error("gbgpu_dense_submul_noalloc: limb planes need " + std::to_string(need) +
                  " bytes, more than the fixed scratch of " +
                  std::to_string(kNoAllocScratchBytes - kStatusBytes) + " bytes");
        return GBGPU_ERANGE;
    }
    DeviceInfo dev;
    int rc = device_init(device, &dev);
    if (rc) return rc;
    void* scratch = nullptr;
    rc = scratch_address(device, &scratch);
    if (rc) return rc;
    if (M == 0 || N == 0 || K == 0) return GBGPU_OK;
    cudaStream_t s = (cudaStream_t)stream;
    int32_t* status = (int32_t*)scratch;
    void* planes = (unsigned char*)scratch + kStatusBytes;
    cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int32_t), s);
    if (e != cudaSuccess) {
        set_error(std::string("noalloc status clear: ") + cudaGetErrorString(e));
        return GBGPU_ECUDA;
    }
    long long launches = 0;
    TcGemmArgs g{(uint32_t)p, M, N, K, A, lda, B, ldb, D, ldd};
    rc = tc_submul(g, planes, s, status, &launches);
    count_launch(launches);
    if (rc) return rc;
    int32_t h = 0;
    e = cudaMemcpyAsync(&h, status, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_error(std::string("noalloc GEMM: ") + cudaGetErrorString(e));
        return GBGPU_ECUDA;
    }
    if (h) {
        set_error("noalloc GEMM: a bounded wait expired");
        return h;
    }
    return GBGPU_OK;
}
