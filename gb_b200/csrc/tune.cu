// tune.cu -- the autotuner of the tensor-core GEMM's tile shape.
//
// k_tc_submul has up to three tile shapes per limb count L (tc_gemm.cu:
// big, mid, small), each best in a different range of the reduction depth K.
// gbgpu_autotune times every candidate shape on this device for every
// (L, K bucket) -- exact modular GEMMs on uniform residues, CUDA events, best
// of three after a warm-up -- and writes the winners to a cache file:
//
//   # gbgpu GEMM tile shapes: limbs kmax shape (0 big, 1 small, 2 mid)
//   2 256 1
//   ...
//
// The library reads that file once per process (GBGPU_TUNE_FILE, else
// $HOME/.cache/gbgpu/gemm_shapes.txt when it exists) and uses it for every
// tensor-core GEMM; without a file, or for a bucket the file does not name,
// it keeps the built-in rule.  Every shape computes the same exact result;
// only the speed differs.  The limb count is not tuned: it follows from p.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <sys/stat.h>

#include "../../include/gbgpu.h"
#include "internal.h"
#include "tc_gemm.h"

namespace gbgpu {

namespace {

constexpr int kBuckets = 7;
constexpr int kKmax[kBuckets] = {128, 256, 512, 1024, 1536, 4096, 1 << 30};
constexpr int kShapeBig = 0, kShapeSmall = 1, kShapeMid = 2;

std::mutex g_mu;
bool g_loaded = false;
int g_table[5][kBuckets];  // [L][bucket], -1: built-in rule

int bucket_of(int K) {
    for (int b = 0; b < kBuckets; ++b)
        if (K <= kKmax[b]) return b;
    return kBuckets - 1;
}

// the built-in rule (measured when the shapes were written)
int default_shape(int L, int K) {
    if (L == 1) return K <= 256 ? kShapeSmall : kShapeBig;
    if (L == 2) return K <= 256 ? kShapeSmall : (K <= 1536 ? kShapeMid : kShapeBig);
    return kShapeBig;
}

bool valid(int L, int kmax, int shape) {
    if (shape == kShapeBig) return true;
    if (shape == kShapeSmall) return L <= 2 && kmax <= 256;
    if (shape == kShapeMid) return L == 2;
    return false;
}

std::string default_path() {
    if (const char* f = getenv("GBGPU_TUNE_FILE")) return f;
    if (const char* h = getenv("HOME")) return std::string(h) + "/.cache/gbgpu/gemm_shapes.txt";
    return "";
}

void load_locked(const std::string& path) {
    for (auto& row : g_table)
        for (int& x : row) x = -1;
    g_loaded = true;
    if (path.empty()) return;
    FILE* f = fopen(path.c_str(), "r");
    if (!f) return;
    char line[256];
    while (fgets(line, sizeof(line), f)) {
        if (line[0] == '#') continue;
        int L = 0, kmax = 0, shape = -1;
        if (sscanf(line, "%d %d %d", &L, &kmax, &shape) != 3) continue;
        if (L < 1 || L > 4) continue;
        const int b = bucket_of(kmax);
        if (kKmax[b] != kmax || !valid(L, kmax, shape)) continue;
        g_table[L][b] = shape;
    }
    fclose(f);
}

__global__ void k_uniform(uint32_t* x, int64_t n, uint32_t p, uint64_t seed) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint64_t z = seed + (uint64_t)i * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        x[i] = (uint32_t)((z ^ (z >> 31)) % p);
    }
}

}  // namespace

int tc_shape_for(int L, int K) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_loaded) load_locked(default_path());
    const int t = g_table[std::min(std::max(L, 1), 4)][bucket_of(K)];
    return t >= 0 ? t : default_shape(L, K);
}

}  // namespace gbgpu

using namespace gbgpu;

extern "C" int gbgpu_autotune(int32_t device, const char* path) {
    DeviceScope scope;
    DeviceInfo dev;
    int rc = device_init(device, &dev);
    if (rc) return rc;
    const std::string out = path && path[0] ? path : default_path();
    if (out.empty()) {
        set_error("gbgpu_autotune: no cache path (GBGPU_TUNE_FILE or HOME)");
        return GBGPU_EINVAL;
    }
    const int M = 4096, N = 4096, Kmax = 8192;
    const uint32_t primes[3] = {251u, 65521u, 0u};
    uint32_t *A = nullptr, *B = nullptr, *D = nullptr;
    void* ws = nullptr;
    int32_t* err = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const size_t ws_bytes = tc_workspace_bytes(65521u, M, N, Kmax);
    auto cleanup = [&]() {
        if (s) cudaStreamSynchronize(s);
        cudaFree(A);
        cudaFree(B);
        cudaFree(D);
        cudaFree(ws);
        cudaFree(err);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (s) cudaStreamDestroy(s);
    };
    if (cudaMalloc(&A, sizeof(uint32_t) * (size_t)M * Kmax) != cudaSuccess ||
        cudaMalloc(&B, sizeof(uint32_t) * (size_t)Kmax * N) != cudaSuccess ||
        cudaMalloc(&D, sizeof(uint32_t) * (size_t)M * N) != cudaSuccess ||
        cudaMalloc(&ws, ws_bytes) != cudaSuccess || cudaMalloc(&err, 64) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        cleanup();
        set_error("gbgpu_autotune: allocation failed");
        return GBGPU_ENOMEM;
    }
    if (cudaMemsetAsync(err, 0, 64, s) != cudaSuccess) {
        cleanup();
        set_error("gbgpu_autotune: status clear failed");
        return GBGPU_ECUDA;
    }
    std::string text = "# gbgpu GEMM tile shapes: limbs kmax shape (0 big, 1 small, 2 mid)\n";
    int table[5][kBuckets];
    for (auto& row : table)
        for (int& x : row) x = -1;
    for (int li = 0; li < 2 && primes[li]; ++li) {
        const uint32_t p = primes[li];
        const int L = limbs_for(p);
        k_uniform<<<1024, 256, 0, s>>>(A, (int64_t)M * Kmax, p, 1);
        k_uniform<<<1024, 256, 0, s>>>(B, (int64_t)Kmax * N, p, 2);
        k_uniform<<<1024, 256, 0, s>>>(D, (int64_t)M * N, p, 3);
        for (int b = 0; b < kBuckets; ++b) {
            const int K = std::min(kKmax[b], Kmax);
            int cands[3], nc = 0;
            for (int sh : {kShapeBig, kShapeSmall, kShapeMid})
                if (valid(L, kKmax[b], sh)) cands[nc++] = sh;
            if (nc < 2) continue;
            float best = 1e30f;
            int best_sh = default_shape(L, K);
            for (int c = 0; c < nc; ++c) {
                TcGemmArgs g{p, M, N, K, A, Kmax, B, N, D, N};
                long long launches = 0;
                float t_min = 1e30f;
                for (int rep = 0; rep < 4; ++rep) {
                    cudaEventRecord(e0, s);
                    rc = tc_submul_shape(g, ws, s, err, &launches, cands[c]);
                    cudaEventRecord(e1, s);
                    if (rc) break;
                    if (cudaEventSynchronize(e1) != cudaSuccess) {
                        rc = GBGPU_ECUDA;
                        break;
                    }
                    float ms = 0;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (rep > 0) t_min = std::min(t_min, ms);  // the first run warms up
                }
                if (rc) {
                    cleanup();
                    return rc;
                }
                if (t_min < best) {
                    best = t_min;
                    best_sh = cands[c];
                }
            }
            table[L][b] = best_sh;
            text += std::to_string(L) + " " + std::to_string(kKmax[b]) + " " +
                    std::to_string(best_sh) + "\n";
        }
    }
    int32_t h_err = 0;
    if (cudaMemcpy(&h_err, err, 4, cudaMemcpyDeviceToHost) != cudaSuccess || h_err) {
        cleanup();
        set_error("gbgpu_autotune: a timed GEMM failed");
        return h_err ? h_err : GBGPU_ECUDA;
    }
    cleanup();
    // write the cache (creating its directory), then use it in this process
    const size_t slash = out.find_last_of('/');
    if (slash != std::string::npos && slash > 0) {
        const std::string dir = out.substr(0, slash);
        for (size_t i = 1; i <= dir.size(); ++i)
            if (i == dir.size() || dir[i] == '/') mkdir(dir.substr(0, i).c_str(), 0755);
    }
    FILE* f = fopen(out.c_str(), "w");
    if (!f) {
        set_error("gbgpu_autotune: cannot write " + out);
        return GBGPU_EINVAL;
    }
    fputs(text.c_str(), f);
    fclose(f);
    std::lock_guard<std::mutex> lock(g_mu);
    for (int L = 0; L < 5; ++L)
        for (int b = 0; b < kBuckets; ++b) g_table[L][b] = table[L][b];
    g_loaded = true;
    return GBGPU_OK;
}
