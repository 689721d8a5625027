// internal.h -- host-side declarations shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "../../include/gbgpu.h"

namespace gbgpu {

struct DeviceInfo {
    int sms;
    int smem_optin;
};

struct Plan;

void set_error(const std::string& s);
void count_launch(long long n);
// Raise the dynamic shared-memory limit of a kernel on the current device to
// at least `bytes`.  The limit only ever grows and is changed under a lock,
// so a launch in one host thread never sees another thread lower it.
cudaError_t ensure_smem_limit(const void* kernel, int bytes);
int device_init(int device, DeviceInfo* info);
// The C-ABI entry points leave the caller's current device as they found it:
// the scope notes it on entry (and makes `device` current when >= 0) and
// restores it on exit.
struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int device = -1) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (device >= 0) cudaSetDevice(device);
    }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
    DeviceScope(const DeviceScope&) = delete;
    DeviceScope& operator=(const DeviceScope&) = delete;
};
// GBGPU_EINVAL with a description of the contract violations in `bits`
// (the error bits of the device-side input checks), GBGPU_OK for none
int err_to_status(uint32_t bits, std::string* msg);

// mode 0: linear_algebra (reduce C|D rows by the known pivots, then reduced
// echelon form of the right block); mode 1: full interreduction of rows with
// distinct leads.
int plan_create(const gbgpu_csr* m, const gbgpu_options* opt, int mode, Plan** out);
int plan_run(Plan* P);
int plan_result(Plan* P, gbgpu_rows* out);
int plan_result_into(Plan* P, int64_t* row_ptr, int32_t* cols, int32_t* vals, int64_t cap_rows,
                     int64_t cap_nnz, int32_t* np, int64_t* nnz);
void plan_destroy(Plan* P);
const gbgpu_stats& plan_stats(const Plan* P);
// waits for a pending small-matrix run and reads its checks and sizes
int settle(Plan* P);
// gb's enlarge_hash_table (src/hash.c:185-240) applied until at least `need`
// entries are free, done as one growth to the final size (boundary.cu)
int grow_hash_table(gbgpu_ht_t* ht, int64_t need);

}  // namespace gbgpu
