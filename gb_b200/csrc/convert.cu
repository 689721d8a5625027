// convert.cu -- the step before the linear algebra on the device: the
// hash -> column mapping of one F4 round (convert_hashes_to_columns,
// src/convert.c:30-135) and the row order (sort_matrix_rows,
// src/order.c:98-131).
//
// Column order (the reference's hcm_cmp, src/order.c:153-235): the lead
// monomials of the known pivots first (hash-data idx 2 before 1), then
//   DRL: higher total degree first, then the smaller exponent of the last
//        variable where two monomials differ;
//   LEX: the larger exponent of the first variable where they differ.
// Monomials of the table are distinct, so this order has no ties and a stable
// LSD radix sort over 64-bit keys -- four exponents of 16 bits per pass, least
// significant group first, the (idx, degree) pass last -- produces exactly it.
// Rows are then ordered by (lead column, length) (sort_matrix_rows); rows that
// tie keep their input order (the reference's qsort leaves ties in an
// unspecified order; any order of tied rows gives the same la answer).
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <sys/time.h>
#include <string>
#include <vector>

#include "../../include/gbgpu.h"
#include "internal.h"

namespace gbgpu {

namespace {

__global__ void k_iota_from(int32_t n, int32_t base, int32_t* out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = base + i;
}

// key of the monomial with hash index h (1-based) for pass `pass`:
// passes 0 .. ng-1 are exponent groups (least significant first), pass ng the
// (idx, degree) key
__global__ void k_col_keys(int32_t n, int32_t nv, const int16_t* __restrict__ exps,
                           const int32_t* __restrict__ deg, const int32_t* __restrict__ idx,
                           int32_t mo, int32_t pass, int32_t ng,
                           const int32_t* __restrict__ hash, uint64_t* key) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int32_t h = hash[i] - 1;
        uint64_t k = 0;
        if (pass == ng) {
            // idx descending, then (DRL) degree descending
            const uint64_t ik = 0xFFFFull - (uint64_t)(uint16_t)idx[h];
            const uint64_t dk = mo == 1 ? 0ull : 0xFFFFFFFFull - (uint64_t)(uint32_t)deg[h];
            k = (ik << 32) | dk;
        } else {
            const int16_t* e = exps + (size_t)h * nv;
            for (int j = 0; j < 4; ++j) {
                uint64_t v;
                int var;
                if (mo == 1) {
                    // LEX: e[0] most significant, descending: group g holds
                    // variables nv-4g-4 .. nv-4g-1, the lower index higher
                    var = nv - 4 * pass - 4 + j;
                    v = var >= 0 ? 0xFFFFull - (uint64_t)(uint16_t)e[var] : 0ull;
                    k |= v << (16 * (3 - j));
                } else {
                    // DRL tie-break: e[nv-1] most significant, ascending: group
                    // g holds variables 4g .. 4g+3, the higher index higher
                    var = 4 * pass + j;
                    v = var < nv ? (uint64_t)(uint16_t)e[var] : 0ull;
                    k |= v << (16 * j);
                }
            }
        }
        key[i] = k;
    }
}

__global__ void k_col_of(int32_t n, const int32_t* __restrict__ hcm, int32_t* col_of) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        col_of[hcm[k]] = k;
}

__global__ void k_count_piv(int32_t n, const int32_t* __restrict__ hcm,
                            const int32_t* __restrict__ idx, int32_t* ncl) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        if (idx[hcm[k] - 1] == 2) atomicAdd(ncl, 1);
}

__global__ void k_row_keys(int32_t nr, const int64_t* __restrict__ row_ptr,
                           const int32_t* __restrict__ hashes, const int32_t* __restrict__ col_of,
                           uint64_t* key, int64_t* len) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nr; i += gridDim.x * blockDim.x) {
        const int64_t b = row_ptr[i], e = row_ptr[i + 1];
        const uint64_t lead = e > b ? (uint64_t)(uint32_t)col_of[hashes[b]] : 0xFFFFFFFFull;
        key[i] = (lead << 32) | (uint64_t)(uint32_t)(e - b);
        len[i] = e - b;
    }
}

__global__ void k_lens_in_order(int32_t nr, const int32_t* __restrict__ order,
                                const int64_t* __restrict__ len, int64_t* out) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nr; k += gridDim.x * blockDim.x)
        out[k] = len[order[k]];
    if (blockIdx.x == 0 && threadIdx.x == 0) out[nr] = 0;
}

// output row k = input row order[k] with its hashes mapped to columns (a warp per row)
__global__ void k_gather_mapped(int32_t nr, const int32_t* __restrict__ order,
                                const int64_t* __restrict__ row_ptr,
                                const int32_t* __restrict__ hashes,
                                const int32_t* __restrict__ col_of,
                                const int64_t* __restrict__ out_ptr, int32_t* out_cols) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int k = warp; k < nr; k += nwarps) {
        const int32_t r = order[k];
        const int64_t b = row_ptr[r], e = row_ptr[r + 1], o = out_ptr[k];
        for (int64_t j = b + lane; j < e; j += 32) out_cols[o + (j - b)] = col_of[hashes[j]];
    }
}

int grid_of(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)); }

}  // namespace

int convert_flat(int32_t nv, int32_t n, const int16_t* exps, const int32_t* deg,
                 const int32_t* idx, int32_t mo, int32_t nr, const int64_t* row_ptr,
                 const int32_t* hashes, int32_t* hcm, int32_t* ncl, int32_t* row_order,
                 int64_t* out_row_ptr, int32_t* out_cols, int device) {
    if (nv < 1 || nv > 4096 || n < 0 || nr < 0 || (mo != 0 && mo != 1) ||
        (n > 0 && (!exps || !deg || !idx || !hcm)) ||
        (nr > 0 && (!row_ptr || !hashes || !row_order || !out_row_ptr || !out_cols)) || !ncl) {
        set_error("gbgpu_convert_hashes_to_columns_flat: bad arguments");
        return GBGPU_EINVAL;
    }
    const int64_t nnz = nr > 0 ? row_ptr[nr] : 0;
    for (int64_t j = 0; j < nnz; ++j)
        if (hashes[j] < 1 || hashes[j] > n) {
            set_error("gbgpu_convert_hashes_to_columns_flat: hash index outside 1..n");
            return GBGPU_EINVAL;
        }
    DeviceInfo dev;
    int rc = device_init(device, &dev);
    if (rc) return rc;
    cudaStream_t s = nullptr;
    std::vector<void*> bufs;
    auto alloc = [&](size_t bytes) -> void* {
        void* q = nullptr;
        if (cudaMallocAsync(&q, std::max<size_t>(bytes, 16), s) != cudaSuccess) q = nullptr;
        bufs.push_back(q);  // a failed allocation is recorded as nullptr
        return q;
    };
    auto done = [&](int code) {
        for (void* q : bufs)
            if (q) cudaFreeAsync(q, s);
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
        return code;
    };
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("stream creation failed");
        return GBGPU_ECUDA;
    }
    int16_t* d_exps = (int16_t*)alloc(sizeof(int16_t) * (size_t)n * nv);
    int32_t* d_deg = (int32_t*)alloc(4 * (size_t)n);
    int32_t* d_idx = (int32_t*)alloc(4 * (size_t)n);
    int32_t* d_ha = (int32_t*)alloc(4 * (size_t)n);
    int32_t* d_hb = (int32_t*)alloc(4 * (size_t)n);
    uint64_t* d_ka = (uint64_t*)alloc(8 * (size_t)std::max(n, nr));
    uint64_t* d_kb = (uint64_t*)alloc(8 * (size_t)std::max(n, nr));
    int32_t* d_colof = (int32_t*)alloc(4 * (size_t)(n + 1));
    int32_t* d_ncl = (int32_t*)alloc(4);
    int64_t* d_rp = (int64_t*)alloc(8 * (size_t)(nr + 1));
    int32_t* d_hashes = (int32_t*)alloc(4 * (size_t)nnz);
    int64_t* d_len = (int64_t*)alloc(8 * (size_t)(nr + 1));
    int64_t* d_lord = (int64_t*)alloc(8 * (size_t)(nr + 1));
    int64_t* d_optr = (int64_t*)alloc(8 * (size_t)(nr + 1));
    int32_t* d_ra = (int32_t*)alloc(4 * (size_t)std::max(nr, 1));
    int32_t* d_rb = (int32_t*)alloc(4 * (size_t)std::max(nr, 1));
    int32_t* d_ocols = (int32_t*)alloc(4 * (size_t)nnz);
    size_t sort_bytes = 0, sort2 = 0, scan_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, d_ka, d_kb, d_ha, d_hb, std::max(n, 1), 0,
                                    64, s);
    cub::DeviceRadixSort::SortPairs(nullptr, sort2, d_ka, d_kb, d_ra, d_rb, std::max(nr, 1), 0, 64,
                                    s);
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, d_lord, d_optr, nr + 1, s);
    void* d_tmp = alloc(std::max(sort_bytes, std::max(sort2, scan_bytes)));
    for (void* q : bufs)
        if (!q) {
            set_error("convert: device allocation failed");
            return done(GBGPU_ENOMEM);
        }
    const size_t tmp_bytes = std::max(sort_bytes, std::max(sort2, scan_bytes));
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t x) {
        if (e == cudaSuccess) e = x;
        return e == cudaSuccess;
    };
    long long launches = 0;
    if (n > 0) {
        ok(cudaMemcpyAsync(d_exps, exps, sizeof(int16_t) * (size_t)n * nv, cudaMemcpyHostToDevice, s));
        ok(cudaMemcpyAsync(d_deg, deg, 4 * (size_t)n, cudaMemcpyHostToDevice, s));
        ok(cudaMemcpyAsync(d_idx, idx, 4 * (size_t)n, cudaMemcpyHostToDevice, s));
        k_iota_from<<<grid_of(n), 256, 0, s>>>(n, 1, d_ha);
        ++launches;
        // LSD: exponent groups (least significant first), then (idx, degree)
        const int ng = (nv + 3) / 4;
        for (int pass = 0; pass <= ng && e == cudaSuccess; ++pass) {
            k_col_keys<<<grid_of(n), 256, 0, s>>>(n, nv, d_exps, d_deg, d_idx, mo, pass, ng, d_ha,
                                                  d_ka);
            size_t b = tmp_bytes;
            ok(cub::DeviceRadixSort::SortPairs(d_tmp, b, d_ka, d_kb, d_ha, d_hb, n, 0, 64, s));
            std::swap(d_ha, d_hb);
            launches += 2;
        }
        ok(cudaMemsetAsync(d_ncl, 0, 4, s));
        k_col_of<<<grid_of(n), 256, 0, s>>>(n, d_ha, d_colof);
        k_count_piv<<<grid_of(n), 256, 0, s>>>(n, d_ha, d_idx, d_ncl);
        launches += 2;
    } else {
        ok(cudaMemsetAsync(d_ncl, 0, 4, s));
    }
    if (nr > 0) {
        ok(cudaMemcpyAsync(d_rp, row_ptr, 8 * (size_t)(nr + 1), cudaMemcpyHostToDevice, s));
        if (nnz > 0) ok(cudaMemcpyAsync(d_hashes, hashes, 4 * (size_t)nnz, cudaMemcpyHostToDevice, s));
        k_row_keys<<<grid_of(nr), 256, 0, s>>>(nr, d_rp, d_hashes, d_colof, d_ka, d_len);
        k_iota_from<<<grid_of(nr), 256, 0, s>>>(nr, 0, d_ra);
        size_t b = tmp_bytes;
        ok(cub::DeviceRadixSort::SortPairs(d_tmp, b, d_ka, d_kb, d_ra, d_rb, nr, 0, 64, s));
        k_lens_in_order<<<grid_of(nr), 256, 0, s>>>(nr, d_rb, d_len, d_lord);
        b = tmp_bytes;
        ok(cub::DeviceScan::ExclusiveSum(d_tmp, b, d_lord, d_optr, nr + 1, s));
        k_gather_mapped<<<grid_of((int64_t)nr * 32), 256, 0, s>>>(nr, d_rb, d_rp, d_hashes, d_colof,
                                                                 d_optr, d_ocols);
        launches += 5;
        ok(cudaMemcpyAsync(row_order, d_rb, 4 * (size_t)nr, cudaMemcpyDeviceToHost, s));
        ok(cudaMemcpyAsync(out_row_ptr, d_optr, 8 * (size_t)(nr + 1), cudaMemcpyDeviceToHost, s));
        if (nnz > 0) ok(cudaMemcpyAsync(out_cols, d_ocols, 4 * (size_t)nnz, cudaMemcpyDeviceToHost, s));
    }
    if (n > 0) ok(cudaMemcpyAsync(hcm, d_ha, 4 * (size_t)n, cudaMemcpyDeviceToHost, s));
    ok(cudaMemcpyAsync(ncl, d_ncl, 4, cudaMemcpyDeviceToHost, s));
    ok(cudaGetLastError());
    ok(cudaStreamSynchronize(s));
    count_launch(launches);
    if (e != cudaSuccess) {
        set_error(std::string("convert: ") + cudaGetErrorString(e));
        return done(GBGPU_ECUDA);
    }
    return done(GBGPU_OK);
}

// stable sort of nr 64-bit keys on the device: order[k] = index of the k-th key
int sort_row_keys(int32_t nr, const uint64_t* keys, int32_t* order, int device) {
    DeviceInfo dev;
    int rc = device_init(device, &dev);
    if (rc) return rc;
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("stream creation failed");
        return GBGPU_ECUDA;
    }
    uint64_t *ka = nullptr, *kb = nullptr;
    int32_t *ra = nullptr, *rb = nullptr;
    void* tmp = nullptr;
    size_t bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, bytes, ka, kb, ra, rb, nr, 0, 64, s);
    cudaError_t e = cudaMallocAsync((void**)&ka, 8 * (size_t)nr, s);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&kb, 8 * (size_t)nr, s);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&ra, 4 * (size_t)nr, s);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&rb, 4 * (size_t)nr, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&tmp, std::max<size_t>(bytes, 16), s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ka, keys, 8 * (size_t)nr, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        k_iota_from<<<grid_of(nr), 256, 0, s>>>(nr, 0, ra);
        e = cub::DeviceRadixSort::SortPairs(tmp, bytes, ka, kb, ra, rb, nr, 0, 64, s);
        count_launch(2);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(order, rb, 4 * (size_t)nr, cudaMemcpyDeviceToHost, s);
    for (void* q : {(void*)ka, (void*)kb, (void*)ra, (void*)rb, tmp})
        if (q) cudaFreeAsync(q, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    else cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (e != cudaSuccess) {
        set_error(std::string("row sort: ") + cudaGetErrorString(e));
        return GBGPU_ECUDA;
    }
    return GBGPU_OK;
}

}  // namespace gbgpu

using namespace gbgpu;

extern "C" int gbgpu_convert_hashes_to_columns_flat(
    int32_t nv, int32_t n, const int16_t* exps, const int32_t* deg, const int32_t* idx,
    int32_t mo, int32_t nr, const int64_t* row_ptr, const int32_t* hashes, int32_t* hcm,
    int32_t* ncl, int32_t* row_order, int64_t* out_row_ptr, int32_t* out_cols, int32_t device) {
    int prev = -1;
    cudaGetDevice(&prev);
    const int rc = convert_flat(nv, n, exps, deg, idx, mo, nr, row_ptr, hashes, hcm, ncl,
                                row_order, out_row_ptr, out_cols, device);
    if (prev >= 0) cudaSetDevice(prev);
    return rc;
}

namespace {

double now_cpu() { return (double)clock() / CLOCKS_PER_SEC; }
double now_wall() {
    struct timeval t;
    gettimeofday(&t, nullptr);
    return (double)t.tv_sec + 1e-6 * (double)t.tv_usec;
}

int device_of_env() {
    const char* d = getenv("GBGPU_DEVICE");
    return d ? atoi(d) : 0;
}

}  // namespace

extern "C" {

int gbgpu_convert_hashes_to_columns_status(int32_t** hcmp, gbgpu_mat_t* mat, gbgpu_stat_t* st,
                                           gbgpu_ht_t* sht) {
    if (!hcmp || !mat || !st || !sht) return GBGPU_EINVAL;
    const double ct0 = now_cpu(), rt0 = now_wall();
    const int32_t n = sht->eld - 1, nv = sht->nv, nr = mat->nr;
    std::vector<int16_t> exps((size_t)std::max(n, 1) * std::max(nv, 1));
    std::vector<int32_t> deg((size_t)std::max(n, 1)), idx((size_t)std::max(n, 1));
    for (int32_t i = 0; i < n; ++i) {
        memcpy(&exps[(size_t)i * nv], sht->ev[i + 1], sizeof(int16_t) * (size_t)nv);
        deg[i] = sht->hd[i + 1].deg;
        idx[i] = sht->hd[i + 1].idx;
    }
    std::vector<int64_t> ptr((size_t)nr + 1, 0);
    for (int32_t i = 0; i < nr; ++i) ptr[i + 1] = ptr[i] + mat->r[i][2];
    std::vector<int32_t> hashes((size_t)std::max<int64_t>(ptr[nr], 1));
    for (int32_t i = 0; i < nr; ++i)
        memcpy(&hashes[ptr[i]], mat->r[i] + 3, sizeof(int32_t) * (size_t)mat->r[i][2]);
    int32_t* hcm = (int32_t*)realloc(*hcmp, sizeof(int32_t) * (size_t)std::max(n, 1));
    if (!hcm) return GBGPU_ENOMEM;
    *hcmp = hcm;
    std::vector<int32_t> order((size_t)std::max(nr, 1)), cols(hashes.size());
    std::vector<int64_t> optr((size_t)nr + 1);
    int32_t ncl = 0;
    int rc = gbgpu_convert_hashes_to_columns_flat(nv, n, exps.data(), deg.data(), idx.data(),
                                                  st->mo == 1 ? 1 : 0, nr, ptr.data(),
                                                  hashes.data(), hcm, &ncl, order.data(),
                                                  optr.data(), cols.data(), device_of_env());
    if (rc) return rc;
    // hash -> column, as the reference stores it (src/convert.c:83-85)
    for (int32_t k = 0; k < n; ++k) sht->hd[hcm[k]].idx = k;
    // every row's entries as columns, rows in the sorted order
    std::vector<gbgpu_hm_t*> rows((size_t)std::max(nr, 1));
    for (int32_t k = 0; k < nr; ++k) {
        gbgpu_hm_t* r = mat->r[order[k]];
        memcpy(r + 3, &cols[optr[k]], sizeof(int32_t) * (size_t)r[2]);
        rows[k] = r;
    }
    for (int32_t k = 0; k < nr; ++k) mat->r[k] = rows[k];
    mat->nru = mat->ncl = ncl;
    mat->nrl = mat->nr - mat->nru;
    mat->ncr = n - ncl;
    st->num_rowsred += mat->nrl;
    st->convert_ctime += now_cpu() - ct0;
    st->convert_rtime += now_wall() - rt0;
    if (st->info_level > 1) {
        int64_t nterms = ptr[nr];
        const double density = nr > 0 && mat->nc > 0
                                   ? (double)nterms * 100.0 / (double)nr / (double)mat->nc
                                   : 0.0;
        printf(" %7d x %-7d %8.3f%%", mat->nr, mat->nc, density);
        fflush(stdout);
    }
    return GBGPU_OK;
}

void gbgpu_convert_hashes_to_columns(int32_t** hcmp, gbgpu_mat_t* mat, gbgpu_stat_t* st,
                                     gbgpu_ht_t* sht) {
    const int rc = gbgpu_convert_hashes_to_columns_status(hcmp, mat, st, sht);
    if (rc) {
        fprintf(stderr, "gbgpu_convert_hashes_to_columns failed (%d): %s\n", rc,
                gbgpu_last_error());
        exit(1);
    }
}

int gbgpu_sort_matrix_rows_status(gbgpu_mat_t* mat) {
    DeviceScope scope;
    if (!mat) return GBGPU_EINVAL;
    const int32_t nr = mat->nr;
    if (nr <= 1) return GBGPU_OK;
    // key = (lead column, length), sorted stably on the device
    std::vector<uint64_t> key((size_t)nr);
    for (int32_t i = 0; i < nr; ++i)
        key[i] = ((uint64_t)(uint32_t)mat->r[i][3] << 32) | (uint64_t)(uint32_t)mat->r[i][2];
    std::vector<int32_t> order((size_t)nr);
    int rc = sort_row_keys(nr, key.data(), order.data(), device_of_env());
    if (rc) return rc;
    std::vector<gbgpu_hm_t*> rows((size_t)nr);
    for (int32_t k = 0; k < nr; ++k) rows[k] = mat->r[order[k]];
    for (int32_t k = 0; k < nr; ++k) mat->r[k] = rows[k];
    return GBGPU_OK;
}

void gbgpu_sort_matrix_rows(gbgpu_mat_t* mat) {
    const int rc = gbgpu_sort_matrix_rows_status(mat);
    if (rc) {
        fprintf(stderr, "gbgpu_sort_matrix_rows failed (%d): %s\n", rc, gbgpu_last_error());
        exit(1);
    }
}

}  // extern "C"
