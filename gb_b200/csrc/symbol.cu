// symbol.cu -- gb's symbolic preprocessing (src/symbol.c:202-272) with the
// reducer search on the device.
//
// Symbolic preprocessing walks the monomials of the round's secondary hash
// table in index order (new ones are appended while it walks) and, for every
// monomial not yet marked, looks for a reducer: the first basis element in
// the lead-monomial list (bs->lmps[0 .. bs->lml)) whose lead monomial divides
// it (short divisor mask, degree, exponents; find_multiplied_reducer,
// src/symbol.c:150-200).  A reducer, multiplied by the quotient, becomes a
// row of the matrix and its terms are inserted into the table
// (multiplied_poly_to_matrix_row, src/hash.c:903-925 and :672-746).
//
// The reducer of a monomial depends only on the monomial and the basis, so
// the device finds the reducers of a whole wave of monomials at once (a warp
// per monomial, 32 basis leads per step, the first match by ballot); the host
// then walks the wave in index order exactly as the reference does (marks,
// column count, rows, insertions), so the table gets the reference's indices
// and the matrix the reference's rows.  Monomials appended by a wave form the
// next wave.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <sys/time.h>
#include <vector>

#include "../../include/gbgpu.h"
#include "internal.h"

namespace gbgpu {

// red[q] = the first i < lml whose lead divides monomial q, -1 for none
// (lead i: exponents lexp[i nv ..], short divisor mask lsdm[i], degree
// ldeg[i]; monomial q: mexp[q nv ..], msdm[q], mdeg[q]); a warp per monomial
__global__ void k_find_reducers(int32_t n, int32_t nv, const int16_t* __restrict__ mexp,
                                const int32_t* __restrict__ msdm,
                                const int32_t* __restrict__ mdeg, int32_t lml,
                                const int16_t* __restrict__ lexp,
                                const int32_t* __restrict__ lsdm,
                                const int32_t* __restrict__ ldeg, int32_t* red) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int q = warp; q < n; q += nwarps) {
        const int16_t* e = mexp + (size_t)q * nv;
        const int32_t ns = ~msdm[q], dq = mdeg[q];
        int found = -1;
        for (int base = 0; base < lml && found < 0; base += 32) {
            const int i = base + lane;
            bool ok = i < lml && (lsdm[i] & ns) == 0 && ldeg[i] <= dq;
            if (ok) {
                const int16_t* f = lexp + (size_t)i * nv;
                for (int k = 0; k < nv; ++k)
                    if (e[k] < f[k]) {
                        ok = false;
                        break;
                    }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, ok);
            if (bal) found = base + __ffs(bal) - 1;
        }
        if (lane == 0) red[q] = found;
    }
}

}  // namespace gbgpu

using namespace gbgpu;

namespace {

double cpu_now() { return (double)clock() / CLOCKS_PER_SEC; }
double wall_now() {
    struct timeval t;
    gettimeofday(&t, nullptr);
    return (double)t.tv_sec + 1e-6 * (double)t.tv_usec;
}

// the device buffers of the calling thread, grown to a high-water mark
struct SymbolScratch {
    int device = -1;
    cudaStream_t s = nullptr;
    int16_t* lexp = nullptr;
    int32_t* lsdm = nullptr;
    int32_t* ldeg = nullptr;
    size_t lcap = 0, lecap = 0;  // leads; their exponent entries (leads x variables)
    int16_t* mexp = nullptr;
    int32_t* msdm = nullptr;
    int32_t* mdeg = nullptr;
    int32_t* red = nullptr;
    size_t mcap = 0, mecap = 0;  // monomials; their exponent entries
};
thread_local SymbolScratch g_sym;

template <class T>
int grow_device(T** p, size_t count) {
    if (*p) cudaFree(*p);
    *p = nullptr;
    if (cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(count, 1)) != cudaSuccess) {
        set_error("symbolic preprocessing: device allocation failed");
        return GBGPU_ENOMEM;
    }
    return GBGPU_OK;
}

// generate_short_divmask (src/hash.c:244-265)
int32_t short_divmask(const int16_t* a, const gbgpu_ht_t* ht) {
    int32_t res = 0, ctr = 0;
    for (int32_t i = 0; i < ht->ndv; ++i)
        for (int32_t j = 0; j < ht->bpv; ++j) {
            if ((int32_t)a[i] >= ht->dm[ctr]) res |= (int32_t)(1u << ctr);
            ++ctr;
        }
    return res;
}

}  // namespace

namespace {

// multiplied_poly_to_matrix_row (src/hash.c:903-925): the matrix row of the
// basis element `poly` times the monomial with exponents em, degree deg and
// hash value hm; every term is found in or inserted into the secondary table
// as insert_multiplied_poly_in_hash_table does (src/hash.c:672-746)
int multiplied_row(gbgpu_ht_t* sht, const gbgpu_ht_t* bht, uint32_t hm, int32_t deg,
                   const int16_t* em, const gbgpu_hm_t* poly, gbgpu_hm_t** out) {
    const int32_t len = poly[2];
    gbgpu_hm_t* row = (gbgpu_hm_t*)malloc(sizeof(gbgpu_hm_t) * (size_t)(len + 3));
    if (!row) return GBGPU_ENOMEM;
    row[0] = poly[0];
    row[1] = poly[1];
    row[2] = poly[2];
    // enlarge_hash_table while sht->eld + len >= sht->esz
    if (int rc = grow_hash_table(sht, (int64_t)len + 1)) {
        free(row);
        return rc;
    }
    const int32_t nv = sht->nv;
    const uint32_t mask = (uint32_t)sht->hsz - 1u;
    for (int32_t l = 3; l < len + 3; ++l) {
        const int32_t t = poly[l];
        const int32_t h = (int32_t)(hm + (uint32_t)bht->hd[t].val);
        const int16_t* eb = bht->ev[t];
        int16_t* n = sht->ev[sht->eld];
        for (int32_t j = 0; j < nv; ++j) n[j] = (int16_t)(em[j] + eb[j]);
        uint32_t k = (uint32_t)h;
        int32_t found = 0;
        for (int32_t i = 0; i < sht->hsz; ++i) {
            k = (k + (uint32_t)i) & mask;
            const int32_t hmk = sht->hmap[k];
            if (!hmk) break;
            if (sht->hd[hmk].val != h) continue;
            if (memcmp(sht->ev[hmk], n, sizeof(int16_t) * (size_t)nv) == 0) {
                found = hmk;
                break;
            }
        }
        if (found) {
            row[l] = found;
            continue;
        }
        const int32_t pos = sht->eld;
        sht->hmap[k] = pos;
        sht->hd[pos].deg = deg + bht->hd[t].deg;
        sht->hd[pos].sdm = short_divmask(n, sht);
        sht->hd[pos].val = h;
        sht->eld = pos + 1;
        row[l] = pos;
    }
    *out = row;
    return GBGPU_OK;
}

}  // namespace

extern "C" {

int gbgpu_symbolic_preprocessing_status(gbgpu_mat_t* mat, const gbgpu_bs_t* bs, gbgpu_stat_t* st,
                                        gbgpu_ht_t* sht, const gbgpu_ht_t* bht) {
    if (!mat || !bs || !st || !sht || !bht) return GBGPU_EINVAL;
    if (sht->nv != bht->nv || sht->hsz <= 0 || (sht->hsz & (sht->hsz - 1)) != 0) {
        set_error("symbolic preprocessing: tables of different variables or a map size that "
                  "is not a power of two");
        return GBGPU_EINVAL;
    }
    const char* dev = getenv("GBGPU_DEVICE");
    DeviceScope scope(dev ? atoi(dev) : 0);
    const double ct0 = cpu_now(), rt0 = wall_now();
    SymbolScratch& g = g_sym;
    int cur = 0;
    cudaGetDevice(&cur);
    if (g.device != cur) {
        g = SymbolScratch{};  // another device: start over (buffers of the old one are kept)
        g.device = cur;
    }
    if (!g.s && cudaStreamCreateWithFlags(&g.s, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("symbolic preprocessing: stream creation failed");
        return GBGPU_ECUDA;
    }
    const int32_t nv = bht->nv, lml = bs->lml;
    int rc;
    // the basis leads, in the order of the lead-monomial list
    // capacities in entries: the variable count differs from one system to the next
    // (a capacity is cleared before its buffers are replaced, so that a failed
    // allocation leaves nothing that a later call would take for a buffer)
    if ((size_t)lml > g.lcap) {
        const size_t cap = std::max<size_t>((size_t)lml, 2 * g.lcap);
        g.lcap = 0;
        if ((rc = grow_device(&g.lsdm, cap)) || (rc = grow_device(&g.ldeg, cap))) return rc;
        g.lcap = cap;
    }
    if ((size_t)lml * nv > g.lecap) {
        const size_t cap = std::max<size_t>((size_t)lml * nv, 2 * g.lecap);
        g.lecap = 0;
        if ((rc = grow_device(&g.lexp, cap))) return rc;
        g.lecap = cap;
    }
    {
        std::vector<int16_t> le((size_t)std::max(lml, 1) * nv);
        std::vector<int32_t> ls((size_t)std::max(lml, 1)), ldg((size_t)std::max(lml, 1));
        for (int32_t i = 0; i < lml; ++i) {
            const int32_t lead = bs->hm[bs->lmps[i]][3];
            memcpy(&le[(size_t)i * nv], bht->ev[lead], sizeof(int16_t) * nv);
            ls[i] = bs->lm[i];
            ldg[i] = bht->hd[lead].deg;
        }
        if (lml > 0 &&
            (cudaMemcpyAsync(g.lexp, le.data(), sizeof(int16_t) * (size_t)lml * nv,
                             cudaMemcpyHostToDevice, g.s) != cudaSuccess ||
             cudaMemcpyAsync(g.lsdm, ls.data(), sizeof(int32_t) * lml, cudaMemcpyHostToDevice,
                             g.s) != cudaSuccess ||
             cudaMemcpyAsync(g.ldeg, ldg.data(), sizeof(int32_t) * lml, cudaMemcpyHostToDevice,
                             g.s) != cudaSuccess ||
             cudaStreamSynchronize(g.s) != cudaSuccess)) {
            set_error("symbolic preprocessing: copy of the basis leads failed");
            return GBGPU_ECUDA;
        }
    }
    // the reducers of monomials [a, b) of the secondary table, on the device
    std::vector<int32_t> red;
    auto reducers = [&](int32_t a, int32_t b) -> int {
        const int32_t n = b - a;
        red.assign((size_t)std::max(n, 1), -1);
        if (n <= 0 || lml <= 0) return GBGPU_OK;
        int r;
        if ((size_t)n > g.mcap) {
            const size_t cap = std::max<size_t>((size_t)n, 2 * g.mcap);
            g.mcap = 0;
            if ((r = grow_device(&g.msdm, cap)) || (r = grow_device(&g.mdeg, cap)) ||
                (r = grow_device(&g.red, cap)))
                return r;
            g.mcap = cap;
        }
        if ((size_t)n * nv > g.mecap) {
            const size_t cap = std::max<size_t>((size_t)n * nv, 2 * g.mecap);
            g.mecap = 0;
            if ((r = grow_device(&g.mexp, cap))) return r;
            g.mecap = cap;
        }
        std::vector<int16_t> me((size_t)n * nv);
        std::vector<int32_t> ms((size_t)n), md((size_t)n);
        for (int32_t q = 0; q < n; ++q) {
            memcpy(&me[(size_t)q * nv], sht->ev[a + q], sizeof(int16_t) * nv);
            ms[q] = sht->hd[a + q].sdm;
            md[q] = sht->hd[a + q].deg;
        }
        cudaMemcpyAsync(g.mexp, me.data(), sizeof(int16_t) * (size_t)n * nv,
                        cudaMemcpyHostToDevice, g.s);
        cudaMemcpyAsync(g.msdm, ms.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, g.s);
        cudaMemcpyAsync(g.mdeg, md.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, g.s);
        const int threads = 256;
        const int blocks = (int)std::min<int64_t>(((int64_t)n * 32 + threads - 1) / threads, 148 * 16);
        k_find_reducers<<<blocks, threads, 0, g.s>>>(n, nv, g.mexp, g.msdm, g.mdeg, lml, g.lexp,
                                                     g.lsdm, g.ldeg, g.red);
        count_launch(1);
        cudaMemcpyAsync(red.data(), g.red, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, g.s);
        if (cudaStreamSynchronize(g.s) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
            set_error("symbolic preprocessing: reducer search failed on the device");
            return GBGPU_ECUDA;
        }
        return GBGPU_OK;
    };
    std::vector<int16_t> etmp((size_t)nv);
    // one monomial in the walk of src/symbol.c:226-258: marked as a column,
    // and its reducer (found on the device) becomes a row
    auto visit = [&](int32_t i, int32_t r) -> int {
        sht->hd[i].idx = 1;
        mat->nc++;
        if (r < 0) return GBGPU_OK;
        const gbgpu_hm_t* b = bs->hm[bs->lmps[r]];
        const int32_t lead = b[3];
        const int32_t d = sht->hd[i].deg - bht->hd[lead].deg;
        const int16_t* e = sht->ev[i];
        const int16_t* f = bht->ev[lead];
        for (int32_t k = 0; k < nv; ++k) etmp[k] = (int16_t)(e[k] - f[k]);
        const uint32_t h = (uint32_t)sht->hd[i].val - (uint32_t)bht->hd[lead].val;
        gbgpu_hm_t* row = nullptr;
        if (int rc2 = multiplied_row(sht, bht, h, d, etmp.data(), b, &row)) return rc2;
        sht->hd[i].idx = 2;
        mat->r[mat->nr++] = row;
        return GBGPU_OK;
    };
    const int32_t oesld = sht->eld;
    if (mat->sz <= 0) mat->sz = 1;
    while (mat->sz <= mat->nr + oesld) mat->sz *= 2;
    gbgpu_hm_t** nr_ = (gbgpu_hm_t**)realloc(mat->r, sizeof(gbgpu_hm_t*) * (size_t)mat->sz);
    if (!nr_) return GBGPU_ENOMEM;
    mat->r = nr_;
    // the monomials present when the walk starts: only those not marked yet
    if ((rc = reducers(1, oesld))) return rc;
    for (int32_t i = 1; i < oesld; ++i) {
        if (sht->hd[i].idx) continue;
        if ((rc = visit(i, red[i - 1]))) return rc;
    }
    // the monomials the rows brought in, wave by wave
    for (int32_t a = oesld; a < sht->eld;) {
        const int32_t b = sht->eld;
        if ((rc = reducers(a, b))) return rc;
        for (int32_t i = a; i < b; ++i) {
            if (mat->sz == mat->nr) {
                mat->sz *= 2;
                nr_ = (gbgpu_hm_t**)realloc(mat->r, sizeof(gbgpu_hm_t*) * (size_t)mat->sz);
                if (!nr_) return GBGPU_ENOMEM;
                mat->r = nr_;
            }
            if ((rc = visit(i, red[i - a]))) return rc;
        }
        a = b;
    }
    nr_ = (gbgpu_hm_t**)realloc(mat->r, sizeof(gbgpu_hm_t*) * (size_t)std::max(mat->nr, 1));
    if (!nr_) return GBGPU_ENOMEM;
    mat->r = nr_;
    mat->sz = mat->nr;
    st->max_sht_size = st->max_sht_size > sht->hsz ? st->max_sht_size : sht->hsz;
    st->symbol_ctime += cpu_now() - ct0;
    st->symbol_rtime += wall_now() - rt0;
    return GBGPU_OK;
}

void gbgpu_symbolic_preprocessing(gbgpu_mat_t* mat, const gbgpu_bs_t* bs, gbgpu_stat_t* st,
                                  gbgpu_ht_t* sht, const gbgpu_ht_t* bht) {
    const int rc = gbgpu_symbolic_preprocessing_status(mat, bs, st, sht, bht);
    if (rc) {
        fprintf(stderr, "gbgpu_symbolic_preprocessing failed (%d): %s\n", rc, gbgpu_last_error());
        exit(1);
    }
}

}  // extern "C"
