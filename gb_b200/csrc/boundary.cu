// boundary.cu -- the drop-in replacements for gb's linear-algebra function
// pointers (src/data.h:269-279) over the mirrored mat_t / bs_t / stat_t, and
// the batched flat entry point.
//
// Ownership follows the reference exactly (src/la_ff_16.c:601-735,
// :737-835, :1322-1392, :1605-1673): input rows are freed by the callee,
// bs coefficient arrays are only read (interreduction frees the basis
// elements like free_basis_elements, src/basis.c:25-57), output rows and
// coefficient arrays are malloc'ed host blocks the basis later adopts and
// frees (src/convert.c:137-280).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <sys/time.h>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/gbgpu.h"
#include "internal.h"
#include "small.h"

using namespace gbgpu;

namespace {

double cpu_seconds() { return (double)clock() / CLOCKS_PER_SEC; }
double wall_seconds() {
    struct timeval t;
    gettimeofday(&t, nullptr);
    return (double)t.tv_sec + 1e-6 * (double)t.tv_usec;
}

// ff_bits as src/io.c:815-828 selects it; the stat_t field is used when set
int coef_bits(const gbgpu_stat_t* st) {
    if (st->ff_bits == 8 || st->ff_bits == 16 || st->ff_bits == 32) return st->ff_bits;
    if (st->fc < 128) return 8;
    if (st->fc < 32768) return 16;
    return 32;
}

int32_t load_cf(const void* const* tab, int bits, int32_t idx, int64_t j) {
    if (bits == 8) return (int32_t)((const int8_t* const*)tab)[idx][j];
    if (bits == 16) return (int32_t)((const int16_t* const*)tab)[idx][j];
    return ((const int32_t* const*)tab)[idx][j];
}

const void* const* bs_table(const gbgpu_bs_t* bs, int bits) {
    if (bits == 8) return (const void* const*)bs->cf_8;
    if (bits == 16) return (const void* const*)bs->cf_16;
    return (const void* const*)bs->cf_32;
}

// mat->r rows -> flat CSR (coefficients from `tab`, reduced into [0, p))
void gather_rows(gbgpu_hm_t* const* rows, int32_t nr, const void* const* tab, int bits,
                 int32_t p, std::vector<int64_t>& ptr, std::vector<int32_t>& cols,
                 std::vector<int32_t>& vals) {
    ptr.assign((size_t)nr + 1, 0);
    for (int32_t i = 0; i < nr; ++i) ptr[i + 1] = ptr[i] + rows[i][2];
    cols.resize((size_t)std::max<int64_t>(ptr[nr], 1));
    vals.resize((size_t)std::max<int64_t>(ptr[nr], 1));
    for (int32_t i = 0; i < nr; ++i) {
        const gbgpu_hm_t* r = rows[i];
        const int64_t off = ptr[i];
        memcpy(&cols[off], r + 3, sizeof(int32_t) * (size_t)r[2]);
        for (int64_t j = 0; j < r[2]; ++j) {
            int32_t v = load_cf(tab, bits, r[0], j) % p;
            vals[off + j] = v < 0 ? v + p : v;
        }
    }
}

// CSR answer -> malloc'ed reference rows and coefficient arrays
int store_rows_raw(gbgpu_mat_t* mat, int bits, int32_t np, const int64_t* row_ptr,
                   const int32_t* ocols, const int32_t* ovals) {
    const gbgpu_rows out{np, np > 0 ? row_ptr[np] : 0, const_cast<int64_t*>(row_ptr),
                         const_cast<int32_t*>(ocols), const_cast<int32_t*>(ovals)};
    gbgpu_hm_t** r = (gbgpu_hm_t**)malloc(sizeof(gbgpu_hm_t*) * (size_t)std::max(np, 1));
    void** cf = (void**)malloc(sizeof(void*) * (size_t)std::max(np, 1));
    if (!r || !cf) return GBGPU_ENOMEM;
    const size_t esz = bits == 8 ? 1 : bits == 16 ? 2 : 4;
    for (int32_t l = 0; l < np; ++l) {
        const int64_t b = out.row_ptr[l], len = out.row_ptr[l + 1] - b;
        gbgpu_hm_t* row = (gbgpu_hm_t*)malloc(sizeof(gbgpu_hm_t) * (size_t)(len + 3));
        void* c = malloc(esz * (size_t)std::max<int64_t>(len, 1));
        if (!row || !c) return GBGPU_ENOMEM;
        row[0] = l;
        row[1] = (gbgpu_hm_t)(len % 4);
        row[2] = (gbgpu_hm_t)len;
        memcpy(row + 3, out.cols + b, sizeof(int32_t) * (size_t)len);
        for (int64_t j = 0; j < len; ++j) {
            const int32_t v = out.vals[b + j];
            if (bits == 8) ((int8_t*)c)[j] = (int8_t)v;
            else if (bits == 16) ((int16_t*)c)[j] = (int16_t)v;
            else ((int32_t*)c)[j] = v;
        }
        r[l] = row;
        cf[l] = c;
    }
    free(mat->r);
    mat->r = r;
    if (bits == 8) {
        free(mat->cf_8);
        mat->cf_8 = (int8_t**)cf;
    } else if (bits == 16) {
        free(mat->cf_16);
        mat->cf_16 = (int16_t**)cf;
    } else {
        free(mat->cf_32);
        mat->cf_32 = (int32_t**)cf;
    }
    mat->np = np;
    return GBGPU_OK;
}

int store_rows(gbgpu_mat_t* mat, int bits, const gbgpu_rows& out) {
    return store_rows_raw(mat, bits, out.np, out.row_ptr, out.cols, out.vals);
}

// mat->r rows -> the small path's pinned staging (coefficients reduced into
// [0, p) as gather_rows does)
struct GatherCtx {
    const gbgpu_mat_t* mat;
    const void* const* tab;
    int bits;
    int32_t p;
};
void fill_from_rows(void* ctx, int64_t* ptr, int32_t* cols, uint32_t* vals) {
    const GatherCtx& g = *(const GatherCtx*)ctx;
    const int32_t nr = g.mat->nr;
    ptr[0] = 0;
    for (int32_t i = 0; i < nr; ++i) {
        const gbgpu_hm_t* r = g.mat->r[i];
        const int64_t off = ptr[i], len = r[2];
        ptr[i + 1] = off + len;
        memcpy(cols + off, r + 3, sizeof(int32_t) * (size_t)len);
        for (int64_t j = 0; j < len; ++j) {
            int32_t v = load_cf(g.tab, g.bits, r[0], j) % g.p;
            vals[off + j] = (uint32_t)(v < 0 ? v + g.p : v);
        }
    }
}

gbgpu_options shim_options() {
    gbgpu_options o{};
    o.form = GBGPU_FORM_AUTO;
    const char* dev = getenv("GBGPU_DEVICE");
    o.device = dev ? atoi(dev) : 0;
    o.check = 1;
    return o;
}

}  // namespace

extern "C" {

int gbgpu_linear_algebra_status(gbgpu_mat_t* mat, const gbgpu_bs_t* bs, gbgpu_stat_t* st) {
    DeviceScope scope;
    if (!mat || !bs || !st) return GBGPU_EINVAL;
    const double ct0 = cpu_seconds(), rt0 = wall_seconds();
    const int bits = coef_bits(st);
    gbgpu_options o = shim_options();
    int rc;
    int64_t nnz = 0;
    for (int32_t i = 0; i < mat->nr; ++i) nnz += mat->r[i][2];
    if (st->fc >= 2 && nnz <= INT32_MAX / 2 &&
        small_eligible(mat->nr, mat->ncl, mat->ncr, o.device)) {
        // small matrix: rows gathered straight into pinned staging, one pass
        GatherCtx g{mat, bs_table(bs, bits), bits, st->fc};
        SmallInput in{st->fc, mat->nr, mat->ncl, mat->ncr, nnz, o.device, fill_from_rows, &g};
        SmallAnswer a;
        if ((rc = small_reduce(in, &a))) return rc;
        // the la functions free their input rows (src/la_ff_16.c:665, :688-691, :804)
        for (int32_t i = 0; i < mat->nr; ++i) free(mat->r[i]);
        if ((rc = store_rows_raw(mat, bits, a.np, a.offs, a.cols, a.vals))) return rc;
    } else {
        std::vector<int64_t> ptr;
        std::vector<int32_t> cols, vals;
        gather_rows(mat->r, mat->nr, bs_table(bs, bits), bits, st->fc, ptr, cols, vals);
        gbgpu_csr m{st->fc, st->laopt, mat->nr, mat->ncl, mat->ncr, ptr.data(), cols.data(),
                    vals.data()};
        gbgpu_rows out{};
        if ((rc = gbgpu_reduce(&m, &o, &out))) return rc;
        for (int32_t i = 0; i < mat->nr; ++i) free(mat->r[i]);
        rc = store_rows(mat, bits, out);
        gbgpu_rows_free(&out);
        if (rc) return rc;
    }
    // the sparse options also reset the row count (src/la_ff_16.c:734)
    const int32_t lo = st->laopt;
    if (!(lo == 1 || lo == 42 || lo == 43)) mat->nr = mat->sz = mat->np;
    st->la_ctime += cpu_seconds() - ct0;
    st->la_rtime += wall_seconds() - rt0;
    st->num_zerored += (mat->nrl - mat->np);
    if (st->info_level > 1) {
        printf("%7d new %7d zero", mat->np, mat->nrl - mat->np);
        fflush(stdout);
    }
    return GBGPU_OK;
}

void gbgpu_linear_algebra(gbgpu_mat_t* mat, const gbgpu_bs_t* bs, gbgpu_stat_t* st) {
    const int rc = gbgpu_linear_algebra_status(mat, bs, st);
    if (rc) {
        fprintf(stderr, "gbgpu_linear_algebra failed (%d): %s\n", rc, gbgpu_last_error());
        exit(1);
    }
}

int gbgpu_interreduce_matrix_rows_status(gbgpu_mat_t* mat, gbgpu_bs_t* bs,
                                         const gbgpu_stat_t* st) {
    DeviceScope scope;
    if (!mat || !bs || !st) return GBGPU_EINVAL;
    if (st->info_level > 1) printf("                        ");
    const int bits = coef_bits(st);
    std::vector<int64_t> ptr;
    std::vector<int32_t> cols, vals;
    gather_rows(mat->r, mat->nr, bs_table(bs, bits), bits, st->fc, ptr, cols, vals);
    gbgpu_options o = shim_options();
    gbgpu_rows out{};
    int rc = gbgpu_interreduce(st->fc, mat->nr, mat->nc, ptr.data(), cols.data(), vals.data(),
                               &o, &out);
    if (rc) return rc;
    // free_basis_elements (src/basis.c:25-57): the basis gives up its elements
    const void* const* tab = bs_table(bs, bits);
    for (int32_t i = 0; i < bs->ld; ++i) {
        free(((void**)tab)[i]);
        free(bs->hm[i]);
    }
    bs->ld = 0;
    for (int32_t i = 0; i < mat->nr; ++i) free(mat->r[i]);
    rc = store_rows(mat, bits, out);
    gbgpu_rows_free(&out);
    return rc;
}

void gbgpu_interreduce_matrix_rows(gbgpu_mat_t* mat, gbgpu_bs_t* bs, const gbgpu_stat_t* st) {
    const int rc = gbgpu_interreduce_matrix_rows_status(mat, bs, st);
    if (rc) {
        fprintf(stderr, "gbgpu_interreduce_matrix_rows failed (%d): %s\n", rc,
                gbgpu_last_error());
        exit(1);
    }
}

// ---------------------------------------------------------------------------
// The linear algebra and the step after it (src/f4.c:306-311) with the answer
// kept on the device in between: gbgpu_linear_algebra_keep leaves the answer
// of the round in the calling thread's slot, and
// gbgpu_convert_sparse_matrix_rows_to_basis_elements turns it into basis
// elements, their columns already mapped to the basis hash table on the
// device (api.cu: gbgpu_plan_first_entry, gbgpu_plan_map_columns).

}  // extern "C"

namespace {

// The kept answer: on the device in a plan, or -- for the matrices the
// one-pass small path reduces, whose answer lands in host memory anyway -- as
// host CSR arrays.
struct KeptAnswer {
    gbgpu_plan* plan = nullptr;
    bool host = false;
    std::vector<int64_t> hptr;
    std::vector<int32_t> hcols, hvals;
    const gbgpu_mat_t* mat = nullptr;
    int32_t np = 0, ncl = 0, ncr = 0;
    int64_t nnz = 0;
    int bits = 32;
};
thread_local KeptAnswer g_kept;

void drop_kept() {
    if (g_kept.plan) gbgpu_plan_destroy(g_kept.plan);
    g_kept = KeptAnswer{};
}

// f(begin, end) over [0, n) split among the host's threads (at most 16, at
// least `grain` items each)
template <class Fn>
void host_parallel(int64_t n, int64_t grain, Fn f) {
    const int64_t hw = std::max<int64_t>(1, std::min<int64_t>(16, std::thread::hardware_concurrency()));
    const int64_t nt = std::max<int64_t>(1, std::min<int64_t>(hw, n / grain));
    if (nt <= 1) {
        f((int64_t)0, n);
        return;
    }
    std::vector<std::thread> th;
    for (int64_t q = 0; q < nt; ++q)
        th.emplace_back([&, q] { f(n * q / nt, n * (q + 1) / nt); });
    for (auto& x : th) x.join();
}

// check_enlarge_basis_ff_{8,16,32} (src/basis.c:149-165 and twins): room
// for `added` more elements, the new reducibility flags cleared
int grow_basis(gbgpu_bs_t* bs, int32_t added, int bits) {
    if (bs->ld + added < bs->sz) return GBGPU_OK;
    const int32_t sz = bs->sz * 2 > bs->ld + added ? bs->sz * 2 : bs->ld + added;
    const size_t esz = bits == 8 ? sizeof(int8_t*) : bits == 16 ? sizeof(int16_t*) : sizeof(int32_t*);
    void** cf = bits == 8 ? (void**)&bs->cf_8 : bits == 16 ? (void**)&bs->cf_16 : (void**)&bs->cf_32;
    void* ncf = realloc(*cf, esz * (size_t)sz);
    void* nhm = realloc(bs->hm, sizeof(gbgpu_hm_t*) * (size_t)sz);
    void* nlm = realloc(bs->lm, sizeof(int32_t) * (size_t)sz);
    void* nlmps = realloc(bs->lmps, sizeof(int32_t) * (size_t)sz);
    void* nred = realloc(bs->red, sizeof(int8_t) * (size_t)sz);
    if (ncf) *cf = ncf;
    if (nhm) bs->hm = (gbgpu_hm_t**)nhm;
    if (nlm) bs->lm = (int32_t*)nlm;
    if (nlmps) bs->lmps = (int32_t*)nlmps;
    if (nred) bs->red = (int8_t*)nred;
    if (!ncf || !nhm || !nlm || !nlmps || !nred) return GBGPU_ENOMEM;
    bs->sz = sz;
    memset(bs->red + bs->ld, 0, (size_t)(sz - bs->ld));
    return GBGPU_OK;
}

}  // namespace

namespace gbgpu {

// enlarge_hash_table (src/hash.c:185-240), called until at least `need` free
// entries remain (src/convert.c:166-168): every call doubles the exponent
// storage and the hash map and reinserts every element, in index order, into
// the cleared map with the table's probe sequence k <- (k + i) mod hsz.  Only
// the last reinsertion decides the map, so one growth to the final size with
// one reinsertion leaves the same table (the same sizes, indices and map
// layout, which the reference's own code probes later), without the
// intermediate copies: fresh zeroed blocks for the map and the hash data.
int grow_hash_table(gbgpu_ht_t* ht, int64_t need) {
    int64_t esz = ht->esz, hsz = ht->hsz;
    const int32_t eld = ht->eld, nv = ht->nv;
    if (esz - eld >= need) return GBGPU_OK;
    while (esz - eld < need) {
        esz *= 2;
        hsz *= 2;
    }
    if (esz > INT32_MAX || hsz > INT32_MAX) {
        set_error("basis hash table would exceed 2^31 entries");
        return GBGPU_ERANGE;
    }
    gbgpu_hd_t* hd = (gbgpu_hd_t*)calloc((size_t)esz, sizeof(gbgpu_hd_t));
    int16_t* blk = (int16_t*)malloc(sizeof(int16_t) * (size_t)esz * (size_t)nv);
    int16_t** ev = (int16_t**)malloc(sizeof(int16_t*) * (size_t)esz);
    int32_t* hmap = (int32_t*)calloc((size_t)hsz, sizeof(int32_t));
    if (!hd || !blk || !ev || !hmap) {
        free(hd);
        free(blk);
        free(ev);
        free(hmap);
        return GBGPU_ENOMEM;
    }
    memcpy(hd, ht->hd, sizeof(gbgpu_hd_t) * (size_t)eld);
    memcpy(blk, ht->ev[0], sizeof(int16_t) * (size_t)eld * (size_t)nv);
    host_parallel(esz, 1 << 16, [&](int64_t a, int64_t b) {
        for (int64_t i = a; i < b; ++i) ev[i] = blk + (size_t)i * (size_t)nv;
    });
    free(ht->hd);
    free(ht->ev[0]);
    free(ht->ev);
    free(ht->hmap);
    ht->hd = hd;
    ht->ev = ev;
    ht->hmap = hmap;
    ht->esz = (int32_t)esz;
    ht->hsz = (int32_t)hsz;
    const uint32_t mask = (uint32_t)hsz - 1u;
    for (int32_t i = 1; i < eld; ++i) {
        uint32_t k = (uint32_t)hd[i].val;
        for (int64_t j = 0; j < hsz; ++j) {
            k = (k + (uint32_t)j) & mask;
            if (hmap[k]) continue;
            hmap[k] = i;
            break;
        }
    }
    return GBGPU_OK;
}

}  // namespace gbgpu

namespace {

// the index of monomial e (hash value h) in the table, inserted at the first
// free slot of its probe sequence when absent, as insert_in_basis_hash_table_
// pivots does it (src/hash.c:604-669): a new element takes the next free
// index with the degree and divisor mask of its secondary-table entry
int32_t table_index(gbgpu_ht_t* ht, const int16_t* e, int32_t h, int32_t deg, int32_t sdm) {
    const int32_t nv = ht->nv, hsz = ht->hsz;
    const uint32_t mask = (uint32_t)hsz - 1u;
    uint32_t k = (uint32_t)h;
    for (int32_t i = 0; i < hsz; ++i) {
        k = (k + (uint32_t)i) & mask;
        const int32_t hm = ht->hmap[k];
        if (!hm) break;
        if (ht->hd[hm].val != h) continue;
        if (memcmp(ht->ev[hm], e, sizeof(int16_t) * (size_t)nv) == 0) return hm;
    }
    const int32_t pos = ht->eld;
    memcpy(ht->ev[pos], e, sizeof(int16_t) * (size_t)nv);
    ht->hmap[k] = pos;
    ht->hd[pos].deg = deg;
    ht->hd[pos].sdm = sdm;
    ht->hd[pos].val = h;
    ht->eld = pos + 1;
    return pos;
}

}  // namespace

extern "C" {

int gbgpu_linear_algebra_keep_status(gbgpu_mat_t* mat, const gbgpu_bs_t* bs, gbgpu_stat_t* st) {
    DeviceScope scope;
    drop_kept();
    if (!mat || !bs || !st) return GBGPU_EINVAL;
    const double ct0 = cpu_seconds(), rt0 = wall_seconds();
    const int bits = coef_bits(st);
    gbgpu_options o = shim_options();
    int64_t in_nnz = 0;
    for (int32_t i = 0; i < mat->nr; ++i) in_nnz += mat->r[i][2];
    if (st->fc >= 2 && in_nnz <= INT32_MAX / 2 &&
        small_eligible(mat->nr, mat->ncl, mat->ncr, o.device)) {
        // one pass; the answer comes back to host memory, where it is kept
        GatherCtx gc{mat, bs_table(bs, bits), bits, st->fc};
        SmallInput in{st->fc, mat->nr, mat->ncl, mat->ncr, in_nnz, o.device, fill_from_rows, &gc};
        SmallAnswer a;
        if (int rc = small_reduce(in, &a)) return rc;
        for (int32_t i = 0; i < mat->nr; ++i) free(mat->r[i]);
        mat->np = a.np;
        if (a.np > 0) {
            g_kept.host = true;
            g_kept.hptr.assign(a.offs, a.offs + a.np + 1);
            g_kept.hcols.assign(a.cols, a.cols + a.nnz);
            g_kept.hvals.assign(a.vals, a.vals + a.nnz);
            g_kept.mat = mat;
            g_kept.np = a.np;
            g_kept.nnz = a.nnz;
            g_kept.ncl = mat->ncl;
            g_kept.ncr = mat->ncr;
            g_kept.bits = bits;
        }
    } else {
    std::vector<int64_t> ptr;
    std::vector<int32_t> cols, vals;
    gather_rows(mat->r, mat->nr, bs_table(bs, bits), bits, st->fc, ptr, cols, vals);
    gbgpu_csr m{st->fc, st->laopt, mat->nr, mat->ncl, mat->ncr, ptr.data(), cols.data(),
                vals.data()};
    gbgpu_plan* plan = nullptr;
    int rc = gbgpu_plan_create(&m, &o, &plan);
    if (!rc) rc = gbgpu_plan_run(plan);
    int32_t np = 0;
    int64_t nnz = 0;
    if (!rc) {
        // a size query: NULL buffers of zero capacity
        rc = gbgpu_plan_result_into(plan, nullptr, nullptr, nullptr, 0, 0, &np, &nnz);
        if (rc == GBGPU_ERANGE) rc = GBGPU_OK;
    }
    if (rc) {
        if (plan) gbgpu_plan_destroy(plan);
        return rc;
    }
    // the la functions free their input rows (src/la_ff_16.c:665, :688-691, :804)
    for (int32_t i = 0; i < mat->nr; ++i) free(mat->r[i]);
    mat->np = np;
    if (np > 0) {
        g_kept.plan = plan;
        g_kept.mat = mat;
        g_kept.np = np;
        g_kept.nnz = nnz;
        g_kept.ncl = mat->ncl;
        g_kept.ncr = mat->ncr;
        g_kept.bits = bits;
    } else {
        gbgpu_plan_destroy(plan);
    }
    }  // plan path
    const int32_t lo = st->laopt;
    if (!(lo == 1 || lo == 42 || lo == 43)) mat->nr = mat->sz = mat->np;
    st->la_ctime += cpu_seconds() - ct0;
    st->la_rtime += wall_seconds() - rt0;
    st->num_zerored += (mat->nrl - mat->np);
    if (st->info_level > 1) {
        printf("%7d new %7d zero", mat->np, mat->nrl - mat->np);
        fflush(stdout);
    }
    return GBGPU_OK;
}

void gbgpu_linear_algebra_keep(gbgpu_mat_t* mat, const gbgpu_bs_t* bs, gbgpu_stat_t* st) {
    const int rc = gbgpu_linear_algebra_keep_status(mat, bs, st);
    if (rc) {
        fprintf(stderr, "gbgpu_linear_algebra_keep failed (%d): %s\n", rc, gbgpu_last_error());
        exit(1);
    }
}

int gbgpu_kept_answer(const gbgpu_mat_t* mat) {
    return (g_kept.plan || g_kept.host) && g_kept.mat == mat && mat && g_kept.np == mat->np ? 1
                                                                                            : 0;
}

int gbgpu_convert_sparse_matrix_rows_to_basis_elements_status(
    gbgpu_mat_t* mat, gbgpu_bs_t* bs, gbgpu_ht_t* bht, const gbgpu_ht_t* sht,
    const int32_t* hcm, gbgpu_stat_t* st) {
    if (!mat || !bs || !bht || !sht || !hcm || !st) return GBGPU_EINVAL;
    if (!gbgpu_kept_answer(mat)) {
        set_error("no answer of gbgpu_linear_algebra_keep for this matrix");
        return GBGPU_EINVAL;
    }
    if (bht->hsz <= 0 || (bht->hsz & (bht->hsz - 1)) != 0 || bht->nv != sht->nv) {
        set_error("basis hash table: size not a power of two, or variables differ");
        return GBGPU_EINVAL;
    }
    const double ct0 = cpu_seconds(), rt0 = wall_seconds();
    const KeptAnswer& ka = g_kept;  // dropped at the end
    const int bits = ka.bits;
    int rc;
    // room for the new elements and for every entry's monomial
    // (src/convert.c:157-168)
    if ((rc = grow_basis(bs, ka.np, bits))) return rc;
    if ((rc = grow_hash_table(bht, ka.nnz))) return rc;
    // the right columns by their first entry in the answer: the order in
    // which the reference meets (and inserts) their monomials
    std::vector<int64_t> first((size_t)std::max(ka.ncr, 1), -1);
    if (ka.host) {
        for (int64_t e = (int64_t)ka.hcols.size() - 1; e >= 0; --e)
            first[ka.hcols[e] - ka.ncl] = e;
    } else if ((rc = gbgpu_plan_first_entry(ka.plan, first.data(), ka.ncr))) {
        return rc;
    }
    std::vector<int32_t> order;
    order.reserve((size_t)ka.ncr);
    for (int32_t j = 0; j < ka.ncr; ++j)
        if (first[j] >= 0) order.push_back(j);
    std::sort(order.begin(), order.end(),
              [&](int32_t a, int32_t b) { return first[a] < first[b]; });
    std::vector<int32_t> map((size_t)std::max(ka.ncr, 1), 0);
    for (int32_t j : order) {
        const int32_t h = hcm[ka.ncl + j];  // the column's monomial in the secondary table
        map[j] = table_index(bht, sht->ev[h], sht->hd[h].val, sht->hd[h].deg, sht->hd[h].sdm);
    }
    // the answer with its entries mapped: rewritten on the device (plan), or
    // here for an answer already in host memory
    gbgpu_rows out{};
    std::vector<int32_t> hmapped;
    if (ka.host) {
        hmapped.resize(ka.hcols.size());
        for (size_t e = 0; e < ka.hcols.size(); ++e) hmapped[e] = map[ka.hcols[e] - ka.ncl];
        out.np = ka.np;
        out.nnz = ka.nnz;
        out.row_ptr = const_cast<int64_t*>(ka.hptr.data());
        out.cols = hmapped.data();
        out.vals = const_cast<int32_t*>(ka.hvals.data());
    } else {
        if ((rc = gbgpu_plan_map_columns(ka.plan, map.data(), ka.ncr))) return rc;
        if ((rc = gbgpu_plan_result(ka.plan, &out))) return rc;
    }
    auto release_out = [&]() {
        if (!ka.host) gbgpu_rows_free(&out);
    };
    // the rows join the basis at bs->ld + i (src/convert.c:225-236); mat keeps
    // the pointer arrays the la would have left
    const int32_t bl = bs->ld, np = out.np;
    const size_t esz = bits == 8 ? 1 : bits == 16 ? 2 : 4;
    void** cf = (void**)malloc(sizeof(void*) * (size_t)std::max(np, 1));
    gbgpu_hm_t** r = (gbgpu_hm_t**)malloc(sizeof(gbgpu_hm_t*) * (size_t)std::max(np, 1));
    if (!cf || !r) {
        free(cf);
        free(r);
        release_out();
        return GBGPU_ENOMEM;
    }
    std::atomic<bool> oom{false};
    host_parallel(np, 8, [&](int64_t ia, int64_t ib) {
      for (int32_t i = (int32_t)ia; i < (int32_t)ib; ++i) {
        const int64_t b0 = out.row_ptr[i], len = out.row_ptr[i + 1] - b0;
        gbgpu_hm_t* row = (gbgpu_hm_t*)malloc(sizeof(gbgpu_hm_t) * (size_t)(len + 3));
        void* c = malloc(esz * (size_t)std::max<int64_t>(len, 1));
        if (!row || !c) {
            free(row);
            free(c);
            oom = true;
            return;
        }
        row[0] = bl + i;
        row[1] = (gbgpu_hm_t)(len % 4);
        row[2] = (gbgpu_hm_t)len;
        memcpy(row + 3, out.cols + b0, sizeof(int32_t) * (size_t)len);
        for (int64_t j = 0; j < len; ++j) {
            const int32_t v = out.vals[b0 + j];
            if (bits == 8) ((int8_t*)c)[j] = (int8_t)v;
            else if (bits == 16) ((int16_t*)c)[j] = (int16_t)v;
            else ((int32_t*)c)[j] = v;
        }
        r[i] = row;
        cf[i] = c;
        bs->hm[bl + i] = row;
        if (bits == 8) bs->cf_8[bl + i] = (int8_t*)c;
        else if (bits == 16) bs->cf_16[bl + i] = (int16_t*)c;
        else bs->cf_32[bl + i] = (int32_t*)c;
      }
    });
    release_out();
    if (oom) {
        // the rows made so far are the basis's (bs->hm, bs->cf_*); the
        // pointer arrays meant for mat are not handed over
        free(cf);
        free(r);
        set_error("basis conversion: host allocation failed");
        return GBGPU_ENOMEM;
    }
    free(mat->r);
    mat->r = r;
    if (bits == 8) {
        free(mat->cf_8);
        mat->cf_8 = (int8_t**)cf;
    } else if (bits == 16) {
        free(mat->cf_16);
        mat->cf_16 = (int16_t**)cf;
    } else {
        free(mat->cf_32);
        mat->cf_32 = (int32_t**)cf;
    }
    drop_kept();
    st->convert_ctime += cpu_seconds() - ct0;
    st->convert_rtime += wall_seconds() - rt0;
    return GBGPU_OK;
}

void gbgpu_convert_sparse_matrix_rows_to_basis_elements(gbgpu_mat_t* mat, gbgpu_bs_t* bs,
                                                        gbgpu_ht_t* bht, const gbgpu_ht_t* sht,
                                                        const int32_t* hcm, gbgpu_stat_t* st) {
    const int rc =
        gbgpu_convert_sparse_matrix_rows_to_basis_elements_status(mat, bs, bht, sht, hcm, st);
    if (rc) {
        fprintf(stderr, "gbgpu_convert_sparse_matrix_rows_to_basis_elements failed (%d): %s\n",
                rc, gbgpu_last_error());
        exit(1);
    }
}

// a batch matrix the one-launch small-matrix kernel takes
static bool batch_small(const gbgpu_csr& m, const gbgpu_options* opt) {
    if (opt && !(opt->form == GBGPU_FORM_AUTO || opt->form == GBGPU_FORM_PLAIN)) return false;
    if (opt && opt->profile) return false;
    if (m.p < 2 || m.nr <= 0 || !m.row_ptr || !m.cols || !m.vals || m.row_ptr[0] != 0) return false;
    if (m.row_ptr[m.nr] < 0 || m.row_ptr[m.nr] > INT32_MAX / 2) return false;  // 32-bit offsets
    const int vb = m.val_bytes ? m.val_bytes : 4;
    if (!(vb == 1 || vb == 2 || vb == 4) || (vb < 4 && (int64_t)m.p >= ((int64_t)1 << (8 * vb))))
        return false;
    return small_batch_bytes(m.nr, m.ncl, m.ncr, opt ? opt->device : 0) > 0;
}

int gbgpu_reduce_batch(int32_t n, const gbgpu_csr* ms, const gbgpu_options* opt,
                       gbgpu_rows* outs, int32_t* status) {
    DeviceScope scope;
    if (n < 0 || (n > 0 && (!ms || !outs || !status))) return GBGPU_EINVAL;
    for (int32_t i = 0; i < n; ++i) {
        memset(&outs[i], 0, sizeof(gbgpu_rows));
        status[i] = GBGPU_OK;
    }
    if (n == 0) return GBGPU_OK;
    {
        // no usable device: no matrix runs, each one says why
        DeviceInfo info;
        if (int rc = device_init(opt ? opt->device : 0, &info)) {
            for (int32_t i = 0; i < n; ++i) status[i] = rc;
            return rc;
        }
    }
    // The small matrices of the batch go to ONE persistent launch (small.cu,
    // a device work queue over the matrices); the others are reduced by a few
    // host workers, each one matrix at a time on a stream of its own, so
    // that their host round trips and small launches interleave on the device
    // (and at most `workers` of them hold device memory at once).  The small
    // launch runs on the calling thread while the workers run.
    std::vector<int32_t> small_idx, big_idx;
    for (int32_t i = 0; i < n; ++i)
        (batch_small(ms[i], opt) ? small_idx : big_idx).push_back(i);
    int workers = 4;
    if (const char* w = getenv("GBGPU_BATCH_WORKERS")) workers = std::max(1, atoi(w));
    workers = std::min<int>(workers, std::max<int>((int)big_idx.size(), 1));
    const int device = opt ? opt->device : 0;
    std::atomic<int32_t> next{0};
    const int32_t n_big = (int32_t)big_idx.size();
    // device-memory gate: the matrices in flight together stay within 60% of
    // the memory free when the batch starts (one matrix always runs)
    size_t free_b = 0, total_b = 0;
    if (cudaSetDevice(device) == cudaSuccess) cudaMemGetInfo(&free_b, &total_b);
    const double budget = 0.6 * (double)free_b;
    double in_flight = 0.0;
    std::mutex gate_mu;
    std::condition_variable gate_cv;
    auto estimate = [&](const gbgpu_csr& m) {
        const double t = std::max(0, m.nr - m.ncl), nc = (double)m.ncl + m.ncr;
        const double nnz = m.nr > 0 && m.row_ptr ? (double)m.row_ptr[m.nr] : 0.0;
        return nnz * 12.0 + (t + m.ncl) * nc * 4.0 + 2.0 * (t + m.ncr) * m.ncl +
               t * (double)m.ncr * 8.0;
    };
    auto work = [&]() {
        if (cudaSetDevice(device) != cudaSuccess) {
            for (int32_t k; (k = next.fetch_add(1)) < n_big;) status[big_idx[k]] = GBGPU_ECUDA;
            return;
        }
        for (int32_t k; (k = next.fetch_add(1)) < n_big;) {
            const int32_t i = big_idx[k];
            const double need = estimate(ms[i]);
            {
                std::unique_lock<std::mutex> lock(gate_mu);
                gate_cv.wait(lock, [&] { return in_flight == 0.0 || in_flight + need <= budget; });
                in_flight += need;
            }
            struct Release {
                std::mutex& mu;
                std::condition_variable& cv;
                double& fl;
                double n;
                ~Release() {
                    {
                        std::lock_guard<std::mutex> lock(mu);
                        fl -= n;
                        if (fl < 1.0) fl = 0.0;
                    }
                    cv.notify_all();
                }
            } release{gate_mu, gate_cv, in_flight, need};
            gbgpu_options o{};
            if (opt) o = *opt;
            o.stream = nullptr;  // the plan creates its own stream
            Plan* P = nullptr;
            int rc = plan_create(&ms[i], &o, 0, &P);
            if (!rc) rc = plan_run(P);
            if (!rc) rc = plan_result(P, &outs[i]);
            if (P) plan_destroy(P);
            status[i] = rc;
            if (rc && getenv("GBGPU_DEBUG"))
                fprintf(stderr, "gbgpu batch matrix %d: status %d: %s\n", i, rc, gbgpu_last_error());
        }
    };
    std::vector<std::thread> pool;
    if (n_big > 0)
        for (int k = 0; k < workers; ++k) pool.emplace_back(work);
    if (!small_idx.empty()) {
        std::vector<const gbgpu_csr*> sm;
        for (int32_t i : small_idx) sm.push_back(&ms[i]);
        std::vector<gbgpu_rows> so(sm.size());
        std::vector<int32_t> ss(sm.size(), GBGPU_OK);
        for (auto& r : so) memset(&r, 0, sizeof(r));
        int rc = small_batch((int32_t)sm.size(), sm.data(), device, so.data(), ss.data());
        for (size_t k = 0; k < sm.size(); ++k) {
            outs[small_idx[k]] = so[k];
            status[small_idx[k]] = rc ? rc : ss[k];
        }
    }
    for (auto& th : pool) th.join();
    return GBGPU_OK;
}

int gbgpu_layout(int64_t* out, int32_t n) {
    const int64_t v[] = {
        (int64_t)sizeof(gbgpu_mat_t),
        (int64_t)offsetof(gbgpu_mat_t, r), (int64_t)offsetof(gbgpu_mat_t, cf_8),
        (int64_t)offsetof(gbgpu_mat_t, cf_16), (int64_t)offsetof(gbgpu_mat_t, cf_32),
        (int64_t)offsetof(gbgpu_mat_t, sz), (int64_t)offsetof(gbgpu_mat_t, np),
        (int64_t)offsetof(gbgpu_mat_t, nr), (int64_t)offsetof(gbgpu_mat_t, nc),
        (int64_t)offsetof(gbgpu_mat_t, nru), (int64_t)offsetof(gbgpu_mat_t, nrl),
        (int64_t)offsetof(gbgpu_mat_t, ncl), (int64_t)offsetof(gbgpu_mat_t, ncr),
        (int64_t)sizeof(gbgpu_bs_t),
        (int64_t)offsetof(gbgpu_bs_t, ld), (int64_t)offsetof(gbgpu_bs_t, hm),
        (int64_t)offsetof(gbgpu_bs_t, cf_8), (int64_t)offsetof(gbgpu_bs_t, cf_16),
        (int64_t)offsetof(gbgpu_bs_t, cf_32),
        (int64_t)sizeof(gbgpu_stat_t),
        (int64_t)offsetof(gbgpu_stat_t, la_ctime), (int64_t)offsetof(gbgpu_stat_t, la_rtime),
        (int64_t)offsetof(gbgpu_stat_t, num_zerored), (int64_t)offsetof(gbgpu_stat_t, fc),
        (int64_t)offsetof(gbgpu_stat_t, laopt), (int64_t)offsetof(gbgpu_stat_t, nthrds),
        (int64_t)offsetof(gbgpu_stat_t, ff_bits), (int64_t)offsetof(gbgpu_stat_t, info_level),
        (int64_t)offsetof(gbgpu_stat_t, mo), (int64_t)offsetof(gbgpu_stat_t, num_rowsred),
        (int64_t)offsetof(gbgpu_stat_t, convert_ctime),
        (int64_t)offsetof(gbgpu_stat_t, convert_rtime),
        (int64_t)sizeof(gbgpu_hd_t), (int64_t)offsetof(gbgpu_hd_t, deg),
        (int64_t)offsetof(gbgpu_hd_t, idx),
        (int64_t)sizeof(gbgpu_ht_t), (int64_t)offsetof(gbgpu_ht_t, ev),
        (int64_t)offsetof(gbgpu_ht_t, hd), (int64_t)offsetof(gbgpu_ht_t, eld),
        (int64_t)offsetof(gbgpu_ht_t, nv),
    };
    const int32_t k = (int32_t)(sizeof(v) / sizeof(v[0]));
    for (int32_t i = 0; i < k && i < n; ++i) out[i] = v[i];
    return k;
}

}  // extern "C"
