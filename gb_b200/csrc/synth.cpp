// synth.cpp -- host generator of the banded A|B/C|D staircase matrices
// (libgbsynth.so, plain C++ with std::thread), for the batched workloads whose
// matrices hold up to hundreds of millions of entries.  The structure is that
// of gb_b200.synth.staircase: known pivots with leads 0..nru-1 (coefficient 1),
// nrl rows with leads uniform in the left block, a per-row density drawn
// uniformly from [dmin, dmax] and split between a band to the right of the lead
// in the left block and a band of the right block around the lead's image;
// inside each band one column per equal stratum (so the columns of a row are
// distinct), coefficients uniform in [1, p).  Every row draws from its own
// generator (splitmix64 of the seed and the row), so the matrix does not depend
// on the thread count.  Rows are ordered by (lead, known pivot first, length),
// the order gb's sort_matrix_rows gives (src/order.c:98-131).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <numeric>
#include <thread>
#include <vector>

namespace {

struct Rng {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    uint64_t below(uint64_t n) { return next() % n; }
};

struct Shape {
    int64_t lead, na, nb;  // lead, entries in the A band (lead excluded), in the B band
    int64_t a_lo, a_hi, b_lo, b_hi;
    int64_t len;
};

Shape shape_of(int64_t i, int64_t nru, int64_t ncr, double dmin, double dmax, double band,
               uint64_t seed) {
    const int64_t ncl = nru, nc = nru + ncr;
    Rng r{seed * 0x100000001B3ull + (uint64_t)i * 0x9E3779B97F4A7C15ull + 1};
    Shape s;
    s.lead = i < nru ? i : (int64_t)r.below((uint64_t)std::max<int64_t>(ncl, 1));
    const int64_t k = std::max<int64_t>(2, std::llround((dmin + (dmax - dmin) * r.unit()) * nc));
    const int64_t ka = k / 2, kb = k - ka;
    const int64_t wa = std::max<int64_t>(1, (int64_t)(band * ka));
    s.a_lo = s.lead + 1;
    s.a_hi = std::min(ncl, s.lead + 1 + wa);
    s.na = std::max<int64_t>(0, std::min(ka - 1, s.a_hi - s.a_lo));
    const int64_t center = ncl + (s.lead * ncr) / std::max<int64_t>(ncl, 1);
    const int64_t wb = std::max<int64_t>(1, (int64_t)(band * kb));
    s.b_lo = std::max(ncl, center - wb / 2);
    s.b_hi = std::min(nc, center + wb - wb / 2);
    s.nb = std::max<int64_t>(0, std::min(kb, s.b_hi - s.b_lo));
    s.len = 1 + s.na + s.nb;
    return s;
}

// one column per stratum [ceil(j w / c), ceil((j + 1) w / c)) of [lo, hi)
void stratified(Rng& r, int64_t lo, int64_t hi, int64_t c, int32_t* out) {
    const int64_t w = hi - lo;
    for (int64_t j = 0; j < c; ++j) {
        const int64_t a = (j * w + c - 1) / c, b = ((j + 1) * w + c - 1) / c;
        out[j] = (int32_t)(lo + a + (int64_t)r.below((uint64_t)std::max<int64_t>(b - a, 1)));
    }
}

template <class F>
void parallel(int64_t n, int threads, const F& f) {
    std::vector<std::thread> ts;
    const int64_t chunk = (n + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        const int64_t a = t * chunk, b = std::min(n, a + chunk);
        if (a >= b) break;
        ts.emplace_back([=, &f] { f(a, b); });
    }
    for (auto& th : ts) th.join();
}

}  // namespace

extern "C" {

// Row lengths in output order: writes row_ptr[nr + 1]; returns nnz (or -1).
int64_t gbsynth_staircase_layout(int32_t nru, int32_t nrl, int32_t ncr, double dmin, double dmax,
                                 double band, uint64_t seed, int32_t threads, int64_t* row_ptr,
                                 int32_t* order) {
    const int64_t nr = (int64_t)nru + nrl;
    if (nru < 0 || nrl < 0 || ncr < 0 || threads < 1) return -1;
    std::vector<int64_t> lead(nr), len(nr);
    parallel(nr, threads, [&](int64_t a, int64_t b) {
        for (int64_t i = a; i < b; ++i) {
            const Shape s = shape_of(i, nru, ncr, dmin, dmax, band, seed);
            lead[i] = s.lead;
            len[i] = s.len;
        }
    });
    for (int64_t i = 0; i < nr; ++i) order[i] = (int32_t)i;
    std::stable_sort(order, order + nr, [&](int32_t x, int32_t y) {
        if (lead[x] != lead[y]) return lead[x] < lead[y];
        const bool lx = x >= nru, ly = y >= nru;
        if (lx != ly) return !lx;
        return len[x] < len[y];
    });
    row_ptr[0] = 0;
    for (int64_t k = 0; k < nr; ++k) row_ptr[k + 1] = row_ptr[k] + len[order[k]];
    return row_ptr[nr];
}

// Entries of every row at its place in the layout above.
int gbsynth_staircase_fill(int32_t nru, int32_t nrl, int32_t ncr, int32_t p, double dmin,
                           double dmax, double band, uint64_t seed, int32_t threads,
                           const int64_t* row_ptr, const int32_t* order, int32_t* cols,
                           int32_t* vals) {
    const int64_t nr = (int64_t)nru + nrl;
    if (p < 2 || threads < 1) return -1;
    parallel(nr, threads, [&](int64_t a, int64_t b) {
        for (int64_t k = a; k < b; ++k) {
            const int64_t i = order[k];
            const Shape s = shape_of(i, nru, ncr, dmin, dmax, band, seed);
            Rng r{(seed ^ 0xD1B54A32D192ED03ull) + (uint64_t)i * 0x632BE59BD9B4E019ull};
            int32_t* c = cols + row_ptr[k];
            int32_t* v = vals + row_ptr[k];
            c[0] = (int32_t)s.lead;
            stratified(r, s.a_lo, s.a_hi, s.na, c + 1);
            stratified(r, s.b_lo, s.b_hi, s.nb, c + 1 + s.na);
            v[0] = 1;
            for (int64_t j = 1; j < s.len; ++j) v[j] = (int32_t)(1 + r.below((uint64_t)p - 1));
        }
    });
    return 0;
}

}  // extern "C"
