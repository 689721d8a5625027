// field.cuh -- exact arithmetic in GF(p), p < 2^31, for the device kernels.
//
// Residues are stored reduced, as uint32 in [0, p).  The row kernels need one
// operation per pivot entry:  acc <- acc - m * v  (mod p), with the multiplier
// m fixed for a whole pivot row.  Two implementations, picked per prime the
// way the reference picks its 17-bit / 31-bit kernel families
// (src/io.c:710-729), but with the bounds of 32-bit lanes:
//
//   FieldSmall (p < 2^16): m * v < 2^32, reduced by a 32-bit Barrett step
//       with mu = floor(2^32 / p).  q = umulhi(t, mu) is floor(t/p) or one
//       less, so one conditional subtraction finishes.
//   FieldMont (2^16 <= p < 2^31, p odd): Montgomery multiplication with
//       R = 2^32.  The multiplier is moved into Montgomery form once per pivot
//       row (prep), so REDC(m R * v) = m v mod p with the data left in normal
//       form.  T + q p < 2 p 2^32 < 2^64 because p < 2^31.
//
// Nothing here uses floating point.
#pragma once
#include <stdint.h>

namespace gbgpu {

struct FieldSmall {
    uint32_t p;
    uint32_t mu;  // floor(2^32 / p)

    static FieldSmall make(uint32_t p_) {
        FieldSmall f;
        f.p = p_;
        f.mu = (uint32_t)((((uint64_t)1) << 32) / p_);
        return f;
    }
    __device__ __forceinline__ uint32_t prep(uint32_t m) const { return m; }
    __device__ __forceinline__ uint32_t mul(uint32_t a, uint32_t b) const {
        const uint32_t t = a * b;
        const uint32_t q = __umulhi(t, mu);
        uint32_t r = t - q * p;
        return r >= p ? r - p : r;
    }
    // acc - m * v mod p, with mp = prep(m)
    __device__ __forceinline__ uint32_t mulsub(uint32_t acc, uint32_t mp, uint32_t v) const {
        const uint32_t r = mul(mp, v);
        return acc >= r ? acc - r : acc + (p - r);
    }
    // a * b mod p for arbitrary a, b < p (normalisation)
    __device__ __forceinline__ uint32_t mulmod(uint32_t a, uint32_t b) const { return mul(a, b); }
    // x * a mod p with ap = prep(a)
    __device__ __forceinline__ uint32_t mulp(uint32_t x, uint32_t ap) const { return mul(ap, x); }
    // a x - m v mod p with one final reduction, ap = prep(a), mn = prep(p - m)
    // (a, p - m in [1, p), x, v in [0, p)): a x reduced to [0, 2p) by one
    // Barrett step, plus (p - m) v, stays below 2p - 1 + (p - 1)^2 = p^2 < 2^32
    __device__ __forceinline__ uint32_t ffsub(uint32_t x, uint32_t ap, uint32_t v,
                                              uint32_t mn) const {
        const uint32_t t = ap * x;
        const uint32_t s = t - __umulhi(t, mu) * p + mn * v;
        const uint32_t q = __umulhi(s, mu);
        const uint32_t r = s - q * p;
        return r >= p ? r - p : r;
    }
    // a^-1 = a^(p-2) mod p (0 < a < p), square and multiply
    __device__ __forceinline__ uint32_t inv(uint32_t a) const {
        uint32_t r = 1u, b = a;
        for (uint32_t e = p - 2u; e; e >>= 1) {
            if (e & 1u) r = mul(r, b);
            b = mul(b, b);
        }
        return r;
    }
};

struct FieldMont {
    uint32_t p;
    uint32_t pneg_inv;  // -p^-1 mod 2^32
    uint32_t r2;        // 2^64 mod p

    static FieldMont make(uint32_t p_) {
        FieldMont f;
        f.p = p_;
        // Newton iteration for p^-1 mod 2^32 (p odd): x <- x (2 - p x)
        uint32_t x = p_;  // correct to 3 bits
        for (int i = 0; i < 5; ++i) x *= 2u - p_ * x;
        f.pneg_inv = (uint32_t)(0u - x);
        const uint64_t r = ((((uint64_t)1) << 32) % p_);
        f.r2 = (uint32_t)((r * r) % p_);
        return f;
    }
    __device__ __forceinline__ uint32_t redc(uint64_t T) const {
        const uint32_t q = (uint32_t)T * pneg_inv;
        const uint64_t t = (T + (uint64_t)q * p) >> 32;
        const uint32_t r = (uint32_t)t;
        return r >= p ? r - p : r;
    }
    __device__ __forceinline__ uint32_t prep(uint32_t m) const {
        return redc((uint64_t)m * r2);  // m R mod p
    }
    __device__ __forceinline__ uint32_t mulsub(uint32_t acc, uint32_t mp, uint32_t v) const {
        const uint32_t r = redc((uint64_t)mp * v);
        return acc >= r ? acc - r : acc + (p - r);
    }
    __device__ __forceinline__ uint32_t mulmod(uint32_t a, uint32_t b) const {
        return redc((uint64_t)prep(a) * b);
    }
    // x * a mod p with ap = prep(a)
    __device__ __forceinline__ uint32_t mulp(uint32_t x, uint32_t ap) const {
        return redc((uint64_t)ap * x);
    }
    // a x - m v mod p with one reduction, ap = prep(a), mn = prep(p - m):
    // T = ap x + mn v < 2 p^2 and REDC(T) = (T + q p) / 2^32 < 2p (p < 2^31)
    __device__ __forceinline__ uint32_t ffsub(uint32_t x, uint32_t ap, uint32_t v,
                                              uint32_t mn) const {
        const uint64_t T = (uint64_t)ap * x + (uint64_t)mn * v;
        const uint32_t q = (uint32_t)T * pneg_inv;
        const uint32_t r = (uint32_t)((T + (uint64_t)q * p) >> 32);
        return r >= p ? r - p : r;
    }
    // a^-1 = a^(p-2) mod p (0 < a < p), square and multiply in Montgomery form
    __device__ __forceinline__ uint32_t inv(uint32_t a) const {
        uint32_t r = prep(1u), b = prep(a);
        for (uint32_t e = p - 2u; e; e >>= 1) {
            if (e & 1u) r = redc((uint64_t)r * b);
            b = redc((uint64_t)b * b);
        }
        return redc(r);
    }
};

// Inverse of a (0 < a < p) by the extended Euclidean algorithm, as the
// reference's mod_p_inverse_32 (src/tools.c:83-110).
__host__ __device__ inline uint32_t inverse_mod(uint32_t a, uint32_t p) {
    // extended Euclid; remainders stay below p < 2^31 (32-bit division),
    // Bezout coefficients stay within (-p, p)
    uint32_t r0 = p, r1 = a % p;
    int64_t s0 = 0, s1 = 1;
    while (r1 != 0) {
        const uint32_t q = r0 / r1;
        const uint32_t r2 = r0 - q * r1;
        r0 = r1;
        r1 = r2;
        const int64_t s2 = s0 - (int64_t)q * s1;
        s0 = s1;
        s1 = s2;
    }
    if (s0 < 0) s0 += p;
    return (uint32_t)s0;
}

}  // namespace gbgpu
