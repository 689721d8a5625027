// lift.cpp -- host-side Chinese remaindering for the multi-modular driver
// (gb_b200/multimod.py).  Plain C++ built by g++ into libgblift.so; no GPU.
//
// Every answer entry is an unsigned integer x in [0, M) held as `nl` 64-bit
// limbs, least significant first; M is the product of the primes added so
// far.  Adding a prime p with residues r makes every x the integer in
// [0, M p) that is x mod M and r mod p:
//
//     x <- x + M ((r - x) M^-1 mod p).
//
// x mod p is a dot product of the 32-bit halves of x with the powers
// 2^(32 j) mod p (each product < 2^64, summed in 128 bits, one final
// reduction), so no limb needs a division.
#include <stdint.h>

#include <algorithm>
#include <thread>
#include <vector>

namespace {

uint64_t mod128(unsigned __int128 v, uint32_t p) { return (uint64_t)(v % p); }

// entries [e0, e1) of gblift_crt_add
void crt_add_range(int64_t e0, int64_t e1, int32_t nl, uint64_t* x, const uint64_t* m,
                   int32_t m_len, const int64_t* r, uint32_t p, uint32_t minv,
                   const uint64_t* pw) {
    for (int64_t e = e0; e < e1; ++e) {
        uint64_t* xe = x + e * (int64_t)nl;
        unsigned __int128 acc = 0;
        for (int i = 0; i < m_len; ++i) {  // x < M: limbs at and above m_len are 0
            acc += (unsigned __int128)(xe[i] & 0xFFFFFFFFu) * pw[2 * i];
            acc += (unsigned __int128)(xe[i] >> 32) * pw[2 * i + 1];
        }
        const uint64_t xm = mod128(acc, p);
        const uint64_t re = (uint64_t)r[e] % p;
        const uint64_t t = (re + p - xm) % p * minv % p;
        // x += t M
        uint64_t carry = 0;
        for (int i = 0; i < m_len; ++i) {
            const unsigned __int128 v = (unsigned __int128)m[i] * t + xe[i] + carry;
            xe[i] = (uint64_t)v;
            carry = (uint64_t)(v >> 64);
        }
        for (int i = m_len; i < nl && carry; ++i) {
            const unsigned __int128 v = (unsigned __int128)xe[i] + carry;
            xe[i] = (uint64_t)v;
            carry = (uint64_t)(v >> 64);
        }
    }
}

}  // namespace

extern "C" {

// x: n entries of nl limbs; m: M as m_len limbs (m_len + 1 <= nl, M < 2^(64 m_len));
// r: n residues in [0, p); minv = M^-1 mod p.  Returns 0, or -1 when the
// limbs cannot hold M p (nl too small) or an argument is out of range.
int gblift_crt_add(int64_t n, int32_t nl, uint64_t* x, const uint64_t* m, int32_t m_len,
                   const int64_t* r, uint32_t p, uint32_t minv) {
    if (n < 0 || nl <= 0 || m_len < 1 || m_len + 1 > nl || p < 2) return -1;
    // 2^(32 j) mod p for the 2 m_len + 2 halves an entry below M p can have
    const int halves = 2 * (m_len + 1);
    std::vector<uint64_t> pw(halves);
    uint64_t w = 1 % p;
    for (int j = 0; j < halves; ++j) {
        pw[j] = w;
        w = (w << 32) % p;
    }
    // entries split over the host's threads (each entry is independent)
    const int64_t grain = 4096;
    const int64_t hw = std::max(1u, std::thread::hardware_concurrency());
    const int64_t nt = std::min<int64_t>(hw, (n + grain - 1) / grain);
    if (nt <= 1) {
        crt_add_range(0, n, nl, x, m, m_len, r, p, minv, pw.data());
    } else {
        std::vector<std::thread> pool;
        const int64_t per = (n + nt - 1) / nt;
        for (int64_t t = 0; t < nt; ++t) {
            const int64_t e0 = t * per, e1 = std::min(n, e0 + per);
            if (e0 < e1)
                pool.emplace_back(crt_add_range, e0, e1, nl, x, m, m_len, r, p, minv, pw.data());
        }
        for (auto& th : pool) th.join();
    }
    return 0;
}

}  // extern "C"
