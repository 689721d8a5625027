// tc_gemm.cu -- exact modular GEMM  D <- (D - A B) mod p  on the int8 tensor
// cores of sm_100a (tcgen05.mma kind::i8, TMA, TMEM), and its plain CUDA-core
// twin.
//
// Residues (uint32 in [0, p), p < 2^31 odd) are split into L unsigned bytes,
// a = sum_i a_i 2^(8i) with L = 1 (p < 2^8), 2 (< 2^16), 3 (< 2^24), 4.  Then
//   A B = sum_w 2^(8w) S_w,   S_w = sum_{i+j=w} A_i B_j,   w = 0 .. 2L-2,
// and every S_w is a u8 x u8 -> s32 tensor-core product accumulated in TMEM.
// At most L limb pairs share a weight, each product is <= 255^2, so a K panel
// of at most floor((2^31-1) / (L 255^2)) columns keeps every S_w below 2^31
// (kPanelBytes below).  After each panel the epilogue folds the weights,
//   v = sum_w REDC(S_w * (2^(8w) R mod p))   (Montgomery, R = 2^32),
// and updates D <- D - v mod p in place, so no partial sum ever leaves [0, p).
// The result is bit-identical to any exact evaluation of (D - A B) mod p.
//
// Pipeline (one CTA per 128 x BN output tile, 192 threads):
//   warp 0      TMA producer: L A-limb tiles (128 x 128 B) and L B-limb tiles
//               (BN x 128 B) per 128-byte K step into a STAGES-deep ring,
//               128-byte swizzle (the canonical K-major UMMA layout);
//   warp 1      TMEM allocation and MMA issue (one elected thread), stage
//               release through tcgen05.commit;
//   warps 2..5  epilogue: tcgen05.ld of the 2L-1 weight accumulators of its
//               32-lane TMEM quarter, fold, read-modify-write of D.
// Every mbarrier wait is bounded (clock64 budget); on expiry the CTA records
// GBGPU_ETIMEDOUT in *err, drains its in-flight copies and frees its TMEM.
// No cluster multicast is used anywhere.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "../../include/gbgpu.h"
#include "field.cuh"
#include "internal.h"
#include "tc_gemm.h"

namespace gbgpu {

// ---------------------------------------------------------------------------
// PTX wrappers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Wait for the phase of parity `parity` to complete, at most `budget` cycles.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long budget) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > budget) return false;
    }
    return true;
}
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"((uint64_t)map), "r"(x), "r"(y), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     bar)
                 : "memory");
}
__device__ __forceinline__ void tc_mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// 32 consecutive TMEM columns of this warp's 32 lanes (one row per thread)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, "
        "[%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// K-major operand tile with 128-byte swizzle: rows of 128 bytes, 8-row
// groups 1024 bytes apart (SBO), LBO unused (1), descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t smem_addr) {
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// ---------------------------------------------------------------------------
// Tile shapes (SHAPE):
//   TC_BIG   long K: 128 x BN tiles, one CTA per SM; one- and two-limb shapes
//            keep their accumulators twice (the next tile's MMAs run while the
//            epilogue drains the last) when 2 x NW x BN fits the 512 TMEM
//            columns: 128 x 256 for L = 1; L = 2 keeps 128 x 128 once (more
//            reuse per operand byte), L = 3, 4 keep 128 x 64 once;
//   TC_MID   two limbs, K up to 1536: 128 x 64 tiles, accumulators twice;
//   TC_SMALL K <= 256, one or two limbs: 128 x 128/64 tiles, two CTAs per SM
//            (TMEM <= 256 columns each), so one CTA's loads and MMAs overlap
//            the other's epilogue.
constexpr int TC_BIG = 0, TC_SMALL = 1, TC_MID = 2;

template <int L, int SHAPE = TC_BIG>
struct TcCfg {
    static constexpr bool SMALL = SHAPE == TC_SMALL;
    static constexpr int BM = 128;
    static constexpr int BK = 128;  // bytes of K per stage (one swizzle row)
    static constexpr int BN =
        SMALL ? (L == 1 ? 128 : 64) : (L == 1 ? 256 : (L == 2 && SHAPE == TC_BIG ? 128 : 64));
    static constexpr int NW = 2 * L - 1;
    // accumulator sets in TMEM (see the shapes above)
    static constexpr int ACC_BUFS = (!SMALL && 2 * (2 * L - 1) * BN <= 512) ? 2 : 1;
    static constexpr int A_BYTES = BM * BK;
    static constexpr int B_BYTES = BN * BK;
    static constexpr int STAGE_BYTES = L * (A_BYTES + B_BYTES);
    static constexpr int STAGES = SMALL ? 1 : (L == 1 ? 4 : (L == 2 ? (BN == 128 ? 3 : 4) : 2));
    static constexpr int ACC_COLS = ACC_BUFS * NW * BN;
    static constexpr int TMEM_COLS =
        ACC_COLS <= 64 ? 64 : (ACC_COLS <= 128 ? 128 : (ACC_COLS <= 256 ? 256 : 512));
    // epilogue warps: two per TMEM lane quarter (each half of the columns) for
    // the one-CTA-per-SM shapes with one or two limbs, one otherwise
    static constexpr int EPI_WARPS = (!SMALL && L <= 2) ? 8 : 4;
    static constexpr int THREADS = 64 + 32 * EPI_WARPS;
    // epilogue staging: a 32 x 32 block per epilogue warp (XOR-swizzled
    // columns) and the D row indices of its 32 rows
    static constexpr int STG_BYTES = EPI_WARPS * 32 * 32 * 4;
    // (64-bit pointers when there is room, 32-bit row indices otherwise)
    static constexpr bool ROW_PTRS = EPI_WARPS == 4;
    static constexpr int ROWP_BYTES = EPI_WARPS * 32 * (ROW_PTRS ? 8 : 4);
    static constexpr int BAR_OFF = STAGES * STAGE_BYTES;
    static constexpr int STG_OFF = BAR_OFF + 256;
    static constexpr int ROWP_OFF = STG_OFF + STG_BYTES;
    static constexpr int USED_BYTES = ROWP_OFF + ROWP_BYTES + 1024 /*align*/;
    // the small shape asks for enough shared memory that at most two CTAs
    // share an SM (their TMEM allocations, 2 x 256 columns, then always fit)
    static constexpr int SMEM_BYTES = SMALL && USED_BYTES < 100 * 1024 ? 100 * 1024 : USED_BYTES;
    static constexpr int MIN_CTAS = SMALL ? 2 : 1;
    // K bytes per panel: L * 255^2 * K < 2^31
    static constexpr int PANEL_KB = L == 1 ? 256 : (L == 2 ? 128 : (L == 3 ? 85 : 64));
    static constexpr uint32_t IDESC = (2u << 4)                      // D = s32
                                      | (0u << 7) | (0u << 10)       // A, B = u8
                                      | ((uint32_t)(BN >> 3) << 17)  // N
                                      | ((uint32_t)(BM >> 4) << 24); // M
    static_assert(!SMALL || L <= 2, "small tiles for one or two limbs only");
    static_assert(!SMALL || 2 * TMEM_COLS <= 512, "two small CTAs share the TMEM");
    static_assert(SMEM_BYTES <= 227 * 1024, "shared memory");
    static_assert(ACC_COLS <= 512, "TMEM columns");
};

// tiles of one batch item are visited in groups of TC_GROUP_M row tiles, all
// column tiles of a group before the next, so that the B tiles of a column are
// reused from L2 by the row tiles of the group
constexpr int TC_GROUP_M = 8;

struct TcParams {
    uint32_t* D;
    int64_t ldd, sD;
    const int32_t* d_rows;  // optional: row m of D is D + d_rows[m] ldd (< 0: not written)
    int64_t sDr;
    int32_t M, N, Mp, Np, nkb, nkbp, batch;
    // nonzero flags of the 128-row x 128-byte A tiles ([Mp/128][nkbp]) and of the
    // BN-row x 128-byte B tiles ([Np/BN][nkbp], nkbp = nkb rounded up to 64, the
    // padding zero); a K step where either tile is
    // zero contributes nothing and is skipped (NULL: no skipping)
    const uint8_t* fa;
    const uint8_t* fb;
    unsigned long long* steps;  // optional: K steps executed, summed over tiles
    uint32_t p, pneg_inv;
    uint32_t mu;     // floor(2^32 / p)
    uint32_t cw[7];  // 2^(8w) R mod p
    int32_t* err;
    long long budget;
};

template <int L, int SHAPE>
__global__ void __launch_bounds__(TcCfg<L, SHAPE>::THREADS, TcCfg<L, SHAPE>::MIN_CTAS)
k_tc_submul(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
            const TcParams prm) {
    using C = TcCfg<L, SHAPE>;
    extern __shared__ uint8_t smem_raw[];
    // 1024-byte aligned tile region (shared-window address)
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    uint8_t* gbase = smem_raw + (base - raw);
    uint64_t* bars = (uint64_t*)(gbase + C::BAR_OFF);
    // bars: full[STAGES], empty[STAGES], tmem_full[ACC_BUFS], tmem_empty[ACC_BUFS];
    // then tmem slot, abort flag
    const uint32_t bar0 = smem_u32(bars);
    auto full_bar = [&](int s) { return bar0 + 8u * s; };
    auto empty_bar = [&](int s) { return bar0 + 8u * (C::STAGES + s); };
    auto tfull_bar = [&](int b) { return bar0 + 8u * (2 * C::STAGES + b); };
    auto tempty_bar = [&](int b) { return bar0 + 8u * (2 * C::STAGES + C::ACC_BUFS + b); };
    volatile uint32_t* tmem_slot = (volatile uint32_t*)(bars + 2 * C::STAGES + 2 * C::ACC_BUFS);
    volatile int* abort_flag = (volatile int*)(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nkb = prm.nkb;
    const int tiles_m = prm.Mp / C::BM, tiles_n = prm.Np / C::BN;
    const int per_z = tiles_m * tiles_n;
    const int total = per_z * prm.batch;
    // tile t -> batch item z, row tile mt, column tile nt (grouped raster)
    auto coords = [&](int t, int& z, int& mt, int& nt) {
        z = t / per_z;
        const int r = t - z * per_z;
        const int span = TC_GROUP_M * tiles_n;
        const int first_m = (r / span) * TC_GROUP_M;
        const int gm = min(TC_GROUP_M, tiles_m - first_m);
        const int rr = r - (r / span) * span;
        mt = first_m + rr % gm;
        nt = rr / gm;
    };
    // flags of the tile's A row block and B column block (NULL: all live)
    const int nkbp = prm.nkbp;
    auto flag_ptrs = [&](int z, int mt, int nt, const uint8_t*& fa, const uint8_t*& fb) {
        fa = prm.fa ? prm.fa + ((size_t)z * tiles_m + mt) * nkbp : nullptr;
        // B flags are kept per 64 rows of B's planes: the tile's BN / 64 rows
        fb = prm.fb ? prm.fb + ((size_t)z * (prm.Np / 64) + (size_t)nt * (C::BN / 64)) * nkbp
                    : nullptr;
    };
    // live K steps [64 ch, 64 ch + 64) of a tile as a bit mask, from 16-byte
    // loads of the A flag row and of the OR of the tile's B flag rows (flags
    // are 0 or 1 bytes)
    auto live_mask = [&](const uint8_t* fa, const uint8_t* fb, int ch) -> uint64_t {
        uint64_t msk = 0;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int kb0 = ch * 64 + v * 16;
            if (kb0 >= nkb) break;  // padding only
            uint4 a = make_uint4(0x01010101u, 0x01010101u, 0x01010101u, 0x01010101u);
            uint4 b = a;
            if (fa) a = *(const uint4*)(fa + kb0);
            if (fb) {
                b = *(const uint4*)(fb + kb0);
#pragma unroll
                for (int r = 1; r < C::BN / 64; ++r) {
                    const uint4 o = *(const uint4*)(fb + (size_t)r * nkbp + kb0);
                    b.x |= o.x;
                    b.y |= o.y;
                    b.z |= o.z;
                    b.w |= o.w;
                }
            }
            const uint32_t w[4] = {a.x & b.x, a.y & b.y, a.z & b.z, a.w & b.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint32_t x = w[j];
                const uint32_t bits = (x & 1u) | ((x >> 7) & 2u) | ((x >> 14) & 4u) | ((x >> 21) & 8u);
                msk |= (uint64_t)bits << (v * 16 + j * 4);
            }
        }
        if (!fa && !fb) {
            // no flags at all: every real K step is live
            const int rem = nkb - ch * 64;
            msk = rem >= 64 ? ~0ull : (rem > 0 ? ((1ull << rem) - 1ull) : 0ull);
        } else if (nkb - ch * 64 < 64) {
            const int rem = nkb - ch * 64;
            msk &= rem > 0 ? ((1ull << rem) - 1ull) : 0ull;
        }
        return msk;
    };
    const int nch = (nkb + 63) / 64;
    auto live_steps = [&](const uint8_t* fa, const uint8_t* fb) {
        int n_it = 0;
        for (int ch = 0; ch < nch; ++ch) n_it += __popcll(live_mask(fa, fb, ch));
        return n_it;
    };

    if (threadIdx.x == 0) {
        for (int s = 0; s < C::STAGES; ++s) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), 1);
        }
        for (int b = 0; b < C::ACC_BUFS; ++b) {
            mbar_init(tfull_bar(b), 1);
            mbar_init(tempty_bar(b), C::EPI_WARPS);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32((const void*)tmem_slot)),
                     "r"((uint32_t)C::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    // Every role walks the same tile sequence and skips the tiles whose
    // product is zero.  The operand ring and the accumulator phases continue
    // across tiles, so the producer fetches the next tile while the epilogue
    // drains the current one.
    if (warp == 0) {
        if (lane == 0) {
            // ---- producer ----
            int it = 0;
            bool stop = false;
            for (int t = blockIdx.x; t < total && !stop; t += gridDim.x) {
                int z, mt, nt;
                coords(t, z, mt, nt);
                const uint8_t *fa, *fb;
                flag_ptrs(z, mt, nt, fa, fb);
                const int m0 = mt * C::BM, n0 = nt * C::BN;
                int n_tile = 0;
                for (int ch = 0; ch < nch && !stop; ++ch) {
                  uint64_t msk = live_mask(fa, fb, ch);
                  while (msk) {
                    const int kb = ch * 64 + __ffsll((long long)msk) - 1;
                    msk &= msk - 1;
                    const int s = it % C::STAGES;
                    const uint32_t ph = (it / C::STAGES) & 1;
                    if (*abort_flag || !mbar_wait(empty_bar(s), ph ^ 1, prm.budget)) {
                        *abort_flag = 1;
                        stop = true;
                        break;
                    }
                    mbar_expect_tx(full_bar(s), C::STAGE_BYTES);
                    const uint32_t st = base + s * C::STAGE_BYTES;
                    for (int l = 0; l < L; ++l)
                        tma_load_2d(st + l * C::A_BYTES, &mapA, kb * C::BK,
                                    (z * L + l) * prm.Mp + m0, full_bar(s));
                    for (int l = 0; l < L; ++l)
                        tma_load_2d(st + L * C::A_BYTES + l * C::B_BYTES, &mapB, kb * C::BK,
                                    (z * L + l) * prm.Np + n0, full_bar(s));
                    ++it;
                    ++n_tile;
                  }
                }
                if (prm.steps && n_tile) atomicAdd(prm.steps, (unsigned long long)n_tile);
            }
            // on abort, let the copies already issued land before the CTA exits
            for (int q = it > C::STAGES ? it - C::STAGES : 0; q < it; ++q)
                mbar_wait(full_bar(q % C::STAGES), (q / C::STAGES) & 1, prm.budget);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer ----
            int it = 0, pc = 0;  // k steps and accumulator panels so far
            bool stop = false;
            for (int t = blockIdx.x; t < total && !stop; t += gridDim.x) {
                int z, mt, nt;
                coords(t, z, mt, nt);
                const uint8_t *fa, *fb;
                flag_ptrs(z, mt, nt, fa, fb);
                const int n_it = live_steps(fa, fb);
                int j = 0;
                for (int ch = 0; ch < nch && !stop; ++ch) {
                  uint64_t msk = live_mask(fa, fb, ch);
                  while (msk) {
                    msk &= msk - 1;
                    const int s = it % C::STAGES;
                    const uint32_t ph = (it / C::STAGES) & 1;
                    const int pk = j % C::PANEL_KB;
                    const int ab = pc % C::ACC_BUFS, au = pc / C::ACC_BUFS;
                    if (pk == 0 && au > 0) {
                        // this accumulator set is free once the epilogue read its last panel
                        if (*abort_flag || !mbar_wait(tempty_bar(ab), (au - 1) & 1, prm.budget)) {
                            *abort_flag = 1;
                            stop = true;
                            break;
                        }
                    }
                    if (*abort_flag || !mbar_wait(full_bar(s), ph, prm.budget)) {
                        *abort_flag = 1;
                        stop = true;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t st = base + s * C::STAGE_BYTES;
                    // the descriptors of the stage's operands: the start address
                    // field holds address / 16 in its low 14 bits, and every
                    // operand of the stage lies below 2^18 bytes, so an offset
                    // adds to the descriptor without a carry out of the field
                    const uint64_t dst = umma_desc_sw128(st);
#pragma unroll
                    for (int i = 0; i < L; ++i) {
#pragma unroll
                        for (int jj = 0; jj < L; ++jj) {
                            const int w = i + jj;
                            const bool first_pair = (i == (w > L - 1 ? w - (L - 1) : 0));
#pragma unroll
                            for (int kk = 0; kk < C::BK / 32; ++kk) {
                                const uint64_t ad = dst + (uint64_t)((i * C::A_BYTES + kk * 32) >> 4);
                                const uint64_t bd =
                                    dst + (uint64_t)((L * C::A_BYTES + jj * C::B_BYTES + kk * 32) >> 4);
                                const uint32_t acc = (pk == 0 && kk == 0 && first_pair) ? 0u : 1u;
                                tc_mma_i8(tmem + (uint32_t)(ab * C::NW * C::BN + w * C::BN), ad, bd,
                                          C::IDESC, acc);
                            }
                        }
                    }
                    tc_commit(empty_bar(s));
                    if (pk == C::PANEL_KB - 1 || j == n_it - 1) {
                        tc_commit(tfull_bar(ab));
                        ++pc;
                    }
                    ++it;
                    ++j;
                  }
                }
            }
        }
    } else {
        // ---- epilogue: warps 2.., TMEM lane quarter warp % 4, column half ----
        // Thread `lane` folds row q*32+lane of the tile; the 32 x 32 result
        // block goes through shared memory so that the read-modify-write of D
        // runs along rows (one 128-byte row segment per warp instruction).
        const int e = warp - 2;
        const int q = warp & 3;
        constexpr int HALVES = C::EPI_WARPS / 4;
        constexpr int COLS = C::BN / HALVES;  // columns of this warp
        const int cbeg = (e / 4) * COLS;
        const int row = q * 32 + lane;
        const uint32_t p = prm.p;
        uint32_t* stg = (uint32_t*)(gbase + C::STG_OFF + (size_t)e * 32 * 32 * 4);
        uint8_t* rowb = gbase + C::ROWP_OFF + (size_t)e * 32 * (C::ROW_PTRS ? 8 : 4);
        int32_t* rowi = (int32_t*)rowb;
        uint32_t** rowp = (uint32_t**)rowb;
        int pc = 0;
        bool stop = false;
        for (int t = blockIdx.x; t < total && !stop; t += gridDim.x) {
            int z, mt, nt;
            coords(t, z, mt, nt);
            const uint8_t *fa, *fb;
            flag_ptrs(z, mt, nt, fa, fb);
            const int n_it = live_steps(fa, fb);
            if (n_it == 0) continue;  // A B is zero on this tile: D stays as it is
            const int npanels = (n_it + C::PANEL_KB - 1) / C::PANEL_KB;
            const int m0 = mt * C::BM, n0 = nt * C::BN;
            const int gm = m0 + row;
            uint32_t* Dz = prm.D + (size_t)z * prm.sD;
            bool rows_here;  // any of this warp's 32 rows is written
            {
                int32_t ri = -1;
                if (gm < prm.M) ri = prm.d_rows ? prm.d_rows[(size_t)z * prm.sDr + gm] : gm;
                __syncwarp();  // the previous tile's readers are done with the rows
                if constexpr (C::ROW_PTRS)
                    rowp[lane] = ri >= 0 ? Dz + (size_t)ri * prm.ldd : nullptr;
                else
                    rowi[lane] = ri;
                rows_here = __any_sync(0xffffffffu, ri >= 0);
                __syncwarp();  // the row table is visible to the whole warp
            }
            // row r of the tile in D (nullptr: not written)
            auto drow = [&](int r) -> uint32_t* {
                if constexpr (C::ROW_PTRS) {
                    return rowp[r];
                } else {
                    const int32_t ri = rowi[r];
                    return ri >= 0 ? Dz + (size_t)ri * prm.ldd : nullptr;
                }
            };
            // D values of a 32 x 32 block (row r, this lane's column)
            auto load_d = [&](int c0, uint32_t (&dv)[32]) {
                const int gn = n0 + c0 + lane;
                const bool col_ok = gn < prm.N;
#pragma unroll
                for (int r = 0; r < 32; ++r) {
                    const uint32_t* rp = drow(r);
                    dv[r] = (rp && col_ok) ? rp[gn] : 0u;
                }
            };
            for (int panel = 0; panel < npanels; ++panel, ++pc) {
                const int ab = pc % C::ACC_BUFS, au = pc / C::ACC_BUFS;
                const uint32_t acc_base = (uint32_t)(ab * C::NW * C::BN);
                // the first block's D values do not depend on the accumulators:
                // their loads are in flight while the MMAs finish (this lane
                // wrote the same addresses in the previous panel, if any).
                // Three and four limbs have no registers to spare for it; with
                // two CTAs per SM the other CTA's epilogue covers the wait.
                constexpr bool EARLY_D = L <= 2 && !C::SMALL;
                uint32_t dv[32];
                if constexpr (EARLY_D) {
                    if (rows_here) load_d(cbeg, dv);
                }
                bool ok = true;
                if (lane == 0) ok = !*abort_flag && mbar_wait(tfull_bar(ab), au & 1, prm.budget);
                ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
                if (!ok) {
                    if (lane == 0) *abort_flag = 1;
                    stop = true;
                    break;
                }
                tc_fence_after();
                // a warp with no row to write keeps only its place in the
                // accumulator handshake
                for (int c0 = cbeg; rows_here && c0 < cbeg + COLS; c0 += 32) {
                    const int gn = n0 + c0 + lane;
                    const bool col_ok = gn < prm.N;
                    // D values of the later blocks, issued before the fold
                    if (!EARLY_D || c0 != cbeg) load_d(c0, dv);
                    uint32_t v[32];
                    if constexpr (L <= 3) {
                        // one Montgomery reduction of the weighted sum:
                        // T = sum_w S_w (2^(8w) R mod p) < (2L - 1) 2^31 p, so
                        // (T + q p) / 2^32 < 2^32, then one Barrett step
                        uint64_t T[32];
#pragma unroll
                        for (int w = 0; w < C::NW; ++w) {
                            uint32_t a[32];
                            tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + acc_base +
                                          (uint32_t)(w * C::BN + c0),
                                      a);
                            const uint32_t cw = prm.cw[w];
#pragma unroll
                            for (int j = 0; j < 32; ++j)
                                T[j] = (w == 0 ? 0ull : T[j]) + (uint64_t)a[j] * cw;
                        }
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            const uint32_t qq = (uint32_t)T[j] * prm.pneg_inv;
                            const uint32_t t = (uint32_t)((T[j] + (uint64_t)qq * p) >> 32);
                            const uint32_t r = t - __umulhi(t, prm.mu) * p;
                            v[j] = r >= p ? r - p : r;
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < 32; ++j) v[j] = 0;
#pragma unroll
                        for (int w = 0; w < C::NW; ++w) {
                            uint32_t a[32];
                            tmem_ld32(tmem + ((uint32_t)(q * 32) << 16) + acc_base +
                                          (uint32_t)(w * C::BN + c0),
                                      a);
                            const uint32_t cw = prm.cw[w];
#pragma unroll
                            for (int j = 0; j < 32; ++j) {
                                const uint64_t T = (uint64_t)a[j] * cw;
                                const uint32_t qq = (uint32_t)T * prm.pneg_inv;
                                uint32_t r = (uint32_t)((T + (uint64_t)qq * p) >> 32);
                                r = r >= p ? r - p : r;
                                const uint32_t sum = v[j] + r;
                                v[j] = sum >= p ? sum - p : sum;
                            }
                        }
                    }
                    // stage (row lane, column j) at [lane][j ^ lane]
#pragma unroll
                    for (int j = 0; j < 32; ++j) stg[lane * 32 + (j ^ lane)] = v[j];
                    __syncwarp();
#pragma unroll
                    for (int r = 0; r < 32; ++r) {
                        uint32_t* rp = drow(r);
                        if (rp && col_ok) {
                            const uint32_t vv = stg[r * 32 + (lane ^ r)];
                            const uint32_t d = dv[r];
                            rp[gn] = d >= vv ? d - vv : d + (p - vv);
                        }
                    }
                    __syncwarp();
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(tempty_bar(ab));
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag) atomicExch(prm.err, GBGPU_ETIMEDOUT);
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"((uint32_t)C::TMEM_COLS)
                     : "memory");
    }
}

// ---------------------------------------------------------------------------
// Limb planes of both operands and their tile flags, one launch per GEMM.
//
// A part (blocks [0, a_blocks)): one 128-row x 128-column tile of A per
// block; out[l][m][k] = byte l of A[m][k], zero padded; row m of A is
// A + a_rows[m] lda when a_rows is given (negative: a zero row).  Every item
// is 16 consecutive k of one row (one 16-byte store per limb); with `vec` (A
// and its row and batch strides 16-byte aligned) a full item is read as four
// 16-byte loads.  The block writes its tile flag fa[mt][kb] (0 or 1).
//
// B part (the other blocks): transposing split, out[l][n][k] = byte l of
// B[k][n]; row k of B is B + b_rows[k] ldb when b_rows is given (negative: a
// zero row).  One 128 (k) x 64 (n) tile per block: rows of B are read 256
// bytes per pair of warps; the bytes go to shared memory as [l][n][k] (rows
// padded to 132 bytes: conflict-free in both phases) and leave as whole
// 128-byte k-rows of every n, four threads per row.  The block writes its flag
// fb[n / 64][kb]; the GEMM ORs the flags of the 64-row groups of its tile.
// With nrange (see TcGemmArgs::b_nrange) a tile outside its rows' column range
// is not read: it is written as zeros when another part of its bn-wide GEMM
// tile is live, and not at all otherwise (the GEMM never loads it).
//
// Every flag of the GEMM is written here, so nothing clears them first.
constexpr int SPLIT_ROW = 132;
struct SplitArgs {
    const uint32_t* A;
    int64_t lda, sA;
    const int32_t* a_rows;
    int64_t sAr;
    int32_t M, K, Mp, Kp, L;
    uint8_t* Ap;
    uint8_t* fa;
    int32_t nkbp, vec;
    const uint32_t* B;
    int64_t ldb, sB;
    const int32_t* b_rows;
    int64_t sBr;
    int32_t N, Np, bn;
    uint8_t* Bp;
    uint8_t* fb;
    const int2* nrange;
    int32_t a_blocks;  // (Mp / 128) (Kp / 128)
};

__global__ void __launch_bounds__(256) k_split_ab(const SplitArgs a) {
    extern __shared__ uint8_t split_smem[];  // [L][64][SPLIT_ROW] bytes (B part)
    __shared__ const uint32_t* rowp[128];
    const int z = blockIdx.z;  // batch item
    const int nkb = a.Kp / 128;
    const int L = a.L;
    if ((int)blockIdx.x < a.a_blocks) {
        // ---- A part ----
        const int mt = blockIdx.x / nkb, kbi = blockIdx.x % nkb;
        const uint32_t* A = a.A + (size_t)z * a.sA;
        const int32_t* a_rows = a.a_rows ? a.a_rows + (size_t)z * a.sAr : nullptr;
        uint8_t* out = a.Ap + (size_t)z * L * a.Mp * a.Kp;
        uint32_t any = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int item = threadIdx.x + 256 * q;
            const int m = mt * 128 + (item >> 3);
            const int k = kbi * 128 + (item & 7) * 16;
            int64_t src = -1;
            if (m < a.M) src = a_rows ? (int64_t)a_rows[m] : (int64_t)m;
            const uint32_t* row = src >= 0 ? A + (size_t)src * a.lda : nullptr;
            uint32_t v[16];
            if (a.vec && row && k + 16 <= a.K) {
                const uint4* r4 = (const uint4*)(row + k);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const uint4 w = r4[u];
                    v[4 * u] = w.x;
                    v[4 * u + 1] = w.y;
                    v[4 * u + 2] = w.z;
                    v[4 * u + 3] = w.w;
                }
            } else {
#pragma unroll
                for (int e = 0; e < 16; ++e) v[e] = (row && k + e < a.K) ? row[k + e] : 0u;
            }
#pragma unroll
            for (int e = 0; e < 16; ++e) any |= v[e];
            for (int l = 0; l < L; ++l) {
                uint32_t w[4];
#pragma unroll
                for (int jj = 0; jj < 4; ++jj)
                    w[jj] = ((v[4 * jj] >> (8 * l)) & 255u) |
                            (((v[4 * jj + 1] >> (8 * l)) & 255u) << 8) |
                            (((v[4 * jj + 2] >> (8 * l)) & 255u) << 16) |
                            (((v[4 * jj + 3] >> (8 * l)) & 255u) << 24);
                *(uint4*)(out + ((size_t)l * a.Mp + m) * a.Kp + k) =
                    make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
        any = __syncthreads_or(any != 0);
        if (threadIdx.x == 0)
            a.fa[((size_t)z * (a.Mp / 128) + mt) * a.nkbp + kbi] = any ? 1 : 0;
        return;
    }
    // ---- B part ----
    const int bq = blockIdx.x - a.a_blocks;
    const int nx = bq % (a.Np / 64), kbi = bq / (a.Np / 64);
    const int k0 = kbi * 128, n0 = nx * 64;
    const uint32_t* B = a.B + (size_t)z * a.sB;
    const int32_t* b_rows = a.b_rows ? a.b_rows + (size_t)z * a.sBr : nullptr;
    uint8_t* out = a.Bp + (size_t)z * L * a.Np * a.Kp;
    uint8_t* flag = a.fb + ((size_t)z * (a.Np / 64) + nx) * a.nkbp + kbi;
    if (a.nrange) {  // uniform over the block
        const int2 rg = k0 < a.K ? a.nrange[kbi] : make_int2(1, 0);
        const int t0 = (n0 / a.bn) * a.bn;
        const bool tile_live = !(rg.y < rg.x || t0 + a.bn <= rg.x || t0 > rg.y);
        if (!tile_live || n0 + 64 <= rg.x || n0 > rg.y) {
            if (threadIdx.x == 0) *flag = 0;
            if (!tile_live) return;
            // zeros: 64 k-rows of 128 bytes per limb, four threads per row
            const int nn = threadIdx.x >> 2, part = threadIdx.x & 3;
            for (int l = 0; l < L; ++l) {
                uint4* dst = (uint4*)(out + ((size_t)l * a.Np + n0 + nn) * a.Kp + k0 + 32 * part);
                dst[0] = make_uint4(0u, 0u, 0u, 0u);
                dst[1] = make_uint4(0u, 0u, 0u, 0u);
            }
            return;
        }
    }
    if (threadIdx.x < 128) {
        const int k = k0 + threadIdx.x;
        int64_t src = -1;
        if (k < a.K) src = b_rows ? (int64_t)b_rows[k] : (int64_t)k;
        rowp[threadIdx.x] = src >= 0 ? B + (size_t)src * a.ldb : nullptr;
    }
    __syncthreads();
    uint32_t any = 0;
    {
        const int c = threadIdx.x & 63, r0 = threadIdx.x >> 6;  // 4 k rows per pass
        const int n = n0 + c;
        // all 32 loads first (no shared-memory store between them)
        uint32_t v[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const uint32_t* rp = rowp[r0 + 4 * i];
            v[i] = (rp && n < a.N) ? rp[n] : 0u;
        }
        for (int l = 0; l < L; ++l) {
            uint8_t* dst = split_smem + ((size_t)l * 64 + c) * SPLIT_ROW + r0;
#pragma unroll
            for (int i = 0; i < 32; ++i) dst[4 * i] = (uint8_t)(v[i] >> (8 * l));
        }
#pragma unroll
        for (int i = 0; i < 32; ++i) any |= v[i];
    }
    any = __syncthreads_or(any != 0);
    // thread: n = tid / 4, bytes [32 part, 32 part + 32) of the 128-byte k row
    const int nn = threadIdx.x >> 2, part = threadIdx.x & 3;
    const int n = n0 + nn;  // n < Np and k0 + 128 <= Kp by the grid
    for (int l = 0; l < L; ++l) {
        const uint32_t* src =
            (const uint32_t*)(split_smem + ((size_t)l * 64 + nn) * SPLIT_ROW + 32 * part);
        uint32_t w[8];
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) w[jj] = src[jj];
        uint4* dst = (uint4*)(out + ((size_t)l * a.Np + n) * a.Kp + k0 + 32 * part);
        dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
        dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
    }
    if (threadIdx.x == 0) *flag = any ? 1 : 0;
}

// row index lists of the plain GEMM (see TcGemmArgs)
struct RowLists {
    const int32_t *a, *b, *d;
    int64_t sa, sb, sd;
};

// ---------------------------------------------------------------------------
// plain CUDA-core modular GEMM: 64 x 64 tile per 256 threads, 4 x 4 per thread;
// b is split into 16-bit halves so 2^16 products fit the u64 partial sums.
__global__ void __launch_bounds__(256)
k_plain_submul(const uint32_t* __restrict__ A, int64_t lda, const uint32_t* __restrict__ B,
               int64_t ldb, uint32_t* D, int64_t ldd, int32_t M, int32_t N, int32_t K,
               int64_t strideA, int64_t strideB, int64_t strideD, RowLists rl, FieldMont f) {
    A += (size_t)blockIdx.z * strideA;
    B += (size_t)blockIdx.z * strideB;
    D += (size_t)blockIdx.z * strideD;
    const int32_t* a_rows = rl.a ? rl.a + (size_t)blockIdx.z * rl.sa : nullptr;
    const int32_t* b_rows = rl.b ? rl.b + (size_t)blockIdx.z * rl.sb : nullptr;
    const int32_t* d_rows = rl.d ? rl.d + (size_t)blockIdx.z * rl.sd : nullptr;
    __shared__ uint32_t sA[16][64 + 1];
    __shared__ uint32_t sB[16][64 + 1];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    // row index of A row m / B row k (negative: zero row)
    auto arow = [&](int m) -> int64_t { return a_rows ? (int64_t)a_rows[m] : (int64_t)m; };
    auto brow = [&](int k) -> int64_t { return b_rows ? (int64_t)b_rows[k] : (int64_t)k; };
    uint64_t lo[4][4], hi[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) lo[i][j] = hi[i][j] = 0;
    int since = 0;
    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int t = threadIdx.x; t < 16 * 64; t += 256) {
            const int kk = t & 15, mm = t >> 4;
            const int m = m0 + mm, k = k0 + kk;
            const int64_t ra = (m < M && k < K) ? arow(m) : -1;
            sA[kk][mm] = ra >= 0 ? A[(size_t)ra * lda + k] : 0u;
            const int nn = t & 63, kr = t >> 6;
            const int n = n0 + nn, k2 = k0 + kr;
            const int64_t rb = (n < N && k2 < K) ? brow(k2) : -1;
            sB[kr][nn] = rb >= 0 ? B[(size_t)rb * ldb + n] : 0u;
        }
        __syncthreads();
#pragma unroll 4
        for (int kk = 0; kk < 16; ++kk) {
            uint32_t a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = sA[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = sB[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    lo[i][j] += (uint64_t)a[i] * (b[j] & 0xFFFFu);
                    hi[i][j] += (uint64_t)a[i] * (b[j] >> 16);
                }
        }
        __syncthreads();
        since += 16;
        if (since >= 32768) {  // keep the partial sums far from 2^64
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    lo[i][j] %= f.p;
                    hi[i][j] %= f.p;
                }
            since = 0;
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = m0 + ty * 4 + i;
        if (m >= M) continue;
        const int64_t rd = d_rows ? (int64_t)d_rows[m] : (int64_t)m;
        if (rd < 0) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = n0 + tx * 4 + j;
            if (n >= N) continue;
            const uint64_t h = (hi[i][j] % f.p) << 16;
            const uint32_t v = (uint32_t)((lo[i][j] % f.p + h % f.p) % f.p);
            const uint32_t d = D[(size_t)rd * ldd + n];
            D[(size_t)rd * ldd + n] = d >= v ? d - v : d + (f.p - v);
        }
    }
}

// ---------------------------------------------------------------------------
// host side
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

static int make_map(CUtensorMap* map, const void* base, int64_t inner, int64_t rows,
                    int box_inner, int box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) {
        set_error("cuTensorMapEncodeTiled unavailable");
        return GBGPU_ENODEV;
    }
    cuuint64_t dims[2] = {(cuuint64_t)inner, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)inner};
    cuuint32_t box[2] = {(cuuint32_t)box_inner, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides,
                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed");
        return GBGPU_ECUDA;
    }
    return GBGPU_OK;
}

static thread_local GemmProfile* g_profile = nullptr;
GemmProfile* gemm_profile() { return g_profile; }
void set_gemm_profile(GemmProfile* p) { g_profile = p; }

int limbs_for(uint32_t p) {
    if (p < (1u << 8)) return 1;
    if (p < (1u << 16)) return 2;
    if (p < (1u << 24)) return 3;
    return 4;
}

// SMs of the current device (persistent GEMM grid)
static int num_sms() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
        return 148;
    return n;
}

template <int L, int SHAPE>
static int tc_run(const TcGemmArgs& g, uint8_t* planes, cudaStream_t s, int32_t* err,
                  long long* launches) {
    using Cfg = TcCfg<L, SHAPE>;
    const int32_t Mp = (g.M + Cfg::BM - 1) / Cfg::BM * Cfg::BM;
    const int32_t Np = (g.N + Cfg::BN - 1) / Cfg::BN * Cfg::BN;
    const int32_t Kp = (g.K + Cfg::BK - 1) / Cfg::BK * Cfg::BK;
    const int32_t nb = g.batch;
    uint8_t* Ap = planes;                                    // [nb][L][Mp][Kp]
    uint8_t* Bp = planes + (size_t)nb * L * Mp * Kp;         // [nb][L][Np][Kp]
    const int32_t nkb = Kp / Cfg::BK;
    const int32_t nkbp = (nkb + 63) / 64 * 64;
    uint8_t* fa = Bp + (size_t)nb * L * Np * Kp;             // [nb][Mp/128][nkbp]
    uint8_t* fb = fa + (size_t)nb * (Mp / Cfg::BM) * nkbp;   // [nb][Np/64][nkbp]
    GemmProfile* prof = gemm_profile();
    if (prof) {
        cudaEvent_t es = nullptr;
        cudaEventCreate(&es);
        cudaEventRecord(es, s);
        prof->split_events.push_back(es);
    }
    {
        SplitArgs sa{};
        sa.A = g.A;
        sa.lda = g.lda;
        sa.sA = g.sA;
        sa.a_rows = g.a_rows;
        sa.sAr = g.sAr;
        sa.M = g.M;
        sa.K = g.K;
        sa.Mp = Mp;
        sa.Kp = Kp;
        sa.L = L;
        sa.Ap = Ap;
        sa.fa = fa;
        sa.nkbp = nkbp;
        sa.vec = ((uintptr_t)g.A % 16 == 0) && g.lda % 4 == 0 && g.sA % 4 == 0;
        sa.B = g.B;
        sa.ldb = g.ldb;
        sa.sB = g.sB;
        sa.b_rows = g.b_rows;
        sa.sBr = g.sBr;
        sa.N = g.N;
        sa.Np = Np;
        sa.bn = Cfg::BN;
        sa.Bp = Bp;
        sa.fb = fb;
        sa.nrange = nb == 1 && !g.b_rows ? g.b_nrange : nullptr;
        sa.a_blocks = (Mp / 128) * (Kp / 128);
        const int64_t blocks = (int64_t)sa.a_blocks + (int64_t)(Np / 64) * (Kp / 128);
        k_split_ab<<<dim3((unsigned)blocks, 1, nb), 256, L * 64 * SPLIT_ROW, s>>>(sa);
        *launches += 1;
    }
    CUtensorMap ma, mb;
    int rc = make_map(&ma, Ap, Kp, (int64_t)nb * L * Mp, Cfg::BK, Cfg::BM);
    if (rc) return rc;
    rc = make_map(&mb, Bp, Kp, (int64_t)nb * L * Np, Cfg::BK, Cfg::BN);
    if (rc) return rc;
    TcParams prm{};
    prm.D = g.D;
    prm.ldd = g.ldd;
    prm.sD = g.sD;
    prm.d_rows = g.d_rows;
    prm.sDr = g.sDr;
    prm.M = g.M;
    prm.N = g.N;
    prm.Mp = Mp;
    prm.Np = Np;
    prm.nkb = nkb;
    prm.nkbp = nkbp;
    prm.fa = fa;
    prm.fb = fb;
    const FieldMont f = FieldMont::make(g.p);
    prm.p = g.p;
    prm.pneg_inv = f.pneg_inv;
    prm.mu = (uint32_t)((((uint64_t)1) << 32) / g.p);
    const uint64_t R = ((uint64_t)1 << 32) % g.p;
    uint64_t pw = 1;
    for (int w = 0; w < 7; ++w) {
        prm.cw[w] = (uint32_t)((pw % g.p) * R % g.p);
        pw = (pw << 8) % g.p;
    }
    prm.err = err;
    prm.budget = 4000000000LL;  // about 2 s at 2 GHz per wait
    cudaError_t e = ensure_smem_limit((const void*)k_tc_submul<L, SHAPE>, Cfg::SMEM_BYTES);
    if (e != cudaSuccess) {
        set_error(std::string("tc smem attribute: ") + cudaGetErrorString(e));
        return GBGPU_ECUDA;
    }
    prm.batch = nb;
    const int64_t tiles = (int64_t)(Np / Cfg::BN) * (Mp / Cfg::BM) * nb;
    const dim3 grid((unsigned)std::max<int64_t>(
        1, std::min<int64_t>(tiles, (int64_t)num_sms() * Cfg::MIN_CTAS)));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (prof) {
        const int slot = (int)prof->events.size();
        prm.steps = slot < prof->capacity ? prof->d_steps + slot : nullptr;
        prof->shape.insert(prof->shape.end(), {g.M, g.N, g.K, nb});
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, s);
    }
    k_tc_submul<L, SHAPE><<<grid, Cfg::THREADS, Cfg::SMEM_BYTES, s>>>(ma, mb, prm);
    ++*launches;
    if (prof) {
        cudaEventRecord(e1, s);
        prof->events.push_back({e0, e1});
        // int8 MACs of one executed K step of one tile
        prof->macs_per_step.push_back((double)Cfg::BM * Cfg::BN * Cfg::BK * L * L);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("tc launch: ") + cudaGetErrorString(e));
        return GBGPU_ECUDA;
    }
    return GBGPU_OK;
}

size_t tc_workspace_bytes(uint32_t p, int32_t M, int32_t N, int32_t K, int32_t batch) {
    const int L = limbs_for(p);
    // planes padded for the widest tile (256 columns), flags counted for the
    // narrowest (64) with flag rows padded to 64 K steps: enough for either
    // tile shape
    const size_t Mp = (size_t)(M + 127) / 128 * 128, Np = (size_t)(N + 255) / 256 * 256;
    const size_t Kp = (size_t)(K + 127) / 128 * 128;
    const size_t nkbp = (Kp / 128 + 63) / 64 * 64;
    const size_t nb = (size_t)(batch > 0 ? batch : 1);
    const size_t flags = nb * (Mp / 128 + Np / 64) * nkbp;
    return nb * L * (Mp + Np) * Kp + ((flags + 255) & ~(size_t)255);
}

int tc_submul(const TcGemmArgs& g, void* workspace, cudaStream_t s, int32_t* err,
              long long* launches) {
    if (g.M <= 0 || g.N <= 0 || g.K <= 0 || g.batch <= 0) return GBGPU_OK;
    if (g.batch > 65535) {
        set_error("tensor-core GEMM: batch too large");
        return GBGPU_ERANGE;
    }
    if ((g.p & 1u) == 0 || g.p < 3) {
        set_error("tensor-core path needs an odd prime");
        return GBGPU_EINVAL;
    }
    return tc_submul_shape(g, workspace, s, err, launches, tc_shape_for(limbs_for(g.p), g.K));
}

// the shapes: 0 big, 1 small (K <= 256, L <= 2), 2 mid (L = 2); any other
// request falls back to the big shape
int tc_submul_shape(const TcGemmArgs& g, void* workspace, cudaStream_t s, int32_t* err,
                    long long* launches, int shape) {
    if (g.M <= 0 || g.N <= 0 || g.K <= 0 || g.batch <= 0) return GBGPU_OK;
    uint8_t* planes = (uint8_t*)workspace;
    const bool small = shape == 1 && g.K <= 256;
    switch (limbs_for(g.p)) {
        case 1:
            return small ? tc_run<1, TC_SMALL>(g, planes, s, err, launches)
                         : tc_run<1, TC_BIG>(g, planes, s, err, launches);
        case 2:
            return small         ? tc_run<2, TC_SMALL>(g, planes, s, err, launches)
                   : shape == 2  ? tc_run<2, TC_MID>(g, planes, s, err, launches)
                                 : tc_run<2, TC_BIG>(g, planes, s, err, launches);
        case 3: return tc_run<3, TC_BIG>(g, planes, s, err, launches);
        default: return tc_run<4, TC_BIG>(g, planes, s, err, launches);
    }
}

int plain_submul(const TcGemmArgs& g, cudaStream_t s, long long* launches) {
    if (g.M <= 0 || g.N <= 0 || g.K <= 0 || g.batch <= 0) return GBGPU_OK;
    dim3 grid((g.N + 63) / 64, (g.M + 63) / 64, g.batch);
    FieldMont f{};
    f.p = g.p;
    const RowLists rl{g.a_rows, g.b_rows, g.d_rows, g.sAr, g.sBr, g.sDr};
    k_plain_submul<<<grid, 256, 0, s>>>(g.A, g.lda, g.B, g.ldb, g.D, g.ldd, g.M, g.N, g.K, g.sA,
                                        g.sB, g.sD, rl, f);
    ++*launches;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("plain gemm launch: ") + cudaGetErrorString(e));
        return GBGPU_ECUDA;
    }
    return GBGPU_OK;
}

}  // namespace gbgpu
