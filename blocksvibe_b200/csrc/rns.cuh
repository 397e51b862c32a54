// Residue-number-system (RNS) multiprecision GEMM on the sm_100a INT8 tensor cores.
//
// C = A B for aligned operands (k_align: integer mantissas of at most NB = 32 L - 2 bits, a common exponent
// per row of A and per column of B).  The exact integer product P = sum_k a b (|P| < K 2^(2 NB)) is computed
// modulo n_p primes p_j < 2^31 whose product M exceeds 4 max |P|, then reconstructed by the Chinese remainder
// theorem and rounded once: the result is bit-identical to the exact schoolbook product (k_gemm_aligned).
//
//   1. k_rns_split: each operand element -> its n_p residues, each cut into four 8-bit digits, written as
//      unsigned int8 matrices in the canonical K-major UMMA layout (core matrices of 8 rows x 16 bytes).
//      Row r of the operand becomes rows 4 r + s (digit s) of the digit matrix.
//   2. k_rns_mma: per (prime, batch, tile) one CTA: both tiles land in shared memory by bulk async copies
//      (cp.async.bulk, the TMA engine) on an mbarrier, one thread issues tcgen05.mma.kind::i8 over K into a
//      TMEM accumulator (128 lanes x TN columns, int32), and the epilogue reads TMEM with tcgen05.ld and folds
//      the 16 digit products of each output, sum_{s,t} D[4i+s][4l+t] 2^(8(s+t)), to a residue mod p_j.
//   3. k_rns_crt: per output, y_j = r_j (M/p_j)^-1 mod p_j, x' = sum_j y_j (M/p_j) exactly in limbs,
//      q = round(x' / M) from two words of x' in integers (crt_quotient: x' / M lies within 1/8 of an integer
//      because |P| < M/8), P = x' - q M, rounded to NB bits with the exponents of its row and column.
//
// Every spin-wait (mbarrier phases) has an iteration limit; on expiry the CTA records an error code in a
// device flag, waits (bounded) for its own copies, frees its TMEM and returns.
#pragma once
#include <cuda_runtime.h>

#include "mp.cuh"

namespace b3d {

// number of primes and limbs of M for L-limb operands and inner dimension K <= 4096
B3D_CX int rns_primes(int L) { return (2 * (32 * L - 2) + 12 + 2 + 30) / 31 + 1; }
B3D_CX int rns_mlimbs(int L) { return (31 * rns_primes(L) + 31) / 32 + 1; }
// dynamic shared memory cap of the tensor-core split and CRT kernels: under the 227 KB per-block opt-in limit
// with room for their few static words (the 1470-bit CRT takes 208 KB)
constexpr int kRnsSmemCap = 224 * 1024;

// per-L tables (device memory, filled by the host: blocksvibe_b200/rns.py)
struct RnsTables {
    const uint32_t* p;       // (np) primes
    const uint64_t* mu;      // (np) floor(2^62 / p)
    const uint32_t* w;       // (np, 8) 2^(8u) mod p, u < 7
    const uint32_t* conv;    // (np, L) 2^(32k) mod p
    const uint32_t* inv;     // (np) (M / p)^-1 mod p
    const uint32_t* mj;      // (np, ML) M / p, little-endian limbs
    const uint32_t* mfull;   // (ML) M
    int np, ml;
    uint64_t mtop;           // floor(M / 2^(32 msw))
    int msw;                 // word offset with 32 msw >= bitlen(M) - 56
};

// The CRT quotient q = round(x' / M) for x' = sum_j y_j M / p_j = P + q M with |P| < M / 8 (the prime count
// guarantees it): from the words msw, msw + 1 of x' (x' < 128 M < 2^(32 msw + 63)) and mtop = floor(M / 2^(32 msw))
// >= 2^23, xt / mtop is within 2^-16 of x' / M, which lies within 1/8 of q: round(xt / mtop) = q, found by seven
// compare-and-add steps (q <= np < 128) in 64-bit integers.  No floating point.
template <int N>
__device__ __forceinline__ uint32_t crt_quotient(const u32 (&x)[N], int msw, uint64_t mtop) {
    uint64_t xt = 0;
#pragma unroll
    for (int c = 0; c < N; c++)
        if (c == msw) xt = ((uint64_t)(c + 1 < N ? x[c + 1] : 0u) << 32) | x[c];
    const uint64_t num = 2 * xt + mtop, den = 2 * mtop;        // round(xt / mtop) = floor(num / den)
    uint32_t q = 0;
#pragma unroll
    for (int b = 6; b >= 0; b--)
        if ((uint64_t)(q + (1u << b)) * den <= num) q += 1u << b;
    return q;
}

// x mod p for x < 2^62, Barrett with mu = floor(2^62 / p), 2^30 < p < 2^31
// (the quotient estimate is at most 3 below the true quotient)
__device__ __forceinline__ uint32_t barrett(uint64_t x, uint32_t p, uint64_t mu) {
    uint64_t xq = x >> 30;                      // < 2^32
    uint64_t qq = (xq * mu) >> 32;              // xq < 2^32, mu < 2^32: the product fits 64 bits
    uint64_t r = x - qq * (uint64_t)p;
#pragma unroll
    for (int c = 0; c < 3; c++) r = r >= p ? r - p : r;
    return (uint32_t)r;
}

// ------------------------------------------------------------------------------------------------
// 1. digits.  Element (b, r, k) of a strided aligned operand (two's complement limb planes, plane stride
// `plane`, element index b * sb + r * sr + k * sk) -> digits of its residues at rows 4 r + s, column k of the
// K-major tiled matrix of (prime j, batch b): out + (j * nb + b) * mat_bytes, tiles of TR rows:
//   byte(row, k) = ((row / TR) * (Kp / 16) + k / 16) * (TR * 16) + ((row % TR) / 8) * 128 + (row % 8) * 16 + k % 16
// Threads cover the padded matrix (rows < Rp, k < Kp); padding is written as zero.
__device__ __forceinline__ size_t tiled_offset(int64_t row, int64_t k, int TR, int64_t Kp) {
    return (size_t)(((row / TR) * (Kp / 16) + k / 16) * (TR * 16) + ((row % TR) / 8) * 128 + (row % 8) * 16 + k % 16);
}

template <int L>
__device__ __forceinline__ uint32_t residue_of(const u32 (&a)[L], bool neg, const RnsTables& tb, int j) {
    const uint32_t* c = tb.conv + (size_t)j * L;
    uint64_t lo = 0, hi = 0;                     // sums of 16-bit halves times constants: < 2 L 2^47
#pragma unroll
    for (int q = 0; q < L; q++) {
        uint32_t cq = __ldg(c + q);
        lo += (uint64_t)(a[q] & 0xFFFFu) * cq;
        hi += (uint64_t)(a[q] >> 16) * cq;
    }
    uint32_t p = __ldg(tb.p + j);
    uint64_t mu = __ldg(tb.mu + j);
    uint32_t r = barrett(((uint64_t)barrett(hi, p, mu) << 16) + barrett(lo, p, mu), p, mu);
    return (neg && r) ? p - r : r;
}

// threads cover (b, r < Rp, k4 < Kp / 4): four consecutive k of one row, one 32-bit store per (prime, digit)
template <int L>
__global__ void k_rns_split(const int32_t* __restrict__ m, int64_t plane, int64_t nb, int64_t R, int64_t K,
                            int64_t sb, int64_t sr, int64_t sk, int64_t Rp, int64_t Kp, int TR, RnsTables tb,
                            uint8_t* __restrict__ out, int64_t mat_bytes) {
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t K4 = Kp / 4;
    if (t >= nb * Rp * K4) return;
    int64_t k0 = (t % K4) * 4, r = (t / K4) % Rp, b = t / (K4 * Rp);
    const int np = tb.np;
    u32 a[4][L];
    bool neg[4], nz[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
        int64_t k = k0 + u;
        if (r < R && k < K) {
            neg[u] = load_mag<L>(m, plane, b * sb + r * sr + k * sk, a[u]);
        } else {
            zero(a[u]);
            neg[u] = false;
        }
        nz[u] = !is_zero(a[u]);
    }
    for (int j = 0; j < np; j++) {
        uint32_t res[4];
#pragma unroll
        for (int u = 0; u < 4; u++) res[u] = nz[u] ? residue_of<L>(a[u], neg[u], tb, j) : 0u;
        uint8_t* base = out + ((size_t)j * nb + b) * mat_bytes;
#pragma unroll
        for (int s = 0; s < 4; s++) {
            uint32_t w = ((res[0] >> (8 * s)) & 0xFFu) | (((res[1] >> (8 * s)) & 0xFFu) << 8) |
                         (((res[2] >> (8 * s)) & 0xFFu) << 16) | (((res[3] >> (8 * s)) & 0xFFu) << 24);
            *reinterpret_cast<uint32_t*>(base + tiled_offset(4 * r + s, k0, TR, Kp)) = w;
        }
    }
}

// ------------------------------------------------------------------------------------------------
// 2. tensor-core product with the residue epilogue
struct RnsMma {
    const uint8_t* X;        // digit matrices of the lane-side operand: (np, nb, tilesX, 128 x Kp)
    const uint8_t* Y;        // digit matrices of the column-side operand: (np, nb, tilesY, TN x Kp)
    int64_t x_mat, y_mat;    // bytes per (prime, batch) matrix
    int64_t nb, NI, NL;      // batch, rows of X (i), rows of Y (l)
    int Kp, TN;              // padded K (multiple of 32, <= 256), column tile (multiple of 16, <= 256)
    int64_t tiles_l;         // column tiles (grid: x = row tiles * tiles_l, y = batch, z = prime)
    int64_t out_b, out_i, out_l;   // output strides (elements) for (b, i, l); prime stride = nb * out_b
    uint32_t* out;           // residues (np, nb, ...), when yb is null
    int* err;                // device error flag (0 = ok)
    uint8_t* yb;             // else: y_j = r_j (M/p_j)^-1 mod p_j as 4 bytes at row e, column 4 j of the CRT operand
    int64_t crt_kp;          // bytes per row of the CRT operand (tiles of 128 rows)
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// bounded wait for phase `parity` of an mbarrier; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    uint32_t addr = smem_u32(bar);
    for (uint32_t it = 0; it < limit; it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P;\n\t}"
            : "=r"(done) : "r"(addr), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

// K-major, no swizzle: core matrices of 8 rows x 16 bytes; lbo = byte stride between K chunks of 16 bytes,
// sbo = byte stride between groups of 8 rows
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;                      // descriptor version for sm_100
    return d;                                    // base offset 0, lbo mode 0, layout SWIZZLE_NONE (0)
}

constexpr uint32_t kWaitLimit = 1u << 24;

#ifdef B3D_RNS_MMA
__global__ void __launch_bounds__(128, 1) k_rns_mma(RnsMma a, RnsTables tb) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar_load, bar_mma;
    __shared__ uint32_t tmem_base_sh;
    __shared__ int fail_sh;

    const int TN = a.TN, Kp = a.Kp;
    const int64_t j = blockIdx.z, b = blockIdx.y;
    const int64_t ti = blockIdx.x / a.tiles_l, tl = blockIdx.x % a.tiles_l;
    uint8_t* sX = smem;
    uint8_t* sY = smem + 128 * Kp;
    const uint32_t xbytes = 128u * Kp, ybytes = (uint32_t)TN * Kp;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    uint32_t ncols = 32;
    while (ncols < (uint32_t)TN) ncols <<= 1;

    if (threadIdx.x == 0) {
        fail_sh = 0;
        mbar_init(&bar_load, 1);
        mbar_init(&bar_mma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_base_sh)), "r"(ncols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_sh;

    if (threadIdx.x == 0) {
        const uint8_t* gx = a.X + (size_t)(j * a.nb + b) * a.x_mat + (size_t)ti * xbytes;
        const uint8_t* gy = a.Y + (size_t)(j * a.nb + b) * a.y_mat + (size_t)tl * ybytes;
        mbar_expect_tx(&bar_load, xbytes + ybytes);
        bulk_copy_g2s(sX, gx, xbytes, &bar_load);
        bulk_copy_g2s(sY, gy, ybytes, &bar_load);
    }
    bool ok = mbar_wait(&bar_load, 0, kWaitLimit);
    if (!ok) atomicExch(&fail_sh, 1);
    __syncthreads();
    bool run = fail_sh == 0;

    if (run && threadIdx.x == 0) {
        // instruction descriptor: s32 accumulator, u8 x u8, both K-major, M = 128, N = TN
        const uint32_t idesc = (2u << 4) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
        const uint32_t ax = smem_u32(sX), ay = smem_u32(sY);
        for (int kk = 0; kk < Kp / 32; kk++) {
            uint64_t da = umma_desc(ax + kk * 2 * (128 * 16), 128 * 16, 128);
            uint64_t db = umma_desc(ay + kk * 2 * (TN * 16), TN * 16, 128);
            uint32_t acc = kk > 0 ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
                ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc) : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     ::"r"(smem_u32(&bar_mma)) : "memory");
    }
    if (run) {
        ok = mbar_wait(&bar_mma, 0, kWaitLimit);
        if (!ok) atomicExch(&fail_sh, 2);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    run = run && fail_sh == 0;

    if (run) {
        // epilogue: lane row = 4 i + s, columns 4 l + t
        const uint32_t p = __ldg(tb.p + j);
        const uint64_t mu = __ldg(tb.mu + j);
        const uint32_t inv = __ldg(tb.inv + j);
        uint32_t w[7];
#pragma unroll
        for (int u = 0; u < 7; u++) w[u] = __ldg(tb.w + j * 8 + u);
        const int row = threadIdx.x;                 // TMEM lane
        const int s = row & 3;
        const int64_t i = ti * 32 + row / 4;
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
        for (int c0 = 0; c0 < TN; c0 += 16) {
            uint32_t d[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
                  "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15])
                : "r"(taddr + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int q = 0; q < 4; q++) {
                uint64_t v = 0;
#pragma unroll
                for (int t = 0; t < 4; t++) v += (uint64_t)d[4 * q + t] * w[s + t];
                v += __shfl_xor_sync(0xFFFFFFFFu, v, 1);
                v += __shfl_xor_sync(0xFFFFFFFFu, v, 2);
                const int64_t l = tl * (TN / 4) + c0 / 4 + q;
                if (s == 0 && i < a.NI && l < a.NL) {
                    uint32_t r = barrett(v, p, mu);
                    const int64_t e = b * a.out_b + i * a.out_i + l * a.out_l;
                    if (a.yb) {
                        uint32_t y = barrett((uint64_t)r * inv, p, mu);
                        *reinterpret_cast<uint32_t*>(a.yb + tiled_offset(e, 4 * j, 128, a.crt_kp)) = y;
                    } else {
                        a.out[j * a.nb * a.out_b + e] = r;
                    }
                }
            }
        }
    }
    if (threadIdx.x == 0 && fail_sh) {              // bounded drain of our own copies and MMAs
        if (!mbar_wait(&bar_load, 0, kWaitLimit)) fail_sh = 3;
        else if (fail_sh == 2 && !mbar_wait(&bar_mma, 0, kWaitLimit)) fail_sh = 4;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
    }
    if (threadIdx.x == 0 && fail_sh) atomicExch(a.err, fail_sh);
}
#endif

#ifdef B3D_RNS_MMA
// 2''. the product with the CRT-operand epilogue, four primes per CTA.  256 threads: thread 0 issues the bulk
// copies (one operand buffer: as soon as the MMAs of prime j have completed, the operands of prime j + 1
// are copied into it while the epilogue of prime j runs) and the MMAs; both warpgroups read TMEM (warp w reads lanes 32 (w % 4), warpgroup h the h-th half of the
// column chunks) and reduce.  The y bytes of the four primes of an output are staged in shared memory and
// leave as one 16-byte store per output (columns 16 g .. 16 g + 15 of the CRT operand).
constexpr int kPrimesPerCta = 4;

__global__ void __launch_bounds__(256, 2) k_rns_mma4(RnsMma a, RnsTables tb) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar_load, bar_mma;
    __shared__ uint32_t tmem_base_sh;
    __shared__ int fail_sh;

    const int TN = a.TN, Kp = a.Kp, np = tb.np;
    const int64_t g = blockIdx.z, b = blockIdx.y;
    const int64_t ti = blockIdx.x / a.tiles_l, tl = blockIdx.x % a.tiles_l;
    const uint32_t xbytes = 128u * Kp, ybytes = (uint32_t)TN * Kp, stage = xbytes + ybytes;
    uint8_t* ysm = smem + (size_t)stage;                 // (32 rows i x TN / 4 columns l) x 16 bytes
    const int warp = threadIdx.x / 32;
    const int j0 = (int)g * kPrimesPerCta;
    const int nj = np - j0 < kPrimesPerCta ? np - j0 : kPrimesPerCta;
    uint32_t ncols = 32;
    while (ncols < (uint32_t)TN) ncols <<= 1;

    if (threadIdx.x == 0) {
        fail_sh = 0;
        mbar_init(&bar_load, 1);
        mbar_init(&bar_mma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_base_sh)), "r"(ncols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_sh;

    int issued = 0, waited = 0, mma_pending = 0;         // thread 0's bookkeeping (for the failure drain)
    if (threadIdx.x == 0) {
        const uint8_t* gx = a.X + (size_t)((int64_t)j0 * a.nb + b) * a.x_mat + (size_t)ti * xbytes;
        const uint8_t* gy = a.Y + (size_t)((int64_t)j0 * a.nb + b) * a.y_mat + (size_t)tl * ybytes;
        mbar_expect_tx(&bar_load, stage);
        bulk_copy_g2s(smem, gx, xbytes, &bar_load);
        bulk_copy_g2s(smem + xbytes, gy, ybytes, &bar_load);
        issued = 1;
    }
    const int row = threadIdx.x & 127, s = row & 3, half = threadIdx.x >> 7;
    const uint32_t taddr = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    const int chunks = TN / 16, c_lo = half ? (chunks + 1) / 2 : 0, c_hi = half ? chunks : (chunks + 1) / 2;
    const uint32_t idesc = (2u << 4) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);

    for (int pi = 0; pi < nj; pi++) {
        const int j = j0 + pi;
        if (!mbar_wait(&bar_load, pi & 1, kWaitLimit)) atomicExch(&fail_sh, 1);
        else if (threadIdx.x == 0) waited = pi + 1;
        __syncthreads();
        if (fail_sh) break;
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");   // after the previous epilogue's reads
            const uint32_t ax = smem_u32(smem), ay = ax + xbytes;
            for (int kk = 0; kk < Kp / 32; kk++) {
                uint64_t da = umma_desc(ax + kk * 2 * (128 * 16), 128 * 16, 128);
                uint64_t db = umma_desc(ay + kk * 2 * (TN * 16), TN * 16, 128);
                uint32_t acc = kk > 0 ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
                    ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc) : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(smem_u32(&bar_mma)) : "memory");
            mma_pending = 1;
        }
        if (!mbar_wait(&bar_mma, pi & 1, kWaitLimit)) atomicExch(&fail_sh, 2);
        else if (threadIdx.x == 0) mma_pending = 0;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        __syncthreads();
        if (fail_sh) break;
        if (threadIdx.x == 0 && pi + 1 < nj) {           // the MMAs are done with the buffer: prime j + 1
            const uint8_t* gx = a.X + (size_t)((int64_t)(j + 1) * a.nb + b) * a.x_mat + (size_t)ti * xbytes;
            const uint8_t* gy = a.Y + (size_t)((int64_t)(j + 1) * a.nb + b) * a.y_mat + (size_t)tl * ybytes;
            mbar_expect_tx(&bar_load, stage);
            bulk_copy_g2s(smem, gx, xbytes, &bar_load);
            bulk_copy_g2s(smem + xbytes, gy, ybytes, &bar_load);
            issued = pi + 2;
        }

        const uint32_t p = __ldg(tb.p + j);
        const uint64_t mu = __ldg(tb.mu + j);
        const uint32_t inv = __ldg(tb.inv + j);
        uint32_t w[7];
#pragma unroll
        for (int u = 0; u < 7; u++) w[u] = __ldg(tb.w + j * 8 + u);
        for (int c = c_lo; c < c_hi; c++) {
            const int c0 = 16 * c;
            uint32_t d[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
                  "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15])
                : "r"(taddr + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            // partial sums of the four outputs q of this chunk (this lane's row digit s), then a
            // reduce-scatter over the four lanes of the row: lane s ends with the full sum of output q = s
            uint64_t pq[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                uint64_t v = 0;
#pragma unroll
                for (int t = 0; t < 4; t++) v += (uint64_t)d[4 * q + t] * w[s + t];
                pq[q] = v;
            }
            const bool hi2 = (s & 2) != 0, hi1 = (s & 1) != 0;
            const uint64_t k0 = hi2 ? pq[2] : pq[0], k1 = hi2 ? pq[3] : pq[1];
            const uint64_t x0 = hi2 ? pq[0] : pq[2], x1 = hi2 ? pq[1] : pq[3];
            const uint64_t a0 = k0 + __shfl_xor_sync(0xFFFFFFFFu, x0, 2);     // outputs (s & 2) + {0, 1}
            const uint64_t a1 = k1 + __shfl_xor_sync(0xFFFFFFFFu, x1, 2);
            const uint64_t v = (hi1 ? a1 : a0) + __shfl_xor_sync(0xFFFFFFFFu, hi1 ? a0 : a1, 1);   // output s
            const uint32_t r = barrett(v, p, mu);
            const uint32_t y = barrett((uint64_t)r * inv, p, mu);
            const int ll = c0 / 4 + s;
            *reinterpret_cast<uint32_t*>(ysm + ((size_t)(row >> 2) * (TN / 4) + ll) * 16 + 4 * pi) = y;
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();                                  // TMEM read out before the next prime's MMAs
    }
    if (!fail_sh) {                                       // one 16-byte store per output
        const int nl = TN / 4, per = 32 * nl;
        const bool lfast = a.out_l == 1;
        for (int x = threadIdx.x; x < per; x += blockDim.x) {
            const int il = lfast ? x / nl : x % 32, ll = lfast ? x % nl : x / 32;
            const int64_t ii = ti * 32 + il, l = tl * nl + ll;
            if (ii < a.NI && l < a.NL) {
                const int64_t e = b * a.out_b + ii * a.out_i + l * a.out_l;
                *reinterpret_cast<uint4*>(a.yb + tiled_offset(e, 4 * (int64_t)j0, 128, a.crt_kp)) =
                    *reinterpret_cast<const uint4*>(ysm + ((size_t)il * nl + ll) * 16);
            }
        }
    }
    if (threadIdx.x == 0 && fail_sh) {                    // bounded drain of our own copies and MMAs
        for (int q = waited; q < issued; q++)
            if (!mbar_wait(&bar_load, q & 1, kWaitLimit)) { fail_sh = 3; break; }
        if (fail_sh != 3 && mma_pending && !mbar_wait(&bar_mma, (waited - 1) & 1, kWaitLimit)) fail_sh = 4;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
    }
    if (threadIdx.x == 0 && fail_sh) atomicExch(a.err, fail_sh);
}
#endif

// ------------------------------------------------------------------------------------------------
// 1'. digits on the tensor cores.  One CTA = a tile of 8 operand rows x 16 columns k (128 elements).  The
// elements' magnitude bytes form A (128 rows x 4 L bytes, K-major in shared memory); the constant
// C[(j, t)][d] = byte t of (2^(8 d) mod p_j) is B (two tiles of NS rows); S = A B^T holds
// sum_d digit_d C[(j, t)][d] < 4 L 255^2, so r_j = sum_t S[4 j + t] 2^(8 t) mod p_j (sign applied after).
// The residue digits are staged in shared memory and written as 16-byte chunks of the same K-major
// digit matrices k_rns_split writes.
struct RnsSplit {
    const int32_t* m; int64_t plane, nb, R, K, sb, sr, sk;   // aligned operand
    int64_t Rp, Kp; int TR; int64_t mat_bytes;               // output digit matrices
    uint8_t* out;
    const uint8_t* C;        // (2 NS x Ks) constant digit matrix, tiles of NS rows
    int Ks, NS;              // K bytes of the magnitudes (multiple of 32) and half of the 4 np columns
    int* err;
};

#ifdef B3D_DEFINE_LAUNCH
template <int L>
__global__ void __launch_bounds__(128, 1) k_rns_split_mma(RnsSplit a, RnsTables tb) {
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar_load, bar_mma;
    __shared__ uint32_t tmem_base_sh;
    __shared__ int fail_sh;
    __shared__ uint8_t neg_sh[128];
    const int Ks = a.Ks, NS = a.NS, np = tb.np;
    uint8_t* sA = smem;                                  // 128 x Ks magnitude bytes
    uint8_t* sC = smem + 128 * Ks;                       // 2 NS x Ks constants
    uint8_t* sD = sC + 2 * NS * Ks;                      // np x 4 x 8 x 16 staged digits
    const int warp = threadIdx.x / 32, t = threadIdx.x;
    const int64_t ktiles = a.Kp / 16, tiles = ktiles * ((a.Rp + 7) / 8), items = tiles * a.nb;
    const uint32_t ncols = 256;                          // one half (NS <= 256 columns) at a time
    if (t == 0) {
        fail_sh = 0;
        mbar_init(&bar_load, 1);
        mbar_init(&bar_mma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_base_sh)), "r"(ncols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_sh;
    if (t == 0) {
        const uint32_t cbytes = 2u * NS * Ks;
        mbar_expect_tx(&bar_load, cbytes);
        bulk_copy_g2s(sC, a.C, cbytes, &bar_load);
    }
    if (!mbar_wait(&bar_load, 0, kWaitLimit)) atomicExch(&fail_sh, 1);
    __syncthreads();
    bool run = fail_sh == 0;
    int mma_h = 0;                                        // pass of the last MMA commit (failure drain)
    // persistent: the constant and the TMEM allocation serve every tile this CTA takes
    for (int64_t item = blockIdx.x; item < items && run; item += gridDim.x) {
    const int64_t b = item / tiles, tile = item % tiles;
    const int64_t r0 = (tile / ktiles) * 8, k0 = (tile % ktiles) * 16;
    // magnitudes of the tile's elements -> A rows e = rr * 16 + kk (load order follows the unit stride)
    {
        const bool rows_fast = a.sr == 1;
        const int rr = rows_fast ? (t % 8) : (t / 16), kk = rows_fast ? (t / 8) : (t % 16);
        const int e = rr * 16 + kk;
        const int64_t r = r0 + rr, k = k0 + kk;
        u32 v[L];
        bool neg = false;
        if (r < a.R && k < a.K) neg = load_mag<L>(a.m, a.plane, b * a.sb + r * a.sr + k * a.sk, v);
        else zero(v);
        neg_sh[e] = neg;
#pragma unroll
        for (int c = 0; c < (4 * L + 15) / 16; c++) {
            uint4 w;
            w.x = 4 * c + 0 < L ? v[4 * c + 0] : 0u;
            w.y = 4 * c + 1 < L ? v[4 * c + 1] : 0u;
            w.z = 4 * c + 2 < L ? v[4 * c + 2] : 0u;
            w.w = 4 * c + 3 < L ? v[4 * c + 3] : 0u;
            *reinterpret_cast<uint4*>(sA + tiled_offset(e, 16 * c, 128, Ks)) = w;
        }
        for (int c = (4 * L + 15) / 16; c < Ks / 16; c++)
            *reinterpret_cast<uint4*>(sA + tiled_offset(e, 16 * c, 128, Ks)) = make_uint4(0, 0, 0, 0);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");    // generic-proxy writes -> tensor core
    __syncthreads();
    // two passes over the halves of the constant matrix, sharing 256 TMEM columns (two CTAs per SM)
    for (int h = 0; h < 2 && run; h++) {
    if (t == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");   // after the first half's TMEM reads
        const uint32_t idesc = (2u << 4) | ((uint32_t)(NS >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
        const uint32_t aa = smem_u32(sA), ac = smem_u32(sC);
        for (int kk = 0; kk < Ks / 32; kk++) {
            uint64_t da = umma_desc(aa + kk * 2 * (128 * 16), 128 * 16, 128);
            uint64_t db = umma_desc(ac + h * NS * Ks + kk * 2 * (NS * 16), NS * 16, 128);
            uint32_t acc = kk > 0 ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "setp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
                ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc) : "memory");
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     ::"r"(smem_u32(&bar_mma)) : "memory");
    }
    mma_h = h;
    if (!mbar_wait(&bar_mma, h, kWaitLimit)) atomicExch(&fail_sh, 2);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    run = fail_sh == 0;
    if (run) {
        // epilogue: element e = t; residues of 4 primes per 16-column chunk, primes of this half
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
        const bool neg = neg_sh[t];
        const int rr = t / 16, kk = t % 16;
        const int jlo = h * (NS / 4), jhi = (h + 1) * (NS / 4) < np ? (h + 1) * (NS / 4) : np;
        for (int j0 = jlo; j0 < jhi; j0 += 4) {
            uint32_t d[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
                  "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15])
                : "r"(taddr + (uint32_t)(4 * j0 - h * NS)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int j = j0 + q;
                if (j >= np) break;
                uint64_t v = (uint64_t)d[4 * q] + ((uint64_t)d[4 * q + 1] << 8) + ((uint64_t)d[4 * q + 2] << 16) +
                             ((uint64_t)d[4 * q + 3] << 24);
                const uint32_t p = __ldg(tb.p + j);
                uint32_t r = barrett(v, p, __ldg(tb.mu + j));
                if (neg && r) r = p - r;
#pragma unroll
                for (int s = 0; s < 4; s++) sD[((j * 4 + s) * 8 + rr) * 16 + kk] = (uint8_t)(r >> (8 * s));
            }
        }
    }
    mma_h = h;
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();                                      // TMEM read out before the second half's MMAs
    }
    __syncthreads();
    if (run) {
        // 16-byte chunks: (prime j, digit s, row rr) -> row 4 (r0 + rr) + s, columns k0 .. k0 + 15
        for (int c = t; c < np * 32; c += 128) {
            const int rr = c % 8, s = (c / 8) % 4, j = c / 32;
            const int64_t r = r0 + rr;
            if (r >= a.Rp) continue;
            uint4 w = *reinterpret_cast<const uint4*>(sD + (size_t)c * 16);
            *reinterpret_cast<uint4*>(a.out + ((size_t)j * a.nb + b) * a.mat_bytes + tiled_offset(4 * r + s, k0, a.TR, a.Kp)) = w;
        }
    }
    __syncthreads();                                      // sD and neg_sh are rewritten by the next tile
    }
    if (t == 0 && fail_sh) {
        if (!mbar_wait(&bar_load, 0, kWaitLimit)) fail_sh = 3;
        else if (fail_sh == 2 && !mbar_wait(&bar_mma, mma_h, kWaitLimit)) fail_sh = 4;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
    }
    if (t == 0 && fail_sh) atomicExch(a.err, fail_sh);
}
#endif

// ------------------------------------------------------------------------------------------------
// 3'. CRT on the tensor cores.  A = the y bytes of 128 outputs (rows e, K = 4 np bytes, from k_rns_mma),
// B = the constant matrix T[pos][4 j + a] = byte (pos - a) of M / p_j (two tiles of NH rows), so that
// S[e][pos] = sum_{j,a} y_{j,a}(e) T[pos][4 j + a] and x' = sum_pos S[pos] 2^(8 pos) = sum_j y_j M / p_j
// exactly (S < 4 np 255^2 < 2^25).  The epilogue thread of output e carries S into limbs, subtracts
// round(x' / M) M (crt_quotient, integers) and rounds once to NB bits.
struct RnsCrt {
    const uint8_t* A;        // (tiles, 128 x Kc) y bytes
    const uint8_t* T;        // (2 NH x Kc) constant Toeplitz digits, tiles of NH rows
    int Kc, NH;              // K bytes (multiple of 32), half of the position count (multiple of 16)
    int64_t n, nbatch, M, N; // outputs, their (b, row, col) shape
    const int64_t* ea;       // (nbatch, M) row exponents
    const int64_t* eb;       // (nbatch, N) column exponents
    int32_t* cm;             // result limb planes
    int64_t* ce;             // result exponents
    int64_t cplane;
    int* err;
};

#ifdef B3D_DEFINE_LAUNCH
template <int L>
__global__ void __launch_bounds__(128, 1) k_rns_crt_mma(RnsCrt a, RnsTables tb) {
    constexpr int ML = rns_mlimbs(L);
    constexpr int NX = ML + 2;
    constexpr int NCH = (4 * ML + 3 + 15) / 16;      // 16-column chunks holding all positions
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar_load, bar_mma;
    __shared__ uint32_t tmem_base_sh;
    __shared__ int fail_sh;
    const int Kc = a.Kc, NH = a.NH;
    uint8_t* sA = smem;
    uint8_t* sT = smem + 128 * Kc;
    const uint32_t abytes = 128u * Kc, tbytes = 2u * NH * Kc;
    const int warp = threadIdx.x / 32;
    const uint32_t ncols = 512;
    if (threadIdx.x == 0) {
        fail_sh = 0;
        mbar_init(&bar_load, 1);
        mbar_init(&bar_mma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_base_sh)), "r"(ncols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_sh;
    // persistent over tiles of 128 outputs: the constant T is loaded once; the next tile's y bytes are copied
    // into sA as soon as the MMAs of the current tile have completed, while its epilogue runs
    const int64_t tiles = (a.n + 127) / 128;
    int issued = 0, waited = 0, mma_pending = 0;          // thread 0's bookkeeping (failure drain)
    if (threadIdx.x == 0 && (int64_t)blockIdx.x < tiles) {
        mbar_expect_tx(&bar_load, abytes + tbytes);
        bulk_copy_g2s(sA, a.A + (size_t)blockIdx.x * abytes, abytes, &bar_load);
        bulk_copy_g2s(sT, a.T, tbytes, &bar_load);
        issued = 1;
    }
    bool run = true;
    int it = 0;
    for (int64_t tile = blockIdx.x; tile < tiles && run; tile += gridDim.x, it++) {
    if (!mbar_wait(&bar_load, it & 1, kWaitLimit)) atomicExch(&fail_sh, 1);
    else if (threadIdx.x == 0) waited = it + 1;
    __syncthreads();
    run = fail_sh == 0;
    if (!run) break;
    if (threadIdx.x == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");   // after the previous epilogue's reads
        const uint32_t idesc = (2u << 4) | ((uint32_t)(NH >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
        const uint32_t aa = smem_u32(sA), at = smem_u32(sT);
        for (int h = 0; h < 2; h++) {
            for (int kk = 0; kk < Kc / 32; kk++) {
                uint64_t da = umma_desc(aa + kk * 2 * (128 * 16), 128 * 16, 128);
                uint64_t db = umma_desc(at + h * NH * Kc + kk * 2 * (NH * 16), NH * 16, 128);
                uint32_t acc = kk > 0 ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
                    ::"r"(tmem + (uint32_t)(h * NH)), "l"(da), "l"(db), "r"(idesc), "r"(acc) : "memory");
            }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     ::"r"(smem_u32(&bar_mma)) : "memory");
        mma_pending = 1;
    }
    if (!mbar_wait(&bar_mma, it & 1, kWaitLimit)) atomicExch(&fail_sh, 2);
    else if (threadIdx.x == 0) mma_pending = 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    run = fail_sh == 0;
    if (!run) break;
    if (threadIdx.x == 0 && tile + gridDim.x < tiles) {  // the MMAs are done with sA: the next tile
        mbar_expect_tx(&bar_load, abytes);
        bulk_copy_g2s(sA, a.A + (size_t)(tile + gridDim.x) * abytes, abytes, &bar_load);
        issued = it + 2;
    }
    const int64_t e = tile * 128 + threadIdx.x;
    {
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
        u32 x[NX];
        uint64_t carry = 0;
#pragma unroll
        for (int ch = 0; ch < NCH; ch++) {
            uint32_t d[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
                  "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]), "=r"(d[15])
                : "r"(taddr + (uint32_t)(16 * ch)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int c = 4 * ch + q;
                uint64_t v = carry + (uint64_t)d[4 * q] + ((uint64_t)d[4 * q + 1] << 8) +
                             ((uint64_t)d[4 * q + 2] << 16) + ((uint64_t)d[4 * q + 3] << 24);
                if (c < NX) x[c] = (uint32_t)v;
                carry = v >> 32;
            }
        }
#pragma unroll
        for (int c = 4 * NCH; c < NX; c++) {
            x[c] = (uint32_t)carry;
            carry >>= 32;
        }
        const uint32_t q = crt_quotient<NX>(x, tb.msw, tb.mtop);
        uint32_t mc = 0;
        uint64_t borrow = 0;
#pragma unroll
        for (int c = 0; c < NX; c++) {
            uint64_t prod = (c < ML ? (uint64_t)q * __ldg(tb.mfull + c) : 0) + mc;
            mc = (uint32_t)(prod >> 32);
            uint64_t v = (uint64_t)x[c] - (uint32_t)prod - borrow;
            x[c] = (uint32_t)v;
            borrow = v >> 63;
        }
        if (e < a.n) {
            const int64_t col = e % a.N, row = (e / a.N) % a.M, b = e / (a.M * a.N);
            const int64_t Ea = a.ea[b * a.M + row], Eb = a.eb[b * a.N + col];
            const bool z = Ea == EZ || Eb == EZ;
            if (z) zero(x);
            store_rounded<L, NX>(a.cm, a.ce, a.cplane, e, x, z ? EZ : Ea + Eb);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();                                      // TMEM read out before the next tile's MMAs
    }
    if (threadIdx.x == 0 && fail_sh) {                    // bounded drain of our own copies and MMAs
        for (int q = waited; q < issued; q++)
            if (!mbar_wait(&bar_load, q & 1, kWaitLimit)) { fail_sh = 3; break; }
        if (fail_sh != 3 && mma_pending && !mbar_wait(&bar_mma, (waited - 1) & 1, kWaitLimit)) fail_sh = 4;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
    }
    if (threadIdx.x == 0 && fail_sh) atomicExch(a.err, fail_sh);
}
#endif

// ------------------------------------------------------------------------------------------------
// 3. reconstruction: residues (np, n) with element index e = b * sb_out ... -> normalised MPF
template <int L>
__global__ void k_rns_crt(const uint32_t* __restrict__ res, int64_t n, const int64_t* __restrict__ ea,
                          const int64_t* __restrict__ eb, int64_t nbatch, int64_t M, int64_t N, RnsTables tb,
                          int32_t* __restrict__ cm, int64_t* __restrict__ ce, int64_t cplane) {
    constexpr int ML = rns_mlimbs(L);
    constexpr int NA = ML + 1;
    int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e >= n) return;
    int64_t col = e % N, row = (e / N) % M, b = e / (M * N);
    int64_t Ea = ea[b * M + row], Eb = eb[b * N + col];
    u32 acc[NA];
    zero(acc);
    const int np = tb.np;
    for (int jj = 0; jj < np; jj++) {
        uint32_t r = res[(size_t)jj * n + e];
        uint32_t p = __ldg(tb.p + jj);
        uint64_t mu = __ldg(tb.mu + jj);
        uint32_t y = barrett((uint64_t)r * __ldg(tb.inv + jj), p, mu);
        // acc += y * (M / p_j)
        const uint32_t* mj = tb.mj + (size_t)jj * ML;
        uint32_t carry = 0;
#pragma unroll
        for (int c = 0; c < ML; c++) {
            uint64_t v = (uint64_t)y * __ldg(mj + c) + acc[c] + carry;
            acc[c] = (uint32_t)v;
            carry = (uint32_t)(v >> 32);
        }
        acc[ML] += carry;
    }
    // subtract round(x' / M) M: the result is the signed product in (-M/8, M/8)
    const uint32_t q = crt_quotient<NA>(acc, tb.msw, tb.mtop);
    uint32_t borrow = 0;
    {
        uint32_t carry = 0;
        u32 qm[NA];
#pragma unroll
        for (int c = 0; c < ML; c++) {
            uint64_t v = (uint64_t)q * __ldg(tb.mfull + c) + carry;
            qm[c] = (uint32_t)v;
            carry = (uint32_t)(v >> 32);
        }
        qm[ML] = carry;
#pragma unroll
        for (int c = 0; c < NA; c++) {
            uint64_t v = (uint64_t)acc[c] - qm[c] - borrow;
            acc[c] = (uint32_t)v;
            borrow = (uint32_t)(v >> 63);
        }
    }
    bool zero_out = Ea == EZ || Eb == EZ;
    if (zero_out) zero(acc);
    store_rounded<L, NA>(cm, ce, cplane, e, acc, zero_out ? EZ : Ea + Eb);
}

}  // namespace b3d

namespace b3d {

// host-side launchers (instantiated per L in inst.cu; the MMA launcher lives in rns_mma.cu)
template <int L>
struct RnsLaunch {
    static int split(const int32_t* m, int64_t plane, int64_t nb, int64_t R, int64_t K, int64_t sb, int64_t sr,
                     int64_t sk, int64_t Rp, int64_t Kp, int TR, const RnsTables& tb, uint8_t* out,
                     int64_t mat_bytes, cudaStream_t st);
    static int crt(const uint32_t* res, int64_t n, const int64_t* ea, const int64_t* eb, int64_t nbatch, int64_t M,
                   int64_t N, const RnsTables& tb, int32_t* cm, int64_t* ce, int64_t cplane, cudaStream_t st);
    static int crt_mma(const RnsCrt& a, const RnsTables& tb, cudaStream_t st);
    static int split_mma(const RnsSplit& a, const RnsTables& tb, cudaStream_t st);
};

#ifdef B3D_DEFINE_LAUNCH
template <int L>
int RnsLaunch<L>::split(const int32_t* m, int64_t plane, int64_t nb, int64_t R, int64_t K, int64_t sb, int64_t sr,
                        int64_t sk, int64_t Rp, int64_t Kp, int TR, const RnsTables& tb, uint8_t* out,
                        int64_t mat_bytes, cudaStream_t st) {
    int64_t n = nb * Rp * (Kp / 4);
    if (n == 0) return 0;
    k_rns_split<L><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(m, plane, nb, R, K, sb, sr, sk, Rp, Kp, TR, tb, out, mat_bytes);
    return (int)cudaGetLastError();
}

template <int L>
int RnsLaunch<L>::crt(const uint32_t* res, int64_t n, const int64_t* ea, const int64_t* eb, int64_t nbatch, int64_t M,
                      int64_t N, const RnsTables& tb, int32_t* cm, int64_t* ce, int64_t cplane, cudaStream_t st) {
    if (n == 0) return 0;
    k_rns_crt<L><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(res, n, ea, eb, nbatch, M, N, tb, cm, ce, cplane);
    return (int)cudaGetLastError();
}

template <int L>
int RnsLaunch<L>::split_mma(const RnsSplit& a, const RnsTables& tb, cudaStream_t st) {
    static unsigned long long configured = 0;            // devices whose shared-memory limit is raised
    const unsigned long long dbit = device_bit();
    const int smem = 128 * a.Ks + 2 * a.NS * a.Ks + tb.np * 512;
    if (!(configured & dbit) || !dbit) {
        int rc = (int)cudaFuncSetAttribute(k_rns_split_mma<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRnsSmemCap);
        if (rc) return rc;
        configured |= dbit;
    }
    if (a.nb == 0 || a.Rp == 0) return 0;
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    const int64_t items = (a.Kp / 16) * ((a.Rp + 7) / 8) * a.nb;
    const int64_t ctas = items < 2 * (int64_t)sms ? items : 2 * (int64_t)sms;   // two CTAs per SM, persistent
    k_rns_split_mma<L><<<(unsigned)ctas, 128, smem, st>>>(a, tb);
    return (int)cudaGetLastError();
}

template <int L>
int RnsLaunch<L>::crt_mma(const RnsCrt& a, const RnsTables& tb, cudaStream_t st) {
    static unsigned long long configured = 0;            // devices whose shared-memory limit is raised
    const unsigned long long dbit = device_bit();
    const int smem = (128 + 2 * a.NH) * a.Kc;
    if (!(configured & dbit) || !dbit) {
        int rc = (int)cudaFuncSetAttribute(k_rns_crt_mma<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, kRnsSmemCap);
        if (rc) return rc;
        configured |= dbit;
    }
    if (a.n == 0) return 0;
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    const int64_t tiles = (a.n + 127) / 128;
    const int64_t ctas = tiles < (int64_t)sms ? tiles : (int64_t)sms;     // persistent, one CTA per SM (TMEM 512)
    k_rns_crt_mma<L><<<(unsigned)ctas, 128, smem, st>>>(a, tb);
    return (int)cudaGetLastError();
}
#endif

}  // namespace b3d
