// Pole step on the sm_100a INT8 tensor cores (tcgen05.mma.kind::i8, s8 x s8 -> s32 accumulators in TMEM).
//
// One stage of the pole step is, per task t, Out[i, n] = sum_j C[i, j] X[j, n] over S x S multiprecision
// constants C (rows aligned, one exponent per row) and S x N numbers X (aligned per column n over j here),
// each output an exact sum rounded once: the same results as k_pole1 / k_pole2 bit for bit.
//
// The exact products are byte convolutions.  Both operands are written in balanced base-256 digits
// (d in [-128, 127]: the bytes of v + 0x8080...80, each minus 128), so that
//     sum_j C[i, j] X[j, n] = sum_p D[p, n] 256^p,   D[p, n] = sum_j sum_u c_ij[p - u] x_jn[u],
// and D is one int8 GEMM per row i: A[p, (j, u')] = c_ij[p - U + 1 + u'] (positions p on the 128 TMEM
// lanes, a Hankel matrix in (p, u')), B[n, (j, u')] = x_jn[U - 1 - u'] (the digits of each X entry reversed
// along K).  The Hankel operand is never materialised: its 16 x 16 blocks depend only on the sum of the
// block coordinates, so one 16-byte window of c_ij per byte offset o, stored at 16 o, is addressed by the
// canonical no-swizzle K-major descriptor with LBO = 256 (next K chunk = 16 offsets on) and SBO = 128
// (next 8 rows = 8 offsets on).  |D| <= S 4 L 2^14 < 2^31: no wrap.
//
// Positions below P0 (a multiple of 16; zero when two 128-lane tiles cover the whole product) are not
// computed.  Their sum is below 2^(8 P0 + 17) in magnitude, far under the rounding point of the result;
// the rounding is kept where no value that close rounds differently (the test of round_safe), and where it
// is not (exact cancellation, a sum at a rounding midpoint) the thread adds the missing positions exactly
// from the digits still in shared memory.
//
// One CTA (128 threads) per (task, column chunk of NC <= 32 columns), persistent over the work list:
//   1. column exponents, then the aligned X digits into the K-major B operand (16-byte stores);
//   2. per row i: the padded digit strings of c_ij (the next row's constants load meanwhile), the Hankel
//      windows (four per thread step, byte permutations of five words, stored in a rotated order that
//      keeps the stores free of bank conflicts), fence.proxy.async, one thread issues MT x S x U / 32 MMAs
//      (M = 128, N = NC, K = 32), commits to an mbarrier and waits for it;
//   3. per tile of 128 positions, tcgen05.ld of the accumulators, transposed through shared memory
//      (D[n][p]); the carry chain (64-bit multiply-adds of four positions per limb) in segments of eight
//      limbs, one per warp and a lane per column, into a shared-memory limb column; then one header thread
//      per column joins the segments' carries, checks the rounding and decides it (top limb, shift, carry
//      and sign extents), and all threads write the rounded limbs, a lane per column (runs of consecutive
//      outputs in each limb plane).
// Every mbarrier wait is bounded; on expiry the CTA records an error code, waits (bounded) for its own MMAs,
// frees its TMEM and returns.
#pragma once
#include <cuda_runtime.h>

#include "kernels.cuh"
#include "rns.cuh"

namespace b3d {

template <int L>
struct PoleMmaGeom {
    static constexpr int NB = nb_bits(L);
    static constexpr int D = 4 * L;                                 // digits of a number
    static constexpr int U = 32 * ((D + 31) / 32);                  // digits per entry along K (MMA K step 32)
    static constexpr int p0_for(int mt) {
        return 8 * L - 1 - 128 * mt <= 0 ? 0 : 16 * ((8 * L - 1 - 128 * mt + 15) / 16);
    }
    // one tile of 128 positions where the dropped part stays 160 bits below the result's rounding point
    static constexpr int MT = (8 * p0_for(1) + 17 <= NB - 160) ? 1 : 2;
    static constexpr int P0 = p0_for(MT);                            // first position computed
    static constexpr int NWIN = 128 * MT + U - 16;                  // Hankel windows per entry (a multiple of 16)
    static constexpr int FAM = 16 * NWIN;                           // bytes of one entry's windows
    static constexpr int PADB = U;                                  // zero bytes before a digit string
    static constexpr int CW = (P0 + 128 * MT + 2 * U) / 4 + 2;      // words of a padded digit string
    static constexpr int NW = 2 * L + 2;                            // accumulator limbs
    static constexpr int EW = P0 / 4 + 1;                           // error of the truncated sum < 2^(32 EW)
    static constexpr int VW = 32 * MT;                              // 4-position words per column
    static constexpr int DS = 128 + 4;                              // words per transposed column of a tile (16-byte rows)
    static_assert(8 * P0 + 17 <= NB - 160, "two tiles must reach the rounding point");
    static_assert(U / 4 + L <= CW, "digit string inside its padded buffer");
    static_assert(NWIN % 4 == 0 && (P0 + 1) % 4 == 1, "window groups start one byte after a word");
};

struct PoleMmaArgs {
    const int32_t* xm; const i64* xe; i64 xplane;   // X: (rows, S, S, B) limb planes
    const int32_t* cm; const i64* ce; i64 cplane;   // constant tables (n, S, S), row exponents (n, S)
    const i64* t_x;                                 // (T) X row per task, or null (row t)
    const i64* t_c;                                 // (T) constant table per task
    const i64* t_o;                                 // (T) output row per task, or null (row t)
    int32_t* om; i64* oe; i64 oplane;               // output (rows, S, S, B)
    i64 T, B;
    int S;
    int stage;                                      // 1: X[a, j, k] summed over j; 2: X[j, b0, k] summed over j
    int NC, nchunks;                                // columns per CTA work item (multiple of 16), chunks per task
    int* err;                                       // device error flag (0 = ok)
};

constexpr int kPoleMmaThreads = 128;
constexpr int kPoleMmaMaxS = 8;
constexpr int kPoleMmaMaxNC = 32;

__host__ __device__ constexpr size_t pm_align(size_t x) { return (x + 127) & ~size_t(127); }

// dynamic shared memory: B operand | Hankel windows, reused by the transposed accumulators and the limb
// columns once the MMAs are done | padded digit strings of two rows (this one and the next) | column exponents
template <int L>
struct PoleMmaSmem {
    using G = PoleMmaGeom<L>;
    static __host__ __device__ size_t bop(int S, int NC) { return pm_align((size_t)S * G::U * NC); }
    static __host__ __device__ size_t dbuf(int NC) { return (size_t)NC * G::DS * 4; }
    static __host__ __device__ size_t hank(int S, int NC) {
        const size_t h = (size_t)S * G::FAM, v = dbuf(NC) + (size_t)G::NW * (NC + 1) * 4;
        return pm_align(h > v ? h : v);
    }
    static __host__ __device__ size_t cdig(int S) { return pm_align((size_t)2 * S * G::CW * 4); }   // two rows
    static __host__ __device__ size_t total(int S, int NC) {
        return bop(S, NC) + hank(S, NC) + cdig(S) + pm_align((size_t)NC * 8);
    }
};

// v (two's complement, L words) -> balanced base-256 digits, four per word (little-endian bytes, as s8)
template <int L> __device__ __forceinline__ void to_balanced(u32 (&v)[L]) {
    u32 c = 0;
#pragma unroll
    for (int k = 0; k < L; k++) {
        const u64 s = (u64)v[k] + 0x80808080u + c;
        c = (u32)(s >> 32);
        v[k] = (u32)s ^ 0x80808080u;
    }
}

__device__ __forceinline__ int sbyte(const uint8_t* p, int i) { return (int)(int8_t)p[i]; }

// Offsets inside a task's (S, S, B) block: X entry (j, column n) at coff(n) + j * jst, output (i, column n) at
// coff(n) + i * jst, with n = a B + k in stage 1 (X[a, j, k], Y[a, i, k]) and n = b0 B + k in stage 2
// (Y[j, b0, k], res[i, b0, k]).  32-bit arithmetic: a block holds S^2 B < 2^31 numbers.
__device__ __forceinline__ int pm_coff(const PoleMmaArgs& a, int n) {
    const int B = (int)a.B;
    return a.stage == 1 ? (n / B) * a.S * B + n % B : n;
}

__device__ __forceinline__ int pm_jst(const PoleMmaArgs& a) { return a.stage == 1 ? (int)a.B : a.S * (int)a.B; }

template <int L> __device__ __forceinline__ void pm_store_zero(const PoleMmaArgs& a, i64 o) {
#pragma unroll
    for (int k = 0; k < L; k++) a.om[k * a.oplane + o] = 0;
    a.oe[o] = EZ;
}

// Magnitude view of a two's complement limb column col[k * st] (k < NW): limb i of |value|.  With neg, z is
// the lowest nonzero limb: -x = ~x + 1, and the +1 only reaches the limbs up to z.
template <int NW>
struct PmCol {
    const u32* col;
    int st, z, lo;                                                  // limbs below lo are zero
    bool neg;
    __device__ __forceinline__ u32 conv(int i, u32 v) const {
        return neg ? (i > z ? ~v : (i == z ? 0u - v : 0u)) : v;
    }
    __device__ __forceinline__ u32 operator()(int i) const {
        return (i < 0 || i >= NW) ? 0u : conv(i, col[i * st]);
    }
    __device__ __forceinline__ void init() {
        neg = (col[(NW - 1) * st] >> 31) != 0;
        z = lo;
        if (neg)
            while (z < NW - 1 && col[z * st] == 0) z++;
    }
    // bit length of the magnitude (0 for zero), by a scan from the top limb
    __device__ __forceinline__ int bitlen() const {
        for (int i = NW - 1; i >= lo; i--) {
            const u32 m = (*this)(i);
            if (m) return 32 * i + 32 - __clz(m);
        }
        return 0;
    }
};

// round_safe of mp.cuh on a magnitude view of bit length bl: every value within 2^(32 EW) rounds alike
template <int L, int EW, class Mag>
__device__ __forceinline__ bool pm_round_safe(const Mag& m, int bl) {
    const int hb = bl - nb_bits(L) - 1;
    if (hb < 32 * EW + 2) return false;
    const u32 flip = ((m(hb >> 5) >> (hb & 31)) & 1u) ? 0u : ~0u;
    for (int k = hb >> 5; k >= EW; k--) {
        const int lo = 32 * k;
        const u32 mask = hb >= lo + 32 ? ~0u : (hb > lo ? (1u << (hb - lo)) - 1u : 0u);
        if ((m(k) ^ flip) & mask) return true;
    }
    return false;
}

// round_mag of mp.cuh on a magnitude view of bit length bl > 0: r and the exponent ein + shift, the same bits.
// The L + 2 limbs the rounding reads are loaded in one batch from the run-time word offset.
template <int L, int NW>
__device__ __forceinline__ i64 pm_round(const PmCol<NW>& m, int bl, i64 ein, u32 (&r)[L]) {
    constexpr int NB = nb_bits(L);
    int s = bl - NB;
    if (s <= 0) {                                                   // fewer than NB bits: exact left shift
        const int q = (-s) >> 5, f = (-s) & 31;
#pragma unroll
        for (int k = 0; k < L; k++) r[k] = fsl(m(k - q - 1), m(k - q), f);
        return ein + s;
    }
    const int q = (s - 1) >> 5, f = (s - 1) & 31;                  // q + L + 1 <= NW
    u32 v[L + 2];
#pragma unroll
    for (int k = 0; k < L + 2; k++) v[k] = q + k < NW ? m.col[(q + k) * m.st] : 0u;
#pragma unroll
    for (int k = 0; k < L + 2; k++) v[k] = q + k < NW ? m.conv(q + k, v[k]) : 0u;
    u32 t[L + 1];
#pragma unroll
    for (int k = 0; k <= L; k++) t[k] = fsr(v[k], v[k + 1], f);
    u32 c = t[0] & 1u;
#pragma unroll
    for (int k = 0; k < L; k++) {
        const u32 x = (t[k] >> 1) | (t[k + 1] << 31);
        const u32 sum = x + c;
        c = (c && sum == 0) ? 1u : 0u;
        r[k] = sum;
    }
    if ((r[L - 1] >> (NB - 32 * (L - 1))) != 0) {
#pragma unroll
        for (int k = 0; k < L; k++) r[k] = (r[k] >> 1) | (k + 1 < L ? r[k + 1] << 31 : 0u);
        s += 1;
    }
    return ein + s;
}

// The rounding of one column decided by its header thread, so that every output limb can then be formed
// on its own: magnitude limbs from the column (neg, z as in PmCol), x = floor(|sum| / 2^s) with s = 32 Q + F,
// the half bit c0, the carry of the rounding reaching limbs 0 .. kc, and for the two's complement store the
// lowest nonzero limb kz of the rounded magnitude.
struct PmHead {
    enum { kZero = 0, kLimbs = 1, kRenorm = 2, kDone = 3 };
    int mode, s, Q, F, z, kc, kz, c0, neg;
};

template <int NW>
__device__ __forceinline__ u32 pm_mag(const u32* col, int st, int i, bool neg, int z) {
    if (i < 0 || i >= NW) return 0u;
    const u32 v = col[i * st];
    return neg ? (i > z ? ~v : (i == z ? 0u - v : 0u)) : v;
}

template <int L, int NW>
__device__ __forceinline__ PmHead pm_head(const PmCol<NW>& m, int bl) {
    constexpr int NB = nb_bits(L);
    PmHead h{};
    h.s = bl - NB;
    h.neg = m.neg;
    h.z = m.z;
    if (h.s <= 0) { h.mode = PmHead::kDone; return h; }
    h.Q = h.s >> 5;
    h.F = h.s & 31;
    h.c0 = (int)((m((h.s - 1) >> 5) >> ((h.s - 1) & 31)) & 1u);
    auto x = [&](int k) { return fsr(m(h.Q + k), m(h.Q + k + 1), h.F); };
    h.mode = PmHead::kLimbs;
    if (h.c0) {
        int k = 0;
        u32 xk = x(0);
        while (xk == 0xFFFFFFFFu && k < L - 1) xk = x(++k);
        h.kc = k;
        h.kz = k;                                                   // rounded limbs below kc are zero, kc is not
        if (k == L - 1 && xk + 1u == (1u << (NB - 32 * (L - 1)))) h.mode = PmHead::kRenorm;
    } else {
        h.kc = -1;
        int k = 0;
        while (k < L - 1 && x(k) == 0u) k++;
        h.kz = k;
    }
    return h;
}

// limb k of the stored (two's complement) result of a header
template <int L, int NW>
__device__ __forceinline__ u32 pm_limb(const PmHead& h, const u32* col, int st, int k) {
    constexpr int NB = nb_bits(L);
    u32 r;
    if (h.mode == PmHead::kZero) return 0u;
    if (h.mode == PmHead::kRenorm) {
        r = k == L - 1 ? 1u << (NB - 1 - 32 * (L - 1)) : 0u;
        return h.neg ? (k == L - 1 ? 0u - r : (k < L - 1 ? 0u : ~r)) : r;
    }
    const u32 xk = fsr(pm_mag<NW>(col, st, h.Q + k, h.neg, h.z), pm_mag<NW>(col, st, h.Q + k + 1, h.neg, h.z), h.F);
    r = xk + (k <= h.kc ? 1u : 0u);
    if (!h.neg) return r;
    return k < h.kz ? 0u : (k == h.kz ? 0u - r : ~r);
}

// limbs [w KQ, (w + 1) KQ) of the stored result (KQ = ceil(L / 4)), written to out[k * plane]: the KQ + 1
// magnitude limbs they read are loaded once
template <int L, int NW>
__device__ __forceinline__ void pm_limbs(const PmHead& h, const u32* col, int st, int w, int32_t* out, i64 plane) {
    constexpr int NB = nb_bits(L), KQ = (L + 3) / 4;
    const int k0 = w * KQ;
    if (h.mode != PmHead::kLimbs) {
#pragma unroll
        for (int q = 0; q < KQ; q++) {
            const int k = k0 + q;
            if (k < L) out[k * plane] = (int32_t)pm_limb<L, NW>(h, col, st, k);
        }
        return;
    }
    u32 mm[KQ + 1];
#pragma unroll
    for (int q = 0; q <= KQ; q++) mm[q] = pm_mag<NW>(col, st, h.Q + k0 + q, h.neg, h.z);
#pragma unroll
    for (int q = 0; q < KQ; q++) {
        const int k = k0 + q;
        if (k < L) {
            const u32 r = fsr(mm[q], mm[q + 1], h.F) + (k <= h.kc ? 1u : 0u);
            out[k * plane] = (int32_t)(!h.neg ? r : (k < h.kz ? 0u : (k == h.kz ? 0u - r : ~r)));
        }
    }
    (void)NB;
}

// col (two's complement limbs, stride st) += sum_{p < P0} D[p, n] 256^p, from the digits in shared memory
// (the rare exact redo)
template <int L>
__device__ void pm_add_low(u32* col, int st, const u32* cdig, const uint8_t* bop, int S, int NC, int n) {
    using G = PoleMmaGeom<L>;
    constexpr int P0 = G::P0, U = G::U, D = G::D;
    i64 c = 0;
    for (int k = 0; k < G::NW; k++) {
        i64 v = 0;
        if (k < P0 / 4) {
            for (int r = 0; r < 4; r++) {
                const int p = 4 * k + r;
                i64 cp = 0;
                for (int j = 0; j < S; j++) {
                    const uint8_t* cd = reinterpret_cast<const uint8_t*>(cdig + j * G::CW) + G::PADB;
                    for (int u = 0; u <= p && u < D; u++) {
                        if (p - u >= D) continue;
                        const int kap = j * U + (U - 1 - u);            // reversed digit index along K
                        const int xd = sbyte(bop, (kap >> 4) * 16 * NC + (n >> 3) * 128 + (n & 7) * 16 + (kap & 15));
                        cp += (i64)sbyte(cd, p - u) * xd;
                    }
                }
                v += cp * ((i64)1 << (8 * r));
            }
        }
        const i64 s = (i64)col[k * st] + v + c;
        col[k * st] = (u32)s;
        c = s >> 32;
    }
}

// warp 1, lane j < S: the digit string of c_ij (its magnitude and sign in c, ng) into a padded buffer
template <int L>
__device__ __forceinline__ void pm_put_digits(u32 (&c)[L], bool ng, u32* dst) {
    if (ng) negate(c);
    to_balanced(c);
#pragma unroll
    for (int k = 0; k < L; k++) dst[k] = c[k];
}

template <int L>
__global__ void __launch_bounds__(kPoleMmaThreads, 3) k_pole_mma(PoleMmaArgs a) {
    using G = PoleMmaGeom<L>;
    using SM = PoleMmaSmem<L>;
    constexpr int U = G::U, MT = G::MT, NW = G::NW, VW = G::VW, CW = G::CW, FAM = G::FAM, NWIN = G::NWIN,
                  DS = G::DS, P0 = G::P0;
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_sh;
    __shared__ int fail_sh;
    __shared__ i64 carr[8][kPoleMmaMaxNC];                          // carry out of each chain segment
    __shared__ i64 er_sh[kPoleMmaMaxS];                             // row exponents of the task's constant
    __shared__ PmHead head[kPoleMmaMaxNC];                          // the rounding of each column
    __shared__ int coff_sh[kPoleMmaMaxNC];                          // column offsets inside the task's block

    const int S = a.S, NC = a.NC, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ncs = NC == 32 ? 5 : 4;                               // NC is 16 or 32
    const bool cthread = warp == 1 && lane < S;                     // the constants' digit strings
    const i64 N = (i64)S * a.B;
    uint8_t* bop = smem;
    uint8_t* hank = smem + SM::bop(S, NC);
    u32* dbuf = reinterpret_cast<u32*>(hank);                       // D[n][p]: reuses the windows after the MMAs
    u32* accs = dbuf + (size_t)NC * DS;                              // limb k of column n at accs[k * (NC + 1) + n]
    const int ast = NC + 1;
    u32* cdig = reinterpret_cast<u32*>(hank + SM::hank(S, NC));    // row r at cdig + (r % 2) S CW
    i64* ecol = reinterpret_cast<i64*>(reinterpret_cast<uint8_t*>(cdig) + SM::cdig(S));
    uint32_t ncols = 32;
    while (ncols < (uint32_t)(MT * NC)) ncols <<= 1;

    for (int q = tid; q < 2 * S * CW; q += blockDim.x) cdig[q] = 0;   // padding stays zero: digits go to [PADB, PADB + D)
    if (tid == 0) {
        fail_sh = 0;
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_sh)), "r"(ncols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_sh;
    // instruction descriptor: s32 accumulator, s8 x s8, both K-major, M = 128, N = NC
    const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NC >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
    // descriptors of the first A and B core matrices; the others differ only in the 14-bit address field
    const uint64_t da0 = umma_desc(smem_u32(hank), 256, 128), db0 = umma_desc(smem_u32(bop), 16 * NC, 128);
    uint32_t phase = 0;
    int pending = 0;                                                // thread 0: a commit not yet waited for

    const i64 items = a.T * a.nchunks;
    for (i64 w = blockIdx.x; w < items; w += gridDim.x) {
        const i64 t = w / a.nchunks;
        const i64 n0 = (w % a.nchunks) * (i64)NC;
        const int nn = (int)(N - n0 < NC ? N - n0 : NC);
        const i64 xrow = a.t_x ? a.t_x[t] : t, crow = a.t_c[t], orow = a.t_o ? a.t_o[t] : t;

        // 1. the constants of row 0 (digits now) and row 1 (loaded, converted during row 0), row exponents
        u32 cn[L];
        bool cneg = false;
        if (cthread) {
            cneg = load_mag<L>(a.cm, a.cplane, crow * S * S + lane, cn);
            er_sh[lane] = a.ce[crow * S + lane];
            pm_put_digits<L>(cn, cneg, cdig + lane * CW + G::PADB / 4);
            if (S > 1) cneg = load_mag<L>(a.cm, a.cplane, (crow * S + 1) * S + lane, cn);
        }
        const i64 xbase = xrow * S * S * a.B, obase = orow * S * S * a.B;
        const int jst = pm_jst(a);
        // column exponents: the largest over j of the nonzero entries (all loads of a column issued at once)
        for (int n = tid; n < NC; n += blockDim.x) {
            i64 E = EZ;
            const int co = n < nn ? pm_coff(a, (int)n0 + n) : 0;
            coff_sh[n] = co;
            if (n < nn) {
                i64 ev[kPoleMmaMaxS];
                int32_t tv[kPoleMmaMaxS];
#pragma unroll
                for (int j = 0; j < kPoleMmaMaxS; j++) {
                    if (j < S) {
                        const i64 ix = xbase + co + j * jst;
                        ev[j] = a.xe[ix];
                        tv[j] = a.xm[(L - 1) * a.xplane + ix];
                    }
                }
#pragma unroll
                for (int j = 0; j < kPoleMmaMaxS; j++)
                    if (j < S && tv[j] != 0 && ev[j] > E) E = ev[j];
            }
            ecol[n] = E;
        }
        __syncthreads();
        // the aligned X digits into the B operand
        for (int it = tid; it < S * NC; it += blockDim.x) {
            const int j = it >> ncs, n = it & (NC - 1);
            u32 dg[L];
            zero(dg);
            const i64 E = ecol[n];
            if (n < nn) {
                const i64 ix = xbase + coff_sh[n] + j * jst;
                u32 x[L];
                const bool neg = load_mag<L>(a.xm, a.xplane, ix, x);
                const i64 ex = a.xe[ix];
                if (E != EZ && !is_zero(x) && ex != EZ && E - ex < 32 * L) {
                    shr(x, (int)(E - ex), dg);
                    if (neg) negate(dg);
                }
            }
            to_balanced(dg);
            uint8_t* col = bop + (n >> 3) * 128 + (n & 7) * 16;
#pragma unroll
            for (int c = 0; c < U / 16; c++) {
                u32 q[4];
#pragma unroll
                for (int r = 0; r < 4; r++) {
                    const int wd = U / 4 - 1 - (4 * c + r);            // reversed words, bytes reversed inside
                    q[r] = wd < L ? __byte_perm(dg[wd], 0, 0x0123) : 0u;
                }
                *reinterpret_cast<uint4*>(col + (size_t)(j * (U / 16) + c) * 16 * NC) = make_uint4(q[0], q[1], q[2], q[3]);
            }
        }
        __syncthreads();

        // 2. rows
        bool stop = false;
        for (int i = 0; i < S; i++) {
            const i64 Er = er_sh[i];
            const u32* cd = cdig + (i & 1) * S * CW;
            if (Er == EZ) {                                          // a zero row of the constant: exact zeros
                for (int n = tid; n < nn; n += blockDim.x) pm_store_zero<L>(a, obase + coff_sh[n] + i * jst);
                if (cthread && i + 1 < S) {
                    pm_put_digits<L>(cn, cneg, cdig + ((i + 1) & 1) * S * CW + lane * CW + G::PADB / 4);
                    if (i + 2 < S) cneg = load_mag<L>(a.cm, a.cplane, (crow * S + i + 2) * S + lane, cn);
                }
                __syncthreads();
                continue;
            }
            // windows o .. o + 3 (o a multiple of 4) start at bytes P0 + 1 + o .. of the padded string: words
            // ws .. ws + 4 shifted by 1 to 4 bytes.  The thread stores them in the rotated order k' = (k + t / 2) % 4
            // so that the eight threads of each store phase cover all 32 banks.
            for (int it = tid; it < S * (NWIN / 4); it += blockDim.x) {
                const int j = it / (NWIN / 4), o = 4 * (it % (NWIN / 4));
                const u32* cw = cd + j * CW + ((P0 + o) >> 2);
                const u32 w0 = cw[0], w1 = cw[1], w2 = cw[2], w3 = cw[3], w4 = cw[4];
                uint4* dst = reinterpret_cast<uint4*>(hank + (size_t)j * FAM + 16 * o);
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const int kp = (k + (tid >> 1)) & 3;
                    const u32 sel = 0x4321u + 0x1111u * (u32)kp;
                    dst[kp] = make_uint4(__byte_perm(w0, w1, sel), __byte_perm(w1, w2, sel), __byte_perm(w2, w3, sel),
                                         __byte_perm(w3, w4, sel));
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // generic writes -> tensor-core reads
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
                for (int mt = 0; mt < MT; mt++) {
#pragma unroll 1
                    for (int j = 0; j < S; j++) {
                        const uint64_t da = da0 + (uint64_t)((j * FAM + 2048 * mt) >> 4);
                        const uint64_t db = db0 + (uint64_t)((j * (U / 16) * 16 * NC) >> 4);
#pragma unroll
                        for (int ks = 0; ks < U / 32; ks++) {
                            const uint32_t accf = (j > 0 || ks > 0) ? 1u : 0u;
                            asm volatile(
                                "{\n\t.reg .pred p;\n\t"
                                "setp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
                                ::"r"(tmem + (uint32_t)(mt * NC)), "l"(da + (uint64_t)(32 * ks)),
                                  "l"(db + (uint64_t)(2 * ks * NC)), "r"(idesc), "r"(accf) : "memory");
                        }
                    }
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                             ::"r"(smem_u32(&bar)) : "memory");
                pending = 1;
                if (!mbar_wait(&bar, phase, kWaitLimit)) fail_sh = 1;
                else pending = 0;
            } else if (cthread && i + 1 < S) {                       // next row's digits while the MMAs run
                pm_put_digits<L>(cn, cneg, cdig + ((i + 1) & 1) * S * CW + lane * CW + G::PADB / 4);
                if (i + 2 < S) cneg = load_mag<L>(a.cm, a.cplane, (crow * S + i + 2) * S + lane, cn);
            }
            phase ^= 1;
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncthreads();
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (fail_sh) { stop = true; break; }

            // 3. per tile of 128 positions: accumulators -> D[n][p] in shared memory (this lane's position p,
            // sixteen columns per load), then the carry chain in four segments of eight limbs (warp s: words
            // 32 mt + 8 s .. + 8 of every column, lane = column), each from a zero carry; the carries out are
            // joined below
#pragma unroll 1
            for (int mt = 0; mt < MT; mt++) {
                const int p = warp * 32 + lane;
#pragma unroll 1
                for (int c0 = 0; c0 < NC; c0 += 16) {
                    uint32_t d[16];
                    asm volatile(
                        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]),
                          "=r"(d[7]), "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]),
                          "=r"(d[14]), "=r"(d[15])
                        : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(mt * NC + c0)));
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int q = 0; q < 16; q++) dbuf[(c0 + q) * DS + p] = d[q];
                }
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncthreads();
                if (lane < nn) {
                    const int n = lane;
                    u32* col = accs + n;
                    const int4* dn = reinterpret_cast<const int4*>(dbuf + (size_t)n * DS);
                    i64 c = 0;
#pragma unroll
                    for (int q = 0; q < 8; q++) {
                        const int k = P0 / 4 + 32 * mt + 8 * warp + q;
                        if (k < NW) {
                            const int4 d = dn[8 * warp + q];
                            const i64 s = c + (i64)d.x + (i64)d.y * 256 + (i64)d.z * 65536 + (i64)d.w * 16777216;
                            col[k * ast] = (u32)s;
                            c = s >> 32;
                        }
                    }
                    carr[4 * mt + warp][n] = c;
                }
                __syncthreads();
            }

            // join the segments, check the rounding (exact redo of the low positions where needed) and decide the
            // rounded number: one header thread per column (column n on warp n % 4, lane n / 4)
            {
                const int n = 4 * lane + warp;
                if (n < nn) {
                    PmHead h{};
                    h.mode = PmHead::kZero;
                    const i64 out = obase + coff_sh[n] + i * jst;
                    const i64 E = ecol[n];
                    if (E != EZ) {
                        u32* col = accs + n;
                        // segment sg (sg >= 1) receives the carry out of segment sg - 1 (all segments at once);
                        // what then runs out of the top of a segment (rare) is passed on in order afterwards
                        constexpr int NSEG = 4 * MT;
                        i64 e[NSEG];
#pragma unroll
                        for (int sg = 0; sg < NSEG; sg++) {
                            i64 c = sg > 0 ? carr[sg - 1][n] : 0;
                            const int k0 = P0 / 4 + 8 * sg, kend = k0 + 8 < NW ? k0 + 8 : NW;
                            for (int k = k0; c != 0 && k < kend; k++) {
                                const i64 v = (i64)col[k * ast] + c;
                                col[k * ast] = (u32)v;
                                c = v >> 32;
                            }
                            e[sg] = c;
                        }
                        i64 x = 0;
#pragma unroll
                        for (int sg = 1; sg < NSEG; sg++) {
                            x += e[sg - 1];
                            const int k0 = P0 / 4 + 8 * sg, kend = k0 + 8 < NW ? k0 + 8 : NW;
                            for (int k = k0; x != 0 && k < kend; k++) {
                                const i64 v = (i64)col[k * ast] + x;
                                col[k * ast] = (u32)v;
                                x = v >> 32;
                            }
                        }
                        i64 C = carr[NSEG - 1][n] + x + e[NSEG - 1];
                        for (int k = P0 / 4 + VW; k < NW; k++) {
                            col[k * ast] = (u32)C;
                            C >>= 32;
                        }
                        PmCol<NW> m{col, ast, 0, P0 / 4, false};
                        m.init();
                        int bl = m.bitlen();
                        if (P0 > 0 && !pm_round_safe<L, G::EW>(m, bl)) {
                            for (int k = 0; k < P0 / 4; k++) col[k * ast] = 0u;
                            pm_add_low<L>(col, ast, cd, bop, S, NC, n);
                            m.lo = 0;
                            m.init();
                            bl = m.bitlen();
                        }
                        if (bl > 0) h = pm_head<L, NW>(m, bl);
                        if (h.mode == PmHead::kDone) {                   // fewer than NB bits: rounded here
                            u32 r[L];
                            const i64 er = pm_round<L, NW>(m, bl, E + Er, r);
                            store_signed<L>(a.om, a.oplane, out, r, m.neg);
                            a.oe[out] = er;
                        } else if (h.mode != PmHead::kZero) {
                            a.oe[out] = E + Er + h.s + (h.mode == PmHead::kRenorm ? 1 : 0);
                        }
                    }
                    if (h.mode == PmHead::kZero) a.oe[out] = EZ;
                    head[n] = h;
                }
            }
            __syncthreads();
            // the rounded limbs: a quarter of the limbs per warp, a lane per column, so that each limb plane is
            // written in runs of consecutive outputs
            if (lane < nn) {
                const PmHead h = head[lane];
                const i64 out = obase + coff_sh[lane] + i * jst;
                if (h.mode != PmHead::kDone) pm_limbs<L, NW>(h, accs + lane, ast, warp, a.om + out, a.oplane);
            }
            __syncthreads();                                         // D, the limb columns and windows are reused
        }
        if (stop) break;
    }
    if (tid == 0 && pending) {                                       // bounded drain of our own MMAs
        if (!mbar_wait(&bar, phase ^ 1, kWaitLimit)) fail_sh = 2;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
    }
    if (tid == 0 && fail_sh) atomicExch(a.err, fail_sh);
}

#ifdef B3D_DEFINE_LAUNCH
// columns per work item: all of a task's S B columns up to kPoleMmaMaxNC, in multiples of 16 (the MMA's N step)
inline int pole_mma_nc(i64 N) { return (int)(N >= kPoleMmaMaxNC ? kPoleMmaMaxNC : ((N + 15) / 16) * 16); }

template <int L>
static int pole_mma_stage(PoleMmaArgs a, cudaStream_t st) {
    if (a.T == 0) return 0;
    const size_t smem = PoleMmaSmem<L>::total(a.S, a.NC);
    static unsigned long long configured = 0;                       // devices whose limits are raised
    const unsigned long long dbit = device_bit();
    if (!(configured & dbit) || !dbit) {
        int rc = (int)cudaFuncSetAttribute(k_pole_mma<L>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (!rc) rc = (int)cudaFuncSetAttribute(k_pole_mma<L>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (rc) return rc;
        configured |= dbit;
    }
    int dev = 0, sms = 0;
    int rc = (int)cudaGetDevice(&dev);
    if (!rc) rc = (int)cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (rc) return rc;
    // resident CTAs per SM: three by the launch bounds (registers), fewer when the shared memory (228 KB per
    // SM: static + dynamic + 1 KB reserved per CTA) or the 512 TMEM columns do not hold three
    static size_t static_smem = 0;
    if (!static_smem) {
        cudaFuncAttributes fa;
        const int rc2 = (int)cudaFuncGetAttributes(&fa, k_pole_mma<L>);
        if (rc2) return rc2;
        static_smem = fa.sharedSizeBytes + 1;
    }
    int ncols = 32;
    while (ncols < PoleMmaGeom<L>::MT * a.NC) ncols <<= 1;
    int occ = (int)((228 * 1024) / (smem + static_smem + 1024));
    if (occ > 3) occ = 3;
    if (occ > 512 / ncols) occ = 512 / ncols;
    if (occ < 1) return (int)cudaErrorInvalidConfiguration;
    const i64 items = a.T * a.nchunks;
    const i64 grid = items < (i64)sms * occ ? items : (i64)sms * occ;
    k_pole_mma<L><<<(unsigned)grid, kPoleMmaThreads, smem, st>>>(a);
    return (int)cudaGetLastError();
}

template <int L>
int Launch<L>::pole_mma(const int32_t* hm, const i64* he, i64 hplane, const int32_t* Rm, const i64* Re, i64 Rplane,
                        const int32_t* Qm, const i64* Qe, i64 Qplane, const i64* t_hrow, const i64* t_R, const i64* t_qL,
                        const i64* t_slot, i64 T, i64 B, int S, int32_t* ym, i64* ye, i64 yplane,
                        int32_t* rm, i64* re, i64 rplane, int* err, cudaStream_t st) {
    if (T == 0) return 0;
    if (S > kPoleMmaMaxS || !err) return (int)cudaErrorInvalidValue;
    const int NC = pole_mma_nc((i64)S * B);
    const int nchunks = (int)(((i64)S * B + NC - 1) / NC);
    PoleMmaArgs s1{hm, he, hplane, Rm, Re, Rplane, t_hrow, t_R, nullptr, ym, ye, yplane, T, B, S, 1, NC, nchunks, err};
    int rc = pole_mma_stage<L>(s1, st);
    if (rc) return rc;
    PoleMmaArgs s2{ym, ye, yplane, Qm, Qe, Qplane, nullptr, t_qL, t_slot, rm, re, rplane, T, B, S, 2, NC, nchunks, err};
    return pole_mma_stage<L>(s2, st);
}
#endif

}  // namespace b3d
