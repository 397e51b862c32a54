// CUDA-core kernels of the blocks_3d hot path (sm_100a): multiprecision alignment, products, batched
// GEMM, the recursion's Cauchy and pole steps, and the derivative moments.  Every kernel is a template
// over the limb count L; inst.cu instantiates the launchers once per L, abi.cu dispatches on L.
#pragma once
#include <type_traits>
#include <cuda_runtime.h>

#include "mp.cuh"

namespace b3d {

// Per-level tables of the Cauchy step (device pointers; see Plan in the Python host code).
struct CauchyLevel {
    i64 m, nb, Mr, Kc, N;          // level, groups, rows per group, columns per group, S^2 B
    i64 hlevels, Jh;               // h_inf layout: (2, hlevels, Jh, N)
    const i64* gsrc;               // (nb) source parity of each group
    const i64* gj;                 // (nb) h_inf spin index of each group
    const i64* rowd;               // (nb, Mr) 2 D' per row
    const i64* nrow;               // (nb) rows in use
    const i64* cold;               // (nb, Kc) 2 D_i per column
    const i64* ncol;               // (nb) columns in use
    const i64* col;                // (nb, Kc) physical slot of each column
};

// Index splits of a flat thread index, in 32-bit arithmetic where the whole index space fits in 31 bits
// (64-bit division is a long software sequence on the GPU; these kernels do little else per thread).
// split2: t = q N + n;  split3: t = (g K + i) N + n.
__device__ __forceinline__ void split2(i64 t, i64 N, i64 total, i64& n, i64& q) {
    if (total < (i64(1) << 31)) {
        const u32 qq = (u32)t / (u32)N;
        n = (u32)t - qq * (u32)N;
        q = qq;
    } else {
        n = t % N;
        q = t / N;
    }
}

__device__ __forceinline__ void split3(i64 t, i64 N, i64 K, i64 total, i64& n, i64& i, i64& g) {
    i64 q;
    split2(t, N, total, n, q);
    if (total < (i64(1) << 31)) {
        i = (u32)q % (u32)K;
        g = (u32)q / (u32)K;
    } else {
        i = q % K;
        g = q / K;
    }
}

// ------------------------------------------------------------------------------------------------
// Alignment: for each (batch b, row r) of a strided view X[b, r, k] (k < K), write the mantissas shifted
// to the row's largest exponent E (truncated below it) and E.  Output element (b, r, k) goes to
// (b * R + r) * K + k, or (b * K + k) * R + r when `kmajor` (columns of a GEMM's right operand).
template <int L>
__global__ void k_align(const int32_t* __restrict__ m, const i64* __restrict__ e, i64 plane,
                        i64 nbatch, i64 R, i64 K, i64 sb, i64 sr, i64 sk, const i64* __restrict__ bidx,
                        int32_t* __restrict__ om, i64* __restrict__ oe, i64 oplane, int kmajor) {
    i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (t >= nbatch * R) return;
    i64 b = t / R, r = t % R;
    i64 base = (bidx ? bidx[b] : b) * sb + r * sr;
    i64 E = EZ;
    for (i64 k = 0; k < K; k++) {
        i64 ek = e[base + k * sk];
        if (ek > E && m[(L - 1) * plane + base + k * sk] != 0) E = ek;
    }
    oe[t] = E;
    for (i64 k = 0; k < K; k++) {
        i64 src = base + k * sk;
        i64 dst = kmajor ? (b * K + k) * R + r : t * K + k;
        u32 a[L];
        bool neg = load_mag<L>(m, plane, src, a);
        i64 ek = e[src];
        u32 s[L];
        if (E == EZ || is_zero(a) || ek == EZ || E - ek >= 32 * L) {
            zero(s);
            neg = false;
        } else {
            shr(a, (int)(E - ek), s);
        }
        store_signed<L>(om, oplane, dst, s, neg);
    }
}

// Exact sums of products, rounded once, computed in two tries (the pole steps).  The first drops the product columns below
// trunc_cols<L>() (mac_signed_mem), which leaves the accumulator within 2^(32 (trunc_cols + 2)) of the exact sum;
// where round_safe shows that no value that close rounds differently, its rounding is the exact sum's.  Elsewhere
// (heavy cancellation, a sum at a rounding midpoint, exact zeros) the second try redoes the sum exactly.  With
// both operands normalised a product has about 64 L bits and the rounding bit sits near bit 32 L, so the first
// try has some 90 bits to spare.
template <int L> B3D_CX int trunc_cols() { return L >= 10 ? L - 5 : 0; }

// sum(std::integral_constant<int, C0>) fills the two's complement accumulator (limb w at acc[w * stride]) and
// returns whether it added any product.  mag receives the magnitude of an accumulator whose rounding equals the
// exact sum's; the return value is its sign.
template <int L, int NW, class Sum> __device__ __forceinline__ bool exact_sum(Sum& sum, u32* acc, int stride,
                                                                               u32 (&mag)[NW]) {
    constexpr int C0 = trunc_cols<L>();
    auto load = [&]() {
#pragma unroll
        for (int w = 0; w < NW; w++) mag[w] = acc[w * stride];
        const bool neg = (mag[NW - 1] >> 31) != 0;
        if (neg) negate(mag);
        return neg;
    };
    const bool any = sum(std::integral_constant<int, C0>());
    bool neg = load();
    if (C0 > 0 && any && !round_safe<L, NW, C0 + 2>(mag)) {
        sum(std::integral_constant<int, 0>());
        neg = load();
    }
    return neg;
}

// Round a magnitude (NW limbs, value mag * 2^ein) and store it normalised with the given sign.
template <int L, int NW> __device__ __forceinline__ void store_rounded_mag(int32_t* m, i64* e, i64 plane, i64 i,
                                                                           const u32 (&mag)[NW], bool neg, i64 ein) {
    u32 r[L];
    i64 er;
    if (!round_mag<L>(mag, ein, r, &er)) neg = false;
    store_signed<L>(m, plane, i, r, neg);
    e[i] = er;
}

// Batched product of aligned operands: C[b, i, j] = sum_k A[b, i, k] B[b, k, j] with A rows and B
// columns already aligned (k_align); exact accumulation, one rounding.  C is contiguous (b, i, j).
constexpr int kGemmThreads = 128;

template <int L>
__global__ void __launch_bounds__(kGemmThreads, 3) k_gemm_aligned(const int32_t* __restrict__ am, const i64* __restrict__ ae, i64 aplane,
                               const int32_t* __restrict__ bm, const i64* __restrict__ be, i64 bplane,
                               i64 nbatch, i64 M, i64 N, i64 K, int32_t* __restrict__ cm, i64* __restrict__ ce,
                               i64 cplane) {
    i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (t >= nbatch * M * N) return;
    i64 j = t % N, i = (t / N) % M, b = t / (M * N);
    i64 Ea = ae[b * M + i], Eb = be[b * N + j];
    constexpr int NW = 2 * L + 2;
    extern __shared__ u32 gemm_acc[];                    // (NW, blockDim.x): this thread's accumulator
    u32* accm = gemm_acc + threadIdx.x;
#pragma unroll
    for (int w = 0; w < NW; w++) accm[w * kGemmThreads] = 0;
    if (Ea != EZ && Eb != EZ) {
        for (i64 k = 0; k < K; k++) {
            u32 a[L], bb[L];
            bool na = load_mag<L>(am, aplane, (b * M + i) * K + k, a);
            if (is_zero(a)) continue;
            bool nb = load_mag<L>(bm, bplane, (b * K + k) * N + j, bb);
            if (is_zero(bb)) continue;
            mac_signed_mem<L, NW>(accm, kGemmThreads, a, bb, na != nb);
        }
    }
    u32 acc[NW];
#pragma unroll
    for (int w = 0; w < NW; w++) acc[w] = accm[w * kGemmThreads];
    store_rounded<L, NW>(cm, ce, cplane, t, acc, (Ea == EZ || Eb == EZ) ? EZ : Ea + Eb);
}

// Elementwise C = A * B (exact product, one rounding); A and B indexed through optional gathers.
template <int L>
__global__ void k_mul(const int32_t* __restrict__ am, const i64* __restrict__ ae, i64 aplane, const i64* __restrict__ aidx,
                      const int32_t* __restrict__ bm, const i64* __restrict__ be, i64 bplane, const i64* __restrict__ bidx,
                      i64 n, int32_t* __restrict__ cm, i64* __restrict__ ce, i64 cplane) {
    i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (t >= n) return;
    i64 ia = aidx ? aidx[t] : t, ib = bidx ? bidx[t] : t;
    u32 a[L], b[L];
    bool na = load_mag<L>(am, aplane, ia, a);
    bool nb = load_mag<L>(bm, bplane, ib, b);
    i64 ea = ae[ia], eb = be[ib];
    constexpr int NW = 2 * L + 1;
    u32 acc[NW];
    zero(acc);
    bool z = is_zero(a) || is_zero(b) || ea == EZ || eb == EZ;
    if (!z) mac_signed<L, NW>(acc, a, b, na != nb);
    store_rounded<L, NW>(cm, ce, cplane, t, acc, z ? EZ : ea + eb);
}

// Elementwise C = A + B (one rounding), optional gathers.
template <int L>
__global__ void k_add(const int32_t* __restrict__ am, const i64* __restrict__ ae, i64 aplane, const i64* __restrict__ aidx,
                      const int32_t* __restrict__ bm, const i64* __restrict__ be, i64 bplane, const i64* __restrict__ bidx,
                      i64 n, int32_t* __restrict__ cm, i64* __restrict__ ce, i64 cplane) {
    i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (t >= n) return;
    i64 ia = aidx ? aidx[t] : t, ib = bidx ? bidx[t] : t;
    u32 a[L], b[L], r[L];
    bool na = load_mag<L>(am, aplane, ia, a);
    bool nb = load_mag<L>(bm, bplane, ib, b);
    bool nr;
    i64 er;
    add_norm<L>(a, na, ae[ia], b, nb, be[ib], r, &nr, &er);
    store_signed<L>(cm, cplane, t, r, nr);
    ce[t] = er;
}

// ------------------------------------------------------------------------------------------------
// Cauchy step of recursion level m, fused with the h_inf term:
//   H[g, r, n] = hinf[gsrc[g], m, gj[g], n] + sum_{i < ncol[g]} 2 / (rowd[g, r] - cold[g, i]) res[col[g, i], n]
// (terms with a vanishing difference are skipped; rows r >= nrow[g] are padding and written as zero).
// The residues of a column (g, n) are aligned to their largest exponent, each term 2 x / d is formed
// exactly up to 32 guard bits (one-limb division), the sum is exact, rounded once, then h_inf is added
// with one more rounding.
template <int L>
__global__ void k_cauchy(const int32_t* __restrict__ rm, const i64* __restrict__ re, i64 rplane,
                         const int32_t* __restrict__ hm, const i64* __restrict__ he, i64 hplane,
                         CauchyLevel lv, int32_t* __restrict__ om, i64* __restrict__ oe, i64 oplane) {
    i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    i64 N = lv.N;
    if (t >= lv.nb * lv.Mr * N) return;
    i64 n = t % N, r = (t / N) % lv.Mr, g = t / (N * lv.Mr);
    if (r >= lv.nrow[g]) {
        u32 z[L];
        zero(z);
        store_signed<L>(om, oplane, t, z, false);
        oe[t] = EZ;
        return;
    }
    i64 hidx = ((lv.gsrc[g] * lv.hlevels + lv.m) * lv.Jh + lv.gj[g]) * N + n;
    u32 h[L];
    bool nh = load_mag<L>(hm, hplane, hidx, h);
    i64 eh = he[hidx];
    i64 ncol = lv.ncol[g];
    const i64* col = lv.col + g * lv.Kc;
    const i64* cold = lv.cold + g * lv.Kc;
    i64 D = lv.rowd[g * lv.Mr + r];
    i64 E = EZ;
    for (i64 i = 0; i < ncol; i++) {
        i64 ix = col[i] * N + n;
        i64 ei = re[ix];
        if (ei > E && rm[(L - 1) * rplane + ix] != 0) E = ei;
    }
    u32 s[L];
    bool ns = false;
    i64 es = EZ;
    if (E != EZ) {
        constexpr int NW = L + 3;
        u32 acc[NW];
        zero(acc);
        for (i64 i = 0; i < ncol; i++) {
            i64 d = D - cold[i];
            if (d == 0) continue;
            i64 ix = col[i] * N + n;
            u32 a[L];
            bool na = load_mag<L>(rm, rplane, ix, a);
            i64 ei = re[ix];
            if (is_zero(a) || ei == EZ || E - ei >= 32 * L) continue;
            u32 x[L];
            shr(a, (int)(E - ei), x);
            if (d < 0) { na = !na; d = -d; }
            u32 q[L + 1];
            div_small<L>(x, (u32)d, q);
            add_signed(acc, q, na);
        }
        bool neg = (acc[NW - 1] >> 31) != 0;
        if (neg) negate(acc);
        if (round_mag<L>(acc, E - 31, s, &es)) ns = neg;   // value = acc 2^(E - 32) x 2
    } else {
        zero(s);
    }
    u32 out[L];
    bool no;
    i64 eo;
    add_norm<L>(s, ns, es, h, nh, eh, out, &no, &eo);
    store_signed<L>(om, oplane, t, out, no);
    oe[t] = eo;
}


// ------------------------------------------------------------------------------------------------
// Cauchy step, second form: X already aligned per column (g, n) (k_cauchy_align: (nb, Kc, N) mantissas and the
// column exponents).  Each term floor(|x| 2^32 / |d|) is produced limb by limb from the top and added with its
// sign into per-limb 64-bit accumulators (no carry chain per term: |acc[k]| < Kc 2^32); two terms are divided
// at once (independent chains); the digit corrections are branch free.  One carry pass, one rounding, then the
// h_inf term is added with one more rounding (as k_cauchy).
struct Div16 {
    u32 d, inv;
};

__device__ __forceinline__ u32 div16_step(u32 cur, const Div16& v, u32* rem) {
    u32 q = umulhi32(cur, v.inv);                 // inv = floor((2^32 - 1) / d): q is at most 2 short
    u32 r = cur - q * v.d;
    bool c1 = r >= v.d;
    q += c1; r -= c1 ? v.d : 0u;
    bool c2 = r >= v.d;
    q += c2; r -= c2 ? v.d : 0u;
    *rem = r;
    return q;
}

template <int L>
__global__ void k_cauchy2(const int32_t* __restrict__ xm, const i64* __restrict__ xe, i64 xplane,
                          const int32_t* __restrict__ hm, const i64* __restrict__ he, i64 hplane,
                          CauchyLevel lv, int32_t* __restrict__ om, i64* __restrict__ oe, i64 oplane) {
    i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    const i64 N = lv.N;
    if (t >= lv.nb * lv.Mr * N) return;
    const i64 n = t % N, r = (t / N) % lv.Mr, g = t / (N * lv.Mr);
    if (r >= lv.nrow[g]) {
        u32 z[L];
        zero(z);
        store_signed<L>(om, oplane, t, z, false);
        oe[t] = EZ;
        return;
    }
    const i64 hidx = ((lv.gsrc[g] * lv.hlevels + lv.m) * lv.Jh + lv.gj[g]) * N + n;
    const i64 E = xe[g * N + n];
    const i64 ncol = lv.ncol[g];
    const i64* cold = lv.cold + g * lv.Kc;
    const i64 D = lv.rowd[g * lv.Mr + r];
    long long acc[L + 1];
#pragma unroll
    for (int k = 0; k <= L; k++) acc[k] = 0;
    if (E != EZ) {
        for (i64 i = 0; i < ncol; i += 2) {
            u32 a0[L], a1[L];
            const bool two = i + 1 < ncol;
            i64 d0 = D - cold[i], d1 = two ? D - cold[i + 1] : 0;
            bool n0 = load_mag<L>(xm, xplane, (g * lv.Kc + i) * N + n, a0);
            bool n1 = false;
            if (two) n1 = load_mag<L>(xm, xplane, (g * lv.Kc + i + 1) * N + n, a1);
            else zero(a1);
            if (d0 < 0) { n0 = !n0; d0 = -d0; }
            if (d1 < 0) { n1 = !n1; d1 = -d1; }
            const bool live0 = d0 != 0, live1 = d1 != 0;
            Div16 v0{live0 ? (u32)d0 : 1u, live0 ? 0xFFFFFFFFu / (u32)d0 : 0xFFFFFFFFu};
            Div16 v1{live1 ? (u32)d1 : 1u, live1 ? 0xFFFFFFFFu / (u32)d1 : 0xFFFFFFFFu};
            const long long s0 = !live0 ? 0 : (n0 ? -1 : 1), s1 = !live1 ? 0 : (n1 ? -1 : 1);
            u32 r0 = 0, r1 = 0;
#pragma unroll
            for (int k = L; k >= 0; k--) {               // quotient limb k of floor(|x| 2^32 / d)
                const u32 l0 = k > 0 ? a0[k - 1] : 0u, l1 = k > 0 ? a1[k - 1] : 0u;
                u32 qh0 = div16_step((r0 << 16) | (l0 >> 16), v0, &r0);
                u32 qh1 = div16_step((r1 << 16) | (l1 >> 16), v1, &r1);
                u32 ql0 = div16_step((r0 << 16) | (l0 & 0xFFFFu), v0, &r0);
                u32 ql1 = div16_step((r1 << 16) | (l1 & 0xFFFFu), v1, &r1);
                acc[k] += s0 * (long long)((qh0 << 16) | ql0) + s1 * (long long)((qh1 << 16) | ql1);
            }
        }
    }
    // carry pass into L + 3 two's complement limbs, value acc 2^(E - 31)
    u32 w[L + 3];
    long long c = 0;
#pragma unroll
    for (int k = 0; k <= L; k++) {
        long long v = acc[k] + c;
        w[k] = (u32)v;
        c = v >> 32;
    }
#pragma unroll
    for (int k = L + 1; k < L + 3; k++) {
        w[k] = (u32)c;
        c >>= 32;
    }
    const bool neg = (w[L + 2] >> 31) != 0;
    if (neg) negate(w);
    u32 s[L];
    i64 es;
    bool ns = false;
    if (E != EZ && round_mag<L>(w, E - 31, s, &es)) ns = neg;
    else { zero(s); es = EZ; }
    u32 h[L], out[L];
    const bool nh = load_mag<L>(hm, hplane, hidx, h);
    bool no;
    i64 eo;
    add_norm<L>(s, ns, es, h, nh, he[hidx], out, &no, &eo);
    store_signed<L>(om, oplane, t, out, no);
    oe[t] = eo;
}

// The Cauchy step with wide quotient digits: the same exact quotients floor(|x| 2^32 / d) as k_cauchy2, but
// the dividend (32 (L + 1) bits) is consumed in W-bit digits from the top, W = 24 when every divisor of the
// level is below 2^8 and 22 below 2^10 (16 otherwise): r < d < 2^(32 - W) keeps (r << W) | digit in 32 bits,
// so one multiply-high step per digit covers W bits instead of 16.  Quotient digits are summed per digit
// position in signed 32-bit registers (|sum| <= ncol (2^W - 1) < 2^31: ncol < 128 for W = 24, < 512 for
// W = 22, checked by the launcher), then carried into limbs: the result is bit-identical to k_cauchy2.
template <int L>
__device__ __forceinline__ u32 dividend_bits(const u32 (&a)[L], int lo, int width) {
    const int li = lo >> 5, bo = lo & 31;                   // dividend limb k = (k == 0 ? 0 : a[k - 1])
    const u32 v0 = li == 0 ? 0u : a[li - 1];
    const u32 v1 = (li + 1 <= L) ? a[li] : 0u;
    const u32 v = bo ? ((v0 >> bo) | (v1 << (32 - bo))) : v0;
    return width >= 32 ? v : (v & ((1u << width) - 1u));
}

constexpr int kCauchyThreads = 128;

template <int L, int W>
__global__ void __launch_bounds__(kCauchyThreads, 3) k_cauchy3(const int32_t* __restrict__ xm, const i64* __restrict__ xe, i64 xplane,
                          const int32_t* __restrict__ hm, const i64* __restrict__ he, i64 hplane,
                          CauchyLevel lv, int32_t* __restrict__ om, i64* __restrict__ oe, i64 oplane) {
    constexpr int TB = 32 * (L + 1), ND = (TB + W - 1) / W;
    i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    const i64 N = lv.N;
    if (t >= lv.nb * lv.Mr * N) return;
    const i64 n = t % N, r = (t / N) % lv.Mr, g = t / (N * lv.Mr);
    if (r >= lv.nrow[g]) {
        u32 z[L];
        zero(z);
        store_signed<L>(om, oplane, t, z, false);
        oe[t] = EZ;
        return;
    }
    const i64 hidx = ((lv.gsrc[g] * lv.hlevels + lv.m) * lv.Jh + lv.gj[g]) * N + n;
    const i64 E = xe[g * N + n];
    const i64 ncol = lv.ncol[g];
    const i64* cold = lv.cold + g * lv.Kc;
    const i64 D = lv.rowd[g * lv.Mr + r];
    extern __shared__ int c3_acc[];                      // (ND, blockDim.x): this thread's digit sums
    int* acc = c3_acc + threadIdx.x;
#pragma unroll
    for (int j = 0; j < ND; j++) acc[j * kCauchyThreads] = 0;
    if (E != EZ) {
        for (i64 i = 0; i < ncol; i += 2) {
            u32 a0[L], a1[L];
            const bool two = i + 1 < ncol;
            i64 d0 = D - cold[i], d1 = two ? D - cold[i + 1] : 0;
            bool n0 = load_mag<L>(xm, xplane, (g * lv.Kc + i) * N + n, a0);
            bool n1 = false;
            if (two) n1 = load_mag<L>(xm, xplane, (g * lv.Kc + i + 1) * N + n, a1);
            else zero(a1);
            if (d0 < 0) { n0 = !n0; d0 = -d0; }
            if (d1 < 0) { n1 = !n1; d1 = -d1; }
            const bool live0 = d0 != 0, live1 = d1 != 0;
            const u32 v0 = live0 ? (u32)d0 : 1u, v1 = live1 ? (u32)d1 : 1u;
            // inv = floor(2^32 / d) (2^32 - 1 for d = 1): for c < 2^32 the estimate umulhi(c, inv) is the
            // quotient or one below it (c inv / 2^32 > c / d - 1), so one correction step suffices
            const u32 i0 = v0 == 1u ? 0xFFFFFFFFu : (u32)(0x100000000ull / v0);
            const u32 i1 = v1 == 1u ? 0xFFFFFFFFu : (u32)(0x100000000ull / v1);
            const int s0 = !live0 ? 0 : (n0 ? -1 : 1), s1 = !live1 ? 0 : (n1 ? -1 : 1);
            u32 r0 = 0, r1 = 0;
#pragma unroll
            for (int j = 0; j < ND; j++) {                  // digit j from the top: dividend bits [lo, lo + width)
                const int lo = W * (ND - 1 - j);
                const int width = j == 0 ? TB - W * (ND - 1) : W;
                const u32 c0 = (r0 << width) | dividend_bits(a0, lo, width);
                const u32 c1 = (r1 << width) | dividend_bits(a1, lo, width);
                u32 q0 = umulhi32(c0, i0), q1 = umulhi32(c1, i1);   // at most 1 short
                r0 = c0 - q0 * v0;
                r1 = c1 - q1 * v1;
                const bool x0 = r0 >= v0, x1 = r1 >= v1;
                q0 += x0; r0 -= x0 ? v0 : 0u;
                q1 += x1; r1 -= x1 ? v1 : 0u;
                acc[j * kCauchyThreads] += s0 * (int)q0 + s1 * (int)q1;
            }
        }
    }
    // digit sums -> signed limb sums (value sum_j acc[j] 2^(W (ND - 1 - j))), then the k_cauchy2 carry pass
    long long accl[L + 2];
#pragma unroll
    for (int k = 0; k < L + 2; k++) accl[k] = 0;
    {
        long long carry = 0;
#pragma unroll
        for (int j = ND - 1; j >= 0; j--) {
            const int lo = W * (ND - 1 - j), k0 = lo >> 5, b0 = lo & 31;
            const long long v = (long long)acc[j * kCauchyThreads] + carry;
            long long part;
            if (j > 0) {                                    // keep W bits here, carry the rest up
                part = v & ((1ll << W) - 1);
                carry = v >> W;
            } else {
                part = v;                                   // top digit: signed, small
            }
            // part 2^b0 = (part mod 2^(32 - b0)) 2^b0 + floor(part / 2^(32 - b0)) 2^32, exact for any part
            const long long lo32 = b0 ? ((part & ((1ll << (32 - b0)) - 1)) << b0) : (part & 0xFFFFFFFFll);
            const long long hi = b0 ? (part >> (32 - b0)) : (part >> 32);
            accl[k0] += lo32;                               // k0 <= L: the dividend has L + 1 limbs
            accl[k0 + 1] += hi;
        }
    }
    u32 w[L + 3];
    long long c = 0;
#pragma unroll
    for (int k = 0; k < L + 2; k++) {
        long long v = accl[k] + c;
        w[k] = (u32)v;
        c = v >> 32;
    }
    w[L + 2] = (u32)c;
    const bool neg = (w[L + 2] >> 31) != 0;
    if (neg) negate(w);
    u32 s[L];
    i64 es;
    bool ns = false;
    if (E != EZ && round_mag<L>(w, E - 31, s, &es)) ns = neg;
    else { zero(s); es = EZ; }
    u32 h[L], out[L];
    const bool nh = load_mag<L>(hm, hplane, hidx, h);
    bool no;
    i64 eo;
    add_norm<L>(s, ns, es, h, nh, he[hidx], out, &no, &eo);
    store_signed<L>(om, oplane, t, out, no);
    oe[t] = eo;
}

// The Cauchy step of k_cauchy3 on sign-magnitude columns (k_cauchy_align_sm: |x| with the sign in the top bit
// of limb L - 1), read limb by limb from memory as the division reaches them instead of held in registers: the
// same quotient digits from the top of the same dividend |x| 2^32, so the results are bit-identical to
// k_cauchy3, with a third of its registers per thread (more resident warps to hide the multiply-high chains).
template <int L>
__device__ __forceinline__ u32 sm_dividend_limb(const int32_t* __restrict__ xm, i64 plane, i64 idx, int k) {
    if (k <= 0 || k > L) return 0u;                          // dividend limb k = |x| limb k - 1; limb 0 is zero
    const u32 v = (u32)__ldg(xm + (i64)(k - 1) * plane + idx);
    return k == L ? (v & 0x7FFFFFFFu) : v;
}

template <int L>
__device__ __forceinline__ u32 sm_dividend_bits(const int32_t* __restrict__ xm, i64 plane, i64 idx, int lo, int width) {
    const int li = lo >> 5, bo = lo & 31;
    const u32 v0 = sm_dividend_limb<L>(xm, plane, idx, li);
    const u32 v = bo ? ((v0 >> bo) | (sm_dividend_limb<L>(xm, plane, idx, li + 1) << (32 - bo))) : v0;
    return width >= 32 ? v : (v & ((1u << width) - 1u));
}

template <int L, int W>
__global__ void __launch_bounds__(kCauchyThreads, 4) k_cauchy4(const int32_t* __restrict__ xm, const i64* __restrict__ xe, i64 xplane,
                          const int32_t* __restrict__ hm, const i64* __restrict__ he, i64 hplane,
                          CauchyLevel lv, int32_t* __restrict__ om, i64* __restrict__ oe, i64 oplane) {
    constexpr int TB = 32 * (L + 1), ND = (TB + W - 1) / W;
    // reciprocals floor(2^32 / v) of the divisors, built once per block: the W = 24 and W = 22 forms are only
    // launched for plans whose divisors are below 2^8 and 2^10 (the W = 16 form divides per term)
    constexpr int NT = W >= 24 ? 256 : (W >= 22 ? 1024 : 1);
    __shared__ u32 inv_tab[NT];
    if (NT > 1) {
        for (int v = threadIdx.x; v < NT; v += blockDim.x) inv_tab[v] = v <= 1 ? 0xFFFFFFFFu : (u32)(0x100000000ull / v);
        __syncthreads();
    }
    i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    const i64 N = lv.N, total = lv.nb * lv.Mr * N;
    if (t >= total) return;
    i64 n, r, g;
    split3(t, N, lv.Mr, total, n, r, g);
    if (r >= lv.nrow[g]) {
        u32 z[L];
        zero(z);
        store_signed<L>(om, oplane, t, z, false);
        oe[t] = EZ;
        return;
    }
    const i64 hidx = ((lv.gsrc[g] * lv.hlevels + lv.m) * lv.Jh + lv.gj[g]) * N + n;
    const i64 E = xe[g * N + n];
    const i64 ncol = lv.ncol[g];
    const i64* cold = lv.cold + g * lv.Kc;
    const i64 D = lv.rowd[g * lv.Mr + r];
    extern __shared__ int c4_acc[];                      // (ND, blockDim.x): this thread's digit sums
    int* acc = c4_acc + threadIdx.x;
#pragma unroll
    for (int j = 0; j < ND; j++) acc[j * kCauchyThreads] = 0;
    if (E != EZ) {
        for (i64 i = 0; i < ncol; i += 2) {
            const bool two = i + 1 < ncol;
            const i64 ix0 = (g * lv.Kc + i) * N + n, ix1 = two ? ix0 + N : ix0;
            const bool n0 = ((u32)__ldg(xm + (i64)(L - 1) * xplane + ix0) >> 31) != 0;
            const bool n1 = ((u32)__ldg(xm + (i64)(L - 1) * xplane + ix1) >> 31) != 0;
            i64 d0 = D - cold[i], d1 = two ? D - cold[i + 1] : 0;
            const int s0 = d0 == 0 ? 0 : ((n0 != (d0 < 0)) ? -1 : 1);
            const int s1 = d1 == 0 ? 0 : ((n1 != (d1 < 0)) ? -1 : 1);
            const u32 v0 = d0 == 0 ? 1u : (u32)(d0 < 0 ? -d0 : d0), v1 = d1 == 0 ? 1u : (u32)(d1 < 0 ? -d1 : d1);
            // inv = floor(2^32 / d) (2^32 - 1 for d = 1): the estimate umulhi(c, inv) is the quotient or one below it
            const u32 i0 = v0 < (u32)NT ? inv_tab[v0] : (v0 == 1u ? 0xFFFFFFFFu : (u32)(0x100000000ull / v0));
            const u32 i1 = v1 < (u32)NT ? inv_tab[v1] : (v1 == 1u ? 0xFFFFFFFFu : (u32)(0x100000000ull / v1));
            u32 r0 = 0, r1 = 0;
#pragma unroll
            for (int j = 0; j < ND; j++) {                  // digit j from the top: dividend bits [lo, lo + width)
                const int lo = W * (ND - 1 - j);
                const int width = j == 0 ? TB - W * (ND - 1) : W;
                const u32 c0 = (r0 << width) | sm_dividend_bits<L>(xm, xplane, ix0, lo, width);
                const u32 c1 = (r1 << width) | sm_dividend_bits<L>(xm, xplane, ix1, lo, width);
                u32 q0 = umulhi32(c0, i0), q1 = umulhi32(c1, i1);
                r0 = c0 - q0 * v0;
                r1 = c1 - q1 * v1;
                const bool x0 = r0 >= v0, x1 = r1 >= v1;
                q0 += x0; r0 -= x0 ? v0 : 0u;
                q1 += x1; r1 -= x1 ? v1 : 0u;
                acc[j * kCauchyThreads] += s0 * (int)q0 + s1 * (int)q1;
            }
        }
    }
    // digit sums -> signed limb sums (value sum_j acc[j] 2^(W (ND - 1 - j))), carried into limbs
    long long accl[L + 2];
#pragma unroll
    for (int k = 0; k < L + 2; k++) accl[k] = 0;
    {
        long long carry = 0;
#pragma unroll
        for (int j = ND - 1; j >= 0; j--) {
            const int lo = W * (ND - 1 - j), k0 = lo >> 5, b0 = lo & 31;
            const long long v = (long long)acc[j * kCauchyThreads] + carry;
            long long part;
            if (j > 0) {
                part = v & ((1ll << W) - 1);
                carry = v >> W;
            } else {
                part = v;
            }
            const long long lo32 = b0 ? ((part & ((1ll << (32 - b0)) - 1)) << b0) : (part & 0xFFFFFFFFll);
            const long long hi = b0 ? (part >> (32 - b0)) : (part >> 32);
            accl[k0] += lo32;
            accl[k0 + 1] += hi;
        }
    }
    u32 w[L + 3];
    long long c = 0;
#pragma unroll
    for (int k = 0; k < L + 2; k++) {
        long long v = accl[k] + c;
        w[k] = (u32)v;
        c = v >> 32;
    }
    w[L + 2] = (u32)c;
    const bool neg = (w[L + 2] >> 31) != 0;
    if (neg) negate(w);
    u32 sres[L];
    i64 es;
    bool ns = false;
    if (E != EZ && round_mag<L>(w, E - 31, sres, &es)) ns = neg;
    else { zero(sres); es = EZ; }
    u32 h[L], out[L];
    const bool nh = load_mag<L>(hm, hplane, hidx, h);
    bool no;
    i64 eo;
    add_norm<L>(sres, ns, es, h, nh, he[hidx], out, &no, &eo);
    store_signed<L>(om, oplane, t, out, no);
    oe[t] = eo;
}

// ------------------------------------------------------------------------------------------------
// The pole kernels keep their 2 L + 2 accumulator limbs in shared memory (one column per thread), so that only
// the operands live in registers: more resident warps to hide the latency of the multiply-add chains.
constexpr int kPoleThreads = 128;

// Pole step, stage 1: Y[t, a, b0, k] = sum_b R[b0, b] H[t_hrow[t], a, b, k]  (R = Rtab[t_R[t]] aligned
// per row; H aligned per column (a, k) over b here).  Y: (T, S, S, B) contiguous.
template <int L>
__global__ void __launch_bounds__(kPoleThreads, 3) k_pole1(const int32_t* __restrict__ hm, const i64* __restrict__ he, i64 hplane,
                        const int32_t* __restrict__ Rm, const i64* __restrict__ Re, i64 Rplane,
                        const i64* __restrict__ t_hrow, const i64* __restrict__ t_R, i64 T, i64 B, int S,
                        int32_t* __restrict__ ym, i64* __restrict__ ye, i64 yplane) {
    i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (idx >= T * S * S * B) return;
    i64 k = idx % B, b0 = (idx / B) % S, a = (idx / (B * S)) % S, t = idx / (B * S * S);
    i64 hrow = t_hrow[t], rk = t_R[t];
    i64 hb = hrow * S * S * B + a * S * B + k;          // H[hrow, a, b, k] at hb + b * B
    i64 E = EZ;
    for (int b = 0; b < S; b++) {
        i64 ix = hb + b * B;
        i64 eb = he[ix];
        if (eb > E && hm[(L - 1) * hplane + ix] != 0) E = eb;
    }
    i64 Er = Re[rk * S + b0];
    constexpr int NW = 2 * L + 2;
    extern __shared__ u32 pole_acc[];                    // (NW, blockDim.x): this thread's column
    u32* acc = pole_acc + threadIdx.x;
    auto sum = [&](auto cols) {                          // acc = the sum from product column cols up
#pragma unroll
        for (int w = 0; w < NW; w++) acc[w * kPoleThreads] = 0;
        bool any = false;
        if (E != EZ && Er != EZ) {
#pragma unroll 1
            for (int b = 0; b < S; b++) {
                u32 x[L], y[L], r[L];
                bool nr = load_mag<L>(Rm, Rplane, (rk * S + b0) * S + b, r);
                if (is_zero(r)) continue;
                i64 ix = hb + b * B;
                bool nx = load_mag<L>(hm, hplane, ix, x);
                i64 ex = he[ix];
                if (is_zero(x) || ex == EZ || E - ex >= 32 * L) continue;
                shr(x, (int)(E - ex), y);
                mac_signed_mem<L, NW, decltype(cols)::value>(acc, kPoleThreads, r, y, nr != nx);
                any = true;
            }
        }
        return any;
    };
    u32 mag[NW];
    const bool neg = exact_sum<L, NW>(sum, acc, kPoleThreads, mag);
    store_rounded_mag<L, NW>(ym, ye, yplane, idx, mag, neg, (E == EZ || Er == EZ) ? EZ : E + Er);
}

// Pole step, stage 2: res[t_slot[t], a0, b0, k] = sum_a QL[a0, a] Y[t, a, b0, k]  (QL = QLtab[t_qL[t]]
// aligned per row; Y aligned per column (b0, k) over a here).
template <int L>
__global__ void __launch_bounds__(kPoleThreads, 3) k_pole2(const int32_t* __restrict__ ym, const i64* __restrict__ ye, i64 yplane,
                        const int32_t* __restrict__ Qm, const i64* __restrict__ Qe, i64 Qplane,
                        const i64* __restrict__ t_qL, const i64* __restrict__ t_slot, i64 T, i64 B, int S,
                        int32_t* __restrict__ rm, i64* __restrict__ re, i64 rplane) {
    i64 idx = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (idx >= T * S * S * B) return;
    i64 k = idx % B, b0 = (idx / B) % S, a0 = (idx / (B * S)) % S, t = idx / (B * S * S);
    i64 qk = t_qL[t];
    i64 yb = t * S * S * B + b0 * B + k;                // Y[t, a, b0, k] at yb + a * S * B
    i64 E = EZ;
    for (int a = 0; a < S; a++) {
        i64 ix = yb + a * S * B;
        i64 ea = ye[ix];
        if (ea > E && ym[(L - 1) * yplane + ix] != 0) E = ea;
    }
    i64 Eq = Qe[qk * S + a0];
    constexpr int NW = 2 * L + 2;
    extern __shared__ u32 pole_acc[];                    // (NW, blockDim.x): this thread's column
    u32* acc = pole_acc + threadIdx.x;
    auto sum = [&](auto cols) {                          // acc = the sum from product column cols up
#pragma unroll
        for (int w = 0; w < NW; w++) acc[w * kPoleThreads] = 0;
        bool any = false;
        if (E != EZ && Eq != EZ) {
#pragma unroll 1
            for (int a = 0; a < S; a++) {
                u32 x[L], y[L], q[L];
                bool nq = load_mag<L>(Qm, Qplane, (qk * S + a0) * S + a, q);
                if (is_zero(q)) continue;
                i64 ix = yb + a * S * B;
                bool nx = load_mag<L>(ym, yplane, ix, x);
                i64 ex = ye[ix];
                if (is_zero(x) || ex == EZ || E - ex >= 32 * L) continue;
                shr(x, (int)(E - ex), y);
                mac_signed_mem<L, NW, decltype(cols)::value>(acc, kPoleThreads, q, y, nq != nx);
                any = true;
            }
        }
        return any;
    };
    u32 mag[NW];
    const bool neg = exact_sum<L, NW>(sum, acc, kPoleThreads, mag);
    i64 out = t_slot[t] * S * S * B + (a0 * S + b0) * B + k;
    store_rounded_mag<L, NW>(rm, re, rplane, out, mag, neg, (E == EZ || Eq == EZ) ? EZ : E + Eq);
}

// ------------------------------------------------------------------------------------------------
// Derivative moments of one recursion level: for each moment entry q (slot, row, n) and column c,
//   y = res[slot, c] * rc^n,   mom[row, kk, c] += n^kk y   (kk <= R)
// mom layout (rows, R + 1, N).  n^kk y is formed exactly from the previous power (one-limb product)
// and rounded before each addition.
constexpr int kMomThreads = 128;

template <int L>
__global__ void __launch_bounds__(kMomThreads, 3) k_moments(const int32_t* __restrict__ rm, const i64* __restrict__ re, i64 rplane,
                          const int32_t* __restrict__ pm, const i64* __restrict__ pe, i64 pplane,
                          const i64* __restrict__ q_slot, const i64* __restrict__ q_row, const i64* __restrict__ q_n,
                          i64 Q, i64 N, int R1, int32_t* __restrict__ mm, i64* __restrict__ me, i64 mplane) {
    i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (t >= Q * N) return;
    i64 c = t % N, q = t / N;
    i64 ix = q_slot[q] * N + c, nn = q_n[q];
    u32 x[L], p[L];
    bool nx = load_mag<L>(rm, rplane, ix, x);
    bool np = load_mag<L>(pm, pplane, nn, p);
    i64 ex = re[ix], ep = pe[nn];
    if (is_zero(x) || is_zero(p) || ex == EZ || ep == EZ) return;
    constexpr int NW = 2 * L + 1;
    extern __shared__ u32 mom_acc[];                     // (NW, blockDim.x): this thread's product
    u32* accm = mom_acc + threadIdx.x;
#pragma unroll
    for (int w = 0; w < NW; w++) accm[w * kMomThreads] = 0;
    mac_signed_mem<L, NW>(accm, kMomThreads, x, p, false);
    u32 acc[NW];
#pragma unroll
    for (int w = 0; w < NW; w++) acc[w] = accm[w * kMomThreads];
    // y = n^kk x p between iterations lives in this thread's shared-memory column (free after the product,
    // words [0, L)); add_norm_col reads it there and uses words [L, 2 L) as its scratch column
    u32* ys = accm;
    i64 ey;
    {
        u32 y[L];
        round_mag<L>(acc, ex + ep, y, &ey);
#pragma unroll
        for (int k = 0; k < L; k++) ys[k * kMomThreads] = y[k];
    }
    const bool ny = nx != np;
    const i64 row = q_row[q];
    for (int kk = 0; kk < R1; kk++) {
        const i64 o = (row * R1 + kk) * N + c;
        {
            u32 v[L], s[L];
            const bool nv = load_mag<L>(mm, mplane, o, v);
            bool ns;
            i64 es;
            add_norm_col<L>(v, nv, me[o], ys, ny, ey, ys + L * kMomThreads, kMomThreads, s, &ns, &es);
            store_signed<L>(mm, mplane, o, s, ns);
            me[o] = es;
        }
        if (kk + 1 < R1) {                             // y *= n (exact, then rounded)
            u32 w[L + 1], y[L];
            u64 carry = 0;
#pragma unroll
            for (int k = 0; k < L; k++) {
                u64 v2 = (u64)ys[k * kMomThreads] * (u64)nn + carry;
                w[k] = (u32)v2;
                carry = v2 >> 32;
            }
            w[L] = (u32)carry;
            if (nn == 0) {                             // 0^kk = 0 for kk >= 1
                ey = EZ;
                zero(y);
            } else {
                round_mag<L>(w, ey, y, &ey);
            }
#pragma unroll
            for (int k = 0; k < L; k++) ys[k * kMomThreads] = y[k];
        }
    }
}

// ------------------------------------------------------------------------------------------------
// Staged derivative moments.  Instead of a read-modify-write of all R + 1 moments of a row at every level,
// each level only stages its terms, and the moments are formed once per window of levels:
//   stage (per level m):  Y[m - m0, row, c] = round(res[slot, c] * rc^n)     (n = m + shift of the row's pole)
//   flush (per window):   mom[row, kk, c] (+)= round( sum_{w < W} n_w^kk Y[w, row, c] ),  n_w = m0 + w + shift
// The window sum is exact for every term above 2^-(32 L + 64) of the largest one (aligned to the largest
// n^kk |Y| of the window, truncated below): one rounding per window and moment order, plus one for the
// addition into the moments of earlier windows.  Staged entries that a level does not write stay zero.
template <int L>
__global__ void __launch_bounds__(kMomThreads, 3) k_moments_stage(const int32_t* __restrict__ rm, const i64* __restrict__ re,
                          i64 rplane, const int32_t* __restrict__ pm, const i64* __restrict__ pe, i64 pplane,
                          const i64* __restrict__ q_slot, const i64* __restrict__ q_row, const i64* __restrict__ q_n,
                          i64 Q, i64 N, i64 w, i64 rows, int32_t* __restrict__ ym, i64* __restrict__ ye, i64 yplane) {
    i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (t >= Q * N) return;
    i64 c, q;
    split2(t, N, Q * N, c, q);
    i64 ix = q_slot[q] * N + c, nn = q_n[q];
    i64 out = (w * rows + q_row[q]) * N + c;
    u32 x[L], p[L];
    bool nx = load_mag<L>(rm, rplane, ix, x);
    bool np = load_mag<L>(pm, pplane, nn, p);
    i64 ex = re[ix], ep = pe[nn];
    if (is_zero(x) || is_zero(p) || ex == EZ || ep == EZ) {
        ye[out] = EZ;
        return;
    }
    constexpr int NW = 2 * L + 1;
    extern __shared__ u32 stage_acc[];                   // (NW, blockDim.x): this thread's product
    u32* accm = stage_acc + threadIdx.x;
#pragma unroll
    for (int k = 0; k < NW; k++) accm[k * kMomThreads] = 0;
    mac_signed_mem<L, NW>(accm, kMomThreads, x, p, false);
    u32 acc[NW];
#pragma unroll
    for (int k = 0; k < NW; k++) acc[k] = accm[k * kMomThreads];
    u32 y[L];
    i64 ey;
    round_mag<L>(acc, ex + ep, y, &ey);
    store_signed<L>(ym, yplane, out, y, nx != np);
    ye[out] = ey;
}

// One thread per (row, column) item, the moment orders in chunks of kFlushKC: for each staged term, the exact
// product |Y| n^k0 (n^k0 from the table nk: nk[(k * NN + n) * KW + j], 32-bit limbs; nkb[k * NN + n] its bit
// length), then times n for each further order of the chunk, each added into that order's accumulator (a
// shared-memory column of L + 3 words, two's complement) at the word and bit offset of its exponent: no barrel
// shifter, one funnel shift per word.  The accumulator of order k keeps the bits from 32 (L + 2) below the bound
// E_k = max_w (e_w + NB + bits(n_w^k)) of its terms (truncated below), then rounds once.
constexpr int kFlushThreads = 64;
constexpr int kFlushKC = 4;

template <int ACC, int NP>
__device__ __forceinline__ void add_at_offset(u32* acc, int stride, const u32 (&P)[NP], i64 off, bool neg) {
    const i64 qq = off >= 0 ? off / 32 : -((-off + 31) / 32);      // floor(off / 32)
    const int f = (int)(off - 32 * qq);
    const int q = (int)qq;
    u32 carry = 0;                                                  // carry (add) or borrow (subtract)
#pragma unroll
    for (int j = 0; j <= NP; j++) {
        const int a = j + q;
        const u32 lo = j > 0 ? P[j - 1] : 0u, hi = j < NP ? P[j] : 0u;
        const u32 v = fsl(lo, hi, f);                               // word j of P 2^f
        if (a < 0 || a >= ACC) continue;                            // below the accumulator: truncated
        const u32 w = acc[a * stride];
        if (!neg) {
            const u32 s1 = w + v, s2 = s1 + carry;
            carry = (s1 < w) | (s2 < s1);
            acc[a * stride] = s2;
        } else {
            const u32 d1 = w - v, d2 = d1 - carry;
            carry = (w < v) | (d1 < carry);
            acc[a * stride] = d2;
        }
    }
    for (int a = NP + 1 + q; carry && a < ACC; a++) {              // propagate to the top
        if (a < 0) continue;
        const u32 w = acc[a * stride];
        if (!neg) { acc[a * stride] = w + 1; carry = w == 0xFFFFFFFFu; }
        else { acc[a * stride] = w - 1; carry = w == 0u; }
    }
}

template <int L, int LO, int KW, bool ACCUMULATE>
__global__ void __launch_bounds__(kFlushThreads) k_moments_flush(const int32_t* __restrict__ ym, const i64* __restrict__ ye,
                          i64 yplane, const i64* __restrict__ row_shift, i64 m0, int W, i64 rows, i64 N, int R1,
                          const u32* __restrict__ nk, const int32_t* __restrict__ nkb, int NN,
                          int32_t* __restrict__ mm, i64* __restrict__ me, i64 mplane) {
    constexpr int NB = nb_bits(L);                       // staged terms: L limbs; moments: LO limbs
    constexpr int ACC = LO + 3;
    constexpr int NP = L + KW + 1;                       // |Y| n^k, k within a chunk: n^k0 < 2^(32 KW), n^3 < 2^32
    extern __shared__ u32 flush_acc[];                   // (kFlushKC * ACC, blockDim.x)
    const i64 item = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (item >= rows * N) return;
    const i64 row = item / N, c = item - row * N;
    const i64 sh = row_shift[row];
    u32* acc = flush_acc + threadIdx.x;
    for (int k0 = 0; k0 < R1; k0 += kFlushKC) {
        const int kc = R1 - k0 < kFlushKC ? R1 - k0 : kFlushKC;
        i64 E[kFlushKC];
#pragma unroll
        for (int kk = 0; kk < kFlushKC; kk++) E[kk] = EZ;
        for (int w = 0; w < W; w++) {
            const i64 ey = ye[(w * rows + row) * N + c];
            const i64 n = m0 + w + sh;
            if (ey == EZ || n >= NN) continue;
#pragma unroll
            for (int kk = 0; kk < kFlushKC; kk++) {
                if (kk >= kc) break;
                const int kb = nkb[(k0 + kk) * NN + n];
                if (kb && ey + NB + kb > E[kk]) E[kk] = ey + NB + kb;
            }
        }
        for (int k = 0; k < kFlushKC * ACC; k++) acc[k * kFlushThreads] = 0;
        for (int w = 0; w < W; w++) {
            const i64 ix = (w * rows + row) * N + c;
            const i64 ey = ye[ix];
            const i64 n = m0 + w + sh;
            if (ey == EZ || n >= NN) continue;
            u32 y[L];
            const bool neg = load_mag<L>(ym, yplane, ix, y);
            u32 P[NP];
            zero(P);
#pragma unroll
            for (int j = 0; j < KW; j++) {               // P = |Y| n^k0
                const u32 b = nk[((i64)k0 * NN + n) * KW + j];
                u32 carry = 0;
#pragma unroll
                for (int i = 0; i < L; i++) {
                    const u64 v = (u64)y[i] * b + P[i + j] + carry;
                    P[i + j] = (u32)v;
                    carry = (u32)(v >> 32);
                }
                P[L + j] += carry;
            }
#pragma unroll 1
            for (int kk = 0; kk < kc; kk++) {
                if (kk > 0) {                            // P *= n (exact)
                    u32 carry = 0;
#pragma unroll
                    for (int i = 0; i < NP; i++) {
                        const u64 v = (u64)P[i] * (u64)n + carry;
                        P[i] = (u32)v;
                        carry = (u32)(v >> 32);
                    }
                }
                if (E[kk] == EZ || nkb[(k0 + kk) * NN + n] == 0) continue;
                add_at_offset<ACC, NP>(acc + kk * ACC * kFlushThreads, kFlushThreads, P, ey - (E[kk] - 32 * (LO + 2)), neg);
            }
        }
        for (int kk = 0; kk < kc; kk++) {
            const i64 o = (row * R1 + k0 + kk) * N + c;
            if (E[kk] == EZ) {
                if (!ACCUMULATE) {
#pragma unroll
                    for (int k = 0; k < LO; k++) mm[k * mplane + o] = 0;
                    me[o] = EZ;
                }
                continue;
            }
            u32 mag[ACC];
#pragma unroll
            for (int k = 0; k < ACC; k++) mag[k] = acc[(kk * ACC + k) * kFlushThreads];
            const bool negs = (mag[ACC - 1] >> 31) != 0;
            if (negs) negate(mag);
            u32 r[LO];
            i64 er;
            bool nr = negs;
            if (!round_mag<LO>(mag, E[kk] - 32 * (LO + 2), r, &er)) nr = false;
            if (ACCUMULATE) {
                u32 v[LO], sum[LO];
                const bool nv = load_mag<LO>(mm, mplane, o, v);
                bool ns;
                i64 es;
                add_norm<LO>(v, nv, me[o], r, nr, er, sum, &ns, &es);
                store_signed<LO>(mm, mplane, o, sum, ns);
                me[o] = es;
            } else {
                store_signed<LO>(mm, mplane, o, r, nr);
                me[o] = er;
            }
        }
    }
}

// ------------------------------------------------------------------------------------------------
// Change of limb count: widening is exact (the mantissa moves up by 32 (LO - LI) bits), narrowing rounds once
// (half away from zero) to 32 LO - 2 bits.
template <int LI, int LO>
__global__ void k_resize(const int32_t* __restrict__ m, const i64* __restrict__ e, i64 plane, i64 n,
                         int32_t* __restrict__ om, i64* __restrict__ oe, i64 oplane) {
    const i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    if (i >= n) return;
    u32 a[LI];
    const bool neg = load_mag<LI>(m, plane, i, a);
    const i64 ea = e[i];
    u32 r[LO];
    i64 er = EZ;
    bool nr = neg;
    if (is_zero(a) || ea == EZ) {
        zero(r);
        nr = false;
    } else if (LO >= LI) {
#pragma unroll
        for (int k = 0; k < LO; k++) r[k] = k >= LO - LI ? a[k - (LO - LI)] : 0u;
        er = ea - 32 * (LO - LI);
    } else if (!round_mag<LO>(a, ea, r, &er)) {
        nr = false;
    }
    store_signed<LO>(om, oplane, i, r, nr);
    oe[i] = er;
}

// ------------------------------------------------------------------------------------------------
// Host-side launchers, one instantiation per limb count (inst.cu).  Each returns a cudaError_t code.
inline unsigned grid_for(i64 n, int th) { return (unsigned)((n + th - 1) / th); }

template <int L>
struct Launch {
    static int align(const int32_t* m, const i64* e, i64 plane, i64 nbatch, i64 R, i64 K, i64 sb, i64 sr, i64 sk,
                     const i64* bidx, int32_t* om, i64* oe, i64 oplane, int kmajor, cudaStream_t st);
    static int gemm_aligned(const int32_t* am, const i64* ae, i64 aplane, const int32_t* bm, const i64* be, i64 bplane,
                            i64 nbatch, i64 M, i64 N, i64 K, int32_t* cm, i64* ce, i64 cplane, cudaStream_t st);
    static int mul(const int32_t* am, const i64* ae, i64 aplane, const i64* aidx, const int32_t* bm, const i64* be,
                   i64 bplane, const i64* bidx, i64 n, int32_t* cm, i64* ce, i64 cplane, cudaStream_t st);
    static int add(const int32_t* am, const i64* ae, i64 aplane, const i64* aidx, const int32_t* bm, const i64* be,
                   i64 bplane, const i64* bidx, i64 n, int32_t* cm, i64* ce, i64 cplane, cudaStream_t st);
    static int cauchy(const int32_t* rm, const i64* re, i64 rplane, const int32_t* hm, const i64* he, i64 hplane,
                      const CauchyLevel& lv, int32_t* om, i64* oe, i64 oplane, cudaStream_t st);
    static int cauchy2(const int32_t* xm, const i64* xe, i64 xplane, const int32_t* hm, const i64* he, i64 hplane,
                       const CauchyLevel& lv, int32_t* om, i64* oe, i64 oplane, cudaStream_t st);
    static int cauchy3(const int32_t* xm, const i64* xe, i64 xplane, const int32_t* hm, const i64* he, i64 hplane,
                       const CauchyLevel& lv, i64 dmax, int32_t* om, i64* oe, i64 oplane, cudaStream_t st);
    static int cauchy4(const int32_t* xm, const i64* xe, i64 xplane, const int32_t* hm, const i64* he, i64 hplane,
                       const CauchyLevel& lv, i64 dmax, int32_t* om, i64* oe, i64 oplane, cudaStream_t st);
    static int pole(const int32_t* hm, const i64* he, i64 hplane, const int32_t* Rm, const i64* Re, i64 Rplane,
                    const int32_t* Qm, const i64* Qe, i64 Qplane, const i64* t_hrow, const i64* t_R, const i64* t_qL,
                    const i64* t_slot, i64 T, i64 B, int S, int32_t* ym, i64* ye, i64 yplane,
                    int32_t* rm, i64* re, i64 rplane, cudaStream_t st);
    // the same pole step on the tensor cores (pole_mma.cuh); err: device flag of bounded-wait expiries
    static int pole_mma(const int32_t* hm, const i64* he, i64 hplane, const int32_t* Rm, const i64* Re, i64 Rplane,
                        const int32_t* Qm, const i64* Qe, i64 Qplane, const i64* t_hrow, const i64* t_R, const i64* t_qL,
                        const i64* t_slot, i64 T, i64 B, int S, int32_t* ym, i64* ye, i64 yplane,
                        int32_t* rm, i64* re, i64 rplane, int* err, cudaStream_t st);
    static int moments(const int32_t* rm, const i64* re, i64 rplane, const int32_t* pm, const i64* pe, i64 pplane,
                       const i64* q_slot, const i64* q_row, const i64* q_n, i64 Q, i64 N, int R1,
                       int32_t* mm, i64* me, i64 mplane, cudaStream_t st);
    static int moments_stage(const int32_t* rm, const i64* re, i64 rplane, const int32_t* pm, const i64* pe, i64 pplane,
                             const i64* q_slot, const i64* q_row, const i64* q_n, i64 Q, i64 N, i64 w, i64 rows,
                             int32_t* ym, i64* ye, i64 yplane, cudaStream_t st);
    static int moments_flush(const int32_t* ym, const i64* ye, i64 yplane, const i64* row_shift, i64 m0, int W, i64 rows,
                             i64 N, int R1, const u32* nk, const int32_t* nkb, int NN, int KW, int accumulate, int LO,
                             int32_t* mm, i64* me, i64 mplane, cudaStream_t st);
    static int resize(const int32_t* m, const i64* e, i64 plane, i64 n, int LO, int32_t* om, i64* oe, i64 oplane,
                      cudaStream_t st);
};

#ifdef B3D_DEFINE_LAUNCH
constexpr int kThreads = 128;

template <int L>
int Launch<L>::align(const int32_t* m, const i64* e, i64 plane, i64 nbatch, i64 R, i64 K, i64 sb, i64 sr, i64 sk,
                     const i64* bidx, int32_t* om, i64* oe, i64 oplane, int kmajor, cudaStream_t st) {
    i64 n = nbatch * R;
    if (n == 0) return 0;
    k_align<L><<<grid_for(n, kThreads), kThreads, 0, st>>>(m, e, plane, nbatch, R, K, sb, sr, sk, bidx, om, oe, oplane, kmajor);
    return (int)cudaGetLastError();
}

template <int L>
int Launch<L>::gemm_aligned(const int32_t* am, const i64* ae, i64 aplane, const int32_t* bm, const i64* be, i64 bplane,
                            i64 nbatch, i64 M, i64 N, i64 K, int32_t* cm, i64* ce, i64 cplane, cudaStream_t st) {
    i64 n = nbatch * M * N;
    if (n == 0) return 0;
    k_gemm_aligned<L><<<grid_for(n, kGemmThreads), kGemmThreads, (2 * L + 2) * kGemmThreads * 4, st>>>(
        am, ae, aplane, bm, be, bplane, nbatch, M, N, K, cm, ce, cplane);
    return (int)cudaGetLastError();
}

template <int L>
int Launch<L>::mul(const int32_t* am, const i64* ae, i64 aplane, const i64* aidx, const int32_t* bm, const i64* be,
                   i64 bplane, const i64* bidx, i64 n, int32_t* cm, i64* ce, i64 cplane, cudaStream_t st) {
    if (n == 0) return 0;
    k_mul<L><<<grid_for(n, kThreads), kThreads, 0, st>>>(am, ae, aplane, aidx, bm, be, bplane, bidx, n, cm, ce, cplane);
    return (int)cudaGetLastError();
}

template <int L>
int Launch<L>::add(const int32_t* am, const i64* ae, i64 aplane, const i64* aidx, const int32_t* bm, const i64* be,
                   i64 bplane, const i64* bidx, i64 n, int32_t* cm, i64* ce, i64 cplane, cudaStream_t st) {
    if (n == 0) return 0;
    k_add<L><<<grid_for(n, kThreads), kThreads, 0, st>>>(am, ae, aplane, aidx, bm, be, bplane, bidx, n, cm, ce, cplane);
    return (int)cudaGetLastError();
}

template <int L>
int Launch<L>::cauchy(const int32_t* rm, const i64* re, i64 rplane, const int32_t* hm, const i64* he, i64 hplane,
                      const CauchyLevel& lv, int32_t* om, i64* oe, i64 oplane, cudaStream_t st) {
    i64 n = lv.nb * lv.Mr * lv.N;
    if (n == 0) return 0;
    k_cauchy<L><<<grid_for(n, kThreads), kThreads, 0, st>>>(rm, re, rplane, hm, he, hplane, lv, om, oe, oplane);
    return (int)cudaGetLastError();
}

template <int L>
int Launch<L>::cauchy2(const int32_t* xm, const i64* xe, i64 xplane, const int32_t* hm, const i64* he, i64 hplane,
                       const CauchyLevel& lv, int32_t* om, i64* oe, i64 oplane, cudaStream_t st) {
    i64 n = lv.nb * lv.Mr * lv.N;
    if (n == 0) return 0;
    k_cauchy2<L><<<grid_for(n, kThreads), kThreads, 0, st>>>(xm, xe, xplane, hm, he, hplane, lv, om, oe, oplane);
    return (int)cudaGetLastError();
}

template <int L>
int Launch<L>::cauchy3(const int32_t* xm, const i64* xe, i64 xplane, const int32_t* hm, const i64* he, i64 hplane,
                       const CauchyLevel& lv, i64 dmax, int32_t* om, i64* oe, i64 oplane, cudaStream_t st) {
    i64 n = lv.nb * lv.Mr * lv.N;
    if (n == 0) return 0;
    constexpr int TB = 32 * (L + 1);
    if (dmax < (1 << 8) && lv.Kc < 128)
        k_cauchy3<L, 24><<<grid_for(n, kCauchyThreads), kCauchyThreads, ((TB + 23) / 24) * kCauchyThreads * 4, st>>>(
            xm, xe, xplane, hm, he, hplane, lv, om, oe, oplane);
    else if (dmax < (1 << 10) && lv.Kc < 512)
        k_cauchy3<L, 22><<<grid_for(n, kCauchyThreads), kCauchyThreads, ((TB + 21) / 22) * kCauchyThreads * 4, st>>>(
            xm, xe, xplane, hm, he, hplane, lv, om, oe, oplane);
    else
        k_cauchy2<L><<<grid_for(n, kThreads), kThreads, 0, st>>>(xm, xe, xplane, hm, he, hplane, lv, om, oe, oplane);
    return (int)cudaGetLastError();
}

template <int L>
int Launch<L>::cauchy4(const int32_t* xm, const i64* xe, i64 xplane, const int32_t* hm, const i64* he, i64 hplane,
                       const CauchyLevel& lv, i64 dmax, int32_t* om, i64* oe, i64 oplane, cudaStream_t st) {
    i64 n = lv.nb * lv.Mr * lv.N;
    if (n == 0) return 0;
    constexpr int TB = 32 * (L + 1);
    if (dmax < (1 << 8) && lv.Kc < 128)
        k_cauchy4<L, 24><<<grid_for(n, kCauchyThreads), kCauchyThreads, ((TB + 23) / 24) * kCauchyThreads * 4, st>>>(
            xm, xe, xplane, hm, he, hplane, lv, om, oe, oplane);
    else if (dmax < (1 << 10) && lv.Kc < 512)
        k_cauchy4<L, 22><<<grid_for(n, kCauchyThreads), kCauchyThreads, ((TB + 21) / 22) * kCauchyThreads * 4, st>>>(
            xm, xe, xplane, hm, he, hplane, lv, om, oe, oplane);
    else
        k_cauchy4<L, 16><<<grid_for(n, kCauchyThreads), kCauchyThreads, ((TB + 15) / 16) * kCauchyThreads * 4, st>>>(
            xm, xe, xplane, hm, he, hplane, lv, om, oe, oplane);
    return (int)cudaGetLastError();
}

template <int L>
int Launch<L>::pole(const int32_t* hm, const i64* he, i64 hplane, const int32_t* Rm, const i64* Re, i64 Rplane,
                    const int32_t* Qm, const i64* Qe, i64 Qplane, const i64* t_hrow, const i64* t_R, const i64* t_qL,
                    const i64* t_slot, i64 T, i64 B, int S, int32_t* ym, i64* ye, i64 yplane,
                    int32_t* rm, i64* re, i64 rplane, cudaStream_t st) {
    i64 n = T * S * S * B;
    if (n == 0) return 0;
    const int smem = (2 * L + 2) * kPoleThreads * 4;   // <= 44 KB (L = 42): no opt-in
    k_pole1<L><<<grid_for(n, kPoleThreads), kPoleThreads, smem, st>>>(hm, he, hplane, Rm, Re, Rplane, t_hrow, t_R, T, B, S,
                                                                       ym, ye, yplane);
    k_pole2<L><<<grid_for(n, kPoleThreads), kPoleThreads, smem, st>>>(ym, ye, yplane, Qm, Qe, Qplane, t_qL, t_slot, T, B,
                                                                       S, rm, re, rplane);
    return (int)cudaGetLastError();
}

template <int L>
int Launch<L>::moments(const int32_t* rm, const i64* re, i64 rplane, const int32_t* pm, const i64* pe, i64 pplane,
                       const i64* q_slot, const i64* q_row, const i64* q_n, i64 Q, i64 N, int R1,
                       int32_t* mm, i64* me, i64 mplane, cudaStream_t st) {
    i64 n = Q * N;
    if (n == 0) return 0;
    k_moments<L><<<grid_for(n, kMomThreads), kMomThreads, (2 * L + 1) * kMomThreads * 4, st>>>(
        rm, re, rplane, pm, pe, pplane, q_slot, q_row, q_n, Q, N, R1, mm, me, mplane);
    return (int)cudaGetLastError();
}

template <int L>
int Launch<L>::moments_stage(const int32_t* rm, const i64* re, i64 rplane, const int32_t* pm, const i64* pe, i64 pplane,
                             const i64* q_slot, const i64* q_row, const i64* q_n, i64 Q, i64 N, i64 w, i64 rows,
                             int32_t* ym, i64* ye, i64 yplane, cudaStream_t st) {
    i64 n = Q * N;
    if (n == 0) return 0;
    k_moments_stage<L><<<grid_for(n, kMomThreads), kMomThreads, (2 * L + 1) * kMomThreads * 4, st>>>(
        rm, re, rplane, pm, pe, pplane, q_slot, q_row, q_n, Q, N, w, rows, ym, ye, yplane);
    return (int)cudaGetLastError();
}

template <int L>
int Launch<L>::moments_flush(const int32_t* ym, const i64* ye, i64 yplane, const i64* row_shift, i64 m0, int W, i64 rows,
                             i64 N, int R1, const u32* nk, const int32_t* nkb, int NN, int KW, int accumulate, int LO,
                             int32_t* mm, i64* me, i64 mplane, cudaStream_t st) {
    const i64 items = rows * N;
    if (items == 0 || W == 0) return 0;
    const unsigned grid = (unsigned)((items + kFlushThreads - 1) / kFlushThreads);
#define B3D_FLUSH(LOC, KWC, AC) do {                                                                       \
        const int smem = kFlushThreads * kFlushKC * ((LOC) + 3) * 4;     /* above 48 KB from 46 limbs: opt in */ \
        static unsigned long long opted = 0;                /* devices whose limit is raised */                  \
        const unsigned long long dbit = device_bit();                                                            \
        if (!(opted & dbit) || !dbit) {                                                                          \
            const int rc = (int)cudaFuncSetAttribute(k_moments_flush<L, LOC, KWC, AC>,                           \
                                                     cudaFuncAttributeMaxDynamicSharedMemorySize, smem);         \
            if (rc) return rc;                                                                                   \
            opted |= dbit;                                                                                       \
        }                                                                                                    \
        k_moments_flush<L, LOC, KWC, AC><<<grid, kFlushThreads, smem, st>>>(ym, ye, yplane, row_shift, m0, W, rows, N, R1, \
                                                                            nk, nkb, NN, mm, me, mplane);    \
    } while (0)
#define B3D_FLUSH_KW(LOC) \
    if (KW <= 2) { if (accumulate) B3D_FLUSH(LOC, 2, true); else B3D_FLUSH(LOC, 2, false); } \
    else if (KW <= 6) { if (accumulate) B3D_FLUSH(LOC, 6, true); else B3D_FLUSH(LOC, 6, false); } \
    else { if (accumulate) B3D_FLUSH(LOC, 12, true); else B3D_FLUSH(LOC, 12, false); }
    if (LO == L) { B3D_FLUSH_KW(L) }
    else if (LO == L + 4) { B3D_FLUSH_KW(L + 4) }
    else return (int)cudaErrorInvalidValue;
#undef B3D_FLUSH_KW
#undef B3D_FLUSH
    return (int)cudaGetLastError();
}

template <int L>
int Launch<L>::resize(const int32_t* m, const i64* e, i64 plane, i64 n, int LO, int32_t* om, i64* oe, i64 oplane,
                      cudaStream_t st) {
    if (n == 0) return 0;
    const unsigned grid = grid_for(n, kThreads);
    if (LO == L) k_resize<L, L><<<grid, kThreads, 0, st>>>(m, e, plane, n, om, oe, oplane);
    else if (LO == L + 4) k_resize<L, L + 4><<<grid, kThreads, 0, st>>>(m, e, plane, n, om, oe, oplane);
    else if (LO == L - 4 && L > 4) k_resize<L, (L > 4 ? L - 4 : L)><<<grid, kThreads, 0, st>>>(m, e, plane, n, om, oe, oplane);
    else return (int)cudaErrorInvalidValue;
    return (int)cudaGetLastError();
}
#endif

// limb counts with compiled kernels: 2 ceil(prec / 64) + 2 for precisions 128 ... 1280 bits, plus 6
#define B3D_FOR_EACH_L(X) X(6) X(10) X(14) X(18) X(22) X(26) X(30) X(34) X(38) X(42) X(46)

}  // namespace b3d
