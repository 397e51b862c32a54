// Multiprecision primitives on register arrays (sm_100a CUDA cores).
//
// Number format ("MPF", the layout of the reference's sdpvibe.mpf as used by blocksvibe): a value is
// m * 2^e with m a signed integer of L 32-bit limbs (two's complement, limb 0 least significant) and e an
// int64 exponent.  Normalised numbers have |m| of exactly NB = 32 L - 2 bits; zero is m = 0, e = EZ.
// Arrays store limb planes: limb k of element i at m[k * plane + i].
//
// Everything here works on fixed-size register arrays (sizes are template parameters, all indexing is
// static), so the compiler keeps the limbs in registers: variable shifts use a log-depth barrel shifter
// instead of a runtime word index.
#pragma once
#include <cstdint>
#ifdef __CUDACC__
#include <cuda_runtime.h>
#endif

namespace b3d {

typedef uint32_t u32;
typedef uint64_t u64;
typedef int64_t i64;

#ifdef __CUDACC__
#define B3D_HD __host__ __device__ __forceinline__
#define B3D_CX __host__ __device__ constexpr
#else
#define B3D_HD inline
#define B3D_CX constexpr
#endif

constexpr i64 EZ = -(i64(1) << 60);       // exponent of zero
B3D_CX int nb_bits(int L) { return 32 * L - 2; }

B3D_HD int clz32(u32 x) {
#ifdef __CUDA_ARCH__
    return __clz(x);
#else
    return x ? __builtin_clz(x) : 32;
#endif
}

B3D_HD u32 umulhi32(u32 a, u32 b) {
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return (u32)(((u64)a * b) >> 32);
#endif
}

// (c2:c1:c0) += a * b  (96-bit column accumulator of product scanning)
B3D_HD void mac96(u32& c0, u32& c1, u32& c2, u32 a, u32 b) {
#ifdef __CUDA_ARCH__
    asm("mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
        "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
        "addc.u32 %2, %2, 0;"
        : "+r"(c0), "+r"(c1), "+r"(c2) : "r"(a), "r"(b));
#else
    u64 p = (u64)a * b;
    u64 lo = (u64)c0 + (u32)p;
    u64 hi = (u64)c1 + (p >> 32) + (lo >> 32);
    c0 = (u32)lo; c1 = (u32)hi; c2 += (u32)(hi >> 32);
#endif
}

template <int N> B3D_HD void zero(u32 (&a)[N]) {
#pragma unroll
    for (int k = 0; k < N; k++) a[k] = 0;
}

// two's complement negation in place
template <int N> B3D_HD void negate(u32 (&a)[N]) {
    u32 c = 1;
#pragma unroll
    for (int k = 0; k < N; k++) {
        u32 v = ~a[k] + c;
        c = (c && v == 0) ? 1u : 0u;
        a[k] = v;
    }
}

template <int N> B3D_HD bool is_zero(const u32 (&a)[N]) {
    u32 o = 0;
#pragma unroll
    for (int k = 0; k < N; k++) o |= a[k];
    return o == 0;
}

// bit length of an unsigned array (0 for zero)
template <int N> B3D_HD int bitlen(const u32 (&a)[N]) {
    int bl = 0;
#pragma unroll
    for (int k = 0; k < N; k++)
        if (a[k]) bl = 32 * k + 32 - clz32(a[k]);
    return bl;
}

// funnel shifts: low 32 bits of (hi:lo) >> b and high 32 bits of (hi:lo) << b, for 0 <= b < 32
B3D_HD u32 fsr(u32 lo, u32 hi, int b) {
#ifdef __CUDA_ARCH__
    return __funnelshift_r(lo, hi, b);
#else
    return b ? ((lo >> b) | (hi << (32 - b))) : lo;
#endif
}

B3D_HD u32 fsl(u32 lo, u32 hi, int b) {
#ifdef __CUDA_ARCH__
    return __funnelshift_l(lo, hi, b);
#else
    return b ? ((hi << b) | (lo >> (32 - b))) : hi;
#endif
}

// out = floor(in / 2^sh), low NO limbs (sh >= 0; any size).  Shifts below one word skip the word stages.
template <int NI, int NO> B3D_HD void shr(const u32 (&in)[NI], int sh, u32 (&out)[NO]) {
    constexpr int NT = (NI > NO + 1 ? NI : NO + 1);
    u32 t[NT];
#pragma unroll
    for (int k = 0; k < NT; k++) t[k] = k < NI ? in[k] : 0u;
    int w = sh >> 5, b = sh & 31;
    if (w >= NI) { zero(out); return; }
    if (w) {
#pragma unroll
        for (int s = 1; s < NT; s <<= 1) {
            if (w & s) {
#pragma unroll
                for (int k = 0; k < NT; k++) t[k] = (k + s < NT) ? t[k + s] : 0u;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < NO; k++) out[k] = fsr(t[k], (k + 1 < NT) ? t[k + 1] : 0u, b);
}

// out = (in * 2^sh) mod 2^(32 NO)  (sh >= 0).  Shifts below one word skip the word stages.
template <int NI, int NO> B3D_HD void shl(const u32 (&in)[NI], int sh, u32 (&out)[NO]) {
    u32 t[NO];
#pragma unroll
    for (int k = 0; k < NO; k++) t[k] = k < NI ? in[k] : 0u;
    int w = sh >> 5, b = sh & 31;
    if (w >= NO) { zero(out); return; }
    if (w) {
#pragma unroll
        for (int s = 1; s < NO; s <<= 1) {
            if (w & s) {
#pragma unroll
                for (int k = NO - 1; k >= 0; k--) t[k] = (k - s >= 0) ? t[k - s] : 0u;
            }
        }
    }
#pragma unroll
    for (int k = NO - 1; k >= 0; k--) out[k] = fsl((k > 0) ? t[k - 1] : 0u, t[k], b);
}

// load one element of a limb-plane array as sign + magnitude
template <int L> B3D_HD bool load_mag(const int32_t* m, i64 plane, i64 i, u32 (&a)[L]) {
#pragma unroll
    for (int k = 0; k < L; k++) a[k] = (u32)m[k * plane + i];
    bool neg = (a[L - 1] >> 31) != 0;
    if (neg) negate(a);
    return neg;
}

template <int L> B3D_HD void store_signed(int32_t* m, i64 plane, i64 i, const u32 (&a)[L], bool neg) {
    u32 t[L];
#pragma unroll
    for (int k = 0; k < L; k++) t[k] = a[k];
    if (neg) negate(t);
#pragma unroll
    for (int k = 0; k < L; k++) m[k * plane + i] = (int32_t)t[k];
}

// Round an unsigned magnitude w (NW limbs, value w * 2^ein) to NB = 32 L - 2 bits, half away from zero.
// Returns false for zero.  r: L-limb magnitude, *eout: exponent.
template <int L, int NW> B3D_HD bool round_mag(const u32 (&w)[NW], i64 ein, u32 (&r)[L], i64* eout) {
    constexpr int NB = nb_bits(L);
    int bl = bitlen(w);
    if (bl == 0) { zero(r); *eout = EZ; return false; }
    int s = bl - NB;
    if (s <= 0) {
        shl(w, -s, r);
        *eout = ein + s;
        return true;
    }
    u32 t[L + 1];
    shr(w, s - 1, t);                      // keeps the rounding bit in bit 0
    u32 c = t[0] & 1u;
#pragma unroll
    for (int k = 0; k < L; k++) {
        u32 v = (t[k] >> 1) | (t[k + 1] << 31);
        u32 sum = v + c;
        c = (c && sum == 0) ? 1u : 0u;
        r[k] = sum;
    }
    // a carry out of bit NB - 1 makes the magnitude 2^NB: renormalise
    if ((r[L - 1] >> (NB - 32 * (L - 1))) != 0) {
        u32 q[L];
        shr(r, 1, q);
#pragma unroll
        for (int k = 0; k < L; k++) r[k] = q[k];
        s += 1;
    }
    *eout = ein + s;
    return true;
}

// Round a two's complement accumulator (NW limbs, value acc * 2^ein) and store it normalised.
template <int L, int NW> B3D_HD void store_rounded(int32_t* m, i64* e, i64 plane, i64 i, const u32 (&acc)[NW], i64 ein) {
    u32 w[NW];
#pragma unroll
    for (int k = 0; k < NW; k++) w[k] = acc[k];
    bool neg = (w[NW - 1] >> 31) != 0;
    if (neg) negate(w);
    u32 r[L];
    i64 er;
    if (!round_mag<L>(w, ein, r, &er)) neg = false;
    store_signed<L>(m, plane, i, r, neg);
    e[i] = er;
}

// acc (two's complement, NW >= 2 L + 1 limbs) += sgn * a * b, a and b magnitudes of L limbs
// (product scanning: one 96-bit column at a time, merged into acc with a signed running carry)
template <int L, int NW> B3D_HD void mac_signed(u32 (&acc)[NW], const u32 (&a)[L], const u32 (&b)[L], bool negative) {
    u32 c0 = 0, c1 = 0, c2 = 0;
    i64 rc = 0;
#pragma unroll
    for (int col = 0; col < 2 * L; col++) {
#pragma unroll
        for (int x = 0; x < L; x++) {
            int y = col - x;
            if (y >= 0 && y < L) mac96(c0, c1, c2, a[x], b[y]);
        }
        i64 r = (i64)acc[col] + (negative ? -(i64)c0 : (i64)c0) + rc;
        acc[col] = (u32)r;
        rc = r >> 32;
        c0 = c1; c1 = c2; c2 = 0;
    }
#pragma unroll
    for (int k = 2 * L; k < NW; k++) {
        i64 r = (i64)acc[k] + rc;
        acc[k] = (u32)r;
        rc = r >> 32;
    }
}

// mac_signed with the accumulator in memory (limb k at acc[k * stride]; shared memory in the pole kernels, so
// that the operands, not the 2 L + 2 accumulator limbs, occupy the registers): same result bit for bit.
// C0 > 0 scans only the columns from C0 up and leaves acc[0 .. C0) alone: the part of a * b it drops,
// sum over x + y < C0 of a[x] b[y] 2^(32 (x + y)), lies in [0, C0 2^(32 (C0 + 1)) (1 + 2^-31)), so n such
// products leave acc within n C0 2^(32 (C0 + 1)) (1 + 2^-31) < 2^(32 (C0 + 2)) of the exact sum (n C0 < 2^31).
template <int L, int NW, int C0 = 0> B3D_HD void mac_signed_mem(u32* acc, int stride, const u32 (&a)[L],
                                                                const u32 (&b)[L], bool negative) {
    u32 c0 = 0, c1 = 0, c2 = 0;
    i64 rc = 0;
#pragma unroll
    for (int col = C0; col < 2 * L; col++) {
#pragma unroll
        for (int x = 0; x < L; x++) {
            int y = col - x;
            if (y >= 0 && y < L) mac96(c0, c1, c2, a[x], b[y]);
        }
        i64 r = (i64)acc[col * stride] + (negative ? -(i64)c0 : (i64)c0) + rc;
        acc[col * stride] = (u32)r;
        rc = r >> 32;
        c0 = c1; c1 = c2; c2 = 0;
    }
#pragma unroll
    for (int k = 2 * L; k < NW; k++) {
        i64 r = (i64)acc[k * stride] + rc;
        acc[k * stride] = (u32)r;
        rc = r >> 32;
    }
}

// Whether round_mag gives the same result for w (an unsigned magnitude) and for every value within 2^(32 EW) of
// it.  Rounding to NB bits, half away from zero, is constant between midpoints of the NB-bit grid, so it is
// enough that no midpoint lies within the error: with hb the half bit of w (bit 0 of round_mag's shifted t),
// the error must lie at least two bits below hb, and the bits of w in [32 EW, hb) must not be all zero when the
// half bit is set (w just above a midpoint) nor all one when it is clear (w just below one).  The nearest
// midpoint of the finer grid below 2^(bitlen - 1) is half a half-unit away, also out of reach.
template <int L, int NW, int EW> B3D_HD bool round_safe(const u32 (&w)[NW]) {
    constexpr int NB = nb_bits(L);
    const int hb = bitlen(w) - NB - 1;
    if (hb < 32 * EW + 2) return false;
    u32 h = 0;
#pragma unroll
    for (int k = EW; k < NW; k++)
        if (k == (hb >> 5)) h = (w[k] >> (hb & 31)) & 1u;
    const u32 flip = h ? 0u : ~0u;
    u32 any = 0;
#pragma unroll
    for (int k = EW; k < NW; k++) {
        const int lo = 32 * k;
        const u32 mask = hb >= lo + 32 ? ~0u : (hb > lo ? (1u << (hb - lo)) - 1u : 0u);
        any |= (w[k] ^ flip) & mask;
    }
    return any != 0;
}

// round_safe for a two's complement accumulator (the rounding acts on its magnitude)
template <int L, int NW, int EW> B3D_HD bool round_safe_signed(const u32 (&acc)[NW]) {
    u32 w[NW];
#pragma unroll
    for (int k = 0; k < NW; k++) w[k] = acc[k];
    if (w[NW - 1] >> 31) negate(w);
    return round_safe<L, NW, EW>(w);
}

// acc (two's complement) += sgn * q, q an unsigned magnitude of NQ limbs (NQ <= NW)
template <int NQ, int NW> B3D_HD void add_signed(u32 (&acc)[NW], const u32 (&q)[NQ], bool negative) {
    i64 rc = 0;
#pragma unroll
    for (int k = 0; k < NW; k++) {
        i64 v = k < NQ ? (i64)q[k] : 0;
        i64 r = (i64)acc[k] + (negative ? -v : v) + rc;
        acc[k] = (u32)r;
        rc = r >> 32;
    }
}

// floor(a * 2^32 / d) for an L-limb magnitude a and 0 < d < 2^16; L + 1 limbs
template <int L> B3D_HD void div_small(const u32 (&a)[L], u32 d, u32 (&q)[L + 1]) {
    u32 inv = 0xFFFFFFFFu / d;
    u32 rem = 0;
#pragma unroll
    for (int k = L; k >= 0; k--) {
        u32 limb = k > 0 ? a[k - 1] : 0u;
        u32 out = 0;
#pragma unroll
        for (int h = 1; h >= 0; h--) {           // two 16-bit digits per limb: cur < d 2^16 <= 2^32
            u32 cur = (rem << 16) | ((limb >> (16 * h)) & 0xFFFFu);
            u32 qq = umulhi32(cur, inv);
            u32 rr = cur - qq * d;
            while (rr >= d) { qq++; rr -= d; }
            out = (out << 16) | qq;
            rem = rr;
        }
        q[k] = out;
    }
}

// r = a + b for normalised operands (one rounding); returns the sign of r through *neg
template <int L> B3D_HD void add_norm(const u32 (&a)[L], bool na, i64 ea, const u32 (&b)[L], bool nb, i64 eb,
                                      u32 (&r)[L], bool* nr, i64* er) {
    bool za = is_zero(a) || ea == EZ, zb = is_zero(b) || eb == EZ;
    if (za && zb) { zero(r); *nr = false; *er = EZ; return; }
    if (za) {
#pragma unroll
        for (int k = 0; k < L; k++) r[k] = b[k];
        *nr = nb; *er = eb; return;
    }
    if (zb) {
#pragma unroll
        for (int k = 0; k < L; k++) r[k] = a[k];
        *nr = na; *er = ea; return;
    }
    i64 top = ea > eb ? ea : eb;
    i64 T = top - 32;                        // common grid: 32 guard bits below the larger operand's ulp
    u32 acc[L + 2];
    zero(acc);
    u32 t[L + 2];
    // the operand with the larger exponent moves up by exactly one word (no barrel shift); the other by
    // 32 - (difference) bits
    const bool abig = ea >= eb;
    const bool sbig = abig ? na : nb, ssmall = abig ? nb : na;
    const i64 ds = (abig ? eb : ea) - T;     // <= 32
    const u32(&sm)[L] = abig ? b : a;
    if (ds >= 0) shl(sm, (int)ds, t); else shr(sm, (int)(-ds > 64 * L ? 64 * L : -ds), t);
    // magnitudes: |big| 2^32 +- |small|, one carry (or borrow) chain; a borrow out means |small| was larger
    bool neg = sbig;
    if (sbig == ssmall) {
        u32 c = 0;
#pragma unroll
        for (int k = 0; k < L + 2; k++) {
            const u64 v = (u64)(k >= 1 && k <= L ? (abig ? a[k - 1] : b[k - 1]) : 0u) + t[k] + c;
            acc[k] = (u32)v;
            c = (u32)(v >> 32);
        }
    } else {
        u32 br = 0;
#pragma unroll
        for (int k = 0; k < L + 2; k++) {
            const u64 v = (u64)(k >= 1 && k <= L ? (abig ? a[k - 1] : b[k - 1]) : 0u) - t[k] - br;
            acc[k] = (u32)v;
            br = (u32)(v >> 63);
        }
        if (br) {
            negate(acc);
            neg = !neg;
        }
    }
    if (!round_mag<L>(acc, T, r, er)) { *nr = false; return; }
    *nr = neg;
}

// add_norm with the second operand in memory (limb k at b[k * stride]; a shared-memory column in the moments
// kernel) and a scratch column of L limbs (same stride): the same result bit for bit.  The smaller operand
// is read from memory at a run-time word offset instead of going through the register barrel shifter: with
// ds = 32 q + f (0 <= f < 32), word k of floor(|small| 2^ds) is fsl(S[k - q - 1], S[k - q], f), S[i] = 0
// outside [0, L).  Fewer live registers, no shifter stages.
template <int L> B3D_HD void add_norm_col(const u32 (&a)[L], bool na, i64 ea, const u32* b, bool nb, i64 eb,
                                          u32* scratch, int stride, u32 (&r)[L], bool* nr, i64* er) {
    u32 bor = 0;
#pragma unroll
    for (int k = 0; k < L; k++) bor |= b[k * stride];
    const bool za = is_zero(a) || ea == EZ, zb = bor == 0 || eb == EZ;
    if (za && zb) { zero(r); *nr = false; *er = EZ; return; }
    if (za) {
#pragma unroll
        for (int k = 0; k < L; k++) r[k] = b[k * stride];
        *nr = nb; *er = eb; return;
    }
    if (zb) {
#pragma unroll
        for (int k = 0; k < L; k++) r[k] = a[k];
        *nr = na; *er = ea; return;
    }
    const i64 top = ea > eb ? ea : eb;
    const i64 T = top - 32;
    const bool abig = ea >= eb;
    const bool sbig = abig ? na : nb, ssmall = abig ? nb : na;
    const i64 ds = (abig ? eb : ea) - T;         // <= 32
    const u32* S = b;
    if (!abig) {                                 // the smaller operand is a: through the scratch column
#pragma unroll
        for (int k = 0; k < L; k++) scratch[k * stride] = a[k];
        S = scratch;
    }
    const i64 dsc = ds < -64 * L ? -64 * L : ds;
    const int q = (int)(dsc >= 0 ? dsc / 32 : -((-dsc + 31) / 32));     // floor(dsc / 32)
    const int f = (int)(dsc - 32 * (i64)q);
    u32 t[L + 2];
    u32 lo = 0;
    {
        const int i = -q - 1;
        lo = (i >= 0 && i < L) ? S[i * stride] : 0u;
    }
#pragma unroll
    for (int k = 0; k < L + 2; k++) {
        const int i = k - q;
        const u32 hi = (i >= 0 && i < L) ? S[i * stride] : 0u;
        t[k] = fsl(lo, hi, f);
        lo = hi;
    }
    u32 acc[L + 2];
    bool neg = sbig;
    if (sbig == ssmall) {
        u32 c = 0;
#pragma unroll
        for (int k = 0; k < L + 2; k++) {
            const u32 big = (k >= 1 && k <= L) ? (abig ? a[k - 1] : b[(k - 1) * stride]) : 0u;
            const u64 v = (u64)big + t[k] + c;
            acc[k] = (u32)v;
            c = (u32)(v >> 32);
        }
    } else {
        u32 br = 0;
#pragma unroll
        for (int k = 0; k < L + 2; k++) {
            const u32 big = (k >= 1 && k <= L) ? (abig ? a[k - 1] : b[(k - 1) * stride]) : 0u;
            const u64 v = (u64)big - t[k] - br;
            acc[k] = (u32)v;
            br = (u32)(v >> 63);
        }
        if (br) {
            negate(acc);
            neg = !neg;
        }
    }
    if (!round_mag<L>(acc, T, r, er)) { *nr = false; return; }
    *nr = neg;
}

#ifdef __CUDACC__
// The current device as a bit of a per-process mask (0 when the device is unknown or beyond 63).  Kernel
// attributes such as a raised shared-memory limit belong to one device's context: launchers keep a mask of
// the devices they have configured, so that a process driving several GPUs sets them on each.
inline unsigned long long device_bit() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    return 1ull << dev;
}
#endif

}  // namespace b3d
