// Decimal output of MPF numbers and blocks_3d's JSON text, on the GPU.
//
// Each number m 2^e (exact) is printed the way blocks_3d's JSON writer prints it (the reference's
// production writer, blocksvibe/b3djson.py:56-80: an MPFR number at the MPF's precision, printed with
// "%.{p}g"): p significant digits rounded to nearest with ties to even, trailing zeros removed, fixed
// notation for decimal exponents -4 <= E < p, otherwise d.ddd e+XX with at least two exponent digits.
//
// Method (exact integer arithmetic, one thread per number):
//   E      = floor(log10 |v|), estimated from the top 64 bits in double and corrected below;
//   D      = floor(|v| 10^k), k = p - 1 - E, computed exactly: |m| 5^k 2^(e+k) for k >= 0 (5^k from a
//            table), |m| 2^(e+k) / 5^-k by exact one-limb divisions for k < 0; the round bit and the sticky
//            bit come from the bits shifted out and the division remainders;
//   check  10^(p-1) <= D < 10^p, else E -= 1 or E += 1 and again (the estimate is off by at most one);
//   round  D += 1 when round && (sticky || D odd); D = 10^p becomes 10^(p-1) with E + 1;
//   digits repeated division of D by 10^9, each digit written straight to its place in the string.
// Strings are built in shared memory and leave the block as 16-byte stores into fixed-stride slots.
//
// Polynomials (blocks_3d's truncation of negligible top coefficients, b3djson.py:160-166) and the text
// assembly (b3djson.py:150-198) are two more kernels: kept sizes plus text lengths per polynomial here, and
// a warp-per-polynomial copy of "skeleton" bytes (brackets, header) and quoted numbers to their offsets
// (k_emit_text, json.cu).
#pragma once
#include <cmath>

#include "mp.cuh"

namespace b3d {

struct DecimalTables {
    const u32* pow5;            // (kmax + 1) rows of fw limbs: 5^k, k = 0 .. kmax
    const int32_t* pow5_limbs;  // limbs in use of 5^k
    const u32* bounds;          // two rows of L - 1 limbs: 10^(p-1), 10^p
    int kmax, fw, p, stride;    // stride: bytes per output slot (multiple of 16, >= p + 12)
};

B3D_CX int dec_digits_max(int L) { return 32 * (L - 2) * 301 / 1000; }     // p of the precision L encodes
B3D_CX int dec_fw_max(int L) { return 3 * dec_digits_max(L) * 2322 / 32000 + 2; }  // limbs of 5^(3 p)
B3D_CX int dec_work(int L) { return L + dec_fw_max(L) + 2; }

// compare a and b of N limbs: -1, 0, 1
template <int N> B3D_HD int cmp_limbs(const u32 (&a)[N], const u32* b) {
#pragma unroll
    for (int k = N - 1; k >= 0; k--)
        if (a[k] != b[k]) return a[k] < b[k] ? -1 : 1;
    return 0;
}

// bit `i` of the W-limb array P (0 outside)
template <int W> B3D_HD u32 bit_of(const u32* P, i64 i) {
    if (i < 0 || i >= 32 * (i64)W) return 0;
    return (P[i >> 5] >> (i & 31)) & 1u;
}

// any bit below position i of P
template <int W> B3D_HD bool any_below(const u32* P, i64 i) {
    if (i <= 0) return false;
    if (i >= 32 * (i64)W) i = 32 * (i64)W;
    const i64 w = i >> 5;
    u32 o = 0;
    for (i64 k = 0; k < w; k++) o |= P[k];
    const int b = (int)(i & 31);
    if (b && w < W) o |= P[w] & ((1u << b) - 1u);
    return o != 0;
}

// D = floor(P / 2^t) (t may be <= 0: a left shift), round = bit t-1, sticky = bits below t-1.
// Returns 1 when D does not fit DW limbs (the decimal exponent estimate was too small), else 0.
template <int W, int DW> B3D_HD int extract_scaled(const u32* P, i64 t, u32 (&D)[DW], bool* rnd, bool* sticky) {
    int bl = 0;
    for (int k = W - 1; k >= 0; k--)
        if (P[k]) { bl = 32 * k + 32 - clz32(P[k]); break; }
    if ((i64)bl - t > 32 * (i64)DW) return 1;
    if (t <= 0) {
        const int s = (int)(-t), w = s >> 5, b = s & 31;
#pragma unroll
        for (int j = 0; j < DW; j++) {
            const int i = j - w;
            const u32 hi = (i >= 0 && i < W) ? P[i] : 0u, lo = (i - 1 >= 0 && i - 1 < W) ? P[i - 1] : 0u;
            D[j] = b ? ((hi << b) | (lo >> (32 - b))) : hi;
        }
        *rnd = false;
        *sticky = false;
        return 0;
    }
    const i64 w = t >> 5;
    const int b = (int)(t & 31);
#pragma unroll
    for (int j = 0; j < DW; j++) {
        const i64 i = w + j;
        const u32 lo = (i < W) ? P[i] : 0u, hi = (i + 1 < W) ? P[i + 1] : 0u;
        D[j] = b ? ((lo >> b) | (hi << (32 - b))) : lo;
    }
    *rnd = bit_of<W>(P, t - 1) != 0;
    *sticky = any_below<W>(P, t - 1);
    return 0;
}

// D = floor(|v| 10^k) for |v| = mag 2^e, with the round and sticky bits of the dropped fraction.
// Returns 0, 1 (D >= 2^(32 DW): exponent estimate too small) or -1 (k outside the tables' range).
template <int L> B3D_HD int scaled_floor(const u32 (&mag)[L], i64 e, i64 k, const DecimalTables& tb,
                                         u32 (&D)[L - 1], bool* rnd, bool* sticky) {
    constexpr int W = dec_work(L);
    u32 P[W];
    for (int j = 0; j < W; j++) P[j] = 0;
    if (k >= 0) {                                           // |m| 5^k, then a shift by e + k
        if (k > tb.kmax) return -1;
        const int nf = tb.pow5_limbs[k];
        if (L + nf > W) return -1;
        const u32* f = tb.pow5 + k * (i64)tb.fw;
        for (int j = 0; j < nf; j++) {
            const u32 fj = f[j];
            u32 c = 0;
#pragma unroll
            for (int i = 0; i < L; i++) {
                const u64 t = (u64)mag[i] * fj + P[i + j] + c;
                P[i + j] = (u32)t;
                c = (u32)(t >> 32);
            }
            P[L + j] = c;
        }
        return extract_scaled<W, L - 1>(P, -(e + k), D, rnd, sticky);
    }
    // k < 0: |m| 2^(e+k+G) / 5^-k, exact floor divisions, then a right shift by G >= 1
    const i64 sft = e + k, G = sft < 0 ? -sft : 1, lsh = sft + G;
    if (lsh > 32 * (i64)(W - L - 1)) return -1;
    {
        const int w = (int)(lsh >> 5), b = (int)(lsh & 31);
        for (int i = 0; i <= L; i++) {
            const u32 lo = i < L ? mag[i] : 0u, lo1 = (i > 0 && i - 1 < L) ? mag[i - 1] : 0u;
            P[i + w] = b ? ((lo << b) | (lo1 >> (32 - b))) : lo;
        }
    }
    bool st = false;
    for (i64 j5 = -k; j5 > 0;) {
        const int c = j5 > 13 ? 13 : (int)j5;             // 5^13 < 2^31
        u32 d = 1;
        for (int q = 0; q < c; q++) d *= 5u;
        u64 r = 0;
        for (int i = W - 1; i >= 0; i--) {
            const u64 cur = (r << 32) | P[i];
            P[i] = (u32)(cur / d);
            r = cur % d;
        }
        st |= r != 0;
        j5 -= c;
    }
    const int code = extract_scaled<W, L - 1>(P, G, D, rnd, sticky);
    *sticky = *sticky || st;
    return code;
}

// the printed form of mag 2^e (mag != 0) with sign `neg` into s; returns its length, or -1 when the
// decimal exponent is outside the supported range (|v| below 10^(-2p-1) or far above 10^p)
template <int L> B3D_HD int format_one(const u32 (&mag)[L], bool neg, i64 e, const DecimalTables& tb, char* s) {
    constexpr int DW = L - 1;
    const int p = tb.p;
    const int bl = bitlen(mag);
    u32 t2[2];
    if (bl > 64) shr(mag, bl - 64, t2);
    else { t2[0] = mag[0]; t2[1] = L > 1 ? mag[1] : 0u; }
    const double top = (double)(((u64)t2[1] << 32) | t2[0]);
    const i64 low = bl > 64 ? bl - 64 : 0;
    i64 E = (i64)floor(log10(top) + (double)(low + e) * 0.30102999566398119521);
    u32 D[DW];
    bool rnd = false, sticky = false;
    for (int attempt = 0;; attempt++) {
        if (attempt == 4) return -1;
        const int code = scaled_floor<L>(mag, e, (i64)p - 1 - E, tb, D, &rnd, &sticky);
        if (code < 0) return -1;
        if (code == 1 || cmp_limbs<DW>(D, tb.bounds + DW) >= 0) { E++; continue; }
        if (cmp_limbs<DW>(D, tb.bounds) < 0) { E--; continue; }
        break;
    }
    if (rnd && (sticky || (D[0] & 1u))) {
        u32 c = 1;
#pragma unroll
        for (int j = 0; j < DW; j++) {
            const u32 v = D[j] + c;
            c = (c && v == 0) ? 1u : 0u;
            D[j] = v;
        }
        if (cmp_limbs<DW>(D, tb.bounds + DW) == 0) {       // rounded up to 10^p
#pragma unroll
            for (int j = 0; j < DW; j++) D[j] = tb.bounds[j];
            E++;
        }
    }
    const int sg = neg ? 1 : 0;
    const bool sci = E < -4 || E >= p;
    // place of digit i (0 = most significant): sci d.ddd; fixed E >= 0 ddd.ddd; fixed E < 0 0.000ddd
    const int lead = sci ? sg : (E >= 0 ? sg : sg + 2 + (int)(-1 - E));
    const int dot = sci ? 1 : (E >= 0 ? (int)E + 1 : p + 1);     // digits before the point (p + 1: none)
    int tz = 0;
    bool nz = false;
    for (int done = 0; done < p; done += 9) {
        u64 r = 0;
#pragma unroll
        for (int j = DW - 1; j >= 0; j--) {
            const u64 cur = (r << 32) | D[j];
            D[j] = (u32)(cur / 1000000000ull);
            r = cur % 1000000000ull;
        }
        u32 chunk = (u32)r;
        for (int q = 0; q < 9 && done + q < p; q++) {
            const int i = p - 1 - (done + q);
            const u32 dg = chunk % 10u;
            chunk /= 10u;
            if (!nz) {
                if (dg == 0) tz++;
                else nz = true;
            }
            s[lead + i + (i >= dot ? 1 : 0)] = (char)('0' + dg);
        }
    }
    if (neg) s[0] = '-';
    const int nd = p - tz;                                  // digits after stripping trailing zeros
    if (sci) {
        int n = sg + nd;
        if (nd > 1) { s[sg + 1] = '.'; n++; }
        s[n++] = 'e';
        s[n++] = E < 0 ? '-' : '+';
        i64 a = E < 0 ? -E : E;
        char buf[20];
        int nb = 0;
        do { buf[nb++] = (char)('0' + a % 10); a /= 10; } while (a);
        if (nb < 2) buf[nb++] = '0';
        while (nb) s[n++] = buf[--nb];
        return n;
    }
    if (E >= 0) {
        if (nd > E + 1) { s[sg + E + 1] = '.'; return sg + nd + 1; }
        return sg + (int)E + 1;
    }
    s[sg] = '0';
    s[sg + 1] = '.';
    for (int z = 0; z < (int)(-1 - E); z++) s[sg + 2 + z] = '0';
    return lead + nd;
}

#ifdef __CUDACC__
constexpr int kFmtThreads = 64;

template <int L>
__global__ void __launch_bounds__(kFmtThreads) k_format_decimal(const int32_t* __restrict__ m, const i64* __restrict__ e,
                                                                i64 plane, i64 n, DecimalTables tb, char* __restrict__ out,
                                                                int32_t* __restrict__ len, long long* __restrict__ err) {
    extern __shared__ __align__(16) char sbuf[];
    const int stride = tb.stride;
    const i64 first = blockIdx.x * (i64)blockDim.x;
    const i64 i = first + threadIdx.x;
    char* s = sbuf + threadIdx.x * stride;
    if (i < n) {
        u32 mag[L];
        const bool neg = load_mag<L>(m, plane, i, mag);
        const i64 ex = e[i];
        int l;
        if (ex == EZ || is_zero(mag)) {
            s[0] = '0';
            l = 1;
        } else {
            l = format_one<L>(mag, neg, ex, tb, s);
            if (l < 0) {                                    // length -1: outside the supported range
                atomicAdd((unsigned long long*)err, 1ull);
                atomicMin(err + 1, (long long)i);
                s[0] = '?';
            }
        }
        len[i] = l;
    }
    __syncthreads();
    const i64 cnt = (n - first) < (i64)blockDim.x ? (n - first) : (i64)blockDim.x;
    const int4* src = reinterpret_cast<const int4*>(sbuf);
    int4* dst = reinterpret_cast<int4*>(out + first * stride);
    const i64 words = cnt * stride / 16;
    for (i64 w = threadIdx.x; w < words; w += blockDim.x) dst[w] = src[w];
}

// normalise mag so that bit 32 L - 1 is set; returns the exponent change
template <int L> __device__ __forceinline__ int normalise(u32 (&a)[L]) {
    const int sh = 32 * L - bitlen(a);
    u32 t[L];
    shl(a, sh, t);
#pragma unroll
    for (int k = 0; k < L; k++) a[k] = t[k];
    return sh;
}

// (ea, a) < (eb, b) for normalised magnitudes
template <int L> __device__ __forceinline__ bool less_norm(i64 ea, const u32 (&a)[L], i64 eb, const u32 (&b)[L]) {
    if (ea != eb) return ea < eb;
#pragma unroll
    for (int k = L - 1; k >= 0; k--)
        if (a[k] != b[k]) return a[k] < b[k];
    return false;
}

// kept size of each polynomial (0: all zero) and the byte length of its text (-1 when a kept coefficient is
// outside the formatter's range; dropped coefficients may be).  blocks_3d's rule, scanning from the top
// coefficient down, keeps the polynomial up to the lowest nonzero coefficient c_d whose higher coefficients are
// all below eps |c_d|:  size = 1 + min { d : c_d != 0 and max_{d' > d} |c_d'| < eps |c_d| }.  One warp per
// polynomial, one coefficient per lane (coalesced loads of the limb planes): chunks of 32 coefficients from the
// top, an exact suffix maximum of the normalised magnitudes by shuffles, carried from chunk to chunk.
template <int L>
__global__ void k_poly_sizes(const int32_t* __restrict__ m, const i64* __restrict__ e, i64 plane,
                             const i64* __restrict__ poly_num, i64 npoly, int D, int eps_shift,
                             const int32_t* __restrict__ len, int32_t* __restrict__ size, i64* __restrict__ text_len) {
    const i64 t = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (t >= npoly) return;                                  // whole warps leave together
    const i64 base = poly_num[t];
    // carried maximum of the coefficients above the current chunk (ce == EZ: none yet)
    u32 cm[L];
    zero(cm);
    i64 ce = EZ;
    int sz = -1;                                             // lowest d with the condition (-1: none yet)
    for (int top = D - 1; top >= 0; top -= 32) {
        const int d = top - lane;                            // lane 0: the highest coefficient of the chunk
        u32 c[L];
        zero(c);
        i64 en = EZ;
        if (d >= 0) {
            load_mag<L>(m, plane, base + d, c);
            const i64 ec = e[base + d];
            if (ec != EZ && !is_zero(c)) en = ec - normalise(c);
            else zero(c);
        }
        // exclusive prefix maximum over lanes 0 .. lane - 1 (the higher coefficients of the chunk), then the carry
        u32 mx[L];
        i64 emx = EZ;
        {
            u32 run[L];
            i64 erun = en;
#pragma unroll
            for (int k = 0; k < L; k++) run[k] = c[k];
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {         // inclusive scan of the maximum towards higher lanes
                u32 o[L];
#pragma unroll
                for (int k = 0; k < L; k++) o[k] = __shfl_up_sync(0xFFFFFFFFu, run[k], off);
                const i64 eo = __shfl_up_sync(0xFFFFFFFFu, erun, off);
                if (lane >= off && eo != EZ && (erun == EZ || less_norm<L>(erun, run, eo, o))) {
#pragma unroll
                    for (int k = 0; k < L; k++) run[k] = o[k];
                    erun = eo;
                }
            }
#pragma unroll
            for (int k = 0; k < L; k++) mx[k] = __shfl_up_sync(0xFFFFFFFFu, run[k], 1);
            emx = __shfl_up_sync(0xFFFFFFFFu, erun, 1);
            if (lane == 0) emx = EZ;
            if (ce != EZ && (emx == EZ || less_norm<L>(emx, mx, ce, cm))) {
#pragma unroll
                for (int k = 0; k < L; k++) mx[k] = cm[k];
                emx = ce;
            }
            // the new carry: the maximum of the whole chunk and the old carry (lane 31's inclusive value)
            u32 last[L];
#pragma unroll
            for (int k = 0; k < L; k++) last[k] = __shfl_sync(0xFFFFFFFFu, run[k], 31);
            const i64 elast = __shfl_sync(0xFFFFFFFFu, erun, 31);
            if (elast != EZ && (ce == EZ || less_norm<L>(ce, cm, elast, last))) {
#pragma unroll
                for (int k = 0; k < L; k++) cm[k] = last[k];
                ce = elast;
            }
        }
        const bool cond = en != EZ && (emx == EZ || less_norm<L>(emx, mx, en - eps_shift, c));
        const unsigned hit = __ballot_sync(0xFFFFFFFFu, cond);
        if (hit) sz = top - (31 - __clz(hit));               // the highest lane with the condition = lowest d
    }
    const int kept = sz < 0 ? 0 : sz + 1;
    // text length: the kept numbers quoted (length + 2) and joined by ",\n"; "\"0\"" for an all-zero polynomial
    i64 tl = 0;
    bool bad = false;
    for (int d0 = 0; d0 < kept; d0 += 32) {
        const int d = d0 + lane;
        if (d < kept) {
            const int l = len[base + d];
            if (l < 0) bad = true;
            else tl += l + 2;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) tl += __shfl_down_sync(0xFFFFFFFFu, tl, off);
    bad = __any_sync(0xFFFFFFFFu, bad);
    if (lane == 0) {
        size[t] = kept;
        text_len[t] = kept == 0 ? 3 : (bad ? -1 : tl + 2 * (i64)(kept - 1));
    }
}

#endif

template <int L> struct DecimalLaunch {
    static int format(const int32_t* m, const i64* e, i64 plane, i64 n, const DecimalTables& tb, char* out,
                      int32_t* len, long long* err, cudaStream_t st);
    static int poly_sizes(const int32_t* m, const i64* e, i64 plane, const i64* poly_num, i64 npoly, int D,
                          int eps_shift, const int32_t* len, int32_t* size, i64* text_len, cudaStream_t st);
};

#if defined(__CUDACC__) && defined(B3D_DEFINE_LAUNCH)
template <int L>
int DecimalLaunch<L>::format(const int32_t* m, const i64* e, i64 plane, i64 n, const DecimalTables& tb, char* out,
                             int32_t* len, long long* err, cudaStream_t st) {
    if (n == 0) return 0;
    const int smem = kFmtThreads * tb.stride;             // <= 64 x 416 bytes: no opt-in needed
    const i64 blocks = (n + kFmtThreads - 1) / kFmtThreads;
    k_format_decimal<L><<<(unsigned)blocks, kFmtThreads, smem, st>>>(m, e, plane, n, tb, out, len, err);
    return (int)cudaGetLastError();
}

template <int L>
int DecimalLaunch<L>::poly_sizes(const int32_t* m, const i64* e, i64 plane, const i64* poly_num, i64 npoly, int D,
                                 int eps_shift, const int32_t* len, int32_t* size, i64* text_len, cudaStream_t st) {
    if (npoly == 0) return 0;
    const i64 blocks = (npoly + 3) / 4;                      // one warp per polynomial
    k_poly_sizes<L><<<(unsigned)blocks, 128, 0, st>>>(m, e, plane, poly_num, npoly, D, eps_shift, len, size, text_len);
    return (int)cudaGetLastError();
}
#endif

}  // namespace b3d
