// The Cauchy step of a recursion level as an RNS GEMM on the tensor cores (rns.cuh), per group g:
//   H_raw[g] = C[g] X[g],  C[g][r][i] = round(2^(NB-1) / (D'_r - D_i)) (one fixed exponent 1 - NB for the
//   whole table: an absolute error of 2^-NB on each 2 / d),  X[g][i][n] = res[col[g][i]][n] aligned per
//   column (g, n);  then H = H_raw + h_inf (one rounding each).
// k_cauchy_align gathers and aligns X; k_cauchy_digits writes the digit matrices of C straight from a table of
// the residues of round(2^(NB-1) / d) for |d| <= dmax; k_cauchy_add_hinf adds the h_inf rows.
#pragma once
#include "kernels.cuh"
#include "rns.cuh"

namespace b3d {

// X[g][i][n] (layout (nb, Kc, N)) aligned to the column's largest exponent, column exponents oe[g * N + n].
// Two kernels: the exponent of each column (g, n), then one thread per element (g, i, n) for the shifts, so
// that a level's nb Kc N elements spread over the whole GPU (consecutive threads: consecutive n, coalesced).
template <int L>
__global__ void k_cauchy_colexp(const int32_t* __restrict__ rm, const i64* __restrict__ re, i64 rplane, CauchyLevel lv,
                                i64* __restrict__ oe) {
    i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    const i64 N = lv.N;
    if (t >= lv.nb * N) return;
    i64 g, n;
    split2(t, N, lv.nb * N, n, g);
    const i64 ncol = lv.ncol[g];
    const i64* col = lv.col + g * lv.Kc;
    i64 E = EZ;
    for (i64 i = 0; i < ncol; i++) {
        const i64 ix = col[i] * N + n;
        const i64 ei = re[ix];
        if (ei > E && rm[(L - 1) * rplane + ix] != 0) E = ei;
    }
    oe[t] = E;
}

template <int L>
__global__ void k_cauchy_align(const int32_t* __restrict__ rm, const i64* __restrict__ re, i64 rplane, CauchyLevel lv,
                               const i64* __restrict__ ce, int32_t* __restrict__ om, i64 oplane) {
    i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    const i64 N = lv.N;
    if (t >= lv.nb * lv.Kc * N) return;
    i64 n, i, g;
    split3(t, N, lv.Kc, lv.nb * lv.Kc * N, n, i, g);
    const i64 E = ce[g * N + n];
    u32 a[L], s[L];
    bool neg = false;
    if (i < lv.ncol[g] && E != EZ) {
        const i64 ix = lv.col[g * lv.Kc + i] * N + n;
        neg = load_mag<L>(rm, rplane, ix, a);
        const i64 ei = re[ix];
        if (is_zero(a) || ei == EZ || E - ei >= 32 * L) { zero(s); neg = false; }
        else shr(a, (int)(E - ei), s);
    } else {
        zero(s);
    }
    store_signed<L>(om, oplane, t, s, neg);
}

// k_cauchy_align with sign-magnitude output: |x| aligned, the sign in bit 31 of limb L - 1 (free: |x| < 2^NB),
// the input form of k_cauchy4
template <int L>
__global__ void k_cauchy_align_sm(const int32_t* __restrict__ rm, const i64* __restrict__ re, i64 rplane, CauchyLevel lv,
                                  const i64* __restrict__ ce, int32_t* __restrict__ om, i64 oplane) {
    i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    const i64 N = lv.N;
    if (t >= lv.nb * lv.Kc * N) return;
    i64 n, i, g;
    split3(t, N, lv.Kc, lv.nb * lv.Kc * N, n, i, g);
    const i64 E = ce[g * N + n];
    u32 a[L], s[L];
    bool neg = false;
    if (i < lv.ncol[g] && E != EZ) {
        const i64 ix = lv.col[g * lv.Kc + i] * N + n;
        neg = load_mag<L>(rm, rplane, ix, a);
        const i64 ei = re[ix];
        if (is_zero(a) || ei == EZ || E - ei >= 32 * L) { zero(s); neg = false; }
        else shr(a, (int)(E - ei), s);
    } else {
        zero(s);
    }
#pragma unroll
    for (int k = 0; k < L; k++) om[k * oplane + t] = (int32_t)(k == L - 1 && neg ? (s[k] | 0x80000000u) : s[k]);
}

#ifdef B3D_RNS_MMA
// digit matrices of C: matrix (prime j, group g), rows 4 r + s, columns i, tiles of TR digit rows; threads over
// (g, r < Rp, i4 < Kp / 4), four consecutive i per thread.  table[(d + dmax) * np + j] = residue of
// round(2^(NB-1) / d) mod p_j (zero for d = 0)
__global__ void k_cauchy_digits(CauchyLevel lv, const uint32_t* __restrict__ table, int64_t dmax, int np, int64_t Rp,
                                int64_t Kp, int TR, int64_t mat_bytes, uint8_t* __restrict__ out) {
    int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t K4 = Kp / 4;
    if (t >= lv.nb * Rp * K4) return;
    const int64_t i0 = (t % K4) * 4, r = (t / K4) % Rp, g = t / (K4 * Rp);
    int64_t row[4];
    bool live[4];
    const bool rok = r < lv.Mr && r < lv.nrow[g];
    const int64_t D = rok ? lv.rowd[g * lv.Mr + r] : 0;
#pragma unroll
    for (int u = 0; u < 4; u++) {
        const int64_t i = i0 + u;
        const bool ok = rok && i < lv.Kc && i < lv.ncol[g];
        const int64_t d = ok ? D - lv.cold[g * lv.Kc + i] : 0;
        live[u] = ok && d != 0 && d >= -dmax && d <= dmax;
        row[u] = (d + dmax) * np;
    }
    for (int j = 0; j < np; j++) {
        uint32_t res[4];
#pragma unroll
        for (int u = 0; u < 4; u++) res[u] = live[u] ? __ldg(table + row[u] + j) : 0u;
        uint8_t* base = out + ((size_t)j * lv.nb + g) * mat_bytes;
#pragma unroll
        for (int s = 0; s < 4; s++) {
            uint32_t w = ((res[0] >> (8 * s)) & 0xFFu) | (((res[1] >> (8 * s)) & 0xFFu) << 8) |
                         (((res[2] >> (8 * s)) & 0xFFu) << 16) | (((res[3] >> (8 * s)) & 0xFFu) << 24);
            *reinterpret_cast<uint32_t*>(base + tiled_offset(4 * r + s, i0, TR, Kp)) = w;
        }
    }
}
#endif

// H[g][r][n] = H_raw[g][r][n] + h_inf[gsrc[g], m, gj[g], n]  (rows r >= nrow[g] are written as zero)
template <int L>
__global__ void k_cauchy_add_hinf(const int32_t* __restrict__ am, const i64* __restrict__ ae, i64 aplane,
                                  const int32_t* __restrict__ hm, const i64* __restrict__ he, i64 hplane, CauchyLevel lv,
                                  int32_t* __restrict__ om, i64* __restrict__ oe, i64 oplane) {
    i64 t = blockIdx.x * (i64)blockDim.x + threadIdx.x;
    const i64 N = lv.N;
    if (t >= lv.nb * lv.Mr * N) return;
    const i64 n = t % N, r = (t / N) % lv.Mr, g = t / (N * lv.Mr);
    u32 a[L], h[L], o[L];
    if (r >= lv.nrow[g]) {
        zero(o);
        store_signed<L>(om, oplane, t, o, false);
        oe[t] = EZ;
        return;
    }
    const i64 hidx = ((lv.gsrc[g] * lv.hlevels + lv.m) * lv.Jh + lv.gj[g]) * N + n;
    bool na = load_mag<L>(am, aplane, t, a);
    bool nh = load_mag<L>(hm, hplane, hidx, h);
    bool no;
    i64 eo;
    add_norm<L>(a, na, ae[t], h, nh, he[hidx], o, &no, &eo);
    store_signed<L>(om, oplane, t, o, no);
    oe[t] = eo;
}

template <int L>
struct CauchyRnsLaunch {
    static int align(const int32_t* rm, const i64* re, i64 rplane, const CauchyLevel& lv, int32_t* om, i64* oe,
                     i64 oplane, cudaStream_t st);
    static int add_hinf(const int32_t* am, const i64* ae, i64 aplane, const int32_t* hm, const i64* he, i64 hplane,
                        const CauchyLevel& lv, int32_t* om, i64* oe, i64 oplane, cudaStream_t st);
    static int align_sm(const int32_t* rm, const i64* re, i64 rplane, const CauchyLevel& lv, int32_t* om, i64* oe,
                        i64 oplane, cudaStream_t st);
};

#ifdef B3D_DEFINE_LAUNCH
template <int L>
int CauchyRnsLaunch<L>::align(const int32_t* rm, const i64* re, i64 rplane, const CauchyLevel& lv, int32_t* om,
                              i64* oe, i64 oplane, cudaStream_t st) {
    const i64 n = lv.nb * lv.N, ne = n * lv.Kc;
    if (n == 0) return 0;
    k_cauchy_colexp<L><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(rm, re, rplane, lv, oe);
    if (ne > 0) k_cauchy_align<L><<<(unsigned)((ne + 127) / 128), 128, 0, st>>>(rm, re, rplane, lv, oe, om, oplane);
    return (int)cudaGetLastError();
}

template <int L>
int CauchyRnsLaunch<L>::align_sm(const int32_t* rm, const i64* re, i64 rplane, const CauchyLevel& lv, int32_t* om,
                                 i64* oe, i64 oplane, cudaStream_t st) {
    const i64 n = lv.nb * lv.N, ne = n * lv.Kc;
    if (n == 0) return 0;
    k_cauchy_colexp<L><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(rm, re, rplane, lv, oe);
    if (ne > 0) k_cauchy_align_sm<L><<<(unsigned)((ne + 127) / 128), 128, 0, st>>>(rm, re, rplane, lv, oe, om, oplane);
    return (int)cudaGetLastError();
}

template <int L>
int CauchyRnsLaunch<L>::add_hinf(const int32_t* am, const i64* ae, i64 aplane, const int32_t* hm, const i64* he,
                                 i64 hplane, const CauchyLevel& lv, int32_t* om, i64* oe, i64 oplane, cudaStream_t st) {
    const i64 n = lv.nb * lv.Mr * lv.N;
    if (n == 0) return 0;
    k_cauchy_add_hinf<L><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(am, ae, aplane, hm, he, hplane, lv, om, oe, oplane);
    return (int)cudaGetLastError();
}
#endif

}  // namespace b3d
