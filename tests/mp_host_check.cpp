// Host check of the multiprecision helpers of blocksvibe_b200/csrc/mp.cuh (compiled by g++ from
// tests/test_mp_host.py; the helpers are __host__ __device__, the same source the kernels use):
//   mac   the truncated product scan (mac_signed_mem with C0 > 0) stays within 2^(32 (C0 + 2)) of the exact sum
//   safe  where round_safe holds, every value within the error bound rounds like the approximation
//   col   add_norm_col (second operand in memory, run-time word offsets) == add_norm, bit for bit
// Prints one "<check> <cases> <failures>" line per check.
#include <cstdio>
#include <random>

#include "mp.cuh"

using namespace b3d;
static std::mt19937_64 rng(20261203);

template <int N> void fill(u32 (&a)[N], int kind) {
    for (int k = 0; k < N; k++) {
        u32 v = (u32)rng();
        if (kind == 1) v = ~0u;                       // all ones: the largest dropped part
        if (kind == 2) v = (rng() & 1) ? ~0u : 0u;
        a[k] = v;
    }
}

template <int L, int C0> long check_mac(int iters) {
    constexpr int NW = 2 * L + 2;
    long bad = 0;
    for (int it = 0; it < iters; it++) {
        const int n = 1 + (int)(rng() % 40);
        u32 ex[NW] = {0}, tr[NW] = {0};
        for (int t = 0; t < n; t++) {
            u32 a[L], b[L];
            fill(a, it % 3);
            fill(b, (it / 3) % 3);
            const bool neg = rng() & 1;
            mac_signed_mem<L, NW, 0>(ex, 1, a, b, neg);
            mac_signed_mem<L, NW, C0>(tr, 1, a, b, neg);
        }
        u32 d[NW];
        i64 br = 0;
        for (int k = 0; k < NW; k++) {
            const i64 v = (i64)ex[k] - tr[k] + br;
            d[k] = (u32)v;
            br = v >> 32;
        }
        if (d[NW - 1] >> 31) negate(d);
        for (int k = C0 + 2; k < NW; k++)
            if (d[k]) { bad++; break; }
    }
    return bad;
}

template <int L> bool same_round(const u32 (&a)[2 * L + 2], const u32 (&b)[2 * L + 2]) {
    u32 ra[L], rb[L];
    i64 ea, eb;
    const bool za = round_mag<L>(a, 0, ra, &ea), zb = round_mag<L>(b, 0, rb, &eb);
    if (za != zb || ea != eb) return false;
    for (int k = 0; k < L; k++)
        if (ra[k] != rb[k]) return false;
    return true;
}

// random magnitudes, many with a planted run of zeros or ones below the half bit (near a midpoint)
template <int L, int EW> long check_safe(int iters, long* nsafe) {
    constexpr int NW = 2 * L + 2, NB = nb_bits(L);
    long bad = 0;
    for (int it = 0; it < iters; it++) {
        u32 w[NW];
        fill(w, 0);
        const int bl = 32 * EW + (int)(rng() % (32 * (NW - EW) - 1)) + 1;
        for (int k = 0; k < NW; k++) {
            const int lo = 32 * k;
            if (lo >= bl) w[k] = 0;
            else if (lo + 32 > bl) w[k] &= (1u << (bl - lo)) - 1;
        }
        w[(bl - 1) >> 5] |= 1u << ((bl - 1) & 31);
        const int hb = bl - NB - 1;
        const int mode = (int)(rng() % 4);
        if (hb > 0 && mode) {
            const int run = (int)(rng() % (hb + 1));
            for (int bit = hb - run; bit < hb; bit++) {
                if (bit < 0) continue;
                if (mode == 1) w[bit >> 5] |= 1u << (bit & 31);
                else w[bit >> 5] &= ~(1u << (bit & 31));
            }
            if (mode == 3) w[hb >> 5] ^= 1u << (hb & 31);
        }
        if (!round_safe<L, NW, EW>(w)) continue;
        (*nsafe)++;
        for (int j = 0; j < 8; j++) {                 // w +- delta, |delta| < 2^(32 EW)
            u32 dl[NW] = {0};
            for (int k = 0; k < EW; k++) dl[k] = j == 0 ? ~0u : (u32)rng();
            u32 v[NW];
            if (!(j & 1)) {
                u64 c = 0;
                for (int k = 0; k < NW; k++) {
                    const u64 s = (u64)w[k] + dl[k] + c;
                    v[k] = (u32)s;
                    c = s >> 32;
                }
            } else {
                i64 b2 = 0;
                for (int k = 0; k < NW; k++) {
                    const i64 s = (i64)w[k] - dl[k] + b2;
                    v[k] = (u32)s;
                    b2 = s >> 32;
                }
            }
            if (!same_round<L>(w, v)) { bad++; break; }
        }
    }
    return bad;
}

template <int L> void number(u32 (&a)[L], i64* e, bool* n) {
    constexpr int NB = nb_bits(L);
    const int kind = (int)(rng() % 8);
    fill(a, 0);
    if (kind == 0) { zero(a); *e = EZ; *n = false; return; }
    if (kind == 1) { zero(a); a[rng() % L] = 1u << (rng() % 32); }                 // short, unnormalised
    if (kind >= 2) {                                                                 // NB bits
        a[L - 1] &= (1u << (NB - 32 * (L - 1))) - 1;
        a[L - 1] |= 1u << (NB - 1 - 32 * (L - 1));
    }
    *e = (i64)(rng() % 200) - 100;
    *n = rng() & 1;
}

template <int L> long check_col(int iters) {
    long bad = 0;
    for (int it = 0; it < iters; it++) {
        u32 a[L], b[L];
        i64 ea, eb;
        bool na, nb;
        number(a, &ea, &na);
        number(b, &eb, &nb);
        const int mode = (int)(rng() % 5);
        if (mode == 1 && ea != EZ && eb != EZ) eb = ea + (i64)(rng() % 65) - 32;              // close exponents
        if (mode == 2 && ea != EZ && eb != EZ) eb = ea + (i64)(rng() % (200 * L)) - 100 * L;  // far apart
        if (mode == 3 && ea != EZ) {                                                          // cancellation
            for (int k = 0; k < L; k++) b[k] = a[k];
            eb = ea;
            nb = !na;
            b[rng() % L] ^= 1u << (rng() % 32);
        }
        u32 r1[L], r2[L];
        bool n1, n2;
        i64 e1, e2;
        add_norm<L>(a, na, ea, b, nb, eb, r1, &n1, &e1);
        constexpr int stride = 3;
        u32 col[stride * L], scratch[stride * L];
        for (int k = 0; k < L; k++) col[k * stride] = b[k];
        add_norm_col<L>(a, na, ea, col, nb, eb, scratch, stride, r2, &n2, &e2);
        bool same = n1 == n2 && e1 == e2;
        for (int k = 0; k < L; k++) same = same && r1[k] == r2[k];
        if (!same) bad++;
    }
    return bad;
}

int main() {
    printf("mac10 %d %ld\n", 20000, check_mac<10, 5>(20000));
    printf("mac34 %d %ld\n", 3000, check_mac<34, 29>(3000));
    long ns = 0, b = check_safe<4, 3>(1000000, &ns);
    printf("safe4 %ld %ld\n", ns, b);
    ns = 0;
    b = check_safe<10, 7>(200000, &ns);
    printf("safe10 %ld %ld\n", ns, b);
    printf("col10 %d %ld\n", 200000, check_col<10>(200000));
    printf("col34 %d %ld\n", 100000, check_col<34>(100000));
    printf("col42 %d %ld\n", 50000, check_col<42>(50000));
    return 0;
}
