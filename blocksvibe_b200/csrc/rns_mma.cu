// The tensor-core residue product (k_rns_mma) and its launcher: one translation unit, independent of L.
#define B3D_RNS_MMA
#include "abi_internal.h"

namespace b3d {

int rns_mma_launch(const RnsMma& a, const RnsTables& tb, cudaStream_t st) {
    static unsigned long long configured = 0;            // devices whose shared-memory limits are raised
    const unsigned long long dbit = device_bit();
    const int smem = (128 + a.TN) * a.Kp;
    if (!(configured & dbit) || !dbit) {
        int rc = (int)cudaFuncSetAttribute(k_rns_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, (128 + 256) * 256);
        if (rc) return rc;
        rc = (int)cudaFuncSetAttribute(k_rns_mma4, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (128 + 256) * 256 + 128 * 256);
        if (rc) return rc;
        configured |= dbit;
    }
    const int64_t tiles_i = (4 * a.NI + 127) / 128;
    const int groups = (tb.np + kPrimesPerCta - 1) / kPrimesPerCta;
    if (a.yb && a.crt_kp >= 16 * groups && a.TN % 16 == 0) {      // CRT operand: four primes per CTA
        const int smem4 = (128 + a.TN) * a.Kp + 128 * a.TN;
        dim3 grid4((unsigned)(tiles_i * a.tiles_l), (unsigned)a.nb, (unsigned)groups);
        k_rns_mma4<<<grid4, 256, smem4, st>>>(a, tb);
        return (int)cudaGetLastError();
    }
    dim3 grid((unsigned)(tiles_i * a.tiles_l), (unsigned)a.nb, (unsigned)tb.np);
    k_rns_mma<<<grid, 128, smem, st>>>(a, tb);
    return (int)cudaGetLastError();
}

int cauchy_digits_launch(const CauchyLevel& lv, const uint32_t* table, int64_t dmax, int np, int64_t Rp, int64_t Kp,
                         int TR, int64_t mat_bytes, uint8_t* out, cudaStream_t st) {
    const int64_t n = lv.nb * Rp * (Kp / 4);
    if (n == 0) return 0;
    k_cauchy_digits<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(lv, table, dmax, np, Rp, Kp, TR, mat_bytes, out);
    return (int)cudaGetLastError();
}

}  // namespace b3d
