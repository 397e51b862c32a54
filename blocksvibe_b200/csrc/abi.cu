// extern "C" entry points of libb3dgpu.so (declared in include/b3dgpu.h): argument checks, dispatch on
// the limb count, error reporting.  No device memory is allocated here.
#include <cstdio>
#include <string>

#include "b3dgpu.h"
#include "abi_internal.h"

namespace b3d {

thread_local std::string g_error;

int fail(int code, const std::string& what) {
    g_error = what;
    return code;
}

int cuda_status(int code, const char* fn) {
    if (code == 0) return 0;
    return fail(code, std::string(fn) + ": " + cudaGetErrorString((cudaError_t)code));
}

}  // namespace b3d

namespace {

using b3d::cuda_status;
using b3d::fail;

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

bool nonneg(int64_t x) { return x >= 0; }

}  // namespace

extern "C" {

int b3d_version(void) { return 100; }

const char* b3d_last_error(void) { return b3d::g_error.c_str(); }

int b3d_supported_limbs(int L) {
    switch (L) {
        case 6: case 10: case 14: case 18: case 22: case 26: case 30: case 34: case 38: case 42: case 46: return 1;
        default: return 0;
    }
}

int b3d_align(int L, const int32_t* m, const int64_t* e, int64_t plane, int64_t nbatch, int64_t R, int64_t K,
              int64_t sb, int64_t sr, int64_t sk, const int64_t* bidx, int32_t* om, int64_t* oe, int64_t oplane,
              int kmajor, void* stream) {
    if (!nonneg(nbatch) || !nonneg(R) || !nonneg(K)) return fail(B3D_E_ARG, "b3d_align: negative size");
    B3D_DISPATCH(L, cuda_status(LX::align(m, e, plane, nbatch, R, K, sb, sr, sk, bidx, om, oe, oplane, kmajor,
                                         as_stream(stream)), "b3d_align"));
}

int b3d_gemm_aligned(int L, const int32_t* am, const int64_t* ae, int64_t aplane, const int32_t* bm,
                     const int64_t* be, int64_t bplane, int64_t nbatch, int64_t M, int64_t N, int64_t K,
                     int32_t* cm, int64_t* ce, int64_t cplane, void* stream) {
    if (!nonneg(nbatch) || !nonneg(M) || !nonneg(N) || !nonneg(K)) return fail(B3D_E_ARG, "b3d_gemm_aligned: negative size");
    B3D_DISPATCH(L, cuda_status(LX::gemm_aligned(am, ae, aplane, bm, be, bplane, nbatch, M, N, K, cm, ce, cplane,
                                                as_stream(stream)), "b3d_gemm_aligned"));
}

int b3d_mul(int L, const int32_t* am, const int64_t* ae, int64_t aplane, const int64_t* aidx,
            const int32_t* bm, const int64_t* be, int64_t bplane, const int64_t* bidx, int64_t n,
            int32_t* cm, int64_t* ce, int64_t cplane, void* stream) {
    if (!nonneg(n)) return fail(B3D_E_ARG, "b3d_mul: negative size");
    B3D_DISPATCH(L, cuda_status(LX::mul(am, ae, aplane, aidx, bm, be, bplane, bidx, n, cm, ce, cplane,
                                       as_stream(stream)), "b3d_mul"));
}

int b3d_add(int L, const int32_t* am, const int64_t* ae, int64_t aplane, const int64_t* aidx,
            const int32_t* bm, const int64_t* be, int64_t bplane, const int64_t* bidx, int64_t n,
            int32_t* cm, int64_t* ce, int64_t cplane, void* stream) {
    if (!nonneg(n)) return fail(B3D_E_ARG, "b3d_add: negative size");
    B3D_DISPATCH(L, cuda_status(LX::add(am, ae, aplane, aidx, bm, be, bplane, bidx, n, cm, ce, cplane,
                                       as_stream(stream)), "b3d_add"));
}

int b3d_cauchy_level(int L, const int32_t* rm, const int64_t* re, int64_t rplane, const int32_t* hm,
                     const int64_t* he, int64_t hplane, const b3d_level_tables* lv, int32_t* om, int64_t* oe,
                     int64_t oplane, void* stream) {
    if (!lv || lv->nb < 0 || lv->Mr < 0 || lv->Kc < 0 || lv->N < 0 || lv->m < 0 || lv->m >= lv->hlevels)
        return fail(B3D_E_ARG, "b3d_cauchy_level: invalid level description");
    b3d::CauchyLevel c{lv->m, lv->nb, lv->Mr, lv->Kc, lv->N, lv->hlevels, lv->Jh, lv->gsrc, lv->gj,
                       lv->rowd, lv->nrow, lv->cold, lv->ncol, lv->col};
    B3D_DISPATCH(L, cuda_status(LX::cauchy(rm, re, rplane, hm, he, hplane, c, om, oe, oplane, as_stream(stream)),
                                "b3d_cauchy_level"));
}

int b3d_pole_level(int L, const int32_t* hm, const int64_t* he, int64_t hplane, const int32_t* Rm,
                   const int64_t* Re, int64_t Rplane, const int32_t* Qm, const int64_t* Qe, int64_t Qplane,
                   const int64_t* t_hrow, const int64_t* t_R, const int64_t* t_qL, const int64_t* t_slot,
                   int64_t T, int64_t B, int S, int32_t* ym, int64_t* ye, int64_t yplane, int32_t* rm,
                   int64_t* re, int64_t rplane, void* stream) {
    if (!nonneg(T) || B < 1 || S < 1) return fail(B3D_E_ARG, "b3d_pole_level: invalid size");
    B3D_DISPATCH(L, cuda_status(LX::pole(hm, he, hplane, Rm, Re, Rplane, Qm, Qe, Qplane, t_hrow, t_R, t_qL, t_slot,
                                        T, B, S, ym, ye, yplane, rm, re, rplane, as_stream(stream)),
                                "b3d_pole_level"));
}

int b3d_pole_level_mma(int L, const int32_t* hm, const int64_t* he, int64_t hplane, const int32_t* Rm,
                       const int64_t* Re, int64_t Rplane, const int32_t* Qm, const int64_t* Qe, int64_t Qplane,
                       const int64_t* t_hrow, const int64_t* t_R, const int64_t* t_qL, const int64_t* t_slot,
                       int64_t T, int64_t B, int S, int32_t* ym, int64_t* ye, int64_t yplane, int32_t* rm,
                       int64_t* re, int64_t rplane, int* err, void* stream) {
    if (!nonneg(T) || B < 1 || S < 1) return fail(B3D_E_ARG, "b3d_pole_level_mma: invalid size");
    if (S > 8) return fail(B3D_E_ARG, "b3d_pole_level_mma: S > 8 (use b3d_pole_level)");
    if (!err) return fail(B3D_E_ARG, "b3d_pole_level_mma: no error flag");
    B3D_DISPATCH(L, cuda_status(LX::pole_mma(hm, he, hplane, Rm, Re, Rplane, Qm, Qe, Qplane, t_hrow, t_R, t_qL, t_slot,
                                            T, B, S, ym, ye, yplane, rm, re, rplane, err, as_stream(stream)),
                                "b3d_pole_level_mma"));
}

int b3d_moments_level(int L, const int32_t* rm, const int64_t* re, int64_t rplane, const int32_t* pm,
                      const int64_t* pe, int64_t pplane, const int64_t* q_slot, const int64_t* q_row,
                      const int64_t* q_n, int64_t Q, int64_t N, int R1, int32_t* mm, int64_t* me, int64_t mplane,
                      void* stream) {
    if (!nonneg(Q) || !nonneg(N) || R1 < 1) return fail(B3D_E_ARG, "b3d_moments_level: invalid size");
    B3D_DISPATCH(L, cuda_status(LX::moments(rm, re, rplane, pm, pe, pplane, q_slot, q_row, q_n, Q, N, R1, mm, me,
                                           mplane, as_stream(stream)), "b3d_moments_level"));
}

int b3d_moments_stage(int L, const int32_t* rm, const int64_t* re, int64_t rplane, const int32_t* pm,
                      const int64_t* pe, int64_t pplane, const int64_t* q_slot, const int64_t* q_row,
                      const int64_t* q_n, int64_t Q, int64_t N, int64_t w, int64_t rows, int32_t* ym, int64_t* ye,
                      int64_t yplane, void* stream) {
    if (!nonneg(Q) || !nonneg(N) || !nonneg(w) || !nonneg(rows)) return fail(B3D_E_ARG, "b3d_moments_stage: invalid size");
    B3D_DISPATCH(L, cuda_status(LX::moments_stage(rm, re, rplane, pm, pe, pplane, q_slot, q_row, q_n, Q, N, w, rows, ym,
                                                 ye, yplane, as_stream(stream)), "b3d_moments_stage"));
}

int b3d_moments_flush(int L, const int32_t* ym, const int64_t* ye, int64_t yplane, const int64_t* row_shift, int64_t m0,
                      int W, int64_t rows, int64_t N, int R1, const uint32_t* nk, const int32_t* nkb, int NN, int KW,
                      int accumulate, int Lout, int32_t* mm, int64_t* me, int64_t mplane, void* stream) {
    if (!nonneg(rows) || !nonneg(N) || !nonneg(m0) || W < 0 || R1 < 1 || R1 > 32 || NN < 1 || KW < 1 || KW > 12)
        return fail(B3D_E_ARG, "b3d_moments_flush: invalid size (1 <= R + 1 <= 32, 1 <= KW <= 12)");
    if ((Lout != L && Lout != L + 4) || !b3d_supported_limbs(Lout))
        return fail(B3D_E_ARG, "b3d_moments_flush: Lout must be L or L + 4 (compiled)");
    B3D_DISPATCH(L, cuda_status(LX::moments_flush(ym, ye, yplane, row_shift, m0, W, rows, N, R1, nk, nkb, NN, KW,
                                                 accumulate, Lout, mm, me, mplane, as_stream(stream)), "b3d_moments_flush"));
}

int b3d_resize(int L, const int32_t* m, const int64_t* e, int64_t plane, int64_t n, int Lout, int32_t* om, int64_t* oe,
               int64_t oplane, void* stream) {
    if (!nonneg(n) || (Lout != L && Lout != L + 4 && Lout != L - 4) || !b3d_supported_limbs(Lout))
        return fail(B3D_E_ARG, "b3d_resize: Lout must be L or L +- 4 (compiled)");
    B3D_DISPATCH(L, cuda_status(LX::resize(m, e, plane, n, Lout, om, oe, oplane, as_stream(stream)), "b3d_resize"));
}

namespace {
b3d::RnsTables tables_of(const b3d_rns_tables* t) {
    return b3d::RnsTables{t->p, t->mu, t->w, t->conv, t->inv, t->mj, t->mfull, t->np, t->ml, t->mtop, t->msw};
}
}  // namespace

int b3d_rns_layout(int L, int* np, int* ml) {
    if (!b3d_supported_limbs(L)) return fail(B3D_E_LIMBS, "no kernels compiled for L = " + std::to_string(L));
    *np = b3d::rns_primes(L);
    *ml = b3d::rns_mlimbs(L);
    return 0;
}

int b3d_rns_split(int L, const int32_t* m, int64_t plane, int64_t nb, int64_t R, int64_t K, int64_t sb, int64_t sr,
                  int64_t sk, int64_t Rp, int64_t Kp, int TR, const b3d_rns_tables* tb, uint8_t* out,
                  int64_t mat_bytes, void* stream) {
    if (!tb || nb < 0 || R < 0 || K < 0 || Rp < R || Kp < K || Kp % 32 || TR % 16 || TR <= 0 || (4 * Rp) % TR ||
        mat_bytes < 4 * Rp * Kp || tb->np != b3d::rns_primes(L))
        return fail(B3D_E_ARG, "b3d_rns_split: invalid sizes or tables");
    b3d::RnsTables t = tables_of(tb);
    B3D_DISPATCH_RNS(L, cuda_status(RX::split(m, plane, nb, R, K, sb, sr, sk, Rp, Kp, TR, t, out, mat_bytes,
                                              as_stream(stream)), "b3d_rns_split"));
}

int b3d_rns_split_mma(int L, const b3d_rns_split_args* a, const b3d_rns_tables* tb, void* stream) {
    if (!a || !tb || tb->np != b3d::rns_primes(L) || a->nb < 0 || a->nb > 65535 || a->R < 0 || a->K < 0 ||
        a->Rp < a->R || a->Kp < a->K || a->Kp % 32 || a->TR % 16 || a->TR <= 0 || (4 * a->Rp) % a->TR ||
        a->mat_bytes < 4 * a->Rp * a->Kp || a->Ks % 32 || a->Ks < 4 * L || a->NS % 16 || a->NS <= 0 ||
        a->NS > 256 || 2 * a->NS < 4 * tb->np || 128 * a->Ks + 2 * a->NS * a->Ks + tb->np * 512 > b3d::kRnsSmemCap)
        return fail(B3D_E_ARG, "b3d_rns_split_mma: invalid sizes or tables");
    b3d::RnsSplit c{a->m, a->plane, a->nb, a->R, a->K, a->sb, a->sr, a->sk, a->Rp, a->Kp, a->TR, a->mat_bytes,
                    a->out, a->C, a->Ks, a->NS, a->err};
    b3d::RnsTables t = tables_of(tb);
    B3D_DISPATCH_RNS(L, cuda_status(RX::split_mma(c, t, as_stream(stream)), "b3d_rns_split_mma"));
}

int b3d_rns_mma(const b3d_rns_mma_args* a, const b3d_rns_tables* tb, void* stream) {
    if (!a || !tb || a->Kp <= 0 || a->Kp > 256 || a->Kp % 32 || a->TN < 16 || a->TN > 256 || a->TN % 16 ||
        a->nb <= 0 || a->nb > 65535 || tb->np <= 0 || tb->np > 65535 || a->NI < 0 || a->NL < 0 ||
        a->tiles_l * (a->TN / 4) < a->NL || a->x_mat < ((4 * a->NI + 127) / 128) * 128 * (int64_t)a->Kp ||
        a->y_mat < a->tiles_l * a->TN * (int64_t)a->Kp)
        return fail(B3D_E_ARG, "b3d_rns_mma: invalid sizes");
    if (a->NI == 0 || a->NL == 0) return 0;
    if (a->yb && (a->crt_kp % 32 || a->crt_kp < 4 * (int64_t)tb->np))
        return fail(B3D_E_ARG, "b3d_rns_mma: CRT operand row too short");
    b3d::RnsMma m{a->X, a->Y, a->x_mat, a->y_mat, a->nb, a->NI, a->NL, a->Kp, a->TN, a->tiles_l, a->out_b, a->out_i,
                  a->out_l, a->out, a->err, a->yb, a->crt_kp};
    return cuda_status(b3d::rns_mma_launch(m, tables_of(tb), as_stream(stream)), "b3d_rns_mma");
}

int b3d_rns_crt_mma(int L, const b3d_rns_crt_args* a, const b3d_rns_tables* tb, void* stream) {
    if (!a || !tb || tb->np != b3d::rns_primes(L) || tb->ml != b3d::rns_mlimbs(L) || a->Kc % 32 ||
        a->Kc < 4 * tb->np || a->NH % 16 || a->NH <= 0 || a->NH > 256 || 2 * a->NH < 4 * tb->ml + 3 ||
        (128 + 2 * a->NH) * a->Kc > b3d::kRnsSmemCap || a->n != a->nbatch * a->M * a->N || a->n < 0)
        return fail(B3D_E_ARG, "b3d_rns_crt_mma: invalid sizes or tables");
    b3d::RnsCrt c{a->A, a->T, a->Kc, a->NH, a->n, a->nbatch, a->M, a->N, a->ea, a->eb, a->cm, a->ce, a->cplane, a->err};
    b3d::RnsTables t = tables_of(tb);
    B3D_DISPATCH_RNS(L, cuda_status(RX::crt_mma(c, t, as_stream(stream)), "b3d_rns_crt_mma"));
}

int b3d_rns_crt(int L, const uint32_t* res, int64_t n, const int64_t* ea, const int64_t* eb, int64_t nbatch,
                int64_t M, int64_t N, const b3d_rns_tables* tb, int32_t* cm, int64_t* ce, int64_t cplane,
                void* stream) {
    if (!tb || n != nbatch * M * N || n < 0 || tb->np != b3d::rns_primes(L) || tb->ml != b3d::rns_mlimbs(L))
        return fail(B3D_E_ARG, "b3d_rns_crt: invalid sizes or tables");
    b3d::RnsTables t = tables_of(tb);
    B3D_DISPATCH_RNS(L, cuda_status(RX::crt(res, n, ea, eb, nbatch, M, N, t, cm, ce, cplane, as_stream(stream)),
                                    "b3d_rns_crt"));
}

namespace {
b3d::CauchyLevel level_of(const b3d_level_tables* lv) {
    return b3d::CauchyLevel{lv->m, lv->nb, lv->Mr, lv->Kc, lv->N, lv->hlevels, lv->Jh, lv->gsrc, lv->gj,
                            lv->rowd, lv->nrow, lv->cold, lv->ncol, lv->col};
}
bool level_ok(const b3d_level_tables* lv) {
    return lv && lv->nb >= 0 && lv->Mr >= 0 && lv->Kc >= 0 && lv->N >= 0 && lv->m >= 0 && lv->m < lv->hlevels;
}
}  // namespace

int b3d_cauchy_align(int L, const int32_t* rm, const int64_t* re, int64_t rplane, const b3d_level_tables* lv,
                     int32_t* om, int64_t* oe, int64_t oplane, void* stream) {
    if (!level_ok(lv)) return fail(B3D_E_ARG, "b3d_cauchy_align: invalid level description");
    b3d::CauchyLevel c = level_of(lv);
    B3D_DISPATCH_CAUCHY(L, cuda_status(CX::align(rm, re, rplane, c, om, oe, oplane, as_stream(stream)), "b3d_cauchy_align"));
}

int b3d_cauchy_align_sm(int L, const int32_t* rm, const int64_t* re, int64_t rplane, const b3d_level_tables* lv,
                        int32_t* om, int64_t* oe, int64_t oplane, void* stream) {
    if (!level_ok(lv)) return fail(B3D_E_ARG, "b3d_cauchy_align_sm: invalid level description");
    b3d::CauchyLevel c = level_of(lv);
    B3D_DISPATCH_CAUCHY(L, cuda_status(CX::align_sm(rm, re, rplane, c, om, oe, oplane, as_stream(stream)),
                                       "b3d_cauchy_align_sm"));
}

int b3d_cauchy_level4(int L, const int32_t* xm, const int64_t* xe, int64_t xplane, const int32_t* hm,
                      const int64_t* he, int64_t hplane, const b3d_level_tables* lv, int64_t dmax, int32_t* om,
                      int64_t* oe, int64_t oplane, void* stream) {
    if (!level_ok(lv)) return fail(B3D_E_ARG, "b3d_cauchy_level4: invalid level description");
    if (dmax < 1 || dmax >= (1 << 16)) return fail(B3D_E_ARG, "b3d_cauchy_level4: dmax must be in [1, 65535]");
    if (dmax >= (1 << 10) && lv->Kc >= 2048)
        return fail(B3D_E_ARG, "b3d_cauchy_level4: more than 2047 columns with 16-bit digits");
    b3d::CauchyLevel c = level_of(lv);
    B3D_DISPATCH(L, cuda_status(LX::cauchy4(xm, xe, xplane, hm, he, hplane, c, dmax, om, oe, oplane, as_stream(stream)),
                                "b3d_cauchy_level4"));
}

int b3d_cauchy_level2(int L, const int32_t* xm, const int64_t* xe, int64_t xplane, const int32_t* hm,
                      const int64_t* he, int64_t hplane, const b3d_level_tables* lv, int32_t* om, int64_t* oe,
                      int64_t oplane, void* stream) {
    if (!level_ok(lv)) return fail(B3D_E_ARG, "b3d_cauchy_level2: invalid level description");
    b3d::CauchyLevel c = level_of(lv);
    B3D_DISPATCH(L, cuda_status(LX::cauchy2(xm, xe, xplane, hm, he, hplane, c, om, oe, oplane, as_stream(stream)),
                                "b3d_cauchy_level2"));
}

int b3d_cauchy_level3(int L, const int32_t* xm, const int64_t* xe, int64_t xplane, const int32_t* hm,
                      const int64_t* he, int64_t hplane, const b3d_level_tables* lv, int64_t dmax, int32_t* om,
                      int64_t* oe, int64_t oplane, void* stream) {
    if (!level_ok(lv)) return fail(B3D_E_ARG, "b3d_cauchy_level3: invalid level description");
    if (dmax < 1 || dmax >= (1 << 16)) return fail(B3D_E_ARG, "b3d_cauchy_level3: dmax must be in [1, 65535]");
    b3d::CauchyLevel c = level_of(lv);
    B3D_DISPATCH(L, cuda_status(LX::cauchy3(xm, xe, xplane, hm, he, hplane, c, dmax, om, oe, oplane, as_stream(stream)),
                                "b3d_cauchy_level3"));
}

int b3d_cauchy_digits(const b3d_level_tables* lv, const uint32_t* table, int64_t dmax, int np, int64_t Rp, int64_t Kp,
                      int TR, int64_t mat_bytes, uint8_t* out, void* stream) {
    if (!level_ok(lv) || dmax < 0 || np <= 0 || Rp < lv->Mr || Kp < lv->Kc || Kp % 32 || TR % 16 || TR <= 0 ||
        (4 * Rp) % TR || mat_bytes < 4 * Rp * Kp)
        return fail(B3D_E_ARG, "b3d_cauchy_digits: invalid sizes");
    return cuda_status(b3d::cauchy_digits_launch(level_of(lv), table, dmax, np, Rp, Kp, TR, mat_bytes, out,
                                                 as_stream(stream)), "b3d_cauchy_digits");
}

int b3d_cauchy_add_hinf(int L, const int32_t* am, const int64_t* ae, int64_t aplane, const int32_t* hm,
                        const int64_t* he, int64_t hplane, const b3d_level_tables* lv, int32_t* om, int64_t* oe,
                        int64_t oplane, void* stream) {
    if (!level_ok(lv)) return fail(B3D_E_ARG, "b3d_cauchy_add_hinf: invalid level description");
    b3d::CauchyLevel c = level_of(lv);
    B3D_DISPATCH_CAUCHY(L, cuda_status(CX::add_hinf(am, ae, aplane, hm, he, hplane, c, om, oe, oplane, as_stream(stream)),
                                       "b3d_cauchy_add_hinf"));
}

}  // extern "C"
