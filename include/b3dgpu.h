/* C ABI of libb3dgpu.so: the B200 (sm_100a) kernels of blocks_3d's drop-in hot path.
 *
 * Numbers are multiprecision floats stored as limb planes: element i of an array with plane stride P has
 * limbs m[k * P + i] (k = 0 .. L-1, 32-bit two's complement, limb 0 least significant) and exponent e[i];
 * its value is m * 2^e.  Normalised values have |m| of exactly 32 L - 2 bits; zero is m = 0 with
 * e = B3D_EZ.  All pointers are device pointers owned by the caller (PyTorch tensors on the host side);
 * index arrays are int64.  `stream` is a cudaStream_t (NULL: the legacy default stream).  Every function
 * returns 0 on success, B3D_E_LIMBS for a limb count without compiled kernels, B3D_E_ARG for invalid
 * sizes, or a positive cudaError_t; b3d_last_error() describes the last failure of the calling thread.
 * Nothing here allocates device memory.
 */
#ifndef B3DGPU_H
#define B3DGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define B3D_EZ (-(((int64_t)1) << 60))
#define B3D_E_LIMBS (-1)
#define B3D_E_ARG (-2)

/* library version (major * 10000 + minor * 100 + patch) */
int b3d_version(void);

/* description of the last failure of the calling thread ("" if none) */
const char* b3d_last_error(void);

/* 1 if kernels are compiled for L limbs, else 0 */
int b3d_supported_limbs(int L);

/* Exponent alignment, the first half of sdpvibe's mpf.gemm / mpf._align_rows as called by the reference
 * (recursion_gpu.py:53-70, smallgemm.py:154-175): for each (batch b, row r) of the strided view
 * X[b, r, k] = element (bidx ? bidx[b] : b) * sb + r * sr + k * sk (k < K), write the mantissas shifted to
 * the row's largest exponent (truncated below it) to om at (b * R + r) * K + k, or (b * K + k) * R + r
 * when kmajor != 0, and the row exponents to oe[b * R + r]. */
int b3d_align(int L, const int32_t* m, const int64_t* e, int64_t plane, int64_t nbatch, int64_t R, int64_t K,
              int64_t sb, int64_t sr, int64_t sk, const int64_t* bidx, int32_t* om, int64_t* oe, int64_t oplane,
              int kmajor, void* stream);

/* Batched multiprecision GEMM on aligned operands, the second half of mpf.gemm (reference
 * recursion_gpu.py:53 gemm, :73 bgemm; smallgemm.py:18-56): C[b, i, j] = sum_k A[b, i, k] B[b, k, j] with
 * A = (am (b, M, K) row-aligned, ae (b, M)) and B = (bm (b, K, N) column-aligned, be (b, N)); exact
 * products and sums, one rounding; C contiguous (b, M, N). */
int b3d_gemm_aligned(int L, const int32_t* am, const int64_t* ae, int64_t aplane, const int32_t* bm,
                     const int64_t* be, int64_t bplane, int64_t nbatch, int64_t M, int64_t N, int64_t K,
                     int32_t* cm, int64_t* ce, int64_t cplane, void* stream);

/* Elementwise C[i] = A[aidx ? aidx[i] : i] * B[bidx ? bidx[i] : i] (mpf.mul: exact product, one rounding;
 * reference recursion_gpu.py:435, derivatives.py:496, :572) */
int b3d_mul(int L, const int32_t* am, const int64_t* ae, int64_t aplane, const int64_t* aidx,
            const int32_t* bm, const int64_t* be, int64_t bplane, const int64_t* bidx, int64_t n,
            int32_t* cm, int64_t* ce, int64_t cplane, void* stream);

/* Elementwise C[i] = A[..] + B[..] (mpf.add: one rounding; reference recursion_gpu.py:457, derivatives.py:573) */
int b3d_add(int L, const int32_t* am, const int64_t* ae, int64_t aplane, const int64_t* aidx,
            const int32_t* bm, const int64_t* be, int64_t bplane, const int64_t* bidx, int64_t n,
            int32_t* cm, int64_t* ce, int64_t cplane, void* stream);

/* Per-level tables of the Cauchy step (reference recursion_gpu.py:242-245 level dict, :368-376 tables) */
typedef struct b3d_level_tables {
    int64_t m, nb, Mr, Kc, N;      /* level, groups, rows per group, columns per group, S^2 B */
    int64_t hlevels, Jh;           /* h_inf layout (2, hlevels, Jh, N) */
    const int64_t* gsrc;           /* (nb) */
    const int64_t* gj;             /* (nb) */
    const int64_t* rowd;           /* (nb, Mr) 2 D' */
    const int64_t* nrow;           /* (nb) */
    const int64_t* cold;           /* (nb, Kc) 2 D_i */
    const int64_t* ncol;           /* (nb) */
    const int64_t* col;            /* (nb, Kc) physical slots */
} b3d_level_tables;

/* Cauchy step of one recursion level fused with the h_inf term (replaces cauchy.cauchy, cauchy.py:73-87,
 * and recursion_gpu.py:451-460 + mpf.add): H[g, r, n] = hinf[gsrc[g], m, gj[g], n]
 * + sum_i 2 / (rowd[g, r] - cold[g, i]) res[col[g, i], n].  res: (nslots, N), hinf: (2, hlevels, Jh, N),
 * H: (nb, Mr, N).  |rowd - cold| must be < 65536. */
int b3d_cauchy_level(int L, const int32_t* rm, const int64_t* re, int64_t rplane, const int32_t* hm,
                     const int64_t* he, int64_t hplane, const b3d_level_tables* lv, int32_t* om, int64_t* oe,
                     int64_t oplane, void* stream);

/* Pole step of one recursion level (replaces Recursion._pole with pole="cuda", recursion_gpu.py:483-492,
 * and the slot scatter :471-472): for each task t, res[t_slot[t]] = QL[t_qL[t]] (H[t_hrow[t]] R[t_R[t]]^T)
 * with H: (rows, S, S, B), Rtab / QLtab: (n, S, S) row-aligned with row exponents (n, S) (b3d_align),
 * scratch Y: (T, S, S, B), res: (nslots, S, S, B). */
int b3d_pole_level(int L, const int32_t* hm, const int64_t* he, int64_t hplane, const int32_t* Rm,
                   const int64_t* Re, int64_t Rplane, const int32_t* Qm, const int64_t* Qe, int64_t Qplane,
                   const int64_t* t_hrow, const int64_t* t_R, const int64_t* t_qL, const int64_t* t_slot,
                   int64_t T, int64_t B, int S, int32_t* ym, int64_t* ye, int64_t yplane, int32_t* rm,
                   int64_t* re, int64_t rplane, void* stream);

/* The same pole step with its exact sums on the INT8 tensor cores (replaces Recursion._pole with
 * pole="gemm", recursion_gpu.py:494-498, and the small GEMMs of smallgemm.py:18-88): per task and row of the
 * constant, one tcgen05 GEMM of balanced base-256 digits (a Hankel matrix of the constant's digits against the
 * reversed digits of the aligned columns), carry chain and one rounding; bit-identical to b3d_pole_level.
 * S <= 8.  err: a device int set nonzero if a bounded wait of the kernel expired (results then incomplete). */
int b3d_pole_level_mma(int L, const int32_t* hm, const int64_t* he, int64_t hplane, const int32_t* Rm,
                       const int64_t* Re, int64_t Rplane, const int32_t* Qm, const int64_t* Qe, int64_t Qplane,
                       const int64_t* t_hrow, const int64_t* t_R, const int64_t* t_qL, const int64_t* t_slot,
                       int64_t T, int64_t B, int S, int32_t* ym, int64_t* ye, int64_t yplane, int32_t* rm,
                       int64_t* re, int64_t rplane, int* err, void* stream);

/* Derivative moments of one recursion level (replaces Derivs.accumulate + momacc, derivatives.py:48-96,
 * :486-510): for each entry q and column c, y = res[q_slot[q], c] * rcpow[q_n[q]] and
 * mom[q_row[q], k, c] += q_n[q]^k y for k < R1.  res: (nslots, N), rcpow: (order + 1), mom: (rows, R1, N). */
int b3d_moments_level(int L, const int32_t* rm, const int64_t* re, int64_t rplane, const int32_t* pm,
                      const int64_t* pe, int64_t pplane, const int64_t* q_slot, const int64_t* q_row,
                      const int64_t* q_n, int64_t Q, int64_t N, int R1, int32_t* mm, int64_t* me, int64_t mplane,
                      void* stream);

/* Staged derivative moments (replaces the per-level momacc and the windowed momflush + mpadd of the reference,
 * derivatives.py:48-188, :474-510).  Stage, once per level m of a window starting at m0 (w = m - m0): for each
 * entry q and column c, Y[(w * rows + q_row[q]) * N + c] = res[q_slot[q], c] * rcpow[q_n[q]] (one rounding);
 * Y exponents the level does not write must be B3D_EZ (the caller clears them per window). */
int b3d_moments_stage(int L, const int32_t* rm, const int64_t* re, int64_t rplane, const int32_t* pm,
                      const int64_t* pe, int64_t pplane, const int64_t* q_slot, const int64_t* q_row,
                      const int64_t* q_n, int64_t Q, int64_t N, int64_t w, int64_t rows, int32_t* ym, int64_t* ye,
                      int64_t yplane, void* stream);

/* Flush a window of W staged levels: mom[(row * R1 + k) * N + c] = (mom +) round(sum_w n^k Y[w, row, c]) with
 * n = m0 + w + row_shift[row] (< NN), the sum exact above 2^-(32 Lout + 64) of its largest term, one rounding (and one
 * for the addition when accumulate != 0); Y has L limbs, the moments Lout = L or L + 4.  nk: n^k as KW 32-bit
 * limbs, nk[(k * NN + n) * KW + j]; nkb[k * NN + n]
 * its bit length.  R1 <= 32, KW <= 12. */
int b3d_moments_flush(int L, const int32_t* ym, const int64_t* ye, int64_t yplane, const int64_t* row_shift, int64_t m0,
                      int W, int64_t rows, int64_t N, int R1, const uint32_t* nk, const int32_t* nkb, int NN, int KW,
                      int accumulate, int Lout, int32_t* mm, int64_t* me, int64_t mplane, void* stream);

/* Change of limb count of n numbers, Lout = L or L +- 4: widening is exact, narrowing rounds once (half away from
 * zero).  The derivative stages run with more limbs than the recursion where their sums cancel (the drop-in's
 * choice; no counterpart in the reference, whose stages share one limb count). */
int b3d_resize(int L, const int32_t* m, const int64_t* e, int64_t plane, int64_t n, int Lout, int32_t* om, int64_t* oe,
               int64_t oplane, void* stream);

/* ---- residue-number-system GEMM on the INT8 tensor cores (tcgen05), the replacement of the reference's
 * un-vendored sdpvibe mpf.gemm (RNS / INT8; called at recursion_gpu.py:53-79, derivatives.py:540-580,
 * output.py:189,211).  Exact products, one rounding: bit-identical to b3d_gemm_aligned. */

/* per-limb-count constant tables (device pointers; built by blocksvibe_b200/rns.py) */
typedef struct b3d_rns_tables {
    const uint32_t* p;       /* (np) primes, 2^30 < p < 2^31 */
    const uint64_t* mu;      /* (np) floor(2^62 / p) */
    const uint32_t* w;       /* (np, 8) 2^(8u) mod p */
    const uint32_t* conv;    /* (np, L) 2^(32k) mod p */
    const uint32_t* inv;     /* (np) (M / p)^-1 mod p */
    const uint32_t* mj;      /* (np, ml) M / p, 32-bit limbs */
    const uint32_t* mfull;   /* (ml) M */
    int np, ml;
    uint64_t mtop;           /* floor(M / 2^(32 msw)): the CRT quotient's integer estimate */
    int msw;                 /* word offset: 32 msw >= bitlen(M) - 56 (so M / 2^(32 msw) >= 2^23) */
} b3d_rns_tables;

/* primes and limbs of M the kernels for L limbs expect (K <= 4096) */
int b3d_rns_layout(int L, int* np, int* ml);

/* aligned operand (b3d_align output, element b * sb + r * sr + k * sk) -> int8 digit matrices of its residues,
 * K-major UMMA core-matrix layout, tiles of TR digit rows, (np, nb, mat_bytes); rows padded to Rp, K to Kp */
int b3d_rns_split(int L, const int32_t* m, int64_t plane, int64_t nb, int64_t R, int64_t K, int64_t sb, int64_t sr,
                  int64_t sk, int64_t Rp, int64_t Kp, int TR, const b3d_rns_tables* tb, uint8_t* out,
                  int64_t mat_bytes, void* stream);

/* the same digit matrices computed on the tensor cores: magnitude bytes x the constant C (2 NS x Ks) */
typedef struct b3d_rns_split_args {
    const int32_t* m;
    int64_t plane, nb, R, K, sb, sr, sk;
    int64_t Rp, Kp;
    int TR;
    int64_t mat_bytes;
    uint8_t* out;
    const uint8_t* C;
    int Ks, NS;
    int* err;
} b3d_rns_split_args;

int b3d_rns_split_mma(int L, const b3d_rns_split_args* args, const b3d_rns_tables* tb, void* stream);

typedef struct b3d_rns_mma_args {
    const uint8_t* X;        /* lane-side digit matrices (tiles of 128 digit rows) */
    const uint8_t* Y;        /* column-side digit matrices (tiles of TN digit rows) */
    int64_t x_mat, y_mat;    /* bytes per (prime, batch) matrix */
    int64_t nb, NI, NL;      /* batch, operand rows of X and of Y */
    int Kp, TN;              /* padded K (multiple of 32, <= 256), column tile (multiple of 16, <= 256) */
    int64_t tiles_l;         /* column tiles */
    int64_t out_b, out_i, out_l;   /* residue output strides (elements) */
    uint32_t* out;           /* (np, nb, ...) residues, when yb is NULL */
    int* err;                /* device error flag, 0 = ok */
    uint8_t* yb;             /* else: y_j = r_j (M/p_j)^-1 mod p_j bytes, row e, column 4 j, of the CRT operand */
    int64_t crt_kp;          /* bytes per row of the CRT operand (multiple of 32) */
} b3d_rns_mma_args;

/* residues of X Y^T per prime with tcgen05.mma.kind::i8 (TMEM accumulators, bulk async copies) */
int b3d_rns_mma(const b3d_rns_mma_args* args, const b3d_rns_tables* tb, void* stream);

/* CRT on the tensor cores: A = y bytes (b3d_rns_mma with yb), T = constant Toeplitz digits of M / p_j
 * (2 NH rows x Kc, built by blocksvibe_b200/rns.py), result rounded to an MPF like b3d_rns_crt */
typedef struct b3d_rns_crt_args {
    const uint8_t* A;
    const uint8_t* T;
    int Kc, NH;
    int64_t n, nbatch, M, N;
    const int64_t* ea;
    const int64_t* eb;
    int32_t* cm;
    int64_t* ce;
    int64_t cplane;
    int* err;
} b3d_rns_crt_args;

int b3d_rns_crt_mma(int L, const b3d_rns_crt_args* args, const b3d_rns_tables* tb, void* stream);

/* CRT reconstruction of (np, n) residues, element e = (b * M + i) * N + l, rounded with exponents
 * ea[b * M + i] + eb[b * N + l] -> normalised MPF C (n) */
int b3d_rns_crt(int L, const uint32_t* res, int64_t n, const int64_t* ea, const int64_t* eb, int64_t nbatch,
                int64_t M, int64_t N, const b3d_rns_tables* tb, int32_t* cm, int64_t* ce, int64_t cplane,
                void* stream);

/* ---- the Cauchy step as an RNS GEMM on the tensor cores (the reference's "rns" Cauchy variant,
 * recursion_gpu.py:456-460: C = +-2/k gathered from a table, bgemm(C, X)); per group g:
 * H_raw[g] = C[g] X[g] with C[g][r][i] = round(2^(NB-1) / (rowd[g][r] - cold[g][i])) (fixed exponent 1 - NB),
 * X[g][i][n] = res[col[g][i]][n] aligned per column. */

/* X (nb, Kc, N) aligned per column (g, n) and its column exponents (nb, N) */
int b3d_cauchy_align(int L, const int32_t* rm, const int64_t* re, int64_t rplane, const b3d_level_tables* lv,
                     int32_t* om, int64_t* oe, int64_t oplane, void* stream);

/* the Cauchy step of b3d_cauchy_level from X already aligned (b3d_cauchy_align): per-limb 64-bit accumulation
 * of the one-limb quotients, two terms per thread, one rounding, plus the h_inf term (the CUDA-core form) */
int b3d_cauchy_level2(int L, const int32_t* xm, const int64_t* xe, int64_t xplane, const int32_t* hm,
                      const int64_t* he, int64_t hplane, const b3d_level_tables* lv, int32_t* om, int64_t* oe,
                      int64_t oplane, void* stream);

/* b3d_cauchy_level2 with wide quotient digits: the caller guarantees that every divisor |rowd - cold| of the
 * level is at most dmax (the plan's maximum, < 2^16); with dmax < 2^8 (2^10) each multiply-high step of the
 * one-limb division yields 24 (22) quotient bits instead of 16.  Results bit-identical to b3d_cauchy_level2. */
int b3d_cauchy_level3(int L, const int32_t* xm, const int64_t* xe, int64_t xplane, const int32_t* hm,
                      const int64_t* he, int64_t hplane, const b3d_level_tables* lv, int64_t dmax, int32_t* om,
                      int64_t* oe, int64_t oplane, void* stream);

/* b3d_cauchy_align with sign-magnitude output (|x| aligned, its sign in bit 31 of limb L - 1): the input of
 * b3d_cauchy_level4 */
int b3d_cauchy_align_sm(int L, const int32_t* rm, const int64_t* re, int64_t rplane, const b3d_level_tables* lv,
                        int32_t* om, int64_t* oe, int64_t oplane, void* stream);

/* b3d_cauchy_level3 on the sign-magnitude columns of b3d_cauchy_align_sm, each column's limbs read from memory
 * as the division reaches them (fewer registers per thread); results bit-identical to b3d_cauchy_level3
 * (replaces cauchy.cauchy, cauchy.py:73-87, like it) */
int b3d_cauchy_level4(int L, const int32_t* xm, const int64_t* xe, int64_t xplane, const int32_t* hm,
                      const int64_t* he, int64_t hplane, const b3d_level_tables* lv, int64_t dmax, int32_t* om,
                      int64_t* oe, int64_t oplane, void* stream);

/* digit matrices of C (as b3d_rns_split writes them) from table[(d + dmax) * np + j] = residues of
 * round(2^(NB-1) / d) */
int b3d_cauchy_digits(const b3d_level_tables* lv, const uint32_t* table, int64_t dmax, int np, int64_t Rp, int64_t Kp,
                      int TR, int64_t mat_bytes, uint8_t* out, void* stream);

/* H = H_raw + h_inf rows of the level (one rounding); padded rows written as zero */
int b3d_cauchy_add_hinf(int L, const int32_t* am, const int64_t* ae, int64_t aplane, const int32_t* hm,
                        const int64_t* he, int64_t hplane, const b3d_level_tables* lv, int32_t* om, int64_t* oe,
                        int64_t oplane, void* stream);

/* Size of the device scratch array of b3d_pole_level_noalloc: reserved on a GPU once the library's module is
 * loaded there (with lazy module loading, no later than the first b3d_pole_level_noalloc call on that GPU) and
 * held until the process exits. */
#define B3D_NOALLOC_SCRATCH_BYTES ((size_t)16 << 20)

/* b3d_pole_level without a caller-provided scratch buffer (no counterpart in the reference: an addition for
 * callers that cannot allocate device memory while they run, e.g. when another allocator owns the device
 * memory or a serving loop budgets it per request).  Same arguments and results as b3d_pole_level minus
 * ym / ye / yplane; the intermediate lives in a fixed array of B3D_NOALLOC_SCRATCH_BYTES, so a call needs
 * T * S^2 * B * (4 L + 8) <= B3D_NOALLOC_SCRATCH_BYTES - 256 bytes (else B3D_E_ARG: split the level's tasks).
 * Allocates nothing.  The array is resolved on the current device (make the stream's device current first); the
 * first call on each device looks its address up and caches it for the life of the process: make that call
 * before any stream capture, and do not call this entry point after a cudaDeviceReset of a device it ran on (the
 * cached address is then stale).  All calls on a device share the array: calls whose kernels overlap on the GPU
 * race. */
int b3d_pole_level_noalloc(int L, const int32_t* hm, const int64_t* he, int64_t hplane, const int32_t* Rm,
                           const int64_t* Re, int64_t Rplane, const int32_t* Qm, const int64_t* Qe, int64_t Qplane,
                           const int64_t* t_hrow, const int64_t* t_R, const int64_t* t_qL, const int64_t* t_slot,
                           int64_t T, int64_t B, int S, int32_t* rm, int64_t* re, int64_t rplane, void* stream);

/* ---- Index plan of the recursion (host memory; replaces the reference's recursion_gpu.Plan,
 *      recursion_gpu.py:136-365, whose tensors it reproduces: logical slots (m, spin, pole) with parity p adding
 *      p * nslots, per level the Cauchy groups (src, tj') with their rows D' and columns, per pole-step task its
 *      slot, H row and keys, every numbering by first appearance, and LIFO slot recycling) ---- */

typedef struct b3d_plan b3d_plan;

/* number of int64 written by b3d_plan_scalars: Smax, Jh, nslots, nphys, zero_slot, dmax, order, number of M keys,
 * of Q keys, of (L, Q) pairs, of (level, spin) layout entries */
#define B3D_PLAN_NSCALARS 11

/* Per-level arrays copied out by b3d_plan_level (int64, any pointer may be NULL to skip it).  With dims
 * (nb, Mr, Kc, T) from b3d_plan_level_dims: gsrc, gj, nrow, ncol (nb); rowd (nb, Mr); col, cold (nb, Kc); per
 * task (T): t_slot (physical), t_hrow (group * Mr + row), t_L / t_R (M key ids), t_q (Q key id), t_qL ((L, Q)
 * pair id), t_p (parity), t_tj (doubled spin), t_kind / t_k (pole). */
typedef struct b3d_plan_level_arrays {
    int64_t *gsrc, *gj, *col, *rowd, *nrow, *cold, *ncol;
    int64_t *t_slot, *t_hrow, *t_L, *t_R, *t_q, *t_qL, *t_p, *t_tj, *t_kind, *t_k;
} b3d_plan_level_arrays;

/* Build the plan of (two_j12, two_j43, two_j_max, order, pseudo_parities[2][2] as 4 int64), with slot recycling
 * when reuse != 0 (reference Plan(..., reuse)).  *out is released with b3d_plan_destroy. */
int b3d_plan_build(int64_t two_j12, int64_t two_j43, int64_t two_j_max, int64_t order, const int64_t* pseudo_parities,
                   int reuse, b3d_plan** out);
void b3d_plan_destroy(b3d_plan* plan);
/* B3D_PLAN_NSCALARS values (above) */
int b3d_plan_scalars(const b3d_plan* plan, int64_t* scalars);
/* mkeys (nM, 5): kind, k, side (0 = L, 1 = R), pseudo-parity, two_j; qkeys (nQ, 4): kind, k, two_j, sign;
 * lqpairs (nLQ, 2): M key id, Q key id; row i = id i (reference Plan.Mkeys / Qkeys / LQpairs) */
int b3d_plan_keys(const b3d_plan* plan, int64_t* mkeys, int64_t* qkeys, int64_t* lqpairs);
/* start (order) and first (layout entries): first logical slot of (m, spin index j) = first[start[m] + j];
 * phys (2 nslots): physical slot of each logical one, -1 where never written */
int b3d_plan_layout(const b3d_plan* plan, int64_t* start, int64_t* first, int64_t* phys);
/* dims[4] = nb, Mr, Kc, T of level m (nb = 0: no task at that level) */
int b3d_plan_level_dims(const b3d_plan* plan, int64_t m, int64_t* dims);
int b3d_plan_level(const b3d_plan* plan, int64_t m, const b3d_plan_level_arrays* arrays);

/* ---- b3d_setup's file (csrc/b3d_setup.cxx:15-21 layout, read by the reference's setup.read, setup.py:128-161) ---- */

/* Host memory.  n numbers of the file, records rec[i * (2 + K) ...] = [size, exp, limb_0 .. limb_{K-1}] (GMP mpf:
 * 64-bit limbs, value sign(size) * sum_t limb_t 2^(64 t) * 2^(64 (exp - K))), rounded once to L limbs (half away
 * from zero): limbs m[k * plane + i], exponents e[i] (B3D_EZ for zero).  Replaces setup.numbers_to_mpf
 * (setup.py:52-74). */
int b3d_setup_numbers(const int64_t* rec, int64_t n, int K, int L, int32_t* m, int64_t plane, int64_t* e);

/* ---- blocks_3d's JSON output (reference blocksvibe/b3djson.py, called from cli._write_one, cli.py:471-490) ---- */

/* Tables of the decimal formatter, built once per (L, p) by the caller: pow5 = 5^k for k = 0 .. kmax as rows of
 * fw limbs (pow5_limbs[k] = limbs in use), bounds = 10^(p-1) and 10^p as two rows of L - 1 limbs; p = digits;
 * stride = bytes per output slot (multiple of 16, p + 12 .. 416).  kmax = 3 p covers |v| >= 10^(-2p-1). */
typedef struct b3d_decimal_tables {
    const uint32_t* pow5;
    const int32_t* pow5_limbs;
    const uint32_t* bounds;
    int kmax, fw, p, stride;
} b3d_decimal_tables;

/* Number i (m, e limb planes) printed as blocks_3d's writer prints it (b3djson.fmt_gmpy + limbs_to_mpfr,
 * b3djson.py:56-80: MPFR "%.{p}g" of the exact value, ties to even) into out[i * stride ...], its length in
 * len[i].  err: two int64 set by the caller to {0, INT64_MAX}; numbers outside the supported decimal range
 * (|v| < 10^(-2p-1), or far above 10^p) get len -1, add 1 to err[0] and lower err[1] to their index.
 * out must be 16-byte aligned. */
int b3d_format_decimal(int L, const int32_t* m, const int64_t* e, int64_t plane, int64_t n,
                       const b3d_decimal_tables* tb, char* out, int32_t* len, int64_t* err, void* stream);

/* Per polynomial t (coefficients poly_num[t] + d, d < D, of the same m / e arrays): the kept size of
 * blocks_3d's truncation of negligible top coefficients (b3djson.py:160-166, eps = 2^-eps_shift; 0 when all
 * coefficients are zero) in size[t], and the byte length of its text (quoted numbers joined by ",\n", or
 * "0" in quotes) in text_len[t], -1 if a kept coefficient has length -1; len = the lengths from
 * b3d_format_decimal. */
int b3d_poly_sizes(int L, const int32_t* m, const int64_t* e, int64_t plane, const int64_t* poly_num, int64_t npoly,
                   int D, int eps_shift, const int32_t* len, int32_t* size, int64_t* text_len, void* stream);

/* Text assembly (b3djson.write_spin / derivs_text, b3djson.py:150-198): for each polynomial t, the skeleton
 * bytes skel[skel_off[t] .. skel_off[t+1]) and then its text (size[t] < 0: none) are written to
 * out[out_off[t] ...], out_off[t] = sum over t' < t of the skeleton plus text lengths. */
int b3d_emit_text(const char* slots, int stride, const int32_t* len, const int64_t* poly_num, const int32_t* size,
                  const int64_t* out_off, const char* skel, const int64_t* skel_off, int64_t npoly, char* out,
                  void* stream);

#ifdef __cplusplus
}
#endif

#endif /* B3DGPU_H */
