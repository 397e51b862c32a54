// C ABI of the decimal formatter and the JSON text assembly (decimal.cuh), and the text-assembly kernel.
#include <string>

#include "../../include/b3dgpu.h"
#include "abi_internal.h"
#include "decimal.cuh"

namespace b3d {
#define B3D_DECL_DEC(L) extern template struct DecimalLaunch<L>;
B3D_FOR_EACH_L(B3D_DECL_DEC)
#undef B3D_DECL_DEC

// one warp per polynomial: its skeleton bytes, then its quoted numbers joined by ",\n" ("0" in quotes
// when all are zero, nothing when size < 0) -- b3djson.py:155-167 for the numbers, the skeleton holds
// everything else of b3djson.py:97-198
__global__ void k_emit_text(const char* __restrict__ slots, int stride, const int32_t* __restrict__ len,
                            const int64_t* __restrict__ poly_num, const int32_t* __restrict__ size,
                            const int64_t* __restrict__ out_off, const char* __restrict__ skel,
                            const int64_t* __restrict__ skel_off, int64_t npoly, char* __restrict__ out) {
    const int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= npoly) return;
    int64_t o = out_off[w];
    const int64_t s0 = skel_off[w], sn = skel_off[w + 1] - s0;
    for (int64_t j = lane; j < sn; j += 32) out[o + j] = skel[s0 + j];
    o += sn;
    const int sz = size[w];
    if (sz < 0) return;
    if (sz == 0) {
        if (lane < 3) out[o + lane] = lane == 1 ? '0' : '"';
        return;
    }
    const int64_t base = poly_num[w];
    for (int d = 0; d < sz; d++) {
        const int l = len[base + d];
        const char* src = slots + (base + d) * (int64_t)stride;
        if (lane == 0) out[o] = '"';
        for (int j = lane; j < l; j += 32) out[o + 1 + j] = src[j];
        o += 1 + l;
        if (d + 1 < sz) {
            if (lane < 3) out[o + lane] = lane == 0 ? '"' : (lane == 1 ? ',' : '\n');
            o += 3;
        } else {
            if (lane == 0) out[o] = '"';
            o += 1;
        }
    }
}
}  // namespace b3d

#define B3D_DISPATCH_DEC(L, CALL)                                              \
    switch (L) {                                                               \
        case 6: { using DX = b3d::DecimalLaunch<6>; return CALL; }             \
        case 10: { using DX = b3d::DecimalLaunch<10>; return CALL; }           \
        case 18: { using DX = b3d::DecimalLaunch<18>; return CALL; }           \
        case 26: { using DX = b3d::DecimalLaunch<26>; return CALL; }           \
        case 30: { using DX = b3d::DecimalLaunch<30>; return CALL; }           \
        case 34: { using DX = b3d::DecimalLaunch<34>; return CALL; }           \
        case 14: { using DX = b3d::DecimalLaunch<14>; return CALL; }\
        case 22: { using DX = b3d::DecimalLaunch<22>; return CALL; }\
        case 38: { using DX = b3d::DecimalLaunch<38>; return CALL; }\
        case 46: { using DX = b3d::DecimalLaunch<46>; return CALL; }\
        case 42: { using DX = b3d::DecimalLaunch<42>; return CALL; }           \
        default: return b3d::fail(B3D_E_LIMBS, "no kernels compiled for L = " + std::to_string(L)); \
    }

using b3d::cuda_status;
using b3d::fail;

static cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

extern "C" {

int b3d_format_decimal(int L, const int32_t* m, const int64_t* e, int64_t plane, int64_t n,
                       const b3d_decimal_tables* tb, char* out, int32_t* len, int64_t* err, void* stream) {
    if (!tb || n < 0 || plane < n || L < 3) return fail(B3D_E_ARG, "b3d_format_decimal: invalid sizes");
    if (tb->p < 1 || tb->p > b3d::dec_digits_max(L))
        return fail(B3D_E_ARG, "b3d_format_decimal: p = " + std::to_string(tb->p) + " digits exceed L = " +
                                   std::to_string(L) + " limbs");
    if (tb->stride % 16 || tb->stride < tb->p + 12 || tb->stride > 416)
        return fail(B3D_E_ARG, "b3d_format_decimal: stride must be a multiple of 16 in [p + 12, 416]");
    if (tb->kmax < 0 || tb->fw < 1 || L + tb->fw > b3d::dec_work(L))
        return fail(B3D_E_ARG, "b3d_format_decimal: power-of-5 table wider than the work array");
    if (reinterpret_cast<uintptr_t>(out) % 16) return fail(B3D_E_ARG, "b3d_format_decimal: out not 16-byte aligned");
    b3d::DecimalTables t{tb->pow5, tb->pow5_limbs, tb->bounds, tb->kmax, tb->fw, tb->p, tb->stride};
    B3D_DISPATCH_DEC(L, cuda_status(DX::format(m, e, plane, n, t, out, len, reinterpret_cast<long long*>(err),
                                               as_stream(stream)), "b3d_format_decimal"));
}

int b3d_poly_sizes(int L, const int32_t* m, const int64_t* e, int64_t plane, const int64_t* poly_num, int64_t npoly,
                   int D, int eps_shift, const int32_t* len, int32_t* size, int64_t* text_len, void* stream) {
    if (npoly < 0 || D < 1 || eps_shift < 0) return fail(B3D_E_ARG, "b3d_poly_sizes: invalid sizes");
    B3D_DISPATCH_DEC(L, cuda_status(DX::poly_sizes(m, e, plane, poly_num, npoly, D, eps_shift, len, size, text_len,
                                                   as_stream(stream)), "b3d_poly_sizes"));
}

int b3d_emit_text(const char* slots, int stride, const int32_t* len, const int64_t* poly_num, const int32_t* size,
                  const int64_t* out_off, const char* skel, const int64_t* skel_off, int64_t npoly, char* out,
                  void* stream) {
    if (npoly < 0 || stride < 1) return fail(B3D_E_ARG, "b3d_emit_text: invalid sizes");
    if (npoly == 0) return 0;
    const int64_t threads = 256, blocks = (npoly * 32 + threads - 1) / threads;
    b3d::k_emit_text<<<(unsigned)blocks, (unsigned)threads, 0, as_stream(stream)>>>(slots, stride, len, poly_num, size,
                                                                                   out_off, skel, skel_off, npoly, out);
    return cuda_status((int)cudaGetLastError(), "b3d_emit_text");
}

}  // extern "C"
