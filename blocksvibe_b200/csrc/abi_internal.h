// Shared by the C ABI translation units: error reporting and the dispatch on the limb count.
#pragma once
#include <string>

#include "kernels.cuh"
#include "rns.cuh"
#include "cauchy_rns.cuh"

namespace b3d {
#define B3D_DECL(L) extern template struct Launch<L>; extern template struct RnsLaunch<L>; extern template struct CauchyRnsLaunch<L>;
B3D_FOR_EACH_L(B3D_DECL)
#undef B3D_DECL

// record `what` as the calling thread's last error (b3d_last_error) and return `code`
int fail(int code, const std::string& what);
// 0 for cudaSuccess, else the error code with its message recorded
int cuda_status(int code, const char* fn);
// tensor-core residue product and the Cauchy coefficient digits (rns_mma.cu)
int rns_mma_launch(const RnsMma& a, const RnsTables& tb, cudaStream_t st);
int cauchy_digits_launch(const CauchyLevel& lv, const uint32_t* table, int64_t dmax, int np, int64_t Rp, int64_t Kp,
                         int TR, int64_t mat_bytes, uint8_t* out, cudaStream_t st);
}  // namespace b3d

#define B3D_DISPATCH_RNS(L, CALL)                                              \
    switch (L) {                                                               \
        case 6: { using RX = b3d::RnsLaunch<6>; return CALL; }                 \
        case 10: { using RX = b3d::RnsLaunch<10>; return CALL; }               \
        case 18: { using RX = b3d::RnsLaunch<18>; return CALL; }               \
        case 26: { using RX = b3d::RnsLaunch<26>; return CALL; }               \
        case 30: { using RX = b3d::RnsLaunch<30>; return CALL; }               \
        case 34: { using RX = b3d::RnsLaunch<34>; return CALL; }               \
        case 14: { using RX = b3d::RnsLaunch<14>; return CALL; }\
        case 22: { using RX = b3d::RnsLaunch<22>; return CALL; }\
        case 38: { using RX = b3d::RnsLaunch<38>; return CALL; }\
        case 46: { using RX = b3d::RnsLaunch<46>; return CALL; }\
        case 42: { using RX = b3d::RnsLaunch<42>; return CALL; }               \
        default: return b3d::fail(B3D_E_LIMBS, "no kernels compiled for L = " + std::to_string(L)); \
    }

#define B3D_DISPATCH_CAUCHY(L, CALL)                                           \
    switch (L) {                                                               \
        case 6: { using CX = b3d::CauchyRnsLaunch<6>; return CALL; }           \
        case 10: { using CX = b3d::CauchyRnsLaunch<10>; return CALL; }         \
        case 18: { using CX = b3d::CauchyRnsLaunch<18>; return CALL; }         \
        case 26: { using CX = b3d::CauchyRnsLaunch<26>; return CALL; }         \
        case 30: { using CX = b3d::CauchyRnsLaunch<30>; return CALL; }         \
        case 34: { using CX = b3d::CauchyRnsLaunch<34>; return CALL; }         \
        case 14: { using CX = b3d::CauchyRnsLaunch<14>; return CALL; }\
        case 22: { using CX = b3d::CauchyRnsLaunch<22>; return CALL; }\
        case 38: { using CX = b3d::CauchyRnsLaunch<38>; return CALL; }\
        case 46: { using CX = b3d::CauchyRnsLaunch<46>; return CALL; }\
        case 42: { using CX = b3d::CauchyRnsLaunch<42>; return CALL; }         \
        default: return b3d::fail(B3D_E_LIMBS, "no kernels compiled for L = " + std::to_string(L)); \
    }

#define B3D_DISPATCH(L, CALL)                                                  \
    switch (L) {                                                               \
        case 6: { using LX = b3d::Launch<6>; return CALL; }                    \
        case 10: { using LX = b3d::Launch<10>; return CALL; }                  \
        case 18: { using LX = b3d::Launch<18>; return CALL; }                  \
        case 26: { using LX = b3d::Launch<26>; return CALL; }                  \
        case 30: { using LX = b3d::Launch<30>; return CALL; }                  \
        case 34: { using LX = b3d::Launch<34>; return CALL; }                  \
        case 14: { using LX = b3d::Launch<14>; return CALL; }\
        case 22: { using LX = b3d::Launch<22>; return CALL; }\
        case 38: { using LX = b3d::Launch<38>; return CALL; }\
        case 46: { using LX = b3d::Launch<46>; return CALL; }\
        case 42: { using LX = b3d::Launch<42>; return CALL; }                  \
        default: return b3d::fail(B3D_E_LIMBS, "no kernels compiled for L = " + std::to_string(L)); \
    }
