// One translation unit per limb count (compiled with -DB3D_L=<L>): instantiates the kernel launchers.
#define B3D_DEFINE_LAUNCH
#include "kernels.cuh"
#include "rns.cuh"
#include "cauchy_rns.cuh"
#include "decimal.cuh"
#include "pole_mma.cuh"

#ifndef B3D_L
#error "compile with -DB3D_L=<limbs>"
#endif

namespace b3d {
template struct Launch<B3D_L>;
template struct RnsLaunch<B3D_L>;
template struct CauchyRnsLaunch<B3D_L>;
template struct DecimalLaunch<B3D_L>;
}
