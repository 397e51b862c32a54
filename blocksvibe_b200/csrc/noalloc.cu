// b3d_pole_level_noalloc: the pole step of one recursion level with its scratch in a fixed device array
// of this library instead of a caller-provided buffer.
//
// Who needs it: callers that cannot allocate device memory at the point where they run a level.  Examples
// are a host program whose whole device memory is owned by another allocator (a PyTorch caching allocator, or
// a serving loop that budgets HBM per request and admits work only inside that budget), and a caller that
// must not trigger cudaMalloc's implicit device-wide synchronisation in the middle of its work.  Such a
// caller still owns and passes every input and output; only the intermediate product H R^T lives here.
//
// Limits and sharing rules:
//  * the scratch is B3D_NOALLOC_SCRATCH_BYTES (16 MiB) of device memory, reserved on a device once this
//    library's module is loaded there (with CUDA's lazy module loading, no later than the first call of this
//    entry point on that device) and held until the process exits; a level needs T * S^2 * B * (4 L + 8)
//    bytes (L-limb numbers and their exponents) and at most B3D_NOALLOC_SCRATCH_BYTES - 256 of them, larger
//    requests are rejected with B3D_E_ARG and a message (split the level's tasks into chunks that fit);
//  * every call on a device uses the same array, which keeps the last call's contents.  Nothing has to
//    start at zero: the first kernel writes every scratch element the second kernel reads.  Calls whose
//    kernels overlap on the GPU (different streams, or several host threads) race on the array: serialise
//    them (one stream, or events);
//  * the array is resolved on the CURRENT device (cudaGetDevice), not on the stream's: make the stream's device
//    current before calling.  The first call on each device looks up the array's device address
//    (cudaGetSymbolAddress) and caches it for the life of the process; make that first call before any stream
//    capture begins.  A cudaDeviceReset (or any other teardown of the primary context) invalidates the cached
//    address, and later calls in the same process would write through it: do not use this entry point in a
//    process after resetting a device it has run on.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "abi_internal.h"
#include "b3dgpu.h"

namespace {

constexpr size_t kScratchBytes = B3D_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_pole_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

// device address of g_pole_scratch on the current device (looked up once per device)
int scratch_address(void** out) {
    int dev = -1;
    int rc = (int)cudaGetDevice(&dev);
    if (rc) return b3d::cuda_status(rc, "b3d_pole_level_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return b3d::fail(B3D_E_ARG, "b3d_pole_level_noalloc: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        rc = (int)cudaGetSymbolAddress(&p, g_pole_scratch);
        if (rc) return b3d::cuda_status(rc, "b3d_pole_level_noalloc: cudaGetSymbolAddress");
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return 0;
}

}  // namespace

extern "C" int b3d_pole_level_noalloc(int L, const int32_t* hm, const int64_t* he, int64_t hplane,
                                      const int32_t* Rm, const int64_t* Re, int64_t Rplane, const int32_t* Qm,
                                      const int64_t* Qe, int64_t Qplane, const int64_t* t_hrow, const int64_t* t_R,
                                      const int64_t* t_qL, const int64_t* t_slot, int64_t T, int64_t B, int S,
                                      int32_t* rm, int64_t* re, int64_t rplane, void* stream) {
    if (T < 0 || B < 1 || S < 1 || S > 64 || L < 1 || L > 64)
        return b3d::fail(B3D_E_ARG, "b3d_pole_level_noalloc: invalid size");
    if (!b3d_supported_limbs(L))
        return b3d::fail(B3D_E_LIMBS, "no kernels compiled for L = " + std::to_string(L));
    if (T == 0) return 0;
    // scratch bytes T * S^2 * B * (4 L + 8), checked factor by factor so that no product can overflow
    const uint64_t num_bytes = 4u * (uint64_t)L + 8u;
    const uint64_t usable = kScratchBytes - 256;                  // room for aligning the exponent block
    const uint64_t row_bytes = (uint64_t)S * (uint64_t)S * num_bytes;          // <= 64 * 64 * 264
    if ((uint64_t)B > usable / row_bytes)
        return b3d::fail(B3D_E_ARG, "b3d_pole_level_noalloc: B = " + std::to_string(B) + " right-hand sides exceed the " +
                                        std::to_string(kScratchBytes >> 20) + " MiB scratch even for one task");
    const uint64_t per = (uint64_t)S * (uint64_t)S * (uint64_t)B;              // per * num_bytes <= usable
    if ((uint64_t)T > usable / (per * num_bytes))
        return b3d::fail(B3D_E_ARG, "b3d_pole_level_noalloc: " + std::to_string(T) + " tasks x " + std::to_string(per) +
                                        " numbers of " + std::to_string(num_bytes) + " bytes exceed the " +
                                        std::to_string(kScratchBytes >> 20) + " MiB scratch; split the level");
    const int64_t n = T * (int64_t)per;
    void* base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;
    int32_t* ym = static_cast<int32_t*>(base);
    const size_t limb_bytes = ((size_t)4 * L * n + 255) & ~(size_t)255;       // exponents on a 256-byte boundary
    int64_t* ye = reinterpret_cast<int64_t*>(static_cast<unsigned char*>(base) + limb_bytes);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    B3D_DISPATCH(L, b3d::cuda_status(LX::pole(hm, he, hplane, Rm, Re, Rplane, Qm, Qe, Qplane, t_hrow, t_R, t_qL, t_slot,
                                              T, B, S, ym, ye, n, rm, re, rplane, st),
                                     "b3d_pole_level_noalloc"));
}
