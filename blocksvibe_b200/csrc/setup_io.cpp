// Numbers of b3d_setup's B3DSETUP file (host C++): GMP mpf records [size exp limb_0 .. limb_{K-1}] (64-bit
// limbs, limb_{K-1} most significant, value = sign(size) * sum_t limb_t 2^(64 t) * 2^(64 (exp - K))) rounded
// once to the drop-in's multiprecision format: L 32-bit two's complement limb planes normalised to
// NB = 32 L - 2 bits (half away from zero on the magnitude, as every other conversion of the library), and an
// exponent (B3D_EZ for zero).  Replaces the reference's setup.numbers_to_mpf (setup.py:52-74), which did the
// same on the GPU with sdpvibe's normalize.
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "b3dgpu.h"

namespace b3d {
int fail(int code, const std::string& what);
}

namespace {

// magnitude as little-endian 32-bit words
int bit_length(const std::vector<uint32_t>& w) {
    for (int i = (int)w.size() - 1; i >= 0; --i)
        if (w[i]) return 32 * i + 32 - __builtin_clz(w[i]);
    return 0;
}

bool get_bit(const std::vector<uint32_t>& w, int64_t b) {
    return b >= 0 && b / 32 < (int64_t)w.size() && ((w[b / 32] >> (b % 32)) & 1u);
}

// w >> s (s >= 0) into n words
std::vector<uint32_t> shr(const std::vector<uint32_t>& w, int64_t s, int n) {
    std::vector<uint32_t> out(n, 0);
    const int64_t q = s / 32, r = s % 32;
    for (int i = 0; i < n; ++i) {
        const int64_t j = i + q;
        uint64_t lo = j < (int64_t)w.size() ? w[j] : 0, hi = j + 1 < (int64_t)w.size() ? w[j + 1] : 0;
        out[i] = (uint32_t)(((hi << 32) | lo) >> r);
    }
    return out;
}

// w << s (s >= 0) into n words
std::vector<uint32_t> shl(const std::vector<uint32_t>& w, int64_t s, int n) {
    std::vector<uint32_t> out(n, 0);
    const int64_t q = s / 32, r = s % 32;
    for (int i = 0; i < n; ++i) {
        const int64_t j = i - q;
        uint64_t lo = (j - 1 >= 0 && j - 1 < (int64_t)w.size()) ? w[j - 1] : 0;
        uint64_t hi = (j >= 0 && j < (int64_t)w.size()) ? w[j] : 0;
        out[i] = (uint32_t)((((hi << 32) | lo) << r) >> 32);
    }
    return out;
}

}  // namespace

extern "C" int b3d_setup_numbers(const int64_t* rec, int64_t n, int K, int L, int32_t* m, int64_t plane, int64_t* e) {
    if ((!rec && n) || n < 0 || K < 1 || L < 3 || plane < n || (n && (!m || !e)))
        return b3d::fail(B3D_E_ARG, "b3d_setup_numbers: invalid arguments");
    const int NB = 32 * L - 2;
    std::vector<uint32_t> w(2 * K);
    for (int64_t i = 0; i < n; ++i) {
        const int64_t* r = rec + i * (2 + K);
        const int64_t size = r[0], ex = r[1];
        std::memcpy(w.data(), r + 2, 8 * (size_t)K);
        const int bl = size == 0 ? 0 : bit_length(w);
        std::vector<uint32_t> a;
        int64_t s = bl - NB, exp2 = 64 * (ex - K);
        if (bl == 0) {
            for (int k = 0; k < L; ++k) m[k * plane + i] = 0;
            e[i] = B3D_EZ;
            continue;
        }
        if (s > 0) {
            a = shr(w, s, L);
            if (get_bit(w, s - 1)) {                      // round half away from zero
                for (int k = 0; k < L && ++a[k] == 0; ++k) {
                }
                if (bit_length(a) > NB) {
                    a = shr(a, 1, L);
                    ++s;
                }
            }
        } else {
            a = shl(w, -s, L);
        }
        if (size < 0) {                                   // two's complement of the magnitude
            uint64_t carry = 1;
            for (int k = 0; k < L; ++k) {
                const uint64_t v = (uint64_t)(uint32_t)~a[k] + carry;
                a[k] = (uint32_t)v;
                carry = v >> 32;
            }
        }
        for (int k = 0; k < L; ++k) m[k * plane + i] = (int32_t)a[k];
        e[i] = exp2 + s;
    }
    return 0;
}
