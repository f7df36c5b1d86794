// Device photon source for the height-field plate (sm_100a): per_texel photon entry points per
// texel, jittered uniformly inside the texel.
//
// Reference: the per-pixel random sampling of the surface in model/caustics.py:78-83
// (rand_like offsets of up to half a texel in each direction) and the per-simulation
// repetition of the reference's loop; there the offsets come from torch's generator on the
// host side of each simulation. Here they come from a counter-based generator, Philox4x32
// with 10 rounds (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as easy as 1, 2, 3",
// SC 2011): the offsets of photon i are a pure function of (seed, offset + i), so a batch of
// simulations draws disjoint streams by offset, with no generator state, no host round trip
// and no random-number buffer.
#include <cstdint>
#include <cuda_runtime.h>

#include "pds_internal.h"

namespace pds {
namespace {

// Philox4x32 constants of the paper: the round multipliers and the key's Weyl increments.
constexpr uint32_t kPhiloxM0 = 0xD2511F53u, kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u, kPhiloxW1 = 0xBB67AE85u;

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = kPhiloxM0 * c.x, hi0 = __umulhi(kPhiloxM0, c.x);
        const uint32_t lo1 = kPhiloxM1 * c.z, hi1 = __umulhi(kPhiloxM1, c.z);
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += kPhiloxW0;
        k1 += kPhiloxW1;
    }
    return c;
}

// [0, 1) from the top 24 bits: exact in float.
__device__ __forceinline__ float unit24(uint32_t u) { return float(u >> 8) * (1.f / 16777216.f); }

// Two photons per thread: one Philox block gives both photons' (x, y) offsets.
__global__ __launch_bounds__(256) void source_kernel(int32_t rows, int32_t cols,
                                                     int32_t per_texel, float texel,
                                                     uint64_t seed, uint64_t offset, int64_t n,
                                                     float* __restrict__ px,
                                                     float* __restrict__ py) {
    const int64_t pairs = (n + 1) >> 1;
    const float cx = 0.5f * float(cols - 1), cy = 0.5f * float(rows - 1);
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < pairs;
         k += int64_t(gridDim.x) * blockDim.x) {
        // Philox block (offset + k) as a 64-bit counter over the first two words
        const uint64_t ctr = offset + uint64_t(k);
        const uint4 r = philox4x32_10(make_uint4(uint32_t(ctr), uint32_t(ctr >> 32), 0u, 0u),
                                      uint32_t(seed), uint32_t(seed >> 32));
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int64_t i = 2 * k + h;
            if (i >= n) break;
            const int64_t t = i / per_texel;
            const float iy = float(t / cols), ix = float(t % cols);
            const float jx = unit24(h ? r.z : r.x) - 0.5f, jy = unit24(h ? r.w : r.y) - 0.5f;
            px[i] = (ix + jx - cx) * texel;
            py[i] = (iy + jy - cy) * texel;
        }
    }
}

}  // namespace

cudaError_t launch_source(int32_t rows, int32_t cols, int32_t per_texel, float texel,
                          uint64_t seed, uint64_t offset, int64_t n, float* px, float* py,
                          cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int64_t pairs = (n + 1) / 2;
    const int64_t blocks = (pairs + 255) / 256;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t cap = int64_t(sms) * 16;
    source_kernel<<<unsigned(blocks < cap ? blocks : cap), 256, 0, st>>>(
        rows, cols, per_texel, texel, seed, offset, n, px, py);
    return cudaGetLastError();
}

}  // namespace pds
