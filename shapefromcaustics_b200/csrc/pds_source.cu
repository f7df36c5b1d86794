// Device photon source for the height-field plate (sm_100a): per_texel photon entry points per
// texel, jittered uniformly inside the texel, as per_texel samples of one photon per texel
// each (photon i: sample i / texels of texel i % texels, texels in raster order).
//
// Reference: the per-pixel random sampling of the surface in model/caustics.py:78-83
// (rand_like offsets of up to half a texel in each direction, one photon per texel) and the
// per-simulation repetition of the reference's loop, which the samples follow; there the
// offsets come from torch's generator on the host side of each simulation. Consecutive
// photons therefore come from neighbouring texels, not from one texel: the splat's tile
// kernels and the refraction backward's patch sums then see spread-out pixels and texels
// instead of the same few. Here they come from a counter-based generator, Philox4x32
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
    const int64_t texels = int64_t(rows) * cols;
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
            // texel of photon i (32-bit quotients where the index fits: a 64-bit division is
            // a long software sequence)
            int64_t t, ty;
            if (uint64_t(i) <= 0xFFFFFFFFull && texels <= 0xFFFFFFFFll) {
                const uint32_t t32 = uint32_t(i) % uint32_t(texels);
                const uint32_t y32 = t32 / uint32_t(cols);
                t = t32;
                ty = y32;
            } else {
                t = i % texels;
                ty = t / cols;
            }
            const float iy = float(ty), ix = float(t - ty * cols);
            const float jx = unit24(h ? r.z : r.x) - 0.5f, jy = unit24(h ? r.w : r.y) - 0.5f;
            px[i] = (ix + jx - cx) * texel;
            py[i] = (iy + jy - cy) * texel;
        }
    }
}

// ---- point light -----------------------------------------------------------------------
// Directions of a point light spread over a rectangle of the plane z = plane_z by a bilinear
// slerp (model/caustics.py:26-70, compute_point_light_dirs): with the corner directions
// c_ab = normalize(corner_ab - light) (a: x min/max, b: y min/max), a photon's direction is
// slerp(slerp(c_00, c_10, u0), slerp(c_01, c_11, u0), u1) for its two uniform numbers
// (u0, u1); its direction differentials are the Frisvad (2012) orthonormal basis of that
// direction (model/utils.py, compute_orthonormal_basis), scaled by
// 2 smoothing sqrt(omega / (pi N)) with omega the rectangle's solid angle seen from the light
// (two triangles, Van Oosterom-Strackee, model/utils.py subtended_angle) and N the photon count
// of all simulations and wavelengths. The reference computes omega on the device and reads it
// back (sbt_angle.item(), caustics.py:60); here every thread computes it from the light's
// parameters, so nothing waits on the host.

// The directions and their bases are formed in double: the basis divides by 1 + d_z, which
// cancels for near-vertical directions (about 7e-4 for a light 10 units above a unit plate),
// so a float32 direction would carry ~1e-4 relative error into the differentials. Each photon
// costs a few hundred double operations once per simulation, outside the splat's hot path.
struct V3d {
    double x, y, z;
};
__device__ __forceinline__ V3d v3(double x, double y, double z) { return {x, y, z}; }
__device__ __forceinline__ double dot3(V3d a, V3d b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3d cross3(V3d a, V3d b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ V3d scale3(double s, V3d a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ V3d add3(V3d a, V3d b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ V3d sub3(V3d a, V3d b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ double norm3(V3d a) { return sqrt(dot3(a, a)); }
__device__ __forceinline__ V3d unit3(V3d a) {
    const double n = norm3(a);
    return n > 0.0 ? scale3(1.0 / n, a) : a;
}

// slerp(p0, p1, t) = (sin((1 - t) w) p0 + sin(t w) p1) / sin(w), w = acos(clamp(p0.p1))
__device__ __forceinline__ V3d slerp3(V3d p0, V3d p1, double t) {
    const double w = acos(fmin(fmax(dot3(p0, p1), -1.0), 1.0));
    const double s = sin(w);
    return scale3(1.0 / s, add3(scale3(sin((1.0 - t) * w), p0), scale3(sin(t * w), p1)));
}

// Solid angle of triangle (v0, v1, v2) seen from o: 2 atan2(d0.(d2 x d1), |d0||d1||d2| +
// |d0| d1.d2 + |d1| d0.d2 + |d2| d0.d1), negative values counted as zero (as the reference
// sums relu of the per-triangle angles).
__device__ __forceinline__ double tri_angle(V3d o, V3d v0, V3d v1, V3d v2) {
    const V3d d0 = sub3(v0, o), d1 = sub3(v1, o), d2 = sub3(v2, o);
    const double n0 = norm3(d0), n1 = norm3(d1), n2 = norm3(d2);
    const double num = dot3(d0, cross3(d2, d1));
    const double den = n0 * n1 * n2 + n0 * dot3(d1, d2) + n1 * dot3(d0, d2) + n2 * dot3(d0, d1);
    const double a = (num == 0.0 && den == 0.0) ? 0.0 : 2.0 * atan2(num, den);
    return fmax(a, 0.0);
}

// [0, 1) from the top 24 bits, in double (exact)
__device__ __forceinline__ double unit24d(uint32_t u) { return double(u >> 8) * (1.0 / 16777216.0); }

__global__ __launch_bounds__(256) void point_light_kernel(pds_point_light L, int64_t n_dir,
                                                          uint64_t seed, uint64_t offset,
                                                          const float* __restrict__ coeffs,
                                                          float* __restrict__ dir,
                                                          float* __restrict__ dth,
                                                          float* __restrict__ dph,
                                                          float* __restrict__ flux) {
    const V3d o = v3(L.position[0], L.position[1], L.position[2]);
    const V3d p00 = v3(L.xmin, L.ymin, L.plane_z), p10 = v3(L.xmax, L.ymin, L.plane_z);
    const V3d p01 = v3(L.xmin, L.ymax, L.plane_z), p11 = v3(L.xmax, L.ymax, L.plane_z);
    const V3d c00 = unit3(sub3(p00, o)), c10 = unit3(sub3(p10, o));
    const V3d c01 = unit3(sub3(p01, o)), c11 = unit3(sub3(p11, o));
    const double omega = tri_angle(o, p00, p10, p01) + tri_angle(o, p01, p10, p11);
    const int wl = L.wavelengths;
    const double total = double(n_dir) * double(L.simulations) * double(wl);
    const double scale = 2.0 * double(L.smoothing) * sqrt(omega / (3.141592653589793 * total));
    const float f = L.energy / float(int64_t(L.simulations) * L.inner);
    const int64_t n = n_dir * wl;
    const int64_t pairs = (n_dir + 1) >> 1;
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < pairs;
         k += int64_t(gridDim.x) * blockDim.x) {
        uint4 r = make_uint4(0u, 0u, 0u, 0u);
        if (!coeffs) {
            const uint64_t ctr = offset + uint64_t(k);
            r = philox4x32_10(make_uint4(uint32_t(ctr), uint32_t(ctr >> 32), 0u, 0u),
                              uint32_t(seed), uint32_t(seed >> 32));
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int64_t i = 2 * k + h;
            if (i >= n_dir) break;
            const double u0 = coeffs ? double(coeffs[i]) : unit24d(h ? r.z : r.x);
            const double u1 = coeffs ? double(coeffs[n_dir + i]) : unit24d(h ? r.w : r.y);
            const V3d lower = slerp3(c00, c10, u0), upper = slerp3(c01, c11, u0);
            const V3d d = slerp3(lower, upper, u1);
            V3d b1, b2;
            if (d.z < -1.0 + 1e-5) {
                b1 = v3(0.0, -1.0, 0.0);
                b2 = v3(-1.0, 0.0, 0.0);
            } else {
                const double a = 1.0 / (1.0 + d.z);
                const double b = -d.x * d.y * a;
                b1 = v3(1.0 - a * d.x * d.x, b, -d.x);
                b2 = v3(b, 1.0 - a * d.y * d.y, -d.y);
            }
            for (int w = 0; w < wl; ++w) {
                const int64_t j = i * wl + w;
                dir[j] = float(d.x); dir[n + j] = float(d.y); dir[2 * n + j] = float(d.z);
                dth[j] = float(scale * b1.x); dth[n + j] = float(scale * b1.y);
                dth[2 * n + j] = float(scale * b1.z);
                dph[j] = float(scale * b2.x); dph[n + j] = float(scale * b2.y);
                dph[2 * n + j] = float(scale * b2.z);
                flux[j] = f;
            }
        }
    }
}

}  // namespace

cudaError_t launch_point_light(const pds_point_light& L, int64_t n_dir, uint64_t seed,
                               uint64_t offset, const float* coeffs, float* dir, float* dth,
                               float* dph, float* flux, cudaStream_t st) {
    if (n_dir <= 0) return cudaSuccess;
    const int64_t pairs = (n_dir + 1) / 2;
    const int64_t blocks = (pairs + 255) / 256;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t cap = int64_t(sms) * 16;
    point_light_kernel<<<unsigned(blocks < cap ? blocks : cap), 256, 0, st>>>(
        L, n_dir, seed, offset, coeffs, dir, dth, dph, flux);
    return cudaGetLastError();
}

cudaError_t launch_source(int32_t rows, int32_t cols, int32_t per_texel, float texel,
                          uint64_t seed, uint64_t offset, int64_t n, float* px, float* py,
                          cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    const int64_t pairs = (n + 1) / 2;
    const int64_t blocks = (pairs + 255) / 256;
    // one wave of resident CTAs (a grid-stride loop; partial extra waves would idle SMs)
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, source_kernel, 256, 0) !=
            cudaSuccess || per_sm < 1)
        per_sm = 1;
    const int64_t cap = int64_t(sms) * per_sm;
    source_kernel<<<unsigned(blocks < cap ? blocks : cap), 256, 0, st>>>(
        rows, cols, per_texel, texel, seed, offset, n, px, py);
    return cudaGetLastError();
}

}  // namespace pds
