// Projected Landweber update of the height-field offset, fused (sm_100a).
//
// The reference's per-iteration update (shape_from_caustics.py:386-398, default options):
//   d = d - tau * grad                                  (gradient step, :387)
//   d = mask * extShrink(d, tau * alpha, lower, upper)  (:397, extShrink :184-189)
//   d = VconsHeur(d, d1, d2, mask, gamma, r)            (:398, VconsHeur :228-241)
// with extShrink(x) = clamp(max(|x| - a, 0) sign(x), lower, upper) and
// VconsHeur: v = sum(d); m = (2r+1)^2 box mean of d (zero padded, count_include_pad);
//   v <= d1: d += mask m sin(v/d1 pi) gamma;  v >= d2: d -= mask m sin((v/d2 - 1) pi) gamma.
// Two kernels: (1) step + shrink + mask into a scratch image, with per-block partial sums;
// (2) every block reduces the partial sums in a fixed order (deterministic v), then applies
// the volume heuristic with the box mean of the scratch image. The reference's volume test
// is a host-side branch on a device scalar; here it stays on the device.
#include <cstdint>
#include <mutex>
#include <cuda_runtime.h>

#include "../../include/pds_b200.h"
#include "pds_internal.h"

namespace pds {
namespace {

constexpr int kThreads = 256;
constexpr float kPi = 3.14159265358979323846f;

__device__ __forceinline__ float ext_shrink(float x, float a, float lo, float hi) {
    const float s = x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f);
    const float v = fmaxf(fabsf(x) - a, 0.f) * s;
    return fmaxf(fminf(v, hi), lo);
}

__global__ __launch_bounds__(kThreads) void lw_shrink_kernel(const float* __restrict__ d,
                                                             const float* __restrict__ g,
                                                             const float* __restrict__ mask,
                                                             int64_t n, pds_landweber p,
                                                             float* __restrict__ t,
                                                             float* __restrict__ partial) {
    __shared__ float red[kThreads / 32];
    float acc = 0.f;
    const int64_t stride = int64_t(gridDim.x) * kThreads;
    for (int64_t i = int64_t(blockIdx.x) * kThreads + threadIdx.x; i < n; i += stride) {
        const float x = d[i] - p.tau * g[i];
        const float v = mask[i] * ext_shrink(x, p.shrink, p.lower, p.upper);
        t[i] = v;
        acc += v;
    }
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < kThreads / 32; ++w) s += red[w];
        partial[blockIdx.x] = s;
    }
}

__global__ __launch_bounds__(kThreads) void lw_volume_kernel(const float* __restrict__ t,
                                                             const float* __restrict__ mask,
                                                             int64_t rows, int64_t cols,
                                                             pds_landweber p,
                                                             const float* __restrict__ partial,
                                                             int nparts, float* __restrict__ d) {
    __shared__ float red[kThreads];
    __shared__ float vol;
    // total of the shrunk image, summed in the same order by every block
    float s = 0.f;
    for (int k = threadIdx.x; k < nparts; k += kThreads) s += partial[k];
    red[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float v = 0.f;
        for (int k = 0; k < kThreads; ++k) v += red[k];
        vol = v;
    }
    __syncthreads();
    const float v = vol;
    float coef = 0.f;
    if (v <= p.d1)
        coef = sinf(v / p.d1 * kPi) * p.gamma;
    else if (v >= p.d2)
        coef = -sinf((v / p.d2 - 1.f) * kPi) * p.gamma;
    const int r = p.radius;
    const float inv_area = 1.f / float((2 * r + 1) * (2 * r + 1));
    const int64_t n = rows * cols;
    const int64_t stride = int64_t(gridDim.x) * kThreads;
    for (int64_t i = int64_t(blockIdx.x) * kThreads + threadIdx.x; i < n; i += stride) {
        const float x = t[i];
        if (coef == 0.f) {
            d[i] = x;
            continue;
        }
        const int64_t y = i / cols, xx = i - y * cols;
        float box = 0.f;
        for (int dy = -r; dy <= r; ++dy) {
            const int64_t yy = y + dy;
            if (yy < 0 || yy >= rows) continue;
            for (int dx = -r; dx <= r; ++dx) {
                const int64_t xc = xx + dx;
                if (xc < 0 || xc >= cols) continue;
                box += t[yy * cols + xc];
            }
        }
        d[i] = x + mask[i] * (box * inv_area) * coef;
    }
}

// Fixed block count (independent of the device, so the scratch size is too): grid-stride
// loops cover any image size.
int lw_blocks(int64_t n) {
    const int64_t b = (n + kThreads - 1) / kThreads;
    return int(b < 1024 ? (b > 0 ? b : 1) : 1024);
}

}  // namespace

size_t landweber_scratch_bytes(int64_t n) {
    return align_up(size_t(n > 0 ? n : 1) * sizeof(float), 256) + size_t(lw_blocks(n)) * sizeof(float);
}

cudaError_t launch_landweber(float* d, const float* g, const float* mask, int64_t rows,
                             int64_t cols, const pds_landweber& p, float* t, float* partial,
                             cudaStream_t st) {
    const int64_t n = rows * cols;
    if (n <= 0) return cudaSuccess;
    const int nb = lw_blocks(n);
    lw_shrink_kernel<<<nb, kThreads, 0, st>>>(d, g, mask, n, p, t, partial);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    lw_volume_kernel<<<nb, kThreads, 0, st>>>(t, mask, rows, cols, p, partial, nb, d);
    return cudaGetLastError();
}

// ---- the allocation-free variant -------------------------------------------------------
// Scratch of pds_landweber_update_noalloc_f32: the shrunk image (up to kNoAllocMaxPixels
// floats) followed by the per-block partial sums (at most 1024 floats, see lw_blocks).
// Every GPU that loads this library holds it (4 MiB + 4 KiB) until the process exits.
constexpr int64_t kNoAllocMaxPixels = int64_t(1) << 20;  // 1024 x 1024
constexpr size_t kNoAllocImageBytes = size_t(kNoAllocMaxPixels) * sizeof(float);
constexpr size_t kNoAllocBytes = kNoAllocImageBytes + 1024 * sizeof(float);
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

int64_t landweber_noalloc_max_pixels() { return kNoAllocMaxPixels; }

// Device addresses of the scratch's two parts on the current device: the shrunk image `t`
// (kNoAllocMaxPixels floats) and the per-block partial sums `partial` right after it. In host
// code the symbol is only a host-side stand-in, so the array's address is looked up once per
// device (with that device current) and cached.
cudaError_t landweber_noalloc_scratch(float** t, float** partial) {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static void* addr[kMaxDevices] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(mu);
    if (addr[dev] == nullptr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        addr[dev] = p;
    }
    unsigned char* base = static_cast<unsigned char*>(addr[dev]);
    *t = reinterpret_cast<float*>(base);
    *partial = reinterpret_cast<float*>(base + kNoAllocImageBytes);
    return cudaSuccess;
}

}  // namespace pds
