// Fused refraction-to-receiver for a glass plate with a height-field top face (sm_100a).
//
// Per photon, from the height field h and the photon's entry point (px, py):
//   surface sample      bilinear h and bilinear Sobel normal N~ = (-dh/dx, -dh/dy, 1) with its
//                       x/y derivatives (model/caustics.py:215-221: replicate padding, kernel
//                       scaled by -1/(8 texel))
//   transfer            positional differentials onto the tangent plane
//                       (model/photon_differential.py:69-78)
//   refraction x2       Snell + Igehy direction differentials (model/caustics.py:176-189),
//                       normal derivative of the normalised normal along the positional
//                       differential (model/renderable_object.py:391-401); flat bottom face
//   receiver            propagation to the receiver plane, normalised coordinates
//   splat inputs        Mp = 2 [Du Dv]^-1, radius = |D|max / 2, Ep = 4 flux / |Du x Dv|
//                       (model/caustics.py:224-239); degenerate photons get channel -1
// and writes the splat inputs (Ep, xp, Mp, cp, radius) in the reference's layouts.
//
// The backward recomputes the chain from h (nothing is stored between the passes), takes the
// derivatives of the splat-input gradients' contraction with respect to the seven
// height-dependent scalars of the photon (height, N~x, N~y and their x/y derivatives; for the
// point light the hit parameter in place of the height) by a hand-written reverse-mode sweep,
// and maps them back onto the photon's 4x4 texel patch through the transposed bilinear and
// Sobel stencils (the chain and its sweeps: pds_chain.cuh, checked on the host against the
// chain instantiated with forward-mode dual numbers by tests/chain_adjoint_check.cu). A CTA's
// patches are summed in shared memory where its photons share a compact region of the field,
// else added with global float atomics.
#include <climits>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pds_b200.h"
#include "pds_chain.cuh"
#include "pds_device.cuh"
#include "pds_internal.h"

namespace pds {
namespace {

using namespace chain;

// Bilinear footprint of a world position on the height-field grid (texel centres at
// integers, clamped to the border).
struct Bilin {
    int x0, y0;
    float ax, ay;
};

__device__ __forceinline__ Bilin bilin(float px, float py, float texel, int H, int W) {
    float fx = qdiv(px, texel) + 0.5f * float(W - 1);
    float fy = qdiv(py, texel) + 0.5f * float(H - 1);
    fx = fminf(fmaxf(fx, 0.f), float(W - 1));
    fy = fminf(fmaxf(fy, 0.f), float(H - 1));
    Bilin b;
    b.x0 = min(int(floorf(fx)), max(W - 2, 0));
    b.y0 = min(int(floorf(fy)), max(H - 2, 0));
    b.ax = fx - float(b.x0);
    b.ay = fy - float(b.y0);
    return b;
}

// Position derivatives of the surface at a sample (for the traced hit).
struct SurfGeo {
    float hx, hy;        // slope of the bilinear height
    float tw_nx, tw_ny;  // d2 Nx / dx dy, d2 Ny / dx dy of the bilinear normal field
};

// The seven scalars of one photon: height, Sobel normal (x, y) and their x/y derivatives;
// with geo, also the position derivatives of the sample. The cell's two rows and columns
// with their Sobel neighbours span the 4x4 texels y0-1..y0+2 x x0-1..x0+2; each is loaded
// once, with its row and column clamped into the field (replicate padding: a texel outside
// the field reads its nearest border texel, for every stencil tap alike).
__device__ __forceinline__ void surface_scalars(const float* h, int H, int W, float texel,
                                                const Bilin& b, float s[K],
                                                SurfGeo* geo = nullptr) {
    const float itex = qdiv(1.f, texel);  // one quotient; the stencils multiply by it
    const float c = -0.125f * itex;
    int col[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) col[q] = min(max(b.x0 - 1 + q, 0), W - 1);
    float t[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const float* row = h + int64_t(min(max(b.y0 - 1 + r, 0), H - 1)) * W;
#pragma unroll
        for (int q = 0; q < 4; ++q) t[r][q] = __ldg(row + col[q]);
    }
    // cell corner (r, q) is texel (r + 1, q + 1); its Sobel taps are rows r .. r + 2 and
    // columns q .. q + 2
    float hv[2][2], nx[2][2], ny[2][2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            hv[r][q] = t[r + 1][q + 1];
            nx[r][q] = c * (t[r][q + 2] - t[r][q] + 2.f * (t[r + 1][q + 2] - t[r + 1][q]) +
                            t[r + 2][q + 2] - t[r + 2][q]);
            ny[r][q] = c * (t[r + 2][q] - t[r][q] + 2.f * (t[r + 2][q + 1] - t[r][q + 1]) +
                            t[r + 2][q + 2] - t[r][q + 2]);
        }
    }
    auto val = [&](float v[2][2]) {
        const float top = v[0][0] + (v[0][1] - v[0][0]) * b.ax;
        const float bot = v[1][0] + (v[1][1] - v[1][0]) * b.ax;
        return top + (bot - top) * b.ay;
    };
    auto ddx = [&](float v[2][2]) {
        return ((v[0][1] - v[0][0]) * (1.f - b.ay) + (v[1][1] - v[1][0]) * b.ay) * itex;
    };
    auto ddy = [&](float v[2][2]) {
        const float top = v[0][0] + (v[0][1] - v[0][0]) * b.ax;
        const float bot = v[1][0] + (v[1][1] - v[1][0]) * b.ax;
        return (bot - top) * itex;
    };
    s[0] = val(hv);
    s[1] = val(nx);
    s[2] = val(ny);
    s[3] = ddx(nx);  // dNx/dx
    s[4] = ddx(ny);  // dNy/dx
    s[5] = ddy(nx);  // dNx/dy
    s[6] = ddy(ny);  // dNy/dy
    if (geo) {
        // the height's slope and the normal field's twist d2/dxdy (the x derivatives above
        // vary along y and the y derivatives along x by it)
        geo->hx = ddx(hv);
        geo->hy = ddy(hv);
        const float it2 = itex * itex;
        geo->tw_nx = ((nx[1][1] - nx[1][0]) - (nx[0][1] - nx[0][0])) * it2;
        geo->tw_ny = ((ny[1][1] - ny[1][0]) - (ny[0][1] - ny[0][0])) * it2;
    }
}

struct RefractArgs {
    const float* h;
    int H, W;
    PlateParams P;
    // batches: simulation k (photons begins[k] .. begins[k + 1] - 1) uses plates[k]; NULL: P
    const pds_plate* plates;
    const int64_t* begins;
    int32_t n_sims;
    const float* px;
    const float* py;
    const float* flux;
    const int64_t* channel;
    int64_t n;
    // forward outputs
    float* Ep;
    float* xp;
    float* Mp;
    int64_t* cp;
    float* radius;
    // backward inputs / output: the splat gradients as arrays, or (rec_inv non-null) as a
    // plan's gradient records
    const float* gE;
    const float* gX;
    const float* gM;
    const uint32_t* rec_inv;
    const float4* rec_stage;
    const uint32_t* rec_counters;
    float* gh;
};

// The splat gradients of photon i (d L / d Ep, xp, Mp[0,0..1], Mp[1,0..1]) from the plan's
// gradient records: the values the gradient spread would write, without the spread and its
// re-read. False for a photon that touches no pixel (zero gradients).
__device__ __forceinline__ bool photon_grads(const RefractArgs& a, int64_t i, int64_t n_tile,
                                             float& gE, float& gx, float& gy, float& g0,
                                             float& g1, float& g3, float& g4) {
    const int64_t n = a.n;
    const uint32_t v = __ldg(a.rec_inv + i);
    const int64_t slot = (v & kWideBit) ? n_tile + int64_t(v & ~kWideBit) : int64_t(v);
    if (v == kInvalidPos || slot >= n) return false;
    const float4 lo = __ldg(a.rec_stage + 2 * slot), hi = __ldg(a.rec_stage + 2 * slot + 1);
    gE = lo.x; gx = lo.y; gy = lo.z; g0 = lo.w;
    g1 = hi.x; g3 = hi.y; g4 = hi.z;
    return true;
}

// The plate of photon i: its simulation's in a batch (photons of a simulation are
// contiguous; bisection over the simulations' first photons), else the call's.
__device__ __forceinline__ PlateParams photon_params(const RefractArgs& a, int64_t i) {
    if (!a.plates) return a.P;
    int lo = 0, hi = a.n_sims - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(a.begins + mid) <= i) lo = mid; else hi = mid - 1;
    }
    return to_params(a.plates[lo]);
}

// Each thread loads its next photon's entry point and flux while it refracts the current one
// (the texel loads depend on the entry point, so an unprefetched photon waits for two memory
// latencies in a row); five CTAs an SM (48 registers) keep the occupancy the prefetch's
// registers would otherwise cost (recon1024: 1.44 -> 1.37 ms).
__global__ __launch_bounds__(256, 5) void refract_fwd_kernel(RefractArgs a) {
    const int64_t n = a.n;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    float npx = 0.f, npy = 0.f, nfl = 0.f;
    if (i < n) {
        npx = a.px[i];
        npy = a.py[i];
        nfl = a.flux[i];
    }
    for (; i < n; i += stride) {
        const float px = npx, py = npy, fl = nfl;
        if (i + stride < n) {
            npx = a.px[i + stride];
            npy = a.py[i + stride];
            nfl = a.flux[i + stride];
        }
        const PlateParams P = photon_params(a, i);
        const Bilin b = bilin(px, py, P.texel, a.H, a.W);
        float s[K];
        surface_scalars(a.h, a.H, a.W, P.texel, b, s);
        float xr, yr, Dux, Duy, Dvx, Dvy;
        plate_chain<float>(s[0], s[1], s[2], s[3], s[4], s[5], s[6], px, py, P, xr, yr, Dux,
                           Duy, Dvx, Dvy);
        const float den = Dux * Dvy - Duy * Dvx;
        const bool good = den != 0.f;
        const float f = qdiv(2.f, good ? den : 1.f);
        a.Mp[i] = f * Dvy;
        a.Mp[n + i] = -f * Dvx;
        a.Mp[2 * n + i] = 0.f;
        a.Mp[3 * n + i] = -f * Duy;
        a.Mp[4 * n + i] = f * Dux;
        a.Mp[5 * n + i] = 0.f;
        a.xp[i] = xr;
        a.xp[n + i] = yr;
        a.radius[i] = 0.5f * fmaxf(sqrtf(Dux * Dux + Duy * Duy), sqrtf(Dvx * Dvx + Dvy * Dvy));
        a.Ep[i] = qdiv(4.f * fl, good ? fabsf(den) : 1.f);
        const int64_t ch = a.channel ? a.channel[i] : 0;
        a.cp[i] = good ? ch : -1;
    }
}

// Adds d L / d height of one photon to its 4x4 texel patch (x0-1..x0+2, y0-1..y0+2) from the
// derivatives c[k] of L with respect to its seven surface scalars: the transposed bilinear
// stencil for the height (k = 0) and the transposed bilinear and Sobel stencils for the normal
// scalars (k = 1..6). Patch texels outside the field fold onto the border (replicate padding).
// add(row, col, value) receives the non-zero patch entries.
template <class Add>
__device__ __forceinline__ void scatter_patch(int H, int W, float texel, const Bilin& b,
                                              const float c[K], Add add) {
    float patch[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int q = 0; q < 4; ++q) patch[r][q] = 0.f;
    const float it = qdiv(1.f, texel);
    const float sob = -0.125f * it;
    const float wv[2][2] = {{(1.f - b.ay) * (1.f - b.ax), (1.f - b.ay) * b.ax},
                            {b.ay * (1.f - b.ax), b.ay * b.ax}};
    const float wx[2][2] = {{-(1.f - b.ay) * it, (1.f - b.ay) * it}, {-b.ay * it, b.ay * it}};
    const float wy[2][2] = {{-(1.f - b.ax) * it, -b.ax * it}, {(1.f - b.ax) * it, b.ax * it}};
#pragma unroll
    for (int r = 0; r < 2; ++r) {
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            patch[r + 1][q + 1] += c[0] * wv[r][q];
            const float gnx = sob * (c[1] * wv[r][q] + c[3] * wx[r][q] + c[5] * wy[r][q]);
            const float gny = sob * (c[2] * wv[r][q] + c[4] * wx[r][q] + c[6] * wy[r][q]);
            // Sobel x at (r, q): +(r-1,q+1) -(r-1,q-1) +2(r,q+1) -2(r,q-1) +(r+1,q+1) -(r+1,q-1)
            patch[r][q + 2] += gnx;
            patch[r][q] -= gnx;
            patch[r + 1][q + 2] += 2.f * gnx;
            patch[r + 1][q] -= 2.f * gnx;
            patch[r + 2][q + 2] += gnx;
            patch[r + 2][q] -= gnx;
            // Sobel y: +(r+1,q-1) -(r-1,q-1) +2(r+1,q) -2(r-1,q) +(r+1,q+1) -(r-1,q+1)
            patch[r + 2][q] += gny;
            patch[r][q] -= gny;
            patch[r + 2][q + 1] += 2.f * gny;
            patch[r][q + 1] -= 2.f * gny;
            patch[r + 2][q + 2] += gny;
            patch[r][q + 2] -= gny;
        }
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int ii = min(max(b.y0 - 1 + r, 0), H - 1);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int jj = min(max(b.x0 - 1 + q, 0), W - 1);
            if (patch[r][q] != 0.f) add(ii, jj, patch[r][q]);
        }
    }
}

// The height-field gradient of a CTA's photons: where the CTA's photons share a compact patch
// of the field (the photon source emits each sample's photons texel by texel in raster order,
// so a CTA's 256 consecutive photons sit in one or two texel rows), their patches are summed
// in shared memory and added to the field once per texel; otherwise (scattered hits) each
// patch entry is a global atomic add. Without it, every photon's 16 patch entries were global
// atomics on a few hot texels.
constexpr int kPatchSmem = 8192;  // floats of the CTA's two shared patch regions (32 KB)

struct PatchAcc {
    float* buf;   // shared region, rw x rh floats, or nullptr: global atomics
    int x0, y0, rw;
    float* gh;
    int W;
    __device__ __forceinline__ void operator()(int ii, int jj, float v) const {
        if (buf)
            atomicAdd(buf + (ii - y0) * rw + (jj - x0), v);
        else
            atomicAdd(gh + int64_t(ii) * W + jj, v);
    }
};

// Sets up the CTA's region from its active photons' cells (bx0, by0; ignored when !active):
// all threads call it. Returns the accumulator (shared region zeroed, or global).
// The accumulator of the region bounded by the cells in bb (min x, max x, min y, max y): the
// shared buffer (cap floats) when the region fits, else global atomics.
__device__ __forceinline__ PatchAcc region_acc(float* buf, int cap, const int* bb, float* gh,
                                               int H, int W) {
    PatchAcc acc;
    acc.gh = gh;
    acc.W = W;
    acc.buf = nullptr;
    acc.x0 = acc.y0 = acc.rw = 0;
    if (bb[0] <= bb[1]) {
        // patch texels: cell - 1 .. cell + 2, clamped into the field (replicate padding)
        const int x0 = max(bb[0] - 1, 0), x1 = min(bb[1] + 2, W - 1);
        const int y0 = max(bb[2] - 1, 0), y1 = min(bb[3] + 2, H - 1);
        const int rw = x1 - x0 + 1, rh = y1 - y0 + 1;
        if (int64_t(rw) * rh <= cap) {
            acc.buf = buf;
            acc.x0 = x0;
            acc.y0 = y0;
            acc.rw = rw;
        }
    }
    return acc;
}

// Clears a shared region (all threads call it).
__device__ __forceinline__ void region_zero(const PatchAcc& acc, const int* bb, int H) {
    if (acc.buf) {
        const int rh = min(bb[3] + 2, H - 1) - acc.y0 + 1;
        for (int k = threadIdx.x; k < acc.rw * rh; k += blockDim.x) acc.buf[k] = 0.f;
    }
}

// Adds a shared region to the field (all threads call it): warps take rows, lanes take
// consecutive columns (coalesced adds, and no division to find a texel's row).
__device__ __forceinline__ void region_flush(const PatchAcc& acc, const int* bb, int H, int W) {
    if (acc.buf) {
        const int y1 = min(bb[3] + 2, H - 1);
        const int rh = y1 - acc.y0 + 1;
        const int warp = int(threadIdx.x >> 5), lane = int(threadIdx.x & 31);
        const int nw = int(blockDim.x >> 5);
        for (int ry = warp; ry < rh; ry += nw) {
            const float* srow = acc.buf + ry * acc.rw;
            float* grow = acc.gh + int64_t(acc.y0 + ry) * W + acc.x0;
            for (int rx = lane; rx < acc.rw; rx += 32) {
                const float v = srow[rx];
                if (v != 0.f) atomicAdd(grow + rx, v);
            }
        }
    }
}

// The bounds of the CTA's active cells into bb (reset beforehand): a warp reduction, then one
// shared atomic per warp and bound.
__device__ __forceinline__ void region_bounds(int* bb, bool active, int bx0, int by0) {
    int lx0 = active ? bx0 : INT_MAX, lx1 = active ? bx0 : INT_MIN;
    int ly0 = active ? by0 : INT_MAX, ly1 = active ? by0 : INT_MIN;
    lx0 = __reduce_min_sync(0xFFFFFFFFu, lx0);
    lx1 = __reduce_max_sync(0xFFFFFFFFu, lx1);
    ly0 = __reduce_min_sync(0xFFFFFFFFu, ly0);
    ly1 = __reduce_max_sync(0xFFFFFFFFu, ly1);
    if ((threadIdx.x & 31) == 0 && lx0 <= lx1) {
        atomicMin(bb + 0, lx0);
        atomicMax(bb + 1, lx1);
        atomicMin(bb + 2, ly0);
        atomicMax(bb + 3, ly1);
    }
}

__device__ __forceinline__ void bounds_reset(int* bb) {
    bb[0] = INT_MAX; bb[1] = INT_MIN; bb[2] = INT_MAX; bb[3] = INT_MIN;
}

// Three CTAs an SM (80 registers): measured 18% faster than the 114-register build at two
// CTAs an SM (16.8 M photons of a 1024^2 field: 2.24 vs 2.73 ms).
//
// Consecutive blocks of a CTA alternate between two shared regions (half of kPatchSmem each)
// and two bound arrays, so that a block's flush needs no barrier after it and the next
// block's bounds need none before them: three barriers a block instead of five. Buffer p of
// block k was last read by block k - 2's flush, which every thread finished before block
// k - 1's first barrier; its bounds are reset by thread 0 after that barrier, and block k's
// bound atomics come after block k - 1's last barrier (recon1024: 4.68 -> 4.49 ms).
template <bool REC>
__global__ __launch_bounds__(256, 3) void refract_bwd_kernel(RefractArgs a) {
    constexpr int kHalf = kPatchSmem / 2;
    __shared__ float smem[2 * kHalf];
    __shared__ int bbs[2][4];
    if (threadIdx.x == 0) {
        bounds_reset(bbs[0]);
        bounds_reset(bbs[1]);
    }
    __syncthreads();
    int p = 0;
    const int64_t n = a.n;
    // tile-path photons of the plan whose gradient records are read (records mode)
    const int64_t n_tile = REC ? min(int64_t(__ldg(a.rec_counters)), n) : 0;
    // CTA-contiguous blocks of 256 photons (their patches share a shared-memory region)
    for (int64_t blk = int64_t(blockIdx.x) * blockDim.x; blk < n;
         blk += int64_t(gridDim.x) * blockDim.x, p ^= 1) {
        const int64_t i = blk + threadIdx.x;
        bool active = i < n;
        Bilin b = {0, 0, 0.f, 0.f};
        float c[K];
        float texel = a.P.texel;
        if (active) {
            const float px = a.px[i], py = a.py[i];
            const PlateParams P = photon_params(a, i);
            texel = P.texel;
            b = bilin(px, py, P.texel, a.H, a.W);
            float s[K];
            surface_scalars(a.h, a.H, a.W, P.texel, b, s);
            if (REC) {
                float gE, gx, gy, g0, g1, g3, g4;
                active = photon_grads(a, i, n_tile, gE, gx, gy, g0, g1, g3, g4) &&
                         plate_chain_adjoint(s, px, py, P, gx, gy, g0, g1, g3, g4,
                                             4.f * a.flux[i] * gE, c);
            } else {
                active = plate_chain_adjoint(s, px, py, P, a.gX[i], a.gX[n + i], a.gM[i],
                                             a.gM[n + i], a.gM[3 * n + i], a.gM[4 * n + i],
                                             4.f * a.flux[i] * a.gE[i], c);
            }
        }
        int* bb = bbs[p];
        region_bounds(bb, active, b.x0, b.y0);
        __syncthreads();
        if (threadIdx.x == 0) bounds_reset(bbs[p ^ 1]);
        const PatchAcc acc = region_acc(smem + p * kHalf, kHalf, bb, a.gh, a.H, a.W);
        region_zero(acc, bb, a.H);
        __syncthreads();
        if (active) scatter_patch(a.H, a.W, texel, b, c, acc);
        __syncthreads();
        region_flush(acc, bb, a.H, a.W);
    }
}

// ---- point light: traced hit on the height field ----------------------------------------
// Photons leave the light at o with unit direction d and direction differentials (Dth, Dph)
// (pds_point_light_source_f32). Their first hit with the bilinear height-field surface is found
// by Newton steps on f(t) = o_z + t d_z - h(o_xy + t d_xy) from the plane z = plane_z (no
// overhangs and no occluding bump before the hit, as the reference's generate_from_point_light
// assumes, model/caustics.py:119). At the hit the positional differentials are the light's
// carried over the length t (model/photon_differential.py:69-78 with Du = Dv = 0 at the light),
// and the chain continues as for the collimated plate with the direction differentials.

// Newton iterations of the trace; false when the ray grazes the surface or its hit lies
// outside the field. b, s, geo: the surface at the hit; t: the ray parameter; fp: f'(t).
__device__ __forceinline__ bool trace_hit(const float* h, int H, int W, float texel,
                                          float plane_z, const Ray& r, float& t, Bilin& b,
                                          float s[K], SurfGeo& geo, float& fp) {
    t = qdiv(r.oz - plane_z, -r.dz);
    const float cx = 0.5f * float(W - 1), cy = 0.5f * float(H - 1);
    for (int it = 0; it < 10; ++it) {
        const float px = r.ox + t * r.dx, py = r.oy + t * r.dy, pz = r.oz + t * r.dz;
        b = bilin(px, py, texel, H, W);
        surface_scalars(h, H, W, texel, b, s, &geo);
        fp = r.dz - (geo.hx * r.dx + geo.hy * r.dy);
        if (!(fabsf(fp) > 1e-6f)) return false;
        const float step = qdiv(pz - s[0], fp);
        t -= step;
        if (fabsf(step) <= 1e-7f * fabsf(t)) break;
    }
    const float px = r.ox + t * r.dx, py = r.oy + t * r.dy;
    const float fx = qdiv(px, texel) + cx, fy = qdiv(py, texel) + cy;
    if (!(fx >= 0.f && fx <= float(W - 1) && fy >= 0.f && fy <= float(H - 1))) return false;
    b = bilin(px, py, texel, H, W);
    surface_scalars(h, H, W, texel, b, s, &geo);
    fp = r.dz - (geo.hx * r.dx + geo.hy * r.dy);
    return fabsf(fp) > 1e-6f;
}

struct PointArgs {
    const float* h;
    int H, W;
    PlateParams P;
    float ox, oy, oz, plane_z;
    const float* dir;   // [3][n]
    const float* dth;   // [3][n]
    const float* dph;   // [3][n]
    const float* flux;
    const int64_t* channel;
    int64_t n;
    float* Ep;
    float* xp;
    float* Mp;
    int64_t* cp;
    float* radius;
    const float* gE;
    const float* gX;
    const float* gM;
    float* gh;
};

__device__ __forceinline__ Ray photon_ray(const PointArgs& a, int64_t i) {
    Ray r;
    r.ox = a.ox; r.oy = a.oy; r.oz = a.oz;
    r.dx = a.dir[i]; r.dy = a.dir[a.n + i]; r.dz = a.dir[2 * a.n + i];
    return r;
}

__global__ __launch_bounds__(256) void point_fwd_kernel(PointArgs a) {
    const int64_t n = a.n;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x) {
        const Ray r = photon_ray(a, i);
        float t, fp, s[K];
        Bilin b;
        SurfGeo geo;
        const bool hit = trace_hit(a.h, a.H, a.W, a.P.texel, a.plane_z, r, t, b, s, geo, fp);
        float xr = 0.f, yr = 0.f, Dux = 0.f, Duy = 0.f, Dvx = 0.f, Dvy = 0.f;
        if (hit) {
            const V3<float> Dt = {a.dth[i], a.dth[n + i], a.dth[2 * n + i]};
            const V3<float> Dp = {a.dph[i], a.dph[n + i], a.dph[2 * n + i]};
            point_chain<float>(t, s[1], s[2], s[3], s[4], s[5], s[6], r, Dt, Dp, a.P, xr, yr, Dux,
                               Duy, Dvx, Dvy);
        }
        const float den = Dux * Dvy - Duy * Dvx;
        const bool good = hit && den != 0.f;
        const float f = qdiv(2.f, good ? den : 1.f);
        a.Mp[i] = f * Dvy;
        a.Mp[n + i] = -f * Dvx;
        a.Mp[2 * n + i] = 0.f;
        a.Mp[3 * n + i] = -f * Duy;
        a.Mp[4 * n + i] = f * Dux;
        a.Mp[5 * n + i] = 0.f;
        a.xp[i] = xr;
        a.xp[n + i] = yr;
        a.radius[i] = 0.5f * fmaxf(sqrtf(Dux * Dux + Duy * Duy), sqrtf(Dvx * Dvx + Dvy * Dvy));
        a.Ep[i] = qdiv(4.f * a.flux[i], good ? fabsf(den) : 1.f);
        const int64_t ch = a.channel ? a.channel[i] : 0;
        a.cp[i] = good ? ch : -1;
    }
}

__global__ __launch_bounds__(256) void point_bwd_kernel(PointArgs a) {
    const int64_t n = a.n;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x) {
        const Ray r = photon_ray(a, i);
        float t, fp, s[K];
        Bilin b;
        SurfGeo geo;
        if (!trace_hit(a.h, a.H, a.W, a.P.texel, a.plane_z, r, t, b, s, geo, fp)) continue;
        const V3<float> Dt = {a.dth[i], a.dth[n + i], a.dth[2 * n + i]};
        const V3<float> Dp = {a.dph[i], a.dph[n + i], a.dph[2 * n + i]};
        float tb, Sb[K];
        if (!point_chain_adjoint(t, s, r, Dt, Dp, a.P, a.gX[i], a.gX[n + i], a.gM[i],
                                 a.gM[n + i], a.gM[3 * n + i], a.gM[4 * n + i],
                                 4.f * a.flux[i] * a.gE[i], tb, Sb))
            continue;
        // d L / d t along the ray: t itself, and the normal scalars following the hit (their
        // position derivatives times d); the hit moves with the heights, dt / dh_j = w_j / f'(t)
        // for the bilinear weights w_j of the hit's cell
        const float Lt = tb + Sb[1] * (s[3] * r.dx + s[5] * r.dy) +
                         Sb[2] * (s[4] * r.dx + s[6] * r.dy) +
                         (Sb[3] * geo.tw_nx + Sb[4] * geo.tw_ny) * r.dy +
                         (Sb[5] * geo.tw_nx + Sb[6] * geo.tw_ny) * r.dx;
        float c[K];
        c[0] = qdiv(Lt, fp);
#pragma unroll
        for (int k = 1; k < K; ++k) c[k] = Sb[k];
        // traced hits follow the photons' random directions, not the field's texel order:
        // global adds
        PatchAcc acc;
        acc.buf = nullptr;
        acc.x0 = acc.y0 = acc.rw = 0;
        acc.gh = a.gh;
        acc.W = a.W;
        scatter_patch(a.H, a.W, a.P.texel, b, c, acc);
    }
}

// Grid of a grid-stride refraction kernel: whole waves of resident CTAs (the occupancy of
// this kernel x SMs, times `waves`), capped by the work. A grid with a partial last wave (the
// backward at three CTAs an SM under a fixed 8-CTAs-an-SM grid: 2.67 waves) leaves the CTAs
// of that wave running their whole share after the others finished (the backward 2% faster
// in one wave; the forward, at four CTAs an SM, measured best at two).
template <typename Kern>
int grid_for(Kern kernel, int64_t n, int waves = 1) {
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const int64_t blocks = (n + 255) / 256;
    const int64_t cap = int64_t(sms) * per_sm * waves;
    return int(blocks < cap ? blocks : cap);
}

}  // namespace

cudaError_t launch_refract_point(bool backward, const float* h, int H, int W,
                                 const pds_plate& plate, const pds_point_light& light,
                                 const float* dir, const float* dth, const float* dph,
                                 const float* flux, const int64_t* channel, int64_t n, float* Ep,
                                 float* xp, float* Mp, int64_t* cp, float* radius,
                                 const float* gE, const float* gX, const float* gM, float* gh,
                                 cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    PointArgs a;
    a.h = h;
    a.H = H;
    a.W = W;
    a.P.texel = plate.texel;
    a.P.ior = plate.ior;
    a.P.dist = plate.receiver_distance;
    a.P.inv_half = 1.f / plate.receiver_half;
    a.P.du0 = 0.f;
    a.P.lx = a.P.ly = a.P.lz = 0.f;
    a.ox = light.position[0];
    a.oy = light.position[1];
    a.oz = light.position[2];
    a.plane_z = light.plane_z;
    a.dir = dir;
    a.dth = dth;
    a.dph = dph;
    a.flux = flux;
    a.channel = channel;
    a.n = n;
    a.Ep = Ep;
    a.xp = xp;
    a.Mp = Mp;
    a.cp = cp;
    a.radius = radius;
    a.gE = gE;
    a.gX = gX;
    a.gM = gM;
    a.gh = gh;
    if (backward)
        point_bwd_kernel<<<grid_for(point_bwd_kernel, n), 256, 0, st>>>(a);
    else
        point_fwd_kernel<<<grid_for(point_fwd_kernel, n), 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_refract(bool backward, const float* h, int H, int W, const pds_plate& plate,
                           const pds_plate* plates, const int64_t* begins, int32_t n_sims,
                           const float* px, const float* py, const float* flux,
                           const int64_t* channel, int64_t n, float* Ep, float* xp, float* Mp,
                           int64_t* cp, float* radius, const float* gE, const float* gX,
                           const float* gM, float* gh, cudaStream_t st, const GradRecords* rec) {
    if (n <= 0) return cudaSuccess;
    RefractArgs a;
    a.h = h;
    a.H = H;
    a.W = W;
    a.P = to_params(plate);
    a.plates = plates;
    a.begins = begins;
    a.n_sims = n_sims;
    a.px = px;
    a.py = py;
    a.flux = flux;
    a.channel = channel;
    a.n = n;
    a.Ep = Ep;
    a.xp = xp;
    a.Mp = Mp;
    a.cp = cp;
    a.radius = radius;
    a.gE = gE;
    a.gX = gX;
    a.gM = gM;
    a.rec_inv = rec ? rec->inv : nullptr;
    a.rec_stage = rec ? reinterpret_cast<const float4*>(rec->stage) : nullptr;
    a.rec_counters = rec ? rec->counters : nullptr;
    a.gh = gh;
    if (backward && rec)
        refract_bwd_kernel<true><<<grid_for(refract_bwd_kernel<true>, n), 256, 0, st>>>(a);
    else if (backward)
        refract_bwd_kernel<false><<<grid_for(refract_bwd_kernel<false>, n), 256, 0, st>>>(a);
    else
        refract_fwd_kernel<<<grid_for(refract_fwd_kernel, n, 2), 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace pds
