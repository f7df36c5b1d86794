// Device-side definitions shared by the photon-differential splatting kernels.
//
// Semantics follow the reference kernel PyOptix/kernel/photon_differentials.cu:
//   footprint set-up  :76-89   (radius cut in double through the 0.5 literal, :80-81;
//                               coord_to_pixel in double, truncating, :46-51)
//   ellipse test      :93      (against the image half-size, in double)
//   kernel            :23-29   (K(s) = 3/pi (1 - s)^2 for s = |u|^2 < 1)
//   derivative        :31-37   (dK/dr = -12/pi r (1 - r^2))
//   pixel position    :39-44   (pixel corner: 2 px / w - 1)
// The integer decisions (centre pixel, radii, ellipse) reproduce the reference bit for bit.
// The real-valued per-pixel offset is evaluated as k * (2/w) + delta, where delta is the
// offset of the centre pixel's corner from the photon, formed in double once per photon;
// the reference forms (2 px / w - 1) - x in float per pixel, which cancels and carries
// ~1e-5 relative error for sub-pixel offsets. Both approximate the same quantity; ours is
// the closer one to the FP64 oracle.
#pragma once

#include <climits>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pds_b200.h"

namespace pds {

constexpr float kThreeOverPi = 0.954929658551372f;     // 3 / pi
constexpr float kTwelveOverPi = 3.819718634205488f;    // 12 / pi

// Record flags (low 4 bits of Rec::packed).
constexpr uint32_t kFlagEllipseAll = 1u;  // :93 test passes for the whole box
constexpr uint32_t kFlagFwdSkip = 2u;     // E <= 0 or NaN: forward deposits nothing (:106)

// Per-photon slot of the plan's inverse map: a sorted position of the tile path, a wide photon
// (kWideBit | index into the wide list), or a photon that touches no pixel.
constexpr uint32_t kWideBit = 0x80000000u;
constexpr uint32_t kInvalidPos = 0xFFFFFFFFu;

// One photon of the tile path, 32 bytes, written once in photon order by the plan kernel
// and gathered by sorted index by the tile kernels.
struct __align__(16) Rec {
    float dx0, dy0;       // corner of the centre pixel minus the photon, normalised units
    float m00, m01, m10, m11;
    float e;              // energy Ep
    uint32_t packed;      // lx:8 | ly:8 | rx:6 | ry:6 | flags:4 (lx, ly: centre pixel in
                          // the tile's apron frame)
};

__host__ __device__ __forceinline__ uint32_t pack_rec(int lx, int ly, int rx, int ry,
                                                      uint32_t flags) {
    return (uint32_t(lx) << 24) | (uint32_t(ly) << 16) | (uint32_t(rx) << 10) |
           (uint32_t(ry) << 4) | flags;
}
__device__ __forceinline__ int rec_lx(uint32_t p) { return int(p >> 24); }
__device__ __forceinline__ int rec_ly(uint32_t p) { return int((p >> 16) & 0xFFu); }
__device__ __forceinline__ int rec_rx(uint32_t p) { return int((p >> 10) & 0x3Fu); }
__device__ __forceinline__ int rec_ry(uint32_t p) { return int((p >> 4) & 0x3Fu); }
__device__ __forceinline__ uint32_t rec_flags(uint32_t p) { return p & 0xFu; }

// Per-photon gradient record of the backward, written in photon order as one 32-byte sector
// (a whole-sector store, no read-for-ownership) and spread into the reference's SoA outputs
// by a coalesced pass.
struct __align__(16) GradRec {
    float gE, gx0, gx1, g00, g01, g10, g11, pad;
};

// Resolved launch configuration (host fills it from pds_config).
struct Cfg {
    int32_t tile;
    int32_t chunk;
    int32_t class_bits;
    int32_t apron;       // min(max_pixel_radius, apron_max), >= 0
    int32_t sw;          // tile + 2 * apron: edge of the shared accumulator
    int32_t spans;       // 1: walk only the support's rows / row spans; 0: the whole box
    int32_t band;        // 1: walk each footprint's sheared band (see Band)
    int32_t rows;        // 1: walk the bands' rows padded to a common count and width per warp
    int32_t min_blocks;  // resident CTAs per SM the forward tile kernels' register budget targets
    int32_t min_blocks_bwd;  // the same for the backward tile kernels
    int32_t coop_r;      // footprint radius from which a photon is splatted by a whole warp
};

// Simulation table: either a device array or one inline descriptor.
struct SimTable {
    const pds_sim* dev;
    int32_t n;
    pds_sim one;
};

__device__ __forceinline__ pds_sim load_sim(const SimTable& t, int s) {
    if (t.dev == nullptr) return t.one;
    return t.dev[s];
}

// Simulation owning photon i (photons of a simulation are contiguous).
__device__ __forceinline__ int find_sim_of_photon(const SimTable& t, int64_t i) {
    if (t.dev == nullptr) return 0;
    int lo = 0, hi = t.n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(&t.dev[mid].photon_begin) <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// First photon after simulation s (the next simulation's photon_begin; no limit for the last).
__device__ __forceinline__ int64_t sim_end(const SimTable& t, int s) {
    if (t.dev == nullptr || s + 1 >= t.n) return INT64_MAX;
    return __ldg(&t.dev[s + 1].photon_begin);
}

// Simulation owning global tile id g.
__device__ __forceinline__ int find_sim_of_tile(const SimTable& t, int64_t g) {
    if (t.dev == nullptr) return 0;
    int lo = 0, hi = t.n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(&t.dev[mid].tile_base) <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Footprint of one photon (photon_differentials.cu:76-87), integer part exact.
struct Footprint {
    int32_t px_c, py_c, rx, ry;
    bool ellipse_all;
};

// The :93 test for one offset, evaluated exactly as the reference does (int32 square,
// float conversion, double division and sum).
__device__ __forceinline__ bool ellipse_ok(int32_t xo, int32_t yo, double w, double h) {
    const float fx = float(int32_t(uint32_t(xo) * uint32_t(xo)));
    const float fy = float(int32_t(uint32_t(yo) * uint32_t(yo)));
    return double(fx) / (0.25 * w * w) + double(fy) / (0.25 * h * h) <= 1.0;
}

__device__ __forceinline__ Footprint make_footprint(float x, float y, float r, int32_t H,
                                                    int32_t W, int32_t mpr) {
    Footprint f;
    const double w = double(float(W)), h = double(float(H));
    // __double2int_rz: truncation with saturation, NaN -> 0 (the GPU semantics of the
    // reference's int32_t(...) casts).
    const int32_t rx = __double2int_rz(ceil(double(r) * 0.5 * w));
    const int32_t ry = __double2int_rz(ceil(double(r) * 0.5 * h));
    f.rx = min(rx, mpr);
    f.ry = min(ry, mpr);
    f.px_c = __double2int_rz((0.5 * double(x) + 0.5) * w);
    f.py_c = __double2int_rz((0.5 * double(y) + 0.5) * h);
    // The corner test sums two terms of at most (2 rx / w)^2 and (2 ry / h)^2; with
    // 4 rx <= w and 4 ry <= h it is at most 1/2 and passes without evaluating it.
    if (f.rx < 0 || f.ry < 0)
        f.ellipse_all = true;
    else if (int64_t(f.rx) * 4 <= int64_t(W) && int64_t(f.ry) * 4 <= int64_t(H))
        f.ellipse_all = true;
    else
        f.ellipse_all = ellipse_ok(f.rx, f.ry, w, h);
    return f;
}

// Clipped box in 64-bit arithmetic; false when empty.
__device__ __forceinline__ bool clip_box(const Footprint& f, int32_t H, int32_t W, int32_t& x0,
                                         int32_t& x1, int32_t& y0, int32_t& y1) {
    if (f.rx < 0 || f.ry < 0) return false;
    const int64_t a = max(int64_t(f.px_c) - f.rx, int64_t(0));
    const int64_t b = min(int64_t(f.px_c) + f.rx, int64_t(W) - 1);
    const int64_t c = max(int64_t(f.py_c) - f.ry, int64_t(0));
    const int64_t d = min(int64_t(f.py_c) + f.ry, int64_t(H) - 1);
    if (a > b || c > d) return false;
    x0 = int32_t(a); x1 = int32_t(b); y0 = int32_t(c); y1 = int32_t(d);
    return true;
}

// Rows and per-row column spans of the support |M d| < 1 (d the normalised offset from the
// photon), in pixel offsets from the centre pixel, one pixel wider on each side than the
// float solution so that every pixel whose float s is below 1 is inside. With
// a = |M e_x|^2, b = (M e_x . M e_y) dy, c = |M e_y|^2 dy^2 - 1 the row's support is
// a dx^2 + 2 b dx + c < 0, and the support's half-height is sqrt(a) / |det M|.
// Degenerate, near-singular or non-finite M falls back to the whole box.
struct Support {
    bool on;
    float a, inv_a, bco, cco, ey;
};

__device__ __forceinline__ Support make_support(float m00, float m01, float m10, float m11,
                                                bool enabled) {
    Support g;
    g.on = false;
    if (!enabled) return g;
    const float a = fmaf(m00, m00, m10 * m10);
    const float det = fmaf(m00, m11, -m01 * m10);
    const float ey = sqrtf(a) / fabsf(det);
    if (!(a > 0.f) || !isfinite(a) || !isfinite(ey)) return g;
    // near-singular M: the float determinant has cancelled, so its support size is unreliable
    if (!(fabsf(det) > 1e-3f * (fabsf(m00 * m11) + fabsf(m01 * m10)))) return g;
    g.on = true;
    g.a = a;
    g.inv_a = 1.f / a;
    g.bco = fmaf(m00, m01, m10 * m11);
    g.cco = fmaf(m01, m01, m11 * m11);
    g.ey = ey;
    return g;
}

// Narrows the row range [ky0, ky1] (offsets from the centre pixel) to the support.
__device__ __forceinline__ void support_rows(const Support& g, float dy0, float inv_sy, int& ky0,
                                             int& ky1) {
    if (!g.on) return;
    ky0 = max(ky0, __float2int_ru((-g.ey - dy0) * inv_sy) - 1);
    ky1 = min(ky1, __float2int_rd((g.ey - dy0) * inv_sy) + 1);
}

// Narrows the column range [kx0, kx1] of the row at normalised offset dy; false if empty.
__device__ __forceinline__ bool support_cols(const Support& g, float dy, float dx0, float inv_sx,
                                             int& kx0, int& kx1) {
    if (!g.on) return true;
    const float b = g.bco * dy;
    const float c = fmaf(g.cco * dy, dy, -1.f);
    const float disc = fmaf(b, b, -g.a * c);
    if (!(disc >= 0.f)) return false;
    const float r = sqrtf(disc);
    const float lo = (-b - r) * g.inv_a, hi = (r - b) * g.inv_a;
    kx0 = max(kx0, __float2int_ru((lo - dx0) * inv_sx) - 1);
    kx1 = min(kx1, __float2int_rd((hi - dx0) * inv_sx) + 1);
    return kx0 <= kx1;
}

// Band: the support |M d| < 1 covered by a sheared parallelogram whose rows all have the
// same width. Row ky (pixel offset from the centre pixel) of the support is centred on the
// column alpha + beta ky and at most hw pixels wide on either side (the half-width of the
// row quadratic, sqrt(a - det^2 dy^2) / a, is largest on the centre line: 1 / sqrt(a)); its
// pixels lie in columns xs(ky) .. xs(ky) + bw - 1 with xs = floor(alpha + beta ky - hw) and
// bw = floor(2 hw) + 2. The band is ~4/pi of the support's area (plus a column), where the
// reference's box can be 40 times it for thin rotated footprints. Pixels whose float s is
// below 1 only by rounding at the support's edge may fall outside; they add (1 - s)^2 ~ 0.
// Degenerate, near-singular or non-finite M: on = false (walk the box).
struct Band {
    bool on;
    int ky0, ky1;  // support rows
    float alpha, beta, hw;
    int bw;
};

// The band's geometry only has to be right to within its margins (a column and the rows'
// rounding), so it uses the approximate reciprocal and reciprocal square root.
// max_hw bounds the band's half-width in pixels (the footprint's box radius plus one): an M
// whose support is wider than the box the radius gives takes the box walk, which the radius
// bounds.
__device__ __forceinline__ Band make_band(float m00, float m01, float m10, float m11, float dx0,
                                          float dy0, float sy, float isx, float isy,
                                          float max_hw) {
    Band b;
    b.on = false;
    const float a = fmaf(m00, m00, m10 * m10);
    const float det = fmaf(m00, m11, -m01 * m10);
    if (!(a > 0.f) || !(a < 1e30f)) return b;
    if (!(fabsf(det) > 1e-3f * (fabsf(m00 * m11) + fabsf(m01 * m10)))) return b;
    const float ra = rsqrtf(a);                                // 1 / sqrt(a)
    const float ey = a * ra * __fdividef(1.f, fabsf(det));     // sqrt(a) / |det|
    const float ia = ra * ra;
    b.hw = isx * ra;
    if (!(b.hw <= max_hw) || !(ey * isy < 1e6f)) return b;
    const float bco = fmaf(m00, m01, m10 * m11);
    b.on = true;
    b.ky0 = __float2int_ru((-ey - dy0) * isy);
    b.ky1 = __float2int_rd((ey - dy0) * isy);
    b.alpha = (-bco * dy0 * ia - dx0) * isx;
    b.beta = -bco * sy * isx * ia;
    b.bw = __float2int_rd(2.f * b.hw) + 2;
    return b;
}

__device__ __forceinline__ int band_start(const Band& b, int ky) {
    return __float2int_rd(fmaf(float(ky), b.beta, b.alpha - b.hw));
}

// The rows a photon's band walk visits inside its clipped box [kxb0, kxb1] x [kyb0, kyb1]
// (pixel offsets from the centre pixel): rows ky0 .. ky0 + rows - 1, each w pixels wide and
// starting at the band's start clamped into [kxb0, kxlast]. A clamped row still holds every
// pixel of its support that lies in the box: the support's pixels of row ky are in
// [xs, xs + bw - 1]; clamping slides that window into the box without dropping any of them,
// and when w is the box width the row is the whole box row. Every visited pixel is in the box,
// so the walks need no per-pixel box test.
struct RowWalk {
    int ky0, rows, w, kxb0, kxlast;
};

__device__ __forceinline__ RowWalk row_walk(const Band& b, int kxb0, int kxb1, int kyb0, int kyb1) {
    RowWalk r;
    r.ky0 = max(b.ky0, kyb0);
    r.rows = max(min(b.ky1, kyb1) - r.ky0 + 1, 0);
    r.w = min(b.bw, kxb1 - kxb0 + 1);
    r.kxb0 = kxb0;
    r.kxlast = kxb1 - r.w + 1;
    return r;
}

__device__ __forceinline__ int row_start(const Band& b, const RowWalk& r, int ky) {
    return min(max(band_start(b, ky), r.kxb0), r.kxlast);
}

// Footprint class of the row walk: 3 bits for the row count and 3 for the row width, levels
// 1, 2, 3, 4, 5-6, 7-8, 9-12, 13+ each. Photons of one class have nearly the same rows and
// widths, so a warp of them pads its rows to a common count and width with little waste.
constexpr int kRowClassBits = 6;

__host__ __device__ __forceinline__ uint32_t row_level(int v) {
    return v <= 4 ? uint32_t((v < 1 ? 1 : v) - 1) : (v <= 6 ? 4u : (v <= 8 ? 5u : (v <= 12 ? 6u : 7u)));
}

__host__ __device__ __forceinline__ uint32_t row_class(int rows, int w) {
    return (row_level(rows) << 3) | row_level(w);
}

// The row class of the plan's sort key, from the band's row range and width in IEEE
// round-to-nearest single-precision operations in a fixed order (no contraction, no
// approximate intrinsics), so that a CPU restatement of the binning reproduces every key bit
// for bit. It follows make_band's geometry (the walks themselves use make_band; a photon whose
// rows or width round differently here lands in a neighbouring class, which only changes how
// photons are grouped). kxb0..kyb1: the clipped box in offsets from the centre pixel; the last
// class when the photon takes the generic walk (no band).
__device__ __forceinline__ uint32_t plan_row_class(float m00, float m01, float m10, float m11,
                                                   float dy0, int32_t W, int32_t H, int rx,
                                                   int kxb0, int kxb1, int kyb0, int kyb1) {
    const float a = __fadd_rn(__fmul_rn(m00, m00), __fmul_rn(m10, m10));
    const float p = __fmul_rn(m00, m11), q = __fmul_rn(m01, m10);
    const float det = __fsub_rn(p, q);
    if (!(a > 0.f) || !(a < 1e30f)) return 63u;
    if (!(fabsf(det) > __fmul_rn(1e-3f, __fadd_rn(fabsf(p), fabsf(q))))) return 63u;
    const float isx = __fmul_rn(0.5f, float(W)), isy = __fmul_rn(0.5f, float(H));
    const float sa = __fsqrt_rn(a);
    const float hw = __fdiv_rn(isx, sa);
    const float ey = __fdiv_rn(sa, fabsf(det));
    if (!(hw <= float(rx) + 1.f) || !(__fmul_rn(ey, isy) < 1e6f)) return 63u;
    const int ky0 = int(ceilf(__fmul_rn(__fsub_rn(-ey, dy0), isy)));
    const int ky1 = int(floorf(__fmul_rn(__fsub_rn(ey, dy0), isy)));
    const int bw = int(floorf(__fmul_rn(2.f, hw))) + 2;
    const int rows = max(min(ky1, kyb1) - max(ky0, kyb0) + 1, 0);
    const int w = min(bw, kxb1 - kxb0 + 1);
    return row_class(rows, w);
}

// delta = (2 p_c / w - 1) - x in double (separately rounded operations, in this order),
// rounded once to float.
__device__ __forceinline__ float corner_offset_step(int32_t p_c, double step, float x) {
    return float(__dsub_rn(__dsub_rn(__dmul_rn(double(p_c), step), 1.0), double(x)));
}

// step = 2 / W of corner_offset, for callers that hoist it out of a loop over photons of one
// image (the same correctly rounded division, so the same offsets)
__device__ __forceinline__ double corner_step(int32_t W) { return __ddiv_rn(2.0, double(W)); }

__device__ __forceinline__ float corner_offset(int32_t p_c, int32_t W, float x) {
    return corner_offset_step(p_c, corner_step(W), x);
}

// Predicated shared-memory add without a branch (the compiler otherwise branches around
// the atomic per pixel).
__device__ __forceinline__ void red_shared_add_if(bool p, const float* addr, float v) {
    const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(addr));
    asm volatile(
        "{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q red.shared.add.f32 [%0], %1;\n\t}"
        :: "r"(a), "f"(v), "r"(int(p)) : "memory");
}

// Shared add of v at shared byte address a + OFF when s < 1 (the kernel's support), as one
// predicated reduction: no branch per pixel.
template <int OFF>
__device__ __forceinline__ void red_shared_inside(uint32_t a, float s, float v) {
    asm volatile(
        "{\n\t.reg .pred q;\n\tsetp.lt.f32 q, %1, 0f3F800000;\n\t@q red.shared.add.f32 [%0+%3], %2;\n\t}"
        :: "r"(a), "f"(s), "f"(v), "n"(OFF) : "memory");
}

}  // namespace pds
