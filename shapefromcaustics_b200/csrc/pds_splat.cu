// Photon-differential splatting kernels for sm_100a.
//
// Reference: PyOptix/kernel/photon_differentials.cu. The reference runs one thread per
// photon over its whole footprint box with one global atomicAdd per covered pixel (forward,
// :60-113) and the same walk reading the upstream gradient (backward, :136-221). Here the
// photons come binned by the plan (pds_plan.cu: records in (simulation, channel, screen tile,
// footprint class) order) and
//
//   fwd_tiles_kernel persistent CTAs take fixed-size chunks of the sorted photons from a work
//                    counter; each tile segment is rasterised into a shared-memory accumulator
//                    covering the tile plus an apron of the largest footprint radius, then
//                    flushed with one coalesced pass of global adds over the touched box.
//   bwd_tiles_kernel same walk; the segment's tile+apron of the upstream gradient is staged
//                    in shared memory once, each photon gathers over its footprint from there
//                    and writes one gradient record (no atomics). The per-pixel work is reduced
//                    to the moments sum(t g), sum(t^2 g), sum(t g d), sum(t g d d^T) of the
//                    offset d, from which dL/dE, dL/dx and dL/dM follow by 2x2 algebra.
//   tail kernels     footprints wider than the apron (direct global path, a warp per photon).
//   grad_scatter     gradient records into the reference's SoA outputs, zero for photons that
//                    touch no pixel.
#include <climits>
#include <cstdint>
#include <cuda_runtime.h>

#include "pds_device.cuh"
#include "pds_internal.h"
#include "pds_splat.h"

namespace pds {

namespace {

// ------------------------------------------------------------------ tiles --------------

// Photon counts of the plan, clamped to the photon count so that a workspace without a plan
// cannot send the kernels outside their arrays.
__device__ __forceinline__ int64_t tile_count(const TileArgs& a) {
    return min(int64_t(a.counters[0]), a.ph.n);
}
__device__ __forceinline__ int64_t wide_count(const TileArgs& a) {
    return min(int64_t(a.counters[1]), a.ph.n - tile_count(a));
}

struct TileInfo {
    int64_t img_off;  // element offset of the (simulation, channel) image plane
    bool in_image;    // the plane lies inside the caller's image buffer
    int32_t W, H;
    int32_t ox, oy;   // pixel coordinates of the accumulator's (0, 0)
    float sx, sy;     // 2 / W, 2 / H
    float isx, isy;   // W / 2, H / 2
};

// float(W), float(H) in double: the reference's w, h of the :93 ellipse test
__device__ __forceinline__ double img_wd(const TileInfo& t) { return double(float(t.W)); }
__device__ __forceinline__ double img_hd(const TileInfo& t) { return double(float(t.H)); }

__device__ __forceinline__ TileInfo decode_tile(const SimTable& st, uint32_t tile, const Cfg& cfg,
                                                int64_t image_elems) {
    const int s = find_sim_of_tile(st, tile);
    const pds_sim sim = load_sim(st, s);
    const int32_t local = int32_t(tile) - sim.tile_base;
    const int32_t tx = local % sim.tiles_x;
    const int32_t r = local / sim.tiles_x;
    const int32_t ty = r % sim.tiles_y;
    const int32_t ch = r / sim.tiles_y;
    TileInfo t;
    t.W = sim.width;
    t.H = sim.height;
    t.img_off = sim.image_offset + int64_t(ch) * sim.height * sim.width;
    t.in_image = t.img_off >= 0 && t.img_off + int64_t(sim.height) * sim.width <= image_elems;
    t.ox = tx * cfg.tile - cfg.apron;
    t.oy = ty * cfg.tile - cfg.apron;
    t.sx = float(2.0 / double(sim.width));
    t.sy = float(2.0 / double(sim.height));
    t.isx = 0.5f * float(sim.width);
    t.isy = 0.5f * float(sim.height);
    return t;
}

// One row of a forward deposit: n pixels from shared byte address a, with
// u = (k M00 sx + b0, k M10 sx + b1) at the k-th pixel, s = |u|^2, and a predicated shared add
// of E 3/pi (1 - s)^2 where s < 1 (the reference's value > 0, photon_differentials.cu:105-106).
// Lanes of a warp hold photons of one footprint class, so n is nearly always warp-uniform and
// the loop stays converged; it is unrolled by two.
__device__ __forceinline__ void fwd_row(int n, uint32_t a, float b0, float b1, float a00,
                                        float a10, float e3) {
    float kf = 0.f;
    int k = 0;
    for (; k + 1 < n; k += 2) {
        const float u0 = fmaf(kf, a00, b0), u1 = fmaf(kf, a10, b1);
        const float v0 = u0 + a00, v1 = u1 + a10;
        const float s = fmaf(u0, u0, u1 * u1), s2 = fmaf(v0, v0, v1 * v1);
        const float t = 1.f - s, t2 = 1.f - s2;
        red_shared_inside<0>(a, s, (t * e3) * t);
        red_shared_inside<4>(a, s2, (t2 * e3) * t2);
        a += 8u;
        kf += 2.f;
    }
    if (k < n) {
        const float u0 = fmaf(kf, a00, b0), u1 = fmaf(kf, a10, b1);
        const float s = fmaf(u0, u0, u1 * u1);
        const float t = 1.f - s;
        red_shared_inside<0>(a, s, (t * e3) * t);
    }
}

// Forward deposit of one photon over its band (see Band): one flattened loop over
// rows x bw pixels, so the trip count depends only on the band's area (photons of a warp
// share an area class), the row changing every bw steps. Pixels outside the reference's
// clipped box are masked off (their add is predicated away).
__device__ __forceinline__ void deposit_band(const Rec& r, const Band& bd, const TileInfo& ti,
                                             int sw, uint32_t acc_base, int pxc, int pyc, int x0,
                                             int x1, int y0, int y1) {
    const int ky0 = max(bd.ky0, y0 - pyc), ky1 = min(bd.ky1, y1 - pyc);
    if (ky0 > ky1) return;
    const int kxb0 = x0 - pxc;
    const uint32_t kxspan = uint32_t(x1 - x0);
    const float e3 = r.e * kThreeOverPi;
    const float a00 = r.m00 * ti.sx, a10 = r.m10 * ti.sx;
    const float m01sy = r.m01 * ti.sy, m11sy = r.m11 * ti.sy;
    const float c00 = fmaf(r.m00, r.dx0, r.m01 * r.dy0), c10 = fmaf(r.m10, r.dx0, r.m11 * r.dy0);
    const int bw = bd.bw;
    const int total = (ky1 - ky0 + 1) * bw;
    int ky = ky0, c = 0;
    int xs = band_start(bd, ky);
    float c0 = fmaf(float(ky), m01sy, c00), c1 = fmaf(float(ky), m11sy, c10);
    uint32_t row = acc_base + 4u * uint32_t((pyc + ky - ti.oy) * sw + (pxc - ti.ox));
    for (int q = 0; q < total; ++q) {
        const int kx = xs + c;
        const bool in = uint32_t(kx - kxb0) <= kxspan;
        const float kf = float(kx);
        const float u0 = fmaf(kf, a00, c0), u1 = fmaf(kf, a10, c1);
        const float s = fmaf(u0, u0, u1 * u1);
        const float t = 1.f - s;
        red_shared_inside<0>(row + 4u * uint32_t(kx), in ? s : 2.f, (t * e3) * t);
        if (++c == bw) {
            c = 0;
            ++ky;
            xs = band_start(bd, ky);
            c0 += m01sy;
            c1 += m11sy;
            row += 4u * uint32_t(sw);
        }
    }
}

// Forward deposit of one photon into the shared accumulator (photon_differentials.cu:91-110).
// With spans on, only the support's rows and row spans are visited; the other box pixels
// add exactly zero in the reference (value > 0 fails, :106). Photons that fail the
// reference's image-half-size ellipse test somewhere in their box (tiny images only) take
// the per-pixel test path.
__device__ __forceinline__ void deposit(const Rec& r, const TileInfo& ti, int sw, bool spans,
                                        bool band, float* acc, int& bx0, int& bx1, int& by0,
                                        int& by1) {
    const uint32_t p = r.packed;
    const uint32_t fl = rec_flags(p);
    if (fl & kFlagFwdSkip) return;
    const int pxc = ti.ox + rec_lx(p), pyc = ti.oy + rec_ly(p);
    const int rx = rec_rx(p), ry = rec_ry(p);
    const int x0 = max(pxc - rx, 0), x1 = min(pxc + rx, ti.W - 1);
    const int y0 = max(pyc - ry, 0), y1 = min(pyc + ry, ti.H - 1);
    bx0 = x0; bx1 = x1; by0 = y0; by1 = y1;
    const float e3 = r.e * kThreeOverPi;
    const bool all = fl & kFlagEllipseAll;
    if (band && all) {
        const Band bd = make_band(r.m00, r.m01, r.m10, r.m11, r.dx0, r.dy0, ti.sy, ti.isx, ti.isy,
                                  float(rx) + 1.f);
        if (bd.on) {
            deposit_band(r, bd, ti, sw, static_cast<uint32_t>(__cvta_generic_to_shared(acc)), pxc,
                         pyc, x0, x1, y0, y1);
            return;
        }
    }
    const Support sup = make_support(r.m00, r.m01, r.m10, r.m11, spans && all);
    const float a00 = r.m00 * ti.sx, a10 = r.m10 * ti.sx;
    const float m01sy = r.m01 * ti.sy, m11sy = r.m11 * ti.sy;
    // u at the centre pixel's corner: M (dx0, dy0)
    const float c00 = fmaf(r.m00, r.dx0, r.m01 * r.dy0), c10 = fmaf(r.m10, r.dx0, r.m11 * r.dy0);
    const uint32_t acc_base = static_cast<uint32_t>(__cvta_generic_to_shared(acc));
    int ky0 = y0 - pyc, ky1 = y1 - pyc;
    support_rows(sup, r.dy0, ti.isy, ky0, ky1);
    if (all) {
        // Each lane starts its row walk at a different row: co-located photons in one warp
        // (focused caustics) then add into different rows at the same time instead of
        // serialising on one shared address.
        const int nrows = ky1 - ky0 + 1;
        int ky = nrows > 0 ? ky0 + int(threadIdx.x & 31) % nrows : ky0;
        for (int j = 0; j < nrows; ++j, ky = (ky == ky1) ? ky0 : ky + 1) {
            const float dy = fmaf(float(ky), ti.sy, r.dy0);
            int kx0 = x0 - pxc, kx1 = x1 - pxc;
            if (!support_cols(sup, dy, r.dx0, ti.isx, kx0, kx1)) continue;
            const float kf = float(kx0);
            const float b0 = fmaf(kf, a00, fmaf(float(ky), m01sy, c00));
            const float b1 = fmaf(kf, a10, fmaf(float(ky), m11sy, c10));
            const uint32_t a = acc_base +
                               4u * uint32_t((pyc + ky - ti.oy) * sw + (pxc + kx0 - ti.ox));
            fwd_row(kx1 - kx0 + 1, a, b0, b1, a00, a10, e3);
        }
    } else {
        for (int ky = ky0; ky <= ky1; ++ky) {
            const float dy = fmaf(float(ky), ti.sy, r.dy0);
            const float c0 = fmaf(r.m00, r.dx0, r.m01 * dy);
            const float c1 = fmaf(r.m10, r.dx0, r.m11 * dy);
            const uint32_t arow = acc_base + 4u * uint32_t((pyc + ky - ti.oy) * sw + (pxc - ti.ox));
            for (int kx = x0 - pxc; kx <= x1 - pxc; ++kx) {
                if (!ellipse_ok(kx, ky, img_wd(ti), img_hd(ti))) continue;
                const float u0 = fmaf(float(kx), a00, c0), u1 = fmaf(float(kx), a10, c1);
                const float s = fmaf(u0, u0, u1 * u1);
                const float t = 1.f - s;
                red_shared_inside<0>(arow + 4u * uint32_t(kx), s, (t * e3) * t);
            }
        }
    }
}

// ---- the padded-row walk (walk 4) -------------------------------------------------------
// Each lane holds one photon and walks its band's rows inside the clipped box (RowWalk). The
// warp pads every lane to the warp's largest row count and row width, so all lanes change
// rows on the same iteration and the loops stay converged; the plan's row classes group
// photons of nearly equal rows and widths into a warp, so little of the padding is wasted.
// Along a row, s = |M d|^2 is a quadratic in the column c, stepped by its first and second
// differences (two adds per pixel). Padding pixels (c >= the lane's width, rows past the
// lane's count) are predicated off.

// Per-lane constants of the row walk of one photon.
struct RowGeo {
    float xs0, beta;        // band start of row ky: floor(xs0 + beta ky) (xs0 = alpha - hw)
    int ky0, rows, w;       // rows ky0 .. ky0 + rows - 1 of w pixels (RowWalk)
    int kxb0, kxlast;       // clamp range of the row starts
    int off;                // accumulator index of the centre pixel: (pyc - oy) sw + pxc - ox
    float a00, a10;         // u step per pixel column: M (sx, 0)
    float b0, b1;           // u step per pixel row: M (0, sy)
    float c00, c10;         // u at the centre pixel's corner: M (dx0, dy0)
    float A;                // |M (sx, 0)|^2: half the second difference of s along a row
};

// The clipped box of a record (pixel coordinates) and its centre pixel.
__device__ __forceinline__ void rec_clip(const Rec& r, const TileInfo& ti, int& pxc, int& pyc,
                                         int& x0, int& x1, int& y0, int& y1) {
    const uint32_t p = r.packed;
    pxc = ti.ox + rec_lx(p);
    pyc = ti.oy + rec_ly(p);
    const int rx = rec_rx(p), ry = rec_ry(p);
    x0 = max(pxc - rx, 0);
    x1 = min(pxc + rx, ti.W - 1);
    y0 = max(pyc - ry, 0);
    y1 = min(pyc + ry, ti.H - 1);
}

// Row walk of a record inside its clipped box (x0..y1, from rec_clip); false when the photon
// needs the generic walk (the image-half-size ellipse quirk of tiny images, or an M without a
// band).
__device__ __forceinline__ bool prep_rows(const Rec& r, const TileInfo& ti, int sw, int pxc,
                                          int pyc, int x0, int x1, int y0, int y1, RowGeo& g) {
    if (!(rec_flags(r.packed) & kFlagEllipseAll)) return false;
    const Band band = make_band(r.m00, r.m01, r.m10, r.m11, r.dx0, r.dy0, ti.sy, ti.isx, ti.isy,
                                float(rec_rx(r.packed)) + 1.f);
    if (!band.on) return false;
    const RowWalk rw = row_walk(band, x0 - pxc, x1 - pxc, y0 - pyc, y1 - pyc);
    g.xs0 = band.alpha - band.hw;
    g.beta = band.beta;
    g.ky0 = rw.ky0;
    g.rows = rw.rows;
    g.w = rw.w;
    g.kxb0 = rw.kxb0;
    g.kxlast = rw.kxlast;
    g.off = (pyc - ti.oy) * sw + (pxc - ti.ox);
    g.a00 = r.m00 * ti.sx;
    g.a10 = r.m10 * ti.sx;
    g.b0 = r.m01 * ti.sy;
    g.b1 = r.m11 * ti.sy;
    g.c00 = fmaf(r.m00, r.dx0, r.m01 * r.dy0);
    g.c10 = fmaf(r.m10, r.dx0, r.m11 * r.dy0);
    g.A = fmaf(g.a00, g.a00, g.a10 * g.a10);
    return true;
}

// First column of row ky (band start clamped into the box), s and its first difference there.
__device__ __forceinline__ int row_begin(const RowGeo& g, int ky, float& s, float& d) {
    const float kyf = float(ky);
    const int xs = min(max(__float2int_rd(fmaf(kyf, g.beta, g.xs0)), g.kxb0), g.kxlast);
    const float kxf = float(xs);
    const float u0 = fmaf(kxf, g.a00, fmaf(kyf, g.b0, g.c00));
    const float u1 = fmaf(kxf, g.a10, fmaf(kyf, g.b1, g.c10));
    s = fmaf(u0, u0, u1 * u1);
    d = fmaf(2.f, fmaf(u0, g.a00, u1 * g.a10), g.A);  // s(c + 1) - s(c) at c = 0
    return xs;
}

// Shared add of v at shared byte address a + OFF when c < w and s < 1, as one predicated
// reduction.
template <int OFF>
__device__ __forceinline__ void red_row(uint32_t a, float s, float v, int c, int w) {
    asm volatile(
        "{\n\t.reg .pred q;\n\tsetp.lt.s32 q, %3, %4;\n\t"
        "setp.lt.and.f32 q, %1, 0f3F800000, q;\n\t@q red.shared.add.f32 [%0+%5], %2;\n\t}"
        :: "r"(a), "f"(s), "f"(v), "r"(c), "r"(w), "n"(OFF) : "memory");
}

// Shared load of the float at shared byte address a when c < w, else 0.
__device__ __forceinline__ float lds_row(uint32_t a, int c, int w) {
    float v;
    asm volatile(
        "{\n\t.reg .pred q;\n\tsetp.lt.s32 q, %2, %3;\n\tmov.b32 %0, 0;\n\t"
        "@q ld.shared.f32 %0, [%1];\n\t}"
        : "=f"(v) : "r"(a), "r"(c), "r"(w) : "memory");
    return v;
}

// Forward deposit of the warp's photons by padded rows. rows = 0 for lanes with nothing to
// walk (their g is not read). Lanes start at rotated rows (lane mod rows), so co-located
// photons of a caustic add into different rows, and so different banks, at the same time.
// Every lane of the warp calls it.
__device__ __forceinline__ void deposit_rows(const RowGeo& g, int rows, float e3, uint32_t acc_base,
                                             int sw) {
    const int rm = __reduce_max_sync(0xFFFFFFFFu, rows);
    if (rm == 0) return;
    const int wm = __reduce_max_sync(0xFFFFFFFFu, rows > 0 ? g.w : 0);
    const int rot = rows > 1 ? int(threadIdx.x & 31) % rows : 0;
    const float dd = 2.f * g.A;
    for (int j = 0; j < rm; ++j) {
        const int wl = j < rows ? g.w : 0;
        int jj = j + rot;
        jj = jj >= rows ? jj - rows : jj;
        const int ky = g.ky0 + jj;
        float s, d;
        const int xs = row_begin(g, ky, s, d);
        uint32_t a = acc_base + 4u * uint32_t(g.off + ky * sw + xs);
        int c = 0;
        for (; c + 2 <= wm; c += 2) {
            const float t = 1.f - s;
            red_row<0>(a, s, (t * e3) * t, c, wl);
            s += d;
            d += dd;
            const float t2 = 1.f - s;
            red_row<4>(a, s, (t2 * e3) * t2, c + 1, wl);
            s += d;
            d += dd;
            a += 8u;
        }
        if (c < wm) {
            const float t = 1.f - s;
            red_row<0>(a, s, (t * e3) * t, c, wl);
        }
    }
}

// Backward moments of the warp's photons by padded rows (no rotation: the gathers read).
// Per row it keeps sum t g, sum t g c and sum t g c^2 over the row's columns c and folds them
// into the photon's moments in the integer x offset kx = xs + c and the normalised y offset,
// as gather_band_rows does. Every lane of the warp calls it.
struct RowMoments {
    float sE, A0t, B1t, B2t, Sy, Sxy, Syy;
};

__device__ __forceinline__ RowMoments gather_rows(const RowGeo& g, int rows, uint32_t tg_base,
                                                 int sw, float sy, float dy0) {
    RowMoments m = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const int rm = __reduce_max_sync(0xFFFFFFFFu, rows);
    if (rm == 0) return m;
    const int wm = __reduce_max_sync(0xFFFFFFFFu, rows > 0 ? g.w : 0);
    const float dd = 2.f * g.A;
    for (int j = 0; j < rm; ++j) {
        const bool act = j < rows;
        const int wl = act ? g.w : 0;
        const int ky = g.ky0 + j;
        float s, d;
        const int xs = row_begin(g, ky, s, d);
        // lanes without this row read nothing (their address is not formed from their rows)
        uint32_t a = act ? tg_base + 4u * uint32_t(g.off + ky * sw + xs) : tg_base;
        float A0 = 0.f, Bc = 0.f, Bcc = 0.f, sEr = 0.f, cf = 0.f;
        int c = 0;
        for (; c + 2 <= wm; c += 2) {
            const float q0 = lds_row(a, c, wl);
            const float q1 = lds_row(a + 4u, c + 1, wl);
            const float t0 = fmaxf(1.f - s, 0.f);
            s += d;
            d += dd;
            const float t1 = fmaxf(1.f - s, 0.f);
            s += d;
            d += dd;
            const float g0 = t0 * q0, g1 = t1 * q1;
            sEr = fmaf(t0, g0, sEr);
            sEr = fmaf(t1, g1, sEr);
            A0 += g0 + g1;
            const float h0 = g0 * cf, h1 = g1 * (cf + 1.f);
            Bc += h0 + h1;
            Bcc = fmaf(h0, cf, Bcc);
            Bcc = fmaf(h1, cf + 1.f, Bcc);
            cf += 2.f;
            a += 8u;
        }
        if (c < wm) {
            const float q0 = lds_row(a, c, wl);
            const float t0 = fmaxf(1.f - s, 0.f);
            const float g0 = t0 * q0;
            sEr = fmaf(t0, g0, sEr);
            A0 += g0;
            const float h0 = g0 * cf;
            Bc += h0;
            Bcc = fmaf(h0, cf, Bcc);
        }
        // sum g kx and sum g kx^2 with kx = xs + c
        const float xf = float(xs);
        const float B1 = fmaf(xf, A0, Bc);
        const float B2 = fmaf(xf, fmaf(xf, A0, 2.f * Bc), Bcc);
        const float dy = fmaf(float(ky), sy, dy0);
        m.sE += sEr;
        m.A0t += A0;
        m.B1t += B1;
        m.B2t += B2;
        m.Sy = fmaf(dy, A0, m.Sy);
        m.Syy = fmaf(dy * dy, A0, m.Syy);
        m.Sxy = fmaf(dy, B1, m.Sxy);  // sum g kx dy; finish_rows adds the dx0 part
    }
    return m;
}


// Photons with a footprint radius of at least cfg.coop_r are splatted by their whole warp:
// lane j takes rows j, j + 32, ... of the photon and walks each row's span of the support
// (|M d| < 1 solved per row, one pixel of margin) rather than the whole box row. Large and
// thin footprints then cost about their support area, co-located photons of a caustic no
// longer make a warp's lanes add into one shared address at once, and with an odd
// accumulator pitch the 32 rows of one column fall in 32 different banks.
__device__ __forceinline__ bool use_coop(const Rec& r, int coop_r) {
    const uint32_t p = r.packed;
    const uint32_t fl = rec_flags(p);
    return coop_r > 0 && (fl & kFlagEllipseAll) && !(fl & kFlagFwdSkip) &&
           (rec_rx(p) >= coop_r || rec_ry(p) >= coop_r);
}

// Records of the next batch of photons are copied global -> shared asynchronously while the
// current batch is splatted (two buffers of kTileThreads records after the tile's shared
// region). Each thread copies and later reads only its own slot, so no barrier is needed:
// cp.async.wait_group makes the thread's own copies visible to it.
__device__ __forceinline__ int stage_offset_floats(int sw) { return (sw * sw + 3) & ~3; }

__device__ __forceinline__ void stage_rec_async(Rec* dst, const Rec* src) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    const char* g = reinterpret_cast<const char*>(src);
    asm volatile(
        "cp.async.cg.shared.global [%0], [%1], 16;\n\t"
        "cp.async.cg.shared.global [%2], [%3], 16;"
        :: "r"(d), "l"(g), "r"(d + 16u), "l"(g + 16) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

__device__ __forceinline__ Rec shfl_rec(const Rec& r, int src) {
    Rec o;
    o.dx0 = __shfl_sync(0xFFFFFFFFu, r.dx0, src);
    o.dy0 = __shfl_sync(0xFFFFFFFFu, r.dy0, src);
    o.m00 = __shfl_sync(0xFFFFFFFFu, r.m00, src);
    o.m01 = __shfl_sync(0xFFFFFFFFu, r.m01, src);
    o.m10 = __shfl_sync(0xFFFFFFFFu, r.m10, src);
    o.m11 = __shfl_sync(0xFFFFFFFFu, r.m11, src);
    o.e = __shfl_sync(0xFFFFFFFFu, r.e, src);
    o.packed = __shfl_sync(0xFFFFFFFFu, r.packed, src);
    return o;
}

// Clipped box of a record in pixel coordinates.
__device__ __forceinline__ void rec_box(const Rec& r, const TileInfo& ti, int& pxc, int& pyc,
                                        int& x0, int& x1, int& y0, int& y1) {
    const uint32_t p = r.packed;
    pxc = ti.ox + rec_lx(p);
    pyc = ti.oy + rec_ly(p);
    const int rx = rec_rx(p), ry = rec_ry(p);
    x0 = max(pxc - rx, 0);
    x1 = min(pxc + rx, ti.W - 1);
    y0 = max(pyc - ry, 0);
    y1 = min(pyc + ry, ti.H - 1);
}

// Forward deposit of one photon by the whole warp (see use_coop).
__device__ __forceinline__ void deposit_coop(const Rec& r, const TileInfo& ti, int sw,
                                             uint32_t acc_base, int lane) {
    int pxc, pyc, x0, x1, y0, y1;
    rec_box(r, ti, pxc, pyc, x0, x1, y0, y1);
    const float e3 = r.e * kThreeOverPi;
    const float a00 = r.m00 * ti.sx, a10 = r.m10 * ti.sx;
    const float m01sy = r.m01 * ti.sy, m11sy = r.m11 * ti.sy;
    const float c00 = fmaf(r.m00, r.dx0, r.m01 * r.dy0), c10 = fmaf(r.m10, r.dx0, r.m11 * r.dy0);
    const Support sup = make_support(r.m00, r.m01, r.m10, r.m11, true);
    int ky0 = y0 - pyc, ky1 = y1 - pyc;
    support_rows(sup, r.dy0, ti.isy, ky0, ky1);
    for (int ky = ky0 + lane; ky <= ky1; ky += 32) {
        const float dy = fmaf(float(ky), ti.sy, r.dy0);
        int kx0 = x0 - pxc, kx1 = x1 - pxc;
        if (!support_cols(sup, dy, r.dx0, ti.isx, kx0, kx1)) continue;
        const float kf = float(kx0);
        const float b0 = fmaf(kf, a00, fmaf(float(ky), m01sy, c00));
        const float b1 = fmaf(kf, a10, fmaf(float(ky), m11sy, c10));
        const uint32_t a = acc_base + 4u * uint32_t((pyc + ky - ti.oy) * sw + (pxc + kx0 - ti.ox));
        fwd_row(kx1 - kx0 + 1, a, b0, b1, a00, a10, e3);
    }
}

__device__ __forceinline__ void bbox_publish(int* sb, int x0, int x1, int y0, int y1) {
    x0 = __reduce_min_sync(0xFFFFFFFFu, x0);
    x1 = __reduce_max_sync(0xFFFFFFFFu, x1);
    y0 = __reduce_min_sync(0xFFFFFFFFu, y0);
    y1 = __reduce_max_sync(0xFFFFFFFFu, y1);
    if ((threadIdx.x & 31) == 0 && x0 <= x1) {
        atomicMin(sb + 0, x0);
        atomicMax(sb + 1, x1);
        atomicMin(sb + 2, y0);
        atomicMax(sb + 3, y1);
    }
}

// Adds the touched box of the accumulator into the image and clears it: warps take rows,
// lanes take consecutive columns. When image rows are 16-byte aligned the adds are 4-wide
// vector reductions (red.global.add.v4.f32) over 4-aligned column groups; columns of a group
// outside the touched box add zero. All-zero groups are skipped.
__device__ __forceinline__ void flush_tile(float* acc, int sw, const TileInfo& ti, float* out,
                                           int* sb) {
    __syncthreads();
    const int x0 = sb[0], x1 = sb[1], y0 = sb[2], y1 = sb[3];
    __syncthreads();
    if (threadIdx.x == 0) {
        sb[0] = INT_MAX; sb[1] = INT_MIN; sb[2] = INT_MAX; sb[3] = INT_MIN;
    }
    if (x0 <= x1 && !ti.in_image) {
        // a plane outside the caller's buffer (an inconsistent simulation table): clear only
        for (int gy = y0 + int(threadIdx.x >> 5); gy <= y1; gy += int(blockDim.x >> 5)) {
            float* arow = acc + (gy - ti.oy) * sw - ti.ox;
            for (int gx = x0 + int(threadIdx.x & 31); gx <= x1; gx += 32) arow[gx] = 0.f;
        }
    } else if (x0 <= x1) {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int nw = blockDim.x >> 5;
        float* img = out + ti.img_off;
        const bool vec = (ti.W & 3) == 0 && (reinterpret_cast<uintptr_t>(img) & 15) == 0;
        if (vec) {
            const int g0 = x0 >> 2, g1 = x1 >> 2;
            for (int gy = y0 + warp; gy <= y1; gy += nw) {
                float* arow = acc + (gy - ti.oy) * sw - ti.ox;
                float* grow = img + int64_t(gy) * ti.W;
                for (int g = g0 + lane; g <= g1; g += 32) {
                    const int gx = g << 2;
                    float v[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int c = gx + j;
                        v[j] = 0.f;
                        if (c >= x0 && c <= x1) {
                            v[j] = arow[c];
                            arow[c] = 0.f;
                        }
                    }
                    if (v[0] != 0.f || v[1] != 0.f || v[2] != 0.f || v[3] != 0.f)
                        atomicAdd(reinterpret_cast<float4*>(grow + gx),
                                  make_float4(v[0], v[1], v[2], v[3]));
                }
            }
        } else {
            for (int gy = y0 + warp; gy <= y1; gy += nw) {
                float* arow = acc + (gy - ti.oy) * sw - ti.ox;
                float* grow = img + int64_t(gy) * ti.W;
                for (int gx = x0 + lane; gx <= x1; gx += 32) {
                    const float v = arow[gx];
                    if (v != 0.f) {
                        atomicAdd(grow + gx, v);
                        arow[gx] = 0.f;
                    }
                }
            }
        }
    }
    __syncthreads();
}

// A run of sorted positions [begin, end) holding one screen tile's photons.
struct Segment {
    uint32_t tile;
    int64_t begin, end;
};

// End of tile t's photons: the start of its successor's first bucket.
__device__ __forceinline__ int64_t tile_end(const TileArgs& a, int64_t t) {
    return int64_t(__ldg(a.start + ((t + 1) << a.cfg.class_bits)));
}

__device__ __forceinline__ Segment first_segment(const TileArgs& a, int64_t chunk, int64_t p0) {
    Segment s;
    // (clamped, like the counters, so that a workspace without a plan stays in its arrays)
    s.tile = uint32_t(min(int64_t(__ldg(a.chunk_tile + chunk)), a.n_tiles - 1));
    s.begin = p0;
    s.end = tile_end(a, s.tile);
    return s;
}

// The segment after sg (sg.end below the tile path's photon count): the first tile after
// sg.tile whose range is not empty, found by doubling steps then bisection (empty tiles are
// usually few, so one probe mostly suffices). Every thread computes it from the same loads.
__device__ __forceinline__ Segment next_segment(const TileArgs& a, const Segment& sg) {
    const int64_t p = sg.end, t = sg.tile, last = a.n_tiles - 1;
    int64_t k = 1;
    while (t + k < last && tile_end(a, t + k) <= p) k <<= 1;
    int64_t lo = t + (k >> 1) + 1, hi = min(t + k, last);
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (tile_end(a, mid) > p) hi = mid; else lo = mid + 1;
    }
    Segment s;
    s.tile = uint32_t(lo);
    s.begin = p;
    s.end = tile_end(a, lo);
    return s;
}

// Next chunk of sorted photons for this CTA: a shared work counter (reset to zero before the
// launch) hands chunks out in order as CTAs finish, so CTAs that drew chunks of large
// footprints do not hold up the others. Nothing waits on it.
__device__ __forceinline__ int64_t next_chunk(uint32_t* queue, uint32_t* slot) {
    __syncthreads();
    if (threadIdx.x == 0) *slot = atomicAdd(queue, 1u);
    __syncthreads();
    return int64_t(*slot);
}

template <int NT, int MINB>
__global__ __launch_bounds__(NT, MINB) void fwd_tiles_kernel(TileArgs a) {
    extern __shared__ float acc[];
    __shared__ int sb[4];
    const Cfg cfg = a.cfg;
    const int sw = cfg.sw;
    Rec* stage = reinterpret_cast<Rec*>(acc + stage_offset_floats(sw));
    for (int k = threadIdx.x; k < sw * sw; k += NT) acc[k] = 0.f;
    if (threadIdx.x == 0) {
        sb[0] = INT_MAX; sb[1] = INT_MIN; sb[2] = INT_MAX; sb[3] = INT_MIN;
    }
    __syncthreads();
    const uint32_t acc_base = static_cast<uint32_t>(__cvta_generic_to_shared(acc));
    const int64_t n_tile = tile_count(a);
    const int64_t nchunks = (n_tile + cfg.chunk - 1) / cfg.chunk;
    __shared__ uint32_t chunk_slot;
    for (int64_t c = next_chunk(a.queue, &chunk_slot); c < nchunks;
         c = next_chunk(a.queue, &chunk_slot)) {
        const int64_t p0 = c * cfg.chunk, p1 = min(p0 + cfg.chunk, n_tile);
        if (p0 + threadIdx.x < p1) stage_rec_async(stage + threadIdx.x, a.srecs + p0 + threadIdx.x);
        cp_async_commit();
        Segment sg = first_segment(a, c, p0);
        TileInfo ti = decode_tile(a.sims, sg.tile, cfg, a.image_elems);
        int buf = 0;
        for (int64_t base = p0; base < p1; base += NT, buf ^= 1) {
            const int64_t i = base + threadIdx.x;
            const bool have = i < p1;
            cp_async_wait_all();
            Rec r = {};
            if (have) r = stage[buf * NT + threadIdx.x];
            if (i + NT < p1) stage_rec_async(stage + (buf ^ 1) * NT + threadIdx.x, a.srecs + i + NT);
            cp_async_commit();
            const int64_t bend = min(base + NT, p1);
            // The batch's segments (runs of one tile) are consecutive thread ranges; each
            // pass handles one and flushes the tile's accumulator when the next one starts.
            // Every pass but the first covers at least one photon, so NT + 1 passes suffice.
            for (int pass = 0; pass <= NT; ++pass) {
                const bool mine = have && i >= sg.begin && i < sg.end;
                const bool coop = mine && use_coop(r, cfg.coop_r);
                int x0 = INT_MAX, x1 = INT_MIN, y0 = INT_MAX, y1 = INT_MIN;
                if (mine && !coop) deposit(r, ti, sw, cfg.spans, cfg.band, acc, x0, x1, y0, y1);
                if (coop) {
                    int pxc, pyc;
                    rec_box(r, ti, pxc, pyc, x0, x1, y0, y1);
                }
                for (uint32_t cm = __ballot_sync(0xFFFFFFFFu, coop); cm; cm &= cm - 1) {
                    const Rec rb = shfl_rec(r, __ffs(cm) - 1);
                    deposit_coop(rb, ti, sw, acc_base, threadIdx.x & 31);
                }
                bbox_publish(sb, x0, x1, y0, y1);
                if (sg.end >= bend) break;
                flush_tile(acc, sw, ti, a.out, sb);
                sg = next_segment(a, sg);
                ti = decode_tile(a.sims, sg.tile, cfg, a.image_elems);
            }
        }
        flush_tile(acc, sw, ti, a.out, sb);
    }
}

// Stages the upstream gradient that a tile's photons read (clipped to the image): the tile and
// the pixels within r of it, r the largest box radius of the tile's photons (the plan's
// tile_r, at most the apron), and the column after them (the band walk reads, and discards,
// the pixel after an odd row's end; the pitch sw = tile + 2 apron + 1 has room for it). The
// apron's outer margin, which no photon of the tile reaches, is not loaded. Warps take rows,
// lanes take consecutive columns.
__device__ __forceinline__ void load_region(float* tg, int sw, const TileInfo& ti,
                                            const float* grad, int apron, uint32_t r) {
    const int m = apron - int(min(r, uint32_t(apron)));
    const int gx0 = max(ti.ox + m, 0), gx1 = min(ti.ox + sw - m, ti.W);
    const int gy0 = max(ti.oy + m, 0), gy1 = min(ti.oy + sw - m, ti.H);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nw = blockDim.x >> 5;
    const float* img = grad + ti.img_off;
    for (int gy = gy0 + warp; gy < gy1; gy += nw) {
        float* trow = tg + (gy - ti.oy) * sw - ti.ox;
        const float* grow = img + int64_t(gy) * ti.W;
        for (int gx = gx0 + lane; gx < gx1; gx += 32)
            trow[gx] = ti.in_image ? __ldg(grow + gx) : 0.f;
    }
}

__device__ __forceinline__ void store_grad(GradRec* stage, uint32_t rid, float gE, float gx0,
                                           float gx1, float g00, float g01, float g10,
                                           float g11) {
    float4* d = reinterpret_cast<float4*>(stage + rid);
    d[0] = make_float4(gE, gx0, gx1, g00);
    d[1] = make_float4(g01, g10, g11, 0.f);
}

// The moments of one photon turned into its gradients. With a = -12/pi E t g (the
// reference's d_silverman(r) E g / r, :193), sums over the support of
//   S  = sum t^2 g,  Sd = sum t g d,  Sdd = sum t g d d^T  (d the normalised offset)
// give  dL/dE = 3/pi S,  dL/dx = -M^T (c M Sd),  dL/dM = c M Sdd  with c = -12/pi E
// (:195-205 summed over the pixels; u = M d).
__device__ __forceinline__ void finish_grad(GradRec* stage, uint32_t rid, float e, float m00,
                                            float m01, float m10, float m11, float sE, float Sx,
                                            float Sy, float Sxx, float Sxy, float Syy) {
    const float c = -kTwelveOverPi * e;
    const float v0 = c * fmaf(m00, Sx, m01 * Sy);
    const float v1 = c * fmaf(m10, Sx, m11 * Sy);
    store_grad(stage, rid, kThreeOverPi * sE, -fmaf(m00, v0, m10 * v1),
               -fmaf(m01, v0, m11 * v1), c * fmaf(m00, Sxx, m01 * Sxy),
               c * fmaf(m00, Sxy, m01 * Syy), c * fmaf(m10, Sxx, m11 * Sxy),
               c * fmaf(m10, Sxy, m11 * Syy));
}

// The gradients of one photon from its row moments: sum g dx = sx B1t + dx0 A0t and
// sum g dx dy = sx (sum g kx dy) + dx0 Sy, with dx = kx sx + dx0.
__device__ __forceinline__ void finish_rows(GradRec* stage, uint32_t slot, const Rec& r,
                                            const TileInfo& ti, const RowMoments& m) {
    const float Sx = fmaf(ti.sx, m.B1t, r.dx0 * m.A0t);
    const float Sxx = fmaf(ti.sx * ti.sx, m.B2t,
                           fmaf(2.f * ti.sx * r.dx0, m.B1t, r.dx0 * r.dx0 * m.A0t));
    const float Sxy = fmaf(ti.sx, m.Sxy, r.dx0 * m.Sy);
    finish_grad(stage, slot, r.e, r.m00, r.m01, r.m10, r.m11, m.sE, Sx, m.Sy, Sxx, Sxy, m.Syy);
}

// One row of a backward gather: n pixels from q, the first at pixel offset k0 (relative to
// the centre pixel). With t = max(1 - s, 0) and g the upstream gradient it accumulates
// sum t^2 g, and over the row sum t g and sum t g k (k the pixel offset); the caller folds
// those into the photon's moments. Unrolled by two; n is nearly always warp-uniform.
__device__ __forceinline__ void bwd_row(int n, const float* q, float k0, float b0, float b1,
                                        float a00, float a10, float& sE, float& A0, float& B1,
                                        float& B2) {
    float kf = 0.f;
    int k = 0;
    for (; k + 1 < n; k += 2) {
        const float u0 = fmaf(kf, a00, b0), u1 = fmaf(kf, a10, b1);
        const float v0 = u0 + a00, v1 = u1 + a10;
        const float s = fmaf(u0, u0, u1 * u1), s2 = fmaf(v0, v0, v1 * v1);
        const float t = fmaxf(1.f - s, 0.f), t2 = fmaxf(1.f - s2, 0.f);
        const float g = t * q[k], g2 = t2 * q[k + 1];
        const float kk = k0 + kf;
        sE = fmaf(t, g, sE);
        sE = fmaf(t2, g2, sE);
        A0 += g + g2;
        const float tk = g * kk, tk2 = g2 * (kk + 1.f);
        B1 += tk + tk2;
        B2 = fmaf(tk, kk, B2);
        B2 = fmaf(tk2, kk + 1.f, B2);
        kf += 2.f;
    }
    if (k < n) {
        const float u0 = fmaf(kf, a00, b0), u1 = fmaf(kf, a10, b1);
        const float s = fmaf(u0, u0, u1 * u1);
        const float t = fmaxf(1.f - s, 0.f);
        const float g = t * q[k];
        const float kk = k0 + kf;
        sE = fmaf(t, g, sE);
        A0 += g;
        const float tk = g * kk;
        B1 += tk;
        B2 = fmaf(tk, kk, B2);
    }
}

// The backward walks the band inside the clipped box. A row is w = min(bw rounded up to
// even, box width) pixels wide and starts at the band's start clamped into
// [kxb0, kxb1 - w + 1]. A clamped row still holds every pixel of its support that lies in the
// box (the support's pixels of row ky are in [xs, xs + bw - 1]; clamping slides that window
// into the box without dropping any of them, and when w is the box width the row is the whole
// box row), so no pixel needs an in-box test. Rows are walked two pixels at a time; when w is
// odd, the second pixel of each row's last pair lies just outside the box and is masked.
struct BandWalk {
    int w, npairs, tail, kxb0, kxlast;
};

__device__ __forceinline__ BandWalk band_walk(const Band& bd, int kxb0, int kxb1) {
    BandWalk b;
    b.w = min((bd.bw + 1) & ~1, kxb1 - kxb0 + 1);
    b.npairs = (b.w + 1) >> 1;
    b.tail = b.w & 1;  // value of the remaining-pair count at which the mask applies
    b.kxb0 = kxb0;
    b.kxlast = kxb1 - b.w + 1;
    return b;
}

__device__ __forceinline__ int band_row_start(const Band& bd, const BandWalk& bw, int ky) {
    return min(max(band_start(bd, ky), bw.kxb0), bw.kxlast);
}

// Backward moments over the band rows ky0..ky1 (ky0 <= ky1). Per row it keeps sum t g and
// sum t g kx (kx the integer pixel offset) and folds them into the y moments at the row
// change; sum t g kx^2 and sum t^2 g run over the whole band. The masked pixel of an odd row
// (just outside the box) is read from the staged tile's spare column (the pitch is odd:
// tile + 2 apron + 1, and a box never reaches past column tile + 2 apron - 1) and its product
// discarded. The two pixels of a step are evaluated as the two lanes of sm_100's packed FP32
// instructions (__ffma2_rn / __fmul2_rn / __fadd2_rn: one instruction for both pixels, each
// lane rounded as its scalar counterpart); the even and odd pixels keep separate partial sums,
// added where a row or the band ends.
struct BandMoments {
    float sE, A0t, B1t, B2, Sy, Sxy, Syy;
};

__device__ __forceinline__ float2 pair(float v) { return make_float2(v, v); }
__device__ __forceinline__ float hsum(float2 v) { return v.x + v.y; }

__device__ __forceinline__ BandMoments gather_band_rows(const Band& bd, const BandWalk& bw,
                                                        int ky, int ky1, const float* row,
                                                        int sw, float a00, float a10, float c0,
                                                        float c1, float m01sy, float m11sy,
                                                        float sy, float dy0, float sx,
                                                        float dx0) {
    BandMoments m = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    const float2 A00 = pair(a00), A10 = pair(a10);
    float2 C0 = pair(c0), C1 = pair(c1);
    float2 SE = pair(0.f), B2 = pair(0.f), A0 = pair(0.f), B1 = pair(0.f);
    int xs = band_row_start(bd, bw, ky);
    float2 KF = make_float2(float(xs), float(xs + 1));
    const float* q = row + xs;
    int rem = bw.npairs;
    for (;;) {
        // u = M d at the two pixels, s = |u|^2, t = max(1 - s, 0)
        const float2 U0 = __ffma2_rn(KF, A00, C0), U1 = __ffma2_rn(KF, A10, C1);
        const float2 S = __ffma2_rn(U0, U0, __fmul2_rn(U1, U1));
        const float2 T = make_float2(fmaxf(1.f - S.x, 0.f), fmaxf(1.f - S.y, 0.f));
        const float2 Q = make_float2(q[0], rem == bw.tail ? 0.f : q[1]);
        const float2 G = __fmul2_rn(T, Q);
        SE = __ffma2_rn(T, G, SE);
        A0 = __fadd2_rn(A0, G);
        const float2 TK = __fmul2_rn(G, KF);
        B1 = __fadd2_rn(B1, TK);
        B2 = __ffma2_rn(TK, KF, B2);
        KF = __fadd2_rn(KF, pair(2.f));
        q += 2;
        if (--rem == 0) {
            const float a0 = hsum(A0), b1 = hsum(B1);
            const float dy = fmaf(float(ky), sy, dy0);
            const float sdx = fmaf(sx, b1, dx0 * a0);
            m.Sy = fmaf(dy, a0, m.Sy);
            m.Sxy = fmaf(dy, sdx, m.Sxy);
            m.Syy = fmaf(dy * dy, a0, m.Syy);
            m.A0t += a0;
            m.B1t += b1;
            if (++ky > ky1) break;
            A0 = pair(0.f);
            B1 = pair(0.f);
            rem = bw.npairs;
            xs = band_row_start(bd, bw, ky);
            KF = make_float2(float(xs), float(xs + 1));
            C0 = __fadd2_rn(C0, pair(m01sy));
            C1 = __fadd2_rn(C1, pair(m11sy));
            row += sw;
            q = row + xs;
        }
    }
    m.sE = hsum(SE);
    m.B2 = hsum(B2);
    return m;
}

// Backward gather of one photon over its band rows ky0..ky1 (see BandWalk); with no row
// inside the box (ky0 > ky1) its gradients are zero.
__device__ __forceinline__ void gather_band(const Rec& r, const Band& bd, const TileInfo& ti,
                                            int sw, const float* tg, uint32_t slot, int pxc,
                                            int pyc, int ky0, int ky1, int kxb0, int kxb1,
                                            GradRec* stage) {
    const float a00 = r.m00 * ti.sx, a10 = r.m10 * ti.sx;
    const float m01sy = r.m01 * ti.sy, m11sy = r.m11 * ti.sy;
    const float c00 = fmaf(r.m00, r.dx0, r.m01 * r.dy0), c10 = fmaf(r.m10, r.dx0, r.m11 * r.dy0);
    const float c0 = fmaf(float(ky0), m01sy, c00), c1 = fmaf(float(ky0), m11sy, c10);
    const float* row = tg + (pyc + ky0 - ti.oy) * sw + (pxc - ti.ox);
    BandMoments m = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (ky0 <= ky1)
        m = gather_band_rows(bd, band_walk(bd, kxb0, kxb1), ky0, ky1, row, sw, a00, a10, c0,
                             c1, m01sy, m11sy, ti.sy, r.dy0, ti.sx, r.dx0);
    const float Sx = fmaf(ti.sx, m.B1t, r.dx0 * m.A0t);
    const float Sxx = fmaf(ti.sx * ti.sx, m.B2,
                           fmaf(2.f * ti.sx * r.dx0, m.B1t, r.dx0 * r.dx0 * m.A0t));
    finish_grad(stage, slot, r.e, r.m00, r.m01, r.m10, r.m11, m.sE, Sx, m.Sy, Sxx, m.Sxy,
                m.Syy);
}

// Backward gather of one photon (photon_differentials.cu:169-218) from the staged gradient.
// Pixels outside the support contribute 0 * g in the reference; with spans on they are not
// visited. The offset d of pixel (kx, ky) is (kx sx + dx0, ky sy + dy0); moments in x are
// kept in the integer offset kx and converted once per photon.
__device__ __forceinline__ void gather(const Rec& r, const TileInfo& ti, int sw, bool spans,
                                       bool band, const float* tg, uint32_t rid,
                                       GradRec* stage) {
    const uint32_t p = r.packed;
    const uint32_t fl = rec_flags(p);
    const int pxc = ti.ox + rec_lx(p), pyc = ti.oy + rec_ly(p);
    const int rx = rec_rx(p), ry = rec_ry(p);
    const int x0 = max(pxc - rx, 0), x1 = min(pxc + rx, ti.W - 1);
    const int y0 = max(pyc - ry, 0), y1 = min(pyc + ry, ti.H - 1);
    const bool all = fl & kFlagEllipseAll;
    if (band && all) {
        const Band bd = make_band(r.m00, r.m01, r.m10, r.m11, r.dx0, r.dy0, ti.sy, ti.isx, ti.isy,
                                  float(rx) + 1.f);
        if (bd.on) {
            const int ky0 = max(bd.ky0, y0 - pyc), ky1 = min(bd.ky1, y1 - pyc);
            gather_band(r, bd, ti, sw, tg, rid, pxc, pyc, ky0, ky1, x0 - pxc, x1 - pxc, stage);
            return;
        }
    }
    const Support sup = make_support(r.m00, r.m01, r.m10, r.m11, spans && all);
    const float a00 = r.m00 * ti.sx, a10 = r.m10 * ti.sx;
    int ky0 = y0 - pyc, ky1 = y1 - pyc;
    support_rows(sup, r.dy0, ti.isy, ky0, ky1);
    float sE = 0.f, A0t = 0.f, B1t = 0.f, B2 = 0.f, Sy = 0.f, Sxy = 0.f, Syy = 0.f;
    for (int ky = ky0; ky <= ky1; ++ky) {
        const float dy = fmaf(float(ky), ti.sy, r.dy0);
        int kx0 = x0 - pxc, kx1 = x1 - pxc;
        if (!support_cols(sup, dy, r.dx0, ti.isx, kx0, kx1)) continue;
        const float c0 = fmaf(r.m00, r.dx0, r.m01 * dy);
        const float c1 = fmaf(r.m10, r.dx0, r.m11 * dy);
        const float* q = tg + (pyc + ky - ti.oy) * sw + (pxc - ti.ox);
        float A0 = 0.f, B1 = 0.f;
        if (all) {
            const float kf = float(kx0);
            bwd_row(kx1 - kx0 + 1, q + kx0, kf, fmaf(kf, a00, c0), fmaf(kf, a10, c1), a00, a10,
                    sE, A0, B1, B2);
        } else {
            for (int kx = kx0; kx <= kx1; ++kx) {
                if (!ellipse_ok(kx, ky, img_wd(ti), img_hd(ti))) continue;
                const float kf = float(kx);
                const float u0 = fmaf(kf, a00, c0), u1 = fmaf(kf, a10, c1);
                const float s = fmaf(u0, u0, u1 * u1);
                const float t = fmaxf(1.f - s, 0.f);
                const float tgv = t * q[kx];
                sE = fmaf(t, tgv, sE);
                A0 += tgv;
                const float tk = tgv * kf;
                B1 += tk;
                B2 = fmaf(tk, kf, B2);
            }
        }
        A0t += A0;
        B1t += B1;
        const float sdx = fmaf(ti.sx, B1, r.dx0 * A0);  // sum t g dx over the row
        Sy = fmaf(dy, A0, Sy);
        Sxy = fmaf(dy, sdx, Sxy);
        Syy = fmaf(dy * dy, A0, Syy);
    }
    const float Sx = fmaf(ti.sx, B1t, r.dx0 * A0t);
    const float Sxx = fmaf(ti.sx * ti.sx, B2, fmaf(2.f * ti.sx * r.dx0, B1t, r.dx0 * r.dx0 * A0t));
    finish_grad(stage, rid, r.e, r.m00, r.m01, r.m10, r.m11, sE, Sx, Sy, Sxx, Sxy, Syy);
}

// Backward gather of one photon by the whole warp (see use_coop): lanes take rows and walk
// their support spans, and a warp reduction hands the moments to the owning lane.
__device__ __forceinline__ void gather_coop(const Rec& r, const TileInfo& ti, int sw,
                                            const float* tg, uint32_t rid, int owner,
                                            GradRec* stage) {
    const int lane = threadIdx.x & 31;
    int pxc, pyc, x0, x1, y0, y1;
    rec_box(r, ti, pxc, pyc, x0, x1, y0, y1);
    const float a00 = r.m00 * ti.sx, a10 = r.m10 * ti.sx;
    const Support sup = make_support(r.m00, r.m01, r.m10, r.m11, true);
    int ky0 = y0 - pyc, ky1 = y1 - pyc;
    support_rows(sup, r.dy0, ti.isy, ky0, ky1);
    float sE = 0.f, A0t = 0.f, B1t = 0.f, B2 = 0.f, Sy = 0.f, Sxy = 0.f, Syy = 0.f;
    for (int ky = ky0 + lane; ky <= ky1; ky += 32) {
        const float dy = fmaf(float(ky), ti.sy, r.dy0);
        int kx0 = x0 - pxc, kx1 = x1 - pxc;
        if (!support_cols(sup, dy, r.dx0, ti.isx, kx0, kx1)) continue;
        const float c0 = fmaf(r.m00, r.dx0, r.m01 * dy);
        const float c1 = fmaf(r.m10, r.dx0, r.m11 * dy);
        const float* q = tg + (pyc + ky - ti.oy) * sw + (pxc - ti.ox);
        float A0 = 0.f, B1 = 0.f;
        const float kf = float(kx0);
        bwd_row(kx1 - kx0 + 1, q + kx0, kf, fmaf(kf, a00, c0), fmaf(kf, a10, c1), a00, a10, sE,
                A0, B1, B2);
        A0t += A0;
        B1t += B1;
        const float sdx = fmaf(ti.sx, B1, r.dx0 * A0);
        Sy = fmaf(dy, A0, Sy);
        Sxy = fmaf(dy, sdx, Sxy);
        Syy = fmaf(dy * dy, A0, Syy);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        sE += __shfl_xor_sync(0xFFFFFFFFu, sE, off);
        A0t += __shfl_xor_sync(0xFFFFFFFFu, A0t, off);
        B1t += __shfl_xor_sync(0xFFFFFFFFu, B1t, off);
        B2 += __shfl_xor_sync(0xFFFFFFFFu, B2, off);
        Sy += __shfl_xor_sync(0xFFFFFFFFu, Sy, off);
        Sxy += __shfl_xor_sync(0xFFFFFFFFu, Sxy, off);
        Syy += __shfl_xor_sync(0xFFFFFFFFu, Syy, off);
    }
    if (lane == owner) {
        const float Sx = fmaf(ti.sx, B1t, r.dx0 * A0t);
        const float Sxx = fmaf(ti.sx * ti.sx, B2, fmaf(2.f * ti.sx * r.dx0, B1t, r.dx0 * r.dx0 * A0t));
        finish_grad(stage, rid, r.e, r.m00, r.m01, r.m10, r.m11, sE, Sx, Sy, Sxx, Sxy, Syy);
    }
}

template <int NT, int MINB>
__global__ __launch_bounds__(NT, MINB) void bwd_tiles_kernel(TileArgs a) {
    extern __shared__ float tg[];
    const Cfg cfg = a.cfg;
    const int sw = cfg.sw;
    const int64_t n_tile = tile_count(a);
    const int64_t nchunks = (n_tile + cfg.chunk - 1) / cfg.chunk;
    __shared__ uint32_t chunk_slot;
    for (int64_t c = next_chunk(a.queue, &chunk_slot); c < nchunks;
         c = next_chunk(a.queue, &chunk_slot)) {
        const int64_t p0 = c * cfg.chunk, p1 = min(p0 + cfg.chunk, n_tile);
        Segment sg = first_segment(a, c, p0);
        TileInfo ti = decode_tile(a.sims, sg.tile, cfg, a.image_elems);
        // next_chunk's barrier ends the previous chunk's reads of the staged tile
        load_region(tg, sw, ti, a.grad, cfg.apron, __ldg(a.tile_r + sg.tile));
        __syncthreads();
        for (int64_t base = p0; base < p1; base += NT) {
            const int64_t i = base + threadIdx.x;
            const bool have = i < p1;
            Rec r = {};
            if (have) r = a.srecs[i];
            const int64_t bend = min(base + NT, p1);
            // consecutive segments of the batch, as in fwd_tiles_kernel; a photon's gradient
            // record goes to its sorted position
            for (int pass = 0; pass <= NT; ++pass) {
                const bool mine = have && i >= sg.begin && i < sg.end;
                const bool coop = mine && use_coop(r, cfg.coop_r);
                if (mine && !coop) gather(r, ti, sw, cfg.spans, cfg.band, tg, uint32_t(i), a.stage);
                for (uint32_t cm = __ballot_sync(0xFFFFFFFFu, coop); cm; cm &= cm - 1) {
                    const int src = __ffs(cm) - 1;
                    const Rec rb = shfl_rec(r, src);
                    const uint32_t slot = uint32_t(base) + (threadIdx.x & ~31u) + uint32_t(src);
                    gather_coop(rb, ti, sw, tg, slot, src, a.stage);
                }
                if (sg.end >= bend) break;
                sg = next_segment(a, sg);
                ti = decode_tile(a.sims, sg.tile, cfg, a.image_elems);
                __syncthreads();
                load_region(tg, sw, ti, a.grad, cfg.apron, __ldg(a.tile_r + sg.tile));
                __syncthreads();
            }
        }
    }
}

// ---- the padded-row walk's kernels (walk 4) ---------------------------------------------
// The same persistent chunk and segment loop as fwd_tiles_kernel / bwd_tiles_kernel, with the
// padded-row walk for the photons that have a band. A lane loads its record in the pass of its
// segment only, and keeps just the row walk's constants across the walk; the rare paths (no
// band, warp-cooperative splat) reload the record out of line, so their registers do not
// burden the walk.

__device__ __noinline__ void deposit_generic(const Rec* rp, TileInfo ti, int sw, bool spans,
                                             float* acc) {
    const Rec r = *rp;
    int x0, x1, y0, y1;
    deposit(r, ti, sw, spans, false, acc, x0, x1, y0, y1);
}

__device__ __noinline__ void deposit_coop_at(const Rec* rp, TileInfo ti, int sw, uint32_t acc_base,
                                             int lane) {
    deposit_coop(*rp, ti, sw, acc_base, lane);
}

__device__ __noinline__ void gather_generic(const Rec* rp, TileInfo ti, int sw, bool spans,
                                            const float* tg, uint32_t rid, GradRec* stage) {
    gather(*rp, ti, sw, spans, false, tg, rid, stage);
}

__device__ __noinline__ void gather_coop_at(const Rec* rp, TileInfo ti, int sw, const float* tg,
                                            uint32_t rid, int owner, GradRec* stage) {
    gather_coop(*rp, ti, sw, tg, rid, owner, stage);
}

template <int NT, int MINB>
__global__ __launch_bounds__(NT, MINB) void fwd_rows_kernel(TileArgs a) {
    extern __shared__ float acc[];
    __shared__ int sb[4];
    __shared__ uint32_t chunk_slot;
    const Cfg cfg = a.cfg;
    const int sw = cfg.sw;
    for (int k = threadIdx.x; k < sw * sw; k += NT) acc[k] = 0.f;
    if (threadIdx.x == 0) {
        sb[0] = INT_MAX; sb[1] = INT_MIN; sb[2] = INT_MAX; sb[3] = INT_MIN;
    }
    __syncthreads();
    const uint32_t acc_base = static_cast<uint32_t>(__cvta_generic_to_shared(acc));
    const int lane = threadIdx.x & 31;
    // photon positions fit in 31 bits (the entry points reject larger calls)
    const int n_tile = int(tile_count(a));
    const int nchunks = (n_tile + cfg.chunk - 1) / cfg.chunk;
    for (int c = int(next_chunk(a.queue, &chunk_slot)); c < nchunks;
         c = int(next_chunk(a.queue, &chunk_slot))) {
        const int p0 = c * cfg.chunk, p1 = min(p0 + cfg.chunk, n_tile);
        Segment sg = first_segment(a, c, p0);
        TileInfo ti = decode_tile(a.sims, sg.tile, cfg, a.image_elems);
        for (int base = p0; base < p1; base += NT) {
            const int i = base + int(threadIdx.x);
            const int bend = min(base + NT, p1);
            for (int pass = 0; pass <= NT; ++pass) {
                const bool mine = i < p1 && i >= sg.begin && i < sg.end;
                RowGeo g;
                int rows = 0;
                float e3 = 0.f;
                bool generic = false, coop = false;
                int x0 = INT_MAX, x1 = INT_MIN, y0 = INT_MAX, y1 = INT_MIN;
                if (mine) {
                    const Rec r = a.srecs[i];
                    coop = use_coop(r, cfg.coop_r);
                    if (coop || !(rec_flags(r.packed) & kFlagFwdSkip)) {
                        int pxc, pyc;
                        rec_clip(r, ti, pxc, pyc, x0, x1, y0, y1);
                        if (!coop) {
                            generic = !prep_rows(r, ti, sw, pxc, pyc, x0, x1, y0, y1, g);
                            rows = generic ? 0 : g.rows;
                            e3 = r.e * kThreeOverPi;
                        }
                    }
                }
                deposit_rows(g, rows, e3, acc_base, sw);
                if (generic) deposit_generic(a.srecs + i, ti, sw, cfg.spans, acc);
                for (uint32_t cm = __ballot_sync(0xFFFFFFFFu, coop); cm; cm &= cm - 1) {
                    const int src = __ffs(cm) - 1;
                    deposit_coop_at(a.srecs + (base + int(threadIdx.x & ~31u) + src), ti, sw,
                                    acc_base, lane);
                }
                bbox_publish(sb, x0, x1, y0, y1);
                if (sg.end >= bend) break;
                flush_tile(acc, sw, ti, a.out, sb);
                sg = next_segment(a, sg);
                ti = decode_tile(a.sims, sg.tile, cfg, a.image_elems);
            }
        }
        flush_tile(acc, sw, ti, a.out, sb);
    }
}

template <int NT, int MINB>
__global__ __launch_bounds__(NT, MINB) void bwd_rows_kernel(TileArgs a) {
    extern __shared__ float tg[];
    __shared__ uint32_t chunk_slot;
    const Cfg cfg = a.cfg;
    const int sw = cfg.sw;
    const uint32_t tg_base = static_cast<uint32_t>(__cvta_generic_to_shared(tg));
    const int n_tile = int(tile_count(a));
    const int nchunks = (n_tile + cfg.chunk - 1) / cfg.chunk;
    for (int c = int(next_chunk(a.queue, &chunk_slot)); c < nchunks;
         c = int(next_chunk(a.queue, &chunk_slot))) {
        const int p0 = c * cfg.chunk, p1 = min(p0 + cfg.chunk, n_tile);
        Segment sg = first_segment(a, c, p0);
        TileInfo ti = decode_tile(a.sims, sg.tile, cfg, a.image_elems);
        // next_chunk's barrier ends the previous chunk's reads of the staged tile
        load_region(tg, sw, ti, a.grad, cfg.apron, __ldg(a.tile_r + sg.tile));
        __syncthreads();
        for (int base = p0; base < p1; base += NT) {
            const int i = base + int(threadIdx.x);
            const int bend = min(base + NT, p1);
            for (int pass = 0; pass <= NT; ++pass) {
                const bool mine = i < p1 && i >= sg.begin && i < sg.end;
                RowGeo g;
                int rows = 0;
                float dy0 = 0.f;
                bool walk = false, generic = false, coop = false;
                if (mine) {
                    const Rec r = a.srecs[i];
                    coop = use_coop(r, cfg.coop_r);
                    if (!coop) {
                        int pxc, pyc, x0, x1, y0, y1;
                        rec_clip(r, ti, pxc, pyc, x0, x1, y0, y1);
                        walk = prep_rows(r, ti, sw, pxc, pyc, x0, x1, y0, y1, g);
                        generic = !walk;
                        rows = walk ? g.rows : 0;
                        dy0 = r.dy0;
                    }
                }
                const RowMoments m = gather_rows(g, rows, tg_base, sw, ti.sy, dy0);
                if (walk) finish_rows(a.stage, uint32_t(i), a.srecs[i], ti, m);
                if (generic)
                    gather_generic(a.srecs + i, ti, sw, cfg.spans, tg, uint32_t(i), a.stage);
                for (uint32_t cm = __ballot_sync(0xFFFFFFFFu, coop); cm; cm &= cm - 1) {
                    const int src = __ffs(cm) - 1;
                    const int slot = base + int(threadIdx.x & ~31u) + src;
                    gather_coop_at(a.srecs + slot, ti, sw, tg, uint32_t(slot), src, a.stage);
                }
                if (sg.end >= bend) break;
                sg = next_segment(a, sg);
                ti = decode_tile(a.sims, sg.tile, cfg, a.image_elems);
                __syncthreads();
                load_region(tg, sw, ti, a.grad, cfg.apron, __ldg(a.tile_r + sg.tile));
                __syncthreads();
            }
        }
    }
}

// ------------------------------------------------------------------ tail ---------------
// Footprints wider than the apron (the plan's wide list) are splatted straight into global
// memory, one warp per photon; their gradient records follow the tile path's in the stage.

struct Direct {
    int pxc, pyc, x0, x1, y0, y1;
    bool all;
    float dx0, dy0, m00, m01, m10, m11, e;
    float sx, sy;
    double wd, hd;
    int64_t img_off;
    int W;
};

__device__ __forceinline__ bool direct_setup(const TileArgs& a, uint32_t rid, Direct& d) {
    const int64_t n = a.ph.n;
    const int s = find_sim_of_photon(a.sims, rid);
    const pds_sim sim = load_sim(a.sims, s);
    const int64_t ch = a.ph.cp[rid];
    const float x = a.ph.X[rid], y = a.ph.X[n + rid];
    const Footprint f = make_footprint(x, y, a.ph.R[rid], sim.height, sim.width, a.mpr);
    if (!clip_box(f, sim.height, sim.width, d.x0, d.x1, d.y0, d.y1)) return false;
    d.pxc = f.px_c;
    d.pyc = f.py_c;
    d.all = f.ellipse_all;
    d.dx0 = corner_offset(f.px_c, sim.width, x);
    d.dy0 = corner_offset(f.py_c, sim.height, y);
    d.m00 = a.ph.M[rid];
    d.m01 = a.ph.M[n + rid];
    d.m10 = a.ph.M[3 * n + rid];
    d.m11 = a.ph.M[4 * n + rid];
    d.e = a.ph.E[rid];
    d.sx = float(2.0 / double(sim.width));
    d.sy = float(2.0 / double(sim.height));
    d.wd = double(float(sim.width));
    d.hd = double(float(sim.height));
    d.img_off = sim.image_offset + ch * sim.height * sim.width;
    if (d.img_off < 0 || d.img_off + int64_t(sim.height) * sim.width > a.image_elems) return false;
    d.W = sim.width;
    return true;
}

__global__ __launch_bounds__(256) void tail_fwd_kernel(TileArgs a) {
    const int64_t n_big = wide_count(a);
    const int lane = threadIdx.x & 31;
    const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
    for (int64_t w = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); w < n_big;
         w += warps) {
        const uint32_t rid = __ldg(a.wide + w);
        Direct d;
        if (!direct_setup(a, rid, d) || !(d.e > 0.f)) continue;
        const float e3 = d.e * kThreeOverPi;
        const int bw = d.x1 - d.x0 + 1;
        const int64_t total = int64_t(bw) * (d.y1 - d.y0 + 1);
        float* img = a.out + d.img_off;
        for (int64_t k = lane; k < total; k += 32) {
            const int py = d.y0 + int(k / bw), px = d.x0 + int(k % bw);
            const int kx = px - d.pxc, ky = py - d.pyc;
            if (!d.all && !ellipse_ok(kx, ky, d.wd, d.hd)) continue;
            const float dx = fmaf(float(kx), d.sx, d.dx0), dy = fmaf(float(ky), d.sy, d.dy0);
            const float u0 = fmaf(d.m00, dx, d.m01 * dy), u1 = fmaf(d.m10, dx, d.m11 * dy);
            const float s = fmaf(u0, u0, u1 * u1);
            if (s < 1.f) {
                const float t = 1.f - s;
                atomicAdd(img + int64_t(py) * d.W + px, t * t * e3);
            }
        }
    }
}

__global__ __launch_bounds__(256) void tail_bwd_kernel(TileArgs a) {
    const int64_t n_tile = tile_count(a), n_big = wide_count(a);
    const int lane = threadIdx.x & 31;
    const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
    for (int64_t w = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); w < n_big;
         w += warps) {
        const uint32_t rid = __ldg(a.wide + w);
        Direct d;
        float sE = 0.f, Sx = 0.f, Sy = 0.f, Sxx = 0.f, Sxy = 0.f, Syy = 0.f;
        const bool any = direct_setup(a, rid, d);
        if (any) {
            const int bw = d.x1 - d.x0 + 1;
            const int64_t total = int64_t(bw) * (d.y1 - d.y0 + 1);
            const float* img = a.grad + d.img_off;
            for (int64_t k = lane; k < total; k += 32) {
                const int py = d.y0 + int(k / bw), px = d.x0 + int(k % bw);
                const int kx = px - d.pxc, ky = py - d.pyc;
                if (!d.all && !ellipse_ok(kx, ky, d.wd, d.hd)) continue;
                const float dx = fmaf(float(kx), d.sx, d.dx0), dy = fmaf(float(ky), d.sy, d.dy0);
                const float u0 = fmaf(d.m00, dx, d.m01 * dy), u1 = fmaf(d.m10, dx, d.m11 * dy);
                const float s = fmaf(u0, u0, u1 * u1);
                const float t = s < 1.f ? 1.f - s : 0.f;
                const float tgv = t * __ldg(img + int64_t(py) * d.W + px);
                sE = fmaf(t, tgv, sE);
                Sx = fmaf(tgv, dx, Sx);
                Sy = fmaf(tgv, dy, Sy);
                Sxx = fmaf(tgv * dx, dx, Sxx);
                Sxy = fmaf(tgv * dx, dy, Sxy);
                Syy = fmaf(tgv * dy, dy, Syy);
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            sE += __shfl_xor_sync(0xFFFFFFFFu, sE, off);
            Sx += __shfl_xor_sync(0xFFFFFFFFu, Sx, off);
            Sy += __shfl_xor_sync(0xFFFFFFFFu, Sy, off);
            Sxx += __shfl_xor_sync(0xFFFFFFFFu, Sxx, off);
            Sxy += __shfl_xor_sync(0xFFFFFFFFu, Sxy, off);
            Syy += __shfl_xor_sync(0xFFFFFFFFu, Syy, off);
        }
        if (lane == 0) {
            if (!any) {
                d.m00 = d.m01 = d.m10 = d.m11 = d.e = 0.f;
            }
            finish_grad(a.stage, uint32_t(n_tile + w), d.e, d.m00, d.m01, d.m10, d.m11, sE, Sx,
                        Sy, Sxx, Sxy, Syy);
        }
    }
}

// Spreads the gradient records into the reference's outputs grad_Ep[N], grad_xp[2][N],
// grad_Mp[2][3][N] (column 2 of grad_Mp is zero, :212, :218) in photon order: each photon's
// record is one 32-byte gather through the plan's inverse map, the writes are coalesced.
// Photons that touch no pixel get zeros.
__device__ __forceinline__ void grad_record(const TileArgs& a, int64_t n, int64_t n_tile,
                                            uint32_t v, float4& lo, float4& hi) {
    const float4* st = reinterpret_cast<const float4*>(a.stage);
    const int64_t slot = (v & kWideBit) ? n_tile + int64_t(v & ~kWideBit) : int64_t(v);
    lo = make_float4(0.f, 0.f, 0.f, 0.f);
    hi = lo;
    if (v != kInvalidPos && slot < n) {
        lo = st[2 * slot];
        hi = st[2 * slot + 1];
    }
}

__global__ __launch_bounds__(256) void grad_scatter_kernel(TileArgs a) {
    const int64_t n = a.ph.n;
    const int64_t n_tile = tile_count(a);
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x) {
        float4 lo, hi;
        grad_record(a, n, n_tile, __ldg(a.inv + i), lo, hi);
        a.gE[i] = lo.x;
        a.gX[i] = lo.y;
        a.gX[n + i] = lo.z;
        a.gM[i] = lo.w;
        a.gM[n + i] = hi.x;
        a.gM[2 * n + i] = 0.f;
        a.gM[3 * n + i] = hi.y;
        a.gM[4 * n + i] = hi.z;
        a.gM[5 * n + i] = 0.f;
    }
}

// The same for 4 photons per thread: quad q holds photons 4q..4q+3 and each output row takes
// them in one 16-byte store, two 8-byte stores or four 4-byte stores, as the row's start
// allows (row r starts N * r elements after its array's start, so for N not a multiple of 4
// rows differ in alignment). The last N % 4 photons are written one by one.
__device__ __forceinline__ void store_quad(float* p, float4 v) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    if ((a & 15) == 0) {
        *reinterpret_cast<float4*>(p) = v;
    } else if ((a & 7) == 0) {
        reinterpret_cast<float2*>(p)[0] = make_float2(v.x, v.y);
        reinterpret_cast<float2*>(p)[1] = make_float2(v.z, v.w);
    } else {
        p[0] = v.x; p[1] = v.y; p[2] = v.z; p[3] = v.w;
    }
}

__global__ __launch_bounds__(256) void grad_scatter4_kernel(TileArgs a) {
    const int64_t n = a.ph.n, nq = n >> 2;
    const int64_t n_tile = tile_count(a);
    const uint4* inv4 = reinterpret_cast<const uint4*>(a.inv);
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int64_t q = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < nq;
         q += int64_t(gridDim.x) * blockDim.x) {
        const uint4 v = __ldg(inv4 + q);
        float4 l0, h0, l1, h1, l2, h2, l3, h3;
        grad_record(a, n, n_tile, v.x, l0, h0);
        grad_record(a, n, n_tile, v.y, l1, h1);
        grad_record(a, n, n_tile, v.z, l2, h2);
        grad_record(a, n, n_tile, v.w, l3, h3);
        const int64_t i = 4 * q;
        store_quad(a.gE + i, make_float4(l0.x, l1.x, l2.x, l3.x));
        store_quad(a.gX + i, make_float4(l0.y, l1.y, l2.y, l3.y));
        store_quad(a.gX + n + i, make_float4(l0.z, l1.z, l2.z, l3.z));
        store_quad(a.gM + i, make_float4(l0.w, l1.w, l2.w, l3.w));
        store_quad(a.gM + n + i, make_float4(h0.x, h1.x, h2.x, h3.x));
        store_quad(a.gM + 2 * n + i, z);
        store_quad(a.gM + 3 * n + i, make_float4(h0.y, h1.y, h2.y, h3.y));
        store_quad(a.gM + 4 * n + i, make_float4(h0.z, h1.z, h2.z, h3.z));
        store_quad(a.gM + 5 * n + i, z);
    }
    // the last n % 4 photons
    const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < (n & 3)) {
        const int64_t i = 4 * nq + t;
        float4 lo, hi;
        grad_record(a, n, n_tile, __ldg(a.inv + i), lo, hi);
        a.gE[i] = lo.x;
        a.gX[i] = lo.y;
        a.gX[n + i] = lo.z;
        a.gM[i] = lo.w;
        a.gM[n + i] = hi.x;
        a.gM[2 * n + i] = 0.f;
        a.gM[3 * n + i] = hi.y;
        a.gM[4 * n + i] = hi.z;
        a.gM[5 * n + i] = 0.f;
    }
}


constexpr int kTileThreads = 256;

int num_sms() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

// Grid of a persistent tile kernel: resident CTAs per SM x SMs, capped by the work.
template <typename K>
int persistent_grid(K kernel, size_t smem, int64_t n_units) {
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTileThreads, smem);
    if (per_sm < 1) per_sm = 1;
    const int64_t g = int64_t(per_sm) * num_sms();
    const int64_t need = n_units > 0 ? n_units : 1;
    return int(g < need ? g : need);
}

template <typename K>
cudaError_t set_smem(K kernel, size_t smem) {
    if (smem <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
}

}  // namespace


// Dynamic shared memory of a tile kernel: the tile's region (sw x sw floats) and, for the
// band forward (staged), the two record buffers after it.
size_t tile_smem(const TileArgs& a, bool staged) {
    const size_t sw = size_t(a.cfg.sw);
    if (!staged) return sw * sw * sizeof(float);
    return (((sw * sw + 3) & ~size_t(3)) * sizeof(float)) + 2 * size_t(kTileThreads) * sizeof(Rec);
}

template <int MINB, bool ROWS>
cudaError_t launch_forward_t(const TileArgs& a, cudaStream_t st) {
    const size_t smem = tile_smem(a, !ROWS);
    auto kern = ROWS ? fwd_rows_kernel<kTileThreads, MINB> : fwd_tiles_kernel<kTileThreads, MINB>;
    cudaError_t e = set_smem(kern, smem);
    if (e != cudaSuccess) return e;
    const int64_t chunks = (a.ph.n + a.cfg.chunk - 1) / a.cfg.chunk;
    if (chunks > 0) {
        const int grid = persistent_grid(kern, smem, chunks);
        kern<<<grid, kTileThreads, smem, st>>>(a);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        const int tgrid = num_sms() * 2;
        tail_fwd_kernel<<<tgrid, 256, 0, st>>>(a);
        e = cudaGetLastError();
    }
    return e;
}

template <int MINB, bool ROWS>
cudaError_t launch_backward_t(const TileArgs& a, cudaStream_t st) {
    const size_t smem = tile_smem(a, false);
    auto kern = ROWS ? bwd_rows_kernel<kTileThreads, MINB> : bwd_tiles_kernel<kTileThreads, MINB>;
    cudaError_t e = set_smem(kern, smem);
    if (e != cudaSuccess) return e;
    const int64_t chunks = (a.ph.n + a.cfg.chunk - 1) / a.cfg.chunk;
    if (chunks > 0) {
        const int grid = persistent_grid(kern, smem, chunks);
        kern<<<grid, kTileThreads, smem, st>>>(a);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        const int tgrid = num_sms() * 2;
        tail_bwd_kernel<<<tgrid, 256, 0, st>>>(a);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        // the quad form needs the inverse map 16-byte aligned (the workspace is) and every
        // output 4-byte aligned; the rows' own alignment is handled per store
        // no outputs: the gradients stay in the workspace as records (read by the refraction
        // backward's records mode)
        if (!a.gE) return cudaSuccess;
        const auto al = [](const void* p, uintptr_t m) {
            return (reinterpret_cast<uintptr_t>(p) & m) == 0;
        };
        const bool vec = al(a.inv, 15) && al(a.gE, 3) && al(a.gX, 3) && al(a.gM, 3);
        const int64_t items = vec ? a.ph.n / 4 : a.ph.n;
        const int64_t sblocks = items > 0 ? (items + 255) / 256 : 1;
        const int64_t scap = int64_t(num_sms()) * 16;
        const unsigned sgrid = unsigned(sblocks < scap ? sblocks : scap);
        if (vec)
            grad_scatter4_kernel<<<sgrid, 256, 0, st>>>(a);
        else
            grad_scatter_kernel<<<sgrid, 256, 0, st>>>(a);
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t launch_forward(const TileArgs& a, cudaStream_t st) {
    if (a.cfg.rows) {
        if (a.cfg.min_blocks >= 4) return launch_forward_t<4, true>(a, st);
        return a.cfg.min_blocks == 3 ? launch_forward_t<3, true>(a, st)
                                     : launch_forward_t<2, true>(a, st);
    }
    if (a.cfg.min_blocks >= 4) return launch_forward_t<4, false>(a, st);
    return a.cfg.min_blocks == 3 ? launch_forward_t<3, false>(a, st)
                                 : launch_forward_t<2, false>(a, st);
}

cudaError_t launch_backward(const TileArgs& a, cudaStream_t st) {
    if (a.cfg.rows) {
        if (a.cfg.min_blocks_bwd >= 4) return launch_backward_t<4, true>(a, st);
        return a.cfg.min_blocks_bwd == 3 ? launch_backward_t<3, true>(a, st)
                                     : launch_backward_t<2, true>(a, st);
    }
    if (a.cfg.min_blocks_bwd >= 4) return launch_backward_t<4, false>(a, st);
    return a.cfg.min_blocks_bwd == 3 ? launch_backward_t<3, false>(a, st)
                                 : launch_backward_t<2, false>(a, st);
}

}  // namespace pds
