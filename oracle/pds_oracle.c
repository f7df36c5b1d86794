/*
 * CPU oracle for photon-differential splatting (PDS). TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's splatting kernels
 *   PyOptix/kernel/photon_differentials.cu:60-113  (pds_cuda_forward_kernel)
 *   PyOptix/kernel/photon_differentials.cu:136-221 (pds_cuda_backward_kernel)
 * with the helper semantics of :23-58 (silverman, d_silverman, pixel_to_coord,
 * coord_to_pixel, matrix_multiply). Only tests, the smoke check and the CPU baseline leg of
 * the benchmark call it; the product never does.
 *
 * Two arithmetic modes:
 *   PDS_ORACLE_FP64 (0): every real-valued quantity in double. This is the accuracy oracle
 *     the CUDA kernels are held to (relative L2 <= 1e-5 forward, <= 1e-4 gradients). The
 *     backward uses the closed form of d/dr K(r^2) * u / r = -12/pi (1 - r^2) u, which is the
 *     finite limit of the reference's expression at r = 0 (where the reference divides 0/0).
 *   PDS_ORACLE_REF32 (1): the reference's own single-precision expression order
 *     (float pixel_to_coord with a float divide, float differences, the float silverman,
 *     the normalised direction u / |u| of :187-190 including its NaN at r = 0). Built with
 *     -ffp-contract=off, so it differs from the reference GPU build only where nvcc
 *     contracted a multiply-add. Used to pin the oracle on fixtures produced by the
 *     reference extension itself.
 *
 * Integer decisions (which pixels a photon touches) are identical in both modes and equal
 * to the reference's: they are computed in double from the float inputs, exactly as the
 * reference's mixed float/double expressions do (coord_to_pixel :46-51 and the radius cut
 * :80-81 promote to double through their 0.5 literals; the ellipse test :93 through 0.25).
 * Conversions double -> int32 follow the CUDA device rule (round toward zero, saturate,
 * NaN -> 0), which is what the reference's int32_t(...) casts do on the GPU.
 *
 * Photons whose channel is outside [0, C) are skipped (the reference checks only c < C,
 * :75, and its negative-channel behaviour is an out-of-bounds write). In the backward such
 * photons get zero gradients (the reference leaves its empty_like outputs unwritten).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PDS_ORACLE_FP64 0
#define PDS_ORACLE_REF32 1

/* CUDA's double -> int32 conversion (cvt.rzi.s32.f64): truncate, saturate, NaN -> 0. */
static int32_t cvt_rzi_s32(double v) {
    if (isnan(v)) return 0;
    if (v >= 2147483647.0) return INT32_MAX;
    if (v <= -2147483648.0) return INT32_MIN;
    return (int32_t)v;
}

/* Per-photon footprint set-up shared by both modes and both directions.
 * Reference: photon_differentials.cu:76-87 (and the same lines :155-165 of the backward). */
typedef struct {
    int32_t px_c, py_c, rx, ry;
    int ellipse_all; /* 1 if the :93 ellipse test passes for every offset of the box */
} footprint_t;

static footprint_t footprint(double x, double y, double r, int64_t H, int64_t W, int32_t mpr) {
    footprint_t f;
    const double w = (double)(float)W, h = (double)(float)H; /* scalar_t w = size(2) */
    int32_t rx = cvt_rzi_s32(ceil(r * 0.5 * w));
    int32_t ry = cvt_rzi_s32(ceil(r * 0.5 * h));
    f.rx = rx < mpr ? rx : mpr;
    f.ry = ry < mpr ? ry : mpr;
    f.px_c = cvt_rzi_s32((0.5 * x + 0.5) * w);
    f.py_c = cvt_rzi_s32((0.5 * y + 0.5) * h);
    if (f.rx >= 0 && f.ry >= 0) {
        /* the test is monotone in |x_off|, |y_off|: the corner decides for the whole box */
        double tx = (double)(float)((int32_t)((uint32_t)f.rx * (uint32_t)f.rx)) / (0.25 * w * w);
        double ty = (double)(float)((int32_t)((uint32_t)f.ry * (uint32_t)f.ry)) / (0.25 * h * h);
        f.ellipse_all = (tx + ty <= 1.0);
    } else {
        f.ellipse_all = 1;
    }
    return f;
}

/* The :93 test for one offset (int32 square as the reference computes it). */
static int ellipse_ok(int32_t xo, int32_t yo, int64_t H, int64_t W) {
    const double w = (double)(float)W, h = (double)(float)H;
    double tx = (double)(float)((int32_t)((uint32_t)xo * (uint32_t)xo)) / (0.25 * w * w);
    double ty = (double)(float)((int32_t)((uint32_t)yo * (uint32_t)yo)) / (0.25 * h * h);
    return tx + ty <= 1.0;
}

/* Clipped box of a photon in pixel space; returns 0 if empty. 64-bit so that saturated
 * centres cannot overflow (the reference's int32 sums wrap to out-of-image values there). */
static int clipped_box(const footprint_t* f, int64_t H, int64_t W, int64_t* x0, int64_t* x1,
                       int64_t* y0, int64_t* y1) {
    if (f->rx < 0 || f->ry < 0) return 0;
    int64_t a = (int64_t)f->px_c - f->rx, b = (int64_t)f->px_c + f->rx;
    int64_t c = (int64_t)f->py_c - f->ry, d = (int64_t)f->py_c + f->ry;
    if (a < 0) a = 0;
    if (b > W - 1) b = W - 1;
    if (c < 0) c = 0;
    if (d > H - 1) d = H - 1;
    *x0 = a; *x1 = b; *y0 = c; *y1 = d;
    return a <= b && c <= d;
}

/* ---------------------------------------------------------------- forward ------------ */
/* Photon arrays are double: float inputs converted exactly, so the integer decisions match
 * the reference's, and finite-difference checks can perturb below float resolution. */

static void forward_one(int64_t i, const double* E, const double* X, const double* M,
                        const int64_t* cp, const double* R, int64_t N, int64_t C, int64_t H,
                        int64_t W, int32_t mpr, int mode, double* out) {
    const int64_t ch = cp[i];
    if (ch < 0 || ch >= C) return;
    const double x = X[i], y = X[N + i], e = E[i];
    footprint_t f = footprint(x, y, R[i], H, W, mpr);
    int64_t x0, x1, y0, y1;
    if (!clipped_box(&f, H, W, &x0, &x1, &y0, &y1)) return;
    double* img = out + ch * H * W;
    const double m0 = M[0 * N + i], m1 = M[1 * N + i], m2 = M[2 * N + i];
    const double m3 = M[3 * N + i], m4 = M[4 * N + i], m5 = M[5 * N + i];
    for (int64_t py = y0; py <= y1; ++py) {
        for (int64_t px = x0; px <= x1; ++px) {
            if (!f.ellipse_all && !ellipse_ok((int32_t)(px - f.px_c), (int32_t)(py - f.py_c), H, W))
                continue;
            if (mode == PDS_ORACLE_FP64) {
                const double dx = 2.0 * (double)px / (double)W - 1.0 - x;
                const double dy = 2.0 * (double)py / (double)H - 1.0 - y;
                const double u0 = m0 * dx + m1 * dy + m2 * 0.0;
                const double u1 = m3 * dx + m4 * dy + m5 * 0.0;
                const double s = u0 * u0 + u1 * u1;
                const double k = s < 1.0 ? 3.0 / M_PI * (1.0 - s) * (1.0 - s) : 0.0;
                const double v = k * e;
                if (v > 0.0) img[py * W + px] += v;
            } else {
                const float wf = (float)W, hf = (float)H;
                const float xf = (float)x, yf = (float)y, ef = (float)e;
                float cx = 2.0f * (float)px;
                cx = cx / wf;
                cx = cx - 1.0f;
                float cy = 2.0f * (float)py;
                cy = cy / hf;
                cy = cy - 1.0f;
                const float dx = cx - xf, dy = cy - yf;
                const float u0 = (float)m0 * dx + (float)m1 * dy + (float)m2 * 0.0f;
                const float u1 = (float)m3 * dx + (float)m4 * dy + (float)m5 * 0.0f;
                const float s = u0 * u0 + u1 * u1;
                float k = 0.0f;
                if (s < 1.0f) k = 3.0f / (float)M_PI * (1.0f - s) * (1.0f - s);
                const float v = k * ef;
                if (v > 0.0f) img[py * W + px] += (double)v;
            }
        }
    }
}

/* out: C*H*W doubles, overwritten. threads <= 0 -> all available. */
void pds_oracle_forward(const double* E, const double* X, const double* M, const int64_t* cp,
                        const double* R, int64_t N, int64_t C, int64_t H, int64_t W,
                        int32_t mpr, int mode, int threads, double* out) {
    const int64_t npix = C * H * W;
    memset(out, 0, (size_t)npix * sizeof(double));
#ifdef _OPENMP
    int nt = threads > 0 ? threads : omp_get_max_threads();
    if (nt > 1 && (double)npix * nt * 8.0 <= 2.0e9) {
        double* priv = (double*)calloc((size_t)npix * (size_t)nt, sizeof(double));
        if (priv) {
#pragma omp parallel num_threads(nt)
            {
                int t = omp_get_thread_num();
                double* mine = priv + (size_t)t * (size_t)npix;
#pragma omp for schedule(static)
                for (int64_t i = 0; i < N; ++i)
                    forward_one(i, E, X, M, cp, R, N, C, H, W, mpr, mode, mine);
#pragma omp for schedule(static)
                for (int64_t p = 0; p < npix; ++p) {
                    double acc = 0.0;
                    for (int k = 0; k < nt; ++k) acc += priv[(size_t)k * (size_t)npix + p];
                    out[p] = acc;
                }
            }
            free(priv);
            return;
        }
    }
#else
    (void)threads;
#endif
    for (int64_t i = 0; i < N; ++i) forward_one(i, E, X, M, cp, R, N, C, H, W, mpr, mode, out);
}

/* ---------------------------------------------------------------- backward ----------- */

static void backward_one(int64_t i, const double* G, const double* E, const double* X,
                         const double* M, const int64_t* cp, const double* R, int64_t N,
                         int64_t C, int64_t H, int64_t W, int32_t mpr, int mode, double* gE,
                         double* gX, double* gM) {
    double ge = 0.0, gx0 = 0.0, gx1 = 0.0, g0 = 0.0, g1 = 0.0, g3 = 0.0, g4 = 0.0;
    const int64_t ch = cp[i];
    if (ch >= 0 && ch < C) {
        const double x = X[i], y = X[N + i], e = E[i];
        footprint_t f = footprint(x, y, R[i], H, W, mpr);
        int64_t x0, x1, y0, y1;
        const double* img = G + ch * H * W;
        const double m0 = M[0 * N + i], m1 = M[1 * N + i], m2 = M[2 * N + i];
        const double m3 = M[3 * N + i], m4 = M[4 * N + i], m5 = M[5 * N + i];
        if (clipped_box(&f, H, W, &x0, &x1, &y0, &y1)) {
            /* float accumulators of the REF32 mode (the reference's scalar_t sums :169-171) */
            float fe = 0.f, fx0 = 0.f, fx1 = 0.f, f0 = 0.f, f1 = 0.f, f3 = 0.f, f4 = 0.f;
            for (int64_t py = y0; py <= y1; ++py) {
                for (int64_t px = x0; px <= x1; ++px) {
                    if (!f.ellipse_all &&
                        !ellipse_ok((int32_t)(px - f.px_c), (int32_t)(py - f.py_c), H, W))
                        continue;
                    const double g = img[py * W + px];
                    if (mode == PDS_ORACLE_FP64) {
                        const double dx = 2.0 * (double)px / (double)W - 1.0 - x;
                        const double dy = 2.0 * (double)py / (double)H - 1.0 - y;
                        const double u0 = m0 * dx + m1 * dy + m2 * 0.0;
                        const double u1 = m3 * dx + m4 * dy + m5 * 0.0;
                        const double s = u0 * u0 + u1 * u1;
                        const double t = s < 1.0 ? 1.0 - s : 0.0;
                        /* 2 dK/ds = -12/pi (1 - s): the reference's d_silverman(r) * u / r */
                        const double a = -12.0 / M_PI * t * e * g;
                        ge += 3.0 / M_PI * t * t * g;
                        gx0 += -a * (m0 * u0 + m3 * u1);
                        gx1 += -a * (m1 * u0 + m4 * u1);
                        g0 += a * u0 * dx;
                        g1 += a * u0 * dy;
                        g3 += a * u1 * dx;
                        g4 += a * u1 * dy;
                    } else {
                        const float wf = (float)W, hf = (float)H;
                        const float xf = (float)x, yf = (float)y, ef = (float)e;
                        const float M0 = (float)m0, M1 = (float)m1, M2 = (float)m2;
                        const float M3 = (float)m3, M4 = (float)m4, M5 = (float)m5;
                        float cx = 2.0f * (float)px;
                        cx = cx / wf;
                        cx = cx - 1.0f;
                        float cy = 2.0f * (float)py;
                        cy = cy / hf;
                        cy = cy - 1.0f;
                        const float dx = cx - xf, dy = cy - yf;
                        const float u0 = M0 * dx + M1 * dy + M2 * 0.0f;
                        const float u1 = M3 * dx + M4 * dy + M5 * 0.0f;
                        const float s = u0 * u0 + u1 * u1;
                        const float r = sqrtf(s);
                        const float n0 = u0 / r, n1 = u1 / r;
                        const float gf = (float)g;
                        float ds = 0.0f;
                        if (r < 1.0f) ds = -12.0f / (float)M_PI * r * (1.0f - s);
                        const float dk = ds * ef * gf;
                        float k = 0.0f;
                        if (s < 1.0f) k = 3.0f / (float)M_PI * (1.0f - s) * (1.0f - s);
                        fe += k * gf;
                        fx0 += -dk * (M0 * n0 + M3 * n1);
                        fx1 += -dk * (M1 * n0 + M4 * n1);
                        f0 += dk * n0 * dx;
                        f1 += dk * n0 * dy;
                        f3 += dk * n1 * dx;
                        f4 += dk * n1 * dy;
                    }
                }
            }
            if (mode != PDS_ORACLE_FP64) {
                ge = fe; gx0 = fx0; gx1 = fx1; g0 = f0; g1 = f1; g3 = f3; g4 = f4;
            }
        }
    }
    gE[i] = ge;
    gX[i] = gx0;
    gX[N + i] = gx1;
    gM[0 * N + i] = g0;
    gM[1 * N + i] = g1;
    gM[2 * N + i] = 0.0;
    gM[3 * N + i] = g3;
    gM[4 * N + i] = g4;
    gM[5 * N + i] = 0.0;
}

/* G: C*H*W doubles (upstream gradient). Outputs: gE[N], gX[2N], gM[6N] (row-major 2x3xN). */
void pds_oracle_backward(const double* G, const double* E, const double* X, const double* M,
                         const int64_t* cp, const double* R, int64_t N, int64_t C, int64_t H,
                         int64_t W, int32_t mpr, int mode, int threads, double* gE,
                         double* gX, double* gM) {
#ifdef _OPENMP
    int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1024) num_threads(nt)
#else
    (void)threads;
#endif
    for (int64_t i = 0; i < N; ++i)
        backward_one(i, G, E, X, M, cp, R, N, C, H, W, mpr, mode, gE, gX, gM);
}

/* ---------------------------------------------------------------- footprints --------- */

/* Per photon: centre pixel, radii, ellipse flag and the number of in-image box pixels the
 * reference visits (the count behind the FLOP accounting). box_pixels = 0 for skipped
 * photons (channel out of range or box outside the image). */
void pds_oracle_footprints(const double* X, const int64_t* cp, const double* R, int64_t N,
                           int64_t C, int64_t H, int64_t W, int32_t mpr, int32_t* out5,
                           int64_t* box_pixels) {
    for (int64_t i = 0; i < N; ++i) {
        footprint_t f = footprint(X[i], X[N + i], R[i], H, W, mpr);
        out5[5 * i + 0] = f.px_c;
        out5[5 * i + 1] = f.py_c;
        out5[5 * i + 2] = f.rx;
        out5[5 * i + 3] = f.ry;
        out5[5 * i + 4] = f.ellipse_all;
        int64_t x0, x1, y0, y1, n = 0;
        if (cp[i] >= 0 && cp[i] < C && clipped_box(&f, H, W, &x0, &x1, &y0, &y1)) {
            if (f.ellipse_all) {
                n = (x1 - x0 + 1) * (y1 - y0 + 1);
            } else {
                for (int64_t py = y0; py <= y1; ++py)
                    for (int64_t px = x0; px <= x1; ++px)
                        n += ellipse_ok((int32_t)(px - f.px_c), (int32_t)(py - f.py_c), H, W);
            }
        }
        box_pixels[i] = n;
    }
}
