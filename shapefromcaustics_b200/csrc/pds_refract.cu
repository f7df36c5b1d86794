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
// Sobel stencils. (The chain templates take T = float here; instantiated with forward-mode
// dual numbers on the host they give the reference derivatives the sweeps were checked
// against.) A CTA's patches are summed in shared memory where
// its photons share a compact region of the field, else added with global float atomics.
#include <climits>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/pds_b200.h"
#include "pds_internal.h"

namespace pds {
namespace {

constexpr int K = 7;  // height-dependent scalars of one photon

__device__ __forceinline__ float dsqrt(float a) { return sqrtf(a); }

template <class T>
struct V3 {
    T x, y, z;
};
template <class T>
__device__ __forceinline__ V3<T> vadd(const V3<T>& a, const V3<T>& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T>
__device__ __forceinline__ V3<T> vsub(const V3<T>& a, const V3<T>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T, class S>
__device__ __forceinline__ V3<T> vscale(const S& s, const V3<T>& a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T>
__device__ __forceinline__ T vdot(const V3<T>& a, const V3<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

template <class T>
__device__ __forceinline__ T cst(float v);
template <>
__device__ __forceinline__ float cst<float>(float v) { return v; }

struct PlateParams {
    float texel, ior, dist, inv_half, du0;
    float lx, ly, lz;  // light direction
};

__host__ __device__ __forceinline__ PlateParams to_params(const pds_plate& p) {
    PlateParams q;
    q.texel = p.texel;
    q.ior = p.ior;
    q.dist = p.receiver_distance;
    q.inv_half = 1.f / p.receiver_half;
    q.du0 = p.du0;
    q.lx = p.light_dir[0];
    q.ly = p.light_dir[1];
    q.lz = p.light_dir[2];
    return q;
}

// Snell refraction of direction d and its differential Dd at unit normal n facing the
// incident side (d.n < 0), with normal derivative dn (model/caustics.py:176-189).
template <class T>
__device__ __forceinline__ void refract(const V3<T>& d, const V3<T>& n, const V3<T>& Dd,
                                        const V3<T>& dn, float eta, V3<T>& out, V3<T>& Dout) {
    T cosi = vdot(d, n);
    const T k = cst<T>(1.f) - eta * eta * (cst<T>(1.f) - cosi * cosi);
    const T neg_sq = -dsqrt(k);
    const T coso = eta * cosi - neg_sq;
    out = vsub(vscale(eta, d), vscale(coso, n));
    const T f = cst<T>(eta) - (eta * eta) * cosi / neg_sq;
    const T q = f * (vdot(Dd, n) + vdot(d, dn));
    Dout = vsub(vscale(eta, Dd), vadd(vscale(coso, dn), vscale(q, n)));
}

// D carried along direction t for length s onto the plane z = const
// (model/photon_differential.py:69-78 with n = e_z).
template <class T>
__device__ __forceinline__ V3<T> transfer_z(const V3<T>& D, const V3<T>& Dd, const T& s,
                                            const V3<T>& t) {
    const T itz = cst<T>(1.f) / t.z;  // one quotient (the same t in both of a photon's calls)
    const T a = D.z * itz;
    const T b = Dd.z * itz;
    return vadd(vsub(D, vscale(a, t)), vscale(s, vsub(Dd, vscale(b, t))));
}

// The refraction chain for one photon. Inputs: the seven height-dependent scalars.
// Outputs: receiver position (normalised) and the receiver-plane differentials (x, y parts).
template <class T>
__device__ __forceinline__ void plate_chain(const T& hz, const T& Nx, const T& Ny, const T& Nxx,
                                            const T& Nyx, const T& Nxy, const T& Nyy, float px,
                                            float py, const PlateParams& P, T& xr, T& yr,
                                            T& Dux, T& Duy, T& Dvx, T& Dvy) {
    const V3<T> d = {cst<T>(P.lx), cst<T>(P.ly), cst<T>(P.lz)};
    const V3<T> Nt = {Nx, Ny, cst<T>(1.f)};
    const T nn = vdot(Nt, Nt);
    const T nlen = dsqrt(nn);
    const V3<T> n = vscale(cst<T>(1.f) / nlen, Nt);
    const T nd = vdot(n, d);
    // source-plane differentials (du0, 0, 0) and (0, du0, 0) onto the tangent plane
    const T dnd = cst<T>(P.du0) / nd;
    const V3<T> Du1 = vsub(V3<T>{cst<T>(P.du0), cst<T>(0.f), cst<T>(0.f)}, vscale(n.x * dnd, d));
    const V3<T> Dv1 = vsub(V3<T>{cst<T>(0.f), cst<T>(P.du0), cst<T>(0.f)}, vscale(n.y * dnd, d));
    // derivative of the normalised normal along each positional differential
    const V3<T> dNu = {Nxx * Du1.x + Nxy * Du1.y, Nyx * Du1.x + Nyy * Du1.y, cst<T>(0.f)};
    const V3<T> dNv = {Nxx * Dv1.x + Nxy * Dv1.y, Nyx * Dv1.x + Nyy * Dv1.y, cst<T>(0.f)};
    const T nl3 = nn * nlen;
    const V3<T> dnu = vscale(cst<T>(1.f) / nl3, vsub(vscale(nn, dNu), vscale(vdot(Nt, dNu), Nt)));
    const V3<T> dnv = vscale(cst<T>(1.f) / nl3, vsub(vscale(nn, dNv), vscale(vdot(Nt, dNv), Nt)));
    // air -> glass at the top face
    const V3<T> zero = {cst<T>(0.f), cst<T>(0.f), cst<T>(0.f)};
    V3<T> t1, Ddu, Ddv, tmp;
    refract(d, n, zero, dnu, 1.f / P.ior, t1, Ddu);
    refract(d, n, zero, dnv, 1.f / P.ior, tmp, Ddv);
    // to the bottom face z = 0
    const T s1 = -hz / t1.z;
    const V3<T> p2 = {cst<T>(px) + s1 * t1.x, cst<T>(py) + s1 * t1.y, cst<T>(0.f)};
    const V3<T> Du2 = transfer_z(Du1, Ddu, s1, t1);
    const V3<T> Dv2 = transfer_z(Dv1, Ddv, s1, t1);
    // glass -> air at the flat bottom face (normal +z faces the glass side)
    const V3<T> ez = {cst<T>(0.f), cst<T>(0.f), cst<T>(1.f)};
    V3<T> t2, Ddu2, Ddv2;
    refract(t1, ez, Ddu, zero, P.ior, t2, Ddu2);
    refract(t1, ez, Ddv, zero, P.ior, tmp, Ddv2);
    // to the receiver plane z = -dist
    const T s2 = cst<T>(-P.dist) / t2.z;
    const V3<T> Du3 = transfer_z(Du2, Ddu2, s2, t2);
    const V3<T> Dv3 = transfer_z(Dv2, Ddv2, s2, t2);
    xr = P.inv_half * (p2.x + s2 * t2.x);
    yr = P.inv_half * (p2.y + s2 * t2.y);
    Dux = P.inv_half * Du3.x;
    Duy = P.inv_half * Du3.y;
    Dvx = P.inv_half * Dv3.x;
    Dvy = P.inv_half * Dv3.y;
}

// ---- reverse mode of the collimated chain ------------------------------------------------
// The backward needs the seven derivatives dL/dS_k of one scalar L; forward-mode duals carry
// seven tangents through every operation (eight times the arithmetic, and a register count
// that leaves one CTA per SM), reverse mode one adjoint sweep. plate_chain_adjoint runs the
// chain of plate_chain<float> forward, keeping its intermediates, then propagates the adjoints
// of the outputs back to the seven scalars, operation by operation (the derivative of each
// step written out below, from the formulas of plate_chain, refract and transfer_z).

struct V3a {
    float x, y, z;
};
__device__ __forceinline__ V3a va(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ float da(const V3a& a, const V3a& b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
__device__ __forceinline__ V3a sa(float s, const V3a& a) { return {s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ V3a pa(const V3a& a, const V3a& b) {
    return {a.x + b.x, a.y + b.y, a.z + b.z};
}
__device__ __forceinline__ V3a ma(const V3a& a, const V3a& b) {
    return {a.x - b.x, a.y - b.y, a.z - b.z};
}
__device__ __forceinline__ void acc3(V3a& a, const V3a& b) {
    a.x += b.x; a.y += b.y; a.z += b.z;
}

// transfer_z: out = D - (D.z / t.z) t + s (Dd - (Dd.z / t.z) t), with itz = 1 / t.z
__device__ __forceinline__ V3a tz_fwd(const V3a& D, const V3a& Dd, float s, const V3a& t,
                                      float itz) {
    const float a = D.z * itz, b = Dd.z * itz;
    return pa(ma(D, sa(a, t)), sa(s, ma(Dd, sa(b, t))));
}

// adjoint of tz_fwd: accumulates into Db (D), Ddb (Dd), sb (s) and tb (t) from ob (out)
__device__ __forceinline__ void tz_adj(const V3a& D, const V3a& Dd, float s, const V3a& t,
                                       float itz, const V3a& ob, V3a& Db, V3a& Ddb, float& sb,
                                       V3a& tb) {
    const float a = D.z * itz, b = Dd.z * itz;
    acc3(Db, ob);
    const float ab = -da(ob, t);
    Db.z += ab * itz;
    tb.z -= ab * a * itz;
    acc3(tb, sa(-(a + s * b), ob));
    sb += da(ob, ma(Dd, sa(b, t)));
    acc3(Ddb, sa(s, ob));
    const float bb = -s * da(ob, t);
    Ddb.z += bb * itz;
    tb.z -= bb * b * itz;
}

// d L / d S for the collimated chain; L from the splat-input gradients (as in the backward
// kernels): gx xr + gy yr + sum of gM times Mp + 4 flux gE / |den|. False for a degenerate
// photon (den == 0: no gradient). Each quotient's denominator is inverted once (eight
// reciprocals) and the sweep multiplies by the inverses.
__device__ __forceinline__ bool plate_chain_adjoint(const float S[K], float px, float py,
                                                    const PlateParams& P, float gx, float gy,
                                                    float g0, float g1, float g3, float g4,
                                                    float cE, float Sb[K]) {
    const float Nx = S[1], Ny = S[2], Nxx = S[3], Nyx = S[4], Nxy = S[5], Nyy = S[6];
    const float hz = S[0];
    const V3a d = va(P.lx, P.ly, P.lz);
    // ---- forward
    const V3a Nt = va(Nx, Ny, 1.f);
    const float nn = Nx * Nx + Ny * Ny + 1.f;
    const float nlen = sqrtf(nn);
    const float inl = 1.f / nlen;
    const V3a n = sa(inl, Nt);
    const float nd = da(n, d);
    const float ind = 1.f / nd;
    const float au = P.du0 * n.x * ind, av = P.du0 * n.y * ind;
    const V3a Du1 = ma(va(P.du0, 0.f, 0.f), sa(au, d));
    const V3a Dv1 = ma(va(0.f, P.du0, 0.f), sa(av, d));
    const V3a dNu = va(Nxx * Du1.x + Nxy * Du1.y, Nyx * Du1.x + Nyy * Du1.y, 0.f);
    const V3a dNv = va(Nxx * Dv1.x + Nxy * Dv1.y, Nyx * Dv1.x + Nyy * Dv1.y, 0.f);
    const float inl3 = inl * inl * inl;  // 1 / (nn nlen)
    const float wu = da(Nt, dNu), wv = da(Nt, dNv);
    const V3a dnu = sa(inl3, ma(sa(nn, dNu), sa(wu, Nt)));
    const V3a dnv = sa(inl3, ma(sa(nn, dNv), sa(wv, Nt)));
    const float e1 = 1.f / P.ior;
    const float cosi = da(d, n);
    const float k1 = 1.f - e1 * e1 * (1.f - cosi * cosi);
    const float ng1 = -sqrtf(k1);
    const float ing1 = 1.f / ng1;
    const float coso = e1 * cosi - ng1;
    const V3a t1 = ma(sa(e1, d), sa(coso, n));
    const float f1 = e1 - (e1 * e1) * cosi * ing1;
    const float ddu = da(d, dnu), ddv = da(d, dnv);
    const float qu = f1 * ddu, qv = f1 * ddv;
    const V3a Ddu = sa(-1.f, pa(sa(coso, dnu), sa(qu, n)));
    const V3a Ddv = sa(-1.f, pa(sa(coso, dnv), sa(qv, n)));
    const float it1z = 1.f / t1.z;
    const float s1 = -hz * it1z;
    const V3a Du2 = tz_fwd(Du1, Ddu, s1, t1, it1z);
    const V3a Dv2 = tz_fwd(Dv1, Ddv, s1, t1, it1z);
    const float e2 = P.ior;
    const float c2 = t1.z;
    const float k2 = 1.f - e2 * e2 * (1.f - c2 * c2);
    const float ng2 = -sqrtf(k2);
    const float ing2 = 1.f / ng2;
    const float coso2 = e2 * c2 - ng2;
    const V3a t2 = ma(sa(e2, t1), va(0.f, 0.f, coso2));
    const float f2 = e2 - (e2 * e2) * c2 * ing2;
    const float q2u = f2 * Ddu.z, q2v = f2 * Ddv.z;
    const V3a Ddu2 = ma(sa(e2, Ddu), va(0.f, 0.f, q2u));
    const V3a Ddv2 = ma(sa(e2, Ddv), va(0.f, 0.f, q2v));
    const float it2z = 1.f / t2.z;
    const float s2 = -P.dist * it2z;
    const V3a Du3 = tz_fwd(Du2, Ddu2, s2, t2, it2z);
    const V3a Dv3 = tz_fwd(Dv2, Ddv2, s2, t2, it2z);
    const float Dux = P.inv_half * Du3.x, Duy = P.inv_half * Du3.y;
    const float Dvx = P.inv_half * Dv3.x, Dvy = P.inv_half * Dv3.y;
    const float den = Dux * Dvy - Duy * Dvx;
    if (den == 0.f) return false;
    // ---- output adjoints: L = gx xr + gy yr + (2 / den) A + cE / |den|
    const float iden = 1.f / den;
    const float f = 2.f * iden;
    const float A = g0 * Dvy - g1 * Dvx - g3 * Duy + g4 * Dux;
    const float denb = (-f * A - cE * copysignf(1.f, den) * iden) * iden;
    const float Duxb = f * g4 + denb * Dvy, Duyb = -f * g3 - denb * Dvx;
    const float Dvxb = -f * g1 - denb * Duy, Dvyb = f * g0 + denb * Dux;
    const float p2xb = P.inv_half * gx, p2yb = P.inv_half * gy;
    // ---- reverse sweep
    V3a t2b = va(P.inv_half * gx * s2, P.inv_half * gy * s2, 0.f);
    float s2b = P.inv_half * (gx * t2.x + gy * t2.y);
    V3a Du2b = va(0.f, 0.f, 0.f), Dv2b = Du2b, Ddu2b = Du2b, Ddv2b = Du2b;
    tz_adj(Du2, Ddu2, s2, t2, it2z, va(P.inv_half * Duxb, P.inv_half * Duyb, 0.f), Du2b, Ddu2b,
           s2b, t2b);
    tz_adj(Dv2, Ddv2, s2, t2, it2z, va(P.inv_half * Dvxb, P.inv_half * Dvyb, 0.f), Dv2b, Ddv2b,
           s2b, t2b);
    t2b.z += s2b * P.dist * it2z * it2z;
    // bottom refraction
    V3a Dub = sa(e2, Ddu2b), Dvb = sa(e2, Ddv2b);  // adjoints of Ddu, Ddv
    const float q2ub = -Ddu2b.z, q2vb = -Ddv2b.z;
    Dub.z += f2 * q2ub;
    Dvb.z += f2 * q2vb;
    const float f2b = Ddu.z * q2ub + Ddv.z * q2vb;
    V3a t1b = sa(e2, t2b);
    const float coso2b = -t2b.z;
    float c2b = e2 * coso2b - (e2 * e2) * ing2 * f2b;
    float ng2b = -coso2b + (e2 * e2) * c2 * ing2 * ing2 * f2b;
    const float k2b = 0.5f * ng2b * ing2;
    c2b += 2.f * e2 * e2 * c2 * k2b;
    t1b.z += c2b;
    // bottom transfer
    V3a Du1b = va(0.f, 0.f, 0.f), Dv1b = Du1b;
    float s1b = p2xb * t1.x + p2yb * t1.y;
    t1b.x += p2xb * s1;
    t1b.y += p2yb * s1;
    tz_adj(Du1, Ddu, s1, t1, it1z, Du2b, Du1b, Dub, s1b, t1b);
    tz_adj(Dv1, Ddv, s1, t1, it1z, Dv2b, Dv1b, Dvb, s1b, t1b);
    const float hzb = -s1b * it1z;
    t1b.z += s1b * hz * it1z * it1z;
    // top refraction (Dd = 0): Ddu = -(coso dnu + qu n), qu = f1 (d . dnu)
    V3a nb = va(0.f, 0.f, 0.f);
    float cosob = -da(Dub, dnu) - da(Dvb, dnv) - da(t1b, n);
    V3a dnub = sa(-coso, Dub), dnvb = sa(-coso, Dvb);
    const float qub = -da(Dub, n), qvb = -da(Dvb, n);
    acc3(nb, sa(-qu, Dub));
    acc3(nb, sa(-qv, Dvb));
    acc3(nb, sa(-coso, t1b));
    const float f1b = qub * ddu + qvb * ddv;
    acc3(dnub, sa(qub * f1, d));
    acc3(dnvb, sa(qvb * f1, d));
    float cosib = e1 * cosob - (e1 * e1) * ing1 * f1b;
    const float ng1b = -cosob + (e1 * e1) * cosi * ing1 * ing1 * f1b;
    const float k1b = 0.5f * ng1b * ing1;
    cosib += 2.f * e1 * e1 * cosi * k1b;
    acc3(nb, sa(cosib, d));
    // dn = (nn dN - w Nt) / nl3
    V3a Ntb = va(0.f, 0.f, 0.f);
    float nnb = 0.f, nl3b = 0.f;
    V3a dNub = sa(nn * inl3, dnub), dNvb = sa(nn * inl3, dnvb);
    const float wub = -da(dnub, Nt) * inl3, wvb = -da(dnvb, Nt) * inl3;
    acc3(dNub, sa(wub, Nt));
    acc3(dNvb, sa(wvb, Nt));
    acc3(Ntb, sa(wub, dNu));
    acc3(Ntb, sa(wvb, dNv));
    acc3(Ntb, sa(-wu * inl3, dnub));
    acc3(Ntb, sa(-wv * inl3, dnvb));
    nnb += (da(dnub, dNu) + da(dnvb, dNv)) * inl3;
    nl3b -= (da(dnub, dnu) + da(dnvb, dnv)) * inl3;
    nnb += 1.5f * nlen * nl3b;
    // dN = (Nxx D.x + Nxy D.y, Nyx D.x + Nyy D.y, 0)
    Sb[3] = dNub.x * Du1.x + dNvb.x * Dv1.x;  // Nxx
    Sb[5] = dNub.x * Du1.y + dNvb.x * Dv1.y;  // Nxy
    Sb[4] = dNub.y * Du1.x + dNvb.y * Dv1.x;  // Nyx
    Sb[6] = dNub.y * Du1.y + dNvb.y * Dv1.y;  // Nyy
    Du1b.x += dNub.x * Nxx + dNub.y * Nyx;
    Du1b.y += dNub.x * Nxy + dNub.y * Nyy;
    Dv1b.x += dNvb.x * Nxx + dNvb.y * Nyx;
    Dv1b.y += dNvb.x * Nxy + dNvb.y * Nyy;
    // Du1 = (du0, 0, 0) - au d, au = du0 n.x / nd (Dv1 with n.y)
    const float aub = -da(Du1b, d), avb = -da(Dv1b, d);
    nb.x += aub * P.du0 * ind;
    nb.y += avb * P.du0 * ind;
    const float ndb = -(aub * au + avb * av) * ind;
    acc3(nb, sa(ndb, d));
    // n = Nt / sqrt(nn)
    acc3(Ntb, sa(inl, nb));
    const float inlb = da(nb, Nt);
    nnb += -0.5f * inl * inl * inl * inlb;  // d inl / d nn = -1 / (2 nn^1.5)
    Sb[0] = hzb;
    Sb[1] = Ntb.x + 2.f * Nx * nnb;
    Sb[2] = Ntb.y + 2.f * Ny * nnb;
    return true;
}

// Bilinear footprint of a world position on the height-field grid (texel centres at
// integers, clamped to the border).
struct Bilin {
    int x0, y0;
    float ax, ay;
};

__device__ __forceinline__ Bilin bilin(float px, float py, float texel, int H, int W) {
    float fx = px / texel + 0.5f * float(W - 1);
    float fy = py / texel + 0.5f * float(H - 1);
    fx = fminf(fmaxf(fx, 0.f), float(W - 1));
    fy = fminf(fmaxf(fy, 0.f), float(H - 1));
    Bilin b;
    b.x0 = min(int(floorf(fx)), max(W - 2, 0));
    b.y0 = min(int(floorf(fy)), max(H - 2, 0));
    b.ax = fx - float(b.x0);
    b.ay = fy - float(b.y0);
    return b;
}

__device__ __forceinline__ float hat(const float* h, int H, int W, int i, int j) {
    i = min(max(i, 0), H - 1);
    j = min(max(j, 0), W - 1);
    return __ldg(h + int64_t(i) * W + j);
}

// Position derivatives of the surface at a sample (for the traced hit).
struct SurfGeo {
    float hx, hy;        // slope of the bilinear height
    float tw_nx, tw_ny;  // d2 Nx / dx dy, d2 Ny / dx dy of the bilinear normal field
};

// The seven scalars of one photon: height, Sobel normal (x, y) and their x/y derivatives;
// with geo, also the position derivatives of the sample.
__device__ __forceinline__ void surface_scalars(const float* h, int H, int W, float texel,
                                                const Bilin& b, float s[K],
                                                SurfGeo* geo = nullptr) {
    const float itex = 1.f / texel;  // one quotient; the stencils multiply by it
    const float c = -0.125f * itex;
    float hv[2][2], nx[2][2], ny[2][2];
#pragma unroll
    for (int r = 0; r < 2; ++r) {
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int i = b.y0 + r, j = min(b.x0 + q, W - 1);
            hv[r][q] = hat(h, H, W, i, j);
            nx[r][q] = c * (hat(h, H, W, i - 1, j + 1) - hat(h, H, W, i - 1, j - 1) +
                            2.f * (hat(h, H, W, i, j + 1) - hat(h, H, W, i, j - 1)) +
                            hat(h, H, W, i + 1, j + 1) - hat(h, H, W, i + 1, j - 1));
            ny[r][q] = c * (hat(h, H, W, i + 1, j - 1) - hat(h, H, W, i - 1, j - 1) +
                            2.f * (hat(h, H, W, i + 1, j) - hat(h, H, W, i - 1, j)) +
                            hat(h, H, W, i + 1, j + 1) - hat(h, H, W, i - 1, j + 1));
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
    // backward inputs / output
    const float* gE;
    const float* gX;
    const float* gM;
    float* gh;
};

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

__global__ __launch_bounds__(256) void refract_fwd_kernel(RefractArgs a) {
    const int64_t n = a.n;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += int64_t(gridDim.x) * blockDim.x) {
        const float px = a.px[i], py = a.py[i];
        const PlateParams P = photon_params(a, i);
        const Bilin b = bilin(px, py, P.texel, a.H, a.W);
        float s[K];
        surface_scalars(a.h, a.H, a.W, P.texel, b, s);
        float xr, yr, Dux, Duy, Dvx, Dvy;
        plate_chain<float>(s[0], s[1], s[2], s[3], s[4], s[5], s[6], px, py, P, xr, yr, Dux,
                           Duy, Dvx, Dvy);
        const float den = Dux * Dvy - Duy * Dvx;
        const bool good = den != 0.f;
        const float f = 2.f / (good ? den : 1.f);
        a.Mp[i] = f * Dvy;
        a.Mp[n + i] = -f * Dvx;
        a.Mp[2 * n + i] = 0.f;
        a.Mp[3 * n + i] = -f * Duy;
        a.Mp[4 * n + i] = f * Dux;
        a.Mp[5 * n + i] = 0.f;
        a.xp[i] = xr;
        a.xp[n + i] = yr;
        a.radius[i] = 0.5f * fmaxf(sqrtf(Dux * Dux + Duy * Duy), sqrtf(Dvx * Dvx + Dvy * Dvy));
        a.Ep[i] = 4.f * a.flux[i] / (good ? fabsf(den) : 1.f);
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
    const float it = 1.f / texel;
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
// in shared memory and added to the
// field once per texel; otherwise (scattered hits) each patch entry is a global atomic add.
// Without it, every photon's 16 patch entries were global atomics on a few hot texels.
constexpr int kPatchSmem = 8192;  // floats of the CTA's shared patch region (32 KB)

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
__device__ __forceinline__ PatchAcc patch_begin(float* smem, int* bb, bool active, int bx0,
                                                int by0, float* gh, int H, int W) {
    if (threadIdx.x == 0) {
        bb[0] = INT_MAX; bb[1] = INT_MIN; bb[2] = INT_MAX; bb[3] = INT_MIN;
    }
    __syncthreads();
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
    __syncthreads();
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
        if (int64_t(rw) * rh <= kPatchSmem) {
            acc.buf = smem;
            acc.x0 = x0;
            acc.y0 = y0;
            acc.rw = rw;
            for (int k = threadIdx.x; k < rw * rh; k += blockDim.x) smem[k] = 0.f;
        }
    }
    __syncthreads();
    return acc;
}

// Adds the CTA's shared region to the field (all threads call it).
__device__ __forceinline__ void patch_end(const PatchAcc& acc, int* bb, int H, int W) {
    __syncthreads();
    if (acc.buf) {
        const int x1 = min(bb[1] + 2, W - 1), y1 = min(bb[3] + 2, H - 1);
        const int rh = y1 - acc.y0 + 1;
        for (int k = threadIdx.x; k < acc.rw * rh; k += blockDim.x) {
            const float v = acc.buf[k];
            if (v != 0.f)
                atomicAdd(acc.gh + int64_t(acc.y0 + k / acc.rw) * W + acc.x0 + k % acc.rw, v);
        }
    }
    __syncthreads();
}

// Three CTAs an SM (80 registers, a few spilled to the L1): measured 18% faster than the
// 114-register build at two CTAs an SM (16.8 M photons of a 1024^2 field: 2.24 vs 2.73 ms).
__global__ __launch_bounds__(256, 3) void refract_bwd_kernel(RefractArgs a) {
    __shared__ float smem[kPatchSmem];
    __shared__ int bb[4];
    const int64_t n = a.n;
    // CTA-contiguous blocks of 256 photons (their patches share a shared-memory region)
    for (int64_t blk = int64_t(blockIdx.x) * blockDim.x; blk < n;
         blk += int64_t(gridDim.x) * blockDim.x) {
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
            active = plate_chain_adjoint(s, px, py, P, a.gX[i], a.gX[n + i], a.gM[i],
                                         a.gM[n + i], a.gM[3 * n + i], a.gM[4 * n + i],
                                         4.f * a.flux[i] * a.gE[i], c);
        }
        const PatchAcc acc = patch_begin(smem, bb, active, b.x0, b.y0, a.gh, a.H, a.W);
        if (active) scatter_patch(a.H, a.W, texel, b, c, acc);
        patch_end(acc, bb, a.H, a.W);
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

struct Ray {
    float ox, oy, oz;
    float dx, dy, dz;
};

// Newton iterations of the trace; false when the ray grazes the surface or its hit lies
// outside the field. b, s, geo: the surface at the hit; t: the ray parameter; fp: f'(t).
__device__ __forceinline__ bool trace_hit(const float* h, int H, int W, float texel,
                                          float plane_z, const Ray& r, float& t, Bilin& b,
                                          float s[K], SurfGeo& geo, float& fp) {
    t = (r.oz - plane_z) / (-r.dz);
    const float cx = 0.5f * float(W - 1), cy = 0.5f * float(H - 1);
    for (int it = 0; it < 10; ++it) {
        const float px = r.ox + t * r.dx, py = r.oy + t * r.dy, pz = r.oz + t * r.dz;
        b = bilin(px, py, texel, H, W);
        surface_scalars(h, H, W, texel, b, s, &geo);
        fp = r.dz - (geo.hx * r.dx + geo.hy * r.dy);
        if (!(fabsf(fp) > 1e-6f)) return false;
        const float step = (pz - s[0]) / fp;
        t -= step;
        if (fabsf(step) <= 1e-7f * fabsf(t)) break;
    }
    const float px = r.ox + t * r.dx, py = r.oy + t * r.dy;
    const float fx = px / texel + cx, fy = py / texel + cy;
    if (!(fx >= 0.f && fx <= float(W - 1) && fy >= 0.f && fy <= float(H - 1))) return false;
    b = bilin(px, py, texel, H, W);
    surface_scalars(h, H, W, texel, b, s, &geo);
    fp = r.dz - (geo.hx * r.dx + geo.hy * r.dy);
    return fabsf(fp) > 1e-6f;
}

// The refraction chain of one point-light photon from its hit parameter t and the six normal
// scalars at the hit (Nx, Ny, dNx/dx, dNy/dx, dNx/dy, dNy/dy).
template <class T>
__device__ __forceinline__ void point_chain(const T& t, const T& Nx, const T& Ny, const T& Nxx,
                                            const T& Nyx, const T& Nxy, const T& Nyy,
                                            const Ray& r, const V3<float>& Dth,
                                            const V3<float>& Dph, const PlateParams& P, T& xr,
                                            T& yr, T& Dux, T& Duy, T& Dvx, T& Dvy) {
    const V3<T> d = {cst<T>(r.dx), cst<T>(r.dy), cst<T>(r.dz)};
    const V3<T> Dt = {cst<T>(Dth.x), cst<T>(Dth.y), cst<T>(Dth.z)};
    const V3<T> Dp = {cst<T>(Dph.x), cst<T>(Dph.y), cst<T>(Dph.z)};
    const V3<T> p1 = {cst<T>(r.ox) + t * d.x, cst<T>(r.oy) + t * d.y, cst<T>(r.oz) + t * d.z};
    const V3<T> Nt = {Nx, Ny, cst<T>(1.f)};
    const T nn = vdot(Nt, Nt);
    const T nlen = dsqrt(nn);
    const V3<T> n = vscale(cst<T>(1.f) / nlen, Nt);
    const T nd = vdot(n, d);
    // positional differentials carried from the light over t onto the tangent plane
    const V3<T> Du1 = vscale(t, vsub(Dt, vscale(vdot(n, Dt) / nd, d)));
    const V3<T> Dv1 = vscale(t, vsub(Dp, vscale(vdot(n, Dp) / nd, d)));
    const V3<T> dNu = {Nxx * Du1.x + Nxy * Du1.y, Nyx * Du1.x + Nyy * Du1.y, cst<T>(0.f)};
    const V3<T> dNv = {Nxx * Dv1.x + Nxy * Dv1.y, Nyx * Dv1.x + Nyy * Dv1.y, cst<T>(0.f)};
    const T nl3 = nn * nlen;
    const V3<T> dnu = vscale(cst<T>(1.f) / nl3, vsub(vscale(nn, dNu), vscale(vdot(Nt, dNu), Nt)));
    const V3<T> dnv = vscale(cst<T>(1.f) / nl3, vsub(vscale(nn, dNv), vscale(vdot(Nt, dNv), Nt)));
    V3<T> t1, Ddu, Ddv, tmp;
    refract(d, n, Dt, dnu, 1.f / P.ior, t1, Ddu);
    refract(d, n, Dp, dnv, 1.f / P.ior, tmp, Ddv);
    const T s1 = -p1.z / t1.z;
    const V3<T> p2 = {p1.x + s1 * t1.x, p1.y + s1 * t1.y, cst<T>(0.f)};
    const V3<T> Du2 = transfer_z(Du1, Ddu, s1, t1);
    const V3<T> Dv2 = transfer_z(Dv1, Ddv, s1, t1);
    const V3<T> ez = {cst<T>(0.f), cst<T>(0.f), cst<T>(1.f)};
    const V3<T> zero = {cst<T>(0.f), cst<T>(0.f), cst<T>(0.f)};
    V3<T> t2, Ddu2, Ddv2;
    refract(t1, ez, Ddu, zero, P.ior, t2, Ddu2);
    refract(t1, ez, Ddv, zero, P.ior, tmp, Ddv2);
    const T s2 = cst<T>(-P.dist) / t2.z;
    const V3<T> Du3 = transfer_z(Du2, Ddu2, s2, t2);
    const V3<T> Dv3 = transfer_z(Dv2, Ddv2, s2, t2);
    xr = P.inv_half * (p2.x + s2 * t2.x);
    yr = P.inv_half * (p2.y + s2 * t2.y);
    Dux = P.inv_half * Du3.x;
    Duy = P.inv_half * Du3.y;
    Dvx = P.inv_half * Dv3.x;
    Dvy = P.inv_half * Dv3.y;
}

// Reverse mode of point_chain (the adjoint sweep of plate_chain_adjoint with the point
// light's differences: the hit p1 = o + t d moves with t, the positional differentials are
// t (D - (n.D / n.d) d) for the light's direction differentials D, and the top refraction
// carries those direction differentials). Returns d L / d t at fixed normal scalars (tb) and
// d L / d S_k for the six normal scalars S[1..6]; L as in plate_chain_adjoint. False for a
// degenerate photon.
__device__ __forceinline__ bool point_chain_adjoint(float t, const float S[K], const Ray& r,
                                                    const V3<float>& Dth,
                                                    const V3<float>& Dph,
                                                    const PlateParams& P, float gx, float gy,
                                                    float g0, float g1, float g3, float g4,
                                                    float cE, float& tb, float Sb[K]) {
    const float Nx = S[1], Ny = S[2], Nxx = S[3], Nyx = S[4], Nxy = S[5], Nyy = S[6];
    const V3a d = va(r.dx, r.dy, r.dz);
    const V3a Dt = va(Dth.x, Dth.y, Dth.z), Dp = va(Dph.x, Dph.y, Dph.z);
    // ---- forward
    const V3a p1 = va(r.ox + t * d.x, r.oy + t * d.y, r.oz + t * d.z);
    const V3a Nt = va(Nx, Ny, 1.f);
    const float nn = Nx * Nx + Ny * Ny + 1.f;
    const float nlen = sqrtf(nn);
    const float inl = 1.f / nlen;
    const V3a n = sa(inl, Nt);
    const float nd = da(n, d);
    const float ind = 1.f / nd;
    const float aT = da(n, Dt) * ind, aP = da(n, Dp) * ind;
    const V3a Eu = ma(Dt, sa(aT, d)), Ev = ma(Dp, sa(aP, d));
    const V3a Du1 = sa(t, Eu), Dv1 = sa(t, Ev);
    const V3a dNu = va(Nxx * Du1.x + Nxy * Du1.y, Nyx * Du1.x + Nyy * Du1.y, 0.f);
    const V3a dNv = va(Nxx * Dv1.x + Nxy * Dv1.y, Nyx * Dv1.x + Nyy * Dv1.y, 0.f);
    const float inl3 = inl * inl * inl;
    const float wu = da(Nt, dNu), wv = da(Nt, dNv);
    const V3a dnu = sa(inl3, ma(sa(nn, dNu), sa(wu, Nt)));
    const V3a dnv = sa(inl3, ma(sa(nn, dNv), sa(wv, Nt)));
    const float e1 = 1.f / P.ior;
    const float cosi = da(d, n);
    const float k1 = 1.f - e1 * e1 * (1.f - cosi * cosi);
    const float ng1 = -sqrtf(k1);
    const float ing1 = 1.f / ng1;
    const float coso = e1 * cosi - ng1;
    const V3a t1 = ma(sa(e1, d), sa(coso, n));
    const float f1 = e1 - (e1 * e1) * cosi * ing1;
    const float ddu = da(Dt, n) + da(d, dnu), ddv = da(Dp, n) + da(d, dnv);
    const float qu = f1 * ddu, qv = f1 * ddv;
    const V3a Ddu = ma(sa(e1, Dt), pa(sa(coso, dnu), sa(qu, n)));
    const V3a Ddv = ma(sa(e1, Dp), pa(sa(coso, dnv), sa(qv, n)));
    const float it1z = 1.f / t1.z;
    const float s1 = -p1.z * it1z;
    const V3a Du2 = tz_fwd(Du1, Ddu, s1, t1, it1z);
    const V3a Dv2 = tz_fwd(Dv1, Ddv, s1, t1, it1z);
    const float e2 = P.ior;
    const float c2 = t1.z;
    const float k2 = 1.f - e2 * e2 * (1.f - c2 * c2);
    const float ng2 = -sqrtf(k2);
    const float ing2 = 1.f / ng2;
    const float coso2 = e2 * c2 - ng2;
    const V3a t2 = ma(sa(e2, t1), va(0.f, 0.f, coso2));
    const float f2 = e2 - (e2 * e2) * c2 * ing2;
    const float q2u = f2 * Ddu.z, q2v = f2 * Ddv.z;
    const V3a Ddu2 = ma(sa(e2, Ddu), va(0.f, 0.f, q2u));
    const V3a Ddv2 = ma(sa(e2, Ddv), va(0.f, 0.f, q2v));
    const float it2z = 1.f / t2.z;
    const float s2 = -P.dist * it2z;
    const V3a Du3 = tz_fwd(Du2, Ddu2, s2, t2, it2z);
    const V3a Dv3 = tz_fwd(Dv2, Ddv2, s2, t2, it2z);
    const float Dux = P.inv_half * Du3.x, Duy = P.inv_half * Du3.y;
    const float Dvx = P.inv_half * Dv3.x, Dvy = P.inv_half * Dv3.y;
    const float den = Dux * Dvy - Duy * Dvx;
    if (den == 0.f) return false;
    // ---- output adjoints
    const float iden = 1.f / den;
    const float f = 2.f * iden;
    const float A = g0 * Dvy - g1 * Dvx - g3 * Duy + g4 * Dux;
    const float denb = (-f * A - cE * copysignf(1.f, den) * iden) * iden;
    const float Duxb = f * g4 + denb * Dvy, Duyb = -f * g3 - denb * Dvx;
    const float Dvxb = -f * g1 - denb * Duy, Dvyb = f * g0 + denb * Dux;
    const float p2xb = P.inv_half * gx, p2yb = P.inv_half * gy;
    // ---- reverse sweep: receiver transfer and bottom refraction as for collimated light
    V3a t2b = va(P.inv_half * gx * s2, P.inv_half * gy * s2, 0.f);
    float s2b = P.inv_half * (gx * t2.x + gy * t2.y);
    V3a Du2b = va(0.f, 0.f, 0.f), Dv2b = Du2b, Ddu2b = Du2b, Ddv2b = Du2b;
    tz_adj(Du2, Ddu2, s2, t2, it2z, va(P.inv_half * Duxb, P.inv_half * Duyb, 0.f), Du2b, Ddu2b,
           s2b, t2b);
    tz_adj(Dv2, Ddv2, s2, t2, it2z, va(P.inv_half * Dvxb, P.inv_half * Dvyb, 0.f), Dv2b, Ddv2b,
           s2b, t2b);
    t2b.z += s2b * P.dist * it2z * it2z;
    V3a Dub = sa(e2, Ddu2b), Dvb = sa(e2, Ddv2b);  // adjoints of Ddu, Ddv
    const float q2ub = -Ddu2b.z, q2vb = -Ddv2b.z;
    Dub.z += f2 * q2ub;
    Dvb.z += f2 * q2vb;
    const float f2b = Ddu.z * q2ub + Ddv.z * q2vb;
    V3a t1b = sa(e2, t2b);
    const float coso2b = -t2b.z;
    float c2b = e2 * coso2b - (e2 * e2) * ing2 * f2b;
    const float ng2b = -coso2b + (e2 * e2) * c2 * ing2 * ing2 * f2b;
    const float k2b = 0.5f * ng2b * ing2;
    c2b += 2.f * e2 * e2 * c2 * k2b;
    t1b.z += c2b;
    // bottom transfer from the hit p1 (p2 = p1 + s1 t1, s1 = -p1.z / t1.z)
    V3a Du1b = va(0.f, 0.f, 0.f), Dv1b = Du1b;
    float s1b = p2xb * t1.x + p2yb * t1.y;
    t1b.x += p2xb * s1;
    t1b.y += p2yb * s1;
    tz_adj(Du1, Ddu, s1, t1, it1z, Du2b, Du1b, Dub, s1b, t1b);
    tz_adj(Dv1, Ddv, s1, t1, it1z, Dv2b, Dv1b, Dvb, s1b, t1b);
    const float p1zb = -s1b * it1z;
    t1b.z += s1b * p1.z * it1z * it1z;
    tb = p2xb * d.x + p2yb * d.y + p1zb * d.z;
    // top refraction with the light's direction differentials:
    // Ddu = e1 Dt - (coso dnu + qu n), qu = f1 (Dt . n + d . dnu)
    V3a nb = va(0.f, 0.f, 0.f);
    const float cosob = -da(Dub, dnu) - da(Dvb, dnv) - da(t1b, n);
    V3a dnub = sa(-coso, Dub), dnvb = sa(-coso, Dvb);
    const float qub = -da(Dub, n), qvb = -da(Dvb, n);
    acc3(nb, sa(-qu, Dub));
    acc3(nb, sa(-qv, Dvb));
    acc3(nb, sa(-coso, t1b));
    const float f1b = qub * ddu + qvb * ddv;
    const float ddub = qub * f1, ddvb = qvb * f1;
    acc3(dnub, sa(ddub, d));
    acc3(dnvb, sa(ddvb, d));
    acc3(nb, sa(ddub, Dt));
    acc3(nb, sa(ddvb, Dp));
    float cosib = e1 * cosob - (e1 * e1) * ing1 * f1b;
    const float ng1b = -cosob + (e1 * e1) * cosi * ing1 * ing1 * f1b;
    const float k1b = 0.5f * ng1b * ing1;
    cosib += 2.f * e1 * e1 * cosi * k1b;
    acc3(nb, sa(cosib, d));
    // dn = (nn dN - w Nt) / nn^1.5
    V3a Ntb = va(0.f, 0.f, 0.f);
    float nnb = 0.f, nl3b = 0.f;
    V3a dNub = sa(nn * inl3, dnub), dNvb = sa(nn * inl3, dnvb);
    const float wub = -da(dnub, Nt) * inl3, wvb = -da(dnvb, Nt) * inl3;
    acc3(dNub, sa(wub, Nt));
    acc3(dNvb, sa(wvb, Nt));
    acc3(Ntb, sa(wub, dNu));
    acc3(Ntb, sa(wvb, dNv));
    acc3(Ntb, sa(-wu * inl3, dnub));
    acc3(Ntb, sa(-wv * inl3, dnvb));
    nnb += (da(dnub, dNu) + da(dnvb, dNv)) * inl3;
    nl3b -= (da(dnub, dnu) + da(dnvb, dnv)) * inl3;
    nnb += 1.5f * nlen * nl3b;
    Sb[3] = dNub.x * Du1.x + dNvb.x * Dv1.x;  // Nxx
    Sb[5] = dNub.x * Du1.y + dNvb.x * Dv1.y;  // Nxy
    Sb[4] = dNub.y * Du1.x + dNvb.y * Dv1.x;  // Nyx
    Sb[6] = dNub.y * Du1.y + dNvb.y * Dv1.y;  // Nyy
    Du1b.x += dNub.x * Nxx + dNub.y * Nyx;
    Du1b.y += dNub.x * Nxy + dNub.y * Nyy;
    Dv1b.x += dNvb.x * Nxx + dNvb.y * Nyx;
    Dv1b.y += dNvb.x * Nxy + dNvb.y * Nyy;
    // Du1 = t (Dt - aT d), aT = (n . Dt) / nd (Dv1 with Dp)
    tb += da(Du1b, Eu) + da(Dv1b, Ev);
    const float aTb = -t * da(Du1b, d), aPb = -t * da(Dv1b, d);
    acc3(nb, sa(aTb * ind, Dt));
    acc3(nb, sa(aPb * ind, Dp));
    const float ndb = -(aTb * aT + aPb * aP) * ind;
    acc3(nb, sa(ndb, d));
    // n = Nt / sqrt(nn)
    acc3(Ntb, sa(inl, nb));
    const float inlb = da(nb, Nt);
    nnb += -0.5f * inl * inl * inl * inlb;
    Sb[0] = 0.f;  // the height enters through t only
    Sb[1] = Ntb.x + 2.f * Nx * nnb;
    Sb[2] = Ntb.y + 2.f * Ny * nnb;
    return true;
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
        const float f = 2.f / (good ? den : 1.f);
        a.Mp[i] = f * Dvy;
        a.Mp[n + i] = -f * Dvx;
        a.Mp[2 * n + i] = 0.f;
        a.Mp[3 * n + i] = -f * Duy;
        a.Mp[4 * n + i] = f * Dux;
        a.Mp[5 * n + i] = 0.f;
        a.xp[i] = xr;
        a.xp[n + i] = yr;
        a.radius[i] = 0.5f * fmaxf(sqrtf(Dux * Dux + Duy * Duy), sqrtf(Dvx * Dvx + Dvy * Dvy));
        a.Ep[i] = 4.f * a.flux[i] / (good ? fabsf(den) : 1.f);
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
        c[0] = Lt / fp;
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

int grid_for(int64_t n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t blocks = (n + 255) / 256;
    const int64_t cap = int64_t(sms) * 8;
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
        point_bwd_kernel<<<grid_for(n), 256, 0, st>>>(a);
    else
        point_fwd_kernel<<<grid_for(n), 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_refract(bool backward, const float* h, int H, int W, const pds_plate& plate,
                           const pds_plate* plates, const int64_t* begins, int32_t n_sims,
                           const float* px, const float* py, const float* flux,
                           const int64_t* channel, int64_t n, float* Ep, float* xp, float* Mp,
                           int64_t* cp, float* radius, const float* gE, const float* gX,
                           const float* gM, float* gh, cudaStream_t st) {
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
    a.gh = gh;
    if (backward)
        refract_bwd_kernel<<<grid_for(n), 256, 0, st>>>(a);
    else
        refract_fwd_kernel<<<grid_for(n), 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace pds
