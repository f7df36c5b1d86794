// The refraction chain of a height-field plate and its reverse-mode adjoints, shared by the
// refraction kernels (pds_refract.cu) and a host build of the adjoint check (the chain
// templates instantiated with forward-mode dual numbers, tests/chain_adjoint_check.cu).
//
// plate_chain: collimated (tilted) light through a plate with a height-field top face and a
// flat bottom face to the receiver plane (model/caustics.py:123-212, the transfer of
// model/photon_differential.py:69-78); point_chain: the same from a point light's hit on the
// surface. plate_chain_adjoint / point_chain_adjoint: one reverse sweep each, from the
// splat-input gradients to the photon's height-dependent scalars.
#pragma once

#include <cmath>
#include <cstdint>

#include "../../include/pds_b200.h"

#define PDS_HD __host__ __device__ __forceinline__

namespace pds {
namespace chain {

constexpr int K = 7;  // height-dependent scalars of one photon

PDS_HD float dsqrt(float a) { return sqrtf(a); }

template <class T>
struct V3 {
    T x, y, z;
};
template <class T>
PDS_HD V3<T> vadd(const V3<T>& a, const V3<T>& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T>
PDS_HD V3<T> vsub(const V3<T>& a, const V3<T>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T, class S>
PDS_HD V3<T> vscale(const S& s, const V3<T>& a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T>
PDS_HD T vdot(const V3<T>& a, const V3<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

template <class T>
PDS_HD T cst(float v);
template <>
PDS_HD float cst<float>(float v) { return v; }

// Single-precision quotients of the chain. On the device they take the hardware reciprocal
// (__fdividef: within 2 ulp of the correctly rounded quotient; a reciprocal and a multiply
// where the IEEE quotient adds a refinement sequence and a range check), on the host (the
// dual-number check's build) the IEEE quotient. Dual numbers divide as they define.
PDS_HD float qdiv(float a, float b) {
#ifdef __CUDA_ARCH__
    return __fdividef(a, b);
#else
    return a / b;
#endif
}
template <class T>
PDS_HD T qdiv(const T& a, const T& b) { return a / b; }

// 1 / sqrt(a) of the chain: on the device the hardware reciprocal square root (rsqrtf, within
// 2 ulp), from which the chain also forms sqrt(a) = a / sqrt(a) (its roots are of norms >= 1
// and of Snell's 1 - eta^2 sin^2, positive short of total internal reflection); on the host
// the IEEE quotient of the IEEE root.
PDS_HD float rsq(float a) {
#ifdef __CUDA_ARCH__
    return rsqrtf(a);
#else
    return 1.f / sqrtf(a);
#endif
}
template <class T>
PDS_HD T rsq(const T& a) { return cst<T>(1.f) / dsqrt(a); }

struct PlateParams {
    float texel, ior, dist, inv_half, du0;
    float lx, ly, lz;  // light direction
};

PDS_HD PlateParams to_params(const pds_plate& p) {
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
PDS_HD void refract(const V3<T>& d, const V3<T>& n, const V3<T>& Dd,
                                        const V3<T>& dn, float eta, V3<T>& out, V3<T>& Dout) {
    T cosi = vdot(d, n);
    const T k = cst<T>(1.f) - eta * eta * (cst<T>(1.f) - cosi * cosi);
    const T rk = rsq(k);
    const T neg_sq = -(k * rk);
    const T coso = eta * cosi - neg_sq;
    out = vsub(vscale(eta, d), vscale(coso, n));
    const T f = cst<T>(eta) + (eta * eta) * cosi * rk;
    const T q = f * (vdot(Dd, n) + vdot(d, dn));
    Dout = vsub(vscale(eta, Dd), vadd(vscale(coso, dn), vscale(q, n)));
}

// D carried along direction t for length s onto the plane z = const
// (model/photon_differential.py:69-78 with n = e_z).
template <class T>
PDS_HD V3<T> transfer_z(const V3<T>& D, const V3<T>& Dd, const T& s,
                                            const V3<T>& t) {
    const T itz = qdiv(cst<T>(1.f), t.z);  // one quotient (the same t in both of a photon's calls)
    const T a = D.z * itz;
    const T b = Dd.z * itz;
    return vadd(vsub(D, vscale(a, t)), vscale(s, vsub(Dd, vscale(b, t))));
}

// The refraction chain for one photon. Inputs: the seven height-dependent scalars.
// Outputs: receiver position (normalised) and the receiver-plane differentials (x, y parts).
template <class T>
PDS_HD void plate_chain(const T& hz, const T& Nx, const T& Ny, const T& Nxx,
                                            const T& Nyx, const T& Nxy, const T& Nyy, float px,
                                            float py, const PlateParams& P, T& xr, T& yr,
                                            T& Dux, T& Duy, T& Dvx, T& Dvy) {
    const V3<T> d = {cst<T>(P.lx), cst<T>(P.ly), cst<T>(P.lz)};
    const V3<T> Nt = {Nx, Ny, cst<T>(1.f)};
    const T nn = vdot(Nt, Nt);
    const T inl = rsq(nn);
    const V3<T> n = vscale(inl, Nt);
    const T nd = vdot(n, d);
    // source-plane differentials (du0, 0, 0) and (0, du0, 0) onto the tangent plane
    const T dnd = qdiv(cst<T>(P.du0), nd);
    const V3<T> Du1 = vsub(V3<T>{cst<T>(P.du0), cst<T>(0.f), cst<T>(0.f)}, vscale(n.x * dnd, d));
    const V3<T> Dv1 = vsub(V3<T>{cst<T>(0.f), cst<T>(P.du0), cst<T>(0.f)}, vscale(n.y * dnd, d));
    // derivative of the normalised normal along each positional differential
    const V3<T> dNu = {Nxx * Du1.x + Nxy * Du1.y, Nyx * Du1.x + Nyy * Du1.y, cst<T>(0.f)};
    const V3<T> dNv = {Nxx * Dv1.x + Nxy * Dv1.y, Nyx * Dv1.x + Nyy * Dv1.y, cst<T>(0.f)};
    const T inl3 = inl * inl * inl;  // 1 / (nn |Nt|)
    const V3<T> dnu = vscale(inl3, vsub(vscale(nn, dNu), vscale(vdot(Nt, dNu), Nt)));
    const V3<T> dnv = vscale(inl3, vsub(vscale(nn, dNv), vscale(vdot(Nt, dNv), Nt)));
    // air -> glass at the top face
    const V3<T> zero = {cst<T>(0.f), cst<T>(0.f), cst<T>(0.f)};
    V3<T> t1, Ddu, Ddv, tmp;
    refract(d, n, zero, dnu, qdiv(1.f, P.ior), t1, Ddu);
    refract(d, n, zero, dnv, qdiv(1.f, P.ior), tmp, Ddv);
    // to the bottom face z = 0
    const T s1 = qdiv(-hz, t1.z);
    const V3<T> p2 = {cst<T>(px) + s1 * t1.x, cst<T>(py) + s1 * t1.y, cst<T>(0.f)};
    const V3<T> Du2 = transfer_z(Du1, Ddu, s1, t1);
    const V3<T> Dv2 = transfer_z(Dv1, Ddv, s1, t1);
    // glass -> air at the flat bottom face (normal +z faces the glass side)
    const V3<T> ez = {cst<T>(0.f), cst<T>(0.f), cst<T>(1.f)};
    V3<T> t2, Ddu2, Ddv2;
    refract(t1, ez, Ddu, zero, P.ior, t2, Ddu2);
    refract(t1, ez, Ddv, zero, P.ior, tmp, Ddv2);
    // to the receiver plane z = -dist
    const T s2 = qdiv(cst<T>(-P.dist), t2.z);
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
PDS_HD V3a va(float x, float y, float z) { return {x, y, z}; }
PDS_HD float da(const V3a& a, const V3a& b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
PDS_HD V3a sa(float s, const V3a& a) { return {s * a.x, s * a.y, s * a.z}; }
PDS_HD V3a pa(const V3a& a, const V3a& b) {
    return {a.x + b.x, a.y + b.y, a.z + b.z};
}
PDS_HD V3a ma(const V3a& a, const V3a& b) {
    return {a.x - b.x, a.y - b.y, a.z - b.z};
}
PDS_HD void acc3(V3a& a, const V3a& b) {
    a.x += b.x; a.y += b.y; a.z += b.z;
}

// transfer_z: out = D - (D.z / t.z) t + s (Dd - (Dd.z / t.z) t), with itz = 1 / t.z
PDS_HD V3a tz_fwd(const V3a& D, const V3a& Dd, float s, const V3a& t,
                                      float itz) {
    const float a = D.z * itz, b = Dd.z * itz;
    return pa(ma(D, sa(a, t)), sa(s, ma(Dd, sa(b, t))));
}

// adjoint of tz_fwd: accumulates into Db (D), Ddb (Dd), sb (s) and tb (t) from ob (out)
PDS_HD void tz_adj(const V3a& D, const V3a& Dd, float s, const V3a& t,
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
PDS_HD bool plate_chain_adjoint(const float S[K], float px, float py,
                                                    const PlateParams& P, float gx, float gy,
                                                    float g0, float g1, float g3, float g4,
                                                    float cE, float Sb[K]) {
    const float Nx = S[1], Ny = S[2], Nxx = S[3], Nyx = S[4], Nxy = S[5], Nyy = S[6];
    const float hz = S[0];
    const V3a d = va(P.lx, P.ly, P.lz);
    // ---- forward
    const V3a Nt = va(Nx, Ny, 1.f);
    const float nn = Nx * Nx + Ny * Ny + 1.f;
    const float inl = rsq(nn);
    const float nlen = nn * inl;
    const V3a n = sa(inl, Nt);
    const float nd = da(n, d);
    const float ind = qdiv(1.f, nd);
    const float au = P.du0 * n.x * ind, av = P.du0 * n.y * ind;
    const V3a Du1 = ma(va(P.du0, 0.f, 0.f), sa(au, d));
    const V3a Dv1 = ma(va(0.f, P.du0, 0.f), sa(av, d));
    const V3a dNu = va(Nxx * Du1.x + Nxy * Du1.y, Nyx * Du1.x + Nyy * Du1.y, 0.f);
    const V3a dNv = va(Nxx * Dv1.x + Nxy * Dv1.y, Nyx * Dv1.x + Nyy * Dv1.y, 0.f);
    const float inl3 = inl * inl * inl;  // 1 / (nn nlen)
    const float wu = da(Nt, dNu), wv = da(Nt, dNv);
    const V3a dnu = sa(inl3, ma(sa(nn, dNu), sa(wu, Nt)));
    const V3a dnv = sa(inl3, ma(sa(nn, dNv), sa(wv, Nt)));
    const float e1 = qdiv(1.f, P.ior);
    const float cosi = da(d, n);
    const float k1 = 1.f - e1 * e1 * (1.f - cosi * cosi);
    const float rk1 = rsq(k1);
    const float ng1 = -(k1 * rk1);
    const float ing1 = -rk1;
    const float coso = e1 * cosi - ng1;
    const V3a t1 = ma(sa(e1, d), sa(coso, n));
    const float f1 = e1 - (e1 * e1) * cosi * ing1;
    const float ddu = da(d, dnu), ddv = da(d, dnv);
    const float qu = f1 * ddu, qv = f1 * ddv;
    const V3a Ddu = sa(-1.f, pa(sa(coso, dnu), sa(qu, n)));
    const V3a Ddv = sa(-1.f, pa(sa(coso, dnv), sa(qv, n)));
    const float it1z = qdiv(1.f, t1.z);
    const float s1 = -hz * it1z;
    const V3a Du2 = tz_fwd(Du1, Ddu, s1, t1, it1z);
    const V3a Dv2 = tz_fwd(Dv1, Ddv, s1, t1, it1z);
    const float e2 = P.ior;
    const float c2 = t1.z;
    const float k2 = 1.f - e2 * e2 * (1.f - c2 * c2);
    const float rk2 = rsq(k2);
    const float ng2 = -(k2 * rk2);
    const float ing2 = -rk2;
    const float coso2 = e2 * c2 - ng2;
    const V3a t2 = ma(sa(e2, t1), va(0.f, 0.f, coso2));
    const float f2 = e2 - (e2 * e2) * c2 * ing2;
    const float q2u = f2 * Ddu.z, q2v = f2 * Ddv.z;
    const V3a Ddu2 = ma(sa(e2, Ddu), va(0.f, 0.f, q2u));
    const V3a Ddv2 = ma(sa(e2, Ddv), va(0.f, 0.f, q2v));
    const float it2z = qdiv(1.f, t2.z);
    const float s2 = -P.dist * it2z;
    const V3a Du3 = tz_fwd(Du2, Ddu2, s2, t2, it2z);
    const V3a Dv3 = tz_fwd(Dv2, Ddv2, s2, t2, it2z);
    const float Dux = P.inv_half * Du3.x, Duy = P.inv_half * Du3.y;
    const float Dvx = P.inv_half * Dv3.x, Dvy = P.inv_half * Dv3.y;
    const float den = Dux * Dvy - Duy * Dvx;
    if (den == 0.f) return false;
    // ---- output adjoints: L = gx xr + gy yr + (2 / den) A + cE / |den|
    const float iden = qdiv(1.f, den);
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

struct Ray {
    float ox, oy, oz;
    float dx, dy, dz;
};

// The refraction chain of one point-light photon from its hit parameter t and the six normal
// scalars at the hit (Nx, Ny, dNx/dx, dNy/dx, dNx/dy, dNy/dy).
template <class T>
PDS_HD void point_chain(const T& t, const T& Nx, const T& Ny, const T& Nxx,
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
    const T inl = rsq(nn);
    const V3<T> n = vscale(inl, Nt);
    const T nd = vdot(n, d);
    // positional differentials carried from the light over t onto the tangent plane
    const V3<T> Du1 = vscale(t, vsub(Dt, vscale(qdiv(vdot(n, Dt), nd), d)));
    const V3<T> Dv1 = vscale(t, vsub(Dp, vscale(qdiv(vdot(n, Dp), nd), d)));
    const V3<T> dNu = {Nxx * Du1.x + Nxy * Du1.y, Nyx * Du1.x + Nyy * Du1.y, cst<T>(0.f)};
    const V3<T> dNv = {Nxx * Dv1.x + Nxy * Dv1.y, Nyx * Dv1.x + Nyy * Dv1.y, cst<T>(0.f)};
    const T inl3 = inl * inl * inl;  // 1 / (nn |Nt|)
    const V3<T> dnu = vscale(inl3, vsub(vscale(nn, dNu), vscale(vdot(Nt, dNu), Nt)));
    const V3<T> dnv = vscale(inl3, vsub(vscale(nn, dNv), vscale(vdot(Nt, dNv), Nt)));
    V3<T> t1, Ddu, Ddv, tmp;
    refract(d, n, Dt, dnu, qdiv(1.f, P.ior), t1, Ddu);
    refract(d, n, Dp, dnv, qdiv(1.f, P.ior), tmp, Ddv);
    const T s1 = qdiv(-p1.z, t1.z);
    const V3<T> p2 = {p1.x + s1 * t1.x, p1.y + s1 * t1.y, cst<T>(0.f)};
    const V3<T> Du2 = transfer_z(Du1, Ddu, s1, t1);
    const V3<T> Dv2 = transfer_z(Dv1, Ddv, s1, t1);
    const V3<T> ez = {cst<T>(0.f), cst<T>(0.f), cst<T>(1.f)};
    const V3<T> zero = {cst<T>(0.f), cst<T>(0.f), cst<T>(0.f)};
    V3<T> t2, Ddu2, Ddv2;
    refract(t1, ez, Ddu, zero, P.ior, t2, Ddu2);
    refract(t1, ez, Ddv, zero, P.ior, tmp, Ddv2);
    const T s2 = qdiv(cst<T>(-P.dist), t2.z);
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
PDS_HD bool point_chain_adjoint(float t, const float S[K], const Ray& r,
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
    const float inl = rsq(nn);
    const float nlen = nn * inl;
    const V3a n = sa(inl, Nt);
    const float nd = da(n, d);
    const float ind = qdiv(1.f, nd);
    const float aT = da(n, Dt) * ind, aP = da(n, Dp) * ind;
    const V3a Eu = ma(Dt, sa(aT, d)), Ev = ma(Dp, sa(aP, d));
    const V3a Du1 = sa(t, Eu), Dv1 = sa(t, Ev);
    const V3a dNu = va(Nxx * Du1.x + Nxy * Du1.y, Nyx * Du1.x + Nyy * Du1.y, 0.f);
    const V3a dNv = va(Nxx * Dv1.x + Nxy * Dv1.y, Nyx * Dv1.x + Nyy * Dv1.y, 0.f);
    const float inl3 = inl * inl * inl;
    const float wu = da(Nt, dNu), wv = da(Nt, dNv);
    const V3a dnu = sa(inl3, ma(sa(nn, dNu), sa(wu, Nt)));
    const V3a dnv = sa(inl3, ma(sa(nn, dNv), sa(wv, Nt)));
    const float e1 = qdiv(1.f, P.ior);
    const float cosi = da(d, n);
    const float k1 = 1.f - e1 * e1 * (1.f - cosi * cosi);
    const float rk1 = rsq(k1);
    const float ng1 = -(k1 * rk1);
    const float ing1 = -rk1;
    const float coso = e1 * cosi - ng1;
    const V3a t1 = ma(sa(e1, d), sa(coso, n));
    const float f1 = e1 - (e1 * e1) * cosi * ing1;
    const float ddu = da(Dt, n) + da(d, dnu), ddv = da(Dp, n) + da(d, dnv);
    const float qu = f1 * ddu, qv = f1 * ddv;
    const V3a Ddu = ma(sa(e1, Dt), pa(sa(coso, dnu), sa(qu, n)));
    const V3a Ddv = ma(sa(e1, Dp), pa(sa(coso, dnv), sa(qv, n)));
    const float it1z = qdiv(1.f, t1.z);
    const float s1 = -p1.z * it1z;
    const V3a Du2 = tz_fwd(Du1, Ddu, s1, t1, it1z);
    const V3a Dv2 = tz_fwd(Dv1, Ddv, s1, t1, it1z);
    const float e2 = P.ior;
    const float c2 = t1.z;
    const float k2 = 1.f - e2 * e2 * (1.f - c2 * c2);
    const float rk2 = rsq(k2);
    const float ng2 = -(k2 * rk2);
    const float ing2 = -rk2;
    const float coso2 = e2 * c2 - ng2;
    const V3a t2 = ma(sa(e2, t1), va(0.f, 0.f, coso2));
    const float f2 = e2 - (e2 * e2) * c2 * ing2;
    const float q2u = f2 * Ddu.z, q2v = f2 * Ddv.z;
    const V3a Ddu2 = ma(sa(e2, Ddu), va(0.f, 0.f, q2u));
    const V3a Ddv2 = ma(sa(e2, Ddv), va(0.f, 0.f, q2v));
    const float it2z = qdiv(1.f, t2.z);
    const float s2 = -P.dist * it2z;
    const V3a Du3 = tz_fwd(Du2, Ddu2, s2, t2, it2z);
    const V3a Dv3 = tz_fwd(Dv2, Ddv2, s2, t2, it2z);
    const float Dux = P.inv_half * Du3.x, Duy = P.inv_half * Du3.y;
    const float Dvx = P.inv_half * Dv3.x, Dvy = P.inv_half * Dv3.y;
    const float den = Dux * Dvy - Duy * Dvx;
    if (den == 0.f) return false;
    // ---- output adjoints
    const float iden = qdiv(1.f, den);
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


}  // namespace chain
}  // namespace pds
