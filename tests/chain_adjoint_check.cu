// Host check of the refraction chain's reverse-mode sweeps (shapefromcaustics_b200/csrc/
// pds_chain.cuh): plate_chain_adjoint and point_chain_adjoint against the chain templates
// instantiated with forward-mode dual numbers (seven tangents, one per height-dependent
// scalar), on seeded random photons. Built and run by tests/test_chain_adjoint.py; prints one
// line per sweep: "<name> trials <n> median <rel> worst <rel>" (relative L2 of the seven
// derivatives).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "../shapefromcaustics_b200/csrc/pds_chain.cuh"

namespace pds {
namespace chain {

struct Dual {
    float v;
    float d[K];
};

inline Dual dconst(float v) {
    Dual r;
    r.v = v;
    for (int k = 0; k < K; ++k) r.d[k] = 0.f;
    return r;
}
inline Dual operator+(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v + b.v;
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
inline Dual operator-(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v - b.v;
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
inline Dual operator-(const Dual& a) {
    Dual r;
    r.v = -a.v;
    for (int k = 0; k < K; ++k) r.d[k] = -a.d[k];
    return r;
}
inline Dual operator*(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v * b.v;
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
inline Dual operator*(float s, const Dual& a) {
    Dual r;
    r.v = s * a.v;
    for (int k = 0; k < K; ++k) r.d[k] = s * a.d[k];
    return r;
}
inline Dual operator/(const Dual& a, const Dual& b) {
    const float inv = 1.f / b.v;
    Dual r;
    r.v = a.v * inv;
    for (int k = 0; k < K; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * inv;
    return r;
}
inline Dual dsqrt(const Dual& a) {
    Dual r;
    r.v = std::sqrt(a.v);
    const float h = 0.5f / r.v;
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * h;
    return r;
}
inline Dual dabs(const Dual& a) { return a.v < 0.f ? -a : a; }
template <>
inline Dual cst<Dual>(float v) { return dconst(v); }

// L of the sweeps: gx xr + gy yr + the M gradients against Mp = 2 [Du Dv]^-1 + cE / |den|
inline Dual loss(const Dual& xr, const Dual& yr, const Dual& Dux, const Dual& Duy,
                 const Dual& Dvx, const Dual& Dvy, float gx, float gy, float g0, float g1,
                 float g3, float g4, float cE) {
    const Dual den = Dux * Dvy - Duy * Dvx;
    const Dual f = dconst(2.f) / den;
    Dual L = gx * xr + gy * yr;
    L = L + g0 * (f * Dvy) + (-g1) * (f * Dvx) + (-g3) * (f * Duy) + g4 * (f * Dux);
    return L + cE * (dconst(1.f) / dabs(den));
}

double rel(const float* a, const Dual& L) {
    double num = 0, den = 0;
    for (int k = 0; k < K; ++k) {
        num += double(a[k] - L.d[k]) * double(a[k] - L.d[k]);
        den += double(L.d[k]) * double(L.d[k]);
    }
    return std::sqrt(num / den);
}

void report(const char* name, std::vector<double>& r) {
    std::sort(r.begin(), r.end());
    std::printf("%s trials %d median %.3e worst %.3e\n", name, int(r.size()), r[r.size() / 2],
                r.back());
}

}  // namespace chain
}  // namespace pds

using namespace pds::chain;

int main() {
    std::mt19937 g(1);
    std::uniform_real_distribution<float> U(-1.f, 1.f);
    std::vector<double> rp, rq;
    for (int trial = 0; trial < 300; ++trial) {  // collimated light, tilted up to ~3 degrees
        PlateParams P;
        P.texel = 0.4f; P.ior = 1.45f + 0.05f * std::fabs(U(g)); P.dist = 30.f;
        P.inv_half = 1.f / 14.f; P.du0 = 0.05f + 0.05f * std::fabs(U(g));
        const float lx = 0.05f * U(g), ly = 0.05f * U(g);
        const float ln = std::sqrt(lx * lx + ly * ly + 1.f);
        P.lx = lx / ln; P.ly = ly / ln; P.lz = -1.f / ln;
        const float S[K] = {1.f + 0.05f * std::fabs(U(g)), 0.1f * U(g), 0.1f * U(g), 0.3f * U(g),
                            0.3f * U(g), 0.3f * U(g), 0.3f * U(g)};
        const float px = 3.f * U(g), py = 3.f * U(g);
        const float gx = U(g), gy = U(g), g0 = 1e-3f * U(g), g1 = 1e-3f * U(g),
                    g3 = 1e-3f * U(g), g4 = 1e-3f * U(g), cE = 1e-4f * U(g);
        float Sb[K];
        if (!plate_chain_adjoint(S, px, py, P, gx, gy, g0, g1, g3, g4, cE, Sb)) continue;
        Dual v[K];
        for (int k = 0; k < K; ++k) { v[k] = dconst(S[k]); v[k].d[k] = 1.f; }
        Dual xr, yr, Dux, Duy, Dvx, Dvy;
        plate_chain<Dual>(v[0], v[1], v[2], v[3], v[4], v[5], v[6], px, py, P, xr, yr, Dux, Duy,
                          Dvx, Dvy);
        rp.push_back(rel(Sb, loss(xr, yr, Dux, Duy, Dvx, Dvy, gx, gy, g0, g1, g3, g4, cE)));
    }
    for (int trial = 0; trial < 300; ++trial) {  // point light: rays from a light 40 above
        PlateParams P;
        P.texel = 0.4f; P.ior = 1.45f + 0.05f * std::fabs(U(g)); P.dist = 30.f;
        P.inv_half = 1.f / 14.f; P.du0 = 0.f; P.lx = P.ly = 0.f; P.lz = -1.f;
        Ray r;
        r.ox = 2.f * U(g); r.oy = 2.f * U(g); r.oz = 40.f;
        const float dx = 0.2f * U(g), dy = 0.2f * U(g);
        const float dn = std::sqrt(dx * dx + dy * dy + 1.f);
        r.dx = dx / dn; r.dy = dy / dn; r.dz = -1.f / dn;
        const V3<float> Dt = {0.01f * (1.f + 0.2f * U(g)), 0.002f * U(g), 0.001f * U(g)};
        const V3<float> Dp = {0.002f * U(g), 0.01f * (1.f + 0.2f * U(g)), 0.001f * U(g)};
        const float t = 39.f + U(g);
        const float S[K] = {0.f, 0.1f * U(g), 0.1f * U(g), 0.3f * U(g), 0.3f * U(g), 0.3f * U(g),
                            0.3f * U(g)};
        const float gx = U(g), gy = U(g), g0 = 1e-3f * U(g), g1 = 1e-3f * U(g),
                    g3 = 1e-3f * U(g), g4 = 1e-3f * U(g), cE = 1e-4f * U(g);
        float tb, Sb[K];
        if (!point_chain_adjoint(t, S, r, Dt, Dp, P, gx, gy, g0, g1, g3, g4, cE, tb, Sb))
            continue;
        Dual v[K];
        for (int k = 0; k < K; ++k) { v[k] = dconst(S[k]); v[k].d[k] = 1.f; }
        v[0].v = t;  // component 0: the hit parameter
        Dual xr, yr, Dux, Duy, Dvx, Dvy;
        point_chain<Dual>(v[0], v[1], v[2], v[3], v[4], v[5], v[6], r, Dt, Dp, P, xr, yr, Dux,
                          Duy, Dvx, Dvy);
        Sb[0] = tb;
        rq.push_back(rel(Sb, loss(xr, yr, Dux, Duy, Dvx, Dvy, gx, gy, g0, g1, g3, g4, cE)));
    }
    report("collimated", rp);
    report("point", rq);
    return 0;
}
