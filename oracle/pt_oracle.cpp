// pt_oracle.cpp — CPU oracle (test infrastructure only; see pt_oracle.h).
//
// Each routine cites the reference source it restates
// (gracejinsotrue/PBRT-renderer-, paths within that project).
#include "pt_oracle.h"

#include <algorithm>
#include <atomic>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <thread>

namespace oracle {

// ---------------------------------------------------------------------------
// Constants (shaders/Common.hlsli:147-154)
// ---------------------------------------------------------------------------
template <class T> constexpr T kPi = T(3.14159265358979323846);
template <class T> constexpr T kInvPi = T(0.31830988618379067154);

template <class T> inline T dot(const V3<T> &a, const V3<T> &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline V3<T> cross(const V3<T> &a, const V3<T> &b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> inline T length(const V3<T> &v) { return std::sqrt(dot(v, v)); }
template <class T> inline V3<T> normalize(const V3<T> &v) { return v * (T(1) / std::sqrt(dot(v, v))); }
template <class T> inline T clampT(T x, T a, T b) { return std::min(std::max(x, a), b); }
template <class T> inline T saturate(T x) { return clampT(x, T(0), T(1)); }
template <class T> inline V3<T> vmax(const V3<T> &a, const V3<T> &b) {
    return {std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)};
}
template <class T> inline V3<T> vmin(const V3<T> &a, const V3<T> &b) {
    return {std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)};
}
template <class T> inline V3<T> vexp(const V3<T> &a) { return {std::exp(a.x), std::exp(a.y), std::exp(a.z)}; }
template <class T> inline T lerp(T a, T b, T t) { return a + (b - a) * t; }
template <class T> inline V3<T> lerp3(const V3<T> &a, const V3<T> &b, T t) { return a + (b - a) * t; }
// HLSL reflect / refract (intrinsic definitions)
template <class T> inline V3<T> reflect(const V3<T> &i, const V3<T> &n) { return i - T(2) * dot(n, i) * n; }
template <class T> inline V3<T> refract(const V3<T> &i, const V3<T> &n, T eta) {
    T ndi = dot(n, i);
    T k = T(1) - eta * eta * (T(1) - ndi * ndi);
    if (k < T(0)) return V3<T>(T(0));
    return eta * i - (eta * ndi + std::sqrt(k)) * n;
}

// ---------------------------------------------------------------------------
// RNG (shaders/RNG.hlsli:9-99)
// ---------------------------------------------------------------------------
inline uint32_t pcg_hash(uint32_t v) {  // RNG.hlsli:9-14
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
inline uint32_t reverse_bits(uint32_t x) {
    x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
    x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
    x = ((x >> 4) & 0x0F0F0F0Fu) | ((x & 0x0F0F0F0Fu) << 4);
    x = ((x >> 8) & 0x00FF00FFu) | ((x & 0x00FF00FFu) << 8);
    return (x >> 16) | (x << 16);
}
inline uint32_t sobol2d(uint32_t index, uint32_t axis) {  // RNG.hlsli:17-30
    if (axis == 0u) return reverse_bits(index);
    uint32_t r = 0u, dirn = 1u << 31;
    for (uint32_t i = index; i != 0u; i >>= 1u) {
        if (i & 1u) r ^= dirn;
        dirn ^= dirn >> 1u;
    }
    return r;
}
inline uint32_t laine_karras(uint32_t x, uint32_t seed) {  // RNG.hlsli:33-41
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}
inline uint32_t owen_scramble(uint32_t x, uint32_t seed) {  // RNG.hlsli:43-49
    return reverse_bits(laine_karras(reverse_bits(x), seed));
}

struct Rng {  // RNG.hlsli:51-70
    uint32_t pixelSeed, sampleIndex, dim, state, pcgWhite, kind;
};
inline Rng init_rng(uint32_t px, uint32_t py, uint32_t w, uint32_t h, uint32_t frame, uint32_t kind) {
    Rng r;
    uint32_t pid = py * w + px;
    r.pixelSeed = pcg_hash(pid ^ 0x9e3779b9u);
    r.sampleIndex = frame;
    r.dim = 0u;
    r.state = pcg_hash(pid + frame * w * h);
    r.pcgWhite = pcg_hash(pid * 0x9e3779b9u + frame * 0x85ebca6bu + 1u);
    r.kind = kind;
    return r;
}
inline float next_float(Rng &r) {  // RNG.hlsli:80-99
    if (r.kind == PT_RNG_PCG_HASH) {
        r.dim++;
        r.pcgWhite = pcg_hash(r.pcgWhite);
        return std::min(float(r.pcgWhite) * 2.3283064365386963e-10f, 0.99999994f);
    }
    uint32_t d = r.dim++;
    uint32_t axis = d & 1u, pad = d >> 1u;
    uint32_t sIdx = owen_scramble(r.sampleIndex, pcg_hash(pad * 0x9e3779b9u + 1u));
    uint32_t v = owen_scramble(sobol2d(sIdx, axis),
                               pcg_hash(r.pixelSeed + pad * 0x6c8e9cf5u + axis * 0x68bc21ebu));
    return std::min(float(v) * 2.3283064365386963e-10f, 0.99999994f);
}

// ---------------------------------------------------------------------------
// Geometry helpers (shaders/GeometryUtils.hlsli:18-228)
// ---------------------------------------------------------------------------
template <class T> inline T balance_heuristic(T a, T b) {  // :18-24
    T s = a + b;
    if (s < T(1e-20)) return T(0);
    return a / s;
}
template <class T> inline void build_onb(const V3<T> &N, V3<T> &Tn, V3<T> &B) {  // :160-165
    V3<T> up = std::fabs(N.y) < T(0.999) ? V3<T>(T(0), T(1), T(0)) : V3<T>(T(1), T(0), T(0));
    Tn = normalize(cross(up, N));
    B = cross(N, Tn);
}
template <class T> inline V3<T> to_local(const V3<T> &v, const V3<T> &Tn, const V3<T> &B, const V3<T> &N) {
    return {dot(v, Tn), dot(v, B), dot(v, N)};
}
template <class T> inline V3<T> to_world(const V3<T> &v, const V3<T> &Tn, const V3<T> &B, const V3<T> &N) {
    return Tn * v.x + B * v.y + N * v.z;
}
inline F3 offset_ray_origin(const F3 &p, const F3 &Ng, const F3 &N) {  // :178-183
    F3 q = p + N * 0.002f;
    q += Ng * std::max(0.0f, -dot(q - p, Ng));
    return q;
}
template <class T> inline V3<T> cosine_sample_hemisphere(T u0, T u1) {  // :189-194
    T r = std::sqrt(u0);
    T phi = T(2) * kPi<T> * u1;
    return {r * std::cos(phi), r * std::sin(phi), std::sqrt(std::max(T(0), T(1) - u0))};
}
template <class T> inline T fresnel_dielectric(T cosI, T etaI, T etaT) {  // :200-219
    if (etaI == etaT) return T(0);
    if (cosI < T(0)) { std::swap(etaI, etaT); cosI = -cosI; }
    T eta = etaI / etaT;
    T s2 = eta * eta * (T(1) - cosI * cosI);
    if (s2 > T(1)) return T(1);
    T cosT = std::sqrt(T(1) - s2);
    T Rs = (etaI * cosI - etaT * cosT) / (etaI * cosI + etaT * cosT);
    T Rp = (etaT * cosI - etaI * cosT) / (etaT * cosI + etaI * cosT);
    return T(0.5) * (Rs * Rs + Rp * Rp);
}
template <class T> inline T luminance(const V3<T> &c) {  // :225-228
    return T(0.212671) * c.x + T(0.715160) * c.y + T(0.072169) * c.z;
}
template <class T> inline T pow5(T x) { return std::pow(x, T(5)); }

// ---------------------------------------------------------------------------
// Beckmann microfacet (shaders/Microfacet.hlsli:13-125)
// ---------------------------------------------------------------------------
template <class T> T beckmann_d(const V3<T> &wh, T a) {
    if (wh.z <= T(0)) return T(0);
    T c2 = wh.z * wh.z, t2 = (T(1) - c2) / c2, c3 = c2 * wh.z, a2 = a * a;
    return std::exp(-t2 / a2) / (kPi<T> * a2 * c3);
}
template <class T> T beckmann_d_cos(const V3<T> &wh, T a) {
    if (wh.z <= T(0)) return T(0);
    T c2 = wh.z * wh.z, t2 = (T(1) - c2) / c2, a2 = a * a;
    return std::exp(-t2 / a2) / (kPi<T> * a2 * c2);
}
template <class T> V3<T> beckmann_sample(T u0, T u1, T a) {
    T phi = T(2) * kPi<T> * u1;
    T t2 = -a * a * std::log(std::max(T(1e-8), T(1) - u0));
    T c = T(1) / std::sqrt(T(1) + t2);
    T s = std::sqrt(std::max(T(0), T(1) - c * c));
    return {s * std::cos(phi), s * std::sin(phi), c};
}
template <class T> T smith_g1(const V3<T> &v, const V3<T> &wh, T a) {
    T dvw = dot(v, wh), dvn = v.z;
    if (dvw / dvn <= T(0)) return T(0);
    T c2 = v.z * v.z;
    if (c2 < T(1e-10)) return T(0);
    T tanT = std::sqrt(std::max(T(0), T(1) - c2)) / std::fabs(v.z);
    if (tanT < T(1e-10)) return T(1);
    T b = T(1) / (a * tanT);
    if (b >= T(1.6)) return T(1);
    T b2 = b * b;
    return (T(3.535) * b + T(2.181) * b2) / (T(1) + T(2.276) * b + T(2.577) * b2);
}
template <class T> V3<T> microfacet_eval(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m) {
    if (wi.z <= T(0) || wo.z <= T(0)) return V3<T>(T(0));
    V3<T> kd = m.albedo;
    T ks = T(1) - std::max(kd.x, std::max(kd.y, kd.z));
    V3<T> diffuse = kd * kInvPi<T>;
    V3<T> wh = normalize(wi + wo);
    T D = beckmann_d(wh, m.alpha);
    T F = fresnel_dielectric(dot(wh, wi), m.extIOR, m.intIOR);
    T G = smith_g1(wi, wh, m.alpha) * smith_g1(wo, wh, m.alpha);
    T denom = T(4) * wi.z * wo.z;
    return diffuse + V3<T>(T(1)) * (ks * D * F * G / std::max(denom, T(1e-10)));
}
template <class T> T microfacet_pdf(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m) {
    if (wi.z <= T(0) || wo.z <= T(0)) return T(0);
    V3<T> kd = m.albedo;
    T ks = T(1) - std::max(kd.x, std::max(kd.y, kd.z));
    V3<T> wh = normalize(wi + wo);
    T Dc = beckmann_d_cos(wh, m.alpha);
    T Jh = T(1) / std::max(T(4) * dot(wh, wo), T(1e-10));
    return ks * Dc * Jh + (T(1) - ks) * wo.z * kInvPi<T>;
}

// Subsurface entry lobe (shaders/Material.hlsli:48-58, 92-100).
template <class T> V3<T> subsurface_eval(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m) {
    if (wi.z <= T(0) || wo.z <= T(0)) return V3<T>(T(0));
    T a = std::max(m.roughness * m.roughness, T(1e-4));
    V3<T> wh = normalize(wi + wo);
    T D = beckmann_d(wh, a);
    T Fr = fresnel_dielectric(dot(wh, wi), m.extIOR, m.intIOR);
    T G = smith_g1(wi, wh, a) * smith_g1(wo, wh, a);
    return V3<T>(T(1)) * (D * Fr * G / std::max(T(4) * wi.z * wo.z, T(1e-10)));
}
template <class T> T subsurface_pdf(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m) {
    if (wi.z <= T(0) || wo.z <= T(0)) return T(0);
    T a = std::max(m.roughness * m.roughness, T(1e-4));
    V3<T> wh = normalize(wi + wo);
    T Fr = fresnel_dielectric(dot(wh, wi), m.extIOR, m.intIOR);
    return Fr * beckmann_d_cos(wh, a) / std::max(T(4) * dot(wh, wo), T(1e-10));
}

// ---------------------------------------------------------------------------
// Disney principled (shaders/Disney.hlsli:10-275)
// ---------------------------------------------------------------------------
template <class T> V3<T> disney_burley(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m) {
    if (wi.z <= T(0) || wo.z <= T(0)) return V3<T>(T(0));
    V3<T> wh = normalize(wi + wo);
    T cd = std::fabs(dot(wo, wh));
    T fd90 = T(0.5) + T(2) * m.roughness * cd * cd;
    T fv = T(1) + (fd90 - T(1)) * pow5(T(1) - wi.z);
    T fl = T(1) + (fd90 - T(1)) * pow5(T(1) - wo.z);
    return m.albedo * kInvPi<T> * fv * fl;
}
template <class T> V3<T> disney_hk(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m) {
    if (wi.z <= T(0) || wo.z <= T(0)) return V3<T>(T(0));
    V3<T> wh = normalize(wi + wo);
    T cd = std::fabs(dot(wo, wh));
    T f90 = m.roughness * cd * cd;
    T fv = T(1) + (f90 - T(1)) * pow5(T(1) - wi.z);
    T fl = T(1) + (f90 - T(1)) * pow5(T(1) - wo.z);
    T cs = std::max(wi.z + wo.z, T(1e-4));
    T ss = T(1.25) * (fv * fl * (T(1) / cs - T(0.5)) + T(0.5));
    return m.albedo * kInvPi<T> * ss;
}
template <class T> V3<T> disney_diffuse_lobe(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m) {
    return lerp3(disney_burley(wi, wo, m), disney_hk(wi, wo, m), m.subsurface);
}
template <class T> T ggx_d(T ndh, T a) {
    if (ndh <= T(0)) return T(0);
    T a2 = a * a;
    T den = ndh * ndh * (a2 - T(1)) + T(1);
    return a2 / std::max(kPi<T> * den * den, T(1e-10));
}
template <class T> T ggx_g1(T ndv, T a) {
    if (ndv <= T(0)) return T(0);
    T a2 = a * a, n2 = ndv * ndv;
    T den = ndv + std::sqrt(a2 + (T(1) - a2) * n2);
    return T(2) * ndv / std::max(den, T(1e-10));
}
template <class T> V3<T> ggx_sample_wh(T u0, T u1, T a) {
    T a2 = a * a;
    T c2 = (T(1) - u0) / std::max(T(1) + (a2 - T(1)) * u0, T(1e-10));
    T c = std::sqrt(saturate(c2));
    T s = std::sqrt(std::max(T(0), T(1) - c2));
    T phi = T(2) * kPi<T> * u1;
    return {s * std::cos(phi), s * std::sin(phi), c};
}
template <class T> T ggx_pdf_wo(const V3<T> &wi, const V3<T> &wo, T a) {
    V3<T> wh = normalize(wi + wo);
    if (wh.z <= T(0)) return T(0);
    return ggx_d(wh.z, a) * wh.z / std::max(T(4) * std::fabs(dot(wh, wo)), T(1e-10));
}
template <class T> V3<T> disney_tint(const Mat<T> &m) {
    T lum = luminance(m.albedo);
    return lum > T(0) ? m.albedo / lum : V3<T>(T(1));
}
template <class T> V3<T> disney_f0(const Mat<T> &m) {
    V3<T> ctint = disney_tint(m);
    V3<T> cspec0 = T(0.08) * m.specular * lerp3(V3<T>(T(1)), ctint, m.specularTint);
    return lerp3(cspec0, m.albedo, m.metallic);
}
template <class T> V3<T> disney_spec_eval(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m) {
    if (wi.z <= T(0) || wo.z <= T(0)) return V3<T>(T(0));
    V3<T> wh = normalize(wi + wo);
    if (wh.z <= T(0)) return V3<T>(T(0));
    T a = std::max(m.roughness * m.roughness, T(1e-4));
    T vdh = std::fabs(dot(wi, wh));
    T D = ggx_d(wh.z, a);
    V3<T> F0 = disney_f0(m);
    T t = pow5(T(1) - vdh);
    V3<T> F = F0 + (V3<T>(T(1)) - F0) * t;
    T G = ggx_g1(wi.z, a) * ggx_g1(wo.z, a);
    return D * F * G / std::max(T(4) * wi.z * wo.z, T(1e-10));
}
template <class T> T disney_spec_pdf(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m) {
    if (wi.z <= T(0) || wo.z <= T(0)) return T(0);
    return ggx_pdf_wo(wi, wo, std::max(m.roughness * m.roughness, T(1e-4)));
}
template <class T> V3<T> disney_sheen(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m) {
    if (m.sheen <= T(0) || wi.z <= T(0) || wo.z <= T(0)) return V3<T>(T(0));
    V3<T> wh = normalize(wi + wo);
    T cd = std::fabs(dot(wo, wh));
    V3<T> csheen = lerp3(V3<T>(T(1)), disney_tint(m), m.sheenTint);
    T fr = pow5(T(1) - cd);
    return m.sheen * csheen * fr;
}
template <class T> T gtr1_d(T ndh, T a) {
    if (ndh <= T(0)) return T(0);
    T a2 = a * a;
    if (a2 >= T(0.9999)) return kInvPi<T>;
    T t = T(1) + (a2 - T(1)) * ndh * ndh;
    return (a2 - T(1)) / (kPi<T> * std::log(a2) * t);
}
template <class T> V3<T> gtr1_sample_wh(T u0, T u1, T a) {
    T a2 = a * a, c2;
    if (a2 >= T(0.9999)) c2 = T(1) - u0;
    else c2 = (T(1) - std::pow(a2, T(1) - u0)) / (T(1) - a2);
    T c = std::sqrt(saturate(c2));
    T s = std::sqrt(std::max(T(0), T(1) - c2));
    T phi = T(2) * kPi<T> * u1;
    return {s * std::cos(phi), s * std::sin(phi), c};
}
template <class T> T gtr1_pdf_wo(const V3<T> &wi, const V3<T> &wo, T a) {
    V3<T> wh = normalize(wi + wo);
    if (wh.z <= T(0)) return T(0);
    return gtr1_d(wh.z, a) * wh.z / std::max(T(4) * std::fabs(dot(wh, wo)), T(1e-10));
}
template <class T> T disney_cc_alpha(const Mat<T> &m) { return lerp(T(0.1), T(0.001), m.clearcoatGloss); }
template <class T> T disney_cc_eval(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m) {
    if (m.clearcoat <= T(0) || wi.z <= T(0) || wo.z <= T(0)) return T(0);
    V3<T> wh = normalize(wi + wo);
    if (wh.z <= T(0)) return T(0);
    T D = gtr1_d(wh.z, disney_cc_alpha(m));
    T vdh = std::fabs(dot(wi, wh));
    T F = T(0.04) + (T(1) - T(0.04)) * pow5(T(1) - vdh);
    T G = ggx_g1(wi.z, T(0.25)) * ggx_g1(wo.z, T(0.25));
    return T(0.25) * m.clearcoat * D * F * G / std::max(T(4) * wi.z * wo.z, T(1e-10));
}
template <class T> T disney_cc_pdf(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m) {
    if (m.clearcoat <= T(0) || wi.z <= T(0) || wo.z <= T(0)) return T(0);
    return gtr1_pdf_wo(wi, wo, disney_cc_alpha(m));
}
template <class T> struct LobeProbs { T d, s, c; };
template <class T> LobeProbs<T> disney_probs(const Mat<T> &m) {  // Disney.hlsli:260-273
    T wd = T(1) - m.metallic, ws = T(1), wc = T(0.25) * m.clearcoat;
    T tot = wd + ws + wc;
    T inv = tot > T(0) ? T(1) / tot : T(0);
    return {wd * inv, ws * inv, wc * inv};
}
template <class T> V3<T> disney_eval(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m) {  // Material.hlsli:30-40
    if (wi.z <= T(0) || wo.z <= T(0)) return V3<T>(T(0));
    V3<T> fd = disney_diffuse_lobe(wi, wo, m);
    V3<T> fs = disney_spec_eval(wi, wo, m);
    V3<T> fsh = disney_sheen(wi, wo, m);
    T fc = disney_cc_eval(wi, wo, m);
    return (T(1) - m.metallic) * (fd + fsh) + fs + fc;
}
template <class T> T disney_pdf(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m) {  // Material.hlsli:74-84
    if (wi.z <= T(0) || wo.z <= T(0)) return T(0);
    LobeProbs<T> p = disney_probs(m);
    return p.d * (wo.z * kInvPi<T>) + p.s * disney_spec_pdf(wi, wo, m) + p.c * disney_cc_pdf(wi, wo, m);
}

// ---------------------------------------------------------------------------
// Chiang 2016 hair BCSDF (shaders/Hair.hlsli:26-432)
// ---------------------------------------------------------------------------
template <class T> T hair_i0(T x) {
    T val = T(0), x2i = T(1), ifact = T(1), i4 = T(1);
    for (int i = 0; i < 10; i++) {
        if (i > 0) { x2i *= x * x; ifact *= T(i); i4 *= T(4); }
        val += x2i / (i4 * ifact * ifact);
    }
    return val;
}
template <class T> T hair_log_i0(T x) {
    if (x > T(12)) return x + T(0.5) * (-std::log(T(2) * kPi<T>) + std::log(T(1) / x) + T(1) / (T(8) * x));
    return std::log(hair_i0(x));
}
template <class T> T hair_mp(T cti, T cto, T sti, T sto, T v) {
    T a = cti * cto / v, b = sti * sto / v;
    if (v <= T(0.1)) return std::exp(hair_log_i0(a) - b - T(1) / v + T(0.6931) + std::log(T(1) / (T(2) * v)));
    return (std::exp(-b) * hair_i0(a)) / (std::sinh(T(1) / v) * T(2) * v);
}
template <class T> T hair_logistic(T x, T s) {
    T ex = std::exp(-std::fabs(x) / s);
    return ex / (s * (T(1) + ex) * (T(1) + ex));
}
template <class T> T hair_logistic_cdf(T x, T s) { return T(1) / (T(1) + std::exp(-x / s)); }
template <class T> T hair_trimmed_logistic(T x, T s, T a, T b) {
    T den = hair_logistic_cdf(b, s) - hair_logistic_cdf(a, s);
    return den > T(1e-10) ? hair_logistic(x, s) / den : T(0);
}
template <class T> T hair_sample_trimmed_logistic(T u, T s, T a, T b) {
    T ca = hair_logistic_cdf(a, s), cb = hair_logistic_cdf(b, s);
    T t = ca + u * (cb - ca);
    t = clampT(t, T(1e-6), T(1) - T(1e-6));
    return -s * std::log(T(1) / t - T(1));
}
template <class T> T hair_phi(int p, T go, T gt) { return T(2) * T(p) * gt - T(2) * go + T(p) * kPi<T>; }
template <class T> T hair_np(T phi, int p, T s, T go, T gt) {
    T dphi = phi - hair_phi(p, go, gt);
    while (dphi > kPi<T>) dphi -= T(2) * kPi<T>;
    while (dphi < -kPi<T>) dphi += T(2) * kPi<T>;
    return hair_trimmed_logistic(dphi, s, -kPi<T>, kPi<T>);
}
template <class T> V3<T> hair_sigma_a_from_color(const V3<T> &C, T bn) {
    T den = T(5.969) - T(0.215) * bn + T(2.532) * bn * bn - T(10.73) * bn * bn * bn +
            T(5.574) * bn * bn * bn * bn + T(0.245) * bn * bn * bn * bn * bn;
    V3<T> s;
    s.x = C.x > T(1e-4) ? std::pow(std::log(C.x) / den, T(2)) : T(100);
    s.y = C.y > T(1e-4) ? std::pow(std::log(C.y) / den, T(2)) : T(100);
    s.z = C.z > T(1e-4) ? std::pow(std::log(C.z) / den, T(2)) : T(100);
    return s;
}
template <class T> struct HairParams { T v[4]; T s; T sin2k[3], cos2k[3]; V3<T> sigma_a; };
template <class T> HairParams<T> hair_params(const Mat<T> &m) {
    HairParams<T> p;
    T bm = m.roughness;
    T v0 = T(0.726) * bm + T(0.812) * bm * bm + T(3.7) * std::pow(bm, T(20));
    v0 = v0 * v0;
    p.v[0] = v0; p.v[1] = T(0.25) * v0; p.v[2] = T(4) * v0; p.v[3] = p.v[2];
    T bn = m.betaN;
    p.s = T(0.626657069) * (T(0.265) * bn + T(1.194) * bn * bn + T(5.372) * std::pow(bn, T(22)));
    T ar = m.alpha * kPi<T> / T(180);
    p.sin2k[0] = std::sin(ar);
    p.cos2k[0] = std::sqrt(std::max(T(0), T(1) - p.sin2k[0] * p.sin2k[0]));
    for (int i = 1; i < 3; i++) {
        p.sin2k[i] = T(2) * p.cos2k[i - 1] * p.sin2k[i - 1];
        p.cos2k[i] = p.cos2k[i - 1] * p.cos2k[i - 1] - p.sin2k[i - 1] * p.sin2k[i - 1];
    }
    p.sigma_a = hair_sigma_a_from_color(m.albedo, bn);
    return p;
}
template <class T> void hair_ap(T cto, T sto, T h, T eta, const V3<T> &sa, V3<T> ap[4]) {
    T etap = std::sqrt(std::max(T(0), eta * eta - sto * sto)) / std::max(cto, T(1e-6));
    T sgt = clampT(h / etap, T(-1), T(1));
    T cgt = std::sqrt(std::max(T(0), T(1) - sgt * sgt));
    T stt = sto / eta;
    T ctt = std::sqrt(std::max(T(0), T(1) - stt * stt));
    V3<T> Tr = vexp(-sa * (T(2) * cgt / std::max(ctt, T(1e-6))));
    T cgo = std::sqrt(std::max(T(0), T(1) - h * h));
    T f = fresnel_dielectric(cto * cgo, T(1), eta);
    ap[0] = V3<T>(f);
    ap[1] = (T(1) - f) * (T(1) - f) * Tr;
    ap[2] = ap[1] * Tr * f;
    V3<T> tf = Tr * f;
    V3<T> den = vmax(V3<T>(T(1)) - tf, V3<T>(T(1e-10)));
    ap[3] = ap[2] * f * Tr / den;
}
template <class T> void hair_tilt(int p, T sto, T cto, const T s2k[3], const T c2k[3], T &sp, T &cp) {
    if (p == 0) { sp = sto * c2k[1] - cto * s2k[1]; cp = cto * c2k[1] + sto * s2k[1]; }
    else if (p == 1) { sp = sto * c2k[0] + cto * s2k[0]; cp = cto * c2k[0] - sto * s2k[0]; }
    else if (p == 2) { sp = sto * c2k[2] + cto * s2k[2]; cp = cto * c2k[2] - sto * s2k[2]; }
    else { sp = sto; cp = cto; }
    cp = std::fabs(cp);
}
template <class T> struct HairFrame { T sto, cto, phio, sti, cti, phii, phi, go, gt, eta; };
template <class T> HairFrame<T> hair_frame(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m, T h) {
    HairFrame<T> f;
    f.sto = wi.x; f.cto = std::sqrt(std::max(T(0), T(1) - f.sto * f.sto)); f.phio = std::atan2(wi.z, wi.y);
    f.sti = wo.x; f.cti = std::sqrt(std::max(T(0), T(1) - f.sti * f.sti)); f.phii = std::atan2(wo.z, wo.y);
    f.phi = f.phii - f.phio;
    f.go = std::asin(clampT(h, T(-1), T(1)));
    f.eta = m.intIOR;
    T etap = std::sqrt(std::max(T(0), f.eta * f.eta - f.sto * f.sto)) / std::max(f.cto, T(1e-6));
    f.gt = std::asin(clampT(h / etap, T(-1), T(1)));
    return f;
}
template <class T> V3<T> hair_eval(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m, T h) {
    HairFrame<T> F = hair_frame(wi, wo, m, h);
    HairParams<T> P = hair_params(m);
    V3<T> ap[4];
    hair_ap(F.cto, F.sto, h, F.eta, P.sigma_a, ap);
    V3<T> fsum(T(0));
    for (int p = 0; p < 3; p++) {
        T sp, cp;
        hair_tilt(p, F.sto, F.cto, P.sin2k, P.cos2k, sp, cp);
        T mp = hair_mp(F.cti, cp, F.sti, sp, P.v[p]);
        T np = hair_np(F.phi, p, P.s, F.go, F.gt);
        fsum += mp * ap[p] * np;
    }
    fsum += hair_mp(F.cti, F.cto, F.sti, F.sto, P.v[3]) * ap[3] / (T(2) * kPi<T>);
    T ac = std::fabs(wo.z);
    if (ac > T(1e-6)) fsum = fsum / ac;
    return fsum;
}
template <class T> T hair_pdf(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m, T h) {
    HairFrame<T> F = hair_frame(wi, wo, m, h);
    HairParams<T> P = hair_params(m);
    V3<T> ap[4];
    hair_ap(F.cto, F.sto, h, F.eta, P.sigma_a, ap);
    T al[4], sum = T(0);
    for (int i = 0; i <= 3; i++) { al[i] = luminance(ap[i]); sum += al[i]; }
    T inv = sum > T(0) ? T(1) / sum : T(0);
    T pdf = T(0);
    for (int p = 0; p < 3; p++) {
        T sp, cp;
        hair_tilt(p, F.sto, F.cto, P.sin2k, P.cos2k, sp, cp);
        pdf += hair_mp(F.cti, cp, F.sti, sp, P.v[p]) * al[p] * inv * hair_np(F.phi, p, P.s, F.go, F.gt);
    }
    pdf += hair_mp(F.cti, F.cto, F.sti, F.sto, P.v[3]) * al[3] * inv * (T(1) / (T(2) * kPi<T>));
    return pdf;
}
// uniforms u[0..3] = the four NextFloat draws of HairBCSDF_Sample (Hair.hlsli:351-432)
template <class T> V3<T> hair_sample(const V3<T> &wi, const T *u, const Mat<T> &m, T h, V3<T> &wo, T &pdf) {
    T sto = wi.x;
    T cto = std::sqrt(std::max(T(0), T(1) - sto * sto));
    T phio = std::atan2(wi.z, wi.y);
    T go = std::asin(clampT(h, T(-1), T(1)));
    T eta = m.intIOR;
    T etap = std::sqrt(std::max(T(0), eta * eta - sto * sto)) / std::max(cto, T(1e-6));
    T gt = std::asin(clampT(h / etap, T(-1), T(1)));
    HairParams<T> P = hair_params(m);
    V3<T> ap[4];
    hair_ap(cto, sto, h, eta, P.sigma_a, ap);
    T apPdf[4], sum = T(0);
    for (int i = 0; i <= 3; i++) { apPdf[i] = luminance(ap[i]); sum += apPdf[i]; }
    T inv = sum > T(0) ? T(1) / sum : T(0);
    for (int j = 0; j <= 3; j++) apPdf[j] *= inv;
    T u0 = u[0];
    int p = 0;
    T cdf = apPdf[0];
    while (p < 3 && u0 > cdf) { p++; cdf += apPdf[p]; }
    T lobeStart = cdf - apPdf[p];
    u0 = clampT((u0 - lobeStart) / std::max(apPdf[p], T(1e-10)), T(0), T(1));
    (void)u0;
    T sp, cp;
    hair_tilt(p, sto, cto, P.sin2k, P.cos2k, sp, cp);
    T u1 = u[1], u2 = u[2];
    T ct = T(1) + P.v[p] * std::log(std::max(u1, T(1e-5)) + (T(1) - u1) * std::exp(T(-2) / P.v[p]));
    T st = std::sqrt(std::max(T(0), T(1) - ct * ct));
    T cphs = std::cos(T(2) * kPi<T> * u2);
    T sti = -ct * sp + st * cphs * cp;
    T cti = std::sqrt(std::max(T(0), T(1) - sti * sti));
    T u3 = u[3];
    T dphi;
    if (p < 3) dphi = hair_phi(p, go, gt) + hair_sample_trimmed_logistic(u3, P.s, -kPi<T>, kPi<T>);
    else dphi = T(2) * kPi<T> * u3;
    T phii = phio + dphi;
    wo = V3<T>(sti, cti * std::cos(phii), cti * std::sin(phii));
    pdf = hair_pdf(wi, wo, m, h);
    if (pdf <= T(0)) return V3<T>(T(0));
    V3<T> f = hair_eval(wi, wo, m, h);
    return f * std::fabs(wo.z) / pdf;
}

// ---------------------------------------------------------------------------
// Material dispatch (shaders/Material.hlsli:18-194)
// ---------------------------------------------------------------------------
template <class T> V3<T> material_eval(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m, T h) {
    switch (m.type) {
        case PT_MAT_DIFFUSE:
            if (wi.z <= T(0) || wo.z <= T(0)) return V3<T>(T(0));
            return m.albedo * kInvPi<T>;
        case PT_MAT_MICROFACET: return microfacet_eval(wi, wo, m);
        case PT_MAT_DISNEY: return disney_eval(wi, wo, m);
        case PT_MAT_HAIR: return hair_eval(wi, wo, m, h);
        case PT_MAT_SUBSURFACE: return subsurface_eval(wi, wo, m);
        default: return V3<T>(T(0));
    }
}
template <class T> T material_pdf(const V3<T> &wi, const V3<T> &wo, const Mat<T> &m, T h) {
    switch (m.type) {
        case PT_MAT_DIFFUSE:
            if (wi.z <= T(0) || wo.z <= T(0)) return T(0);
            return wo.z * kInvPi<T>;
        case PT_MAT_MICROFACET: return microfacet_pdf(wi, wo, m);
        case PT_MAT_DISNEY: return disney_pdf(wi, wo, m);
        case PT_MAT_HAIR: return hair_pdf(wi, wo, m, h);
        case PT_MAT_SUBSURFACE: return subsurface_pdf(wi, wo, m);
        default: return T(0);
    }
}
// Mirror / dielectric scattering of the shader's delta branch
// (shaders/Shaders.hlsl:419-472) restated in the local shading frame of a BSDF
// query: wi toward the viewer, z the outward normal, wi.z < 0 a query from
// inside (the shader's hitBackFace, which turns N to the ray's side and swaps
// the IORs).  u: the dielectric's Fresnel draw.  Weight 1, pdf 0 (discrete).
template <class T>
V3<T> delta_sample(const V3<T> &wi, const Mat<T> &m, T u, V3<T> &wo, T &pdf) {
    bool back = wi.z < T(0);
    V3<T> I = -wi, N(T(0), T(0), back ? T(-1) : T(1));
    pdf = T(0);
    if (m.type == PT_MAT_MIRROR) {
        wo = reflect(I, N);
        return V3<T>(T(1));
    }
    T etaI = back ? m.intIOR : m.extIOR, etaT = back ? m.extIOR : m.intIOR;
    T Fr = fresnel_dielectric(dot(-I, N), etaI, etaT);
    if (u < Fr) wo = reflect(I, N);
    else {
        wo = refract(I, N, etaI / etaT);
        if (dot(wo, wo) < T(0.001)) wo = reflect(I, N);
    }
    return V3<T>(T(1));
}

// u: the uniforms MaterialSample draws, in draw order; *used = how many.
template <class T>
V3<T> material_sample(const V3<T> &wi, const T *u, const Mat<T> &m, T h, V3<T> &wo, T &pdf, int *used) {
    *used = 0;
    switch (m.type) {
        case PT_MAT_DIFFUSE: {
            if (wi.z <= T(0)) { wo = V3<T>(T(0), T(0), T(1)); pdf = T(0); return V3<T>(T(0)); }
            *used = 2;
            wo = cosine_sample_hemisphere(u[0], u[1]);
            pdf = wo.z * kInvPi<T>;
            return m.albedo;
        }
        case PT_MAT_MICROFACET: {  // Microfacet.hlsli:93-125
            if (wi.z <= T(0)) { wo = V3<T>(T(0), T(0), T(1)); pdf = T(0); return V3<T>(T(0)); }
            *used = 2;
            V3<T> kd = m.albedo;
            T ks = T(1) - std::max(kd.x, std::max(kd.y, kd.z));
            T ux = u[0], uy = u[1];
            if (ux < ks) {
                ux /= ks;
                V3<T> wh = beckmann_sample(ux, uy, m.alpha);
                wo = T(2) * dot(wh, wi) * wh - wi;
            } else {
                ux = (ux - ks) / (T(1) - ks);
                wo = cosine_sample_hemisphere(ux, uy);
            }
            if (wo.z <= T(0)) { pdf = T(0); return V3<T>(T(0)); }
            pdf = microfacet_pdf(wi, wo, m);
            if (pdf <= T(0)) return V3<T>(T(0));
            return microfacet_eval(wi, wo, m) * wo.z / pdf;
        }
        case PT_MAT_DISNEY: {  // Material.hlsli:127-183
            if (wi.z <= T(0)) { wo = V3<T>(T(0), T(0), T(1)); pdf = T(0); return V3<T>(T(0)); }
            *used = 3;
            LobeProbs<T> p = disney_probs(m);
            T u0 = u[0];
            if (u0 < p.d) {
                wo = cosine_sample_hemisphere(u[1], u[2]);
            } else if (u0 < p.d + p.s) {
                T a = std::max(m.roughness * m.roughness, T(1e-4));
                V3<T> wh = ggx_sample_wh(u[1], u[2], a);
                wo = T(2) * dot(wh, wi) * wh - wi;
            } else {
                V3<T> wh = gtr1_sample_wh(u[1], u[2], disney_cc_alpha(m));
                wo = T(2) * dot(wh, wi) * wh - wi;
            }
            if (wo.z <= T(0)) { pdf = T(0); return V3<T>(T(0)); }
            pdf = p.d * (wo.z * kInvPi<T>) + p.s * disney_spec_pdf(wi, wo, m) + p.c * disney_cc_pdf(wi, wo, m);
            if (pdf <= T(0)) return V3<T>(T(0));
            V3<T> ft = (T(1) - m.metallic) * (disney_diffuse_lobe(wi, wo, m) + disney_sheen(wi, wo, m)) +
                       disney_spec_eval(wi, wo, m) + disney_cc_eval(wi, wo, m);
            return ft * wo.z / pdf;
        }
        case PT_MAT_HAIR:
            *used = 4;
            return hair_sample(wi, u, m, h, wo, pdf);
        default:
            wo = V3<T>(T(0), T(0), T(1));
            pdf = T(0);
            return V3<T>(T(0));
    }
}

// ---------------------------------------------------------------------------
// Henyey-Greenstein (shaders/Volume.hlsl:31-65)
// ---------------------------------------------------------------------------
template <class T> T hg(T c, T g) {
    T g2 = g * g;
    T den = T(1) + g2 - T(2) * g * c;
    return (T(1) / (T(4) * kPi<T>)) * (T(1) - g2) / (den * std::sqrt(std::max(den, T(1e-8))));
}
template <class T> V3<T> sample_hg(const V3<T> &wo, T g, T xi1, T xi2, T &pdf) {
    T c;
    if (std::fabs(g) < T(1e-3)) c = T(1) - T(2) * xi1;
    else {
        T sqr = (T(1) - g * g) / (T(1) + g - T(2) * g * xi1);
        c = (T(1) + g * g - sqr * sqr) / (T(2) * g);
        c = clampT(c, T(-1), T(1));
    }
    T s = std::sqrt(std::max(T(0), T(1) - c * c));
    T phi = T(2) * kPi<T> * xi2;
    V3<T> Tn, B;
    build_onb(wo, Tn, B);
    V3<T> wi = s * std::cos(phi) * Tn + s * std::sin(phi) * B + c * wo;
    pdf = hg(c, g);
    return normalize(wi);
}

// ---------------------------------------------------------------------------
// Scene
// ---------------------------------------------------------------------------
struct Bvh {
    struct Node { F3 lo, hi; uint32_t left, right, start, count; };  // count>0: leaf
    std::vector<Node> nodes;
    std::vector<uint32_t> prims;
};

struct Grid { uint32_t w, h, d; std::vector<float> v; };

struct Scene {
    std::vector<float> pos, nrm, uv, tan;
    std::vector<uint32_t> idx;
    std::vector<pt_material> mats;
    std::vector<float> emitterCdf;
    std::vector<uint32_t> emitterList;
    uint32_t emitterCount = 0;
    // envmap
    uint32_t envW = 0, envH = 0;
    std::vector<float> env;  // RGBA
    std::vector<float> marg, cond;
    // alias tables: rows (H) then per-row columns (H x W)
    std::vector<float> rowProb, colProb, aliasPdf;
    std::vector<uint32_t> rowAlias, colAlias;
    float envScale = 1.0f, evComp = 0.0f;
    std::vector<pt_volume> vols;
    std::vector<Grid> grids;
    std::vector<Grid> majorants;  // per volume (w = 0: none)
    // global triangle list: (mesh, local prim)
    std::vector<uint32_t> triMesh, triPrim;
    Bvh bvh;
    std::string err;
    // material textures: RGBA8 mip chains (level l of texture t starts at
    // texel texOff[t][l]), sRGB byte -> linear table
    struct Tex { uint32_t w, h, levels, srgb; std::vector<size_t> off; };
    std::vector<Tex> tex;
    std::vector<uint8_t> texels;  // 4 bytes per texel
    float srgbLut[256];
    bool hasAlpha = false;
};

static inline F3 ld3(const std::vector<float> &b, uint32_t i) { return F3(b[3 * i], b[3 * i + 1], b[3 * i + 2]); }

// ---- emitter CDFs: src/cpu/mesh.cpp:24-40 + include/dpdf.h + src/gpu/DXRApp_Scene.cpp:243-299
static void build_emitters(Scene &s) {
    std::vector<float> all;
    s.emitterList.clear();
    for (uint32_t i = 0; i < s.mats.size(); i++) {
        pt_material &m = s.mats[i];
        uint32_t nt = m.indexCount / 3;
        std::vector<float> cdf(1, 0.0f);
        for (uint32_t t = 0; t < nt; t++) {
            const uint32_t *f = &s.idx[m.indexOffset + 3 * t];
            F3 p0 = ld3(s.pos, m.vertexOffset + f[0]);
            F3 p1 = ld3(s.pos, m.vertexOffset + f[1]);
            F3 p2 = ld3(s.pos, m.vertexOffset + f[2]);
            F3 c = cross(p1 - p0, p2 - p0);
            cdf.push_back(cdf.back() + 0.5f * std::sqrt(dot(c, c)));
        }
        float sum = cdf.back();
        if (sum > 0) {
            float inv = 1.0f / sum;
            for (size_t k = 1; k < cdf.size(); k++) cdf[k] *= inv;
            cdf.back() = 1.0f;
        }
        m.surfaceArea = sum;
        m.emitterCdfOffset = 0;
        m.emitterSelectionProb = 0.0f;
        if (m.isEmitter) {
            m.emitterCdfOffset = (uint32_t)all.size();
            all.insert(all.end(), cdf.begin(), cdf.end());
            s.emitterList.push_back(i);
        }
    }
    uint32_t ne = (uint32_t)s.emitterList.size();
    std::vector<float> pc(ne + 1, 0.0f);
    for (uint32_t k = 0; k < ne; k++) {
        const pt_material &m = s.mats[s.emitterList[k]];
        float l = 0.2126f * m.radiance[0] + 0.7152f * m.radiance[1] + 0.0722f * m.radiance[2];
        pc[k + 1] = pc[k] + l * m.surfaceArea;
    }
    float tot = pc[ne];
    if (tot > 0.0f) {
        float inv = 1.0f / tot;
        for (uint32_t k = 1; k <= ne; k++) pc[k] *= inv;
    } else {
        for (uint32_t k = 0; k <= ne; k++) pc[k] = float(k) / float(std::max(ne, 1u));
    }
    pc[ne] = 1.0f;
    for (uint32_t k = 0; k < ne; k++) s.mats[s.emitterList[k]].emitterSelectionProb = pc[k + 1] - pc[k];
    for (uint32_t k = 0; k < ne; k++) s.mats[s.emitterList[k]].emitterCdfOffset += ne + 1;
    all.insert(all.begin(), pc.begin(), pc.end());
    s.emitterCdf = all;
    s.emitterCount = ne;
}

// ---- envmap distribution: src/gpu/DXRApp_Textures.cpp:281-389
static void build_env(Scene &s) {
    const uint32_t W = s.envW, H = s.envH;
    s.cond.assign((size_t)H * (W + 1), 0.0f);
    s.marg.assign(H + 1, 0.0f);
    std::vector<float> rowSums(H);
    const float PI = 3.14159265358979323846f;
    for (uint32_t y = 0; y < H; ++y) {
        float theta = PI * (y + 0.5f) / (float)H;
        float st = std::sin(theta);
        size_t rb = (size_t)y * (W + 1);
        s.cond[rb] = 0.0f;
        float rs = 0.0f;
        for (uint32_t x = 0; x < W; ++x) {
            const float *p = &s.env[((size_t)y * W + x) * 4];
            float w = (0.2126f * p[0] + 0.7152f * p[1] + 0.0722f * p[2]) * st;
            if (w < 0.0f) w = 0.0f;
            rs += w;
            s.cond[rb + x + 1] = rs;
        }
        rowSums[y] = rs;
        if (rs > 0.0f) {
            float inv = 1.0f / rs;
            for (uint32_t x = 1; x <= W; ++x) s.cond[rb + x] *= inv;
        } else {
            for (uint32_t x = 0; x <= W; ++x) s.cond[rb + x] = (float)x / (float)W;
        }
    }
    double total = 0.0;
    for (uint32_t y = 0; y < H; ++y) total += rowSums[y];
    s.marg[0] = 0.0f;
    if (total > 0.0) {
        double acc = 0.0, invT = 1.0 / total;
        for (uint32_t y = 0; y < H; ++y) {
            acc += rowSums[y];
            s.marg[y + 1] = (float)(acc * invT);
        }
        s.marg[H] = 1.0f;
    } else {
        for (uint32_t y = 0; y <= H; ++y) s.marg[y] = (float)y / (float)H;
    }
}

// ---- alias tables (new in this build; same target density as the CDF)
// Walker/Vose construction in FP64 over weights w(x,y) = max(lum*sin(theta_y), 0),
// rows by their FP64 row sums, columns within each row.  pdf per pixel is
// (rowSum/total) * (w/rowSum) in FP64, rounded to float once.
static void build_alias_1d(const std::vector<double> &w, float *prob, uint32_t *alias) {
    const size_t n = w.size();
    double sum = 0.0;
    for (double x : w) sum += x;
    if (!(sum > 0.0)) {
        for (size_t i = 0; i < n; i++) { prob[i] = 1.0f; alias[i] = (uint32_t)i; }
        return;
    }
    std::vector<double> q(n);
    std::vector<uint32_t> small, large;
    for (size_t i = 0; i < n; i++) {
        q[i] = w[i] * (double)n / sum;
        (q[i] < 1.0 ? small : large).push_back((uint32_t)i);
    }
    // deterministic Vose: process stacks in index order
    std::reverse(small.begin(), small.end());
    std::reverse(large.begin(), large.end());
    while (!small.empty() && !large.empty()) {
        uint32_t l = small.back(); small.pop_back();
        uint32_t g = large.back(); large.pop_back();
        prob[l] = (float)q[l];
        alias[l] = g;
        q[g] = (q[g] + q[l]) - 1.0;
        if (q[g] < 1.0) small.push_back(g); else large.push_back(g);
    }
    while (!large.empty()) { uint32_t g = large.back(); large.pop_back(); prob[g] = 1.0f; alias[g] = g; }
    while (!small.empty()) { uint32_t l = small.back(); small.pop_back(); prob[l] = 1.0f; alias[l] = l; }
}
static void build_env_alias(Scene &s) {
    const uint32_t W = s.envW, H = s.envH;
    const double PI = 3.14159265358979323846;
    s.rowProb.assign(H, 0.0f); s.rowAlias.assign(H, 0);
    s.colProb.assign((size_t)H * W, 0.0f); s.colAlias.assign((size_t)H * W, 0);
    s.aliasPdf.assign((size_t)H * W, 0.0f);
    std::vector<double> rowSum(H, 0.0), wrow(W);
    double total = 0.0;
    std::vector<double> wall((size_t)H * W);
    for (uint32_t y = 0; y < H; y++) {
        float st = std::sin(3.14159265358979323846f * (y + 0.5f) / (float)H);
        double rs = 0.0;
        for (uint32_t x = 0; x < W; x++) {
            const float *p = &s.env[((size_t)y * W + x) * 4];
            float w = (0.2126f * p[0] + 0.7152f * p[1] + 0.0722f * p[2]) * st;
            double wd = w < 0.0f ? 0.0 : (double)w;
            wall[(size_t)y * W + x] = wd;
            rs += wd;
        }
        rowSum[y] = rs;
        total += rs;
    }
    build_alias_1d(rowSum, s.rowProb.data(), s.rowAlias.data());
    for (uint32_t y = 0; y < H; y++) {
        for (uint32_t x = 0; x < W; x++) wrow[x] = wall[(size_t)y * W + x];
        build_alias_1d(wrow, &s.colProb[(size_t)y * W], &s.colAlias[(size_t)y * W]);
        for (uint32_t x = 0; x < W; x++) {
            double pp;
            if (total > 0.0) pp = rowSum[y] > 0.0 ? wall[(size_t)y * W + x] / total : 0.0;
            else pp = 1.0 / ((double)W * (double)H);
            s.aliasPdf[(size_t)y * W + x] = (float)(pp * (double)W * (double)H / (2.0 * PI * PI));
        }
    }
}

// ---- envmap lookups (shaders/Envmap.hlsli)
// Bilinear texel fetch with the reference's s1 sampler: wrap U, clamp V
// (src/gpu/DXRApp_Pipeline.cpp:56-61), texel centres at (i + 0.5) / N.
static F3 env_bilinear(const Scene &s, float u, float v) {
    const int W = (int)s.envW, H = (int)s.envH;
    float x = u * (float)W - 0.5f, y = v * (float)H - 0.5f;
    float fx0 = std::floor(x), fy0 = std::floor(y);
    float fx = x - fx0, fy = y - fy0;
    int x0 = (int)fx0, y0 = (int)fy0;
    int xa = ((x0 % W) + W) % W, xb = (((x0 + 1) % W) + W) % W;
    int ya = std::min(std::max(y0, 0), H - 1), yb = std::min(std::max(y0 + 1, 0), H - 1);
    auto px = [&](int xx, int yy) {
        const float *p = &s.env[((size_t)yy * W + xx) * 4];
        return F3(p[0], p[1], p[2]);
    };
    F3 a = px(xa, ya) * (1.0f - fx) + px(xb, ya) * fx;
    F3 b = px(xa, yb) * (1.0f - fx) + px(xb, yb) * fx;
    return a * (1.0f - fy) + b * fy;
}
static F3 eval_env(const Scene &s, F3 dir) {  // Envmap.hlsli:15-24
    F3 d = normalize(dir);
    float phi = std::atan2(d.z, d.x);
    if (phi < 0.0f) phi += 2.0f * kPi<float>;
    float theta = std::acos(clampT(d.y, -1.0f, 1.0f));
    return env_bilinear(s, phi / (2.0f * kPi<float>), theta / kPi<float>) * s.envScale;
}
static uint32_t cdf_search(const float *buf, uint32_t n, float u) {  // Envmap.hlsli:31-45, Emitter.hlsli:17-31
    uint32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        uint32_t mid = (lo + hi) / 2;
        if (buf[mid] <= u) lo = mid + 1;
        else hi = mid;
    }
    return (uint32_t)std::max(0, (int)lo - 1);
}
static void sample_env_cdf(const Scene &s, float u1, float u2, F3 &dir, F3 &rad, float &pdf) {  // Envmap.hlsli:58-101
    const uint32_t W = s.envW, H = s.envH;
    uint32_t y = cdf_search(s.marg.data(), H + 1, u1);
    float m0 = s.marg[y], m1 = s.marg[y + 1];
    float pMar = m1 - m0;
    float jv = pMar > 1e-20f ? saturate((u1 - m0) / pMar) : 0.5f;
    const float *row = &s.cond[(size_t)y * (W + 1)];
    uint32_t x = cdf_search(row, W + 1, u2);
    float c0 = row[x], c1 = row[x + 1];
    float pCon = c1 - c0;
    float ju = pCon > 1e-20f ? saturate((u2 - c0) / pCon) : 0.5f;
    float u = ((float)x + ju) / (float)W;
    float v = ((float)y + jv) / (float)H;
    float phi = 2.0f * kPi<float> * u, theta = kPi<float> * v;
    float st = std::sin(theta), ct = std::cos(theta);
    dir = F3(st * std::cos(phi), ct, st * std::sin(phi));
    rad = env_bilinear(s, u, v) * s.envScale;
    float pPix = pMar * pCon;
    float den = 2.0f * kPi<float> * kPi<float> * std::max(st, 1e-8f);
    pdf = pPix * (float)(W * H) / den;
}
static float env_pdf_cdf(const Scene &s, F3 dir) {  // Envmap.hlsli:109-135
    const uint32_t W = s.envW, H = s.envH;
    F3 d = normalize(dir);
    float phi = std::atan2(d.z, d.x);
    if (phi < 0.0f) phi += 2.0f * kPi<float>;
    float theta = std::acos(clampT(d.y, -1.0f, 1.0f));
    float st = std::sin(theta);
    float u = phi / (2.0f * kPi<float>), v = theta / kPi<float>;
    uint32_t x = std::min((uint32_t)(u * (float)W), W - 1);
    uint32_t y = std::min((uint32_t)(v * (float)H), H - 1);
    float pMar = s.marg[y + 1] - s.marg[y];
    const float *row = &s.cond[(size_t)y * (W + 1)];
    float pCon = row[x + 1] - row[x];
    float den = 2.0f * kPi<float> * kPi<float> * std::max(st, 1e-8f);
    return pMar * pCon * (float)(W * H) / den;
}
// Alias-mode sampling: row by alias table on u1, column by alias table on u2;
// the leftover fraction of each uniform is the in-texel jitter.
static inline uint32_t alias_pick(const float *prob, const uint32_t *alias, uint32_t n, float u, float &frac) {
    float sc = u * (float)n;
    uint32_t i = std::min((uint32_t)sc, n - 1);
    float f = sc - (float)i;
    float p = prob[i];
    if (f < p) { frac = p > 0.0f ? f / p : 0.5f; return i; }
    frac = p < 1.0f ? (f - p) / (1.0f - p) : 0.5f;
    return alias[i];
}
static void sample_env_alias(const Scene &s, float u1, float u2, F3 &dir, F3 &rad, float &pdf) {
    const uint32_t W = s.envW, H = s.envH;
    float jv, ju;
    uint32_t y = alias_pick(s.rowProb.data(), s.rowAlias.data(), H, u1, jv);
    uint32_t x = alias_pick(&s.colProb[(size_t)y * W], &s.colAlias[(size_t)y * W], W, u2, ju);
    jv = saturate(jv); ju = saturate(ju);
    float u = ((float)x + ju) / (float)W;
    float v = ((float)y + jv) / (float)H;
    float phi = 2.0f * kPi<float> * u, theta = kPi<float> * v;
    float st = std::sin(theta), ct = std::cos(theta);
    dir = F3(st * std::cos(phi), ct, st * std::sin(phi));
    rad = env_bilinear(s, u, v) * s.envScale;
    pdf = s.aliasPdf[(size_t)y * W + x] / std::max(st, 1e-8f);
}
static float env_pdf_alias(const Scene &s, F3 dir) {
    const uint32_t W = s.envW, H = s.envH;
    F3 d = normalize(dir);
    float phi = std::atan2(d.z, d.x);
    if (phi < 0.0f) phi += 2.0f * kPi<float>;
    float theta = std::acos(clampT(d.y, -1.0f, 1.0f));
    float st = std::sin(theta);
    float u = phi / (2.0f * kPi<float>), v = theta / kPi<float>;
    uint32_t x = std::min((uint32_t)(u * (float)W), W - 1);
    uint32_t y = std::min((uint32_t)(v * (float)H), H - 1);
    return s.aliasPdf[(size_t)y * W + x] / std::max(st, 1e-8f);
}

// ---------------------------------------------------------------------------
// Geometry access (shaders/GeometryUtils.hlsli:44-113)
// ---------------------------------------------------------------------------
static inline void tri_idx(const Scene &s, uint32_t mesh, uint32_t prim, uint32_t &i0, uint32_t &i1, uint32_t &i2) {
    const pt_material &m = s.mats[mesh];
    uint32_t base = m.indexOffset + prim * 3;
    i0 = m.vertexOffset + s.idx[base]; i1 = m.vertexOffset + s.idx[base + 1]; i2 = m.vertexOffset + s.idx[base + 2];
}
static F3 geometric_normal(const Scene &s, uint32_t mesh, uint32_t prim) {
    uint32_t i0, i1, i2;
    tri_idx(s, mesh, prim, i0, i1, i2);
    F3 p0 = ld3(s.pos, i0), p1 = ld3(s.pos, i1), p2 = ld3(s.pos, i2);
    return normalize(cross(p1 - p0, p2 - p0));
}
static F3 interp_normal(const Scene &s, uint32_t mesh, uint32_t prim, float bx, float by) {
    uint32_t i0, i1, i2;
    tri_idx(s, mesh, prim, i0, i1, i2);
    F3 n0 = ld3(s.nrm, i0), n1 = ld3(s.nrm, i1), n2 = ld3(s.nrm, i2);
    float w0 = 1.0f - bx - by;
    F3 n = n0 * w0 + n1 * bx + n2 * by;
    float l2 = dot(n, n);
    if (l2 < 1e-8f) return geometric_normal(s, mesh, prim);
    return n * (1.0f / std::sqrt(l2));
}
static void interp_uv(const Scene &s, uint32_t mesh, uint32_t prim, float bx, float by, float &u, float &v) {
    uint32_t i0, i1, i2;
    tri_idx(s, mesh, prim, i0, i1, i2);
    float w0 = 1.0f - bx - by;
    u = s.uv[2 * i0] * w0 + s.uv[2 * i1] * bx + s.uv[2 * i2] * by;
    v = s.uv[2 * i0 + 1] * w0 + s.uv[2 * i1 + 1] * bx + s.uv[2 * i2 + 1] * by;
}
static F3 interp_tangent(const Scene &s, uint32_t mesh, uint32_t prim, float bx, float by) {
    uint32_t i0, i1, i2;
    tri_idx(s, mesh, prim, i0, i1, i2);
    F3 t0 = ld3(s.tan, i0), t1 = ld3(s.tan, i1), t2 = ld3(s.tan, i2);
    float w0 = 1.0f - bx - by;
    F3 t = t0 * w0 + t1 * bx + t2 * by;
    float l2 = dot(t, t);
    return l2 > 1e-8f ? t * (1.0f / std::sqrt(l2)) : F3(0.0f);
}

// ---------------------------------------------------------------------------
// Material textures (shaders/Shaders.hlsl:232-315, shaders/GeometryUtils.hlsli:
// 120-154, src/gpu/DXRApp_Textures.cpp:34-176): RGBA8 with a box-filtered mip
// chain, sRGB colour maps decoded per texel, trilinear filtering with wrap
// addressing (the hardware sampler s0), LOD from the hit's UV footprint.
// ---------------------------------------------------------------------------
static void build_textures(Scene &s, const pt_scene_desc *d) {
    for (uint32_t i = 0; i < 256; i++) {  // the _SRGB decode, in double
        double v = i / 255.0;
        s.srgbLut[i] = (float)(v <= 0.04045 ? v / 12.92 : std::pow((v + 0.055) / 1.055, 2.4));
    }
    for (uint32_t t = 0; t < d->num_textures; t++) {
        const pt_texture &src = d->textures[t];
        Scene::Tex tx{src.width, src.height, 1, src.srgb ? 1u : 0u, {}};
        for (uint32_t dim = std::max(src.width, src.height); dim > 1; dim >>= 1) tx.levels++;
        tx.off.push_back(s.texels.size() / 4);
        s.texels.insert(s.texels.end(), src.rgba8, src.rgba8 + (size_t)src.width * src.height * 4);
        uint32_t pw = src.width, ph = src.height;
        for (uint32_t l = 1; l < tx.levels; l++) {  // integer mean of 2 x 2, edges repeated
            uint32_t mw = std::max(pw / 2, 1u), mh = std::max(ph / 2, 1u);
            size_t prev = tx.off[l - 1], cur = s.texels.size() / 4;
            tx.off.push_back(cur);
            s.texels.resize((cur + (size_t)mw * mh) * 4);
            for (uint32_t y = 0; y < mh; y++)
                for (uint32_t x = 0; x < mw; x++) {
                    uint32_t sx = std::min(x * 2, pw - 1), sy = std::min(y * 2, ph - 1);
                    uint32_t sx1 = std::min(sx + 1, pw - 1), sy1 = std::min(sy + 1, ph - 1);
                    for (int c = 0; c < 4; c++) {
                        auto at = [&](uint32_t xx, uint32_t yy) { return (int)s.texels[(prev + (size_t)yy * pw + xx) * 4 + c]; };
                        s.texels[(cur + (size_t)y * mw + x) * 4 + c] =
                            (uint8_t)((at(sx, sy) + at(sx1, sy) + at(sx, sy1) + at(sx1, sy1)) / 4);
                    }
                }
            pw = mw;
            ph = mh;
        }
        s.tex.push_back(std::move(tx));
    }
    for (const pt_material &m : s.mats)
        if (m.indexCount && m.alphaTexIndex != PT_NO_TEXTURE) s.hasAlpha = true;
}
struct F4 { float x, y, z, w; };
static F4 lerp4(F4 a, F4 b, float t) {
    return {a.x + (b.x - a.x) * t, a.y + (b.y - a.y) * t, a.z + (b.z - a.z) * t, a.w + (b.w - a.w) * t};
}
static F4 tex_texel(const Scene &s, const Scene::Tex &t, uint32_t level, int W, int x, int y) {
    const uint8_t *c = &s.texels[(t.off[level] + (size_t)y * W + x) * 4];
    if (t.srgb) return {s.srgbLut[c[0]], s.srgbLut[c[1]], s.srgbLut[c[2]], (float)c[3] / 255.0f};
    return {(float)c[0] / 255.0f, (float)c[1] / 255.0f, (float)c[2] / 255.0f, (float)c[3] / 255.0f};
}
static F4 tex_bilinear(const Scene &s, const Scene::Tex &t, uint32_t level, float u, float v) {
    const int W = (int)std::max(t.w >> level, 1u), H = (int)std::max(t.h >> level, 1u);
    u -= std::floor(u);
    v -= std::floor(v);
    float x = u * (float)W - 0.5f, y = v * (float)H - 0.5f;
    float fx0 = std::floor(x), fy0 = std::floor(y);
    float fx = x - fx0, fy = y - fy0;
    int x0 = std::isfinite(fx0) ? (int)fx0 : 0, y0 = std::isfinite(fy0) ? (int)fy0 : 0;
    int xa = ((x0 % W) + W) % W, xb = (((x0 + 1) % W) + W) % W;
    int ya = ((y0 % H) + H) % H, yb = (((y0 + 1) % H) + H) % H;
    F4 top = lerp4(tex_texel(s, t, level, W, xa, ya), tex_texel(s, t, level, W, xb, ya), fx);
    F4 bot = lerp4(tex_texel(s, t, level, W, xa, yb), tex_texel(s, t, level, W, xb, yb), fx);
    return lerp4(top, bot, fy);
}
static F4 tex_sample(const Scene &s, uint32_t index, float u, float v, float lod) {
    const Scene::Tex &t = s.tex[index];
    lod = std::min(std::max(lod, 0.0f), (float)(t.levels - 1));
    uint32_t l0 = (uint32_t)std::floor(lod);
    float f = lod - (float)l0;
    F4 a = tex_bilinear(s, t, l0, u, v);
    if (f > 0.0f && l0 + 1 < t.levels) a = lerp4(a, tex_bilinear(s, t, l0 + 1, u, v), f);
    return a;
}
static float uv_footprint(const Scene &s, uint32_t mesh, uint32_t prim, float hitT, uint32_t W, uint32_t H) {  // :120-145
    uint32_t i0, i1, i2;
    tri_idx(s, mesh, prim, i0, i1, i2);
    F3 p0 = ld3(s.pos, i0), p1 = ld3(s.pos, i1), p2 = ld3(s.pos, i2);
    float u0 = s.uv[2 * i0], v0 = s.uv[2 * i0 + 1], u1 = s.uv[2 * i1], v1 = s.uv[2 * i1 + 1];
    float u2 = s.uv[2 * i2], v2 = s.uv[2 * i2 + 1];
    float worldArea = 0.5f * length(cross(p1 - p0, p2 - p0));
    float uvArea = 0.5f * std::fabs((u1 - u0) * (v2 - v0) - (u2 - u0) * (v1 - v0));
    if (worldArea < 1e-12f || uvArea < 1e-12f) return 0.0f;
    float pixelAngle = 1.0f / (float)std::max(W, H);
    return hitT * pixelAngle * std::sqrt(uvArea / worldArea);
}
static float tex_lod(const Scene &s, uint32_t index, float footprint) {  // :148-154
    const Scene::Tex &t = s.tex[index];
    float tpp = footprint * (float)std::max(t.w, t.h);
    return std::max(std::log2(std::max(tpp, 1.0f)), 0.0f);
}
// Shaders.hlsl:232-315 on a copy of the hit's material; bends N.
static void apply_textures(const Scene &s, pt_material &m, uint32_t mesh, uint32_t prim, float hitT, float bx, float by,
                           F3 &N, uint32_t W, uint32_t H) {
    float foot = uv_footprint(s, mesh, prim, hitT, W, H);
    float u, v;
    interp_uv(s, mesh, prim, bx, by, u, v);
    F3 alb(m.albedo[0], m.albedo[1], m.albedo[2]);
    if (m.albedoTexIndex != PT_NO_TEXTURE) {
        F4 c = tex_sample(s, m.albedoTexIndex, u, v, tex_lod(s, m.albedoTexIndex, foot));
        alb = F3(c.x, c.y, c.z);
    }
    if (m.normalTexIndex != PT_NO_TEXTURE) {
        uint32_t i0, i1, i2;
        tri_idx(s, mesh, prim, i0, i1, i2);
        F3 p0 = ld3(s.pos, i0), p1 = ld3(s.pos, i1), p2 = ld3(s.pos, i2);
        F3 e1 = p1 - p0, e2 = p2 - p0;
        float u0 = s.uv[2 * i0], v0 = s.uv[2 * i0 + 1];
        float du1 = s.uv[2 * i1] - u0, dv1 = s.uv[2 * i1 + 1] - v0;
        float du2 = s.uv[2 * i2] - u0, dv2 = s.uv[2 * i2 + 1] - v0;
        float det = du1 * dv2 - du2 * dv1;
        F3 T, B;
        if (std::fabs(det) > 1e-8f) {
            float invDet = 1.0f / det;
            T = normalize((dv2 * e1 - dv1 * e2) * invDet);
            T = normalize(T - N * dot(N, T));
            B = cross(N, T);
        } else {
            build_onb(N, T, B);
        }
        F4 c = tex_sample(s, m.normalTexIndex, u, v, tex_lod(s, m.normalTexIndex, foot));
        F3 tn = F3(c.x, c.y, c.z) * 2.0f - F3(1.0f);
        N = normalize(T * tn.x + B * tn.y + N * tn.z);
    }
    m.albedo[0] = alb.x; m.albedo[1] = alb.y; m.albedo[2] = alb.z;
    if (m.type != PT_MAT_HAIR && m.roughnessTexIndex != PT_NO_TEXTURE) {
        float r = tex_sample(s, m.roughnessTexIndex, u, v, tex_lod(s, m.roughnessTexIndex, foot)).x;
        m.alpha = r;
        m.roughness = r;
    }
    if (m.specularTexIndex != PT_NO_TEXTURE)
        m.specular = tex_sample(s, m.specularTexIndex, u, v, tex_lod(s, m.specularTexIndex, foot)).x * 0.5f;
    if (m.subsurfaceTexIndex != PT_NO_TEXTURE)
        m.subsurface = tex_sample(s, m.subsurfaceTexIndex, u, v, tex_lod(s, m.subsurfaceTexIndex, foot)).x;
}
static bool has_shading_textures(const pt_material &m) {
    return m.albedoTexIndex != PT_NO_TEXTURE || m.normalTexIndex != PT_NO_TEXTURE ||
           m.roughnessTexIndex != PT_NO_TEXTURE || m.specularTexIndex != PT_NO_TEXTURE ||
           m.subsurfaceTexIndex != PT_NO_TEXTURE;
}
// Stochastic alpha of an alpha-mapped candidate (shaders/RayQueryTrace.hlsli:
// 50-62, 100-112): alpha at level 0 (.r; shadow rays: .a when below 1),
// ignored below 0.01, kept with probability alpha^2.  The uniform is a hash
// of (path seed, ray key, triangle) instead of the reference's PCG stream
// threaded through candidates in hardware order, so the outcome of each
// candidate does not depend on the traversal order.
static bool alpha_pass(const Scene &s, uint32_t g, float bx, float by, uint32_t seed, uint32_t key, bool shadow) {
    const pt_material &m = s.mats[s.triMesh[g]];
    float u, v;
    interp_uv(s, s.triMesh[g], s.triPrim[g], bx, by, u, v);
    F4 c = tex_sample(s, m.alphaTexIndex, u, v, 0.0f);
    float a = shadow ? (c.w < 1.0f ? c.w : c.x) : c.x;
    if (a < 0.01f) return false;
    uint32_t x = pcg_hash(seed ^ pcg_hash(key * 0x9e3779b9u ^ g));
    float xi = std::min(float(x) * 2.3283064365386963e-10f, 0.99999994f);
    return !(a * a < xi);
}
static inline uint32_t alpha_seed(uint32_t pixelSeed, uint32_t sample) {
    return pcg_hash(pixelSeed * 0x85ebca6bu ^ pcg_hash(sample + 0x27d4eb2fu));
}
static inline uint32_t alpha_key(uint32_t bounce, uint32_t kind) { return bounce * 4u + kind; }
static inline bool alpha_mapped(const Scene &s, uint32_t g) {
    return s.mats[s.triMesh[g]].alphaTexIndex != PT_NO_TEXTURE;
}

// ---------------------------------------------------------------------------
// BVH: binned SAH (16 bins, largest axis) as in src/cpu/accel.cpp:55-324,
// single-threaded; triangle test = Moller-Trumbore of src/cpu/mesh.cpp:51-89.
// ---------------------------------------------------------------------------
static void tri_verts(const Scene &s, uint32_t g, F3 &p0, F3 &p1, F3 &p2) {
    uint32_t i0, i1, i2;
    tri_idx(s, s.triMesh[g], s.triPrim[g], i0, i1, i2);
    p0 = ld3(s.pos, i0); p1 = ld3(s.pos, i1); p2 = ld3(s.pos, i2);
}
static void build_bvh(Scene &s) {
    uint32_t n = (uint32_t)s.triMesh.size();
    Bvh &b = s.bvh;
    b.nodes.clear();
    b.prims.resize(n);
    std::vector<F3> lo(n), hi(n), ce(n);
    for (uint32_t i = 0; i < n; i++) {
        F3 p0, p1, p2;
        tri_verts(s, i, p0, p1, p2);
        lo[i] = vmin(p0, vmin(p1, p2));
        hi[i] = vmax(p0, vmax(p1, p2));
        ce[i] = (lo[i] + hi[i]) * 0.5f;
        b.prims[i] = i;
    }
    if (n == 0) return;
    struct Item { uint32_t node, start, end; };
    std::vector<Item> stack;
    b.nodes.push_back({});
    stack.push_back({0, 0, n});
    while (!stack.empty()) {
        Item it = stack.back();
        stack.pop_back();
        F3 bl(std::numeric_limits<float>::infinity()), bh(-std::numeric_limits<float>::infinity());
        F3 cl = bl, ch = bh;
        for (uint32_t i = it.start; i < it.end; i++) {
            uint32_t p = b.prims[i];
            bl = vmin(bl, lo[p]); bh = vmax(bh, hi[p]);
            cl = vmin(cl, ce[p]); ch = vmax(ch, ce[p]);
        }
        Bvh::Node nd{bl, bh, 0, 0, it.start, it.end - it.start};
        uint32_t cnt = it.end - it.start;
        F3 ext = ch - cl;
        int axis = ext.x > ext.y ? (ext.x > ext.z ? 0 : 2) : (ext.y > ext.z ? 1 : 2);
        if (cnt <= 4 || ext[axis] <= 0.0f) { b.nodes[it.node] = nd; continue; }
        const int NB = 16;
        uint32_t bc[NB] = {};
        F3 blo[NB], bhi[NB];
        for (int k = 0; k < NB; k++) { blo[k] = F3(std::numeric_limits<float>::infinity()); bhi[k] = F3(-std::numeric_limits<float>::infinity()); }
        float mn = cl[axis], inv = NB / ext[axis];
        auto binOf = [&](uint32_t p) { return std::min(NB - 1, (int)((ce[p][axis] - mn) * inv)); };
        for (uint32_t i = it.start; i < it.end; i++) {
            uint32_t p = b.prims[i];
            int k = binOf(p);
            bc[k]++; blo[k] = vmin(blo[k], lo[p]); bhi[k] = vmax(bhi[k], hi[p]);
        }
        auto area = [](F3 l, F3 h) { F3 d = h - l; if (d.x < 0) return 0.0f; return 2.0f * (d.x * d.y + d.y * d.z + d.z * d.x); };
        float best = std::numeric_limits<float>::infinity();
        int bestK = -1;
        for (int k = 1; k < NB; k++) {
            F3 ll(std::numeric_limits<float>::infinity()), lh(-std::numeric_limits<float>::infinity()), rl = ll, rh = lh;
            uint32_t lc = 0, rc = 0;
            for (int j = 0; j < k; j++) if (bc[j]) { ll = vmin(ll, blo[j]); lh = vmax(lh, bhi[j]); lc += bc[j]; }
            for (int j = k; j < NB; j++) if (bc[j]) { rl = vmin(rl, blo[j]); rh = vmax(rh, bhi[j]); rc += bc[j]; }
            if (!lc || !rc) continue;
            float c = area(ll, lh) * lc + area(rl, rh) * rc;
            if (c < best) { best = c; bestK = k; }
        }
        uint32_t mid;
        if (bestK < 0) {
            mid = it.start + cnt / 2;
            std::nth_element(b.prims.begin() + it.start, b.prims.begin() + mid, b.prims.begin() + it.end,
                             [&](uint32_t a, uint32_t c) { return ce[a][axis] < ce[c][axis]; });
        } else {
            auto m = std::partition(b.prims.begin() + it.start, b.prims.begin() + it.end,
                                    [&](uint32_t p) { return binOf(p) < bestK; });
            mid = (uint32_t)(m - b.prims.begin());
        }
        uint32_t L = (uint32_t)b.nodes.size(), R = L + 1;
        b.nodes.push_back({});
        b.nodes.push_back({});
        nd.left = L; nd.right = R; nd.count = 0;
        b.nodes[it.node] = nd;
        stack.push_back({L, it.start, mid});
        stack.push_back({R, mid, it.end});
    }
}
static inline bool box_hit(const F3 &lo, const F3 &hi, const F3 &o, const F3 &invd, float tmin, float tmax) {
    float t0 = tmin, t1 = tmax;
    for (int a = 0; a < 3; a++) {
        float tn = (lo[a] - o[a]) * invd[a], tf = (hi[a] - o[a]) * invd[a];
        if (tn > tf) std::swap(tn, tf);
        if (!(tn <= tf)) { if (std::isnan(tn) || std::isnan(tf)) continue; }
        t0 = std::max(t0, tn);
        t1 = std::min(t1, tf);
    }
    return t0 <= t1 * 1.00000024f;
}
// Moller-Trumbore (src/cpu/mesh.cpp:51-89).  The reference's GPU path
// intersects in ray-tracing hardware whose arithmetic is not published; this
// restatement fixes one: fused multiply-adds in a set order (a*b - c*d as
// fma(a, b, -(c*d)), dot products as fma(z, z', fma(y, y', x*x'))), which the
// kernels and the reference build's ray-query stand-in use too.
static inline float dot_f(const F3 &a, const F3 &b) { return std::fmaf(a.z, b.z, std::fmaf(a.y, b.y, a.x * b.x)); }
static inline F3 cross_f(const F3 &a, const F3 &b) {
    return F3(std::fmaf(a.y, b.z, -(a.z * b.y)), std::fmaf(a.z, b.x, -(a.x * b.z)), std::fmaf(a.x, b.y, -(a.y * b.x)));
}
static bool tri_hit(const F3 &p0, const F3 &p1, const F3 &p2, const F3 &o, const F3 &d, float tmin, float tmax,
                    float &u, float &v, float &t) {
    F3 e1 = p1 - p0, e2 = p2 - p0;
    F3 pv = cross_f(d, e2);
    float det = dot_f(e1, pv);
    if (det > -1e-8f && det < 1e-8f) return false;
    float inv = 1.0f / det;
    F3 tv = o - p0;
    u = dot_f(tv, pv) * inv;
    if (u < 0.0f || u > 1.0f) return false;
    F3 qv = cross_f(tv, e1);
    v = dot_f(d, qv) * inv;
    if (v < 0.0f || u + v > 1.0f) return false;
    t = dot_f(e2, qv) * inv;
    return t >= tmin && t <= tmax;
}
static thread_local uint64_t g_ext_rays = 0, g_shadow_rays = 0;
struct Hit { bool hit; float t, u, v; uint32_t mesh, prim, gid; };
static Hit trace_closest(const Scene &s, F3 o, F3 d, float tmin, float tmax, uint32_t seed = 0, uint32_t key = 0) {
    Hit h{false, tmax, 0, 0, 0, 0, 0};
    g_ext_rays++;
    if (s.bvh.nodes.empty()) return h;
    F3 invd(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    uint32_t stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
        const Bvh::Node &n = s.bvh.nodes[stack[--sp]];
        if (!box_hit(n.lo, n.hi, o, invd, tmin, h.t)) continue;
        if (n.count) {
            for (uint32_t i = n.start; i < n.start + n.count; i++) {
                uint32_t g = s.bvh.prims[i];
                F3 p0, p1, p2;
                tri_verts(s, g, p0, p1, p2);
                float u, v, t;
                if (tri_hit(p0, p1, p2, o, d, tmin, h.t, u, v, t)) {
                    // equal-t ties resolve to the lower global triangle id
                    if (!h.hit || t < h.t || (t == h.t && g < h.gid)) {
                        if (s.hasAlpha && alpha_mapped(s, g) && !alpha_pass(s, g, u, v, seed, key, false)) continue;
                        h.hit = true; h.t = t; h.u = u; h.v = v; h.gid = g;
                    }
                }
            }
        } else {
            stack[sp++] = n.left;
            stack[sp++] = n.right;
        }
    }
    if (h.hit) { h.mesh = s.triMesh[h.gid]; h.prim = s.triPrim[h.gid]; }
    return h;
}
// TraceShadowInline (shaders/RayQueryTrace.hlsli:88-129) for scenes without
// alpha textures: an opaque hit occludes; mirror/dielectric surfaces in
// [tmin, tmax] attenuate by (1 - Fr) with |cos| against the geometric normal.
static bool trace_shadow(const Scene &s, F3 o, F3 d, float tmin, float tmax, F3 &trans, uint32_t seed = 0,
                         uint32_t key = 0) {
    trans = F3(1.0f);
    g_shadow_rays++;
    if (s.bvh.nodes.empty()) return false;
    F3 invd(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    uint32_t stack[128];
    int sp = 0;
    stack[sp++] = 0;
    // Collect glass hits first so the product is order independent.
    std::vector<std::pair<uint32_t, float>> glass;
    while (sp) {
        const Bvh::Node &n = s.bvh.nodes[stack[--sp]];
        if (!box_hit(n.lo, n.hi, o, invd, tmin, tmax)) continue;
        if (n.count) {
            for (uint32_t i = n.start; i < n.start + n.count; i++) {
                uint32_t g = s.bvh.prims[i];
                F3 p0, p1, p2;
                tri_verts(s, g, p0, p1, p2);
                float u, v, t;
                if (!tri_hit(p0, p1, p2, o, d, tmin, tmax, u, v, t)) continue;
                if (s.hasAlpha && alpha_mapped(s, g)) {  // occludes when the stochastic test keeps it
                    if (alpha_pass(s, g, u, v, seed, key, true)) return true;
                    continue;
                }
                const pt_material &m = s.mats[s.triMesh[g]];
                if (m.type == PT_MAT_MIRROR || m.type == PT_MAT_DIELECTRIC) glass.push_back({g, t});
                else return true;
            }
        } else {
            stack[sp++] = n.left;
            stack[sp++] = n.right;
        }
    }
    std::sort(glass.begin(), glass.end());
    for (auto &gt : glass) {
        const pt_material &m = s.mats[s.triMesh[gt.first]];
        F3 Ng = geometric_normal(s, s.triMesh[gt.first], s.triPrim[gt.first]);
        float cosI = std::fabs(dot(d, Ng));
        float Fr = fresnel_dielectric(cosI, m.extIOR, m.intIOR);
        trans = trans * (1.0f - Fr);
    }
    return false;
}

// ---------------------------------------------------------------------------
// Volumes (shaders/Volume.hlsl, src/gpu/DXRApp_Scene.cpp:625-641)
// ---------------------------------------------------------------------------
static void build_majorants(Scene &s) {
    s.majorants.assign(s.vols.size(), Grid{0, 0, 0, {}});
    for (size_t i = 0; i < s.vols.size(); i++) {
        const pt_volume &v = s.vols[i];
        if (!(v.flags & PT_VOLUME_HETEROGENEOUS) || v.density_grid == PT_NO_TEXTURE) continue;
        const Grid &g = s.grids[v.density_grid];
        const uint32_t B = 4;
        Grid m{(g.w + B - 1) / B, (g.h + B - 1) / B, (g.d + B - 1) / B, {}};
        m.v.assign((size_t)m.w * m.h * m.d, 0.0f);
        for (uint32_t z = 0; z < g.d; z++)
            for (uint32_t y = 0; y < g.h; y++)
                for (uint32_t x = 0; x < g.w; x++) {
                    float dd = g.v[(size_t)x + (size_t)g.w * (y + (size_t)g.h * z)];
                    size_t mi = (size_t)(x / B) + (size_t)m.w * ((y / B) + (size_t)m.h * (z / B));
                    m.v[mi] = std::max(m.v[mi], dd);
                }
        s.majorants[i] = std::move(m);
    }
}
static inline F3 vol_sigma_t(const pt_volume &v) {
    return F3(v.sigma_a[0] + v.sigma_s[0], v.sigma_a[1] + v.sigma_s[1], v.sigma_a[2] + v.sigma_s[2]);
}
static inline float vol_sigma_t_max(const pt_volume &v) {
    F3 s = vol_sigma_t(v);
    return std::max(s.x, std::max(s.y, s.z));
}
static bool ray_aabb(F3 o, F3 d, F3 bmin, F3 bmax, float &tn, float &tf) {  // Volume.hlsl:15-27
    F3 inv(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    F3 t0 = (bmin - o) * inv, t1 = (bmax - o) * inv;
    F3 a = vmin(t0, t1), b = vmax(t0, t1);
    tn = std::max(std::max(a.x, a.y), a.z);
    tf = std::min(std::min(b.x, b.y), b.z);
    return tf >= std::max(tn, 0.0f);
}
// Trilinear fetch with the reference's s2 sampler (clamp in u, v, w).
static float grid_trilinear(const Grid &g, float u, float v, float w) {
    float x = u * g.w - 0.5f, y = v * g.h - 0.5f, z = w * g.d - 0.5f;
    float fx0 = std::floor(x), fy0 = std::floor(y), fz0 = std::floor(z);
    float fx = x - fx0, fy = y - fy0, fz = z - fz0;
    int x0 = (int)fx0, y0 = (int)fy0, z0 = (int)fz0;
    auto c = [](int a, int n) { return std::min(std::max(a, 0), n - 1); };
    int xa = c(x0, g.w), xb = c(x0 + 1, g.w), ya = c(y0, g.h), yb = c(y0 + 1, g.h), za = c(z0, g.d), zb = c(z0 + 1, g.d);
    auto at = [&](int xx, int yy, int zz) { return g.v[(size_t)xx + (size_t)g.w * (yy + (size_t)g.h * zz)]; };
    float c00 = at(xa, ya, za) * (1 - fx) + at(xb, ya, za) * fx;
    float c10 = at(xa, yb, za) * (1 - fx) + at(xb, yb, za) * fx;
    float c01 = at(xa, ya, zb) * (1 - fx) + at(xb, ya, zb) * fx;
    float c11 = at(xa, yb, zb) * (1 - fx) + at(xb, yb, zb) * fx;
    float c0 = c00 * (1 - fy) + c10 * fy, c1 = c01 * (1 - fy) + c11 * fy;
    return c0 * (1 - fz) + c1 * fz;
}
static float vol_density(const Scene &s, const pt_volume &v, F3 p) {  // Volume.hlsl:98-105
    if (!(v.flags & PT_VOLUME_HETEROGENEOUS) || v.density_grid == PT_NO_TEXTURE) return 1.0f;
    F3 vmn(v.vmin[0], v.vmin[1], v.vmin[2]), vmx(v.vmax[0], v.vmax[1], v.vmax[2]);
    F3 uvw = (p - vmn) / vmax(vmx - vmn, F3(1e-6f));
    return grid_trilinear(s.grids[v.density_grid], uvw.x, uvw.y, uvw.z);
}
static void local_majorant(const Scene &s, uint32_t vi, F3 pos, F3 dir, float &mu, float &bd) {  // Volume.hlsl:119-164
    const pt_volume &v = s.vols[vi];
    float gmu = vol_sigma_t_max(v);
    const Grid &m = s.majorants[vi];
    if (m.w == 0) { mu = gmu; bd = 1e20f; return; }
    F3 mres((float)m.w, (float)m.h, (float)m.d);
    F3 vmn(v.vmin[0], v.vmin[1], v.vmin[2]), vmx(v.vmax[0], v.vmax[1], v.vmax[2]);
    F3 size = vmax(vmx - vmn, F3(1e-6f));
    F3 bws = size / mres;
    F3 nc = (pos - vmn) / size;
    F3 bf = nc * mres;
    int bc[3];
    int res[3] = {(int)m.w, (int)m.h, (int)m.d};
    for (int i = 0; i < 3; i++) bc[i] = std::min(std::max((int)bf[i], 0), res[i] - 1);
    float dbm = m.v[(size_t)bc[0] + (size_t)m.w * (bc[1] + (size_t)m.h * bc[2])];
    mu = dbm * gmu;
    float dv[3];
    for (int i = 0; i < 3; i++) {
        if (std::fabs(dir[i]) < 1e-20f) dv[i] = 1e20f;
        else {
            float ne = (float)bc[i] + (dir[i] > 0.0f ? 1.0f : 0.0f);
            float we = vmn[i] + ne * bws[i];
            float dd = (we - pos[i]) / dir[i];
            dv[i] = std::max(dd, 1e-5f);
        }
    }
    bd = std::min(dv[0], std::min(dv[1], dv[2]));
}
struct Seg { uint32_t vi; float tn, tf; };
static uint32_t enumerate_segments(const Scene &s, F3 o, F3 d, float tmax, Seg segs[8]) {  // Volume.hlsl:186-215
    uint32_t count = 0;
    for (uint32_t i = 0; i < s.vols.size() && count < 8; i++) {
        const pt_volume &v = s.vols[i];
        float tn, tf;
        if (!ray_aabb(o, d, F3(v.vmin[0], v.vmin[1], v.vmin[2]), F3(v.vmax[0], v.vmax[1], v.vmax[2]), tn, tf)) continue;
        tn = std::max(tn, 0.0f);
        tf = std::min(tf, tmax);
        if (tf <= tn) continue;
        uint32_t p = count;
        for (; p > 0; p--) {
            if (segs[p - 1].tn <= tn) break;
            segs[p] = segs[p - 1];
        }
        segs[p] = {i, tn, tf};
        count++;
    }
    return count;
}
static bool null_collision(const Scene &s, uint32_t vi, F3 o, F3 d, float tn, float tf, Rng &rng, F3 &w, float &ts) {  // Volume.hlsl:236-319
    const pt_volume &v = s.vols[vi];
    float gmu = vol_sigma_t_max(v);
    F3 stv = vol_sigma_t(v);
    float t = tn;
    for (uint32_t step = 0; step < 512; step++) {
        F3 pos = o + d * t;
        float lmu, bd;
        local_majorant(s, vi, pos, d, lmu, bd);
        if (lmu < 1e-8f) {
            t += bd;
            if (t >= tf) { ts = tf; return false; }
            continue;
        }
        float xi = std::max(next_float(rng), 1e-10f);
        float dt = -std::log(xi) / lmu;
        if (dt > bd) {
            t += bd;
            if (t >= tf) { ts = tf; return false; }
            continue;
        }
        t += dt;
        if (t >= tf) { ts = tf; return false; }
        F3 np = o + d * t;
        float dens = vol_density(s, v, np);
        float pr = saturate((dens * gmu) / std::max(lmu, 1e-20f));
        if (pr >= 1.0f - 1e-6f || next_float(rng) < pr) {
            w = w * (stv / std::max(gmu, 1e-20f));
            ts = t;
            return true;
        }
        F3 sn = lmu - dens * stv;
        float den = std::max(lmu * (1.0f - pr), 1e-20f);
        w = w * (sn / den);
    }
    ts = tf;
    return false;
}
static F3 ratio_tracking(const Scene &s, uint32_t vi, F3 o, F3 d, float tn, float tf, Rng &rng) {  // Volume.hlsl:326-372
    const pt_volume &v = s.vols[vi];
    F3 stv = vol_sigma_t(v);
    F3 tr(1.0f);
    float t = tn;
    for (uint32_t step = 0; step < 512; step++) {
        F3 pos = o + d * t;
        float lmu, bd;
        local_majorant(s, vi, pos, d, lmu, bd);
        if (lmu < 1e-8f) {
            t += bd;
            if (t >= tf) return tr;
            continue;
        }
        float xi = std::max(next_float(rng), 1e-10f);
        float dt = -std::log(xi) / lmu;
        if (dt > bd) {
            t += bd;
            if (t >= tf) return tr;
            continue;
        }
        t += dt;
        if (t >= tf) return tr;
        F3 np = o + d * t;
        float dens = vol_density(s, v, np);
        F3 sn = lmu - dens * stv;
        tr = tr * (sn / std::max(lmu, 1e-20f));
        if (std::max(tr.x, std::max(tr.y, tr.z)) < 1e-6f) return F3(0.0f);
    }
    return tr;
}
static bool sample_free_flight(const Scene &s, F3 o, F3 d, float tmax, Rng &rng, F3 &w, float &ts, uint32_t &svi) {  // Volume.hlsl:381-415
    ts = tmax;
    svi = 0;
    if (s.vols.empty()) return false;
    Seg segs[8];
    uint32_t c = enumerate_segments(s, o, d, tmax, segs);
    for (uint32_t k = 0; k < c; k++) {
        const pt_volume &v = s.vols[segs[k].vi];
        if (vol_sigma_t_max(v) < 1e-8f) continue;
        float th;
        if (null_collision(s, segs[k].vi, o, d, segs[k].tn, segs[k].tf, rng, w, th)) {
            ts = th;
            svi = segs[k].vi;
            return true;
        }
    }
    return false;
}
static F3 multi_volume_tr(const Scene &s, F3 o, F3 d, float tmax, Rng &rng) {  // Volume.hlsl:419-454
    if (s.vols.empty()) return F3(1.0f);
    Seg segs[8];
    uint32_t c = enumerate_segments(s, o, d, tmax, segs);
    F3 tr(1.0f);
    for (uint32_t k = 0; k < c; k++) {
        const pt_volume &v = s.vols[segs[k].vi];
        F3 st = vol_sigma_t(v);
        if (std::max(st.x, std::max(st.y, st.z)) < 1e-8f) continue;
        F3 seg;
        if (v.flags & PT_VOLUME_HETEROGENEOUS) seg = ratio_tracking(s, segs[k].vi, o, d, segs[k].tn, segs[k].tf, rng);
        else seg = vexp(-st * (segs[k].tf - segs[k].tn));
        tr = tr * seg;
        if (std::max(tr.x, std::max(tr.y, tr.z)) < 1e-6f) return F3(0.0f);
    }
    return tr;
}

// ---------------------------------------------------------------------------
// Emitters / NEE (shaders/Emitter.hlsli:17-434)
// ---------------------------------------------------------------------------
struct EmitterSample { F3 pos, nrm, rad; float pdfArea; uint32_t id; bool valid; };
static EmitterSample sample_emitter(const Scene &s, Rng &rng) {  // Emitter.hlsli:43-89
    EmitterSample es{};
    es.valid = false;
    if (s.emitterCount == 0) return es;
    uint32_t pick = std::min((uint32_t)(next_float(rng) * float(s.emitterCount)), s.emitterCount - 1);
    es.id = s.emitterList[pick];
    es.valid = true;
    const pt_material &m = s.mats[es.id];
    es.rad = F3(m.radiance[0], m.radiance[1], m.radiance[2]);
    uint32_t nt = m.indexCount / 3;
    float u = next_float(rng);
    uint32_t tri = std::min(cdf_search(&s.emitterCdf[m.emitterCdfOffset], nt + 1, u), nt - 1);
    uint32_t i0, i1, i2;
    tri_idx(s, es.id, tri, i0, i1, i2);
    F3 p0 = ld3(s.pos, i0), p1 = ld3(s.pos, i1), p2 = ld3(s.pos, i2);
    float r1 = next_float(rng), r2 = next_float(rng);
    float sr1 = std::sqrt(r1);
    es.pos = (1.0f - sr1) * p0 + sr1 * (1.0f - r2) * p1 + sr1 * r2 * p2;
    es.nrm = normalize(cross(p1 - p0, p2 - p0));
    es.pdfArea = 1.0f / (m.surfaceArea * float(s.emitterCount));
    return es;
}
static float emitter_pdf_sa(const Scene &s, const pt_material &m, F3 hp, F3 sp, F3 n) {  // Emitter.hlsli:91-103
    F3 d = hp - sp;
    float d2 = dot(d, d);
    if (d2 < 1e-12f) return 0.0f;
    float dist = std::sqrt(d2);
    float cl = std::fabs(dot(n, -d / dist));
    if (cl < 1e-8f) return 0.0f;
    return (1.0f / (m.surfaceArea * float(s.emitterCount))) * d2 / cl;
}

struct Ctx { const Scene *s; uint32_t envMode; };
static inline void env_sample(const Ctx &c, float u1, float u2, F3 &dir, F3 &rad, float &pdf) {
    if (c.envMode == PT_ENV_ALIAS) sample_env_alias(*c.s, u1, u2, dir, rad, pdf);
    else sample_env_cdf(*c.s, u1, u2, dir, rad, pdf);
}
static inline float env_pdf(const Ctx &c, F3 d) {
    return c.envMode == PT_ENV_ALIAS ? env_pdf_alias(*c.s, d) : env_pdf_cdf(*c.s, d);
}

static F3 mis_direct(const Ctx &c, F3 hp, F3 N, F3 Ng, F3 T, F3 B, F3 wil, const Mat<float> &m, float h, Rng &rng,
                     uint32_t aseed, uint32_t bounce) {  // Emitter.hlsli:105-153
    const Scene &s = *c.s;
    EmitterSample es = sample_emitter(s, rng);
    if (!es.valid) return F3(0.0f);
    F3 tl = es.pos - hp;
    float dist = length(tl);
    F3 ww = tl / dist;
    float ct = dot(N, ww), cl = dot(es.nrm, -ww);
    bool hair = m.type == PT_MAT_HAIR;
    if ((!hair && ct <= 0.0f) || cl <= 0.0f) return F3(0.0f);
    float act = hair ? std::fabs(ct) : ct;
    F3 sng = hair ? (dot(ww, Ng) >= 0.0f ? Ng : -Ng) : Ng;
    F3 so = offset_ray_origin(hp, sng, sng);
    F3 trans;
    if (trace_shadow(s, so, ww, 0.0f, dist - 0.001f, trans, aseed, alpha_key(bounce, 1u))) return F3(0.0f);
    F3 wol = to_local(ww, T, B, N);
    F3 f = material_eval(wil, wol, m, h);
    float pb = material_pdf(wil, wol, m, h);
    float pe = es.pdfArea * dist * dist / cl;
    float w = balance_heuristic(pe, pb);
    F3 vt = multi_volume_tr(s, so, ww, dist, rng);
    return es.rad * f * act / std::max(pe, 1e-20f) * w * vt * trans;
}
// EvalLightCandidate (Emitter.hlsli:166-199): unshadowed integrand, scalar
// target pHat = lum(f Le cos) and the solid-angle pdf of the emitter sample.
static bool ris_candidate(const EmitterSample &es, F3 hp, F3 N, F3 T, F3 B, F3 wil, const Mat<float> &m, float h,
                          F3 &wiw, float &dist, F3 &integ, float &pHat, float &pSA) {
    integ = F3(0.0f);
    pHat = 0.0f;
    pSA = 0.0f;
    F3 toLight = es.pos - hp;
    dist = length(toLight);
    if (dist < 1e-6f) {
        wiw = F3(0.0f, 0.0f, 1.0f);
        return false;
    }
    wiw = toLight / dist;
    float cosSurface = dot(N, wiw), cosLight = dot(es.nrm, -wiw);
    bool hair = m.type == PT_MAT_HAIR;
    if ((!hair && cosSurface <= 0.0f) || cosLight <= 1e-8f) return false;
    float absCos = hair ? std::fabs(cosSurface) : cosSurface;
    F3 f = material_eval(wil, to_local(wiw, T, B, N), m, h);
    integ = f * es.rad * absCos;
    pHat = dot(integ, F3(0.2126f, 0.7152f, 0.0722f));
    pSA = es.pdfArea * dist * dist / cosLight;
    return pHat > 0.0f && pSA > 0.0f;
}
// RISDirectIllumination (Emitter.hlsli:201-271), RIS_M = 8 candidates streamed
// through a one-sample reservoir, the survivor shadow-tested and MIS-weighted
// against the BSDF with the candidate's solid-angle pdf.
static F3 ris_direct(const Ctx &c, F3 hp, F3 N, F3 Ng, F3 T, F3 B, F3 wil, const Mat<float> &m, float h, Rng &rng,
                     uint32_t aseed, uint32_t bounce) {
    const Scene &s = *c.s;
    EmitterSample y{};
    y.valid = false;
    float wSum = 0.0f, pHatY = 0.0f;
    for (int i = 0; i < 8; i++) {
        EmitterSample cnd = sample_emitter(s, rng);
        if (!cnd.valid) continue;
        F3 wiwC, integC;
        float distC, pHatC, pSAC;
        if (!ris_candidate(cnd, hp, N, T, B, wil, m, h, wiwC, distC, integC, pHatC, pSAC)) continue;
        float w = pHatC / pSAC;
        wSum += w;
        if (next_float(rng) < w / std::max(wSum, 1e-20f)) {
            y = cnd;
            pHatY = pHatC;
        }
    }
    if (!y.valid || pHatY <= 0.0f) return F3(0.0f);
    float W = (wSum / 8.0f) / pHatY;
    F3 wiw, integ;
    float dist, pHat, pSA;
    if (!ris_candidate(y, hp, N, T, B, wil, m, h, wiw, dist, integ, pHat, pSA)) return F3(0.0f);
    bool hair = m.type == PT_MAT_HAIR;
    F3 sng = hair ? (dot(wiw, Ng) >= 0.0f ? Ng : -Ng) : Ng;
    F3 so = offset_ray_origin(hp, sng, sng);
    F3 trans;
    if (trace_shadow(s, so, wiw, 0.0f, dist - 0.001f, trans, aseed, alpha_key(bounce, 1u))) return F3(0.0f);
    float pdfBsdf = material_pdf(wil, to_local(wiw, T, B, N), m, h);
    float wMis = balance_heuristic(pSA, pdfBsdf);
    F3 vt = multi_volume_tr(s, so, wiw, dist, rng);
    return integ * W * wMis * vt * trans;
}
static F3 env_direct(const Ctx &c, F3 hp, F3 N, F3 Ng, F3 T, F3 B, F3 wil, const Mat<float> &m, float h, Rng &rng,
                     uint32_t aseed, uint32_t bounce) {  // Emitter.hlsli:275-326
    const Scene &s = *c.s;
    float u1 = next_float(rng), u2 = next_float(rng);
    F3 ww, Le;
    float pe;
    env_sample(c, u1, u2, ww, Le, pe);
    if (pe <= 0.0f) return F3(0.0f);
    float ct = dot(N, ww);
    bool hair = m.type == PT_MAT_HAIR;
    if (!hair && ct <= 0.0f) return F3(0.0f);
    float act = hair ? std::fabs(ct) : ct;
    F3 sng = hair ? (dot(ww, Ng) >= 0.0f ? Ng : -Ng) : Ng;
    F3 so = offset_ray_origin(hp, sng, sng);
    F3 trans;
    if (trace_shadow(s, so, ww, 0.0f, 1e20f, trans, aseed, alpha_key(bounce, 2u))) return F3(0.0f);
    F3 wol = to_local(ww, T, B, N);
    F3 f = material_eval(wil, wol, m, h);
    float pb = material_pdf(wil, wol, m, h);
    float w = balance_heuristic(pe, pb);
    F3 vt = multi_volume_tr(s, so, ww, 1e20f, rng);
    return Le * f * act / std::max(pe, 1e-20f) * w * vt * trans;
}
static bool vol_nee_skip(const pt_volume &v, F3 p) {
    F3 st = vol_sigma_t(v);
    float smin = std::min(st.x, std::min(st.y, st.z));
    F3 dmn = p - F3(v.vmin[0], v.vmin[1], v.vmin[2]);
    F3 dmx = F3(v.vmax[0], v.vmax[1], v.vmax[2]) - p;
    float md = std::min(std::min(dmn.x, dmn.y), std::min(dmn.z, std::min(dmx.x, std::min(dmx.y, dmx.z))));
    return md * smin > 8.0f;
}
static F3 vol_nee_area(const Ctx &c, F3 sp, F3 wo, uint32_t vi, Rng &rng, uint32_t aseed, uint32_t bounce) {  // Emitter.hlsli:334-390
    const Scene &s = *c.s;
    const pt_volume &v = s.vols[vi];
    if (vol_nee_skip(v, sp)) return F3(0.0f);
    EmitterSample es = sample_emitter(s, rng);
    if (!es.valid) return F3(0.0f);
    F3 tl = es.pos - sp;
    float dist = length(tl);
    F3 wi = tl / dist;
    float cl = dot(es.nrm, -wi);
    if (cl <= 0.0f) return F3(0.0f);
    F3 trans;
    if (trace_shadow(s, sp, wi, 0.001f, dist - 0.001f, trans, aseed, alpha_key(bounce, 1u))) return F3(0.0f);
    float fp = hg(dot(wo, wi), v.phase_g);
    float pe = es.pdfArea * dist * dist / cl;
    float w = balance_heuristic(pe, fp);
    F3 vt = multi_volume_tr(s, sp, wi, dist, rng);
    return es.rad * fp / std::max(pe, 1e-20f) * w * vt * trans;
}
static F3 vol_nee_env(const Ctx &c, F3 sp, F3 wo, uint32_t vi, Rng &rng, uint32_t aseed, uint32_t bounce) {  // Emitter.hlsli:392-434
    const Scene &s = *c.s;
    const pt_volume &v = s.vols[vi];
    if (vol_nee_skip(v, sp)) return F3(0.0f);
    float u1 = next_float(rng), u2 = next_float(rng);
    F3 wi, Le;
    float pe;
    env_sample(c, u1, u2, wi, Le, pe);
    if (pe <= 0.0f) return F3(0.0f);
    F3 trans;
    if (trace_shadow(s, sp, wi, 0.001f, 1e20f, trans, aseed, alpha_key(bounce, 2u))) return F3(0.0f);
    float fp = hg(dot(wo, wi), v.phase_g);
    float w = balance_heuristic(pe, fp);
    F3 vt = multi_volume_tr(s, sp, wi, 1e20f, rng);
    return Le * fp / std::max(pe, 1e-20f) * w * vt * trans;
}

// Draw k uniforms from the path's sampler, in order.
static inline void draw(Rng &rng, float *u, int k) { for (int i = 0; i < k; i++) u[i] = next_float(rng); }

// ---------------------------------------------------------------------------
// SubsurfaceWalk (shaders/Subsurface.hlsli:49-144): random walk inside the
// closed mesh `mesh` from pos along dir; scalar extinction sigmaT, per-channel
// albedo alpha, HG phase g, Fresnel at the boundary (reflect back or leave),
// Russian roulette after 5 steps, at most 256 steps.  Returns true with the
// exit point, direction, outward normal and throughput factor; a hit on other
// geometry or an absorbed walk returns false.  Interior rays take the alpha
// test with key kind 3.
// ---------------------------------------------------------------------------
static bool subsurface_walk(const Scene &s, F3 pos, F3 dir, uint32_t mesh, float sigmaT, F3 alpha, float g,
                            float intIOR, float extIOR, Rng &rng, uint32_t aseed, uint32_t bounce, F3 &exitPos,
                            F3 &exitDir, F3 &exitN, F3 &tmul) {
    tmul = F3(1.0f);
    exitPos = pos;
    exitDir = dir;
    exitN = dir;
    for (int step = 0; step < 256; step++) {
        float d = sigmaT > 0.0f ? -std::log(std::max(next_float(rng), 1e-10f)) / sigmaT : 1e30f;
        Hit p = trace_closest(s, pos, dir, 1e-4f, d, aseed, alpha_key(bounce, 3u));
        if (p.hit && p.t < d) {
            if (p.mesh != mesh) {
                tmul = F3(0.0f);
                return false;
            }
            F3 bPos = pos + dir * p.t;
            F3 Nb = normalize(interp_normal(s, p.mesh, p.prim, p.u, p.v));
            if (dot(Nb, dir) < 0.0f) Nb = -Nb;
            float cosI = dot(dir, Nb);
            float Fr = fresnel_dielectric(cosI, intIOR, extIOR);
            if (next_float(rng) < Fr) {
                dir = normalize(reflect(dir, Nb));
                pos = bPos - Nb * 1e-4f;
                continue;
            }
            F3 outDir = refract(dir, -Nb, intIOR / extIOR);
            if (dot(outDir, outDir) < 1e-8f) {
                dir = normalize(reflect(dir, Nb));
                pos = bPos - Nb * 1e-4f;
                continue;
            }
            exitPos = bPos;
            exitDir = normalize(outDir);
            exitN = Nb;
            return true;
        }
        pos = pos + dir * d;
        tmul *= alpha;
        float x1 = next_float(rng), x2 = next_float(rng), pp;
        dir = sample_hg(dir, g, x1, x2, pp);
        if (step > 4) {
            float q = std::min(std::max(std::max(tmul.x, std::max(tmul.y, tmul.z)), 0.05f), 0.95f);
            if (next_float(rng) >= q) {
                tmul = F3(0.0f);
                return false;
            }
            tmul = tmul / q;
        }
    }
    tmul = F3(0.0f);
    return false;
}

// ---------------------------------------------------------------------------
// The path (shaders/Shaders.hlsl:25-651, RayGen), one camera sample.
// ---------------------------------------------------------------------------
struct PathStats { uint64_t ext = 0, shadow = 0; };
// Radiance-cache termination with a cache that returns the constant `value`
// (the library's rule: a path ends at the first non-emitting surface vertex
// reached by a rough bounce and adds throughput x cache there).  Used to
// check the library's termination logic independently of its network.
struct CacheConst { float value[3]; float roughThr; };
static F3 trace_path(const Ctx &c, const pt_render_params &P, uint32_t px, uint32_t py, uint32_t frame, PathStats *st,
                     const CacheConst *cc = nullptr) {
    const Scene &s = *c.s;
    const pt_camera &cam = P.camera;
    Rng rng = init_rng(px, py, P.width, P.height, frame, P.rng_kind);
    float jx = next_float(rng), jy = next_float(rng);
    float ux = ((float)px + jx) / (float)P.width;
    float uy = ((float)py + jy) / (float)P.height;
    uy = 1.0f - uy;
    F3 cpos(cam.pos[0], cam.pos[1], cam.pos[2]);
    F3 llc(cam.llc[0], cam.llc[1], cam.llc[2]);
    F3 hor(cam.horizontal[0], cam.horizontal[1], cam.horizontal[2]);
    F3 ver(cam.vertical[0], cam.vertical[1], cam.vertical[2]);
    F3 dir = normalize(llc + ux * hor + uy * ver - cpos);
    F3 ro = cpos, rd = dir;
    float tmin = 0.001f, tmax = 1e20f;
    if (cam.lens_radius > 0.0f) {  // Shaders.hlsl:68-92
        F3 fwd = normalize(llc + 0.5f * hor + 0.5f * ver - cpos);
        F3 right = normalize(hor), up = normalize(ver);
        float ft = cam.focal_distance / dot(dir, fwd);
        F3 fp = cpos + dir * ft;
        float u1 = next_float(rng), u2 = next_float(rng);
        float r = std::sqrt(u1) * cam.lens_radius;
        float th = 2.0f * kPi<float> * u2;
        F3 lo = (r * std::cos(th)) * right + (r * std::sin(th)) * up;
        ro = cpos + lo;
        rd = normalize(fp - ro);
    }
    F3 Lo(0.0f), thr(1.0f);
    float lastPdf = 0.0f, eta = 1.0f;
    bool rough = false;  // the last bounce was rough (radiance-cache termination)
    const uint32_t aseed = s.hasAlpha ? alpha_seed(rng.pixelSeed, rng.sampleIndex) : 0u;
    for (int bounce = 0; bounce < (int)P.max_depth; bounce++) {
        Hit hit = trace_closest(s, ro, rd, tmin, tmax, aseed, alpha_key((uint32_t)bounce, 0u));
        if (st) st->ext++;
        bool volScat = false;
        if (!s.vols.empty()) {  // Shaders.hlsl:133-179
            float tSurf = hit.hit ? hit.t : 1e20f;
            float tsc;
            uint32_t svi;
            F3 vw(1.0f);
            bool sc = sample_free_flight(s, ro, rd, tSurf, rng, vw, tsc, svi);
            thr *= vw;
            if (sc) {
                volScat = true;
                const pt_volume &v = s.vols[svi];
                F3 sst = vol_sigma_t(v);
                F3 spos = ro + tsc * rd;
                thr *= F3(v.sigma_s[0], v.sigma_s[1], v.sigma_s[2]) / vmax(sst, F3(1e-20f));
                Lo += thr * vol_nee_area(c, spos, rd, svi, rng, aseed, (uint32_t)bounce);
                Lo += thr * vol_nee_env(c, spos, rd, svi, rng, aseed, (uint32_t)bounce);
                float x1 = next_float(rng), x2 = next_float(rng);
                float pp;
                F3 nd = sample_hg(rd, v.phase_g, x1, x2, pp);
                ro = spos; rd = nd; tmin = 0.0f; tmax = 1e20f;
                lastPdf = std::max(pp, 1e-20f);
                rough = true;
            }
        }
        if (volScat) {
        } else if (!hit.hit) {  // Shaders.hlsl:188-212
            F3 env = eval_env(s, rd);
            if (lastPdf == 0.0f) Lo += thr * env;
            else {
                float pe = env_pdf(c, rd);
                float w = balance_heuristic(lastPdf, pe);
                Lo += thr * env * w;
            }
            break;
        } else {
            F3 hp = ro + rd * hit.t;
            F3 N = normalize(interp_normal(s, hit.mesh, hit.prim, hit.u, hit.v));
            F3 Ng = normalize(geometric_normal(s, hit.mesh, hit.prim));
            pt_material pm = s.mats[hit.mesh];
            float hu, hv;
            interp_uv(s, hit.mesh, hit.prim, hit.u, hit.v, hu, hv);
            bool back = dot(Ng, rd) > 0.0f;
            if (back) Ng = -Ng;
            if (dot(N, Ng) < 0.0f) N = -N;
            if (has_shading_textures(pm)) apply_textures(s, pm, hit.mesh, hit.prim, hit.t, hit.u, hit.v, N, P.width, P.height);
            Mat<float> m = Mat<float>::from(pm);
            if (pm.isEmitter) {  // Shaders.hlsl:317-335
                F3 rad(pm.radiance[0], pm.radiance[1], pm.radiance[2]);
                if (lastPdf == 0.0f) Lo += thr * rad;
                else {
                    float pe = emitter_pdf_sa(s, pm, hp, ro, N);
                    Lo += thr * rad * balance_heuristic(lastPdf, pe);
                }
                break;
            }
            if (cc && rough) {
                Lo += thr * F3(cc->value[0], cc->value[1], cc->value[2]);
                break;
            }
            F3 T, B;
            float h = 0.0f;
            if (pm.type == PT_MAT_HAIR) {  // Shaders.hlsl:340-387
                F3 ht = interp_tangent(s, hit.mesh, hit.prim, hit.u, hit.v);
                if (dot(ht, ht) > 1e-8f) {
                    ht = normalize(ht);
                    h = hv * 2.0f - 1.0f;
                } else {
                    uint32_t i0, i1, i2;
                    tri_idx(s, hit.mesh, hit.prim, i0, i1, i2);
                    F3 p0 = ld3(s.pos, i0), p1 = ld3(s.pos, i1), p2 = ld3(s.pos, i2);
                    float a0u = s.uv[2 * i0], a0v = s.uv[2 * i0 + 1], a1u = s.uv[2 * i1], a1v = s.uv[2 * i1 + 1],
                          a2u = s.uv[2 * i2], a2v = s.uv[2 * i2 + 1];
                    F3 e1 = p1 - p0, e2 = p2 - p0;
                    float d1u = a1u - a0u, d1v = a1v - a0v, d2u = a2u - a0u, d2v = a2v - a0v;
                    float det = d1u * d2v - d2u * d1v;
                    if (std::fabs(det) > 1e-8f) {
                        float id = 1.0f / det;
                        ht = normalize((-d1u * e1 + d2u * e2) * id);
                    } else {
                        build_onb(N, ht, B);
                    }
                    h = hu * 2.0f - 1.0f;
                }
                T = normalize(ht - N * dot(ht, N));
                B = cross(N, T);
            } else {
                build_onb(N, T, B);
                h = 0.0f;
            }
            {  // terminator bend, Shaders.hlsl:402-411
                F3 V = -rd;
                float ndv = dot(N, V);
                if (ndv <= 0.0f && dot(V, Ng) > 0.0f) {
                    N = normalize(N + V * (1e-3f - ndv));
                    build_onb(N, T, B);
                }
            }
            F3 wil = to_local(-rd, T, B, N);
            if (pm.type == PT_MAT_MIRROR) {  // Shaders.hlsl:419-427
                F3 rf = reflect(rd, N);
                ro = hp + Ng * 0.001f; rd = rf; tmin = 0.0f; tmax = 1e20f;
                lastPdf = 0.0f;
                rough = false;
            } else if (pm.type == PT_MAT_DIELECTRIC) {  // Shaders.hlsl:429-472
                F3 I = rd, Nf = N;
                float etaI, etaT;
                if (!back) { etaI = pm.extIOR; etaT = pm.intIOR; }
                else { etaI = pm.intIOR; etaT = pm.extIOR; }
                float cosI = dot(-I, Nf);
                float Fr = fresnel_dielectric(cosI, etaI, etaT);
                F3 nd;
                bool refr = false;
                float rv = next_float(rng);
                if (rv < Fr) nd = reflect(I, Nf);
                else {
                    nd = refract(I, Nf, etaI / etaT);
                    if (dot(nd, nd) < 0.001f) nd = reflect(I, Nf);
                    else refr = true;
                }
                F3 on = dot(nd, Ng) > 0.0f ? Ng : -Ng;
                ro = hp + on * 0.001f; rd = nd; tmin = 0.0f; tmax = 1e20f;
                lastPdf = 0.0f;
                if (refr) eta *= etaI / etaT;
                rough = false;
            } else if (pm.type == PT_MAT_DIFFUSE || pm.type == PT_MAT_MICROFACET || pm.type == PT_MAT_DISNEY ||
                       pm.type == PT_MAT_HAIR) {  // Shaders.hlsl:473-511
                if (P.flags & PT_RENDER_RIS_NEE) Lo += thr * ris_direct(c, hp, N, Ng, T, B, wil, m, h, rng, aseed, (uint32_t)bounce);
                else Lo += thr * mis_direct(c, hp, N, Ng, T, B, wil, m, h, rng, aseed, (uint32_t)bounce);
                if (st && s.emitterCount) st->shadow++;
                Lo += thr * env_direct(c, hp, N, Ng, T, B, wil, m, h, rng, aseed, (uint32_t)bounce);
                if (st) st->shadow++;
                float u[4];
                int k = (pm.type == PT_MAT_DIFFUSE || pm.type == PT_MAT_MICROFACET) ? 2 : (pm.type == PT_MAT_DISNEY ? 3 : 4);
                // MaterialSample returns before drawing when wi.z <= 0 (all but hair)
                if (pm.type != PT_MAT_HAIR && wil.z <= 0.0f) k = 0;
                draw(rng, u, k);
                F3 wol;
                float bp;
                int used;
                F3 wt = material_sample(wil, u, m, h, wol, bp, &used);
                if (bp <= 0.0f || (wt.x == 0.0f && wt.y == 0.0f && wt.z == 0.0f)) break;
                F3 ww = to_world(wol, T, B, N);
                F3 on = pm.type == PT_MAT_HAIR ? (dot(ww, Ng) >= 0.0f ? Ng : -Ng) : Ng;
                ro = offset_ray_origin(hp, on, on); rd = ww; tmin = 0.0f; tmax = 1e20f;
                thr *= wt;
                lastPdf = std::max(bp, 1e-20f);
                if (cc)
                    rough = pm.type == PT_MAT_DIFFUSE || pm.type == PT_MAT_HAIR ||
                            (pm.type == PT_MAT_MICROFACET && pm.alpha >= cc->roughThr) ||
                            (pm.type == PT_MAT_DISNEY && pm.roughness >= cc->roughThr);
            } else if (pm.type == PT_MAT_SUBSURFACE) {  // Shaders.hlsl:515-611
                F3 I = rd;
                m.roughness = m.roughness * (1.0f + std::min(std::max(m.specular * 2.0f, 0.0f), 1.0f) * (0.65f - 1.0f));
                const float rough = m.roughness;
                const float aR = std::max(rough * rough, 1e-4f);
                F3 wiL = to_local(-I, T, B, N);
                F3 wmL(0.0f, 0.0f, 1.0f);
                if (rough > 1e-3f) {
                    float u0 = next_float(rng), u1 = next_float(rng);
                    wmL = beckmann_sample(u0, u1, aR);
                }
                F3 wm = normalize(to_world(wmL, T, B, N));
                float cosThetaM = dot(-I, wm);
                if (cosThetaM <= 0.0f) {
                    wm = N;
                    wmL = F3(0.0f, 0.0f, 1.0f);
                    cosThetaM = dot(-I, N);
                }
                float G1i = rough > 1e-3f ? smith_g1(wiL, wmL, aR) : 1.0f;
                float Fr = fresnel_dielectric(cosThetaM, m.extIOR, m.intIOR);
                Lo += thr * mis_direct(c, hp, N, Ng, T, B, wil, m, h, rng, aseed, (uint32_t)bounce);
                if (st && s.emitterCount) st->shadow++;
                Lo += thr * env_direct(c, hp, N, Ng, T, B, wil, m, h, rng, aseed, (uint32_t)bounce);
                if (st) st->shadow++;
                if (next_float(rng) < Fr) {
                    F3 refl = reflect(I, wm);
                    F3 woL = to_local(refl, T, B, N);
                    if (woL.z <= 0.0f) break;  // reflected below the surface
                    float weight = rough > 1e-3f
                                       ? G1i * smith_g1(woL, wmL, aR) * cosThetaM / std::max(wiL.z * wmL.z, 1e-6f)
                                       : 1.0f;
                    float pdfSpec = rough > 1e-3f ? Fr * beckmann_d_cos(wmL, aR) / std::max(4.0f * cosThetaM, 1e-6f)
                                                  : 0.0f;
                    ro = hp + Ng * 0.001f; rd = refl; tmin = 0.0f; tmax = 1e20f;
                    thr = thr * weight;
                    lastPdf = pdfSpec;
                } else {
                    F3 refr = refract(I, wm, m.extIOR / m.intIOR);
                    if (dot(refr, refr) < 1e-8f) {
                        ro = hp + Ng * 0.001f; rd = reflect(I, wm); tmin = 0.0f; tmax = 1e20f;
                        lastPdf = 0.0f;
                    } else {
                        F3 tint(pm.sheen, pm.sheenTint, pm.clearcoat);
                        F3 aSharp = m.albedo, aBlur = m.albedo, detail(1.0f);
                        if (pm.albedoTexIndex != PT_NO_TEXTURE) {  // albedo blurred 4 mip levels up
                            float foot = uv_footprint(s, hit.mesh, hit.prim, hit.t, P.width, P.height);
                            float tu, tv;
                            interp_uv(s, hit.mesh, hit.prim, hit.u, hit.v, tu, tv);
                            F4 cb = tex_sample(s, pm.albedoTexIndex, tu, tv, tex_lod(s, pm.albedoTexIndex, foot) + 4.0f);
                            aBlur = F3(cb.x, cb.y, cb.z);
                            F3 r = aSharp / vmax(aBlur, F3(1e-3f));
                            detail = F3(std::min(std::max(r.x, 0.5f), 2.0f), std::min(std::max(r.y, 0.5f), 2.0f),
                                        std::min(std::max(r.z, 0.5f), 2.0f));
                        }
                        F3 A = aBlur * tint, A2 = A * A, A3 = A2 * A;
                        float sigmaT = 1.0f / std::max(m.subsurface, 1e-4f);
                        F3 e = -5.09406f * A + 2.61188f * A2 - 4.31805f * A3;
                        F3 alb = F3(1.0f) - F3(std::exp(e.x), std::exp(e.y), std::exp(e.z));
                        F3 ep, ed, en, tm;
                        bool exited = subsurface_walk(s, hp - Ng * 0.001f, normalize(refr), hit.mesh, sigmaT, alb,
                                                      m.anisotropic, m.intIOR, m.extIOR, rng, aseed,
                                                      (uint32_t)bounce, ep, ed, en, tm);
                        if (!exited) break;
                        thr *= tm * detail;
                        ro = offset_ray_origin(ep, en, en); rd = ed; tmin = 0.0f; tmax = 1e20f;
                        lastPdf = 0.0f;
                    }
                }
            } else {
                break;
            }
        }
        if (bounce >= 3) {  // Shaders.hlsl:620-626
            float q = std::min(std::max(thr.x, std::max(thr.y, thr.z)) * eta * eta, 0.95f);
            if (next_float(rng) >= q) break;
            thr /= q;
        }
    }
    if (std::isnan(Lo.x) || std::isnan(Lo.y) || std::isnan(Lo.z) || std::isinf(Lo.x) || std::isinf(Lo.y) || std::isinf(Lo.z))
        Lo = F3(0.0f);
    return Lo;
}

}  // namespace oracle

// ===========================================================================
// extern "C" surface for the tests (ctypes)
// ===========================================================================
using namespace oracle;

extern "C" {

void *or_scene_create(const pt_scene_desc *d) {
    auto *s = new Scene();
    s->pos.assign(d->positions, d->positions + 3 * (size_t)d->num_vertices);
    s->nrm = d->normals ? std::vector<float>(d->normals, d->normals + 3 * (size_t)d->num_vertices)
                        : std::vector<float>(3 * (size_t)d->num_vertices, 0.0f);
    s->uv = d->texcoords ? std::vector<float>(d->texcoords, d->texcoords + 2 * (size_t)d->num_vertices)
                         : std::vector<float>(2 * (size_t)d->num_vertices, 0.0f);
    s->tan = d->tangents ? std::vector<float>(d->tangents, d->tangents + 3 * (size_t)d->num_vertices)
                         : std::vector<float>(3 * (size_t)d->num_vertices, 0.0f);
    s->idx.assign(d->indices, d->indices + d->num_indices);
    s->mats.assign(d->materials, d->materials + d->num_meshes);
    for (uint32_t m = 0; m < d->num_meshes; m++)
        for (uint32_t t = 0; t < s->mats[m].indexCount / 3; t++) { s->triMesh.push_back(m); s->triPrim.push_back(t); }
    build_emitters(*s);
    s->envW = d->env_width; s->envH = d->env_height;
    s->env.assign((size_t)s->envW * s->envH * 4, 0.0f);
    for (size_t i = 0; i < (size_t)s->envW * s->envH; i++)
        for (int c = 0; c < 3; c++) s->env[4 * i + c] = d->env_rgb[3 * i + c];
    s->envScale = d->env_scale;
    s->evComp = d->ev_compensation;
    build_env(*s);
    build_env_alias(*s);
    s->vols.assign(d->volumes, d->volumes + d->num_volumes);
    for (uint32_t g = 0; g < d->num_grids; g++) {
        Grid gr{d->grids[g].w, d->grids[g].h, d->grids[g].d, {}};
        gr.v.assign(d->grids[g].data, d->grids[g].data + (size_t)gr.w * gr.h * gr.d);
        s->grids.push_back(std::move(gr));
    }
    build_majorants(*s);
    build_textures(*s, d);
    build_bvh(*s);
    return s;
}
void or_scene_destroy(void *s) { delete static_cast<Scene *>(s); }

void or_scene_materials(void *sp, pt_material *out) {
    Scene *s = static_cast<Scene *>(sp);
    std::memcpy(out, s->mats.data(), s->mats.size() * sizeof(pt_material));
}
uint32_t or_scene_emitter_cdf(void *sp, float *out) {
    Scene *s = static_cast<Scene *>(sp);
    if (out) std::memcpy(out, s->emitterCdf.data(), s->emitterCdf.size() * sizeof(float));
    return (uint32_t)s->emitterCdf.size();
}
void or_env_cdf(void *sp, float *marg, float *cond) {
    Scene *s = static_cast<Scene *>(sp);
    std::memcpy(marg, s->marg.data(), s->marg.size() * 4);
    std::memcpy(cond, s->cond.data(), s->cond.size() * 4);
}
void or_env_sample(void *sp, uint32_t mode, const float *u, size_t n, float *dir, float *rad, float *pdf) {
    Scene *s = static_cast<Scene *>(sp);
    Ctx c{s, mode};
    for (size_t i = 0; i < n; i++) {
        F3 d, r;
        float p;
        env_sample(c, u[2 * i], u[2 * i + 1], d, r, p);
        dir[3 * i] = d.x; dir[3 * i + 1] = d.y; dir[3 * i + 2] = d.z;
        rad[3 * i] = r.x; rad[3 * i + 1] = r.y; rad[3 * i + 2] = r.z;
        pdf[i] = p;
    }
}
void or_env_pdf(void *sp, uint32_t mode, const float *dir, size_t n, float *pdf, float *rad) {
    Scene *s = static_cast<Scene *>(sp);
    Ctx c{s, mode};
    for (size_t i = 0; i < n; i++) {
        F3 d(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
        pdf[i] = env_pdf(c, d);
        if (rad) { F3 r = eval_env(*s, d); rad[3 * i] = r.x; rad[3 * i + 1] = r.y; rad[3 * i + 2] = r.z; }
    }
}

void or_rng_batch(uint32_t kind, const uint32_t *pix, const uint32_t *smp, size_t n, uint32_t dims, uint32_t w,
                  uint32_t h, float *out) {
    for (size_t i = 0; i < n; i++) {
        Rng r = init_rng(pix[i] % w, pix[i] / w, w, h, smp[i], kind);
        for (uint32_t d = 0; d < dims; d++) out[i * dims + d] = next_float(r);
    }
}

// precision: 0 = float32 (the shader arithmetic), 1 = float64
void or_bsdf_eval(int precision, const pt_material *mats, const uint32_t *mi, const float *wi, const float *wo,
                  const float *hh, size_t n, float *f, float *pdf) {
    for (size_t i = 0; i < n; i++) {
        const pt_material &pm = mats[mi ? mi[i] : 0];
        float h = hh ? hh[i] : 0.0f;
        if (precision == 1) {
            Mat<double> m = Mat<double>::from(pm);
            V3<double> a(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]), b(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
            V3<double> r = material_eval(a, b, m, (double)h);
            f[3 * i] = (float)r.x; f[3 * i + 1] = (float)r.y; f[3 * i + 2] = (float)r.z;
            pdf[i] = (float)material_pdf(a, b, m, (double)h);
        } else {
            Mat<float> m = Mat<float>::from(pm);
            F3 a(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]), b(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
            F3 r = material_eval(a, b, m, h);
            f[3 * i] = r.x; f[3 * i + 1] = r.y; f[3 * i + 2] = r.z;
            pdf[i] = material_pdf(a, b, m, h);
        }
    }
}
void or_bsdf_sample(int precision, const pt_material *mats, const uint32_t *mi, const float *wi, const float *u,
                    const float *hh, size_t n, float *wo, float *wt, float *pdf) {
    for (size_t i = 0; i < n; i++) {
        const pt_material &pm = mats[mi ? mi[i] : 0];
        float h = hh ? hh[i] : 0.0f;
        int used;
        if (precision == 1) {
            Mat<double> m = Mat<double>::from(pm);
            V3<double> a(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]), o;
            double uu[4] = {u[4 * i], u[4 * i + 1], u[4 * i + 2], u[4 * i + 3]};
            double p;
            bool delta = pm.type == PT_MAT_MIRROR || pm.type == PT_MAT_DIELECTRIC;
            V3<double> r = delta ? delta_sample(a, m, uu[0], o, p) : material_sample(a, uu, m, (double)h, o, p, &used);
            wo[3 * i] = (float)o.x; wo[3 * i + 1] = (float)o.y; wo[3 * i + 2] = (float)o.z;
            wt[3 * i] = (float)r.x; wt[3 * i + 1] = (float)r.y; wt[3 * i + 2] = (float)r.z;
            pdf[i] = (float)p;
        } else {
            Mat<float> m = Mat<float>::from(pm);
            F3 a(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]), o;
            float p;
            bool delta = pm.type == PT_MAT_MIRROR || pm.type == PT_MAT_DIELECTRIC;
            F3 r = delta ? delta_sample(a, m, u[4 * i], o, p) : material_sample(a, &u[4 * i], m, h, o, p, &used);
            wo[3 * i] = o.x; wo[3 * i + 1] = o.y; wo[3 * i + 2] = o.z;
            wt[3 * i] = r.x; wt[3 * i + 1] = r.y; wt[3 * i + 2] = r.z;
            pdf[i] = p;
        }
    }
}
void or_phase_sample(int precision, const float *g, const float *wo, const float *u, size_t n, float *wi, float *pdf) {
    for (size_t i = 0; i < n; i++) {
        if (precision == 1) {
            V3<double> w(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
            double p;
            V3<double> r = sample_hg(w, (double)g[i], (double)u[2 * i], (double)u[2 * i + 1], p);
            wi[3 * i] = (float)r.x; wi[3 * i + 1] = (float)r.y; wi[3 * i + 2] = (float)r.z;
            pdf[i] = (float)p;
        } else {
            F3 w(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
            float p;
            F3 r = sample_hg(w, g[i], u[2 * i], u[2 * i + 1], p);
            wi[3 * i] = r.x; wi[3 * i + 1] = r.y; wi[3 * i + 2] = r.z;
            pdf[i] = p;
        }
    }
}

// CPU LBVH for topology parity (new in this build; the reference uses the
// driver's BVH).  Morton codes of triangle-bounds centroids quantised to 10
// bits per axis over the centroid bounds, stable sort by code, then the radix
// tree of Karras 2012 ("Maximizing Parallelism in the Construction of BVHs,
// Octrees, and k-d Trees", Fig. 4), with equal codes ordered by position.
static uint32_t expand_bits10(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
static int lbvh_delta(const std::vector<uint32_t> &k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    if (k[i] == k[j]) return 32 + __builtin_clz((uint32_t)(i ^ j));
    return __builtin_clz(k[i] ^ k[j]);
}
void or_lbvh(void *sp, uint32_t *morton, uint32_t *sorted, int32_t *children) {
    Scene *s = static_cast<Scene *>(sp);
    const int n = (int)s->triMesh.size();
    if (n == 0) return;
    std::vector<F3> cen(n);
    F3 bl(std::numeric_limits<float>::infinity()), bh(-std::numeric_limits<float>::infinity());
    for (int g = 0; g < n; g++) {
        F3 p0, p1, p2;
        tri_verts(*s, (uint32_t)g, p0, p1, p2);
        F3 lo = vmin(p0, vmin(p1, p2)), hi = vmax(p0, vmax(p1, p2));
        cen[g] = F3((lo.x + hi.x) * 0.5f, (lo.y + hi.y) * 0.5f, (lo.z + hi.z) * 0.5f);
        bl = vmin(bl, cen[g]);
        bh = vmax(bh, cen[g]);
    }
    std::vector<uint32_t> codes(n), ids(n);
    for (int g = 0; g < n; g++) {
        uint32_t q[3];
        for (int a = 0; a < 3; a++) {
            float ext = bh[a] - bl[a];
            float x = ext > 0.0f ? (cen[g][a] - bl[a]) / ext : 0.0f;
            q[a] = (uint32_t)std::min(std::max(x * 1024.0f, 0.0f), 1023.0f);
        }
        codes[g] = (expand_bits10(q[0]) << 2) | (expand_bits10(q[1]) << 1) | expand_bits10(q[2]);
        ids[g] = (uint32_t)g;
    }
    std::stable_sort(ids.begin(), ids.end(), [&](uint32_t a, uint32_t b) { return codes[a] < codes[b]; });
    std::vector<uint32_t> keys(n);
    for (int i = 0; i < n; i++) keys[i] = codes[ids[i]];
    if (morton) std::memcpy(morton, codes.data(), n * 4);
    if (sorted) std::memcpy(sorted, ids.data(), n * 4);
    if (!children) return;
    for (int i = 0; i < n - 1; i++) {
        int d = (lbvh_delta(keys, n, i, i + 1) - lbvh_delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
        int dmin = lbvh_delta(keys, n, i, i - d);
        int lmax = 2;
        while (lbvh_delta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
        int l = 0;
        for (int t = lmax / 2; t >= 1; t /= 2)
            if (lbvh_delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
        int j = i + l * d;
        int dnode = lbvh_delta(keys, n, i, j);
        int sp2 = 0, t = l;
        do {  // binary search for the split: t = ceil(l / 2), ceil(l / 4), ..., 1
            t = (t + 1) >> 1;
            if (lbvh_delta(keys, n, i, i + (sp2 + t) * d) > dnode) sp2 += t;
        } while (t > 1);
        int gamma = i + sp2 * d + std::min(d, 0);
        int lo = std::min(i, j), hi = std::max(i, j);
        children[2 * i] = (lo == gamma) ? ~gamma : gamma;
        children[2 * i + 1] = (hi == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    }
}

void or_trace_closest(void *sp, const float *rays, size_t n, pt_hit *out) {
    Scene *s = static_cast<Scene *>(sp);
    for (size_t i = 0; i < n; i++) {
        const float *r = &rays[8 * i];
        Hit h = trace_closest(*s, F3(r[0], r[1], r[2]), F3(r[4], r[5], r[6]), r[3], r[7], (uint32_t)i, 0u);
        out[i] = pt_hit{h.hit ? h.t : 0.0f, h.mesh, h.prim, h.u, h.v, h.hit ? 1u : 0u};
    }
}
void or_trace_shadow(void *sp, const float *rays, size_t n, uint32_t *occ, float *trans) {
    Scene *s = static_cast<Scene *>(sp);
    for (size_t i = 0; i < n; i++) {
        const float *r = &rays[8 * i];
        F3 t;
        occ[i] = trace_shadow(*s, F3(r[0], r[1], r[2]), F3(r[4], r[5], r[6]), r[3], r[7], t, (uint32_t)i, 0u) ? 1u : 0u;
        trans[3 * i] = t.x; trans[3 * i + 1] = t.y; trans[3 * i + 2] = t.z;
    }
}

// Render spp samples per pixel into sum (RGBA: xyz = sum L, w = count), in the
// reference's accumulation order (per pixel, frame by frame, float32).
// per_path (optional): W*H*spp*3 floats, Lo of every path (frame-major).
// threads <= 0: all hardware threads.  Returns 0 or -1 (unsupported scene).
static int render_impl(void *sp, const pt_render_params *P, float *sum, float *per_path, int threads,
                       uint64_t *counters, const CacheConst *cc);
int or_render(void *sp, const pt_render_params *P, float *sum, float *per_path, int threads, uint64_t *counters) {
    return render_impl(sp, P, sum, per_path, threads, counters, nullptr);
}
// or_render with radiance-cache termination into a constant cache (value: 3
// floats, rough_threshold as the library's pt_cache_params field).
int or_render_cached(void *sp, const pt_render_params *P, float *sum, float *per_path, int threads,
                     const float *value, float rough_threshold) {
    CacheConst cc{{value[0], value[1], value[2]}, rough_threshold};
    return render_impl(sp, P, sum, per_path, threads, nullptr, &cc);
}
static int render_impl(void *sp, const pt_render_params *P, float *sum, float *per_path, int threads,
                       uint64_t *counters, const CacheConst *cc) {
    Scene *s = static_cast<Scene *>(sp);
    Ctx c{s, P->env_sampling};
    const uint32_t W = P->width, H = P->height;
    const uint32_t TS = 32;  // NORI_BLOCK_SIZE, include/block.h:17
    const uint32_t tx = (W + TS - 1) / TS, ty = (H + TS - 1) / TS;
    std::atomic<uint32_t> next{0};
    std::atomic<uint64_t> next_ext{0}, next_sh{0};
    int nt = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    auto work = [&]() {
        PathStats ps;
        for (;;) {
            uint32_t t = next.fetch_add(1);
            if (t >= tx * ty) break;
            uint32_t x0 = (t % tx) * TS, y0 = (t / tx) * TS;
            for (uint32_t y = y0; y < std::min(H, y0 + TS); y++)
                for (uint32_t x = x0; x < std::min(W, x0 + TS); x++) {
                    float *acc = &sum[4 * ((size_t)y * W + x)];
                    for (uint32_t k = 0; k < P->spp; k++) {
                        F3 L = trace_path(c, *P, x, y, P->sample_offset + k, counters ? &ps : nullptr, cc);
                        acc[0] = acc[0] + L.x; acc[1] = acc[1] + L.y; acc[2] = acc[2] + L.z; acc[3] = acc[3] + 1.0f;
                        if (per_path) {
                            float *pp = &per_path[3 * ((size_t)k * W * H + (size_t)y * W + x)];
                            pp[0] = L.x; pp[1] = L.y; pp[2] = L.z;
                        }
                    }
                }
        }
        next_ext += ps.ext;
        next_sh += ps.shadow;
    };
    std::vector<std::thread> th;
    for (int i = 0; i < nt; i++) th.emplace_back(work);
    for (auto &t : th) t.join();
    if (counters) { counters[0] = next_ext.load(); counters[1] = next_sh.load(); }
    return 0;
}

}  // extern "C"
