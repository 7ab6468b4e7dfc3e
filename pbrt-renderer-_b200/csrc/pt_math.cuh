// pt_math.cuh — shading math of the path tracer, shared by the CUDA kernels
// and the C++17 Nori host plugins (compiled as plain C++ there).
//
// Everything restates the reference's shader math
// (gracejinsotrue/PBRT-renderer-, shaders/*.hlsli, cited per function) in
// float32, in the reference's evaluation order.  Differences from a plain
// transcription: pow(x, 5) is evaluated by multiplication and FMA
// contraction is allowed, both rounding-level; the Sobol dimension-1 matrix
// product uses an exact byte-table form of the same GF(2) product.
#pragma once

#include <stdint.h>

#include "../../include/pt.h"

#if defined(__CUDACC__)
#define PT_HD __host__ __device__ __forceinline__
#else
#include <cmath>
#include <algorithm>
#define PT_HD inline
#endif

namespace ptm {

#if !defined(__CUDACC__)
struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
struct float2 { float x, y; };
inline float3 make_float3(float a, float b, float c) { return {a, b, c}; }
inline float2 make_float2(float a, float b) { return {a, b}; }
using std::fabs; using std::sqrt; using std::exp; using std::log; using std::sin; using std::cos;
using std::atan2; using std::asin; using std::acos; using std::pow; using std::sinh; using std::floor;
PT_HD float fminf_(float a, float b) { return a < b ? a : b; }
PT_HD float fmaxf_(float a, float b) { return a > b ? a : b; }
#define PT_FMIN fminf_
#define PT_FMAX fmaxf_
#else
using ::float3; using ::float4; using ::float2; using ::make_float3; using ::make_float2;
#define PT_FMIN fminf
#define PT_FMAX fmaxf
#endif

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618379067154f;

// HLSL min/max return the second operand when the first is NaN-free compare fails;
// these follow the (a < b ? a : b) form used by the oracle.
PT_HD float mn(float a, float b) { return a < b ? a : b; }
PT_HD float mx(float a, float b) { return a > b ? a : b; }
PT_HD float clampf(float x, float a, float b) { return mn(mx(x, a), b); }
PT_HD float sat(float x) { return clampf(x, 0.0f, 1.0f); }

// Round-to-nearest products and sums that the compiler may not fuse into an
// FMA: for expressions that cancel (the HG denominator near |g| -> 1), where
// a fused product shifts the result by many ulps against the unfused order.
#if defined(__CUDA_ARCH__)
PT_HD float rmul(float a, float b) { return __fmul_rn(a, b); }
PT_HD float radd(float a, float b) { return __fadd_rn(a, b); }
PT_HD float rsub(float a, float b) { return __fsub_rn(a, b); }
#else
PT_HD float rmul(float a, float b) { return a * b; }
PT_HD float radd(float a, float b) { return a + b; }
PT_HD float rsub(float a, float b) { return a - b; }
#endif

PT_HD float3 v3(float a) { return make_float3(a, a, a); }
PT_HD float3 v3(float a, float b, float c) { return make_float3(a, b, c); }
PT_HD float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
PT_HD float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
PT_HD float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
PT_HD float3 operator/(float3 a, float3 b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
PT_HD float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
PT_HD float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
PT_HD float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
PT_HD float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
PT_HD float3 operator-(float s, float3 a) { return make_float3(s - a.x, s - a.y, s - a.z); }
PT_HD float3 &operator+=(float3 &a, float3 b) { a = a + b; return a; }
PT_HD float3 &operator*=(float3 &a, float3 b) { a = a * b; return a; }
PT_HD float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PT_HD float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
PT_HD float len(float3 v) { return sqrtf(dot(v, v)); }
PT_HD float3 normalize(float3 v) { return v * (1.0f / sqrtf(dot(v, v))); }
PT_HD float3 vmin(float3 a, float3 b) { return make_float3(mn(a.x, b.x), mn(a.y, b.y), mn(a.z, b.z)); }
PT_HD float3 vmax(float3 a, float3 b) { return make_float3(mx(a.x, b.x), mx(a.y, b.y), mx(a.z, b.z)); }
PT_HD float3 vexp(float3 a) { return make_float3(expf(a.x), expf(a.y), expf(a.z)); }
PT_HD float3 lerp3(float3 a, float3 b, float t) { return a + (b - a) * t; }
PT_HD float lerpf(float a, float b, float t) { return a + (b - a) * t; }
PT_HD float maxc(float3 v) { return mx(v.x, mx(v.y, v.z)); }
PT_HD float pow5(float x) { float x2 = x * x; return x2 * x2 * x; }
PT_HD float3 reflect(float3 i, float3 n) { return i - 2.0f * dot(n, i) * n; }
PT_HD float3 refract(float3 i, float3 n, float eta) {
    float ndi = dot(n, i);
    float k = 1.0f - eta * eta * (1.0f - ndi * ndi);
    if (k < 0.0f) return v3(0.0f);
    return eta * i - (eta * ndi + sqrtf(k)) * n;
}
PT_HD float get(float3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

// ---------------------------------------------------------------------------
// Sample generator (shaders/RNG.hlsli:9-99)
// ---------------------------------------------------------------------------
PT_HD uint32_t pcg_hash(uint32_t v) {
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
}
PT_HD uint32_t brev(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __brev(x);
#else
    x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
    x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
    x = ((x >> 4) & 0x0F0F0F0Fu) | ((x & 0x0F0F0F0Fu) << 4);
    x = ((x >> 8) & 0x00FF00FFu) | ((x & 0x00FF00FFu) << 8);
    return (x >> 16) | (x << 16);
#endif
}
// Sobol dimension 1 (RNG.hlsli:17-30) is the GF(2) product of a fixed 32x32
// matrix with the index; sobol1_table(k, b) is that product for byte b at
// byte position k, so the product is the XOR of four table entries.
PT_HD uint32_t sobol1_loop(uint32_t index) {
    uint32_t r = 0u, dirn = 1u << 31;
    for (uint32_t i = index; i != 0u; i >>= 1u) {
        if (i & 1u) r ^= dirn;
        dirn ^= dirn >> 1u;
    }
    return r;
}
PT_HD uint32_t laine_karras(uint32_t x, uint32_t seed) {
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}
PT_HD uint32_t owen(uint32_t x, uint32_t seed) { return brev(laine_karras(brev(x), seed)); }
PT_HD float u32_to_unit(uint32_t v) { return mn(float(v) * 2.3283064365386963e-10f, 0.99999994f); }

// Path sampler state: dimension counter + white-noise stream (PCG mode).
struct Rng {
    uint32_t pixelSeed, sampleIndex, dim, white, kind;
};
PT_HD Rng rng_init(uint32_t pid, uint32_t npix, uint32_t frame, uint32_t kind) {  // RNG.hlsli:60-70
    Rng r;
    r.pixelSeed = pcg_hash(pid ^ 0x9e3779b9u);
    r.sampleIndex = frame;
    r.dim = 0u;
    r.white = pcg_hash(pid * 0x9e3779b9u + frame * 0x85ebca6bu + 1u);
    r.kind = kind;
    (void)npix;
    return r;
}

// ---------------------------------------------------------------------------
// Geometry helpers (shaders/GeometryUtils.hlsli)
// ---------------------------------------------------------------------------
PT_HD float balance(float a, float b) {  // :18-24
    float s = a + b;
    if (s < 1e-20f) return 0.0f;
    return a / s;
}
PT_HD void build_onb(float3 N, float3 &T, float3 &B) {  // :160-165
    float3 up = fabsf(N.y) < 0.999f ? v3(0.0f, 1.0f, 0.0f) : v3(1.0f, 0.0f, 0.0f);
    T = normalize(cross(up, N));
    B = cross(N, T);
}
PT_HD float3 to_local(float3 v, float3 T, float3 B, float3 N) { return v3(dot(v, T), dot(v, B), dot(v, N)); }
PT_HD float3 to_world(float3 v, float3 T, float3 B, float3 N) { return T * v.x + B * v.y + N * v.z; }
PT_HD float3 offset_origin(float3 p, float3 Ng, float3 N) {  // :178-183
    float3 q = p + N * 0.002f;
    q += Ng * mx(0.0f, -dot(q - p, Ng));
    return q;
}
PT_HD float3 cos_hemi(float u0, float u1) {  // :189-194
    float r = sqrtf(u0);
    float phi = 2.0f * kPi * u1;
    return v3(r * cosf(phi), r * sinf(phi), sqrtf(mx(0.0f, 1.0f - u0)));
}
PT_HD float fresnel(float cosI, float etaI, float etaT) {  // :200-219
    if (etaI == etaT) return 0.0f;
    if (cosI < 0.0f) { float t = etaI; etaI = etaT; etaT = t; cosI = -cosI; }
    float eta = etaI / etaT;
    float s2 = eta * eta * (1.0f - cosI * cosI);
    if (s2 > 1.0f) return 1.0f;
    float cosT = sqrtf(1.0f - s2);
    float Rs = (etaI * cosI - etaT * cosT) / (etaI * cosI + etaT * cosT);
    float Rp = (etaT * cosI - etaI * cosT) / (etaT * cosI + etaI * cosT);
    return 0.5f * (Rs * Rs + Rp * Rp);
}
// Mirror and dielectric (delta BSDFs), shaders/Shaders.hlsl:419-472: the
// direction a hit scatters into.  rd is the incoming ray's direction, N the
// shading normal turned to the side the ray arrives from (at a back-face hit
// the shader flips Ng and N with it), back whether the ray hit the back face.
// u is the dielectric's Fresnel draw (a mirror draws nothing).  A dielectric
// reflects with probability Fr, else refracts (reflecting on total internal
// reflection); etaScale is etaI / etaT after a refraction, else 1.  Delta
// BSDFs leave the throughput unchanged and have no pdf (lastBsdfPdf = 0).
// Every product and sum of the delta branch rounded on its own, in the
// oracle's order (no contraction): the result is the oracle's float32 value,
// and the same in every kernel that inlines it.
PT_HD float dot_nf(float3 a, float3 b) { return radd(radd(rmul(a.x, b.x), rmul(a.y, b.y)), rmul(a.z, b.z)); }
PT_HD float3 axpy_nf(float s, float3 x, float3 y) {  // s * x + y
    return make_float3(radd(rmul(s, x.x), y.x), radd(rmul(s, x.y), y.y), radd(rmul(s, x.z), y.z));
}
PT_HD float3 reflect_nf(float3 i, float3 n) {  // i - 2 dot(n, i) n
    const float k = rmul(2.0f, dot_nf(n, i));
    return make_float3(rsub(i.x, rmul(k, n.x)), rsub(i.y, rmul(k, n.y)), rsub(i.z, rmul(k, n.z)));
}
PT_HD float3 refract_nf(float3 i, float3 n, float eta) {  // eta i - (eta dot(n, i) + sqrt(k)) n
    const float ndi = dot_nf(n, i);
    const float k = rsub(1.0f, rmul(rmul(eta, eta), rsub(1.0f, rmul(ndi, ndi))));
    if (k < 0.0f) return v3(0.0f);
    const float c = radd(rmul(eta, ndi), sqrtf(k));
    return make_float3(rsub(rmul(eta, i.x), rmul(c, n.x)), rsub(rmul(eta, i.y), rmul(c, n.y)),
                       rsub(rmul(eta, i.z), rmul(c, n.z)));
}
PT_HD float fresnel_nf(float cosI, float etaI, float etaT) {  // :200-219
    if (etaI == etaT) return 0.0f;
    if (cosI < 0.0f) { float t = etaI; etaI = etaT; etaT = t; cosI = -cosI; }
    float eta = etaI / etaT;
    float s2 = rmul(rmul(eta, eta), rsub(1.0f, rmul(cosI, cosI)));
    if (s2 > 1.0f) return 1.0f;
    float cosT = sqrtf(rsub(1.0f, s2));
    float Rs = rsub(rmul(etaI, cosI), rmul(etaT, cosT)) / radd(rmul(etaI, cosI), rmul(etaT, cosT));
    float Rp = rsub(rmul(etaT, cosI), rmul(etaI, cosT)) / radd(rmul(etaT, cosI), rmul(etaI, cosT));
    return rmul(0.5f, radd(rmul(Rs, Rs), rmul(Rp, Rp)));
}
PT_HD float3 delta_scatter(uint32_t type, float3 rd, float3 N, bool back, float intIOR, float extIOR, float u,
                           float &etaScale) {
    etaScale = 1.0f;
    if (type == PT_MAT_MIRROR) return reflect_nf(rd, N);
    float etaI = back ? intIOR : extIOR, etaT = back ? extIOR : intIOR;
    float Fr = fresnel_nf(dot_nf(-rd, N), etaI, etaT);
    if (u < Fr) return reflect_nf(rd, N);
    float3 nd = refract_nf(rd, N, etaI / etaT);
    if (dot_nf(nd, nd) < 0.001f) return reflect_nf(rd, N);
    etaScale = etaI / etaT;
    return nd;
}
// The same in the local shading frame (BSDF query convention: wi points to the
// viewer, z is the outward normal; wi.z < 0 is a query from inside): returns
// the throughput weight (1), sets wo and pdf = 0 (a discrete measure).
PT_HD float3 delta_sample(float3 wi, const pt_material &m, float u, float3 &wo, float &pdf) {
    bool back = wi.z < 0.0f;
    float es;
    wo = delta_scatter(m.type, -wi, v3(0.0f, 0.0f, back ? -1.0f : 1.0f), back, m.intIOR, m.extIOR, u, es);
    pdf = 0.0f;
    return v3(1.0f);
}
PT_HD float luminance(float3 c) { return 0.212671f * c.x + 0.715160f * c.y + 0.072169f * c.z; }  // :225-228
PT_HD float3 albedo(const pt_material &m) { return v3(m.albedo[0], m.albedo[1], m.albedo[2]); }

// ---------------------------------------------------------------------------
// Beckmann microfacet (shaders/Microfacet.hlsli:13-125)
// ---------------------------------------------------------------------------
PT_HD float beckmann_d(float3 wh, float a) {
    if (wh.z <= 0.0f) return 0.0f;
    float c2 = wh.z * wh.z, t2 = (1.0f - c2) / c2, c3 = c2 * wh.z, a2 = a * a;
    return expf(-t2 / a2) / (kPi * a2 * c3);
}
PT_HD float beckmann_d_cos(float3 wh, float a) {
    if (wh.z <= 0.0f) return 0.0f;
    float c2 = wh.z * wh.z, t2 = (1.0f - c2) / c2, a2 = a * a;
    return expf(-t2 / a2) / (kPi * a2 * c2);
}
PT_HD float3 beckmann_sample(float u0, float u1, float a) {
    float phi = 2.0f * kPi * u1;
    float t2 = -a * a * logf(mx(1e-8f, 1.0f - u0));
    float c = 1.0f / sqrtf(1.0f + t2);
    float s = sqrtf(mx(0.0f, 1.0f - c * c));
    return v3(s * cosf(phi), s * sinf(phi), c);
}
PT_HD float smith_g1(float3 v, float3 wh, float a) {
    float dvw = dot(v, wh), dvn = v.z;
    if (dvw / dvn <= 0.0f) return 0.0f;
    float c2 = v.z * v.z;
    if (c2 < 1e-10f) return 0.0f;
    float tanT = sqrtf(mx(0.0f, 1.0f - c2)) / fabsf(v.z);
    if (tanT < 1e-10f) return 1.0f;
    float b = 1.0f / (a * tanT);
    if (b >= 1.6f) return 1.0f;
    float b2 = b * b;
    return (3.535f * b + 2.181f * b2) / (1.0f + 2.276f * b + 2.577f * b2);
}
PT_HD float3 microfacet_eval(float3 wi, float3 wo, const pt_material &m) {
    if (wi.z <= 0.0f || wo.z <= 0.0f) return v3(0.0f);
    float3 kd = albedo(m);
    float ks = 1.0f - maxc(kd);
    float3 wh = normalize(wi + wo);
    float D = beckmann_d(wh, m.alpha);
    float F = fresnel(dot(wh, wi), m.extIOR, m.intIOR);
    float G = smith_g1(wi, wh, m.alpha) * smith_g1(wo, wh, m.alpha);
    return kd * kInvPi + v3(1.0f) * (ks * D * F * G / mx(4.0f * wi.z * wo.z, 1e-10f));
}
PT_HD float microfacet_pdf(float3 wi, float3 wo, const pt_material &m) {
    if (wi.z <= 0.0f || wo.z <= 0.0f) return 0.0f;
    float ks = 1.0f - maxc(albedo(m));
    float3 wh = normalize(wi + wo);
    float Jh = 1.0f / mx(4.0f * dot(wh, wo), 1e-10f);
    return ks * beckmann_d_cos(wh, m.alpha) * Jh + (1.0f - ks) * wo.z * kInvPi;
}

// Subsurface entry lobe (Material.hlsli:48-58,92-100): Beckmann reflection
// with Fresnel at the half vector, alpha = max(roughness^2, 1e-4).  The walk
// under the surface is a shading event (Subsurface.hlsli), not a BSDF sample.
PT_HD float3 subsurface_eval(float3 wi, float3 wo, const pt_material &m) {
    if (wi.z <= 0.0f || wo.z <= 0.0f) return v3(0.0f);
    float a = mx(m.roughness * m.roughness, 1e-4f);
    float3 wh = normalize(wi + wo);
    float D = beckmann_d(wh, a);
    float Fr = fresnel(dot(wh, wi), m.extIOR, m.intIOR);
    float G = smith_g1(wi, wh, a) * smith_g1(wo, wh, a);
    return v3(1.0f) * (D * Fr * G / mx(4.0f * wi.z * wo.z, 1e-10f));
}
PT_HD float subsurface_pdf(float3 wi, float3 wo, const pt_material &m) {
    if (wi.z <= 0.0f || wo.z <= 0.0f) return 0.0f;
    float a = mx(m.roughness * m.roughness, 1e-4f);
    float3 wh = normalize(wi + wo);
    float Fr = fresnel(dot(wh, wi), m.extIOR, m.intIOR);
    return Fr * beckmann_d_cos(wh, a) / mx(4.0f * dot(wh, wo), 1e-10f);
}
// SubsurfaceParams (Subsurface.hlsli:24-31): scalar extinction 1 / mean free
// path and the per-channel single-scattering albedo of colour A.
PT_HD void subsurface_params(float3 A, float d, float &sigmaT, float3 &alpha) {
    sigmaT = 1.0f / mx(d, 1e-4f);
    float3 A2 = A * A, A3 = A2 * A;
    alpha = v3(1.0f) - vexp(-5.09406f * A + 2.61188f * A2 - 4.31805f * A3);
}

// ---------------------------------------------------------------------------
// Disney principled (shaders/Disney.hlsli:10-275, Material.hlsli:30-40,74-84)
// ---------------------------------------------------------------------------
struct DisneyPre {  // per-material terms that do not depend on directions
    float3 base, f0, csheen;
    float alpha, ccAlpha, pD, pS, pC;
};
PT_HD DisneyPre disney_pre(const pt_material &m) {
    DisneyPre p;
    p.base = albedo(m);
    float lum = luminance(p.base);
    float3 tint = lum > 0.0f ? p.base / v3(lum) : v3(1.0f);
    float3 cspec0 = 0.08f * m.specular * lerp3(v3(1.0f), tint, m.specularTint);
    p.f0 = lerp3(cspec0, p.base, m.metallic);
    p.csheen = lerp3(v3(1.0f), tint, m.sheenTint);
    p.alpha = mx(m.roughness * m.roughness, 1e-4f);
    p.ccAlpha = lerpf(0.1f, 0.001f, m.clearcoatGloss);
    float wd = 1.0f - m.metallic, ws = 1.0f, wc = 0.25f * m.clearcoat;
    float tot = wd + ws + wc;
    float inv = tot > 0.0f ? 1.0f / tot : 0.0f;
    p.pD = wd * inv; p.pS = ws * inv; p.pC = wc * inv;
    return p;
}
PT_HD float ggx_d(float ndh, float a) {
    if (ndh <= 0.0f) return 0.0f;
    float a2 = a * a;
    float den = ndh * ndh * (a2 - 1.0f) + 1.0f;
    return a2 / mx(kPi * den * den, 1e-10f);
}
PT_HD float ggx_g1(float ndv, float a) {
    if (ndv <= 0.0f) return 0.0f;
    float a2 = a * a;
    float den = ndv + sqrtf(a2 + (1.0f - a2) * ndv * ndv);
    return 2.0f * ndv / mx(den, 1e-10f);
}
PT_HD float gtr1_d(float ndh, float a) {
    if (ndh <= 0.0f) return 0.0f;
    float a2 = a * a;
    if (a2 >= 0.9999f) return kInvPi;
    float t = 1.0f + (a2 - 1.0f) * ndh * ndh;
    return (a2 - 1.0f) / (kPi * logf(a2) * t);
}
// f and pdf of the full Disney BSDF for local wi (towards viewer), wo (light).
PT_HD void disney_eval_pdf(float3 wi, float3 wo, const pt_material &m, const DisneyPre &p, float3 &f, float &pdf) {
    f = v3(0.0f);
    pdf = 0.0f;
    if (wi.z <= 0.0f || wo.z <= 0.0f) return;
    float3 wh = normalize(wi + wo);
    float cd = fabsf(dot(wo, wh));
    float fwi = pow5(1.0f - wi.z), fwo = pow5(1.0f - wo.z);
    // Burley diffuse + Hanrahan-Krueger blend (Disney.hlsli:10-48)
    float fd90 = 0.5f + 2.0f * m.roughness * cd * cd;
    float3 fB = p.base * kInvPi * ((1.0f + (fd90 - 1.0f) * fwi) * (1.0f + (fd90 - 1.0f) * fwo));
    float f90 = m.roughness * cd * cd;
    float cs = mx(wi.z + wo.z, 1e-4f);
    float ss = 1.25f * ((1.0f + (f90 - 1.0f) * fwi) * (1.0f + (f90 - 1.0f) * fwo) * (1.0f / cs - 0.5f) + 0.5f);
    float3 fSS = p.base * kInvPi * ss;
    float3 fd = lerp3(fB, fSS, m.subsurface);
    // GGX specular (Disney.hlsli:114-135)
    float3 fs = v3(0.0f);
    float pdfS = 0.0f, pdfC = 0.0f, fc = 0.0f;
    if (wh.z > 0.0f) {
        float vdh = fabsf(dot(wi, wh));
        float D = ggx_d(wh.z, p.alpha);
        float3 F = p.f0 + (v3(1.0f) - p.f0) * pow5(1.0f - vdh);
        float G = ggx_g1(wi.z, p.alpha) * ggx_g1(wo.z, p.alpha);
        fs = D * F * G / mx(4.0f * wi.z * wo.z, 1e-10f);
        pdfS = D * wh.z / mx(4.0f * fabsf(dot(wh, wo)), 1e-10f);
        if (m.clearcoat > 0.0f) {  // GTR1 clearcoat (Disney.hlsli:209-240)
            float Dc = gtr1_d(wh.z, p.ccAlpha);
            float Fc = 0.04f + (1.0f - 0.04f) * pow5(1.0f - vdh);
            float Gc = ggx_g1(wi.z, 0.25f) * ggx_g1(wo.z, 0.25f);
            fc = 0.25f * m.clearcoat * Dc * Fc * Gc / mx(4.0f * wi.z * wo.z, 1e-10f);
            pdfC = Dc * wh.z / mx(4.0f * fabsf(dot(wh, wo)), 1e-10f);
        }
    }
    float3 fsh = v3(0.0f);
    if (m.sheen > 0.0f) fsh = m.sheen * p.csheen * pow5(1.0f - cd);  // Disney.hlsli:145-160
    f = (1.0f - m.metallic) * (fd + fsh) + fs + v3(fc);
    pdf = p.pD * (wo.z * kInvPi) + p.pS * pdfS + p.pC * pdfC;
}
PT_HD float3 ggx_sample_wh(float u0, float u1, float a) {
    float a2 = a * a;
    float c2 = (1.0f - u0) / mx(1.0f + (a2 - 1.0f) * u0, 1e-10f);
    float c = sqrtf(sat(c2)), s = sqrtf(mx(0.0f, 1.0f - c2));
    float phi = 2.0f * kPi * u1;
    return v3(s * cosf(phi), s * sinf(phi), c);
}
PT_HD float3 gtr1_sample_wh(float u0, float u1, float a) {
    float a2 = a * a, c2;
    if (a2 >= 0.9999f) c2 = 1.0f - u0;
    else c2 = (1.0f - powf(a2, 1.0f - u0)) / (1.0f - a2);
    float c = sqrtf(sat(c2)), s = sqrtf(mx(0.0f, 1.0f - c2));
    float phi = 2.0f * kPi * u1;
    return v3(s * cosf(phi), s * sinf(phi), c);
}

// ---------------------------------------------------------------------------
// Chiang 2016 hair (shaders/Hair.hlsli:26-432)
// ---------------------------------------------------------------------------
PT_HD float hair_i0(float x) {
    float val = 0.0f, x2i = 1.0f, ifact = 1.0f, i4 = 1.0f;
    for (int i = 0; i < 10; i++) {
        if (i > 0) { x2i *= x * x; ifact *= float(i); i4 *= 4.0f; }
        val += x2i / (i4 * ifact * ifact);
    }
    return val;
}
PT_HD float hair_log_i0(float x) {
    if (x > 12.0f) return x + 0.5f * (-logf(2.0f * kPi) + logf(1.0f / x) + 1.0f / (8.0f * x));
    return logf(hair_i0(x));
}
PT_HD float hair_mp(float cti, float cto, float sti, float sto, float v) {
    float a = cti * cto / v, b = sti * sto / v;
    if (v <= 0.1f) return expf(hair_log_i0(a) - b - 1.0f / v + 0.6931f + logf(1.0f / (2.0f * v)));
    return (expf(-b) * hair_i0(a)) / (sinhf(1.0f / v) * 2.0f * v);
}
PT_HD float logistic_cdf(float x, float s) { return 1.0f / (1.0f + expf(-x / s)); }
PT_HD float hair_np(float phi, int p, float s, float go, float gt) {
    float dphi = phi - (2.0f * float(p) * gt - 2.0f * go + float(p) * kPi);
    // |dphi| < 8 pi for finite inputs; the bound only guards non-finite ones
    for (int k = 0; k < 8 && dphi > kPi; k++) dphi -= 2.0f * kPi;
    for (int k = 0; k < 8 && dphi < -kPi; k++) dphi += 2.0f * kPi;
    float den = logistic_cdf(kPi, s) - logistic_cdf(-kPi, s);
    if (!(den > 1e-10f)) return 0.0f;
    float ex = expf(-fabsf(dphi) / s);
    return ex / (s * (1.0f + ex) * (1.0f + ex)) / den;
}
struct HairPre {
    float v[4], s, sin2k[3], cos2k[3];
    float3 sigma_a;
};
PT_HD HairPre hair_pre(const pt_material &m) {
    HairPre p;
    float bm = m.roughness;
    float v0 = 0.726f * bm + 0.812f * bm * bm + 3.7f * powf(bm, 20.0f);
    v0 = v0 * v0;
    p.v[0] = v0; p.v[1] = 0.25f * v0; p.v[2] = 4.0f * v0; p.v[3] = p.v[2];
    float bn = m.betaN;
    p.s = 0.626657069f * (0.265f * bn + 1.194f * bn * bn + 5.372f * powf(bn, 22.0f));
    float ar = m.alpha * kPi / 180.0f;
    p.sin2k[0] = sinf(ar);
    p.cos2k[0] = sqrtf(mx(0.0f, 1.0f - p.sin2k[0] * p.sin2k[0]));
    for (int i = 1; i < 3; i++) {
        p.sin2k[i] = 2.0f * p.cos2k[i - 1] * p.sin2k[i - 1];
        p.cos2k[i] = p.cos2k[i - 1] * p.cos2k[i - 1] - p.sin2k[i - 1] * p.sin2k[i - 1];
    }
    float den = 5.969f - 0.215f * bn + 2.532f * bn * bn - 10.73f * bn * bn * bn + 5.574f * bn * bn * bn * bn +
                0.245f * bn * bn * bn * bn * bn;
    float3 C = albedo(m);
    float l0 = logf(C.x) / den, l1 = logf(C.y) / den, l2 = logf(C.z) / den;
    p.sigma_a = v3(C.x > 1e-4f ? l0 * l0 : 100.0f, C.y > 1e-4f ? l1 * l1 : 100.0f, C.z > 1e-4f ? l2 * l2 : 100.0f);
    return p;
}
PT_HD void hair_ap(float cto, float sto, float h, float eta, float3 sa, float3 ap[4]) {
    float etap = sqrtf(mx(0.0f, eta * eta - sto * sto)) / mx(cto, 1e-6f);
    float sgt = clampf(h / etap, -1.0f, 1.0f);
    float cgt = sqrtf(mx(0.0f, 1.0f - sgt * sgt));
    float stt = sto / eta;
    float ctt = sqrtf(mx(0.0f, 1.0f - stt * stt));
    float3 Tr = vexp(-sa * (2.0f * cgt / mx(ctt, 1e-6f)));
    float cgo = sqrtf(mx(0.0f, 1.0f - h * h));
    float f = fresnel(cto * cgo, 1.0f, eta);
    ap[0] = v3(f);
    ap[1] = (1.0f - f) * (1.0f - f) * Tr;
    ap[2] = ap[1] * Tr * f;
    float3 den = vmax(v3(1.0f) - Tr * f, v3(1e-10f));
    ap[3] = ap[2] * f * Tr / den;
}
PT_HD void hair_tilt(int p, float sto, float cto, const HairPre &P, float &sp, float &cp) {
    if (p == 0) { sp = sto * P.cos2k[1] - cto * P.sin2k[1]; cp = cto * P.cos2k[1] + sto * P.sin2k[1]; }
    else if (p == 1) { sp = sto * P.cos2k[0] + cto * P.sin2k[0]; cp = cto * P.cos2k[0] - sto * P.sin2k[0]; }
    else if (p == 2) { sp = sto * P.cos2k[2] + cto * P.sin2k[2]; cp = cto * P.cos2k[2] - sto * P.sin2k[2]; }
    else { sp = sto; cp = cto; }
    cp = fabsf(cp);
}
// Combined f (already divided by |cos theta_i|) and pdf (HairBCSDF_Eval + _Pdf).
PT_HD void hair_eval_pdf(float3 wi, float3 wo, const pt_material &m, const HairPre &P, float h, float3 &f, float &pdf) {
    float sto = wi.x, cto = sqrtf(mx(0.0f, 1.0f - sto * sto)), phio = atan2f(wi.z, wi.y);
    float sti = wo.x, cti = sqrtf(mx(0.0f, 1.0f - sti * sti)), phii = atan2f(wo.z, wo.y);
    float phi = phii - phio;
    float go = asinf(clampf(h, -1.0f, 1.0f));
    float eta = m.intIOR;
    float etap = sqrtf(mx(0.0f, eta * eta - sto * sto)) / mx(cto, 1e-6f);
    float gt = asinf(clampf(h / etap, -1.0f, 1.0f));
    float3 ap[4];
    hair_ap(cto, sto, h, eta, P.sigma_a, ap);
    float al[4], sum = 0.0f;
    for (int i = 0; i < 4; i++) { al[i] = luminance(ap[i]); sum += al[i]; }
    float inv = sum > 0.0f ? 1.0f / sum : 0.0f;
    float3 fs = v3(0.0f);
    float ps = 0.0f;
    for (int p = 0; p < 3; p++) {
        float sp, cp;
        hair_tilt(p, sto, cto, P, sp, cp);
        float mp = hair_mp(cti, cp, sti, sp, P.v[p]);
        float np = hair_np(phi, p, P.s, go, gt);
        fs += mp * ap[p] * np;
        ps += mp * al[p] * inv * np;
    }
    float mp3 = hair_mp(cti, cto, sti, sto, P.v[3]);
    fs += mp3 * ap[3] / (2.0f * kPi);
    ps += mp3 * al[3] * inv * (1.0f / (2.0f * kPi));
    float ac = fabsf(wo.z);
    if (ac > 1e-6f) fs = fs / v3(ac);
    f = fs;
    pdf = ps;
}
// HairBCSDF_Sample direction part (Hair.hlsli:351-421) with the four uniforms.
PT_HD float3 hair_sample_dir(float3 wi, const float *u, const pt_material &m, const HairPre &P, float h) {
    float sto = wi.x, cto = sqrtf(mx(0.0f, 1.0f - sto * sto)), phio = atan2f(wi.z, wi.y);
    float go = asinf(clampf(h, -1.0f, 1.0f));
    float eta = m.intIOR;
    float etap = sqrtf(mx(0.0f, eta * eta - sto * sto)) / mx(cto, 1e-6f);
    float gt = asinf(clampf(h / etap, -1.0f, 1.0f));
    float3 ap[4];
    hair_ap(cto, sto, h, eta, P.sigma_a, ap);
    float apPdf[4], sum = 0.0f;
    for (int i = 0; i < 4; i++) { apPdf[i] = luminance(ap[i]); sum += apPdf[i]; }
    float inv = sum > 0.0f ? 1.0f / sum : 0.0f;
    for (int j = 0; j < 4; j++) apPdf[j] *= inv;
    float u0 = u[0];
    int p = 0;
    float cdf = apPdf[0];
    while (p < 3 && u0 > cdf) { p++; cdf += apPdf[p]; }
    float sp, cp;
    hair_tilt(p, sto, cto, P, sp, cp);
    float u1 = u[1], u2 = u[2];
    float ct = 1.0f + P.v[p] * logf(mx(u1, 1e-5f) + (1.0f - u1) * expf(-2.0f / P.v[p]));
    float st = sqrtf(mx(0.0f, 1.0f - ct * ct));
    float cphs = cosf(2.0f * kPi * u2);
    float sti = -ct * sp + st * cphs * cp;
    float cti = sqrtf(mx(0.0f, 1.0f - sti * sti));
    float u3 = u[3];
    float dphi;
    if (p < 3) {
        float ca = logistic_cdf(-kPi, P.s), cb = logistic_cdf(kPi, P.s);
        float t = clampf(ca + u3 * (cb - ca), 1e-6f, 1.0f - 1e-6f);
        dphi = (2.0f * float(p) * gt - 2.0f * go + float(p) * kPi) + (-P.s * logf(1.0f / t - 1.0f));
    } else {
        dphi = 2.0f * kPi * u3;
    }
    float phii = phio + dphi;
    return v3(sti, cti * cosf(phii), cti * sinf(phii));
}

// ---------------------------------------------------------------------------
// Material dispatch (shaders/Material.hlsli:18-194)
// ---------------------------------------------------------------------------
// The dispatchers take the material type as an explicit key: a kernel that
// serves one material class passes a compile-time constant and keeps only
// that branch.
PT_HD void material_eval_pdf_t(uint32_t type, float3 wi, float3 wo, const pt_material &m, float h, float3 &f,
                               float &pdf) {
    switch (type) {
        case PT_MAT_DIFFUSE:
            if (wi.z <= 0.0f || wo.z <= 0.0f) { f = v3(0.0f); pdf = 0.0f; }
            else { f = albedo(m) * kInvPi; pdf = wo.z * kInvPi; }
            return;
        case PT_MAT_MICROFACET:
            f = microfacet_eval(wi, wo, m);
            pdf = microfacet_pdf(wi, wo, m);
            return;
        case PT_MAT_DISNEY: {
            DisneyPre p = disney_pre(m);
            disney_eval_pdf(wi, wo, m, p, f, pdf);
            return;
        }
        case PT_MAT_HAIR: {
            HairPre p = hair_pre(m);
            hair_eval_pdf(wi, wo, m, p, h, f, pdf);
            return;
        }
        case PT_MAT_SUBSURFACE:
            f = subsurface_eval(wi, wo, m);
            pdf = subsurface_pdf(wi, wo, m);
            return;
        default:
            f = v3(0.0f);
            pdf = 0.0f;
    }
}
PT_HD void material_eval_pdf(float3 wi, float3 wo, const pt_material &m, float h, float3 &f, float &pdf) {
    material_eval_pdf_t(m.type, wi, wo, m, h, f, pdf);
}
// Number of NextFloat draws MaterialSample makes for this material and wi.
PT_HD int material_sample_dims_t(uint32_t type, float3 wi) {
    switch (type) {
        case PT_MAT_DIFFUSE: case PT_MAT_MICROFACET: return wi.z <= 0.0f ? 0 : 2;
        case PT_MAT_DISNEY: return wi.z <= 0.0f ? 0 : 3;
        case PT_MAT_HAIR: return 4;
        default: return 0;
    }
}
PT_HD int material_sample_dims(const pt_material &m, float3 wi) { return material_sample_dims_t(m.type, wi); }
// MaterialSample with its uniforms supplied: returns f*cos/pdf, sets wo, pdf.
PT_HD float3 material_sample_t(uint32_t type, float3 wi, const float *u, const pt_material &m, float h, float3 &wo,
                               float &pdf) {
    switch (type) {
        case PT_MAT_DIFFUSE:
            if (wi.z <= 0.0f) { wo = v3(0.0f, 0.0f, 1.0f); pdf = 0.0f; return v3(0.0f); }
            wo = cos_hemi(u[0], u[1]);
            pdf = wo.z * kInvPi;
            return albedo(m);
        case PT_MAT_MICROFACET: {
            if (wi.z <= 0.0f) { wo = v3(0.0f, 0.0f, 1.0f); pdf = 0.0f; return v3(0.0f); }
            float ks = 1.0f - maxc(albedo(m));
            float ux = u[0], uy = u[1];
            if (ux < ks) {
                ux /= ks;
                float3 wh = beckmann_sample(ux, uy, m.alpha);
                wo = 2.0f * dot(wh, wi) * wh - wi;
            } else {
                ux = (ux - ks) / (1.0f - ks);
                wo = cos_hemi(ux, uy);
            }
            if (wo.z <= 0.0f) { pdf = 0.0f; return v3(0.0f); }
            pdf = microfacet_pdf(wi, wo, m);
            if (pdf <= 0.0f) return v3(0.0f);
            return microfacet_eval(wi, wo, m) * wo.z / pdf;
        }
        case PT_MAT_DISNEY: {
            if (wi.z <= 0.0f) { wo = v3(0.0f, 0.0f, 1.0f); pdf = 0.0f; return v3(0.0f); }
            DisneyPre p = disney_pre(m);
            if (u[0] < p.pD) {
                wo = cos_hemi(u[1], u[2]);
            } else if (u[0] < p.pD + p.pS) {
                float3 wh = ggx_sample_wh(u[1], u[2], p.alpha);
                wo = 2.0f * dot(wh, wi) * wh - wi;
            } else {
                float3 wh = gtr1_sample_wh(u[1], u[2], p.ccAlpha);
                wo = 2.0f * dot(wh, wi) * wh - wi;
            }
            if (wo.z <= 0.0f) { pdf = 0.0f; return v3(0.0f); }
            float3 f;
            disney_eval_pdf(wi, wo, m, p, f, pdf);
            if (pdf <= 0.0f) return v3(0.0f);
            return f * wo.z / pdf;
        }
        case PT_MAT_HAIR: {
            HairPre p = hair_pre(m);
            wo = hair_sample_dir(wi, u, m, p, h);
            float3 f;
            hair_eval_pdf(wi, wo, m, p, h, f, pdf);
            if (pdf <= 0.0f) return v3(0.0f);
            return f * fabsf(wo.z) / pdf;
        }
        default:
            wo = v3(0.0f, 0.0f, 1.0f);
            pdf = 0.0f;
            return v3(0.0f);
    }
}
PT_HD float3 material_sample(float3 wi, const float *u, const pt_material &m, float h, float3 &wo, float &pdf) {
    return material_sample_t(m.type, wi, u, m, h, wo, pdf);
}

// ---------------------------------------------------------------------------
// Henyey-Greenstein (shaders/Volume.hlsl:31-65)
// ---------------------------------------------------------------------------
PT_HD float hg(float c, float g) {
    float g2 = rmul(g, g);
    float den = rsub(radd(1.0f, g2), rmul(2.0f * g, c));
    return rmul(1.0f / (4.0f * kPi), 1.0f - g2) / rmul(den, sqrtf(mx(den, 1e-8f)));
}
PT_HD float3 sample_hg(float3 wo, float g, float xi1, float xi2, float &pdf) {
    float c;
    if (fabsf(g) < 1e-3f) c = rsub(1.0f, 2.0f * xi1);
    else {
        float g2 = rmul(g, g);
        float sq = (1.0f - g2) / rsub(radd(1.0f, g), rmul(2.0f * g, xi1));
        c = clampf(rsub(radd(1.0f, g2), rmul(sq, sq)) / (2.0f * g), -1.0f, 1.0f);
    }
    float s = sqrtf(mx(0.0f, 1.0f - c * c));
    float phi = 2.0f * kPi * xi2;
    float3 T, B;
    build_onb(wo, T, B);
    float3 wi = s * cosf(phi) * T + s * sinf(phi) * B + c * wo;
    pdf = hg(c, g);
    return normalize(wi);
}

}  // namespace ptm
