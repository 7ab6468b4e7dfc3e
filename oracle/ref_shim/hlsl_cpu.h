// hlsl_cpu.h — the HLSL types, intrinsics and DXR objects the reference
// shaders use, implemented on the CPU so that the reference's own shader
// source (gracejinsotrue/PBRT-renderer-, shaders/*.hlsl(i)) compiles as C++.
//
// TEST INFRASTRUCTURE ONLY (see oracle/build_ref.py).  The shader files are
// never copied into this repository: build_ref.py rewrites them mechanically
// from the reference checkout into oracle/_ref/gen/ (git-ignored) and
// compiles them together with this header and ref_entry.cpp.
//
// Everything lives in namespace ref so the shader's unqualified calls
// (sqrt, min, pow, ...) resolve to the overloads here, with HLSL semantics,
// and never to <cmath>'s double versions.  Compile with
// -fsingle-precision-constant so unsuffixed literals are float as in HLSL.
//
// Hardware stand-ins (documented, not pinned by the reference): bilinear /
// trilinear filtering uses float weights; RayQuery reports candidates in
// increasing t.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#undef M_PI

namespace ref {

typedef unsigned int uint;

struct bool3 { bool x, y, z; };

struct uint2 {
    uint x, y;
    uint2() = default;
    uint2(uint a, uint b) : x(a), y(b) {}
};
struct float2 {
    union { struct { float x, y; }; struct { float r, g; }; };
    float2() = default;
    float2(float a, float b) { x = a; y = b; }
    explicit float2(const uint2 &u) { x = (float)u.x; y = (float)u.y; }
    float &operator[](int i) { return i == 0 ? x : y; }
};
struct uint3 {
    uint x, y, z;
    uint3() = default;
    uint3(uint a, uint b, uint c) : x(a), y(b), z(c) {}
    uint2 xy() const { return uint2(x, y); }
};
struct float3 {
    union { struct { float x, y, z; }; struct { float r, g, b; }; };
    float3() = default;
    float3(float a, float b_, float c) { x = a; y = b_; z = c; }
    float &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
struct float4 {
    union { struct { float x, y, z, w; }; struct { float r, g, b, a; }; };
    float4() = default;
    float4(float a_, float b_, float c, float d) { x = a_; y = b_; z = c; w = d; }
    float4(const float3 &v, float d) { x = v.x; y = v.y; z = v.z; w = d; }
    float3 xyz() const { return float3(x, y, z); }
    float3 rgb() const { return float3(x, y, z); }
};
struct int3 {
    int x, y, z;
    int3() = default;
    int3(int a, int b, int c) : x(a), y(b), z(c) {}
    explicit int3(const float3 &v) : x((int)v.x), y((int)v.y), z((int)v.z) {}
    int &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    int operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
struct int4 {
    int x, y, z, w;
    int4(const int3 &v, int d) : x(v.x), y(v.y), z(v.z), w(d) {}
};

// float2
inline float2 operator+(const float2 &a, const float2 &b) { return float2(a.x + b.x, a.y + b.y); }
inline float2 operator-(const float2 &a, const float2 &b) { return float2(a.x - b.x, a.y - b.y); }
inline float2 operator/(const float2 &a, const float2 &b) { return float2(a.x / b.x, a.y / b.y); }
inline float2 operator*(const float2 &a, float s) { return float2(a.x * s, a.y * s); }
// float3
inline float3 operator-(const float3 &a) { return float3(-a.x, -a.y, -a.z); }
inline float3 operator+(const float3 &a, const float3 &b) { return float3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline float3 operator-(const float3 &a, const float3 &b) { return float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float3 operator*(const float3 &a, const float3 &b) { return float3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float3 operator/(const float3 &a, const float3 &b) { return float3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline float3 operator*(const float3 &a, float s) { return float3(a.x * s, a.y * s, a.z * s); }
inline float3 operator*(float s, const float3 &a) { return float3(s * a.x, s * a.y, s * a.z); }
inline float3 operator/(const float3 &a, float s) { return float3(a.x / s, a.y / s, a.z / s); }
inline float3 operator+(const float3 &a, float s) { return float3(a.x + s, a.y + s, a.z + s); }
inline float3 operator-(const float3 &a, float s) { return float3(a.x - s, a.y - s, a.z - s); }
inline float3 operator-(float s, const float3 &a) { return float3(s - a.x, s - a.y, s - a.z); }
inline float3 operator/(float s, const float3 &a) { return float3(s / a.x, s / a.y, s / a.z); }
inline float3 operator+(float s, const float3 &a) { return float3(s + a.x, s + a.y, s + a.z); }
inline float3 &operator+=(float3 &a, const float3 &b) { return a = a + b; }
inline float3 &operator*=(float3 &a, const float3 &b) { return a = a * b; }
inline float3 &operator*=(float3 &a, float s) { return a = a * s; }
inline float3 &operator/=(float3 &a, float s) { return a = a / s; }
inline bool3 operator==(const float3 &a, float s) { return {a.x == s, a.y == s, a.z == s}; }
// float4
inline float4 operator+(const float4 &a, const float4 &b) { return float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
// int3
inline int3 operator-(const int3 &a, const int3 &b) { return int3(a.x - b.x, a.y - b.y, a.z - b.z); }

// scalar intrinsics (float overloads only, as HLSL float math)
inline float sqrt(float x) { return std::sqrt(x); }
inline float rsqrt(float x) { return 1.0f / std::sqrt(x); }
inline float exp(float x) { return std::exp(x); }
inline float log(float x) { return std::log(x); }
inline float log2(float x) { return std::log2(x); }
inline float pow(float x, float y) { return std::pow(x, y); }
inline float sin(float x) { return std::sin(x); }
inline float cos(float x) { return std::cos(x); }
inline float sinh(float x) { return std::sinh(x); }
inline float acos(float x) { return std::acos(x); }
inline float asin(float x) { return std::asin(x); }
inline float atan2(float y, float x) { return std::atan2(y, x); }
inline float abs(float x) { return std::fabs(x); }
inline float floor(float x) { return std::floor(x); }
inline float min(float a, float b) { return a < b ? a : b; }
inline float max(float a, float b) { return a > b ? a : b; }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline uint min(uint a, uint b) { return a < b ? a : b; }
inline uint max(uint a, uint b) { return a > b ? a : b; }
inline float clamp(float x, float a, float b) { return min(max(x, a), b); }
inline float saturate(float x) { return clamp(x, 0.0f, 1.0f); }
inline bool isnan(float x) { return std::isnan(x); }
inline bool isinf(float x) { return std::isinf(x); }
inline uint reversebits(uint x) {
    x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
    x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
    x = ((x >> 4) & 0x0F0F0F0Fu) | ((x & 0x0F0F0F0Fu) << 4);
    x = ((x >> 8) & 0x00FF00FFu) | ((x & 0x00FF00FFu) << 8);
    return (x >> 16) | (x << 16);
}
inline float asfloat(uint u) { float f; std::memcpy(&f, &u, 4); return f; }
inline float3 asfloat(const uint3 &u) { return float3(asfloat(u.x), asfloat(u.y), asfloat(u.z)); }
inline float2 asfloat(const uint2 &u) { return float2(asfloat(u.x), asfloat(u.y)); }
// vector intrinsics
inline float dot(const float3 &a, const float3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float3 cross(const float3 &a, const float3 &b) {
    return float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float length(const float3 &v) { return std::sqrt(dot(v, v)); }
inline float3 normalize(const float3 &v) { return v * (1.0f / std::sqrt(dot(v, v))); }
inline float3 reflect(const float3 &i, const float3 &n) { return i - 2.0f * dot(n, i) * n; }
inline float3 refract(const float3 &i, const float3 &n, float eta) {
    float ndi = dot(n, i);
    float k = 1.0f - eta * eta * (1.0f - ndi * ndi);
    if (k < 0.0f) return float3(0, 0, 0);
    return eta * i - (eta * ndi + std::sqrt(k)) * n;
}
inline float3 min(const float3 &a, const float3 &b) { return float3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline float3 max(const float3 &a, const float3 &b) { return float3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline float3 exp(const float3 &a) { return float3(exp(a.x), exp(a.y), exp(a.z)); }
inline float3 pow(const float3 &a, float y) { return float3(pow(a.x, y), pow(a.y, y), pow(a.z, y)); }
inline float3 saturate(const float3 &a) { return float3(saturate(a.x), saturate(a.y), saturate(a.z)); }
inline float3 clamp(const float3 &x, const float3 &a, const float3 &b) { return min(max(x, a), b); }
inline float3 lerp(const float3 &a, const float3 &b, float t) { return a + (b - a) * t; }
inline float lerp(float a, float b, float t) { return a + (b - a) * t; }
inline int3 clamp(const int3 &x, const int3 &a, const int3 &b) {
    return int3(min(max(x.x, a.x), b.x), min(max(x.y, a.y), b.y), min(max(x.z, a.z), b.z));
}
inline bool3 isnan(const float3 &v) { return {std::isnan(v.x), std::isnan(v.y), std::isnan(v.z)}; }
inline bool3 isinf(const float3 &v) { return {std::isinf(v.x), std::isinf(v.y), std::isinf(v.z)}; }
inline bool any(const bool3 &b) { return b.x || b.y || b.z; }
inline bool all(const bool3 &b) { return b.x && b.y && b.z; }

// ---- resources ------------------------------------------------------------
enum AddressMode { ADDR_WRAP, ADDR_CLAMP };
struct SamplerState { AddressMode u = ADDR_WRAP, v = ADDR_WRAP, w = ADDR_WRAP; };
struct RaytracingAccelerationStructure {};

inline int address(int i, int n, AddressMode m) {
    if (m == ADDR_WRAP) return ((i % n) + n) % n;
    return i < 0 ? 0 : (i >= n ? n - 1 : i);
}

template <class T = float4>
struct Texture2D_t {
    uint w = 0, h = 0;
    const float4 *data = nullptr;
    void GetDimensions(uint &W, uint &H) const { W = w; H = h; }
    float4 fetch(int x, int y) const { return data[(size_t)y * w + x]; }
    // Bilinear, level 0 (mip maps are not built by this stand-in).
    float4 SampleLevel(const SamplerState &s, const float2 &uv, float) const {
        float x = uv.x * (float)w - 0.5f, y = uv.y * (float)h - 0.5f;
        float fx0 = std::floor(x), fy0 = std::floor(y);
        float fx = x - fx0, fy = y - fy0;
        int xa = address((int)fx0, (int)w, s.u), xb = address((int)fx0 + 1, (int)w, s.u);
        int ya = address((int)fy0, (int)h, s.v), yb = address((int)fy0 + 1, (int)h, s.v);
        float4 a = fetch(xa, ya), b = fetch(xb, ya), c = fetch(xa, yb), d = fetch(xb, yb);
        float4 r;
        for (int k = 0; k < 4; k++) {
            float *pr = &r.x;
            const float *pa = &a.x, *pb = &b.x, *pc = &c.x, *pd = &d.x;
            float top = pa[k] * (1.0f - fx) + pb[k] * fx;
            float bot = pc[k] * (1.0f - fx) + pd[k] * fx;
            pr[k] = top * (1.0f - fy) + bot * fy;
        }
        return r;
    }
};
template <class T = float>
struct Texture3D_t {
    uint w = 0, h = 0, d = 0;
    const float *data = nullptr;
    void GetDimensions(uint, uint &W, uint &H, uint &D, uint &L) const { W = w; H = h; D = d; L = 1; }
    float at(int x, int y, int z) const { return data[(size_t)x + (size_t)w * (y + (size_t)h * z)]; }
    float Load(const int4 &c) const { return at(c.x, c.y, c.z); }
    float SampleLevel(const SamplerState &s, const float3 &uvw, float) const {
        float x = uvw.x * w - 0.5f, y = uvw.y * h - 0.5f, z = uvw.z * d - 0.5f;
        float fx0 = std::floor(x), fy0 = std::floor(y), fz0 = std::floor(z);
        float fx = x - fx0, fy = y - fy0, fz = z - fz0;
        int xa = address((int)fx0, w, s.u), xb = address((int)fx0 + 1, w, s.u);
        int ya = address((int)fy0, h, s.v), yb = address((int)fy0 + 1, h, s.v);
        int za = address((int)fz0, d, s.w), zb = address((int)fz0 + 1, d, s.w);
        float c00 = at(xa, ya, za) * (1 - fx) + at(xb, ya, za) * fx;
        float c10 = at(xa, yb, za) * (1 - fx) + at(xb, yb, za) * fx;
        float c01 = at(xa, ya, zb) * (1 - fx) + at(xb, ya, zb) * fx;
        float c11 = at(xa, yb, zb) * (1 - fx) + at(xb, yb, zb) * fx;
        float c0 = c00 * (1 - fy) + c10 * fy, c1 = c01 * (1 - fy) + c11 * fy;
        return c0 * (1 - fz) + c1 * fz;
    }
};
template <class T>
struct RWTexture2D {
    uint w = 0, h = 0;
    std::vector<T> px;
    T &operator[](const uint2 &p) { return px[(size_t)p.y * w + p.x]; }
};
template <class T>
struct StructuredBuffer {
    const T *data = nullptr;
    const T &operator[](uint i) const { return data[i]; }
};
struct ByteAddressBuffer {
    const uint *data = nullptr;
    uint Load(uint off) const { return data[off / 4]; }
    uint2 Load2(uint off) const { return uint2(data[off / 4], data[off / 4 + 1]); }
    uint3 Load3(uint off) const { return uint3(data[off / 4], data[off / 4 + 1], data[off / 4 + 2]); }
};

// ---- DXR -------------------------------------------------------------------
struct RayDesc { float3 Origin; float TMin; float3 Direction; float TMax; };
struct BuiltInTriangleIntersectionAttributes { float2 barycentrics; };

enum : uint {
    RAY_FLAG_NONE = 0,
    RAY_FLAG_ACCEPT_FIRST_HIT_AND_END_SEARCH = 0x4,
    RAY_FLAG_SKIP_CLOSEST_HIT_SHADER = 0x8,
};
enum : uint { CANDIDATE_NON_OPAQUE_TRIANGLE = 0, CANDIDATE_PROCEDURAL_PRIMITIVE = 1 };
enum : uint { COMMITTED_NOTHING = 0, COMMITTED_TRIANGLE_HIT = 1 };

// One triangle the ray crosses in [TMin, TMax] (provided by ref_entry.cpp).
struct Candidate { float t, u, v; uint inst, prim, gid; bool opaque; };
void collect_candidates(const RayDesc &ray, std::vector<Candidate> &out, bool accept_first);  // sorted by (t, gid)

extern int g_max_bounces;  // MAX_BOUNCES (see build_ref.py)
extern thread_local uint3 g_dispatch_index;
extern uint3 g_dispatch_dims;
inline uint3 DispatchRaysIndex() { return g_dispatch_index; }
inline uint3 DispatchRaysDimensions() { return g_dispatch_dims; }
// Entry points of the DXR pipeline path (compiled, never called here).
inline float RayTCurrent() { return 0.0f; }
inline uint InstanceID() { return 0; }
inline uint PrimitiveIndex() { return 0; }
inline void IgnoreHit() {}
inline float3 WorldRayDirection() { return float3(0, 0, 1); }

// Inline ray query: candidates are visited in increasing t; opaque ones are
// committed by traversal itself (ending the query), non-opaque ones are
// handed to the shader through Proceed().
template <uint FLAGS>
struct RayQuery {
    std::vector<Candidate> cands;
    size_t next = 0;
    int cur = -1;
    bool committed = false, done = false;
    Candidate com{};
    void TraceRayInline(const RaytracingAccelerationStructure &, uint, uint, const RayDesc &ray) {
        cands.clear();
        collect_candidates(ray, cands, (FLAGS & RAY_FLAG_ACCEPT_FIRST_HIT_AND_END_SEARCH) != 0);
        next = 0; cur = -1; committed = false; done = false;
    }
    bool Proceed() {
        if (done) return false;
        while (next < cands.size()) {
            const Candidate &c = cands[next++];
            if (committed && c.t > com.t) break;
            if (c.opaque) { com = c; committed = true; done = true; return false; }
            cur = (int)(next - 1);
            return true;
        }
        done = true;
        return false;
    }
    uint CandidateType() const { return CANDIDATE_NON_OPAQUE_TRIANGLE; }
    uint CandidateInstanceID() const { return cands[cur].inst; }
    uint CandidatePrimitiveIndex() const { return cands[cur].prim; }
    float2 CandidateTriangleBarycentrics() const { return float2(cands[cur].u, cands[cur].v); }
    void CommitNonOpaqueTriangleHit() {
        com = cands[cur];
        committed = true;
        // Later candidates are farther; with ACCEPT_FIRST_HIT the search ends.
        done = true;
    }
    uint CommittedStatus() const { return committed ? COMMITTED_TRIANGLE_HIT : COMMITTED_NOTHING; }
    float CommittedRayT() const { return com.t; }
    uint CommittedInstanceID() const { return com.inst; }
    uint CommittedPrimitiveIndex() const { return com.prim; }
    float2 CommittedTriangleBarycentrics() const { return float2(com.u, com.v); }
};

}  // namespace ref
