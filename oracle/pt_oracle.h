// pt_oracle.h — CPU oracle for the path-tracing hot path.
//
// TEST INFRASTRUCTURE ONLY.  This is a scalar C++17 restatement of the
// reference's DXR megakernel (gracejinsotrue/PBRT-renderer-,
// shaders/Shaders.hlsl:25-651 and the .hlsli files it includes), used by the
// tests, the smoke check and the CPU-baseline leg of bench.py as the checker.
// The product (libpt) never links, loads or calls it.
//
// Parity pins: the restatement is checked against (a) the reference's own
// shader source compiled for the CPU through oracle/ref_shim (built by
// oracle/build_ref.py into oracle/_ref/, this container only), and (b) the
// analytic golden values the reference's validation suite states
// (Beer-Lambert exp(-2), white furnaces).
//
// Arithmetic follows the shaders in IEEE float32 (FP contraction off, float
// literals), so integer work (RNG, CDF searches, BVH topology) is bit-exact
// and float work matches to rounding.  The BSDF / phase / envmap routines are
// templates so the tests can evaluate them in FP64 as the reference of the
// reference.
#pragma once

#include <cmath>
#include <cstdint>
#include <vector>

#include "../include/pt.h"

namespace oracle {

template <class T>
struct V3 {
    T x, y, z;
    V3() = default;
    constexpr V3(T a, T b, T c) : x(a), y(b), z(c) {}
    explicit constexpr V3(T a) : x(a), y(a), z(a) {}
    template <class U>
    explicit V3(const V3<U> &o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
    T &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    V3 operator-() const { return {-x, -y, -z}; }
    V3 operator+(const V3 &o) const { return {x + o.x, y + o.y, z + o.z}; }
    V3 operator-(const V3 &o) const { return {x - o.x, y - o.y, z - o.z}; }
    V3 operator*(const V3 &o) const { return {x * o.x, y * o.y, z * o.z}; }
    V3 operator/(const V3 &o) const { return {x / o.x, y / o.y, z / o.z}; }
    V3 operator*(T s) const { return {x * s, y * s, z * s}; }
    V3 operator/(T s) const { return {x / s, y / s, z / s}; }
    V3 operator+(T s) const { return {x + s, y + s, z + s}; }
    V3 operator-(T s) const { return {x - s, y - s, z - s}; }
    V3 &operator+=(const V3 &o) { return *this = *this + o; }
    V3 &operator*=(const V3 &o) { return *this = *this * o; }
    V3 &operator/=(T s) { return *this = *this / s; }
};
template <class T>
inline V3<T> operator*(T s, const V3<T> &v) { return {s * v.x, s * v.y, s * v.z}; }
template <class T>
inline V3<T> operator-(T s, const V3<T> &v) { return {s - v.x, s - v.y, s - v.z}; }

using F3 = V3<float>;

// Material parameters in the precision of the evaluation.
template <class T>
struct Mat {
    uint32_t type;
    V3<T> albedo;
    T intIOR, extIOR, alpha;
    T roughness, metallic, specular, specularTint, sheen, sheenTint, subsurface,
        clearcoat, clearcoatGloss, anisotropic, betaN;
    static Mat from(const pt_material &m) {
        Mat r;
        r.type = m.type;
        r.albedo = V3<T>(T(m.albedo[0]), T(m.albedo[1]), T(m.albedo[2]));
        r.intIOR = m.intIOR; r.extIOR = m.extIOR; r.alpha = m.alpha;
        r.roughness = m.roughness; r.metallic = m.metallic; r.specular = m.specular;
        r.specularTint = m.specularTint; r.sheen = m.sheen; r.sheenTint = m.sheenTint;
        r.subsurface = m.subsurface; r.clearcoat = m.clearcoat;
        r.clearcoatGloss = m.clearcoatGloss; r.anisotropic = m.anisotropic; r.betaN = m.betaN;
        return r;
    }
};

}  // namespace oracle
