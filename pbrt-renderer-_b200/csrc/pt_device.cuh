// pt_device.cuh — device-side scene view, sampler, envmap, volume, emitter
// and 8-wide BVH traversal routines of libpt (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pt_math.cuh"

namespace pt {

using namespace ptm;

// Dense float grid, x fastest.
struct DevGrid {
    uint32_t w, h, d;
    const float *data;
};

// BVH8 node, 80 bytes (5 x 16 B), in this library's own layout:
//   n0 = (p.x, p.y, p.z, e.x | e.y << 8 | e.z << 16 | imask << 24)
//   n1 = (child_base, tri_base, meta[0..3], meta[4..7])
//   n2 = (qlo.x[0..3], qlo.x[4..7], qlo.y[0..3], qlo.y[4..7])
//   n3 = (qlo.z[0..3], qlo.z[4..7], qhi.x[0..3], qhi.x[4..7])
//   n4 = (qhi.y[0..3], qhi.y[4..7], qhi.z[0..3], qhi.z[4..7])
// Child i's box is p + [qlo_i, qhi_i] * 2^(e - 127) per axis.  imask bit i:
// child i is an internal node (index child_base + rank of i among internal
// children).  meta[i] = (bits << 5) | position, one formula for every child:
// a hit ORs bits << position into the node's hit mask.  Internal child:
// bits 1 at position 24 + i; leaf of c (1..3) triangles at tri_base + offset:
// bits 2^c - 1 at position offset (< 24); empty slot: 0.  Child slots follow
// the octant of the child's centre within the node, so visiting slot
// (k ^ oct) for k = 0..7 is near-to-far for rays of octant oct.
struct BVH8Node { uint4 n[5]; };

struct DevScene {
    // geometry in BVH8 leaf order: 3 x float4 per triangle
    // (v0.xyz, gid bits), (e1 = v1 - v0, alpha flag bits), (e2 = v2 - v0, 0);
    // alpha flag = 1 when the triangle's material has an alpha map
    const float4 *tri;
    const BVH8Node *nodes;
    uint32_t numTris, numNodes;
    const uint32_t *triMesh;      // global triangle id -> mesh
    const uint32_t *meshFirstTri; // mesh -> first global triangle id
    const pt_material *mats;
    const uint32_t *meshClass;    // mesh -> shading class of its hits
    uint32_t numMeshes;
    uint32_t hasGlass;            // any mirror/dielectric mesh (non-opaque for shadow rays)
    const float *pos, *nrm, *uv, *tan;
    const uint32_t *idx;
    // emitters (src/gpu/DXRApp_Scene.cpp:243-299)
    const float *emitterCdf;
    const uint32_t *emitterList;
    uint32_t emitterCount;
    // envmap (RGBA float32) + sampling tables
    const float4 *env;
    uint32_t envW, envH;
    float envScale;
    const float *marg, *cond;
    const uint16_t *margGuide, *condGuide;  // guide tables of the CDFs (null: rows wider than 65,535)
    const float *rowProb, *colProb, *aliasPdf;
    const uint32_t *rowAlias, *colAlias;
    // volumes
    const pt_volume *vols;
    const DevGrid *dens, *maj;  // per volume; w == 0: none
    uint32_t numVols;
    // sampler tables
    const uint32_t *sobol1;     // 4 x 256 GF(2) product table of Sobol dimension 1
    // material textures: RGBA8 mip chains, sRGB decode table
    const struct DevTexture *tex;
    const uchar4 *texels;
    const float *srgbLut;       // 256 entries: sRGB-encoded byte -> linear
    uint32_t numTex;
    uint32_t hasAlpha;          // any alpha-mapped mesh (alpha-tested triangles)
    uint32_t hasSubsurface;     // any subsurface (type 6) mesh: shading traces its walks inline
    uint32_t mediaWavefront;    // media, all homogeneous, no subsurface: free flights in the closest-hit
                                // kernel, medium events as their own shading class, NEE deferred
    uint32_t mediaTrDeferred;   // heterogeneous media in the wavefront (on request): the medium
                                // transmittance of an NEE ray is estimated in the shadow kernel, only
                                // when the ray is unoccluded, from its own random stream
};

// One texture's mip chain in DevScene::texels (level l: max(w >> l, 1) x
// max(h >> l, 1) texels starting at off[l]).
constexpr int kMaxTexLevels = 16;
struct DevTexture {
    uint32_t w, h, levels, srgb;
    uint32_t off[kMaxTexLevels];
};

// ---------------------------------------------------------------------------
// sampler (shaders/RNG.hlsli:80-99)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float next_float(Rng &r, const uint32_t *__restrict__ tab) {
    if (r.kind == PT_RNG_PCG_HASH) {
        r.dim++;
        r.white = pcg_hash(r.white);
        return u32_to_unit(r.white);
    }
    uint32_t d = r.dim++;
    uint32_t axis = d & 1u, pad = d >> 1u;
    uint32_t sIdx = owen(r.sampleIndex, pcg_hash(pad * 0x9e3779b9u + 1u));
    uint32_t s;
    if (axis == 0u) s = brev(sIdx);
    else s = __ldg(&tab[sIdx & 255u]) ^ __ldg(&tab[256u + ((sIdx >> 8) & 255u)]) ^
             __ldg(&tab[512u + ((sIdx >> 16) & 255u)]) ^ __ldg(&tab[768u + (sIdx >> 24)]);
    uint32_t v = owen(s, pcg_hash(r.pixelSeed + pad * 0x6c8e9cf5u + axis * 0x68bc21ebu));
    return u32_to_unit(v);
}

// ---------------------------------------------------------------------------
// geometry access (shaders/GeometryUtils.hlsli:44-113)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float3 ld3(const float *b, uint32_t i) {
    return make_float3(__ldg(b + 3 * i), __ldg(b + 3 * i + 1), __ldg(b + 3 * i + 2));
}
__device__ __forceinline__ void tri_vidx(const DevScene &S, uint32_t mesh, uint32_t prim, uint32_t &i0, uint32_t &i1,
                                         uint32_t &i2) {
    const pt_material &m = S.mats[mesh];
    uint32_t base = m.indexOffset + prim * 3u;
    i0 = m.vertexOffset + __ldg(S.idx + base);
    i1 = m.vertexOffset + __ldg(S.idx + base + 1);
    i2 = m.vertexOffset + __ldg(S.idx + base + 2);
}
__device__ __forceinline__ float3 geometric_normal(const DevScene &S, uint32_t i0, uint32_t i1, uint32_t i2) {
    float3 p0 = ld3(S.pos, i0), p1 = ld3(S.pos, i1), p2 = ld3(S.pos, i2);
    return normalize(cross(p1 - p0, p2 - p0));
}

// ---------------------------------------------------------------------------
// envmap (shaders/Envmap.hlsli); bilinear with wrap U / clamp V
// (sampler s1 of src/gpu/DXRApp_Pipeline.cpp:56-61), texel centres at i+0.5
// ---------------------------------------------------------------------------
__device__ __forceinline__ float3 env_bilinear(const DevScene &S, float u, float v) {
    const int W = (int)S.envW, H = (int)S.envH;
    float x = u * (float)W - 0.5f, y = v * (float)H - 0.5f;
    float fx0 = floorf(x), fy0 = floorf(y);
    float fx = x - fx0, fy = y - fy0;
    int x0 = (int)fx0, y0 = (int)fy0;
    int xa = ((x0 % W) + W) % W, xb = (((x0 + 1) % W) + W) % W;
    int ya = min(max(y0, 0), H - 1), yb = min(max(y0 + 1, 0), H - 1);
    float4 a = __ldg(&S.env[(size_t)ya * W + xa]), b = __ldg(&S.env[(size_t)ya * W + xb]);
    float4 c = __ldg(&S.env[(size_t)yb * W + xa]), d = __ldg(&S.env[(size_t)yb * W + xb]);
    float3 top = make_float3(a.x, a.y, a.z) * (1.0f - fx) + make_float3(b.x, b.y, b.z) * fx;
    float3 bot = make_float3(c.x, c.y, c.z) * (1.0f - fx) + make_float3(d.x, d.y, d.z) * fx;
    return top * (1.0f - fy) + bot * fy;
}
__device__ __forceinline__ void dir_to_uv(float3 dir, float &u, float &v, float &sinTheta) {
    float3 d = normalize(dir);
    float phi = atan2f(d.z, d.x);
    if (phi < 0.0f) phi += 2.0f * kPi;
    float theta = acosf(clampf(d.y, -1.0f, 1.0f));
    sinTheta = sinf(theta);
    u = phi / (2.0f * kPi);
    v = theta / kPi;
}
__device__ __forceinline__ float3 eval_env(const DevScene &S, float3 dir) {  // Envmap.hlsli:15-24
    float u, v, st;
    dir_to_uv(dir, u, v, st);
    return env_bilinear(S, u, v) * S.envScale;
}
// The first index in [lo, hi) whose CDF value exceeds u, else hi.
__device__ __forceinline__ uint32_t cdf_upper(const float *buf, uint32_t lo, uint32_t hi, float u) {
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (__ldg(buf + mid) <= u) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ uint32_t cdf_search(const float *buf, uint32_t n, float u) {  // Envmap.hlsli:31-45
    return (uint32_t)max(0, (int)cdf_upper(buf, 0, n - 1, u) - 1);
}
// The same search narrowed by a guide table (Chen and Asau's cutpoint
// method): guide[k] = cdf_upper(buf, 0, n - 1, k / kCdfGuide) for k = 0 ..
// kCdfGuide.  For u in [k, k + 1) / kCdfGuide (exact: kCdfGuide is a power of
// two) the search result is monotone in u, so it lies in [guide[k],
// guide[k + 1]], and the loop over that range returns the same index as over
// the whole CDF; a few steps instead of log2(n).
constexpr uint32_t kCdfGuide = 256;
__device__ __forceinline__ uint32_t cdf_search_guided(const float *buf, const uint16_t *guide, float u) {
    const uint32_t k = min((uint32_t)(u * (float)kCdfGuide), kCdfGuide - 1u);
    return (uint32_t)max(0, (int)cdf_upper(buf, __ldg(guide + k), __ldg(guide + k + 1), u) - 1);
}
__device__ __forceinline__ float3 env_dir_from_uv(float u, float v, float &st) {
    float phi = 2.0f * kPi * u, theta = kPi * v;
    float ct;
    sincosf(theta, &st, &ct);
    float sp, cp;
    sincosf(phi, &sp, &cp);
    return make_float3(st * cp, ct, st * sp);
}
__device__ __forceinline__ void env_sample_cdf(const DevScene &S, float u1, float u2, float3 &dir, float3 &rad,
                                               float &pdf) {  // Envmap.hlsli:58-101
    const uint32_t W = S.envW, H = S.envH;
    uint32_t y = S.margGuide ? cdf_search_guided(S.marg, S.margGuide, u1) : cdf_search(S.marg, H + 1, u1);
    float m0 = __ldg(S.marg + y), m1 = __ldg(S.marg + y + 1);
    float pMar = m1 - m0;
    float jv = pMar > 1e-20f ? sat((u1 - m0) / pMar) : 0.5f;
    const float *row = S.cond + (size_t)y * (W + 1);
    uint32_t x = S.condGuide ? cdf_search_guided(row, S.condGuide + (size_t)y * (kCdfGuide + 1), u2)
                             : cdf_search(row, W + 1, u2);
    float c0 = __ldg(row + x), c1 = __ldg(row + x + 1);
    float pCon = c1 - c0;
    float ju = pCon > 1e-20f ? sat((u2 - c0) / pCon) : 0.5f;
    float u = ((float)x + ju) / (float)W;
    float v = ((float)y + jv) / (float)H;
    float st;
    dir = env_dir_from_uv(u, v, st);
    rad = env_bilinear(S, u, v) * S.envScale;
    pdf = pMar * pCon * (float)(W * H) / (2.0f * kPi * kPi * mx(st, 1e-8f));
}
__device__ __forceinline__ float env_pdf_cdf(const DevScene &S, float3 dir) {  // Envmap.hlsli:109-135
    const uint32_t W = S.envW, H = S.envH;
    float u, v, st;
    dir_to_uv(dir, u, v, st);
    uint32_t x = min((uint32_t)(u * (float)W), W - 1);
    uint32_t y = min((uint32_t)(v * (float)H), H - 1);
    float pMar = __ldg(S.marg + y + 1) - __ldg(S.marg + y);
    const float *row = S.cond + (size_t)y * (W + 1);
    float pCon = __ldg(row + x + 1) - __ldg(row + x);
    return pMar * pCon * (float)(W * H) / (2.0f * kPi * kPi * mx(st, 1e-8f));
}
// Alias-table form: O(1) row and column picks; the leftover fraction of each
// uniform is the in-texel jitter.  Density: the same lum * sin(theta) weights.
__device__ __forceinline__ uint32_t alias_pick(const float *prob, const uint32_t *alias, uint32_t n, float u,
                                               float &frac) {
    float sc = u * (float)n;
    uint32_t i = min((uint32_t)sc, n - 1);
    float f = sc - (float)i;
    float p = __ldg(prob + i);
    if (f < p) { frac = p > 0.0f ? f / p : 0.5f; return i; }
    frac = p < 1.0f ? (f - p) / (1.0f - p) : 0.5f;
    return __ldg(alias + i);
}
__device__ __forceinline__ void env_sample_alias(const DevScene &S, float u1, float u2, float3 &dir, float3 &rad,
                                                 float &pdf) {
    const uint32_t W = S.envW, H = S.envH;
    float jv, ju;
    uint32_t y = alias_pick(S.rowProb, S.rowAlias, H, u1, jv);
    uint32_t x = alias_pick(S.colProb + (size_t)y * W, S.colAlias + (size_t)y * W, W, u2, ju);
    float u = ((float)x + sat(ju)) / (float)W;
    float v = ((float)y + sat(jv)) / (float)H;
    float st;
    dir = env_dir_from_uv(u, v, st);
    rad = env_bilinear(S, u, v) * S.envScale;
    pdf = __ldg(S.aliasPdf + (size_t)y * W + x) / mx(st, 1e-8f);
}
__device__ __forceinline__ float env_pdf_alias(const DevScene &S, float3 dir) {
    const uint32_t W = S.envW, H = S.envH;
    float u, v, st;
    dir_to_uv(dir, u, v, st);
    uint32_t x = min((uint32_t)(u * (float)W), W - 1);
    uint32_t y = min((uint32_t)(v * (float)H), H - 1);
    return __ldg(S.aliasPdf + (size_t)y * W + x) / mx(st, 1e-8f);
}
__device__ __forceinline__ void env_sample(const DevScene &S, uint32_t mode, float u1, float u2, float3 &d, float3 &r,
                                           float &p) {
    if (mode == PT_ENV_ALIAS) env_sample_alias(S, u1, u2, d, r, p);
    else env_sample_cdf(S, u1, u2, d, r, p);
}
__device__ __forceinline__ float env_pdf(const DevScene &S, uint32_t mode, float3 d) {
    return mode == PT_ENV_ALIAS ? env_pdf_alias(S, d) : env_pdf_cdf(S, d);
}

// ---------------------------------------------------------------------------
// emitters (shaders/Emitter.hlsli:17-103)
// ---------------------------------------------------------------------------
struct EmitterSample {
    float3 pos, nrm, rad;
    float pdfArea;
    bool valid;
};
__device__ __forceinline__ EmitterSample sample_emitter(const DevScene &S, Rng &rng) {
    EmitterSample es;
    es.valid = false;
    if (S.emitterCount == 0) return es;
    uint32_t pick = min((uint32_t)(next_float(rng, S.sobol1) * float(S.emitterCount)), S.emitterCount - 1);
    uint32_t id = __ldg(S.emitterList + pick);
    const pt_material &m = S.mats[id];
    es.valid = true;
    es.rad = make_float3(m.radiance[0], m.radiance[1], m.radiance[2]);
    uint32_t nt = m.indexCount / 3u;
    float u = next_float(rng, S.sobol1);
    uint32_t tri = min(cdf_search(S.emitterCdf + m.emitterCdfOffset, nt + 1, u), nt - 1);
    uint32_t i0, i1, i2;
    tri_vidx(S, id, tri, i0, i1, i2);
    float3 p0 = ld3(S.pos, i0), p1 = ld3(S.pos, i1), p2 = ld3(S.pos, i2);
    float r1 = next_float(rng, S.sobol1), r2 = next_float(rng, S.sobol1);
    float sr1 = sqrtf(r1);
    es.pos = (1.0f - sr1) * p0 + sr1 * (1.0f - r2) * p1 + sr1 * r2 * p2;
    es.nrm = normalize(cross(p1 - p0, p2 - p0));
    es.pdfArea = 1.0f / (m.surfaceArea * float(S.emitterCount));
    return es;
}
__device__ __forceinline__ float emitter_pdf_sa(const DevScene &S, const pt_material &m, float3 hp, float3 sp, float3 n) {
    float3 d = hp - sp;
    float d2 = dot(d, d);
    if (d2 < 1e-12f) return 0.0f;
    float dist = sqrtf(d2);
    float cl = fabsf(dot(n, -d / v3(dist)));
    if (cl < 1e-8f) return 0.0f;
    return (1.0f / (m.surfaceArea * float(S.emitterCount))) * d2 / cl;
}

// ---------------------------------------------------------------------------
// volumes (shaders/Volume.hlsl)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float3 vsigma_t(const pt_volume &v) {
    return make_float3(v.sigma_a[0] + v.sigma_s[0], v.sigma_a[1] + v.sigma_s[1], v.sigma_a[2] + v.sigma_s[2]);
}
__device__ __forceinline__ float vsigma_t_max(const pt_volume &v) { return maxc(vsigma_t(v)); }
__device__ __forceinline__ bool ray_aabb(float3 o, float3 d, float3 bmin, float3 bmax, float &tn, float &tf) {
    float3 inv = make_float3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    float3 t0 = (bmin - o) * inv, t1 = (bmax - o) * inv;
    float3 a = vmin(t0, t1), b = vmax(t0, t1);
    tn = mx(mx(a.x, a.y), a.z);
    tf = mn(mn(b.x, b.y), b.z);
    return tf >= mx(tn, 0.0f);
}
// The null-collision walk branches on positions that land exactly on brick
// boundaries and on densities compared against uniforms, so the volume code
// uses uncontracted IEEE operations (the reference's order) throughout.
__device__ __forceinline__ float xmad(float a, float b, float c) { return __fadd_rn(__fmul_rn(a, b), c); }
__device__ __forceinline__ float3 xpos(float3 o, float3 d, float t) {
    return make_float3(__fadd_rn(o.x, __fmul_rn(d.x, t)), __fadd_rn(o.y, __fmul_rn(d.y, t)),
                       __fadd_rn(o.z, __fmul_rn(d.z, t)));
}
__device__ __forceinline__ float xlerp(float a, float b, float f) {
    return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, f)), __fmul_rn(b, f));
}
__device__ __forceinline__ float grid_trilinear(const DevGrid &g, float u, float v, float w) {  // sampler s2: clamp
    float x = __fsub_rn(__fmul_rn(u, (float)g.w), 0.5f), y = __fsub_rn(__fmul_rn(v, (float)g.h), 0.5f),
          z = __fsub_rn(__fmul_rn(w, (float)g.d), 0.5f);
    float fx0 = floorf(x), fy0 = floorf(y), fz0 = floorf(z);
    float fx = x - fx0, fy = y - fy0, fz = z - fz0;
    int x0 = (int)fx0, y0 = (int)fy0, z0 = (int)fz0;
    int W = g.w, H = g.h, D = g.d;
    int xa = min(max(x0, 0), W - 1), xb = min(max(x0 + 1, 0), W - 1);
    int ya = min(max(y0, 0), H - 1), yb = min(max(y0 + 1, 0), H - 1);
    int za = min(max(z0, 0), D - 1), zb = min(max(z0 + 1, 0), D - 1);
    auto at = [&](int xx, int yy, int zz) { return __ldg(g.data + (size_t)xx + (size_t)W * (yy + (size_t)H * zz)); };
    float c00 = xlerp(at(xa, ya, za), at(xb, ya, za), fx);
    float c10 = xlerp(at(xa, yb, za), at(xb, yb, za), fx);
    float c01 = xlerp(at(xa, ya, zb), at(xb, ya, zb), fx);
    float c11 = xlerp(at(xa, yb, zb), at(xb, yb, zb), fx);
    float c0 = xlerp(c00, c10, fy), c1 = xlerp(c01, c11, fy);
    return xlerp(c0, c1, fz);
}
__device__ __forceinline__ float vol_density(const DevScene &S, uint32_t vi, float3 p) {  // Volume.hlsl:98-105
    const pt_volume &v = S.vols[vi];
    if (!(v.flags & PT_VOLUME_HETEROGENEOUS) || S.dens[vi].w == 0) return 1.0f;
    float3 vmn = make_float3(v.vmin[0], v.vmin[1], v.vmin[2]), vmxx = make_float3(v.vmax[0], v.vmax[1], v.vmax[2]);
    float3 uvw = (p - vmn) / vmax(vmxx - vmn, v3(1e-6f));
    return grid_trilinear(S.dens[vi], uvw.x, uvw.y, uvw.z);
}
__device__ __forceinline__ void local_majorant(const DevScene &S, uint32_t vi, float3 pos, float3 dir, float &mu,
                                               float &bd) {  // Volume.hlsl:119-164
    const pt_volume &v = S.vols[vi];
    float gmu = vsigma_t_max(v);
    const DevGrid &m = S.maj[vi];
    if (m.w == 0) { mu = gmu; bd = 1e20f; return; }
    float3 mres = make_float3((float)m.w, (float)m.h, (float)m.d);
    float3 vmn = make_float3(v.vmin[0], v.vmin[1], v.vmin[2]), vmxx = make_float3(v.vmax[0], v.vmax[1], v.vmax[2]);
    float3 size = vmax(vmxx - vmn, v3(1e-6f));
    float3 bws = size / mres;
    float3 bf = (pos - vmn) / size * mres;
    int bc[3];
    int res[3] = {(int)m.w, (int)m.h, (int)m.d};
    for (int i = 0; i < 3; i++) bc[i] = min(max((int)get(bf, i), 0), res[i] - 1);
    mu = __ldg(m.data + (size_t)bc[0] + (size_t)m.w * (bc[1] + (size_t)m.h * bc[2])) * gmu;
    float dv[3];
    for (int i = 0; i < 3; i++) {
        float di = get(dir, i);
        if (fabsf(di) < 1e-20f) dv[i] = 1e20f;
        else {
            float ne = (float)bc[i] + (di > 0.0f ? 1.0f : 0.0f);
            float we = __fadd_rn(get(vmn, i), __fmul_rn(ne, get(bws, i)));
            dv[i] = mx((we - get(pos, i)) / di, 1e-5f);
        }
    }
    bd = mn(dv[0], mn(dv[1], dv[2]));
}
struct Seg { uint32_t vi; float tn, tf; };
__device__ __forceinline__ uint32_t enumerate_segments(const DevScene &S, float3 o, float3 d, float tmax, Seg segs[8]) {
    uint32_t count = 0;
    for (uint32_t i = 0; i < S.numVols && count < 8; i++) {
        const pt_volume &v = S.vols[i];
        float tn, tf;
        if (!ray_aabb(o, d, make_float3(v.vmin[0], v.vmin[1], v.vmin[2]), make_float3(v.vmax[0], v.vmax[1], v.vmax[2]),
                      tn, tf))
            continue;
        tn = mx(tn, 0.0f);
        tf = mn(tf, tmax);
        if (tf <= tn) continue;
        uint32_t p = count;
        for (; p > 0; p--) {
            if (segs[p - 1].tn <= tn) break;
            segs[p] = segs[p - 1];
        }
        segs[p].vi = i; segs[p].tn = tn; segs[p].tf = tf;
        count++;
    }
    return count;
}
__device__ inline bool null_collision(const DevScene &S, uint32_t vi, float3 o, float3 d, float tn, float tf, Rng &rng,
                               float3 &w, float &ts) {  // Volume.hlsl:236-319
    const pt_volume &v = S.vols[vi];
    float gmu = vsigma_t_max(v);
    float3 stv = vsigma_t(v);
    float t = tn;
    for (uint32_t step = 0; step < 512; step++) {
        float3 pos = xpos(o, d, t);
        float lmu, bd;
        local_majorant(S, vi, pos, d, lmu, bd);
        if (lmu < 1e-8f) {
            t += bd;
            if (t >= tf) { ts = tf; return false; }
            continue;
        }
        float xi = mx(next_float(rng, S.sobol1), 1e-10f);
        float dt = -logf(xi) / lmu;
        if (dt > bd) {
            t += bd;
            if (t >= tf) { ts = tf; return false; }
            continue;
        }
        t += dt;
        if (t >= tf) { ts = tf; return false; }
        float dens = vol_density(S, vi, xpos(o, d, t));
        float pr = sat((dens * gmu) / mx(lmu, 1e-20f));
        if (pr >= 1.0f - 1e-6f || next_float(rng, S.sobol1) < pr) {
            w = w * (stv / v3(mx(gmu, 1e-20f)));
            ts = t;
            return true;
        }
        float3 sn = make_float3(__fsub_rn(lmu, __fmul_rn(dens, stv.x)), __fsub_rn(lmu, __fmul_rn(dens, stv.y)),
                                __fsub_rn(lmu, __fmul_rn(dens, stv.z)));
        w = w * (sn / v3(mx(lmu * (1.0f - pr), 1e-20f)));
    }
    ts = tf;
    return false;
}
__device__ inline float3 ratio_tracking(const DevScene &S, uint32_t vi, float3 o, float3 d, float tn, float tf, Rng &rng) {
    const pt_volume &v = S.vols[vi];  // Volume.hlsl:326-372
    float3 stv = vsigma_t(v);
    float3 tr = v3(1.0f);
    float t = tn;
    for (uint32_t step = 0; step < 512; step++) {
        float3 pos = xpos(o, d, t);
        float lmu, bd;
        local_majorant(S, vi, pos, d, lmu, bd);
        if (lmu < 1e-8f) {
            t += bd;
            if (t >= tf) return tr;
            continue;
        }
        float xi = mx(next_float(rng, S.sobol1), 1e-10f);
        float dt = -logf(xi) / lmu;
        if (dt > bd) {
            t += bd;
            if (t >= tf) return tr;
            continue;
        }
        t += dt;
        if (t >= tf) return tr;
        float dens = vol_density(S, vi, xpos(o, d, t));
        float3 sn = make_float3(__fsub_rn(lmu, __fmul_rn(dens, stv.x)), __fsub_rn(lmu, __fmul_rn(dens, stv.y)),
                                __fsub_rn(lmu, __fmul_rn(dens, stv.z)));
        tr = tr * (sn / v3(mx(lmu, 1e-20f)));
        if (maxc(tr) < 1e-6f) return v3(0.0f);
    }
    return tr;
}
__device__ inline bool sample_free_flight(const DevScene &S, float3 o, float3 d, float tmax, Rng &rng, float3 &w, float &ts,
                                   uint32_t &svi) {  // Volume.hlsl:381-415
    ts = tmax;
    svi = 0;
    if (S.numVols == 0) return false;
    Seg segs[8];
    uint32_t c = enumerate_segments(S, o, d, tmax, segs);
    for (uint32_t k = 0; k < c; k++) {
        if (vsigma_t_max(S.vols[segs[k].vi]) < 1e-8f) continue;
        float th;
        if (null_collision(S, segs[k].vi, o, d, segs[k].tn, segs[k].tf, rng, w, th)) {
            ts = th;
            svi = segs[k].vi;
            return true;
        }
    }
    return false;
}
__device__ inline float3 multi_volume_tr(const DevScene &S, float3 o, float3 d, float tmax, Rng &rng) {  // Volume.hlsl:419-454
    if (S.numVols == 0) return v3(1.0f);
    Seg segs[8];
    uint32_t c = enumerate_segments(S, o, d, tmax, segs);
    float3 tr = v3(1.0f);
    for (uint32_t k = 0; k < c; k++) {
        const pt_volume &v = S.vols[segs[k].vi];
        float3 st = vsigma_t(v);
        if (maxc(st) < 1e-8f) continue;
        float3 seg;
        if (v.flags & PT_VOLUME_HETEROGENEOUS) seg = ratio_tracking(S, segs[k].vi, o, d, segs[k].tn, segs[k].tf, rng);
        else seg = vexp(-st * (segs[k].tf - segs[k].tn));
        tr = tr * seg;
        if (maxc(tr) < 1e-6f) return v3(0.0f);
    }
    return tr;
}

// ---------------------------------------------------------------------------
// material textures: trilinear, wrap in u and v (sampler s0 of
// src/gpu/DXRApp_Pipeline.cpp:49-53), texel centres at i + 0.5; sRGB texels
// are decoded to linear before filtering, as an _SRGB format is
// ---------------------------------------------------------------------------
__device__ __forceinline__ float4 tex_texel(const DevScene &S, const DevTexture &t, uint32_t level, int W, int x,
                                            int y) {
    uchar4 c = __ldg(&S.texels[t.off[level] + (uint32_t)y * (uint32_t)W + (uint32_t)x]);
    if (t.srgb)
        return make_float4(__ldg(S.srgbLut + c.x), __ldg(S.srgbLut + c.y), __ldg(S.srgbLut + c.z),
                           (float)c.w / 255.0f);
    return make_float4((float)c.x / 255.0f, (float)c.y / 255.0f, (float)c.z / 255.0f, (float)c.w / 255.0f);
}
__device__ __forceinline__ float4 lerp4(float4 a, float4 b, float t) {
    return make_float4(a.x + (b.x - a.x) * t, a.y + (b.y - a.y) * t, a.z + (b.z - a.z) * t, a.w + (b.w - a.w) * t);
}
__device__ __forceinline__ float4 tex_bilinear(const DevScene &S, const DevTexture &t, uint32_t level, float u,
                                               float v) {
    const int W = (int)max(t.w >> level, 1u), H = (int)max(t.h >> level, 1u);
    u -= floorf(u);
    v -= floorf(v);
    float x = u * (float)W - 0.5f, y = v * (float)H - 0.5f;
    float fx0 = floorf(x), fy0 = floorf(y);
    float fx = x - fx0, fy = y - fy0;
    int x0 = (int)fx0, y0 = (int)fy0;
    int xa = ((x0 % W) + W) % W, xb = (((x0 + 1) % W) + W) % W;
    int ya = ((y0 % H) + H) % H, yb = (((y0 + 1) % H) + H) % H;
    float4 top = lerp4(tex_texel(S, t, level, W, xa, ya), tex_texel(S, t, level, W, xb, ya), fx);
    float4 bot = lerp4(tex_texel(S, t, level, W, xa, yb), tex_texel(S, t, level, W, xb, yb), fx);
    return lerp4(top, bot, fy);
}
// SampleLevel(g_sampler, uv, lod): linear between the two nearest mip levels.
__device__ __forceinline__ float4 tex_sample(const DevScene &S, uint32_t index, float u, float v, float lod) {
    const DevTexture &t = S.tex[index];
    lod = fminf(fmaxf(lod, 0.0f), (float)(t.levels - 1));
    uint32_t l0 = (uint32_t)floorf(lod);
    float f = lod - (float)l0;
    float4 a = tex_bilinear(S, t, l0, u, v);
    if (f > 0.0f && l0 + 1 < t.levels) a = lerp4(a, tex_bilinear(S, t, l0 + 1, u, v), f);
    return a;
}
// ComputeUVFootprint (shaders/GeometryUtils.hlsli:120-145): world-space pixel
// footprint at distance hitT mapped to UV space by the triangle's UV/world
// area ratio.
__device__ __forceinline__ float uv_footprint(const DevScene &S, uint32_t mesh, uint32_t prim, float hitT,
                                              uint32_t width, uint32_t height) {
    uint32_t i0, i1, i2;
    tri_vidx(S, mesh, prim, i0, i1, i2);
    float3 p0 = ld3(S.pos, i0), p1 = ld3(S.pos, i1), p2 = ld3(S.pos, i2);
    float u0 = __ldg(S.uv + 2 * i0), v0 = __ldg(S.uv + 2 * i0 + 1);
    float u1 = __ldg(S.uv + 2 * i1), v1 = __ldg(S.uv + 2 * i1 + 1);
    float u2 = __ldg(S.uv + 2 * i2), v2 = __ldg(S.uv + 2 * i2 + 1);
    float worldArea = 0.5f * len(cross(p1 - p0, p2 - p0));
    float uvArea = 0.5f * fabsf((u1 - u0) * (v2 - v0) - (u2 - u0) * (v1 - v0));
    if (worldArea < 1e-12f || uvArea < 1e-12f) return 0.0f;
    float pixelAngle = 1.0f / (float)max(width, height);
    return hitT * pixelAngle * sqrtf(uvArea / worldArea);
}
// ComputeTexLOD (shaders/GeometryUtils.hlsli:148-154).
__device__ __forceinline__ float tex_lod(const DevScene &S, uint32_t index, float footprint) {
    const DevTexture &t = S.tex[index];
    float texelsPerPixel = footprint * (float)max(t.w, t.h);
    return fmaxf(log2f(fmaxf(texelsPerPixel, 1.0f)), 0.0f);
}
__device__ __forceinline__ float2 interp_uv(const DevScene &S, uint32_t i0, uint32_t i1, uint32_t i2, float b1,
                                            float b2) {
    float w0 = 1.0f - b1 - b2;
    return make_float2(__ldg(S.uv + 2 * i0) * w0 + __ldg(S.uv + 2 * i1) * b1 + __ldg(S.uv + 2 * i2) * b2,
                       __ldg(S.uv + 2 * i0 + 1) * w0 + __ldg(S.uv + 2 * i1 + 1) * b1 + __ldg(S.uv + 2 * i2 + 1) * b2);
}

// Stochastic alpha test of an alpha-mapped candidate hit (PrimaryAnyHit /
// ShadowAnyHit of shaders/RayQueryTrace.hlsli:50-62,100-112): alpha from
// mip level 0 (closest hit: .r; shadow: .a when below 1, else .r), ignored
// below 0.01, kept with probability alpha^2.  The reference draws the
// uniform from a PCG stream threaded through the candidates in hardware
// traversal order; here it is a hash of (path seed, ray key, triangle), so
// the decision for a candidate does not depend on the order in which a
// traversal meets the candidates.
__device__ __forceinline__ bool alpha_pass(const DevScene &S, uint32_t gid, float b1, float b2, uint32_t seed,
                                           uint32_t key, bool shadow) {
    uint32_t mesh = __ldg(S.triMesh + gid);
    uint32_t prim = gid - __ldg(S.meshFirstTri + mesh);
    uint32_t i0, i1, i2;
    tri_vidx(S, mesh, prim, i0, i1, i2);
    float2 uv = interp_uv(S, i0, i1, i2, b1, b2);
    float4 c = tex_sample(S, __ldg(&S.mats[mesh].alphaTexIndex), uv.x, uv.y, 0.0f);
    float a = shadow ? (c.w < 1.0f ? c.w : c.x) : c.x;
    if (a < 0.01f) return false;
    float xi = u32_to_unit(pcg_hash(seed ^ pcg_hash(key * 0x9e3779b9u ^ gid)));
    return !(a * a < xi);
}
// Per-path seed of the alpha tests, fixed for the path: the sampler's pixel
// seed and sample index.
__device__ __forceinline__ uint32_t alpha_seed(uint32_t pixelSeed, uint32_t sample) {
    return pcg_hash(pixelSeed * 0x85ebca6bu ^ pcg_hash(sample + 0x27d4eb2fu));
}
// Ray keys: extension ray of bounce b, area / envmap NEE shadow ray of bounce b.
__device__ __forceinline__ uint32_t alpha_key(uint32_t bounce, uint32_t kind) { return bounce * 4u + kind; }

// ---------------------------------------------------------------------------
// BVH8 traversal
// ---------------------------------------------------------------------------
constexpr int kTraversalStack = 32;

struct Hit {
    float t, u, v;
    uint32_t gid;  // 0xFFFFFFFF: miss
};

// Moller-Trumbore (src/cpu/mesh.cpp:51-89) on (v0, e1, e2).
// Moller-Trumbore with fused multiply-adds in one fixed order, the order
// the oracle (and the reference build's ray-query stand-in) evaluates it:
// a*b - c*d as fma(a, b, -(c*d)), dot products as fma(z, z', fma(y, y',
// x*x')).  Explicit intrinsics, so the compiler contracts nothing else: the
// decision and t, u, v are the oracle's bit for bit, and hit ids differ only
// where traversal order breaks an equal-t tie or a ray grazes a box.
__device__ __forceinline__ float dot_f(float3 a, float3 b) {
    return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, __fmul_rn(a.x, b.x)));
}
__device__ __forceinline__ float3 cross_f(float3 a, float3 b) {
    return make_float3(__fmaf_rn(a.y, b.z, -__fmul_rn(a.z, b.y)), __fmaf_rn(a.z, b.x, -__fmul_rn(a.x, b.z)),
                       __fmaf_rn(a.x, b.y, -__fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ bool tri_test(float3 o, float3 d, float4 a, float4 b, float4 c, float tmin, float tmax,
                                         float &t, float &u, float &v) {
    float3 e1 = make_float3(b.x, b.y, b.z), e2 = make_float3(c.x, c.y, c.z);
    float3 pv = cross_f(d, e2);
    float det = dot_f(e1, pv);
    if (det > -1e-8f && det < 1e-8f) return false;
    float inv = __frcp_rn(det);  // correctly rounded: the value of 1.0f / det
    float3 tv = o - make_float3(a.x, a.y, a.z);
    u = __fmul_rn(dot_f(tv, pv), inv);
    if (u < 0.0f || u > 1.0f) return false;
    float3 qv = cross_f(tv, e1);
    v = __fmul_rn(dot_f(d, qv), inv);
    if (v < 0.0f || __fadd_rn(u, v) > 1.0f) return false;
    t = __fmul_rn(dot_f(e2, qv), inv);
    return t >= tmin && t <= tmax;
}

struct RayPre {
    float3 o, d, idir;
    uint32_t oct;
};
__device__ __forceinline__ RayPre ray_pre(float3 o, float3 d) {
    RayPre r;
    r.o = o;
    r.d = d;
    const float eps = 8.271806125530277e-25f;  // 2^-80: keeps 1/d finite
    r.idir = make_float3(1.0f / (fabsf(d.x) > eps ? d.x : copysignf(eps, d.x)),
                         1.0f / (fabsf(d.y) > eps ? d.y : copysignf(eps, d.y)),
                         1.0f / (fabsf(d.z) > eps ? d.z : copysignf(eps, d.z)));
    r.oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
    return r;
}
__device__ __forceinline__ uint32_t byte_of(uint32_t w, uint32_t i) { return (w >> (8u * i)) & 0xFFu; }
// Byte `i` of w as a float, exactly (float)byte: one byte permute builds the
// bits of 2^23 + byte (exponent 0x4B, byte in the low mantissa bits) and an
// exact subtraction removes 2^23.  Runs on the ALU and FMA pipes instead of
// the conversion unit.
__device__ __forceinline__ float byte_as_float(uint32_t w, uint32_t i) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7540u | i)) - 8388608.0f;
}

// Three-input float max / min (PTX 8.8, sm_100): the same value as two
// chained fmaxf / fminf in one ALU instruction.
__device__ __forceinline__ float fmax3(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float fmin3(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// Intersect the 8 children of node `ni`: internal hits (in near-to-far visit
// order, bit k = slot k ^ oct) into gHits, triangle hits into tHits.
__device__ __forceinline__ void intersect_node(const DevScene &S, uint32_t ni, const RayPre &r, float tmin, float tmax,
                                               uint32_t &gBase, uint32_t &gImask, uint32_t &gHits, uint32_t &tBase,
                                               uint32_t &tHits) {
    const uint4 *np = S.nodes[ni].n;
    uint4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2), n3 = __ldg(np + 3), n4 = __ldg(np + 4);
    float px = __uint_as_float(n0.x), py = __uint_as_float(n0.y), pz = __uint_as_float(n0.z);
    uint32_t ex = n0.w & 0xFFu, ey = (n0.w >> 8) & 0xFFu, ez = (n0.w >> 16) & 0xFFu;
    float sx = __uint_as_float(ex << 23) * r.idir.x;
    float sy = __uint_as_float(ey << 23) * r.idir.y;
    float sz = __uint_as_float(ez << 23) * r.idir.z;
    float ox = (px - r.o.x) * r.idir.x, oy = (py - r.o.y) * r.idir.y, oz = (pz - r.o.z) * r.idir.z;
    gBase = n1.x;
    tBase = n1.y;
    gImask = n0.w >> 24;
    // internal children (meta bits 3 and 4 set: position >= 24) take their
    // position XOR the ray octant, four meta bytes at a time
    uint32_t oct4 = r.oct * 0x01010101u;
    uint32_t ma = n1.z ^ (((n1.z >> 3) & (n1.z >> 4) & 0x01010101u) * 7u & oct4);
    uint32_t mb = n1.w ^ (((n1.w >> 3) & (n1.w >> 4) & 0x01010101u) * 7u & oct4);
    uint32_t hits = 0;
    // near/far plane words per axis by ray sign
    uint32_t lxa = n2.x, lxb = n2.y, hxa = n3.z, hxb = n3.w;
    uint32_t lya = n2.z, lyb = n2.w, hya = n4.x, hyb = n4.y;
    uint32_t lza = n3.x, lzb = n3.y, hza = n4.z, hzb = n4.w;
    if (r.idir.x < 0.0f) { uint32_t t0 = lxa, t1 = lxb; lxa = hxa; lxb = hxb; hxa = t0; hxb = t1; }
    if (r.idir.y < 0.0f) { uint32_t t0 = lya, t1 = lyb; lya = hya; lyb = hyb; hya = t0; hyb = t1; }
    if (r.idir.z < 0.0f) { uint32_t t0 = lza, t1 = lzb; lza = hza; lzb = hzb; hza = t0; hzb = t1; }
#pragma unroll
    for (uint32_t i = 0; i < 8; i++) {
        uint32_t sel = i & 3u;
        // x and y planes through the conversion unit, z through byte_as_float:
        // both exact; the split balances the ALU, FMA and XU pipes (measured
        // on B200: all-ALU and all-XU decodes are both slower)
        float tnx = fmaf((float)byte_of(i < 4 ? lxa : lxb, sel), sx, ox);
        float tfx = fmaf((float)byte_of(i < 4 ? hxa : hxb, sel), sx, ox);
        float tny = fmaf((float)byte_of(i < 4 ? lya : lyb, sel), sy, oy);
        float tfy = fmaf((float)byte_of(i < 4 ? hya : hyb, sel), sy, oy);
        float tnz = fmaf(byte_as_float(i < 4 ? lza : lzb, sel), sz, oz);
        float tfz = fmaf(byte_as_float(i < 4 ? hza : hzb, sel), sz, oz);
        float t0 = fmax3(tnx, tny, fmaxf(tnz, tmin));
        float t1 = fmin3(tfx, tfy, fminf(tfz, tmax));
        uint32_t meta = byte_of(i < 4 ? ma : mb, sel);
        if (t0 <= t1 * 1.00000024f) hits |= (meta >> 5) << (meta & 31u);
    }
    gHits = hits >> 24;
    tHits = hits & 0x00FFFFFFu;
}

// Resumable traversal state: the kernels with per-lane ray replacement run
// it one node at a time; trace_closest / trace_shadow run it to the end.
// The node stack is a separate object: indexed at run time, it lives in
// local memory, and must not drag the scalar state there with it.
struct Trav {
    RayPre r;
    float tmin, tmax;
    uint32_t seed, key;  // alpha tests: path seed and ray key
    uint32_t gBase, gImask, gHits, tBase, tHits;
    uint32_t visits;
    int sp;
};
// An entry is (child base, internal mask << 8 | pending hit bits).
struct TravStack {  // all entries in local memory
    uint32_t base[kTraversalStack], mask[kTraversalStack];
    __device__ __forceinline__ void put(int i, uint32_t b, uint32_t m) { base[i] = b; mask[i] = m; }
    __device__ __forceinline__ uint2 get(int i) const { return make_uint2(base[i], mask[i]); }
};
// The first SH entries in shared memory, the rest in local memory.  `col`
// is this thread's column of a block-wide [SH][STRIDE] uint2 array: entry i
// of the block's threads lies in consecutive words (no bank conflicts).
template <int SH, int STRIDE>
struct SplitStack {
    uint2 *col;
    uint2 spill[kTraversalStack - SH];
    __device__ __forceinline__ void put(int i, uint32_t b, uint32_t m) {
        if (i < SH) col[i * STRIDE] = make_uint2(b, m);
        else spill[i - SH] = make_uint2(b, m);
    }
    __device__ __forceinline__ uint2 get(int i) const { return i < SH ? col[i * STRIDE] : spill[i - SH]; }
};
__device__ __forceinline__ void trav_init(Trav &T, const DevScene &S, float3 o, float3 d, float tmin, float tmax,
                                          uint32_t seed = 0u, uint32_t key = 0u) {
    T.r = ray_pre(o, d);
    T.tmin = tmin;
    T.tmax = tmax;
    T.seed = seed;
    T.key = key;
    T.sp = 0;
    T.visits = 1;
    T.gHits = T.tHits = 0;
    if (S.numNodes) intersect_node(S, 0, T.r, tmin, tmax, T.gBase, T.gImask, T.gHits, T.tBase, T.tHits);
}
// Next node: pop the nearest pending child (from this node or the stack) and
// intersect it.  Returns false when nothing is left (or on an error, which
// is flagged in *err).
template <class Stack>
__device__ __forceinline__ bool trav_next_node(Trav &T, Stack &K, const DevScene &S, float tmax, uint32_t *err) {
    if (T.gHits == 0) {
        if (T.sp == 0) return false;
        --T.sp;
        const uint2 e = K.get(T.sp);
        T.gBase = e.x;
        T.gImask = e.y >> 8;
        T.gHits = e.y & 0xFFu;
    }
    uint32_t k = __ffs(T.gHits) - 1;
    T.gHits &= T.gHits - 1;
    uint32_t slot = k ^ T.r.oct;
    uint32_t child = T.gBase + __popc(T.gImask & ((1u << slot) - 1u));
    if (++T.visits > S.numNodes || child >= S.numNodes) {
        if (err) atomicOr(err, 4u);
        return false;
    }
    if (T.gHits) {
        if (T.sp == kTraversalStack) {
            if (err) atomicOr(err, 1u);
            return false;
        }
        K.put(T.sp, T.gBase, (T.gImask << 8) | T.gHits);
        ++T.sp;
    }
    intersect_node(S, child, T.r, T.tmin, tmax, T.gBase, T.gImask, T.gHits, T.tBase, T.tHits);
    return true;
}
// Closest-hit step: the current node's triangles, then the next node.
// Returns true when the traversal has finished.
template <class Stack>
__device__ __forceinline__ bool trav_step_closest(Trav &T, Stack &K, const DevScene &S, Hit &h, uint32_t *err) {
    while (T.tHits) {
        uint32_t j = __ffs(T.tHits) - 1;
        T.tHits &= T.tHits - 1;
        const float4 *tp = S.tri + 3u * (T.tBase + j);
        float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
        float t, u, v;
        if (tri_test(T.r.o, T.r.d, a, b, c, T.tmin, h.t, t, u, v)) {
            uint32_t g = __float_as_uint(a.w);
            if (t < h.t || (t == h.t && g < h.gid)) {
                // b.w != 0: the triangle's material has an alpha map
                if (__float_as_uint(b.w) && !alpha_pass(S, g, u, v, T.seed, T.key, false)) continue;
                h.t = t; h.u = u; h.v = v; h.gid = g;
            }
        }
    }
    return !trav_next_node(T, K, S, h.t, err);
}
// Any-hit step (shadow rays).  Sets `occluded` and returns true at the first
// opaque hit; mirror/dielectric hits multiply `trans` by (1 - Fr).
template <class Stack>
__device__ __forceinline__ bool trav_step_shadow(Trav &T, Stack &K, const DevScene &S, float3 &trans,
                                                 bool &occluded, uint32_t *err) {
    while (T.tHits) {
        uint32_t j = __ffs(T.tHits) - 1;
        T.tHits &= T.tHits - 1;
        const float4 *tp = S.tri + 3u * (T.tBase + j);
        float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
        float t, u, v;
        if (tri_test(T.r.o, T.r.d, a, b, c, T.tmin, T.tmax, t, u, v)) {
            uint32_t g = __float_as_uint(a.w);
            if (__float_as_uint(b.w)) {  // alpha-mapped: occludes when the stochastic test keeps it
                if (alpha_pass(S, g, u, v, T.seed, T.key, true)) { occluded = true; return true; }
                continue;
            }
            if (!S.hasGlass) { occluded = true; return true; }
            uint32_t mesh = __ldg(S.triMesh + g);
            const pt_material &m = S.mats[mesh];
            if (m.type != PT_MAT_MIRROR && m.type != PT_MAT_DIELECTRIC) { occluded = true; return true; }
            float3 Ng = normalize(cross(make_float3(b.x, b.y, b.z), make_float3(c.x, c.y, c.z)));
            float Fr = fresnel(fabsf(dot(T.r.d, Ng)), m.extIOR, m.intIOR);
            trans = trans * (1.0f - Fr);
        }
    }
    return !trav_next_node(T, K, S, T.tmax, err);
}

// Closest hit (TraceClosestInline semantics for opaque geometry).  Sets *err
// on stack overflow or a runaway visit count.
template <class Stack>
__device__ __forceinline__ Hit trace_closest_on(Stack &K, const DevScene &S, float3 o, float3 d, float tmin,
                                                float tmax, uint32_t *err, uint32_t seed = 0u, uint32_t key = 0u) {
    Hit h;
    h.t = tmax; h.u = 0.0f; h.v = 0.0f; h.gid = 0xFFFFFFFFu;
    if (S.numNodes == 0) return h;
    Trav T;
    trav_init(T, S, o, d, tmin, tmax, seed, key);
    while (!trav_step_closest(T, K, S, h, err)) {
    }
    return h;
}
__device__ __forceinline__ Hit trace_closest(const DevScene &S, float3 o, float3 d, float tmin, float tmax,
                                             uint32_t *err, uint32_t seed = 0u, uint32_t key = 0u) {
    TravStack K;
    return trace_closest_on(K, S, o, d, tmin, tmax, err, seed, key);
}

// Occlusion (TraceShadowInline, shaders/RayQueryTrace.hlsli:88-129, for
// scenes without alpha textures): the first opaque hit in [tmin, tmax]
// occludes; mirror/dielectric surfaces multiply `trans` by (1 - Fr).
template <class Stack>
__device__ __forceinline__ bool trace_shadow_on(Stack &K, const DevScene &S, float3 o, float3 d, float tmin,
                                                float tmax, float3 &trans, uint32_t *err, uint32_t seed = 0u,
                                                uint32_t key = 0u) {
    trans = v3(1.0f);
    if (S.numNodes == 0) return false;
    Trav T;
    trav_init(T, S, o, d, tmin, tmax, seed, key);
    bool occ = false;
    while (!trav_step_shadow(T, K, S, trans, occ, err)) {
    }
    return occ;
}
__device__ __forceinline__ bool trace_shadow(const DevScene &S, float3 o, float3 d, float tmin, float tmax,
                                             float3 &trans, uint32_t *err, uint32_t seed = 0u, uint32_t key = 0u) {
    TravStack K;
    return trace_shadow_on(K, S, o, d, tmin, tmax, trans, err, seed, key);
}

}  // namespace pt
