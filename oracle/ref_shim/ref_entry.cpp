// ref_entry.cpp — drives the reference's own shader code (rewritten to C++
// by oracle/build_ref.py) on the CPU.  TEST INFRASTRUCTURE ONLY.
//
// The shader TU is included inside namespace ref.  This file supplies what
// the D3D12 host (gracejinsotrue/PBRT-renderer-, src/gpu/DXRApp_*.cpp)
// supplies on Windows: resource contents, the envmap CDFs
// (src/gpu/DXRApp_Textures.cpp:281-389), the emitter CDFs
// (src/gpu/DXRApp_Scene.cpp:243-299 over src/cpu/mesh.cpp:24-40), the volume
// majorant grids (src/gpu/DXRApp_Scene.cpp:625-641), the per-frame
// DispatchRays loop (src/gpu/DXRApp.cpp:84-118), and a stand-in for the RT
// cores (BVH + Moller-Trumbore of src/cpu/mesh.cpp:51-89).
#include "hlsl_cpu.h"

#include <algorithm>
#include <atomic>
#include <limits>
#include <thread>

#include "../../include/pt.h"

namespace ref {
#include "Shaders.hlsl"
}  // namespace ref

namespace ref {
thread_local uint3 g_dispatch_index;
uint3 g_dispatch_dims;
int g_max_bounces = 32;

static_assert(sizeof(GPUMaterial) == sizeof(pt_material), "GPUMaterial layout");

struct HostScene {
    std::vector<pt_material> mats;
    std::vector<float> pos, nrm, uv, tan;
    std::vector<uint> idx;
    std::vector<float> emitterCdf, marg, cond;
    std::vector<float4> env;
    std::vector<GPUVolume> vols;
    std::vector<std::vector<float>> grids;  // densities then majorants
    std::vector<uint3> gridDims;
    std::vector<bool> opaque;               // per mesh (instance flags)
    std::vector<uint> triMesh, triPrim;
    struct Node { float lo[3], hi[3]; uint left, right, start, count, axis; };
    std::vector<Node> nodes;
    std::vector<uint> prims;
};
static HostScene g_host;

static void tri_verts(uint g, float3 &p0, float3 &p1, float3 &p2) {
    const pt_material &m = g_host.mats[g_host.triMesh[g]];
    uint base = m.indexOffset + g_host.triPrim[g] * 3;
    auto V = [&](uint i) {
        uint k = m.vertexOffset + g_host.idx[base + i];
        return float3(g_host.pos[3 * k], g_host.pos[3 * k + 1], g_host.pos[3 * k + 2]);
    };
    p0 = V(0); p1 = V(1); p2 = V(2);
}

// The ray-query stand-in's tree: a binned SAH build with the cost model of
// the reference's CPU accelerator (src/cpu/accel.cpp:55-324): 16 centroid
// bins along the node's largest axis, cost 2 C_trav + C_isect (n_L A_L +
// n_R A_R) / A with both costs 1, against C_isect n for a leaf; nodes of
// fewer than 32 triangles, or where the bins find no better split, get an
// exact sweep over the sorted centroids of all three axes.  Leaves where no
// split is cheaper.  Depth is capped so traversal's 128-entry stack holds.
static void build_bvh() {
    uint n = (uint)g_host.triMesh.size();
    g_host.prims.resize(n);
    std::vector<float3> ce(n), lo(n), hi(n);
    for (uint i = 0; i < n; i++) {
        float3 a, b, c;
        tri_verts(i, a, b, c);
        lo[i] = min(a, min(b, c));
        hi[i] = max(a, max(b, c));
        ce[i] = (lo[i] + hi[i]) * 0.5f;
        g_host.prims[i] = i;
    }
    g_host.nodes.clear();
    if (!n) return;
    struct Box {
        float3 l{1e30f, 1e30f, 1e30f}, h{-1e30f, -1e30f, -1e30f};
        void add(const float3 &a, const float3 &b) { l = min(l, a); h = max(h, b); }
        void add(const Box &o) { l = min(l, o.l); h = max(h, o.h); }
        float area() const {
            if (l.x > h.x) return 0.0f;
            float3 e = h - l;
            return 2.0f * (e.x * e.y + e.y * e.z + e.z * e.x);
        }
    };
    constexpr int kBins = 16, kSerial = 32, kMaxDepth = 100;
    struct It { uint node, s, e, depth; };
    std::vector<It> st{{0, 0, n, 0}};
    g_host.nodes.push_back({});
    uint *P = g_host.prims.data();
    std::vector<float> rightArea(n + 1);
    while (!st.empty()) {
        It it = st.back();
        st.pop_back();
        HostScene::Node nd{};
        Box bb;
        for (uint i = it.s; i < it.e; i++) bb.add(lo[P[i]], hi[P[i]]);
        for (int a = 0; a < 3; a++) { nd.lo[a] = bb.l[a]; nd.hi[a] = bb.h[a]; }
        const uint cnt = it.e - it.s;
        const float A = bb.area();
        float bestCost = (float)cnt;  // a leaf
        int bestAxis = -1;
        uint split = 0;  // triangles left of the split, in the order of bestAxis
        float3 ext = bb.h - bb.l;
        int ax = ext.x > ext.y ? (ext.x > ext.z ? 0 : 2) : (ext.y > ext.z ? 1 : 2);
        bool binned = false;
        if (cnt >= kSerial && A > 0.0f && ext[ax] > 0.0f) {
            float cmin = bb.l[ax], scale = kBins / ext[ax];
            uint binCnt[kBins] = {};
            Box binBox[kBins];
            auto binOf = [&](uint g) { return std::min(std::max((int)((ce[g][ax] - cmin) * scale), 0), kBins - 1); };
            for (uint i = it.s; i < it.e; i++) {
                int b = binOf(P[i]);
                binCnt[b]++;
                binBox[b].add(lo[P[i]], hi[P[i]]);
            }
            Box left[kBins];
            uint leftCnt[kBins];
            left[0] = binBox[0];
            leftCnt[0] = binCnt[0];
            for (int b = 1; b < kBins; b++) {
                left[b] = left[b - 1];
                left[b].add(binBox[b]);
                leftCnt[b] = leftCnt[b - 1] + binCnt[b];
            }
            Box right = binBox[kBins - 1];
            int bestBin = -1;
            for (int b = kBins - 2; b >= 0; b--) {
                float c = 2.0f + (leftCnt[b] * left[b].area() + (cnt - leftCnt[b]) * right.area()) / A;
                if (c < bestCost && leftCnt[b] > 0 && leftCnt[b] < cnt) { bestCost = c; bestBin = b; }
                right.add(binBox[b]);
            }
            if (bestBin >= 0) {
                uint *mid = std::partition(P + it.s, P + it.e, [&](uint g) { return binOf(g) <= bestBin; });
                split = (uint)(mid - (P + it.s));
                bestAxis = ax;
                binned = true;
            }
        }
        if (!binned && cnt > 1 && A > 0.0f) {  // exact sweep, every axis
            for (int a = 0; a < 3; a++) {
                std::sort(P + it.s, P + it.e, [&](uint x, uint y) { return ce[x][a] < ce[y][a] || (ce[x][a] == ce[y][a] && x < y); });
                Box r;
                for (uint i = cnt; i >= 1; i--) {
                    r.add(lo[P[it.s + i - 1]], hi[P[it.s + i - 1]]);
                    rightArea[i - 1] = r.area();
                }
                Box l;
                for (uint i = 1; i < cnt; i++) {
                    l.add(lo[P[it.s + i - 1]], hi[P[it.s + i - 1]]);
                    float c = 2.0f + (i * l.area() + (cnt - i) * rightArea[i]) / A;
                    if (c < bestCost) { bestCost = c; bestAxis = a; split = i; }
                }
            }
            if (bestAxis >= 0 && bestAxis != 2)  // the last sort was along z
                std::sort(P + it.s, P + it.e, [&](uint x, uint y) {
                    return ce[x][bestAxis] < ce[y][bestAxis] || (ce[x][bestAxis] == ce[y][bestAxis] && x < y);
                });
        }
        if (bestAxis < 0 || it.depth >= kMaxDepth) {
            if (bestAxis < 0 || cnt <= 4) { nd.start = it.s; nd.count = cnt; g_host.nodes[it.node] = nd; continue; }
        }
        if (it.depth >= kMaxDepth) {  // deep and still large: median split on the largest axis
            bestAxis = ax;
            split = cnt / 2;
            std::nth_element(P + it.s, P + it.s + split, P + it.e, [&](uint x, uint y) { return ce[x][ax] < ce[y][ax]; });
        }
        uint L = (uint)g_host.nodes.size();
        g_host.nodes.push_back({});
        g_host.nodes.push_back({});
        nd.left = L; nd.right = L + 1; nd.count = 0; nd.axis = (uint)bestAxis;
        g_host.nodes[it.node] = nd;
        st.push_back({L, it.s, it.s + split, it.depth + 1});
        st.push_back({L + 1, it.s + split, it.e, it.depth + 1});
    }
}

// The ray-tracing hardware's triangle test stand-in: Moller-Trumbore with
// fused multiply-adds in a set order (the arithmetic of the hardware the
// reference runs on is not published; the oracle and the kernels use this one).
static inline float dot_f(const float3 &a, const float3 &b) {
    return std::fmaf(a.z, b.z, std::fmaf(a.y, b.y, a.x * b.x));
}
static inline float3 cross_f(const float3 &a, const float3 &b) {
    return float3(std::fmaf(a.y, b.z, -(a.z * b.y)), std::fmaf(a.z, b.x, -(a.x * b.z)),
                  std::fmaf(a.x, b.y, -(a.y * b.x)));
}
static bool mt(const float3 &p0, const float3 &p1, const float3 &p2, const RayDesc &r, float &u, float &v, float &t) {
    float3 e1 = p1 - p0, e2 = p2 - p0;
    float3 pv = cross_f(r.Direction, e2);
    float det = dot_f(e1, pv);
    if (det > -1e-8f && det < 1e-8f) return false;
    float inv = 1.0f / det;
    float3 tv = r.Origin - p0;
    u = dot_f(tv, pv) * inv;
    if (u < 0.0f || u > 1.0f) return false;
    float3 qv = cross_f(tv, e1);
    v = dot_f(r.Direction, qv) * inv;
    if (v < 0.0f || u + v > 1.0f) return false;
    t = dot_f(e2, qv) * inv;
    return t >= r.TMin && t <= r.TMax;
}

// Candidates the query reports, in (t, triangle id) order: the non-opaque
// triangles in front of the nearest opaque one, then that opaque one (which
// commits and ends the query).  Opaque hits shrink the search interval as
// traversal finds them; an occlusion query (accept_first) stops at the first
// opaque hit, whose commit alone decides its result.
void collect_candidates(const RayDesc &r, std::vector<Candidate> &out, bool accept_first) {
    if (g_host.nodes.empty()) return;
    float inv[3] = {1.0f / r.Direction.x, 1.0f / r.Direction.y, 1.0f / r.Direction.z};
    float o[3] = {r.Origin.x, r.Origin.y, r.Origin.z};
    uint stack[128];
    int sp = 0;
    stack[sp++] = 0;
    RayDesc q = r;  // q.TMax: nearest opaque hit so far
    bool haveOpaque = false;
    Candidate best{};
    auto before = [](const Candidate &a, const Candidate &b) { return a.t < b.t || (a.t == b.t && a.gid < b.gid); };
    while (sp) {
        const HostScene::Node &n = g_host.nodes[stack[--sp]];
        float t0 = q.TMin, t1 = q.TMax;
        for (int a = 0; a < 3; a++) {
            float tn = (n.lo[a] - o[a]) * inv[a], tf = (n.hi[a] - o[a]) * inv[a];
            if (tn > tf) std::swap(tn, tf);
            if (std::isnan(tn) || std::isnan(tf)) continue;
            t0 = std::max(t0, tn);
            t1 = std::min(t1, tf);
        }
        if (!(t0 <= t1 * 1.00000024f)) continue;
        if (n.count) {
            for (uint i = n.start; i < n.start + n.count; i++) {
                uint g = g_host.prims[i];
                float3 p0, p1, p2;
                tri_verts(g, p0, p1, p2);
                float u, v, t;
                if (!mt(p0, p1, p2, q, u, v, t)) continue;
                Candidate c{t, u, v, g_host.triMesh[g], g_host.triPrim[g], g, (bool)g_host.opaque[g_host.triMesh[g]]};
                if (c.opaque) {
                    if (!haveOpaque || before(c, best)) { best = c; haveOpaque = true; q.TMax = t; }
                    if (accept_first) { out.clear(); out.push_back(best); return; }
                } else {
                    out.push_back(c);
                }
            }
        } else if (sp + 2 <= 128) {  // near child (along the split axis) on top
            bool leftNear = r.Direction[(int)n.axis] >= 0.0f;
            stack[sp++] = leftNear ? n.right : n.left;
            stack[sp++] = leftNear ? n.left : n.right;
        }
    }
    if (haveOpaque) {
        out.erase(std::remove_if(out.begin(), out.end(), [&](const Candidate &c) { return !before(c, best); }),
                  out.end());
        out.push_back(best);
    }
    std::sort(out.begin(), out.end(), before);
}

static void bind_u32(ByteAddressBuffer &b, const void *p) { b.data = static_cast<const uint *>(p); }

}  // namespace ref

using namespace ref;

extern "C" {

int ref_scene_create(const pt_scene_desc *d) {
    HostScene &s = g_host;
    s = HostScene();
    size_t nv = d->num_vertices;
    s.pos.assign(d->positions, d->positions + 3 * nv);
    s.nrm = d->normals ? std::vector<float>(d->normals, d->normals + 3 * nv) : std::vector<float>(3 * nv, 0.0f);
    s.uv = d->texcoords ? std::vector<float>(d->texcoords, d->texcoords + 2 * nv) : std::vector<float>(2 * nv, 0.0f);
    s.tan = d->tangents ? std::vector<float>(d->tangents, d->tangents + 3 * nv) : std::vector<float>(3 * nv, 0.0f);
    s.idx.assign(d->indices, d->indices + d->num_indices);
    s.mats.assign(d->materials, d->materials + d->num_meshes);
    // Mesh::activate area DiscretePDF + CreateSceneBuffers emitter CDFs.
    std::vector<float> all;
    std::vector<uint> emitters;
    for (uint i = 0; i < s.mats.size(); i++) {
        pt_material &m = s.mats[i];
        uint nt = m.indexCount / 3;
        std::vector<float> cdf{0.0f};
        for (uint t = 0; t < nt; t++) {
            s.triMesh.push_back(i);
            s.triPrim.push_back(t);
            float3 p0, p1, p2;
            tri_verts((uint)s.triMesh.size() - 1, p0, p1, p2);
            float3 c = cross(p1 - p0, p2 - p0);
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
        m.emitterSelectionProb = 0;
        if (m.isEmitter) {
            m.emitterCdfOffset = (uint)all.size();
            all.insert(all.end(), cdf.begin(), cdf.end());
            emitters.push_back(i);
        }
    }
    uint ne = (uint)emitters.size();
    std::vector<float> pc(ne + 1, 0.0f);
    for (uint k = 0; k < ne; k++) {
        const pt_material &m = s.mats[emitters[k]];
        pc[k + 1] = pc[k] + (0.2126f * m.radiance[0] + 0.7152f * m.radiance[1] + 0.0722f * m.radiance[2]) * m.surfaceArea;
    }
    if (pc[ne] > 0.0f) { float inv = 1.0f / pc[ne]; for (uint k = 1; k <= ne; k++) pc[k] *= inv; }
    else for (uint k = 0; k <= ne; k++) pc[k] = float(k) / float(std::max(ne, 1u));
    pc[ne] = 1.0f;
    for (uint k = 0; k < ne; k++) {
        s.mats[emitters[k]].emitterSelectionProb = pc[k + 1] - pc[k];
        s.mats[emitters[k]].emitterCdfOffset += ne + 1;
    }
    all.insert(all.begin(), pc.begin(), pc.end());
    s.emitterCdf = all.empty() ? std::vector<float>(1, 0.0f) : all;
    s.opaque.resize(s.mats.size());
    for (size_t i = 0; i < s.mats.size(); i++)
        s.opaque[i] = !(s.mats[i].type == PT_MAT_MIRROR || s.mats[i].type == PT_MAT_DIELECTRIC ||
                        s.mats[i].alphaTexIndex != PT_NO_TEXTURE);
    // Envmap + BuildEnvmapDistribution.
    const uint W = d->env_width, H = d->env_height;
    s.env.resize((size_t)W * H);
    for (size_t i = 0; i < (size_t)W * H; i++) s.env[i] = float4(d->env_rgb[3 * i], d->env_rgb[3 * i + 1], d->env_rgb[3 * i + 2], 1.0f);
    s.cond.assign((size_t)H * (W + 1), 0.0f);
    s.marg.assign(H + 1, 0.0f);
    std::vector<float> rowSums(H);
    const float M_PI_F = 3.14159265358979323846f;
    for (uint y = 0; y < H; ++y) {
        float theta = M_PI_F * (y + 0.5f) / (float)H;
        float sinTheta = std::sin(theta);
        size_t rb = (size_t)y * (W + 1);
        float rowSum = 0.0f;
        for (uint x = 0; x < W; ++x) {
            const float4 &p = s.env[(size_t)y * W + x];
            float w = (0.2126f * p.x + 0.7152f * p.y + 0.0722f * p.z) * sinTheta;
            if (w < 0.0f) w = 0.0f;
            rowSum += w;
            s.cond[rb + x + 1] = rowSum;
        }
        rowSums[y] = rowSum;
        if (rowSum > 0.0f) { float inv = 1.0f / rowSum; for (uint x = 1; x <= W; ++x) s.cond[rb + x] *= inv; }
        else for (uint x = 0; x <= W; ++x) s.cond[rb + x] = (float)x / (float)W;
    }
    double total = 0.0;
    for (uint y = 0; y < H; ++y) total += rowSums[y];
    if (total > 0.0) {
        double acc = 0.0, invT = 1.0 / total;
        for (uint y = 0; y < H; ++y) { acc += rowSums[y]; s.marg[y + 1] = (float)(acc * invT); }
        s.marg[H] = 1.0f;
    } else for (uint y = 0; y <= H; ++y) s.marg[y] = (float)y / (float)H;
    // Volumes, density grids and 4^3 brick majorants.
    for (uint g = 0; g < d->num_grids; g++) {
        const pt_grid &gr = d->grids[g];
        s.grids.emplace_back(gr.data, gr.data + (size_t)gr.w * gr.h * gr.d);
        s.gridDims.push_back(uint3(gr.w, gr.h, gr.d));
    }
    for (uint i = 0; i < d->num_volumes; i++) {
        const pt_volume &pv = d->volumes[i];
        GPUVolume v{};
        v.vMin = float3(pv.vmin[0], pv.vmin[1], pv.vmin[2]);
        v.vMax = float3(pv.vmax[0], pv.vmax[1], pv.vmax[2]);
        v.sigmaA = float3(pv.sigma_a[0], pv.sigma_a[1], pv.sigma_a[2]);
        v.sigmaS = float3(pv.sigma_s[0], pv.sigma_s[1], pv.sigma_s[2]);
        v.phaseG = pv.phase_g;
        v.flags = pv.flags;
        v.densityTexIndex = VOLUME_INVALID_TEX;
        v.majorantTexIndex = VOLUME_INVALID_TEX;
        if ((pv.flags & PT_VOLUME_HETEROGENEOUS) && pv.density_grid != PT_NO_TEXTURE) {
            v.densityTexIndex = pv.density_grid;
            uint3 dm = s.gridDims[pv.density_grid];
            const uint B = 4;
            uint mW = (dm.x + B - 1) / B, mH = (dm.y + B - 1) / B, mD = (dm.z + B - 1) / B;
            std::vector<float> maj((size_t)mW * mH * mD, 0.0f);
            const std::vector<float> &data = s.grids[pv.density_grid];
            for (uint z = 0; z < dm.z; z++)
                for (uint y = 0; y < dm.y; y++)
                    for (uint x = 0; x < dm.x; x++) {
                        float dd = data[(size_t)x + (size_t)dm.x * (y + (size_t)dm.y * z)];
                        size_t mi = (size_t)(x / B) + (size_t)mW * ((y / B) + (size_t)mH * (z / B));
                        maj[mi] = std::max(maj[mi], dd);
                    }
            v.majorantTexIndex = (uint)s.grids.size();
            s.grids.push_back(std::move(maj));
            s.gridDims.push_back(uint3(mW, mH, mD));
        }
        s.vols.push_back(v);
    }
    if (s.grids.size() > 64) return -1;
    // Bind resources.
    g_materials.data = reinterpret_cast<const GPUMaterial *>(s.mats.data());
    bind_u32(g_normals, s.nrm.data());
    bind_u32(g_indices, s.idx.data());
    bind_u32(g_vertices, s.pos.data());
    bind_u32(g_emitterCdf, s.emitterCdf.data());
    bind_u32(g_texcoords, s.uv.data());
    bind_u32(g_tangents, s.tan.data());
    bind_u32(g_envmapMarginalCdf, s.marg.data());
    bind_u32(g_envmapConditionalCdf, s.cond.data());
    g_envmap.w = W; g_envmap.h = H; g_envmap.data = s.env.data();
    g_sampler = SamplerState{ADDR_WRAP, ADDR_WRAP, ADDR_WRAP};
    g_envmapSampler = SamplerState{ADDR_WRAP, ADDR_CLAMP, ADDR_CLAMP};
    g_volumeSampler = SamplerState{ADDR_CLAMP, ADDR_CLAMP, ADDR_CLAMP};
    g_volumes.data = s.vols.data();
    for (size_t g = 0; g < s.grids.size(); g++) {
        g_volumeDensities[g].w = s.gridDims[g].x;
        g_volumeDensities[g].h = s.gridDims[g].y;
        g_volumeDensities[g].d = s.gridDims[g].z;
        g_volumeDensities[g].data = s.grids[g].data();
    }
    meshCount = (uint)s.mats.size();
    emitterCount = ne;
    volumeCount = (uint)s.vols.size();
    envmapScale = d->env_scale;
    evCompensation = d->ev_compensation;
    build_bvh();
    return 0;
}

// Camera constants + frame loop: one RayGen per pixel per frame, frames in
// order (g_accum carries the running sum as in the reference).
int ref_render(const pt_render_params *P, float *sum, int threads) {
    const pt_camera &c = P->camera;
    camPos = float3(c.pos[0], c.pos[1], c.pos[2]);
    camLowerLeftCorner = float3(c.llc[0], c.llc[1], c.llc[2]);
    camHorizontal = float3(c.horizontal[0], c.horizontal[1], c.horizontal[2]);
    camVertical = float3(c.vertical[0], c.vertical[1], c.vertical[2]);
    lensRadius = c.lens_radius;
    focalDistance = c.focal_distance;
    g_max_bounces = (int)P->max_depth;  // MAX_BOUNCES is bound to this variable at build time
    if (P->rng_kind != PT_RNG_SOBOL_OWEN || P->env_sampling != PT_ENV_CDF) return -3;
    const uint W = P->width, H = P->height;
    g_dispatch_dims = uint3(W, H, 1);
    for (auto *t : {&g_accum, &g_albedo, &g_normal, &g_output}) {
        t->w = W; t->h = H;
        t->px.assign((size_t)W * H, float4(0, 0, 0, 0));
    }
    int nt = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    for (uint f = 0; f < P->spp; f++) {
        frameCount = P->sample_offset + f;
        // frameCount == 0 resets the accumulator; later frames read it back.
        std::atomic<uint> next{0};
        auto work = [&]() {
            for (;;) {
                uint row = next.fetch_add(1);
                if (row >= H) break;
                for (uint x = 0; x < W; x++) {
                    g_dispatch_index = uint3(x, row, 0);
                    RayGen();
                }
            }
        };
        std::vector<std::thread> th;
        for (int i = 0; i < nt; i++) th.emplace_back(work);
        for (auto &t : th) t.join();
    }
    for (size_t i = 0; i < (size_t)W * H; i++) {
        sum[4 * i] = g_accum.px[i].x; sum[4 * i + 1] = g_accum.px[i].y;
        sum[4 * i + 2] = g_accum.px[i].z; sum[4 * i + 3] = g_accum.px[i].w;
    }
    return 0;
}

void ref_scene_materials(pt_material *out) { std::memcpy(out, g_host.mats.data(), g_host.mats.size() * sizeof(pt_material)); }
uint32_t ref_max_bounces(void) { return (uint32_t)g_max_bounces; }

void ref_rng(const uint32_t *pix, const uint32_t *smp, size_t n, uint32_t dims, uint32_t w, uint32_t h, float *out) {
    for (size_t i = 0; i < n; i++) {
        RNG r = InitRNG(uint2(pix[i] % w, pix[i] / w), uint2(w, h), smp[i]);
        for (uint32_t d = 0; d < dims; d++) out[i * dims + d] = NextFloat(r);
    }
}
void ref_bsdf_eval(const pt_material *mats, const uint32_t *mi, const float *wi, const float *wo, const float *hh,
                   size_t n, float *f, float *pdf) {
    for (size_t i = 0; i < n; i++) {
        GPUMaterial m;
        std::memcpy(&m, &mats[mi ? mi[i] : 0], sizeof(m));
        float3 a(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]), b(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
        float h = hh ? hh[i] : 0.0f;
        float3 r = MaterialEval(a, b, m, h);
        f[3 * i] = r.x; f[3 * i + 1] = r.y; f[3 * i + 2] = r.z;
        pdf[i] = MaterialPdf(a, b, m, h);
    }
}
// MaterialSample with the path sampler positioned at dimension dim0 of
// (pixel, sample) in a width x height frame.
void ref_bsdf_sample(const pt_material *mats, const uint32_t *mi, const float *wi, const float *hh,
                     const uint32_t *pix, const uint32_t *smp, uint32_t dim0, uint32_t w, uint32_t h, size_t n,
                     float *wo, float *wt, float *pdf) {
    for (size_t i = 0; i < n; i++) {
        GPUMaterial m;
        std::memcpy(&m, &mats[mi ? mi[i] : 0], sizeof(m));
        RNG r = InitRNG(uint2(pix[i] % w, pix[i] / w), uint2(w, h), smp[i]);
        r.dim = dim0;
        float3 a(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]), o;
        float p;
        float3 res = MaterialSample(a, r, m, hh ? hh[i] : 0.0f, o, p);
        wo[3 * i] = o.x; wo[3 * i + 1] = o.y; wo[3 * i + 2] = o.z;
        wt[3 * i] = res.x; wt[3 * i + 1] = res.y; wt[3 * i + 2] = res.z;
        pdf[i] = p;
    }
}
void ref_hg_sample(const float *g, const float *wo, const uint32_t *pix, const uint32_t *smp, uint32_t dim0, uint32_t w,
                   uint32_t h, size_t n, float *wi, float *pdf) {
    for (size_t i = 0; i < n; i++) {
        RNG r = InitRNG(uint2(pix[i] % w, pix[i] / w), uint2(w, h), smp[i]);
        r.dim = dim0;
        float p;
        float3 res = SampleHG(float3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), g[i], r, p);
        wi[3 * i] = res.x; wi[3 * i + 1] = res.y; wi[3 * i + 2] = res.z;
        pdf[i] = p;
    }
}
void ref_env_sample(const float *u, size_t n, float *dir, float *rad, float *pdf) {
    for (size_t i = 0; i < n; i++) {
        float3 d, r;
        float p;
        SampleEnvmap(u[2 * i], u[2 * i + 1], d, r, p);
        dir[3 * i] = d.x; dir[3 * i + 1] = d.y; dir[3 * i + 2] = d.z;
        rad[3 * i] = r.x; rad[3 * i + 1] = r.y; rad[3 * i + 2] = r.z;
        pdf[i] = p;
    }
}
void ref_env_pdf(const float *dir, size_t n, float *pdf, float *rad) {
    for (size_t i = 0; i < n; i++) {
        float3 d(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
        pdf[i] = EnvmapPdfDirection(d);
        float3 r = EvalEnvmap(d);
        rad[3 * i] = r.x; rad[3 * i + 1] = r.y; rad[3 * i + 2] = r.z;
    }
}
void ref_env_cdf(float *marg, float *cond) {
    std::memcpy(marg, g_host.marg.data(), g_host.marg.size() * 4);
    std::memcpy(cond, g_host.cond.data(), g_host.cond.size() * 4);
}

}  // extern "C"
