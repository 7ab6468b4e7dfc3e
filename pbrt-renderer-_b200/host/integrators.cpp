// integrators.cpp — the "path_mis" and "direct" integrators the reference's
// scene files request (38 of its XML scenes; it registers neither), rendering
// through libpt, plus the scene flattening and camera conversion of its
// D3D12 host (gracejinsotrue/PBRT-renderer-, src/gpu/DXRApp_Scene.cpp,
// src/gpu/DXRApp_Textures.cpp, src/gpu/DXRApp_Camera.cpp).
#include <cstdio>
#include <cstring>
#include <unordered_map>

#include "nori/nori.h"

namespace nori {

std::vector<float> RenderResult::mean() const {
    std::vector<float> m((size_t)width * height * 3, 0.0f);
    for (size_t i = 0; i < (size_t)width * height; i++) {
        float w = sum[4 * i + 3] > 0 ? sum[4 * i + 3] : 1.0f;
        for (int c = 0; c < 3; c++) m[3 * i + c] = sum[4 * i + c] / w;
    }
    return m;
}

// CreateSceneBuffers (src/gpu/DXRApp_Scene.cpp:172-451), CreateTextures
// (src/gpu/DXRApp_Textures.cpp:448-537), LoadEnvmap
// (src/gpu/DXRApp_Textures.cpp:181-275), SetupVolumes + LoadVolume
// (src/gpu/DXRApp_Scene.cpp:453-548).  Emitter CDFs, surface areas, mip
// chains, the envmap tables and majorant grids are built by pt_upload_scene.
void flattenScene(const Scene *scene, FlatScene &out) {
    out = FlatScene{};
    uint32_t nv = 0, ni = 0;
    // Textures are keyed by resolved path: a file named by several materials
    // (or maps) loads once, with the colour space of its first use; a file
    // that cannot be read leaves the map unset (the constant parameter is used).
    std::unordered_map<std::string, uint32_t> texCache;
    auto texture = [&](const std::string &rel, bool srgb) -> uint32_t {
        if (rel.empty()) return PT_NO_TEXTURE;
        std::string path = resolvePath(rel, scene->getBaseDir());
        auto it = texCache.find(path);
        if (it != texCache.end()) return it->second;
        std::vector<uint8_t> rgba;
        uint32_t w = 0, h = 0;
        try {
            loadImageRGBA8(path, w, h, rgba);
        } catch (const std::exception &e) {
            std::fprintf(stderr, "[texture] Failed to load: %s (%s)\n", path.c_str(), e.what());
            return PT_NO_TEXTURE;
        }
        uint32_t index = (uint32_t)out.texData.size();
        out.texData.push_back(std::move(rgba));
        out.textures.push_back(pt_texture{w, h, nullptr, srgb ? 1u : 0u});
        out.texPaths.push_back(path);
        texCache[path] = index;
        return index;
    };
    for (const Mesh *mesh : scene->getMeshes()) {
        BSDFGPUData gd = mesh->getBSDF()->getGPUData();
        pt_material m = toGPUMaterial(gd);
        // metallic maps are loaded by the reference but read by no shader: not loaded here
        m.albedoTexIndex = texture(gd.albedoTexture, true);
        m.normalTexIndex = texture(gd.normalTexture, false);
        m.roughnessTexIndex = texture(gd.roughnessTexture, false);
        m.specularTexIndex = texture(gd.specularTexture, false);
        m.subsurfaceTexIndex = texture(gd.subsurfaceTexture, false);
        m.alphaTexIndex = texture(gd.alphaTexture, false);
        if (mesh->isEmitter()) {
            Color3f Le = mesh->getEmitter()->getRadiance();
            m.isEmitter = 1;
            for (int c = 0; c < 3; c++) m.radiance[c] = Le[c];
        }
        uint32_t vc = mesh->getVertexCount(), ic = mesh->getTriangleCount() * 3;
        m.vertexOffset = nv;
        m.indexOffset = ni;
        m.vertexCount = vc;
        m.indexCount = ic;
        out.mats.push_back(m);
        const auto &V = mesh->getVertexPositions();
        out.pos.insert(out.pos.end(), V.begin(), V.end());
        const auto &N = mesh->getVertexNormals();
        if (N.size() == (size_t)vc * 3) out.nrm.insert(out.nrm.end(), N.begin(), N.end());
        else out.nrm.insert(out.nrm.end(), (size_t)vc * 3, 0.0f);
        const auto &F = mesh->getIndices();
        out.idx.insert(out.idx.end(), F.begin(), F.end());
        const auto &UV = mesh->getVertexTexCoords();
        bool hair = mesh->hasTangents();
        for (uint32_t v = 0; v < vc; v++) {
            if (UV.size() == (size_t)vc * 2) {
                out.uv.push_back(UV[2 * v]);
                out.uv.push_back(hair ? UV[2 * v + 1] : 1.0f - UV[2 * v + 1]);  // V flip for OBJ meshes
            } else {
                out.uv.push_back(0.0f);
                out.uv.push_back(0.0f);
            }
        }
        const auto &T = mesh->getVertexTangents();
        if (T.size() == (size_t)vc * 3) out.tan.insert(out.tan.end(), T.begin(), T.end());
        else out.tan.insert(out.tan.end(), (size_t)vc * 3, 0.0f);
        nv += vc;
        ni += ic;
    }
    for (size_t t = 0; t < out.textures.size(); t++) out.textures[t].rgba8 = out.texData[t].data();
    // envmap: the reference falls back to a 1x1 0.5 grey texel when the HDR cannot be read
    std::string hdr = resolvePath(scene->getEnvmap(), scene->getBaseDir());
    if (!loadHDR(hdr, out.env, out.envW, out.envH)) {
        std::fprintf(stderr, "[envmap] No HDR at '%s' - falling back to flat gray.\n", hdr.c_str());
        out.envW = out.envH = 1;
        out.env.assign(3, 0.5f);
    }
    out.envScale = scene->getEnvmapScale();
    out.evCompensation = scene->getEvCompensation();
    if (const Medium *med = scene->getMedium()) {
        BoundingBox3f b = med->hasExplicitBounds() ? med->getExplicitBounds() : scene->getBoundingBox();
        Color3f sa = med->getSigmaARGB(), ss = med->getSigmaSRGB();
        pt_volume v{};
        for (int i = 0; i < 3; i++) {
            v.vmin[i] = b.min[i]; v.vmax[i] = b.max[i];
            v.sigma_a[i] = sa[i]; v.sigma_s[i] = ss[i];
        }
        v.phase_g = med->getPhaseG();
        v.flags = med->isHeterogeneous() ? PT_VOLUME_HETEROGENEOUS : 0u;
        v.density_grid = PT_NO_TEXTURE;
        if (med->isHeterogeneous() && !med->getVolumePath().empty()) {
            std::vector<float> data;
            uint32_t w, h, d;
            std::string p = resolvePath(med->getVolumePath(), scene->getBaseDir());
            if (loadVol(p, data, w, h, d)) {
                v.density_grid = (uint32_t)out.gridData.size();
                out.gridData.push_back(std::move(data));
                out.grids.push_back(pt_grid{w, h, d, nullptr});
            } else {
                std::fprintf(stderr, "[volume] WARNING: could not open '%s'\n", p.c_str());
            }
        }
        out.vols.push_back(v);
    }
    for (size_t g = 0; g < out.gridData.size(); g++) out.grids[g].data = out.gridData[g].data();
}

pt_scene_desc FlatScene::desc() const {
    pt_scene_desc d;
    std::memset(&d, 0, sizeof(d));
    d.num_vertices = (uint32_t)(pos.size() / 3);
    d.positions = pos.data();
    d.normals = nrm.data();
    d.texcoords = uv.data();
    d.tangents = tan.data();
    d.num_indices = (uint32_t)idx.size();
    d.indices = idx.data();
    d.num_meshes = (uint32_t)mats.size();
    d.materials = mats.data();
    d.env_width = envW;
    d.env_height = envH;
    d.env_rgb = env.data();
    d.env_scale = envScale;
    d.ev_compensation = evCompensation;
    d.num_volumes = (uint32_t)vols.size();
    d.volumes = vols.data();
    d.num_grids = (uint32_t)grids.size();
    d.grids = grids.data();
    d.num_textures = (uint32_t)textures.size();
    d.textures = textures.data();
    return d;
}

// SetupCamera + RecomputeCameraPlane (src/gpu/DXRApp_Camera.cpp:23-112):
// four Nori camera rays -> position, yaw/pitch, vertical fov and the x flip,
// then the lower-left corner / horizontal / vertical image plane.
pt_camera cameraConstants(const Camera *cam, int width, int height) {
    float w = (float)width, h = (float)height;
    Ray3f bl, br, tl, ctr;
    Point2f ap(0, 0);
    cam->sampleRay(bl, Point2f(0, h), ap);
    cam->sampleRay(br, Point2f(w, h), ap);
    cam->sampleRay(tl, Point2f(0, 0), ap);
    cam->sampleRay(ctr, Point2f(w / 2, h / 2), ap);
    Point3f pos = bl.o;
    Vector3f fwd = ctr.d.normalized();
    float yaw = std::atan2(fwd.x(), fwd.z());
    float pitch = std::asin(fwd.y());
    auto project = [&](const Ray3f &r) { return pos + r.d * (1.0f / r.d.dot(fwd)); };
    Point3f Pbl = project(bl), Pbr = project(br), Ptl = project(tl);
    float halfHeight = (Ptl - Pbl).norm() * 0.5f;
    float fovY = 2.0f * std::atan(halfHeight);
    Vector3f dxrRight(std::cos(yaw), 0.0f, -std::sin(yaw));
    float xflip = (Pbr - Pbl).normalized().dot(dxrRight) >= 0.0f ? 1.0f : -1.0f;
    float cy = std::cos(yaw), sy = std::sin(yaw), cp = std::cos(pitch), sp = std::sin(pitch);
    float f[3] = {sy * cp, sp, cy * cp};
    float r[3] = {cy, 0.0f, -sy};
    float u[3] = {f[1] * r[2] - f[2] * r[1], f[2] * r[0] - f[0] * r[2], f[0] * r[1] - f[1] * r[0]};
    float aspect = w / h;
    float halfH = std::tan(fovY * 0.5f), halfW = halfH * aspect;
    pt_camera c{};
    for (int i = 0; i < 3; i++) {
        c.pos[i] = pos[i];
        c.llc[i] = pos[i] + f[i] - xflip * halfW * r[i] - halfH * u[i];
        c.horizontal[i] = xflip * 2.0f * halfW * r[i];
        c.vertical[i] = 2.0f * halfH * u[i];
    }
    c.lens_radius = cam->getLensRadius();
    c.focal_distance = cam->getFocalDistance();
    return c;
}

GPUIntegrator::GPUIntegrator(const PropertyList &p, uint32_t defaultDepth) {
    m_maxDepth = (uint32_t)p.getInteger("maxDepth", (int)defaultDepth);
    m_device = p.getInteger("device", 0);
    std::string rng = p.getString("rng", "sobol");
    m_rng = rng == "pcg" ? PT_RNG_PCG_HASH : PT_RNG_SOBOL_OWEN;
    std::string env = p.getString("envSampling", "cdf");
    m_envSampling = env == "alias" ? PT_ENV_ALIAS : PT_ENV_CDF;
}
GPUIntegrator::~GPUIntegrator() {
    if (m_ctx) pt_destroy(m_ctx);
}
void GPUIntegrator::preprocess(const Scene *scene) {
    m_scene = scene;
    flattenScene(scene, m_flat);
    m_desc = m_flat.desc();
    const Camera *cam = scene->getCamera();
    m_width = cam->getOutputSize()[0];
    m_height = cam->getOutputSize()[1];
    m_cam = nori::cameraConstants(cam, m_width, m_height);
    if (!m_ctx) {
        int rc = pt_create(&m_ctx, m_device);
        if (rc != PT_OK) throw NoriException("path tracer: no CUDA device (pt_create = " + std::to_string(rc) + ")");
    }
    int rc = pt_upload_scene(m_ctx, &m_desc);
    if (rc != PT_OK) throw NoriException(std::string("pt_upload_scene: ") + pt_last_error(m_ctx));
}
Color3f GPUIntegrator::Li(const Scene *, Sampler *, const Ray3f &) const {
    throw NoriException("GPU integrators trace whole frames: call render() (Integrator::Li is not evaluated per ray)");
}
RenderResult GPUIntegrator::render(uint32_t spp, uint32_t sampleOffset, RenderResult *film) {
    if (!m_ctx || !m_scene) throw NoriException("render() before preprocess()");
    RenderResult local;
    RenderResult &R = film ? *film : local;
    if (R.width != m_width || R.height != m_height || R.sum.size() != (size_t)m_width * m_height * 4) {
        R.width = m_width;
        R.height = m_height;
        R.sum.assign((size_t)m_width * m_height * 4, 0.0f);
        R.comp.assign((size_t)m_width * m_height * 4, 0.0f);
    }
    pt_render_params P{};
    P.width = (uint32_t)m_width;
    P.height = (uint32_t)m_height;
    P.spp = spp;
    P.sample_offset = sampleOffset;
    P.max_depth = m_maxDepth;
    P.rng_kind = m_rng;
    P.env_sampling = m_envSampling;
    P.camera = m_cam;
    pt_film F{(uint32_t)m_width, (uint32_t)m_height, R.sum.data(), R.comp.data(), PT_MEM_HOST};
    int rc = pt_render(m_ctx, &P, &F, &R.stats);
    if (rc != PT_OK) throw NoriException(std::string("pt_render: ") + pt_last_error(m_ctx));
    return film ? R : local;
}
std::string GPUIntegrator::toString() const { return "GPUIntegrator[maxDepth = " + std::to_string(m_maxDepth) + "]"; }

class PathMIS : public GPUIntegrator {  // Shaders.hlsl RayGen: MAX_BOUNCES = 32
public:
    explicit PathMIS(const PropertyList &p) : GPUIntegrator(p, 32) {}
    std::string toString() const override { return "PathMIS[maxDepth = " + std::to_string(m_maxDepth) + "]"; }
};
// Direct illumination: emission + one bounce of light / envmap NEE with MIS.
class Direct : public GPUIntegrator {
public:
    explicit Direct(const PropertyList &p) : GPUIntegrator(p, 1) { m_maxDepth = 1; }
    std::string toString() const override { return "Direct[]"; }
};

NORI_REGISTER_CLASS(PathMIS, "path_mis")
NORI_REGISTER_CLASS(Direct, "direct")

}  // namespace nori
