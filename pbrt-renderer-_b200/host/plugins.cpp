// plugins.cpp — the Nori plugins of the C++17 host: BSDFs, area emitter,
// media, perspective camera, independent sampler, Gaussian filter, OBJ mesh
// and the scene (reference: src/cpu/*.cpp of gracejinsotrue/PBRT-renderer-).
//
// BSDF eval/pdf/sample use the same shading math as the CUDA kernels
// (csrc/pt_math.cuh, compiled here as plain C++), i.e. the reference's shader
// models; the reference's CPU Disney and hair classes return Lambertian
// stand-ins instead.  BSDF::sample receives two uniforms (the Nori API);
// Disney's lobe choice and the hair lobe choice reuse the first one by
// remapping it inside the chosen lobe, and the hair azimuth takes the low bits
// of the second.
#include <algorithm>
#include <cstring>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <unordered_map>

#include "nori/nori.h"
#include "pt_math.cuh"

namespace nori {

namespace {

ptm::float3 F(const Vec3 &v) { return ptm::make_float3(v[0], v[1], v[2]); }
Vec3 V(const ptm::float3 &v) { return Vec3(v.x, v.y, v.z); }
Color3f C(const ptm::float3 &v) { return Color3f(v.x, v.y, v.z); }

}  // namespace

pt_material toGPUMaterial(const BSDFGPUData &d) {  // src/gpu/DXRApp_Scene.cpp:183-233
    pt_material m;
    std::memset(&m, 0, sizeof(m));
    m.type = (uint32_t)d.type;
    for (int i = 0; i < 3; i++) m.albedo[i] = d.albedo[i];
    m.intIOR = d.intIOR;
    m.extIOR = d.extIOR;
    m.alpha = d.alpha;
    uint32_t *tex = &m.albedoTexIndex;
    for (int i = 0; i < 7; i++) tex[i] = PT_NO_TEXTURE;
    m.roughness = d.roughness; m.metallic = d.metallic; m.specular = d.specular; m.specularTint = d.specularTint;
    m.sheen = d.sheen; m.sheenTint = d.sheenTint; m.subsurface = d.subsurface; m.clearcoat = d.clearcoat;
    m.clearcoatGloss = d.clearcoatGloss; m.anisotropic = d.anisotropic; m.betaN = d.betaN;
    return m;
}

// Evaluation through the shared shading math.
class MathBSDF : public BSDF {
public:
    Color3f eval(const BSDFQueryRecord &bRec) const override {
        if (bRec.measure != ESolidAngle) return Color3f(0.0f);
        pt_material m = toGPUMaterial(getGPUData());
        ptm::float3 f;
        float p;
        ptm::material_eval_pdf(F(bRec.wi), F(bRec.wo), m, bRec.h, f, p);
        return C(f);
    }
    float pdf(const BSDFQueryRecord &bRec) const override {
        if (bRec.measure != ESolidAngle) return 0.0f;
        pt_material m = toGPUMaterial(getGPUData());
        ptm::float3 f;
        float p;
        ptm::material_eval_pdf(F(bRec.wi), F(bRec.wo), m, bRec.h, f, p);
        return p;
    }
    Color3f sample(BSDFQueryRecord &bRec, const Point2f &s) const override {
        pt_material m = toGPUMaterial(getGPUData());
        float u[4] = {s.x(), s.y(), 0.0f, 0.0f};
        if (m.type == PT_MAT_DISNEY) {
            ptm::DisneyPre p = ptm::disney_pre(m);
            float lo = 0.0f, w = p.pD;
            if (s.x() >= p.pD && s.x() < p.pD + p.pS) { lo = p.pD; w = p.pS; }
            else if (s.x() >= p.pD + p.pS) { lo = p.pD + p.pS; w = p.pC; }
            u[1] = std::min(w > 0.0f ? (s.x() - lo) / w : 0.0f, 0.99999994f);
            u[2] = s.y();
        } else if (m.type == PT_MAT_HAIR) {
            u[1] = s.x();
            u[2] = s.y();
            float sc = s.y() * 4096.0f;
            u[3] = sc - std::floor(sc);
        }
        ptm::float3 wo;
        float pdfv;
        ptm::float3 wt = ptm::material_sample(F(bRec.wi), u, m, bRec.h, wo, pdfv);
        bRec.wo = V(wo);
        bRec.eta = 1.0f;
        bRec.measure = ESolidAngle;
        if (!(pdfv > 0.0f)) return Color3f(0.0f);
        return C(wt);
    }
};

// ---- diffuse (src/cpu/diffuse.cpp) --------------------------------------------
class Diffuse : public MathBSDF {
public:
    explicit Diffuse(const PropertyList &p) {
        m_albedo = p.getColor("albedo", Color3f(0.5f));
        m_textures[0] = p.getString("albedoTexture", "");
        m_textures[1] = p.getString("normalTexture", "");
        m_textures[2] = p.getString("roughnessTexture", "");
        m_textures[3] = p.getString("metallicTexture", "");
        m_alphaTexture = p.getString("alphaTexture", "");
    }
    bool isDiffuse() const override { return true; }
    BSDFGPUData getGPUData() const override {
        BSDFGPUData d;
        d.type = BSDFGPUData::DIFFUSE;
        for (int i = 0; i < 3; i++) d.albedo[i] = m_albedo[i];
        d.albedoTexture = m_textures[0]; d.normalTexture = m_textures[1];
        d.roughnessTexture = m_textures[2]; d.metallicTexture = m_textures[3];
        d.alphaTexture = m_alphaTexture;
        return d;
    }
    std::string toString() const override { return "Diffuse[albedo = " + m_albedo.toString() + "]"; }

private:
    Color3f m_albedo;
    std::string m_textures[4], m_alphaTexture;
};

// ---- mirror (src/cpu/mirror.cpp) ---------------------------------------------
class Mirror : public BSDF {
public:
    explicit Mirror(const PropertyList &) {}
    Color3f eval(const BSDFQueryRecord &) const override { return Color3f(0.0f); }
    float pdf(const BSDFQueryRecord &) const override { return 0.0f; }
    Color3f sample(BSDFQueryRecord &bRec, const Point2f &) const override {
        if (bRec.wi.z() <= 0) return Color3f(0.0f);
        bRec.wo = Vector3f(-bRec.wi.x(), -bRec.wi.y(), bRec.wi.z());
        bRec.measure = EDiscrete;
        bRec.eta = 1.0f;
        return Color3f(1.0f);
    }
    BSDFGPUData getGPUData() const override {
        BSDFGPUData d;
        d.type = BSDFGPUData::MIRROR;
        d.albedo[0] = d.albedo[1] = d.albedo[2] = 1.0f;
        return d;
    }
    std::string toString() const override { return "Mirror[]"; }
};

// ---- dielectric (src/cpu/dielectric.cpp) -------------------------------------
class Dielectric : public BSDF {
public:
    explicit Dielectric(const PropertyList &p) {
        m_intIOR = p.getFloat("intIOR", 1.5046f);
        m_extIOR = p.getFloat("extIOR", 1.000277f);
        m_tint = p.getColor("tintColor", Color3f(1.0f));
    }
    Color3f eval(const BSDFQueryRecord &) const override { return Color3f(0.0f); }
    float pdf(const BSDFQueryRecord &) const override { return 0.0f; }
    Color3f sample(BSDFQueryRecord &bRec, const Point2f &s) const override {
        float cosI = bRec.wi.z();
        float Fr = ptm::fresnel(cosI, m_extIOR, m_intIOR);
        bRec.measure = EDiscrete;
        if (s.x() < Fr) {
            bRec.wo = Vector3f(-bRec.wi.x(), -bRec.wi.y(), bRec.wi.z());
            bRec.eta = 1.0f;
            return Color3f(1.0f);
        }
        float etaI = m_extIOR, etaT = m_intIOR;
        Vec3 n(0, 0, 1);
        if (cosI < 0.0f) { std::swap(etaI, etaT); n = Vec3(0, 0, -1); cosI = -cosI; }
        float eta = etaI / etaT;
        float s2 = eta * eta * (1.0f - cosI * cosI);
        if (s2 > 1.0f) {
            bRec.wo = Vector3f(-bRec.wi.x(), -bRec.wi.y(), bRec.wi.z());
            bRec.eta = 1.0f;
            return Color3f(1.0f);
        }
        float cosT = std::sqrt(1.0f - s2);
        bRec.wo = eta * (-bRec.wi) + (eta * cosI - cosT) * n;
        bRec.eta = eta;
        return Color3f(1.0f);
    }
    BSDFGPUData getGPUData() const override {
        BSDFGPUData d;
        d.type = BSDFGPUData::DIELECTRIC;
        for (int i = 0; i < 3; i++) d.albedo[i] = m_tint[i];
        d.intIOR = m_intIOR;
        d.extIOR = m_extIOR;
        return d;
    }
    std::string toString() const override { return "Dielectric[]"; }

private:
    float m_intIOR, m_extIOR;
    Color3f m_tint;
};

// ---- microfacet (src/cpu/microfacet.cpp) -------------------------------------
class Microfacet : public MathBSDF {
public:
    explicit Microfacet(const PropertyList &p) {
        m_alpha = p.getFloat("alpha", 0.1f);
        m_intIOR = p.getFloat("intIOR", 1.5046f);
        m_extIOR = p.getFloat("extIOR", 1.000277f);
        m_kd = p.getColor("kd", Color3f(0.5f));
        m_textures[0] = p.getString("albedoTexture", "");
        m_textures[1] = p.getString("normalTexture", "");
        m_textures[2] = p.getString("roughnessTexture", "");
        m_textures[3] = p.getString("metallicTexture", "");
    }
    BSDFGPUData getGPUData() const override {
        BSDFGPUData d;
        d.type = BSDFGPUData::MICROFACET;
        for (int i = 0; i < 3; i++) d.albedo[i] = m_kd[i];
        d.intIOR = m_intIOR; d.extIOR = m_extIOR; d.alpha = m_alpha;
        d.albedoTexture = m_textures[0]; d.normalTexture = m_textures[1];
        d.roughnessTexture = m_textures[2]; d.metallicTexture = m_textures[3];
        return d;
    }
    std::string toString() const override { return "Microfacet[]"; }

private:
    float m_alpha, m_intIOR, m_extIOR;
    Color3f m_kd;
    std::string m_textures[4];
};

// ---- Disney (src/cpu/disney.cpp) -------------------------------------------------
class Disney : public MathBSDF {
public:
    explicit Disney(const PropertyList &p) {
        if (p.getColor("baseColor", Color3f(-1.f)).r() >= 0.f) m_base = p.getColor("baseColor");
        else m_base = p.getColor("albedo", Color3f(0.8f));
        m_v[0] = p.getFloat("roughness", 0.5f);
        m_v[1] = p.getFloat("metallic", 0.0f);
        m_v[2] = p.getFloat("specular", 0.5f);
        m_v[3] = p.getFloat("specularTint", 0.0f);
        m_v[4] = p.getFloat("sheen", 0.0f);
        m_v[5] = p.getFloat("sheenTint", 0.5f);
        m_v[6] = p.getFloat("subsurface", 0.0f);
        m_v[7] = p.getFloat("clearcoat", 0.0f);
        m_v[8] = p.getFloat("clearcoatGloss", 1.0f);
        m_v[9] = p.getFloat("anisotropic", 0.0f);
        const char *tn[] = {"albedoTexture", "normalTexture", "roughnessTexture", "metallicTexture",
                            "specularTexture", "subsurfaceTexture", "alphaTexture"};
        for (int i = 0; i < 7; i++) m_tex[i] = p.getString(tn[i], "");
    }
    bool isDiffuse() const override { return true; }
    BSDFGPUData getGPUData() const override {
        BSDFGPUData d;
        d.type = BSDFGPUData::DISNEY;
        for (int i = 0; i < 3; i++) d.albedo[i] = m_base[i];
        d.roughness = m_v[0]; d.metallic = m_v[1]; d.specular = m_v[2]; d.specularTint = m_v[3];
        d.sheen = m_v[4]; d.sheenTint = m_v[5]; d.subsurface = m_v[6]; d.clearcoat = m_v[7];
        d.clearcoatGloss = m_v[8]; d.anisotropic = m_v[9];
        d.albedoTexture = m_tex[0]; d.normalTexture = m_tex[1]; d.roughnessTexture = m_tex[2];
        d.metallicTexture = m_tex[3]; d.specularTexture = m_tex[4]; d.subsurfaceTexture = m_tex[5];
        d.alphaTexture = m_tex[6];
        return d;
    }
    std::string toString() const override { return "Disney[baseColor = " + m_base.toString() + "]"; }

private:
    Color3f m_base;
    float m_v[10];
    std::string m_tex[7];
};

// ---- hair BSDF (src/cpu/hair.cpp:326-423) ------------------------------------------
class HairBSDF : public MathBSDF {
public:
    explicit HairBSDF(const PropertyList &p) {
        m_color = p.getColor("color", Color3f(0.28f, 0.15f, 0.06f));
        m_betaM = p.getFloat("beta_m", 0.25f);
        m_betaN = p.getFloat("beta_n", 0.3f);
        m_alpha = p.getFloat("alpha", 2.0f);
        m_eta = p.getFloat("eta", 1.55f);
        m_alphaTexture = p.getString("alphaTexture", "");
    }
    BSDFGPUData getGPUData() const override {
        BSDFGPUData d;
        d.type = BSDFGPUData::HAIR;
        for (int i = 0; i < 3; i++) d.albedo[i] = m_color[i];
        d.roughness = m_betaM;
        d.alpha = m_alpha;
        d.intIOR = m_eta;
        d.betaN = m_betaN;
        d.alphaTexture = m_alphaTexture;
        return d;
    }
    std::string toString() const override { return "HairBSDF[color = " + m_color.toString() + "]"; }

private:
    Color3f m_color;
    float m_betaM, m_betaN, m_alpha, m_eta;
    std::string m_alphaTexture;
};

// ---- subsurface (src/cpu/subsurface.cpp): the GPU renders the random walk
// (type 6); the CPU eval is the reference's Lambertian stand-in.  Field reuse
// as the reference's: radius -> subsurface, g -> anisotropic, tint -> sheen /
// sheenTint / clearcoat.
class Subsurface : public BSDF {
public:
    explicit Subsurface(const PropertyList &p) {
        m_albedo = p.getColor("albedo", Color3f(0.8f, 0.5f, 0.4f));
        m_radius = p.getFloat("radius", 0.1f);
        m_intIOR = p.getFloat("intIOR", 1.33f);
        m_extIOR = p.getFloat("extIOR", 1.000277f);
        m_g = p.getFloat("g", 0.0f);
        m_roughness = p.getFloat("roughness", 0.3f);
        m_tint = p.getColor("tint", Color3f(1.f, 1.f, 1.f));
        m_specular = p.getFloat("specular", 0.0f);
        m_tex[0] = p.getString("albedoTexture", "");
        m_tex[1] = p.getString("normalTexture", "");
        m_tex[2] = p.getString("roughnessTexture", "");
        m_tex[3] = p.getString("specularTexture", "");
    }
    Color3f eval(const BSDFQueryRecord &b) const override {
        if (b.measure != ESolidAngle || b.wi.z() <= 0 || b.wo.z() <= 0) return Color3f(0.0f);
        return m_albedo * ptm::kInvPi;
    }
    float pdf(const BSDFQueryRecord &b) const override {
        if (b.measure != ESolidAngle || b.wi.z() <= 0 || b.wo.z() <= 0) return 0.0f;
        return ptm::kInvPi * b.wo.z();
    }
    Color3f sample(BSDFQueryRecord &b, const Point2f &s) const override {
        if (b.wi.z() <= 0) return Color3f(0.0f);
        b.measure = ESolidAngle;
        b.wo = V(ptm::cos_hemi(s.x(), s.y()));
        b.eta = 1.0f;
        return m_albedo;
    }
    BSDFGPUData getGPUData() const override {
        BSDFGPUData d;
        d.type = BSDFGPUData::SUBSURFACE;
        for (int i = 0; i < 3; i++) d.albedo[i] = m_albedo[i];
        d.intIOR = m_intIOR; d.extIOR = m_extIOR; d.subsurface = m_radius; d.anisotropic = m_g;
        d.roughness = m_roughness; d.sheen = m_tint.r(); d.sheenTint = m_tint.g(); d.clearcoat = m_tint.b();
        d.specular = m_specular;
        d.albedoTexture = m_tex[0]; d.normalTexture = m_tex[1]; d.roughnessTexture = m_tex[2];
        d.specularTexture = m_tex[3];
        return d;
    }
    std::string toString() const override { return "Subsurface[]"; }

private:
    Color3f m_albedo, m_tint;
    float m_radius, m_intIOR, m_extIOR, m_g, m_roughness, m_specular;
    std::string m_tex[4];
};

// ---- area emitter (src/cpu/area.cpp) ----------------------------------------------
class AreaLight : public Emitter {
public:
    explicit AreaLight(const PropertyList &p) { m_radiance = p.getColor("radiance"); }
    Color3f getRadiance() const override { return m_radiance; }
    Color3f sample(const Point2f &s, Point3f &p, Normal3f &n, float &pdf) const override {
        m_mesh->samplePosition(s, p, n, pdf);
        return m_radiance;
    }
    float pdf() const override { return 1.0f / m_mesh->getDiscretePDF().getSum(); }
    std::string toString() const override { return "AreaLight[radiance = " + m_radiance.toString() + "]"; }

private:
    Color3f m_radiance;
};

// ---- media (src/cpu/homogeneous.cpp, src/cpu/heterogeneous.cpp) -----------------------
class HomogeneousMedium : public Medium {
public:
    explicit HomogeneousMedium(const PropertyList &p) {
        m_sa = readScalarOrColor(p, "sigmaA", 0.0f);
        m_ss = readScalarOrColor(p, "sigmaS", 0.3f);
        m_g = p.getFloat("g", 0.0f);
        Point3f bmin = p.getPoint("boundsMin", Point3f(1e18f)), bmax = p.getPoint("boundsMax", Point3f(-1e18f));
        m_explicit = bmin.x() < 1e17f && bmax.x() > -1e17f;
        if (m_explicit) m_bounds = BoundingBox3f(bmin, bmax);
    }
    float getSigmaA() const override { return m_sa.r(); }
    float getSigmaS() const override { return m_ss.r(); }
    Color3f getSigmaARGB() const override { return m_sa; }
    Color3f getSigmaSRGB() const override { return m_ss; }
    float getPhaseG() const override { return m_g; }
    bool hasExplicitBounds() const override { return m_explicit; }
    BoundingBox3f getExplicitBounds() const override { return m_bounds; }
    std::string toString() const override { return "HomogeneousMedium[]"; }

private:
    Color3f m_sa, m_ss;
    float m_g;
    bool m_explicit = false;
    BoundingBox3f m_bounds;
};

class HeterogeneousMedium : public Medium {
public:
    explicit HeterogeneousMedium(const PropertyList &p) {
        m_sa = readScalarOrColor(p, "sigmaA", 0.0f);
        m_ss = readScalarOrColor(p, "sigmaS", 5.0f);
        m_g = p.getFloat("g", 0.85f);
        m_path = p.getString("volume", "");
        m_bounds = BoundingBox3f(p.getPoint("boundsMin"), p.getPoint("boundsMax"));
    }
    float getSigmaA() const override { return m_sa.r(); }
    float getSigmaS() const override { return m_ss.r(); }
    Color3f getSigmaARGB() const override { return m_sa; }
    Color3f getSigmaSRGB() const override { return m_ss; }
    float getPhaseG() const override { return m_g; }
    bool isHeterogeneous() const override { return true; }
    std::string getVolumePath() const override { return m_path; }
    bool hasExplicitBounds() const override { return true; }
    BoundingBox3f getExplicitBounds() const override { return m_bounds; }
    std::string toString() const override { return "HeterogeneousMedium[volume = " + m_path + "]"; }

private:
    Color3f m_sa, m_ss;
    float m_g;
    std::string m_path;
    BoundingBox3f m_bounds;
};

// ---- Gaussian filter (src/cpu/rfilter.cpp) ----------------------------------------------
class GaussianFilter : public ReconstructionFilter {
public:
    explicit GaussianFilter(const PropertyList &p) {
        m_radius = p.getFloat("radius", 2.0f);
        m_stddev = p.getFloat("stddev", 0.5f);
        m_alpha = std::exp(-m_stddev * m_stddev * m_radius * m_radius);
    }
    float eval(float x) const override { return std::max(0.0f, std::exp(-m_stddev * m_stddev * x * x) - m_alpha); }
    std::string toString() const override { return "GaussianFilter[]"; }

private:
    float m_stddev, m_alpha;
};

// ---- perspective camera (src/cpu/perspective.cpp) -------------------------------------------
class PerspectiveCamera : public Camera {
public:
    explicit PerspectiveCamera(const PropertyList &p) {
        m_outputSize[0] = p.getInteger("width", 1280);
        m_outputSize[1] = p.getInteger("height", 720);
        m_cameraToWorld = p.getTransform("toWorld", Transform());
        m_fov = p.getFloat("fov", 30.0f);
        m_near = p.getFloat("nearClip", 1e-4f);
        m_far = p.getFloat("farClip", 1e4f);
        m_lensRadius = p.getFloat("lensRadius", 0.0f);
        m_focalDistance = p.getFloat("focalDistance", 1.0f);
    }
    void activate() override {
        float aspect = m_outputSize[0] / (float)m_outputSize[1];
        float recip = 1.0f / (m_far - m_near), cot = 1.0f / std::tan(degToRad(m_fov / 2.0f));
        float P[4][4] = {{cot, 0, 0, 0}, {0, cot, 0, 0}, {0, 0, m_far * recip, -m_near * m_far * recip}, {0, 0, 1, 0}};
        float T[4][4] = {{1, 0, 0, -1.0f}, {0, 1, 0, -1.0f / aspect}, {0, 0, 1, 0}, {0, 0, 0, 1}};
        float S[4][4] = {{-0.5f, 0, 0, 0}, {0, -0.5f * aspect, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}};
        m_sampleToCamera = (Transform(S) * Transform(T) * Transform(P)).inverse();
        if (!m_rfilter) m_rfilter = static_cast<ReconstructionFilter *>(NoriObjectFactory::createInstance("gaussian", PropertyList()));
    }
    Color3f sampleRay(Ray3f &ray, const Point2f &pos, const Point2f &aperture) const override {
        Point3f nearP = m_sampleToCamera.point(Point3f(pos.x() / m_outputSize[0], pos.y() / m_outputSize[1], 0.0f));
        Vector3f d = nearP.normalized();
        Point3f o(0.0f, 0.0f, 0.0f);
        if (m_lensRadius > 0.0f) {
            float r = std::sqrt(aperture.x()) * m_lensRadius, th = 2.0f * M_PI_F * aperture.y();
            Point3f lens(r * std::cos(th), r * std::sin(th), 0.0f);
            float ft = m_focalDistance / d.z();
            Point3f focus = d * ft;
            o = lens;
            d = (focus - lens).normalized();
        }
        float invZ = 1.0f / d.z();
        ray.o = m_cameraToWorld.point(o);
        ray.d = m_cameraToWorld.vector(d);
        ray.mint = m_near * invZ;
        ray.maxt = m_far * invZ;
        return Color3f(1.0f);
    }
    float getLensRadius() const override { return m_lensRadius; }
    float getFocalDistance() const override { return m_focalDistance; }
    void addChild(NoriObject *obj) override {
        if (obj->getClassType() != EReconstructionFilter)
            throw NoriException("Camera::addChild(<" + classTypeName(obj->getClassType()) + ">) is not supported!");
        if (m_rfilter) throw NoriException("Camera: tried to register multiple reconstruction filters!");
        m_rfilter = static_cast<ReconstructionFilter *>(obj);
    }
    std::string toString() const override { return "PerspectiveCamera[]"; }

private:
    Transform m_sampleToCamera, m_cameraToWorld;
    float m_fov, m_near, m_far, m_lensRadius, m_focalDistance;
};

// ---- independent sampler (src/cpu/independent.cpp) -------------------------------------------
// PCG32 (O'Neill, pcg-random.org: 64-bit LCG state, XSH-RR output), unit
// floats from the top 23 bits.
class Independent : public Sampler {
public:
    explicit Independent(const PropertyList &p) { m_sampleCount = (size_t)p.getInteger("sampleCount", 1); seed(0, 1); }
    std::unique_ptr<Sampler> clone() const override { return std::unique_ptr<Sampler>(new Independent(*this)); }
    void generate() override {}
    void advance() override {}
    float next1D() override { return nextFloat(); }
    Point2f next2D() override { float a = nextFloat(); float b = nextFloat(); return Point2f(a, b); }
    void seed(uint64_t initstate, uint64_t initseq) {
        state = 0u;
        inc = (initseq << 1u) | 1u;
        nextUInt();
        state += initstate;
        nextUInt();
    }
    std::string toString() const override { return "Independent[sampleCount = " + std::to_string(m_sampleCount) + "]"; }

private:
    uint64_t state = 0, inc = 1;
    uint32_t nextUInt() {
        uint64_t old = state;
        state = old * 6364136223846793005ULL + inc;
        uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        return (xs >> rot) | (xs << ((~rot + 1u) & 31));
    }
    float nextFloat() {
        uint32_t u = (nextUInt() >> 9) | 0x3f800000u;
        float f;
        std::memcpy(&f, &u, 4);
        return f - 1.0f;
    }
};

// ---- meshes (src/cpu/mesh.cpp, src/cpu/obj.cpp) -------------------------------------------------
Mesh::~Mesh() {
    delete m_bsdf;
    delete m_emitter;
}
void Mesh::activate() {
    if (!m_bsdf) m_bsdf = static_cast<BSDF *>(NoriObjectFactory::createInstance("diffuse", PropertyList()));
    m_dpdf.clear();
    for (uint32_t i = 0; i < getTriangleCount(); ++i) m_dpdf.append(surfaceArea(i));
    m_dpdf.normalize();
}
float Mesh::surfaceArea(uint32_t index) const {
    const uint32_t *f = &m_F[3 * index];
    Vec3 p0(m_V[3 * f[0]], m_V[3 * f[0] + 1], m_V[3 * f[0] + 2]);
    Vec3 p1(m_V[3 * f[1]], m_V[3 * f[1] + 1], m_V[3 * f[1] + 2]);
    Vec3 p2(m_V[3 * f[2]], m_V[3 * f[2] + 1], m_V[3 * f[2] + 2]);
    return 0.5f * (p1 - p0).cross(p2 - p0).norm();
}
void Mesh::samplePosition(const Point2f &sample, Point3f &p, Normal3f &n, float &pdf) const {
    float reused = sample.x();
    size_t t = m_dpdf.sampleReuse(reused);
    const uint32_t *f = &m_F[3 * t];
    Vec3 p0(m_V[3 * f[0]], m_V[3 * f[0] + 1], m_V[3 * f[0] + 2]);
    Vec3 p1(m_V[3 * f[1]], m_V[3 * f[1] + 1], m_V[3 * f[1] + 2]);
    Vec3 p2(m_V[3 * f[2]], m_V[3 * f[2] + 1], m_V[3 * f[2] + 2]);
    float a = 1.0f - std::sqrt(1.0f - reused);
    float b = sample.y() * std::sqrt(1.0f - reused);
    p = p0 * a + p1 * b + p2 * (1.0f - a - b);
    n = (p1 - p0).cross(p2 - p0).normalized();
    pdf = 1.0f / m_dpdf.getSum();
}
void Mesh::addChild(NoriObject *obj) {
    switch (obj->getClassType()) {
        case EBSDF:
            if (m_bsdf) throw NoriException("Mesh: tried to register multiple BSDF instances!");
            m_bsdf = static_cast<BSDF *>(obj);
            break;
        case EEmitter: {
            Emitter *e = static_cast<Emitter *>(obj);
            if (m_emitter) throw NoriException("Mesh: tried to register multiple Emitter instances!");
            m_emitter = e;
            e->setMesh(this);
            break;
        }
        default:
            throw NoriException("Mesh::addChild(<" + classTypeName(obj->getClassType()) + ">) is not supported!");
    }
}
std::string Mesh::toString() const {
    return "Mesh[name = \"" + m_name + "\", vertexCount = " + std::to_string(getVertexCount()) +
           ", triangleCount = " + std::to_string(getTriangleCount()) + "]";
}

class WavefrontOBJ : public Mesh {
public:
    explicit WavefrontOBJ(const PropertyList &propList) {
        std::string filename = resolvePath(propList.getString("filename"));
        std::ifstream is(filename);
        if (is.fail()) throw NoriException("Unable to open OBJ file \"" + filename + "\"!");
        Transform trafo = propList.getTransform("toWorld", Transform());
        std::vector<Vec3> positions, normals;
        std::vector<Point2f> texcoords;
        struct Key { int p, uv, n; bool operator==(const Key &o) const { return p == o.p && uv == o.uv && n == o.n; } };
        struct KeyHash { size_t operator()(const Key &k) const { return ((size_t)k.p * 73856093u) ^ ((size_t)k.uv * 19349663u) ^ ((size_t)k.n * 83492791u); } };
        std::unordered_map<Key, uint32_t, KeyHash> vmap;
        std::vector<Key> verts;
        std::vector<uint32_t> indices;
        auto parseVert = [](const std::string &s) {
            Key k{0, 0, 0};
            int *f[3] = {&k.p, &k.uv, &k.n};
            size_t b = 0;
            for (int i = 0; i < 3 && b <= s.size(); i++) {
                size_t e = s.find('/', b);
                std::string t = s.substr(b, e == std::string::npos ? std::string::npos : e - b);
                if (!t.empty()) *f[i] = std::atoi(t.c_str());
                if (e == std::string::npos) break;
                b = e + 1;
            }
            return k;
        };
        std::string line;
        while (std::getline(is, line)) {
            std::istringstream ls(line);
            std::string prefix;
            ls >> prefix;
            if (prefix == "v") {
                Vec3 p;
                ls >> p.x() >> p.y() >> p.z();
                p = trafo.point(p);
                m_bbox.expandBy(p);
                positions.push_back(p);
            } else if (prefix == "vt") {
                Point2f t;
                ls >> t.x() >> t.y();
                texcoords.push_back(t);
            } else if (prefix == "vn") {
                Vec3 n;
                ls >> n.x() >> n.y() >> n.z();
                normals.push_back(trafo.normal(n).normalized());
            } else if (prefix == "f") {
                std::string a[4];
                ls >> a[0] >> a[1] >> a[2] >> a[3];
                Key v[6] = {parseVert(a[0]), parseVert(a[1]), parseVert(a[2])};
                int nv = 3;
                if (!a[3].empty()) { v[3] = parseVert(a[3]); v[4] = v[0]; v[5] = v[2]; nv = 6; }
                for (int i = 0; i < nv; i++) {
                    auto it = vmap.find(v[i]);
                    if (it == vmap.end()) {
                        vmap[v[i]] = (uint32_t)verts.size();
                        indices.push_back((uint32_t)verts.size());
                        verts.push_back(v[i]);
                    } else {
                        indices.push_back(it->second);
                    }
                }
            }
        }
        m_F = indices;
        m_V.resize(verts.size() * 3);
        for (size_t i = 0; i < verts.size(); i++) {
            if (verts[i].p < 1 || verts[i].p > (int)positions.size()) throw NoriException("OBJ: bad vertex index");
            const Vec3 &p = positions[verts[i].p - 1];
            m_V[3 * i] = p[0]; m_V[3 * i + 1] = p[1]; m_V[3 * i + 2] = p[2];
        }
        m_N.assign(verts.size() * 3, 0.0f);
        if (!normals.empty()) {
            for (size_t i = 0; i < verts.size(); i++) {
                const Vec3 &n = normals.at(verts[i].n - 1);
                m_N[3 * i] = n[0]; m_N[3 * i + 1] = n[1]; m_N[3 * i + 2] = n[2];
            }
        } else {  // angle-weighted smooth normals (src/cpu/obj.cpp:96-127)
            auto P = [&](uint32_t i) { return Vec3(m_V[3 * i], m_V[3 * i + 1], m_V[3 * i + 2]); };
            auto ang = [](const Vec3 &a, const Vec3 &b) {
                float d = a.normalized().dot(b.normalized());
                return std::acos(std::max(-1.0f, std::min(1.0f, d)));
            };
            std::vector<Vec3> acc(verts.size(), Vec3(0.0f));
            for (size_t t = 0; t < m_F.size() / 3; t++) {
                uint32_t i0 = m_F[3 * t], i1 = m_F[3 * t + 1], i2 = m_F[3 * t + 2];
                Vec3 e1 = P(i1) - P(i0), e2 = P(i2) - P(i0);
                Vec3 fn = e1.cross(e2);
                acc[i0] = acc[i0] + fn * ang(e1, e2);
                acc[i1] = acc[i1] + fn * ang(P(i0) - P(i1), P(i2) - P(i1));
                acc[i2] = acc[i2] + fn * ang(P(i0) - P(i2), P(i1) - P(i2));
            }
            for (size_t i = 0; i < verts.size(); i++) {
                float l = acc[i].norm();
                Vec3 n = l > 1e-8f ? acc[i] / l : acc[i];
                m_N[3 * i] = n[0]; m_N[3 * i + 1] = n[1]; m_N[3 * i + 2] = n[2];
            }
        }
        if (!texcoords.empty()) {
            m_UV.resize(verts.size() * 2);
            for (size_t i = 0; i < verts.size(); i++) {
                const Point2f &t = texcoords.at(verts[i].uv - 1);
                m_UV[2 * i] = t.x(); m_UV[2 * i + 1] = t.y();
            }
        }
        m_name = filename;
    }
};

// ---- hair strands (src/cpu/hair.cpp:43-322) -----------------------------------------------------
// A Cem Yuksel HAIR file (128-byte little-endian header "HAIR", strand and
// point counts, a flag word selecting the optional arrays, defaults; then
// the arrays: segments u16 per strand, points 3 x f32, thickness f32,
// transparency f32, colour 3 x f32 per point) tessellated into tubes of
// `sides` vertices per ring.  The vertex layout is the one the hair shading
// reads: UV = (position along the strand, (h + 1) / 2) with h = -cos(angle
// around the tube), tangent = strand direction at the ring.
class HairMesh : public Mesh {
public:
    explicit HairMesh(const PropertyList &propList) {
        std::string filename = resolvePath(propList.getString("filename"));
        int sides = propList.getInteger("sides", 6);
        float radiusScale = propList.getFloat("radiusScale", 1.0f);
        int maxStrands = propList.getInteger("maxStrands", -1);
        Transform trafo = propList.getTransform("toWorld", Transform());
        if (sides < 3) throw NoriException("hair: \"sides\" must be at least 3");
        std::ifstream f(filename, std::ios::binary);
        if (!f) throw NoriException("hair: cannot open \"" + filename + "\"");
        unsigned char hdr[128];
        f.read(reinterpret_cast<char *>(hdr), 128);
        if (!f || std::memcmp(hdr, "HAIR", 4) != 0) throw NoriException("hair: \"" + filename + "\" is not a HAIR file");
        auto u32 = [&](int o) { uint32_t v; std::memcpy(&v, hdr + o, 4); return v; };
        auto f32 = [&](int o) { float v; std::memcpy(&v, hdr + o, 4); return v; };
        const uint32_t numStrands = u32(4), numPoints = u32(8), flags = u32(12), defSegs = u32(16);
        const float defThickness = f32(20);
        if (!(flags & 2u)) throw NoriException("hair: \"" + filename + "\" has no points array");
        std::vector<uint16_t> segs;
        if (flags & 1u) {
            segs.resize(numStrands);
            f.read(reinterpret_cast<char *>(segs.data()), (std::streamsize)numStrands * 2);
        }
        std::vector<float> pts((size_t)numPoints * 3), thick;
        f.read(reinterpret_cast<char *>(pts.data()), (std::streamsize)pts.size() * 4);
        if (flags & 4u) {
            thick.resize(numPoints);
            f.read(reinterpret_cast<char *>(thick.data()), (std::streamsize)numPoints * 4);
        }
        if (!f) throw NoriException("hair: \"" + filename + "\" is truncated");
        // strand point ranges; the counts must add up to numPoints
        std::vector<std::pair<uint32_t, uint32_t>> strands;  // (first point, point count)
        uint64_t at = 0;
        for (uint32_t s = 0; s < numStrands; s++) {
            uint32_t n = (segs.empty() ? defSegs : segs[s]) + 1u;
            strands.push_back({(uint32_t)at, n});
            at += n;
        }
        if (at != numPoints) throw NoriException("hair: \"" + filename + "\": strand point counts do not add up");
        if (maxStrands > 0 && (uint32_t)maxStrands < numStrands) strands.resize((size_t)maxStrands);
        auto P = [&](uint32_t i) { return trafo.point(Vec3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2])); };
        const float kTwoPi = 6.28318530717958647692f;
        for (const auto &st : strands) {
            const uint32_t first = st.first, n = st.second;
            if (n < 2) continue;
            const uint32_t ring0 = (uint32_t)(m_V.size() / 3);
            for (uint32_t p = 0; p < n; p++) {
                Vec3 c = P(first + p);
                m_bbox.expandBy(c);
                Vec3 t = p == 0 ? P(first + 1) - P(first) : p == n - 1 ? P(first + p) - P(first + p - 1)
                                                                     : P(first + p + 1) - P(first + p - 1);
                t = t.normalized();
                Vec3 ref = std::abs(t.x()) < 0.9f ? Vec3(1.0f, 0.0f, 0.0f) : Vec3(0.0f, 1.0f, 0.0f);
                Vec3 b = t.cross(ref).normalized();
                Vec3 nr = t.cross(b).normalized();
                float radius = (thick.empty() ? defThickness : thick[first + p]) * 0.5f * radiusScale;
                float along = (float)p / (float)(n - 1);
                for (int k = 0; k < sides; k++) {
                    float ang = kTwoPi * (float)k / (float)sides;
                    Vec3 radial = b * std::cos(ang) + nr * std::sin(ang);
                    Vec3 v = c + radial * radius;
                    Vec3 nn = radial.normalized();
                    float h = -std::cos(ang);
                    for (int a = 0; a < 3; a++) { m_V.push_back(v[a]); m_N.push_back(nn[a]); m_T.push_back(t[a]); }
                    m_UV.push_back(along);
                    m_UV.push_back((h + 1.0f) * 0.5f);
                }
                if (p > 0) {  // two triangles per quad between this ring and the previous one
                    uint32_t prev = ring0 + (p - 1) * (uint32_t)sides, cur = ring0 + p * (uint32_t)sides;
                    for (uint32_t k = 0; k < (uint32_t)sides; k++) {
                        uint32_t k1 = (k + 1) % (uint32_t)sides;
                        uint32_t tri[6] = {prev + k, prev + k1, cur + k1, prev + k, cur + k1, cur + k};
                        m_F.insert(m_F.end(), tri, tri + 6);
                    }
                }
            }
        }
        if (m_F.empty()) throw NoriException("hair: \"" + filename + "\" has no strand with two points");
        m_name = filename;
    }
};

// ---- scene (src/cpu/scene.cpp) ------------------------------------------------------------------
Scene::Scene(const PropertyList &p) {
    m_envmap = p.getString("envmap", "textures/white_furnace.hdr");
    m_envmapScale = p.getFloat("envmapScale", 1.0f);
    m_evCompensation = p.getFloat("evCompensation", 0.0f);
}
Scene::~Scene() {
    for (Mesh *m : m_meshes) delete m;
    delete m_sampler;
    delete m_camera;
    delete m_integrator;
    delete m_medium;
}
void Scene::activate() {
    for (Mesh *m : m_meshes) {
        const BoundingBox3f &b = m->getBoundingBox();
        if (b.isValid()) { m_bbox.expandBy(b.min); m_bbox.expandBy(b.max); }
    }
    // The reference's GPU build ignores the integrator tag and always runs its
    // path tracer (MAX_BOUNCES 32; src/cpu/scene.cpp:36-37 only warns), so a
    // scene without one gets the GPU path tracer here.
    if (!m_integrator) {
        std::fprintf(stderr, "Warning: No integrator was specified; rendering with path_mis.\n");
        m_integrator = static_cast<Integrator *>(NoriObjectFactory::createInstance("path_mis", PropertyList()));
    }
    if (!m_camera) throw NoriException("No camera was specified!");
    if (!m_sampler) m_sampler = static_cast<Sampler *>(NoriObjectFactory::createInstance("independent", PropertyList()));
}
void Scene::addChild(NoriObject *obj) {
    switch (obj->getClassType()) {
        case EMesh: m_meshes.push_back(static_cast<Mesh *>(obj)); break;
        case EEmitter: break;  // area emitters are children of meshes
        case ESampler:
            if (m_sampler) throw NoriException("There can only be one sampler per scene!");
            m_sampler = static_cast<Sampler *>(obj);
            break;
        case ECamera:
            if (m_camera) throw NoriException("There can only be one camera per scene!");
            m_camera = static_cast<Camera *>(obj);
            break;
        case EIntegrator:
            if (m_integrator) throw NoriException("There can only be one integrator per scene!");
            m_integrator = static_cast<Integrator *>(obj);
            break;
        case EMedium:
            if (m_medium) throw NoriException("There can only be one medium per scene!");
            m_medium = static_cast<Medium *>(obj);
            break;
        default:
            throw NoriException("Scene::addChild(<" + classTypeName(obj->getClassType()) + ">) is not supported!");
    }
}
std::string Scene::toString() const {
    return "Scene[meshes = " + std::to_string(m_meshes.size()) + ", envmap = \"" + m_envmap + "\"]";
}

NORI_REGISTER_CLASS(Diffuse, "diffuse")
NORI_REGISTER_CLASS(Mirror, "mirror")
NORI_REGISTER_CLASS(Dielectric, "dielectric")
NORI_REGISTER_CLASS(Microfacet, "microfacet")
NORI_REGISTER_CLASS(Disney, "disney")
NORI_REGISTER_CLASS(HairBSDF, "hair_bsdf")
NORI_REGISTER_CLASS(Subsurface, "subsurface")
NORI_REGISTER_CLASS(AreaLight, "area")
NORI_REGISTER_CLASS(HomogeneousMedium, "homogeneous")
NORI_REGISTER_CLASS(HeterogeneousMedium, "heterogeneous")
NORI_REGISTER_CLASS(GaussianFilter, "gaussian")
NORI_REGISTER_CLASS(PerspectiveCamera, "perspective")
NORI_REGISTER_CLASS(Independent, "independent")
NORI_REGISTER_CLASS(WavefrontOBJ, "obj")
NORI_REGISTER_CLASS(HairMesh, "hair")
NORI_REGISTER_CLASS(Scene, "scene")

}  // namespace nori
