// nori.h — the Nori plugin API of the reference (gracejinsotrue/PBRT-renderer-,
// include/*.h), restated in C++17 without Eigen/TBB/pugixml, on top of libpt.
//
// Same names, argument meanings and error behaviour as the reference:
// NoriObject / NoriObjectFactory / NORI_REGISTER_CLASS (include/object.h),
// PropertyList (include/proplist.h), loadFromXML (include/parser.h), BSDF /
// BSDFQueryRecord / BSDFGPUData (include/bsdf.h), Emitter (include/emitter.h),
// Medium (include/medium.h), Camera (include/camera.h), Sampler
// (include/sampler.h), Mesh (include/mesh.h), Scene (include/scene.h) and
// Integrator (include/integrator.h).  Errors are NoriException.
//
// Differences, by design: the vector types are small structs with Eigen-like
// accessors (x(), dot(), cross(), norm(), normalized()); the "path_mis" and
// "direct" integrators, which the reference's scene files request but which
// it never implemented, exist and render on the GPU through libpt; the
// Disney and hair BSDFs evaluate the real models (the reference's CPU
// versions are Lambertian stand-ins for its shader code).
#pragma once

#include <cmath>
#include <cstdint>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/pt.h"

namespace nori {

// ---- errors ------------------------------------------------------------------
class NoriException : public std::runtime_error {
public:
    explicit NoriException(const std::string &msg) : std::runtime_error(msg) {}
};

constexpr float Epsilon = 1e-4f;  // include/common.h:38
constexpr float M_PI_F = 3.14159265358979323846f;
inline float degToRad(float v) { return v * (M_PI_F / 180.0f); }

// ---- small math types --------------------------------------------------------
struct Vec3 {
    float v[3] = {0, 0, 0};
    Vec3() = default;
    Vec3(float a, float b, float c) : v{a, b, c} {}
    explicit Vec3(float a) : v{a, a, a} {}
    float &x() { return v[0]; }
    float &y() { return v[1]; }
    float &z() { return v[2]; }
    float x() const { return v[0]; }
    float y() const { return v[1]; }
    float z() const { return v[2]; }
    float &operator[](int i) { return v[i]; }
    float operator[](int i) const { return v[i]; }
    Vec3 operator+(const Vec3 &o) const { return {v[0] + o.v[0], v[1] + o.v[1], v[2] + o.v[2]}; }
    Vec3 operator-(const Vec3 &o) const { return {v[0] - o.v[0], v[1] - o.v[1], v[2] - o.v[2]}; }
    Vec3 operator-() const { return {-v[0], -v[1], -v[2]}; }
    Vec3 operator*(float s) const { return {v[0] * s, v[1] * s, v[2] * s}; }
    Vec3 operator/(float s) const { return {v[0] / s, v[1] / s, v[2] / s}; }
    Vec3 cwiseProduct(const Vec3 &o) const { return {v[0] * o.v[0], v[1] * o.v[1], v[2] * o.v[2]}; }
    float dot(const Vec3 &o) const { return v[0] * o.v[0] + v[1] * o.v[1] + v[2] * o.v[2]; }
    Vec3 cross(const Vec3 &o) const {
        return {v[1] * o.v[2] - v[2] * o.v[1], v[2] * o.v[0] - v[0] * o.v[2], v[0] * o.v[1] - v[1] * o.v[0]};
    }
    float squaredNorm() const { return dot(*this); }
    float norm() const { return std::sqrt(squaredNorm()); }
    Vec3 normalized() const { return *this / norm(); }
};
inline Vec3 operator*(float s, const Vec3 &a) { return a * s; }
using Vector3f = Vec3;
using Point3f = Vec3;
using Normal3f = Vec3;

struct Point2f {
    float v[2] = {0, 0};
    Point2f() = default;
    Point2f(float a, float b) : v{a, b} {}
    float &x() { return v[0]; }
    float &y() { return v[1]; }
    float x() const { return v[0]; }
    float y() const { return v[1]; }
};
using Vector2f = Point2f;

struct Color3f {
    float c[3] = {0, 0, 0};
    Color3f() = default;
    explicit Color3f(float s) : c{s, s, s} {}
    Color3f(float r_, float g_, float b_) : c{r_, g_, b_} {}
    float &r() { return c[0]; }
    float &g() { return c[1]; }
    float &b() { return c[2]; }
    float r() const { return c[0]; }
    float g() const { return c[1]; }
    float b() const { return c[2]; }
    float operator[](int i) const { return c[i]; }
    float &operator[](int i) { return c[i]; }
    Color3f operator*(const Color3f &o) const { return {c[0] * o.c[0], c[1] * o.c[1], c[2] * o.c[2]}; }
    Color3f operator*(float s) const { return {c[0] * s, c[1] * s, c[2] * s}; }
    Color3f operator+(const Color3f &o) const { return {c[0] + o.c[0], c[1] + o.c[1], c[2] + o.c[2]}; }
    float getLuminance() const { return c[0] * 0.212671f + c[1] * 0.715160f + c[2] * 0.072169f; }  // src/cpu/common.cpp:207-209
    std::string toString() const;
};

// 4x4 affine transform with its inverse (include/transform.h).
struct Transform {
    float m[4][4];
    float inv[4][4];
    Transform();
    explicit Transform(const float mat[4][4]);
    Transform inverse() const;
    Transform operator*(const Transform &t) const;
    Point3f point(const Point3f &p) const;     // homogeneous point
    Vector3f vector(const Vector3f &v) const;  // direction (no translation)
    Normal3f normal(const Normal3f &n) const;  // inverse transpose
    std::string toString() const;
};

struct BoundingBox3f {
    Point3f min{1e30f, 1e30f, 1e30f}, max{-1e30f, -1e30f, -1e30f};
    BoundingBox3f() = default;
    BoundingBox3f(const Point3f &a, const Point3f &b) : min(a), max(b) {}
    void expandBy(const Point3f &p) {
        for (int i = 0; i < 3; i++) { min[i] = std::min(min[i], p[i]); max[i] = std::max(max[i], p[i]); }
    }
    bool isValid() const { return min[0] <= max[0] && min[1] <= max[1] && min[2] <= max[2]; }
};

struct Ray3f {  // include/ray.h
    Point3f o;
    Vector3f d;
    float mint = Epsilon, maxt = INFINITY;
};

// ---- properties (include/proplist.h) -----------------------------------------
class PropertyList {
public:
    void setBoolean(const std::string &name, bool value);
    bool getBoolean(const std::string &name) const;
    bool getBoolean(const std::string &name, bool defaultValue) const;
    void setInteger(const std::string &name, int value);
    int getInteger(const std::string &name) const;
    int getInteger(const std::string &name, int defaultValue) const;
    void setFloat(const std::string &name, float value);
    float getFloat(const std::string &name) const;
    float getFloat(const std::string &name, float defaultValue) const;
    void setString(const std::string &name, const std::string &value);
    std::string getString(const std::string &name) const;
    std::string getString(const std::string &name, const std::string &defaultValue) const;
    void setColor(const std::string &name, const Color3f &value);
    Color3f getColor(const std::string &name) const;
    Color3f getColor(const std::string &name, const Color3f &defaultValue) const;
    void setPoint(const std::string &name, const Point3f &value);
    Point3f getPoint(const std::string &name) const;
    Point3f getPoint(const std::string &name, const Point3f &defaultValue) const;
    void setVector(const std::string &name, const Vector3f &value);
    Vector3f getVector(const std::string &name) const;
    Vector3f getVector(const std::string &name, const Vector3f &defaultValue) const;
    void setTransform(const std::string &name, const Transform &value);
    Transform getTransform(const std::string &name) const;
    Transform getTransform(const std::string &name, const Transform &defaultValue) const;

private:
    enum Type { Boolean, Integer, Float, String, Color, Point, Vector, TransformT };
    struct Property {
        Type type;
        bool b = false;
        int i = 0;
        float f = 0;
        std::string s;
        Color3f c;
        Vec3 p;
        Transform t;
    };
    const Property *find(const std::string &name, Type type, bool required) const;
    void put(const std::string &name, Property p);
    std::map<std::string, Property> m_props;
};

// ---- objects (include/object.h) -----------------------------------------------
class NoriObject {
public:
    enum EClassType {
        EScene = 0, EMesh, EBSDF, EPhaseFunction, EEmitter, EMedium, ECamera, EIntegrator, ESampler, ETest,
        EReconstructionFilter, EClassTypeCount
    };
    virtual ~NoriObject() {}
    virtual EClassType getClassType() const = 0;
    virtual void addChild(NoriObject *child);
    virtual void setParent(NoriObject *) {}
    virtual void activate() {}
    virtual std::string toString() const = 0;
    static std::string classTypeName(EClassType type);
};

class NoriObjectFactory {
public:
    using Constructor = std::function<NoriObject *(const PropertyList &)>;
    static void registerClass(const std::string &name, const Constructor &constr);
    static NoriObject *createInstance(const std::string &name, const PropertyList &propList);
    static std::vector<std::string> registeredClasses();
};

#define NORI_REGISTER_CLASS(cls, name)                                                     \
    static nori::NoriObject *cls##_create(const nori::PropertyList &list) { return new cls(list); } \
    static struct cls##_ {                                                                 \
        cls##_() { nori::NoriObjectFactory::registerClass(name, cls##_create); }           \
    } cls##__NORI_;

// ---- BSDF (include/bsdf.h) -------------------------------------------------------
enum EMeasure { EUnknownMeasure = 0, ESolidAngle, EDiscrete };

struct BSDFQueryRecord {
    Vector3f wi, wo;
    float eta = 1.0f;
    EMeasure measure = EUnknownMeasure;
    Point2f uv;
    float h = 0.0f;  // hair fibre offset in [-1, 1] (the shader's UV-derived h)
    explicit BSDFQueryRecord(const Vector3f &wi_) : wi(wi_) {}
    BSDFQueryRecord(const Vector3f &wi_, const Vector3f &wo_, EMeasure m) : wi(wi_), wo(wo_), measure(m) {}
};

struct BSDFGPUData {
    enum Type { DIFFUSE = 0, MIRROR = 1, DIELECTRIC = 2, MICROFACET = 3, DISNEY = 4, HAIR = 5, SUBSURFACE = 6 };
    int type = DIFFUSE;
    float albedo[3] = {0.5f, 0.5f, 0.5f};
    float intIOR = 1.5046f, extIOR = 1.000277f, alpha = 0.1f;
    std::string albedoTexture, normalTexture, roughnessTexture, metallicTexture, specularTexture,
        subsurfaceTexture, alphaTexture;
    float roughness = 0.5f, metallic = 0.0f, specular = 0.5f, specularTint = 0.0f, sheen = 0.0f,
          sheenTint = 0.5f, subsurface = 0.0f, clearcoat = 0.0f, clearcoatGloss = 1.0f, anisotropic = 0.0f;
    float betaN = 0.3f;
};

class BSDF : public NoriObject {
public:
    virtual Color3f sample(BSDFQueryRecord &bRec, const Point2f &sample) const = 0;
    virtual Color3f eval(const BSDFQueryRecord &bRec) const = 0;
    virtual float pdf(const BSDFQueryRecord &bRec) const = 0;
    EClassType getClassType() const override { return EBSDF; }
    virtual bool isDiffuse() const { return false; }
    virtual BSDFGPUData getGPUData() const { return BSDFGPUData{}; }
};
// The GPU material record (pt_material) of a BSDF's GPU data.
pt_material toGPUMaterial(const BSDFGPUData &d);

// ---- mesh / emitter / medium ------------------------------------------------------
class Emitter;

struct DiscretePDF {  // include/dpdf.h
    std::vector<float> cdf{0.0f};
    float sum = 0.0f, normalization = 0.0f;
    bool normalized = false;
    void clear() { cdf.assign(1, 0.0f); normalized = false; }
    void append(float v) { cdf.push_back(cdf.back() + v); }
    size_t size() const { return cdf.size() - 1; }
    float normalize();
    float getSum() const { return sum; }
    size_t sample(float u) const;
    size_t sampleReuse(float &u) const;
};

class Mesh : public NoriObject {
public:
    ~Mesh() override;
    void activate() override;
    uint32_t getTriangleCount() const { return (uint32_t)m_F.size() / 3; }
    uint32_t getVertexCount() const { return (uint32_t)m_V.size() / 3; }
    float surfaceArea(uint32_t index) const;
    void samplePosition(const Point2f &sample, Point3f &p, Normal3f &n, float &pdf) const;
    const std::vector<float> &getVertexPositions() const { return m_V; }  // 3 floats per vertex
    const std::vector<float> &getVertexNormals() const { return m_N; }
    const std::vector<float> &getVertexTexCoords() const { return m_UV; }
    const std::vector<float> &getVertexTangents() const { return m_T; }
    const std::vector<uint32_t> &getIndices() const { return m_F; }
    bool hasTangents() const { return !m_T.empty(); }
    const BSDF *getBSDF() const { return m_bsdf; }
    bool isEmitter() const { return m_emitter != nullptr; }
    Emitter *getEmitter() { return m_emitter; }
    const Emitter *getEmitter() const { return m_emitter; }
    const DiscretePDF &getDiscretePDF() const { return m_dpdf; }
    const BoundingBox3f &getBoundingBox() const { return m_bbox; }
    void addChild(NoriObject *child) override;
    std::string toString() const override;
    EClassType getClassType() const override { return EMesh; }

protected:
    std::string m_name;
    std::vector<float> m_V, m_N, m_UV, m_T;
    std::vector<uint32_t> m_F;
    BSDF *m_bsdf = nullptr;
    Emitter *m_emitter = nullptr;
    BoundingBox3f m_bbox;
    DiscretePDF m_dpdf;
};

class Emitter : public NoriObject {
public:
    virtual Color3f getRadiance() const = 0;
    virtual Color3f sample(const Point2f &sample, Point3f &p, Normal3f &n, float &pdf) const = 0;
    virtual float pdf() const = 0;
    void setMesh(Mesh *mesh) { m_mesh = mesh; }
    const Mesh *getMesh() const { return m_mesh; }
    EClassType getClassType() const override { return EEmitter; }

protected:
    Mesh *m_mesh = nullptr;
};

Color3f readScalarOrColor(const PropertyList &propList, const std::string &name, float scalarDefault);

class Medium : public NoriObject {
public:
    virtual float getSigmaA() const = 0;
    virtual float getSigmaS() const = 0;
    virtual Color3f getSigmaARGB() const { return Color3f(getSigmaA()); }
    virtual Color3f getSigmaSRGB() const { return Color3f(getSigmaS()); }
    virtual float getPhaseG() const = 0;
    virtual bool isHeterogeneous() const { return false; }
    virtual std::string getVolumePath() const { return ""; }
    virtual bool hasExplicitBounds() const = 0;
    virtual BoundingBox3f getExplicitBounds() const = 0;
    EClassType getClassType() const override { return EMedium; }
};

// ---- camera / sampler / filter ---------------------------------------------------------
class ReconstructionFilter : public NoriObject {
public:
    float getRadius() const { return m_radius; }
    virtual float eval(float x) const = 0;
    EClassType getClassType() const override { return EReconstructionFilter; }

protected:
    float m_radius = 0.0f;
};

class Camera : public NoriObject {
public:
    virtual Color3f sampleRay(Ray3f &ray, const Point2f &samplePosition, const Point2f &apertureSample) const = 0;
    const int *getOutputSize() const { return m_outputSize; }
    virtual float getLensRadius() const { return 0.0f; }
    virtual float getFocalDistance() const { return 1.0f; }
    const ReconstructionFilter *getReconstructionFilter() const { return m_rfilter; }
    EClassType getClassType() const override { return ECamera; }

protected:
    int m_outputSize[2] = {1280, 720};
    ReconstructionFilter *m_rfilter = nullptr;
};

class Sampler : public NoriObject {
public:
    virtual std::unique_ptr<Sampler> clone() const = 0;
    virtual void generate() = 0;
    virtual void advance() = 0;
    virtual float next1D() = 0;
    virtual Point2f next2D() = 0;
    virtual size_t getSampleCount() const { return m_sampleCount; }
    EClassType getClassType() const override { return ESampler; }

protected:
    size_t m_sampleCount = 1;
};

// ---- scene / integrator ----------------------------------------------------------------
class Integrator;

class Scene : public NoriObject {
public:
    explicit Scene(const PropertyList &);
    ~Scene() override;
    const Integrator *getIntegrator() const { return m_integrator; }
    Integrator *getIntegrator() { return m_integrator; }
    const Camera *getCamera() const { return m_camera; }
    const Sampler *getSampler() const { return m_sampler; }
    const Medium *getMedium() const { return m_medium; }
    const std::vector<Mesh *> &getMeshes() const { return m_meshes; }
    const BoundingBox3f &getBoundingBox() const { return m_bbox; }
    const std::string &getEnvmap() const { return m_envmap; }
    float getEnvmapScale() const { return m_envmapScale; }
    float getEvCompensation() const { return m_evCompensation; }
    // directory of the scene file: what the scene names by relative path resolves there first
    const std::string &getBaseDir() const { return m_baseDir; }
    void setBaseDir(const std::string &dir) { m_baseDir = dir; }
    void activate() override;
    void addChild(NoriObject *obj) override;
    std::string toString() const override;
    EClassType getClassType() const override { return EScene; }

private:
    std::vector<Mesh *> m_meshes;
    Integrator *m_integrator = nullptr;
    Sampler *m_sampler = nullptr;
    Camera *m_camera = nullptr;
    Medium *m_medium = nullptr;
    BoundingBox3f m_bbox;
    std::string m_envmap, m_baseDir;
    float m_envmapScale = 1.0f, m_evCompensation = 0.0f;
};

// Film of a GPU render: per pixel sum of (L, 1) and its Kahan compensation.
struct RenderResult {
    int width = 0, height = 0;
    std::vector<float> sum, comp;  // 4 x width x height
    pt_stats stats{};
    std::vector<float> mean() const;  // 3 x width x height: sum.xyz / sum.w
};

class Integrator : public NoriObject {
public:
    ~Integrator() override {}
    virtual void preprocess(const Scene *scene) { (void)scene; }
    virtual Color3f Li(const Scene *scene, Sampler *sampler, const Ray3f &ray) const = 0;
    EClassType getClassType() const override { return EIntegrator; }
};

// A scene flattened into the arrays pt_upload_scene takes.  desc() points
// into the vectors, so the FlatScene outlives every upload made from it.
struct FlatScene {
    std::vector<float> pos, nrm, uv, tan, env;
    std::vector<uint32_t> idx;
    std::vector<pt_material> mats;
    uint32_t envW = 0, envH = 0;
    std::vector<pt_volume> vols;
    std::vector<std::vector<float>> gridData;
    std::vector<pt_grid> grids;
    std::vector<std::vector<uint8_t>> texData;  // RGBA8, level 0
    std::vector<pt_texture> textures;
    std::vector<std::string> texPaths;  // resolved file of each texture
    float envScale = 1.0f, evCompensation = 0.0f;
    pt_scene_desc desc() const;
};

// The GPU integrators ("path_mis", "direct"): preprocess() flattens the scene
// and uploads it through pt_upload_scene; render() runs pt_render.
class GPUIntegrator : public Integrator {
public:
    explicit GPUIntegrator(const PropertyList &props, uint32_t defaultDepth);
    ~GPUIntegrator() override;
    void preprocess(const Scene *scene) override;
    Color3f Li(const Scene *scene, Sampler *sampler, const Ray3f &ray) const override;
    // Render `spp` samples per pixel starting at sample `sampleOffset`; adds
    // into `film` when given (progressive), else into a fresh film.
    RenderResult render(uint32_t spp, uint32_t sampleOffset = 0, RenderResult *film = nullptr);
    pt_camera cameraConstants() const { return m_cam; }
    const pt_scene_desc &sceneDesc() const { return m_desc; }
    uint32_t maxDepth() const { return m_maxDepth; }
    std::string toString() const override;

protected:
    int m_device = 0;
    uint32_t m_maxDepth;
    uint32_t m_rng = PT_RNG_SOBOL_OWEN, m_envSampling = PT_ENV_CDF;
    pt_ctx *m_ctx = nullptr;
    const Scene *m_scene = nullptr;
    pt_camera m_cam{};
    int m_width = 0, m_height = 0;
    // flattened scene (CreateSceneBuffers, CreateTextures); kept alive while uploaded
    FlatScene m_flat;
    pt_scene_desc m_desc{};
};

// ---- loading -------------------------------------------------------------------------------
NoriObject *loadFromXML(const std::string &filename);
// Linear HDR image as an uncompressed OpenEXR file (rgb: W*H*3, top row first).
void writeEXR(const std::string &path, int width, int height, const float *rgb);

// Flatten a scene the way src/gpu/DXRApp_Scene.cpp:172-493 and
// src/gpu/DXRApp_Textures.cpp:181-275,448-537 do (shared with GPUIntegrator).
void flattenScene(const Scene *scene, FlatScene &out);
// A PNG / TGA / BMP / PPM / PGM image as 8-bit RGBA, top row first (the
// 4-channel load of src/gpu/DXRApp_Textures.cpp:34-40).  Throws
// NoriException for unreadable, malformed or unsupported files.
void loadImageRGBA8(const std::string &path, uint32_t &width, uint32_t &height, std::vector<uint8_t> &rgba);
// Camera constants of src/gpu/DXRApp_Camera.cpp:23-112 from a Nori camera.
pt_camera cameraConstants(const Camera *cam, int width, int height);

// File resolution relative to the scene file (filesystem/resolver.h): an
// absolute name as is, else baseDir/name when readable, else the first
// readable entry of the search paths (the directory of the XML being loaded
// while it loads, and any the caller pushed), else the name unchanged.
std::string resolvePath(const std::string &name, const std::string &baseDir = std::string());
void pushSearchPath(const std::string &dir);
void popSearchPath();
// Radiance .hdr (RGBE) loader; returns false when the file cannot be read.
bool loadHDR(const std::string &path, std::vector<float> &rgb, uint32_t &w, uint32_t &h);
// .vol density grid ("VOL1", W, H, D, bbox, float data): src/gpu/DXRApp_Scene.cpp:495-548.
bool loadVol(const std::string &path, std::vector<float> &data, uint32_t &w, uint32_t &h, uint32_t &d);

}  // namespace nori
