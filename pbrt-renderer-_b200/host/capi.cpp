// capi.cpp — a C surface over the Nori host for tools and tests (ctypes).
#include <cstdio>
#include <cstring>

#include "nori/nori.h"

using namespace nori;

namespace {
void seterr(char *err, size_t n, const char *msg) {
    if (err && n) {
        std::strncpy(err, msg, n - 1);
        err[n - 1] = 0;
    }
}
}  // namespace

extern "C" {

// Load a Nori XML scene; returns a Scene* or NULL (message in err).
void *nori_load(const char *xml, char *err, size_t errlen) {
    try {
        NoriObject *o = loadFromXML(xml);
        if (o->getClassType() != NoriObject::EScene) {
            delete o;
            seterr(err, errlen, "root object is not a scene");
            return nullptr;
        }
        return o;
    } catch (const std::exception &e) {
        seterr(err, errlen, e.what());
        return nullptr;
    }
}

void nori_free(void *scene) { delete static_cast<Scene *>(scene); }

// width, height, spp (sampler), meshes, triangles, emitters, has_medium, max_depth (0 = no GPU integrator)
int nori_info(void *scene, uint32_t *out8) {
    const Scene *s = static_cast<const Scene *>(scene);
    uint32_t tris = 0, em = 0;
    for (const Mesh *m : s->getMeshes()) { tris += m->getTriangleCount(); em += m->isEmitter() ? 1 : 0; }
    const GPUIntegrator *gi = dynamic_cast<const GPUIntegrator *>(s->getIntegrator());
    uint32_t v[8] = {(uint32_t)s->getCamera()->getOutputSize()[0], (uint32_t)s->getCamera()->getOutputSize()[1],
                     (uint32_t)s->getSampler()->getSampleCount(), (uint32_t)s->getMeshes().size(), tris, em,
                     s->getMedium() ? 1u : 0u, gi ? gi->maxDepth() : 0u};
    std::memcpy(out8, v, sizeof(v));
    return 0;
}

// The scene's envmapScale (no GPU needed).
float nori_env_scale(void *scene) { return static_cast<const Scene *>(scene)->getEnvmapScale(); }

// Camera constants the GPU integrator uses (no GPU needed).
int nori_camera(void *scene, pt_camera *out) {
    const Scene *s = static_cast<const Scene *>(scene);
    const Camera *c = s->getCamera();
    *out = cameraConstants(c, c->getOutputSize()[0], c->getOutputSize()[1]);
    return 0;
}

// Flattened materials in mesh order (no GPU needed); returns the count.
uint32_t nori_materials(void *scene, pt_material *out, uint32_t maxCount) {
    FlatScene f;
    flattenScene(static_cast<const Scene *>(scene), f);
    for (uint32_t i = 0; i < f.mats.size() && i < maxCount; i++) out[i] = f.mats[i];
    return (uint32_t)f.mats.size();
}

// One flattened scene array (no GPU needed): which = 0 positions, 1 normals,
// 2 texcoords, 3 tangents (floats), 4 indices (u32), 5 envmap RGB (floats),
// 6 envmap width, 7 texture count.  Copies into out when it is not NULL;
// returns the element count (the width for 6, the count for 7).
uint64_t nori_flat(void *scene, int which, void *out) {
    FlatScene f;
    flattenScene(static_cast<const Scene *>(scene), f);
    const std::vector<float> *v[] = {&f.pos, &f.nrm, &f.uv, &f.tan, nullptr, &f.env};
    if (which == 6) return f.envW;
    if (which == 7) return f.textures.size();
    if (which == 4) {
        if (out) std::memcpy(out, f.idx.data(), f.idx.size() * 4);
        return f.idx.size();
    }
    if (which < 0 || which > 5) return 0;
    if (out) std::memcpy(out, v[which]->data(), v[which]->size() * 4);
    return v[which]->size();
}

// Texture `index` of the flattened scene (no GPU needed): wh_srgb receives
// width, height, sRGB flag; the RGBA8 texels are copied into rgba when it is
// not NULL.  Returns the byte count, or 0 for an index out of range.
uint64_t nori_texture(void *scene, uint32_t index, uint32_t *wh_srgb, uint8_t *rgba) {
    FlatScene f;
    flattenScene(static_cast<const Scene *>(scene), f);
    if (index >= f.textures.size()) return 0;
    const pt_texture &t = f.textures[index];
    if (wh_srgb) {
        wh_srgb[0] = t.width;
        wh_srgb[1] = t.height;
        wh_srgb[2] = t.srgb;
    }
    if (rgba) std::memcpy(rgba, f.texData[index].data(), f.texData[index].size());
    return f.texData[index].size();
}

// Decode one image file to RGBA8 (no scene needed): wh receives width and
// height; the texels are copied into rgba when it is not NULL and cap bytes
// hold them.  Returns the byte count, or 0 with err set.
uint64_t nori_load_image(const char *path, uint32_t *wh, uint8_t *rgba, uint64_t cap, char *err, size_t errlen) {
    try {
        std::vector<uint8_t> px;
        uint32_t w = 0, h = 0;
        loadImageRGBA8(path ? path : "", w, h, px);
        if (wh) {
            wh[0] = w;
            wh[1] = h;
        }
        if (rgba && cap >= px.size()) std::memcpy(rgba, px.data(), px.size());
        return px.size();
    } catch (const std::exception &e) {
        seterr(err, errlen, e.what());
        return 0;
    }
}

// Write W x H x 3 floats (top row first) as an uncompressed OpenEXR file.
// Returns 0 or -1 (err set).
int nori_write_exr(const char *path, int width, int height, const float *rgb, char *err, size_t errlen) {
    try {
        writeEXR(path ? path : "", width, height, rgb);
        return 0;
    } catch (const std::exception &e) {
        seterr(err, errlen, e.what());
        return -1;
    }
}

// Render spp samples from sample_offset with the scene's GPU integrator into
// host films (4 x W x H floats each; added to).  Returns 0 or -1 (err set).
int nori_render(void *scene, uint32_t spp, uint32_t sample_offset, float *sum, float *comp, pt_stats *stats,
                char *err, size_t errlen) {
    try {
        Scene *s = static_cast<Scene *>(scene);
        GPUIntegrator *gi = dynamic_cast<GPUIntegrator *>(s->getIntegrator());
        if (!gi) throw NoriException("the scene has no GPU integrator (path_mis / direct)");
        if (!gi->cameraConstants().horizontal[0] && !gi->cameraConstants().vertical[1]) gi->preprocess(s);
        RenderResult film;
        int W = s->getCamera()->getOutputSize()[0], H = s->getCamera()->getOutputSize()[1];
        film.width = W;
        film.height = H;
        film.sum.assign(sum, sum + (size_t)W * H * 4);
        film.comp.assign(comp, comp + (size_t)W * H * 4);
        gi->render(spp, sample_offset, &film);
        std::memcpy(sum, film.sum.data(), film.sum.size() * 4);
        std::memcpy(comp, film.comp.data(), film.comp.size() * 4);
        if (stats) *stats = film.stats;
        return 0;
    } catch (const std::exception &e) {
        seterr(err, errlen, e.what());
        return -1;
    }
}

}  // extern "C"
