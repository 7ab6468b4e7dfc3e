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

// Camera constants the GPU integrator uses (no GPU needed).
int nori_camera(void *scene, pt_camera *out) {
    const Scene *s = static_cast<const Scene *>(scene);
    const Camera *c = s->getCamera();
    *out = cameraConstants(c, c->getOutputSize()[0], c->getOutputSize()[1]);
    return 0;
}

// Flattened materials in mesh order (no GPU needed); returns the count.
uint32_t nori_materials(void *scene, pt_material *out, uint32_t maxCount) {
    const Scene *s = static_cast<const Scene *>(scene);
    std::vector<float> pos, nrm, uv, tan, env;
    std::vector<uint32_t> idx;
    std::vector<pt_material> mats;
    std::vector<pt_volume> vols;
    std::vector<std::vector<float>> grids;
    std::vector<pt_grid> gd;
    uint32_t w, h;
    flattenScene(s, pos, nrm, uv, tan, idx, mats, env, w, h, vols, grids, gd);
    for (uint32_t i = 0; i < mats.size() && i < maxCount; i++) out[i] = mats[i];
    return (uint32_t)mats.size();
}

// One flattened scene array (no GPU needed): which = 0 positions, 1 normals,
// 2 texcoords, 3 tangents (floats), 4 indices (u32), 5 envmap RGB (floats),
// 6 envmap width.  Copies into out when it is not NULL; returns the element
// count (the width for 6).
uint64_t nori_flat(void *scene, int which, void *out) {
    const Scene *s = static_cast<const Scene *>(scene);
    std::vector<float> pos, nrm, uv, tan, env;
    std::vector<uint32_t> idx;
    std::vector<pt_material> mats;
    std::vector<pt_volume> vols;
    std::vector<std::vector<float>> grids;
    std::vector<pt_grid> gd;
    uint32_t w, h;
    flattenScene(s, pos, nrm, uv, tan, idx, mats, env, w, h, vols, grids, gd);
    const std::vector<float> *f[] = {&pos, &nrm, &uv, &tan, nullptr, &env};
    if (which == 6) return w;
    if (which == 4) {
        if (out) std::memcpy(out, idx.data(), idx.size() * 4);
        return idx.size();
    }
    if (which < 0 || which > 5) return 0;
    if (out) std::memcpy(out, f[which]->data(), f[which]->size() * 4);
    return f[which]->size();
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
