// pt_internal.h — context and shared declarations of libpt.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "pt_device.cuh"

#define PT_CUDA(call)                                                                  \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess) return ctx->fail(PT_E_CUDA, #call, cudaGetErrorString(e_)); \
    } while (0)

// Device error flag bits (raised by kernels, read after a sync).
enum : uint32_t {
    PT_DEVERR_STACK = 1u,     // traversal stack overflow
    PT_DEVERR_QUEUE = 2u,     // queue overflow
    PT_DEVERR_BVH = 4u,       // traversal visited more nodes than exist
    PT_DEVERR_CACHE = 8u,     // a radiance-cache kernel's bounded wait gave up
};

// Shading classes: the closest-hit kernel sorts each path into one of these
// queues and one shading kernel per class present in the scene runs with its
// material type fixed at compile time.
enum ShadeClass : int {
    CLS_ANY = -1,  // no classification (scenes with media: the medium decides first)
    CLS_MISS = 0,
    CLS_EMIT = 1,     // emitter hit (any material type)
    CLS_DELTA = 2,    // mirror, dielectric
    CLS_DIFFUSE = 3,
    CLS_MICRO = 4,
    CLS_DISNEY = 5,
    CLS_HAIR = 6,
    CLS_TEX = 7,  // + CLS_TEX: the same class for materials with shading textures
    CLS_MEDIUM = 14,  // a scattering event in a (homogeneous) medium, found by the closest-hit kernel
    CLS_N = 15
};
// The reference's hasAnyTex (shaders/Shaders.hlsl:232-236): texture maps the
// shading reads (alpha maps act in the traversal, metallic maps nowhere).
__host__ __device__ inline bool has_shading_textures(const pt_material &m) {
    return m.albedoTexIndex != PT_NO_TEXTURE || m.normalTexIndex != PT_NO_TEXTURE ||
           m.roughnessTexIndex != PT_NO_TEXTURE || m.specularTexIndex != PT_NO_TEXTURE ||
           m.subsurfaceTexIndex != PT_NO_TEXTURE;
}
__host__ __device__ inline int shade_class(bool hit, bool emitter, uint32_t type, bool textured = false) {
    if (!hit) return CLS_MISS;
    int c;
    if (emitter) c = CLS_EMIT;
    else switch (type) {
        case PT_MAT_MIRROR: case PT_MAT_DIELECTRIC: c = CLS_DELTA; break;
        case PT_MAT_DIFFUSE: c = CLS_DIFFUSE; break;
        case PT_MAT_MICROFACET: c = CLS_MICRO; break;
        case PT_MAT_DISNEY: c = CLS_DISNEY; break;
        default: c = CLS_HAIR;  // upload admits no other type
    }
    return textured ? c + CLS_TEX : c;
}

// Words of the per-wave counter block (WaveBuffers::counters).  The claim
// positions of the work-stealing traversal kernels sit right after the
// counts that are zeroed together with them each bounce: the shadow count
// (word 2) and the class counts (words 8 .. 8 + CLS_N).
constexpr int kCounterWords = 32;
constexpr int kCntShadow = 2, kCntStealExt = 3, kCntClass = 8, kCntStealShadow = kCntClass + CLS_N;
constexpr int kCntTailRays = 24;  // uint64: extension rays of the tail kernel
static_assert(kCntStealShadow + 1 <= kCntTailRays && kCntTailRays + 2 <= kCounterWords,
              "class queue counts and the tail's ray count must fit the counter block");

// Per-wave buffers of the wavefront integrator (structure of arrays).
struct WaveBuffers {
    size_t cap = 0;
    // path state, indexed by path slot
    float4 *thr_pdf = nullptr;  // throughput.xyz, last BSDF pdf
    float4 *lo_eta = nullptr;   // Lo.xyz, eta
    float4 *pendA = nullptr;    // pending area-light NEE contribution
    float4 *pendE = nullptr;    // pending envmap NEE contribution
    uint4 *rng = nullptr;       // dim, white-noise state, bounce, flags
    // ray queues (double buffered), indexed by queue position
    uint32_t *qslot[2] = {nullptr, nullptr};
    float4 *qo[2] = {nullptr, nullptr};  // origin, tmin
    float4 *qd[2] = {nullptr, nullptr};  // direction, tmax
    float4 *qhit = nullptr;              // t, gid bits, u, v
    uint32_t *cls = nullptr;             // CLS_N queues of ray-queue positions, cap each
    // shadow queue (two per path per bounce at most)
    uint32_t *sslot = nullptr;           // slot | kind << 31
    float4 *so = nullptr, *sd = nullptr, *sX = nullptr, *sthr = nullptr;
    // counters: [0] ray count q0, [1] ray count q1, [2] shadow count, [3]
    // k_extend claim position, [4..7] total extension / shadow rays (two
    // uint64), [8 .. 8+CLS_N) class queue counts, [8+CLS_N] k_shadow claim
    // position; kCounterWords words in all
    uint32_t *counters = nullptr;
};

// A render's launch sequence captured as a CUDA graph, with the configuration
// it was captured for (everything baked into its launches).  The sample
// offset is not baked: the kernels read it from device memory.
struct RenderGraph {
    cudaGraphExec_t exec = nullptr;
    uint32_t width = 0, height = 0, spp = 0, maxDepth = 0, rngKind = 0, envSampling = 0;
    pt_camera cam{};
    size_t cap = 0;
    const void *sum = nullptr, *comp = nullptr;
    uint64_t sceneGen = 0, waveGen = 0;
    uint32_t cached = 0, trainOn = 0;  // radiance-cache configuration baked into the launches
    uint32_t risNee = 0, flags = 0;
    uint64_t cacheGen = 0;
    uint32_t shadowCap = 0, cacheStall = 0, tailMax = 0, tailMode = 0;  // test hooks baked into the launches
    uint64_t launches = 0;
};

// Radiance cache state (pt_cache.cu): FP32 master weights, Adam moments,
// the inference average, the BF16 images the kernels copy into shared
// memory, and the per-render query / training-record buffers.
struct RadianceCache {
    bool ready = false;
    pt_cache_params params{};
    float bmin[3] = {0, 0, 0}, binv[3] = {1, 1, 1};
    bool boundsFromScene = true;
    float *w = nullptr, *m = nullptr, *v = nullptr, *ema = nullptr, *grad = nullptr;
    float *gradPart = nullptr;  // per training CTA (numSMs slots): its summed weight gradient
    uint8_t *imgTrain = nullptr, *imgInfer = nullptr;
    // counters: [0] Adam steps, [1] queries of the wave, [2] records of the
    // call, [3] loss sum (float bits), [4] records of the last step, [5]
    // queries of the call, [6] first record not yet given a target, [7] the
    // chance (float) that a path at a cache vertex trains, set after each call,
    // [8] loss of the step being trained (float), [9] / [10] first / end
    // record of the wave whose targets were set last, [11] CTAs finished in
    // the current Adam launch (reset by the last)
    uint32_t *ctr = nullptr;
    size_t queryCap = 0;
    float4 *q[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // record float4 x 4, weight
    size_t recCap = 0;       // record buffers: twice params.train_records
    bool firstCall = true;   // no cached render yet: rc_render_setup sets the training chance
    // x 4, throughput, Lo so far, target, cache value at the vertex
    float4 *rec[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    // the training inputs (x 4) and targets of the call's records in a fixed
    // order (each wave's records by path slot), and the ordering's scratch
    float4 *recOrd[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    uint32_t *ordScratch = nullptr;
    uint64_t gen = 1;  // bumped when buffers move
    float lastKernelMs = 0.0f;  // network kernel of the last batch call (CUDA events)
    float renderInferMs = 0.0f, renderTrainMs = 0.0f;  // network kernels of the last stage-timed render
};

// Batched renders (pt_render_batch): the device request table, per-slot
// request / pixel / sample, per-wave completion events, the launch graph of
// the last batch shape, staging of host films, and the autotuned launch shape.
struct BatchState {
    void *reqs = nullptr;  // PT_BATCH_MAX_REQUESTS device records
    uint2 *slotInfo = nullptr;
    size_t slotCap = 0;
    std::vector<cudaEvent_t> ev;  // one per wave
    cudaGraphExec_t exec = nullptr;
    std::vector<uint64_t> key;
    uint64_t launches = 0;
    void *films = nullptr;  // device copies of host films
    size_t filmBytes = 0;
    uint32_t tunedWave = 0;  // 0: not tuned
    float tunedGrid = 1.0f;
    uint64_t tunedSceneGen = 0;
};

struct pt_ctx {
    int device = 0;
    int numSMs = 148;
    // test hooks (pt_debug_set): shadow-queue capacity override (0 = default)
    // and the polls of the cache kernels' up-front stall (0 = off)
    uint32_t dbgShadowCap = 0, dbgCacheStall = 0, dbgTail = 0, dbgWidePlan = 0;
    cudaStream_t stream = nullptr;     // stream all work is issued on
    cudaStream_t ownStream = nullptr;  // created by pt_create, destroyed by pt_destroy
    cudaEvent_t ev[2] = {nullptr, nullptr};  // brackets each render (stats.ms_total)
    // host films: the upload runs on copyStream beside the render, and the
    // render's first film kernel waits for filmReady (recorded by pt_render
    // before every render: after the upload, or on the render stream)
    cudaStream_t copyStream = nullptr;
    cudaEvent_t filmReady = nullptr, streamMark = nullptr;
    std::string err;
    std::vector<void *> sceneAllocs;  // freed on re-upload / destroy
    pt::DevScene S{};
    bool hasScene = false;
    uint32_t clsMask = 0;  // bit c: shading class c occurs in the scene
    uint32_t numTris = 0;
    uint32_t numWide = 0;
    uint32_t *d_morton = nullptr, *d_sorted = nullptr;
    int32_t *d_binChildren = nullptr;
    uint32_t *d_sobol1 = nullptr;
    uint32_t *d_err = nullptr;  // [0] device error flags, [1] sample offset of the running render
    WaveBuffers W;
    RenderGraph graph;
    uint64_t sceneGen = 1, waveGen = 1;  // bumped when scene / wave buffers are replaced
    float sceneMin[3] = {0, 0, 0}, sceneMax[3] = {1, 1, 1};  // vertex bounds of the uploaded scene
    RadianceCache cache;
    BatchState batch;
    // scratch of the batch entry points
    void *scratch = nullptr;
    size_t scratchBytes = 0;

    int fail(int code, const char *what, const char *detail = nullptr) {
        err = what;
        if (detail) { err += ": "; err += detail; }
        return code;
    }
    template <class T>
    cudaError_t alloc_scene(T **p, size_t count) {
        cudaError_t e = cudaMalloc((void **)p, count * sizeof(T) + 16);
        if (e == cudaSuccess) sceneAllocs.push_back((void *)*p);
        return e;
    }
    void free_scene() {
        sceneGen++;
        for (void *p : sceneAllocs) cudaFree(p);
        sceneAllocs.clear();
        hasScene = false;
        S = pt::DevScene{};
        d_morton = d_sorted = nullptr;
        d_binChildren = nullptr;
    }
};

// Device scratch for host-memory batch calls: grows, never shrinks.
inline int scratch(pt_ctx *ctx, size_t bytes, char **out) {
    if (ctx->scratchBytes < bytes) {
        if (ctx->scratch) cudaFree(ctx->scratch);
        ctx->scratch = nullptr;
        ctx->scratchBytes = 0;
        cudaError_t e = cudaMalloc(&ctx->scratch, bytes);
        if (e != cudaSuccess) return ctx->fail(PT_E_NOMEM, "scratch", cudaGetErrorString(e));
        ctx->scratchBytes = bytes;
    }
    *out = (char *)ctx->scratch;
    return PT_OK;
}
inline size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

// Stage host arrays into device scratch (location == PT_MEM_HOST) or pass
// device pointers through.  `ins` are copied in; `outs` copied back by finish().
struct Staging {
    pt_ctx *ctx;
    uint32_t loc;
    struct Buf { const void *host; size_t bytes; void *dev; bool out; };
    std::vector<Buf> bufs;
    int setup() {
        if (loc == PT_MEM_DEVICE) {
            for (auto &b : bufs) b.dev = const_cast<void *>(b.host);
            return PT_OK;
        }
        size_t tot = 0;
        for (auto &b : bufs) tot += al256(b.bytes);
        char *base;
        int rc = scratch(ctx, tot + 256, &base);
        if (rc) return rc;
        for (auto &b : bufs) {
            if (!b.host) { b.dev = nullptr; continue; }
            b.dev = base;
            base += al256(b.bytes);
            if (!b.out) {
                cudaError_t e = cudaMemcpyAsync(b.dev, b.host, b.bytes, cudaMemcpyHostToDevice, ctx->stream);
                if (e != cudaSuccess) return ctx->fail(PT_E_CUDA, "staging copy", cudaGetErrorString(e));
            }
        }
        return PT_OK;
    }
    int finish() {
        if (loc == PT_MEM_HOST)
            for (auto &b : bufs)
                if (b.out && b.host) {
                    cudaError_t e = cudaMemcpyAsync(const_cast<void *>(b.host), b.dev, b.bytes, cudaMemcpyDeviceToHost,
                                                    ctx->stream);
                    if (e != cudaSuccess) return ctx->fail(PT_E_CUDA, "staging copy back", cudaGetErrorString(e));
                }
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) return ctx->fail(PT_E_CUDA, "batch kernel", cudaGetErrorString(e));
        return PT_OK;
    }
    void *add(const void *p, size_t bytes, bool out) {
        bufs.push_back({p, bytes, nullptr, out});
        return nullptr;
    }
    void *dev(size_t i) { return bufs[i].dev; }
};

// pt_bvh.cu: builds S.tri / S.nodes / S.triMesh / S.meshFirstTri and the
// parity exports on the device from the uploaded geometry.
int pt_build_bvh_device(pt_ctx *ctx, const uint32_t *d_meshFirstTri, uint32_t numTris);
// pt_render.cu
int pt_render_impl(pt_ctx *ctx, const pt_render_params *p, float *d_sum, float *d_comp, pt_stats *stats);
int pt_wave_free(pt_ctx *ctx);
// pt_cache.cu
void pt_cache_free(pt_ctx *ctx);
int pt_cache_prepare(pt_ctx *ctx, size_t queryCap);  // query buffers for a cached render
int rc_render_setup(pt_ctx *ctx, size_t waveCap, uint64_t callPaths);  // checks, bounds, query buffers
cudaError_t rc_enqueue_resolve(pt_ctx *ctx, cudaStream_t st, float4 *lo_eta);
// the wave's records: training targets, then their fixed order (keyRange: their order keys lie below it)
cudaError_t rc_enqueue_targets(pt_ctx *ctx, cudaStream_t st, float4 *lo_eta, uint4 *rng, const float4 *pendA,
                               const float4 *pendE, uint32_t keyRange);
// one training step s of kRcStepsPerCall: the network kernel (adam = false) or its Adam update (adam = true)
cudaError_t rc_enqueue_train(pt_ctx *ctx, cudaStream_t st, uint32_t s, bool adam);
constexpr uint32_t kRcStepsPerCall = 4;  // Adam steps per cached render call, on interleaved quarters of its records
void pt_graph_free(pt_ctx *ctx);
void pt_batch_free(pt_ctx *ctx);
