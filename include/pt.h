/*
 * pt.h — C ABI of libpt, the sm_100a wavefront path tracer.
 *
 * Plain C: fixed-width integers, plain pointers and sizes, no C++ or torch
 * types.  Every entry point returns 0 on success or a negative PT_E* code;
 * the message of the last failure on a context is pt_last_error(ctx).
 * Nothing throws across this boundary and no kernel traps: device-side
 * failures (queue overflow, step caps) raise a device flag that the host
 * reads after the stream synchronises and turns into PT_E_DEVICE.
 *
 * A context owns one CUDA stream and the device copy of one scene.  A
 * context is used by one host thread at a time; several contexts may live
 * side by side (also on different devices).
 *
 * Each entry point names the reference interface it replaces
 * (gracejinsotrue/PBRT-renderer-, path within that project).
 */
#ifndef PT_H
#define PT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PT_ABI_VERSION 4

/* ---- status codes ---------------------------------------------------- */
#define PT_OK 0
#define PT_E_INVALID (-1)     /* bad argument (null pointer, size, enum)   */
#define PT_E_CUDA (-2)        /* a CUDA runtime call failed                */
#define PT_E_NOMEM (-3)       /* device or host allocation failed          */
#define PT_E_NOSCENE (-4)     /* render/trace before pt_upload_scene       */
#define PT_E_DEVICE (-5)      /* a kernel raised the device error flag     */
#define PT_E_UNSUPPORTED (-6) /* feature not built into this library       */
#define PT_E_LIMIT (-7)       /* request larger than a fixed-size buffer   */

/* ---- material types: include/bsdf.h:48-57 (BSDFGPUData::Type) -------- */
#define PT_MAT_DIFFUSE 0
#define PT_MAT_MIRROR 1
#define PT_MAT_DIELECTRIC 2
#define PT_MAT_MICROFACET 3
#define PT_MAT_DISNEY 4
#define PT_MAT_HAIR 5
#define PT_MAT_SUBSURFACE 6

#define PT_NO_TEXTURE 0xFFFFFFFFu

/*
 * pt_material — one record per mesh, the GPUMaterial layout of
 * shaders/Common.hlsli:55-89 (36 x 4 bytes = 144 bytes, same field order).
 * Field aliasing follows the reference plugins: hair stores beta_m in
 * `roughness`, the cuticle tilt in degrees in `alpha` and eta in `intIOR`
 * (src/cpu/hair.cpp:389-403); subsurface stores the mean free path in
 * `subsurface`, g in `anisotropic` and its tint in sheen/sheenTint/clearcoat
 * (src/cpu/subsurface.cpp:69-90).
 * The caller fills type, colours, parameters, isEmitter/radiance and the
 * index/vertex ranges; pt_upload_scene fills surfaceArea, emitterCdfOffset
 * and emitterSelectionProb the way src/gpu/DXRApp_Scene.cpp:172-299 does.
 */
typedef struct pt_material {
    uint32_t type;
    float albedo[3];
    float intIOR;
    float extIOR;
    float alpha;
    uint32_t isEmitter;
    float radiance[3];
    uint32_t indexOffset;  /* first index of this mesh in pt_scene_desc.indices */
    uint32_t vertexOffset; /* added to this mesh's (local) indices              */
    uint32_t indexCount;   /* 3 x triangle count                               */
    uint32_t vertexCount;
    float surfaceArea;
    uint32_t emitterCdfOffset;
    uint32_t albedoTexIndex;
    uint32_t normalTexIndex;
    uint32_t roughnessTexIndex;
    uint32_t metallicTexIndex;
    uint32_t specularTexIndex;
    uint32_t subsurfaceTexIndex;
    uint32_t alphaTexIndex;
    float roughness;
    float metallic;
    float specular;
    float specularTint;
    float sheen;
    float sheenTint;
    float subsurface;
    float clearcoat;
    float clearcoatGloss;
    float anisotropic;
    float betaN;
    float emitterSelectionProb;
} pt_material;

/* GPUVolume flags: shaders/Common.hlsli:121-139 */
#define PT_VOLUME_HETEROGENEOUS 0x1u

/*
 * pt_volume — one participating medium (shaders/Common.hlsli:124-139).
 * density_grid indexes pt_scene_desc.grids (PT_NO_TEXTURE for none); the
 * 4^3-brick majorant grid of src/gpu/DXRApp_Scene.cpp:625-641 is built by
 * the library on the device.
 */
typedef struct pt_volume {
    float vmin[3];
    float vmax[3];
    float sigma_a[3];
    float sigma_s[3];
    float phase_g;
    uint32_t flags;
    uint32_t density_grid;
} pt_volume;

/* Dense float32 density grid, x fastest (src/gpu/DXRApp_Scene.cpp:531-545). */
typedef struct pt_grid {
    uint32_t w, h, d;
    const float *data;
} pt_grid;

/*
 * pt_texture — one material texture as LoadTexture loads it
 * (src/gpu/DXRApp_Textures.cpp:34-176): 8-bit RGBA, row 0 = top of the
 * image, `srgb` = 1 for colour data stored sRGB-encoded (albedo maps; decoded
 * to linear per texel before filtering), 0 for linear data (normal,
 * roughness, specular, subsurface, alpha maps).  The library builds the mip
 * chain.  pt_material's *TexIndex fields index pt_scene_desc.textures.
 */
typedef struct pt_texture {
    uint32_t width, height;
    const uint8_t *rgba8; /* 4 x width x height bytes */
    uint32_t srgb;
} pt_texture;

/*
 * pt_scene_desc — the flattened scene CreateSceneBuffers uploads
 * (src/gpu/DXRApp_Scene.cpp:172-451).  Arrays are host memory owned by the
 * caller; pt_upload_scene copies them.  `indices` are local to each mesh
 * (the mesh's vertexOffset is added), exactly like the reference buffers.
 * normals / texcoords / tangents may be NULL (zero-filled like the
 * reference).  The envmap is RGB float32, W x H, row 0 = top (theta = 0).
 */
typedef struct pt_scene_desc {
    uint32_t num_vertices;
    const float *positions; /* 3 x num_vertices */
    const float *normals;   /* 3 x num_vertices or NULL */
    const float *texcoords; /* 2 x num_vertices or NULL (already V-flipped) */
    const float *tangents;  /* 3 x num_vertices or NULL (hair strands) */
    uint32_t num_indices;
    const uint32_t *indices;
    uint32_t num_meshes;
    const pt_material *materials;
    uint32_t env_width, env_height;
    const float *env_rgb; /* 3 x W x H */
    float env_scale;
    float ev_compensation;
    uint32_t num_volumes;
    const pt_volume *volumes;
    uint32_t num_grids;
    const pt_grid *grids;
    uint32_t num_textures;
    const pt_texture *textures;
} pt_scene_desc;

/* Camera constants of shaders/Common.hlsli:31-51, built as
 * src/gpu/DXRApp_Camera.cpp:23-112 does (lower-left corner + image plane). */
typedef struct pt_camera {
    float pos[3];
    float llc[3];
    float horizontal[3];
    float vertical[3];
    float lens_radius;
    float focal_distance;
} pt_camera;

/* Sample generators of shaders/RNG.hlsli:226-274. */
#define PT_RNG_SOBOL_OWEN 0 /* USE_SOBOL=1 (the reference default) */
#define PT_RNG_PCG_HASH 1   /* USE_SOBOL=0 white-noise PCG stream  */

/* Envmap light sampling. */
#define PT_ENV_CDF 0   /* 2D CDF inversion of shaders/Envmap.hlsli:58-101 (same mapping) */
#define PT_ENV_ALIAS 1 /* Walker alias table from FP64 prefix sums (same pdf) */

typedef struct pt_render_params {
    uint32_t width, height;
    uint32_t spp;           /* samples per pixel rendered by this call            */
    uint32_t sample_offset; /* first sample index (the reference's frameCount)    */
    uint32_t max_depth;     /* MAX_BOUNCES (shaders/Common.hlsli:151-153)         */
    uint32_t rng_kind;      /* PT_RNG_*                                           */
    uint32_t env_sampling;  /* PT_ENV_*                                           */
    uint32_t wave_paths;    /* paths in flight per wave (0 = library default)    */
    uint32_t flags;         /* PT_RENDER_*                                        */
    pt_camera camera;
} pt_render_params;

/* pt_render_params.flags */
#define PT_RENDER_STAGE_TIMING 0x1u /* fill pt_stats.ms_* per stage (CUDA events per launch) */
#define PT_RENDER_RADIANCE_CACHE 0x2u /* terminate paths into the radiance cache (pt_cache_init) */
#define PT_RENDER_RIS_NEE 0x4u /* area-light NEE by resampled importance sampling: the reference's
                                  USE_RIS=1 build (RISDirectIllumination, shaders/Emitter.hlsli:155-271) */
#define PT_RENDER_MEDIA_WAVEFRONT 0x8u /* heterogeneous media in the wavefront form (deferred NEE shadow
                                          rays; ratio tracking drawn before visibility is known: the same
                                          estimator with another order of draws than the reference).
                                          Scenes whose media are all homogeneous use it always. */

/* Film: per pixel Σ(L, 1) as RGBA float32 (shaders/Shaders.hlsl:632-634)
 * plus the Kahan compensation of the same shape.  location 0 = host
 * memory (copied in and out by the call), 1 = device memory of ctx's device. */
#define PT_MEM_HOST 0
#define PT_MEM_DEVICE 1
typedef struct pt_film {
    uint32_t width, height;
    float *sum;  /* 4 x W x H */
    float *comp; /* 4 x W x H */
    uint32_t location;
} pt_film;

typedef struct pt_stats {
    uint64_t paths;
    uint64_t extension_rays;
    uint64_t shadow_rays;
    uint64_t waves;
    uint64_t bounces;  /* wavefront iterations launched (closest-hit kernel launches) */
    uint64_t launches; /* kernels this call launched */
    float ms_total;    /* device time of the render, CUDA events on the context's stream */
    /* per stage, with PT_RENDER_STAGE_TIMING (0 otherwise): */
    float ms_raygen;   /* camera rays */
    float ms_extend;   /* closest-hit traversal */
    float ms_shade;    /* surface / medium / light events */
    float ms_shadow;   /* any-hit traversal */
    float ms_film;     /* film accumulation */
    float ms_cache;    /* radiance-cache inference, training targets, training step */
    /* The last bounces of a wave, once few paths are left, run as one kernel
     * (each path to its end: closest hit, shading, NEE): its device time
     * (with PT_RENDER_STAGE_TIMING) and the extension rays it traced (part of
     * extension_rays; its shadow rays are part of shadow_rays). */
    float ms_tail;
    uint64_t tail_extension_rays;
} pt_stats;

typedef struct pt_ctx pt_ctx;

/* ---- context ------------------------------------------------------------
 * Replaces DXRApp construction + OnInit (src/gpu/DXRApp.cpp:44-79). */
int pt_create(pt_ctx **out, int device);
int pt_destroy(pt_ctx *ctx);
/* Use an existing CUDA stream (a cudaStream_t passed as void*, NULL = the
 * context's own stream) for all later work of ctx.  The caller keeps
 * ownership of the stream.  No reference counterpart (DXRApp owns its queue,
 * src/gpu/DXRApp_Device.cpp). */
int pt_set_stream(pt_ctx *ctx, void *stream);

/* Test hooks for the device error paths; no counterpart in the reference.
 * They make the library's own bounded checks fire without any fault:
 * - PT_DEBUG_SHADOW_QUEUE_CAP: shadow-ray queue capacity of later pt_render
 *   calls (0 = the default, two per path).  Below the number of NEE rays a
 *   render makes, shadow rays beyond it are dropped and the render returns
 *   PT_E_DEVICE (queue overflow); no memory beyond the queue is touched.
 * - PT_DEBUG_CACHE_STALL: radiance-cache kernels first wait `value` polls on
 *   a barrier nothing arrives at, before they issue any copy or tensor-core
 *   work, then take their error exit (TMEM freed): the call returns
 *   PT_E_DEVICE.  0 = off.
 * - PT_DEBUG_TAIL: which bounces the tail kernel takes, so that tests can
 *   compare both forms: 0 = the default rule, 1 = never (the per-bounce
 *   kernels run every render to its last bounce), 2 = whenever few paths are
 *   left at bounce 4, however few bounces remain.
 * - PT_DEBUG_WIDE_PLAN: value 1 makes later scene uploads collapse the BVH
 *   by the least-area plan, which by default only trees too large for the
 *   L2 use, so that tests can check those trees on small scenes.
 * Setting a hook back to 0 restores normal operation on the same context. */
#define PT_DEBUG_SHADOW_QUEUE_CAP 1u
#define PT_DEBUG_CACHE_STALL 2u
#define PT_DEBUG_TAIL 3u
#define PT_DEBUG_WIDE_PLAN 4u
int pt_debug_set(pt_ctx *ctx, uint32_t what, uint64_t value);
const char *pt_last_error(const pt_ctx *ctx);
int pt_abi_version(void);

/* ---- scene --------------------------------------------------------------
 * Replaces CreateAccelerationStructure + CreateSceneBuffers + SetupVolumes
 * + BuildEnvmapDistribution (src/gpu/DXRApp_Scene.cpp:37-493,
 * src/gpu/DXRApp_Textures.cpp:281-389): copies the scene, builds the LBVH
 * and its 8-wide compressed form, the emitter CDFs, the envmap CDFs and
 * alias table, and the volume majorant grids on the device. */
int pt_upload_scene(pt_ctx *ctx, const pt_scene_desc *scene);

/* ---- render ---------------------------------------------------------------
 * Replaces OnRender/DispatchRays of RayGen once per spp
 * (src/gpu/DXRApp.cpp:84-118, shaders/Shaders.hlsl:25-651): renders
 * params->spp samples per pixel starting at params->sample_offset and adds
 * them into film.  stats may be NULL. */
int pt_render(pt_ctx *ctx, const pt_render_params *params, pt_film *film, pt_stats *stats);

/* ---- batched render requests ---------------------------------------------
 * No counterpart in the reference (one DispatchRays per frame).  Renders n
 * requests of one scene — each its own image size, spp, sample offset, max
 * depth, camera and film — as one wavefront: the requests' paths are laid
 * out shortest request first and processed in waves that span requests; the
 * launch sequence is captured as a CUDA graph per batch shape and replayed.
 * rng_kind, env_sampling and flags must agree across the batch;
 * wave_paths of requests[0] (0 = the tuned or default size) sets the wave.
 * request_ms (n floats, may be NULL): device time from the batch's start to
 * the end of the wave that finished each request.  Each request's image
 * equals the same request rendered alone by pt_render. */
#define PT_BATCH_MAX_REQUESTS 256u
#define PT_BATCH_MAX_PIXELS (1u << 24) /* per request */
typedef struct pt_request {
    pt_render_params params;
    pt_film film;
} pt_request;
int pt_render_batch(pt_ctx *ctx, const pt_request *requests, uint32_t n, float *request_ms, pt_stats *stats);
/* Autotuner of the batch launch shape: times the batch (films untouched:
 * it renders into scratch films) for each candidate wave size and traversal
 * grid, keeps the fastest for later pt_render_batch calls on this scene. */
typedef struct pt_batch_tuning {
    uint32_t wave_paths;    /* chosen paths per wave */
    float traversal_grid;   /* chosen traversal / shading grid, share of full occupancy */
    float ms;               /* its batch time */
    uint32_t candidates;    /* configurations timed */
    float candidate_ms[16]; /* their times, in trial order */
    uint32_t candidate_wave[16];
    float candidate_grid[16];
} pt_batch_tuning;
int pt_batch_autotune(pt_ctx *ctx, const pt_request *requests, uint32_t n, pt_batch_tuning *out);

/* ---- parity entry points (batched, device or host arrays) ----------------
 * wi, wo: local-frame directions, 3 floats each; h: hair offset per query
 * (may be NULL = 0).  Replace MaterialEval / MaterialPdf / MaterialSample
 * (shaders/Material.hlsli:18-194), which the Nori plugins expose as
 * BSDF::eval / pdf / sample (include/bsdf.h:111-139).
 * mat_index selects per-query materials from `materials` (may be NULL =
 * material 0 for all).  For sample, `u` holds PT_SAMPLE_DIMS uniforms per
 * query consumed in the order the shader's NextFloat calls make.  All
 * pointers are host memory unless location == PT_MEM_DEVICE. */
#define PT_SAMPLE_DIMS 4
int pt_bsdf_eval_batch(pt_ctx *ctx, const pt_material *materials, uint32_t num_materials,
                       const uint32_t *mat_index, const float *wi, const float *wo,
                       const float *h, size_t n, float *f_out, float *pdf_out, uint32_t location);
/* pt_bsdf_eval_batch without any allocation and without a context; no
 * counterpart in the reference.  For callers that must not allocate device
 * memory (cudaFree synchronises the whole device, stalling a render running
 * on another stream; or all device memory was reserved up front).  Host
 * arrays are staged through one fixed 3 MiB array in the library's static
 * device memory, so with PT_MEM_HOST at most PT_NOALLOC_MAX_QUERIES queries
 * and PT_NOALLOC_MAX_MATERIALS materials per call (PT_E_LIMIT otherwise);
 * PT_MEM_DEVICE arrays are used in place and have no limit.
 * - Runs on the calling thread's current device and on `stream` (a
 *   cudaStream_t; NULL = the default stream); returns after the stream
 *   synchronises.
 * - The first call on a device looks up the array's device address (with
 *   that device current) and keeps it; make that first call before any
 *   stream capture.
 * - The array is one per device and process: calls that overlap in time on
 *   the same device (other threads or streams) race on it.  Serialise them.
 * - The kept address belongs to the device's primary context: after a
 *   cudaDeviceReset, or from a thread whose current context is not the
 *   primary one, it no longer names the array.  Callers that reset a device
 *   must not call this function on it again in the same process.
 * Errors are status codes only (no context to hold a message). */
#define PT_NOALLOC_MAX_QUERIES 65536u
#define PT_NOALLOC_MAX_MATERIALS 256u
int pt_bsdf_eval_batch_noalloc(void *stream, const pt_material *materials, uint32_t num_materials,
                               const uint32_t *mat_index, const float *wi, const float *wo,
                               const float *h, size_t n, float *f_out, float *pdf_out,
                               uint32_t location);
int pt_bsdf_sample_batch(pt_ctx *ctx, const pt_material *materials, uint32_t num_materials,
                         const uint32_t *mat_index, const float *wi, const float *u,
                         const float *h, size_t n, float *wo_out, float *weight_out,
                         float *pdf_out, uint32_t location);

/* Henyey-Greenstein eval/sample (shaders/Volume.hlsl:31-65).  wo: travel
 * direction (3 floats), u: 2 uniforms per query; outputs the sampled
 * direction and pdf. */
int pt_phase_sample_batch(pt_ctx *ctx, const float *g, const float *wo, const float *u, size_t n,
                          float *wi_out, float *pdf_out, uint32_t location);

/* Envmap sample / pdf / eval against the uploaded scene
 * (shaders/Envmap.hlsli:15-135).  u: 2 uniforms per query. */
int pt_env_sample_batch(pt_ctx *ctx, uint32_t env_sampling, const float *u, size_t n,
                        float *dir_out, float *radiance_out, float *pdf_out, uint32_t location);
int pt_env_pdf_batch(pt_ctx *ctx, uint32_t env_sampling, const float *dir, size_t n, float *pdf_out,
                     float *radiance_out, uint32_t location);
/* Device copies of the envmap marginal (H+1) and conditional (H*(W+1)) CDFs. */
int pt_env_read_cdf(pt_ctx *ctx, float *marginal, float *conditional);

/* Owen-scrambled Sobol / PCG sample generator (shaders/RNG.hlsli:184-274):
 * out[i*dims + d] = NextFloat for pixel pixel_ids[i], sample sample_ids[i],
 * dimensions 0..dims-1, frame size width x height. */
int pt_rng_batch(pt_ctx *ctx, uint32_t rng_kind, const uint32_t *pixel_ids, const uint32_t *sample_ids,
                 size_t n, uint32_t dims, uint32_t width, uint32_t height, float *out,
                 uint32_t location);

/* ---- acceleration structure (topology parity + ray queries) --------------
 * Replaces the BLAS/TLAS build (src/gpu/DXRApp_Scene.cpp:37-170) with the
 * LBVH of the uploaded scene.  morton_out: one 30-bit code per triangle in
 * global triangle order (may be NULL); sorted_prims_out: triangle ids in
 * LBVH leaf order; nodes_out: (n-1) internal nodes x 2 child links
 * (a link >= 0 is an internal node, ~link a leaf slot) of the radix tree
 * as built, before the treelet passes that shape the traversed tree.
 * Host memory. */
int pt_bvh_info(pt_ctx *ctx, uint32_t *num_triangles, uint32_t *num_wide_nodes);
int pt_bvh_read(pt_ctx *ctx, uint32_t *morton_out, uint32_t *sorted_prims_out, int32_t *nodes_out);

/* pt_hit: the HitPayload of shaders/Common.hlsli:158-166 (t, instance =
 * mesh id, primitive id local to the mesh, barycentrics). */
typedef struct pt_hit {
    float t;
    uint32_t mesh;
    uint32_t prim;
    float u, v;
    uint32_t hit;
} pt_hit;

/* rays: n x 8 floats (ox, oy, oz, tmin, dx, dy, dz, tmax).
 * Closest hit (TraceClosestInline, shaders/RayQueryTrace.hlsli:36-81) and
 * occlusion (TraceShadowInline, shaders/RayQueryTrace.hlsli:88-129;
 * occluded_out = 1 when an opaque surface blocks, transmission_out = the
 * product of (1 - Fr) over mirror/dielectric surfaces crossed, 3 floats).
 * Alpha-mapped triangles take the stochastic alpha test with the ray's index
 * in the batch as its seed. */
int pt_trace_closest(pt_ctx *ctx, const float *rays, size_t n, pt_hit *out, uint32_t location);
int pt_trace_shadow(pt_ctx *ctx, const float *rays, size_t n, uint32_t *occluded_out,
                    float *transmission_out, uint32_t location);

/* ---- radiance cache ---------------------------------------------------------
 * No counterpart in the reference (its paths run to Russian roulette).  A
 * neural radiance cache after Müller et al. 2021: a fully fused MLP of 64
 * encoded inputs, 5 hidden layers of 64 (ReLU) and 3 outputs (RGB), BF16
 * operands on the tensor cores with FP32 accumulation, trained online.
 * With PT_RENDER_RADIANCE_CACHE a render ends each path at the first surface
 * vertex reached after a rough bounce (diffuse, hair, microfacet / Disney at
 * or above rough_threshold) and adds throughput x cache(vertex).  A subset of
 * the paths reaching that vertex (about train_records per call, at most
 * max_train_fraction of them) continues past it; its
 * suffix, itself ended in the cache at its next rough bounce (self-training),
 * gives the radiance estimate the network is trained on after the render
 * (one Adam step per call on relative L2 loss).  One training path in
 * unbiased_every continues without the cache instead.
 *
 * Records (pt_cache_encode_batch): 16 floats per query — position,
 * roughness; direction toward the previous vertex, 0; shading normal, 0;
 * albedo, 0.  Features: 64 floats per query (the network's input).
 * Parameters: PT_CACHE_PARAMS floats, layer by layer, each [out][in]
 * row-major (64x64 x 5, then 16x64 of which rows 0..2 are used). */
#define PT_CACHE_PARAMS 21504u
#define PT_CACHE_FEATURES 64u
#define PT_CACHE_RECORD_FLOATS 16u
#define PT_CACHE_MAX_RECORDS 262144u
#define PT_CACHE_NO_TRAIN 0x1u /* render with the cache, take no training paths and no steps */
typedef struct pt_cache_params {
    /* training paths a render call aims at (0 = 65536; <= PT_CACHE_MAX_RECORDS).
     * The record buffers hold twice that; the training chance of a call is
     * set from the cache vertices of the call before (the first call: from
     * its path count), and each wave's records are ordered by path slot
     * before training, so a cached render sequence repeats bit for bit unless
     * a call's cache vertices more than double from the call before (records
     * past the buffers are dropped in scheduling order). */
    uint32_t train_records;
    uint32_t unbiased_every; /* one training path in this many runs without the cache (0 = none) */
    float rough_threshold;   /* microfacet alpha / Disney roughness counted as rough (0 = 0.3) */
    float learning_rate;     /* Adam step size (0 = 5e-3); beta1 0.9, beta2 0.99, eps 1e-8 */
    float ema;               /* decay of the weight average used for inference (0 = none) */
    uint32_t seed;           /* weight initialisation */
    uint32_t flags;          /* PT_CACHE_* */
    float bbox_min[3];       /* position normalisation; bbox_max <= bbox_min: the scene's bounds */
    float bbox_max[3];
    float max_train_fraction; /* at most this share of cache vertices trains (0 = 0.25) */
} pt_cache_params;
typedef struct pt_cache_stats {
    uint64_t steps;        /* Adam steps taken */
    uint32_t last_records; /* records in the last step */
    float last_loss;       /* mean relative L2 loss of the last step */
    uint64_t queries;      /* cache queries of the last render */
    float last_kernel_ms;  /* device time of the last batch call's network kernel (infer / train) */
    /* the last cached render made with PT_RENDER_STAGE_TIMING (0 otherwise):
     * device time of its inference kernels (all waves; `queries` rows) and of
     * its training kernels (forward, backward, weight gradients of every
     * step; not the launches that sum the CTAs' gradients and apply Adam),
     * and the rows those processed */
    float last_render_infer_ms;
    float last_render_train_ms;
    uint64_t last_render_train_rows;
} pt_cache_stats;
/* (Re)initialise the cache of ctx: weights from params->seed, zero moments. */
int pt_cache_init(pt_ctx *ctx, const pt_cache_params *params);
int pt_cache_release(pt_ctx *ctx);
/* Copy the FP32 parameters out (get != NULL) and/or replace them (set != NULL;
 * moments reset, the inference average restarts from the new weights). */
int pt_cache_weights(pt_ctx *ctx, float *get, const float *set);
/* Batched network entry points (parity): records -> features, features ->
 * outputs (3 per query, the inference weights), and features + targets (3
 * per query) -> the summed parameter gradient of the relative L2 loss
 * sum_c (y_c - t_c)^2 / (y_c^2 + 0.01) (denominator held constant) and the
 * loss sum, or one Adam step on it. */
int pt_cache_encode_batch(pt_ctx *ctx, const float *records, size_t n, float *features, uint32_t location);
int pt_cache_infer_batch(pt_ctx *ctx, const float *features, size_t n, float *out, uint32_t location);
int pt_cache_gradient_batch(pt_ctx *ctx, const float *features, const float *targets, size_t n,
                            float *grad_out, float *loss_out, uint32_t location);
int pt_cache_train_batch(pt_ctx *ctx, const float *features, const float *targets, size_t n, float *loss_out,
                         uint32_t location);
int pt_cache_get_stats(pt_ctx *ctx, pt_cache_stats *out);

#ifdef __cplusplus
}
#endif

#endif /* PT_H */
