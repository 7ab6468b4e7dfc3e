// pt_render.cu — the wavefront integrator of libpt (sm_100a).
//
// Restates RayGen (gracejinsotrue/PBRT-renderer-, shaders/Shaders.hlsl:25-651)
// as a sequence of kernels over waves of paths:
//
//   raygen -> [ extend -> shade -> shadow ] x max_depth -> film
//
// * extend: closest-hit BVH8 traversal of the ray queue -> hit records, and
//   each path's queue position into the queue of its shading class (miss,
//   emitter, delta, diffuse, microfacet, Disney, hair).
// * shade: one kernel per shading class present in the scene, its material
//   type fixed at compile time; one thread per path: folds the previous
//   bounce's NEE results into Lo, handles the miss / emitter / surface event,
//   samples NEE (shadow rays to the shadow queue) and the BSDF (next ray
//   queue), Russian roulette.  Path slots stay fixed; queues hold slot ids
//   and are compacted with one atomic per warp (ballot + popc).
// * shadow: any-hit traversal; writes thr * (X * transmission) or thr * 0
//   into the path's pending slot, folded in by the next shade (or by film),
//   so Lo receives the same float additions in the same order as RayGen.
// * film: per pixel, the wave's samples in sample order, Kahan-compensated
//   float32 accumulation of (L, 1).
//
// The sampler is counter-based (pixel, sample, dimension), so each path draws
// the same dimensions as RayGen.  In scenes with participating media the
// reference traces NEE shadow rays before deciding whether to draw ratio
// tracking samples (Emitter.hlsli:138-148); there shade traces its shadow
// rays inline to keep that order.
#include <algorithm>

#include "pt_internal.h"

namespace pt {

constexpr uint32_t kFlagPending = 1u;
// Shadow queue entries: path slot (< 2^30) | kShadowTrLater | NEE kind << 31.
constexpr uint32_t kShadowTrLater = 1u << 30, kShadowSlotMask = kShadowTrLater - 1u;
// radiance-cache path flags (rng.w); the record index of a training path sits above bit 8
constexpr uint32_t kFlagRough = 2u;     // the last bounce scattered off a rough surface or a medium
constexpr uint32_t kFlagTrain = 4u;     // training path
constexpr uint32_t kFlagUnbiased = 8u;  // training path whose suffix does not use the cache
constexpr uint32_t kFlagHasRec = 16u;   // its training record has been written
constexpr int kBlock = 256;

// One request of a batched render (pt_render_batch), in the device table.
struct ReqDev {
    uint64_t pathStart;  // first path id of the request in the batch's path order
    uint32_t width, height, npix, spp, sampleOffset, maxDepth;
    pt_camera cam;
    float4 *sum, *comp;  // film (device memory)
};

struct WaveArgs {
    DevScene S;
    uint32_t width, height, npix;
    uint32_t spp, spp32, spp8, fullTilePix;  // the call's samples, those in groups of 32, then of 8; pixels in full 8 x 4 tiles
    uint64_t recKeyBase;  // a training record's order key: sample x npix + position - recKeyBase (this wave)
    uint32_t recKeyRange; // keys of this wave's records lie in [0, recKeyRange)
    const uint32_t *sampleOffset;  // -> sample index of path id 0 of this render call
    uint32_t rngKind, envMode, maxDepth;
    uint64_t waveStart;      // first path id of the wave
    uint32_t waveCount;
    pt_camera cam;
    // buffers
    float4 *thr_pdf, *lo_eta, *pendA, *pendE;
    uint4 *rng;
    uint32_t *qslotIn, *qslotOut;
    float4 *qoIn, *qdIn, *qoOut, *qdOut, *qhit;
    uint32_t *sslot;
    float4 *so, *sd, *sX, *sthr;
    uint32_t *cntIn, *cntOut, *cntShadow;
    uint32_t *stealExt, *stealShadow;  // next unclaimed queue position of k_extend / k_shadow
    uint32_t bounce;                   // bounce of the kernels of this launch (uniform over the queue)
    uint32_t *cls, *cntCls;  // shading-class queues (CLS_N x clsStride) and their counts
    uint32_t clsStride;
    unsigned long long *rayTotals;  // [0] extension, [1] shadow
    unsigned long long *tailRays;   // extension rays of k_tail (also in rayTotals[0])
    uint32_t tailMax;               // k_tail takes a wave's paths when at most this many are left
    uint32_t *err;
    uint32_t shadowCap;
    // radiance cache (cacheOn == 0: plain path tracing)
    uint32_t cacheOn, trainOn, unbiasedEvery, recCap, queryCap;
    float roughThr;
    const float *trainProb;  // chance that a path reaching a cache vertex trains (device, per call)
    float4 *cq[5];      // queries: 4 record float4 + throughput weight
    uint32_t *cqCount;
    float4 *cr[7];      // training records: 4 record float4, throughput, Lo so far, target
    uint32_t *crCount;
    uint32_t risNee;  // PT_RENDER_RIS_NEE: area-light NEE by resampled importance sampling
    // batched render (batch != 0): requests and, per path slot, (pixel | request << 24, sample index)
    uint32_t batch, numReqs;
    const ReqDev *reqs;
    uint2 *slotInfo;
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Add this thread's count of rays of kind k (0 extension, 1 shadow) to the
// render's totals: one atomic per warp.
__device__ __forceinline__ void add_rays(const WaveArgs &A, int k, uint32_t c) {
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xFFFFFFFFu, c, o);
    if (lane_id() == 0 && c) atomicAdd(&A.rayTotals[k], (unsigned long long)c);
}

// Warp-aggregated append: returns this lane's slot in the queue.
__device__ __forceinline__ uint32_t warp_append(uint32_t *counter, bool pred) {
    uint32_t active = __activemask();
    uint32_t mask = __ballot_sync(active, pred);
    if (!pred) return 0xFFFFFFFFu;
    uint32_t leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane_id() == leader) base = atomicAdd(counter, __popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + __popc(mask & ((1u << lane_id()) - 1u));
}

// Pixel of position p of the path order.  Positions run over 8 x 4 pixel
// tiles (one warp's paths cover one tile: compact bundles of camera rays),
// tiles row by row; pixels right of the last full tile column or below the
// last full tile row follow in row-major order.  A bijection on [0, W*H).
__device__ __forceinline__ uint32_t tile_pixel_wh(uint32_t W, uint32_t H, uint32_t p) {
    const uint32_t Wt = W / 8u, Ht = H / 4u;
    const uint32_t full = 32u * Wt * Ht;
    if (p < full) {
        uint32_t t = p >> 5, w = p & 31u;
        return ((t / Wt) * 4u + (w >> 3)) * W + (t % Wt) * 8u + (w & 7u);
    }
    uint32_t q = p - full, rw = W - 8u * Wt;
    if (q < 4u * Ht * rw) return (q / rw) * W + 8u * Wt + q % rw;
    q -= 4u * Ht * rw;
    return (4u * Ht + q / W) * W + q % W;
}
__device__ __forceinline__ uint32_t tile_pixel(const WaveArgs &A, uint32_t p) {
    return tile_pixel_wh(A.width, A.height, p);
}
// Request of batch path id pid: the last request whose first path id <= pid.
__device__ __forceinline__ uint32_t find_request(const WaveArgs &A, uint64_t pid) {
    uint32_t lo = 0, hi = A.numReqs;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (A.reqs[mid].pathStart <= pid) lo = mid;
        else hi = mid;
    }
    return lo;
}
// Path order of a render call (path id -> pixel position of tile_pixel,
// sample of the call).  The call's samples go in groups, so that a warp's
// 32 paths are camera rays of few pixels: first as many groups of 32 as
// fit (a warp = 32 samples of one pixel; consecutive warps follow the pixel
// positions), then groups of 8 (within a group, each 8 x 4 tile's eight
// 2 x 2 pixel blocks in turn, a block's 32 paths being its 4 pixels x the 8
// samples; positions outside the full tiles take the group's samples one
// after the other), and the remaining samples one after the other over the
// pixel positions.  A bijection; path_id is its inverse (the film sums each
// pixel's samples in sample order through it).  Measured on the 64-sphere
// frame (Mpaths/s): one sample at a time 1849, groups of 8 1958, groups of
// 32 2040; the 10 M-triangle scene at 16 spp per call: 466 -> 489 with 8.
__host__ __device__ inline void path_pos_sample(const WaveArgs &A, uint64_t pid, uint32_t &p, uint32_t &s) {
    const uint32_t npix = A.npix;
    const uint64_t g32 = (uint64_t)A.spp32 * npix;
    if (pid < g32) {
        const uint64_t gsz = 32ull * npix;
        const uint32_t c = (uint32_t)(pid / gsz), r = (uint32_t)(pid % gsz);
        p = r >> 5;
        s = 32u * c + (r & 31u);
        return;
    }
    pid -= g32;
    const uint64_t g8 = (uint64_t)A.spp8 * npix;
    if (pid < g8) {
        const uint64_t gsz = 8ull * npix;
        const uint32_t c = (uint32_t)(pid / gsz), r = (uint32_t)(pid % gsz), full = A.fullTilePix;
        if (r < 8u * full) {
            const uint32_t t = r >> 8, q = r & 255u, b = q >> 5, u = q & 31u, i = u & 3u;
            p = 32u * t + ((2u * (b >> 2) + (i >> 1)) << 3) + 2u * (b & 3u) + (i & 1u);
            s = A.spp32 + 8u * c + (u >> 2);
        } else {
            const uint32_t r2 = r - 8u * full, rem = npix - full;
            p = full + r2 % rem;
            s = A.spp32 + 8u * c + r2 / rem;
        }
        return;
    }
    const uint64_t q = pid - g8;
    p = (uint32_t)(q % npix);
    s = A.spp32 + A.spp8 + (uint32_t)(q / npix);
}
__device__ __forceinline__ uint64_t path_id(const WaveArgs &A, uint32_t p, uint32_t s) {
    const uint32_t npix = A.npix;
    if (s < A.spp32) return (uint64_t)(s >> 5) * 32u * npix + 32ull * p + (s & 31u);
    const uint64_t base = (uint64_t)A.spp32 * npix;
    const uint32_t s2 = s - A.spp32;
    if (s2 < A.spp8) {
        const uint64_t gbase = base + (uint64_t)(s2 >> 3) * 8u * npix;
        const uint32_t si = s2 & 7u, full = A.fullTilePix;
        if (p < full) {
            const uint32_t t = p >> 5, w = p & 31u, row = w >> 3, col = w & 7u;
            return gbase + 256ull * t + 32u * ((row >> 1) * 4u + (col >> 1)) + 4u * si + (row & 1u) * 2u + (col & 1u);
        }
        return gbase + 8ull * full + (uint64_t)si * (npix - full) + (p - full);
    }
    return base + (uint64_t)A.spp8 * npix + (uint64_t)(s2 - A.spp8) * npix + p;
}
// The first and last sample of sample s's group.
__host__ __device__ inline void path_group(const WaveArgs &A, uint32_t s, uint32_t &lo, uint32_t &hi) {
    if (s < A.spp32) {
        lo = s & ~31u;
        hi = s | 31u;
    } else if (s - A.spp32 < A.spp8) {
        lo = A.spp32 + ((s - A.spp32) & ~7u);
        hi = A.spp32 + ((s - A.spp32) | 7u);
    } else {
        lo = hi = s;
    }
}
__device__ __forceinline__ void path_coords(const WaveArgs &A, uint32_t slot, uint32_t &pix, uint32_t &frame) {
    if (A.batch) {
        uint2 si = A.slotInfo[slot];
        pix = si.x & 0xFFFFFFu;
        frame = si.y;
        return;
    }
    uint32_t p, s;
    path_pos_sample(A, A.waveStart + slot, p, s);
    pix = tile_pixel(A, p);
    frame = __ldg(A.sampleOffset) + s;
}
// Per-request image size and depth of a path (the render's own without a batch).
__device__ __forceinline__ uint32_t path_depth(const WaveArgs &A, uint32_t slot) {
    return A.batch ? A.reqs[A.slotInfo[slot].x >> 24].maxDepth : A.maxDepth;
}
__device__ __forceinline__ uint2 path_image(const WaveArgs &A, uint32_t slot) {
    if (!A.batch) return make_uint2(A.width, A.height);
    const ReqDev &q = A.reqs[A.slotInfo[slot].x >> 24];
    return make_uint2(q.width, q.height);
}
__device__ __forceinline__ Rng load_rng(const WaveArgs &A, uint32_t slot, uint4 st) {
    uint32_t pix, frame;
    path_coords(A, slot, pix, frame);
    Rng r;
    r.pixelSeed = pcg_hash(pix ^ 0x9e3779b9u);
    r.sampleIndex = frame;
    r.dim = st.x;
    r.white = st.y;
    r.kind = A.rngKind;
    return r;
}

// ---- raygen: camera rays (Shaders.hlsl:55-92) ------------------------------
__global__ void k_raygen(WaveArgs A) {
    uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= A.waveCount) return;
    uint32_t pix, frame, W = A.width, H = A.height, npix = A.npix;
    const pt_camera *cp = &A.cam;
    if (A.batch) {  // the path's request, pixel and sample; kept per slot for the later kernels
        uint64_t pid = A.waveStart + slot;
        uint32_t q = find_request(A, pid);
        const ReqDev &R = A.reqs[q];
        W = R.width; H = R.height; npix = R.npix;
        uint64_t local = pid - R.pathStart;
        pix = tile_pixel_wh(W, H, (uint32_t)(local % npix));
        frame = R.sampleOffset + (uint32_t)(local / npix);
        A.slotInfo[slot] = make_uint2(pix | (q << 24), frame);
        cp = &R.cam;
    } else {
        path_coords(A, slot, pix, frame);
    }
    uint32_t px = pix % W, py = pix / W;
    Rng r = rng_init(pix, npix, frame, A.rngKind);
    float jx = next_float(r, A.S.sobol1), jy = next_float(r, A.S.sobol1);
    float ux = ((float)px + jx) / (float)W;
    float uy = 1.0f - ((float)py + jy) / (float)H;
    const pt_camera &c = *cp;
    float3 cpos = make_float3(c.pos[0], c.pos[1], c.pos[2]);
    float3 llc = make_float3(c.llc[0], c.llc[1], c.llc[2]);
    float3 hor = make_float3(c.horizontal[0], c.horizontal[1], c.horizontal[2]);
    float3 ver = make_float3(c.vertical[0], c.vertical[1], c.vertical[2]);
    float3 dir = normalize(llc + ux * hor + uy * ver - cpos);
    float3 ro = cpos, rd = dir;
    if (c.lens_radius > 0.0f) {
        float3 fwd = normalize(llc + 0.5f * hor + 0.5f * ver - cpos);
        float3 right = normalize(hor), up = normalize(ver);
        float ft = c.focal_distance / dot(dir, fwd);
        float3 fp = cpos + dir * ft;
        float u1 = next_float(r, A.S.sobol1), u2 = next_float(r, A.S.sobol1);
        float rr = sqrtf(u1) * c.lens_radius;
        float th = 2.0f * kPi * u2;
        ro = cpos + (rr * cosf(th)) * right + (rr * sinf(th)) * up;
        rd = normalize(fp - ro);
    }
    // the first ray queue is in slot order (its slot index is the position:
    // the kernels of bounce 0 do not read it)
    A.qoOut[slot] = make_float4(ro.x, ro.y, ro.z, 0.001f);
    A.qdOut[slot] = make_float4(rd.x, rd.y, rd.z, 1e20f);
    // the first shading pass starts every path from throughput 1 and Lo 0
    // without loading them; they are stored only where something reads them
    // first: the film (no bounce) and the medium free flights of k_extend
    if (A.S.mediaWavefront || path_depth(A, slot) == 0) {
        A.thr_pdf[slot] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        A.lo_eta[slot] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    }
    A.rng[slot] = make_uint4(r.dim, r.white, 0u, 0u);
    if (slot == 0) *A.cntOut = A.waveCount;
}

// Append queue position i to the queue of class c: lanes with the same class
// share one atomic (match_any + popc).
__device__ __forceinline__ void class_append(const WaveArgs &A, int c, uint32_t i) {
    uint32_t peers = __match_any_sync(__activemask(), c);
    uint32_t leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane_id() == leader) base = atomicAdd(A.cntCls + c, __popc(peers));
    base = __shfl_sync(peers, base, leader);
    __stcs(A.cls + (size_t)c * A.clsStride + base + __popc(peers & ((1u << lane_id()) - 1u)), i);
}

// ---- extend: closest hit (+ sort into shading classes) -----------------------
template <bool CLASSIFY>
__device__ __forceinline__ void finish_extend(const WaveArgs &A, uint32_t i, const Hit &h) {
    __stcs(A.qhit + i, make_float4(h.t, __uint_as_float(h.gid), h.u, h.v));
    if (CLASSIFY) {
        int c = h.gid == 0xFFFFFFFFu ? (int)CLS_MISS : (int)__ldg(A.S.meshClass + __ldg(A.S.triMesh + h.gid));
        class_append(A, c, i);
    }
}
// Traversal stacks of k_extend / k_shadow: the first kSharedStack entries of
// each thread in shared memory (kSharedStack x kBlock x 8 bytes per block),
// deeper entries in local memory.
#ifndef PT_SHARED_STACK
#define PT_SHARED_STACK 0
#endif
constexpr int kSharedStack = PT_SHARED_STACK;
template <int SH>
struct QueueStack {
    using type = SplitStack<SH, kBlock>;
};
template <>
struct QueueStack<0> {
    using type = TravStack;
};
template <int SH, int STRIDE>
__device__ __forceinline__ void bind_stack(SplitStack<SH, STRIDE> &K, uint2 *col) {
    K.col = col;
}
__device__ __forceinline__ void bind_stack(TravStack &, uint2 *) {}
#define PT_QUEUE_STACK(K)                                                \
    __shared__ uint2 stk_[kSharedStack > 0 ? kSharedStack : 1][kBlock]; \
    QueueStack<kSharedStack>::type K;                                    \
    bind_stack(K, &stk_[0][threadIdx.x]);

// Traversal kernels run 4 blocks of 256 threads per SM (64 registers).  The
// opaque-scene forms fit that by themselves (and are left to the compiler:
// the same bound stated explicitly schedules them worse); the media forms
// (free flight after the closest hit, ratio tracking on shadow rays) would
// take 80 registers and 3 blocks, so their entry points state the bound —
// their traversal waits on DRAM in large scenes and wants the warps more than
// those registers.
constexpr int kTraversalBlocksPerSm = 4;


// Persistent work-stealing over a ray queue: each warp claims the next 32
// queue positions with one atomic (so a warp's rays stay neighbours in the
// queue) until the queue is exhausted.  Returns the claimed base, uniform
// across the warp; all 32 lanes must call it together.
__device__ __forceinline__ uint32_t claim32(uint32_t *next) {
    uint32_t base = 0;
    if (lane_id() == 0) base = atomicAdd(next, 32u);
    return __shfl_sync(0xFFFFFFFFu, base, 0);
}

// MEDIA: the free flight of Shaders.hlsl:133-179 follows the closest hit here
// (draws from the path's stream in the shader's order); a scattering event
// goes to the medium class with (t, volume | 1 << 31) in the hit record and
// the throughput gets the flight's weight.  Homogeneous media only: their
// shadow-ray transmittance draws nothing, so NEE can be deferred.
template <bool CLASSIFY, bool MEDIA, class Stack>
__device__ __forceinline__ void extend_one(const WaveArgs &A, uint32_t i, Stack &K) {
    // queue data streams through once: evict-first loads and stores keep
    // the BVH nodes and triangles resident in L2
    float4 o = __ldcs(A.qoIn + i), d = __ldcs(A.qdIn + i);
    uint32_t aseed = 0, akey = 0;
    if (A.S.hasAlpha) {  // alpha tests: the path's seed, key of this bounce's extension ray
        uint32_t slot = A.bounce == 0u ? i : A.qslotIn[i];
        Rng r = load_rng(A, slot, A.rng[slot]);
        aseed = alpha_seed(r.pixelSeed, r.sampleIndex);
        akey = alpha_key(A.rng[slot].z, 0u);
    }
    Hit h = trace_closest_on(K, A.S, make_float3(o.x, o.y, o.z), make_float3(d.x, d.y, d.z), o.w, d.w, A.err, aseed,
                             akey);
    if (MEDIA) {
        const uint32_t slot = A.bounce == 0u ? i : A.qslotIn[i];
        uint4 st = A.rng[slot];
        Rng r = load_rng(A, slot, st);
        float3 vw = v3(1.0f);
        float tsc;
        uint32_t svi;
        bool sc = sample_free_flight(A.S, make_float3(o.x, o.y, o.z), make_float3(d.x, d.y, d.z),
                                     h.gid != 0xFFFFFFFFu ? h.t : 1e20f, r, vw, tsc, svi);
        if (r.dim != st.x || r.white != st.y) {
            st.x = r.dim;
            st.y = r.white;
            A.rng[slot] = st;
        }
        if (vw.x != 1.0f || vw.y != 1.0f || vw.z != 1.0f) {
            float4 tp = A.thr_pdf[slot];
            float3 t3 = make_float3(tp.x, tp.y, tp.z) * vw;
            A.thr_pdf[slot] = make_float4(t3.x, t3.y, t3.z, tp.w);
        }
        if (sc) {
            A.qhit[i] = make_float4(tsc, __uint_as_float(svi | 0x80000000u), 0.0f, 0.0f);
            class_append(A, CLS_MEDIUM, i);
            return;
        }
    }
    finish_extend<CLASSIFY>(A, i, h);
}
template <bool CLASSIFY, bool MEDIA>
__device__ __forceinline__ void extend_queue(const WaveArgs &A) {
    // warps claim the queue in order: the 32 rays of a warp are neighbours in
    // the queue (coherent traversal), and the class queues and the next ray
    // queue keep that order for the kernels that follow
    const uint32_t n = *(volatile uint32_t *)A.cntIn;
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&A.rayTotals[0], (unsigned long long)n);
    PT_QUEUE_STACK(K)
    for (uint32_t base; (base = claim32(A.stealExt)) < n;) {
        const uint32_t i = base + lane_id();
        if (i < n) extend_one<CLASSIFY, MEDIA>(A, i, K);
    }
}
template <bool CLASSIFY>
__global__ void __launch_bounds__(kBlock) k_extend(WaveArgs A) {
    extend_queue<CLASSIFY, false>(A);
}
__global__ void __launch_bounds__(kBlock, kTraversalBlocksPerSm) k_extend_media(WaveArgs A) {
    extend_queue<true, true>(A);
}

// ---- shadow: any hit -> pending NEE contribution ---------------------------
// Shadow queue entry: path slot | kShadowTrLater | kind (0 area, 1 envmap) << 31.
template <bool MEDIA_TR, class Stack>
__device__ __forceinline__ void shadow_one(const WaveArgs &A, uint32_t i, Stack &K) {
    float4 o = __ldcs(A.so + i), d = __ldcs(A.sd + i);
    float3 tr;
    uint32_t aseed = 0, akey = 0;
    if (A.S.hasAlpha) {  // the shading kernel already advanced the path's bounce counter
        uint32_t s = A.sslot[i], slot = s & kShadowSlotMask;
        Rng r = load_rng(A, slot, A.rng[slot]);
        aseed = alpha_seed(r.pixelSeed, r.sampleIndex);
        akey = alpha_key(A.rng[slot].z - 1u, (s >> 31) ? 2u : 1u);
    }
    bool occ = trace_shadow_on(K, A.S, make_float3(o.x, o.y, o.z), make_float3(d.x, d.y, d.z), o.w, d.w, tr, A.err,
                               aseed, akey);
    float4 X = __ldcs(A.sX + i), Th = __ldcs(A.sthr + i);
    uint32_t s = __ldcs(A.sslot + i);
    const uint32_t slot = s & kShadowSlotMask;
    if (MEDIA_TR && !occ && (s & kShadowTrLater)) {
        // the ray's medium transmittance (ratio tracking, Volume.hlsl:326-372),
        // estimated only now that the ray is known to be unoccluded: its own
        // white-noise stream, keyed by pixel, sample, bounce and NEE kind.  The
        // shading kernel integrated to the light (area: tmax + 0.001)
        Rng r = load_rng(A, slot, A.rng[slot]);
        Rng t;
        t.kind = PT_RNG_PCG_HASH;
        t.pixelSeed = r.pixelSeed;
        t.sampleIndex = r.sampleIndex;
        t.dim = 0u;
        t.white = pcg_hash(r.pixelSeed ^ pcg_hash(r.sampleIndex ^ pcg_hash(((A.rng[slot].z - 1u) << 1) + (s >> 31) +
                                                                          0x3C6EF372u)));
        const float tm = d.w < 1e19f ? d.w + 0.001f : d.w;
        tr = tr * multi_volume_tr(A.S, make_float3(o.x, o.y, o.z), make_float3(d.x, d.y, d.z), tm, t);
    }
    float3 thr = make_float3(Th.x, Th.y, Th.z);
    float3 R = occ ? thr * v3(0.0f) : thr * (make_float3(X.x, X.y, X.z) * tr);
    float4 out = make_float4(R.x, R.y, R.z, 0.0f);
    if (s >> 31) __stcs(A.pendE + slot, out);
    else __stcs(A.pendA + slot, out);
}
// MEDIA_TR: the form for heterogeneous media in the wavefront
// (transmittance of unoccluded rays, k_shadow_media); k_shadow carries none
// of that code.
template <bool MEDIA_TR>
__device__ __forceinline__ void shadow_queue(const WaveArgs &A) {
    // appends past the capacity were dropped (and flagged): only what was stored is read
    const uint32_t n = min(*(volatile uint32_t *)A.cntShadow, A.shadowCap);
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&A.rayTotals[1], (unsigned long long)n);
    PT_QUEUE_STACK(K)
    for (uint32_t base; (base = claim32(A.stealShadow)) < n;) {
        const uint32_t i = base + lane_id();
        if (i < n) shadow_one<MEDIA_TR>(A, i, K);
    }
}
__global__ void __launch_bounds__(kBlock) k_shadow(WaveArgs A) { shadow_queue<false>(A); }
__global__ void __launch_bounds__(kBlock, kTraversalBlocksPerSm) k_shadow_media(WaveArgs A) {
    shadow_queue<true>(A);
}

// One NEE estimate, deferred: either a shadow ray carrying X (everything but
// visibility/transmission) or, when the estimate is zero before any trace,
// the final thr * 0 written straight to the pending slot.
struct NeeOut {
    bool ray;
    bool traced;   // the inline form traced its shadow ray (ray counts)
    bool trLater;  // medium transmittance left to the shadow kernel (not in X)
    float3 o, d, X;
    float tmin, tmax;
};

// MISDirectIllumination (Emitter.hlsli:105-153) up to the shadow trace.
template <bool INLINE, bool MEDIA = false>
__device__ __forceinline__ float3 nee_area(const WaveArgs &A, float3 hp, float3 N, float3 Ng, float3 T, float3 B,
                                           float3 wil, uint32_t type, const pt_material &m, float h, Rng &rng,
                                           NeeOut &out, uint32_t aseed, uint32_t bounce) {
    const DevScene &S = A.S;
    out.ray = false;
    out.trLater = false;
    EmitterSample es = sample_emitter(S, rng);
    if (!es.valid) return v3(0.0f);
    float3 tl = es.pos - hp;
    float dist = len(tl);
    float3 ww = tl / v3(dist);
    float ct = dot(N, ww), cl = dot(es.nrm, -ww);
    bool hair = type == PT_MAT_HAIR;
    if ((!hair && ct <= 0.0f) || cl <= 0.0f) return v3(0.0f);
    float act = hair ? fabsf(ct) : ct;
    float3 sng = hair ? (dot(ww, Ng) >= 0.0f ? Ng : -Ng) : Ng;
    float3 so = offset_origin(hp, sng, sng);
    float3 trans = v3(1.0f);
    if (INLINE) {
        out.traced = true;
        if (trace_shadow(S, so, ww, 0.0f, dist - 0.001f, trans, A.err, aseed, alpha_key(bounce, 1u))) return v3(0.0f);
    }
    float3 f;
    float pb;
    material_eval_pdf_t(type, wil, to_local(ww, T, B, N), m, h, f, pb);
    float pe = es.pdfArea * dist * dist / cl;
    float w = balance(pe, pb);
    out.trLater = !INLINE && MEDIA && S.mediaTrDeferred;
    float3 vt = (INLINE || (MEDIA && S.mediaWavefront && !out.trLater)) ? multi_volume_tr(S, so, ww, dist, rng) : v3(1.0f);
    float3 X = es.rad * f * act / v3(mx(pe, 1e-20f)) * w * vt;
    if (INLINE) return X * trans;
    out.ray = true;
    out.o = so; out.d = ww; out.tmin = 0.0f; out.tmax = dist - 0.001f; out.X = X;
    return v3(0.0f);
}
// EvalLightCandidate (Emitter.hlsli:166-199): unshadowed integrand, scalar
// target pHat = lum(f Le cos) and the solid-angle pdf of the emitter sample.
__device__ __forceinline__ bool ris_candidate(const EmitterSample &es, float3 hp, float3 N, float3 T, float3 B,
                                              float3 wil, uint32_t type, const pt_material &m, float h, float3 &wiw,
                                              float &dist, float3 &integ, float &pHat, float &pSA) {
    integ = v3(0.0f);
    pHat = 0.0f;
    pSA = 0.0f;
    float3 tl = es.pos - hp;
    dist = len(tl);
    if (dist < 1e-6f) {
        wiw = make_float3(0.0f, 0.0f, 1.0f);
        return false;
    }
    wiw = tl / v3(dist);
    float cs = dot(N, wiw), cl = dot(es.nrm, -wiw);
    bool hair = type == PT_MAT_HAIR;
    if ((!hair && cs <= 0.0f) || cl <= 1e-8f) return false;
    float ac = hair ? fabsf(cs) : cs;
    float3 f;
    float pb;
    material_eval_pdf_t(type, wil, to_local(wiw, T, B, N), m, h, f, pb);
    integ = f * es.rad * ac;
    pHat = dot(integ, make_float3(0.2126f, 0.7152f, 0.0722f));
    pSA = es.pdfArea * dist * dist / cl;
    return pHat > 0.0f && pSA > 0.0f;
}
// RISDirectIllumination (Emitter.hlsli:201-271) up to the shadow trace: 8
// candidates through a one-sample reservoir, the survivor re-evaluated and
// MIS-weighted against the BSDF with its solid-angle pdf (the same pdf the
// emitter-hit MIS weight uses).
template <bool INLINE, bool MEDIA = false>
__device__ __forceinline__ float3 nee_ris(const WaveArgs &A, float3 hp, float3 N, float3 Ng, float3 T, float3 B,
                                          float3 wil, uint32_t type, const pt_material &m, float h, Rng &rng,
                                          NeeOut &out, uint32_t aseed, uint32_t bounce) {
    const DevScene &S = A.S;
    out.ray = false;
    out.trLater = false;
    EmitterSample y;
    y.valid = false;
    float wSum = 0.0f, pHatY = 0.0f;
    for (int i = 0; i < 8; i++) {
        EmitterSample c = sample_emitter(S, rng);
        if (!c.valid) continue;
        float3 wiwC, integC;
        float distC, pHatC, pSAC;
        if (!ris_candidate(c, hp, N, T, B, wil, type, m, h, wiwC, distC, integC, pHatC, pSAC)) continue;
        float w = pHatC / pSAC;
        wSum += w;
        if (next_float(rng, S.sobol1) < w / mx(wSum, 1e-20f)) {
            y = c;
            pHatY = pHatC;
        }
    }
    if (!y.valid || pHatY <= 0.0f) return v3(0.0f);
    float W = (wSum / 8.0f) / pHatY;
    float3 wiw, integ;
    float dist, pHat, pSA;
    if (!ris_candidate(y, hp, N, T, B, wil, type, m, h, wiw, dist, integ, pHat, pSA)) return v3(0.0f);
    bool hair = type == PT_MAT_HAIR;
    float3 sng = hair ? (dot(wiw, Ng) >= 0.0f ? Ng : -Ng) : Ng;
    float3 so = offset_origin(hp, sng, sng);
    float3 trans = v3(1.0f);
    if (INLINE) {
        out.traced = true;
        if (trace_shadow(S, so, wiw, 0.0f, dist - 0.001f, trans, A.err, aseed, alpha_key(bounce, 1u))) return v3(0.0f);
    }
    float3 fu;
    float pdfBsdf;
    material_eval_pdf_t(type, wil, to_local(wiw, T, B, N), m, h, fu, pdfBsdf);
    float wMis = balance(pSA, pdfBsdf);
    out.trLater = !INLINE && MEDIA && S.mediaTrDeferred;
    float3 vt = (INLINE || (MEDIA && S.mediaWavefront && !out.trLater)) ? multi_volume_tr(S, so, wiw, dist, rng) : v3(1.0f);
    float3 X = integ * v3(W) * v3(wMis) * vt;
    if (INLINE) return X * trans;
    out.ray = true;
    out.o = so; out.d = wiw; out.tmin = 0.0f; out.tmax = dist - 0.001f; out.X = X;
    return v3(0.0f);
}
// EnvmapDirectIllumination (Emitter.hlsli:275-326) up to the shadow trace.
template <bool INLINE, bool MEDIA = false>
__device__ __forceinline__ float3 nee_env(const WaveArgs &A, float3 hp, float3 N, float3 Ng, float3 T, float3 B,
                                          float3 wil, uint32_t type, const pt_material &m, float h, Rng &rng,
                                          NeeOut &out, uint32_t aseed, uint32_t bounce) {
    const DevScene &S = A.S;
    out.ray = false;
    out.trLater = false;
    float u1 = next_float(rng, S.sobol1), u2 = next_float(rng, S.sobol1);
    float3 ww, Le;
    float pe;
    env_sample(S, A.envMode, u1, u2, ww, Le, pe);
    if (pe <= 0.0f) return v3(0.0f);
    float ct = dot(N, ww);
    bool hair = type == PT_MAT_HAIR;
    if (!hair && ct <= 0.0f) return v3(0.0f);
    float act = hair ? fabsf(ct) : ct;
    float3 sng = hair ? (dot(ww, Ng) >= 0.0f ? Ng : -Ng) : Ng;
    float3 so = offset_origin(hp, sng, sng);
    float3 trans = v3(1.0f);
    if (INLINE) {
        out.traced = true;
        if (trace_shadow(S, so, ww, 0.0f, 1e20f, trans, A.err, aseed, alpha_key(bounce, 2u))) return v3(0.0f);
    }
    float3 f;
    float pb;
    material_eval_pdf_t(type, wil, to_local(ww, T, B, N), m, h, f, pb);
    float w = balance(pe, pb);
    out.trLater = !INLINE && MEDIA && S.mediaTrDeferred;
    float3 vt = (INLINE || (MEDIA && S.mediaWavefront && !out.trLater)) ? multi_volume_tr(S, so, ww, 1e20f, rng) : v3(1.0f);
    float3 X = Le * f * act / v3(mx(pe, 1e-20f)) * w * vt;
    if (INLINE) return X * trans;
    out.ray = true;
    out.o = so; out.d = ww; out.tmin = 0.0f; out.tmax = 1e20f; out.X = X;
    return v3(0.0f);
}
// Volume NEE (Emitter.hlsli:334-434), always traced inline.
__device__ bool vol_nee_skip(const pt_volume &v, float3 p) {
    float3 st = vsigma_t(v);
    float smin = mn(st.x, mn(st.y, st.z));
    float3 dmn = p - make_float3(v.vmin[0], v.vmin[1], v.vmin[2]);
    float3 dmx = make_float3(v.vmax[0], v.vmax[1], v.vmax[2]) - p;
    float md = mn(mn(dmn.x, dmn.y), mn(dmn.z, mn(dmx.x, mn(dmx.y, dmx.z))));
    return md * smin > 8.0f;
}
// Volume NEE (Emitter.hlsli:334-434): traced inline (INLINE), or up to the
// shadow trace with the trace deferred (homogeneous media in the wavefront,
// whose transmittance along the shadow ray draws nothing).
template <bool INLINE>
__device__ float3 vol_nee_area(const WaveArgs &A, float3 sp, float3 wo, uint32_t vi, Rng &rng, uint32_t aseed,
                               uint32_t bounce, NeeOut &out) {
    const DevScene &S = A.S;
    out.ray = false;
    out.trLater = false;
    const pt_volume &v = S.vols[vi];
    if (vol_nee_skip(v, sp)) return v3(0.0f);
    EmitterSample es = sample_emitter(S, rng);
    if (!es.valid) return v3(0.0f);
    float3 tl = es.pos - sp;
    float dist = len(tl);
    float3 wi = tl / v3(dist);
    float cl = dot(es.nrm, -wi);
    if (cl <= 0.0f) return v3(0.0f);
    float3 trans = v3(1.0f);
    if (INLINE) out.traced = true;
    if (INLINE && trace_shadow(S, sp, wi, 0.001f, dist - 0.001f, trans, A.err, aseed, alpha_key(bounce, 1u)))
        return v3(0.0f);
    float fp = hg(dot(wo, wi), v.phase_g);
    float pe = es.pdfArea * dist * dist / cl;
    float w = balance(pe, fp);
    out.trLater = !INLINE && S.mediaTrDeferred;
    float3 vt = out.trLater ? v3(1.0f) : multi_volume_tr(S, sp, wi, dist, rng);
    float3 X = es.rad * fp / v3(mx(pe, 1e-20f)) * w * vt;
    if (INLINE) return X * trans;
    out.ray = true;
    out.o = sp; out.d = wi; out.tmin = 0.001f; out.tmax = dist - 0.001f; out.X = X;
    return v3(0.0f);
}
template <bool INLINE>
__device__ float3 vol_nee_env(const WaveArgs &A, float3 sp, float3 wo, uint32_t vi, Rng &rng, uint32_t aseed,
                              uint32_t bounce, NeeOut &out) {
    const DevScene &S = A.S;
    out.ray = false;
    out.trLater = false;
    const pt_volume &v = S.vols[vi];
    if (vol_nee_skip(v, sp)) return v3(0.0f);
    float u1 = next_float(rng, S.sobol1), u2 = next_float(rng, S.sobol1);
    float3 wi, Le;
    float pe;
    env_sample(S, A.envMode, u1, u2, wi, Le, pe);
    if (pe <= 0.0f) return v3(0.0f);
    float3 trans = v3(1.0f);
    if (INLINE) out.traced = true;
    if (INLINE && trace_shadow(S, sp, wi, 0.001f, 1e20f, trans, A.err, aseed, alpha_key(bounce, 2u)))
        return v3(0.0f);
    float fp = hg(dot(wo, wi), v.phase_g);
    float w = balance(pe, fp);
    out.trLater = !INLINE && S.mediaTrDeferred;
    float3 vt = out.trLater ? v3(1.0f) : multi_volume_tr(S, sp, wi, 1e20f, rng);
    float3 X = Le * fp / v3(mx(pe, 1e-20f)) * w * vt;
    if (INLINE) return X * trans;
    out.ray = true;
    out.o = sp; out.d = wi; out.tmin = 0.001f; out.tmax = 1e20f; out.X = X;
    return v3(0.0f);
}

__device__ __forceinline__ void push_shadow(const WaveArgs &A, bool pred, uint32_t slot, uint32_t kind,
                                            const NeeOut &o, float3 thr) {
    uint32_t pos = warp_append(A.cntShadow, pred);
    if (!pred) return;
    if (pos >= A.shadowCap) { atomicOr(A.err, (uint32_t)PT_DEVERR_QUEUE); return; }
    A.sslot[pos] = slot | (kind << 31) | (o.trLater ? kShadowTrLater : 0u);
    A.so[pos] = make_float4(o.o.x, o.o.y, o.o.z, o.tmin);
    A.sd[pos] = make_float4(o.d.x, o.d.y, o.d.z, o.tmax);
    A.sX[pos] = make_float4(o.X.x, o.X.y, o.X.z, 0.0f);
    A.sthr[pos] = make_float4(thr.x, thr.y, thr.z, 0.0f);
}

// Material type served by a surface shading class.
__host__ __device__ constexpr uint32_t class_type(int c) {
    return c == CLS_DIFFUSE ? PT_MAT_DIFFUSE : c == CLS_MICRO ? PT_MAT_MICROFACET
                                             : c == CLS_DISNEY ? PT_MAT_DISNEY : PT_MAT_HAIR;
}

// ---- shade: one bounce of RayGen's loop body (Shaders.hlsl:108-627) --------
// CLS == CLS_ANY: every path of the ray queue, events dispatched at run time
// (media scenes).  Otherwise the paths of one shading class, whose event and
// material type are then compile-time facts: each class gets a small kernel.
// Resident blocks per SM the shading kernels are compiled for.  The Disney
// kernel is latency-bound: 3 blocks (80 registers, a few spills) beat 2
// blocks (112 registers, none) by 7 % on B200.  The others get the count
// their register use gives anyway (a bound makes the compiler spend up to it).
template <int CLS>
struct ShadeBlocks {
    static constexpr int base = CLS < 0 ? CLS : CLS == CLS_MEDIUM ? CLS : CLS % CLS_TEX;
    static constexpr int value = base == CLS_MISS ? 5 : (base == CLS_EMIT || base == CLS_DELTA) ? 4
                                                      : base == CLS_DISNEY ? 4 : base == CLS_MEDIUM ? 3 : 2;
};

// SubsurfaceWalk (Subsurface.hlsli:49-144): random walk inside the closed
// mesh `mesh` from pos along dir; scalar extinction sigmaT, per-channel albedo
// alpha, HG phase g, Fresnel at the boundary (reflect back or leave), Russian
// roulette after 5 steps, at most 256 steps.  True with the exit point,
// direction, outward normal and throughput factor; a hit on other geometry or
// an absorbed walk gives false.  Interior rays take the alpha test with key
// kind 3.
__device__ bool subsurface_walk(const WaveArgs &A, float3 pos, float3 dir, uint32_t mesh, float sigmaT, float3 alpha,
                                float g, float intIOR, float extIOR, Rng &rng, uint32_t aseed, uint32_t bounce,
                                float3 &exitPos, float3 &exitDir, float3 &exitN, float3 &tmul) {
    const DevScene &S = A.S;
    tmul = v3(1.0f);
    exitPos = pos;
    exitDir = dir;
    exitN = dir;
    for (int step = 0; step < 256; step++) {
        float d = sigmaT > 0.0f ? -logf(mx(next_float(rng, S.sobol1), 1e-10f)) / sigmaT : 1e30f;
        Hit p = trace_closest(S, pos, dir, 1e-4f, d, A.err, aseed, alpha_key(bounce, 3u));
        if (p.gid != 0xFFFFFFFFu && p.t < d) {
            const uint32_t hm = __ldg(S.triMesh + p.gid);
            if (hm != mesh) {
                tmul = v3(0.0f);
                return false;
            }
            const uint32_t prim = p.gid - __ldg(S.meshFirstTri + hm);
            uint32_t i0, i1, i2;
            tri_vidx(S, hm, prim, i0, i1, i2);
            float3 bPos = pos + dir * p.t;
            float w0 = 1.0f - p.u - p.v;
            float3 nn = ld3(S.nrm, i0) * w0 + ld3(S.nrm, i1) * p.u + ld3(S.nrm, i2) * p.v;
            float l2 = dot(nn, nn);
            float3 p0 = ld3(S.pos, i0), p1 = ld3(S.pos, i1), p2 = ld3(S.pos, i2);
            float3 Nb = normalize(l2 < 1e-8f ? normalize(cross(p1 - p0, p2 - p0)) : nn * (1.0f / sqrtf(l2)));
            if (dot(Nb, dir) < 0.0f) Nb = -Nb;
            float Fr = fresnel(dot(dir, Nb), intIOR, extIOR);
            if (next_float(rng, S.sobol1) < Fr) {
                dir = normalize(reflect(dir, Nb));
                pos = bPos - Nb * 1e-4f;
                continue;
            }
            float3 outDir = refract(dir, -Nb, intIOR / extIOR);
            if (dot(outDir, outDir) < 1e-8f) {
                dir = normalize(reflect(dir, Nb));
                pos = bPos - Nb * 1e-4f;
                continue;
            }
            exitPos = bPos;
            exitDir = normalize(outDir);
            exitN = Nb;
            return true;
        }
        pos = pos + dir * d;
        tmul *= alpha;
        float x1 = next_float(rng, S.sobol1), x2 = next_float(rng, S.sobol1), pp;
        dir = sample_hg(dir, g, x1, x2, pp);
        if (step > 4) {
            float q = clampf(maxc(tmul), 0.05f, 0.95f);
            if (next_float(rng, S.sobol1) >= q) {
                tmul = v3(0.0f);
                return false;
            }
            tmul = tmul / v3(q);
        }
    }
    tmul = v3(0.0f);
    return false;
}

// Texture maps at a surface hit (Shaders.hlsl:232-315): albedo (sRGB),
// normal map in the frame of the triangle's UV derivatives, roughness (not
// for hair, whose `roughness` is beta_m), specular (x 0.5), subsurface; each
// at the mip level of the hit's UV footprint.  Overrides m's fields, bends N.
__device__ __forceinline__ void apply_textures(const DevScene &S, pt_material &m, uint32_t mesh, uint32_t prim,
                                               float hitT, uint32_t i0, uint32_t i1, uint32_t i2, float b1, float b2,
                                               float3 &N, uint32_t width, uint32_t height) {
    const float foot = uv_footprint(S, mesh, prim, hitT, width, height);
    const float2 uv = interp_uv(S, i0, i1, i2, b1, b2);
    float3 alb = make_float3(m.albedo[0], m.albedo[1], m.albedo[2]);
    if (m.albedoTexIndex != PT_NO_TEXTURE) {
        float4 c = tex_sample(S, m.albedoTexIndex, uv.x, uv.y, tex_lod(S, m.albedoTexIndex, foot));
        alb = make_float3(c.x, c.y, c.z);
    }
    if (m.normalTexIndex != PT_NO_TEXTURE) {
        float3 p0 = ld3(S.pos, i0), p1 = ld3(S.pos, i1), p2 = ld3(S.pos, i2);
        float3 e1 = p1 - p0, e2 = p2 - p0;
        float u0 = __ldg(S.uv + 2 * i0), v0 = __ldg(S.uv + 2 * i0 + 1);
        float du1 = __ldg(S.uv + 2 * i1) - u0, dv1 = __ldg(S.uv + 2 * i1 + 1) - v0;
        float du2 = __ldg(S.uv + 2 * i2) - u0, dv2 = __ldg(S.uv + 2 * i2 + 1) - v0;
        float det = du1 * dv2 - du2 * dv1;
        float3 T, B;
        if (fabsf(det) > 1e-8f) {
            float invDet = 1.0f / det;
            T = normalize((dv2 * e1 - dv1 * e2) * invDet);
            T = normalize(T - N * dot(N, T));
            B = cross(N, T);
        } else {
            build_onb(N, T, B);
        }
        float4 c = tex_sample(S, m.normalTexIndex, uv.x, uv.y, tex_lod(S, m.normalTexIndex, foot));
        float3 tn = make_float3(c.x, c.y, c.z) * 2.0f - v3(1.0f);
        N = normalize(T * tn.x + B * tn.y + N * tn.z);
    }
    m.albedo[0] = alb.x;
    m.albedo[1] = alb.y;
    m.albedo[2] = alb.z;
    if (m.type != PT_MAT_HAIR && m.roughnessTexIndex != PT_NO_TEXTURE) {
        float r = tex_sample(S, m.roughnessTexIndex, uv.x, uv.y, tex_lod(S, m.roughnessTexIndex, foot)).x;
        m.alpha = r;
        m.roughness = r;
    }
    if (m.specularTexIndex != PT_NO_TEXTURE)
        m.specular = tex_sample(S, m.specularTexIndex, uv.x, uv.y, tex_lod(S, m.specularTexIndex, foot)).x * 0.5f;
    if (m.subsurfaceTexIndex != PT_NO_TEXTURE)
        m.subsurface = tex_sample(S, m.subsurfaceTexIndex, uv.x, uv.y, tex_lod(S, m.subsurfaceTexIndex, foot)).x;
}

// Radiance-cache record of a surface vertex: position + roughness input,
// direction toward the previous vertex + path slot, shading normal, albedo.
__device__ __forceinline__ void cache_record(float4 *const *buf, uint32_t i, float3 p, float3 wo, float3 n,
                                             const pt_material &m, uint32_t type, uint32_t slot) {
    float rough = type == PT_MAT_MICROFACET ? m.alpha : type == PT_MAT_DISNEY ? m.roughness
                  : (type == PT_MAT_MIRROR || type == PT_MAT_DIELECTRIC) ? 0.0f : 1.0f;
    buf[0][i] = make_float4(p.x, p.y, p.z, rough);
    buf[1][i] = make_float4(wo.x, wo.y, wo.z, __uint_as_float(slot));
    buf[2][i] = make_float4(n.x, n.y, n.z, 0.0f);
    buf[3][i] = make_float4(m.albedo[0], m.albedo[1], m.albedo[2], 0.0f);
}
// A BSDF-sampled bounce that ends the path into the cache at its next vertex.
__device__ __forceinline__ bool rough_bounce(const WaveArgs &A, uint32_t type, const pt_material &m) {
    return type == PT_MAT_DIFFUSE || type == PT_MAT_HAIR || (type == PT_MAT_MICROFACET && m.alpha >= A.roughThr) ||
           (type == PT_MAT_DISNEY && m.roughness >= A.roughThr);
}

// CLS + CLS_TEX: the kernel of class CLS for materials with shading textures.
// EXTRA: the instantiation for RIS NEE and homogeneous media in the wavefront;
// the default one carries neither (their code would raise register pressure).
// What one shading event leaves for the kernel around it: whether the path
// goes on and with which ray, and its deferred NEE rays.
struct ShadeOut {
    bool cont;
    uint32_t slot;
    float3 no, nd;
    float ntmin;
    NeeOut neeA, neeE;
    float3 thrNee;
};
// The shading event of ray-queue position i (active: i is a real entry).
template <bool INLINE, int CLS, bool EXTRA>
__device__ __forceinline__ void shade_item(const WaveArgs &A, bool active, uint32_t i, ShadeOut &O) {
    constexpr int C = ShadeBlocks<CLS>::base;    // the event / material class
    constexpr bool TEX = CLS >= (int)CLS_TEX && CLS != (int)CLS_MEDIUM;  // shading textures present
    const DevScene &S = A.S;
    bool cont = false;
    uint32_t slot = 0;
    float3 thr = v3(1.0f), Lo = v3(0.0f);
    float lastPdf = 0.0f, eta = 1.0f;
    uint4 st = make_uint4(0, 0, 0, 0);
    float3 no = v3(0.0f), nd = v3(0.0f);
    float ntmin = 0.0f;
    NeeOut neeA, neeE;
    neeA.ray = neeE.ray = false;
    neeA.traced = neeE.traced = false;
    neeA.trLater = neeE.trLater = false;
    float3 thrNee = v3(0.0f);
    Rng rng;
    if (active) {
        slot = A.bounce == 0u ? i : A.qslotIn[i];
        // bounce 0 outside the medium wavefront: the initial state, known
        const bool fresh = A.bounce == 0u && !S.mediaWavefront;
        float4 tp = fresh ? make_float4(1.0f, 1.0f, 1.0f, 0.0f) : A.thr_pdf[slot];
        float4 le = fresh ? make_float4(0.0f, 0.0f, 0.0f, 1.0f) : A.lo_eta[slot];
        st = A.rng[slot];
        thr = make_float3(tp.x, tp.y, tp.z);
        lastPdf = tp.w;
        Lo = make_float3(le.x, le.y, le.z);
        eta = fabsf(le.w);  // the sign of w flags pending NEE for the film
        if (st.w & kFlagPending) {  // NEE of the previous bounce, in RayGen's order
            float4 pa = A.pendA[slot], pe = A.pendE[slot];
            Lo += make_float3(pa.x, pa.y, pa.z);
            Lo += make_float3(pe.x, pe.y, pe.z);
            st.w &= ~kFlagPending;
        }
        rng = load_rng(A, slot, st);
        const uint32_t aseed = S.hasAlpha ? alpha_seed(rng.pixelSeed, rng.sampleIndex) : 0u;
        float4 o4 = A.qoIn[i], d4 = A.qdIn[i], h4 = A.qhit[i];
        float3 ro = make_float3(o4.x, o4.y, o4.z), rd = make_float3(d4.x, d4.y, d4.z);
        uint32_t gid = __float_as_uint(h4.y);
        bool hit = gid != 0xFFFFFFFFu;
        bool volScat = false;
        if (INLINE && S.numVols > 0) {  // Shaders.hlsl:133-179
            float tSurf = hit ? h4.x : 1e20f;
            float tsc;
            uint32_t svi;
            float3 vw = v3(1.0f);
            bool sc = sample_free_flight(S, ro, rd, tSurf, rng, vw, tsc, svi);
            thr *= vw;
            if (sc) {
                volScat = true;
                const pt_volume &v = S.vols[svi];
                float3 spos = xpos(ro, rd, tsc);
                thr *= make_float3(v.sigma_s[0], v.sigma_s[1], v.sigma_s[2]) / vmax(vsigma_t(v), v3(1e-20f));
                Lo += thr * vol_nee_area<true>(A, spos, rd, svi, rng, aseed, st.z, neeA);
                Lo += thr * vol_nee_env<true>(A, spos, rd, svi, rng, aseed, st.z, neeE);
                float x1 = next_float(rng, S.sobol1), x2 = next_float(rng, S.sobol1);
                float pp;
                nd = sample_hg(rd, v.phase_g, x1, x2, pp);
                no = spos;
                ntmin = 0.0f;
                lastPdf = mx(pp, 1e-20f);
                cont = true;
                st.w |= kFlagRough;
            }
        }
        if (EXTRA && C == CLS_MEDIUM) {  // scattering in a homogeneous medium (Shaders.hlsl:149-178), NEE deferred
            const uint32_t svi = gid & 0x7FFFFFFFu;
            const pt_volume &v = S.vols[svi];
            float3 spos = xpos(ro, rd, h4.x);
            thr *= make_float3(v.sigma_s[0], v.sigma_s[1], v.sigma_s[2]) / vmax(vsigma_t(v), v3(1e-20f));
            vol_nee_area<false>(A, spos, rd, svi, rng, aseed, st.z, neeA);
            vol_nee_env<false>(A, spos, rd, svi, rng, aseed, st.z, neeE);
            thrNee = thr;
            if (!neeA.ray) A.pendA[slot] = make_float4(thr.x * 0.0f, thr.y * 0.0f, thr.z * 0.0f, 0.0f);
            if (!neeE.ray) A.pendE[slot] = make_float4(thr.x * 0.0f, thr.y * 0.0f, thr.z * 0.0f, 0.0f);
            st.w |= kFlagPending;
            float x1 = next_float(rng, S.sobol1), x2 = next_float(rng, S.sobol1);
            float pp;
            nd = sample_hg(rd, v.phase_g, x1, x2, pp);
            no = spos;
            ntmin = 0.0f;
            lastPdf = mx(pp, 1e-20f);
            cont = true;
            st.w |= kFlagRough;
        } else if (volScat) {
        } else if (C == CLS_MISS || (C == CLS_ANY && !hit)) {  // Shaders.hlsl:188-212
            float3 env = eval_env(S, rd);
            if (lastPdf == 0.0f) Lo += thr * env;
            else Lo += thr * env * balance(lastPdf, env_pdf(S, A.envMode, rd));
        } else if (C != CLS_MISS) {
            uint32_t mesh = __ldg(S.triMesh + gid);
            uint32_t prim = gid - __ldg(S.meshFirstTri + mesh);
            pt_material m = S.mats[mesh];
            const uint32_t type = C >= CLS_DIFFUSE ? class_type(C) : m.type;
            uint32_t i0, i1, i2;
            tri_vidx(S, mesh, prim, i0, i1, i2);
            float bx = h4.z, by = h4.w, w0 = 1.0f - bx - by;
            float3 hp = ro + rd * h4.x;
            float3 p0 = ld3(S.pos, i0), p1 = ld3(S.pos, i1), p2 = ld3(S.pos, i2);
            float3 Ng = normalize(normalize(cross(p1 - p0, p2 - p0)));
            float3 nn = ld3(S.nrm, i0) * w0 + ld3(S.nrm, i1) * bx + ld3(S.nrm, i2) * by;
            float l2 = dot(nn, nn);
            float3 N = normalize(l2 < 1e-8f ? normalize(cross(p1 - p0, p2 - p0)) : nn * (1.0f / sqrtf(l2)));
            bool back = dot(Ng, rd) > 0.0f;
            if (back) Ng = -Ng;
            if (dot(N, Ng) < 0.0f) N = -N;
            if (TEX || (C == CLS_ANY && has_shading_textures(m)))
            {
                const uint2 wh = path_image(A, slot);
                apply_textures(S, m, mesh, prim, h4.x, i0, i1, i2, bx, by, N, wh.x, wh.y);
            }
            // Radiance cache: the first surface vertex after a rough bounce ends
            // the path (a query, resolved after the wave), or, with probability
            // *trainProb, records its state there and the path goes on as a
            // training path (its suffix ends at its own next cache vertex, or
            // for one in unbiasedEvery, runs without the cache).
            bool cacheStop = false;
            if (A.cacheOn && (st.w & kFlagRough) && !(C == CLS_EMIT || (C == CLS_ANY && m.isEmitter))) {
                bool train = (st.w & kFlagTrain) != 0;
                if (!train && A.trainOn) {
                    const uint32_t hsh = pcg_hash(pcg_hash(rng.pixelSeed ^ (rng.sampleIndex * 0x9E3779B9u)) ^ st.z);
                    if ((float)(hsh >> 8) * (1.0f / 16777216.0f) < __ldg(A.trainProb)) {
                        uint32_t r = warp_append(A.crCount, true);
                        if (r < A.recCap) {
                            cache_record(A.cr, r, hp, -rd, N, m, type, slot);
                            {  // its order key, independent of the path order: sample-major
                                uint32_t kp, ks;
                                path_pos_sample(A, A.waveStart + slot, kp, ks);
                                A.cr[2][r].w = __uint_as_float(
                                    (uint32_t)((uint64_t)ks * A.npix + kp - A.recKeyBase));
                            }
                            A.cr[4][r] = make_float4(thr.x, thr.y, thr.z, 0.0f);
                            A.cr[5][r] = make_float4(Lo.x, Lo.y, Lo.z, 0.0f);
                            st.w |= kFlagTrain | kFlagHasRec | (r << 8);
                            if (A.unbiasedEvery && pcg_hash(hsh) % A.unbiasedEvery == 0) st.w |= kFlagUnbiased;
                            train = true;
                            // the image takes this path as it takes the others (prefix +
                            // throughput x cache here); its suffix only feeds training
                            uint32_t q = warp_append(A.cqCount, true);
                            if (q < A.queryCap) {
                                cache_record(A.cq, q, hp, -rd, N, m, type, r | 0x80000000u);
                                A.cq[4][q] = make_float4(thr.x, thr.y, thr.z, 0.0f);
                            } else {
                                atomicOr(A.err, (uint32_t)PT_DEVERR_QUEUE);
                            }
                        }
                    }
                    if (train) {
                    } else {
                        uint32_t q = warp_append(A.cqCount, true);
                        if (q < A.queryCap) {
                            cache_record(A.cq, q, hp, -rd, N, m, type, slot);
                            A.cq[4][q] = make_float4(thr.x, thr.y, thr.z, 0.0f);
                        } else {
                            atomicOr(A.err, (uint32_t)PT_DEVERR_QUEUE);
                        }
                        cacheStop = true;
                    }
                } else if (!(train && (st.w & kFlagUnbiased))) {
                    uint32_t q = warp_append(A.cqCount, true);
                    if (q < A.queryCap) {
                        cache_record(A.cq, q, hp, -rd, N, m, type, slot);
                        A.cq[4][q] = make_float4(thr.x, thr.y, thr.z, 0.0f);
                    } else {
                        atomicOr(A.err, (uint32_t)PT_DEVERR_QUEUE);
                    }
                    cacheStop = true;
                }
            }
            if (C == CLS_EMIT || (C == CLS_ANY && m.isEmitter)) {  // Shaders.hlsl:317-335
                float3 rad = make_float3(m.radiance[0], m.radiance[1], m.radiance[2]);
                if (lastPdf == 0.0f) Lo += thr * rad;
                else Lo += thr * rad * balance(lastPdf, emitter_pdf_sa(S, m, hp, ro, N));
            } else if (C != CLS_EMIT && !cacheStop) {
                float3 T, B;
                float h = 0.0f;
                if (type == PT_MAT_HAIR) {  // Shaders.hlsl:340-387
                    float hu = __ldg(S.uv + 2 * i0) * w0 + __ldg(S.uv + 2 * i1) * bx + __ldg(S.uv + 2 * i2) * by;
                    float hv = __ldg(S.uv + 2 * i0 + 1) * w0 + __ldg(S.uv + 2 * i1 + 1) * bx +
                               __ldg(S.uv + 2 * i2 + 1) * by;
                    float3 ht = ld3(S.tan, i0) * w0 + ld3(S.tan, i1) * bx + ld3(S.tan, i2) * by;
                    float tl2 = dot(ht, ht);
                    ht = tl2 > 1e-8f ? ht * (1.0f / sqrtf(tl2)) : v3(0.0f);
                    if (dot(ht, ht) > 1e-8f) {
                        ht = normalize(ht);
                        h = hv * 2.0f - 1.0f;
                    } else {
                        float a0u = __ldg(S.uv + 2 * i0), a0v = __ldg(S.uv + 2 * i0 + 1);
                        float d1u = __ldg(S.uv + 2 * i1) - a0u, d1v = __ldg(S.uv + 2 * i1 + 1) - a0v;
                        float d2u = __ldg(S.uv + 2 * i2) - a0u, d2v = __ldg(S.uv + 2 * i2 + 1) - a0v;
                        float det = d1u * d2v - d2u * d1v;
                        if (fabsf(det) > 1e-8f) ht = normalize((-d1u * (p1 - p0) + d2u * (p2 - p0)) * (1.0f / det));
                        else build_onb(N, ht, B);
                        h = hu * 2.0f - 1.0f;
                    }
                    T = normalize(ht - N * dot(ht, N));
                    B = cross(N, T);
                } else {
                    build_onb(N, T, B);
                }
                {  // terminator bend, Shaders.hlsl:402-411
                    float3 V = -rd;
                    float ndv = dot(N, V);
                    if (ndv <= 0.0f && dot(V, Ng) > 0.0f) {
                        N = normalize(N + V * (1e-3f - ndv));
                        build_onb(N, T, B);
                    }
                }
                float3 wil = to_local(-rd, T, B, N);
                if (type == PT_MAT_MIRROR) {  // Shaders.hlsl:419-427
                    float es;
                    nd = delta_scatter(PT_MAT_MIRROR, rd, N, back, m.intIOR, m.extIOR, 0.0f, es);
                    no = axpy_nf(0.001f, Ng, hp);
                    lastPdf = 0.0f;
                    cont = true;
                    st.w &= ~kFlagRough;
                } else if (type == PT_MAT_DIELECTRIC) {  // Shaders.hlsl:429-472
                    float es;
                    nd = delta_scatter(PT_MAT_DIELECTRIC, rd, N, back, m.intIOR, m.extIOR,
                                       next_float(rng, S.sobol1), es);
                    no = axpy_nf(0.001f, dot_nf(nd, Ng) > 0.0f ? Ng : -Ng, hp);
                    lastPdf = 0.0f;
                    eta *= es;
                    cont = true;
                    st.w &= ~kFlagRough;
                } else if (C != CLS_DELTA &&
                           (type == PT_MAT_DIFFUSE || type == PT_MAT_MICROFACET || type == PT_MAT_DISNEY ||
                            type == PT_MAT_HAIR)) {  // Shaders.hlsl:473-511
                    float3 ra = ((INLINE || EXTRA) && A.risNee)
                                    ? nee_ris<INLINE, EXTRA>(A, hp, N, Ng, T, B, wil, type, m, h, rng, neeA, aseed, st.z)
                                    : nee_area<INLINE, EXTRA>(A, hp, N, Ng, T, B, wil, type, m, h, rng, neeA, aseed, st.z);
                    float3 re = nee_env<INLINE, EXTRA>(A, hp, N, Ng, T, B, wil, type, m, h, rng, neeE, aseed, st.z);
                    if (INLINE) {
                        Lo += thr * ra;
                        Lo += thr * re;
                    } else {
                        thrNee = thr;
                        if (!neeA.ray) A.pendA[slot] = make_float4(thr.x * 0.0f, thr.y * 0.0f, thr.z * 0.0f, 0.0f);
                        if (!neeE.ray) A.pendE[slot] = make_float4(thr.x * 0.0f, thr.y * 0.0f, thr.z * 0.0f, 0.0f);
                        st.w |= kFlagPending;
                    }
                    float u[4];
                    int k = material_sample_dims_t(type, wil);
                    for (int j = 0; j < k; j++) u[j] = next_float(rng, S.sobol1);
                    float3 wol;
                    float bp;
                    float3 wt = material_sample_t(type, wil, u, m, h, wol, bp);
                    if (!(bp <= 0.0f || (wt.x == 0.0f && wt.y == 0.0f && wt.z == 0.0f))) {
                        float3 ww = to_world(wol, T, B, N);
                        float3 on = type == PT_MAT_HAIR ? (dot(ww, Ng) >= 0.0f ? Ng : -Ng) : Ng;
                        no = offset_origin(hp, on, on);
                        nd = ww;
                        thr *= wt;
                        lastPdf = mx(bp, 1e-20f);
                        cont = true;
                        if (A.cacheOn) st.w = rough_bounce(A, type, m) ? (st.w | kFlagRough) : (st.w & ~kFlagRough);
                    }
                } else if (C == CLS_ANY && type == PT_MAT_SUBSURFACE) {  // Shaders.hlsl:515-611
                    // rough dielectric entry (Beckmann half vector, Fresnel choice),
                    // NEE with the entry lobe, then reflect or walk the interior
                    const float3 I = rd;
                    m.roughness = m.roughness * (1.0f + sat(m.specular * 2.0f) * (0.65f - 1.0f));
                    const float rough = m.roughness;
                    const float aR = mx(rough * rough, 1e-4f);
                    float3 wmL = make_float3(0.0f, 0.0f, 1.0f);
                    if (rough > 1e-3f) {
                        float u0 = next_float(rng, S.sobol1), u1 = next_float(rng, S.sobol1);
                        wmL = beckmann_sample(u0, u1, aR);
                    }
                    float3 wm = normalize(to_world(wmL, T, B, N));
                    float cosThetaM = dot(-I, wm);
                    if (cosThetaM <= 0.0f) {
                        wm = N;
                        wmL = make_float3(0.0f, 0.0f, 1.0f);
                        cosThetaM = dot(-I, N);
                    }
                    const float G1i = rough > 1e-3f ? smith_g1(wil, wmL, aR) : 1.0f;
                    const float Fr = fresnel(cosThetaM, m.extIOR, m.intIOR);
                    Lo += thr * nee_area<INLINE>(A, hp, N, Ng, T, B, wil, type, m, h, rng, neeA, aseed, st.z);
                    Lo += thr * nee_env<INLINE>(A, hp, N, Ng, T, B, wil, type, m, h, rng, neeE, aseed, st.z);
                    if (next_float(rng, S.sobol1) < Fr) {
                        float3 refl = reflect(I, wm);
                        float3 woL = to_local(refl, T, B, N);
                        if (woL.z > 0.0f) {  // else reflected below the surface: the path ends
                            float weight = rough > 1e-3f ? G1i * smith_g1(woL, wmL, aR) * cosThetaM /
                                                               mx(wil.z * wmL.z, 1e-6f)
                                                         : 1.0f;
                            float pdfSpec = rough > 1e-3f
                                                ? Fr * beckmann_d_cos(wmL, aR) / mx(4.0f * cosThetaM, 1e-6f)
                                                : 0.0f;
                            no = hp + Ng * 0.001f;
                            nd = refl;
                            thr = thr * weight;
                            lastPdf = pdfSpec;
                            cont = true;
                        }
                    } else {
                        float3 refr = refract(I, wm, m.extIOR / m.intIOR);
                        if (dot(refr, refr) < 1e-8f) {
                            no = hp + Ng * 0.001f;
                            nd = reflect(I, wm);
                            lastPdf = 0.0f;
                            cont = true;
                        } else {
                            const float3 tint = make_float3(m.sheen, m.sheenTint, m.clearcoat);
                            const float3 aSharp = make_float3(m.albedo[0], m.albedo[1], m.albedo[2]);
                            float3 aBlur = aSharp, detail = v3(1.0f);
                            if (m.albedoTexIndex != PT_NO_TEXTURE) {  // albedo blurred 4 mip levels up
                                const uint2 wh = path_image(A, slot);
                                const float foot = uv_footprint(S, mesh, prim, h4.x, wh.x, wh.y);
                                const float2 tuv = interp_uv(S, i0, i1, i2, bx, by);
                                float4 cb = tex_sample(S, m.albedoTexIndex, tuv.x, tuv.y,
                                                       tex_lod(S, m.albedoTexIndex, foot) + 4.0f);
                                aBlur = make_float3(cb.x, cb.y, cb.z);
                                float3 r = aSharp / vmax(aBlur, v3(1e-3f));
                                detail = make_float3(clampf(r.x, 0.5f, 2.0f), clampf(r.y, 0.5f, 2.0f),
                                                     clampf(r.z, 0.5f, 2.0f));
                            }
                            float sigmaT;
                            float3 alb;
                            subsurface_params(aBlur * tint, m.subsurface, sigmaT, alb);
                            float3 ep, ed, en, tm;
                            if (subsurface_walk(A, hp - Ng * 0.001f, normalize(refr), mesh, sigmaT, alb,
                                                m.anisotropic, m.intIOR, m.extIOR, rng, aseed, st.z, ep, ed, en,
                                                tm)) {
                                thr *= tm * detail;
                                no = offset_origin(ep, en, en);
                                nd = ed;
                                lastPdf = 0.0f;
                                cont = true;
                            }
                        }
                    }
                }
            }
        }
        // Russian roulette after bounce 3 (Shaders.hlsl:620-626)
        if (cont && st.z >= 3u) {
            float q = mn(maxc(thr) * eta * eta, 0.95f);
            if (next_float(rng, S.sobol1) >= q) cont = false;
            else thr = thr / v3(q);
        }
        st.z += 1u;
        if (st.z >= path_depth(A, slot)) cont = false;
        st.x = rng.dim;
        st.y = rng.white;
        // a finished path's throughput is read by nothing, and its RNG
        // state only by the shadow kernel's alpha tests and the cache's
        // target pass
        if (cont) A.thr_pdf[slot] = make_float4(thr.x, thr.y, thr.z, lastPdf);
        // w = eta, negative while NEE of this bounce is pending: the film
        // reads the flag here instead of the path's RNG state
        A.lo_eta[slot] = make_float4(Lo.x, Lo.y, Lo.z, (st.w & kFlagPending) ? -eta : eta);
        if (cont || S.hasAlpha || A.cacheOn) A.rng[slot] = st;
    }
    O.cont = cont;
    O.slot = slot;
    O.no = no;
    O.nd = nd;
    O.ntmin = ntmin;
    O.neeA = neeA;
    O.neeE = neeE;
    O.thrNee = thrNee;
}
template <bool INLINE, int CLS, bool EXTRA = false>
__global__ void __launch_bounds__(kBlock, ShadeBlocks<CLS>::value) k_shade(WaveArgs A) {
    uint32_t n = CLS == CLS_ANY ? *(volatile uint32_t *)A.cntIn : *(volatile uint32_t *)(A.cntCls + CLS);
    uint32_t iters = (n + gridDim.x * blockDim.x - 1) / (gridDim.x * blockDim.x);
    uint32_t traced = 0;
    for (uint32_t it = 0; it < iters; it++) {
        uint32_t q = (it * gridDim.x + blockIdx.x) * blockDim.x + threadIdx.x;
        bool active = q < n;
        uint32_t i = q;
        if (CLS != CLS_ANY && active) i = A.cls[(size_t)(CLS < 0 ? 0 : CLS) * A.clsStride + q];
        ShadeOut O;
        shade_item<INLINE, CLS, EXTRA>(A, active, i, O);
        if (!INLINE) {
            push_shadow(A, active && O.neeA.ray, O.slot, 0u, O.neeA, O.thrNee);
            push_shadow(A, active && O.neeE.ray, O.slot, 1u, O.neeE, O.thrNee);
        } else if (active) {
            traced += (O.neeA.traced ? 1u : 0u) + (O.neeE.traced ? 1u : 0u);
        }
        uint32_t pos = warp_append(A.cntOut, active && O.cont);
        if (active && O.cont) {
            A.qslotOut[pos] = O.slot;
            A.qoOut[pos] = make_float4(O.no.x, O.no.y, O.no.z, O.ntmin);
            A.qdOut[pos] = make_float4(O.nd.x, O.nd.y, O.nd.z, 1e20f);
        }
    }
    if (INLINE) add_rays(A, 1, traced);
}

// ---- the tail of a wave: its remaining bounces in one launch --------------------
// From bounce PT_TAIL_BOUNCE on a wave may carry few paths, but every bounce's
// kernels still last as long as their slowest ray (about 0.23 ms per bounce
// of the bench frame, 12 bounces of 16).  When at most kTailMaxPaths paths
// are left, k_tail runs each to its end in one thread, its next ray kept in
// the path's own queue position, and k_tail_close empties the queue so the
// per-bounce kernels that follow (launched either way) find nothing; with
// more paths left k_tail returns at once and the per-bounce kernels go on.
// It is launched only when at least kTailMinRemaining bounces remain: one
// thread per path keeps a warp's finished lanes idle until its longest path
// ends (the per-bounce kernels compact them away every bounce), so the tail
// pays only where it saves many per-bounce latency floors.  Measured with
// the tail forced on (Mpaths/s): the 64-sphere scene at depth 16, 4 / 16 / 64
// spp: 901 -> 1054, 1463 -> 1614, 1779 -> 1853; the Cornell box at depth 8,
// 2 / 4 / 16 spp: 124 -> 100, 210 -> 155, 390 -> 196.  2^18 live paths let
// the tail take the Cornell box at 16 spp; 2^17 does not, and keeps the
// 64-sphere scene's gain.
// The result does not depend on which runs: the tail calls the same shading
// instantiations as the per-bounce kernels — the class-specialized ones, with
// each deferred NEE ray resolved in place with k_shadow's arithmetic, or for
// scenes shaded inline the inline one — in the same order per path.
// 0 = no tail.
#ifndef PT_TAIL_BOUNCE
#define PT_TAIL_BOUNCE 4
#endif
constexpr uint32_t kTailBounce = PT_TAIL_BOUNCE;
constexpr uint32_t kTailMaxPaths = 1u << 17;
constexpr uint32_t kTailMinRemaining = 8;

// A deferred NEE ray of a shading event, resolved here as k_shadow resolves a
// queued one (its default instantiation): the pending record for the path's
// next shading event or the film.
template <class Stack>
__device__ __forceinline__ void tail_shadow(const WaveArgs &A, Stack &K, uint32_t slot, uint32_t kind, const NeeOut &ne,
                                            float3 thr) {
    uint32_t aseed = 0, akey = 0;
    if (A.S.hasAlpha) {  // the shading event already advanced the path's bounce counter
        Rng r = load_rng(A, slot, A.rng[slot]);
        aseed = alpha_seed(r.pixelSeed, r.sampleIndex);
        akey = alpha_key(A.rng[slot].z - 1u, kind ? 2u : 1u);
    }
    float3 tr;
    bool occ = trace_shadow_on(K, A.S, ne.o, ne.d, ne.tmin, ne.tmax, tr, A.err, aseed, akey);
    float3 R = occ ? thr * v3(0.0f) : thr * (ne.X * tr);
    float4 out = make_float4(R.x, R.y, R.z, 0.0f);
    if (kind) __stcs(A.pendE + slot, out);
    else __stcs(A.pendA + slot, out);
}
// One shading event of queue position i with the per-bounce kernels' code.
template <bool INLINE, class Stack>
__device__ __forceinline__ void tail_shade(const WaveArgs &A, Stack &K, uint32_t i, ShadeOut &O, uint32_t &traced) {
    if (INLINE) {
        shade_item<true, CLS_ANY, false>(A, true, i, O);
        traced += (O.neeA.traced ? 1u : 0u) + (O.neeE.traced ? 1u : 0u);
        return;
    }
    const uint32_t gid = __float_as_uint(A.qhit[i].y);
    const int c = gid == 0xFFFFFFFFu ? (int)CLS_MISS : (int)__ldg(A.S.meshClass + __ldg(A.S.triMesh + gid));
    switch (c) {
        case CLS_MISS: shade_item<false, CLS_MISS, false>(A, true, i, O); break;
        case CLS_EMIT: shade_item<false, CLS_EMIT, false>(A, true, i, O); break;
        case CLS_DELTA: shade_item<false, CLS_DELTA, false>(A, true, i, O); break;
        case CLS_DIFFUSE: shade_item<false, CLS_DIFFUSE, false>(A, true, i, O); break;
        case CLS_MICRO: shade_item<false, CLS_MICRO, false>(A, true, i, O); break;
        case CLS_DISNEY: shade_item<false, CLS_DISNEY, false>(A, true, i, O); break;
        case CLS_HAIR: shade_item<false, CLS_HAIR, false>(A, true, i, O); break;
        case CLS_TEX + CLS_EMIT: shade_item<false, CLS_TEX + CLS_EMIT, false>(A, true, i, O); break;
        case CLS_TEX + CLS_DELTA: shade_item<false, CLS_TEX + CLS_DELTA, false>(A, true, i, O); break;
        case CLS_TEX + CLS_DIFFUSE: shade_item<false, CLS_TEX + CLS_DIFFUSE, false>(A, true, i, O); break;
        case CLS_TEX + CLS_MICRO: shade_item<false, CLS_TEX + CLS_MICRO, false>(A, true, i, O); break;
        case CLS_TEX + CLS_DISNEY: shade_item<false, CLS_TEX + CLS_DISNEY, false>(A, true, i, O); break;
        default: shade_item<false, CLS_TEX + CLS_HAIR, false>(A, true, i, O); break;
    }
    if (O.neeA.ray) {
        tail_shadow(A, K, O.slot, 0u, O.neeA, O.thrNee);
        ++traced;
    }
    if (O.neeE.ray) {
        tail_shadow(A, K, O.slot, 1u, O.neeE, O.thrNee);
        ++traced;
    }
}
template <bool INLINE>
__global__ void __launch_bounds__(kBlock, 2) k_tail(WaveArgs A) {
    const uint32_t n = *(volatile uint32_t *)A.cntIn;
    if (n > A.tailMax) return;  // uniform: the per-bounce kernels take the rest
    PT_QUEUE_STACK(K)
    uint32_t ext = 0, traced = 0;
    for (uint32_t base; (base = claim32(A.stealExt)) < n;) {
        const uint32_t i = base + lane_id();
        bool live = i < n;
        while (live) {  // each lane its own path
            extend_one<false, false>(A, i, K);
            ++ext;
            ShadeOut O;
            tail_shade<INLINE>(A, K, i, O, traced);
            live = O.cont;
            if (live) {
                A.qoIn[i] = make_float4(O.no.x, O.no.y, O.no.z, O.ntmin);
                A.qdIn[i] = make_float4(O.nd.x, O.nd.y, O.nd.z, 1e20f);
            }
        }
    }
    add_rays(A, 0, ext);
    add_rays(A, 1, traced);
    for (int o = 16; o > 0; o >>= 1) ext += __shfl_xor_sync(0xFFFFFFFFu, ext, o);
    if (lane_id() == 0 && ext) atomicAdd(A.tailRays, (unsigned long long)ext);
}
// After k_tail: if it ran, its paths are done and the queue is empty.
__global__ void k_tail_close(WaveArgs A) {
    if (*A.cntIn <= A.tailMax) *A.cntIn = 0u;
}

// ---- film: Kahan-compensated accumulation of (L, 1), samples in order -------
// (Shaders.hlsl:629-634: NaN/Inf guard, then accum += (Lo, 1)).
__device__ __forceinline__ void kahan(float &s, float &c, float x) {
    float y = x - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
}
// One thread per pixel position: the wave's samples of the pixel, in sample
// order (path_id), Kahan-added to the film.
__global__ void k_film(WaveArgs A, float4 *sum, float4 *comp) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= A.npix) return;
    const uint64_t first = A.waveStart, last = A.waveStart + A.waveCount;
    // the samples the wave can hold: its first and last paths' samples, widened to their groups
    uint32_t p0, s0, p1, s1;
    path_pos_sample(A, first, p0, s0);
    path_pos_sample(A, last - 1, p1, s1);
    uint32_t lo, hi;
    path_group(A, s0, s0, hi);
    path_group(A, s1, lo, s1);
    s1 = min(s1, A.spp - 1u);
    bool any = false;
    float4 s = make_float4(0.0f, 0.0f, 0.0f, 0.0f), c = s;
    const uint32_t pix = tile_pixel(A, p);
    for (uint32_t smp = s0; smp <= s1; smp++) {
        const uint64_t pid = path_id(A, p, smp);
        if (pid < first || pid >= last) continue;
        if (!any) {
            s = sum[pix];
            c = comp[pix];
            any = true;
        }
        uint32_t slot = (uint32_t)(pid - first);
        float4 le = A.lo_eta[slot];
        float3 L = make_float3(le.x, le.y, le.z);
        if (le.w < 0.0f) {  // NEE of the last bounce pending
            float4 pa = A.pendA[slot], pe = A.pendE[slot];
            L += make_float3(pa.x, pa.y, pa.z);
            L += make_float3(pe.x, pe.y, pe.z);
        }
        if (isnan(L.x) || isnan(L.y) || isnan(L.z) || isinf(L.x) || isinf(L.y) || isinf(L.z)) L = v3(0.0f);
        kahan(s.x, c.x, L.x);
        kahan(s.y, c.y, L.y);
        kahan(s.z, c.z, L.z);
        kahan(s.w, c.w, 1.0f);
    }
    if (any) {
        sum[pix] = s;
        comp[pix] = c;
    }
}

// Film of request q for the paths of this wave (k_film's order: per pixel,
// the wave's samples of the request in sample order).
__global__ void k_film_req(WaveArgs A, uint32_t q) {
    const ReqDev &R = A.reqs[q];
    const uint64_t ps = R.pathStart, pe = R.pathStart + (uint64_t)R.npix * R.spp;
    const uint64_t ws = A.waveStart, we = A.waveStart + A.waveCount;
    const uint64_t lo = (ws > ps ? ws : ps) - ps, hi = (we < pe ? we : pe) - ps;
    if (hi <= lo) return;
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= min(hi - lo, (uint64_t)R.npix)) return;
    uint32_t pix = tile_pixel_wh(R.width, R.height, (uint32_t)((lo + t) % R.npix));
    float4 s = R.sum[pix], c = R.comp[pix];
    for (uint64_t l = lo + t; l < hi; l += R.npix) {
        uint32_t slot = (uint32_t)(ps + l - ws);
        float4 le = A.lo_eta[slot];
        float3 L = make_float3(le.x, le.y, le.z);
        if (le.w < 0.0f) {  // NEE of the last bounce pending
            float4 pa = A.pendA[slot], pe4 = A.pendE[slot];
            L += make_float3(pa.x, pa.y, pa.z);
            L += make_float3(pe4.x, pe4.y, pe4.z);
        }
        if (isnan(L.x) || isnan(L.y) || isnan(L.z) || isinf(L.x) || isinf(L.y) || isinf(L.z)) L = v3(0.0f);
        kahan(s.x, c.x, L.x);
        kahan(s.y, c.y, L.y);
        kahan(s.z, c.z, L.z);
        kahan(s.w, c.w, 1.0f);
    }
    R.sum[pix] = s;
    R.comp[pix] = c;
}

}  // namespace pt

using namespace pt;

static int grid_for(pt_ctx *ctx, const void *fn) {
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, kBlock, 0) != cudaSuccess || blocks < 1) blocks = 1;
    return blocks * ctx->numSMs;
}

int pt_wave_free(pt_ctx *ctx) {
    WaveBuffers &W = ctx->W;
    void *ps[] = {W.thr_pdf, W.lo_eta, W.pendA, W.pendE, W.rng, W.qslot[0], W.qslot[1], W.qo[0], W.qo[1],
                  W.qd[0], W.qd[1], W.qhit, W.cls, W.sslot, W.so, W.sd, W.sX, W.sthr, W.counters};
    for (void *p : ps)
        if (p) cudaFree(p);
    W = WaveBuffers{};
    return PT_OK;
}

// Bytes of wave state per path slot: 5 float4/uint4 of path state, two ray
// queues (slot + origin + direction), the hit buffer, one entry in each
// shading-class queue, and two shadow-queue
// entries (slot + origin + direction + contribution + throughput).
constexpr size_t kWaveBytesPerPath = 5 * 16 + 2 * (4 + 16 + 16) + 16 + 4 * CLS_N + 2 * (4 + 4 * 16);
// Default wave cap: 2^26 paths (~22 GB of state).  Larger renders run as
// several waves, whose tails are small at this size, instead of regrowing the
// buffers (a free + malloc of tens of GB that would stall the render).
constexpr size_t kMaxWavePaths = (size_t)1 << 26;
static_assert(kWaveBytesPerPath == 364, "wave state layout");

static int wave_alloc(pt_ctx *ctx, size_t cap) {
    if (ctx->W.cap >= cap) return PT_OK;
    pt_wave_free(ctx);
    WaveBuffers &W = ctx->W;
    size_t sc = 2 * cap;
    cudaError_t e = cudaSuccess;
    auto A = [&](void **p, size_t bytes) { if (e == cudaSuccess) e = cudaMalloc(p, bytes); };
    A((void **)&W.thr_pdf, cap * 16); A((void **)&W.lo_eta, cap * 16);
    A((void **)&W.pendA, cap * 16); A((void **)&W.pendE, cap * 16); A((void **)&W.rng, cap * 16);
    for (int k = 0; k < 2; k++) { A((void **)&W.qslot[k], cap * 4); A((void **)&W.qo[k], cap * 16); A((void **)&W.qd[k], cap * 16); }
    A((void **)&W.qhit, cap * 16);
    A((void **)&W.cls, cap * 4 * CLS_N);
    A((void **)&W.sslot, sc * 4); A((void **)&W.so, sc * 16); A((void **)&W.sd, sc * 16);
    A((void **)&W.sX, sc * 16); A((void **)&W.sthr, sc * 16);
    A((void **)&W.counters, kCounterWords * sizeof(uint32_t));
    if (e != cudaSuccess) {
        pt_wave_free(ctx);
        return ctx->fail(PT_E_NOMEM, "wave buffers", cudaGetErrorString(e));
    }
    W.cap = cap;
    ctx->waveGen++;
    return PT_OK;
}

namespace {
using Kernel = void (*)(WaveArgs);
// per class; entry CLS_TEX + CLS_MISS (a textured miss) never receives paths
template <bool X>
struct ShadeTable {
    static constexpr Kernel k[CLS_N] = {
        k_shade<false, CLS_MISS, X>,            k_shade<false, CLS_EMIT, X>,
        k_shade<false, CLS_DELTA, X>,           k_shade<false, CLS_DIFFUSE, X>,
        k_shade<false, CLS_MICRO, X>,           k_shade<false, CLS_DISNEY, X>,
        k_shade<false, CLS_HAIR, X>,            k_shade<false, CLS_MISS, X>,
        k_shade<false, CLS_TEX + CLS_EMIT, X>,  k_shade<false, CLS_TEX + CLS_DELTA, X>,
        k_shade<false, CLS_TEX + CLS_DIFFUSE, X>, k_shade<false, CLS_TEX + CLS_MICRO, X>,
        k_shade<false, CLS_TEX + CLS_DISNEY, X>, k_shade<false, CLS_TEX + CLS_HAIR, X>,
        k_shade<false, CLS_MEDIUM, true>};
};
// per class: the default kernels, and the EXTRA ones (RIS NEE, media in the wavefront)
const Kernel *const kShadeCls = ShadeTable<false>::k;
const Kernel *const kShadeClsX = ShadeTable<true>::k;
int gExt = 0, gExtC = 0, gExtM = 0, gShadeI = 0, gShadow = 0, gShadowM = 0, gCls[CLS_N], gClsX[CLS_N];
int gTail = 0, gTailI = 0;

// STG_CACHE_INFER / STG_CACHE_TRAIN: the cache's network kernels, reported
// in ms_cache with the rest of the cache's work and on their own in the
// cache statistics
enum {
    STG_RAYGEN, STG_EXTEND, STG_SHADE, STG_SHADOW, STG_FILM, STG_CACHE, STG_CACHE_INFER, STG_CACHE_TRAIN, STG_TAIL,
    STG_N
};
// The bounce at which k_tail may take a wave's remaining paths (depth: never):
// with at least kTailMinRemaining bounces after it, or any (tail mode 2:
// tests).  Not for cached renders, RIS NEE or media in the wavefront form
// (other shading instantiations).
inline uint32_t tail_bounce(uint32_t depth, const WaveArgs &A, uint32_t tailMode) {
    const bool enough = depth >= kTailBounce + kTailMinRemaining || tailMode == 2u;
    return (kTailBounce > 0 && kTailBounce < depth && enough && !A.cacheOn && !A.risNee && !A.S.mediaWavefront)
               ? kTailBounce
               : depth;
}
struct Mark { int stage; cudaEvent_t a, b; };

// Issues one render's work on a stream: directly (optionally with an event
// pair around every launch), or into a stream capture.
struct Enqueue {
    cudaStream_t st;
    bool timing;
    std::vector<Mark> marks;
    uint64_t launches = 0;
    void begin(int stage) {
        launches++;
        if (!timing) return;
        Mark m{stage, nullptr, nullptr};
        cudaEventCreate(&m.a);
        cudaEventCreate(&m.b);
        cudaEventRecord(m.a, st);
        marks.push_back(m);
    }
    void end() {
        if (timing) cudaEventRecord(marks.back().b, st);
    }
};

// Grid sizes of the traversal and shading kernels (grid-stride loops).
struct Grids {
    int ext, extC, extM, shadeI, shadow, shadowM;
    const int *cls, *clsX;
    int tail, tailI;
};

// Raygen and `depth` bounces of one wave (A.waveStart / A.waveCount set).
// Returns the first failing call's status (cudaSuccess if none).
cudaError_t enqueue_paths(const pt_ctx *ctx, Enqueue &E, WaveArgs &A, uint32_t depth, const Grids &G) {
    const WaveBuffers &B = ctx->W;
    const bool inl = (ctx->S.numVols > 0 && !A.S.mediaWavefront) || ctx->S.hasSubsurface;
    cudaStream_t st = E.st;
    cudaError_t err = cudaSuccess;
    auto chk = [&](cudaError_t e) {
        if (err == cudaSuccess && e != cudaSuccess) err = e;
    };
    A.qslotOut = B.qslot[0]; A.qoOut = B.qo[0]; A.qdOut = B.qd[0]; A.cntOut = B.counters + 0;
    E.begin(STG_RAYGEN);
    k_raygen<<<(A.waveCount + kBlock - 1) / kBlock, kBlock, 0, st>>>(A);
    E.end();
    int cur = 0;
    for (uint32_t b = 0; b < depth; b++) {
        A.bounce = b;
        A.qslotIn = B.qslot[cur]; A.qoIn = B.qo[cur]; A.qdIn = B.qd[cur]; A.cntIn = B.counters + cur;
        A.qslotOut = B.qslot[1 - cur]; A.qoOut = B.qo[1 - cur]; A.qdOut = B.qd[1 - cur];
        A.cntOut = B.counters + (1 - cur);
        chk(cudaMemsetAsync(A.cntOut, 0, 4, st));
        chk(cudaMemsetAsync(A.cntShadow, 0, 8, st));  // shadow count and the extend claim position
        if (b == tail_bounce(depth, A, ctx->dbgTail)) {  // the remaining bounces of every path in one launch, when few are left
            E.begin(STG_TAIL);
            if (inl) k_tail<true><<<G.tailI, kBlock, 0, st>>>(A);
            else k_tail<false><<<G.tail, kBlock, 0, st>>>(A);
            k_tail_close<<<1, 1, 0, st>>>(A);
            E.end();
        }
        if (inl) {
            E.begin(STG_EXTEND);
            k_extend<false><<<G.ext, kBlock, 0, st>>>(A);
            E.end();
            E.begin(STG_SHADE);
            k_shade<true, CLS_ANY><<<G.shadeI, kBlock, 0, st>>>(A);
            E.end();
        } else {
            // class counts and the shadow claim position after them
            chk(cudaMemsetAsync(A.cntCls, 0, (CLS_N + 1) * sizeof(uint32_t), st));
            E.begin(STG_EXTEND);
            if (A.S.mediaWavefront) k_extend_media<<<G.extM, kBlock, 0, st>>>(A);
            else k_extend<true><<<G.extC, kBlock, 0, st>>>(A);
            E.end();
            const bool extra = A.risNee || A.S.mediaWavefront;
            const uint32_t mask = ctx->clsMask | (A.S.mediaWavefront ? 1u << CLS_MEDIUM : 0u);
            for (int c = 0; c < CLS_N; c++) {
                if (!((mask >> c) & 1u)) continue;
                E.begin(STG_SHADE);
                if (extra) kShadeClsX[c]<<<G.clsX[c], kBlock, 0, st>>>(A);
                else kShadeCls[c]<<<G.cls[c], kBlock, 0, st>>>(A);
                E.end();
            }
            E.begin(STG_SHADOW);
            if (A.S.mediaTrDeferred) k_shadow_media<<<G.shadowM, kBlock, 0, st>>>(A);
            else k_shadow<<<G.shadow, kBlock, 0, st>>>(A);
            E.end();
        }
        cur = 1 - cur;
    }
    return err;
}

// Returns the first failing call's status (cudaSuccess if none).
cudaError_t enqueue_render(const pt_ctx *ctx, Enqueue &E, WaveArgs A, const pt_render_params *P, size_t cap,
                           uint64_t total, uint64_t npix, float *d_sum, float *d_comp) {
    const WaveBuffers &B = ctx->W;
    cudaStream_t st = E.st;
    cudaError_t err = cudaSuccess;
    auto chk = [&](cudaError_t e) {
        if (err == cudaSuccess && e != cudaSuccess) err = e;
    };
    const bool cached = A.cacheOn != 0;
    const Grids G{gExt, gExtC, gExtM, gShadeI, gShadow, gShadowM, gCls, gClsX, gTail, gTailI};
    chk(cudaMemsetAsync(B.counters, 0, kCounterWords * sizeof(uint32_t), st));
    chk(cudaMemsetAsync(ctx->d_err, 0, 4, st));
    if (cached) {  // per-call cache counters: records [2], queries of the call [5], records with targets [6]
        chk(cudaMemsetAsync(A.crCount, 0, 4, st));
        chk(cudaMemsetAsync(ctx->cache.ctr + 5, 0, 8, st));
    }
    for (uint64_t ws = 0; ws < total; ws += cap) {
        A.waveStart = ws;
        A.waveCount = (uint32_t)std::min<uint64_t>(cap, total - ws);
        {  // the samples this wave holds (whole groups of 8): its training records' key range
            uint32_t p0, s0, p1, s1;
            path_pos_sample(A, A.waveStart, p0, s0);
            path_pos_sample(A, A.waveStart + A.waveCount - 1, p1, s1);
            uint32_t lo, hi;
            path_group(A, s0, s0, hi);
            path_group(A, s1, lo, s1);
            s1 = std::min(s1, A.spp - 1u);
            A.recKeyBase = (uint64_t)s0 * A.npix;
            A.recKeyRange = (uint32_t)std::min<uint64_t>((uint64_t)(s1 - s0 + 1) * A.npix, 0xFFFFFFFFull);
        }
        if (cached) chk(cudaMemsetAsync(A.cqCount, 0, 4, st));
        chk(enqueue_paths(ctx, E, A, P->max_depth, G));
        if (cached) {
            // cache queries of this wave: lo_eta[slot] += throughput x cache, or
            // the cache value at a training record's vertex
            E.begin(STG_CACHE_INFER);
            chk(rc_enqueue_resolve(const_cast<pt_ctx *>(ctx), st, A.lo_eta));
            E.end();
            // training targets from the suffixes, then the training paths' image
            // values (prefix + throughput x cache); counts the wave's queries
            E.begin(STG_CACHE);
            chk(rc_enqueue_targets(const_cast<pt_ctx *>(ctx), st, A.lo_eta, A.rng, A.pendA, A.pendE, A.recKeyRange));
            E.end();
        }
        uint32_t cover = (uint32_t)npix;  // k_film: one thread per pixel position
        if (ws == 0) {  // the film's contents (a host film's upload may still be in flight)
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            chk(cudaStreamIsCapturing(st, &cs));
            chk(cudaStreamWaitEvent(st, ctx->filmReady,
                                    cs == cudaStreamCaptureStatusActive ? cudaEventWaitExternal : 0u));
        }
        E.begin(STG_FILM);
        k_film<<<(cover + kBlock - 1) / kBlock, kBlock, 0, st>>>(A, (float4 *)d_sum, (float4 *)d_comp);
        E.end();
        chk(cudaGetLastError());  // launch-configuration errors of this wave
    }
    if (cached && A.trainOn) {  // training steps on the call's records
        for (uint32_t step = 0; step < kRcStepsPerCall; step++) {
            E.begin(STG_CACHE_TRAIN);
            chk(rc_enqueue_train(const_cast<pt_ctx *>(ctx), st, step, false));
            E.end();
            E.begin(STG_CACHE);
            chk(rc_enqueue_train(const_cast<pt_ctx *>(ctx), st, step, true));
            E.end();
        }
    }
    return err;
}

__global__ void k_set_u32(uint32_t *p, uint32_t v) { *p = v; }


bool graph_matches(const pt_ctx *ctx, const pt_render_params *P, size_t cap, const float *sum, const float *comp,
                   const WaveArgs &A) {
    const RenderGraph &G = ctx->graph;
    return G.exec && G.width == P->width && G.height == P->height && G.spp == P->spp && G.maxDepth == P->max_depth &&
           G.rngKind == P->rng_kind && G.envSampling == P->env_sampling && G.cap == cap && G.sum == sum &&
           G.comp == comp && G.sceneGen == ctx->sceneGen && G.waveGen == ctx->waveGen &&
           G.cached == A.cacheOn && G.trainOn == A.trainOn && (!A.cacheOn || G.cacheGen == ctx->cache.gen) &&
           G.risNee == A.risNee && G.flags == (P->flags & ~PT_RENDER_STAGE_TIMING) &&
           G.shadowCap == A.shadowCap && G.cacheStall == ctx->dbgCacheStall && G.tailMax == A.tailMax &&
           G.tailMode == ctx->dbgTail &&
           memcmp(&G.cam, &P->camera, sizeof(pt_camera)) == 0;
}
}  // namespace

void pt_graph_free(pt_ctx *ctx) {
    if (ctx->graph.exec) cudaGraphExecDestroy(ctx->graph.exec);
    ctx->graph = RenderGraph{};
}

int pt_render_impl(pt_ctx *ctx, const pt_render_params *P, float *d_sum, float *d_comp, pt_stats *stats) {
    const uint32_t W = P->width, H = P->height;
    const uint64_t npix = (uint64_t)W * H;
    const uint64_t total = npix * P->spp;
    // Default wave: the whole render, up to kMaxWavePaths and half of the
    // free device memory.  Each bounce of a wave ends with a latency-bound
    // tail (a few slow traversals), so fewer, larger waves amortise it; the
    // 59 M paths of a 1280 x 720 x 64 frame take ~21 GB.
    // The free-memory query runs only when the buffers would have to grow: it
    // is a driver call that can block on other clients of the driver.
    size_t cap = P->wave_paths;
    if (!cap) {
        size_t want = (size_t)std::min<uint64_t>(total, kMaxWavePaths);
        if (want <= ctx->W.cap) {
            cap = want;
        } else {
            size_t freeB = 0, totalB = 0;
            if (cudaMemGetInfo(&freeB, &totalB) != cudaSuccess) freeB = (size_t)4 << 30;
            size_t fit = (freeB / 2 + ctx->W.cap * kWaveBytesPerPath / 2) / kWaveBytesPerPath;
            cap = std::max<size_t>(std::min(want, fit), std::min<size_t>(want, (size_t)1 << 16));
        }
    }
    if (npix <= cap) cap = (cap / npix) * npix;
    if (cap > total) cap = (size_t)total;
    if (cap == 0) return PT_OK;
    int rc = wave_alloc(ctx, cap);
    if (rc) return rc;
    cudaStream_t st = ctx->stream;
    WaveBuffers &B = ctx->W;
    if (!gExt) {
        gExt = grid_for(ctx, (const void *)k_extend<false>);
        gExtC = grid_for(ctx, (const void *)k_extend<true>);
        gExtM = grid_for(ctx, (const void *)k_extend_media);
        gShadeI = grid_for(ctx, (const void *)k_shade<true, CLS_ANY>);
        gShadow = grid_for(ctx, (const void *)k_shadow);
        gShadowM = grid_for(ctx, (const void *)k_shadow_media);
        for (int c = 0; c < CLS_N; c++) {
            gCls[c] = grid_for(ctx, (const void *)kShadeCls[c]);
            gClsX[c] = grid_for(ctx, (const void *)kShadeClsX[c]);
        }
        gTail = grid_for(ctx, (const void *)k_tail<false>);
        gTailI = grid_for(ctx, (const void *)k_tail<true>);
    }
    WaveArgs A;
    A.S = ctx->S;
    A.width = W; A.height = H; A.npix = (uint32_t)npix;
    A.spp = P->spp;
    A.spp32 = P->spp & ~31u;  // samples in groups of 32, then of 8 (path_pos_sample)
    A.spp8 = (P->spp - A.spp32) & ~7u;
    A.fullTilePix = 32u * (W / 8u) * (H / 4u);
    A.sampleOffset = ctx->d_err + 1;
    A.rngKind = P->rng_kind; A.envMode = P->env_sampling; A.maxDepth = P->max_depth;
    A.cam = P->camera;
    A.thr_pdf = B.thr_pdf; A.lo_eta = B.lo_eta; A.pendA = B.pendA; A.pendE = B.pendE; A.rng = B.rng;
    A.qhit = B.qhit;
    A.sslot = B.sslot; A.so = B.so; A.sd = B.sd; A.sX = B.sX; A.sthr = B.sthr;
    A.cntShadow = B.counters + kCntShadow;
    A.stealExt = B.counters + kCntStealExt;
    A.stealShadow = B.counters + kCntStealShadow;
    A.cntCls = B.counters + kCntClass;
    A.cls = B.cls;
    A.clsStride = (uint32_t)B.cap;
    A.rayTotals = (unsigned long long *)(B.counters + 4);
    A.tailRays = (unsigned long long *)(B.counters + kCntTailRays);
    A.tailMax = ctx->dbgTail == 1u ? 0u : kTailMaxPaths;
    A.err = ctx->d_err;
    A.shadowCap = (uint32_t)(2 * B.cap);
    if (ctx->dbgShadowCap) A.shadowCap = std::min(A.shadowCap, ctx->dbgShadowCap);
    A.batch = 0; A.numReqs = 0; A.reqs = nullptr; A.slotInfo = nullptr;
    A.risNee = (P->flags & PT_RENDER_RIS_NEE) ? 1u : 0u;
    if ((P->flags & PT_RENDER_MEDIA_WAVEFRONT) && A.S.numVols > 0 && !A.S.hasSubsurface && !A.S.mediaWavefront) {
        A.S.mediaWavefront = 1u;  // heterogeneous media (homogeneous-only scenes have it already)
        A.S.mediaTrDeferred = 1u;
    }
    A.cacheOn = (P->flags & PT_RENDER_RADIANCE_CACHE) ? 1u : 0u;
    A.trainOn = A.unbiasedEvery = A.recCap = A.queryCap = 0;
    A.roughThr = 0.0f;
    A.trainProb = nullptr;
    for (float4 *&q : A.cq) q = nullptr;
    for (float4 *&r : A.cr) r = nullptr;
    A.cqCount = A.crCount = nullptr;
    if (A.cacheOn) {
        if ((rc = rc_render_setup(ctx, B.cap, total))) return rc;
        const RadianceCache &C = ctx->cache;
        A.roughThr = C.params.rough_threshold;
        A.unbiasedEvery = C.params.unbiased_every;
        A.recCap = (uint32_t)C.recCap;
        A.trainOn = (C.params.flags & PT_CACHE_NO_TRAIN) ? 0u : 1u;
        A.queryCap = (uint32_t)C.queryCap;
        A.trainProb = reinterpret_cast<const float *>(C.ctr + 7);
        for (int k = 0; k < 5; k++) A.cq[k] = C.q[k];
        for (int k = 0; k < 7; k++) A.cr[k] = C.rec[k];
        A.cqCount = C.ctr + 1;
        A.crCount = C.ctr + 2;
    }
    const uint64_t waves = (total + cap - 1) / cap;
    // Without per-launch timing the render replays a CUDA graph of its launch
    // sequence, captured on the first call with this configuration: no host
    // gaps between the ~100 launches of a render.
    const bool timing = (P->flags & PT_RENDER_STAGE_TIMING) != 0;
    bool useGraph = !timing;
    if (useGraph && !graph_matches(ctx, P, cap, d_sum, d_comp, A)) {
        pt_graph_free(ctx);
        Enqueue E{ctx->ownStream, false, {}, 0};
        cudaGraph_t g = nullptr;
        cudaGraphExec_t exec = nullptr;
        bool ok = cudaStreamBeginCapture(ctx->ownStream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            cudaError_t qe = enqueue_render(ctx, E, A, P, cap, total, npix, d_sum, d_comp);
            ok = cudaStreamEndCapture(ctx->ownStream, &g) == cudaSuccess && g && qe == cudaSuccess;
        }
        ok = ok && cudaGraphInstantiate(&exec, g, 0) == cudaSuccess;
        if (g) cudaGraphDestroy(g);
        if (ok) {
            RenderGraph &G = ctx->graph;
            G.exec = exec;
            G.width = W; G.height = H; G.spp = P->spp; G.maxDepth = P->max_depth;
            G.rngKind = P->rng_kind; G.envSampling = P->env_sampling; G.cam = P->camera;
            G.cap = cap; G.sum = d_sum; G.comp = d_comp;
            G.sceneGen = ctx->sceneGen; G.waveGen = ctx->waveGen;
            G.cached = A.cacheOn; G.trainOn = A.trainOn; G.cacheGen = ctx->cache.gen; G.risNee = A.risNee;
            G.flags = P->flags & ~PT_RENDER_STAGE_TIMING;
            G.shadowCap = A.shadowCap; G.cacheStall = ctx->dbgCacheStall; G.tailMax = A.tailMax;
            G.tailMode = ctx->dbgTail;
            G.launches = E.launches;
        } else {  // capture unavailable: issue the launches directly
            cudaGetLastError();
            useGraph = false;
        }
    }
    cudaEvent_t *ev = ctx->ev;
    cudaEventRecord(ev[0], st);
    k_set_u32<<<1, 1, 0, st>>>(ctx->d_err + 1, P->sample_offset);
    Enqueue E{st, timing, {}, 0};
    uint64_t launches = 1;
    if (useGraph) {
        PT_CUDA(cudaGraphLaunch(ctx->graph.exec, st));
        launches += ctx->graph.launches;
    } else {
        cudaError_t qe = enqueue_render(ctx, E, A, P, cap, total, npix, d_sum, d_comp);
        launches += E.launches;
        if (qe != cudaSuccess) {
            cudaStreamSynchronize(st);
            for (Mark &m : E.marks) { cudaEventDestroy(m.a); cudaEventDestroy(m.b); }
            return ctx->fail(PT_E_CUDA, "render launch", cudaGetErrorString(qe));
        }
    }
    cudaEventRecord(ev[1], st);
    uint32_t hostCnt[kCounterWords];
    PT_CUDA(cudaMemcpyAsync(hostCnt, B.counters, sizeof(hostCnt), cudaMemcpyDeviceToHost, st));
    uint32_t derr = 0;
    PT_CUDA(cudaMemcpyAsync(&derr, ctx->d_err, 4, cudaMemcpyDeviceToHost, st));
    cudaError_t se = cudaStreamSynchronize(st);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev[0], ev[1]);
    float stage[STG_N] = {};
    for (Mark &m : E.marks) {
        float t = 0.0f;
        if (se == cudaSuccess) cudaEventElapsedTime(&t, m.a, m.b);
        stage[m.stage] += t;
        cudaEventDestroy(m.a);
        cudaEventDestroy(m.b);
    }
    if (se != cudaSuccess) return ctx->fail(PT_E_CUDA, "render", cudaGetErrorString(se));
    if (derr)
        return ctx->fail(PT_E_DEVICE, (derr & PT_DEVERR_STACK) ? "traversal stack overflow"
                                      : (derr & PT_DEVERR_BVH) ? "traversal visited more nodes than the BVH has"
                                      : (derr & PT_DEVERR_CACHE) ? "radiance cache kernel: a tensor-core wait timed out"
                                                                 : "queue overflow");
    if (stats) {
        unsigned long long tot[2];
        memcpy(tot, hostCnt + 4, sizeof(tot));
        stats->paths = total;
        stats->extension_rays = tot[0];
        stats->shadow_rays = tot[1];
        stats->waves = waves;
        stats->bounces = waves * P->max_depth;
        stats->launches = launches;
        stats->ms_total = ms;
        stats->ms_raygen = stage[STG_RAYGEN];
        stats->ms_extend = stage[STG_EXTEND];
        stats->ms_shade = stage[STG_SHADE];
        stats->ms_shadow = stage[STG_SHADOW];
        stats->ms_film = stage[STG_FILM];
        stats->ms_cache = stage[STG_CACHE] + stage[STG_CACHE_INFER] + stage[STG_CACHE_TRAIN];
        stats->ms_tail = stage[STG_TAIL];
        memcpy(&stats->tail_extension_rays, hostCnt + kCntTailRays, 8);
        if (timing && A.cacheOn) {
            ctx->cache.renderInferMs = stage[STG_CACHE_INFER];
            ctx->cache.renderTrainMs = stage[STG_CACHE_TRAIN];
        }
    }
    return PT_OK;
}

// ===========================================================================
// Batched requests
// ===========================================================================
void pt_batch_free(pt_ctx *ctx) {
    BatchState &Bt = ctx->batch;
    if (Bt.exec) cudaGraphExecDestroy(Bt.exec);
    for (cudaEvent_t e : Bt.ev) cudaEventDestroy(e);
    if (Bt.reqs) cudaFree(Bt.reqs);
    if (Bt.slotInfo) cudaFree(Bt.slotInfo);
    if (Bt.films) cudaFree(Bt.films);
    ctx->batch = BatchState{};
}

namespace {
struct BatchPlan {
    std::vector<uint32_t> order;        // request index by path order (shortest first)
    std::vector<uint64_t> start;        // first path id, path order
    uint64_t total = 0;
    size_t cap = 0;
    std::vector<uint64_t> waveStart;
    std::vector<uint32_t> waveDepth;
    std::vector<std::vector<uint32_t>> waveReqs;  // requests (path order) with paths in the wave
    std::vector<uint32_t> lastWave;     // per request (path order)
};

int batch_check(pt_ctx *ctx, const pt_request *R, uint32_t n) {
    if (!n || n > PT_BATCH_MAX_REQUESTS) return ctx->fail(PT_E_INVALID, "batch size outside 1..PT_BATCH_MAX_REQUESTS");
    for (uint32_t i = 0; i < n; i++) {
        const pt_render_params &P = R[i].params;
        const pt_film &F = R[i].film;
        if (!P.width || !P.height || !P.spp || !P.max_depth) return ctx->fail(PT_E_INVALID, "empty request");
        if ((uint64_t)P.width * P.height >= PT_BATCH_MAX_PIXELS)
            return ctx->fail(PT_E_INVALID, "request above PT_BATCH_MAX_PIXELS pixels");
        if (F.width != P.width || F.height != P.height || !F.sum || !F.comp)
            return ctx->fail(PT_E_INVALID, "request film does not match");
        if (P.rng_kind != R[0].params.rng_kind || P.env_sampling != R[0].params.env_sampling ||
            P.flags != R[0].params.flags)
            return ctx->fail(PT_E_INVALID, "rng_kind, env_sampling and flags must agree across a batch");
        if (P.rng_kind > PT_RNG_PCG_HASH || P.env_sampling > PT_ENV_ALIAS) return ctx->fail(PT_E_INVALID, "bad enum");
        if (P.flags & PT_RENDER_RADIANCE_CACHE) return ctx->fail(PT_E_UNSUPPORTED, "radiance cache in a batch");
    }
    return PT_OK;
}

BatchPlan batch_plan(const pt_request *R, uint32_t n, size_t cap) {
    BatchPlan pl;
    pl.order.resize(n);
    for (uint32_t i = 0; i < n; i++) pl.order[i] = i;
    auto paths = [&](uint32_t i) { return (uint64_t)R[i].params.width * R[i].params.height * R[i].params.spp; };
    std::stable_sort(pl.order.begin(), pl.order.end(), [&](uint32_t a, uint32_t b) { return paths(a) < paths(b); });
    for (uint32_t k = 0; k < n; k++) {
        pl.start.push_back(pl.total);
        pl.total += paths(pl.order[k]);
    }
    pl.cap = (size_t)std::min<uint64_t>(cap, pl.total);
    pl.lastWave.assign(n, 0);
    uint32_t k = 0;
    for (uint64_t ws = 0; ws < pl.total; ws += pl.cap) {
        const uint64_t we = std::min<uint64_t>(ws + pl.cap, pl.total);
        std::vector<uint32_t> rq;
        uint32_t depth = 0;
        while (k < n && pl.start[k] + paths(pl.order[k]) <= ws) k++;
        for (uint32_t j = k; j < n && pl.start[j] < we; j++) {
            rq.push_back(j);
            depth = std::max(depth, R[pl.order[j]].params.max_depth);
            pl.lastWave[j] = (uint32_t)pl.waveStart.size();
        }
        pl.waveStart.push_back(ws);
        pl.waveDepth.push_back(depth);
        pl.waveReqs.push_back(rq);
    }
    return pl;
}

cudaError_t enqueue_batch(const pt_ctx *ctx, Enqueue &E, WaveArgs A, const BatchPlan &pl, const Grids &G,
                          const ReqDev *hostReqs, const std::vector<cudaEvent_t> &ev, const char **where) {
    const WaveBuffers &B = ctx->W;
    cudaStream_t st = E.st;
    cudaError_t err = cudaSuccess;
    const char *at = "";
    auto chk = [&](cudaError_t e, const char *w = "") {
        if (err == cudaSuccess && e != cudaSuccess) { err = e; at = w; }
    };
    chk(cudaMemsetAsync(B.counters, 0, kCounterWords * sizeof(uint32_t), st), "memset counters");
    chk(cudaMemsetAsync(ctx->d_err, 0, 4, st), "memset err");
    for (size_t w = 0; w < pl.waveStart.size(); w++) {
        A.waveStart = pl.waveStart[w];
        A.waveCount = (uint32_t)std::min<uint64_t>(pl.cap, pl.total - A.waveStart);
        chk(enqueue_paths(ctx, E, A, pl.waveDepth[w], G), "paths");
        for (uint32_t j : pl.waveReqs[w]) {
            const ReqDev &R = hostReqs[j];
            const uint64_t ps = R.pathStart, pe = ps + (uint64_t)R.npix * R.spp;
            const uint64_t lo = std::max<uint64_t>(A.waveStart, ps), hi = std::min<uint64_t>(A.waveStart + A.waveCount, pe);
            const uint64_t cover = std::min<uint64_t>(hi - lo, R.npix);
            E.begin(STG_FILM);
            k_film_req<<<(unsigned)((cover + kBlock - 1) / kBlock), kBlock, 0, st>>>(A, j);
            E.end();
            chk(cudaGetLastError(), "film launch");
        }
        // an external record node: the event is recorded when the graph runs
        // (a plain record inside a capture is only an ordering edge)
        chk(cudaEventRecordWithFlags(ev[w], st, cudaEventRecordExternal), "event record");
        chk(cudaGetLastError(), "wave launches");
    }
    if (where) *where = at;
    return err;
}

// One batch: plan, staging of host films, graph (re)capture, launch, timings.
// tuneFilm != nullptr: every request renders into that device scratch film
// (autotuning), the callers' films are untouched.
int render_batch(pt_ctx *ctx, const pt_request *R, uint32_t n, float *request_ms, pt_stats *stats, size_t capIn,
                 float gridScale, float *tuneFilm, float *msOut) {
    int rc = batch_check(ctx, R, n);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    BatchState &Bt = ctx->batch;
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; i++) total += (uint64_t)R[i].params.width * R[i].params.height * R[i].params.spp;
    size_t cap = capIn ? capIn : R[0].params.wave_paths;
    if (!cap && Bt.tunedWave && Bt.tunedSceneGen == ctx->sceneGen) cap = Bt.tunedWave;
    if (!cap) cap = (size_t)std::min<uint64_t>(total, kMaxWavePaths);
    cap = (size_t)std::min<uint64_t>(cap, total);
    if (cap > ctx->W.cap) {  // grow within half the free memory, as a single render does
        size_t freeB = 0, totalB = 0;
        if (cudaMemGetInfo(&freeB, &totalB) != cudaSuccess) freeB = (size_t)4 << 30;
        size_t fit = (freeB / 2 + ctx->W.cap * kWaveBytesPerPath / 2) / (kWaveBytesPerPath + 8);
        cap = std::max<size_t>(std::min(cap, fit), std::min<size_t>(cap, (size_t)1 << 16));
    }
    if ((rc = wave_alloc(ctx, cap))) return rc;
    if (Bt.slotCap < cap) {
        if (Bt.slotInfo) cudaFree(Bt.slotInfo);
        Bt.slotInfo = nullptr;
        Bt.slotCap = 0;
        if (cudaMalloc(&Bt.slotInfo, cap * sizeof(uint2)) != cudaSuccess) return ctx->fail(PT_E_NOMEM, "batch slots");
        Bt.slotCap = cap;
    }
    if (!Bt.reqs && cudaMalloc(&Bt.reqs, PT_BATCH_MAX_REQUESTS * sizeof(ReqDev)) != cudaSuccess)
        return ctx->fail(PT_E_NOMEM, "batch request table");
    if (!gExt) {
        gExt = grid_for(ctx, (const void *)k_extend<false>);
        gExtC = grid_for(ctx, (const void *)k_extend<true>);
        gExtM = grid_for(ctx, (const void *)k_extend_media);
        gShadeI = grid_for(ctx, (const void *)k_shade<true, CLS_ANY>);
        gShadow = grid_for(ctx, (const void *)k_shadow);
        gShadowM = grid_for(ctx, (const void *)k_shadow_media);
        for (int c = 0; c < CLS_N; c++) {
            gCls[c] = grid_for(ctx, (const void *)kShadeCls[c]);
            gClsX[c] = grid_for(ctx, (const void *)kShadeClsX[c]);
        }
        gTail = grid_for(ctx, (const void *)k_tail<false>);
        gTailI = grid_for(ctx, (const void *)k_tail<true>);
    }
    if (gridScale <= 0.0f) gridScale = (Bt.tunedWave && Bt.tunedSceneGen == ctx->sceneGen) ? Bt.tunedGrid : 1.0f;
    auto sc = [&](int g) { return std::max(ctx->numSMs, (int)((float)g * gridScale)); };
    int clsG[CLS_N], clsGX[CLS_N];
    for (int c = 0; c < CLS_N; c++) {
        clsG[c] = sc(gCls[c]);
        clsGX[c] = sc(gClsX[c]);
    }
    const Grids G{sc(gExt), sc(gExtC), sc(gExtM), sc(gShadeI), sc(gShadow), sc(gShadowM), clsG, clsGX, sc(gTail),
                  sc(gTailI)};

    const BatchPlan pl = batch_plan(R, n, cap);
    // films: the callers' device films, device copies of host films, or the tuning scratch
    size_t stage = 0;
    for (uint32_t i = 0; i < n; i++)
        if (!tuneFilm && R[i].film.location == PT_MEM_HOST) stage += 2 * (size_t)R[i].params.width * R[i].params.height * 16;
    if (stage > Bt.filmBytes) {
        if (Bt.films) cudaFree(Bt.films);
        Bt.films = nullptr;
        Bt.filmBytes = 0;
        if (cudaMalloc(&Bt.films, stage) != cudaSuccess) return ctx->fail(PT_E_NOMEM, "batch film staging");
        Bt.filmBytes = stage;
    }
    std::vector<ReqDev> hostReqs(n);
    std::vector<float *> devSum(n), devComp(n);
    size_t off = 0;
    for (uint32_t k = 0; k < n; k++) {
        const uint32_t i = pl.order[k];
        const pt_render_params &P = R[i].params;
        const size_t bytes = (size_t)P.width * P.height * 16;
        float *ds = R[i].film.sum, *dc = R[i].film.comp;
        if (tuneFilm) {
            ds = tuneFilm;
            dc = tuneFilm + 4 * (size_t)P.width * P.height;
        } else if (R[i].film.location == PT_MEM_HOST) {
            ds = (float *)((char *)Bt.films + off);
            dc = (float *)((char *)Bt.films + off + bytes);
            off += 2 * bytes;
            PT_CUDA(cudaMemcpyAsync(ds, R[i].film.sum, bytes, cudaMemcpyHostToDevice, ctx->stream));
            PT_CUDA(cudaMemcpyAsync(dc, R[i].film.comp, bytes, cudaMemcpyHostToDevice, ctx->stream));
        }
        devSum[i] = ds;
        devComp[i] = dc;
        ReqDev &q = hostReqs[k];
        q.pathStart = pl.start[k];
        q.width = P.width; q.height = P.height; q.npix = P.width * P.height; q.spp = P.spp;
        q.sampleOffset = P.sample_offset; q.maxDepth = P.max_depth;
        q.cam = P.camera;
        q.sum = (float4 *)ds;
        q.comp = (float4 *)dc;
    }
    while (Bt.ev.size() < pl.waveStart.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return ctx->fail(PT_E_CUDA, "batch events");
        Bt.ev.push_back(e);
    }
    WaveBuffers &B = ctx->W;
    WaveArgs A;
    memset(&A, 0, sizeof(A));
    A.S = ctx->S;
    A.width = hostReqs[0].width; A.height = hostReqs[0].height; A.npix = hostReqs[0].npix;
    A.spp = A.spp32 = A.spp8 = A.fullTilePix = 0u;  // batches keep their own path order (slotInfo)
    A.recKeyBase = 0u;
    A.recKeyRange = 0u;
    A.sampleOffset = ctx->d_err + 1;
    A.rngKind = R[0].params.rng_kind; A.envMode = R[0].params.env_sampling; A.maxDepth = 0;
    A.thr_pdf = B.thr_pdf; A.lo_eta = B.lo_eta; A.pendA = B.pendA; A.pendE = B.pendE; A.rng = B.rng;
    A.qhit = B.qhit;
    A.sslot = B.sslot; A.so = B.so; A.sd = B.sd; A.sX = B.sX; A.sthr = B.sthr;
    A.cntShadow = B.counters + kCntShadow;
    A.stealExt = B.counters + kCntStealExt;
    A.stealShadow = B.counters + kCntStealShadow;
    A.cntCls = B.counters + kCntClass;
    A.cls = B.cls;
    A.clsStride = (uint32_t)B.cap;
    A.rayTotals = (unsigned long long *)(B.counters + 4);
    A.tailRays = (unsigned long long *)(B.counters + kCntTailRays);
    A.tailMax = ctx->dbgTail == 1u ? 0u : kTailMaxPaths;
    A.err = ctx->d_err;
    A.shadowCap = (uint32_t)(2 * B.cap);
    A.batch = 1; A.numReqs = n; A.reqs = (const ReqDev *)Bt.reqs; A.slotInfo = Bt.slotInfo;
    A.risNee = (R[0].params.flags & PT_RENDER_RIS_NEE) ? 1u : 0u;
    if ((R[0].params.flags & PT_RENDER_MEDIA_WAVEFRONT) && A.S.numVols > 0 && !A.S.hasSubsurface &&
        !A.S.mediaWavefront) {
        A.S.mediaWavefront = 1u;  // heterogeneous media (homogeneous-only scenes have it already)
        A.S.mediaTrDeferred = 1u;
    }
    // the launch graph depends on the batch's shape, not on cameras, offsets or films (device table)
    std::vector<uint64_t> key = {n, pl.cap, R[0].params.rng_kind, R[0].params.env_sampling, R[0].params.flags,
                                 ctx->sceneGen,
                                 ctx->waveGen, (uint64_t)(uintptr_t)Bt.slotInfo, (uint64_t)(uint32_t)G.extC,
                                 (uint64_t)(uint32_t)G.shadow, (uint64_t)(uint32_t)clsG[CLS_DISNEY], A.tailMax,
                                 ctx->dbgTail};
    for (uint32_t k = 0; k < n; k++) {
        key.push_back(hostReqs[k].width | ((uint64_t)hostReqs[k].height << 32));
        key.push_back(hostReqs[k].spp | ((uint64_t)hostReqs[k].maxDepth << 32));
    }
    if (!Bt.exec || Bt.key != key) {
        if (Bt.exec) cudaGraphExecDestroy(Bt.exec);
        Bt.exec = nullptr;
        Enqueue E{ctx->ownStream, false, {}, 0};
        cudaGraph_t g = nullptr;
        const char *step = "begin capture";
        cudaError_t ce = cudaStreamBeginCapture(ctx->ownStream, cudaStreamCaptureModeThreadLocal);
        if (ce == cudaSuccess) {
            const char *at = "";
            cudaError_t qe = enqueue_batch(ctx, E, A, pl, G, hostReqs.data(), Bt.ev, &at);
            ce = cudaStreamEndCapture(ctx->ownStream, &g);
            step = "end capture";
            if (ce == cudaSuccess && qe != cudaSuccess) {
                ce = qe;
                step = at;
            }
        }
        if (ce == cudaSuccess) {
            ce = cudaGraphInstantiate(&Bt.exec, g, 0);
            step = "instantiate";
        }
        if (g) cudaGraphDestroy(g);
        if (ce != cudaSuccess) {
            cudaGetLastError();
            Bt.exec = nullptr;
            std::string what = std::string("batch graph capture (") + step + ")";
            return ctx->fail(PT_E_CUDA, what.c_str(), cudaGetErrorString(ce));
        }
        Bt.key = key;
        Bt.launches = E.launches;
    }
    cudaStream_t st = ctx->stream;
    PT_CUDA(cudaMemcpyAsync(Bt.reqs, hostReqs.data(), n * sizeof(ReqDev), cudaMemcpyHostToDevice, st));
    cudaEventRecord(ctx->ev[0], st);
    PT_CUDA(cudaGraphLaunch(Bt.exec, st));
    cudaEventRecord(ctx->ev[1], st);
    uint32_t hostCnt[kCounterWords];
    PT_CUDA(cudaMemcpyAsync(hostCnt, B.counters, sizeof(hostCnt), cudaMemcpyDeviceToHost, st));
    uint32_t derr = 0;
    PT_CUDA(cudaMemcpyAsync(&derr, ctx->d_err, 4, cudaMemcpyDeviceToHost, st));
    if (!tuneFilm)
        for (uint32_t i = 0; i < n; i++)
            if (R[i].film.location == PT_MEM_HOST) {
                const size_t bytes = (size_t)R[i].params.width * R[i].params.height * 16;
                PT_CUDA(cudaMemcpyAsync(R[i].film.sum, devSum[i], bytes, cudaMemcpyDeviceToHost, st));
                PT_CUDA(cudaMemcpyAsync(R[i].film.comp, devComp[i], bytes, cudaMemcpyDeviceToHost, st));
            }
    cudaError_t se = cudaStreamSynchronize(st);
    if (se != cudaSuccess) return ctx->fail(PT_E_CUDA, "batch render", cudaGetErrorString(se));
    if (derr)
        return ctx->fail(PT_E_DEVICE, (derr & PT_DEVERR_STACK) ? "traversal stack overflow"
                                      : (derr & PT_DEVERR_BVH) ? "traversal visited more nodes than the BVH has"
                                                               : "queue overflow");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    if (msOut) *msOut = ms;
    if (request_ms)
        for (uint32_t k = 0; k < n; k++) {
            float t = 0.0f;
            if (cudaEventElapsedTime(&t, ctx->ev[0], Bt.ev[pl.lastWave[k]]) != cudaSuccess) {
                cudaGetLastError();
                return ctx->fail(PT_E_CUDA, "batch request timing");
            }
            request_ms[pl.order[k]] = t;
        }
    if (stats) {
        unsigned long long tot[2];
        memcpy(tot, hostCnt + 4, sizeof(tot));
        memset(stats, 0, sizeof(*stats));
        stats->paths = pl.total;
        stats->extension_rays = tot[0];
        stats->shadow_rays = tot[1];
        stats->waves = pl.waveStart.size();
        uint64_t bounces = 0;
        for (uint32_t d : pl.waveDepth) bounces += d;
        stats->bounces = bounces;
        stats->launches = Bt.launches;
        stats->ms_total = ms;
        memcpy(&stats->tail_extension_rays, hostCnt + kCntTailRays, 8);
    }
    return PT_OK;
}
}  // namespace

extern "C" int pt_render_batch(pt_ctx *ctx, const pt_request *requests, uint32_t n, float *request_ms,
                               pt_stats *stats) {
    if (!ctx) return PT_E_INVALID;
    if (!requests) return ctx->fail(PT_E_INVALID, "null requests");
    if (!ctx->hasScene) return ctx->fail(PT_E_NOSCENE, "no scene uploaded");
    return render_batch(ctx, requests, n, request_ms, stats, 0, 0.0f, nullptr, nullptr);
}

extern "C" int pt_batch_autotune(pt_ctx *ctx, const pt_request *requests, uint32_t n, pt_batch_tuning *out) {
    if (!ctx) return PT_E_INVALID;
    if (!requests || !out) return ctx->fail(PT_E_INVALID, "null argument");
    if (!ctx->hasScene) return ctx->fail(PT_E_NOSCENE, "no scene uploaded");
    int rc = batch_check(ctx, requests, n);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    uint64_t total = 0, maxPix = 0;
    for (uint32_t i = 0; i < n; i++) {
        total += (uint64_t)requests[i].params.width * requests[i].params.height * requests[i].params.spp;
        maxPix = std::max<uint64_t>(maxPix, (uint64_t)requests[i].params.width * requests[i].params.height);
    }
    float *film = nullptr;
    if (cudaMalloc(&film, maxPix * 32) != cudaSuccess) return ctx->fail(PT_E_NOMEM, "tuning film");
    // candidates: wave sizes from the whole batch down to 2^22 paths, full and half traversal grids
    std::vector<size_t> waves;
    for (uint64_t w = std::min<uint64_t>(total, kMaxWavePaths);; w >>= 1) {
        waves.push_back((size_t)w);
        if (w <= ((uint64_t)1 << 22) || waves.size() == 4) break;
    }
    const float grids[2] = {1.0f, 0.5f};
    memset(out, 0, sizeof(*out));
    float best = 1e30f;
    for (size_t w : waves)
        for (float g : grids) {
            float ms = 0.0f;
            for (int rep = 0; rep < 2 && rc == PT_OK; rep++)  // the first run captures the graph
                rc = render_batch(ctx, requests, n, nullptr, nullptr, w, g, film, &ms);
            if (rc) break;
            if (out->candidates < 16) {
                out->candidate_ms[out->candidates] = ms;
                out->candidate_wave[out->candidates] = (uint32_t)std::min<uint64_t>(w, total);
                out->candidate_grid[out->candidates] = g;
                out->candidates++;
            }
            if (ms < best) {
                best = ms;
                out->wave_paths = (uint32_t)std::min<uint64_t>(w, total);
                out->traversal_grid = g;
                out->ms = ms;
            }
        }
    cudaFree(film);
    if (rc) return rc;
    ctx->batch.tunedWave = out->wave_paths;
    ctx->batch.tunedGrid = out->traversal_grid;
    ctx->batch.tunedSceneGen = ctx->sceneGen;
    return PT_OK;
}
