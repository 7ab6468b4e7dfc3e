// pt_cache.cu — the radiance cache of libpt: a fully fused BF16 MLP on the
// sm_100a tensor cores (tcgen05.mma, operands in shared memory, FP32
// accumulators in tensor memory), its training step and Adam update, and the
// host entry points.  No counterpart in the reference.
//
// Kernel structure (one CTA = 128 threads = one 128-row tile per pass):
// * the BF16 weight image (43 KB) is placed in shared memory by one bulk
//   copy per CTA and stays there for all of the CTA's tiles;
// * each thread encodes one row (query);
// * per layer one thread issues 4 MMAs (K = 64 in steps of 16) into TMEM
//   and commits them to an mbarrier; the 4 warps read their 32 TMEM lanes
//   back (tcgen05.ld) and apply ReLU;
// * inference writes each layer's BF16 input to tensor memory (tcgen05.st)
//   and reads A from there, so only the weights are read from shared memory;
// * training keeps all six activation tiles in shared memory, runs the
//   backward pass with the same MMAs on transposed views of the same images
//   (K-major for dZ.W, MN-major for dZ^T.A), accumulates the weight
//   gradients in TMEM across the CTA's tiles and stores the sum in the CTA's
//   own slot, which a reduce kernel adds in slot order.
// Every mbarrier wait is bounded; a timeout raises an error flag and the CTA
// frees its tensor memory and returns.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>

#include "pt_cache.cuh"
#include "pt_internal.h"

namespace pt {

constexpr int kRcThreads = 128;
constexpr uint32_t kTileBytes = kRcTile * kRcIn * 2;  // 16 KB: one 128 x 64 BF16 tile
constexpr uint32_t kGradBytes = 2 * kTileBytes;       // dZ tiles carry a zero upper half (M = 128 views)
constexpr uint32_t kTrainSmem = kRcImageBytes + 6 * kTileBytes + 2 * kGradBytes + 64;
static_assert(kTrainSmem <= 227 * 1024, "training kernel shared memory");
constexpr uint32_t kDevErrCache = PT_DEVERR_CACHE;

struct RcNet {
    const uint8_t *img;  // BF16 weight image
    float bmin[3], binv[3];
    uint32_t *err;
    uint32_t stallPolls;  // test hook: polls of the up-front stall (0 = none)
};

// Input of one row: a record (encoded here) or a ready feature vector.
template <int SRC>
struct RcRows;
template <>
struct RcRows<0> {  // features n x 64, targets n x 3 (training)
    const float *feat, *targ;
    uint32_t n;
    __device__ uint32_t count() const { return n; }
    __device__ void load(const RcNet &, uint32_t row, float f[kRcIn]) const {
        const float4 *p = reinterpret_cast<const float4 *>(feat + (size_t)row * kRcIn);
#pragma unroll
        for (int k = 0; k < kRcIn / 4; k++) {
            float4 v = p[k];
            f[4 * k] = v.x; f[4 * k + 1] = v.y; f[4 * k + 2] = v.z; f[4 * k + 3] = v.w;
        }
    }
    __device__ float3 target(uint32_t row) const {
        return make_float3(targ[3 * row], targ[3 * row + 1], targ[3 * row + 2]);
    }
    // a row's inputs in flight: fetch issues the loads, decode uses them
    struct Raw {
        float4 v[kRcIn / 4];
        float3 tg;
    };
    __device__ void fetch(uint32_t row, bool withTarget, Raw &r) const {
        const float4 *p = reinterpret_cast<const float4 *>(feat + (size_t)row * kRcIn);
#pragma unroll
        for (int k = 0; k < kRcIn / 4; k++) r.v[k] = __ldcs(p + k);
        if (withTarget) r.tg = target(row);
    }
    __device__ void decode(const RcNet &, const Raw &r, float f[kRcIn]) const {
#pragma unroll
        for (int k = 0; k < kRcIn / 4; k++) {
            f[4 * k] = r.v[k].x; f[4 * k + 1] = r.v[k].y; f[4 * k + 2] = r.v[k].z; f[4 * k + 3] = r.v[k].w;
        }
    }
};
template <>
struct RcRows<1> {  // records (render queries or training records): rows phase, phase + stride, ...
    const float4 *r0, *r1, *r2, *r3, *tgt;
    const uint32_t *cnt;
    uint32_t cap;
    uint32_t stride = 1, phase = 0;
    __device__ uint32_t total() const { return min(*(volatile const uint32_t *)cnt, cap); }
    __device__ uint32_t count() const {
        uint32_t n = total();
        return n > phase ? (n - phase + stride - 1) / stride : 0u;
    }
    __device__ void load(const RcNet &N, uint32_t row, float f[kRcIn]) const {
        const uint32_t i = row * stride + phase;
        rc_encode(r0[i], r1[i], r2[i], r3[i], N.bmin, N.binv, f);
    }
    __device__ float3 target(uint32_t row) const {
        float4 t = tgt[row * stride + phase];
        return make_float3(t.x, t.y, t.z);
    }
    struct Raw {
        float4 q[4];
        float3 tg;
    };
    __device__ void fetch(uint32_t row, bool withTarget, Raw &r) const {
        const uint32_t i = row * stride + phase;
        r.q[0] = r0[i]; r.q[1] = r1[i]; r.q[2] = r2[i]; r.q[3] = r3[i];
        if (withTarget) r.tg = target(row);
    }
    __device__ void decode(const RcNet &N, const Raw &r, float f[kRcIn]) const {
        rc_encode(r.q[0], r.q[1], r.q[2], r.q[3], N.bmin, N.binv, f);
    }
};

// ---- weight staging and TMEM set-up shared by the kernels -------------------
struct CtaCtl {
    uint32_t mbW, mbM, tbase, td, tl;  // td: the accumulator (lane 0), tl: this warp's lanes of TMEM
    uint32_t phase;
    bool ok;
    bool copyIssued, mmaPending;  // what an error exit still has to wait for
};
__device__ __forceinline__ void rc_setup(CtaCtl &c, uint8_t *W, uint64_t *bars, uint32_t *tslot, const uint8_t *img,
                                         uint32_t cols, uint32_t stallPolls) {
    const uint32_t t = threadIdx.x, warp = t >> 5;
    c.mbW = smem_u32(bars);
    c.mbM = smem_u32(bars + 1);
    if (t == 0) {
        mbar_init(c.mbW, 1);
        mbar_init(c.mbM, 1);
        mbar_fence_init();
    }
    __syncthreads();
    // Test hook: a wait that runs out.  Nothing arrives at mbM before an MMA
    // is committed to it, so with no copy or MMA issued yet every thread gives
    // up after stallPolls polls and the CTA takes the error exit below.
    bool ok = true;
    if (stallPolls) ok = __syncthreads_and(mbar_wait(c.mbM, 0, stallPolls)) != 0;
    if (ok && t == 0) {
        mbar_expect_tx(c.mbW, kRcImageBytes);
        bulk_g2s(smem_u32(W), img, kRcImageBytes, c.mbW);
    }
    c.copyIssued = ok;
    c.mmaPending = false;
    __syncwarp();
    if (warp == 0) tmem_alloc(smem_u32(tslot), cols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    c.tbase = *tslot;
    c.td = c.tbase;
    c.tl = c.tbase + ((warp * 32u) << 16);
    c.phase = 0;
    c.ok = ok && __syncthreads_and(mbar_wait(c.mbW, 0)) != 0;  // ok is uniform across the CTA
}
// Wait for the MMAs committed to mbM; uniform across the CTA.
__device__ __forceinline__ bool rc_wait_mma(CtaCtl &c) {
    bool done = mbar_wait(c.mbM, c.phase);
    bool all = __syncthreads_and(done) != 0;
    if (all) c.phase ^= 1u;
    else c.mmaPending = true;
    tc_fence_after();
    return all;
}
__device__ __forceinline__ void rc_teardown(CtaCtl &c, uint32_t cols, uint32_t *err) {
    if (!c.ok) {
        if (threadIdx.x == 0) atomicOr(err, kDevErrCache);
        if (c.copyIssued) mbar_wait(c.mbW, 0, 1u << 20);          // the weight copy, if still in flight
        if (c.mmaPending) mbar_wait(c.mbM, c.phase, 1u << 20);  // MMAs of the wait that gave up
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if ((threadIdx.x >> 5) == 0) tmem_free(c.tbase, cols);
}
// Forward MMAs of layer l: D[0:N) = A (128 x 64) . W_l^T.
__device__ __forceinline__ void rc_issue_forward(const CtaCtl &c, const uint8_t *A, const uint8_t *W, int l) {
    const uint32_t N = rc_rows(l);
    tc_fence_after();
    const uint32_t idesc = umma_idesc(128, N, 0, 0);
#pragma unroll
    for (int s = 0; s < 4; s++) {
        uint64_t ad = umma_desc(smem_u32(A) + s * 2 * (kRcTile * 16), kRcTile * 16, 128);
        uint64_t bd = umma_desc(smem_u32(W) + rc_image_base(l) + s * 2 * (N * 16), N * 16, 128);
        umma_bf16(c.td, ad, bd, idesc, s > 0 ? 1u : 0u);
    }
    umma_commit(c.mbM);
}

// ---- inference: features / render queries -> radiance ------------------------
// MODE 0: rows from a feature array, outputs to out[n x 3].
// MODE 1: rows from render queries; lo_eta[slot] += weight * max(y, 0).
struct RcInferArgs {
    RcNet net;
    RcRows<0> feat;
    RcRows<1> qry;
    const float4 *qw;  // per query: throughput weight
    float *out;
    float4 *lo_eta;
    float4 *recCache;  // cache value at training-record vertices (queries tagged with bit 31)
};
// the row source of each mode: feature arrays (batch entry points) or records
template <int MODE>
__device__ __forceinline__ const auto &infer_rows(const RcInferArgs &a) {
    if constexpr (MODE == 0) return a.feat;
    else return a.qry;
}
// Inference keeps each layer's input in tensor memory: the epilogue reads the
// FP32 accumulator (TMEM columns [0, 64)), applies ReLU, rounds to BF16 and
// writes the packed pairs to columns [64, 96) with tcgen05.st, and the next
// layer's MMAs read A from there (only the weights come from shared memory).
// No activation tile in shared memory: a CTA holds the 43 KB weight image and
// 128 TMEM columns.  CTAs per SM (measured): 3 for feature arrays, whose
// 256-byte rows are prefetched in registers, 4 for render queries.
template <int MODE>
constexpr uint32_t kRcInferCtasPerSm = MODE == 0 ? 3u : 4u;
constexpr uint32_t kRcInferCols = 128;
constexpr uint32_t kRcInferA = 64;  // first TMEM column of the layer input
constexpr uint32_t kInferSmem = kRcImageBytes + 64;  // + mbarriers, TMEM slot
static_assert(4 * (kInferSmem + 1024) <= 228 * 1024, "inference CTAs per SM: shared memory");
static_assert(4 * kRcInferCols <= 512, "inference CTAs per SM: tensor memory");

// Forward MMAs of layer l with A in tensor memory: D[0:N) = A . W_l^T.
__device__ __forceinline__ void rc_issue_forward_ts(const CtaCtl &c, const uint8_t *W, int l) {
    const uint32_t N = rc_rows(l);
    tc_fence_after();
    const uint32_t idesc = umma_idesc(128, N, 0, 0);
#pragma unroll
    for (int s = 0; s < 4; s++) {
        uint64_t bd = umma_desc(smem_u32(W) + rc_image_base(l) + s * 2 * (N * 16), N * 16, 128);
        umma_bf16_ts(c.td, c.tbase + kRcInferA + 8 * s, bd, idesc, s > 0 ? 1u : 0u);
    }
    umma_commit(c.mbM);
}

template <int MODE>
__global__ void __launch_bounds__(kRcThreads, kRcInferCtasPerSm<MODE>) k_rc_infer(RcInferArgs a) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t *W = sm;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + kRcImageBytes);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2);
    const uint32_t t = threadIdx.x;
    const uint32_t n = MODE == 0 ? a.feat.count() : a.qry.count();
    const uint32_t ntiles = (n + kRcTile - 1) / kRcTile;
    if (blockIdx.x >= ntiles) return;  // uniform: before any set-up
    CtaCtl c;
    // each tile's inputs are loaded while the tile before it runs its layers:
    // the first here, the next one right after a tile decodes its own
    const auto &rows = infer_rows<MODE>(a);
    typename std::remove_reference_t<decltype(rows)>::Raw raw;
    if (blockIdx.x * kRcTile + t < n) rows.fetch(blockIdx.x * kRcTile + t, false, raw);
    rc_setup(c, W, bars, tslot, a.net.img, kRcInferCols, a.net.stallPolls);
    const uint32_t aIn = c.tl + kRcInferA;  // this warp's lanes of the layer input
    for (uint32_t tile = blockIdx.x; tile < ntiles && c.ok; tile += gridDim.x) {
        const uint32_t row = tile * kRcTile + t;
        const bool valid = row < n;
        {
            float f[kRcIn];
            if (valid) {
                rows.decode(a.net, raw, f);
            } else {
#pragma unroll
                for (int k = 0; k < kRcIn; k++) f[k] = 0.0f;
            }
            uint32_t pk[32];
#pragma unroll
            for (int k = 0; k < 32; k++) pk[k] = pack_bf16(f[2 * k], f[2 * k + 1]);
            tmem_st32(aIn, pk);
        }
        // render queries: what the last step reads, requested now
        uint32_t tag = 0;
        float4 qw = make_float4(0.0f, 0.0f, 0.0f, 0.0f), le = qw;
        if constexpr (MODE != 0) {
            if (valid) {
                tag = __float_as_uint(raw.q[1].w);
                if (!(tag & 0x80000000u)) {
                    qw = a.qw[row];
                    le = a.lo_eta[tag];
                }
            }
        }
        {
            const uint32_t nrow = row + gridDim.x * kRcTile;
            if (nrow < n) rows.fetch(nrow, false, raw);
        }
        tmem_wait_st();
        tc_fence_before();
        __syncthreads();
        for (int l = 0; l < kRcLayers && c.ok; l++) {
            if (t == 0) rc_issue_forward_ts(c, W, l);
            if (!(c.ok = rc_wait_mma(c))) break;
            if (l < kRcLayers - 1) {
                float v[64];
                tmem_ld32(c.tl, v);
                tmem_ld32(c.tl + 32, v + 32);
                tmem_wait_ld();
                uint32_t pk[32];
#pragma unroll
                for (int k = 0; k < 32; k++) pk[k] = pack_bf16_relu(v[2 * k], v[2 * k + 1]);
                tmem_st32(aIn, pk);
                tmem_wait_st();
            } else {
                float v[16];
                tmem_ld16(c.tl, v);
                tmem_wait_ld();
                if (valid) {
                    if (MODE == 0) {
                        a.out[3 * (size_t)row] = v[0];
                        a.out[3 * (size_t)row + 1] = v[1];
                        a.out[3 * (size_t)row + 2] = v[2];
                    } else {
                        if (tag & 0x80000000u) {  // a training record's vertex: keep the value
                            a.recCache[tag & 0x7FFFFFFFu] =
                                make_float4(fmaxf(v[0], 0.0f), fmaxf(v[1], 0.0f), fmaxf(v[2], 0.0f), 0.0f);
                        } else {
                            // Lo += throughput * cache, rounded as two operations (no FMA)
                            le.x = __fadd_rn(le.x, __fmul_rn(qw.x, fmaxf(v[0], 0.0f)));
                            le.y = __fadd_rn(le.y, __fmul_rn(qw.y, fmaxf(v[1], 0.0f)));
                            le.z = __fadd_rn(le.z, __fmul_rn(qw.z, fmaxf(v[2], 0.0f)));
                            a.lo_eta[tag] = le;
                        }
                    }
                }
            }
            tc_fence_before();
            __syncthreads();
        }
    }
    rc_teardown(c, kRcInferCols, a.net.err);
}

// ---- training: forward, relative L2 loss, backward, weight gradients ---------
struct RcTrainArgs {
    RcNet net;
    RcRows<0> feat;
    RcRows<1> rec;
    float *part;     // per CTA, kRcParams FP32: the CTA's summed gradient (overwritten; zeros from a CTA
                     // that trained nothing); k_rc_grad_reduce adds the slots in order
    float *lossSum;  // added to
};
template <int MODE>
__device__ __forceinline__ const auto &train_rows(const RcTrainArgs &a) {
    if constexpr (MODE == 0) return a.feat;
    else return a.rec;
}
// TMEM columns: [0, 64) layer output / input gradient, [64 + 64 l, 128 + 64 l)
// the weight gradient of layer l.
template <int MODE>
__global__ void __launch_bounds__(kRcThreads, 1) k_rc_train(RcTrainArgs a) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t *W = sm;
    uint8_t *Act = sm + kRcImageBytes;                     // 6 tiles: A_0 (input) .. A_5
    uint8_t *dZo = Act + 6 * kTileBytes;                   // output-layer gradient (16 columns used)
    uint8_t *dZ = dZo + kGradBytes;                        // hidden-layer gradient
    uint64_t *bars = reinterpret_cast<uint64_t *>(dZ + kGradBytes);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 2);
    const uint32_t t = threadIdx.x;
    const uint32_t n = MODE == 0 ? a.feat.count() : a.rec.count();
    const uint32_t ntiles = (n + kRcTile - 1) / kRcTile;
    float4 *slot = reinterpret_cast<float4 *>(a.part + (size_t)blockIdx.x * kRcParams);
    if (blockIdx.x >= ntiles) {  // nothing to train: an empty slot
        for (uint32_t i = t; i < kRcParams / 4; i += kRcThreads) slot[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    // the dZ images are read as M = 128 operands: their upper halves (and the
    // unused columns of dZo) must hold zeros
    for (uint32_t i = t; i < 2 * kGradBytes / 16; i += kRcThreads)
        reinterpret_cast<uint4 *>(dZo)[i] = make_uint4(0, 0, 0, 0);
    fence_async_smem();
    CtaCtl c;
    // the next tile's inputs load while this tile runs forward and backward
    const auto &rows = train_rows<MODE>(a);
    typename std::remove_reference_t<decltype(rows)>::Raw raw;
    if (blockIdx.x * kRcTile + t < n) rows.fetch(blockIdx.x * kRcTile + t, true, raw);
    rc_setup(c, W, bars, tslot, a.net.img, 512, a.net.stallPolls);
    float loss = 0.0f;
    bool first = true;
    for (uint32_t tile = blockIdx.x; tile < ntiles && c.ok; tile += gridDim.x) {
        const uint32_t row = tile * kRcTile + t;
        const bool valid = row < n;
        float f[kRcIn];
        float3 tg = make_float3(0.0f, 0.0f, 0.0f);
        if (valid) {
            rows.decode(a.net, raw, f);
            tg = raw.tg;
        } else {
#pragma unroll
            for (int k = 0; k < kRcIn; k++) f[k] = 0.0f;
        }
        {
            const uint32_t nrow = row + gridDim.x * kRcTile;
            if (nrow < n) rows.fetch(nrow, true, raw);
        }
        store_row_bf16(Act, t, f);
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        // forward
        for (int l = 0; l < kRcLayers && c.ok; l++) {
            if (t == 0) rc_issue_forward(c, Act + l * kTileBytes, W, l);
            if (!(c.ok = rc_wait_mma(c))) break;
            if (l < kRcLayers - 1) {
                float v[64];
                tmem_ld64(c.tl, v);
                tmem_wait_ld();
#pragma unroll
                for (int k = 0; k < 64; k++) v[k] = fmaxf(v[k], 0.0f);
                store_row_bf16(Act + (l + 1) * kTileBytes, t, v);
            } else {
                float v[16];
                tmem_ld16(c.tl, v);
                tmem_wait_ld();
                const float y[3] = {v[0], v[1], v[2]}, tt[3] = {tg.x, tg.y, tg.z};
                float g[16];
#pragma unroll
                for (int k = 0; k < 16; k++) g[k] = 0.0f;
                if (valid) {
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        float d = y[k] - tt[k], den = y[k] * y[k] + 0.01f;
                        loss += d * d / den;
                        g[k] = 2.0f * d / den;
                    }
                }
                uint4 w0 = make_uint4(pack_bf16(g[0], g[1]), pack_bf16(g[2], g[3]), pack_bf16(g[4], g[5]),
                                      pack_bf16(g[6], g[7]));
                uint4 w1 = make_uint4(pack_bf16(g[8], g[9]), pack_bf16(g[10], g[11]), pack_bf16(g[12], g[13]),
                                      pack_bf16(g[14], g[15]));
                *reinterpret_cast<uint4 *>(dZo + rc_core_offset(t, 0, kRcTile)) = w0;
                *reinterpret_cast<uint4 *>(dZo + rc_core_offset(t, 8, kRcTile)) = w1;
            }
            fence_async_smem();
            tc_fence_before();
            __syncthreads();
        }
        // backward: layer l consumes dZ_l (dZo for the output layer)
        for (int l = kRcLayers - 1; l >= 0 && c.ok; l--) {
            const uint8_t *G = l == kRcLayers - 1 ? dZo : dZ;
            const uint32_t Kout = rc_rows(l);
            if (t == 0) {
                tc_fence_after();
                // dW_l += dZ_l^T . A_l : M = 128 (rows = out, zero above Kout), N = 64, K = 128 (batch)
                const uint32_t idw = umma_idesc(128, 64, 1, 1);
#pragma unroll
                for (int s = 0; s < 8; s++) {
                    uint64_t ad = umma_desc(smem_u32(G) + s * 256, 128, kRcTile * 16);
                    uint64_t bd = umma_desc(smem_u32(Act + l * kTileBytes) + s * 256, 128, kRcTile * 16);
                    umma_bf16(c.tbase + 64 + 64 * l, ad, bd, idw, (first && s == 0) ? 0u : 1u);
                }
                if (l > 0) {
                    // dA_l = dZ_l . W_l : M = 128 (batch), N = 64 (in), K = Kout
                    const uint32_t ida = umma_idesc(128, 64, 0, 1);
                    for (uint32_t s = 0; s < Kout / 16; s++) {
                        uint64_t ad = umma_desc(smem_u32(G) + s * 2 * (kRcTile * 16), kRcTile * 16, 128);
                        uint64_t bd = umma_desc(smem_u32(W) + rc_image_base(l) + s * 256, 128, Kout * 16);
                        umma_bf16(c.tbase, ad, bd, ida, s > 0 ? 1u : 0u);
                    }
                }
                umma_commit(c.mbM);
            }
            if (!(c.ok = rc_wait_mma(c))) break;
            if (l > 0) {  // dZ_{l-1} = dA_l (x) [A_l > 0]
                float v[64], act[64];
                tmem_ld64(c.tl, v);
                tmem_wait_ld();
                load_row_bf16(Act + l * kTileBytes, t, act);
#pragma unroll
                for (int k = 0; k < 64; k++) v[k] = act[k] > 0.0f ? v[k] : 0.0f;
                store_row_bf16(dZ, t, v);
                fence_async_smem();
            }
            tc_fence_before();
            __syncthreads();
        }
        first = false;
    }
    // the CTA's weight gradients into its slot: thread t holds row t (an
    // output unit) of each layer, 64 consecutive parameters; plain stores, the
    // slots are summed afterwards in a fixed order (no float atomics)
    if (c.ok && !first) {
        tc_fence_after();
        for (int l = 0; l < kRcLayers; l++) {
            float v[64];
            tmem_ld64(c.tl + 64 + 64 * l, v);
            tmem_wait_ld();
            if (t < (uint32_t)rc_rows(l)) {
                float4 *g = slot + (rc_param_base(l) + t * kRcIn) / 4;
#pragma unroll
                for (int k = 0; k < 16; k++) g[k] = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
            }
        }
    } else {  // a wait gave up (the call reports it): leave nothing in the slot
        for (uint32_t i = t; i < kRcParams / 4; i += kRcThreads) slot[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xFFFFFFFFu, loss, o);
    if ((t & 31) == 0 && c.ok) atomicAdd(a.lossSum, loss);
    rc_teardown(c, 512, a.net.err);
}

// The training CTAs' gradient slots summed in slot order (deterministic), added to grad.
__global__ void __launch_bounds__(256) k_rc_grad_reduce(const float *part, uint32_t slots, float *grad) {
    const uint32_t p = blockIdx.x * 256u + threadIdx.x;
    if (p >= kRcParams) return;
    float s = 0.0f;
    for (uint32_t k = 0; k < slots; k++) s += __ldcs(part + (size_t)k * kRcParams + p);
    grad[p] += s;
}
constexpr uint32_t kReduceBlocks = (kRcParams + 255) / 256;

// ---- Adam (one CTA): FP32 master weights -> BF16 images ------------------------
struct RcAdamArgs {
    float *w, *m, *v, *ema, *grad;
    uint8_t *imgTrain, *imgInfer;
    uint32_t *ctr;           // [0] steps (read, incremented), [4] records of the step (written)
    const uint32_t *nrec;    // records of the call; this step's gradient sums over rows phase + k stride
    uint32_t nrecCap;     // capacity of the record buffers
    uint32_t nrecTarget;  // records a render call aims at (train_records)
    uint32_t stride, phase;
    float lr, emaDecay;
    float *lossSum;          // mean loss of the step -> ctr[3] as float bits; reset
    uint32_t updateProb;     // last step of a render call: set ctr[7] for the next call
    float maxFrac;           // upper bound of ctr[7]
};
__device__ __forceinline__ void put_bf16(uint8_t *img, int i, float x) {
    int l = i < rc_param_base(5) ? i / (kRcWidth * kRcIn) : 5;
    int j = i - rc_param_base(l);
    int o = j / kRcIn, in = j % kRcIn;
    *reinterpret_cast<__nv_bfloat16 *>(img + rc_image_base(l) + rc_core_offset(o, in, rc_rows(l))) =
        __float2bfloat16_rn(x);
}
// One parameter's Adam update from its gradient sum over n records (3 outputs
// each): FP32 master weight, moments and inference average, then both BF16
// images.
__device__ __forceinline__ void rc_adam_param(const RcAdamArgs &a, int i, float gradSum, uint32_t n,
                                              uint32_t step) {
    const float b1 = 0.9f, b2 = 0.99f, eps = 1e-8f;
    const float gs = 1.0f / (3.0f * (float)n);
    const float bc1 = 1.0f - powf(b1, (float)step), bc2 = 1.0f - powf(b2, (float)step);
    float g = gradSum * gs;
    if (!isfinite(g)) g = 0.0f;
    float m = b1 * a.m[i] + (1.0f - b1) * g;
    float v = b2 * a.v[i] + (1.0f - b2) * g * g;
    a.m[i] = m;
    a.v[i] = v;
    float w = a.w[i] - a.lr * (m / bc1) / (sqrtf(v / bc2) + eps);
    a.w[i] = w;
    float e = (step == 1u || a.emaDecay == 0.0f) ? w : a.emaDecay * a.ema[i] + (1.0f - a.emaDecay) * w;
    a.ema[i] = e;
    put_bf16(a.imgTrain, i, w);
    put_bf16(a.imgInfer, i, e);
}
__global__ void __launch_bounds__(1024) k_rc_adam(RcAdamArgs a) {
    __shared__ uint32_t sStep, sN;
    if (threadIdx.x == 0) {
        sStep = a.ctr[0] + 1u;
        uint32_t tot = min(*a.nrec, a.nrecCap);
        sN = tot > a.phase ? (tot - a.phase + a.stride - 1) / a.stride : 0u;
        if (a.updateProb) {
            // training chance of the next call: about nrecTarget records out
            // of this call's cache vertices (queries + records)
            float verts = (float)a.ctr[5];  // every cache vertex made a query (training ones too)
            reinterpret_cast<float *>(a.ctr)[7] =
                verts > 0.0f ? fminf(a.maxFrac, (float)a.nrecTarget / verts) : a.maxFrac;
        }
    }
    __syncthreads();
    const uint32_t n = sN, step = sStep;
    if (n == 0) return;
    for (int i = threadIdx.x; i < kRcParams; i += blockDim.x) {
        const float g = a.grad[i];
        a.grad[i] = 0.0f;
        rc_adam_param(a, i, g, n, step);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        a.ctr[0] = step;
        a.ctr[4] = n;
        a.ctr[3] = __float_as_uint(*a.lossSum / (3.0f * (float)n));
        *a.lossSum = 0.0f;
    }
}

// A render call's training step, second half: the CTAs' gradient slots
// summed in slot order (the same sums as k_rc_grad_reduce) and the Adam
// update of k_rc_adam, one thread per parameter over the whole GPU.  Every
// CTA reads the step counter first; the last CTA to finish (a ticket in
// ctr[11]) writes the step's counters and, on the call's last step, the
// next call's training chance.
__global__ void __launch_bounds__(256) k_rc_adam_slots(RcAdamArgs a, const float *part, uint32_t slots) {
    const uint32_t step = a.ctr[0] + 1u;
    const uint32_t tot = min(*a.nrec, a.nrecCap);
    const uint32_t n = tot > a.phase ? (tot - a.phase + a.stride - 1) / a.stride : 0u;
    auto updateProb = [&]() {
        // training chance of the next call: about nrecTarget records out of
        // this call's cache vertices (queries + records)
        float verts = (float)a.ctr[5];  // every cache vertex made a query (training ones too)
        reinterpret_cast<float *>(a.ctr)[7] = verts > 0.0f ? fminf(a.maxFrac, (float)a.nrecTarget / verts) : a.maxFrac;
    };
    if (n == 0) {  // no records in this step: no update
        if (a.updateProb && blockIdx.x == 0 && threadIdx.x == 0) updateProb();
        return;
    }
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kRcParams) {
        float sum = 0.0f;
        for (uint32_t k = 0; k < slots; k++) sum += __ldcs(part + (size_t)k * kRcParams + i);
        rc_adam_param(a, (int)i, sum, n, step);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(a.ctr + 11, 1u) == gridDim.x - 1) {  // every CTA has read ctr[0]
            a.ctr[11] = 0u;
            a.ctr[0] = step;
            a.ctr[4] = n;
            a.ctr[3] = __float_as_uint(*a.lossSum / (3.0f * (float)n));
            *a.lossSum = 0.0f;
            if (a.updateProb) updateProb();
        }
    }
}

__global__ void k_rc_set_chance(float *chance, float p) { *chance = p; }

// Images from the FP32 weights (initialisation, pt_cache_weights).
__global__ void k_rc_images(const float *w, uint8_t *imgTrain, uint8_t *imgInfer, float *ema) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kRcParams; i += gridDim.x * blockDim.x) {
        ema[i] = w[i];
        put_bf16(imgTrain, i, w[i]);
        put_bf16(imgInfer, i, w[i]);
    }
}

// Training targets of the records written in this wave: the radiance the
// path gathered after its record vertex, divided by the throughput there.
// Records [ctr[6], count) belong to the wave that just ended (ctr[6] moves
// on in k_rc_ord_scan, after every kernel that reads it here).  The training
// path then takes the value a terminated path would have there, prefix +
// throughput x cache (lo_eta), with its pending NEE dropped.
__global__ void __launch_bounds__(256) k_rc_targets(RcRows<1> rec, float4 *beta, float4 *lo0, float4 *tgt,
                                                   const float4 *recCache, const uint32_t *ctr, float4 *lo_eta,
                                                   uint4 *rng, const float4 *pendA, const float4 *pendE) {
    const uint32_t s0 = ctr[6], s1 = rec.total();
    for (uint32_t r = s0 + blockIdx.x * blockDim.x + threadIdx.x; r < s1; r += gridDim.x * blockDim.x) {
        uint32_t slot = __float_as_uint(rec.r1[r].w);
        float4 le = lo_eta[slot];
        float L[3] = {le.x, le.y, le.z};
        if (rng[slot].w & 1u) {  // NEE of the last bounce, folded in as the film does
            float4 pa = pendA[slot], pe = pendE[slot];
            L[0] += pa.x; L[1] += pa.y; L[2] += pa.z;
            L[0] += pe.x; L[1] += pe.y; L[2] += pe.z;
        }
        float4 b = beta[r], l0 = lo0[r];
        const float bb[3] = {b.x, b.y, b.z}, ll[3] = {l0.x, l0.y, l0.z};
        float o[3];
        for (int k = 0; k < 3; k++) {
            float x = bb[k] > 1e-8f ? (L[k] - ll[k]) / bb[k] : 0.0f;
            o[k] = isfinite(x) ? fmaxf(x, 0.0f) : 0.0f;
        }
        tgt[r] = make_float4(o[0], o[1], o[2], 0.0f);
        const float4 cv = recCache[r];
        lo_eta[slot] = make_float4(__fadd_rn(l0.x, __fmul_rn(b.x, cv.x)), __fadd_rn(l0.y, __fmul_rn(b.y, cv.y)),
                                   __fadd_rn(l0.z, __fmul_rn(b.z, cv.z)), fabsf(le.w));  // nothing pending now
        uint4 st = rng[slot];
        st.w &= ~1u;
        rng[slot] = st;
    }
}

// ---- the records of a wave in a fixed order ------------------------------------
// Records are appended by the shading kernels in whatever order their warps
// run, and an Adam step's batch and its gradient sums follow record order.
// Each wave's records are therefore put in the order of their key (rec[2].w:
// sample x pixels + pixel position, from the wave's first sample group; a
// path leaves at most one record per wave, so keys are distinct, and they do
// not depend on the order in which the wave runs its paths): counted into
// kRcOrdBuckets buckets of consecutive keys, scanned, scattered with their
// keys, and each record placed at its bucket's offset plus its rank by key
// among the bucket's few records; the training inputs and targets are copied
// to recOrd there.  Training reads recOrd, and cached renders repeat bit for
// bit.  The wave's records are [ctr[6], count) until k_rc_ord_scan records
// that range in ctr[9], ctr[10] and moves ctr[6] on.
constexpr uint32_t kRcOrdBuckets = 4096;
__device__ __forceinline__ uint32_t rc_ord_key(const float4 *r2, uint32_t r) {
    return __float_as_uint(__ldg(reinterpret_cast<const float *>(r2 + r) + 3));
}
__device__ __forceinline__ uint32_t rc_ord_bucket(uint32_t key, uint32_t keyRange) {
    // keys lie below keyRange; the clamp keeps any other value in bounds
    return min((uint32_t)(((uint64_t)key * kRcOrdBuckets) / max(keyRange, 1u)), kRcOrdBuckets - 1u);
}
__global__ void __launch_bounds__(256) k_rc_ord_count(RcRows<1> rec, const uint32_t *ctr, uint32_t keyRange,
                                                      uint32_t *cnt) {
    const uint32_t s0 = ctr[6], s1 = rec.total();
    for (uint32_t r = s0 + blockIdx.x * blockDim.x + threadIdx.x; r < s1; r += gridDim.x * blockDim.x)
        atomicAdd(cnt + rc_ord_bucket(rc_ord_key(rec.r2, r), keyRange), 1u);
}
// One block: exclusive scan of the bucket counts into off (kRcOrdBuckets + 1
// entries) and the scatter cursors; then the wave's record range moves to
// ctr[9], ctr[10], ctr[6] to its end, and the wave's queries join the call's.
__global__ void __launch_bounds__(1024) k_rc_ord_scan(RcRows<1> rec, const uint32_t *cnt, uint32_t *off,
                                                      uint32_t *cur, uint32_t *ctr) {
    constexpr uint32_t kPer = kRcOrdBuckets / 1024;
    __shared__ uint32_t part[1024];
    const uint32_t t = threadIdx.x;
    uint32_t c[kPer], sum = 0;
#pragma unroll
    for (uint32_t k = 0; k < kPer; k++) {
        c[k] = cnt[kPer * t + k];
        sum += c[k];
    }
    part[t] = sum;
    __syncthreads();
    for (uint32_t o = 1; o < 1024; o <<= 1) {
        const uint32_t v = t >= o ? part[t - o] : 0u;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    uint32_t base = part[t] - sum;
#pragma unroll
    for (uint32_t k = 0; k < kPer; k++) {
        off[kPer * t + k] = base;
        cur[kPer * t + k] = base;
        base += c[k];
    }
    if (t == 1023) off[kRcOrdBuckets] = part[1023];
    if (t == 0) {
        const uint32_t s0 = ctr[6], s1 = rec.total();
        ctr[9] = s0;
        ctr[10] = s1;
        ctr[6] = s1;
        ctr[5] += ctr[1];
    }
}
// Record indices and their keys into bucket order (order within a bucket:
// whatever the atomics give; the place kernel ranks by key).
__global__ void __launch_bounds__(256) k_rc_ord_scatter(const float4 *r2, const uint32_t *ctr, uint32_t keyRange,
                                                        uint32_t *cur, uint2 *tmp) {
    const uint32_t s0 = ctr[9], s1 = ctr[10];
    for (uint32_t r = s0 + blockIdx.x * blockDim.x + threadIdx.x; r < s1; r += gridDim.x * blockDim.x) {
        const uint32_t key = rc_ord_key(r2, r);
        tmp[atomicAdd(cur + rc_ord_bucket(key, keyRange), 1u)] = make_uint2(r, key);
    }
}
struct RcOrdCopy {
    const float4 *src[5];  // inputs x 4, target
    float4 *dst[5];
};
// One thread per scattered record: its position is its bucket's offset plus
// the number of the bucket's records with a smaller key; the record's
// training inputs and target are copied to ctr[9] + that position.
__global__ void __launch_bounds__(256) k_rc_ord_place(RcOrdCopy a, const uint32_t *ctr, uint32_t keyRange,
                                                      const uint32_t *off, const uint2 *tmp) {
    const uint32_t s0 = ctr[9], n = ctr[10] - s0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint2 e = tmp[j];
        const uint32_t b = rc_ord_bucket(e.y, keyRange), lo = off[b], hi = off[b + 1];
        uint32_t rank = 0;
        for (uint32_t i = lo; i < hi; i++) rank += tmp[i].y < e.y ? 1u : 0u;
        const uint32_t d = s0 + lo + rank;
#pragma unroll
        for (int k = 0; k < 5; k++) a.dst[k][d] = a.src[k][e.x];
    }
}

__global__ void k_rc_encode(const float4 *rec, uint32_t n, float bx, float by, float bz, float ix, float iy, float iz,
                            float *feat) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float bmin[3] = {bx, by, bz}, binv[3] = {ix, iy, iz};
    float f[kRcIn];
    rc_encode(rec[4 * i], rec[4 * i + 1], rec[4 * i + 2], rec[4 * i + 3], bmin, binv, f);
    for (int k = 0; k < kRcIn; k++) feat[(size_t)i * kRcIn + k] = f[k];
}

}  // namespace pt

using namespace pt;

// ---- host side ------------------------------------------------------------------
namespace {
bool gRcAttr = false;
int rc_attrs(pt_ctx *ctx) {
    if (gRcAttr) return PT_OK;
    const void *fns[] = {(const void *)k_rc_infer<0>, (const void *)k_rc_infer<1>};
    for (const void *f : fns)
        if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, kInferSmem) != cudaSuccess)
            return ctx->fail(PT_E_CUDA, "cache kernel attributes");
    const void *tf[] = {(const void *)k_rc_train<0>, (const void *)k_rc_train<1>};
    for (const void *f : tf)
        if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, kTrainSmem) != cudaSuccess)
            return ctx->fail(PT_E_CUDA, "cache kernel attributes");
    gRcAttr = true;
    return PT_OK;
}
RcNet rc_net(const pt_ctx *ctx, const uint8_t *img) {
    RcNet n;
    n.img = img;
    for (int k = 0; k < 3; k++) {
        n.bmin[k] = ctx->cache.bmin[k];
        n.binv[k] = ctx->cache.binv[k];
    }
    n.err = ctx->d_err;
    n.stallPolls = ctx->dbgCacheStall;
    return n;
}
// Cache bounds: the parameters' box, else the scene's vertex bounds.
void rc_bounds(pt_ctx *ctx) {
    RadianceCache &C = ctx->cache;
    const pt_cache_params &P = C.params;
    bool own = P.bbox_max[0] > P.bbox_min[0] && P.bbox_max[1] > P.bbox_min[1] && P.bbox_max[2] > P.bbox_min[2];
    const float *lo = own ? P.bbox_min : ctx->sceneMin, *hi = own ? P.bbox_max : ctx->sceneMax;
    for (int k = 0; k < 3; k++) {
        float e = hi[k] - lo[k];
        C.bmin[k] = lo[k];
        C.binv[k] = e > 0.0f ? 1.0f / e : 1.0f;
    }
}
int rc_check(pt_ctx *ctx) {
    if (!ctx) return PT_E_INVALID;
    if (!ctx->cache.ready) return ctx->fail(PT_E_INVALID, "radiance cache not initialised (pt_cache_init)");
    cudaSetDevice(ctx->device);
    return rc_attrs(ctx);
}
int rc_device_error(pt_ctx *ctx) {
    uint32_t derr = 0;
    if (cudaMemcpy(&derr, ctx->d_err, 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return ctx->fail(PT_E_CUDA, "cache error flag");
    if (derr & kDevErrCache) {
        cudaMemset(ctx->d_err, 0, 4);
        return ctx->fail(PT_E_DEVICE, "radiance cache kernel: a tensor-core wait timed out");
    }
    return PT_OK;
}
unsigned rc_grid(const pt_ctx *ctx, uint32_t n, unsigned perSM) {
    unsigned tiles = (n + kRcTile - 1) / kRcTile;
    return std::max(1u, std::min(tiles, (unsigned)ctx->numSMs * perSM));
}
}  // namespace

// ---- launches of a cached render (stream-ordered, capturable) ------------------
cudaError_t rc_enqueue_resolve(pt_ctx *ctx, cudaStream_t st, float4 *lo_eta) {
    const RadianceCache &C = ctx->cache;
    RcInferArgs a{};
    a.net = rc_net(ctx, C.imgInfer);
    a.qry.r0 = C.q[0]; a.qry.r1 = C.q[1]; a.qry.r2 = C.q[2]; a.qry.r3 = C.q[3];
    a.qry.cnt = C.ctr + 1;
    a.qry.cap = (uint32_t)C.queryCap;
    a.qw = C.q[4];
    a.lo_eta = lo_eta;
    a.recCache = C.rec[7];
    k_rc_infer<1><<<ctx->numSMs * kRcInferCtasPerSm<1>, kRcThreads, kInferSmem, st>>>(a);
    return cudaGetLastError();
}
cudaError_t rc_enqueue_targets(pt_ctx *ctx, cudaStream_t st, float4 *lo_eta, uint4 *rng, const float4 *pendA,
                               const float4 *pendE, uint32_t keyRange) {
    const RadianceCache &C = ctx->cache;
    RcRows<1> rec{C.rec[0], C.rec[1], C.rec[2], C.rec[3], C.rec[6], C.ctr + 2, (uint32_t)C.recCap, 1u, 0u};
    k_rc_targets<<<(unsigned)ctx->numSMs, 256, 0, st>>>(rec, C.rec[4], C.rec[5], C.rec[6], C.rec[7], C.ctr, lo_eta,
                                                         rng, pendA, pendE);
    // the wave's records in slot order (scratch: counts, offsets, cursors, (record, slot) pairs)
    uint32_t *cnt = C.ordScratch, *off = cnt + kRcOrdBuckets, *cur = off + kRcOrdBuckets + 1;
    uint2 *tmp = reinterpret_cast<uint2 *>(cur + kRcOrdBuckets + 1);  // 8-byte aligned: 3 x 4096 + 2 words before
    cudaError_t e = cudaMemsetAsync(cnt, 0, kRcOrdBuckets * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    const unsigned g = (unsigned)ctx->numSMs;
    k_rc_ord_count<<<g, 256, 0, st>>>(rec, C.ctr, keyRange, cnt);
    k_rc_ord_scan<<<1, 1024, 0, st>>>(rec, cnt, off, cur, C.ctr);
    k_rc_ord_scatter<<<g, 256, 0, st>>>(C.rec[2], C.ctr, keyRange, cur, tmp);
    RcOrdCopy oc{{C.rec[0], C.rec[1], C.rec[2], C.rec[3], C.rec[6]},
                 {C.recOrd[0], C.recOrd[1], C.recOrd[2], C.recOrd[3], C.recOrd[4]}};
    k_rc_ord_place<<<g, 256, 0, st>>>(oc, C.ctr, keyRange, off, tmp);
    return cudaGetLastError();
}
// kRcStepsPerCall (pt_internal.h) Adam steps per render call, step s on
// records s, s + steps, ... (interleaved, so each batch spans the whole frame).
cudaError_t rc_enqueue_train(pt_ctx *ctx, cudaStream_t st, uint32_t s, bool adam) {
    RadianceCache &C = ctx->cache;
    float *lossDev = reinterpret_cast<float *>(C.ctr + 8);
    if (!adam) {  // the step's gradient over records s, s + kRcStepsPerCall, ...
        cudaError_t e = cudaMemsetAsync(lossDev, 0, 4, st);
        if (e != cudaSuccess) return e;
        RcTrainArgs a{};
        a.net = rc_net(ctx, C.imgTrain);
        a.rec = RcRows<1>{C.recOrd[0], C.recOrd[1], C.recOrd[2], C.recOrd[3], C.recOrd[4], C.ctr + 2, (uint32_t)C.recCap,
                          kRcStepsPerCall, s};
        a.part = C.gradPart;
        a.lossSum = lossDev;
        k_rc_train<1><<<ctx->numSMs, kRcThreads, kTrainSmem, st>>>(a);
    } else {  // the slots' sum and the Adam update in one launch
        RcAdamArgs d{C.w, C.m, C.v, C.ema, C.grad, C.imgTrain, C.imgInfer, C.ctr, C.ctr + 2, (uint32_t)C.recCap,
                     C.params.train_records, kRcStepsPerCall, s, C.params.learning_rate, C.params.ema, lossDev,
                     s + 1 == kRcStepsPerCall ? 1u : 0u, C.params.max_train_fraction};
        k_rc_adam_slots<<<kReduceBlocks, 256, 0, st>>>(d, C.gradPart, (uint32_t)ctx->numSMs);
    }
    return cudaGetLastError();
}
int rc_render_setup(pt_ctx *ctx, size_t waveCap, uint64_t callPaths) {
    int rc = rc_check(ctx);
    if (rc) return rc;
    rc_bounds(ctx);
    RadianceCache &C = ctx->cache;
    if (C.firstCall && callPaths) {
        // no call before to count cache vertices: a path has at most one, so
        // 1.5 x train_records / paths keeps the first call's records well
        // inside the buffers (twice the target) and their choice repeatable
        const float p = std::min(C.params.max_train_fraction, 1.5f * (float)C.params.train_records / (float)callPaths);
        k_rc_set_chance<<<1, 1, 0, ctx->stream>>>(reinterpret_cast<float *>(C.ctr + 7), p);  // stream-ordered, no sync
        if (cudaGetLastError() != cudaSuccess) return ctx->fail(PT_E_CUDA, "cache training chance");
        C.firstCall = false;
    }
    // a path makes at most two queries per wave: at its cache vertex and, as a
    // training path, at the end of its suffix
    return pt_cache_prepare(ctx, 2 * waveCap);
}

void pt_cache_free(pt_ctx *ctx) {
    RadianceCache &C = ctx->cache;
    void *ps[] = {C.w, C.m, C.v, C.ema, C.grad, C.gradPart, C.imgTrain, C.imgInfer, C.ctr, C.ordScratch};
    for (void *p : ps)
        if (p) cudaFree(p);
    for (float4 *p : C.q)
        if (p) cudaFree(p);
    for (float4 *p : C.rec)
        if (p) cudaFree(p);
    for (float4 *p : C.recOrd)
        if (p) cudaFree(p);
    uint64_t gen = C.gen + 1;
    C = RadianceCache{};
    C.gen = gen;
}

int pt_cache_prepare(pt_ctx *ctx, size_t queryCap) {
    RadianceCache &C = ctx->cache;
    if (C.queryCap >= queryCap) return PT_OK;
    for (float4 *&p : C.q) {
        if (p) cudaFree(p);
        p = nullptr;
    }
    C.queryCap = 0;
    C.gen++;
    for (float4 *&p : C.q)
        if (cudaMalloc(&p, queryCap * sizeof(float4)) != cudaSuccess)
            return ctx->fail(PT_E_NOMEM, "cache query buffers");
    C.queryCap = queryCap;
    return PT_OK;
}

extern "C" {

int pt_cache_init(pt_ctx *ctx, const pt_cache_params *params) {
    if (!ctx || !params) return PT_E_INVALID;
    if (params->train_records > PT_CACHE_MAX_RECORDS) return ctx->fail(PT_E_INVALID, "train_records above the maximum");
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    pt_cache_free(ctx);
    RadianceCache &C = ctx->cache;
    C.params = *params;
    if (!C.params.train_records) C.params.train_records = 65536u;
    if (C.params.rough_threshold <= 0.0f) C.params.rough_threshold = 0.3f;
    if (C.params.learning_rate <= 0.0f) C.params.learning_rate = 5e-3f;
    if (C.params.max_train_fraction <= 0.0f || C.params.max_train_fraction > 1.0f) C.params.max_train_fraction = 0.25f;
    rc_bounds(ctx);
    cudaError_t e = cudaSuccess;
    auto A = [&](void **p, size_t b) { if (e == cudaSuccess) e = cudaMalloc(p, b); };
    for (float **p : {&C.w, &C.m, &C.v, &C.ema, &C.grad}) A((void **)p, kRcParams * sizeof(float));
    A((void **)&C.gradPart, (size_t)ctx->numSMs * kRcParams * sizeof(float));
    A((void **)&C.imgTrain, kRcImageBytes);
    A((void **)&C.imgInfer, kRcImageBytes);
    A((void **)&C.ctr, 16 * sizeof(uint32_t));
    // record buffers hold twice the target: a call overflows them only when
    // its cache vertices more than double from the call before
    C.recCap = 2 * (size_t)C.params.train_records;
    C.firstCall = true;
    for (float4 *&p : C.rec) A((void **)&p, C.recCap * sizeof(float4));
    for (float4 *&p : C.recOrd) A((void **)&p, C.recCap * sizeof(float4));
    A((void **)&C.ordScratch, (3 * kRcOrdBuckets + 2 + 2 * C.recCap) * sizeof(uint32_t));
    if (e != cudaSuccess) {
        pt_cache_free(ctx);
        return ctx->fail(PT_E_NOMEM, "radiance cache", cudaGetErrorString(e));
    }
    // He-uniform initialisation of the hidden layers; the output layer starts
    // small so the untrained cache returns about zero
    std::vector<float> w(kRcParams, 0.0f);
    std::mt19937 rng(params->seed);
    for (int l = 0; l < kRcLayers; l++) {
        float lim = l < kRcLayers - 1 ? std::sqrt(6.0f / kRcIn) : 0.01f;
        std::uniform_real_distribution<float> U(-lim, lim);
        for (int o = 0; o < rc_rows(l); o++)
            for (int i = 0; i < kRcIn; i++)
                w[rc_param_base(l) + o * kRcIn + i] = (l == kRcLayers - 1 && o >= 3) ? 0.0f : U(rng);
    }
    cudaMemcpy(C.w, w.data(), w.size() * 4, cudaMemcpyHostToDevice);
    for (float *p : {C.m, C.v, C.grad}) cudaMemset(p, 0, kRcParams * sizeof(float));
    cudaMemset(C.imgTrain, 0, kRcImageBytes);
    cudaMemset(C.imgInfer, 0, kRcImageBytes);
    cudaMemset(C.ctr, 0, 16 * sizeof(uint32_t));
    cudaMemcpy(C.ctr + 7, &C.params.max_train_fraction, 4, cudaMemcpyHostToDevice);  // see rc_render_setup
    k_rc_images<<<21, 1024>>>(C.w, C.imgTrain, C.imgInfer, C.ema);
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return ctx->fail(PT_E_CUDA, "cache initialisation", cudaGetErrorString(e));
    C.ready = true;
    return PT_OK;
}

int pt_cache_release(pt_ctx *ctx) {
    if (!ctx) return PT_E_INVALID;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    pt_cache_free(ctx);
    return PT_OK;
}

int pt_cache_weights(pt_ctx *ctx, float *get, const float *set) {
    int rc = rc_check(ctx);
    if (rc) return rc;
    RadianceCache &C = ctx->cache;
    cudaStreamSynchronize(ctx->stream);
    if (get && cudaMemcpy(get, C.w, kRcParams * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
        return ctx->fail(PT_E_CUDA, "cache weights");
    if (set) {
        if (cudaMemcpy(C.w, set, kRcParams * 4, cudaMemcpyHostToDevice) != cudaSuccess)
            return ctx->fail(PT_E_CUDA, "cache weights");
        for (float *p : {C.m, C.v, C.grad}) cudaMemset(p, 0, kRcParams * sizeof(float));
        cudaMemset(C.ctr, 0, 16 * sizeof(uint32_t));
        cudaMemcpy(C.ctr + 7, &C.params.max_train_fraction, 4, cudaMemcpyHostToDevice);
        C.firstCall = true;
        k_rc_images<<<21, 1024>>>(C.w, C.imgTrain, C.imgInfer, C.ema);
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return ctx->fail(PT_E_CUDA, "cache weights", cudaGetErrorString(e));
    }
    return PT_OK;
}

int pt_cache_encode_batch(pt_ctx *ctx, const float *records, size_t n, float *features, uint32_t loc) {
    int rc = rc_check(ctx);
    if (rc) return rc;
    if (!records || !features) return ctx->fail(PT_E_INVALID, "null argument");
    if (!n) return PT_OK;
    if (n > 0xFFFFFFFFull) return ctx->fail(PT_E_INVALID, "too many records");
    Staging s{ctx, loc, {}};
    s.add(records, n * kRcRecFloats * 4, false);
    s.add(features, n * kRcIn * 4, true);
    if ((rc = s.setup())) return rc;
    const RadianceCache &C = ctx->cache;
    k_rc_encode<<<(unsigned)((n + 127) / 128), 128, 0, ctx->stream>>>(
        (const float4 *)s.dev(0), (uint32_t)n, C.bmin[0], C.bmin[1], C.bmin[2], C.binv[0], C.binv[1], C.binv[2],
        (float *)s.dev(1));
    return s.finish();
}

int pt_cache_infer_batch(pt_ctx *ctx, const float *features, size_t n, float *out, uint32_t loc) {
    int rc = rc_check(ctx);
    if (rc) return rc;
    if (!features || !out) return ctx->fail(PT_E_INVALID, "null argument");
    if (!n) return PT_OK;
    if (n > 0x7FFFFFFFull) return ctx->fail(PT_E_INVALID, "too many queries");
    Staging s{ctx, loc, {}};
    s.add(features, n * kRcIn * 4, false);
    s.add(out, n * 12, true);
    if ((rc = s.setup())) return rc;
    RcInferArgs a{};
    a.net = rc_net(ctx, ctx->cache.imgInfer);
    a.feat.feat = (const float *)s.dev(0);
    a.feat.n = (uint32_t)n;
    a.out = (float *)s.dev(1);
    cudaEventRecord(ctx->ev[0], ctx->stream);
    k_rc_infer<0><<<rc_grid(ctx, (uint32_t)n, kRcInferCtasPerSm<0>), kRcThreads, kInferSmem, ctx->stream>>>(a);
    cudaEventRecord(ctx->ev[1], ctx->stream);
    if ((rc = s.finish())) return rc;
    cudaEventElapsedTime(&ctx->cache.lastKernelMs, ctx->ev[0], ctx->ev[1]);
    return rc_device_error(ctx);
}

static int rc_train_impl(pt_ctx *ctx, const float *features, const float *targets, size_t n, float *grad,
                         float *loss, uint32_t loc, bool step) {
    int rc = rc_check(ctx);
    if (rc) return rc;
    if (!features || !targets) return ctx->fail(PT_E_INVALID, "null argument");
    if (n > PT_CACHE_MAX_RECORDS) return ctx->fail(PT_E_INVALID, "too many records");
    RadianceCache &C = ctx->cache;
    Staging s{ctx, loc, {}};
    s.add(features, n * kRcIn * 4, false);
    s.add(targets, n * 12, false);
    if ((rc = s.setup())) return rc;
    float *lossDev = reinterpret_cast<float *>(C.ctr + 8);
    uint32_t *nDev = C.ctr + 9;
    uint32_t n32 = (uint32_t)n;
    cudaMemsetAsync(lossDev, 0, 4, ctx->stream);
    cudaMemcpyAsync(nDev, &n32, 4, cudaMemcpyHostToDevice, ctx->stream);
    if (n) {
        RcTrainArgs a{};
        a.net = rc_net(ctx, C.imgTrain);
        a.feat.feat = (const float *)s.dev(0);
        a.feat.targ = (const float *)s.dev(1);
        a.feat.n = n32;
        a.part = C.gradPart;
        a.lossSum = lossDev;
        const unsigned grid = rc_grid(ctx, n32, 1);
        cudaEventRecord(ctx->ev[0], ctx->stream);
        k_rc_train<0><<<grid, kRcThreads, kTrainSmem, ctx->stream>>>(a);
        k_rc_grad_reduce<<<kReduceBlocks, 256, 0, ctx->stream>>>(C.gradPart, grid, C.grad);
        cudaEventRecord(ctx->ev[1], ctx->stream);
    }
    float lossHost = 0.0f;
    cudaMemcpyAsync(&lossHost, lossDev, 4, cudaMemcpyDeviceToHost, ctx->stream);
    if (step) {
        RcAdamArgs d{C.w, C.m, C.v, C.ema, C.grad, C.imgTrain, C.imgInfer, C.ctr, nDev, PT_CACHE_MAX_RECORDS,
                     PT_CACHE_MAX_RECORDS, 1u, 0u, C.params.learning_rate, C.params.ema, lossDev, 0u, 1.0f};
        k_rc_adam<<<1, 1024, 0, ctx->stream>>>(d);
    } else if (grad) {
        cudaMemcpyAsync(grad, C.grad, kRcParams * 4, cudaMemcpyDeviceToHost, ctx->stream);
        cudaMemsetAsync(C.grad, 0, kRcParams * 4, ctx->stream);
    }
    if ((rc = s.finish())) return rc;
    if (n) cudaEventElapsedTime(&C.lastKernelMs, ctx->ev[0], ctx->ev[1]);
    if (loss) *loss = lossHost;
    return rc_device_error(ctx);
}

int pt_cache_gradient_batch(pt_ctx *ctx, const float *features, const float *targets, size_t n, float *grad,
                            float *loss, uint32_t loc) {
    if (ctx && !grad) return ctx->fail(PT_E_INVALID, "null argument");
    return rc_train_impl(ctx, features, targets, n, grad, loss, loc, false);
}

int pt_cache_train_batch(pt_ctx *ctx, const float *features, const float *targets, size_t n, float *loss,
                         uint32_t loc) {
    return rc_train_impl(ctx, features, targets, n, nullptr, loss, loc, true);
}

int pt_cache_get_stats(pt_ctx *ctx, pt_cache_stats *out) {
    int rc = rc_check(ctx);
    if (rc) return rc;
    if (!out) return ctx->fail(PT_E_INVALID, "null argument");
    uint32_t c[16];
    cudaStreamSynchronize(ctx->stream);
    if (cudaMemcpy(c, ctx->cache.ctr, sizeof(c), cudaMemcpyDeviceToHost) != cudaSuccess)
        return ctx->fail(PT_E_CUDA, "cache counters");
    out->steps = c[0];
    out->last_records = c[4];
    memcpy(&out->last_loss, &c[3], 4);
    out->queries = c[5];
    out->last_kernel_ms = ctx->cache.lastKernelMs;
    out->last_render_infer_ms = ctx->cache.renderInferMs;
    out->last_render_train_ms = ctx->cache.renderTrainMs;
    out->last_render_train_rows = std::min<uint64_t>(c[2], ctx->cache.recCap);
    return PT_OK;
}

}  // extern "C"
