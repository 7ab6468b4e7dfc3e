// pt_api.cu — the C ABI of libpt (include/pt.h).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <new>

#include "pt_internal.h"

using namespace pt;

// ===========================================================================
// scene-build kernels
// ===========================================================================
namespace pt {

// Conditional CDF rows of BuildEnvmapDistribution
// (src/gpu/DXRApp_Textures.cpp:281-389): one thread per row, sequential
// float prefix sum in the reference's order, so the bits match.
__global__ void k_env_rows(uint32_t W, uint32_t H, const float4 *__restrict__ env, const float *__restrict__ sinRow,
                           float *cond, float *rowSums) {
    uint32_t y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= H) return;
    float st = sinRow[y];
    size_t rb = (size_t)y * (W + 1);
    cond[rb] = 0.0f;
    float rs = 0.0f;
    for (uint32_t x = 0; x < W; x++) {
        float4 p = env[(size_t)y * W + x];
        float l = __fadd_rn(__fadd_rn(__fmul_rn(0.2126f, p.x), __fmul_rn(0.7152f, p.y)), __fmul_rn(0.0722f, p.z));
        float w = __fmul_rn(l, st);
        if (w < 0.0f) w = 0.0f;
        rs = __fadd_rn(rs, w);
        cond[rb + x + 1] = rs;
    }
    rowSums[y] = rs;
    if (rs > 0.0f) {
        float inv = __fdiv_rn(1.0f, rs);
        for (uint32_t x = 1; x <= W; x++) cond[rb + x] = __fmul_rn(cond[rb + x], inv);
    } else {
        for (uint32_t x = 0; x <= W; x++) cond[rb + x] = __fdiv_rn((float)x, (float)W);
    }
}
// Marginal CDF: FP64 running sum over rows (single thread, the reference order).
__global__ void k_env_marginal(uint32_t H, const float *__restrict__ rowSums, float *marg) {
    double total = 0.0;
    for (uint32_t y = 0; y < H; y++) total = __dadd_rn(total, (double)rowSums[y]);
    marg[0] = 0.0f;
    if (total > 0.0) {
        double acc = 0.0, inv = __ddiv_rn(1.0, total);
        for (uint32_t y = 0; y < H; y++) {
            acc = __dadd_rn(acc, (double)rowSums[y]);
            marg[y + 1] = (float)__dmul_rn(acc, inv);
        }
        marg[H] = 1.0f;
    } else {
        for (uint32_t y = 0; y <= H; y++) marg[y] = __fdiv_rn((float)y, (float)H);
    }
}
// Guide tables of the CDF search (cdf_search_guided): for every conditional
// row and the marginal, the search index at u = k / kCdfGuide, k = 0 .. kCdfGuide.
__global__ void k_env_guides(uint32_t W, uint32_t H, const float *marg, const float *cond, uint16_t *margGuide,
                             uint16_t *condGuide) {
    const uint32_t per = kCdfGuide + 1, total = (H + 1) * per;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const uint32_t r = i / per, k = i % per;
        const float u = (float)k / (float)kCdfGuide;  // exact
        if (r < H) condGuide[i] = (uint16_t)cdf_upper(cond + (size_t)r * (W + 1), 0, W, u);
        else margGuide[k] = (uint16_t)cdf_upper(marg, 0, H, u);
    }
}
// FP64 texel weights and row sums of the alias tables.
__global__ void k_alias_weights(uint32_t W, uint32_t H, const float4 *__restrict__ env, const float *__restrict__ sinRow,
                                double *wall, double *rowSum) {
    uint32_t y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= H) return;
    float st = sinRow[y];
    double rs = 0.0;
    for (uint32_t x = 0; x < W; x++) {
        float4 p = env[(size_t)y * W + x];
        float l = __fadd_rn(__fadd_rn(__fmul_rn(0.2126f, p.x), __fmul_rn(0.7152f, p.y)), __fmul_rn(0.0722f, p.z));
        float w = __fmul_rn(l, st);
        double wd = w < 0.0f ? 0.0 : (double)w;
        wall[(size_t)y * W + x] = wd;
        rs = __dadd_rn(rs, wd);
    }
    rowSum[y] = rs;
}
// Vose alias construction over n weights (FP64), deterministic stack order.
__device__ void alias_1d(const double *w, uint32_t n, float *prob, uint32_t *alias, double *q, uint32_t *stk) {
    double sum = 0.0;
    for (uint32_t i = 0; i < n; i++) sum = __dadd_rn(sum, w[i]);
    if (!(sum > 0.0)) {
        for (uint32_t i = 0; i < n; i++) { prob[i] = 1.0f; alias[i] = i; }
        return;
    }
    // small stack grows up from stk[0], large stack down from stk[n-1];
    // both are filled in reverse index order so the lowest index pops first
    uint32_t ns = 0, nl = 0;
    for (uint32_t k = 0; k < n; k++) {
        uint32_t i = n - 1 - k;
        q[i] = __ddiv_rn(__dmul_rn(w[i], (double)n), sum);
    }
    for (uint32_t k = 0; k < n; k++) {
        uint32_t i = n - 1 - k;
        if (q[i] < 1.0) stk[ns++] = i;
        else stk[n - 1 - (nl++)] = i;
    }
    while (ns > 0 && nl > 0) {
        uint32_t l = stk[--ns];
        uint32_t g = stk[n - 1 - (--nl)];
        prob[l] = (float)q[l];
        alias[l] = g;
        q[g] = __dsub_rn(__dadd_rn(q[g], q[l]), 1.0);
        if (q[g] < 1.0) stk[ns++] = g;
        else stk[n - 1 - (nl++)] = g;
    }
    while (nl > 0) { uint32_t g = stk[n - 1 - (--nl)]; prob[g] = 1.0f; alias[g] = g; }
    while (ns > 0) { uint32_t l = stk[--ns]; prob[l] = 1.0f; alias[l] = l; }
}
__global__ void k_alias_rows(uint32_t W, uint32_t H, const double *wall, const double *rowSum, float *colProb,
                             uint32_t *colAlias, float *aliasPdf, double *q, uint32_t *stk, const double *total) {
    uint32_t y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= H) return;
    size_t o = (size_t)y * W;
    alias_1d(wall + o, W, colProb + o, colAlias + o, q + o, stk + o);
    const double PI = 3.14159265358979323846;
    double tot = *total;
    for (uint32_t x = 0; x < W; x++) {
        double pp;
        if (tot > 0.0) pp = rowSum[y] > 0.0 ? __ddiv_rn(wall[o + x], tot) : 0.0;
        else pp = __ddiv_rn(1.0, __dmul_rn((double)W, (double)H));
        aliasPdf[o + x] = (float)__ddiv_rn(__dmul_rn(__dmul_rn(pp, (double)W), (double)H), 2.0 * PI * PI);
    }
}
__global__ void k_alias_marginal(uint32_t H, const double *rowSum, float *rowProb, uint32_t *rowAlias, double *q,
                                 uint32_t *stk, double *total) {
    double t = 0.0;
    for (uint32_t y = 0; y < H; y++) t = __dadd_rn(t, rowSum[y]);
    *total = t;
    alias_1d(rowSum, H, rowProb, rowAlias, q, stk);
}
// 4^3-brick maximum density (src/gpu/DXRApp_Scene.cpp:625-641).
__global__ void k_majorant(DevGrid g, DevGrid m, float *out) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m.w * m.h * m.d) return;
    uint32_t bx = i % m.w, by = (i / m.w) % m.h, bz = i / (m.w * m.h);
    float v = 0.0f;
    for (uint32_t z = bz * 4; z < min(bz * 4 + 4, g.d); z++)
        for (uint32_t y = by * 4; y < min(by * 4 + 4, g.h); y++)
            for (uint32_t x = bx * 4; x < min(bx * 4 + 4, g.w); x++)
                v = fmaxf(v, g.data[(size_t)x + (size_t)g.w * (y + (size_t)g.h * z)]);
    out[i] = v;
}

// ---- batch kernels ----------------------------------------------------------
__global__ void k_bsdf_eval(const pt_material *mats, uint32_t nm, const uint32_t *mi, const float *wi, const float *wo,
                            const float *hh, size_t n, float *f, float *pdf) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t k = mi ? min(mi[i], nm - 1) : 0u;
    pt_material m = mats[k];
    float3 a = make_float3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
    float3 b = make_float3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]);
    float3 r;
    float p;
    material_eval_pdf(a, b, m, hh ? hh[i] : 0.0f, r, p);
    f[3 * i] = r.x; f[3 * i + 1] = r.y; f[3 * i + 2] = r.z;
    pdf[i] = p;
}
__global__ void k_bsdf_sample(const pt_material *mats, uint32_t nm, const uint32_t *mi, const float *wi, const float *u,
                              const float *hh, size_t n, float *wo, float *wt, float *pdf) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t k = mi ? min(mi[i], nm - 1) : 0u;
    pt_material m = mats[k];
    float3 a = make_float3(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
    float uu[4] = {u[4 * i], u[4 * i + 1], u[4 * i + 2], u[4 * i + 3]};
    float3 o;
    float p;
    float3 r = (m.type == PT_MAT_MIRROR || m.type == PT_MAT_DIELECTRIC)
                   ? delta_sample(a, m, uu[0], o, p)
                   : material_sample(a, uu, m, hh ? hh[i] : 0.0f, o, p);
    wo[3 * i] = o.x; wo[3 * i + 1] = o.y; wo[3 * i + 2] = o.z;
    wt[3 * i] = r.x; wt[3 * i + 1] = r.y; wt[3 * i + 2] = r.z;
    pdf[i] = p;
}
__global__ void k_phase_sample(const float *g, const float *wo, const float *u, size_t n, float *wi, float *pdf) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float p;
    float3 r = sample_hg(make_float3(wo[3 * i], wo[3 * i + 1], wo[3 * i + 2]), g[i], u[2 * i], u[2 * i + 1], p);
    wi[3 * i] = r.x; wi[3 * i + 1] = r.y; wi[3 * i + 2] = r.z;
    pdf[i] = p;
}
__global__ void k_env_sample(DevScene S, uint32_t mode, const float *u, size_t n, float *dir, float *rad, float *pdf) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 d, r;
    float p;
    env_sample(S, mode, u[2 * i], u[2 * i + 1], d, r, p);
    dir[3 * i] = d.x; dir[3 * i + 1] = d.y; dir[3 * i + 2] = d.z;
    rad[3 * i] = r.x; rad[3 * i + 1] = r.y; rad[3 * i + 2] = r.z;
    pdf[i] = p;
}
__global__ void k_env_pdf(DevScene S, uint32_t mode, const float *dir, size_t n, float *pdf, float *rad) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float3 d = make_float3(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
    pdf[i] = env_pdf(S, mode, d);
    float3 r = eval_env(S, d);
    rad[3 * i] = r.x; rad[3 * i + 1] = r.y; rad[3 * i + 2] = r.z;
}
__global__ void k_rng(const uint32_t *tab, uint32_t kind, const uint32_t *pix, const uint32_t *smp, size_t n,
                      uint32_t dims, uint32_t npix, float *out) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Rng r = rng_init(pix[i], npix, smp[i], kind);
    for (uint32_t d = 0; d < dims; d++) out[i * dims + d] = next_float(r, tab);
}
__global__ void k_trace_closest(DevScene S, const float *rays, size_t n, pt_hit *out, uint32_t *err) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *r = rays + 8 * i;
    // alpha tests: path seed = ray index, key 0
    Hit h = trace_closest(S, make_float3(r[0], r[1], r[2]), make_float3(r[4], r[5], r[6]), r[3], r[7], err,
                          (uint32_t)i, 0u);
    pt_hit o;
    if (h.gid != 0xFFFFFFFFu) {
        uint32_t m = S.triMesh[h.gid];
        o = pt_hit{h.t, m, h.gid - S.meshFirstTri[m], h.u, h.v, 1u};
    } else {
        o = pt_hit{0.0f, 0u, 0u, 0.0f, 0.0f, 0u};
    }
    out[i] = o;
}
__global__ void k_trace_shadow(DevScene S, const float *rays, size_t n, uint32_t *occ, float *tr, uint32_t *err) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *r = rays + 8 * i;
    float3 t;
    occ[i] = trace_shadow(S, make_float3(r[0], r[1], r[2]), make_float3(r[4], r[5], r[6]), r[3], r[7], t, err,
                          (uint32_t)i, 0u) ? 1u : 0u;
    tr[3 * i] = t.x; tr[3 * i + 1] = t.y; tr[3 * i + 2] = t.z;
}

}  // namespace pt

// ===========================================================================
// helpers
// ===========================================================================
static inline unsigned blocks_for(size_t n, unsigned b = 256) { return (unsigned)((n + b - 1) / b); }


// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int pt_abi_version(void) { return PT_ABI_VERSION; }

int pt_create(pt_ctx **out, int device) {
    if (!out) return PT_E_INVALID;
    *out = nullptr;
    pt_ctx *ctx = new (std::nothrow) pt_ctx();
    if (!ctx) return PT_E_NOMEM;
    ctx->device = device;
    auto bail = [&](int code) { delete ctx; return code; };
    if (cudaSetDevice(device) != cudaSuccess) return bail(PT_E_CUDA);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return bail(PT_E_CUDA);
    ctx->numSMs = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&ctx->ownStream, cudaStreamNonBlocking) != cudaSuccess) return bail(PT_E_CUDA);
    ctx->stream = ctx->ownStream;
    if (cudaEventCreate(&ctx->ev[0]) != cudaSuccess || cudaEventCreate(&ctx->ev[1]) != cudaSuccess)
        return bail(PT_E_CUDA);
    if (cudaStreamCreateWithFlags(&ctx->copyStream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->filmReady, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->streamMark, cudaEventDisableTiming) != cudaSuccess)
        return bail(PT_E_CUDA);
    uint32_t tab[1024];
    for (uint32_t k = 0; k < 4; k++)
        for (uint32_t b = 0; b < 256; b++) tab[256 * k + b] = ptm::sobol1_loop(b << (8 * k));
    if (cudaMalloc(&ctx->d_sobol1, sizeof(tab)) != cudaSuccess) return bail(PT_E_NOMEM);
    cudaMemcpy(ctx->d_sobol1, tab, sizeof(tab), cudaMemcpyHostToDevice);
    if (cudaMalloc(&ctx->d_err, 16) != cudaSuccess) return bail(PT_E_NOMEM);
    cudaMemset(ctx->d_err, 0, 16);
    ctx->S.sobol1 = ctx->d_sobol1;
    *out = ctx;
    return PT_OK;
}

int pt_destroy(pt_ctx *ctx) {
    if (!ctx) return PT_E_INVALID;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    pt_graph_free(ctx);
    pt_batch_free(ctx);
    ctx->free_scene();
    pt_wave_free(ctx);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->d_sobol1) cudaFree(ctx->d_sobol1);
    if (ctx->d_err) cudaFree(ctx->d_err);
    for (cudaEvent_t e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->copyStream) {
        cudaStreamSynchronize(ctx->copyStream);
        cudaStreamDestroy(ctx->copyStream);
    }
    if (ctx->filmReady) cudaEventDestroy(ctx->filmReady);
    if (ctx->streamMark) cudaEventDestroy(ctx->streamMark);
    if (ctx->ownStream) cudaStreamDestroy(ctx->ownStream);
    delete ctx;
    return PT_OK;
}

int pt_set_stream(pt_ctx *ctx, void *stream) {
    if (!ctx) return PT_E_INVALID;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->stream = stream ? (cudaStream_t)stream : ctx->ownStream;
    return PT_OK;
}

int pt_debug_set(pt_ctx *ctx, uint32_t what, uint64_t value) {
    if (!ctx) return PT_E_INVALID;
    if (value > 0xFFFFFFFFull) return ctx->fail(PT_E_INVALID, "debug value out of range");
    if (what == PT_DEBUG_SHADOW_QUEUE_CAP) ctx->dbgShadowCap = (uint32_t)value;
    else if (what == PT_DEBUG_CACHE_STALL) ctx->dbgCacheStall = (uint32_t)value;
    else if (what == PT_DEBUG_WIDE_PLAN) ctx->dbgWidePlan = value ? 1u : 0u;
    else if (what == PT_DEBUG_TAIL) {
        if (value > 2) return ctx->fail(PT_E_INVALID, "tail mode: 0, 1 or 2");
        ctx->dbgTail = (uint32_t)value;
    }
    else return ctx->fail(PT_E_INVALID, "unknown debug hook");
    return PT_OK;
}

const char *pt_last_error(const pt_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

// LoadTexture's mip chain (src/gpu/DXRApp_Textures.cpp:49-95): levels halve
// (integer division, at least 1) down to 1 x 1, each texel the truncated
// integer mean of the 2 x 2 texels below it, edge texels repeated.
static void build_mips(const pt_texture &t, std::vector<uchar4> &texels, DevTexture &dt) {
    uint32_t levels = 1;
    for (uint32_t dim = std::max(t.width, t.height); dim > 1; dim >>= 1) levels++;
    dt.w = t.width;
    dt.h = t.height;
    dt.levels = levels;
    dt.srgb = t.srgb ? 1u : 0u;
    size_t base = texels.size();
    dt.off[0] = (uint32_t)base;
    texels.resize(base + (size_t)t.width * t.height);
    std::memcpy(&texels[base], t.rgba8, (size_t)t.width * t.height * 4);
    uint32_t pw = t.width, ph = t.height;
    for (uint32_t m = 1; m < levels; m++) {
        uint32_t mw = std::max(pw / 2, 1u), mh = std::max(ph / 2, 1u);
        size_t src = dt.off[m - 1], dst = texels.size();
        dt.off[m] = (uint32_t)dst;
        texels.resize(dst + (size_t)mw * mh);
        for (uint32_t y = 0; y < mh; y++)
            for (uint32_t x = 0; x < mw; x++) {
                uint32_t sx = std::min(x * 2, pw - 1), sy = std::min(y * 2, ph - 1);
                uint32_t sx1 = std::min(sx + 1, pw - 1), sy1 = std::min(sy + 1, ph - 1);
                const uchar4 a = texels[src + (size_t)sy * pw + sx], b = texels[src + (size_t)sy * pw + sx1];
                const uchar4 c = texels[src + (size_t)sy1 * pw + sx], e = texels[src + (size_t)sy1 * pw + sx1];
                texels[dst + (size_t)y * mw + x] =
                    make_uchar4((unsigned char)((a.x + b.x + c.x + e.x) / 4), (unsigned char)((a.y + b.y + c.y + e.y) / 4),
                                (unsigned char)((a.z + b.z + c.z + e.z) / 4), (unsigned char)((a.w + b.w + c.w + e.w) / 4));
            }
        pw = mw;
        ph = mh;
    }
}

// sRGB-encoded byte -> linear (the _SRGB format decode: v / 12.92 up to
// 0.04045, ((v + 0.055) / 1.055)^2.4 above), evaluated in double.
static float srgb_to_linear(uint32_t byte) {
    double v = byte / 255.0;
    return (float)(v <= 0.04045 ? v / 12.92 : std::pow((v + 0.055) / 1.055, 2.4));
}

static int upload_textures(pt_ctx *ctx, const pt_scene_desc *d) {
    DevScene &S = ctx->S;
    std::vector<DevTexture> dts(std::max(1u, d->num_textures));
    std::vector<uchar4> texels;
    for (uint32_t t = 0; t < d->num_textures; t++) build_mips(d->textures[t], texels, dts[t]);
    if (texels.empty()) texels.push_back(make_uchar4(0, 0, 0, 0));
    float lut[256];
    for (uint32_t i = 0; i < 256; i++) lut[i] = srgb_to_linear(i);
    DevTexture *dtex;
    uchar4 *dtexels;
    float *dlut;
    PT_CUDA(ctx->alloc_scene(&dtex, dts.size()));
    PT_CUDA(ctx->alloc_scene(&dtexels, texels.size()));
    PT_CUDA(ctx->alloc_scene(&dlut, 256));
    PT_CUDA(cudaMemcpyAsync(dtex, dts.data(), dts.size() * sizeof(DevTexture), cudaMemcpyHostToDevice, ctx->stream));
    PT_CUDA(cudaMemcpyAsync(dtexels, texels.data(), texels.size() * 4, cudaMemcpyHostToDevice, ctx->stream));
    PT_CUDA(cudaMemcpyAsync(dlut, lut, sizeof(lut), cudaMemcpyHostToDevice, ctx->stream));
    // the host arrays above are freed on return: finish the copies first
    PT_CUDA(cudaStreamSynchronize(ctx->stream));
    S.tex = dtex;
    S.texels = dtexels;
    S.srgbLut = dlut;
    S.numTex = d->num_textures;
    return PT_OK;
}

int pt_upload_scene(pt_ctx *ctx, const pt_scene_desc *d) {
    if (!ctx) return PT_E_INVALID;
    if (!d) return ctx->fail(PT_E_INVALID, "null scene");
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->free_scene();
    if (d->num_vertices && !d->positions) return ctx->fail(PT_E_INVALID, "positions is null");
    if (d->num_indices && !d->indices) return ctx->fail(PT_E_INVALID, "indices is null");
    if (d->num_meshes && !d->materials) return ctx->fail(PT_E_INVALID, "materials is null");
    if (d->num_volumes && !d->volumes) return ctx->fail(PT_E_INVALID, "volumes is null");
    // --- validation + per-mesh first triangle (meshes in index order) -------
    std::vector<pt_material> mats(d->materials, d->materials + d->num_meshes);
    std::vector<uint32_t> meshFirstTri(std::max(1u, d->num_meshes), 0);
    uint32_t numTris = 0;
    bool hasGlass = false, hasAlpha = false, hasSubsurface = false;
    uint32_t clsMask = 1u << CLS_MISS;  // shading classes the scene can produce
    std::vector<uint32_t> meshClass(std::max(1u, d->num_meshes), 0u);
    for (uint32_t m = 0; m < d->num_meshes; m++) {
        const pt_material &pm = mats[m];
        if (pm.type > PT_MAT_SUBSURFACE) return ctx->fail(PT_E_INVALID, "unknown material type");
        const uint32_t *tex = &pm.albedoTexIndex;  // albedo .. alpha: 7 consecutive indices
        for (int t = 0; t < 7; t++)
            if (tex[t] != PT_NO_TEXTURE && tex[t] >= d->num_textures)
                return ctx->fail(PT_E_INVALID, "material texture index out of range");
        if (pm.indexCount % 3) return ctx->fail(PT_E_INVALID, "indexCount is not a multiple of 3");
        if ((uint64_t)pm.indexOffset + pm.indexCount > d->num_indices) return ctx->fail(PT_E_INVALID, "index range");
        if ((uint64_t)pm.vertexOffset + pm.vertexCount > d->num_vertices) return ctx->fail(PT_E_INVALID, "vertex range");
        for (uint32_t k = 0; k < pm.indexCount; k++)
            if (d->indices[pm.indexOffset + k] >= pm.vertexCount) return ctx->fail(PT_E_INVALID, "index out of range");
        meshFirstTri[m] = numTris;
        numTris += pm.indexCount / 3;
        hasGlass |= pm.type == PT_MAT_MIRROR || pm.type == PT_MAT_DIELECTRIC;
        hasSubsurface |= pm.indexCount && pm.type == PT_MAT_SUBSURFACE;
        meshClass[m] = (uint32_t)shade_class(true, pm.isEmitter != 0, pm.type, has_shading_textures(pm));
        if (pm.indexCount) clsMask |= 1u << meshClass[m];
        if (pm.indexCount && pm.alphaTexIndex != PT_NO_TEXTURE) hasAlpha = true;
    }
    if (d->num_textures && !d->textures) return ctx->fail(PT_E_INVALID, "textures is null");
    for (uint32_t t = 0; t < d->num_textures; t++) {
        const pt_texture &tx = d->textures[t];
        if (!tx.rgba8 || !tx.width || !tx.height) return ctx->fail(PT_E_INVALID, "empty texture");
        if (tx.width > 32768u || tx.height > 32768u) return ctx->fail(PT_E_INVALID, "texture larger than 32768");
    }
    for (uint32_t v = 0; v < d->num_volumes; v++) {
        const pt_volume &vol = d->volumes[v];
        if (vol.density_grid != PT_NO_TEXTURE && vol.density_grid >= d->num_grids)
            return ctx->fail(PT_E_INVALID, "volume density_grid out of range");
    }
    for (uint32_t g = 0; g < d->num_grids; g++)
        if (!d->grids[g].data || !d->grids[g].w || !d->grids[g].h || !d->grids[g].d)
            return ctx->fail(PT_E_INVALID, "empty density grid");
    // --- area DiscretePDFs and the emitter CDF buffer (host, the reference's
    //     float accumulation order: src/cpu/mesh.cpp:24-40, include/dpdf.h,
    //     src/gpu/DXRApp_Scene.cpp:243-299) ------------------------------------
    std::vector<float> all;
    std::vector<uint32_t> emitters;
    for (uint32_t m = 0; m < d->num_meshes; m++) {
        pt_material &pm = mats[m];
        const uint32_t nt = pm.indexCount / 3;
        std::vector<float> cdf;
        if (pm.isEmitter) cdf.reserve(nt + 1);
        float acc = 0.0f;
        if (pm.isEmitter) cdf.push_back(0.0f);
        for (uint32_t t = 0; t < nt; t++) {
            const uint32_t *f = d->indices + pm.indexOffset + 3 * t;
            const float *p0 = d->positions + 3 * (size_t)(pm.vertexOffset + f[0]);
            const float *p1 = d->positions + 3 * (size_t)(pm.vertexOffset + f[1]);
            const float *p2 = d->positions + 3 * (size_t)(pm.vertexOffset + f[2]);
            float ax = p1[0] - p0[0], ay = p1[1] - p0[1], az = p1[2] - p0[2];
            float bx = p2[0] - p0[0], by = p2[1] - p0[1], bz = p2[2] - p0[2];
            float cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
            float a = 0.5f * std::sqrt(cx * cx + cy * cy + cz * cz);
            acc = acc + a;
            if (pm.isEmitter) cdf.push_back(acc);
        }
        pm.surfaceArea = acc;
        pm.emitterCdfOffset = 0;
        pm.emitterSelectionProb = 0.0f;
        if (pm.isEmitter) {
            if (acc > 0.0f) {
                float inv = 1.0f / acc;
                for (size_t k = 1; k < cdf.size(); k++) cdf[k] *= inv;
                cdf.back() = 1.0f;
            }
            pm.emitterCdfOffset = (uint32_t)all.size();
            all.insert(all.end(), cdf.begin(), cdf.end());
            emitters.push_back(m);
        }
    }
    const uint32_t ne = (uint32_t)emitters.size();
    std::vector<float> pc(ne + 1, 0.0f);
    for (uint32_t k = 0; k < ne; k++) {
        const pt_material &pm = mats[emitters[k]];
        float l = 0.2126f * pm.radiance[0] + 0.7152f * pm.radiance[1] + 0.0722f * pm.radiance[2];
        pc[k + 1] = pc[k] + l * pm.surfaceArea;
    }
    if (pc[ne] > 0.0f) {
        float inv = 1.0f / pc[ne];
        for (uint32_t k = 1; k <= ne; k++) pc[k] *= inv;
    } else {
        for (uint32_t k = 0; k <= ne; k++) pc[k] = float(k) / float(std::max(ne, 1u));
    }
    pc[ne] = 1.0f;
    for (uint32_t k = 0; k < ne; k++) {
        mats[emitters[k]].emitterSelectionProb = pc[k + 1] - pc[k];
        mats[emitters[k]].emitterCdfOffset += ne + 1;
    }
    all.insert(all.begin(), pc.begin(), pc.end());
    // --- device copies ---------------------------------------------------------
    DevScene &S = ctx->S;
    S.sobol1 = ctx->d_sobol1;
    const size_t nv = d->num_vertices;
    {  // vertex bounds (the radiance cache's default position box)
        float lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
        if (nv) {
            for (int k = 0; k < 3; k++) lo[k] = hi[k] = d->positions[k];
            for (size_t v = 1; v < nv; v++)
                for (int k = 0; k < 3; k++) {
                    lo[k] = std::min(lo[k], d->positions[3 * v + k]);
                    hi[k] = std::max(hi[k], d->positions[3 * v + k]);
                }
        }
        for (int k = 0; k < 3; k++) {
            ctx->sceneMin[k] = lo[k];
            ctx->sceneMax[k] = hi[k];
        }
    }
    float *dpos, *dnrm, *duv, *dtan, *dcdf;
    uint32_t *didx, *dmft, *demit;
    pt_material *dmats;
    cudaStream_t st = ctx->stream;
    PT_CUDA(ctx->alloc_scene(&dpos, 3 * nv + 3));
    PT_CUDA(ctx->alloc_scene(&dnrm, 3 * nv + 3));
    PT_CUDA(ctx->alloc_scene(&duv, 2 * nv + 2));
    PT_CUDA(ctx->alloc_scene(&dtan, 3 * nv + 3));
    PT_CUDA(ctx->alloc_scene(&didx, (size_t)d->num_indices + 1));
    PT_CUDA(ctx->alloc_scene(&dmats, std::max<size_t>(1, mats.size())));
    PT_CUDA(ctx->alloc_scene(&dmft, meshFirstTri.size()));
    PT_CUDA(ctx->alloc_scene(&dcdf, all.size() + 1));
    PT_CUDA(ctx->alloc_scene(&demit, (size_t)ne + 1));
    uint32_t *dmcls;
    PT_CUDA(ctx->alloc_scene(&dmcls, meshClass.size()));
    auto h2d = [&](void *dst, const void *src, size_t bytes) -> int {
        if (!bytes) return PT_OK;
        cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st);
        return e == cudaSuccess ? PT_OK : ctx->fail(PT_E_CUDA, "upload", cudaGetErrorString(e));
    };
    int rc;
    if ((rc = h2d(dpos, d->positions, 3 * nv * 4))) return rc;
    if (d->normals) { if ((rc = h2d(dnrm, d->normals, 3 * nv * 4))) return rc; }
    else PT_CUDA(cudaMemsetAsync(dnrm, 0, 3 * nv * 4 + 12, st));
    if (d->texcoords) { if ((rc = h2d(duv, d->texcoords, 2 * nv * 4))) return rc; }
    else PT_CUDA(cudaMemsetAsync(duv, 0, 2 * nv * 4 + 8, st));
    if (d->tangents) { if ((rc = h2d(dtan, d->tangents, 3 * nv * 4))) return rc; }
    else PT_CUDA(cudaMemsetAsync(dtan, 0, 3 * nv * 4 + 12, st));
    if ((rc = h2d(didx, d->indices, (size_t)d->num_indices * 4))) return rc;
    if ((rc = h2d(dmats, mats.data(), mats.size() * sizeof(pt_material)))) return rc;
    if ((rc = h2d(dmft, meshFirstTri.data(), meshFirstTri.size() * 4))) return rc;
    if ((rc = h2d(dcdf, all.data(), all.size() * 4))) return rc;
    if ((rc = h2d(demit, emitters.data(), emitters.size() * 4))) return rc;
    if ((rc = h2d(dmcls, meshClass.data(), meshClass.size() * 4))) return rc;
    if ((rc = upload_textures(ctx, d))) return rc;
    S.hasAlpha = hasAlpha ? 1u : 0u;
    S.hasSubsurface = hasSubsurface ? 1u : 0u;
    {  // homogeneous media only (and no subsurface walks): the wavefront form
        bool homog = d->num_volumes > 0;
        for (uint32_t v = 0; v < d->num_volumes; v++)
            if (d->volumes[v].flags & PT_VOLUME_HETEROGENEOUS) homog = false;
        S.mediaWavefront = (homog && !hasSubsurface) ? 1u : 0u;
        S.mediaTrDeferred = 0u;
        if (S.mediaWavefront) clsMask |= 1u << CLS_MEDIUM;
    }
    S.pos = dpos; S.nrm = dnrm; S.uv = duv; S.tan = dtan; S.idx = didx;
    S.mats = dmats; S.meshClass = dmcls; S.numMeshes = d->num_meshes; S.meshFirstTri = dmft;
    S.emitterCdf = dcdf; S.emitterList = demit; S.emitterCount = ne;
    S.hasGlass = hasGlass ? 1u : 0u;
    // --- BVH ----------------------------------------------------------------------
    if ((rc = pt_build_bvh_device(ctx, dmft, numTris))) return rc;
    // --- envmap -------------------------------------------------------------------
    uint32_t W = d->env_width, H = d->env_height;
    std::vector<float4> env4;
    if (!W || !H || !d->env_rgb) {
        W = H = 1;
        env4.assign(1, make_float4(0, 0, 0, 1));
    } else {
        env4.resize((size_t)W * H);
        for (size_t i = 0; i < env4.size(); i++)
            env4[i] = make_float4(d->env_rgb[3 * i], d->env_rgb[3 * i + 1], d->env_rgb[3 * i + 2], 1.0f);
    }
    std::vector<float> sinRow(H);
    const float PIf = 3.14159265358979323846f;
    for (uint32_t y = 0; y < H; y++) sinRow[y] = std::sin(PIf * (y + 0.5f) / (float)H);
    float4 *denv;
    float *dmarg, *dcond, *drowsum, *dsin, *drowProb, *dcolProb, *dapdf;
    uint32_t *drowAlias, *dcolAlias;
    const size_t WH = (size_t)W * H;
    PT_CUDA(ctx->alloc_scene(&denv, WH));
    PT_CUDA(ctx->alloc_scene(&dmarg, H + 1));
    PT_CUDA(ctx->alloc_scene(&dcond, (size_t)H * (W + 1)));
    PT_CUDA(ctx->alloc_scene(&drowProb, H));
    PT_CUDA(ctx->alloc_scene(&drowAlias, H));
    PT_CUDA(ctx->alloc_scene(&dcolProb, WH));
    PT_CUDA(ctx->alloc_scene(&dcolAlias, WH));
    PT_CUDA(ctx->alloc_scene(&dapdf, WH));
    uint16_t *dmguide = nullptr, *dcguide = nullptr;  // 16-bit indices: rows up to 65,535 texels
    if (W < 65536u && H < 65536u) {
        PT_CUDA(ctx->alloc_scene(&dmguide, kCdfGuide + 1));
        PT_CUDA(ctx->alloc_scene(&dcguide, (size_t)H * (kCdfGuide + 1)));
    }
    if ((rc = h2d(denv, env4.data(), WH * sizeof(float4)))) return rc;
    {
        // temporaries: sin table, row sums, FP64 weights, Vose scratch
        double *wall, *rowSum, *q, *total;
        uint32_t *stk;
        cudaError_t e = cudaSuccess;
        void *tmps[7] = {};
        e = cudaMalloc(&tmps[0], H * 4 + 16); dsin = (float *)tmps[0];
        if (e == cudaSuccess) e = cudaMalloc(&tmps[1], H * 4 + 16); drowsum = (float *)tmps[1];
        if (e == cudaSuccess) e = cudaMalloc(&tmps[2], WH * 8 + 16); wall = (double *)tmps[2];
        if (e == cudaSuccess) e = cudaMalloc(&tmps[3], H * 8 + 16); rowSum = (double *)tmps[3];
        if (e == cudaSuccess) e = cudaMalloc(&tmps[4], std::max<size_t>(WH, H) * 8 + 16); q = (double *)tmps[4];
        if (e == cudaSuccess) e = cudaMalloc(&tmps[5], std::max<size_t>(WH, H) * 4 + 16); stk = (uint32_t *)tmps[5];
        if (e == cudaSuccess) e = cudaMalloc(&tmps[6], 16); total = (double *)tmps[6];
        auto freeTmps = [&]() { for (void *p : tmps) if (p) cudaFree(p); };
        if (e != cudaSuccess) { freeTmps(); return ctx->fail(PT_E_NOMEM, "envmap temporaries"); }
        cudaMemcpyAsync(dsin, sinRow.data(), H * 4, cudaMemcpyHostToDevice, st);
        k_env_rows<<<blocks_for(H, 64), 64, 0, st>>>(W, H, denv, dsin, dcond, drowsum);
        k_env_marginal<<<1, 1, 0, st>>>(H, drowsum, dmarg);
        if (dmguide) k_env_guides<<<256, 256, 0, st>>>(W, H, dmarg, dcond, dmguide, dcguide);
        k_alias_weights<<<blocks_for(H, 64), 64, 0, st>>>(W, H, denv, dsin, wall, rowSum);
        k_alias_marginal<<<1, 1, 0, st>>>(H, rowSum, drowProb, drowAlias, q, stk, total);
        k_alias_rows<<<blocks_for(H, 64), 64, 0, st>>>(W, H, wall, rowSum, dcolProb, dcolAlias, dapdf, q, stk, total);
        e = cudaStreamSynchronize(st);
        freeTmps();
        if (e != cudaSuccess) return ctx->fail(PT_E_CUDA, "envmap tables", cudaGetErrorString(e));
    }
    S.env = denv; S.envW = W; S.envH = H; S.envScale = d->env_scale;
    S.marg = dmarg; S.cond = dcond;
    S.margGuide = dmguide; S.condGuide = dcguide;
    S.rowProb = drowProb; S.rowAlias = drowAlias; S.colProb = dcolProb; S.colAlias = dcolAlias; S.aliasPdf = dapdf;
    // --- volumes ------------------------------------------------------------------
    S.numVols = d->num_volumes;
    if (d->num_volumes) {
        pt_volume *dvols;
        DevGrid *ddens, *dmaj;
        PT_CUDA(ctx->alloc_scene(&dvols, d->num_volumes));
        PT_CUDA(ctx->alloc_scene(&ddens, d->num_volumes));
        PT_CUDA(ctx->alloc_scene(&dmaj, d->num_volumes));
        std::vector<DevGrid> hd(d->num_volumes), hm(d->num_volumes);
        std::vector<float *> gridDev(d->num_grids, nullptr);
        for (uint32_t g = 0; g < d->num_grids; g++) {
            const pt_grid &gr = d->grids[g];
            size_t cnt = (size_t)gr.w * gr.h * gr.d;
            PT_CUDA(ctx->alloc_scene(&gridDev[g], cnt));
            if ((rc = h2d(gridDev[g], gr.data, cnt * 4))) return rc;
        }
        for (uint32_t v = 0; v < d->num_volumes; v++) {
            const pt_volume &vol = d->volumes[v];
            hd[v] = DevGrid{0, 0, 0, nullptr};
            hm[v] = DevGrid{0, 0, 0, nullptr};
            if ((vol.flags & PT_VOLUME_HETEROGENEOUS) && vol.density_grid != PT_NO_TEXTURE) {
                const pt_grid &gr = d->grids[vol.density_grid];
                hd[v] = DevGrid{gr.w, gr.h, gr.d, gridDev[vol.density_grid]};
                DevGrid m{(gr.w + 3) / 4, (gr.h + 3) / 4, (gr.d + 3) / 4, nullptr};
                float *md;
                PT_CUDA(ctx->alloc_scene(&md, (size_t)m.w * m.h * m.d));
                k_majorant<<<blocks_for((size_t)m.w * m.h * m.d), 256, 0, st>>>(hd[v], m, md);
                m.data = md;
                hm[v] = m;
            }
        }
        if ((rc = h2d(dvols, d->volumes, d->num_volumes * sizeof(pt_volume)))) return rc;
        if ((rc = h2d(ddens, hd.data(), hd.size() * sizeof(DevGrid)))) return rc;
        if ((rc = h2d(dmaj, hm.data(), hm.size() * sizeof(DevGrid)))) return rc;
        S.vols = dvols; S.dens = ddens; S.maj = dmaj;
    }
    PT_CUDA(cudaStreamSynchronize(st));
    ctx->clsMask = clsMask;
    ctx->hasScene = true;
    return PT_OK;
}

int pt_render(pt_ctx *ctx, const pt_render_params *p, pt_film *film, pt_stats *stats) {
    if (!ctx) return PT_E_INVALID;
    if (!p || !film || !film->sum || !film->comp) return ctx->fail(PT_E_INVALID, "null params or film");
    if (!ctx->hasScene) return ctx->fail(PT_E_NOSCENE, "no scene uploaded");
    if (!p->width || !p->height) return ctx->fail(PT_E_INVALID, "empty image");
    if (film->width != p->width || film->height != p->height) return ctx->fail(PT_E_INVALID, "film size mismatch");
    if (p->rng_kind > PT_RNG_PCG_HASH || p->env_sampling > PT_ENV_ALIAS) return ctx->fail(PT_E_INVALID, "bad enum");
    if ((uint64_t)p->width * p->height > 0x7FFFFFFFull) return ctx->fail(PT_E_INVALID, "image too large");
    if (p->spp == 0 || p->max_depth == 0) return PT_OK;
    cudaSetDevice(ctx->device);
    const size_t bytes = (size_t)p->width * p->height * 16;
    float *dsum = film->sum, *dcomp = film->comp;
    bool host = film->location == PT_MEM_HOST;
    if (host) {
        char *base;
        int rc = scratch(ctx, 2 * bytes, &base);
        if (rc) return rc;
        dsum = (float *)base;
        dcomp = (float *)(base + bytes);
        // the upload overlaps the render (only its film kernel reads the
        // film): on the copy stream, after the render stream's earlier work
        // on the staging memory
        PT_CUDA(cudaEventRecord(ctx->streamMark, ctx->stream));
        PT_CUDA(cudaStreamWaitEvent(ctx->copyStream, ctx->streamMark, 0));
        PT_CUDA(cudaMemcpyAsync(dsum, film->sum, bytes, cudaMemcpyHostToDevice, ctx->copyStream));
        PT_CUDA(cudaMemcpyAsync(dcomp, film->comp, bytes, cudaMemcpyHostToDevice, ctx->copyStream));
        PT_CUDA(cudaEventRecord(ctx->filmReady, ctx->copyStream));
    } else {
        PT_CUDA(cudaEventRecord(ctx->filmReady, ctx->stream));
    }
    int rc = pt_render_impl(ctx, p, dsum, dcomp, stats);
    if (rc) {
        // an early error return must not leave the upload in flight: the
        // staging memory is reused by the next call and the caller may free
        // the host film once this returns
        if (host) cudaStreamSynchronize(ctx->copyStream);
        return rc;
    }
    if (host) {
        PT_CUDA(cudaMemcpyAsync(film->sum, dsum, bytes, cudaMemcpyDeviceToHost, ctx->stream));
        PT_CUDA(cudaMemcpyAsync(film->comp, dcomp, bytes, cudaMemcpyDeviceToHost, ctx->stream));
        PT_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    return PT_OK;
}

int pt_bsdf_eval_batch(pt_ctx *ctx, const pt_material *materials, uint32_t nm, const uint32_t *mi, const float *wi,
                       const float *wo, const float *h, size_t n, float *f, float *pdf, uint32_t loc) {
    if (!ctx) return PT_E_INVALID;
    if (!materials || !nm || !wi || !wo || !f || !pdf) return ctx->fail(PT_E_INVALID, "null argument");
    if (!n) return PT_OK;
    cudaSetDevice(ctx->device);
    Staging s{ctx, loc, {}};
    s.add(materials, nm * sizeof(pt_material), false);
    s.add(mi, mi ? n * 4 : 0, false);
    s.add(wi, n * 12, false);
    s.add(wo, n * 12, false);
    s.add(h, h ? n * 4 : 0, false);
    s.add(f, n * 12, true);
    s.add(pdf, n * 4, true);
    int rc = s.setup();
    if (rc) return rc;
    k_bsdf_eval<<<blocks_for(n), 256, 0, ctx->stream>>>((pt_material *)s.dev(0), nm, (uint32_t *)s.dev(1),
                                                         (float *)s.dev(2), (float *)s.dev(3), (float *)s.dev(4), n,
                                                         (float *)s.dev(5), (float *)s.dev(6));
    return s.finish();
}

// ---- BSDF evaluation without any allocation ---------------------------------
// pt_bsdf_eval_batch stages host arrays through a context's scratch, which
// grows with cudaMalloc/cudaFree, and needs a context, whose creation
// allocates.  Some callers cannot allow that: a plugin that queries BSDFs on
// the side while a render keeps another stream of the same device busy
// (cudaFree synchronises the whole device and would stall that render), or a
// host that reserved its device memory up front and must not fail a query
// on an allocation later.  This variant stages through one fixed array in
// the module's static device memory instead, and runs the same kernel.
//
// Layout of the array, every part 256-byte aligned: materials, then
// mat_index, wi, wo, h, f, pdf for PT_NOALLOC_MAX_QUERIES queries.
// Nothing in it has to start at zero: each call overwrites the inputs it
// uses, the kernel reads an optional input only when the caller passed it,
// and it writes every output element below n before anything reads it.
namespace {
constexpr size_t kNaMat = (PT_NOALLOC_MAX_MATERIALS * sizeof(pt_material) + 255) & ~(size_t)255;
constexpr size_t kNaU32 = (PT_NOALLOC_MAX_QUERIES * 4 + 255) & ~(size_t)255;
constexpr size_t kNaF3 = (PT_NOALLOC_MAX_QUERIES * 12 + 255) & ~(size_t)255;
constexpr size_t kNaOffMi = kNaMat;
constexpr size_t kNaOffWi = kNaOffMi + kNaU32;
constexpr size_t kNaOffWo = kNaOffWi + kNaF3;
constexpr size_t kNaOffH = kNaOffWo + kNaF3;
constexpr size_t kNaOffF = kNaOffH + kNaU32;
constexpr size_t kNaOffPdf = kNaOffF + kNaF3;
constexpr size_t kNaBytes = kNaOffPdf + kNaU32;  // 3,182,592 bytes
static_assert(kNaBytes == 3182592, "static staging size");
constexpr int kNaMaxDevices = 64;
std::atomic<char *> g_noallocAddr[kNaMaxDevices];  // per device ordinal, set on first use
}  // namespace
static __device__ __align__(256) unsigned char g_noallocStage[kNaBytes];

int pt_bsdf_eval_batch_noalloc(void *stream, const pt_material *materials, uint32_t nm, const uint32_t *mi,
                               const float *wi, const float *wo, const float *h, size_t n, float *f, float *pdf,
                               uint32_t loc) {
    if (!materials || !nm || !wi || !wo || !f || !pdf) return PT_E_INVALID;
    if (loc != PT_MEM_HOST && loc != PT_MEM_DEVICE) return PT_E_INVALID;
    if (loc == PT_MEM_HOST && (n > PT_NOALLOC_MAX_QUERIES || nm > PT_NOALLOC_MAX_MATERIALS)) return PT_E_LIMIT;
    if (!n) return PT_OK;
    cudaStream_t st = (cudaStream_t)stream;
    if (loc == PT_MEM_DEVICE) {  // arrays used in place: no staging at all
        k_bsdf_eval<<<blocks_for(n), 256, 0, st>>>(materials, nm, mi, wi, wo, h, n, f, pdf);
        if (cudaGetLastError() != cudaSuccess) return PT_E_CUDA;
        return cudaStreamSynchronize(st) == cudaSuccess ? PT_OK : PT_E_CUDA;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return PT_E_CUDA;
    if (dev < 0 || dev >= kNaMaxDevices) return PT_E_INVALID;
    // First call on a device: look up where the array lives on it (with that
    // device current).  Two threads racing here store the same address.
    char *base = g_noallocAddr[dev].load(std::memory_order_acquire);
    if (!base) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noallocStage) != cudaSuccess || !p) return PT_E_CUDA;
        base = (char *)p;
        g_noallocAddr[dev].store(base, std::memory_order_release);
    }
    auto h2d = [&](size_t off, const void *src, size_t bytes) {
        return cudaMemcpyAsync(base + off, src, bytes, cudaMemcpyHostToDevice, st) == cudaSuccess;
    };
    if (!h2d(0, materials, nm * sizeof(pt_material)) || (mi && !h2d(kNaOffMi, mi, n * 4)) ||
        !h2d(kNaOffWi, wi, n * 12) || !h2d(kNaOffWo, wo, n * 12) || (h && !h2d(kNaOffH, h, n * 4)))
        return PT_E_CUDA;
    k_bsdf_eval<<<blocks_for(n), 256, 0, st>>>((const pt_material *)base, nm,
                                                mi ? (const uint32_t *)(base + kNaOffMi) : nullptr,
                                                (const float *)(base + kNaOffWi), (const float *)(base + kNaOffWo),
                                                h ? (const float *)(base + kNaOffH) : nullptr, n,
                                                (float *)(base + kNaOffF), (float *)(base + kNaOffPdf));
    if (cudaGetLastError() != cudaSuccess) return PT_E_CUDA;
    if (cudaMemcpyAsync(f, base + kNaOffF, n * 12, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(pdf, base + kNaOffPdf, n * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return PT_E_CUDA;
    return cudaStreamSynchronize(st) == cudaSuccess ? PT_OK : PT_E_CUDA;
}

int pt_bsdf_sample_batch(pt_ctx *ctx, const pt_material *materials, uint32_t nm, const uint32_t *mi, const float *wi,
                         const float *u, const float *h, size_t n, float *wo, float *wt, float *pdf, uint32_t loc) {
    if (!ctx) return PT_E_INVALID;
    if (!materials || !nm || !wi || !u || !wo || !wt || !pdf) return ctx->fail(PT_E_INVALID, "null argument");
    if (!n) return PT_OK;
    cudaSetDevice(ctx->device);
    Staging s{ctx, loc, {}};
    s.add(materials, nm * sizeof(pt_material), false);
    s.add(mi, mi ? n * 4 : 0, false);
    s.add(wi, n * 12, false);
    s.add(u, n * 16, false);
    s.add(h, h ? n * 4 : 0, false);
    s.add(wo, n * 12, true);
    s.add(wt, n * 12, true);
    s.add(pdf, n * 4, true);
    int rc = s.setup();
    if (rc) return rc;
    k_bsdf_sample<<<blocks_for(n), 256, 0, ctx->stream>>>((pt_material *)s.dev(0), nm, (uint32_t *)s.dev(1),
                                                           (float *)s.dev(2), (float *)s.dev(3), (float *)s.dev(4), n,
                                                           (float *)s.dev(5), (float *)s.dev(6), (float *)s.dev(7));
    return s.finish();
}

int pt_phase_sample_batch(pt_ctx *ctx, const float *g, const float *wo, const float *u, size_t n, float *wi, float *pdf,
                          uint32_t loc) {
    if (!ctx) return PT_E_INVALID;
    if (!g || !wo || !u || !wi || !pdf) return ctx->fail(PT_E_INVALID, "null argument");
    if (!n) return PT_OK;
    cudaSetDevice(ctx->device);
    Staging s{ctx, loc, {}};
    s.add(g, n * 4, false);
    s.add(wo, n * 12, false);
    s.add(u, n * 8, false);
    s.add(wi, n * 12, true);
    s.add(pdf, n * 4, true);
    int rc = s.setup();
    if (rc) return rc;
    k_phase_sample<<<blocks_for(n), 256, 0, ctx->stream>>>((float *)s.dev(0), (float *)s.dev(1), (float *)s.dev(2), n,
                                                            (float *)s.dev(3), (float *)s.dev(4));
    return s.finish();
}

int pt_env_sample_batch(pt_ctx *ctx, uint32_t mode, const float *u, size_t n, float *dir, float *rad, float *pdf,
                        uint32_t loc) {
    if (!ctx) return PT_E_INVALID;
    if (!ctx->hasScene) return ctx->fail(PT_E_NOSCENE, "no scene uploaded");
    if (!u || !dir || !rad || !pdf || mode > PT_ENV_ALIAS) return ctx->fail(PT_E_INVALID, "bad argument");
    if (!n) return PT_OK;
    cudaSetDevice(ctx->device);
    Staging s{ctx, loc, {}};
    s.add(u, n * 8, false);
    s.add(dir, n * 12, true);
    s.add(rad, n * 12, true);
    s.add(pdf, n * 4, true);
    int rc = s.setup();
    if (rc) return rc;
    k_env_sample<<<blocks_for(n), 256, 0, ctx->stream>>>(ctx->S, mode, (float *)s.dev(0), n, (float *)s.dev(1),
                                                          (float *)s.dev(2), (float *)s.dev(3));
    return s.finish();
}

int pt_env_pdf_batch(pt_ctx *ctx, uint32_t mode, const float *dir, size_t n, float *pdf, float *rad, uint32_t loc) {
    if (!ctx) return PT_E_INVALID;
    if (!ctx->hasScene) return ctx->fail(PT_E_NOSCENE, "no scene uploaded");
    if (!dir || !pdf || !rad || mode > PT_ENV_ALIAS) return ctx->fail(PT_E_INVALID, "bad argument");
    if (!n) return PT_OK;
    cudaSetDevice(ctx->device);
    Staging s{ctx, loc, {}};
    s.add(dir, n * 12, false);
    s.add(pdf, n * 4, true);
    s.add(rad, n * 12, true);
    int rc = s.setup();
    if (rc) return rc;
    k_env_pdf<<<blocks_for(n), 256, 0, ctx->stream>>>(ctx->S, mode, (float *)s.dev(0), n, (float *)s.dev(1),
                                                       (float *)s.dev(2));
    return s.finish();
}

int pt_env_read_cdf(pt_ctx *ctx, float *marginal, float *conditional) {
    if (!ctx) return PT_E_INVALID;
    if (!ctx->hasScene) return ctx->fail(PT_E_NOSCENE, "no scene uploaded");
    if (!marginal || !conditional) return ctx->fail(PT_E_INVALID, "null argument");
    cudaSetDevice(ctx->device);
    PT_CUDA(cudaMemcpyAsync(marginal, ctx->S.marg, (ctx->S.envH + 1) * 4, cudaMemcpyDeviceToHost, ctx->stream));
    PT_CUDA(cudaMemcpyAsync(conditional, ctx->S.cond, (size_t)ctx->S.envH * (ctx->S.envW + 1) * 4,
                            cudaMemcpyDeviceToHost, ctx->stream));
    PT_CUDA(cudaStreamSynchronize(ctx->stream));
    return PT_OK;
}

int pt_rng_batch(pt_ctx *ctx, uint32_t kind, const uint32_t *pix, const uint32_t *smp, size_t n, uint32_t dims,
                 uint32_t width, uint32_t height, float *out, uint32_t loc) {
    if (!ctx) return PT_E_INVALID;
    if (!pix || !smp || !out || kind > PT_RNG_PCG_HASH || !width || !height) return ctx->fail(PT_E_INVALID, "bad argument");
    if (!n || !dims) return PT_OK;
    cudaSetDevice(ctx->device);
    Staging s{ctx, loc, {}};
    s.add(pix, n * 4, false);
    s.add(smp, n * 4, false);
    s.add(out, n * dims * 4, true);
    int rc = s.setup();
    if (rc) return rc;
    k_rng<<<blocks_for(n), 256, 0, ctx->stream>>>(ctx->d_sobol1, kind, (uint32_t *)s.dev(0), (uint32_t *)s.dev(1), n,
                                                   dims, width * height, (float *)s.dev(2));
    return s.finish();
}

int pt_bvh_info(pt_ctx *ctx, uint32_t *num_triangles, uint32_t *num_wide_nodes) {
    if (!ctx) return PT_E_INVALID;
    if (!ctx->hasScene) return ctx->fail(PT_E_NOSCENE, "no scene uploaded");
    if (num_triangles) *num_triangles = ctx->numTris;
    if (num_wide_nodes) *num_wide_nodes = ctx->numWide;
    return PT_OK;
}

int pt_bvh_read(pt_ctx *ctx, uint32_t *morton, uint32_t *sorted, int32_t *nodes) {
    if (!ctx) return PT_E_INVALID;
    if (!ctx->hasScene) return ctx->fail(PT_E_NOSCENE, "no scene uploaded");
    cudaSetDevice(ctx->device);
    const uint32_t n = ctx->numTris;
    if (n == 0) return PT_OK;
    if (morton) PT_CUDA(cudaMemcpyAsync(morton, ctx->d_morton, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (sorted) PT_CUDA(cudaMemcpyAsync(sorted, ctx->d_sorted, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (nodes && n > 1)
        PT_CUDA(cudaMemcpyAsync(nodes, ctx->d_binChildren, (size_t)(n - 1) * 8, cudaMemcpyDeviceToHost, ctx->stream));
    PT_CUDA(cudaStreamSynchronize(ctx->stream));
    return PT_OK;
}

int pt_trace_closest(pt_ctx *ctx, const float *rays, size_t n, pt_hit *out, uint32_t loc) {
    if (!ctx) return PT_E_INVALID;
    if (!ctx->hasScene) return ctx->fail(PT_E_NOSCENE, "no scene uploaded");
    if (!rays || !out) return ctx->fail(PT_E_INVALID, "null argument");
    if (!n) return PT_OK;
    cudaSetDevice(ctx->device);
    Staging s{ctx, loc, {}};
    s.add(rays, n * 32, false);
    s.add(out, n * sizeof(pt_hit), true);
    int rc = s.setup();
    if (rc) return rc;
    cudaMemsetAsync(ctx->d_err, 0, 4, ctx->stream);
    k_trace_closest<<<blocks_for(n), 256, 0, ctx->stream>>>(ctx->S, (float *)s.dev(0), n, (pt_hit *)s.dev(1),
                                                             ctx->d_err);
    rc = s.finish();
    if (rc) return rc;
    uint32_t e = 0;
    cudaMemcpy(&e, ctx->d_err, 4, cudaMemcpyDeviceToHost);
    return e ? ctx->fail(PT_E_DEVICE, "traversal stack overflow") : PT_OK;
}

int pt_trace_shadow(pt_ctx *ctx, const float *rays, size_t n, uint32_t *occ, float *tr, uint32_t loc) {
    if (!ctx) return PT_E_INVALID;
    if (!ctx->hasScene) return ctx->fail(PT_E_NOSCENE, "no scene uploaded");
    if (!rays || !occ || !tr) return ctx->fail(PT_E_INVALID, "null argument");
    if (!n) return PT_OK;
    cudaSetDevice(ctx->device);
    Staging s{ctx, loc, {}};
    s.add(rays, n * 32, false);
    s.add(occ, n * 4, true);
    s.add(tr, n * 12, true);
    int rc = s.setup();
    if (rc) return rc;
    cudaMemsetAsync(ctx->d_err, 0, 4, ctx->stream);
    k_trace_shadow<<<blocks_for(n), 256, 0, ctx->stream>>>(ctx->S, (float *)s.dev(0), n, (uint32_t *)s.dev(1),
                                                            (float *)s.dev(2), ctx->d_err);
    rc = s.finish();
    if (rc) return rc;
    uint32_t e = 0;
    cudaMemcpy(&e, ctx->d_err, 4, cudaMemcpyDeviceToHost);
    return e ? ctx->fail(PT_E_DEVICE, "traversal stack overflow") : PT_OK;
}

}  // extern "C"
