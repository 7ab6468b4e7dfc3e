// pt_cache.cuh — the radiance cache's network layout, input encoding and the
// sm_100a primitives its kernels are built from (tcgen05 MMA with TMEM
// accumulators, bulk copies, mbarriers).  No counterpart in the reference:
// the cache is an addition to the path tracer (Müller et al. 2021, "Real-time
// Neural Radiance Caching for Path Tracing").
//
// Network: 64 encoded inputs -> 5 hidden layers of 64 (ReLU, no biases; input
// 49 is a constant 1) -> 16 linear outputs, of which 0..2 are RGB radiance.
// Operands are BF16, accumulation FP32.  Weight W_l is stored [out][in].
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace pt {

constexpr int kRcIn = 64;
constexpr int kRcWidth = 64;
constexpr int kRcOut = 16;         // output rows of the last layer (3 used)
constexpr int kRcLayers = 6;       // 5 hidden + output
constexpr int kRcTile = 128;       // rows per MMA tile (one TMEM lane each)
constexpr int kRcParams = 5 * kRcWidth * kRcIn + kRcOut * kRcWidth;  // 21,504
constexpr int kRcImageBytes = 2 * kRcParams;                          // 43,008
constexpr int kRcRecFloats = 16;   // a query / training record: 4 float4

__host__ __device__ constexpr int rc_rows(int l) { return l < 5 ? kRcWidth : kRcOut; }
// Offset of layer l in the canonical FP32 parameter vector ([l][out][in]).
__host__ __device__ constexpr int rc_param_base(int l) { return l * kRcWidth * kRcIn; }
// Byte offset of layer l in the BF16 weight image.
__host__ __device__ constexpr int rc_image_base(int l) { return 2 * rc_param_base(l); }

// Shared-memory image of an R x 64 BF16 operand (R rows, K = 64 columns):
// 8 x 8 "core matrices" of 128 contiguous bytes (8 rows of 16 bytes), the
// row groups of one 8-column chunk together, chunks R * 16 bytes apart.  The
// tcgen05 no-swizzle canonical layout: read K-major (rows = M or N) with
// SBO = 128 B, LBO = R * 16 B, or MN-major (rows = K) with SBO = R * 16 B,
// LBO = 128 B.  Weights live in global memory in this image so that one bulk
// copy places a layer.
__host__ __device__ constexpr uint32_t rc_core_offset(uint32_t r, uint32_t c, uint32_t R) {
    return (c >> 3) * (R * 16u) + (r >> 3) * 128u + (r & 7u) * 16u + (c & 7u) * 2u;
}

// ---- input encoding ------------------------------------------------------------
// Record (4 float4): (position, roughness), (direction toward the previous
// vertex, slot bits), (shading normal, -), (albedo, -).  Features: position
// in scene-box units [0,1]^3, sin / cos of 2^j pi p for j = 0..5 per axis,
// direction, normal, roughness, albedo, a constant 1, zeros.
constexpr int kRcFeatConst = 49;

__device__ __forceinline__ void rc_encode(const float4 q0, const float4 q1, const float4 q2, const float4 q3,
                                          const float bmin[3], const float binv[3], float f[kRcIn]) {
    const float p[3] = {(q0.x - bmin[0]) * binv[0], (q0.y - bmin[1]) * binv[1], (q0.z - bmin[2]) * binv[2]};
#pragma unroll
    for (int a = 0; a < 3; a++) f[a] = p[a];
#pragma unroll
    for (int j = 0; j < 6; j++) {
#pragma unroll
        for (int a = 0; a < 3; a++) {
            float s, c;
            sincospif(p[a] * (float)(1 << j), &s, &c);
            f[3 + 6 * j + 2 * a] = s;
            f[4 + 6 * j + 2 * a] = c;
        }
    }
    f[39] = q1.x; f[40] = q1.y; f[41] = q1.z;
    f[42] = q2.x; f[43] = q2.y; f[44] = q2.z;
    f[45] = q0.w;
    f[46] = q3.x; f[47] = q3.y; f[48] = q3.z;
    f[kRcFeatConst] = 1.0f;
#pragma unroll
    for (int k = 50; k < kRcIn; k++) f[k] = 0.0f;
}

// ---- sm_100a primitives ------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
// Shared-memory matrix descriptor, no swizzle (layout type 0), version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: BF16 A and B, FP32 D, M x N, majors.
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t M, uint32_t N, uint32_t aMN, uint32_t bMN) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (aMN << 15) | (bMN << 16) | ((N >> 3) << 17) | ((M >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t dTmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dTmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
// The same with A read from tensor memory: 128 lanes (rows of A) x K / 2
// columns, column c of lane m holding A[m][2c] (low half) and A[m][2c + 1].
__device__ __forceinline__ void umma_bf16_ts(uint32_t dTmem, uint32_t aTmem, uint64_t b, uint32_t idesc,
                                             uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(dTmem),
        "r"(aTmem), "l"(b), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
// Bounded wait for phase `parity` of an mbarrier; false after `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint32_t limit = 1u << 22) {
    for (uint32_t i = 0; i < limit; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// Global -> shared bulk copy (16-byte aligned, size a multiple of 16),
// completion counted on mbar's transaction count.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t mbar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}

// TMEM allocation by one full warp; the address is written to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t slotSmem, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slotSmem), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}

// 32 lanes x 16 / 64 consecutive FP32 columns: thread t of the warp gets lane
// (warp's quarter) * 32 + t.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float v[64]) {
    tmem_ld16(taddr, v);
    tmem_ld16(taddr + 16, v + 16);
    tmem_ld16(taddr + 32, v + 32);
    tmem_ld16(taddr + 48, v + 48);
}

// 32 lanes x 32 consecutive FP32 columns in one instruction.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float v[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// 32 lanes x 32 consecutive 32-bit columns from registers (thread t of the
// warp writes lane (warp's quarter) * 32 + t).
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t r[32]) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
                 "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
                 "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]),
                 "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]),
                 "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&h);
}
// Row r (of 128) of an activation tile, 64 values -> BF16 image.
__device__ __forceinline__ void store_row_bf16(uint8_t *tile, uint32_t r, const float v[64]) {
#pragma unroll
    for (int c = 0; c < 8; c++) {
        uint4 w = make_uint4(pack_bf16(v[8 * c], v[8 * c + 1]), pack_bf16(v[8 * c + 2], v[8 * c + 3]),
                             pack_bf16(v[8 * c + 4], v[8 * c + 5]), pack_bf16(v[8 * c + 6], v[8 * c + 7]));
        *reinterpret_cast<uint4 *>(tile + rc_core_offset(r, 8 * c, kRcTile)) = w;
    }
}
// max(a, 0) and max(b, 0) rounded to BF16 in one instruction, a in the low
// half; the same bits as pack_bf16(fmaxf(a, 0), fmaxf(b, 0)) for every
// non-NaN input (a NaN stays NaN).
__device__ __forceinline__ uint32_t pack_bf16_relu(float a, float b) {
    uint32_t d;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(b), "f"(a));
    return d;
}
__device__ __forceinline__ void load_row_bf16(const uint8_t *tile, uint32_t r, float v[64]) {
#pragma unroll
    for (int c = 0; c < 8; c++) {
        uint4 w = *reinterpret_cast<const uint4 *>(tile + rc_core_offset(r, 8 * c, kRcTile));
        const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            v[8 * c + 2 * k] = __uint_as_float(ws[k] << 16);
            v[8 * c + 2 * k + 1] = __uint_as_float(ws[k] & 0xFFFF0000u);
        }
    }
}

}  // namespace pt
