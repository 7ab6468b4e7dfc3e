// pt_bvh.cu — GPU acceleration-structure build of libpt.
//
// Replaces the driver's BLAS/TLAS build (src/gpu/DXRApp_Scene.cpp:37-170 of
// gracejinsotrue/PBRT-renderer-) with:
//   1. per-triangle bounds and 30-bit Morton codes of the centroids,
//   2. a stable radix sort of (code, triangle id): four 8-bit passes of
//      per-tile digit counts, one scan, and an order-keeping scatter,
//   3. the Karras 2012 binary radix tree over the sorted codes (ties broken by
//      position, so the topology is a pure function of the input),
//   4. bottom-up bounds with one atomic per internal node,
//   5. treelet restructuring (Karras & Aila 2013, "Fast Parallel Construction
//      of High-Quality Bounding Volume Hierarchies"): in bottom-up passes,
//      every node with >= 7 triangles below grows a treelet of 7 leaves by
//      opening its largest-area leaf, finds the topology of least surface-area
//      cost over those leaves by dynamic programming over the 127 leaf
//      subsets, and rewires the treelet's 6 internal nodes to it when that
//      lowers the cost,
//   6. a top-down collapse into 8-wide nodes: each wide node takes its binary
//      root's two children and repeatedly opens the child with the largest
//      surface area until it has 8; subtrees of <= 3 triangles become leaves.
//      Child boxes are quantised to 8 bits per plane against a power-of-two
//      grid with directed rounding, so every stored box contains its child.
//      Trees too large for the L2 are collapsed instead by a least-area
//      plan (dynamic programming over the binary tree); a result deeper than
//      the traversal stack is collapsed the other way, then, if still too
//      deep, from the radix tree.
#include "pt_internal.h"

namespace pt {

constexpr uint32_t kLeafMax = 3;

// ---- stable LSD radix sort of (code, id) pairs, 8-bit digits -------------------
// One pass per digit (shift 0, 8, 16, 24).  k_rs_hist counts each tile's
// digits, stored digit-major (hist[d * tiles + tile]) so that one exclusive
// scan gives every (digit, tile) its first output position; k_rs_scatter
// walks its tile in rounds of 256 keys in input order and places each key at
// its digit's next position plus its rank among the round's equal digits
// (earlier warps, then earlier lanes: __match_any_sync), so equal keys keep
// their order and the result is the unique stable sort.
constexpr uint32_t kRsThreads = 256, kRsRounds = 64, kRsTile = kRsThreads * kRsRounds;  // 16,384 keys per tile
__global__ void __launch_bounds__(kRsThreads) k_rs_hist(const uint32_t *keys, uint32_t n, uint32_t shift,
                                                        uint32_t tiles, uint32_t *hist) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0u;
    __syncthreads();
    const uint32_t base = blockIdx.x * kRsTile;
    for (uint32_t i = threadIdx.x; i < kRsTile; i += kRsThreads) {
        const uint32_t j = base + i;
        if (j < n) atomicAdd(&h[(keys[j] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}
// One block: exclusive scan of m counts in place (contiguous runs per thread).
__global__ void __launch_bounds__(1024) k_rs_scan(uint32_t *a, uint32_t m) {
    __shared__ uint32_t part[1024];
    const uint32_t t = threadIdx.x, per = (m + 1023) / 1024, lo = min(m, t * per), hi = min(m, lo + per);
    uint32_t sum = 0;
    for (uint32_t i = lo; i < hi; i++) sum += a[i];
    part[t] = sum;
    __syncthreads();
    for (uint32_t o = 1; o < 1024; o <<= 1) {
        const uint32_t v = t >= o ? part[t - o] : 0u;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    uint32_t run = part[t] - sum;
    for (uint32_t i = lo; i < hi; i++) {
        const uint32_t c = a[i];
        a[i] = run;
        run += c;
    }
}
__global__ void __launch_bounds__(kRsThreads) k_rs_scatter(const uint32_t *keys, const uint32_t *vals, uint32_t n,
                                                           uint32_t shift, uint32_t tiles, const uint32_t *off,
                                                           uint32_t *keysOut, uint32_t *valsOut) {
    constexpr uint32_t kWarps = kRsThreads / 32;
    __shared__ uint32_t next[256];          // this tile's next output position of each digit
    __shared__ uint32_t wcnt[kWarps][256];  // the current round's count of each digit per warp
    const uint32_t t = threadIdx.x, lane = t & 31u, w = t >> 5;
    next[t] = off[t * tiles + blockIdx.x];
    const uint32_t base = blockIdx.x * kRsTile;
    for (uint32_t r = 0; r < kRsRounds; r++) {
#pragma unroll
        for (uint32_t k = 0; k < kWarps; k++) wcnt[k][t] = 0u;  // thread t owns column t
        __syncthreads();
        const uint32_t j = base + r * kRsThreads + t;
        const bool valid = j < n;
        uint32_t key = 0u, val = 0u, d = 256u + lane;  // past the end: a digit no other lane has
        if (valid) {
            key = keys[j];
            val = vals[j];
            d = (key >> shift) & 255u;
        }
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
        if (valid && lane == (uint32_t)__ffs(peers) - 1u) wcnt[w][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            uint32_t pos = next[d] + __popc(peers & ((1u << lane) - 1u));
            for (uint32_t k = 0; k < w; k++) pos += wcnt[k][d];
            keysOut[pos] = key;
            valsOut[pos] = val;
        }
        __syncthreads();
        uint32_t tot = 0u;
#pragma unroll
        for (uint32_t k = 0; k < kWarps; k++) tot += wcnt[k][t];
        next[t] += tot;  // read by other threads only after the next round's first barrier
    }
}

__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

// Triangle bounds, mesh of each triangle and centroid (exact float ops).
__global__ void k_tri_bounds(uint32_t n, const uint32_t *__restrict__ meshFirstTri, uint32_t numMeshes,
                             const pt_material *__restrict__ mats, const uint32_t *__restrict__ idx,
                             const float *__restrict__ pos, uint32_t *triMesh, float4 *lo, float4 *hi,
                             float4 *cen) {
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    uint32_t a = 0, b = numMeshes;  // last mesh with meshFirstTri <= g
    while (b - a > 1) {
        uint32_t m = (a + b) >> 1;
        if (meshFirstTri[m] <= g) a = m; else b = m;
    }
    const pt_material &m = mats[a];
    uint32_t base = m.indexOffset + 3u * (g - meshFirstTri[a]);
    float3 p0 = ld3(pos, m.vertexOffset + idx[base]);
    float3 p1 = ld3(pos, m.vertexOffset + idx[base + 1]);
    float3 p2 = ld3(pos, m.vertexOffset + idx[base + 2]);
    float3 l = vmin(p0, vmin(p1, p2)), h = vmax(p0, vmax(p1, p2));
    triMesh[g] = a;
    lo[g] = make_float4(l.x, l.y, l.z, 0.0f);
    hi[g] = make_float4(h.x, h.y, h.z, 0.0f);
    cen[g] = make_float4(__fmul_rn(__fadd_rn(l.x, h.x), 0.5f), __fmul_rn(__fadd_rn(l.y, h.y), 0.5f),
                         __fmul_rn(__fadd_rn(l.z, h.z), 0.5f), 0.0f);
}

__device__ __forceinline__ uint32_t f2ord(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}
// bounds[0..2] = ordered min, bounds[3..5] = ordered max of the centroids
__global__ void k_centroid_bounds(uint32_t n, const float4 *__restrict__ cen, uint32_t *bounds) {
    uint32_t mn3[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, mx3[3] = {0u, 0u, 0u};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 c = cen[i];
        float v[3] = {c.x, c.y, c.z};
        for (int a = 0; a < 3; a++) {
            uint32_t o = f2ord(v[a]);
            mn3[a] = min(mn3[a], o);
            mx3[a] = max(mx3[a], o);
        }
    }
    for (int a = 0; a < 3; a++) {
        for (int off = 16; off; off >>= 1) {
            mn3[a] = min(mn3[a], __shfl_xor_sync(0xFFFFFFFFu, mn3[a], off));
            mx3[a] = max(mx3[a], __shfl_xor_sync(0xFFFFFFFFu, mx3[a], off));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&bounds[a], mn3[a]);
            atomicMax(&bounds[3 + a], mx3[a]);
        }
    }
}
__global__ void k_morton(uint32_t n, const float4 *__restrict__ cen, const uint32_t *__restrict__ bounds,
                         uint32_t *codes, uint32_t *ids) {
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    float4 c = cen[g];
    float v[3] = {c.x, c.y, c.z};
    uint32_t q[3];
    for (int a = 0; a < 3; a++) {
        float lo = ord2f(bounds[a]), hi = ord2f(bounds[3 + a]);
        float ext = __fsub_rn(hi, lo);
        float x = ext > 0.0f ? __fdiv_rn(__fsub_rn(v[a], lo), ext) : 0.0f;
        float s = fminf(fmaxf(__fmul_rn(x, 1024.0f), 0.0f), 1023.0f);
        q[a] = (uint32_t)s;
    }
    codes[g] = (expand_bits(q[0]) << 2) | (expand_bits(q[1]) << 1) | expand_bits(q[2]);
    ids[g] = g;
}

__device__ __forceinline__ int delta(const uint32_t *k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    uint32_t a = k[i], b = k[j];
    if (a == b) return 32 + __clz((uint32_t)(i ^ j));
    return __clz(a ^ b);
}
// Karras 2012, Figure 4: internal node i of the radix tree over sorted keys.
__global__ void k_karras(int n, const uint32_t *__restrict__ keys, int32_t *children, int32_t *intParent,
                         int32_t *leafParent, uint32_t *rangeFirst, uint32_t *rangeLast) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = delta(keys, n, i, i - d);
    int lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2)
        if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = delta(keys, n, i, j);
    int s = 0, div = 2, t = (l + div - 1) / div;
    for (;;) {
        if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
        if (t == 1) break;
        div *= 2;
        t = (l + div - 1) / div;
    }
    int gamma = i + s * d + min(d, 0);
    int lo = min(i, j), hi = max(i, j);
    int left = (lo == gamma) ? ~gamma : gamma;
    int right = (hi == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    children[2 * i] = left;
    children[2 * i + 1] = right;
    if (left >= 0) intParent[left] = i; else leafParent[~left] = i;
    if (right >= 0) intParent[right] = i; else leafParent[~right] = i;
    rangeFirst[i] = lo;
    rangeLast[i] = hi;
    if (i == 0) intParent[0] = -1;
}
__global__ void k_refit(int n, const uint32_t *__restrict__ sorted, const float4 *__restrict__ tlo,
                        const float4 *__restrict__ thi, const int32_t *__restrict__ children,
                        const int32_t *__restrict__ intParent, const int32_t *__restrict__ leafParent,
                        float4 *leafLo, float4 *leafHi, float4 *intLo, float4 *intHi, uint32_t *flags) {
    int leaf = blockIdx.x * blockDim.x + threadIdx.x;
    if (leaf >= n) return;
    uint32_t g = sorted[leaf];
    leafLo[leaf] = tlo[g];
    leafHi[leaf] = thi[g];
    if (n == 1) return;
    int node = leafParent[leaf];
    for (int guard = 0; node >= 0 && guard < n; guard++) {
        __threadfence();
        if (atomicAdd(&flags[node], 1u) == 0u) return;  // first arrival: sibling finishes the node
        int c0 = children[2 * node], c1 = children[2 * node + 1];
        float4 l0 = c0 >= 0 ? __ldcg(&intLo[c0]) : __ldcg(&leafLo[~c0]);
        float4 h0 = c0 >= 0 ? __ldcg(&intHi[c0]) : __ldcg(&leafHi[~c0]);
        float4 l1 = c1 >= 0 ? __ldcg(&intLo[c1]) : __ldcg(&leafLo[~c1]);
        float4 h1 = c1 >= 0 ? __ldcg(&intHi[c1]) : __ldcg(&leafHi[~c1]);
        intLo[node] = make_float4(fminf(l0.x, l1.x), fminf(l0.y, l1.y), fminf(l0.z, l1.z), 0.0f);
        intHi[node] = make_float4(fmaxf(h0.x, h1.x), fmaxf(h0.y, h1.y), fmaxf(h0.z, h1.z), 0.0f);
        node = intParent[node];
    }
}

// Triangles under each internal node of the radix tree (its key range).
__global__ void k_range_count(int n, const uint32_t *__restrict__ rangeFirst, const uint32_t *__restrict__ rangeLast,
                              uint32_t *cnt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n - 1) cnt[i] = rangeLast[i] - rangeFirst[i] + 1u;
}

__device__ __forceinline__ float area(float4 l, float4 h) {
    float dx = h.x - l.x, dy = h.y - l.y, dz = h.z - l.z;
    return dx * dy + dy * dz + dz * dx;
}

// ---- treelet restructuring --------------------------------------------------
// Surface-area cost of a binary subtree: kCostNode x area of every internal
// node + kCostTri x area of every triangle leaf (areas of the boxes).
constexpr float kCostNode = 1.2f, kCostTri = 1.0f;
constexpr int kTreeletLeaves = 7;
constexpr uint32_t kTreeletMinTris = 7;
constexpr int kTreeletPasses = 3;

struct TreeletIn {
    int n;
    int32_t *children;                // rewired in place
    int32_t *intParent, *leafParent;  // rewired in place
    const float4 *leafLo, *leafHi;
    float4 *intLo, *intHi;            // treelet internal nodes get the bounds of their new subtrees
    float *cost;                      // subtree cost of each internal node
    uint32_t *cnt;                    // triangles under each internal node
    uint32_t *flags;                  // arrivals per internal node, zero before each pass
    uint32_t *rewired;                // treelets rewired in this pass
};

__device__ __forceinline__ void node_box(const TreeletIn &T, int32_t x, float4 &lo, float4 &hi) {
    lo = x >= 0 ? __ldcg(&T.intLo[x]) : T.leafLo[~x];
    hi = x >= 0 ? __ldcg(&T.intHi[x]) : T.leafHi[~x];
}

// Treelet of root R (whose two children are c0, c1 and whose subtree cost is
// `cur` as the tree stands): returns the subtree cost after the step.
__device__ float treelet_restructure(const TreeletIn &T, int32_t R, int32_t c0, int32_t c1, float cur) {
    int32_t L[kTreeletLeaves], I[kTreeletLeaves - 1];
    float4 lo[kTreeletLeaves], hi[kTreeletLeaves];
    float la[kTreeletLeaves];
    int m = 2, ni = 1;
    I[0] = R;
    L[0] = c0;
    L[1] = c1;
    for (int i = 0; i < 2; i++) {
        node_box(T, L[i], lo[i], hi[i]);
        la[i] = area(lo[i], hi[i]);
    }
    while (m < kTreeletLeaves) {  // open the internal leaf of largest area
        int best = -1;
        float ba = -1.0f;
        for (int i = 0; i < m; i++)
            if (L[i] >= 0 && la[i] > ba) { ba = la[i]; best = i; }
        if (best < 0) break;
        int32_t x = L[best];
        I[ni++] = x;
        L[best] = __ldcg(&T.children[2 * x]);
        L[m] = __ldcg(&T.children[2 * x + 1]);
        node_box(T, L[best], lo[best], hi[best]);
        node_box(T, L[m], lo[m], hi[m]);
        la[best] = area(lo[best], hi[best]);
        la[m] = area(lo[m], hi[m]);
        m++;
    }
    if (m < 3) return cur;
    float copt[1 << kTreeletLeaves];
    uint8_t part[1 << kTreeletLeaves];
    const uint32_t full = (1u << m) - 1u;
    for (int i = 0; i < m; i++)
        copt[1u << i] = L[i] >= 0 ? __ldcg(&T.cost[L[i]]) : kCostTri * la[i];
    // subsets in increasing order: every proper subset of S is smaller than S
    for (uint32_t S = 3; S <= full; S++) {
        if (__popc(S) < 2) continue;
        float4 bl = make_float4(3e38f, 3e38f, 3e38f, 0.0f), bh = make_float4(-3e38f, -3e38f, -3e38f, 0.0f);
        for (uint32_t b = S; b; b &= b - 1) {
            int i = __ffs(b) - 1;
            bl = make_float4(fminf(bl.x, lo[i].x), fminf(bl.y, lo[i].y), fminf(bl.z, lo[i].z), 0.0f);
            bh = make_float4(fmaxf(bh.x, hi[i].x), fmaxf(bh.y, hi[i].y), fmaxf(bh.z, hi[i].z), 0.0f);
        }
        const uint32_t low = S & (0u - S);
        float best = 3e38f;
        uint32_t bp = low;
        // splits (P, S \ P) with P holding the lowest leaf of S: each once
        for (uint32_t P = (S - 1u) & S; P; P = (P - 1u) & S) {
            if (!(P & low)) continue;
            float c = copt[P] + copt[S ^ P];
            if (c < best) { best = c; bp = P; }
        }
        copt[S] = kCostNode * area(bl, bh) + best;
        part[S] = (uint8_t)bp;
    }
    if (!(copt[full] < cur * 0.99999f)) return cur;
    // rewire: the subset of each new internal node, R first
    uint32_t stS[kTreeletLeaves - 1];
    int32_t stN[kTreeletLeaves - 1];
    int sp = 0, used = 1;
    stS[sp] = full;
    stN[sp++] = R;
    while (sp > 0) {
        --sp;
        const uint32_t S = stS[sp];
        const int32_t node = stN[sp];
        const uint32_t side[2] = {part[S], S ^ part[S]};
        uint32_t tris = 0;
        float4 bl = make_float4(3e38f, 3e38f, 3e38f, 0.0f), bh = make_float4(-3e38f, -3e38f, -3e38f, 0.0f);
        for (int k = 0; k < 2; k++) {
            int32_t c;
            if (__popc(side[k]) == 1) {
                c = L[__ffs(side[k]) - 1];
            } else {
                c = I[used++];
                stS[sp] = side[k];
                stN[sp++] = c;
            }
            T.children[2 * node + k] = c;
            if (c >= 0) T.intParent[c] = node;
            else T.leafParent[~c] = node;
        }
        for (uint32_t b = S; b; b &= b - 1) {
            int i = __ffs(b) - 1;
            bl = make_float4(fminf(bl.x, lo[i].x), fminf(bl.y, lo[i].y), fminf(bl.z, lo[i].z), 0.0f);
            bh = make_float4(fmaxf(bh.x, hi[i].x), fmaxf(bh.y, hi[i].y), fmaxf(bh.z, hi[i].z), 0.0f);
            tris += L[i] >= 0 ? __ldcg(&T.cnt[L[i]]) : 1u;
        }
        if (node != R) {
            T.intLo[node] = bl;
            T.intHi[node] = bh;
            T.cost[node] = copt[S];
            T.cnt[node] = tris;
        }
    }
    atomicAdd(T.rewired, 1u);
    return copt[full];
}

// One bottom-up pass, one thread per triangle leaf: the second thread to
// reach an internal node finishes it (both subtrees are final by then).
__global__ void k_treelet(TreeletIn T) {
    int leaf = blockIdx.x * blockDim.x + threadIdx.x;
    if (leaf >= T.n || T.n < 2) return;
    int32_t node = __ldcg(&T.leafParent[leaf]);
    for (int guard = 0; node >= 0 && guard < T.n; guard++) {
        __threadfence();
        if (atomicAdd(&T.flags[node], 1u) == 0u) return;
        __threadfence();
        int32_t c0 = __ldcg(&T.children[2 * node]), c1 = __ldcg(&T.children[2 * node + 1]);
        float4 l, h;
        node_box(T, c0, l, h);
        float k0 = c0 >= 0 ? __ldcg(&T.cost[c0]) : kCostTri * area(l, h);
        uint32_t n0 = c0 >= 0 ? __ldcg(&T.cnt[c0]) : 1u;
        node_box(T, c1, l, h);
        float k1 = c1 >= 0 ? __ldcg(&T.cost[c1]) : kCostTri * area(l, h);
        uint32_t n1 = c1 >= 0 ? __ldcg(&T.cnt[c1]) : 1u;
        node_box(T, node, l, h);
        float c = kCostNode * area(l, h) + k0 + k1;
        if (n0 + n1 >= kTreeletMinTris) c = treelet_restructure(T, node, c0, c1, c);
        T.cost[node] = c;
        T.cnt[node] = n0 + n1;
        node = __ldcg(&T.intParent[node]);
    }
}

// ---- collapse plan: least summed area of the wide nodes (Ylitie, Karras and
// Laine 2017, "Efficient Incoherent Ray Traversal on GPUs Through Compressed
// Wide BVHs", section 3) -------------------------------------------------------
// Leaf slots are the maximal subtrees of <= kLeafMax triangles, a fixed set,
// so the tree's cost that the collapse can change is the summed box area of
// its wide nodes.  cost[8 node + i - 1]: the least such sum over node's
// subtree when it takes at most i child slots of the wide node above it
// (leaf slots: 0).  plan[8 node + i - 1]: 0 = node fills one slot itself (a
// leaf slot or a wide node of its own), k > 0 = node is opened, k slots to
// its first child and i - k to its second.  planW[node]: the split of node's
// own 8 slots when it is a wide node.  Bottom-up like k_refit.
__global__ void k_wide_plan(int n, const int32_t *__restrict__ children, const int32_t *__restrict__ intParent,
                            const int32_t *__restrict__ leafParent, const uint32_t *__restrict__ cnt,
                            const float4 *__restrict__ intLo, const float4 *__restrict__ intHi, float *cost,
                            uint8_t *plan, uint8_t *planW, uint32_t *flags) {
    int leaf = blockIdx.x * blockDim.x + threadIdx.x;
    if (leaf >= n || n == 1) return;
    int node = leafParent[leaf];
    for (int guard = 0; node >= 0 && guard < n; guard++) {
        __threadfence();
        if (atomicAdd(&flags[node], 1u) == 0u) return;  // first arrival: sibling finishes the node
        float *cn = cost + 8 * (size_t)node;
        uint8_t *pn = plan + 8 * (size_t)node;
        if (cnt[node] <= kLeafMax) {
            for (int i = 0; i < 8; i++) { cn[i] = 0.0f; pn[i] = 0; }
            planW[node] = 0;
        } else {
            const int32_t c0 = children[2 * node], c1 = children[2 * node + 1];
            float d0[8], d1[8];
            const bool w0 = c0 >= 0 && cnt[c0] > kLeafMax, w1 = c1 >= 0 && cnt[c1] > kLeafMax;
            for (int i = 0; i < 8; i++) {
                d0[i] = w0 ? __ldcg(cost + 8 * (size_t)c0 + i) : 0.0f;
                d1[i] = w1 ? __ldcg(cost + 8 * (size_t)c1 + i) : 0.0f;
            }
            // j slots split between the children, each at least one: the least sum, first k on ties
            auto split = [&](int j, int &bk) {
                float b = 3.0e38f;
                bk = 1;
                for (int k = 1; k < j; k++) {
                    const float v = d0[k - 1] + d1[j - k - 1];
                    if (v < b) { b = v; bk = k; }
                }
                return b;
            };
            int kw;
            const float single = area(intLo[node], intHi[node]) + split(8, kw);
            planW[node] = (uint8_t)kw;
            cn[0] = single;
            pn[0] = 0;
            for (int j = 2; j <= 8; j++) {
                int k;
                const float sj = split(j, k);
                if (sj < single) { cn[j - 1] = sj; pn[j - 1] = (uint8_t)k; }
                else { cn[j - 1] = single; pn[j - 1] = 0; }
            }
        }
        node = intParent[node];
    }
}

struct CollapseIn {
    int n;
    const int32_t *children;
    const uint32_t *cnt;  // triangles under each internal node
    uint32_t maxWide;     // capacity of `nodes`
    const float4 *leafLo, *leafHi, *intLo, *intHi;
    const uint32_t *sorted;
    const uint32_t *triMesh, *meshFirstTri;
    const pt_material *mats;
    const uint32_t *idx;
    const float *pos;
    BVH8Node *nodes;
    float4 *tri;
    uint32_t *counters;  // [0] wide nodes allocated, [1] triangles written, [2] next queue size, [3] error
    const uint8_t *plan, *planW;  // k_wide_plan's choices (null: open the largest child until 8)
};

// Exponent e (biased) with (hi - lo) / 2^(e-127) <= 255, from an upper bound.
__device__ __forceinline__ uint32_t quant_exp(float lo, float hi) {
    float r = __fdiv_ru(__fsub_ru(hi, lo), 255.0f);
    uint32_t b = __float_as_uint(r);
    uint32_t e = (b >> 23) & 0xFFu;
    if (b & 0x7FFFFFu) e += 1;
    return max(e, 1u);
}

// One thread per wide node of the current level.
__global__ void k_collapse(CollapseIn C, const int2 *__restrict__ qin, uint32_t qn, int2 *qout) {
    uint32_t qi = blockIdx.x * blockDim.x + threadIdx.x;
    if (qi >= qn) return;
    int2 item = qin[qi];
    int32_t root = item.x;  // binary node (>= 0 internal, < 0 leaf)
    uint32_t wide = (uint32_t)item.y;
    int32_t ch[8];
    int cnt = 0;
    if (root >= 0) {
        ch[0] = C.children[2 * root];
        ch[1] = C.children[2 * root + 1];
        cnt = 2;
    } else {
        ch[0] = root;
        cnt = 1;
    }
    auto openable = [&](int32_t r) { return r >= 0 && C.cnt[r] > kLeafMax; };
    if (root >= 0 && C.plan && openable(root)) {  // (a root of <= kLeafMax triangles keeps its two children)
        // the plan's children: (binary node, slots) pairs, first child first;
        // the slots on the stack sum to at most 8, one or more each
        int32_t stn[8];
        int sts[8], sp = 0;
        const int kw = C.planW[root];
        stn[sp] = ch[1]; sts[sp++] = 8 - kw;
        stn[sp] = ch[0]; sts[sp++] = kw;
        cnt = 0;
        while (sp > 0) {
            const int32_t m = stn[--sp];
            const int j = sts[sp];
            const int k = openable(m) ? C.plan[8 * (size_t)m + j - 1] : 0;
            if (k <= 0 || k >= j) { ch[cnt++] = m; continue; }
            stn[sp] = C.children[2 * m + 1]; sts[sp++] = j - k;
            stn[sp] = C.children[2 * m]; sts[sp++] = k;
        }
    }
    while (!C.plan && cnt < 8) {
        int best = -1;
        float ba = -1.0f;
        for (int i = 0; i < cnt; i++)
            if (openable(ch[i])) {
                float a = area(C.intLo[ch[i]], C.intHi[ch[i]]);
                if (a > ba) { ba = a; best = i; }
            }
        if (best < 0) break;
        int32_t r = ch[best];
        ch[best] = C.children[2 * r];
        ch[cnt++] = C.children[2 * r + 1];
    }
    float4 clo[8], chi[8];
    float4 nlo = make_float4(3e38f, 3e38f, 3e38f, 0), nhi = make_float4(-3e38f, -3e38f, -3e38f, 0);
    for (int i = 0; i < cnt; i++) {
        int32_t r = ch[i];
        clo[i] = r >= 0 ? C.intLo[r] : C.leafLo[~r];
        chi[i] = r >= 0 ? C.intHi[r] : C.leafHi[~r];
        nlo = make_float4(fminf(nlo.x, clo[i].x), fminf(nlo.y, clo[i].y), fminf(nlo.z, clo[i].z), 0);
        nhi = make_float4(fmaxf(nhi.x, chi[i].x), fmaxf(nhi.y, chi[i].y), fmaxf(nhi.z, chi[i].z), 0);
    }
    // slot assignment by octant of the child centre
    float cx = 0.5f * (nlo.x + nhi.x), cy = 0.5f * (nlo.y + nhi.y), cz = 0.5f * (nlo.z + nhi.z);
    int slotOf[8];
    uint32_t used = 0;
    for (int i = 0; i < cnt; i++) {
        float mx_ = 0.5f * (clo[i].x + chi[i].x), my_ = 0.5f * (clo[i].y + chi[i].y), mz_ = 0.5f * (clo[i].z + chi[i].z);
        uint32_t o = (mx_ > cx ? 1u : 0u) | (my_ > cy ? 2u : 0u) | (mz_ > cz ? 4u : 0u);
        int best = -1, bd = 99;
        for (uint32_t s = 0; s < 8; s++)
            if (!((used >> s) & 1u)) {
                int dd = __popc(s ^ o);
                if (dd < bd) { bd = dd; best = (int)s; }
            }
        slotOf[i] = best;
        used |= 1u << best;
    }
    int child[8];
    for (int s = 0; s < 8; s++) child[s] = -1;
    for (int i = 0; i < cnt; i++) child[slotOf[i]] = i;
    // allocation
    uint32_t nInt = 0, nTri = 0, imask = 0;
    for (int s = 0; s < 8; s++) {
        if (child[s] < 0) continue;
        int32_t r = ch[child[s]];
        if (openable(r)) { nInt++; imask |= 1u << s; }
        else nTri += r >= 0 ? C.cnt[r] : 1u;
    }
    uint32_t childBase = nInt ? atomicAdd(&C.counters[0], nInt) : 0u;
    uint32_t triBase = atomicAdd(&C.counters[1], nTri);
    uint32_t qpos = nInt ? atomicAdd(&C.counters[2], nInt) : 0u;
    // a malformed tree (more nodes, queue entries or triangles than the
    // buffers hold) is reported, never written past the buffers
    if ((uint64_t)childBase + nInt > C.maxWide || (uint64_t)qpos + nInt > (uint64_t)C.n ||
        (uint64_t)triBase + nTri > (uint64_t)C.n || wide >= C.maxWide) {
        atomicOr(&C.counters[3], 2u);
        return;
    }
    // quantisation grid
    uint32_t ex = quant_exp(nlo.x, nhi.x), ey = quant_exp(nlo.y, nhi.y), ez = quant_exp(nlo.z, nhi.z);
    float ix = __uint_as_float((254u - ex) << 23), iy = __uint_as_float((254u - ey) << 23),
          iz = __uint_as_float((254u - ez) << 23);  // 2^(127 - e)
    uint8_t meta[8], qlx[8], qly[8], qlz[8], qhx[8], qhy[8], qhz[8];
    uint32_t rank = 0, toff = 0;
    for (int s = 0; s < 8; s++) {
        meta[s] = 0;
        qlx[s] = qly[s] = qlz[s] = 255;
        qhx[s] = qhy[s] = qhz[s] = 0;
        if (child[s] < 0) continue;
        int i = child[s];
        int32_t r = ch[i];
        qlx[s] = (uint8_t)min(255.0f, fmaxf(0.0f, floorf(__fmul_rd(__fsub_rd(clo[i].x, nlo.x), ix))));
        qly[s] = (uint8_t)min(255.0f, fmaxf(0.0f, floorf(__fmul_rd(__fsub_rd(clo[i].y, nlo.y), iy))));
        qlz[s] = (uint8_t)min(255.0f, fmaxf(0.0f, floorf(__fmul_rd(__fsub_rd(clo[i].z, nlo.z), iz))));
        qhx[s] = (uint8_t)min(255.0f, fmaxf(0.0f, ceilf(__fmul_ru(__fsub_ru(chi[i].x, nlo.x), ix))));
        qhy[s] = (uint8_t)min(255.0f, fmaxf(0.0f, ceilf(__fmul_ru(__fsub_ru(chi[i].y, nlo.y), iy))));
        qhz[s] = (uint8_t)min(255.0f, fmaxf(0.0f, ceilf(__fmul_ru(__fsub_ru(chi[i].z, nlo.z), iz))));
        // meta = (hit bits << 5) | bit position: an internal child sets bit
        // 24 + slot, a leaf sets one bit per triangle from its offset up
        // (< 24: at most 8 leaves of kLeafMax <= 3 triangles).
        if ((imask >> s) & 1u) {
            meta[s] = (uint8_t)(0x20u | 24u | s);
            qout[qpos + rank] = make_int2(r, (int)(childBase + rank));
            rank++;
        } else {
            // the subtree's triangle leaves, left to right (<= kLeafMax)
            uint32_t lv[kLeafMax], count = 0;
            int32_t stk[kLeafMax + 1];
            int sp = 0;
            stk[sp++] = r;
            while (sp > 0) {
                int32_t x = stk[--sp];
                if (x < 0) {
                    if (count < kLeafMax) lv[count++] = (uint32_t)(~x);
                } else if (sp + 2 <= (int)kLeafMax + 1) {
                    stk[sp++] = C.children[2 * x + 1];
                    stk[sp++] = C.children[2 * x];
                }
            }
            const uint32_t want = r >= 0 ? C.cnt[r] : 1u;  // the count this node allocated
            if (count != want || toff + count > nTri) {
                atomicOr(&C.counters[3], 1u);
                count = min(min(count, want), nTri - min(toff, nTri));
            }
            meta[s] = (uint8_t)((((1u << count) - 1u) << 5) | toff);
            for (uint32_t k = 0; k < count; k++) {
                uint32_t g = C.sorted[lv[k]];
                uint32_t mesh = C.triMesh[g];
                const pt_material &m = C.mats[mesh];
                uint32_t base = m.indexOffset + 3u * (g - C.meshFirstTri[mesh]);
                float3 p0 = ld3(C.pos, m.vertexOffset + C.idx[base]);
                float3 p1 = ld3(C.pos, m.vertexOffset + C.idx[base + 1]);
                float3 p2 = ld3(C.pos, m.vertexOffset + C.idx[base + 2]);
                float3 e1 = p1 - p0, e2 = p2 - p0;
                float4 *t = C.tri + 3u * (triBase + toff + k);
                t[0] = make_float4(p0.x, p0.y, p0.z, __uint_as_float(g));
                t[1] = make_float4(e1.x, e1.y, e1.z, __uint_as_float(m.alphaTexIndex != PT_NO_TEXTURE ? 1u : 0u));
                t[2] = make_float4(e2.x, e2.y, e2.z, 0.0f);
            }
            toff += count;
        }
    }
    auto pack4 = [](const uint8_t *b) {
        return (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
    };
    BVH8Node nd;
    nd.n[0] = make_uint4(__float_as_uint(nlo.x), __float_as_uint(nlo.y), __float_as_uint(nlo.z),
                         ex | (ey << 8) | (ez << 16) | (imask << 24));
    nd.n[1] = make_uint4(childBase, triBase, pack4(meta), pack4(meta + 4));
    nd.n[2] = make_uint4(pack4(qlx), pack4(qlx + 4), pack4(qly), pack4(qly + 4));
    nd.n[3] = make_uint4(pack4(qlz), pack4(qlz + 4), pack4(qhx), pack4(qhx + 4));
    nd.n[4] = make_uint4(pack4(qhy), pack4(qhy + 4), pack4(qhz), pack4(qhz + 4));
    C.nodes[wide] = nd;
}

}  // namespace pt

using namespace pt;

// Exact floating-point bounds are needed by the element subtraction in
// k_collapse's e1/e2: they use the same IEEE subtraction as the oracle.
int pt_build_bvh_device(pt_ctx *ctx, const uint32_t *d_meshFirstTri, uint32_t n) {
    cudaStream_t st = ctx->stream;
    DevScene &S = ctx->S;
    ctx->numTris = n;
    ctx->numWide = 0;
    S.numTris = n;
    S.numNodes = 0;
    if (n == 0) return PT_OK;
    uint32_t *triMesh, *codes, *ids, *codesS, *idsS, *bounds, *flags, *counters, *rf, *rl;
    float4 *tlo, *thi, *cen, *leafLo, *leafHi, *intLo, *intHi;
    int32_t *children, *intParent, *leafParent;
    PT_CUDA(ctx->alloc_scene(&triMesh, n));
    PT_CUDA(ctx->alloc_scene(&codes, n));
    PT_CUDA(ctx->alloc_scene(&codesS, n));
    PT_CUDA(ctx->alloc_scene(&idsS, n));
    PT_CUDA(ctx->alloc_scene(&children, 2 * (size_t)max(n - 1, 1u)));
    // temporaries
    std::vector<void *> tmp;
    auto talloc = [&](void **p, size_t bytes) {
        cudaError_t e = cudaMalloc(p, bytes + 16);
        if (e == cudaSuccess) tmp.push_back(*p);
        return e;
    };
    auto cleanup = [&]() { for (void *p : tmp) cudaFree(p); };
#define TA(p, bytes)                                                                   \
    do {                                                                               \
        cudaError_t e_ = talloc((void **)&(p), (bytes));                               \
        if (e_ != cudaSuccess) { cleanup(); return ctx->fail(PT_E_NOMEM, "bvh temp", cudaGetErrorString(e_)); } \
    } while (0)
    TA(ids, n * 4);
    TA(tlo, n * 16); TA(thi, n * 16); TA(cen, n * 16);
    TA(bounds, 6 * 4);
    TA(intParent, (size_t)max(n - 1, 1u) * 4); TA(leafParent, (size_t)n * 4);
    TA(rf, (size_t)max(n - 1, 1u) * 4); TA(rl, (size_t)max(n - 1, 1u) * 4);
    TA(leafLo, n * 16); TA(leafHi, n * 16);
    TA(intLo, (size_t)max(n - 1, 1u) * 16); TA(intHi, (size_t)max(n - 1, 1u) * 16);
    TA(flags, (size_t)max(n - 1, 1u) * 4);
    TA(counters, 4 * 4);
    int2 *qa, *qb;
    TA(qa, (size_t)n * 8); TA(qb, (size_t)n * 8);
    const int B = 256;
    uint32_t G = (n + B - 1) / B;
    k_tri_bounds<<<G, B, 0, st>>>(n, d_meshFirstTri, S.numMeshes, S.mats, S.idx, S.pos, triMesh, tlo, thi, cen);
    uint32_t binit[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
    cudaMemcpyAsync(bounds, binit, sizeof(binit), cudaMemcpyHostToDevice, st);
    k_centroid_bounds<<<min(G, 1024u), B, 0, st>>>(n, cen, bounds);
    k_morton<<<G, B, 0, st>>>(n, cen, bounds, codes, ids);
    {  // (codes, ids) -> (codesS, idsS) by the 30-bit code; `codes` stays unsorted (read back for parity)
        const uint32_t tiles = (n + kRsTile - 1) / kRsTile;
        uint32_t *rsHist, *kA, *vA;
        TA(rsHist, (size_t)256 * tiles * 4);
        TA(kA, (size_t)n * 4);
        TA(vA, (size_t)n * 4);
        const uint32_t *kin = codes, *vin = ids;
        uint32_t *kout[4] = {kA, codesS, kA, codesS}, *vout[4] = {vA, idsS, vA, idsS};
        for (int p = 0; p < 4; p++) {
            k_rs_hist<<<tiles, kRsThreads, 0, st>>>(kin, n, 8u * p, tiles, rsHist);
            k_rs_scan<<<1, 1024, 0, st>>>(rsHist, 256u * tiles);
            k_rs_scatter<<<tiles, kRsThreads, 0, st>>>(kin, vin, n, 8u * p, tiles, rsHist, kout[p], vout[p]);
            kin = kout[p];
            vin = vout[p];
        }
    }
    if (n > 1) {
        k_karras<<<(n - 1 + B - 1) / B, B, 0, st>>>((int)n, codesS, children, intParent, leafParent, rf, rl);
        cudaMemsetAsync(flags, 0, (size_t)(n - 1) * 4, st);
    }
    k_refit<<<G, B, 0, st>>>((int)n, idsS, tlo, thi, children, intParent, leafParent, leafLo, leafHi, intLo, intHi,
                             flags);
    // the radix tree stays as built in `children` (pt_bvh_read); the
    // treelet passes rewire a copy
    uint32_t *cnt, *rewired;
    int32_t *tch, *tip, *tlp;
    float *cost;
    const size_t ni = (size_t)max(n - 1, 1u);
    TA(cnt, ni * 4); TA(cost, ni * 4); TA(rewired, 4);
    TA(tch, ni * 8); TA(tip, ni * 4); TA(tlp, (size_t)n * 4);
    float *planCost;
    uint8_t *planSlots, *planWide;
    TA(planCost, ni * 8 * 4); TA(planSlots, ni * 8); TA(planWide, ni);
    if (n > 1) {
        k_range_count<<<(n - 1 + B - 1) / B, B, 0, st>>>((int)n, rf, rl, cnt);
        cudaMemcpyAsync(tch, children, (size_t)(n - 1) * 8, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(tip, intParent, (size_t)(n - 1) * 4, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(tlp, leafParent, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
        TreeletIn T{(int)n, tch, tip, tlp, leafLo, leafHi, intLo, intHi, cost, cnt, flags, rewired};
        for (int pass = 0; pass < kTreeletPasses; pass++) {
            cudaMemsetAsync(flags, 0, (size_t)(n - 1) * 4, st);
            cudaMemsetAsync(rewired, 0, 4, st);
            k_treelet<<<G, B, 0, st>>>(T);
            if (pass + 1 == kTreeletPasses) break;
            // a pass that rewires nothing leaves the tree as it found it, and
            // the next pass would decide the same: stop
            uint32_t changed = 0;
            cudaError_t ce = cudaMemcpyAsync(&changed, rewired, 4, cudaMemcpyDeviceToHost, st);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
            if (ce != cudaSuccess) { cleanup(); return ctx->fail(PT_E_CUDA, "bvh treelets", cudaGetErrorString(ce)); }
            if (changed == 0) break;
        }
    }
    // collapse: wide nodes <= max(1, n - 1); triangles exactly n
    BVH8Node *nodes;
    float4 *tri;
    uint32_t maxWide = max(1u, n - 1);
    cudaError_t e1 = ctx->alloc_scene(&nodes, maxWide);
    cudaError_t e2 = ctx->alloc_scene(&tri, 3 * (size_t)n);
    if (e1 != cudaSuccess || e2 != cudaSuccess) { cleanup(); return ctx->fail(PT_E_NOMEM, "bvh nodes"); }
    // Two collapses of the restructured tree: greedy (the largest child
    // opened until 8) and k_wide_plan's least-area plan.  Which goes first
    // depends on whether the tree's nodes and triangles (~71 bytes per
    // triangle) fit in the L2.  If they do, traversal runs from L2 and the
    // greedy tree is the faster one: the 64-sphere scene at 1866 vs 1846
    // Mpaths/s, the Cornell box at 390 vs 382.  If they do not, traversal
    // waits on DRAM for each node, and the plan's fewer node visits win:
    // the 10 M-triangle scene at 467 vs 458.  A result deeper than the
    // traversal stack is collapsed the other way, and only then does the
    // build fall back to the radix tree (its depth is bounded by the key
    // bits plus the index bits of equal keys).
    int l2 = 0;
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, ctx->device);
    const bool planFirst = ctx->dbgWidePlan || (uint64_t)n * 71u > (uint64_t)(l2 > 0 ? l2 : 126 << 20);
    uint32_t cnt4[4];
    for (int attempt = 0; attempt < 3; attempt++) {
        const bool radix = attempt == 2 || n == 1;
        const bool usePlan = attempt == (planFirst ? 0 : 1);
        if (attempt == 2) {  // restore the radix tree's bounds and counts
            cudaMemsetAsync(flags, 0, (size_t)(n - 1) * 4, st);
            k_refit<<<G, B, 0, st>>>((int)n, idsS, tlo, thi, children, intParent, leafParent, leafLo, leafHi, intLo,
                                     intHi, flags);
            k_range_count<<<(n - 1 + B - 1) / B, B, 0, st>>>((int)n, rf, rl, cnt);
        }
        const uint8_t *plan = nullptr, *planW = nullptr;
        if (usePlan && n > 1) {  // the collapse plan of the restructured tree
            cudaMemsetAsync(flags, 0, (size_t)(n - 1) * 4, st);
            k_wide_plan<<<G, B, 0, st>>>((int)n, radix ? children : tch, radix ? intParent : tip,
                                         radix ? leafParent : tlp, cnt, intLo, intHi, planCost, planSlots,
                                         planWide, flags);
            plan = planSlots;
            planW = planWide;
        }
        CollapseIn C{(int)n, radix ? children : tch, cnt, maxWide, leafLo, leafHi, intLo, intHi, idsS, triMesh,
                     d_meshFirstTri, S.mats, S.idx, S.pos, nodes, tri, counters, plan, planW};
        int2 root = make_int2(n > 1 ? 0 : ~0, 0);
        cudaMemcpyAsync(qa, &root, sizeof(root), cudaMemcpyHostToDevice, st);
        uint32_t cinit[4] = {1u, 0u, 0u, 0u};
        cudaMemcpyAsync(counters, cinit, sizeof(cinit), cudaMemcpyHostToDevice, st);
        uint32_t qn = 1;
        int levels = 0;
        while (qn > 0) {
            cudaMemsetAsync(counters + 2, 0, 4, st);
            k_collapse<<<(qn + 127) / 128, 128, 0, st>>>(C, qa, qn, qb);
            PT_CUDA(cudaMemcpyAsync(&qn, counters + 2, 4, cudaMemcpyDeviceToHost, st));
            PT_CUDA(cudaStreamSynchronize(st));
            std::swap(qa, qb);
            if (++levels > 64) { cleanup(); return ctx->fail(PT_E_DEVICE, "bvh collapse did not terminate"); }
        }
        PT_CUDA(cudaMemcpyAsync(cnt4, counters, sizeof(cnt4), cudaMemcpyDeviceToHost, st));
        cudaError_t se = cudaStreamSynchronize(st);
        if (se != cudaSuccess) { cleanup(); return ctx->fail(PT_E_CUDA, "bvh build", cudaGetErrorString(se)); }
        if (levels <= kTraversalStack || radix) break;
    }
    cleanup();
    if (cnt4[3] != 0u) return ctx->fail(PT_E_DEVICE, "bvh collapse: leaf triangle count mismatch");
    if (cnt4[1] != n) return ctx->fail(PT_E_DEVICE, "bvh collapse lost triangles");
    S.tri = tri;
    S.nodes = nodes;
    S.numNodes = cnt4[0];
    S.triMesh = triMesh;
    ctx->numWide = cnt4[0];
    ctx->d_morton = codes;
    ctx->d_sorted = idsS;
    ctx->d_binChildren = children;
    (void)codesS;
    return PT_OK;
#undef TA
}
