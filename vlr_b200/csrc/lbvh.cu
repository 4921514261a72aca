// LBVH construction on the GPU:
//   1. centroid bounds (block reduction + one ordered-int atomic per CTA);
//   2. 30-bit Morton codes of the quantised centroids;
//   3. stable LSD radix sort of (code, primitive) pairs, 4-bit digits;
//   4. Karras (2012) hierarchy over the sorted codes, ties broken by position;
//   5. bottom-up refit with one arrival counter per internal node;
//   6. triangles re-packed in sorted order for traversal.
// Every integer result (codes, order, topology) and every box (min/max of the
// input floats) is deterministic, so a host build of the same algorithm
// reproduces it bit for bit.  Compiled without FMA contraction so the float
// quantisation step rounds like the host build.
#include "lbvh_build.h"

#include <cuda_runtime.h>
#include <cfloat>
#include <stdexcept>
#include <string>

namespace vlrb {

namespace {

__device__ __forceinline__ uint32_t floatToOrdered(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float orderedToFloat(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

__device__ __forceinline__ V3 loadVertex(const float* v, uint32_t tri, int k) {
    const float* p = v + 9 * static_cast<size_t>(tri) + 3 * k;
    return V3(p[0], p[1], p[2]);
}

// Centroid of a triangle: (v0 + v1 + v2) * (1/3), summed left to right.  The
// product is rounded on its own (__fmul_rn): left to the compiler it fuses
// with the "- lo" of the quantisation into one FMA, which moves centroids that
// sit on a cell boundary into the neighbouring cell.
__device__ __forceinline__ V3 centroidOf(const float* verts, uint32_t i) {
    V3 a = loadVertex(verts, i, 0), b = loadVertex(verts, i, 1), c = loadVertex(verts, i, 2);
    V3 s = a + b + c;
    const float third = 1.0f / 3.0f;
    return V3(__fmul_rn(s.x, third), __fmul_rn(s.y, third), __fmul_rn(s.z, third));
}

__global__ void centroidBoundsKernel(const float* verts, uint32_t n, uint32_t* ordBox /* 6 */) {
    __shared__ uint32_t s[6];
    if (threadIdx.x < 3) s[threadIdx.x] = 0xFFFFFFFFu;
    else if (threadIdx.x < 6) s[threadIdx.x] = 0u;
    __syncthreads();
    uint32_t lo[3] = { 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu }, hi[3] = { 0u, 0u, 0u };
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        V3 c = centroidOf(verts, i);
        uint32_t o[3] = { floatToOrdered(c.x), floatToOrdered(c.y), floatToOrdered(c.z) };
        for (int k = 0; k < 3; ++k) { lo[k] = min(lo[k], o[k]); hi[k] = max(hi[k], o[k]); }
    }
    for (int k = 0; k < 3; ++k) {
        for (int off = 16; off > 0; off >>= 1) {
            lo[k] = min(lo[k], __shfl_xor_sync(0xFFFFFFFFu, lo[k], off));
            hi[k] = max(hi[k], __shfl_xor_sync(0xFFFFFFFFu, hi[k], off));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int k = 0; k < 3; ++k) { atomicMin(&s[k], lo[k]); atomicMax(&s[3 + k], hi[k]); }
    }
    __syncthreads();
    if (threadIdx.x < 3) atomicMin(&ordBox[threadIdx.x], s[threadIdx.x]);
    else if (threadIdx.x < 6) atomicMax(&ordBox[threadIdx.x], s[threadIdx.x]);
}

__device__ __forceinline__ uint32_t spreadBits10(uint32_t x) {
    x &= 0x3FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

__global__ void mortonKernel(const float* verts, uint32_t n, const uint32_t* ordBox,
                             uint32_t* codes, uint32_t* prims) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float lo[3], scale[3];
    for (int k = 0; k < 3; ++k) {
        lo[k] = orderedToFloat(ordBox[k]);
        float ext = orderedToFloat(ordBox[3 + k]) - lo[k];
        scale[k] = ext > 0.0f ? 1024.0f / ext : 0.0f;
    }
    V3 c = centroidOf(verts, i);
    float cc[3] = { c.x, c.y, c.z };
    uint32_t q[3];
    for (int k = 0; k < 3; ++k) {
        float f = (cc[k] - lo[k]) * scale[k];
        int qi = static_cast<int>(f);
        q[k] = static_cast<uint32_t>(qi < 0 ? 0 : (qi > 1023 ? 1023 : qi));
    }
    codes[i] = (spreadBits10(q[0]) << 2) | (spreadBits10(q[1]) << 1) | spreadBits10(q[2]);
    prims[i] = i;
}

// ---- stable LSD radix sort, 4-bit digits, tile of 256 threads x 16 items
constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kRadix = 16;

__global__ void radixHistKernel(const uint32_t* keys, uint32_t n, int shift, uint32_t* hist /* [16][numTiles] */) {
    __shared__ uint32_t s[kRadix];
    if (threadIdx.x < kRadix) s[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * kSortTile;
    for (int k = 0; k < kSortItems; ++k) {
        uint32_t i = base + k * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&s[(keys[i] >> shift) & (kRadix - 1)], 1u);
    }
    __syncthreads();
    if (threadIdx.x < kRadix) hist[threadIdx.x * gridDim.x + blockIdx.x] = s[threadIdx.x];
}

// Exclusive scan of the [digit][tile] histogram in one CTA of 1024 threads.
__global__ void radixScanKernel(uint32_t* hist, uint32_t count) {
    __shared__ uint32_t partial[1024];
    const uint32_t per = (count + 1023) / 1024;
    const uint32_t begin = threadIdx.x * per;
    uint32_t sum = 0;
    for (uint32_t i = begin; i < begin + per && i < count; ++i) sum += hist[i];
    partial[threadIdx.x] = sum;
    __syncthreads();
    for (uint32_t off = 1; off < 1024; off <<= 1) {
        uint32_t v = threadIdx.x >= off ? partial[threadIdx.x - off] : 0u;
        __syncthreads();
        partial[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = partial[threadIdx.x] - sum;
    for (uint32_t i = begin; i < begin + per && i < count; ++i) {
        uint32_t v = hist[i];
        hist[i] = run;
        run += v;
    }
}

__global__ void radixScatterKernel(const uint32_t* keysIn, const uint32_t* valsIn, uint32_t n, int shift,
                                   const uint32_t* offsets, uint32_t* keysOut, uint32_t* valsOut) {
    __shared__ uint32_t cnt[kRadix][kSortThreads + 1];
    const uint32_t base = blockIdx.x * kSortTile + threadIdx.x * kSortItems;
    uint32_t local[kRadix];
    for (int d = 0; d < kRadix; ++d) local[d] = 0;
    uint32_t key[kSortItems];
    for (int k = 0; k < kSortItems; ++k) {
        uint32_t i = base + k;
        key[k] = i < n ? keysIn[i] : 0u;
        if (i < n) local[(key[k] >> shift) & (kRadix - 1)]++;
    }
    for (int d = 0; d < kRadix; ++d) cnt[d][threadIdx.x] = local[d];
    __syncthreads();
    // 16 threads each scan one digit's column over the CTA's threads.
    if (threadIdx.x < kRadix) {
        uint32_t run = 0;
        for (int t = 0; t < kSortThreads; ++t) {
            uint32_t v = cnt[threadIdx.x][t];
            cnt[threadIdx.x][t] = run;
            run += v;
        }
    }
    __syncthreads();
    uint32_t pos[kRadix];
    for (int d = 0; d < kRadix; ++d)
        pos[d] = offsets[d * gridDim.x + blockIdx.x] + cnt[d][threadIdx.x];
    for (int k = 0; k < kSortItems; ++k) {
        uint32_t i = base + k;
        if (i < n) {
            uint32_t d = (key[k] >> shift) & (kRadix - 1);
            uint32_t p = pos[d]++;
            keysOut[p] = key[k];
            valsOut[p] = valsIn[i];
        }
    }
}

// ---- Karras hierarchy
__device__ __forceinline__ int prefixDelta(const uint32_t* codes, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    uint32_t a = codes[i], b = codes[j];
    if (a == b) return 32 + __clz(static_cast<uint32_t>(i ^ j));
    return __clz(a ^ b);
}

__global__ void karrasKernel(const uint32_t* codes, int n, int32_t* children /* [n-1][2] */,
                             int32_t* parentOfNode /* n-1 */, int32_t* parentOfLeaf /* n */) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = (prefixDelta(codes, n, i, i + 1) - prefixDelta(codes, n, i, i - 1)) >= 0 ? 1 : -1;
    int dMin = prefixDelta(codes, n, i, i - d);
    int lMax = 2;
    while (prefixDelta(codes, n, i, i + lMax * d) > dMin) lMax <<= 1;
    int l = 0;
    for (int t = lMax >> 1; t >= 1; t >>= 1)
        if (prefixDelta(codes, n, i, i + (l + t) * d) > dMin) l += t;
    int j = i + l * d;
    int dNode = prefixDelta(codes, n, i, j);
    int s = 0;
    int t = l;
    do {
        t = (t + 1) >> 1;
        if (prefixDelta(codes, n, i, i + (s + t) * d) > dNode) s += t;
    } while (t > 1);
    int gamma = i + s * d + (d < 0 ? d : 0);
    int lo = i < j ? i : j, hi = i < j ? j : i;
    int left = (lo == gamma) ? ~gamma : gamma;
    int right = (hi == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    children[2 * i + 0] = left;
    children[2 * i + 1] = right;
    if (left >= 0) parentOfNode[left] = i; else parentOfLeaf[~left] = i;
    if (right >= 0) parentOfNode[right] = i; else parentOfLeaf[~right] = i;
    if (i == 0) parentOfNode[0] = -1;
}

__device__ __forceinline__ void triBox(const float* verts, uint32_t prim, V3* lo, V3* hi) {
    V3 a = loadVertex(verts, prim, 0), b = loadVertex(verts, prim, 1), c = loadVertex(verts, prim, 2);
    *lo = vmin3(vmin3(a, b), c);
    *hi = vmax3(vmax3(a, b), c);
}

// Bottom-up refit: the second thread to arrive at a node computes its two
// child boxes (the first one exits), so every node is written exactly once.
__global__ void refitKernel(const float* verts, const uint32_t* sortedPrims, int n, const int32_t* children,
                            const int32_t* parentOfNode, const int32_t* parentOfLeaf, uint32_t* arrivals,
                            float* nodeBox /* [n-1][6] */, BvhNode* nodes) {
    int leaf = blockIdx.x * blockDim.x + threadIdx.x;
    if (leaf >= n) return;
    int node = parentOfLeaf[leaf];
    // Parent links start at -1; every index is range-checked so a malformed
    // hierarchy ends the walk instead of reaching outside the arrays.
    while (node >= 0 && node < n - 1) {
        __threadfence();
        if (atomicAdd(&arrivals[node], 1u) == 0u) return;
        __threadfence();
        V3 lo[2], hi[2];
        int c[2] = { children[2 * node + 0], children[2 * node + 1] };
        if (c[0] >= n - 1 || c[1] >= n - 1 || ~c[0] >= n || ~c[1] >= n) return;
        for (int k = 0; k < 2; ++k) {
            if (c[k] < 0) {
                triBox(verts, sortedPrims[~c[k]], &lo[k], &hi[k]);
            }
            else {
                const float* b = nodeBox + 6 * c[k];
                lo[k] = V3(__ldcg(b + 0), __ldcg(b + 1), __ldcg(b + 2));
                hi[k] = V3(__ldcg(b + 3), __ldcg(b + 4), __ldcg(b + 5));
            }
        }
        V3 ulo = vmin3(lo[0], lo[1]), uhi = vmax3(hi[0], hi[1]);
        float* ob = nodeBox + 6 * node;
        __stcg(ob + 0, ulo.x); __stcg(ob + 1, ulo.y); __stcg(ob + 2, ulo.z);
        __stcg(ob + 3, uhi.x); __stcg(ob + 4, uhi.y); __stcg(ob + 5, uhi.z);
        BvhNode nd;
        nd.lo0 = make_float4(lo[0].x, lo[0].y, lo[0].z, __int_as_float(c[0]));
        nd.hi0 = make_float4(hi[0].x, hi[0].y, hi[0].z, 0.0f);
        nd.lo1 = make_float4(lo[1].x, lo[1].y, lo[1].z, __int_as_float(c[1]));
        nd.hi1 = make_float4(hi[1].x, hi[1].y, hi[1].z, 0.0f);
        nodes[node] = nd;
        node = parentOfNode[node];
    }
}

__global__ void packTrisKernel(const float* verts, const uint32_t* sortedPrims, uint32_t n, BvhTri* tris) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t p = sortedPrims[i];
    V3 a = loadVertex(verts, p, 0), b = loadVertex(verts, p, 1), c = loadVertex(verts, p, 2);
    BvhTri t;
    t.v0 = make_float4(a.x, a.y, a.z, __uint_as_float(p));
    t.v1 = make_float4(b.x, b.y, b.z, 0.0f);
    t.v2 = make_float4(c.x, c.y, c.z, 0.0f);
    tris[i] = t;
}

// ---- treelet restructuring (Karras and Aila, "Fast Parallel Construction of
// High-Quality Bounding Volume Hierarchies", HPG 2013), one warp per
// treelet: every internal node with at least gamma triangles below it becomes
// the root of a treelet of up to 7 leaves (grown by opening the leaf of
// largest surface area), and the treelet's topology is replaced by the one of
// least SAH cost found by dynamic programming over the 127 leaf subsets.  The
// pass runs bottom up with one arrival counter per node, so a treelet is
// optimised after everything below it.  The result depends only on the
// subtree below each root, not on the order the threads run in, and every
// float operation is rounded explicitly, so the host restatement reproduces
// it bit for bit.
constexpr int kTreeletLeaves = 7;
constexpr int kTreeletSubsets = 1 << kTreeletLeaves;
constexpr float kSahNodeCost = 1.2f, kSahTriCost = 1.0f;

__device__ __forceinline__ float surfaceArea(const V3 &lo, const V3 &hi) {
    const float dx = __fsub_rn(hi.x, lo.x), dy = __fsub_rn(hi.y, lo.y), dz = __fsub_rn(hi.z, lo.z);
    return __fmul_rn(2.0f, __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dz, dx)));
}

__device__ __forceinline__ BvhNode loadNodeCg(const BvhNode* p) {
    const float4* q = reinterpret_cast<const float4*>(p);
    BvhNode nd;
    nd.lo0 = __ldcg(q + 0); nd.hi0 = __ldcg(q + 1); nd.lo1 = __ldcg(q + 2); nd.hi1 = __ldcg(q + 3);
    return nd;
}

__global__ void parentsKernel(const int32_t* children, int n, int32_t* parentOfNode, int32_t* parentOfLeaf) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    for (int k = 0; k < 2; ++k) {
        int c = children[2 * i + k];
        if (c >= 0 && c < n - 1) parentOfNode[c] = i;
        else if (c < 0 && ~c < n) parentOfLeaf[~c] = i;
    }
    if (i == 0) parentOfNode[0] = -1;
}

struct TreeletLeaf {
    int ref;
    V3 lo, hi;
    float cost;
    uint32_t count;
};

__device__ __forceinline__ TreeletLeaf treeletLeaf(int ref, const float4 &lo, const float4 &hi, const float* cost,
                                                   const uint32_t* count) {
    TreeletLeaf t;
    t.ref = ref;
    t.lo = V3(lo.x, lo.y, lo.z);
    t.hi = V3(hi.x, hi.y, hi.z);
    if (ref >= 0) { t.cost = __ldcg(cost + ref); t.count = __ldcg(count + ref); }
    else { t.cost = __fmul_rn(kSahTriCost, surfaceArea(t.lo, t.hi)); t.count = 1u; }
    return t;
}

__device__ __forceinline__ void subsetBox(const TreeletLeaf* L, int nl, int s, V3* lo, V3* hi) {
    bool first = true;
    for (int i = 0; i < nl; ++i) {
        if (!((s >> i) & 1)) continue;
        if (first) { *lo = L[i].lo; *hi = L[i].hi; first = false; }
        else { *lo = vmin3(*lo, L[i].lo); *hi = vmax3(*hi, L[i].hi); }
    }
}

// Per-warp dynamic-programming tables in shared memory.
struct TreeletTables {
    float area[kTreeletSubsets];
    float cost[kTreeletSubsets];
    uint8_t split[kTreeletSubsets];
};

// Optimises the treelet rooted at `root` (cost `rootCost` with its current
// topology) with the whole warp: every lane forms the same treelet, the lanes
// share the subsets of each size of the dynamic program, and lane `owner`
// writes the new topology.  Returns the root's cost afterwards (the same in
// every lane).  All control flow is warp-uniform.
__device__ float warpTreelet(int root, float rootCost, int owner, int n, int32_t* children, float* nodeBox,
                             BvhNode* nodes, float* cost, uint32_t* count, uint32_t* restructured,
                             TreeletTables &T) {
    const int lane = threadIdx.x & 31;
    const BvhNode rootNode = loadNodeCg(nodes + root);
    TreeletLeaf L[kTreeletLeaves];
    int inner[kTreeletLeaves - 1];
    int nl = 2, ni = 0;
    inner[ni++] = root;
    L[0] = treeletLeaf(__float_as_int(rootNode.lo0.w), rootNode.lo0, rootNode.hi0, cost, count);
    L[1] = treeletLeaf(__float_as_int(rootNode.lo1.w), rootNode.lo1, rootNode.hi1, cost, count);
    while (nl < kTreeletLeaves) {
        int best = -1;
        float bestArea = -1.0f;
        for (int j = 0; j < nl; ++j) {
            if (L[j].ref < 0) continue;
            const float a = surfaceArea(L[j].lo, L[j].hi);
            if (a > bestArea) { bestArea = a; best = j; }
        }
        if (best < 0) break;
        const int x = L[best].ref;
        if (x >= n - 1) return rootCost;
        const BvhNode xn = loadNodeCg(nodes + x);
        const int x0 = __float_as_int(xn.lo0.w), x1 = __float_as_int(xn.lo1.w);
        if (x0 >= n - 1 || x1 >= n - 1 || ~x0 >= n || ~x1 >= n) return rootCost;
        inner[ni++] = x;
        L[best] = treeletLeaf(x0, xn.lo0, xn.hi0, cost, count);
        L[nl++] = treeletLeaf(x1, xn.lo1, xn.hi1, cost, count);
    }
    const int full = (1 << nl) - 1;
    for (int s = lane + 1; s <= full; s += 32) {
        V3 lo, hi;
        subsetBox(L, nl, s, &lo, &hi);
        T.area[s] = surfaceArea(lo, hi);
    }
    for (int i = 0; i < nl; ++i)
        if (lane == i) T.cost[1 << i] = L[i].cost;
    __syncwarp();
    for (int size = 2; size <= nl; ++size) {
        for (int s = lane + 1; s <= full; s += 32) {
            if (__popc(s) != size) continue;
            const int low = s & -s;
            float best = FLT_MAX;
            int bp = 0;
            for (int p = (s - 1) & s; p; p = (p - 1) & s) {
                if (!(p & low)) continue;
                const float c = __fadd_rn(T.cost[p], T.cost[s ^ p]);
                if (c < best) { best = c; bp = p; }
            }
            T.cost[s] = __fadd_rn(__fmul_rn(kSahNodeCost, T.area[s]), best);
            T.split[s] = static_cast<uint8_t>(bp);
        }
        __syncwarp();
    }
    const float newCost = T.cost[full];
    if (!(newCost < __fmul_rn(rootCost, 0.9999f))) { __syncwarp(); return rootCost; }
    if (lane == owner) {
        // New topology: subsets in breadth-first order onto the treelet's
        // inner nodes (the root keeps its index, so its parent's reference
        // stays valid).
        int qs[kTreeletLeaves - 1], qn[kTreeletLeaves - 1];
        int qh = 0, qt = 0, next = 1;
        qs[qt] = full; qn[qt] = root; ++qt;
        while (qh < qt) {
            const int s = qs[qh], x = qn[qh];
            ++qh;
            const int part[2] = { T.split[s], s ^ T.split[s] };
            int ref[2];
            V3 lo[2], hi[2];
            uint32_t cnt = 0;
            for (int k = 0; k < 2; ++k) {
                const int q = part[k];
                subsetBox(L, nl, q, &lo[k], &hi[k]);
                if ((q & (q - 1)) == 0) {
                    const int i = __ffs(q) - 1;
                    ref[k] = L[i].ref;
                    cnt += L[i].count;
                }
                else {
                    ref[k] = inner[next++];
                    qs[qt] = q; qn[qt] = ref[k]; ++qt;
                    for (int i = 0; i < nl; ++i) if ((q >> i) & 1) cnt += L[i].count;
                }
            }
            children[2 * x + 0] = ref[0];
            children[2 * x + 1] = ref[1];
            BvhNode nd;
            nd.lo0 = make_float4(lo[0].x, lo[0].y, lo[0].z, __int_as_float(ref[0]));
            nd.hi0 = make_float4(hi[0].x, hi[0].y, hi[0].z, 0.0f);
            nd.lo1 = make_float4(lo[1].x, lo[1].y, lo[1].z, __int_as_float(ref[1]));
            nd.hi1 = make_float4(hi[1].x, hi[1].y, hi[1].z, 0.0f);
            float4* np = reinterpret_cast<float4*>(nodes + x);
            __stcg(np + 0, nd.lo0); __stcg(np + 1, nd.hi0); __stcg(np + 2, nd.lo1); __stcg(np + 3, nd.hi1);
            const V3 ulo = vmin3(lo[0], lo[1]), uhi = vmax3(hi[0], hi[1]);
            float* ob = nodeBox + 6 * x;
            __stcg(ob + 0, ulo.x); __stcg(ob + 1, ulo.y); __stcg(ob + 2, ulo.z);
            __stcg(ob + 3, uhi.x); __stcg(ob + 4, uhi.y); __stcg(ob + 5, uhi.z);
            __stcg(cost + x, T.cost[s]);
            __stcg(count + x, cnt);
        }
        atomicAdd(restructured, 1u);
    }
    __syncwarp();
    return newCost;
}

constexpr int kTreeletThreads = 256;

// One bottom-up pass, one thread per leaf climbing while it is the second
// arrival at a node: each node's SAH cost and triangle count from its
// children, then, for every node over >= gamma triangles, the warp optimises
// the treelet rooted there.  The warp stays converged: lanes that have
// stopped climbing keep helping with the others' treelets.
__global__ void __launch_bounds__(kTreeletThreads) treeletKernel(int n, uint32_t gamma, int32_t* children,
                                                                 float* nodeBox, BvhNode* nodes,
                                                                 const int32_t* parentOfNode,
                                                                 const int32_t* parentOfLeaf, uint32_t* arrivals,
                                                                 float* cost, uint32_t* count,
                                                                 uint32_t* restructured) {
    __shared__ TreeletTables tables[kTreeletThreads / 32];
    TreeletTables &T = tables[threadIdx.x >> 5];
    const int leaf = blockIdx.x * blockDim.x + threadIdx.x;
    bool active = leaf < n;
    int node = active ? parentOfLeaf[leaf] : -1;
    int guard = 0;
    while (__any_sync(0xFFFFFFFFu, active)) {
        bool work = false;
        if (active) {
            if (node < 0 || node >= n - 1 || guard++ >= n) active = false;
            else {
                __threadfence();
                if (atomicAdd(&arrivals[node], 1u) == 0u) active = false;
                else { __threadfence(); work = true; }
            }
        }
        float c = 0.0f;
        uint32_t cnt = 0;
        if (work) {
            const BvhNode nd = loadNodeCg(nodes + node);
            const int c0 = __float_as_int(nd.lo0.w), c1 = __float_as_int(nd.lo1.w);
            if (c0 >= n - 1 || c1 >= n - 1 || ~c0 >= n || ~c1 >= n) { work = false; active = false; }
            else {
                const TreeletLeaf a = treeletLeaf(c0, nd.lo0, nd.hi0, cost, count);
                const TreeletLeaf b = treeletLeaf(c1, nd.lo1, nd.hi1, cost, count);
                const V3 ulo = vmin3(a.lo, b.lo), uhi = vmax3(a.hi, b.hi);
                c = __fadd_rn(__fadd_rn(__fmul_rn(kSahNodeCost, surfaceArea(ulo, uhi)), a.cost), b.cost);
                cnt = a.count + b.count;
            }
        }
        uint32_t pending = __ballot_sync(0xFFFFFFFFu, work && cnt >= gamma);
        while (pending) {
            const int src = __ffs(pending) - 1;
            pending &= pending - 1;
            const int root = __shfl_sync(0xFFFFFFFFu, node, src);
            const float rootCost = __shfl_sync(0xFFFFFFFFu, c, src);
            const float nc = warpTreelet(root, rootCost, src, n, children, nodeBox, nodes, cost, count,
                                         restructured, T);
            if ((threadIdx.x & 31) == src) c = nc;
        }
        if (work) {
            __stcg(cost + node, c);
            __stcg(count + node, cnt);
            node = parentOfNode[node];
        }
    }
}

inline void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("lbvh ") + what + ": " + cudaGetErrorString(e));
}

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

} // namespace

size_t lbvhScratchBytes(uint32_t n) {
    const size_t numTiles = (n + kSortTile - 1) / kSortTile;
    size_t b = 0;
    b += align256(6 * 4);                       // ordered centroid box
    b += 4 * align256(size_t(n) * 4);           // codes/prims ping-pong
    b += align256(size_t(kRadix) * numTiles * 4); // histogram
    b += align256(size_t(n) * 4);               // parentOfLeaf
    b += align256(size_t(n) * 4);               // parentOfNode
    b += align256(size_t(n) * 4);               // arrivals
    b += align256(size_t(n) * 24);              // node boxes
    return b;
}

void lbvhBuild(const float* verts, uint32_t n, void* scratch, LbvhOutput* out, cudaStream_t stream) {
    if (n == 0) return;
    char* s = static_cast<char*>(scratch);
    auto take = [&](size_t bytes) { char* p = s; s += align256(bytes); return p; };
    const uint32_t numTiles = (n + kSortTile - 1) / kSortTile;
    uint32_t* ordBox = reinterpret_cast<uint32_t*>(take(6 * 4));
    uint32_t* keysA = reinterpret_cast<uint32_t*>(take(size_t(n) * 4));
    uint32_t* valsA = reinterpret_cast<uint32_t*>(take(size_t(n) * 4));
    uint32_t* keysB = reinterpret_cast<uint32_t*>(take(size_t(n) * 4));
    uint32_t* valsB = reinterpret_cast<uint32_t*>(take(size_t(n) * 4));
    uint32_t* hist = reinterpret_cast<uint32_t*>(take(size_t(kRadix) * numTiles * 4));
    int32_t* parentOfLeaf = reinterpret_cast<int32_t*>(take(size_t(n) * 4));
    int32_t* parentOfNode = reinterpret_cast<int32_t*>(take(size_t(n) * 4));
    uint32_t* arrivals = reinterpret_cast<uint32_t*>(take(size_t(n) * 4));
    float* nodeBox = reinterpret_cast<float*>(take(size_t(n) * 24));

    // Ordered-int centroid box: min = 0xFFFFFFFF x3, max = 0 x3.  Set by
    // memsets on the stream (no host source buffer involved).
    ck(cudaMemsetAsync(ordBox, 0xFF, 3 * sizeof(uint32_t), stream), "init box min");
    ck(cudaMemsetAsync(ordBox + 3, 0, 3 * sizeof(uint32_t), stream), "init box max");
    const uint32_t tb = 256;
    const uint32_t blocks = (n + tb - 1) / tb;
    const uint32_t redBlocks = blocks < 1184 ? blocks : 1184;
    centroidBoundsKernel<<<redBlocks, tb, 0, stream>>>(verts, n, ordBox);
    mortonKernel<<<blocks, tb, 0, stream>>>(verts, n, ordBox, keysA, valsA);
    uint32_t* kin = keysA; uint32_t* vin = valsA; uint32_t* kout = keysB; uint32_t* vout = valsB;
    for (int shift = 0; shift < 30; shift += 4) {
        radixHistKernel<<<numTiles, kSortThreads, 0, stream>>>(kin, n, shift, hist);
        radixScanKernel<<<1, 1024, 0, stream>>>(hist, kRadix * numTiles);
        radixScatterKernel<<<numTiles, kSortThreads, 0, stream>>>(kin, vin, n, shift, hist, kout, vout);
        uint32_t* t = kin; kin = kout; kout = t;
        t = vin; vin = vout; vout = t;
    }
    ck(cudaMemcpyAsync(out->sortedCodes, kin, size_t(n) * 4, cudaMemcpyDeviceToDevice, stream), "codes");
    ck(cudaMemcpyAsync(out->sortedPrims, vin, size_t(n) * 4, cudaMemcpyDeviceToDevice, stream), "prims");
    if (n > 1) {
        ck(cudaMemsetAsync(arrivals, 0, size_t(n) * 4, stream), "arrivals");
        ck(cudaMemsetAsync(parentOfLeaf, 0xFF, size_t(n) * 4, stream), "leaf parents");
        ck(cudaMemsetAsync(parentOfNode, 0xFF, size_t(n) * 4, stream), "node parents");
        karrasKernel<<<(n - 1 + tb - 1) / tb, tb, 0, stream>>>(out->sortedCodes, static_cast<int>(n),
                                                                out->children, parentOfNode, parentOfLeaf);
        refitKernel<<<blocks, tb, 0, stream>>>(verts, out->sortedPrims, static_cast<int>(n), out->children,
                                               parentOfNode, parentOfLeaf, arrivals, nodeBox, out->nodes);
        ck(cudaMemcpyAsync(out->nodeBoxes, nodeBox, size_t(n - 1) * 24, cudaMemcpyDeviceToDevice, stream), "boxes");
    }
    packTrisKernel<<<blocks, tb, 0, stream>>>(verts, out->sortedPrims, n, out->tris);
    ck(cudaGetLastError(), "launch");
}

// Leaf depth (internal nodes on the root path) by walking the parent links
// up; the maximum over all leaves lands in *maxDepth.  A walk longer than n
// steps (a malformed tree) stops there and reports n + 1.
__global__ void leafDepthKernel(const int32_t* parentOfNode, const int32_t* parentOfLeaf, uint32_t n,
                                uint32_t* maxDepth) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t d = 0;
    if (i < n) {
        int node = parentOfLeaf[i];
        while (node >= 0 && d <= n) {
            ++d;
            node = parentOfNode[node];
        }
    }
    for (int o = 16; o > 0; o >>= 1) d = max(d, __shfl_xor_sync(0xFFFFFFFFu, d, o));
    if ((threadIdx.x & 31u) == 0 && d > 0) atomicMax(maxDepth, d);
}

size_t lbvhOptimizeScratchBytes(uint32_t n) {
    return 5 * align256(size_t(n) * 4) + 256;
}

void lbvhOptimize(uint32_t n, uint32_t rounds, void* scratch, LbvhOutput* out, uint32_t* restructuredDev,
                  cudaStream_t stream) {
    if (n < 3 || rounds == 0) return;
    char* s = static_cast<char*>(scratch);
    auto take = [&](size_t bytes) { char* p = s; s += align256(bytes); return p; };
    int32_t* parentOfNode = reinterpret_cast<int32_t*>(take(size_t(n) * 4));
    int32_t* parentOfLeaf = reinterpret_cast<int32_t*>(take(size_t(n) * 4));
    uint32_t* arrivals = reinterpret_cast<uint32_t*>(take(size_t(n) * 4));
    float* cost = reinterpret_cast<float*>(take(size_t(n) * 4));
    uint32_t* count = reinterpret_cast<uint32_t*>(take(size_t(n) * 4));
    uint32_t* restructured = restructuredDev ? restructuredDev : reinterpret_cast<uint32_t*>(take(4));
    ck(cudaMemsetAsync(restructured, 0, 4, stream), "treelet counter");
    const uint32_t tb = 256;
    uint32_t gamma = kTreeletLeaves;
    for (uint32_t r = 0; r < rounds; ++r) {
        ck(cudaMemsetAsync(arrivals, 0, size_t(n) * 4, stream), "arrivals");
        ck(cudaMemsetAsync(parentOfLeaf, 0xFF, size_t(n) * 4, stream), "leaf parents");
        ck(cudaMemsetAsync(parentOfNode, 0xFF, size_t(n) * 4, stream), "node parents");
        parentsKernel<<<(n - 1 + tb - 1) / tb, tb, 0, stream>>>(out->children, static_cast<int>(n), parentOfNode,
                                                                 parentOfLeaf);
        treeletKernel<<<(n + kTreeletThreads - 1) / kTreeletThreads, kTreeletThreads, 0, stream>>>(
            static_cast<int>(n), gamma, out->children, out->nodeBoxes, out->nodes, parentOfNode, parentOfLeaf,
            arrivals, cost, count, restructured);
        gamma *= 2;
    }
    ck(cudaGetLastError(), "treelet launch");
}

uint32_t lbvhMaxLeafDepth(uint32_t n, const int32_t* children, void* scratch, cudaStream_t stream) {
    if (n < 2) return 0;
    char* s = static_cast<char*>(scratch);
    auto take = [&](size_t bytes) { char* p = s; s += align256(bytes); return p; };
    int32_t* parentOfNode = reinterpret_cast<int32_t*>(take(size_t(n) * 4));
    int32_t* parentOfLeaf = reinterpret_cast<int32_t*>(take(size_t(n) * 4));
    uint32_t* maxDepth = reinterpret_cast<uint32_t*>(take(4));
    const uint32_t tb = 256;
    ck(cudaMemsetAsync(parentOfLeaf, 0xFF, size_t(n) * 4, stream), "leaf parents");
    ck(cudaMemsetAsync(parentOfNode, 0xFF, size_t(n) * 4, stream), "node parents");
    ck(cudaMemsetAsync(maxDepth, 0, 4, stream), "depth");
    parentsKernel<<<(n - 1 + tb - 1) / tb, tb, 0, stream>>>(children, static_cast<int>(n), parentOfNode, parentOfLeaf);
    leafDepthKernel<<<(n + tb - 1) / tb, tb, 0, stream>>>(parentOfNode, parentOfLeaf, n, maxDepth);
    ck(cudaGetLastError(), "depth launch");
    uint32_t depth = 0;
    ck(cudaMemcpyAsync(&depth, maxDepth, 4, cudaMemcpyDeviceToHost, stream), "depth readback");
    ck(cudaStreamSynchronize(stream), "depth sync");
    return depth;
}

size_t lbvhTraversableScratchBytes(uint32_t n) {
    const size_t a = lbvhScratchBytes(n), b = lbvhOptimizeScratchBytes(n);
    return a > b ? a : b;
}

uint32_t lbvhBuildTraversable(const float* verts, uint32_t n, uint32_t rounds, void* scratch, LbvhOutput* out,
                              uint32_t* restructuredDev, cudaStream_t stream) {
    lbvhBuild(verts, n, scratch, out, stream);
    if (rounds == 0 || n < 3) return lbvhMaxLeafDepth(n, out->children, scratch, stream);
    lbvhOptimize(n, rounds, scratch, out, restructuredDev, stream);
    const uint32_t depth = lbvhMaxLeafDepth(n, out->children, scratch, stream);
    if (depth <= static_cast<uint32_t>(kTraversalStack)) return depth;
    // Restructuring deepened a path past the traversal stack: use the plain
    // LBVH, whose depth the key bits bound (at most 30 + 32 levels).
    lbvhBuild(verts, n, scratch, out, stream);
    if (restructuredDev) ck(cudaMemsetAsync(restructuredDev, 0, 4, stream), "treelet counter");
    return lbvhMaxLeafDepth(n, out->children, scratch, stream);
}

} // namespace vlrb
