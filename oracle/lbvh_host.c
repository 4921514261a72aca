/* Host build of the linear BVH (TEST INFRASTRUCTURE ONLY: the oracle for the
 * GPU build in vlr_b200/csrc/lbvh.cu).
 *
 * The reference has no BVH code of its own (OptiX builds its acceleration
 * structures, libVLR/scene.cpp:1318-1328), so this file restates the
 * published algorithm the GPU builder follows, sequentially:
 *   Morton codes: centroid (v0+v1+v2)*(1/3), quantised to 10 bits per axis
 *     over the centroid bounds, bits interleaved x2 y1 z0;
 *   sort: stable sort of (code, primitive index) by code;
 *   hierarchy: Karras, "Maximizing Parallelism in the Construction of BVHs,
 *     Octrees, and k-d Trees" (HPG 2012), ties broken by sorted position;
 *   boxes: per internal node, the union of its children's boxes.
 * Compiled without FMA contraction (x86-64 baseline has none), so every float
 * operation rounds as the GPU build's does. */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static uint32_t spread10(uint32_t x) {
    x &= 0x3FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

static void centroid(const float* v, uint32_t i, float c[3]) {
    const float* p = v + 9 * (size_t)i;
    const float third = 1.0f / 3.0f;
    for (int k = 0; k < 3; ++k) {
        float s = p[k] + p[3 + k];
        s = s + p[6 + k];
        c[k] = s * third;
    }
}

static int clz32(uint32_t x) { return x ? __builtin_clz(x) : 32; }

static int delta(const uint32_t* codes, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    if (codes[i] == codes[j]) return 32 + clz32((uint32_t)(i ^ j));
    return clz32(codes[i] ^ codes[j]);
}

typedef struct { uint32_t code, prim; } Pair;

static int cmpPair(const void* a, const void* b) {
    const Pair* x = (const Pair*)a;
    const Pair* y = (const Pair*)b;
    if (x->code != y->code) return x->code < y->code ? -1 : 1;
    return x->prim < y->prim ? -1 : (x->prim > y->prim);   /* prim order = stability */
}

/* verts: n triangles x 9 floats.  Outputs: sortedCodes[n], sortedPrims[n],
 * children[2(n-1)], nodeBoxes[6(n-1)].  Returns 0 on success. */
int oracle_lbvh_build(const float* verts, uint32_t n, uint32_t* sortedCodes, uint32_t* sortedPrims,
                      int32_t* children, float* nodeBoxes) {
    if (n == 0) return 0;
    float lo[3] = { 0, 0, 0 }, hi[3] = { 0, 0, 0 };
    for (uint32_t i = 0; i < n; ++i) {
        float c[3];
        centroid(verts, i, c);
        for (int k = 0; k < 3; ++k) {
            if (i == 0 || c[k] < lo[k]) lo[k] = c[k];
            if (i == 0 || c[k] > hi[k]) hi[k] = c[k];
        }
    }
    float scale[3];
    for (int k = 0; k < 3; ++k) {
        float ext = hi[k] - lo[k];
        scale[k] = ext > 0.0f ? 1024.0f / ext : 0.0f;
    }
    Pair* pairs = (Pair*)malloc(sizeof(Pair) * n);
    if (!pairs) return -1;
    for (uint32_t i = 0; i < n; ++i) {
        float c[3];
        uint32_t q[3];
        centroid(verts, i, c);
        for (int k = 0; k < 3; ++k) {
            float f = (c[k] - lo[k]) * scale[k];
            int qi = (int)f;
            q[k] = (uint32_t)(qi < 0 ? 0 : (qi > 1023 ? 1023 : qi));
        }
        pairs[i].code = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
        pairs[i].prim = i;
    }
    qsort(pairs, n, sizeof(Pair), cmpPair);
    for (uint32_t i = 0; i < n; ++i) { sortedCodes[i] = pairs[i].code; sortedPrims[i] = pairs[i].prim; }
    free(pairs);
    if (n == 1) return 0;
    const int N = (int)n;
    int32_t* parent = (int32_t*)malloc(sizeof(int32_t) * (size_t)N);
    for (int i = 0; i < N - 1; ++i) {
        int d = (delta(sortedCodes, N, i, i + 1) - delta(sortedCodes, N, i, i - 1)) >= 0 ? 1 : -1;
        int dMin = delta(sortedCodes, N, i, i - d);
        int lMax = 2;
        while (delta(sortedCodes, N, i, i + lMax * d) > dMin) lMax <<= 1;
        int l = 0;
        for (int t = lMax >> 1; t >= 1; t >>= 1)
            if (delta(sortedCodes, N, i, i + (l + t) * d) > dMin) l += t;
        int j = i + l * d;
        int dNode = delta(sortedCodes, N, i, j);
        int s = 0, t = l;
        do {
            t = (t + 1) >> 1;
            if (delta(sortedCodes, N, i, i + (s + t) * d) > dNode) s += t;
        } while (t > 1);
        int gamma = i + s * d + (d < 0 ? d : 0);
        int mn = i < j ? i : j, mx = i < j ? j : i;
        children[2 * i] = (mn == gamma) ? ~gamma : gamma;
        children[2 * i + 1] = (mx == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    }
    /* boxes bottom-up: post-order traversal from the root */
    int32_t* stack = (int32_t*)malloc(sizeof(int32_t) * (size_t)N * 2);
    uint8_t* done = (uint8_t*)calloc((size_t)N, 1);
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        int node = stack[sp - 1];
        int ready = 1;
        for (int k = 0; k < 2; ++k) {
            int c = children[2 * node + k];
            if (c >= 0 && !done[c]) { stack[sp++] = c; ready = 0; }
        }
        if (!ready) continue;
        --sp;
        float blo[2][3], bhi[2][3];
        for (int k = 0; k < 2; ++k) {
            int c = children[2 * node + k];
            if (c < 0) {
                const float* p = verts + 9 * (size_t)sortedPrims[~c];
                for (int a = 0; a < 3; ++a) {
                    float m0 = p[a] < p[3 + a] ? p[a] : p[3 + a];
                    float M0 = p[a] > p[3 + a] ? p[a] : p[3 + a];
                    blo[k][a] = m0 < p[6 + a] ? m0 : p[6 + a];
                    bhi[k][a] = M0 > p[6 + a] ? M0 : p[6 + a];
                }
            }
            else {
                for (int a = 0; a < 3; ++a) { blo[k][a] = nodeBoxes[6 * c + a]; bhi[k][a] = nodeBoxes[6 * c + 3 + a]; }
            }
        }
        for (int a = 0; a < 3; ++a) {
            nodeBoxes[6 * node + a] = blo[0][a] < blo[1][a] ? blo[0][a] : blo[1][a];
            nodeBoxes[6 * node + 3 + a] = bhi[0][a] > bhi[1][a] ? bhi[0][a] : bhi[1][a];
        }
        done[node] = 1;
    }
    free(stack);
    free(done);
    free(parent);
    return 0;
}
