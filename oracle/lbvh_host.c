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

/* ---- treelet restructuring (Karras and Aila, "Fast Parallel Construction
 * of High-Quality Bounding Volume Hierarchies", HPG 2013), restated
 * sequentially for the GPU pass in vlr_b200/csrc/lbvh.cu: per round
 * (gamma = 7, 14, 28, ...), every internal node in post-order gets its SAH
 * cost (1.2 x area for a node, 1.0 x area for a triangle) and triangle count
 * from its children; a node with >= gamma triangles roots a treelet of up to
 * 7 leaves, grown by opening the leaf of largest area (first of equals), and
 * the treelet is rebuilt with the least-cost topology from a dynamic program
 * over its leaf subsets when that is below 0.9999 x its current cost.  The
 * new inner nodes take the treelet's node indices in breadth-first order of
 * their subsets, the root keeping its own. */
typedef struct { int ref; float lo[3], hi[3]; float cost; uint32_t count; } TLeaf;

static float boxArea(const float lo[3], const float hi[3]) {
    float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    float s = dx * dy + dy * dz;
    s = s + dz * dx;
    return 2.0f * s;
}

static void refBox(const float* verts, const uint32_t* prims, const float* nodeBoxes, int ref, float lo[3],
                   float hi[3]) {
    if (ref >= 0) {
        for (int a = 0; a < 3; ++a) { lo[a] = nodeBoxes[6 * ref + a]; hi[a] = nodeBoxes[6 * ref + 3 + a]; }
        return;
    }
    const float* p = verts + 9 * (size_t)prims[~ref];
    for (int a = 0; a < 3; ++a) {
        float m0 = p[a] < p[3 + a] ? p[a] : p[3 + a];
        float M0 = p[a] > p[3 + a] ? p[a] : p[3 + a];
        lo[a] = m0 < p[6 + a] ? m0 : p[6 + a];
        hi[a] = M0 > p[6 + a] ? M0 : p[6 + a];
    }
}

static TLeaf makeLeaf(const float* verts, const uint32_t* prims, const float* nodeBoxes, const float* cost,
                      const uint32_t* count, int ref) {
    TLeaf t;
    t.ref = ref;
    refBox(verts, prims, nodeBoxes, ref, t.lo, t.hi);
    if (ref >= 0) { t.cost = cost[ref]; t.count = count[ref]; }
    else { t.cost = 1.0f * boxArea(t.lo, t.hi); t.count = 1; }
    return t;
}

static void unionBox(const TLeaf* L, int nl, int s, float lo[3], float hi[3]) {
    int first = 1;
    for (int i = 0; i < nl; ++i) {
        if (!((s >> i) & 1)) continue;
        for (int a = 0; a < 3; ++a) {
            if (first) { lo[a] = L[i].lo[a]; hi[a] = L[i].hi[a]; }
            else {
                lo[a] = L[i].lo[a] < lo[a] ? L[i].lo[a] : lo[a];
                hi[a] = L[i].hi[a] > hi[a] ? L[i].hi[a] : hi[a];
            }
        }
        first = 0;
    }
}

static float treelet(const float* verts, const uint32_t* prims, int32_t* children, float* nodeBoxes, float* cost,
                     uint32_t* count, int root, float rootCost, uint32_t* restructured) {
    TLeaf L[7];
    int inner[6];
    int nl = 2, ni = 0;
    inner[ni++] = root;
    L[0] = makeLeaf(verts, prims, nodeBoxes, cost, count, children[2 * root]);
    L[1] = makeLeaf(verts, prims, nodeBoxes, cost, count, children[2 * root + 1]);
    while (nl < 7) {
        int best = -1;
        float bestArea = -1.0f;
        for (int j = 0; j < nl; ++j) {
            if (L[j].ref < 0) continue;
            float a = boxArea(L[j].lo, L[j].hi);
            if (a > bestArea) { bestArea = a; best = j; }
        }
        if (best < 0) break;
        int x = L[best].ref;
        inner[ni++] = x;
        L[best] = makeLeaf(verts, prims, nodeBoxes, cost, count, children[2 * x]);
        L[nl++] = makeLeaf(verts, prims, nodeBoxes, cost, count, children[2 * x + 1]);
    }
    const int full = (1 << nl) - 1;
    float A[128], C[128];
    uint8_t P[128];
    for (int s = 1; s <= full; ++s) {
        float lo[3], hi[3];
        unionBox(L, nl, s, lo, hi);
        A[s] = boxArea(lo, hi);
    }
    for (int i = 0; i < nl; ++i) C[1 << i] = L[i].cost;
    for (int s = 1; s <= full; ++s) {
        if ((s & (s - 1)) == 0) continue;
        int low = s & -s;
        float best = 3.402823466e+38f;
        int bp = 0;
        for (int p = (s - 1) & s; p; p = (p - 1) & s) {
            if (!(p & low)) continue;
            float c = C[p] + C[s ^ p];
            if (c < best) { best = c; bp = p; }
        }
        C[s] = 1.2f * A[s] + best;
        P[s] = (uint8_t)bp;
    }
    if (!(C[full] < rootCost * 0.9999f)) return rootCost;
    int qs[6], qn[6], qh = 0, qt = 0, next = 1;
    qs[qt] = full; qn[qt] = root; ++qt;
    while (qh < qt) {
        int s = qs[qh], x = qn[qh];
        ++qh;
        int part[2] = { P[s], s ^ P[s] };
        float lo[2][3], hi[2][3];
        uint32_t cnt = 0;
        for (int k = 0; k < 2; ++k) {
            int q = part[k], ref;
            unionBox(L, nl, q, lo[k], hi[k]);
            if ((q & (q - 1)) == 0) {
                int i = __builtin_ctz((unsigned)q);
                ref = L[i].ref;
                cnt += L[i].count;
            }
            else {
                ref = inner[next++];
                qs[qt] = q; qn[qt] = ref; ++qt;
                for (int i = 0; i < nl; ++i) if ((q >> i) & 1) cnt += L[i].count;
            }
            children[2 * x + k] = ref;
        }
        for (int a = 0; a < 3; ++a) {
            nodeBoxes[6 * x + a] = lo[0][a] < lo[1][a] ? lo[0][a] : lo[1][a];
            nodeBoxes[6 * x + 3 + a] = hi[0][a] > hi[1][a] ? hi[0][a] : hi[1][a];
        }
        cost[x] = C[s];
        count[x] = cnt;
    }
    ++*restructured;
    return C[full];
}

/* children/nodeBoxes: an LBVH from oracle_lbvh_build, modified in place.
 * Returns the number of treelets rebuilt, or -1. */
int oracle_lbvh_optimize(const float* verts, uint32_t n, const uint32_t* sortedPrims, int32_t* children,
                         float* nodeBoxes, uint32_t rounds) {
    if (n < 3 || rounds == 0) return 0;
    const int N = (int)n;
    float* cost = (float*)malloc(sizeof(float) * (size_t)N);
    uint32_t* count = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)N);
    int32_t* order = (int32_t*)malloc(sizeof(int32_t) * (size_t)N);
    int32_t* stack = (int32_t*)malloc(sizeof(int32_t) * (size_t)N * 2);
    uint8_t* seen = (uint8_t*)malloc((size_t)N);
    if (!cost || !count || !order || !stack || !seen) return -1;
    uint32_t restructured = 0, gamma = 7;
    for (uint32_t r = 0; r < rounds; ++r, gamma *= 2) {
        memset(seen, 0, (size_t)N);
        int sp = 0, no = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            int x = stack[sp - 1];
            if (!seen[x]) {
                seen[x] = 1;
                for (int k = 0; k < 2; ++k) if (children[2 * x + k] >= 0) stack[sp++] = children[2 * x + k];
                continue;
            }
            --sp;
            order[no++] = x;
        }
        for (int k = 0; k < no; ++k) {
            int x = order[k];
            TLeaf a = makeLeaf(verts, sortedPrims, nodeBoxes, cost, count, children[2 * x]);
            TLeaf b = makeLeaf(verts, sortedPrims, nodeBoxes, cost, count, children[2 * x + 1]);
            float lo[3], hi[3];
            for (int q = 0; q < 3; ++q) {
                lo[q] = a.lo[q] < b.lo[q] ? a.lo[q] : b.lo[q];
                hi[q] = a.hi[q] > b.hi[q] ? a.hi[q] : b.hi[q];
            }
            float c = 1.2f * boxArea(lo, hi) + a.cost;
            c = c + b.cost;
            uint32_t cnt = a.count + b.count;
            if (cnt >= gamma)
                c = treelet(verts, sortedPrims, children, nodeBoxes, cost, count, x, c, &restructured);
            cost[x] = c;
            count[x] = cnt;
        }
    }
    free(cost); free(count); free(order); free(stack); free(seen);
    return (int)restructured;
}
