// Collapse of a binary LBVH into compressed wide nodes, on the GPU.
//
// The binary hierarchy of az_bvh_build.cu (nodes plus the sorted primitive
// range of every inner node) is turned into WideNode records one tree level
// at a time: every work item of a level is a binary node that becomes one wide
// node.  A thread per item opens the child with the largest surface area until
// the node has `width` (2, 4 or 8) children; subtrees of at most `max_leaf`
// primitives become leaf children.  Children are placed in the slot matching
// the octant of their centre relative to the node centre, so a ray visits
// slots near-first by XOR-ing with its direction octant.  Child boxes are
// quantised conservatively to an 8-bit grid per node.
//
// Each level runs a count kernel (inner children and leaf primitives per item),
// an inclusive scan of the packed counts, and a write kernel that recomputes
// the same expansion, quantises the boxes, and writes the node, the next
// level's items (inner children get consecutive node indices in slot order)
// and the primitive permutation (a node's leaf primitives are consecutive from
// its prim_base).  The allocation order comes from the scan, so the layout is
// the same on every build.
#include <cub/cub.cuh>

#include <cfloat>
#include <cmath>
#include <cstring>

#include "az_internal.h"

namespace az {
namespace {

struct CItem {
    uint32_t ref;     // binary node (global index); for a single primitive its sorted position + leaf_base
    uint32_t first;   // first sorted position of the subtree's primitives (+ leaf_base)
    uint32_t count;   // primitives in the subtree
    uint32_t prim;    // 1: a single primitive reference
    float lo[3], hi[3];
};

struct CParams {
    const azd::BVHNode *nodes;   // global indices
    const uint2 *range;          // per binary node: (first sorted position + leaf_base, count)
    const uint32_t *perm;        // sorted position -> unsorted local primitive index
    uint32_t leaf_base;          // sorted position 0 as it appears in leaf references
    uint32_t max_leaf, width;
};

__device__ __forceinline__ CItem child_item(const CParams &P, const azd::BVHNode &n, int c) {
    CItem it;
    const uint32_t ref = c == 0 ? n.ch.x : n.ch.y, cnt = c == 0 ? n.ch.z : n.ch.w;
    const float4 bx = n.bx, by = n.by, bz = n.bz;
    it.lo[0] = c == 0 ? bx.x : bx.z;
    it.hi[0] = c == 0 ? bx.y : bx.w;
    it.lo[1] = c == 0 ? by.x : by.z;
    it.hi[1] = c == 0 ? by.y : by.w;
    it.lo[2] = c == 0 ? bz.x : bz.z;
    it.hi[2] = c == 0 ? bz.y : bz.w;
    it.ref = ref;
    if (cnt) {
        it.prim = 1;
        it.first = ref;
        it.count = 1;
    } else {
        const uint2 r = P.range[ref];
        it.prim = 0;
        it.first = r.x;
        it.count = r.y;
    }
    return it;
}

__device__ __forceinline__ double area_of(const CItem &k) {
    const double dx = fmax(0.0, (double)k.hi[0] - k.lo[0]), dy = fmax(0.0, (double)k.hi[1] - k.lo[1]),
                 dz = fmax(0.0, (double)k.hi[2] - k.lo[2]);
    return dx * dy + dy * dz + dz * dx;
}

// The children of the wide node made from `item` (greedy surface-area opening).
__device__ int expand(const CParams &P, const CItem &item, CItem kids[8]) {
    int nk = 0;
    if (item.prim || item.count <= P.max_leaf) {
        kids[nk++] = item;   // a hierarchy of at most max_leaf primitives: one leaf child
    } else {
        const azd::BVHNode n = P.nodes[item.ref];
        kids[nk++] = child_item(P, n, 0);
        kids[nk++] = child_item(P, n, 1);
    }
    while (nk < (int)P.width) {
        int best = -1;
        double best_area = -1.0;
        for (int i = 0; i < nk; i++) {
            if (kids[i].prim || kids[i].count < 2) continue;
            // open big subtrees first; small ones only while slots are free
            const double a = area_of(kids[i]) * (kids[i].count > P.max_leaf ? 2.0 : 1.0);
            if (a > best_area) {
                best_area = a;
                best = i;
            }
        }
        if (best < 0) break;
        const azd::BVHNode n = P.nodes[kids[best].ref];
        const CItem a = child_item(P, n, 0), b = child_item(P, n, 1);
        kids[best] = a;
        kids[nk++] = b;
    }
    return nk;
}

__global__ void k_collapse_count(CParams P, const CItem *items, uint32_t n_items, unsigned long long *counts) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_items) return;
    CItem kids[8];
    const int nk = expand(P, items[i], kids);
    uint32_t inner = 0, prims = 0;
    for (int k = 0; k < nk; k++) {
        if (kids[k].count > P.max_leaf) inner++;
        else prims += kids[k].count;
    }
    counts[i] = ((unsigned long long)inner << 32) | prims;
}

// ceil(log2(x)) for x > 0, exactly (frexp gives x = m 2^k with m in [0.5, 1)).
__device__ __forceinline__ int ceil_log2(double x) {
    int k;
    const double m = frexp(x, &k);
    return m == 0.5 ? k - 1 : k;
}

// Writes the wide node of item i (global index self_base + i), its inner
// children as items of the next level and its leaf primitives' permutation.
__global__ void k_collapse_write(CParams P, const CItem *items, uint32_t n_items, const unsigned long long *counts,
                                 const unsigned long long *incl, uint32_t self_base, uint32_t next_base,
                                 uint32_t prim_base, uint32_t prim_cursor, azd::WideNode *wide, CItem *next_items,
                                 uint32_t *out_perm, uint32_t *err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_items) return;
    CItem kids[8];
    const int nk = expand(P, items[i], kids);
    const unsigned long long off = incl[i] - counts[i];
    const uint32_t inner_off = (uint32_t)(off >> 32), prim_off = (uint32_t)(off & 0xFFFFFFFFull);

    // node bounds and slot assignment: child centre octant relative to the node centre
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int k = 0; k < nk; k++)
        for (int a = 0; a < 3; a++) {
            lo[a] = fminf(lo[a], kids[k].lo[a]);
            hi[a] = fmaxf(hi[a], kids[k].hi[a]);
        }
    double cen[8][3];
    for (int k = 0; k < nk; k++)
        for (int a = 0; a < 3; a++) {
            const double ext = fmax(1e-30, (double)hi[a] - lo[a]);
            cen[k][a] = (0.5 * ((double)kids[k].lo[a] + kids[k].hi[a]) - 0.5 * ((double)lo[a] + hi[a])) / ext;
        }
    int slot_of[8], kid_of[8];
    for (int s = 0; s < 8; s++) {
        slot_of[s] = -1;
        kid_of[s] = -1;
    }
    // repeatedly the best (child, slot) pair of the free ones; ties to the lowest child, then slot
    for (int round = 0; round < nk; round++) {
        double best = -DBL_MAX;
        int bk = -1, bs = -1;
        for (int k = 0; k < nk; k++) {
            if (slot_of[k] >= 0) continue;
            for (int s = 0; s < 8; s++) {
                if (kid_of[s] >= 0) continue;
                double sc = 0.0;
                for (int a = 0; a < 3; a++) sc += ((s >> a) & 1) ? cen[k][a] : -cen[k][a];
                if (bk < 0 || sc > best) {
                    best = sc;
                    bk = k;
                    bs = s;
                }
            }
        }
        slot_of[bk] = bs;
        kid_of[bs] = bk;
    }

    // quantisation: per axis a grid origin p and a power-of-two step with at
    // least one full step of slack on both sides of every child box; the slab
    // test folds the byte-to-float bias into its FMA at a cost of up to half a step
    azd::WideNode w;
    float p[3];
    int e[3];
    for (int a = 0; a < 3; a++) {
        const double mag = fmax(fabs((double)lo[a]), fabs((double)hi[a]));
        const double ext = fmax((double)hi[a] - lo[a], fmax(mag * 1e-6, 1e-30));
        int ex = max(-126, min(127, ceil_log2(ext / 251.0)));
        for (int guard = 0; guard < 300; guard++) {
            const double step = ldexp(1.0, ex);
            float pa = __double2float_rn((double)lo[a] - step);   // a float at least one step below lo
            for (int g2 = 0; g2 < 4 && (double)pa > (double)lo[a] - step; g2++) pa = nextafterf(pa, -FLT_MAX);
            const double top = ceil(((double)hi[a] - pa) / step) + 1.0;   // hi's byte, with slack
            p[a] = pa;
            e[a] = ex;
            if (top <= 255.0 || ex >= 127) break;
            ex++;
        }
    }
    w.px = p[0];
    w.py = p[1];
    w.pz = p[2];
    w.ex = (uint8_t)(e[0] + 127);
    w.ey = (uint8_t)(e[1] + 127);
    w.ez = (uint8_t)(e[2] + 127);
    uint8_t *qlo[3] = {w.qlo_x, w.qlo_y, w.qlo_z}, *qhi[3] = {w.qhi_x, w.qhi_y, w.qhi_z};
    for (int s = 0; s < 8; s++) {
        w.meta[s] = 0;
        for (int a = 0; a < 3; a++) {
            qlo[a][s] = 255;   // empty slot: lo > hi, never entered
            qhi[a][s] = 0;
        }
    }
    bool bad = false;
    for (int k = 0; k < nk; k++) {
        const int s = slot_of[k];
        for (int a = 0; a < 3; a++) {
            const double step = ldexp(1.0, e[a]);
            const double l = floor(((double)kids[k].lo[a] - p[a]) / step) - 1.0;   // one step of slack
            const double h = ceil(((double)kids[k].hi[a] - p[a]) / step) + 1.0;
            qlo[a][s] = (uint8_t)fmax(0.0, fmin(255.0, l));
            qhi[a][s] = (uint8_t)fmax(0.0, fmin(255.0, h));
            // the decoded box must hold the child with a full step to spare on both sides
            if ((double)p[a] + qlo[a][s] * step > (double)kids[k].lo[a] - step ||
                (double)p[a] + qhi[a][s] * step < (double)kids[k].hi[a] + step)
                bad = true;
        }
    }
    if (bad) atomicOr(err, 1u);

    // inner children: consecutive node indices in slot order; leaf primitives
    // consecutive from prim_base in slot order
    w.child_base = next_base + inner_off;
    w.prim_base = prim_base + prim_cursor + prim_off;
    uint32_t rank = 0, poff = 0;
    uint8_t imask = 0;
    for (int s = 0; s < 8; s++) {
        const int k = kid_of[s];
        if (k < 0) continue;
        if (kids[k].count > P.max_leaf) {
            imask |= (uint8_t)(1u << s);
            next_items[inner_off + rank] = kids[k];
            rank++;
        } else {
            const uint32_t sorted0 = kids[k].first - P.leaf_base;
            for (uint32_t j = 0; j < kids[k].count; j++)
                out_perm[prim_cursor + prim_off + poff + j] = P.perm[sorted0 + j];
            w.meta[s] = (uint8_t)((kids[k].count << 5) | poff);
            poff += kids[k].count;
        }
    }
    w.imask = imask;
    wide[self_base + i] = w;
}

// The root item: the root binary node with the union of its children's boxes.
__global__ void k_collapse_root(CParams P, uint32_t bin_root, CItem *items) {
    const azd::BVHNode n = P.nodes[bin_root];
    CItem r;
    r.ref = bin_root;
    r.prim = 0;
    r.first = P.range[bin_root].x;
    r.count = P.range[bin_root].y;
    r.lo[0] = fminf(n.bx.x, n.bx.z);
    r.hi[0] = fmaxf(n.bx.y, n.bx.w);
    r.lo[1] = fminf(n.by.x, n.by.z);
    r.hi[1] = fmaxf(n.by.y, n.by.w);
    r.lo[2] = fminf(n.bz.x, n.bz.z);
    r.hi[2] = fmaxf(n.bz.y, n.bz.w);
    items[0] = r;
}

// Every primitive must appear exactly once in the permutation.
__global__ void k_perm_check(const uint32_t *perm, uint32_t n, uint32_t *seen, uint32_t *err) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t v = perm[j];
    if (v >= n || atomicAdd(&seen[v], 1u) != 0) atomicOr(err, 2u);
}

template <typename T>
struct DevScratch {
    T *p = nullptr;
    ~DevScratch() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t n) { return cudaMalloc((void **)&p, (n ? n : 1) * sizeof(T)); }
};

}  // namespace

int CollapseToWide(const azd::BVHNode *d_nodes, const uint2 *d_range, uint32_t bin_root, uint32_t n,
                   uint32_t leaf_base, const uint32_t *d_sorted_perm, uint32_t max_leaf, uint32_t width,
                   azd::WideNode *d_wide, uint32_t wide_cap, uint32_t *wide_count, uint32_t *d_out_perm,
                   cudaStream_t st, uint32_t *root_out, uint32_t *depth_out) {
    if (max_leaf < 1 || max_leaf > 3) return SetError(AZ_ERR_INVALID_ARGUMENT, "leaf size must be 1..3");
    if (width != 2 && width != 4 && width != 8) return SetError(AZ_ERR_INVALID_ARGUMENT, "BVH width must be 2, 4 or 8");
    if (n == 0) return SetError(AZ_ERR_INVALID_ARGUMENT, "empty hierarchy");
    // a wide node per binary node at most: every node is made from a distinct one
    const uint32_t max_items = n > 1 ? n - 1 : 1;
    DevScratch<CItem> items_a, items_b;
    DevScratch<unsigned long long> counts, incl, total;
    DevScratch<uint32_t> flags;   // [0] error bits, [1..n] permutation check
    DevScratch<unsigned char> temp;
    AZ_CUDA_TRY(items_a.alloc(max_items));
    AZ_CUDA_TRY(items_b.alloc(max_items));
    AZ_CUDA_TRY(counts.alloc(max_items));
    AZ_CUDA_TRY(incl.alloc(max_items));
    AZ_CUDA_TRY(flags.alloc((size_t)n + 1));
    size_t temp_bytes = 0;
    AZ_CUDA_TRY(cub::DeviceScan::InclusiveSum(nullptr, temp_bytes, counts.p, incl.p, (int)max_items, st));
    AZ_CUDA_TRY(temp.alloc(temp_bytes));
    AZ_CUDA_TRY(cudaMemsetAsync(flags.p, 0, ((size_t)n + 1) * sizeof(uint32_t), st));

    CParams P;
    P.nodes = d_nodes;
    P.range = d_range;
    P.perm = d_sorted_perm;
    P.leaf_base = leaf_base;
    P.max_leaf = max_leaf;
    P.width = width;
    const uint32_t root = *wide_count;
    if (root + 1 > wide_cap) return SetError(AZ_ERR_CUDA, "BVH collapse: node pool too small");
    k_collapse_root<<<1, 1, 0, st>>>(P, bin_root, items_a.p);
    AZ_CUDA_TRY(cudaGetLastError());
    CItem *cur = items_a.p, *nxt = items_b.p;
    uint32_t n_items = 1, self_base = root, prim_cursor = 0, depth = 0;
    const int B = 128;
    for (uint32_t level = 0; n_items > 0; level++) {
        if (level > 4096) return SetError(AZ_ERR_CUDA, "BVH collapse: hierarchy deeper than 4096 levels");
        const uint32_t grid = (n_items + B - 1) / B;
        k_collapse_count<<<grid, B, 0, st>>>(P, cur, n_items, counts.p);
        AZ_CUDA_TRY(cudaGetLastError());
        AZ_CUDA_TRY(cub::DeviceScan::InclusiveSum(temp.p, temp_bytes, counts.p, incl.p, (int)n_items, st));
        unsigned long long tot = 0;
        AZ_CUDA_TRY(cudaMemcpyAsync(&tot, incl.p + (n_items - 1), sizeof(tot), cudaMemcpyDeviceToHost, st));
        AZ_CUDA_TRY(cudaStreamSynchronize(st));
        const uint32_t inner_total = (uint32_t)(tot >> 32), prim_total = (uint32_t)(tot & 0xFFFFFFFFull);
        const uint32_t next_base = self_base + n_items;
        if ((uint64_t)next_base + inner_total > wide_cap || inner_total > max_items)
            return SetError(AZ_ERR_CUDA, "BVH collapse: node pool too small");
        if ((uint64_t)prim_cursor + prim_total > n) return SetError(AZ_ERR_CUDA, "BVH collapse: primitive overflow");
        k_collapse_write<<<grid, B, 0, st>>>(P, cur, n_items, counts.p, incl.p, self_base, next_base, leaf_base,
                                             prim_cursor, d_wide, nxt, d_out_perm, flags.p);
        AZ_CUDA_TRY(cudaGetLastError());
        prim_cursor += prim_total;
        self_base = next_base;
        n_items = inner_total;
        if (inner_total) depth = level + 1;
        CItem *t = cur;
        cur = nxt;
        nxt = t;
    }
    if (prim_cursor != n) return SetError(AZ_ERR_CUDA, "BVH collapse lost primitives");
    k_perm_check<<<(n + 255) / 256, 256, 0, st>>>(d_out_perm, n, flags.p + 1, flags.p);
    AZ_CUDA_TRY(cudaGetLastError());
    uint32_t errbits = 0;
    AZ_CUDA_TRY(cudaMemcpyAsync(&errbits, flags.p, sizeof(errbits), cudaMemcpyDeviceToHost, st));
    AZ_CUDA_TRY(cudaStreamSynchronize(st));
    if (errbits & 1u) return SetError(AZ_ERR_CUDA, "BVH collapse: a quantised box does not contain its child");
    if (errbits & 2u) return SetError(AZ_ERR_CUDA, "BVH collapse did not produce a permutation of the primitives");
    *wide_count = self_base;
    *root_out = root;
    if (depth_out) *depth_out = depth;
    return AZ_OK;
}

}  // namespace az
