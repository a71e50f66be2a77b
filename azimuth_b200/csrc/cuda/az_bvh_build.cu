// GPU LBVH construction (Karras, "Maximizing Parallelism in the Construction
// of BVHs, Octrees, and k-d Trees", HPG 2012): 63-bit Morton codes (21 bits per
// axis) of the box centroids, a radix sort of (code, primitive) pairs, one
// thread per internal node to find its range and split (equal codes are told
// apart by their sorted position, as in the paper), and a bottom-up pass that
// fills each node with the (slightly enlarged) boxes of both children.
#include <cub/cub.cuh>

#include <cfloat>

#include "az_internal.h"

namespace az {
namespace {

// 21 bits spread to every third bit of a 63-bit word.
__device__ __forceinline__ unsigned long long spread3(unsigned long long v) {
    v &= 0x1FFFFFull;
    v = (v | (v << 32)) & 0x001F00000000FFFFull;
    v = (v | (v << 16)) & 0x001F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__global__ void k_bounds_reduce(const float4 *lo, const float4 *hi, uint32_t n, float *out6) {
    // centroid bounds: one block, strided
    __shared__ float s[6][256];
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        float4 a = lo[i], b = hi[i];
        float c[3] = {0.5f * (a.x + b.x), 0.5f * (a.y + b.y), 0.5f * (a.z + b.z)};
        for (int k = 0; k < 3; k++) {
            mn[k] = fminf(mn[k], c[k]);
            mx[k] = fmaxf(mx[k], c[k]);
        }
    }
    for (int k = 0; k < 3; k++) {
        s[k][threadIdx.x] = mn[k];
        s[3 + k][threadIdx.x] = mx[k];
    }
    __syncthreads();
    for (uint32_t st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st)
            for (int k = 0; k < 3; k++) {
                s[k][threadIdx.x] = fminf(s[k][threadIdx.x], s[k][threadIdx.x + st]);
                s[3 + k][threadIdx.x] = fmaxf(s[3 + k][threadIdx.x], s[3 + k][threadIdx.x + st]);
            }
        __syncthreads();
    }
    if (threadIdx.x < 6) out6[threadIdx.x] = s[threadIdx.x][0];
}

__global__ void k_morton(const float4 *lo, const float4 *hi, uint32_t n, const float *bounds6,
                         unsigned long long *keys, uint32_t *vals) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 a = lo[i], b = hi[i];
    double c[3] = {0.5 * ((double)a.x + b.x), 0.5 * ((double)a.y + b.y), 0.5 * ((double)a.z + b.z)};
    unsigned long long q[3];
    for (int k = 0; k < 3; k++) {
        double ext = (double)bounds6[3 + k] - bounds6[k];
        double u = ext > 0.0 ? (c[k] - bounds6[k]) / ext : 0.5;
        u = fmin(fmax(u, 0.0), 1.0);
        q[k] = (unsigned long long)fmin(u * 2097152.0, 2097151.0);
    }
    keys[i] = (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
    vals[i] = i;
}

// Common-prefix length of sorted keys i and j; equal keys continue with the
// bits of their positions (Karras 2012, section 4).
__device__ __forceinline__ int delta(const unsigned long long *k, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    unsigned long long a = k[i], b = k[j];
    if (a == b) return 64 + __clz((uint32_t)(i ^ j));
    return __clzll(a ^ b);
}

// One thread per internal node i in [0, n-2]: children (internal index or
// leaf flagged with bit 31), parents, and the node's sorted primitive range.
__global__ void k_karras(const unsigned long long *k, int n, uint32_t *left, uint32_t *right, int *parent_int,
                         int *parent_leaf, uint2 *range, uint32_t leaf_base) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = (delta(k, n, i, i + 1) - delta(k, n, i, i - 1)) > 0 ? 1 : -1;
    int dmin = delta(k, n, i, i - d);
    int lmax = 2;
    while (delta(k, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(k, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = delta(k, n, i, j);
    int s = 0;
    int t = l;
    do {
        t = (t + 1) >> 1;
        if (delta(k, n, i, i + (s + t) * d) > dnode) s += t;
    } while (t > 1);
    int gamma = i + s * d + min(d, 0);
    int lo = min(i, j), hi = max(i, j);
    range[i] = make_uint2(leaf_base + (uint32_t)lo, (uint32_t)(hi - lo + 1));
    uint32_t lc, rc;
    if (lo == gamma) {
        lc = 0x80000000u | (uint32_t)gamma;
        parent_leaf[gamma] = i;
    } else {
        lc = (uint32_t)gamma;
        parent_int[gamma] = i;
    }
    if (hi == gamma + 1) {
        rc = 0x80000000u | (uint32_t)(gamma + 1);
        parent_leaf[gamma + 1] = i;
    } else {
        rc = (uint32_t)(gamma + 1);
        parent_int[gamma + 1] = i;
    }
    left[i] = lc;
    right[i] = rc;
}

__device__ __forceinline__ void pad_box(float4 &lo, float4 &hi) {
    // enlarge by 2^-19 of the largest magnitude so that rounding in the slab
    // test never rejects a primitive lying on a face of its box
    float m = fmaxf(fmaxf(fmaxf(fabsf(lo.x), fabsf(lo.y)), fmaxf(fabsf(lo.z), fabsf(hi.x))),
                    fmaxf(fabsf(hi.y), fabsf(hi.z)));
    float p = m * 1.9073486328125e-06f + 1e-30f;
    lo.x -= p; lo.y -= p; lo.z -= p;
    hi.x += p; hi.y += p; hi.z += p;
}

// Bottom-up: one thread per leaf walks to the root; the second child to
// arrive at a node writes it.
__global__ void k_fill(const uint32_t *order, const float4 *plo, const float4 *phi, int n,
                       const uint32_t *left, const uint32_t *right, const int *parent_int, const int *parent_leaf,
                       float4 *ilo, float4 *ihi, unsigned int *visits, azd::BVHNode *nodes, uint32_t node_base,
                       uint32_t leaf_base) {
    int leaf = blockIdx.x * blockDim.x + threadIdx.x;
    if (leaf >= n) return;
    int node = parent_leaf[leaf];
    for (int guard = 0; node >= 0 && guard < n; guard++) {
        __threadfence();
        if (atomicAdd(&visits[node], 1u) == 0) return;  // first arrival: the sibling finishes the node
        __threadfence();
        uint32_t c[2] = {left[node], right[node]};
        float4 blo[2], bhi[2];
        uint32_t ref[2], cnt[2];
        for (int s = 0; s < 2; s++) {
            if (c[s] & 0x80000000u) {
                uint32_t li = c[s] & 0x7FFFFFFFu;
                uint32_t prim = order[li];
                blo[s] = plo[prim];
                bhi[s] = phi[prim];
                ref[s] = leaf_base + li;
                cnt[s] = 1;
            } else {
                blo[s] = __ldcg(ilo + c[s]);
                bhi[s] = __ldcg(ihi + c[s]);
                ref[s] = node_base + c[s];
                cnt[s] = 0;
            }
        }
        float4 ulo = make_float4(fminf(blo[0].x, blo[1].x), fminf(blo[0].y, blo[1].y), fminf(blo[0].z, blo[1].z), 0);
        float4 uhi = make_float4(fmaxf(bhi[0].x, bhi[1].x), fmaxf(bhi[0].y, bhi[1].y), fmaxf(bhi[0].z, bhi[1].z), 0);
        __stcg(ilo + node, ulo);
        __stcg(ihi + node, uhi);
        pad_box(blo[0], bhi[0]);
        pad_box(blo[1], bhi[1]);
        azd::BVHNode out;
        out.bx = make_float4(blo[0].x, bhi[0].x, blo[1].x, bhi[1].x);
        out.by = make_float4(blo[0].y, bhi[0].y, blo[1].y, bhi[1].y);
        out.bz = make_float4(blo[0].z, bhi[0].z, blo[1].z, bhi[1].z);
        out.ch = make_uint4(ref[0], ref[1], cnt[0], cnt[1]);
        nodes[node_base + node] = out;
        node = parent_int[node];
    }
}

__global__ void k_copy_u32(const uint32_t *src, uint32_t n, uint32_t *dst) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i];
}

__global__ void k_single(const float4 *lo, const float4 *hi, azd::BVHNode *nodes, uint2 *range, uint32_t node_base,
                         uint32_t leaf_base, uint32_t *perm) {
    float4 a = lo[0], b = hi[0];
    pad_box(a, b);
    azd::BVHNode out;
    // child 1 is an empty box (lo > hi) that no ray enters
    out.bx = make_float4(a.x, b.x, FLT_MAX, -FLT_MAX);
    out.by = make_float4(a.y, b.y, FLT_MAX, -FLT_MAX);
    out.bz = make_float4(a.z, b.z, FLT_MAX, -FLT_MAX);
    out.ch = make_uint4(leaf_base, leaf_base, 1u, 1u);
    nodes[node_base] = out;
    range[node_base] = make_uint2(leaf_base, 1u);
    perm[0] = 0;
}

template <typename T>
struct Scratch {
    T *p = nullptr;
    ~Scratch() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t n) { return cudaMalloc((void **)&p, n * sizeof(T) + 16); }
};

// ---- PLOC: parallel locally-ordered clustering (Meister, Bittner, "Parallel
// Locally-Ordered Clustering for Bounding Volume Hierarchy Construction",
// IEEE TVCG 2018).  The clusters, kept in Morton order, each find the
// neighbour within `radius` positions whose merged box has the smallest
// surface area; mutual nearest neighbours merge (the lower position keeps
// the new node), and the survivors are compacted.  Ties go to the lowest
// position, and node numbers come from scans, so the tree is the same on
// every build.

constexpr int kPlocRadius = 24;
constexpr uint32_t kLeafBit = 0x80000000u;

__device__ __forceinline__ float merged_area(float4 alo, float4 ahi, float4 blo, float4 bhi) {
    const float dx = fmaxf(ahi.x, bhi.x) - fminf(alo.x, blo.x);
    const float dy = fmaxf(ahi.y, bhi.y) - fminf(alo.y, blo.y);
    const float dz = fmaxf(ahi.z, bhi.z) - fminf(alo.z, blo.z);
    return dx * dy + dy * dz + dz * dx;
}

__global__ void k_ploc_init(const uint32_t *order, const float4 *plo, const float4 *phi, uint32_t n, uint32_t *ids,
                            float4 *lo, float4 *hi) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    ids[i] = kLeafBit | i;   // leaf: its sorted position
    lo[i] = plo[order[i]];
    hi[i] = phi[order[i]];
}

__global__ void k_ploc_nn(const float4 *lo, const float4 *hi, uint32_t count, int radius, uint32_t *nn) {
    const int i = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (i >= (int)count) return;
    const float4 a0 = lo[i], a1 = hi[i];
    float best = FLT_MAX;
    int bj = i == 0 ? 1 : i - 1;
    const int j0 = max(0, i - radius), j1 = min((int)count - 1, i + radius);
    for (int j = j0; j <= j1; j++) {
        if (j == i) continue;
        const float a = merged_area(a0, a1, __ldg(lo + j), __ldg(hi + j));
        if (a < best) {
            best = a;
            bj = j;
        }
    }
    nn[i] = (uint32_t)bj;
}

// Per cluster: bit 32 "creates a node" (mutual pair, lower position), bit 0 "survives".
__global__ void k_ploc_flags(const uint32_t *nn, uint32_t count, unsigned long long *flags) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const uint32_t j = nn[i];
    const bool mutual = nn[j] == i;
    flags[i] = ((unsigned long long)(mutual && i < j) << 32) | (unsigned long long)!(mutual && i > j);
}

__device__ __forceinline__ uint32_t cluster_count(uint32_t id, const uint32_t *node_count) {
    return (id & kLeafBit) ? 1u : node_count[id];
}

__global__ void k_ploc_merge(const uint32_t *ids, const float4 *lo, const float4 *hi, const uint32_t *nn,
                             uint32_t count, const unsigned long long *flags, const unsigned long long *incl,
                             uint32_t node_begin, uint32_t *new_ids, float4 *new_lo, float4 *new_hi,
                             uint32_t *node_left, uint32_t *node_right, float4 *node_lo, float4 *node_hi,
                             uint32_t *node_count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const unsigned long long f = flags[i];
    if (!(f & 1ull)) return;   // merged into its lower neighbour's node
    const unsigned long long ex = incl[i] - f;
    const uint32_t pos = (uint32_t)(ex & 0xFFFFFFFFull);
    if (f >> 32) {
        const uint32_t j = nn[i], id = node_begin + (uint32_t)(ex >> 32);
        const uint32_t a = ids[i], b = ids[j];
        const float4 alo = lo[i], ahi = hi[i], blo = lo[j], bhi = hi[j];
        const float4 ulo = make_float4(fminf(alo.x, blo.x), fminf(alo.y, blo.y), fminf(alo.z, blo.z), 0.0f);
        const float4 uhi = make_float4(fmaxf(ahi.x, bhi.x), fmaxf(ahi.y, bhi.y), fmaxf(ahi.z, bhi.z), 0.0f);
        node_left[id] = a;
        node_right[id] = b;
        node_lo[id] = ulo;
        node_hi[id] = uhi;
        node_count[id] = cluster_count(a, node_count) + cluster_count(b, node_count);
        new_ids[pos] = id;
        new_lo[pos] = ulo;
        new_hi[pos] = uhi;
    } else {
        new_ids[pos] = ids[i];
        new_lo[pos] = lo[i];
        new_hi[pos] = hi[i];
    }
}

// Depth-first positions, top-down one merge round at a time (a node's parent
// was made in a later round): the left child starts where its parent does,
// the right child after the left child's primitives.
__global__ void k_ploc_first(uint32_t node_begin, uint32_t nodes, const uint32_t *node_left,
                             const uint32_t *node_right, const uint32_t *node_count, uint32_t *node_first,
                             uint32_t *leaf_first) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nodes) return;
    const uint32_t id = node_begin + k, f = node_first[id];
    const uint32_t a = node_left[id], b = node_right[id];
    const uint32_t fb = f + cluster_count(a, node_count);
    if (a & kLeafBit) leaf_first[a & ~kLeafBit] = f;
    else node_first[a] = f;
    if (b & kLeafBit) leaf_first[b & ~kLeafBit] = fb;
    else node_first[b] = fb;
}

__global__ void k_ploc_emit(uint32_t n_nodes, const uint32_t *node_left, const uint32_t *node_right,
                            const float4 *node_lo, const float4 *node_hi, const uint32_t *node_count,
                            const uint32_t *node_first, const uint32_t *leaf_first, const float4 *plo,
                            const float4 *phi, const uint32_t *order, azd::BVHNode *nodes, uint2 *range,
                            uint32_t node_base, uint32_t leaf_base, uint32_t *err) {
    const uint32_t id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n_nodes) return;
    const uint32_t n = n_nodes + 1;
    const uint32_t c[2] = {node_left[id], node_right[id]};
    float4 blo[2], bhi[2];
    uint32_t ref[2], cnt[2];
    for (int s = 0; s < 2; s++) {
        if (c[s] & kLeafBit) {
            const uint32_t li = c[s] & ~kLeafBit;
            blo[s] = plo[order[li]];
            bhi[s] = phi[order[li]];
            uint32_t pos = leaf_first[li];
            if (pos >= n) {   // a leaf the depth-first pass did not reach: a broken tree
                atomicOr(err, 1u);
                pos = 0;
            }
            ref[s] = leaf_base + pos;
            cnt[s] = 1;
        } else {
            blo[s] = node_lo[c[s]];
            bhi[s] = node_hi[c[s]];
            ref[s] = node_base + c[s];
            cnt[s] = 0;
        }
    }
    pad_box(blo[0], bhi[0]);
    pad_box(blo[1], bhi[1]);
    azd::BVHNode out;
    out.bx = make_float4(blo[0].x, bhi[0].x, blo[1].x, bhi[1].x);
    out.by = make_float4(blo[0].y, bhi[0].y, blo[1].y, bhi[1].y);
    out.bz = make_float4(blo[0].z, bhi[0].z, blo[1].z, bhi[1].z);
    out.ch = make_uint4(ref[0], ref[1], cnt[0], cnt[1]);
    nodes[node_base + id] = out;
    uint32_t first = node_first[id], count = node_count[id];
    if ((uint64_t)first + count > n || count < 2) {
        atomicOr(err, 1u);
        first = 0;
        count = 2;
    }
    range[node_base + id] = make_uint2(leaf_base + first, count);
}

// Sorted position -> depth-first position: the primitive order the leaves' references use.
__global__ void k_ploc_perm(const uint32_t *order, const uint32_t *leaf_first, uint32_t n, uint32_t *perm) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n && leaf_first[s] < n) perm[leaf_first[s]] = order[s];   // the collapse checks it is a permutation
}

}  // namespace

int BuildPLOC(const float4 *d_lo, const float4 *d_hi, uint32_t n, azd::BVHNode *d_nodes, uint2 *d_range,
              uint32_t node_base, uint32_t leaf_base, uint32_t *d_perm, cudaStream_t stream, uint32_t *root_out) {
    if (n <= 2) return BuildLBVH(d_lo, d_hi, n, d_nodes, d_range, node_base, leaf_base, d_perm, stream, root_out);
    Scratch<float> bounds;
    Scratch<unsigned long long> keys, keys_sorted, flags, incl;
    Scratch<uint32_t> vals, order, ids_a, ids_b, nn, nl, nr, ncount, nfirst, lfirst;
    Scratch<float4> lo_a, hi_a, lo_b, hi_b, nlo, nhi;
    Scratch<unsigned char> temp, temp2;
    Scratch<uint32_t> err;
    AZ_CUDA_TRY(err.alloc(1));
    AZ_CUDA_TRY(cudaMemsetAsync(err.p, 0, sizeof(uint32_t), stream));
    AZ_CUDA_TRY(bounds.alloc(6));
    AZ_CUDA_TRY(keys.alloc(n));
    AZ_CUDA_TRY(keys_sorted.alloc(n));
    AZ_CUDA_TRY(vals.alloc(n));
    AZ_CUDA_TRY(order.alloc(n));
    AZ_CUDA_TRY(ids_a.alloc(n));
    AZ_CUDA_TRY(ids_b.alloc(n));
    AZ_CUDA_TRY(lo_a.alloc(n));
    AZ_CUDA_TRY(hi_a.alloc(n));
    AZ_CUDA_TRY(lo_b.alloc(n));
    AZ_CUDA_TRY(hi_b.alloc(n));
    AZ_CUDA_TRY(nn.alloc(n));
    AZ_CUDA_TRY(flags.alloc(n));
    AZ_CUDA_TRY(incl.alloc(n));
    AZ_CUDA_TRY(nl.alloc(n));
    AZ_CUDA_TRY(nr.alloc(n));
    AZ_CUDA_TRY(nlo.alloc(n));
    AZ_CUDA_TRY(nhi.alloc(n));
    AZ_CUDA_TRY(ncount.alloc(n));
    AZ_CUDA_TRY(nfirst.alloc(n));
    AZ_CUDA_TRY(lfirst.alloc(n));
    size_t temp_bytes = 0, temp2_bytes = 0;
    AZ_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys.p, keys_sorted.p, vals.p, order.p, (int)n, 0,
                                                63, stream));
    AZ_CUDA_TRY(temp.alloc(temp_bytes));
    AZ_CUDA_TRY(cub::DeviceScan::InclusiveSum(nullptr, temp2_bytes, flags.p, incl.p, (int)n, stream));
    AZ_CUDA_TRY(temp2.alloc(temp2_bytes));
    const int B = 256;
    k_bounds_reduce<<<1, 256, 0, stream>>>(d_lo, d_hi, n, bounds.p);
    k_morton<<<(n + B - 1) / B, B, 0, stream>>>(d_lo, d_hi, n, bounds.p, keys.p, vals.p);
    AZ_CUDA_TRY(cudaGetLastError());
    AZ_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp.p, temp_bytes, keys.p, keys_sorted.p, vals.p, order.p, (int)n, 0,
                                                63, stream));
    k_ploc_init<<<(n + B - 1) / B, B, 0, stream>>>(order.p, d_lo, d_hi, n, ids_a.p, lo_a.p, hi_a.p);
    AZ_CUDA_TRY(cudaGetLastError());
    std::vector<std::pair<uint32_t, uint32_t>> rounds;   // nodes made per round: (first id, count)
    uint32_t count = n, made = 0;
    uint32_t *ids = ids_a.p, *ids2 = ids_b.p;
    float4 *lo = lo_a.p, *hi = hi_a.p, *lo2 = lo_b.p, *hi2 = hi_b.p;
    for (int round = 0; count > 1; round++) {
        if (round > (int)n) return SetError(AZ_ERR_CUDA, "PLOC made no progress");
        const uint32_t grid = (count + B - 1) / B;
        k_ploc_nn<<<grid, B, 0, stream>>>(lo, hi, count, kPlocRadius, nn.p);
        k_ploc_flags<<<grid, B, 0, stream>>>(nn.p, count, flags.p);
        AZ_CUDA_TRY(cudaGetLastError());
        AZ_CUDA_TRY(cub::DeviceScan::InclusiveSum(temp2.p, temp2_bytes, flags.p, incl.p, (int)count, stream));
        k_ploc_merge<<<grid, B, 0, stream>>>(ids, lo, hi, nn.p, count, flags.p, incl.p, made, ids2, lo2, hi2, nl.p, nr.p,
                                            nlo.p, nhi.p, ncount.p);
        AZ_CUDA_TRY(cudaGetLastError());
        unsigned long long tot = 0;
        AZ_CUDA_TRY(cudaMemcpyAsync(&tot, incl.p + (count - 1), sizeof(tot), cudaMemcpyDeviceToHost, stream));
        AZ_CUDA_TRY(cudaStreamSynchronize(stream));
        const uint32_t merges = (uint32_t)(tot >> 32), survivors = (uint32_t)(tot & 0xFFFFFFFFull);
        if (merges == 0 || made + merges > n - 1) return SetError(AZ_ERR_CUDA, "PLOC made no progress");
        rounds.push_back({made, merges});
        made += merges;
        count = survivors;
        std::swap(ids, ids2);
        std::swap(lo, lo2);
        std::swap(hi, hi2);
    }
    if (made != n - 1) return SetError(AZ_ERR_CUDA, "PLOC did not build a binary tree");
    // depth-first positions from the root (the last node made) down
    const uint32_t root = n - 2;
    AZ_CUDA_TRY(cudaMemsetAsync(nfirst.p, 0, (size_t)n * sizeof(uint32_t), stream));
    AZ_CUDA_TRY(cudaMemsetAsync(lfirst.p, 0xFF, (size_t)n * sizeof(uint32_t), stream));
    for (size_t r = rounds.size(); r-- > 0;) {
        const uint32_t k = rounds[r].second;
        k_ploc_first<<<(k + B - 1) / B, B, 0, stream>>>(rounds[r].first, k, nl.p, nr.p, ncount.p, nfirst.p, lfirst.p);
    }
    AZ_CUDA_TRY(cudaGetLastError());
    k_ploc_emit<<<(n - 1 + B - 1) / B, B, 0, stream>>>(n - 1, nl.p, nr.p, nlo.p, nhi.p, ncount.p, nfirst.p, lfirst.p,
                                                       d_lo, d_hi, order.p, d_nodes, d_range, node_base, leaf_base,
                                                       err.p);
    k_ploc_perm<<<(n + B - 1) / B, B, 0, stream>>>(order.p, lfirst.p, n, d_perm);
    AZ_CUDA_TRY(cudaGetLastError());
    uint32_t err_h = 0;
    AZ_CUDA_TRY(cudaMemcpyAsync(&err_h, err.p, sizeof(err_h), cudaMemcpyDeviceToHost, stream));
    AZ_CUDA_TRY(cudaStreamSynchronize(stream));   // scratch is freed on return
    if (err_h) return SetError(AZ_ERR_CUDA, "PLOC: the depth-first numbering of the tree failed");
    *root_out = node_base + root;
    return AZ_OK;
}

int BuildLBVH(const float4 *d_lo, const float4 *d_hi, uint32_t n, azd::BVHNode *d_nodes, uint2 *d_range,
              uint32_t node_base, uint32_t leaf_base, uint32_t *d_perm, cudaStream_t stream, uint32_t *root_out) {
    if (n == 0) {
        *root_out = 0xFFFFFFFFu;
        return AZ_OK;
    }
    *root_out = node_base;
    if (n == 1) {
        k_single<<<1, 1, 0, stream>>>(d_lo, d_hi, d_nodes, d_range, node_base, leaf_base, d_perm);
        AZ_CUDA_TRY(cudaGetLastError());
        return AZ_OK;
    }
    Scratch<float> bounds;
    Scratch<unsigned long long> keys, keys_sorted;
    Scratch<uint32_t> vals, vals_sorted;
    Scratch<uint32_t> left, right;
    Scratch<int> parent_int, parent_leaf;
    Scratch<float4> ilo, ihi;
    Scratch<unsigned int> visits;
    Scratch<unsigned char> temp;
    AZ_CUDA_TRY(bounds.alloc(6));
    AZ_CUDA_TRY(keys.alloc(n));
    AZ_CUDA_TRY(keys_sorted.alloc(n));
    AZ_CUDA_TRY(vals.alloc(n));
    AZ_CUDA_TRY(vals_sorted.alloc(n));
    AZ_CUDA_TRY(left.alloc(n));
    AZ_CUDA_TRY(right.alloc(n));
    AZ_CUDA_TRY(parent_int.alloc(n));
    AZ_CUDA_TRY(parent_leaf.alloc(n));
    AZ_CUDA_TRY(ilo.alloc(n));
    AZ_CUDA_TRY(ihi.alloc(n));
    AZ_CUDA_TRY(visits.alloc(n));
    size_t temp_bytes = 0;
    AZ_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys.p, keys_sorted.p, vals.p, vals_sorted.p,
                                                (int)n, 0, 63, stream));
    AZ_CUDA_TRY(temp.alloc(temp_bytes));
    const int B = 256;
    uint32_t grid = (n + B - 1) / B;
    k_bounds_reduce<<<1, 256, 0, stream>>>(d_lo, d_hi, n, bounds.p);
    k_morton<<<grid, B, 0, stream>>>(d_lo, d_hi, n, bounds.p, keys.p, vals.p);
    AZ_CUDA_TRY(cudaGetLastError());
    AZ_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp.p, temp_bytes, keys.p, keys_sorted.p, vals.p, vals_sorted.p,
                                                (int)n, 0, 63, stream));
    AZ_CUDA_TRY(cudaMemsetAsync(parent_int.p, 0xFF, n * sizeof(int), stream));   // root's parent = -1
    AZ_CUDA_TRY(cudaMemsetAsync(visits.p, 0, n * sizeof(unsigned int), stream));
    k_karras<<<grid, B, 0, stream>>>(keys_sorted.p, (int)n, left.p, right.p, parent_int.p, parent_leaf.p,
                                     d_range + node_base, leaf_base);
    k_fill<<<grid, B, 0, stream>>>(vals_sorted.p, d_lo, d_hi, (int)n, left.p, right.p, parent_int.p, parent_leaf.p,
                                   ilo.p, ihi.p, visits.p, d_nodes, node_base, leaf_base);
    k_copy_u32<<<grid, B, 0, stream>>>(vals_sorted.p, n, d_perm);
    AZ_CUDA_TRY(cudaGetLastError());
    // scratch is freed when this returns: finish the work that uses it
    AZ_CUDA_TRY(cudaStreamSynchronize(stream));
    return AZ_OK;
}

}  // namespace az
