// Neural path guiding: the network's kernels (hash-grid encoding, fully
// fused MLP forward and backward on BF16 tensor cores, loss, Adam) and the
// guided render driver.  Network and proposal are described in az_guide.cuh.
//
// The MLP runs warp-synchronously on 16 rows at a time with
// mma.sync.m16n8k16 (BF16 inputs, FP32 accumulation): the accumulator
// fragments of one layer are, after ReLU and conversion, exactly the A
// fragments of the next, so activations stay in registers; weights sit in
// shared memory already arranged as B fragments (one 8-byte load per lane
// per 16x8 tile).  Training keeps each layer's input in shared memory for the
// backward pass: dX = dY W^T on the tensor cores with a second, transposed
// copy of the fragments, dW = X^T dY on the tensor cores with operands
// gathered from the row-major copies and accumulated per block in shared
// memory (each entry summed by one warp in a fixed order), and the encoding
// gradient scattered into the hash grid as fixed-point integers; training is
// therefore deterministic: the same rows give the same step bit for bit.
// Adam keeps FP32 master weights and refreshes the BF16 fragments and the
// FP16 grid after every step.
#include <cub/cub.cuh>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "az_guide.cuh"
#include "az_internal.h"
#include "az_render.h"
#include "az_shade.cuh"
#include "azimuth_gpu.h"

namespace az {
namespace {

using namespace azd;

constexpr int W = GUIDE_WIDTH;
constexpr int NW = GUIDE_LAYERS * W * W;             // MLP weights
constexpr int NFRAG = GUIDE_LAYERS * 4 * 8 * 32;     // B fragments (uint2) per copy
constexpr int XS = W + 8;                            // row stride (bf16) of the shared activation copies
constexpr int OS = W + 4;                            // row stride (fp32) of the shared output rows
constexpr int kWarps = 4;                            // warps per block of the training kernel
constexpr int kInferWarps = 8;                       // warps per block of the inference kernel

// Parameters of the network as the kernels see them.
struct GuideNetDev {
    const __nv_bfloat16 *wtc; // tcgen05 B operands, 64 x 64 K-major in 8x8 core matrices: per layer W^T
                              // (forward), then per layer W (dX of the backward pass)
    const uint2 *wf;          // forward B fragments [layer][kk][nn][lane]
    const uint2 *wt;          // transposed B fragments for dX = dY W^T
    const float *bias;        // output-layer bias [64]
    const __half2 *grid;      // [level][GUIDE_T] features
    uint32_t res[GUIDE_LEVELS];
    float lo[3], inv_ext[3];  // position normalisation onto [0, 1]^3
};

// Byte offset of element (r, k) of a 64-column K-major operand in the
// canonical no-swizzle layout of tcgen05.mma: 8 x 8 core matrices of 128
// contiguous bytes (8 rows of 16 bytes), the 8 core matrices of a row group
// along K at 128-byte steps (leading byte offset), row groups at 1024-byte
// steps (stride byte offset).
__host__ __device__ __forceinline__ uint32_t tc_offset(uint32_t r, uint32_t k) {
    return ((r >> 3) * 8u + (k >> 3)) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ float2 unpack_bf16(uint32_t u) {
    __nv_bfloat162 v = *reinterpret_cast<__nv_bfloat162 *>(&u);
    return __bfloat1622float2(v);
}

__device__ __forceinline__ void mma16816(float (&c)[4], const uint32_t *a, uint2 b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

__device__ __forceinline__ f3 normalise_pos(const GuideNetDev &N, f3 p) {
    return mk(fminf(1.0f, fmaxf(0.0f, (p.x - N.lo[0]) * N.inv_ext[0])),
              fminf(1.0f, fmaxf(0.0f, (p.y - N.lo[1]) * N.inv_ext[1])),
              fminf(1.0f, fmaxf(0.0f, (p.z - N.lo[2]) * N.inv_ext[2])));
}

// Trilinear corners of level l at normalised position p.
struct Corners {
    uint32_t idx[8];
    float w[8];
};

__device__ __forceinline__ void grid_corners(const GuideNetDev &N, int l, f3 p, Corners &c) {
    const uint32_t res = N.res[l];
    const float fr = (float)res;
    const float x = p.x * fr, y = p.y * fr, z = p.z * fr;
    const uint32_t ix = min((uint32_t)x, res - 1u), iy = min((uint32_t)y, res - 1u), iz = min((uint32_t)z, res - 1u);
    const float fx = x - (float)ix, fy = y - (float)iy, fz = z - (float)iz;
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const uint32_t dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
        c.w[k] = (dx ? fx : 1.0f - fx) * (dy ? fy : 1.0f - fy) * (dz ? fz : 1.0f - fz);
        c.idx[k] = (uint32_t)l * GUIDE_T + guide_index(ix + dx, iy + dy, iz + dz, res);
    }
}

__device__ __forceinline__ float2 grid_feature(const GuideNetDev &N, int l, f3 p) {
    Corners c;
    grid_corners(N, l, p, c);
    float2 f = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const float2 v = __half22float2(N.grid[c.idx[k]]);
        f.x += c.w[k] * v.x;
        f.y += c.w[k] * v.y;
    }
    return f;
}

// Network inputs of rows g and g + 8 of the warp's 16-row tile as the A
// fragments of the first layer.  Input columns: 0..31 the hash-grid features
// (level l at 2l, 2l+1), 32..34 the normal, 35..37 the outgoing direction,
// 38 a constant 1, the rest 0.  Lane (g, t) holds, per row, columns 2t, 2t+1,
// 2t+8, 2t+9 of each 16-column tile: grid levels t, t+4, t+8, t+12.
__device__ __forceinline__ void encode_rows(const GuideNetDev &N, f3 p0, f3 n0, f3 o0, f3 p1, f3 n1, f3 o1,
                                            uint32_t t, uint32_t (&act)[16]) {
#pragma unroll
    for (int kk = 0; kk < 2; kk++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int l = (int)t + 4 * h + 8 * kk;
            const float2 a = grid_feature(N, l, p0), b = grid_feature(N, l, p1);
            act[kk * 4 + 2 * h + 0] = pack_bf16(a.x, a.y);
            act[kk * 4 + 2 * h + 1] = pack_bf16(b.x, b.y);
        }
    const float e0[8] = {n0.x, n0.y, n0.z, o0.x, o0.y, o0.z, 1.0f, 0.0f};
    const float e1[8] = {n1.x, n1.y, n1.z, o1.x, o1.y, o1.z, 1.0f, 0.0f};
    act[8] = pack_bf16(e0[2 * t], e0[2 * t + 1]);
    act[9] = pack_bf16(e1[2 * t], e1[2 * t + 1]);
    act[10] = act[11] = 0u;
    act[12] = act[13] = act[14] = act[15] = 0u;
}

// One layer: acc (8 column tiles of 16x8) = A (16x64) * B (64x64).
__device__ __forceinline__ void layer_mma(const uint32_t (&act)[16], const uint2 *frag, uint32_t lane,
                                          float (&acc)[8][4]) {
#pragma unroll
    for (int nn = 0; nn < 8; nn++) {
        acc[nn][0] = acc[nn][1] = acc[nn][2] = acc[nn][3] = 0.0f;
#pragma unroll
        for (int kk = 0; kk < 4; kk++) mma16816(acc[nn], &act[kk * 4], frag[(kk * 8 + nn) * 32 + lane]);
    }
}

// Accumulators (D fragments) to the next layer's A fragments, after ReLU.
__device__ __forceinline__ void relu_to_act(const float (&acc)[8][4], uint32_t (&act)[16]) {
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
        act[kk * 4 + 0] = pack_bf16(fmaxf(acc[2 * kk][0], 0.0f), fmaxf(acc[2 * kk][1], 0.0f));
        act[kk * 4 + 1] = pack_bf16(fmaxf(acc[2 * kk][2], 0.0f), fmaxf(acc[2 * kk][3], 0.0f));
        act[kk * 4 + 2] = pack_bf16(fmaxf(acc[2 * kk + 1][0], 0.0f), fmaxf(acc[2 * kk + 1][1], 0.0f));
        act[kk * 4 + 3] = pack_bf16(fmaxf(acc[2 * kk + 1][2], 0.0f), fmaxf(acc[2 * kk + 1][3], 0.0f));
    }
}

// A fragments of a 16x64 tile to its row-major BF16 copy (row stride XS).
__device__ __forceinline__ void store_act(const uint32_t (&act)[16], __nv_bfloat16 *X, uint32_t g, uint32_t t) {
#pragma unroll
    for (int kk = 0; kk < 4; kk++) {
        *reinterpret_cast<uint32_t *>(X + g * XS + 16 * kk + 2 * t) = act[kk * 4 + 0];
        *reinterpret_cast<uint32_t *>(X + (g + 8) * XS + 16 * kk + 2 * t) = act[kk * 4 + 1];
        *reinterpret_cast<uint32_t *>(X + g * XS + 16 * kk + 2 * t + 8) = act[kk * 4 + 2];
        *reinterpret_cast<uint32_t *>(X + (g + 8) * XS + 16 * kk + 2 * t + 8) = act[kk * 4 + 3];
    }
}

// Output-layer accumulators plus bias to rows of `out` (row stride OS).
__device__ __forceinline__ void store_out(const float (&acc)[8][4], const float *bias, float *out, uint32_t g,
                                          uint32_t t) {
#pragma unroll
    for (int nn = 0; nn < 8; nn++) {
        const int c = 8 * nn + 2 * t;
        out[g * OS + c] = acc[nn][0] + bias[c];
        out[g * OS + c + 1] = acc[nn][1] + bias[c + 1];
        out[(g + 8) * OS + c] = acc[nn][2] + bias[c];
        out[(g + 8) * OS + c + 1] = acc[nn][3] + bias[c + 1];
    }
}

// Raw outputs of one row to the proposal (az_guide.cuh).
__device__ void decode_lobes(const float *o, GuideLobes &G) {
    float mx = -FLT_MAX;
#pragma unroll
    for (int k = 0; k < GUIDE_LOBES; k++) mx = fmaxf(mx, o[5 * k + 4]);
    float e[GUIDE_LOBES], se = 0.0f;
#pragma unroll
    for (int k = 0; k < GUIDE_LOBES; k++) {
        e[k] = __expf(o[5 * k + 4] - mx);
        se += e[k];
    }
    float cum = 0.0f;
#pragma unroll
    for (int k = 0; k < GUIDE_LOBES; k++) {
        const float m0 = o[5 * k], m1 = o[5 * k + 1], m2 = o[5 * k + 2];
        const float inv = rsqrtf(m0 * m0 + m1 * m1 + m2 * m2 + 1e-12f);
        const float kap = __expf(fminf(GUIDE_LOGK_MAX, fmaxf(GUIDE_LOGK_MIN, o[5 * k + 3])));
        const float pk = e[k] / se;
        G.mk[k] = make_float4(m0 * inv, m1 * inv, m2 * inv, kap);
        G.c[k] = pk * kap / (2.0f * GUIDE_PI * -expm1f(-2.0f * kap));
        cum += pk;
        G.cdf[k] = cum;
    }
    G.cdf[GUIDE_LOBES - 1] = 1.0f;
    const float s = 1.0f / (1.0f + __expf(-o[40]));
    G.alpha = GUIDE_ALPHA_MIN + GUIDE_ALPHA_SPAN * s;
    G.pad[0] = G.pad[1] = G.pad[2] = 0.0f;
}

// Loss -w log q(wi) of one row and its gradient with respect to the 41 raw
// outputs (written to d[0..63], zeros past 40).
__device__ float loss_grad(const float *o, f3 n, f3 wi, float w, float *d) {
    float mx = -FLT_MAX;
    for (int k = 0; k < GUIDE_LOBES; k++) mx = fmaxf(mx, o[5 * k + 4]);
    float pi[GUIDE_LOBES], f[GUIDE_LOBES], mu[GUIDE_LOBES][3], len[GUIDE_LOBES], kap[GUIDE_LOBES], cw[GUIDE_LOBES];
    bool inside[GUIDE_LOBES];
    float se = 0.0f;
    for (int k = 0; k < GUIDE_LOBES; k++) {
        pi[k] = expf(o[5 * k + 4] - mx);
        se += pi[k];
    }
    float qv = 0.0f;
    for (int k = 0; k < GUIDE_LOBES; k++) {
        pi[k] /= se;
        const float m0 = o[5 * k], m1 = o[5 * k + 1], m2 = o[5 * k + 2];
        len[k] = sqrtf(m0 * m0 + m1 * m1 + m2 * m2 + 1e-12f);
        mu[k][0] = m0 / len[k];
        mu[k][1] = m1 / len[k];
        mu[k][2] = m2 / len[k];
        const float lk = o[5 * k + 3];
        inside[k] = lk > GUIDE_LOGK_MIN && lk < GUIDE_LOGK_MAX;
        kap[k] = expf(fminf(GUIDE_LOGK_MAX, fmaxf(GUIDE_LOGK_MIN, lk)));
        cw[k] = mu[k][0] * wi.x + mu[k][1] * wi.y + mu[k][2] * wi.z;
        f[k] = kap[k] / (2.0f * GUIDE_PI * -expm1f(-2.0f * kap[k])) * expf(kap[k] * (cw[k] - 1.0f));
        qv += pi[k] * f[k];
    }
    const float s = 1.0f / (1.0f + expf(-o[40]));
    const float alpha = GUIDE_ALPHA_MIN + GUIDE_ALPHA_SPAN * s;
    const float pc = fmaxf(0.0f, dot(n, wi)) / GUIDE_PI;
    const float q = fmaxf(alpha * qv + (1.0f - alpha) * pc, 1e-30f);
    const float g = -w / q;
    for (int j = 0; j < W; j++) d[j] = 0.0f;
    d[40] = g * (qv - pc) * GUIDE_ALPHA_SPAN * s * (1.0f - s);
    float dotp = 0.0f;
    float gp[GUIDE_LOBES];
    for (int k = 0; k < GUIDE_LOBES; k++) {
        gp[k] = g * alpha * f[k];
        dotp += pi[k] * gp[k];
    }
    for (int k = 0; k < GUIDE_LOBES; k++) {
        d[5 * k + 4] = pi[k] * (gp[k] - dotp);
        const float gf = g * alpha * pi[k] * f[k];   // d loss / d log f_k
        const float dlk = 1.0f / kap[k] - 2.0f / expm1f(2.0f * kap[k]) + (cw[k] - 1.0f);
        d[5 * k + 3] = inside[k] ? gf * dlk * kap[k] : 0.0f;
        const float gm0 = gf * kap[k] * wi.x, gm1 = gf * kap[k] * wi.y, gm2 = gf * kap[k] * wi.z;
        const float pr = gm0 * mu[k][0] + gm1 * mu[k][1] + gm2 * mu[k][2];
        d[5 * k + 0] = (gm0 - pr * mu[k][0]) / len[k];
        d[5 * k + 1] = (gm1 - pr * mu[k][1]) / len[k];
        d[5 * k + 2] = (gm2 - pr * mu[k][2]) / len[k];
    }
    return -w * logf(q);
}

// Column c of rows r0 and r1 of a row-major BF16 tile, packed (r0 in the low half).
__device__ __forceinline__ uint32_t pack2(const __nv_bfloat16 *X, int r0, int r1, int c) {
    const uint32_t a = *reinterpret_cast<const unsigned short *>(X + r0 * XS + c);
    const uint32_t b = *reinterpret_cast<const unsigned short *>(X + r1 * XS + c);
    return a | (b << 16);
}

__device__ __forceinline__ void load_frags(uint2 *dst, const uint2 *src) {
    for (int i = threadIdx.x; i < NFRAG; i += blockDim.x) dst[i] = src[i];
}

// ---- inference over the extension queue of one level ----
constexpr size_t kInferSmem = NFRAG * sizeof(uint2) + (size_t)kInferWarps * 16 * OS * sizeof(float) + W * sizeof(float);

__global__ void __launch_bounds__(kInferWarps * 32) k_guide_infer(DevScene S, WaveQueues Q, uint32_t level, GuideNetDev N,
                                                             GuideLobes *out) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint2 *s_wf = reinterpret_cast<uint2 *>(smem);
    float *s_outs = reinterpret_cast<float *>(s_wf + NFRAG);
    float *s_bias = s_outs + kInferWarps * 16 * OS;
    load_frags(s_wf, N.wf);
    for (int i = threadIdx.x; i < W; i += blockDim.x) s_bias[i] = N.bias[i];
    __syncthreads();
    const int buf = level & 1;
    const uint32_t n = min(Q.counts[level], Q.cap_q);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3u;
    float *out_rows = s_outs + warp * 16 * OS;
    const uint32_t tiles = (n + 15u) / 16u;
    for (uint32_t tile = blockIdx.x * kInferWarps + warp; tile < tiles; tile += gridDim.x * kInferWarps) {
        f3 p[2], nr[2], wo[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const uint32_t i = tile * 16u + g + 8u * h;
            p[h] = nr[h] = wo[h] = mk(0.0f, 0.0f, 1.0f);
            if (i < n) {
                const uint4 hh = Q.hit[i];
                const float4 o4 = Q.o[buf][i], d4 = Q.d[buf][i];
                if (hh.w != 0xFFFFFFFFu) {
                    Ray r;
                    r.o = mk(o4.x, o4.y, o4.z);
                    r.d = mk(d4.x, d4.y, d4.z);
                    r.time = o4.w;
                    Hit hit;
                    hit.t = __uint_as_float(hh.x);
                    hit.tl = __uint_as_float(hh.y);
                    hit.prim = hh.z;
                    hit.ent = hh.w;
                    guide_query(S, r, hit, p[h], nr[h]);
                    p[h] = normalise_pos(N, p[h]);
                    wo[h] = -r.d;
                }
            }
        }
        uint32_t act[16];
        encode_rows(N, p[0], nr[0], wo[0], p[1], nr[1], wo[1], t, act);
        float acc[8][4];
#pragma unroll
        for (int l = 0; l < GUIDE_LAYERS; l++) {
            layer_mma(act, s_wf + l * 4 * 8 * 32, lane, acc);
            if (l + 1 < GUIDE_LAYERS) relu_to_act(acc, act);
        }
        store_out(acc, s_bias, out_rows, g, t);
        __syncwarp();
        if (lane < 16) {
            const uint32_t i = tile * 16u + lane;
            if (i < n) {
                GuideLobes G;
                decode_lobes(out_rows + lane * OS, G);
                float4 *dst = reinterpret_cast<float4 *>(out + i);
                const float4 *src = reinterpret_cast<const float4 *>(&G);
#pragma unroll
                for (int j = 0; j < 13; j++) dst[j] = src[j];
            }
        }
        __syncwarp();
    }
}

// ---- the same inference on the 5th-generation tensor cores (tcgen05) ----
// One CTA of 256 threads takes 128 rows at a time, two threads per row (the
// row's two halves): each thread gathers eight of the row's sixteen hash-grid
// levels (the half of the row that also holds the normal, direction and
// constant writes those) straight into the shared-memory A operand; one
// elected thread issues, per layer, four tcgen05.mma (M = 128 rows, N = 64
// units, K = 16 each; BF16 operands in shared memory, FP32 accumulator in
// tensor memory) and commits them to an mbarrier; every thread then reads
// its half of its row (32 columns) back from tensor memory (warps w and
// w + 4 share lanes 32 (w % 4) ..), applies the ReLU and writes its half of
// the next layer's A operand, or, after the output layer, the first half
// decodes the proposal with outputs 32..40 from the second.  Two threads per
// row keep twice the gathers in flight per row at 64 registers a thread.
// Waits on the mbarrier are bounded: on a timeout the kernel sets *err, stops
// issuing work and frees its tensor memory.
// ROWS: caller rows (GuideRow, normalised weights ignored) to raw outputs
// (64 floats per row) instead of a level's queue entries to proposals.
constexpr uint32_t kTcRows = 128;
constexpr uint32_t kTcThreads = 256;
constexpr int kTcHi = 9;   // outputs 32..40 handed from the second half of a row to the first
constexpr size_t kTcSmem = (size_t)kTcRows * W * 2 + (size_t)NW * 2 + (size_t)kTcRows * kTcHi * sizeof(float) +
                           W * sizeof(float) + 16;
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(W >> 3) << 17) | ((kTcRows >> 4) << 24);
constexpr uint32_t kTcWaitLimit = 1u << 20;   // polls of an mbarrier (a layer completes in microseconds)

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (no swizzle, K-major, sm_100 version
// field): core matrices along K 128 bytes apart, row groups `sbo` bytes apart
// (1024 for a 64-wide K, 2048 for the 128-wide K of the transposed operands).
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t sbo = 1024u) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           ((uint64_t)1 << 46);
}

// One tcgen05.mma (M = 128, N = 64, K = 16, BF16 in, FP32 accumulator at
// tensor-memory address d): D = A B^T, plus D when `accumulate`; no output
// lane disabled.  Issued by one thread.
__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n}" ::"r"(d),
        "l"(a), "l"(b), "r"(kTcIdesc), "r"(accumulate), "r"(0u)
        : "memory");
}

// Arrives on the mbarrier once every tcgen05.mma issued so far has completed.
__device__ __forceinline__ void tc_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity) {
    for (uint32_t it = 0; it < kTcWaitLimit; it++) {
        uint32_t done;
        asm volatile("{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.b32 %0, 1, 0, p;\n}"
                     : "=r"(done)
                     : "r"(mbar), "r"(parity)
                     : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 consecutive accumulator columns of this thread's lane.
__device__ __forceinline__ void tc_load16(uint32_t taddr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}

// Row `r` of the A operand from 64 floats (BF16, 8 chunks of 16 bytes).
__device__ __forceinline__ void tc_store_row(unsigned char *A, uint32_t r, const float *x, bool relu) {
#pragma unroll
    for (int kc = 0; kc < 8; kc++) {
        uint4 q;
        uint32_t *u = reinterpret_cast<uint32_t *>(&q);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float a = x[8 * kc + 2 * j], b = x[8 * kc + 2 * j + 1];
            if (relu) {
                a = fmaxf(a, 0.0f);
                b = fmaxf(b, 0.0f);
            }
            u[j] = pack_bf16(a, b);
        }
        *reinterpret_cast<uint4 *>(A + tc_offset(r, 8u * kc)) = q;
    }
}

// Chunks KC0 .. KC0 + NKC - 1 (8 columns each) of row r of the A operand from
// x[0 .. 8 NKC), as BF16.
template <int KC0, int NKC>
__device__ __forceinline__ void tc_store_chunks(unsigned char *A, uint32_t r, const float *x, bool relu) {
#pragma unroll
    for (int c = 0; c < NKC; c++) {
        uint4 q;
        uint32_t *u = reinterpret_cast<uint32_t *>(&q);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float a = x[8 * c + 2 * j], b = x[8 * c + 2 * j + 1];
            if (relu) {
                a = fmaxf(a, 0.0f);
                b = fmaxf(b, 0.0f);
            }
            u[j] = pack_bf16(a, b);
        }
        *reinterpret_cast<uint4 *>(A + tc_offset(r, 8u * (KC0 + c))) = q;
    }
}

template <bool ROWS>
__global__ void __launch_bounds__(kTcThreads, 4) k_guide_mlp_tc(DevScene S, WaveQueues Q, uint32_t level,
                                                                GuideNetDev N, GuideLobes *out, const GuideRow *rows,
                                                                uint32_t nrows, float *raw, uint32_t *err,
                                                                const uint32_t *order = nullptr) {
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char *A = smem;                                   // 128 x 64 BF16
    unsigned char *B = A + kTcRows * W * 2;                    // 4 layers x 64 x 64 BF16
    float *s_hi = reinterpret_cast<float *>(B + NW * 2);       // [128][kTcHi] outputs 32..40 for the decode
    float *s_bias = s_hi + kTcRows * kTcHi;
    uint64_t *s_mbar = reinterpret_cast<uint64_t *>(s_bias + W);
    uint32_t *s_tmem = reinterpret_cast<uint32_t *>(s_mbar + 1);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t r = tid & (kTcRows - 1u), half = tid / kTcRows;   // row of the tile, which half of it
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(N.wtc);
        uint4 *dst = reinterpret_cast<uint4 *>(B);
        for (uint32_t i = tid; i < (uint32_t)NW * 2 / 16; i += blockDim.x) dst[i] = src[i];
    }
    for (uint32_t i = tid; i < (uint32_t)W; i += blockDim.x) s_bias[i] = N.bias[i];
    const uint32_t mbar = smem_u32(s_mbar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(s_tmem)),
                     "r"((uint32_t)W)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // the B operands, for the tensor cores
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *s_tmem;
    // this warp's 32 lanes (warps w and w + 4 share lanes 32 (w % 4) ..), this half's 32 columns
    const uint32_t lane_addr = tmem + ((32u * (warp & 3u)) << 16) + 32u * half;
    const int buf = level & 1;
    const uint32_t n = ROWS ? nrows : min(Q.counts[level], Q.cap_q);
    const uint32_t tiles = (n + kTcRows - 1) / kTcRows;
    const uint32_t adesc0 = smem_u32(A), bdesc0 = smem_u32(B);
    uint32_t phase = 0;
    bool ok = true;
    for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        // the tile's rows: queue entries in order, or in the spatial order of `order`
        const uint32_t k = tile * kTcRows + r;
        const uint32_t i = order && k < n ? order[k] : k;
        // ---- this row's network inputs: half 0 gathers grid levels 0..7,
        // half 1 levels 8..15 and writes the normal, direction and constant ----
        f3 p = mk(0.0f, 0.0f, 1.0f), nr = p, wo = p;
        if (i < n) {
            if (ROWS) {
                const GuideRow row = rows[i];
                p = normalise_pos(N, mk(row.pos_w.x, row.pos_w.y, row.pos_w.z));
                nr = mk(row.n.x, row.n.y, row.n.z);
                wo = mk(row.wo.x, row.wo.y, row.wo.z);
            } else {
                const uint4 hh = Q.hit[i];
                if (hh.w != 0xFFFFFFFFu) {
                    const float4 o4 = Q.o[buf][i], d4 = Q.d[buf][i];
                    Ray ray;
                    ray.o = mk(o4.x, o4.y, o4.z);
                    ray.d = mk(d4.x, d4.y, d4.z);
                    ray.time = o4.w;
                    Hit hit;
                    hit.t = __uint_as_float(hh.x);
                    hit.tl = __uint_as_float(hh.y);
                    hit.prim = hh.z;
                    hit.ent = hh.w;
                    guide_query(S, ray, hit, p, nr);
                    p = normalise_pos(N, p);
                    wo = -ray.d;
                }
            }
        }
        float x[32];
#pragma unroll
        for (int l = 0; l < GUIDE_LEVELS / 2; l++) {
            const float2 f = grid_feature(N, l + (int)half * (GUIDE_LEVELS / 2), p);
            x[2 * l] = f.x;
            x[2 * l + 1] = f.y;
        }
        if (half == 0) {
            tc_store_chunks<0, 2>(A, r, x, false);
        } else {
            tc_store_chunks<2, 2>(A, r, x, false);
            x[0] = nr.x; x[1] = nr.y; x[2] = nr.z;
            x[3] = wo.x; x[4] = wo.y; x[5] = wo.z;
            x[6] = 1.0f;
#pragma unroll
            for (int j = 7; j < 32; j++) x[j] = 0.0f;
            tc_store_chunks<4, 4>(A, r, x, false);
        }
        for (int l = 0; l < GUIDE_LAYERS; l++) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // A written by this thread
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
            if (tid == 0) {
                const uint32_t bl = bdesc0 + (uint32_t)l * W * W * 2;
#pragma unroll
                for (uint32_t ks = 0; ks < (uint32_t)W / 16; ks++)   // accumulate after the first K step
                    tc_mma(tmem, tc_desc(adesc0 + ks * 256u), tc_desc(bl + ks * 256u), ks);
                tc_commit(mbar);
            }
            // every thread decides alike whether the layer arrived
            const bool got = tc_wait(mbar, phase);
            if (__syncthreads_or(!got)) {
                ok = false;
                if (tid == 0 && err) atomicOr(err, 1u);
                break;
            }
            phase ^= 1u;
            tc_fence_after();
            tc_load16(lane_addr, x);
            tc_load16(lane_addr + 16u, x + 16);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (l + 1 < GUIDE_LAYERS) {
                if (half == 0) tc_store_chunks<0, 4>(A, r, x, true);
                else tc_store_chunks<4, 4>(A, r, x, true);
            } else {
#pragma unroll
                for (int j = 0; j < 32; j++) x[j] += s_bias[32 * half + j];
                if (ROWS) {
                    if (i < n)
                        for (int j = 0; j < 32; j++) raw[(size_t)i * W + 32 * half + j] = x[j];
                } else {
                    // the decode reads outputs 0..40: half 1 hands 32..40 to half 0
                    if (half == 1) {
#pragma unroll
                        for (int j = 0; j < kTcHi; j++) s_hi[r * kTcHi + j] = x[j];
                    }
                    __syncthreads();
                    if (half == 0 && i < n) {
                        float o[41];
#pragma unroll
                        for (int j = 0; j < 32; j++) o[j] = x[j];
#pragma unroll
                        for (int j = 0; j < 41 - 32; j++) o[32 + j] = s_hi[r * kTcHi + j];
                        GuideLobes G;
                        decode_lobes(o, G);
                        float4 *dst = reinterpret_cast<float4 *>(out + i);
                        const float4 *src = reinterpret_cast<const float4 *>(&G);
#pragma unroll
                        for (int j = 0; j < 13; j++) dst[j] = src[j];
                    }
                }
            }
        }
    }
    // every thread is past its last tensor-memory read (or the failed wait)
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (!ok && tid == 0) tc_wait(mbar, phase);   // let a commit still in flight land before freeing
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)W) : "memory");
}

// ---- training targets from the recorded vertices of a finished wave ----
// Deterministic: every record gets its weight (0: unusable) and flag, an
// exclusive scan of the flags gives each usable record its row, so rows keep
// the records' order whatever order the threads run in.
__global__ void k_guide_weights(const GuideRecord *rec, uint32_t total, uint32_t n_rec, const float4 *accum,
                                float *weight, uint32_t *flag) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        const GuideRecord R = rec[k];
        float w = 0.0f;
        if (R.tpc.w == 1.0f && R.snap.w == 1.0f && R.pos_q.w > 0.0f) {
            const float4 a = accum[k % n_rec];
            // radiance along wi: what the child's subtree added, divided by its throughput
            const float lx = R.tpc.x > 1e-20f ? (a.x - R.snap.x) / R.tpc.x : 0.0f;
            const float ly = R.tpc.y > 1e-20f ? (a.y - R.snap.y) / R.tpc.y : 0.0f;
            const float lz = R.tpc.z > 1e-20f ? (a.z - R.snap.z) / R.tpc.z : 0.0f;
            const float lum = fmaxf(0.0f, 0.2126f * lx + 0.7152f * ly + 0.0722f * lz);
            const float cs = fmaxf(0.0f, R.n.x * R.wi.x + R.n.y * R.wi.y + R.n.z * R.wi.z);
            // KL objective toward the density proportional to L(wi) cos: weight F / q
            w = lum * cs / R.pos_q.w;
            if (!(w > 0.0f) || !isfinite(w)) w = 0.0f;
        }
        weight[k] = w;
        flag[k] = w > 0.0f ? 1u : 0u;
    }
}

// Usable record k to row pos[k] (the first `cap` only); the kept weights also
// go to wk[pos] (zero elsewhere) for the weight sum; count = kept rows.
__global__ void k_guide_compact(const GuideRecord *rec, uint32_t total, const float *weight, const uint32_t *flag,
                                const uint32_t *pos, GuideRow *rows, float *wk, uint32_t cap, uint32_t *count) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        if (k == total - 1) *count = min(pos[k] + flag[k], cap);
        if (!flag[k] || pos[k] >= cap) continue;
        const GuideRecord R = rec[k];
        GuideRow r;
        r.pos_w = make_float4(R.pos_q.x, R.pos_q.y, R.pos_q.z, weight[k]);
        r.n = R.n;
        r.wo = R.wo;
        r.wi = R.wi;
        rows[pos[k]] = r;
        wk[pos[k]] = weight[k];
    }
}

// ---- forward, loss and backward over training rows ----
// Deterministic gradients: within a block the MLP weight and output-bias
// gradients are summed by the warp that owns them (dW rows 16w..16w+15 and
// bias columns 16w..16w+15 belong to warp w), over the block's four tiles in
// a fixed order; every block writes its sums, its loss and nothing else to
// its own slot of `part`, which k_guide_reduce adds up block by block.  The
// hash-grid gradient is scattered as 64-bit fixed point (2^-32 units), whose
// integer additions give the same sum in any order.  Row weights are scaled
// by count / wsum (mean weight 1) and then capped at `wcap`, so that a rare
// path with a huge radiance estimate cannot pull the proposal onto itself
// (any proposal leaves the estimator unbiased).  Optional outputs for tests:
// raw outputs (n x 64) and encoding gradients (n x 32).
constexpr int kPart = NW + W + 4;            // floats per block slot: dW, db, loss (padded)
constexpr float kGridFix = 4294967296.0f;    // fixed-point scale of the grid gradient

struct TrainArgs {
    const GuideRow *rows;
    const uint32_t *count;    // rows used: min(*count, cap)
    uint32_t cap;
    const float *wsum;        // null: weights used as given
    float wcap;               // cap on a normalised row weight (with wsum)
    float *part;              // [gridDim.x][kPart]
    unsigned long long *grid_grad;   // [entry][2] fixed point, or null
    float *dbg_out, *dbg_enc;
};

constexpr size_t kTrainSmem = 2 * NFRAG * sizeof(uint2) + (size_t)GUIDE_LAYERS * W * W * sizeof(float) +
                              W * sizeof(float) * 2 + kWarps * sizeof(float) +
                              (size_t)kWarps * ((GUIDE_LAYERS + 1) * 16 * XS * sizeof(__nv_bfloat16) +
                                                16 * OS * sizeof(float));

__device__ __forceinline__ unsigned long long to_fixed(float v) {
    v = fminf(fmaxf(v, -1e8f), 1e8f);
    return (unsigned long long)__float2ll_rn(v * kGridFix);
}

__global__ void __launch_bounds__(kWarps * 32) k_guide_train(GuideNetDev N, TrainArgs A) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint2 *s_wf = reinterpret_cast<uint2 *>(smem);
    uint2 *s_wt = s_wf + NFRAG;
    float *s_dw = reinterpret_cast<float *>(s_wt + NFRAG);
    float *s_bias = s_dw + GUIDE_LAYERS * W * W;
    float *s_db = s_bias + W;
    float *s_loss = s_db + W;
    unsigned char *per_warp = reinterpret_cast<unsigned char *>(s_loss + kWarps);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3u;
    const size_t warp_bytes = (GUIDE_LAYERS + 1) * 16 * XS * sizeof(__nv_bfloat16) + 16 * OS * sizeof(float);
    auto warp_x = [&](uint32_t w) {   // [layer][16][XS] inputs of warp w's tile
        return reinterpret_cast<__nv_bfloat16 *>(per_warp + w * warp_bytes);
    };
    __nv_bfloat16 *s_x = warp_x(warp);
    __nv_bfloat16 *s_dy = s_x + GUIDE_LAYERS * 16 * XS;                                    // [16][XS]
    float *s_o = reinterpret_cast<float *>(s_dy + 16 * XS);                                 // [16][OS]
    load_frags(s_wf, N.wf);
    load_frags(s_wt, N.wt);
    for (int i = threadIdx.x; i < GUIDE_LAYERS * W * W; i += blockDim.x) s_dw[i] = 0.0f;
    for (int i = threadIdx.x; i < W; i += blockDim.x) {
        s_bias[i] = N.bias[i];
        s_db[i] = 0.0f;
    }
    __syncthreads();
    const uint32_t n = min(*A.count, A.cap);
    const float wscale = A.wsum ? (float)n / fmaxf(*A.wsum, 1e-30f) : 1.0f;
    const float wcap = A.wsum && A.wcap > 0.0f ? A.wcap : FLT_MAX;
    float loss_acc = 0.0f;
    const uint32_t tiles = (n + 15u) / 16u;
    const uint32_t groups = (tiles + kWarps - 1u) / kWarps;
    // every warp of the block runs the same iterations (a warp past the last
    // tile works on rows past n, which contribute nothing)
    for (uint32_t grp = blockIdx.x; grp < groups; grp += gridDim.x) {
        const uint32_t tile = grp * kWarps + warp;
        // ---- forward, keeping each layer's input ----
        f3 p[2], nr[2], wo[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const uint32_t i = tile * 16u + g + 8u * h;
            p[h] = nr[h] = wo[h] = mk(0.0f, 0.0f, 1.0f);
            if (i < n) {
                const GuideRow r = A.rows[i];
                p[h] = normalise_pos(N, mk(r.pos_w.x, r.pos_w.y, r.pos_w.z));
                nr[h] = mk(r.n.x, r.n.y, r.n.z);
                wo[h] = mk(r.wo.x, r.wo.y, r.wo.z);
            }
        }
        uint32_t act[16];
        encode_rows(N, p[0], nr[0], wo[0], p[1], nr[1], wo[1], t, act);
        float acc[8][4];
#pragma unroll
        for (int l = 0; l < GUIDE_LAYERS; l++) {
            store_act(act, s_x + l * 16 * XS, g, t);
            layer_mma(act, s_wf + l * 4 * 8 * 32, lane, acc);
            if (l + 1 < GUIDE_LAYERS) relu_to_act(acc, act);
        }
        store_out(acc, s_bias, s_o, g, t);
        __syncwarp();
        // ---- loss and output gradient, one row per lane ----
        if (lane < 16) {
            const uint32_t i = tile * 16u + lane;
            float *o = s_o + lane * OS;
            if (A.dbg_out && i < n)
                for (int j = 0; j < W; j++) A.dbg_out[(size_t)i * W + j] = o[j];
            float d[W];
            if (i < n) {
                const GuideRow r = A.rows[i];
                loss_acc += loss_grad(o, mk(r.n.x, r.n.y, r.n.z), mk(r.wi.x, r.wi.y, r.wi.z),
                                      fminf(r.pos_w.w * wscale, wcap), d);
            } else {
                for (int j = 0; j < W; j++) d[j] = 0.0f;
            }
            for (int j = 0; j < W; j++) o[j] = d[j];
        }
        __syncwarp();
        // BF16 row-major copy of dY of the output layer
        for (int e = lane; e < 16 * W; e += 32) {
            const int r = e / W, c = e % W;
            s_dy[r * XS + c] = __float2bfloat16_rn(s_o[r * OS + c]);
        }
        __syncwarp();
        // dY of the output layer as A fragments
        uint32_t dya[16];
#pragma unroll
        for (int kk = 0; kk < 4; kk++) {
            dya[kk * 4 + 0] = *reinterpret_cast<const uint32_t *>(s_dy + g * XS + 16 * kk + 2 * t);
            dya[kk * 4 + 1] = *reinterpret_cast<const uint32_t *>(s_dy + (g + 8) * XS + 16 * kk + 2 * t);
            dya[kk * 4 + 2] = *reinterpret_cast<const uint32_t *>(s_dy + g * XS + 16 * kk + 2 * t + 8);
            dya[kk * 4 + 3] = *reinterpret_cast<const uint32_t *>(s_dy + (g + 8) * XS + 16 * kk + 2 * t + 8);
        }
        // ---- backward through the layers ----
        for (int l = GUIDE_LAYERS - 1; l >= 0; l--) {
            __syncthreads();   // every warp's X_l and dY_l are in shared memory
            // dW_l += X_l^T dY_l over the block's four tiles in order: warp w
            // owns the input units 16w..16w+15 (M), all 64 output units (N)
            {
                const int c0 = 16 * (int)warp + (int)g;
                float c[8][4];
#pragma unroll
                for (int nn = 0; nn < 8; nn++) c[nn][0] = c[nn][1] = c[nn][2] = c[nn][3] = 0.0f;
                for (uint32_t src = 0; src < (uint32_t)kWarps; src++) {
                    const __nv_bfloat16 *X = warp_x(src) + l * 16 * XS;
                    const __nv_bfloat16 *DY = warp_x(src) + GUIDE_LAYERS * 16 * XS;
                    uint32_t a[4];
                    a[0] = pack2(X, 2 * t, 2 * t + 1, c0);
                    a[1] = pack2(X, 2 * t, 2 * t + 1, c0 + 8);
                    a[2] = pack2(X, 2 * t + 8, 2 * t + 9, c0);
                    a[3] = pack2(X, 2 * t + 8, 2 * t + 9, c0 + 8);
#pragma unroll
                    for (int nn = 0; nn < 8; nn++) {
                        const int oc = 8 * nn + (int)g;
                        uint2 b;
                        b.x = pack2(DY, 2 * t, 2 * t + 1, oc);
                        b.y = pack2(DY, 2 * t + 8, 2 * t + 9, oc);
                        mma16816(c[nn], a, b);
                    }
                }
                float *dw = s_dw + l * W * W;
#pragma unroll
                for (int nn = 0; nn < 8; nn++) {
                    const int col = 8 * nn + 2 * (int)t;
                    dw[c0 * W + col] += c[nn][0];
                    dw[c0 * W + col + 1] += c[nn][1];
                    dw[(c0 + 8) * W + col] += c[nn][2];
                    dw[(c0 + 8) * W + col + 1] += c[nn][3];
                }
                if (l == GUIDE_LAYERS - 1 && lane < 16) {
                    // output-bias gradient: warp w owns columns 16w..16w+15
                    const int j = 16 * (int)warp + (int)lane;
                    float sacc = 0.0f;
                    for (uint32_t src = 0; src < (uint32_t)kWarps; src++) {
                        const float *o = reinterpret_cast<const float *>(warp_x(src) + (GUIDE_LAYERS + 1) * 16 * XS);
                        for (int r = 0; r < 16; r++) sacc += o[r * OS + j];
                    }
                    s_db[j] += sacc;
                }
            }
            __syncthreads();   // the dW reads are done before dY_{l-1} replaces dY_l
            // dX_l = dY_l W_l^T
            float dx[8][4];
            layer_mma(dya, s_wt + l * 4 * 8 * 32, lane, dx);
            __syncwarp();
            const __nv_bfloat16 *X = s_x + l * 16 * XS;
            if (l > 0) {
                // through the ReLU that produced X_l: dY_{l-1} = dX_l where X_l > 0
#pragma unroll
                for (int kk = 0; kk < 4; kk++) {
                    const float2 x00 = unpack_bf16(*reinterpret_cast<const uint32_t *>(X + g * XS + 16 * kk + 2 * t));
                    const float2 x01 = unpack_bf16(*reinterpret_cast<const uint32_t *>(X + (g + 8) * XS + 16 * kk + 2 * t));
                    const float2 x10 = unpack_bf16(*reinterpret_cast<const uint32_t *>(X + g * XS + 16 * kk + 2 * t + 8));
                    const float2 x11 = unpack_bf16(*reinterpret_cast<const uint32_t *>(X + (g + 8) * XS + 16 * kk + 2 * t + 8));
                    dya[kk * 4 + 0] = pack_bf16(x00.x > 0.0f ? dx[2 * kk][0] : 0.0f, x00.y > 0.0f ? dx[2 * kk][1] : 0.0f);
                    dya[kk * 4 + 1] = pack_bf16(x01.x > 0.0f ? dx[2 * kk][2] : 0.0f, x01.y > 0.0f ? dx[2 * kk][3] : 0.0f);
                    dya[kk * 4 + 2] = pack_bf16(x10.x > 0.0f ? dx[2 * kk + 1][0] : 0.0f, x10.y > 0.0f ? dx[2 * kk + 1][1] : 0.0f);
                    dya[kk * 4 + 3] = pack_bf16(x11.x > 0.0f ? dx[2 * kk + 1][2] : 0.0f, x11.y > 0.0f ? dx[2 * kk + 1][3] : 0.0f);
                }
                store_act(dya, s_dy, g, t);
                __syncwarp();
            } else {
                // encoding gradient: columns 0..31, level 4 nn + t at 8 nn + 2t
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const uint32_t i = tile * 16u + g + 8u * h;
                    if (i >= n) continue;
#pragma unroll
                    for (int nn = 0; nn < 4; nn++) {
                        const int lv = 4 * nn + (int)t;
                        const float gx = dx[nn][2 * h], gy = dx[nn][2 * h + 1];
                        if (A.dbg_enc) {
                            A.dbg_enc[(size_t)i * 32 + 2 * lv] = gx;
                            A.dbg_enc[(size_t)i * 32 + 2 * lv + 1] = gy;
                        }
                        if (A.grid_grad) {
                            Corners c;
                            grid_corners(N, lv, p[h], c);
#pragma unroll
                            for (int k = 0; k < 8; k++) {
                                atomicAdd(&A.grid_grad[2 * (size_t)c.idx[k]], to_fixed(c.w[k] * gx));
                                atomicAdd(&A.grid_grad[2 * (size_t)c.idx[k] + 1], to_fixed(c.w[k] * gy));
                            }
                        }
                    }
                }
            }
        }
        __syncwarp();
    }
    // the block's loss: lanes, then warps, in a fixed order
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) loss_acc += __shfl_down_sync(0xFFFFFFFFu, loss_acc, off);
    if (lane == 0) s_loss[warp] = loss_acc;
    __syncthreads();
    float *part = A.part + (size_t)blockIdx.x * kPart;
    for (int i = threadIdx.x; i < GUIDE_LAYERS * W * W; i += blockDim.x) part[i] = s_dw[i];
    for (int i = threadIdx.x; i < W; i += blockDim.x) part[NW + i] = s_db[i];
    if (threadIdx.x == 0) {
        float l = 0.0f;
        for (int w = 0; w < kWarps; w++) l += s_loss[w];
        part[NW + W] = l;
    }
}

// ---- the same training step on the 5th-generation tensor cores (tcgen05) ----
// One CTA of 128 threads per SM takes 128 rows at a time, one row per thread,
// and keeps the whole step's tensor work on tcgen05.mma (M = 128, N = 64,
// K = 16 per instruction, BF16 operands in shared memory, FP32 accumulators in
// tensor memory):
//   forward   X_{l+1} = ReLU(X_l W_l), Y = X_3 W_3 + b  (A = X_l, 64-wide K)
//   backward  dX_l = dY_l W_l^T                          (A = dY_l, 64-wide K)
//             dW_l += X_l^T dY_l                         (K = the tile's 128 rows)
// The dW products need the rows as K: every thread also writes its row of X_l
// and dY_l into transposed operands (element (unit u, row r) at
// tc_offset_t(u, r)).  Their M is the 64 input units; the instruction's other
// 64 rows read the next 16 KB of shared memory and land in tensor-memory
// lanes 64..127, which are never read.  dW_l accumulates in its own 64
// tensor-memory columns over all the CTA's tiles in tile order, so the sums
// do not depend on timing; after the last tile warps 0 and 1 (lanes 0..63)
// write them to the CTA's slot of `part`, which k_guide_reduce adds up in
// block order like the mma.sync kernel's.  Output-bias gradients and the loss
// are summed in fixed order through shared memory; the hash-grid gradient is
// scattered in fixed point as in k_guide_train.  Waits on the mbarrier are
// bounded: on a timeout *err is set and the CTA stops (its slot then holds
// what it had).
__host__ __device__ __forceinline__ uint32_t tc_offset_t(uint32_t u, uint32_t r) {
    return ((u >> 3) * 16u + (r >> 3)) * 128u + (u & 7u) * 16u + (r & 7u) * 2u;
}

constexpr uint32_t kTcOp = kTcRows * W * 2;             // bytes of one 128 x 64 BF16 operand
constexpr uint32_t kTcTrainCols = 512;                  // tensor memory: scratch + 4 dW accumulators (320 used)
// shared memory: X (A layout), X_l^T for l = 0..3, dY (A layout), dY^T, W^T
// and W per layer (B operands of the forward and of dX), dY in FP32 for the
// bias gradient, bias, bias gradient, loss, mbarrier, tensor-memory address
constexpr size_t kTcTrainSmem = (size_t)kTcOp * 7 + (size_t)NW * 2 * 2 + (size_t)kTcRows * W * sizeof(float) +
                                2 * W * sizeof(float) + kTcRows / 32 * sizeof(float) + 16;

// this thread's row of a transposed operand (u = 0..63 at row r), as BF16
__device__ __forceinline__ void tc_store_col(unsigned char *T, uint32_t r, const float *x) {
#pragma unroll
    for (int u = 0; u < W; u++)
        *reinterpret_cast<__nv_bfloat16 *>(T + tc_offset_t((uint32_t)u, r)) = __float2bfloat16_rn(x[u]);
}

__global__ void __launch_bounds__(kTcRows, 1) k_guide_train_tc(GuideNetDev N, TrainArgs A, uint32_t *err) {
    extern __shared__ __align__(16) unsigned char smem[];
    unsigned char *XA = smem;                      // X_l, rows (A operand of the forward)
    unsigned char *XT = XA + kTcOp;                // X_l^T, l = 0..3
    unsigned char *DYA = XT + 4 * kTcOp;           // dY_l, rows (A operand of dX)
    unsigned char *DYT = DYA + kTcOp;              // dY_l^T (B operand of dW)
    unsigned char *WF = DYT + kTcOp;               // per layer W^T: row = output unit (forward)
    unsigned char *WB = WF + NW * 2;               // per layer W: row = input unit (dX)
    float *s_o = reinterpret_cast<float *>(WB + NW * 2);   // [128][64] dY in FP32
    float *s_bias = s_o + kTcRows * W;
    float *s_db = s_bias + W;
    float *s_loss = s_db + W;
    uint64_t *s_mbar = reinterpret_cast<uint64_t *>(s_loss + kTcRows / 32);
    uint32_t *s_tmem = reinterpret_cast<uint32_t *>(s_mbar + 1);
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(N.wtc);
        uint4 *dst = reinterpret_cast<uint4 *>(WF);
        for (uint32_t i = tid; i < (uint32_t)NW * 2 * 2 / 16; i += blockDim.x) dst[i] = src[i];
    }
    for (uint32_t i = tid; i < (uint32_t)W; i += blockDim.x) {
        s_bias[i] = N.bias[i];
        s_db[i] = 0.0f;
    }
    const uint32_t mbar = smem_u32(s_mbar);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(s_tmem)),
                     "r"(kTcTrainCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *s_tmem;
    const uint32_t lane_addr = (32u * warp) << 16;
    const uint32_t sXA = smem_u32(XA), sXT = smem_u32(XT), sDYA = smem_u32(DYA), sDYT = smem_u32(DYT),
                   sWF = smem_u32(WF), sWB = smem_u32(WB);
    const uint32_t n = min(*A.count, A.cap);
    const float wscale = A.wsum ? (float)n / fmaxf(*A.wsum, 1e-30f) : 1.0f;
    const float wcap = A.wsum && A.wcap > 0.0f ? A.wcap : FLT_MAX;
    const uint32_t tiles = (n + kTcRows - 1) / kTcRows;
    float loss_acc = 0.0f;
    uint32_t phase = 0;
    bool ok = true, has_acc = false;
    // every thread: make the operands written so far visible to the tensor
    // cores, then one thread issues; false when the wait gave up
    auto sync_issue_wait = [&](auto issue) -> bool {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
            issue();
            tc_commit(mbar);
        }
        const bool got = tc_wait(mbar, phase);
        if (__syncthreads_or(!got)) {
            if (tid == 0 && err) atomicOr(err, 1u);
            return false;
        }
        phase ^= 1u;
        tc_fence_after();
        return true;
    };
    for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const uint32_t i = tile * kTcRows + tid;
        f3 p = mk(0.0f, 0.0f, 1.0f), nr = p, wo = p;
        GuideRow row;
        if (i < n) {
            row = A.rows[i];
            p = normalise_pos(N, mk(row.pos_w.x, row.pos_w.y, row.pos_w.z));
            nr = mk(row.n.x, row.n.y, row.n.z);
            wo = mk(row.wo.x, row.wo.y, row.wo.z);
        }
        float x[W];
#pragma unroll
        for (int l = 0; l < GUIDE_LEVELS; l++) {
            const float2 f = grid_feature(N, l, p);
            x[2 * l] = f.x;
            x[2 * l + 1] = f.y;
        }
        x[32] = nr.x; x[33] = nr.y; x[34] = nr.z;
        x[35] = wo.x; x[36] = wo.y; x[37] = wo.z;
        x[38] = 1.0f;
#pragma unroll
        for (int j = 39; j < W; j++) x[j] = 0.0f;
        tc_store_row(XA, tid, x, false);
        tc_store_col(XT, tid, x);
        // ---- forward ----
        for (int l = 0; l < GUIDE_LAYERS && ok; l++) {
            ok = sync_issue_wait([&] {
#pragma unroll
                for (uint32_t ks = 0; ks < (uint32_t)W / 16; ks++)
                    tc_mma(tmem, tc_desc(sXA + ks * 256u), tc_desc(sWF + (uint32_t)l * W * W * 2 + ks * 256u), ks);
            });
            if (!ok) break;
#pragma unroll
            for (int c = 0; c < 4; c++) tc_load16(tmem + lane_addr + 16u * c, x + 16 * c);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (l + 1 < GUIDE_LAYERS) {
#pragma unroll
                for (int j = 0; j < W; j++) x[j] = fmaxf(x[j], 0.0f);
                tc_store_row(XA, tid, x, false);
                tc_store_col(XT + (l + 1) * kTcOp, tid, x);
            }
        }
        if (!ok) break;
        // ---- loss and output gradient of this thread's row ----
#pragma unroll
        for (int j = 0; j < W; j++) x[j] += s_bias[j];
        if (A.dbg_out && i < n)
            for (int j = 0; j < W; j++) A.dbg_out[(size_t)i * W + j] = x[j];
        float d[W];
        if (i < n) {
            loss_acc += loss_grad(x, mk(row.n.x, row.n.y, row.n.z), mk(row.wi.x, row.wi.y, row.wi.z),
                                  fminf(row.pos_w.w * wscale, wcap), d);
        } else {
#pragma unroll
            for (int j = 0; j < W; j++) d[j] = 0.0f;
        }
#pragma unroll
        for (int j = 0; j < W; j++) s_o[tid * W + j] = d[j];
        tc_store_row(DYA, tid, d, false);
        tc_store_col(DYT, tid, d);
        // ---- backward ----
        for (int l = GUIDE_LAYERS - 1; l >= 0 && ok; l--) {
            const bool acc = has_acc;
            ok = sync_issue_wait([&] {
                // dW_l (+)= X_l^T dY_l over this tile's rows
#pragma unroll
                for (uint32_t ks = 0; ks < kTcRows / 16; ks++)
                    tc_mma(tmem + 64u * (uint32_t)(l + 1), tc_desc(sXT + (uint32_t)l * kTcOp + ks * 256u, 2048u),
                           tc_desc(sDYT + ks * 256u, 2048u), (acc || ks) ? 1u : 0u);
                // dX_l = dY_l W_l^T
#pragma unroll
                for (uint32_t ks = 0; ks < (uint32_t)W / 16; ks++)
                    tc_mma(tmem, tc_desc(sDYA + ks * 256u), tc_desc(sWB + (uint32_t)l * W * W * 2 + ks * 256u), ks);
            });
            if (!ok) break;
            if (l == GUIDE_LAYERS - 1 && tid < (uint32_t)W) {
                // output-bias gradient: thread j sums column j over the rows in order
                float s = 0.0f;
                for (uint32_t r = 0; r < kTcRows; r++) s += s_o[r * W + tid];
                s_db[tid] += s;
            }
#pragma unroll
            for (int c = 0; c < 4; c++) tc_load16(tmem + lane_addr + 16u * c, x + 16 * c);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (l > 0) {
                // through the ReLU that produced X_l: dY_{l-1} = dX_l where X_l > 0
                const unsigned char *T = XT + l * kTcOp;
#pragma unroll
                for (int u = 0; u < W; u++) {
                    const float xv = __bfloat162float(
                        *reinterpret_cast<const __nv_bfloat16 *>(T + tc_offset_t((uint32_t)u, tid)));
                    d[u] = xv > 0.0f ? x[u] : 0.0f;
                }
                tc_store_row(DYA, tid, d, false);
                tc_store_col(DYT, tid, d);
            } else if (i < n) {
                // encoding gradient: columns 2 lv, 2 lv + 1 of dX_0
                for (int lv = 0; lv < GUIDE_LEVELS; lv++) {
                    const float gx = x[2 * lv], gy = x[2 * lv + 1];
                    if (A.dbg_enc) {
                        A.dbg_enc[(size_t)i * 32 + 2 * lv] = gx;
                        A.dbg_enc[(size_t)i * 32 + 2 * lv + 1] = gy;
                    }
                    if (A.grid_grad) {
                        Corners c;
                        grid_corners(N, lv, p, c);
#pragma unroll
                        for (int k = 0; k < 8; k++) {
                            atomicAdd(&A.grid_grad[2 * (size_t)c.idx[k]], to_fixed(c.w[k] * gx));
                            atomicAdd(&A.grid_grad[2 * (size_t)c.idx[k] + 1], to_fixed(c.w[k] * gy));
                        }
                    }
                }
            }
        }
        has_acc = true;
    }
    // every thread is past its last tensor-memory read (or the failed wait)
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (!ok && tid == 0) tc_wait(mbar, phase);   // let a commit still in flight land
    __syncthreads();
    float *part = A.part + (size_t)blockIdx.x * kPart;
    if (warp < 2) {
        // dW_l[u][o] at tensor-memory lane u (0..63), column 64 (l + 1) + o
        const uint32_t u = 32u * warp + lane;
        for (int l = 0; l < GUIDE_LAYERS; l++) {
            float v[W];
#pragma unroll
            for (int c = 0; c < 4; c++) tc_load16(tmem + lane_addr + 64u * (uint32_t)(l + 1) + 16u * c, v + 16 * c);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            for (int o = 0; o < W; o++) part[(size_t)l * W * W + u * W + o] = has_acc && ok ? v[o] : 0.0f;
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) loss_acc += __shfl_down_sync(0xFFFFFFFFu, loss_acc, off);
    if (lane == 0) s_loss[warp] = loss_acc;
    __syncthreads();
    for (uint32_t j = tid; j < (uint32_t)W; j += blockDim.x) part[NW + j] = s_db[j];
    if (tid == 0) {
        float l = 0.0f;
        for (uint32_t w = 0; w < kTcRows / 32; w++) l += s_loss[w];
        part[NW + W] = l;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcTrainCols) : "memory");
}

// Block slots of k_guide_train added up in block order: w_grad, b_grad, loss.
__global__ void k_guide_reduce(const float *part, uint32_t blocks, float *w_grad, float *b_grad, float *loss) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < (uint32_t)(NW + W + 1); i += gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (uint32_t b = 0; b < blocks; b++) s += part[(size_t)b * kPart + i];
        if (i < (uint32_t)NW) w_grad[i] = s;
        else if (i < (uint32_t)(NW + W)) b_grad[i - NW] = s;
        else *loss = s;
    }
}

// ---- Adam (Kingma, Ba 2015) with FP32 master weights; gradients are cleared ----
struct AdamStep {
    float lr, b1, b2, eps, c1, c2;   // c1, c2: bias corrections 1 / (1 - b^t)
};

__global__ void k_adam(float *w, float *g, float *m, float *v, uint32_t n, AdamStep a) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        g[i] = 0.0f;
        const float mi = a.b1 * m[i] + (1.0f - a.b1) * gi, vi = a.b2 * v[i] + (1.0f - a.b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= a.lr * (mi * a.c1) / (sqrtf(vi * a.c2) + a.eps);
    }
}

__global__ void k_adam_grid(float2 *w, unsigned long long *gq, float2 *m, float2 *v, __half2 *feat, uint32_t n,
                            AdamStep a) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        // the fixed-point sums back to float (two's complement: a negative sum wraps)
        const float2 gi = make_float2((float)(long long)gq[2 * (size_t)i] * (1.0f / kGridFix),
                                      (float)(long long)gq[2 * (size_t)i + 1] * (1.0f / kGridFix));
        if (gi.x == 0.0f && gi.y == 0.0f && m[i].x == 0.0f && m[i].y == 0.0f) continue;   // never touched
        gq[2 * (size_t)i] = 0ull;
        gq[2 * (size_t)i + 1] = 0ull;
        float2 mi = m[i], vi = v[i], wi = w[i];
        mi.x = a.b1 * mi.x + (1.0f - a.b1) * gi.x;
        mi.y = a.b1 * mi.y + (1.0f - a.b1) * gi.y;
        vi.x = a.b2 * vi.x + (1.0f - a.b2) * gi.x * gi.x;
        vi.y = a.b2 * vi.y + (1.0f - a.b2) * gi.y * gi.y;
        wi.x -= a.lr * (mi.x * a.c1) / (sqrtf(vi.x * a.c2) + a.eps);
        wi.y -= a.lr * (mi.y * a.c1) / (sqrtf(vi.y * a.c2) + a.eps);
        m[i] = mi;
        v[i] = vi;
        w[i] = wi;
        feat[i] = __float22half2_rn(wi);
    }
}

// BF16 B fragments of every layer from the FP32 master weights W[l][k][n]:
// forward (k = input unit, n = output unit) and transposed (for dY W^T).
// W^T of every layer in the tcgen05 operand layout (row n = output unit, K = input unit).
__global__ void k_tc_weights(const float *w, __nv_bfloat16 *wtc) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (uint32_t)NW) return;
    const uint32_t l = idx / (W * W), n = (idx / W) % W, k = idx % W;
    unsigned char *base = reinterpret_cast<unsigned char *>(wtc) + (size_t)l * W * W * 2;
    // forward: row n = output unit, K = input unit; backward (dX): row n = input unit, K = output unit
    *reinterpret_cast<__nv_bfloat16 *>(base + tc_offset(n, k)) = __float2bfloat16_rn(w[l * W * W + k * W + n]);
    *reinterpret_cast<__nv_bfloat16 *>(base + (size_t)NW * 2 + tc_offset(n, k)) =
        __float2bfloat16_rn(w[l * W * W + n * W + k]);
}

__global__ void k_frags(const float *w, uint2 *wf, uint2 *wt) {
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (uint32_t)NFRAG) return;
    const uint32_t lane = idx & 31u, nn = (idx >> 5) & 7u, kk = (idx >> 8) & 3u, l = idx >> 10;
    const uint32_t g = lane >> 2, t = lane & 3u;
    const float *Wl = w + l * W * W;
    const uint32_t k0 = 16 * kk + 2 * t, c = 8 * nn + g;
    wf[idx] = make_uint2(pack_bf16(Wl[k0 * W + c], Wl[(k0 + 1) * W + c]),
                         pack_bf16(Wl[(k0 + 8) * W + c], Wl[(k0 + 9) * W + c]));
    wt[idx] = make_uint2(pack_bf16(Wl[c * W + k0], Wl[c * W + k0 + 1]), pack_bf16(Wl[c * W + k0 + 8], Wl[c * W + k0 + 9]));
}

__global__ void k_half_grid(const float2 *w, __half2 *feat, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        feat[i] = __float22half2_rn(w[i]);
}

constexpr uint32_t kGridN = GUIDE_LEVELS * GUIDE_T;   // float2 entries of the grid

// SplitMix64 for the seeded initialisation.
struct InitRng {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    float uniform(float a, float b) { return a + (b - a) * (float)((next() >> 11) * (1.0 / 9007199254740992.0)); }
};

}  // namespace

struct GuideState {
    int device = 0;
    GuideNetDev net{};
    float *w = nullptr, *w_grad = nullptr, *w_m = nullptr, *w_v = nullptr;
    float *bias = nullptr, *b_grad = nullptr, *b_m = nullptr, *b_v = nullptr;
    uint2 *wf = nullptr, *wt = nullptr;
    __nv_bfloat16 *wtc = nullptr;
    uint32_t *tc_error = nullptr;   // set by the tcgen05 kernel when a wait gives up
    bool use_tc = true;             // network on the tcgen05 kernels (else the mma.sync ones)
    __half2 *feat = nullptr;
    float2 *grid = nullptr, *grid_m = nullptr, *grid_v = nullptr;
    unsigned long long *grid_grad = nullptr;   // [entry][2], fixed point (k_guide_train)
    float *part = nullptr;                     // per-block gradient slots of k_guide_train
    // scratch of the deterministic row compaction (k_guide_weights / k_guide_compact)
    float *rec_weight = nullptr, *kept_weight = nullptr;
    uint32_t *rec_flag = nullptr, *rec_pos = nullptr;
    void *cub_temp = nullptr;
    size_t rec_cap = 0, cub_bytes = 0;
    uint32_t n_rec = 0;             // samples per wave whose vertices are recorded
    uint32_t steps_per_wave = 4;    // Adam steps on each wave's rows
    GuideRow *rows = nullptr;
    uint32_t rows_cap = 0;
    uint32_t *count = nullptr;      // [0] rows, then scratch
    float *wsum = nullptr, *loss = nullptr;
    float lr = 1e-2f;
    uint32_t step = 0;
    uint64_t trained_rows = 0;
    float last_loss = 0.0f;
    std::vector<void *> allocs;
    int sms = 148;
    int tc_blocks = 4;              // resident CTAs per SM of the tcgen05 inference kernel
    bool order_rows = true;         // tcgen05 inference visits a level's rows in spatial order
    uint32_t *row_keys = nullptr, *row_order = nullptr;   // [row_cap] (OrderRows)
    uint32_t row_cap = 0;
    uint32_t *bin_counts = nullptr, *bin_offsets = nullptr;
    unsigned char *bin_scan_temp = nullptr;
    size_t bin_scan_bytes = 0;
    std::mutex mu;

    ~GuideState() {
        for (void *p : allocs)
            if (p) cudaFree(p);
        for (void *p : {(void *)rec_weight, (void *)rec_flag, (void *)rec_pos, cub_temp, (void *)row_keys,
                        (void *)row_order})
            if (p) cudaFree(p);
    }
    template <typename T>
    T *Alloc(size_t n) {
        void *p = nullptr;
        if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return nullptr;
        allocs.push_back(p);
        return (T *)p;
    }
};

namespace {

// World bounds of the scene from its top-level root node.
void SceneBounds(const GpuScene &G, float lo[3], float hi[3]) {
    for (int a = 0; a < 3; a++) {
        lo[a] = -1.0f;
        hi[a] = 1.0f;
    }
    if (G.dev.tlas_root == 0xFFFFFFFFu) return;
    WideNode n;
    if (cudaMemcpy(&n, G.dev.wnodes + G.dev.tlas_root, sizeof(n), cudaMemcpyDeviceToHost) != cudaSuccess) return;
    const float p[3] = {n.px, n.py, n.pz};
    const uint8_t e[3] = {n.ex, n.ey, n.ez};
    const uint8_t *ql[3] = {n.qlo_x, n.qlo_y, n.qlo_z}, *qh[3] = {n.qhi_x, n.qhi_y, n.qhi_z};
    double l[3] = {1e30, 1e30, 1e30}, h[3] = {-1e30, -1e30, -1e30};
    for (int s = 0; s < 8; s++) {
        if (!((n.imask >> s) & 1u) && n.meta[s] == 0) continue;   // empty slot
        for (int a = 0; a < 3; a++) {
            const double step = std::ldexp(1.0, (int)e[a] - 127);
            l[a] = std::min(l[a], (double)p[a] + ql[a][s] * step);
            h[a] = std::max(h[a], (double)p[a] + qh[a][s] * step);
        }
    }
    for (int a = 0; a < 3; a++)
        if (l[a] < h[a]) {
            lo[a] = (float)l[a];
            hi[a] = (float)h[a];
        }
}

int RefreshFragments(GuideState &g, cudaStream_t st) {
    k_frags<<<(NFRAG + 255) / 256, 256, 0, st>>>(g.w, g.wf, g.wt);
    k_tc_weights<<<(NW + 255) / 256, 256, 0, st>>>(g.w, g.wtc);
    AZ_CUDA_TRY(cudaGetLastError());
    return AZ_OK;
}

// A normalised training row weight (mean 1) counts at most this much.
constexpr float kWeightCap = 25.0f;

// One training step over rows[0 .. min(*count, cap)): gradients, then Adam.
int TrainStep(GuideState &g, const GuideRow *rows, const uint32_t *count, uint32_t cap, const float *wsum,
              cudaStream_t st, float *dbg_out = nullptr, float *dbg_enc = nullptr, bool apply = true) {
    TrainArgs A;
    A.rows = rows;
    A.count = count;
    A.cap = cap;
    A.wsum = wsum;
    A.wcap = kWeightCap;
    A.part = g.part;
    A.grid_grad = g.grid_grad;
    A.dbg_out = dbg_out;
    A.dbg_enc = dbg_enc;
    if (g.use_tc) k_guide_train_tc<<<g.sms, kTcRows, kTcTrainSmem, st>>>(g.net, A, g.tc_error);
    else k_guide_train<<<g.sms, kWarps * 32, kTrainSmem, st>>>(g.net, A);
    k_guide_reduce<<<(NW + W + 1 + 255) / 256, 256, 0, st>>>(g.part, (uint32_t)g.sms, g.w_grad, g.b_grad, g.loss);
    AZ_CUDA_TRY(cudaGetLastError());
    if (!apply) return AZ_OK;
    g.step++;
    AdamStep a;
    a.lr = g.lr;
    a.b1 = 0.9f;
    a.b2 = 0.99f;
    a.eps = 1e-8f;
    a.c1 = (float)(1.0 / (1.0 - std::pow(0.9, (double)g.step)));
    a.c2 = (float)(1.0 / (1.0 - std::pow(0.99, (double)g.step)));
    k_adam<<<16, 256, 0, st>>>(g.w, g.w_grad, g.w_m, g.w_v, NW, a);
    k_adam<<<1, 64, 0, st>>>(g.bias, g.b_grad, g.b_m, g.b_v, W, a);
    k_adam_grid<<<g.sms * 8, 256, 0, st>>>(g.grid, g.grid_grad, g.grid_m, g.grid_v, g.feat, kGridN, a);
    AZ_CUDA_TRY(cudaGetLastError());
    return RefreshFragments(g, st);
}

}  // namespace

int CreateGuide(const GpuScene &G, const az_guide_config *cfg, GuideState **out) {
    std::unique_ptr<GuideState> g(new GuideState());
    g->device = G.device;
    cudaDeviceGetAttribute(&g->sms, cudaDevAttrMultiProcessorCount, G.device);
    g->lr = cfg && cfg->learning_rate > 0.0f ? cfg->learning_rate : 1e-2f;
    g->n_rec = cfg && cfg->record_samples ? cfg->record_samples : (1u << 17);
    g->steps_per_wave = cfg && cfg->steps_per_wave ? cfg->steps_per_wave : 4u;
    g->rows_cap = cfg && cfg->train_batch ? cfg->train_batch : (1u << 18);
    g->use_tc = !(cfg && cfg->kernels == AZ_GUIDE_MMA_SYNC);
    g->order_rows = !(cfg && cfg->queue_order_rows);
    const uint64_t seed = cfg ? cfg->seed : 0;
    g->w = g->Alloc<float>(NW);
    g->w_grad = g->Alloc<float>(NW);
    g->w_m = g->Alloc<float>(NW);
    g->w_v = g->Alloc<float>(NW);
    g->bias = g->Alloc<float>(W);
    g->b_grad = g->Alloc<float>(W);
    g->b_m = g->Alloc<float>(W);
    g->b_v = g->Alloc<float>(W);
    g->wf = g->Alloc<uint2>(NFRAG);
    g->wt = g->Alloc<uint2>(NFRAG);
    g->wtc = g->Alloc<__nv_bfloat16>(2 * NW);
    g->tc_error = g->Alloc<uint32_t>(1);
    g->feat = g->Alloc<__half2>(kGridN);
    g->grid = g->Alloc<float2>(kGridN);
    g->grid_grad = g->Alloc<unsigned long long>(2 * (size_t)kGridN);
    g->part = g->Alloc<float>((size_t)g->sms * kPart);
    g->grid_m = g->Alloc<float2>(kGridN);
    g->grid_v = g->Alloc<float2>(kGridN);
    g->rows = g->Alloc<GuideRow>(g->rows_cap);
    g->count = g->Alloc<uint32_t>(4);
    g->wsum = g->Alloc<float>(1);
    g->loss = g->Alloc<float>(1);
    for (void *p : g->allocs)
        if (!p) return SetError(AZ_ERR_OUT_OF_MEMORY, "path guide parameters");
    // Xavier-uniform weights, small uniform grid features; output biases
    // start at kappa = e and alpha = 0.05 + 0.9 sigmoid(-2) (mostly cosine
    // sampling until the network has learned something)
    InitRng r{seed * 0x2545F4914F6CDD1Dull + 0x1234567ull};
    std::vector<float> w(NW), b(W, 0.0f);
    const float lim = std::sqrt(6.0f / (W + W));
    for (int i = 0; i < NW; i++) w[i] = r.uniform(-lim, lim);
    for (int k = 0; k < GUIDE_LOBES; k++) b[5 * k + 3] = 1.0f;
    b[40] = -2.0f;
    std::vector<float2> grid(kGridN);
    for (uint32_t i = 0; i < kGridN; i++) grid[i] = make_float2(r.uniform(-1e-4f, 1e-4f), r.uniform(-1e-4f, 1e-4f));
    AZ_CUDA_TRY(cudaMemcpy(g->w, w.data(), NW * sizeof(float), cudaMemcpyHostToDevice));
    AZ_CUDA_TRY(cudaMemcpy(g->bias, b.data(), W * sizeof(float), cudaMemcpyHostToDevice));
    AZ_CUDA_TRY(cudaMemcpy(g->grid, grid.data(), kGridN * sizeof(float2), cudaMemcpyHostToDevice));
    AZ_CUDA_TRY(cudaMemset(g->w_grad, 0, NW * sizeof(float)));
    AZ_CUDA_TRY(cudaMemset(g->w_m, 0, NW * sizeof(float)));
    AZ_CUDA_TRY(cudaMemset(g->w_v, 0, NW * sizeof(float)));
    AZ_CUDA_TRY(cudaMemset(g->b_grad, 0, W * sizeof(float)));
    AZ_CUDA_TRY(cudaMemset(g->b_m, 0, W * sizeof(float)));
    AZ_CUDA_TRY(cudaMemset(g->b_v, 0, W * sizeof(float)));
    AZ_CUDA_TRY(cudaMemset(g->grid_grad, 0, 2 * (size_t)kGridN * sizeof(unsigned long long)));
    AZ_CUDA_TRY(cudaMemset(g->grid_m, 0, kGridN * sizeof(float2)));
    AZ_CUDA_TRY(cudaMemset(g->grid_v, 0, kGridN * sizeof(float2)));
    k_half_grid<<<g->sms * 8, 256>>>(g->grid, g->feat, kGridN);
    int rc = RefreshFragments(*g, nullptr);
    if (rc != AZ_OK) return rc;
    AZ_CUDA_TRY(cudaFuncSetAttribute(k_guide_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrainSmem));
    AZ_CUDA_TRY(cudaFuncSetAttribute(k_guide_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInferSmem));
    AZ_CUDA_TRY(cudaMemset(g->tc_error, 0, sizeof(uint32_t)));
    AZ_CUDA_TRY(cudaFuncSetAttribute(k_guide_mlp_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
    AZ_CUDA_TRY(cudaFuncSetAttribute(k_guide_mlp_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem));
    AZ_CUDA_TRY(
        cudaFuncSetAttribute(k_guide_train_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcTrainSmem));
    // the whole unified L1/shared array as shared memory for the kernels that
    // keep their weights there: without the preference the driver may keep the
    // larger L1 split, and one inference CTA of 54 KB per SM fits instead of four
    for (const void *k : {(const void *)k_guide_mlp_tc<false>, (const void *)k_guide_mlp_tc<true>,
                          (const void *)k_guide_train_tc, (const void *)k_guide_infer, (const void *)k_guide_train})
        AZ_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         (int)cudaSharedmemCarveoutMaxShared));
    // four resident inference CTAs per SM: the most that 64 registers a thread
    // and 55 KB of shared memory a CTA allow (each holds 64 of the SM's 512
    // tensor-memory columns while it runs); a grid of that many per SM
    g->tc_blocks = 4;
    // network view
    g->net.wtc = g->wtc;
    g->net.wf = g->wf;
    g->net.wt = g->wt;
    g->net.bias = g->bias;
    g->net.grid = g->feat;
    for (int l = 0; l < GUIDE_LEVELS; l++) g->net.res[l] = (uint32_t)std::floor(16.0 * std::pow(2.0, 7.0 * l / 15.0));
    float lo[3], hi[3];
    SceneBounds(G, lo, hi);
    for (int a = 0; a < 3; a++) {
        const float ext = std::max(hi[a] - lo[a], 1e-6f);
        g->net.lo[a] = lo[a];
        g->net.inv_ext[a] = 1.0f / ext;
    }
    AZ_CUDA_TRY(cudaDeviceSynchronize());
    *out = g.release();
    return AZ_OK;
}

void DestroyGuide(GuideState *g) { delete g; }

int GuidePrepareWave(GuideState &g, WaveBuffers &W, WaveQueues &Q, uint32_t cap_q, uint32_t levels, cudaStream_t st) {
    if (W.guide_lobes_cap < cap_q) {
        if (W.guide_lobes) cudaFree(W.guide_lobes);
        W.guide_lobes = nullptr;
        W.guide_lobes_cap = 0;
        if (cudaMalloc((void **)&W.guide_lobes, (size_t)cap_q * sizeof(GuideLobes)) != cudaSuccess)
            return SetError(AZ_ERR_OUT_OF_MEMORY, "path guide proposals");
        W.guide_lobes_cap = cap_q;
    }
    Q.lobes = W.guide_lobes;
    Q.cap_q = std::min<uint32_t>(Q.cap_q, (uint32_t)W.guide_lobes_cap);
    Q.rec = nullptr;
    Q.n_rec = 0;
    Q.rec_levels = 0;
    if (levels == 0) return AZ_OK;   // not training: no records
    const size_t need = (size_t)levels * g.n_rec;
    if (W.guide_rec_cap < need) {
        if (W.guide_rec) cudaFree(W.guide_rec);
        W.guide_rec = nullptr;
        W.guide_rec_cap = 0;
        if (cudaMalloc((void **)&W.guide_rec, need * sizeof(GuideRecord)) != cudaSuccess)
            return SetError(AZ_ERR_OUT_OF_MEMORY, "path guide records");
        W.guide_rec_cap = need;
    }
    // records of earlier waves must not be mistaken for this wave's
    AZ_CUDA_TRY(cudaMemsetAsync(W.guide_rec, 0, need * sizeof(GuideRecord), st));
    Q.rec = W.guide_rec;
    Q.n_rec = g.n_rec;
    Q.rec_levels = levels;
    return AZ_OK;
}

// ---- spatial order of a level's inference rows ----
// Neighbouring rows of a tile gather the same coarse hash-grid cells when
// their hit points are close, and those gathers then hit in L1.  A level's
// queue entries are bucketed by the 12-bit Morton code of the cell of their
// hit point (o + t d) in a 16^3 grid over the guide's box (misses in bucket
// 0): a histogram, an exclusive scan, a scatter with warp-aggregated
// atomics.  Rows within a bucket keep no particular order; the proposals do
// not depend on the order in which rows are evaluated.
constexpr uint32_t kSortBins = 4096;

__device__ __forceinline__ uint32_t spread4(uint32_t v) {   // bits b3..b0 to b9, b6, b3, b0
    return (v & 1u) | ((v & 2u) << 2) | ((v & 4u) << 4) | ((v & 8u) << 6);
}

__device__ __forceinline__ uint32_t row_bin(const WaveQueues &Q, int buf, uint32_t i, const GuideNetDev &N) {
    const uint4 hh = Q.hit[i];
    if (hh.w == 0xFFFFFFFFu) return 0u;
    const float4 o = Q.o[buf][i], d = Q.d[buf][i];
    const float t = __uint_as_float(hh.x);
    const f3 p = normalise_pos(N, mk(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z));
    const uint32_t x = min((uint32_t)(p.x * 16.0f), 15u), y = min((uint32_t)(p.y * 16.0f), 15u),
                   z = min((uint32_t)(p.z * 16.0f), 15u);
    return (spread4(x) << 2) | (spread4(y) << 1) | spread4(z);
}

// PASS 0: count rows per bin (keys kept); PASS 1: place every row at its bin's
// next slot.  Loop bounds are warp-uniform so that lanes with equal keys can
// share one atomic.
template <int PASS>
__global__ void k_guide_bins(WaveQueues Q, uint32_t level, GuideNetDev N, uint32_t *keys, uint32_t *bins,
                             uint32_t *order) {
    const uint32_t n = min(Q.counts[level], Q.cap_q);
    const int buf = level & 1;
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t b = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); b < n; b += gridDim.x * blockDim.x) {
        const uint32_t i = b + lane;
        const bool live = i < n;
        uint32_t key = 0xFFFFFFFFu;
        if (live) {
            if (PASS == 0) {
                key = row_bin(Q, buf, i, N);
                keys[i] = key;
            } else {
                key = keys[i];
            }
        }
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, key);
        const uint32_t leader = __ffs(peers) - 1u;
        uint32_t base = 0;
        if (live && lane == leader) base = atomicAdd(&bins[key], (uint32_t)__popc(peers));
        if (PASS == 1) {
            base = __shfl_sync(0xFFFFFFFFu, base, leader);
            if (live) order[base + __popc(peers & ((1u << lane) - 1u))] = i;
        }
    }
}

static int OrderRows(GuideState &g, const WaveQueues &Q, uint32_t level, cudaStream_t st);

int GuideInfer(GuideState &g, const GpuScene &G, const WaveQueues &Q, uint32_t level, cudaStream_t st) {
    if (g.use_tc) {
        const uint32_t *order = nullptr;
        if (g.order_rows) {
            int rc = OrderRows(g, Q, level, st);
            if (rc != AZ_OK) return rc;
            order = g.row_order;
        }
        k_guide_mlp_tc<false><<<g.sms * g.tc_blocks, kTcThreads, kTcSmem, st>>>(G.dev, Q, level, g.net, Q.lobes,
                                                                             nullptr, 0, nullptr, g.tc_error, order);
    } else
        k_guide_infer<<<g.sms * 3, kInferWarps * 32, kInferSmem, st>>>(G.dev, Q, level, g.net, Q.lobes);
    AZ_CUDA_TRY(cudaGetLastError());
    return AZ_OK;
}

static int OrderRows(GuideState &g, const WaveQueues &Q, uint32_t level, cudaStream_t st) {
    if (g.row_cap < Q.cap_q) {
        for (void **p : {(void **)&g.row_keys, (void **)&g.row_order}) {
            if (*p) cudaFree(*p);
            *p = nullptr;
        }
        g.row_cap = 0;
        if (cudaMalloc((void **)&g.row_keys, (size_t)Q.cap_q * sizeof(uint32_t)) != cudaSuccess ||
            cudaMalloc((void **)&g.row_order, (size_t)Q.cap_q * sizeof(uint32_t)) != cudaSuccess)
            return SetError(AZ_ERR_OUT_OF_MEMORY, "path guide row order");
        g.row_cap = Q.cap_q;
    }
    if (!g.bin_counts) {
        size_t bytes = 0;
        AZ_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, bytes, g.bin_counts, g.bin_offsets, (int)kSortBins));
        g.bin_scan_bytes = bytes;
        g.bin_counts = g.Alloc<uint32_t>(kSortBins);
        g.bin_offsets = g.Alloc<uint32_t>(kSortBins);
        g.bin_scan_temp = g.Alloc<unsigned char>(std::max<size_t>(bytes, 16));
        if (!g.bin_counts || !g.bin_offsets || !g.bin_scan_temp) return SetError(AZ_ERR_OUT_OF_MEMORY, "row bins");
    }
    AZ_CUDA_TRY(cudaMemsetAsync(g.bin_counts, 0, kSortBins * sizeof(uint32_t), st));
    const int grid = g.sms * 8;
    k_guide_bins<0><<<grid, 256, 0, st>>>(Q, level, g.net, g.row_keys, g.bin_counts, nullptr);
    size_t bytes = g.bin_scan_bytes;
    AZ_CUDA_TRY(cub::DeviceScan::ExclusiveSum(g.bin_scan_temp, bytes, g.bin_counts, g.bin_offsets, (int)kSortBins, st));
    k_guide_bins<1><<<grid, 256, 0, st>>>(Q, level, g.net, g.row_keys, g.bin_offsets, g.row_order);
    AZ_CUDA_TRY(cudaGetLastError());
    return AZ_OK;
}

int GuideTrainWave(GuideState &g, const WaveQueues &Q, cudaStream_t st) {
    AZ_CUDA_TRY(cudaMemsetAsync(g.count, 0, 4 * sizeof(uint32_t), st));
    AZ_CUDA_TRY(cudaMemsetAsync(g.wsum, 0, sizeof(float), st));
    const uint32_t total = Q.n_rec * Q.rec_levels;
    if (total == 0) return AZ_OK;
    if (g.rec_cap < total) {
        for (void **p : {(void **)&g.rec_weight, (void **)&g.rec_flag, (void **)&g.rec_pos, &g.cub_temp}) {
            if (*p) cudaFree(*p);
            *p = nullptr;
        }
        g.rec_cap = 0;
        size_t scan_bytes = 0, sum_bytes = 0;
        AZ_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, g.rec_flag, g.rec_pos, (int)total));
        AZ_CUDA_TRY(cub::DeviceReduce::Sum(nullptr, sum_bytes, g.kept_weight, g.wsum, (int)g.rows_cap));
        g.cub_bytes = std::max(scan_bytes, sum_bytes);
        if (cudaMalloc((void **)&g.rec_weight, (size_t)total * sizeof(float) + (size_t)g.rows_cap * sizeof(float)) !=
                cudaSuccess ||
            cudaMalloc((void **)&g.rec_flag, (size_t)total * sizeof(uint32_t)) != cudaSuccess ||
            cudaMalloc((void **)&g.rec_pos, (size_t)total * sizeof(uint32_t)) != cudaSuccess ||
            cudaMalloc(&g.cub_temp, g.cub_bytes) != cudaSuccess)
            return SetError(AZ_ERR_OUT_OF_MEMORY, "path guide training scratch");
        g.rec_cap = total;
    }
    g.kept_weight = g.rec_weight + g.rec_cap;   // rows_cap floats after the records' weights
    const int grid = g.sms * 4;
    k_guide_weights<<<grid, 256, 0, st>>>(Q.rec, total, Q.n_rec, Q.accum, g.rec_weight, g.rec_flag);
    size_t bytes = g.cub_bytes;
    AZ_CUDA_TRY(cub::DeviceScan::ExclusiveSum(g.cub_temp, bytes, g.rec_flag, g.rec_pos, (int)total, st));
    AZ_CUDA_TRY(cudaMemsetAsync(g.kept_weight, 0, (size_t)g.rows_cap * sizeof(float), st));
    k_guide_compact<<<grid, 256, 0, st>>>(Q.rec, total, g.rec_weight, g.rec_flag, g.rec_pos, g.rows, g.kept_weight,
                                          g.rows_cap, g.count);
    bytes = g.cub_bytes;
    AZ_CUDA_TRY(cub::DeviceReduce::Sum(g.cub_temp, bytes, g.kept_weight, g.wsum, (int)g.rows_cap, st));
    AZ_CUDA_TRY(cudaGetLastError());
    for (uint32_t k = 0; k < g.steps_per_wave; k++) {
        int rc = TrainStep(g, g.rows, g.count, g.rows_cap, g.wsum, st);
        if (rc != AZ_OK) return rc;
    }
    return AZ_OK;
}

}  // namespace az

using namespace az;

struct az_guide {
    GuideState *impl;
};

namespace az {
GuideState *GuideOf(az_guide *g) { return g ? g->impl : nullptr; }
int GuideCheck(GuideState &g, cudaStream_t st) {
    uint32_t e = 0;
    AZ_CUDA_TRY(cudaMemcpyAsync(&e, g.tc_error, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    AZ_CUDA_TRY(cudaStreamSynchronize(st));
    if (!e) return AZ_OK;
    AZ_CUDA_TRY(cudaMemsetAsync(g.tc_error, 0, sizeof(uint32_t), st));
    return SetError(AZ_ERR_CUDA, "tensor-core proposals: a wait on the MMA gave up");
}
std::mutex &GuideLock(GuideState &g) { return g.mu; }
}  // namespace az

extern "C" int az_guide_create(az_gpu_scene *scene, const az_guide_config *cfg, az_guide **out) {
    if (!scene || !scene->impl || !out) return SetError(AZ_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    AZ_CUDA_TRY(cudaSetDevice(scene->impl->device));
    GuideState *g = nullptr;
    int rc = CreateGuide(*scene->impl, cfg, &g);
    if (rc != AZ_OK) return rc;
    *out = new az_guide{g};
    return AZ_OK;
}

extern "C" void az_guide_destroy(az_guide *g) {
    if (!g) return;
    cudaSetDevice(g->impl->device);
    cudaDeviceSynchronize();
    DestroyGuide(g->impl);
    delete g;
}

extern "C" int az_guide_info(az_guide *g, uint32_t *res, float *lo, float *inv_ext, uint32_t *steps) {
    if (!g) return SetError(AZ_ERR_INVALID_ARGUMENT, "null guide");
    for (int l = 0; l < GUIDE_LEVELS && res; l++) res[l] = g->impl->net.res[l];
    for (int a = 0; a < 3; a++) {
        if (lo) lo[a] = g->impl->net.lo[a];
        if (inv_ext) inv_ext[a] = g->impl->net.inv_ext[a];
    }
    if (steps) *steps = g->impl->step;
    return AZ_OK;
}

extern "C" int az_guide_get_params(az_guide *g, float *mlp, float *bias, float *grid) {
    if (!g) return SetError(AZ_ERR_INVALID_ARGUMENT, "null guide");
    GuideState &s = *g->impl;
    AZ_CUDA_TRY(cudaSetDevice(s.device));
    AZ_CUDA_TRY(cudaDeviceSynchronize());
    if (mlp) AZ_CUDA_TRY(cudaMemcpy(mlp, s.w, NW * sizeof(float), cudaMemcpyDeviceToHost));
    if (bias) AZ_CUDA_TRY(cudaMemcpy(bias, s.bias, W * sizeof(float), cudaMemcpyDeviceToHost));
    if (grid) AZ_CUDA_TRY(cudaMemcpy(grid, s.grid, kGridN * sizeof(float2), cudaMemcpyDeviceToHost));
    return AZ_OK;
}

extern "C" int az_guide_set_params(az_guide *g, const float *mlp, const float *bias, const float *grid) {
    if (!g) return SetError(AZ_ERR_INVALID_ARGUMENT, "null guide");
    GuideState &s = *g->impl;
    AZ_CUDA_TRY(cudaSetDevice(s.device));
    AZ_CUDA_TRY(cudaDeviceSynchronize());
    if (mlp) AZ_CUDA_TRY(cudaMemcpy(s.w, mlp, NW * sizeof(float), cudaMemcpyHostToDevice));
    if (bias) AZ_CUDA_TRY(cudaMemcpy(s.bias, bias, W * sizeof(float), cudaMemcpyHostToDevice));
    if (grid) {
        AZ_CUDA_TRY(cudaMemcpy(s.grid, grid, kGridN * sizeof(float2), cudaMemcpyHostToDevice));
        k_half_grid<<<s.sms * 8, 256>>>(s.grid, s.feat, kGridN);
    }
    int rc = RefreshFragments(s, nullptr);
    if (rc != AZ_OK) return rc;
    AZ_CUDA_TRY(cudaDeviceSynchronize());
    return AZ_OK;
}

// Rows are host arrays of 16 floats: position, weight, normal, 0, outgoing
// direction, 0, incident direction, 0 (the GuideRow layout).
static int UploadRows(GuideState &s, const float *rows, uint32_t n, GuideRow **d_rows, uint32_t **d_count) {
    *d_rows = nullptr;
    *d_count = nullptr;
    AZ_CUDA_TRY(cudaMalloc((void **)d_rows, std::max<size_t>(n, 1) * sizeof(GuideRow)));
    AZ_CUDA_TRY(cudaMalloc((void **)d_count, sizeof(uint32_t)));
    AZ_CUDA_TRY(cudaMemcpy(*d_rows, rows, (size_t)n * sizeof(GuideRow), cudaMemcpyHostToDevice));
    AZ_CUDA_TRY(cudaMemcpy(*d_count, &n, sizeof(uint32_t), cudaMemcpyHostToDevice));
    return AZ_OK;
}

extern "C" int az_guide_eval(az_guide *g, const float *rows, uint32_t n, float *outputs, float *loss,
                             float *mlp_grad, float *bias_grad, float *enc_grad) {
    if (!g || (n && !rows)) return SetError(AZ_ERR_INVALID_ARGUMENT, "null argument");
    GuideState &s = *g->impl;
    AZ_CUDA_TRY(cudaSetDevice(s.device));
    GuideRow *d_rows = nullptr;
    uint32_t *d_count = nullptr;
    float *d_out = nullptr, *d_enc = nullptr;
    int rc = UploadRows(s, rows, n, &d_rows, &d_count);
    if (rc == AZ_OK && outputs && cudaMalloc((void **)&d_out, std::max<size_t>(n, 1) * W * sizeof(float)) != cudaSuccess)
        rc = SetError(AZ_ERR_OUT_OF_MEMORY, "eval outputs");
    if (rc == AZ_OK && enc_grad && cudaMalloc((void **)&d_enc, std::max<size_t>(n, 1) * 32 * sizeof(float)) != cudaSuccess)
        rc = SetError(AZ_ERR_OUT_OF_MEMORY, "eval gradients");
    if (rc == AZ_OK) {
        cudaMemset(s.w_grad, 0, NW * sizeof(float));
        cudaMemset(s.b_grad, 0, W * sizeof(float));
        // the grid gradient is not needed here: pass none
        unsigned long long *gg = s.grid_grad;
        s.grid_grad = nullptr;
        rc = TrainStep(s, d_rows, d_count, n, nullptr, nullptr, d_out, d_enc, false);
        s.grid_grad = gg;
    }
    if (rc == AZ_OK) {
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) rc = CudaError(e, "guide eval");
    }
    if (rc == AZ_OK) rc = GuideCheck(s, nullptr);
    if (rc == AZ_OK && outputs) cudaMemcpy(outputs, d_out, (size_t)n * W * sizeof(float), cudaMemcpyDeviceToHost);
    if (rc == AZ_OK && enc_grad) cudaMemcpy(enc_grad, d_enc, (size_t)n * 32 * sizeof(float), cudaMemcpyDeviceToHost);
    if (rc == AZ_OK && loss) cudaMemcpy(loss, s.loss, sizeof(float), cudaMemcpyDeviceToHost);
    if (rc == AZ_OK && mlp_grad) cudaMemcpy(mlp_grad, s.w_grad, NW * sizeof(float), cudaMemcpyDeviceToHost);
    if (rc == AZ_OK && bias_grad) cudaMemcpy(bias_grad, s.b_grad, W * sizeof(float), cudaMemcpyDeviceToHost);
    cudaMemset(s.w_grad, 0, NW * sizeof(float));
    cudaMemset(s.b_grad, 0, W * sizeof(float));
    cudaFree(d_rows);
    cudaFree(d_count);
    if (d_out) cudaFree(d_out);
    if (d_enc) cudaFree(d_enc);
    return rc;
}

extern "C" int az_guide_train(az_guide *g, const float *rows, uint32_t n, uint32_t steps, float *losses) {
    if (!g || (n && !rows)) return SetError(AZ_ERR_INVALID_ARGUMENT, "null argument");
    GuideState &s = *g->impl;
    AZ_CUDA_TRY(cudaSetDevice(s.device));
    GuideRow *d_rows = nullptr;
    uint32_t *d_count = nullptr;
    int rc = UploadRows(s, rows, n, &d_rows, &d_count);
    for (uint32_t k = 0; k < steps && rc == AZ_OK; k++) {
        rc = TrainStep(s, d_rows, d_count, n, nullptr, nullptr);
        if (rc == AZ_OK && losses) {
            cudaError_t e = cudaMemcpy(&losses[k], s.loss, sizeof(float), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) rc = CudaError(e, "guide train");
        }
    }
    if (rc == AZ_OK) {
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) rc = CudaError(e, "guide train");
    }
    if (rc == AZ_OK) rc = GuideCheck(s, nullptr);
    cudaFree(d_rows);
    cudaFree(d_count);
    return rc;
}

extern "C" int az_guide_infer(az_guide *g, const float *rows, uint32_t n, float *outputs) {
    if (!g || (n && (!rows || !outputs))) return SetError(AZ_ERR_INVALID_ARGUMENT, "null argument");
    GuideState &s = *g->impl;
    AZ_CUDA_TRY(cudaSetDevice(s.device));
    if (n == 0) return AZ_OK;
    GuideRow *d_rows = nullptr;
    uint32_t *d_count = nullptr;
    float *d_out = nullptr;
    int rc = UploadRows(s, rows, n, &d_rows, &d_count);
    if (rc == AZ_OK && cudaMalloc((void **)&d_out, (size_t)n * W * sizeof(float)) != cudaSuccess)
        rc = SetError(AZ_ERR_OUT_OF_MEMORY, "inference outputs");
    if (rc == AZ_OK) {
        cudaMemset(s.tc_error, 0, sizeof(uint32_t));
        DevScene none;
        memset(&none, 0, sizeof(none));
        WaveQueues q;
        memset(&q, 0, sizeof(q));
        k_guide_mlp_tc<true><<<std::min<uint32_t>((n + kTcRows - 1) / kTcRows, (uint32_t)(s.sms * s.tc_blocks)),
                               kTcThreads, kTcSmem>>>(
            none, q, 0, s.net, nullptr, d_rows, n, d_out, s.tc_error);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e != cudaSuccess) rc = CudaError(e, "guide inference");
    }
    uint32_t terr = 0;
    if (rc == AZ_OK) cudaMemcpy(&terr, s.tc_error, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    if (rc == AZ_OK && terr) rc = SetError(AZ_ERR_CUDA, "tensor-core inference: a wait on the MMA gave up");
    if (rc == AZ_OK) cudaMemcpy(outputs, d_out, (size_t)n * W * sizeof(float), cudaMemcpyDeviceToHost);
    cudaFree(d_rows);
    cudaFree(d_count);
    if (d_out) cudaFree(d_out);
    return rc;
}
