// Neural path guiding: device-side pieces shared by the guide kernels
// (az_guide.cu) and the shading kernel.
//
// The guide maps a surface point (position, geometric normal, outgoing
// direction) to a proposal density over incident directions: a mixture of 8
// von Mises-Fisher lobes, mixed with cosine-weighted hemisphere sampling by a
// learned selection probability alpha (one-sample MIS with the balance
// heuristic: q(w) = alpha * q_vmf(w) + (1 - alpha) * cos / pi), so any
// direction the cosine term can produce keeps a positive density and the
// estimator stays unbiased.
//
// Network: a multiresolution hash-grid encoding of the position (Mueller,
// Evans, Schied, Keller, "Instant Neural Graphics Primitives with a
// Multiresolution Hash Encoding", SIGGRAPH 2022: 16 levels, 2^19 entries per
// level, 2 features per entry, geometric growth of the grid resolution from
// 16 to 2048 cells, spatial hash with primes 1, 2654435761, 805459861) plus
// the normal, the outgoing direction and a constant 1 -> 64 inputs, three
// hidden layers of 64 with ReLU, and a 64-wide output layer of which 41
// values are used: per lobe a mean direction (3, normalised), log kappa and
// a mixture logit, then the selection logit.  The mixture parameterisation
// and the KL-divergence training objective follow Mueller, McWilliams, Rousselle,
// Gross, Novak, "Neural Importance Sampling" (ToG 2019) and Dong, Wang, Fan,
// Zhang, Wang, Zhou, "Neural Parametric Mixtures for Path Guiding" (SIGGRAPH
// 2023).
#pragma once
#include <cstdint>

#include "az_device_math.cuh"

namespace azd {

constexpr int GUIDE_LEVELS = 16;
constexpr int GUIDE_LOG2_T = 19;
constexpr uint32_t GUIDE_T = 1u << GUIDE_LOG2_T;   // entries per level
constexpr int GUIDE_WIDTH = 64;                     // inputs, hidden units, outputs
constexpr int GUIDE_LAYERS = 4;                     // 3 hidden + output
constexpr int GUIDE_LOBES = 8;
constexpr int GUIDE_OUTPUTS = GUIDE_LOBES * 5 + 1;  // 41 used outputs
constexpr float GUIDE_LOGK_MIN = -3.0f, GUIDE_LOGK_MAX = 5.0f;   // kappa in [0.05, 148]
// alpha in [0.05, 0.8]: at least a fifth of the samples stay cosine-distributed
// (defensive mixture), so a direction the guide misjudges gains at most 5x the
// cosine-sampling weight at a vertex
constexpr float GUIDE_ALPHA_MIN = 0.05f, GUIDE_ALPHA_SPAN = 0.75f;
constexpr float GUIDE_PI = 3.14159265358979f;

// Grid resolution of level l: floor(16 * b^l), b = (2048 / 16)^(1 / 15),
// evaluated once on the host in double precision (GuideNetDev.res).

// Index of grid vertex (x, y, z) of a level with `res` cells per axis:
// dense when the (res + 1)^3 vertices fit in the table, hashed otherwise.
__host__ __device__ __forceinline__ uint32_t guide_index(uint32_t x, uint32_t y, uint32_t z, uint32_t res) {
    const uint64_t n1 = (uint64_t)res + 1u;
    if (n1 * n1 * n1 <= GUIDE_T) return (uint32_t)(x + n1 * (y + n1 * z));
    return (x * 1u ^ y * 2654435761u ^ z * 805459861u) & (GUIDE_T - 1u);
}

// Proposal of one surface point: lobes (mean, kappa), per-lobe pdf factors
// c_k = pi_k * kappa_k / (2 pi (1 - exp(-2 kappa_k))), cumulative mixture
// weights for lobe selection, and alpha.
struct __align__(16) GuideLobes {
    float4 mk[GUIDE_LOBES];     // mean direction, kappa
    float c[GUIDE_LOBES];
    float cdf[GUIDE_LOBES];     // cdf[k] = pi_0 + ... + pi_k
    float alpha;
    float pad[3];
};
static_assert(sizeof(GuideLobes) == 13 * 16, "GuideLobes is 13 float4");

__device__ __forceinline__ float guide_vmf_mixture_pdf(const GuideLobes &G, f3 w) {
    float q = 0.0f;
#pragma unroll
    for (int k = 0; k < GUIDE_LOBES; k++) {
        const float4 m = G.mk[k];
        q += G.c[k] * __expf(m.w * (m.x * w.x + m.y * w.y + m.z * w.z - 1.0f));
    }
    return q;
}

// q(w) = alpha q_vmf(w) + (1 - alpha) max(0, n.w) / pi
__device__ __forceinline__ float guide_mixture_pdf(const GuideLobes &G, f3 n, f3 w) {
    const float cs = fmaxf(0.0f, dot(n, w));
    return G.alpha * guide_vmf_mixture_pdf(G, w) + (1.0f - G.alpha) * cs * (1.0f / GUIDE_PI);
}

// The same mixture with the selection probability `alpha` given (any alpha
// in [0, 1] gives an unbiased one-sample MIS estimator).
__device__ __forceinline__ float guide_mixture_pdf_alpha(const GuideLobes &G, float alpha, f3 n, f3 w) {
    const float cs = fmaxf(0.0f, dot(n, w));
    return alpha * guide_vmf_mixture_pdf(G, w) + (1.0f - alpha) * cs * (1.0f / GUIDE_PI);
}

// Direction from lobe `k` (Wood 1994 / Jakob 2012 closed form for the vMF
// on the sphere): cos theta = 1 + log(u1 + (1 - u1) exp(-2 kappa)) / kappa.
__device__ __forceinline__ f3 guide_sample_lobe(const GuideLobes &G, int k, float u1, float u2) {
    const float4 m = G.mk[k];
    const float kap = m.w;
    float ct = 1.0f + __logf(u1 + (1.0f - u1) * __expf(-2.0f * kap)) / kap;
    ct = fminf(1.0f, fmaxf(-1.0f, ct));
    const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
    const float ph = 2.0f * GUIDE_PI * u2;
    f3 mu = mk(m.x, m.y, m.z), U, V;
    onb(mu, U, V);
    return normalize(U * (st * __cosf(ph)) + V * (st * __sinf(ph)) + mu * ct);
}

__device__ __forceinline__ int guide_pick_lobe(const GuideLobes &G, float u) {
    int k = 0;
#pragma unroll
    for (int j = 0; j < GUIDE_LOBES - 1; j++) k += u >= G.cdf[j] ? 1 : 0;
    return k;
}

// One scattering vertex recorded for training (first n_rec samples of a wave,
// paths that never branched).  `snap` is the sample's accumulated radiance
// when its child vertex is shaded: what arrives along `wi` is then
// (final accumulation - snap) / tp_child.
struct __align__(16) GuideRecord {
    float4 pos_q;    // hit point, pdf q(wi) the direction was sampled with
    float4 n;        // geometric normal (network input), w unused
    float4 wo;       // outgoing direction (towards the previous vertex)
    float4 wi;       // sampled scattering direction
    float4 tpc;      // child's path throughput, w = 1 when the child was queued
    float4 snap;     // accumulation before the child vertex adds anything; w = 1 once written
};

// A training row: position, normal, outgoing and incident direction, weight.
struct __align__(16) GuideRow {
    float4 pos_w;    // position, KL weight F(wi) / q(wi)
    float4 n;
    float4 wo;
    float4 wi;
};

}  // namespace azd
