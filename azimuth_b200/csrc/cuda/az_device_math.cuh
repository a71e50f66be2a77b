// Device-side float3 math with azimuth's operation order.
//
// The translation units whose results must round like azimuth's scalar C++
// (src/azimuth_math.cpp:572-1348) -- primitive tests, camera rays, shading,
// mesh ingestion -- are compiled with --fmad=false, so a*b+c rounds twice
// there; divisions and square roots are IEEE (-prec-div/-prec-sqrt default).
// Fused multiply-adds appear there only where the code asks for them
// explicitly (box tests in the traversal).  The path guide's unit is compiled
// with contraction (azimuth_b200/build.py, CONTRACTED).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace azd {

#define AZD_PI_F32 ((float)3.14159265359)   // azimuth's Pi_f32 (src/azimuth_math.h:3-4)

struct f3 {
    float x, y, z;
};

__host__ __device__ __forceinline__ f3 mk(float x, float y, float z) { return f3{x, y, z}; }
__host__ __device__ __forceinline__ f3 operator+(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ f3 operator-(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ f3 operator*(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ f3 operator*(float s, f3 a) { return mk(s * a.x, s * a.y, s * a.z); }
__host__ __device__ __forceinline__ f3 operator-(f3 a) { return mk(-a.x, -a.y, -a.z); }
__host__ __device__ __forceinline__ f3 had(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
__host__ __device__ __forceinline__ float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ f3 cross(f3 a, f3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ float length(f3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
// Normalize, src/azimuth_math.cpp:1298-1313 (zero vector stays zero)
__host__ __device__ __forceinline__ f3 normalize(f3 a) {
    float l = length(a);
    if (l != 0.0f) return mk(a.x / l, a.y / l, a.z / l);
    return mk(0.0f, 0.0f, 0.0f);
}
// Reflect, src/azimuth_math.cpp:1335-1348
__host__ __device__ __forceinline__ f3 reflect(f3 v, f3 r) { return (2.0f * dot(v, r)) * r - v; }
__host__ __device__ __forceinline__ bool is_zero(f3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }
__host__ __device__ __forceinline__ float comp(f3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

// 3x4 affine matrix rows (azimuth's mat4 E[0..2][0..3]; the 4th row is 0 0 0 1).
struct m34 {
    float e[12];
};

// PointToWorld, src/azimuth_math.cpp:1775-1800
__host__ __device__ __forceinline__ f3 point_xf(const m34 &m, f3 v) {
    return mk(m.e[0] * v.x + m.e[1] * v.y + m.e[2] * v.z + m.e[3],
              m.e[4] * v.x + m.e[5] * v.y + m.e[6] * v.z + m.e[7],
              m.e[8] * v.x + m.e[9] * v.y + m.e[10] * v.z + m.e[11]);
}
// VectorToWorld, src/azimuth_math.cpp:1803-1826
__host__ __device__ __forceinline__ f3 vector_xf(const m34 &m, f3 v) {
    return mk(m.e[0] * v.x + m.e[1] * v.y + m.e[2] * v.z, m.e[4] * v.x + m.e[5] * v.y + m.e[6] * v.z,
              m.e[8] * v.x + m.e[9] * v.y + m.e[10] * v.z);
}
// NormalToWorld with the inverse matrix, src/azimuth_math.cpp:1828-1843
__host__ __device__ __forceinline__ f3 normal_xf(const m34 &inv, f3 v) {
    return normalize(mk(inv.e[0] * v.x + inv.e[4] * v.y + inv.e[8] * v.z,
                        inv.e[1] * v.x + inv.e[5] * v.y + inv.e[9] * v.z,
                        inv.e[2] * v.x + inv.e[6] * v.y + inv.e[10] * v.z));
}
// OrthonormalBasis (Duff et al. 2017), src/azimuth_math.cpp:1845-1863
__host__ __device__ __forceinline__ void onb(f3 w, f3 &u, f3 &v) {
    if (w.z < 0.0f) {
        const float a = 1.0f / (1.0f - w.z);
        const float b = w.x * w.y * a;
        u = mk(1.0f - w.x * w.x * a, -b, w.x);
        v = mk(b, w.y * w.y * a - 1.0f, -w.y);
    } else {
        const float a = 1.0f / (1.0f + w.z);
        const float b = -w.x * w.y * a;
        u = mk(1.0f - w.x * w.x * a, b, -w.x);
        v = mk(b, 1.0f - w.y * w.y * a, -w.y);
    }
}

// ---------------------------------------------------------------------------
// Counter-based RNG: Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
// Draw `dim` of tree node (level, digits) of camera sample (pixel, sample) is
// lane dim&3 of Philox(counter = {pixel, sample, digits, level<<24 | dim>>2},
// key = seed), mapped to [0,1) as (x >> 8) * 2^-24.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                                       uint32_t k0, uint32_t k1, uint32_t out[4]) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
        uint32_t lo0 = 0xD2511F53u * c0, hi0 = __umulhi(0xD2511F53u, c0);
        uint32_t lo1 = 0xCD9E8D57u * c2, hi1 = __umulhi(0xCD9E8D57u, c2);
#else
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32), lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
#endif
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

__host__ __device__ __forceinline__ float u24(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

// One tree node's draw stream.  Consecutive draws share one Philox block of 4.
struct NodeRng {
    uint32_t pixel, sample, digits, level;
    uint32_t k0, k1;
    uint32_t dim;
    uint32_t cache[4];
    uint32_t cached_block;  // dim >> 2 of `cache`, or 0xFFFFFFFF

    __host__ __device__ __forceinline__ void init(uint64_t seed, uint32_t px, uint32_t smp, uint32_t dg,
                                                  uint32_t lv) {
        pixel = px; sample = smp; digits = dg; level = lv;
        k0 = (uint32_t)seed; k1 = (uint32_t)(seed >> 32);
        dim = 0;
        cached_block = 0xFFFFFFFFu;
    }
    __host__ __device__ __forceinline__ void skip(uint32_t n) { dim += n; }
    __host__ __device__ __forceinline__ float next() {
        uint32_t blk = dim >> 2;
        if (blk != cached_block) {
            philox4x32_10(pixel, sample, digits, (level << 24) | blk, k0, k1, cache);
            cached_block = blk;
        }
        // select instead of indexing, so the block stays in registers
        const uint32_t k = dim++ & 3u;
        return u24(k == 0u ? cache[0] : (k == 1u ? cache[1] : (k == 2u ? cache[2] : cache[3])));
    }
};

// Digits of child `k` (0..3) of a node at `level` (the child is at level+1).
__host__ __device__ __forceinline__ uint32_t child_digits(uint32_t digits, uint32_t level, uint32_t k) {
    uint32_t cl = level + 1;
    if (cl >= 2 && cl - 2 < 16) digits |= (k & 3u) << (2u * (cl - 2u));
    return digits;
}

}  // namespace azd
