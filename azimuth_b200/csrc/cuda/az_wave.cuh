// Device helpers shared by the wave kernels: the queue pushes of the shading
// stage, the per-sample sums, and the mapping from a wave slot to its pixel
// and sample.  Included by the traversal translation unit (az_render.cu,
// compiled without FMA contraction so that the primitive tests round like
// azimuth) and by the shading translation unit (az_shade_kernel.cu).
#pragma once
#include "az_render.h"
#include "az_scene_dev.cuh"

namespace az {

// Shadow-query kinds (CalculateLighting occlusion rules, src/azimuth_main.cpp:685-712)
enum : uint32_t {
    SHADOW_TMAX = 0,     // point/area/spot: occluded by a hit with t < 1 - ShadowRay epsilon
    SHADOW_ANY = 1,      // directional light and environment ray: occluded by any hit
    SHADOW_ENTITY = 2,   // entity light: occluded unless the nearest hit is the light's entity
    SHADOW_ENTITY_FULL = 3   // the same for a light too large for the two-phase test: k_shadow_full
};

// flags packed into d.w of a path entry
// PF_BRANCHED: an ancestor vertex spawned more than one child (its
// descendants are not used for training the path guide)
// PF_SCENE: in a tile wave of several scenes, the entry's scene index
enum : uint32_t { PF_INSIDE = 1u, PF_ATTEN = 2u, PF_BRANCHED = 4u, PF_SCENE_SHIFT = 16u, PF_SCENE = 0xFF0000u };

// A shadow entry's meta word: kind (2 bits) | scene index (8 bits) | light index (22 bits)
__host__ __device__ __forceinline__ uint32_t shadow_meta(uint32_t kind, uint32_t scene, uint32_t light) {
    return (kind << 30) | ((scene & 0xFFu) << 22) | (light & 0x3FFFFFu);
}
__host__ __device__ __forceinline__ uint32_t shadow_kind(uint32_t meta) { return meta >> 30; }
__host__ __device__ __forceinline__ uint32_t shadow_scene(uint32_t meta) { return (meta >> 22) & 0xFFu; }
__host__ __device__ __forceinline__ uint32_t shadow_light(uint32_t meta) { return meta & 0x3FFFFFu; }

// Most scenes a tile wave can hold (the 8-bit scene index above)
constexpr uint32_t kMaxWaveScenes = 256;

__host__ __device__ __forceinline__ void sample_of(const CameraParams &cam, uint64_t s, uint32_t &row,
                                                   uint32_t &col, uint32_t &sx, uint32_t &sy) {
    uint64_t pix = s % cam.npix, k = s / cam.npix;
    row = cam.r0 + (uint32_t)(pix / cam.wsc);
    col = cam.c0 + (uint32_t)(pix % cam.wsc);
    sx = (uint32_t)(k % cam.sqrt_spp);
    sy = (uint32_t)(k / cam.sqrt_spp);
}

__device__ __forceinline__ uint32_t push_slot(uint32_t *counter) {
    // warp-aggregated atomic increment
    uint32_t mask = __activemask();
    int lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(mask, base, leader);
    return base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
}

__device__ __forceinline__ void add_accum(float4 *accum, uint32_t slot, azd::f3 v) {
    if (azd::is_zero(v)) return;
    atomicAdd(&accum[slot], make_float4(v.x, v.y, v.z, 0.0f));   // one vector atomic (sm_90 and later)
}

__device__ __forceinline__ void push_path(const WaveQueues &Q, int buf, uint32_t level, azd::f3 o, float time,
                                          azd::f3 d, uint32_t flags, azd::f3 tp, uint32_t slot, azd::f3 att,
                                          uint32_t digits) {
    uint32_t i = push_slot(&Q.counts[level]);
    if (i >= Q.cap_q) {
        Q.counts[AZ_COUNT_OVERFLOW] = 1;   // this wave is re-run with fewer samples
        return;
    }
    Q.o[buf][i] = make_float4(o.x, o.y, o.z, time);
    Q.d[buf][i] = make_float4(d.x, d.y, d.z, __uint_as_float(flags));
    Q.tp[buf][i] = make_float4(tp.x, tp.y, tp.z, __uint_as_float(slot));
    Q.att[buf][i] = make_float4(att.x, att.y, att.z, 0.0f);
    Q.digits[buf][i] = digits;
}

__device__ __forceinline__ void push_shadow(const WaveQueues &Q, uint32_t level, azd::f3 o, float time, azd::f3 d,
                                            float tmax, azd::f3 c, uint32_t slot, uint32_t kind, uint32_t light,
                                            uint32_t scene = 0u) {
    uint32_t i = push_slot(&Q.counts[AZ_COUNT_SHADOW + level]);
    if (i >= Q.cap_s) {
        Q.counts[AZ_COUNT_OVERFLOW] = 1;
        return;
    }
    Q.so[i] = make_float4(o.x, o.y, o.z, time);
    Q.sd[i] = make_float4(d.x, d.y, d.z, tmax);
    Q.sc[i] = make_float4(c.x, c.y, c.z, __uint_as_float(slot));
    Q.smeta[i] = shadow_meta(kind, scene, light);
}

// The shading kernel specialised for the scene's features (DevScene.features)
// and for guided scattering (Q.lobes set); defined in az_shade_kernel.cu.
void LaunchShade(int grid, const azd::DevScene &S, const CameraParams &cam, const WaveQueues &Q, uint64_t start,
                 uint32_t L, cudaStream_t st);

}  // namespace az
