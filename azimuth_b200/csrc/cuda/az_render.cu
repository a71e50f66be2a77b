// Wavefront path tracer reproducing azimuth's estimator (TraceRay,
// src/azimuth_main.cpp:966-1133) on the GPU.
//
// A camera sample in azimuth is a recursive tree: every non-emitting hit adds
// its direct light and ambient term and recurses into a diffuse scatter ray,
// a mirror ray and the dielectric refraction and reflection rays.  Here every
// tree node is one queue entry carrying the product of the weights above it
// ("throughput"); levels are processed breadth-first over a wave of samples:
//
//   camera  -> queue[1]                    (GetSampleCoord + GetRayForPixel)
//   per level L = 1 .. MaxRecursionDepth+1:
//     extend  queue[L]  -> hits            (RayEntityIntersection)
//     shade   hits      -> queue[L+1], shadow queue, per-sample sums
//     shadow  shadow queue -> per-sample sums (the visibility tests of CalculateLighting)
//   splat   per-sample sums -> film        (ComputeSampleWeight, box or Gaussian)
//
// The counter RNG is keyed by the tree node, so the order in which the GPU
// visits nodes does not change any random number: the result equals azimuth's
// own tree up to float summation order.  Child nodes whose weight is exactly
// zero (e.g. the scatter ray of a pure mirror) are not traced; azimuth traces
// them and multiplies their radiance by zero.
#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "az_internal.h"
#include "az_render.h"
#include "az_shade.cuh"
#include "az_wave.cuh"

namespace az {
namespace {

using namespace azd;

// GetSampleCoord + GetRayForPixel (src/azimuth_main.cpp:1135-1178) of camera
// sample s into wave slot i.
__device__ __forceinline__ void camera_node(const CameraParams &cam, const WaveQueues &Q, uint64_t s, uint64_t seed,
                                            uint32_t i) {
    uint32_t row, col, sx, sy;
    sample_of(cam, s, row, col, sx, sy);
    NodeRng rng;
    rng.init(seed, (row << 16) | col, (sy << 16) | sx, 0u, 0u);
    float cx = (float)col + (0.5f * cam.inv_sqrt + (float)sx * cam.inv_sqrt);
    float cy = (float)row + (0.5f * cam.inv_sqrt + (float)sy * cam.inv_sqrt);
    // the lens pair is drawn y first: GCC evaluates the two Random01()
    // arguments of Vec2(...) right to left in the oracle build
    float ly = rng.next() - 0.5f;
    float lx = rng.next() - 0.5f;
    lx *= cam.aperture;
    ly *= cam.aperture;
    f3 offx = cam.axx * lx, offy = cam.axy * ly;
    f3 dir = normalize(cam.base + cx * cam.stepx - cy * cam.stepy - offx - offy);
    f3 o = cam.pos + offx + offy;
    float time = rng.next();
    Q.o[1][i] = make_float4(o.x, o.y, o.z, time);
    Q.d[1][i] = make_float4(dir.x, dir.y, dir.z, __uint_as_float(cam.scene << PF_SCENE_SHIFT));
    Q.tp[1][i] = make_float4(1.0f, 1.0f, 1.0f, __uint_as_float(i));
    Q.att[1][i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    Q.digits[1][i] = 0u;
    Q.accum[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

__global__ void k_camera(CameraParams cam, WaveQueues Q, uint64_t wave_start, uint32_t n) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t seed = cam.seed;
    if (Q.wave) {
        wave_start = Q.wave[0];
        n = (uint32_t)Q.wave[1];
        seed = Q.wave[2];
        if (i == 0) Q.counts[1] = n;   // the level-1 queue is the wave itself
    }
    if (i >= n) return;
    camera_node(cam, Q, wave_start + i, seed, i);
}

// Camera samples of a tile wave: each block takes the next tile of the wave's
// work queue (`next`, zeroed before the launch) until the queue is empty.
__global__ void k_camera_tiles(const Tile *tiles, uint32_t ntiles, uint32_t *next, WaveQueues Q, uint2 *slot_map) {
    __shared__ uint32_t taken;
    for (;;) {
        if (threadIdx.x == 0) taken = atomicAdd(next, 1u);
        __syncthreads();
        const uint32_t t = taken;
        __syncthreads();   // every thread has read `taken` before it is overwritten
        if (t >= ntiles) return;
        const Tile T = tiles[t];
        const CameraParams &cam = Q.job_cams[T.job];
        for (uint32_t k = threadIdx.x; k < T.count; k += blockDim.x) {
            camera_node(cam, Q, (uint64_t)T.first + k, cam.seed, T.slot + k);
            slot_map[T.slot + k] = make_uint2(T.job, T.first + k);
        }
    }
}

// Persistent traversal kernels.  Each warp reserves rays of the level's queue
// in batches; a lane whose query has finished takes the next reserved ray at
// its next step, so no lane idles until its warp's slowest ray is done.
constexpr uint32_t kFetchBatch = 64;
constexpr uint32_t kLaneIdle = 0xFFFFFFFFu, kLaneDone = 0xFFFFFFFEu;

struct WarpFetch {
    uint32_t next = 0, end = 0;
    bool exhausted = false;

    // Hands the idle lanes of the warp new indices below n (kLaneDone when the
    // queue is exhausted).  Called by all 32 lanes.
    __device__ __forceinline__ bool refill(uint32_t *counter, uint32_t n, uint32_t &idx) {
        const uint32_t lane = threadIdx.x & 31u;
        const uint32_t idle = __ballot_sync(0xFFFFFFFFu, idx == kLaneIdle);
        if (!idle) return false;
        if (next >= end && !exhausted) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(counter, kFetchBatch);
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (base >= n) {
                exhausted = true;
            } else {
                next = base;
                end = min(base + kFetchBatch, n);
            }
        }
        const uint32_t avail = end - next;
        bool got = false;
        if (idx == kLaneIdle) {
            const uint32_t rank = __popc(idle & ((1u << lane) - 1u));
            if (rank < avail) {
                idx = next + rank;
                got = true;
            } else if (exhausted) {
                idx = kLaneDone;
            }
        }
        next += min(avail, (uint32_t)__popc(idle));
        return got;
    }
};

// Sort keys that group a level's queue by where its rays start: a 15-bit
// Morton code of the origin's cell in a 32^3 grid over the scene bounds, for
// extension rays the top 13 bits of it and the direction octant.  Entries past
// the queue's size get the largest key, so after a stable sort the first
// `size` indices are the queue's own.
__global__ void k_order_keys(DevScene S, WaveQueues Q, uint32_t level, int shadow, uint32_t cap, uint32_t *keys,
                             uint32_t *vals) {
    const uint32_t n = shadow ? min(Q.counts[AZ_COUNT_SHADOW + level], Q.cap_s) : min(Q.counts[level], Q.cap_q);
    const int buf = level & 1;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += gridDim.x * blockDim.x) {
        uint32_t key = 0xFFFFu;
        if (i < n) {
            const float4 o = shadow ? Q.so[i] : Q.o[buf][i];
            uint32_t c[3];
            const float p[3] = {o.x, o.y, o.z};
            for (int a = 0; a < 3; a++) {
                const float u = (p[a] - S.box_lo[a]) * S.box_scale[a] * 32.0f;
                c[a] = u > 0.0f ? min((uint32_t)u, 31u) : 0u;   // NaN and below the box: cell 0
            }
            uint32_t m = 0;
            for (int b = 4; b >= 0; b--)
                m = (m << 3) | (((c[0] >> b) & 1u) << 2) | (((c[1] >> b) & 1u) << 1) | ((c[2] >> b) & 1u);
            if (shadow) {
                key = m;
            } else {
                const float4 d = Q.d[buf][i];
                const uint32_t oct = (d.x < 0.0f ? 4u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 1u : 0u);
                key = ((m >> 2) << 3) | oct;
            }
        }
        keys[i] = key;
        vals[i] = i;
    }
}

// How a traversal kernel maps queries to threads:
//   MODE_LOOP     one query per thread at a time in a grid-stride loop, each
//                 thread running its query to the end in one loop
//   MODE_LOCKSTEP the same assignment, but the warp advances its 32 queries
//                 one traversal step at a time and reconverges after every
//                 step
//   MODE_FETCH    persistent warps: a lane takes the next query of the queue
//                 as soon as its own ends (batches of kFetchBatch per warp)
//   MODE_FETCHP   the same, with traversal steps that pop the stack first
//                 and visit the popped group in the same step (Tracer
//                 POP_FIRST), so lanes coming back from a pop join the
//                 warp's node visits instead of idling through them
//   MODE_STAGED   MODE_FETCHP with the node fetches of each step staged
//                 through shared memory by the whole warp (stage_nodes)
enum : int { MODE_LOOP = 0, MODE_LOCKSTEP = 1, MODE_FETCH = 2, MODE_FETCHP = 3, MODE_STAGED = 4 };

// WT: triangles by the watertight test (AZ_FLAG_WATERTIGHT) instead of azimuth's.
// MULTI: a tile wave of several scenes (persistent modes only): each query is
// traced in the scene its entry names (WaveQueues.scenes).
// SPH: the top-level sphere test inline (Tracer SPH).
template <int BLOCK, int MINB, int MODE, bool WT = false, bool MULTI = false, bool SPH = false>
__global__ void __launch_bounds__(BLOCK, MINB) k_extend(DevScene S, CameraParams cam, WaveQueues Q, uint32_t level) {
    const int buf = level & 1;
    const uint32_t n = min(Q.counts[level], Q.cap_q);
    uint32_t *cnt = cam.count_traversal ? Q.counts + AZ_COUNT_NODES : nullptr;
    uint32_t *err = Q.counts + AZ_COUNT_ERROR;
    if (MODE == MODE_LOCKSTEP) {
        Tracer<Q_CLOSEST, false, WT, SPH> T;
        uint2 stack[AZD_WSTACK];
        // warp-uniform loop bound: every lane of a warp sees the same base
        for (uint32_t base = blockIdx.x * BLOCK + (threadIdx.x & ~31u); base < n; base += gridDim.x * BLOCK) {
            const uint32_t k = base + (threadIdx.x & 31u);
            bool live = k < n;
            const uint32_t i = live && Q.eorder ? Q.eorder[k] : k;
            if (live) {
                const float4 o = Q.o[buf][i], d = Q.d[buf][i];
                Ray r;
                r.o = mk(o.x, o.y, o.z);
                r.d = mk(d.x, d.y, d.z);
                r.time = o.w;
                T.init(S, r, cam.cull != 0, cam.eps_isect, FLT_MAX, stack);
            }
            while (__any_sync(0xFFFFFFFFu, live)) {
                if (live && T.step(S, stack, err)) {
                    const Hit &h = T.best;
                    Q.hit[i] = make_uint4(__float_as_uint(h.t), __float_as_uint(h.tl), h.prim, h.ent);
                    T.flush_counts(cnt);
                    live = false;
                }
            }
        }
        return;
    }
    if (MODE == MODE_LOOP) {
        // one query per thread at a time, grid-stride over the queue
        for (uint32_t k = blockIdx.x * BLOCK + threadIdx.x; k < n; k += gridDim.x * BLOCK) {
            const uint32_t i = Q.eorder ? Q.eorder[k] : k;
            const float4 o = Q.o[buf][i], d = Q.d[buf][i];
            Ray r;
            r.o = mk(o.x, o.y, o.z);
            r.d = mk(d.x, d.y, d.z);
            r.time = o.w;
            Hit h;
            trace<Q_CLOSEST, WT>(S, r, cam.cull != 0, cam.eps_isect, FLT_MAX, h, cnt, err);
            Q.hit[i] = make_uint4(__float_as_uint(h.t), __float_as_uint(h.tl), h.prim, h.ent);
        }
        return;
    }
    uint32_t *fetch = Q.counts + AZ_COUNT_FETCH + level;
    constexpr bool STAGED = MODE == MODE_STAGED;
    static_assert(!(STAGED && MULTI), "staged fetching serves one scene");
    __shared__ uint4 s_stage[STAGED ? BLOCK / 32 * 160 : 1];
    Tracer<Q_CLOSEST, MODE == MODE_FETCHP || STAGED, WT, SPH> T;
    uint2 stack[AZD_WSTACK];
    WarpFetch wf;
    uint32_t idx = kLaneIdle, qi = 0;   // work item and its queue entry
    uint32_t si = 0;                    // MULTI: the entry's scene
    while (true) {
        if (wf.refill(fetch, n, idx)) {
            qi = Q.eorder ? Q.eorder[idx] : idx;
            const float4 o = Q.o[buf][qi], d = Q.d[buf][qi];
            Ray r;
            r.o = mk(o.x, o.y, o.z);
            r.d = mk(d.x, d.y, d.z);
            r.time = o.w;
            if (MULTI) si = (__float_as_uint(d.w) & PF_SCENE) >> PF_SCENE_SHIFT;
            T.init(MULTI ? Q.scenes[si] : S, r, cam.cull != 0, cam.eps_isect, FLT_MAX, stack);
        }
        if (__all_sync(0xFFFFFFFFu, idx == kLaneDone)) break;
        bool fin;
        if (STAGED) {
            const bool live = idx < n;
            uint32_t node = T.kNoNode;
            fin = live && T.begin(S, stack, err, node);
            uint4 w[5];
            stage_nodes(S.wnodes, node, s_stage + (threadIdx.x >> 5) * 160u, w);
            fin = live && (fin || T.finish(S, stack, err, node, w));
        } else {
            fin = idx < n && T.step(MULTI ? Q.scenes[si] : S, stack, err);
        }
        if (fin) {
            const Hit &h = T.best;
            Q.hit[qi] = make_uint4(__float_as_uint(h.t), __float_as_uint(h.tl), h.prim, h.ent);
            T.flush_counts(cnt);
            idx = kLaneIdle;
        }
    }
}

// Visibility of the queued light samples; unoccluded ones are added to their
// sample.  Entity lights: occluded unless the nearest hit is the light's
// entity, so the light's own nearest hit is found exactly first and the query
// looks for anything else before it.
// Visibility of the SHADOW_ENTITY_FULL queries of the shadow queue (entity
// lights too large for the two-phase test): one full nearest-hit query each,
// visible when the nearest hit is the light's entity (src/azimuth_main.cpp:694-712).
// Launched only for scenes that have such a light.
template <bool WT, bool MULTI = false>
__global__ void __launch_bounds__(128) k_shadow_full(DevScene S0, CameraParams cam, WaveQueues Q, uint32_t level) {
    const uint32_t n = min(Q.counts[AZ_COUNT_SHADOW + level], Q.cap_s);
    uint32_t *cnt = cam.count_traversal ? Q.counts + AZ_COUNT_SNODES : nullptr;
    uint32_t *err = Q.counts + AZ_COUNT_ERROR;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t meta = Q.smeta[i];
        if (shadow_kind(meta) != SHADOW_ENTITY_FULL) continue;
        const DevScene &S = MULTI ? Q.scenes[shadow_scene(meta)] : S0;
        const float4 o = Q.so[i], d = Q.sd[i], c = Q.sc[i];
        const DevLight &L = S.lights[shadow_light(meta)];
        Ray r;
        r.o = mk(o.x, o.y, o.z);
        r.d = mk(d.x, d.y, d.z);
        r.time = o.w;
        Hit h;
        const bool any = trace<Q_CLOSEST, WT>(S, r, false, 0.0f, FLT_MAX, h, cnt, err);
        if (!any || S.ents[h.ent].uid == L.uid) add_accum(Q.accum, __float_as_uint(c.w), mk(c.x, c.y, c.z));
    }
}

template <int BLOCK, int MINB, int MODE, bool WT = false, bool MULTI = false, bool SPH = false>
__global__ void __launch_bounds__(BLOCK, MINB) k_shadow(DevScene S, CameraParams cam, WaveQueues Q, uint32_t level) {
    const uint32_t n = min(Q.counts[AZ_COUNT_SHADOW + level], Q.cap_s);
    uint32_t *cnt = cam.count_traversal ? Q.counts + AZ_COUNT_SNODES : nullptr;
    uint32_t *err = Q.counts + AZ_COUNT_ERROR;
    if (MODE == MODE_LOCKSTEP) {
        Tracer<Q_ANY, false, WT, SPH> T;
        uint2 stack[AZD_WSTACK];
        for (uint32_t base = blockIdx.x * BLOCK + (threadIdx.x & ~31u); base < n; base += gridDim.x * BLOCK) {
            const uint32_t k = base + (threadIdx.x & 31u);
            bool live = k < n;
            const uint32_t i = live && Q.sorder ? Q.sorder[k] : k;
            float4 c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            if (live) {
                const float4 o = Q.so[i], d = Q.sd[i];
                c = Q.sc[i];
                const uint32_t meta = Q.smeta[i];
                const uint32_t kind = shadow_kind(meta), li = shadow_light(meta);
                Ray r;
                r.o = mk(o.x, o.y, o.z);
                r.d = mk(d.x, d.y, d.z);
                r.time = o.w;
                if (kind == SHADOW_ENTITY_FULL) {
                    live = false;   // k_shadow_full
                } else if (kind == SHADOW_ENTITY) {
                    const LightHit lh = light_entity_hit_call(S.ents, S.light_tris, S.lights + li, r);
                    T.init(S, r, false, 0.0f, lh.hit ? lh.t : FLT_MAX, stack, S.lights[li].ent_index);
                } else {
                    T.init(S, r, false, 0.0f, kind == SHADOW_ANY ? FLT_MAX : d.w, stack);
                }
            }
            while (__any_sync(0xFFFFFFFFu, live)) {
                if (live && T.step(S, stack, err)) {
                    if (!T.hit_any) add_accum(Q.accum, __float_as_uint(c.w), mk(c.x, c.y, c.z));
                    T.flush_counts(cnt);
                    live = false;
                }
            }
        }
        return;
    }
    if (MODE == MODE_LOOP) {
        for (uint32_t k = blockIdx.x * BLOCK + threadIdx.x; k < n; k += gridDim.x * BLOCK) {
            const uint32_t i = Q.sorder ? Q.sorder[k] : k;
            const float4 o = Q.so[i], d = Q.sd[i], c = Q.sc[i];
            const uint32_t meta = Q.smeta[i];
            const uint32_t kind = shadow_kind(meta), li = shadow_light(meta);
            Ray r;
            r.o = mk(o.x, o.y, o.z);
            r.d = mk(d.x, d.y, d.z);
            r.time = o.w;
            Hit h;
            bool visible;
            if (kind == SHADOW_ENTITY_FULL) {
                continue;   // k_shadow_full
            } else if (kind == SHADOW_ENTITY) {
                const LightHit lh = light_entity_hit_call(S.ents, S.light_tris, S.lights + li, r);
                visible = !trace<Q_ANY, WT>(S, r, false, 0.0f, lh.hit ? lh.t : FLT_MAX, h, cnt, err,
                                            S.lights[li].ent_index);
            } else {
                visible = !trace<Q_ANY, WT>(S, r, false, 0.0f, kind == SHADOW_ANY ? FLT_MAX : d.w, h, cnt, err);
            }
            if (visible) add_accum(Q.accum, __float_as_uint(c.w), mk(c.x, c.y, c.z));
        }
        return;
    }
    uint32_t *fetch = Q.counts + AZ_COUNT_FETCH + AZ_MAX_LEVELS + level;
    constexpr bool STAGED = MODE == MODE_STAGED;
    static_assert(!(STAGED && MULTI), "staged fetching serves one scene");
    __shared__ uint4 s_stage[STAGED ? BLOCK / 32 * 160 : 1];
    Tracer<Q_ANY, MODE == MODE_FETCHP || STAGED, WT, SPH> T;
    uint2 stack[AZD_WSTACK];
    WarpFetch wf;
    uint32_t idx = kLaneIdle;
    uint32_t si = 0;   // MULTI: the entry's scene
    float4 c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    while (true) {
        if (wf.refill(fetch, n, idx)) {
            const uint32_t qi = Q.sorder ? Q.sorder[idx] : idx;
            const float4 o = Q.so[qi], d = Q.sd[qi];
            c = Q.sc[qi];
            const uint32_t meta = Q.smeta[qi];
            const uint32_t kind = shadow_kind(meta), li = shadow_light(meta);
            if (MULTI) si = shadow_scene(meta);
            const DevScene &Sq = MULTI ? Q.scenes[si] : S;
            Ray r;
            r.o = mk(o.x, o.y, o.z);
            r.d = mk(d.x, d.y, d.z);
            r.time = o.w;
            if (kind == SHADOW_ENTITY_FULL) {
                idx = kLaneIdle;   // k_shadow_full
            } else if (kind == SHADOW_ENTITY) {
                const LightHit lh = light_entity_hit_call(Sq.ents, Sq.light_tris, Sq.lights + li, r);
                T.init(Sq, r, false, 0.0f, lh.hit ? lh.t : FLT_MAX, stack, Sq.lights[li].ent_index);
            } else {
                T.init(Sq, r, false, 0.0f, kind == SHADOW_ANY ? FLT_MAX : d.w, stack);
            }
        }
        if (__all_sync(0xFFFFFFFFu, idx == kLaneDone)) break;
        bool fin;
        if (STAGED) {
            const bool live = idx < n;
            uint32_t node = T.kNoNode;
            fin = live && T.begin(S, stack, err, node);
            uint4 w[5];
            stage_nodes(S.wnodes, node, s_stage + (threadIdx.x >> 5) * 160u, w);
            fin = live && (fin || T.finish(S, stack, err, node, w));
        } else {
            fin = idx < n && T.step(MULTI ? Q.scenes[si] : S, stack, err);
        }
        if (fin) {
            if (!T.hit_any) add_accum(Q.accum, __float_as_uint(c.w), mk(c.x, c.y, c.z));
            T.flush_counts(cnt);
            idx = kLaneIdle;
        }
    }
}

// ComputeSampleWeight (src/azimuth_main.cpp:1209-1254) for every sample of the wave.
// ComputeSampleWeight (src/azimuth_main.cpp:1209-1254): sample s's sum `a`
// into the film, box or Gaussian footprint.
__device__ __forceinline__ void splat_sample(const CameraParams &cam, az_pixel *film, uint64_t s, float4 a) {
    uint32_t row, col, sx, sy;
    sample_of(cam, s, row, col, sx, sy);
    float4 *f = reinterpret_cast<float4 *>(film);
    if (cam.filter == AZ_Filter_Box) {
        atomicAdd(&f[(size_t)row * cam.width + col], make_float4(a.x, a.y, a.z, 1.0f));
        return;
    }
    float cx = (float)col + (0.5f * cam.inv_sqrt + (float)sx * cam.inv_sqrt);
    float cy = (float)row + (0.5f * cam.inv_sqrt + (float)sy * cam.inv_sqrt);
    int32_t w1 = (int32_t)cam.width - 1, h1 = (int32_t)cam.height - 1;
    int32_t x0 = max((int32_t)col - cam.gk, 0), x1 = min((int32_t)col + cam.gk, w1);
    int32_t y0 = max((int32_t)row - cam.gk, 0), y1 = min((int32_t)row + cam.gk, h1);
    for (int32_t gy = y0; gy <= y1; gy++)
        for (int32_t gx = x0; gx <= x1; gx++) {
            float dx = cx - ((float)gx + 0.5f), dy = cy - ((float)gy + 0.5f);
            float d2 = dx * dx + dy * dy;
            float g = cam.g_norm * expf(cam.g_neg * d2);
            atomicAdd(&f[(size_t)gy * cam.width + gx], make_float4(a.x * g, a.y * g, a.z * g, g));
        }
}

__global__ void k_splat(CameraParams cam, WaveQueues Q, uint64_t wave_start, uint32_t n, az_pixel *film) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (Q.wave) {
        wave_start = Q.wave[0];
        n = (uint32_t)Q.wave[1];
    }
    if (i >= n) return;
    if (Q.counts[AZ_COUNT_OVERFLOW]) return;   // the wave is re-run
    if (cam.sample_out) {
        cam.sample_out[wave_start + i] = Q.accum[i];
        return;
    }
    splat_sample(cam, film, wave_start + i, Q.accum[i]);
}

// The samples of a tile wave, each into its own job's film.
__global__ void k_splat_tiles(WaveQueues Q, uint32_t n, az_pixel *const *films) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (Q.counts[AZ_COUNT_OVERFLOW]) return;   // the wave is re-run
    const uint2 js = Q.slot_map[i];
    splat_sample(Q.job_cams[js.x], films[js.x], js.y, Q.accum[i]);
}

// Launch configurations of the two traversal kernels: threads per block,
// minimum resident blocks per SM (which caps registers), and whether warps
// fetch rays persistently (a lane takes a new ray as soon as its query ends)
// or one query per thread in a grid-stride loop; chosen per scene by
// az_gpu_autotune.
struct Variant {
    int block, minb, mode;
};
constexpr Variant kVariants[] = {{128, 1, MODE_LOOP},     {128, 6, MODE_LOOP},     {128, 8, MODE_LOOP},
                                 {256, 1, MODE_LOOP},     {256, 3, MODE_LOOP},     {64, 1, MODE_LOOP},
                                 {64, 12, MODE_LOOP},     {128, 8, MODE_FETCH},    {128, 6, MODE_FETCH},
                                 {256, 3, MODE_FETCH},    {128, 8, MODE_LOCKSTEP}, {128, 6, MODE_LOCKSTEP},
                                 {256, 3, MODE_LOCKSTEP}, {64, 12, MODE_LOCKSTEP}, {128, 7, MODE_FETCH},
                                 {128, 6, MODE_FETCHP},   {128, 7, MODE_FETCHP},   {128, 8, MODE_FETCHP},
                                 {128, 6, MODE_STAGED},   {128, 8, MODE_STAGED}};
constexpr uint32_t kVariantCount = sizeof(kVariants) / sizeof(kVariants[0]);
static_assert(kVariantCount == AZ_LAUNCH_VARIANTS, "variant table and header disagree");

// Scenes with spheres at the top level get the kernels with the sphere test
// inline (a one-thread-per-query loop always has it inline).
template <int B, int M, int P>
void LaunchTraversal(bool shadow, int sms, const DevScene &S, const CameraParams &cam, const WaveQueues &Q,
                     uint32_t L, cudaStream_t st) {
    const int grid = sms * (2048 / B);
    if (P != MODE_LOOP && S.top_spheres) {
        if (shadow) k_shadow<B, M, P, false, false, true><<<grid, B, 0, st>>>(S, cam, Q, L);
        else k_extend<B, M, P, false, false, true><<<grid, B, 0, st>>>(S, cam, Q, L);
        return;
    }
    if (shadow) k_shadow<B, M, P><<<grid, B, 0, st>>>(S, cam, Q, L);
    else k_extend<B, M, P><<<grid, B, 0, st>>>(S, cam, Q, L);
}

void LaunchTraversalVariant(uint32_t v, bool shadow, int sms, const DevScene &S, const CameraParams &cam,
                            const WaveQueues &Q, uint32_t L, cudaStream_t st) {
    const int fgrid = sms * 16;
    if (Q.scenes) {
        // a tile wave of several scenes: one launch configuration, 128 threads, at most 64 registers,
        // persistent fetching (variant 8), the sphere test inline when any scene has top-level spheres
        if (cam.watertight) {
            if (shadow && S.full_light_queries) k_shadow_full<true, true><<<fgrid, 128, 0, st>>>(S, cam, Q, L);
            if (shadow) k_shadow<128, 8, MODE_FETCH, true, true><<<fgrid, 128, 0, st>>>(S, cam, Q, L);
            else k_extend<128, 8, MODE_FETCH, true, true><<<fgrid, 128, 0, st>>>(S, cam, Q, L);
        } else {
            if (shadow && S.full_light_queries) k_shadow_full<false, true><<<fgrid, 128, 0, st>>>(S, cam, Q, L);
            if (S.top_spheres) {
                if (shadow) k_shadow<128, 8, MODE_FETCH, false, true, true><<<fgrid, 128, 0, st>>>(S, cam, Q, L);
                else k_extend<128, 8, MODE_FETCH, false, true, true><<<fgrid, 128, 0, st>>>(S, cam, Q, L);
            } else {
                if (shadow) k_shadow<128, 8, MODE_FETCH, false, true><<<fgrid, 128, 0, st>>>(S, cam, Q, L);
                else k_extend<128, 8, MODE_FETCH, false, true><<<fgrid, 128, 0, st>>>(S, cam, Q, L);
            }
        }
        return;
    }
    if (cam.watertight) {
        // the watertight test has one launch configuration: 128 threads, pop-first persistent fetching
        if (shadow && S.full_light_queries) k_shadow_full<true><<<fgrid, 128, 0, st>>>(S, cam, Q, L);
        if (shadow) k_shadow<128, 6, MODE_FETCHP, true><<<fgrid, 128, 0, st>>>(S, cam, Q, L);
        else k_extend<128, 6, MODE_FETCHP, true><<<fgrid, 128, 0, st>>>(S, cam, Q, L);
        return;
    }
    if (shadow && S.full_light_queries) k_shadow_full<false><<<fgrid, 128, 0, st>>>(S, cam, Q, L);
    switch (v) {
        case 0: LaunchTraversal<128, 1, MODE_LOOP>(shadow, sms, S, cam, Q, L, st); break;
        case 1: LaunchTraversal<128, 6, MODE_LOOP>(shadow, sms, S, cam, Q, L, st); break;
        case 3: LaunchTraversal<256, 1, MODE_LOOP>(shadow, sms, S, cam, Q, L, st); break;
        case 4: LaunchTraversal<256, 3, MODE_LOOP>(shadow, sms, S, cam, Q, L, st); break;
        case 5: LaunchTraversal<64, 1, MODE_LOOP>(shadow, sms, S, cam, Q, L, st); break;
        case 6: LaunchTraversal<64, 12, MODE_LOOP>(shadow, sms, S, cam, Q, L, st); break;
        case 7: LaunchTraversal<128, 8, MODE_FETCH>(shadow, sms, S, cam, Q, L, st); break;
        case 8: LaunchTraversal<128, 6, MODE_FETCH>(shadow, sms, S, cam, Q, L, st); break;
        case 9: LaunchTraversal<256, 3, MODE_FETCH>(shadow, sms, S, cam, Q, L, st); break;
        case 10: LaunchTraversal<128, 8, MODE_LOCKSTEP>(shadow, sms, S, cam, Q, L, st); break;
        case 11: LaunchTraversal<128, 6, MODE_LOCKSTEP>(shadow, sms, S, cam, Q, L, st); break;
        case 12: LaunchTraversal<256, 3, MODE_LOCKSTEP>(shadow, sms, S, cam, Q, L, st); break;
        case 13: LaunchTraversal<64, 12, MODE_LOCKSTEP>(shadow, sms, S, cam, Q, L, st); break;
        case 14: LaunchTraversal<128, 7, MODE_FETCH>(shadow, sms, S, cam, Q, L, st); break;
        case 15: LaunchTraversal<128, 6, MODE_FETCHP>(shadow, sms, S, cam, Q, L, st); break;
        case 16: LaunchTraversal<128, 7, MODE_FETCHP>(shadow, sms, S, cam, Q, L, st); break;
        case 17: LaunchTraversal<128, 8, MODE_FETCHP>(shadow, sms, S, cam, Q, L, st); break;
        case 18: LaunchTraversal<128, 6, MODE_STAGED>(shadow, sms, S, cam, Q, L, st); break;
        case 19: LaunchTraversal<128, 8, MODE_STAGED>(shadow, sms, S, cam, Q, L, st); break;
        default: LaunchTraversal<128, 8, MODE_LOOP>(shadow, sms, S, cam, Q, L, st); break;
    }
}

}  // namespace

// Camera basis and pixel steps of ProduceImageInLinearSpace
// (src/azimuth_main.cpp:1265-1347), evaluated on the host in float.
int SetupCamera(const az_camera *c, az_scissor sc, int32_t filter, uint32_t cull, const az_epsilon_values *eps,
                uint64_t seed, CameraParams &cam) {
    using azd::f3;
    auto v = [](const az_vec3 &a) { return azd::mk(a.x, a.y, a.z); };
    if (c->Resolution.x == 0 || c->Resolution.y == 0 || c->Resolution.x > 65535 || c->Resolution.y > 65535)
        return SetError(AZ_ERR_INVALID_ARGUMENT, "camera resolution must be 1..65535 per axis");
    f3 gaze = v(c->Gaze);
    if (c->GazeIsPoint) gaze = v(c->Gaze) - v(c->Position);
    f3 gn = azd::normalize(gaze);
    f3 az = -gn, ax, ay;
    if (c->IsLeftHanded) {
        ax = azd::normalize(azd::cross(azd::normalize(v(c->Up)), gn));
        ay = azd::cross(ax, az);
    } else {
        ax = azd::normalize(azd::cross(gn, azd::normalize(v(c->Up))));
        ay = azd::cross(az, ax);
    }
    float fdn = 1.0f;
    if (c->FocusDistance != 0.0f) fdn = c->FocusDistance / c->NearDistance;
    memset(&cam, 0, sizeof(cam));
    cam.width = c->Resolution.x;
    cam.height = c->Resolution.y;
    az_vec4 np = c->NearPlane;   // r, l, b, t
    if (c->Type == AZ_Camera_Simple) {
        float hh = c->NearDistance * tanf((c->FovY / 2.0f / 180.0f) * (float)3.14159265359);
        float ar = (float)cam.width / (float)cam.height;
        float wh = ar * hh;
        np.w = +hh;
        np.z = -hh;
        np.x = +wh;
        np.y = -wh;
    }
    float psx = (np.x - np.y) / (float)cam.width, psy = (np.w - np.z) / (float)cam.height;
    cam.stepx = ax * psx * fdn;
    cam.stepy = ay * psy * fdn;
    f3 tl = v(c->Position) + c->NearDistance * gn + np.y * ax + np.w * ay;
    cam.base = (tl - v(c->Position)) * fdn;
    cam.pos = v(c->Position);
    cam.axx = ax;
    cam.axy = ay;
    cam.aperture = c->ApertureSize;
    cam.sqrt_spp = (uint32_t)sqrtf((float)c->SampleCount);
    cam.inv_sqrt = 1.0f / cam.sqrt_spp;
    float gr = 1.5f, sigma = gr / 3.0f, two = 2.0f * (sigma * sigma);
    cam.g_neg = -1.0f / two;
    cam.g_norm = 1.0f / (two * (float)3.14159265359);
    cam.gk = (int32_t)ceilf(gr - 0.5f);
    uint32_t r1 = std::min(sc.Max.y, cam.height), c1 = std::min(sc.Max.x, cam.width);
    cam.r0 = sc.Min.y;
    cam.c0 = sc.Min.x;
    cam.hsc = r1 > cam.r0 ? r1 - cam.r0 : 0;
    cam.wsc = c1 > cam.c0 ? c1 - cam.c0 : 0;
    cam.npix = (uint64_t)cam.hsc * cam.wsc;
    if (filter != AZ_Filter_Box && filter != AZ_Filter_Gaussian) return SetError(AZ_ERR_INVALID_ARGUMENT, "unknown filter");
    cam.filter = filter;
    cam.seed = seed;
    cam.eps_isect = eps ? eps->Intersection : 0.0f;
    cam.eps_shadow = eps ? eps->ShadowRay : 0.000275f;
    cam.cull = cull;
    return AZ_OK;
}

WaveBuffers::~WaveBuffers() {
    DropGraph();
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (wave_host) cudaFreeHost(wave_host);
    if (guide_lobes) cudaFree(guide_lobes);
    if (guide_rec) cudaFree(guide_rec);
    for (void *p : {(void *)okey[0], (void *)okey[1], (void *)oval, (void *)oidx_e, (void *)oidx_s, otemp})
        if (p) cudaFree(p);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (side) cudaStreamDestroy(side);
}

int WaveBuffers::EnsureSide() {
    if (side) return AZ_OK;
    // non-blocking: the side stream only ever runs after waiting on an event
    // of the render stream, which orders it after the caller's earlier work
    cudaStream_t s = nullptr;
    cudaEvent_t f = nullptr, j = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&f, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&j, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        if (f) cudaEventDestroy(f);
        if (s) cudaStreamDestroy(s);
        return CudaError(e, "creating the wave's side stream");
    }
    side = s;
    ev_fork = f;
    ev_join = j;
    return AZ_OK;
}

int WaveBuffers::EnsureOrder(uint32_t cap) {
    if (cap <= ocap && otemp) return AZ_OK;
    DropGraph();   // it refers to the buffers replaced below
    for (uint32_t **p : {&okey[0], &okey[1], &oval, &oidx_e, &oidx_s}) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    if (otemp) cudaFree(otemp);
    otemp = nullptr;
    ocap = 0;
    for (uint32_t **p : {&okey[0], &okey[1], &oval, &oidx_e, &oidx_s})
        if (cudaMalloc((void **)p, (size_t)cap * sizeof(uint32_t)) != cudaSuccess) {
            *p = nullptr;
            return SetError(AZ_ERR_OUT_OF_MEMORY, "queue ordering buffers");
        }
    size_t bytes = 0;
    AZ_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, bytes, okey[0], okey[1], oval, oidx_e, (int)cap, 0, 16));
    if (cudaMalloc(&otemp, bytes) != cudaSuccess) {
        otemp = nullptr;
        return SetError(AZ_ERR_OUT_OF_MEMORY, "queue ordering scratch");
    }
    otemp_bytes = bytes;
    ocap = cap;
    return AZ_OK;
}

void WaveBuffers::DropGraph() {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
    graph_key.clear();
}

int WaveBuffers::Ensure(uint32_t chunk, uint32_t cap_q, uint32_t cap_s) {
    if (chunk <= this->chunk && cap_q <= q.cap_q && cap_s <= q.cap_s && !ptrs.empty()) return AZ_OK;
    DropGraph();   // it refers to the buffers freed below
    for (void *p : ptrs)
        if (p) cudaFree(p);
    ptrs.clear();
    memset(&q, 0, sizeof(q));
    auto alloc = [&](size_t bytes) -> void * {
        void *p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return p;
    };
    for (int b = 0; b < 2; b++) {
        q.o[b] = (float4 *)alloc((size_t)cap_q * sizeof(float4));
        q.d[b] = (float4 *)alloc((size_t)cap_q * sizeof(float4));
        q.tp[b] = (float4 *)alloc((size_t)cap_q * sizeof(float4));
        q.att[b] = (float4 *)alloc((size_t)cap_q * sizeof(float4));
        q.digits[b] = (uint32_t *)alloc((size_t)cap_q * sizeof(uint32_t));
        if (!q.o[b] || !q.d[b] || !q.tp[b] || !q.att[b] || !q.digits[b]) return SetError(AZ_ERR_OUT_OF_MEMORY, "wave queues");
    }
    q.hit = (uint4 *)alloc((size_t)cap_q * sizeof(uint4));
    q.so = (float4 *)alloc((size_t)cap_s * sizeof(float4));
    q.sd = (float4 *)alloc((size_t)cap_s * sizeof(float4));
    q.sc = (float4 *)alloc((size_t)cap_s * sizeof(float4));
    q.smeta = (uint32_t *)alloc((size_t)cap_s * sizeof(uint32_t));
    q.accum = (float4 *)alloc((size_t)chunk * sizeof(float4));
    q.counts = (uint32_t *)alloc(AZ_COUNT_TOTAL * sizeof(uint32_t));
    wave_dev = (uint64_t *)alloc(4 * sizeof(uint64_t));
    if (!q.hit || !q.so || !q.sd || !q.sc || !q.smeta || !q.accum || !q.counts || !wave_dev)
        return SetError(AZ_ERR_OUT_OF_MEMORY, "wave queues");
    if (!wave_host && cudaMallocHost((void **)&wave_host, 4 * sizeof(uint64_t)) != cudaSuccess) {
        wave_host = nullptr;
        return SetError(AZ_ERR_OUT_OF_MEMORY, "wave descriptor");
    }
    q.cap_q = cap_q;
    q.cap_s = cap_s;
    this->chunk = chunk;
    return AZ_OK;
}

// CUDA events between the stages of every level; summed per stage.
struct StageTimer {
    std::vector<cudaEvent_t> ev;
    std::vector<int> kind;   // event k ends stage kind[k]-1 when kind[k] > 0
    float ms[3] = {0, 0, 0};
    void Mark(cudaStream_t st, int k) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, st);
        ev.push_back(e);
        kind.push_back(k);
    }
    void Collect() {   // after a stream synchronize
        for (size_t i = 1; i < ev.size(); i++) {
            if (kind[i] >= 1 && kind[i - 1] == kind[i] - 1) {
                float t = 0.0f;
                cudaEventElapsedTime(&t, ev[i - 1], ev[i]);
                ms[kind[i] - 1] += t;
            }
        }
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
        ev.clear();
        kind.clear();
    }
    ~StageTimer() {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
};

// Renders samples [start, start+n) of the scissor into `film`; returns the
// per-wave counters (path and shadow queue sizes per level, overflow flag).
// Launches of one wave.  With `capture`, the launches read the wave's first
// sample, size and seed from W.wave_dev (set before every replay of the
// captured graph) and size their grids for `n` = the largest wave.
// Sorts the extension (shadow = 0) or shadow queue of `level` by origin cell
// into its visiting order (k_order_keys + a 16-bit radix sort).
static int OrderQueue(const GpuScene &G, const WaveQueues &Q, WaveBuffers &W, uint32_t level, int shadow, int sms,
                      cudaStream_t st, RenderCounters &rc) {
    const uint32_t cap = shadow ? Q.cap_s : Q.cap_q;
    k_order_keys<<<sms * 8, 256, 0, st>>>(G.dev, Q, level, shadow, cap, W.okey[0], W.oval);
    rc.launches++;
    AZ_CUDA_TRY(cub::DeviceRadixSort::SortPairs(W.otemp, W.otemp_bytes, W.okey[0], W.okey[1], W.oval,
                                                shadow ? W.oidx_s : W.oidx_e, (int)cap, 0, 16, st));
    return AZ_OK;
}

// The device side of a tile wave (az_gpu_render_tiles): the wave's tiles, the
// counter its camera kernel pulls them with, and the jobs' cameras and films.
struct TileWave {
    const Tile *tiles;
    uint32_t ntiles;
    uint32_t *next;
    uint2 *slot_map;
    const CameraParams *cams;
    az_pixel *const *films;
    const DevScene *scenes;   // jobs of several scenes: their device records (null: one scene)
    const DevScene *dev;      // and the host record the launches are chosen for (null: the scene's own)
};

static int RenderWave(const GpuScene &G, const CameraParams &cam, WaveBuffers &W, uint64_t start, uint32_t n,
                      az_pixel *film, cudaStream_t st, int sms, RenderCounters &rc, StageTimer *timer,
                      GuideState *guide, bool train, bool capture = false, const TileWave *tw = nullptr) {
    WaveQueues Q = W.q;
    if (tw) {
        Q.slot_map = tw->slot_map;
        Q.job_cams = tw->cams;
        Q.scenes = tw->scenes;
    }
    // the scene the launches are chosen for: a tile wave of several scenes
    // passes one whose features, depth and light kinds cover all of them
    const DevScene &D = tw && tw->dev ? *tw->dev : G.dev;
    if (capture) Q.wave = W.wave_dev;
    if (cam.order & kOrderExtend) Q.eorder = W.oidx_e;
    if (cam.order & kOrderShadow) Q.sorder = W.oidx_s;
    // While the guide trains, its early proposals can be far from the light
    // field; capping the chance of sampling them at one half keeps every
    // sample's weight within twice cosine sampling's (the estimate stays
    // unbiased for any cap).  Inference-only renders use the learned value.
    Q.guide_alpha_max = train ? 0.5f : 1.0f;
    const uint32_t levels = std::min<uint32_t>(D.max_depth + 1, AZ_MAX_LEVELS - 2);
    if (guide) {
        // proposals for every queue entry this wave can hold (the queue is capped to match)
        int grc = GuidePrepareWave(*guide, W, Q, std::min<uint32_t>(Q.cap_q, n + n / 2 + 1024), train ? levels : 0u, st);
        if (grc != AZ_OK) return grc;
    }
    AZ_CUDA_TRY(cudaMemsetAsync(Q.counts, 0, AZ_COUNT_TOTAL * sizeof(uint32_t), st));
    if (!capture) {
        uint32_t first = n;
        AZ_CUDA_TRY(cudaMemcpyAsync(Q.counts + 1, &first, sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    }
    if (tw) {
        AZ_CUDA_TRY(cudaMemsetAsync(tw->next, 0, sizeof(uint32_t), st));
        k_camera_tiles<<<std::min<uint32_t>(tw->ntiles, (uint32_t)sms * 8), 256, 0, st>>>(tw->tiles, tw->ntiles,
                                                                                          tw->next, Q, tw->slot_map);
    } else {
        k_camera<<<(n + 255) / 256, 256, 0, st>>>(cam, Q, start, n);
    }
    rc.launches++;
    const int grid = sms * 16;
    const uint32_t v = cam.variant;
    // Level L's visibility queries need only its shading; level L+1's
    // closest-hit queries need the same.  Run them side by side (visibility
    // on the side stream) so that the tail of one fills with the other's work;
    // the next shading waits for both.  Not with stage timing, nor with queue
    // ordering (both orderings share one sort scratch).
    const bool overlap = W.side && !timer && !cam.order && !cam.serial_levels;
    if (overlap) {
        LaunchTraversalVariant(v, false, sms, D, cam, Q, 1, st);
        for (uint32_t L = 1; L <= levels; L++) {
            if (guide && L + 1 <= D.max_depth + 1) {   // the deepest level spawns nothing to guide
                int grc = GuideInfer(*guide, G, Q, L, st);
                if (grc != AZ_OK) return grc;
                rc.launches++;
            }
            LaunchShade(grid, D, cam, Q, start, L, st);
            AZ_CUDA_TRY(cudaEventRecord(W.ev_fork, st));
            AZ_CUDA_TRY(cudaStreamWaitEvent(W.side, W.ev_fork, 0));
            LaunchTraversalVariant(cam.shadow_variant, true, sms, D, cam, Q, L, W.side);
            AZ_CUDA_TRY(cudaEventRecord(W.ev_join, W.side));
            if (L < levels) LaunchTraversalVariant(v, false, sms, D, cam, Q, L + 1, st);
            AZ_CUDA_TRY(cudaStreamWaitEvent(st, W.ev_join, 0));
            rc.launches += D.full_light_queries ? 4 : 3;
            rc.extend_launches++;
        }
    }
    for (uint32_t L = 1; L <= levels && !overlap; L++) {
        if (timer) timer->Mark(st, 0);
        if (cam.order & kOrderExtend) {
            int orc = OrderQueue(G, Q, W, L, 0, sms, st, rc);
            if (orc != AZ_OK) return orc;
        }
        LaunchTraversalVariant(v, false, sms, D, cam, Q, L, st);
        if (guide && L + 1 <= D.max_depth + 1) {   // the deepest level spawns nothing to guide
            int grc = GuideInfer(*guide, G, Q, L, st);
            if (grc != AZ_OK) return grc;
            rc.launches++;
        }
        if (timer) timer->Mark(st, 1);
        LaunchShade(grid, D, cam, Q, start, L, st);
        if (timer) timer->Mark(st, 2);
        if (cam.order & kOrderShadow) {
            int orc = OrderQueue(G, Q, W, L, 1, sms, st, rc);
            if (orc != AZ_OK) return orc;
        }
        LaunchTraversalVariant(cam.shadow_variant, true, sms, D, cam, Q, L, st);
        if (timer) timer->Mark(st, 3);
        rc.launches += D.full_light_queries ? 4 : 3;
        rc.extend_launches++;
    }
    if (guide && train) {
        int grc = GuideTrainWave(*guide, Q, st);
        if (grc != AZ_OK) return grc;
        rc.launches += 7;
    }
    if (tw) k_splat_tiles<<<(n + 255) / 256, 256, 0, st>>>(Q, n, tw->films);
    else k_splat<<<(n + 255) / 256, 256, 0, st>>>(cam, Q, start, n, film);
    rc.launches++;
    AZ_CUDA_TRY(cudaGetLastError());
    return AZ_OK;
}

// One wave through the captured graph of W (capturing it first when the
// scene, camera, film, launch configuration or largest wave changed).
static int ReplayWave(const GpuScene &G, const CameraParams &cam, WaveBuffers &W, uint64_t start, uint32_t n,
                      uint32_t n_max, az_pixel *film, cudaStream_t st, int sms, RenderCounters &rc) {
    struct Key {
        const GpuScene *g;
        az_pixel *film;
        CameraParams cam;
        uint32_t n_max, cap_q, cap_s;
        int sms;
        const void *q0;
    } key;
    memset(&key, 0, sizeof(key));
    key.g = &G;
    key.film = film;
    key.cam = cam;
    key.cam.seed = 0;   // read from the descriptor
    key.n_max = n_max;
    key.cap_q = W.q.cap_q;
    key.cap_s = W.q.cap_s;
    key.sms = sms;
    key.q0 = W.q.o[0];
    const unsigned char *kb = reinterpret_cast<const unsigned char *>(&key);
    RenderCounters launches{};
    if (!W.graph || W.graph_key.size() != sizeof(key) || memcmp(W.graph_key.data(), kb, sizeof(key)) != 0) {
        W.DropGraph();
        AZ_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int crc = RenderWave(G, cam, W, 0, n_max, film, st, sms, launches, nullptr, nullptr, false, true);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(st, &graph);
        if (crc != AZ_OK) {
            if (graph) cudaGraphDestroy(graph);
            return crc;
        }
        if (e != cudaSuccess) return CudaError(e, "capturing the wave launches");
        e = cudaGraphInstantiate(&W.graph, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            W.graph = nullptr;
            return CudaError(e, "instantiating the wave graph");
        }
        W.graph_key.assign(kb, kb + sizeof(key));
        W.graph_launches = launches.launches;
        W.graph_extend_launches = launches.extend_launches;
    }
    W.wave_host[0] = start;
    W.wave_host[1] = n;
    W.wave_host[2] = cam.seed;
    AZ_CUDA_TRY(cudaMemcpyAsync(W.wave_dev, W.wave_host, 3 * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    AZ_CUDA_TRY(cudaGraphLaunch(W.graph, st));
    rc.launches += W.graph_launches;
    rc.extend_launches += W.graph_extend_launches;
    return AZ_OK;
}

// The queue ordering of a render: the flags', else the scene's choice.
static uint32_t QueueOrder(const GpuScene &G, const az_render_opts *opts) {
    const uint32_t f = opts ? opts->flags : 0u;
    if (f & AZ_FLAG_ORDER_NONE) return 0u;
    if (f & (AZ_FLAG_ORDER_SHADOW | AZ_FLAG_ORDER_EXTEND))
        return ((f & AZ_FLAG_ORDER_SHADOW) ? kOrderShadow : 0u) | ((f & AZ_FLAG_ORDER_EXTEND) ? kOrderExtend : 0u);
    return G.order;
}

// The default wave of a render: as many camera samples as a quarter of the
// free device memory holds in wave queues, a power of two from 2^22 to 2^26.
// Bigger waves keep the launches of the deep tree levels, where most paths
// have ended, full (C1: 427 ms per frame at 2^22, 393 at 2^24, 383 at 2^26).
// The queues `W` already holds count as free, so that repeated renders of a
// scene keep their wave size.
static uint32_t DefaultWave(uint32_t per_node_shadow, const WaveBuffers &W) {
    uint64_t n = 1u << 22;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return (uint32_t)n;
    }
    // per sample: 1.5 queue entries of 168 bytes (two ping-pong sets of four
    // float4, digits, hit), shadow entries of 52 bytes, one float4 sum
    const double shadow_entries = std::min(1.5 * std::max(per_node_shadow, 1u), 4.0);
    const double per_sample = 1.5 * 168.0 + shadow_entries * 52.0 + 16.0;
    const double held = W.ptrs.empty() ? 0.0
                                       : (double)W.q.cap_q * 168.0 + (double)W.q.cap_s * 52.0 + (double)W.chunk * 16.0;
    const uint64_t fit = (uint64_t)(((double)free_b + held) / 4.0 / per_sample);
    while (n * 2 <= fit && n < (1u << 26)) n *= 2;
    return (uint32_t)n;
}

int Render(GpuScene &G, az_pixel *film, const az_camera *camera, const az_epsilon_values *eps, az_scissor sc,
           int32_t filter, uint32_t cull, const az_render_opts *opts, cudaStream_t st, az_render_stats *stats,
           GuideState *guide, bool train, WaveBuffers *wave_buffers, float4 *sample_out) {
    CameraParams cam;
    int rc = SetupCamera(camera, sc, filter, cull, eps, opts ? opts->seed : 0, cam);
    if (rc != AZ_OK) return rc;
    cam.sample_out = sample_out;
    cam.count_traversal = opts && (opts->flags & AZ_FLAG_COUNT_TRAVERSAL) ? 1u : 0u;
    cam.env_importance = opts && (opts->flags & AZ_FLAG_ENV_IMPORTANCE) && G.dev.env_rows ? 1u : 0u;
    cam.variant = opts && opts->variant ? opts->variant - 1 : G.variant;
    if (cam.variant >= kVariantCount) return SetError(AZ_ERR_INVALID_ARGUMENT, "unknown launch variant");
    // a variant the caller names applies to both traversal kernels
    cam.shadow_variant = (opts && opts->variant) || G.shadow_variant >= kVariantCount ? cam.variant : G.shadow_variant;
    cam.order = QueueOrder(G, opts);
    cam.serial_levels = opts && (opts->flags & AZ_FLAG_SERIAL_LEVELS) ? 1u : 0u;
    cam.watertight = opts && (opts->flags & AZ_FLAG_WATERTIGHT) ? 1u : 0u;
    if (G.dev.max_depth + 1 > AZ_MAX_LEVELS - 2) return SetError(AZ_ERR_UNSUPPORTED, "MaxRecursionDepth above 61");
    const uint64_t all = cam.npix * (uint64_t)cam.sqrt_spp * cam.sqrt_spp;
    // a part of the camera-sample sequence (one GPU's share of a frame)
    uint64_t begin = 0, end = all;
    if (opts && opts->sample_parts > 1) {
        if (opts->sample_part >= opts->sample_parts)
            return SetError(AZ_ERR_INVALID_ARGUMENT, "sample_part must be below sample_parts");
        begin = all / opts->sample_parts * opts->sample_part +
                std::min<uint64_t>(opts->sample_part, all % opts->sample_parts);
        end = begin + all / opts->sample_parts + (opts->sample_part < all % opts->sample_parts ? 1 : 0);
    }
    const uint64_t total = end - begin;
    if (stats) memset(stats, 0, sizeof(*stats));
    if (total == 0) return AZ_OK;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, G.device);
    uint32_t per_node_shadow = G.dev.light_count + (G.dev.use_env_map ? 1u : 0u);
    WaveBuffers &W = wave_buffers ? *wave_buffers : G.waves;
    uint32_t chunk = opts && opts->chunk_samples ? opts->chunk_samples : DefaultWave(per_node_shadow, W);
    // a training render updates the guide after every wave: smaller waves, more updates
    if (guide && train && !(opts && opts->chunk_samples)) chunk = 1u << 20;
    // the visit counters are 32-bit per wave: counting renders keep 2^22-sample waves
    if (cam.count_traversal && !(opts && opts->chunk_samples)) chunk = std::min(chunk, 1u << 22);
    chunk = (uint32_t)std::min<uint64_t>(chunk, total);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (stats) {
        AZ_CUDA_TRY(cudaEventCreate(&e0));
        AZ_CUDA_TRY(cudaEventCreate(&e1));
        AZ_CUDA_TRY(cudaEventRecord(e0, st));
    }
    RenderCounters counters{};
    std::vector<uint32_t> host_counts(AZ_COUNT_TOTAL);
    std::unique_ptr<StageTimer> timer;
    if (stats && opts && (opts->flags & AZ_FLAG_TIME_STAGES)) timer.reset(new StageTimer());
    // The launches of a wave run as one CUDA graph, captured once per scene,
    // camera, film and launch configuration and replayed for every wave with
    // its first sample, size and seed in a 24-byte descriptor.  Not for stage
    // timing, guided renders, or a legacy default stream (which cannot be
    // captured).
    const bool use_graph = !(opts && (opts->flags & AZ_FLAG_NO_GRAPH)) && !timer && !guide && st != nullptr &&
                           st != cudaStreamLegacy && st != cudaStreamPerThread;
    uint64_t pos = begin;
    while (pos < end) {
        uint32_t n = (uint32_t)std::min<uint64_t>(chunk, end - pos);
        uint32_t cap_q = std::max<uint32_t>(n + n / 2, 1024);
        uint32_t cap_s = std::max<uint32_t>((uint32_t)std::min<uint64_t>((uint64_t)cap_q * std::max(per_node_shadow, 1u),
                                                                         (uint64_t)n * 4), 1024);
        rc = W.Ensure(n, cap_q, cap_s);
        if (rc != AZ_OK) return rc;
        if (cam.order && (rc = W.EnsureOrder(std::max(W.q.cap_q, W.q.cap_s))) != AZ_OK) return rc;
        if (!cam.serial_levels && (rc = W.EnsureSide()) != AZ_OK) return rc;
        if (use_graph) {
            rc = ReplayWave(G, cam, W, pos, n, chunk, film, st, sms, counters);
        } else {
            rc = RenderWave(G, cam, W, pos, n, film, st, sms, counters, timer.get(), guide, train);
        }
        if (rc != AZ_OK) return rc;
        AZ_CUDA_TRY(cudaMemcpyAsync(host_counts.data(), W.q.counts, AZ_COUNT_TOTAL * sizeof(uint32_t),
                                    cudaMemcpyDeviceToHost, st));
        AZ_CUDA_TRY(cudaStreamSynchronize(st));
        if (timer) timer->Collect();
        if (host_counts[AZ_COUNT_ERROR])
            return SetError(AZ_ERR_CUDA, "BVH traversal exceeded its step limit (corrupt hierarchy)");
        if (host_counts[AZ_COUNT_OVERFLOW]) {
            // a queue overflowed: this wave wrote nothing; retry it with half the samples
            if (n <= 1024) return SetError(AZ_ERR_OUT_OF_MEMORY, "wave queue overflow with 1024 samples");
            chunk = std::max<uint32_t>(n / 2, 1024);
            counters.retries++;
            continue;
        }
        for (uint32_t L = 1; L < AZ_MAX_LEVELS; L++) {
            counters.extend += host_counts[L];
            counters.shadow += host_counts[AZ_COUNT_SHADOW + L];
        }
        counters.nodes += host_counts[AZ_COUNT_NODES];
        counters.prims += host_counts[AZ_COUNT_NODES + 1];
        counters.snodes += host_counts[AZ_COUNT_SNODES];
        counters.sprims += host_counts[AZ_COUNT_SNODES + 1];
        counters.chunks++;
        pos += n;
    }
    if (stats) {
        AZ_CUDA_TRY(cudaEventRecord(e1, st));
        AZ_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        stats->samples = total;
        stats->extend_rays = counters.extend;
        stats->shadow_rays = counters.shadow;
        stats->chunks = counters.chunks;
        stats->retries = counters.retries;
        stats->kernel_launches = counters.launches;
        stats->gpu_ms = ms;
        stats->node_visits = counters.nodes;
        stats->prim_visits = counters.prims;
        stats->shadow_node_visits = counters.snodes;
        stats->shadow_prim_visits = counters.sprims;
        stats->extend_launches = (uint32_t)counters.extend_launches;
        if (timer) {
            stats->extend_ms = timer->ms[0];
            stats->shade_ms = timer->ms[1];
            stats->shadow_ms = timer->ms[2];
        }
    }
    return AZ_OK;
}

int RenderTiles(GpuScene &G, std::vector<TileJob> &jobs, const az_render_opts *opts, cudaStream_t st,
                az_render_stats *stats, cudaEvent_t origin) {
    if (stats) memset(stats, 0, sizeof(*stats));
    if (jobs.empty()) return AZ_OK;
    const uint32_t nj = (uint32_t)jobs.size();
    // the jobs' scenes: one, or a table the kernels index per queue entry
    std::vector<GpuScene *> scenes;
    std::vector<uint32_t> scene_of(nj, 0);
    for (uint32_t j = 0; j < nj; j++) {
        GpuScene *sg = jobs[j].scene ? jobs[j].scene : &G;
        if (sg->device != G.device) return SetError(AZ_ERR_INVALID_ARGUMENT, "tile jobs on different devices");
        auto it = std::find(scenes.begin(), scenes.end(), sg);
        if (it == scenes.end()) {
            if (scenes.size() == kMaxWaveScenes)
                return SetError(AZ_ERR_UNSUPPORTED, "a tile render of more than 256 scenes");
            scenes.push_back(sg);
            it = scenes.end() - 1;
        }
        scene_of[j] = (uint32_t)(it - scenes.begin());
    }
    const bool multi = scenes.size() > 1;
    // the record the launches are chosen for: the first scene's, with the
    // features, light kinds and depth of all of them
    DevScene wave_dev = scenes[0]->dev;
    uint32_t per_node_shadow = 0;
    for (GpuScene *sg : scenes) {
        const DevScene &d = sg->dev;
        if (d.max_depth + 1 > AZ_MAX_LEVELS - 2) return SetError(AZ_ERR_UNSUPPORTED, "MaxRecursionDepth above 61");
        wave_dev.features |= d.features;
        wave_dev.full_light_queries |= d.full_light_queries;
        wave_dev.top_spheres += d.top_spheres;
        wave_dev.max_depth = std::max(wave_dev.max_depth, d.max_depth);
        per_node_shadow = std::max(per_node_shadow, d.light_count + (d.use_env_map ? 1u : 0u));
    }
    std::vector<CameraParams> cams(nj);
    uint64_t total = 0;
    for (uint32_t j = 0; j < nj; j++) {
        const TileJob &J = jobs[j];
        const GpuScene &Gj = *scenes[scene_of[j]];
        if (!J.film || !J.camera) return SetError(AZ_ERR_INVALID_ARGUMENT, "tile job without film or camera");
        CameraParams &c = cams[j];
        int rc = SetupCamera(J.camera, J.scissor, J.filter, J.cull, J.eps, J.seed, c);
        if (rc != AZ_OK) return rc;
        c.scene = scene_of[j];
        c.count_traversal = opts && (opts->flags & AZ_FLAG_COUNT_TRAVERSAL) ? 1u : 0u;
        c.env_importance = opts && (opts->flags & AZ_FLAG_ENV_IMPORTANCE) && Gj.dev.env_rows ? 1u : 0u;
        c.variant = opts && opts->variant ? opts->variant - 1 : G.variant;
        if (c.variant >= kVariantCount) return SetError(AZ_ERR_INVALID_ARGUMENT, "unknown launch variant");
        c.shadow_variant = (opts && opts->variant) || G.shadow_variant >= kVariantCount ? c.variant : G.shadow_variant;
        // several scenes: no queue ordering (its keys use one scene's bounds)
        c.order = multi ? 0u : QueueOrder(G, opts);
        c.serial_levels = opts && (opts->flags & AZ_FLAG_SERIAL_LEVELS) ? 1u : 0u;
        c.watertight = opts && (opts->flags & AZ_FLAG_WATERTIGHT) ? 1u : 0u;
        // the traversal and shading kernels take these from the wave's first job
        if (c.eps_isect != cams[0].eps_isect || c.eps_shadow != cams[0].eps_shadow || c.cull != cams[0].cull)
            return SetError(AZ_ERR_INVALID_ARGUMENT, "the jobs of a tile render need the same epsilons and culling");
        const uint64_t samples = c.npix * (uint64_t)c.sqrt_spp * c.sqrt_spp;
        if (samples >= (1ull << 32)) return SetError(AZ_ERR_UNSUPPORTED, "a tile job with 2^32 samples or more");
        jobs[j].samples = samples;
        jobs[j].done_ms = 0.0f;
        total += samples;
    }
    if (total == 0) return AZ_OK;
    // every job's samples in runs of kTile consecutive sample indices (one
    // sample number over a run of pixels: coherent camera rays), jobs in order
    constexpr uint32_t kTile = 4096;
    std::vector<Tile> tiles;
    std::vector<size_t> last_tile(nj, 0);
    for (uint32_t j = 0; j < nj; j++) {
        for (uint64_t first = 0; first < jobs[j].samples; first += kTile)
            tiles.push_back(Tile{j, (uint32_t)first, (uint32_t)std::min<uint64_t>(kTile, jobs[j].samples - first), 0u});
        last_tile[j] = tiles.size();   // one past the job's last tile
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, G.device);
    uint32_t chunk = opts && opts->chunk_samples ? opts->chunk_samples : DefaultWave(per_node_shadow, G.waves);
    chunk = std::max<uint32_t>(chunk, kTile);
    WaveBuffers &W = G.waves;
    // device tables: cameras, films, this wave's tiles, the work-queue counter, slot -> (job, sample)
    struct DevBuf {
        void *p = nullptr;
        ~DevBuf() {
            if (p) cudaFree(p);
        }
    } d_cams, d_films, d_tiles, d_next, d_slots, d_scenes;
    std::vector<az_pixel *> films(nj);
    for (uint32_t j = 0; j < nj; j++) films[j] = jobs[j].film;
    AZ_CUDA_TRY(cudaMalloc(&d_cams.p, nj * sizeof(CameraParams)));
    AZ_CUDA_TRY(cudaMalloc(&d_films.p, nj * sizeof(az_pixel *)));
    AZ_CUDA_TRY(cudaMalloc(&d_tiles.p, (chunk / kTile + 2 + nj) * sizeof(Tile)));
    AZ_CUDA_TRY(cudaMalloc(&d_next.p, sizeof(uint32_t)));
    AZ_CUDA_TRY(cudaMalloc(&d_slots.p, (size_t)chunk * sizeof(uint2)));
    AZ_CUDA_TRY(cudaMemcpyAsync(d_cams.p, cams.data(), nj * sizeof(CameraParams), cudaMemcpyHostToDevice, st));
    AZ_CUDA_TRY(cudaMemcpyAsync(d_films.p, films.data(), nj * sizeof(az_pixel *), cudaMemcpyHostToDevice, st));
    std::vector<DevScene> scene_recs;
    if (multi) {
        for (GpuScene *sg : scenes) scene_recs.push_back(sg->dev);
        AZ_CUDA_TRY(cudaMalloc(&d_scenes.p, scene_recs.size() * sizeof(DevScene)));
        AZ_CUDA_TRY(cudaMemcpyAsync(d_scenes.p, scene_recs.data(), scene_recs.size() * sizeof(DevScene),
                                    cudaMemcpyHostToDevice, st));
    }
    struct Events {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        ~Events() {
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        }
    } ev;
    AZ_CUDA_TRY(cudaEventCreate(&ev.e0));
    AZ_CUDA_TRY(cudaEventCreate(&ev.e1));
    AZ_CUDA_TRY(cudaEventRecord(ev.e0, st));
    RenderCounters counters{};
    std::vector<uint32_t> host_counts(AZ_COUNT_TOTAL);
    size_t ti = 0;
    while (ti < tiles.size()) {
        // the wave: the next tiles while they fit in `chunk` samples (the
        // tile table holds at most chunk / kTile + 2 + nj of them)
        uint32_t n = 0;
        size_t te = ti;
        while (te < tiles.size() && n + tiles[te].count <= chunk) {
            tiles[te].slot = n;
            n += tiles[te].count;
            te++;
        }
        const uint32_t ntiles = (uint32_t)(te - ti);
        const uint32_t cap_q = std::max<uint32_t>(n + n / 2, 1024);
        const uint32_t cap_s = std::max<uint32_t>(
            (uint32_t)std::min<uint64_t>((uint64_t)cap_q * std::max(per_node_shadow, 1u), (uint64_t)n * 4), 1024);
        int rc = W.Ensure(n, cap_q, cap_s);
        if (rc != AZ_OK) return rc;
        if (cams[0].order && (rc = W.EnsureOrder(std::max(W.q.cap_q, W.q.cap_s))) != AZ_OK) return rc;
        if (!cams[0].serial_levels && (rc = W.EnsureSide()) != AZ_OK) return rc;
        AZ_CUDA_TRY(cudaMemcpyAsync(d_tiles.p, tiles.data() + ti, ntiles * sizeof(Tile), cudaMemcpyHostToDevice, st));
        TileWave tw{(const Tile *)d_tiles.p, ntiles, (uint32_t *)d_next.p, (uint2 *)d_slots.p,
                    (const CameraParams *)d_cams.p, (az_pixel *const *)d_films.p,
                    multi ? (const DevScene *)d_scenes.p : nullptr, multi ? &wave_dev : nullptr};
        rc = RenderWave(G, cams[0], W, 0, n, nullptr, st, sms, counters, nullptr, nullptr, false, false, &tw);
        if (rc != AZ_OK) return rc;
        AZ_CUDA_TRY(cudaMemcpyAsync(host_counts.data(), W.q.counts, AZ_COUNT_TOTAL * sizeof(uint32_t),
                                    cudaMemcpyDeviceToHost, st));
        AZ_CUDA_TRY(cudaEventRecord(ev.e1, st));
        AZ_CUDA_TRY(cudaEventSynchronize(ev.e1));
        if (host_counts[AZ_COUNT_ERROR])
            return SetError(AZ_ERR_CUDA, "BVH traversal exceeded its step limit (corrupt hierarchy)");
        if (host_counts[AZ_COUNT_OVERFLOW]) {
            // a queue overflowed: this wave wrote nothing; retry it with half the samples
            if (n <= kTile) return SetError(AZ_ERR_OUT_OF_MEMORY, "wave queue overflow with one tile");
            chunk = std::max<uint32_t>(n / 2, kTile);
            counters.retries++;
            continue;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, origin ? origin : ev.e0, ev.e1);
        for (uint32_t j = 0; j < nj; j++)
            if (last_tile[j] > ti && last_tile[j] <= te) jobs[j].done_ms = ms;
        for (uint32_t L = 1; L < AZ_MAX_LEVELS; L++) {
            counters.extend += host_counts[L];
            counters.shadow += host_counts[AZ_COUNT_SHADOW + L];
        }
        counters.nodes += host_counts[AZ_COUNT_NODES];
        counters.prims += host_counts[AZ_COUNT_NODES + 1];
        counters.snodes += host_counts[AZ_COUNT_SNODES];
        counters.sprims += host_counts[AZ_COUNT_SNODES + 1];
        counters.chunks++;
        ti = te;
    }
    if (stats) {
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ev.e0, ev.e1);
        stats->samples = total;
        stats->extend_rays = counters.extend;
        stats->shadow_rays = counters.shadow;
        stats->chunks = counters.chunks;
        stats->retries = counters.retries;
        stats->kernel_launches = counters.launches;
        stats->gpu_ms = ms;
        stats->node_visits = counters.nodes;
        stats->prim_visits = counters.prims;
        stats->shadow_node_visits = counters.snodes;
        stats->shadow_prim_visits = counters.sprims;
        stats->extend_launches = (uint32_t)counters.extend_launches;
    }
    return AZ_OK;
}

// Times every launch variant on a band of the frame (the middle eighth of the
// scissor's rows, all samples) and keeps the fastest for this scene.
int Autotune(GpuScene &G, const az_camera *camera, const az_epsilon_values *eps, az_scissor sc, int32_t filter,
             uint32_t cull, const az_render_opts *opts, cudaStream_t st, uint32_t *best_out, float *ms_out) {
    CameraParams cam;
    int rc = SetupCamera(camera, sc, filter, cull, eps, opts ? opts->seed : 0, cam);
    if (rc != AZ_OK) return rc;
    // at least ~2^20 samples so that the timing is not dominated by launch overhead
    const uint64_t per_row = (uint64_t)cam.wsc * cam.sqrt_spp * cam.sqrt_spp;
    uint32_t rows = std::max<uint32_t>(cam.hsc / 8, (uint32_t)std::min<uint64_t>(cam.hsc, (1u << 20) / std::max<uint64_t>(per_row, 1) + 1));
    rows = std::max<uint32_t>(1, std::min(rows, cam.hsc));
    az_scissor band = sc;
    band.Min.y = cam.r0 + (cam.hsc - rows) / 2;
    band.Max.y = band.Min.y + rows;
    band.Min.x = cam.c0;
    band.Max.x = cam.c0 + cam.wsc;
    size_t bytes = (size_t)cam.width * cam.height * sizeof(az_pixel);
    az_pixel *film = nullptr;
    AZ_CUDA_TRY(cudaMalloc((void **)&film, bytes));
    float best_ms = FLT_MAX;
    uint32_t best = 0;
    az_render_opts o;
    if (opts) o = *opts;
    else memset(&o, 0, sizeof(o));
    for (uint32_t v = 0; v < kVariantCount && rc == AZ_OK; v++) {
        o.variant = v + 1;
        o.flags &= ~(uint32_t)AZ_FLAG_TIME_STAGES;
        az_render_stats stats;
        float vms = FLT_MAX;
        for (int rep = 0; rep < 3 && rc == AZ_OK; rep++) {   // the first run warms caches and allocates queues
            rc = Render(G, film, camera, eps, band, filter, cull, &o, st, &stats);
            if (rep > 0) vms = std::min(vms, stats.gpu_ms);
        }
        if (rc == AZ_OK && vms < best_ms) {
            best_ms = vms;
            best = v;
        }
    }
    // then the queue ordering with that launch configuration, unless the caller fixed it
    const uint32_t order_flags = AZ_FLAG_ORDER_SHADOW | AZ_FLAG_ORDER_EXTEND | AZ_FLAG_ORDER_NONE;
    uint32_t best_order = QueueOrder(G, opts);
    if (rc == AZ_OK && !(opts && (opts->flags & order_flags))) {
        o.variant = best + 1;
        for (uint32_t ord : {0u, kOrderShadow, kOrderExtend, kOrderShadow | kOrderExtend}) {
            if (ord == best_order || rc != AZ_OK) continue;
            o.flags = (o.flags & ~(order_flags | (uint32_t)AZ_FLAG_TIME_STAGES)) |
                      (ord == 0 ? (uint32_t)AZ_FLAG_ORDER_NONE
                                : ((ord & kOrderShadow) ? (uint32_t)AZ_FLAG_ORDER_SHADOW : 0u) |
                                      ((ord & kOrderExtend) ? (uint32_t)AZ_FLAG_ORDER_EXTEND : 0u));
            az_render_stats stats;
            float oms = FLT_MAX;
            for (int rep = 0; rep < 3 && rc == AZ_OK; rep++) {
                rc = Render(G, film, camera, eps, band, filter, cull, &o, st, &stats);
                if (rep > 0) oms = std::min(oms, stats.gpu_ms);
            }
            if (rc == AZ_OK && oms < best_ms) {
                best_ms = oms;
                best_order = ord;
            }
        }
    }
    // then the shadow queries' configuration alone, with the extension's fixed
    uint32_t best_shadow = best;
    if (rc == AZ_OK) {
        const uint32_t keep_variant = G.variant, keep_order = G.order, keep_shadow = G.shadow_variant;
        G.variant = best;
        G.order = best_order;
        o.variant = 0;   // the scene's configuration, with the shadow variant under test
        o.flags &= ~(uint32_t)AZ_FLAG_TIME_STAGES;
        if (!(opts && (opts->flags & order_flags))) o.flags &= ~order_flags;
        for (uint32_t v = 0; v < kVariantCount && rc == AZ_OK; v++) {
            if (v == best) continue;
            G.shadow_variant = v;
            az_render_stats stats;
            float vms = FLT_MAX;
            for (int rep = 0; rep < 3 && rc == AZ_OK; rep++) {
                rc = Render(G, film, camera, eps, band, filter, cull, &o, st, &stats);
                if (rep > 0) vms = std::min(vms, stats.gpu_ms);
            }
            if (rc == AZ_OK && vms < best_ms) {
                best_ms = vms;
                best_shadow = v;
            }
        }
        G.variant = keep_variant;
        G.order = keep_order;
        G.shadow_variant = keep_shadow;
    }
    cudaFree(film);
    if (rc != AZ_OK) return rc;
    G.variant = best;
    G.shadow_variant = best_shadow;
    G.order = best_order;
    if (best_out) *best_out = best + 1;
    if (ms_out) *ms_out = best_ms;
    return AZ_OK;
}

// ---- closest-hit queries for the parity tests ----
namespace {
template <bool WT>
__global__ void k_closest(DevScene S, const az_ray3 *rays, uint32_t n, uint32_t cull, float eps, uint32_t *hit,
                          uint32_t *uid, uint32_t *face, float *t) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    az_ray3 rr = rays[i];
    Ray r;
    r.o = mk(rr.Origin.x, rr.Origin.y, rr.Origin.z);
    r.d = mk(rr.Direction.x, rr.Direction.y, rr.Direction.z);
    r.time = rr.T;
    Hit h;
    bool ok = trace<Q_CLOSEST, WT>(S, r, cull != 0, eps, FLT_MAX, h);
    hit[i] = ok ? 1u : 0u;
    uid[i] = ok ? S.ents[h.ent].uid : 0xFFFFFFFFu;
    face[i] = ok && h.prim != 0xFFFFFFFFu ? S.tri_attr[h.prim].face_id : 0xFFFFFFFFu;
    t[i] = ok ? h.t : 0.0f;
}
}  // namespace

int ClosestHit(GpuScene &G, const az_ray3 *rays, uint32_t n, int32_t cull, float eps, uint32_t *out_hit,
               uint32_t *out_uid, uint32_t *out_face, float *out_t, cudaStream_t st, bool watertight) {
    if (n == 0) return AZ_OK;
    void *buf = nullptr;
    size_t bytes = (size_t)n * (sizeof(az_ray3) + 3 * sizeof(uint32_t) + sizeof(float)) + 64;
    AZ_CUDA_TRY(cudaMalloc(&buf, bytes));
    char *p = (char *)buf;
    az_ray3 *d_rays = (az_ray3 *)p;
    p += ((size_t)n * sizeof(az_ray3) + 15) & ~(size_t)15;
    uint32_t *d_hit = (uint32_t *)p;
    uint32_t *d_uid = d_hit + n;
    uint32_t *d_face = d_uid + n;
    float *d_t = (float *)(d_face + n);
    int rc = AZ_OK;
    cudaError_t e = cudaMemcpyAsync(d_rays, rays, (size_t)n * sizeof(az_ray3), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        if (watertight)
            k_closest<true><<<(n + 127) / 128, 128, 0, st>>>(G.dev, d_rays, n, (uint32_t)cull, eps, d_hit, d_uid,
                                                              d_face, d_t);
        else
            k_closest<false><<<(n + 127) / 128, 128, 0, st>>>(G.dev, d_rays, n, (uint32_t)cull, eps, d_hit, d_uid,
                                                               d_face, d_t);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_hit, d_hit, n * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_uid, d_uid, n * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_face, d_face, n * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(out_t, d_t, n * 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = CudaError(e, "closest-hit query");
    cudaFree(buf);
    return rc;
}

}  // namespace az

// ---------------------------------------------------------------------------
// az_gpu_render_noalloc: the same render with the wave queues in a fixed
// static device array, for callers that must not allocate device memory.
// ---------------------------------------------------------------------------
namespace az {
namespace {

constexpr uint32_t kStaticWave = 16384;                          // camera samples per wave, maximum
constexpr uint32_t kStaticCapQ = kStaticWave + kStaticWave / 2;  // path-queue entries per level buffer
constexpr uint32_t kStaticCapS = 4 * kStaticCapQ;                // light-sample (shadow) entries
constexpr size_t Align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kQ16 = Align256((size_t)kStaticCapQ * 16), kQ4 = Align256((size_t)kStaticCapQ * 4);
constexpr size_t kS16 = Align256((size_t)kStaticCapS * 16), kS4 = Align256((size_t)kStaticCapS * 4);
constexpr size_t kA16 = Align256((size_t)kStaticWave * 16), kC4 = Align256((size_t)AZ_COUNT_TOTAL * 4);
constexpr size_t kStaticBytes = 2 * (4 * kQ16 + kQ4) + kQ16 + 3 * kS16 + kS4 + kA16 + kC4;  // 9,110,784 B

// One copy per GPU that loads this library, held until the process exits.
// Host code must not use this name as an address: it resolves the device
// address once per device with cudaGetSymbolAddress (StaticWaveScratch).
static __device__ __align__(256) unsigned char g_wave_scratch[kStaticBytes];

std::mutex g_wave_scratch_mu;
void *g_wave_scratch_addr[256] = {};

// Device address of g_wave_scratch on the current device (set-up on first use).
int StaticWaveScratch(int device, void **out) {
    std::lock_guard<std::mutex> lock(g_wave_scratch_mu);
    if (device < 0 || device >= 256) return SetError(AZ_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    if (!g_wave_scratch_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_wave_scratch);
        if (e != cudaSuccess) return CudaError(e, "cudaGetSymbolAddress(wave scratch)");
        g_wave_scratch_addr[device] = p;
    }
    *out = g_wave_scratch_addr[device];
    return AZ_OK;
}

WaveQueues CarveStaticQueues(unsigned char *p) {
    WaveQueues q;
    memset(&q, 0, sizeof(q));
    for (int b = 0; b < 2; b++) {
        q.o[b] = (float4 *)p; p += kQ16;
        q.d[b] = (float4 *)p; p += kQ16;
        q.tp[b] = (float4 *)p; p += kQ16;
        q.att[b] = (float4 *)p; p += kQ16;
        q.digits[b] = (uint32_t *)p; p += kQ4;
    }
    q.hit = (uint4 *)p; p += kQ16;
    q.so = (float4 *)p; p += kS16;
    q.sd = (float4 *)p; p += kS16;
    q.sc = (float4 *)p; p += kS16;
    q.smeta = (uint32_t *)p; p += kS4;
    q.accum = (float4 *)p; p += kA16;
    q.counts = (uint32_t *)p;
    q.cap_q = kStaticCapQ;
    q.cap_s = kStaticCapS;
    return q;
}

}  // namespace
}  // namespace az

extern "C" int az_gpu_render_noalloc(az_gpu_scene *scene, az_pixel *film, const az_camera *camera,
                                     const az_epsilon_values *epsilons, az_scissor scissor, int32_t filter_type,
                                     uint32_t backface_culling, const az_render_opts *opts) {
    using namespace az;
    if (!scene || !scene->impl || !film || !camera) return SetError(AZ_ERR_INVALID_ARGUMENT, "null argument");
    const GpuScene &G = *scene->impl;
    const int device = opts ? opts->device : G.device;
    uint32_t wave = opts && opts->chunk_samples ? opts->chunk_samples : kStaticWave;
    if (wave > kStaticWave)
        return SetError(AZ_ERR_INVALID_ARGUMENT,
                        "chunk_samples " + std::to_string(wave) + " exceeds the static wave scratch of " +
                            std::to_string(kStaticWave) + " camera samples");
    if (G.dev.max_depth + 1 > AZ_MAX_LEVELS - 2) return SetError(AZ_ERR_UNSUPPORTED, "MaxRecursionDepth above 61");
    AZ_CUDA_TRY(cudaSetDevice(device));
    cudaStream_t st = opts && opts->stream ? (cudaStream_t)opts->stream : cudaStreamPerThread;
    void *base = nullptr;
    int rc = StaticWaveScratch(device, &base);
    if (rc != AZ_OK) return rc;
    CameraParams cam;
    rc = SetupCamera(camera, scissor, filter_type, backface_culling, epsilons, opts ? opts->seed : 0, cam);
    if (rc != AZ_OK) return rc;
    cam.variant = opts && opts->variant ? opts->variant - 1 : G.variant;
    if (cam.variant >= kVariantCount) return SetError(AZ_ERR_INVALID_ARGUMENT, "unknown launch variant");
    // a variant the caller names applies to both traversal kernels
    cam.shadow_variant = (opts && opts->variant) || G.shadow_variant >= kVariantCount ? cam.variant : G.shadow_variant;
    // flags whose work would need buffers of their own or a statistics output
    const uint32_t flags = opts ? opts->flags : 0u;
    const uint32_t refused = AZ_FLAG_COUNT_TRAVERSAL | AZ_FLAG_TIME_STAGES | AZ_FLAG_ORDER_SHADOW | AZ_FLAG_ORDER_EXTEND;
    if (flags & refused)
        return SetError(AZ_ERR_INVALID_ARGUMENT,
                        "az_gpu_render_noalloc does not take AZ_FLAG_COUNT_TRAVERSAL, AZ_FLAG_TIME_STAGES, "
                        "AZ_FLAG_ORDER_SHADOW or AZ_FLAG_ORDER_EXTEND");
    cam.env_importance = (flags & AZ_FLAG_ENV_IMPORTANCE) && G.dev.env_rows ? 1u : 0u;
    cam.watertight = (flags & AZ_FLAG_WATERTIGHT) ? 1u : 0u;
    const uint64_t total = cam.npix * (uint64_t)cam.sqrt_spp * cam.sqrt_spp;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const WaveQueues Q = CarveStaticQueues((unsigned char *)base);
    const uint32_t levels = std::min<uint32_t>(G.dev.max_depth + 1, AZ_MAX_LEVELS - 2);
    const int grid = sms * 16;
    uint32_t host_counts[AZ_COUNT_TOTAL];
    uint64_t pos = 0;
    while (pos < total) {
        const uint32_t n = (uint32_t)std::min<uint64_t>(wave, total - pos);
        // the array keeps the previous call's contents: the counters start at
        // zero, every other entry is written before it is read
        AZ_CUDA_TRY(cudaMemsetAsync(Q.counts, 0, AZ_COUNT_TOTAL * sizeof(uint32_t), st));
        AZ_CUDA_TRY(cudaMemcpyAsync(Q.counts + 1, &n, sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        k_camera<<<(n + 255) / 256, 256, 0, st>>>(cam, Q, pos, n);
        for (uint32_t L = 1; L <= levels; L++) {
            LaunchTraversalVariant(cam.variant, false, sms, G.dev, cam, Q, L, st);
            LaunchShade(grid, G.dev, cam, Q, pos, L, st);
            LaunchTraversalVariant(cam.shadow_variant, true, sms, G.dev, cam, Q, L, st);
        }
        k_splat<<<(n + 255) / 256, 256, 0, st>>>(cam, Q, pos, n, film);
        AZ_CUDA_TRY(cudaGetLastError());
        AZ_CUDA_TRY(cudaMemcpyAsync(host_counts, Q.counts, sizeof(host_counts), cudaMemcpyDeviceToHost, st));
        AZ_CUDA_TRY(cudaStreamSynchronize(st));
        if (host_counts[AZ_COUNT_ERROR])
            return SetError(AZ_ERR_CUDA, "BVH traversal exceeded its step limit (corrupt hierarchy)");
        if (host_counts[AZ_COUNT_OVERFLOW]) {
            // the wave wrote nothing to the film; rerun it with half the samples
            if (n <= 256) return SetError(AZ_ERR_OUT_OF_MEMORY, "static wave queues overflow with 256 samples");
            wave = n / 2;
            continue;
        }
        pos += n;
    }
    return AZ_OK;
}
