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

namespace az {
namespace {

using namespace azd;

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
enum : uint32_t { PF_INSIDE = 1u, PF_ATTEN = 2u, PF_BRANCHED = 4u };

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

__device__ __forceinline__ void add_accum(float4 *accum, uint32_t slot, f3 v) {
    if (is_zero(v)) return;
    atomicAdd(&accum[slot], make_float4(v.x, v.y, v.z, 0.0f));   // one vector atomic (sm_90 and later)
}

__device__ __forceinline__ void push_path(const WaveQueues &Q, int buf, uint32_t level, f3 o, float time, f3 d,
                                          uint32_t flags, f3 tp, uint32_t slot, f3 att, uint32_t digits) {
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

__device__ __forceinline__ void push_shadow(const WaveQueues &Q, uint32_t level, f3 o, float time, f3 d,
                                            float tmax, f3 c, uint32_t slot, uint32_t kind, uint32_t uid) {
    uint32_t i = push_slot(&Q.counts[AZ_COUNT_SHADOW + level]);
    if (i >= Q.cap_s) {
        Q.counts[AZ_COUNT_OVERFLOW] = 1;
        return;
    }
    Q.so[i] = make_float4(o.x, o.y, o.z, time);
    Q.sd[i] = make_float4(d.x, d.y, d.z, tmax);
    Q.sc[i] = make_float4(c.x, c.y, c.z, __uint_as_float(slot));
    Q.smeta[i] = (kind << 30) | (uid & 0x3FFFFFFFu);
}

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
    Q.d[1][i] = make_float4(dir.x, dir.y, dir.z, __uint_as_float(0u));
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
enum : int { MODE_LOOP = 0, MODE_LOCKSTEP = 1, MODE_FETCH = 2 };

template <int BLOCK, int MINB, int MODE>
__global__ void __launch_bounds__(BLOCK, MINB) k_extend(DevScene S, CameraParams cam, WaveQueues Q, uint32_t level) {
    const int buf = level & 1;
    const uint32_t n = min(Q.counts[level], Q.cap_q);
    uint32_t *cnt = cam.count_traversal ? Q.counts + AZ_COUNT_NODES : nullptr;
    uint32_t *err = Q.counts + AZ_COUNT_ERROR;
    if (MODE == MODE_LOCKSTEP) {
        Tracer<Q_CLOSEST> T;
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
            trace<Q_CLOSEST>(S, r, cam.cull != 0, cam.eps_isect, FLT_MAX, h, cnt, err);
            Q.hit[i] = make_uint4(__float_as_uint(h.t), __float_as_uint(h.tl), h.prim, h.ent);
        }
        return;
    }
    uint32_t *fetch = Q.counts + AZ_COUNT_FETCH + level;
    Tracer<Q_CLOSEST> T;
    uint2 stack[AZD_WSTACK];
    WarpFetch wf;
    uint32_t idx = kLaneIdle, qi = 0;   // work item and its queue entry
    while (true) {
        if (wf.refill(fetch, n, idx)) {
            qi = Q.eorder ? Q.eorder[idx] : idx;
            const float4 o = Q.o[buf][qi], d = Q.d[buf][qi];
            Ray r;
            r.o = mk(o.x, o.y, o.z);
            r.d = mk(d.x, d.y, d.z);
            r.time = o.w;
            T.init(S, r, cam.cull != 0, cam.eps_isect, FLT_MAX, stack);
        }
        if (__all_sync(0xFFFFFFFFu, idx == kLaneDone)) break;
        if (idx < n && T.step(S, stack, err)) {
            const Hit &h = T.best;
            Q.hit[qi] = make_uint4(__float_as_uint(h.t), __float_as_uint(h.tl), h.prim, h.ent);
            T.flush_counts(cnt);
            idx = kLaneIdle;
        }
    }
}

__device__ __forceinline__ f3 ld3(const float *p) { return mk(p[0], p[1], p[2]); }

// One tree node: direct light, ambient and children (TraceRay body,
// src/azimuth_main.cpp:974-1130).  FEAT (DevScene.features) compiles out the
// parts a scene cannot reach: textures, environment map, mirror/dielectric
// branches, point/area/directional/spot lights.
template <int BLOCK, uint32_t FEAT, bool GUIDED, bool TILES = false>
__global__ void __launch_bounds__(BLOCK) k_shade(DevScene S, CameraParams cam, WaveQueues Q, uint64_t wave_start,
                                                 uint32_t level) {
    constexpr bool TEX = FEAT & FEAT_TEXTURES, ENV = FEAT & FEAT_ENV, SPECIAL = FEAT & FEAT_SPECIAL,
                   LIGHTS = FEAT & FEAT_ANALYTIC_LIGHTS;
    const int buf = level & 1, nbuf = buf ^ 1;
    const uint32_t n = min(Q.counts[level], Q.cap_q);
    const bool can_spawn = level + 1 <= S.max_depth + 1;   // child's RecursionDepth <= MaxRecursionDepth
    const float seps = cam.eps_shadow;
    uint64_t seed = cam.seed;
    if (Q.wave) {
        wave_start = Q.wave[0];
        seed = Q.wave[2];
    }
    for (uint32_t i = blockIdx.x * BLOCK + threadIdx.x; i < n; i += gridDim.x * BLOCK) {
        const float4 o4 = Q.o[buf][i], d4 = Q.d[buf][i], tp4 = Q.tp[buf][i];
        const uint4 hh = Q.hit[i];
        const uint32_t flags = __float_as_uint(d4.w);
        const uint32_t slot = __float_as_uint(tp4.w);
        f3 tp = mk(tp4.x, tp4.y, tp4.z);
        Ray r;
        r.o = mk(o4.x, o4.y, o4.z);
        r.d = mk(d4.x, d4.y, d4.z);
        r.time = o4.w;
        Hit h;
        h.t = __uint_as_float(hh.x);
        h.tl = __uint_as_float(hh.y);
        h.prim = hh.z;
        h.ent = hh.w;
        // the sample's pixel; in a tile wave (TILES) its own job's camera,
        // whose seed and film size are read again where they are needed
        uint32_t row, col, sx, sy;
        uint32_t job = 0;
        if (TILES) {
            const uint2 js = Q.slot_map[slot];
            job = js.x;
            sample_of(Q.job_cams[job], js.y, row, col, sx, sy);
        } else {
            sample_of(cam, wave_start + slot, row, col, sx, sy);
        }
        // path-guide training: this node is the only child of the vertex recorded
        // one level up, so the sample's sum now holds everything up to that
        // vertex's level
        const bool recordable = GUIDED && Q.rec && slot < Q.n_rec && !(flags & PF_BRANCHED);
        if (recordable && level >= 2 && level - 2 < Q.rec_levels) {
            const float4 a = Q.accum[slot];
            Q.rec[(size_t)(level - 2) * Q.n_rec + slot].snap = make_float4(a.x, a.y, a.z, 1.0f);
        }
        if (h.ent == 0xFFFFFFFFu) {
            // a miss returns 0, except for the primary ray, whose sample then takes
            // the background (RayTravelDistance == 0, src/azimuth_main.cpp:1374-1384)
            if (level == 1) {
                const uint32_t fw = TILES ? Q.job_cams[job].width : cam.width;
                const uint32_t fh = TILES ? Q.job_cams[job].height : cam.height;
                add_accum(Q.accum, slot, background(S, r.d, (int32_t)fw - 1, (int32_t)fh - 1, row, col));
            }
            continue;
        }
        const bool inside = (flags & PF_INSIDE) != 0;
        if (flags & PF_ATTEN) {
            // Beer attenuation of a refracted or internally reflected subtree by
            // the distance to its first hit (src/azimuth_main.cpp:921-935, :955-962)
            float4 a = Q.att[buf][i];
            tp = had(tp, mk(expf(a.x * h.t), expf(a.y * h.t), expf(a.z * h.t)));
        }
        const DevEntity &e = S.ents[h.ent];
        if (e.is_emitter) {
            add_accum(Q.accum, slot, had(tp, ld3(e.radiance)));   // :984-985
            continue;
        }
        NodeRng rng;
        const uint32_t digits = Q.digits[buf][i];
        rng.init(TILES ? Q.job_cams[job].seed : seed, (row << 16) | col, (sy << 16) | sx, digits, level);
        const Surface s = surface_at<TEX>(S, r, h);
        const DevMaterial &m = S.materials[e.material];
        f3 dcol = ld3(m.diffuse), scol = ld3(m.specular);
        f3 local = mk(0.0f, 0.0f, 0.0f);   // this node's own radiance (before `tp`)
        bool ignore_ambient = false;
        if (TEX && e.texture_index) {
            const DevTexture &tex = S.textures[e.texture_index - 1];
            f3 ts = sample_texture(S, tex, s.p, s.u, s.v);
            if (tex.blend == 0) {           // ReplaceAll: DiffuseContribution starts at (1,1,1)
                dcol = ts;
                local = dcol;
                ignore_ambient = true;
            } else if (tex.blend == 1) {    // ReplaceDiffuse
                dcol = ts;
            } else {                        // BlendDiffuse
                dcol = dcol + ts;
                dcol = dcol * 0.5f;
            }
        }
        // CalculateLighting (:605-779): one sample and one visibility test per light
        for (uint32_t li = 0; li < S.light_count; li++) {
            const DevLight &L = S.lights[li];
            f3 ldir = mk(0.0f, 0.0f, 0.0f), I = ld3(L.intensity);
            uint32_t kind = SHADOW_TMAX;
            float falloff = 1.0f, ldist = 1.0f, invpdf = 1.0f;
            if (!LIGHTS || L.type == LIGHT_ENTITY) {
                sample_entity_light(S, L, s.p, rng, ldir, invpdf);
                I = ld3(L.intensity);
                kind = entity_light_needs_full_query(L) ? SHADOW_ENTITY_FULL : SHADOW_ENTITY;
            } else if (L.type == LIGHT_POINT) {
                ldir = ld3(L.position) - s.p;
                ldist = length(ldir);
            } else if (L.type == LIGHT_AREA) {
                // GCC evaluates the second Random01() of this sum first
                float u1 = rng.next();
                float u0 = rng.next();
                f3 lp = ld3(L.position) + ld3(L.edge0) * u0 + ld3(L.edge1) * u1;
                falloff = dot(normalize(lp - s.p), ld3(L.normal));
                if (falloff < 0.0f) falloff *= -1.0f;
                ldir = lp - s.p;
                ldist = length(ldir);
            } else if (L.type == LIGHT_DIRECTIONAL) {
                ldir = normalize(-ld3(L.position));
                kind = SHADOW_ANY;
            } else if (L.type == LIGHT_SPOT) {
                ldir = ld3(L.position) - s.p;
                ldist = length(ldir);
                float ct = dot(normalize(-ldir), normalize(ld3(L.spot_dir)));
                if (ct < L.cos_half_coverage) {
                    falloff = 0.0f;
                } else if (ct > L.cos_half_falloff) {
                    falloff = 1.0f;
                } else {
                    falloff = (ct - L.cos_half_coverage) / (L.cos_half_falloff - L.cos_half_coverage);
                    falloff = powf(falloff, 4.0f);
                    if (falloff < 0.0f) falloff = 0.0f;
                    else if (falloff > 1.0f) falloff = 1.0f;
                }
            }
            if (ldist == 0.0f) ldist = 0.001f;
            if (inside) continue;   // no direct light inside a dielectric (:714)
            f3 dc, sc;
            if (!light_contribution(dc, sc, m, I, ldir, r.d, s.n, ldist, falloff, invpdf)) continue;
            f3 c = had(tp, had(dcol, dc) + had(scol, sc));
            if (is_zero(c)) continue;
            // entity lights carry the light index (their identity test needs the light)
            push_shadow(Q, level, s.p + (ldir * seps), r.time, ldir, 1.0f - seps, c, slot, kind,
                        kind >= SHADOW_ENTITY ? li : 0u);
        }
        if (ENV && S.use_env_map) {
            // cosine-sampled environment ray (:724-778); not gated by InsideDielectric
            f3 Ld;
            float env_invpdf;
            if (cam.env_importance) {
                // the same two draws, through one-sample MIS of the map's luminance CDF and cosine sampling
                const float u1 = rng.next(), u2 = rng.next();
                env_invpdf = sample_env_mis(S, s.n, u1, u2, Ld);
            } else {
                float phi = 2.0f * AZD_PI_F32 * rng.next();
                float cp = cosf(phi), sp = sinf(phi);
                float theta = asinf(sqrtf(rng.next()));
                float ct = cosf(theta), st = sinf(theta);
                f3 U, V;
                onb(s.n, U, V);
                Ld = normalize(U * st * cp + V * st * sp + s.n * ct);
                float ca = dot(Ld, s.n);
                if (ca == 0.0f) ca = 0.000001f;
                env_invpdf = AZD_PI_F32 / ca;
            }
            float u = (-atan2f(Ld.z, Ld.x) + AZD_PI_F32) / (2.0f * AZD_PI_F32), v = acosf(Ld.y) / AZD_PI_F32;
            f3 I = sample_texture(S, S.textures[S.env_texture], mk(u, v, 1.0f), u, v);
            f3 dc, sc;
            if (env_invpdf > 0.0f && light_contribution(dc, sc, m, I, Ld, r.d, s.n, 1.0f, 1.0f, env_invpdf)) {
                f3 c = had(tp, had(dcol, dc) + had(scol, sc));
                if (!is_zero(c)) push_shadow(Q, level, s.p + (Ld * seps), r.time, Ld, FLT_MAX, c, slot, SHADOW_ANY, 0u);
            }
        }
        uint32_t next_child = 0;
        // a vertex that may spawn more than one child marks its subtree
        const bool multi = SPECIAL && S.path_trace && (m.is_mirror || m.transparent);
        const uint32_t bflag = ((flags & PF_BRANCHED) || multi) ? PF_BRANCHED : 0u;
        if (S.path_trace) {
            // diffuse scatter ray (:1029-1083): child 0
            f3 Sd;
            float invpdf, qpdf = 0.0f;
            if (GUIDED && can_spawn) {
                // path guiding: one-sample MIS of the learned vMF mixture and
                // cosine sampling, weighted by the mixture density (the deepest
                // level spawns no child: it has no proposals, and its records
                // keep density 0, which training skips)
                const GuideLobes &G = Q.lobes[i];
                const float alpha = fminf(G.alpha, Q.guide_alpha_max);
                const float us = rng.next();
                if (us < alpha) {
                    const int k = guide_pick_lobe(G, rng.next());
                    const float u1 = rng.next();
                    Sd = guide_sample_lobe(G, k, u1, rng.next());
                } else {
                    const float theta = asinf(sqrtf(rng.next()));
                    const float phi = 2.0f * AZD_PI_F32 * rng.next();
                    f3 U, V;
                    onb(s.n, U, V);
                    Sd = normalize(U * (sinf(theta) * cosf(phi)) + V * (sinf(theta) * sinf(phi)) + s.n * cosf(theta));
                }
                qpdf = guide_mixture_pdf_alpha(G, alpha, s.n, Sd);
                invpdf = qpdf > 0.0f ? 1.0f / qpdf : 0.0f;
            } else {
                float theta = S.importance_sampling ? asinf(sqrtf(rng.next())) : acosf(rng.next());
                float ct = cosf(theta), st = sinf(theta);
                float phi = 2.0f * AZD_PI_F32 * rng.next();
                float cp = cosf(phi), sp = sinf(phi);
                f3 U, V;
                onb(s.n, U, V);
                Sd = normalize(U * st * cp + V * st * sp + s.n * ct);
                if (S.importance_sampling) {
                    float cs = dot(Sd, s.n);
                    if (cs == 0.0f) cs = 0.000001f;
                    invpdf = AZD_PI_F32 / cs;
                } else {
                    invpdf = AZD_PI_F32 * 2.0f;
                }
            }
            f3 dc, sc, ctp = mk(0.0f, 0.0f, 0.0f);
            bool queued = false;
            if (can_spawn && invpdf > 0.0f &&
                light_contribution(dc, sc, m, mk(1.0f, 1.0f, 1.0f), Sd, r.d, s.n, 1.0f, 1.0f, invpdf)) {
                ctp = had(tp, had(dcol, dc) + had(scol, sc));
                if (!is_zero(ctp)) {
                    push_path(Q, nbuf, level + 1, s.p + (Sd * seps), r.time, Sd, (flags & PF_INSIDE) | bflag, ctp,
                              slot, mk(0.0f, 0.0f, 0.0f), child_digits(digits, level, 0));
                    queued = true;
                }
            }
            if (recordable && !multi && level - 1 < Q.rec_levels) {
                f3 gp, gn;
                guide_query(S, r, h, gp, gn);
                GuideRecord &R = Q.rec[(size_t)(level - 1) * Q.n_rec + slot];
                R.pos_q = make_float4(gp.x, gp.y, gp.z, qpdf);
                R.n = make_float4(gn.x, gn.y, gn.z, 0.0f);
                R.wo = make_float4(-r.d.x, -r.d.y, -r.d.z, 0.0f);
                R.wi = make_float4(Sd.x, Sd.y, Sd.z, 0.0f);
                R.tpc = make_float4(ctp.x, ctp.y, ctp.z, queued ? 1.0f : 0.0f);
            }
            next_child = 1;
        }
        // ReplaceAll's (1,1,1) start value and the ambient term (:1000-1020, :1086-1099)
        f3 own = local;
        if ((!inside || !m.transparent) && !ignore_ambient) own = own + had(ld3(m.ambient), ld3(S.ambient));
        add_accum(Q.accum, slot, had(tp, own));
        if (!SPECIAL) continue;
        if (m.is_mirror) {
            // CalculateMirrorContribution (:781-854)
            f3 rd = reflect(-r.d, s.n);
            if (m.glossiness != 0.0f) {
                f3 rp = mk(fabsf(rd.x), fabsf(rd.y), fabsf(rd.z));
                if (rp.x < rp.y) {
                    if (rp.x < rp.z) { rp = rd; rp.x = rp.x < 0.0f ? -1.0f : 1.0f; }
                    else { rp = rd; rp.z = rp.z < 0.0f ? -1.0f : 1.0f; }
                } else {
                    if (rp.y < rp.z) { rp = rd; rp.y = rp.y < 0.0f ? -1.0f : 1.0f; }
                    else { rp = rd; rp.z = rp.z < 0.0f ? -1.0f : 1.0f; }
                }
                rp = normalize(rp);
                f3 uu = cross(rp, rd), vv = cross(uu, rd);
                // GCC evaluates the second Random01() of this sum first
                float b = rng.next();
                float a = rng.next();
                rd = rd + (2.0f * m.glossiness) * (uu * (a - 0.5f) + vv * (b - 0.5f));
                rd = normalize(rd);
            }
            f3 ctp = had(tp, ld3(m.mirror));
            if (can_spawn && !is_zero(ctp))
                push_path(Q, nbuf, level + 1, s.p + (rd * 0.000825f), r.time, rd, (flags & PF_INSIDE) | bflag, ctp,
                          slot, mk(0.0f, 0.0f, 0.0f), child_digits(digits, level, next_child));
            next_child++;
        }
        if (m.transparent) {
            // CalculateTransparencyContribution (:856-964)
            f3 T = ld3(m.transparency);
            float to = m.refraction_index, from = 1.0f;
            if (inside) {
                from = m.refraction_index;
                to = 1.0f;
            }
            f3 N = s.n;
            float ct = -dot(r.d, N);
            if (ct < 0.0f) {
                N = -s.n;
                ct = -dot(r.d, N);
            }
            float ratio = from / to;
            float delta = 1.0f - (ratio * ratio) * (1.0f - ct * ct);
            float refl;
            f3 att = mk(T.x - 1.0f, T.y - 1.0f, T.z - 1.0f);
            if (delta <= 0.0f) {
                refl = 1.0f;
            } else {
                float cphi = sqrtf(delta);
                float cair = inside ? cphi : ct;
                float icair = 1.0f - cair;
                float q = (from - to) / (from + to);
                float r0 = q * q;
                refl = r0 + (1.0f - r0) * powf(icair, 5.0f);
                f3 td = (r.d + N * ct) * ratio - N * cphi;
                td = normalize(td);
                f3 ctp = tp * (1.0f - refl);
                if (can_spawn && !is_zero(ctp))
                    push_path(Q, nbuf, level + 1, s.p + (td * 0.0001f), r.time, td,
                              (inside ? 0u : PF_INSIDE) | (inside ? 0u : PF_ATTEN) | bflag, ctp, slot, att,
                              child_digits(digits, level, next_child));
                next_child++;
            }
            f3 rd = reflect(-r.d, N);
            f3 ctp = tp * refl;
            if (can_spawn && !is_zero(ctp))
                push_path(Q, nbuf, level + 1, s.p + (rd * 0.0001f), r.time, rd,
                          (inside ? PF_INSIDE : 0u) | (inside ? PF_ATTEN : 0u) | bflag, ctp, slot, att,
                          child_digits(digits, level, next_child));
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
__global__ void __launch_bounds__(128) k_shadow_full(DevScene S, CameraParams cam, WaveQueues Q, uint32_t level) {
    const uint32_t n = min(Q.counts[AZ_COUNT_SHADOW + level], Q.cap_s);
    uint32_t *cnt = cam.count_traversal ? Q.counts + AZ_COUNT_NODES : nullptr;
    uint32_t *err = Q.counts + AZ_COUNT_ERROR;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t meta = Q.smeta[i];
        if ((meta >> 30) != SHADOW_ENTITY_FULL) continue;
        const float4 o = Q.so[i], d = Q.sd[i], c = Q.sc[i];
        const DevLight &L = S.lights[meta & 0x3FFFFFFFu];
        Ray r;
        r.o = mk(o.x, o.y, o.z);
        r.d = mk(d.x, d.y, d.z);
        r.time = o.w;
        Hit h;
        const bool any = trace<Q_CLOSEST>(S, r, false, 0.0f, FLT_MAX, h, cnt, err);
        if (!any || S.ents[h.ent].uid == L.uid) add_accum(Q.accum, __float_as_uint(c.w), mk(c.x, c.y, c.z));
    }
}

template <int BLOCK, int MINB, int MODE>
__global__ void __launch_bounds__(BLOCK, MINB) k_shadow(DevScene S, CameraParams cam, WaveQueues Q, uint32_t level) {
    const uint32_t n = min(Q.counts[AZ_COUNT_SHADOW + level], Q.cap_s);
    uint32_t *cnt = cam.count_traversal ? Q.counts + AZ_COUNT_NODES : nullptr;
    uint32_t *err = Q.counts + AZ_COUNT_ERROR;
    if (MODE == MODE_LOCKSTEP) {
        Tracer<Q_ANY> T;
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
                const uint32_t kind = meta >> 30, li = meta & 0x3FFFFFFFu;
                Ray r;
                r.o = mk(o.x, o.y, o.z);
                r.d = mk(d.x, d.y, d.z);
                r.time = o.w;
                if (kind == SHADOW_ENTITY_FULL) {
                    live = false;   // k_shadow_full
                } else if (kind == SHADOW_ENTITY) {
                    const DevLight &L = S.lights[li];
                    float tl = FLT_MAX;
                    const int lh = light_entity_hit(S, L, r, tl);
                    T.init(S, r, false, 0.0f, lh ? tl : FLT_MAX, stack, L.ent_index);
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
            const uint32_t kind = meta >> 30, li = meta & 0x3FFFFFFFu;
            Ray r;
            r.o = mk(o.x, o.y, o.z);
            r.d = mk(d.x, d.y, d.z);
            r.time = o.w;
            Hit h;
            bool visible;
            if (kind == SHADOW_ENTITY_FULL) {
                continue;   // k_shadow_full
            } else if (kind == SHADOW_ENTITY) {
                const DevLight &L = S.lights[li];
                float tl = FLT_MAX;
                const int lh = light_entity_hit(S, L, r, tl);
                visible = !trace<Q_ANY>(S, r, false, 0.0f, lh ? tl : FLT_MAX, h, cnt, err, L.ent_index);
            } else {
                visible = !trace<Q_ANY>(S, r, false, 0.0f, kind == SHADOW_ANY ? FLT_MAX : d.w, h, cnt, err);
            }
            if (visible) add_accum(Q.accum, __float_as_uint(c.w), mk(c.x, c.y, c.z));
        }
        return;
    }
    uint32_t *fetch = Q.counts + AZ_COUNT_FETCH + AZ_MAX_LEVELS + level;
    Tracer<Q_ANY> T;
    uint2 stack[AZD_WSTACK];
    WarpFetch wf;
    uint32_t idx = kLaneIdle;
    float4 c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    while (true) {
        if (wf.refill(fetch, n, idx)) {
            const uint32_t qi = Q.sorder ? Q.sorder[idx] : idx;
            const float4 o = Q.so[qi], d = Q.sd[qi];
            c = Q.sc[qi];
            const uint32_t meta = Q.smeta[qi];
            const uint32_t kind = meta >> 30, li = meta & 0x3FFFFFFFu;
            Ray r;
            r.o = mk(o.x, o.y, o.z);
            r.d = mk(d.x, d.y, d.z);
            r.time = o.w;
            if (kind == SHADOW_ENTITY_FULL) {
                idx = kLaneIdle;   // k_shadow_full
            } else if (kind == SHADOW_ENTITY) {
                const DevLight &L = S.lights[li];
                float tl = FLT_MAX;
                const int lh = light_entity_hit(S, L, r, tl);
                T.init(S, r, false, 0.0f, lh ? tl : FLT_MAX, stack, L.ent_index);
            } else {
                T.init(S, r, false, 0.0f, kind == SHADOW_ANY ? FLT_MAX : d.w, stack);
            }
        }
        if (__all_sync(0xFFFFFFFFu, idx == kLaneDone)) break;
        if (idx < n && T.step(S, stack, err)) {
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

constexpr int kBlock = 128;

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
                                 {256, 3, MODE_LOCKSTEP}, {64, 12, MODE_LOCKSTEP}};
constexpr uint32_t kVariantCount = sizeof(kVariants) / sizeof(kVariants[0]);
static_assert(kVariantCount == AZ_LAUNCH_VARIANTS, "variant table and header disagree");

template <uint32_t F>
void LaunchShadeF(int grid, const DevScene &S, const CameraParams &cam, const WaveQueues &Q, uint64_t start,
                  uint32_t L, cudaStream_t st, bool guided) {
    if (Q.slot_map) k_shade<kBlock, F, false, true><<<grid, kBlock, 0, st>>>(S, cam, Q, start, L);   // tile wave
    else if (guided) k_shade<kBlock, F, true><<<grid, kBlock, 0, st>>>(S, cam, Q, start, L);
    else k_shade<kBlock, F, false><<<grid, kBlock, 0, st>>>(S, cam, Q, start, L);
}

// The shading kernel specialised for the scene's features (DevScene.features)
// and for guided scattering (Q.lobes set).
void LaunchShade(int grid, const DevScene &S, const CameraParams &cam, const WaveQueues &Q, uint64_t start,
                 uint32_t L, cudaStream_t st) {
    const bool guided = Q.lobes != nullptr;
    switch (S.features & 15u) {
        case 0: LaunchShadeF<0>(grid, S, cam, Q, start, L, st, guided); break;
        case 1: LaunchShadeF<1>(grid, S, cam, Q, start, L, st, guided); break;
        case 2: LaunchShadeF<2>(grid, S, cam, Q, start, L, st, guided); break;
        case 3: LaunchShadeF<3>(grid, S, cam, Q, start, L, st, guided); break;
        case 4: LaunchShadeF<4>(grid, S, cam, Q, start, L, st, guided); break;
        case 5: LaunchShadeF<5>(grid, S, cam, Q, start, L, st, guided); break;
        case 6: LaunchShadeF<6>(grid, S, cam, Q, start, L, st, guided); break;
        case 7: LaunchShadeF<7>(grid, S, cam, Q, start, L, st, guided); break;
        case 8: LaunchShadeF<8>(grid, S, cam, Q, start, L, st, guided); break;
        case 9: LaunchShadeF<9>(grid, S, cam, Q, start, L, st, guided); break;
        case 10: LaunchShadeF<10>(grid, S, cam, Q, start, L, st, guided); break;
        case 11: LaunchShadeF<11>(grid, S, cam, Q, start, L, st, guided); break;
        case 12: LaunchShadeF<12>(grid, S, cam, Q, start, L, st, guided); break;
        case 13: LaunchShadeF<13>(grid, S, cam, Q, start, L, st, guided); break;
        case 14: LaunchShadeF<14>(grid, S, cam, Q, start, L, st, guided); break;
        default: LaunchShadeF<15>(grid, S, cam, Q, start, L, st, guided); break;
    }
}

template <int B, int M, int P>
void LaunchTraversal(bool shadow, int sms, const DevScene &S, const CameraParams &cam, const WaveQueues &Q,
                     uint32_t L, cudaStream_t st) {
    const int grid = sms * (2048 / B);
    if (shadow) k_shadow<B, M, P><<<grid, B, 0, st>>>(S, cam, Q, L);
    else k_extend<B, M, P><<<grid, B, 0, st>>>(S, cam, Q, L);
}

void LaunchTraversalVariant(uint32_t v, bool shadow, int sms, const DevScene &S, const CameraParams &cam,
                            const WaveQueues &Q, uint32_t L, cudaStream_t st) {
    if (shadow && S.full_light_queries) k_shadow_full<<<sms * 16, 128, 0, st>>>(S, cam, Q, L);
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
};

static int RenderWave(const GpuScene &G, const CameraParams &cam, WaveBuffers &W, uint64_t start, uint32_t n,
                      az_pixel *film, cudaStream_t st, int sms, RenderCounters &rc, StageTimer *timer,
                      GuideState *guide, bool train, bool capture = false, const TileWave *tw = nullptr) {
    WaveQueues Q = W.q;
    if (tw) {
        Q.slot_map = tw->slot_map;
        Q.job_cams = tw->cams;
    }
    if (capture) Q.wave = W.wave_dev;
    if (cam.order & kOrderExtend) Q.eorder = W.oidx_e;
    if (cam.order & kOrderShadow) Q.sorder = W.oidx_s;
    // While the guide trains, its early proposals can be far from the light
    // field; capping the chance of sampling them at one half keeps every
    // sample's weight within twice cosine sampling's (the estimate stays
    // unbiased for any cap).  Inference-only renders use the learned value.
    Q.guide_alpha_max = train ? 0.5f : 1.0f;
    const uint32_t levels = std::min<uint32_t>(G.dev.max_depth + 1, AZ_MAX_LEVELS - 2);
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
    for (uint32_t L = 1; L <= levels; L++) {
        if (timer) timer->Mark(st, 0);
        if (cam.order & kOrderExtend) {
            int orc = OrderQueue(G, Q, W, L, 0, sms, st, rc);
            if (orc != AZ_OK) return orc;
        }
        LaunchTraversalVariant(v, false, sms, G.dev, cam, Q, L, st);
        if (guide && L + 1 <= G.dev.max_depth + 1) {   // the deepest level spawns nothing to guide
            int grc = GuideInfer(*guide, G, Q, L, st);
            if (grc != AZ_OK) return grc;
            rc.launches++;
        }
        if (timer) timer->Mark(st, 1);
        LaunchShade(grid, G.dev, cam, Q, start, L, st);
        if (timer) timer->Mark(st, 2);
        if (cam.order & kOrderShadow) {
            int orc = OrderQueue(G, Q, W, L, 1, sms, st, rc);
            if (orc != AZ_OK) return orc;
        }
        LaunchTraversalVariant(cam.shadow_variant, true, sms, G.dev, cam, Q, L, st);
        if (timer) timer->Mark(st, 3);
        rc.launches += G.dev.full_light_queries ? 4 : 3;
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
           GuideState *guide, bool train, WaveBuffers *wave_buffers) {
    CameraParams cam;
    int rc = SetupCamera(camera, sc, filter, cull, eps, opts ? opts->seed : 0, cam);
    if (rc != AZ_OK) return rc;
    cam.count_traversal = opts && (opts->flags & AZ_FLAG_COUNT_TRAVERSAL) ? 1u : 0u;
    cam.env_importance = opts && (opts->flags & AZ_FLAG_ENV_IMPORTANCE) && G.dev.env_rows ? 1u : 0u;
    cam.variant = opts && opts->variant ? opts->variant - 1 : G.variant;
    if (cam.variant >= kVariantCount) return SetError(AZ_ERR_INVALID_ARGUMENT, "unknown launch variant");
    // a variant the caller names applies to both traversal kernels
    cam.shadow_variant = (opts && opts->variant) || G.shadow_variant >= kVariantCount ? cam.variant : G.shadow_variant;
    cam.order = QueueOrder(G, opts);
    if (G.dev.max_depth + 1 > AZ_MAX_LEVELS - 2) return SetError(AZ_ERR_UNSUPPORTED, "MaxRecursionDepth above 61");
    uint64_t total = cam.npix * (uint64_t)cam.sqrt_spp * cam.sqrt_spp;
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
    uint64_t pos = 0;
    while (pos < total) {
        uint32_t n = (uint32_t)std::min<uint64_t>(chunk, total - pos);
        uint32_t cap_q = std::max<uint32_t>(n + n / 2, 1024);
        uint32_t cap_s = std::max<uint32_t>((uint32_t)std::min<uint64_t>((uint64_t)cap_q * std::max(per_node_shadow, 1u),
                                                                         (uint64_t)n * 4), 1024);
        rc = W.Ensure(n, cap_q, cap_s);
        if (rc != AZ_OK) return rc;
        if (cam.order && (rc = W.EnsureOrder(std::max(W.q.cap_q, W.q.cap_s))) != AZ_OK) return rc;
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
                az_render_stats *stats) {
    if (stats) memset(stats, 0, sizeof(*stats));
    if (jobs.empty()) return AZ_OK;
    if (G.dev.max_depth + 1 > AZ_MAX_LEVELS - 2) return SetError(AZ_ERR_UNSUPPORTED, "MaxRecursionDepth above 61");
    const uint32_t nj = (uint32_t)jobs.size();
    std::vector<CameraParams> cams(nj);
    uint64_t total = 0;
    for (uint32_t j = 0; j < nj; j++) {
        const TileJob &J = jobs[j];
        if (!J.film || !J.camera) return SetError(AZ_ERR_INVALID_ARGUMENT, "tile job without film or camera");
        CameraParams &c = cams[j];
        int rc = SetupCamera(J.camera, J.scissor, J.filter, J.cull, J.eps, J.seed, c);
        if (rc != AZ_OK) return rc;
        c.count_traversal = opts && (opts->flags & AZ_FLAG_COUNT_TRAVERSAL) ? 1u : 0u;
        c.env_importance = opts && (opts->flags & AZ_FLAG_ENV_IMPORTANCE) && G.dev.env_rows ? 1u : 0u;
        c.variant = opts && opts->variant ? opts->variant - 1 : G.variant;
        if (c.variant >= kVariantCount) return SetError(AZ_ERR_INVALID_ARGUMENT, "unknown launch variant");
        c.shadow_variant = (opts && opts->variant) || G.shadow_variant >= kVariantCount ? c.variant : G.shadow_variant;
        c.order = QueueOrder(G, opts);
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
    const uint32_t per_node_shadow = G.dev.light_count + (G.dev.use_env_map ? 1u : 0u);
    uint32_t chunk = opts && opts->chunk_samples ? opts->chunk_samples : DefaultWave(per_node_shadow, G.waves);
    chunk = std::max<uint32_t>(chunk, kTile);
    WaveBuffers &W = G.waves;
    // device tables: cameras, films, this wave's tiles, the work-queue counter, slot -> (job, sample)
    struct DevBuf {
        void *p = nullptr;
        ~DevBuf() {
            if (p) cudaFree(p);
        }
    } d_cams, d_films, d_tiles, d_next, d_slots;
    std::vector<az_pixel *> films(nj);
    for (uint32_t j = 0; j < nj; j++) films[j] = jobs[j].film;
    AZ_CUDA_TRY(cudaMalloc(&d_cams.p, nj * sizeof(CameraParams)));
    AZ_CUDA_TRY(cudaMalloc(&d_films.p, nj * sizeof(az_pixel *)));
    AZ_CUDA_TRY(cudaMalloc(&d_tiles.p, (chunk / kTile + 2 + nj) * sizeof(Tile)));
    AZ_CUDA_TRY(cudaMalloc(&d_next.p, sizeof(uint32_t)));
    AZ_CUDA_TRY(cudaMalloc(&d_slots.p, (size_t)chunk * sizeof(uint2)));
    AZ_CUDA_TRY(cudaMemcpyAsync(d_cams.p, cams.data(), nj * sizeof(CameraParams), cudaMemcpyHostToDevice, st));
    AZ_CUDA_TRY(cudaMemcpyAsync(d_films.p, films.data(), nj * sizeof(az_pixel *), cudaMemcpyHostToDevice, st));
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
        AZ_CUDA_TRY(cudaMemcpyAsync(d_tiles.p, tiles.data() + ti, ntiles * sizeof(Tile), cudaMemcpyHostToDevice, st));
        TileWave tw{(const Tile *)d_tiles.p, ntiles, (uint32_t *)d_next.p, (uint2 *)d_slots.p,
                    (const CameraParams *)d_cams.p, (az_pixel *const *)d_films.p};
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
        cudaEventElapsedTime(&ms, ev.e0, ev.e1);
        for (uint32_t j = 0; j < nj; j++)
            if (last_tile[j] > ti && last_tile[j] <= te) jobs[j].done_ms = ms;
        for (uint32_t L = 1; L < AZ_MAX_LEVELS; L++) {
            counters.extend += host_counts[L];
            counters.shadow += host_counts[AZ_COUNT_SHADOW + L];
        }
        counters.nodes += host_counts[AZ_COUNT_NODES];
        counters.prims += host_counts[AZ_COUNT_NODES + 1];
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
    bool ok = trace<Q_CLOSEST>(S, r, cull != 0, eps, FLT_MAX, h);
    hit[i] = ok ? 1u : 0u;
    uid[i] = ok ? S.ents[h.ent].uid : 0xFFFFFFFFu;
    face[i] = ok && h.prim != 0xFFFFFFFFu ? S.tri_attr[h.prim].face_id : 0xFFFFFFFFu;
    t[i] = ok ? h.t : 0.0f;
}
}  // namespace

int ClosestHit(GpuScene &G, const az_ray3 *rays, uint32_t n, int32_t cull, float eps, uint32_t *out_hit,
               uint32_t *out_uid, uint32_t *out_face, float *out_t, cudaStream_t st) {
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
        k_closest<<<(n + 127) / 128, 128, 0, st>>>(G.dev, d_rays, n, (uint32_t)cull, eps, d_hit, d_uid, d_face, d_t);
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
