// Closest-hit and occlusion queries on the device scene.
//
// Primitive tests reproduce azimuth's arithmetic exactly (same operation
// order, IEEE rounding, no contraction): the Cramer triangle test
// (src/azimuth_main.cpp:147-243), the transformed, moving sphere
// (:64-146) and the mesh-instance path (:244-281: motion, GetLocalRay with a
// re-normalised direction, world t recomputed from the local hit point).
// The hierarchy is this library's own 8-wide compressed BVH, traversed
// near-first with t-pruning on conservative boxes; it finds the same nearest
// primitive as azimuth's exhaustive BVH walk except for exact ties and rays
// that graze a box azimuth's slab test rejects.
#pragma once
#include <cfloat>

#include "az_scene_dev.cuh"

namespace azd {

struct Ray {
    f3 o, d;
    float time;
};

// GetLocalRay, src/azimuth_ray.h:24-66
__device__ __forceinline__ Ray local_ray(Ray r, const m34 &m) {
    Ray l;
    l.o = point_xf(m, r.o);
    l.d = normalize(vector_xf(m, r.d));
    l.time = r.time;
    return l;
}

// GetLocalRay for a transform that is the identity with no motion: the bits
// local_ray() gives (x * 1 + y * 0 + z * 0 + 0 is x, a -0 becoming +0; the
// re-normalised direction), without the matrix products.  Only the sign of an
// exactly zero direction component can differ, which changes no distance.
__device__ __forceinline__ Ray local_ray_identity(const Ray &r) {
    Ray l;
    l.o = mk(r.o.x + 0.0f, r.o.y + 0.0f, r.o.z + 0.0f);
    l.d = normalize(r.d);
    l.time = r.time;
    return l;
}

struct Hit {
    float t;        // azimuth's Hit.t (world)
    float tl;       // local t of the primitive test (triangle: in its mesh space)
    uint32_t prim;  // triangle index, or 0xFFFFFFFF for a sphere
    uint32_t ent;   // dense entity index, 0xFFFFFFFF = miss
};

// Sphere, src/azimuth_main.cpp:64-146.  Returns the world t (WorldT) and the
// local quadratic root; the caller keeps the hit only if it beats its best.
__device__ __forceinline__ bool sphere_test(const DevEntity &e, Ray r, float eps, float &t_world, float &t_local) {
    f3 motion = r.time * mk(e.motion[0], e.motion[1], e.motion[2]);
    r.o = r.o - motion;
    Ray lr = local_ray(r, e.inv);
    float radius = e.radius;
    f3 c = mk(e.center[0], e.center[1], e.center[2]);
    f3 dist = lr.o - c;
    float A = dot(lr.d, lr.d);
    float B = dot(dist, lr.d);
    float C = dot(dist, dist) - radius * radius;
    float disc = B * B - (A * C);
    if (!(disc > 0.0f)) return false;
    float sq = sqrtf(disc);
    float t1 = (-B + sq) / (A), t2 = (-B - sq) / (A);
    float t = FLT_MAX;
    if (t1 > eps && t2 > eps) t = t1 < t2 ? t1 : t2;
    else if (t1 > eps) t = t1;
    else if (t2 > eps) t = t2;
    if (!(t > eps && t < FLT_MAX)) return false;
    f3 hp = lr.o + (lr.d * t);
    f3 wp = point_xf(e.xf, hp) + motion;
    float wt = length(wp - r.o - motion) / length(r.d);
    if (!(wt > eps && wt < FLT_MAX)) return false;
    t_world = wt;
    t_local = t;
    return true;
}

// Cramer triangle test, src/azimuth_main.cpp:147-243, on the precomputed
// differences E1 = P0-P1, E2 = P0-P2 (identical bits to azimuth's A,B,D,E,G,H).
__device__ __forceinline__ bool tri_test(const DevTri &tr, const Ray &r, bool cull, float eps, float tmax,
                                         float &t_out, float &beta_out, float &gamma_out) {
    const float p0x = tr.a.x, p0y = tr.a.y, p0z = tr.a.z;
    const float A = tr.a.w, D = tr.b.x, G = tr.b.y;      // P0 - P1
    const float B = tr.b.z, E = tr.b.w, H = tr.c.x;      // P0 - P2
    if (cull) {
        f3 fn = mk(tr.c.y, tr.c.z, tr.c.w);
        if (!(dot(r.d, fn) < 0.0f)) return false;
    }
    const float C = r.d.x, F = r.d.y, I = r.d.z;
    float detM = (A * E * I) + (D * H * C) + (G * B * F) - (C * E * G) - (F * H * A) - (I * B * D);
    float K = p0x - r.o.x, M = p0y - r.o.y, N = p0z - r.o.z;
    float detB = (K * E * I) + (M * H * C) + (N * B * F) - (C * E * N) - (F * H * K) - (I * B * M);
    const float lower = -0.000001f;
    // Division-free pre-rejects: only cases where azimuth's test is certain to
    // fail (the quotient is out of range by far more than its rounding), so
    // every accepted hit still comes from azimuth's exact divisions below.
    const float am = fabsf(detM);
    const float sb = detM < 0.0f ? -detB : detB;
    if (!(sb > -0.001f * am && sb <= 1.001f * am)) return false;
    float beta = detB / detM;
    if (!(beta > lower && beta <= 1.0f)) return false;
    float detG = (A * M * I) + (D * N * C) + (G * K * F) - (C * M * G) - (F * N * A) - (I * K * D);
    const float sg = detM < 0.0f ? -detG : detG;
    if (!(sg > -0.001f * am && sg <= 1.001f * am)) return false;
    float gamma = detG / detM;
    if (!(gamma > lower && gamma <= 1.0f)) return false;
    float alpha = 1.0f - beta - gamma;
    if (!(alpha > lower)) return false;
    float detT = (A * E * N) + (D * H * K) + (G * B * M) - (K * E * G) - (M * H * A) - (N * B * D);
    const float st = detM < 0.0f ? -detT : detT;
    if (eps >= 0.0f && !(st > 0.0f)) return false;                // t <= 0 <= eps
    if (st >= tmax * 1.0001f * am) return false;                   // t >= tmax
    float t = detT / detM;
    if (!(t > eps && t < tmax)) return false;
    t_out = t;
    beta_out = beta;
    gamma_out = gamma;
    return true;
}

// Watertight ray/triangle test (Woop, Benthin, Wald, "Watertight Ray/Triangle
// Intersection", JCGT 2(1), 2013), the production alternative to azimuth's
// Cramer test (AZ_FLAG_WATERTIGHT).  The ray is sheared once so that it runs
// along +z; a triangle's vertices, taken relative to the origin and sheared
// the same way, give three 2D edge functions whose signs decide the hit.
// Neighbouring triangles compute the edge functions of a shared edge from the
// same vertex bits with the same operations, so the values are exact
// negatives of each other and no ray passes between them; a zero edge value
// is recomputed in double precision.  Every product and sum below is an
// explicit round-to-nearest operation, never fused.
struct WtRay {
    uint32_t kx, ky, kz;   // the axes of the sheared frame; kz = largest |d|
    float sx, sy, sz;      // shear d[kx]/d[kz], d[ky]/d[kz] and scale 1/d[kz]
};

__device__ __forceinline__ WtRay wt_setup(f3 d) {
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    WtRay w;
    w.kz = ax > ay ? (ax > az ? 0u : 2u) : (ay > az ? 1u : 2u);
    w.kx = w.kz == 2u ? 0u : w.kz + 1u;
    w.ky = w.kx == 2u ? 0u : w.kx + 1u;
    const float dz = comp(d, (int)w.kz);
    if (dz < 0.0f) {   // keep the winding: swap the other two axes
        const uint32_t k = w.kx;
        w.kx = w.ky;
        w.ky = k;
    }
    w.sx = comp(d, (int)w.kx) / dz;
    w.sy = comp(d, (int)w.ky) / dz;
    w.sz = 1.0f / dz;
    return w;
}

__device__ __forceinline__ bool tri_test_wt(const DevTriVerts &v, const Ray &r, const WtRay &w, bool cull, float eps,
                                            float tmax, float &t_out) {
    if (cull) {
        f3 fn = mk(v.c.y, v.c.z, v.c.w);
        if (!(dot(r.d, fn) < 0.0f)) return false;   // azimuth's back-face rule
    }
    const f3 A = mk(__fsub_rn(v.a.x, r.o.x), __fsub_rn(v.a.y, r.o.y), __fsub_rn(v.a.z, r.o.z));
    const f3 B = mk(__fsub_rn(v.a.w, r.o.x), __fsub_rn(v.b.x, r.o.y), __fsub_rn(v.b.y, r.o.z));
    const f3 C = mk(__fsub_rn(v.b.z, r.o.x), __fsub_rn(v.b.w, r.o.y), __fsub_rn(v.c.x, r.o.z));
    const float Az = comp(A, (int)w.kz), Bz = comp(B, (int)w.kz), Cz = comp(C, (int)w.kz);
    const float Ax = __fsub_rn(comp(A, (int)w.kx), __fmul_rn(w.sx, Az));
    const float Ay = __fsub_rn(comp(A, (int)w.ky), __fmul_rn(w.sy, Az));
    const float Bx = __fsub_rn(comp(B, (int)w.kx), __fmul_rn(w.sx, Bz));
    const float By = __fsub_rn(comp(B, (int)w.ky), __fmul_rn(w.sy, Bz));
    const float Cx = __fsub_rn(comp(C, (int)w.kx), __fmul_rn(w.sx, Cz));
    const float Cy = __fsub_rn(comp(C, (int)w.ky), __fmul_rn(w.sy, Cz));
    float U = __fsub_rn(__fmul_rn(Cx, By), __fmul_rn(Cy, Bx));
    float V = __fsub_rn(__fmul_rn(Ax, Cy), __fmul_rn(Ay, Cx));
    float W = __fsub_rn(__fmul_rn(Bx, Ay), __fmul_rn(By, Ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        // on an edge in float: decide in double, where these products are exact
        U = (float)__dsub_rn(__dmul_rn((double)Cx, (double)By), __dmul_rn((double)Cy, (double)Bx));
        V = (float)__dsub_rn(__dmul_rn((double)Ax, (double)Cy), __dmul_rn((double)Ay, (double)Cx));
        W = (float)__dsub_rn(__dmul_rn((double)Bx, (double)Ay), __dmul_rn((double)By, (double)Ax));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = __fadd_rn(__fadd_rn(U, V), W);
    if (det == 0.0f) return false;
    const float T = __fadd_rn(__fadd_rn(__fmul_rn(U, __fmul_rn(w.sz, Az)), __fmul_rn(V, __fmul_rn(w.sz, Bz))),
                              __fmul_rn(W, __fmul_rn(w.sz, Cz)));
    const float t = T / det;
    if (!(t > eps && t < tmax)) return false;
    t_out = t;
    return true;
}

__device__ __forceinline__ DevTriVerts load_tri_verts(const DevTriVerts *v, uint32_t i) {
    const float4 *p = reinterpret_cast<const float4 *>(v + i);
    DevTriVerts t;
    t.a = __ldg(p + 0);
    t.b = __ldg(p + 1);
    t.c = __ldg(p + 2);
    return t;
}

// Reciprocal direction for the box tests; components are kept at most 1e18
// in magnitude so that 2^23 * grid step * 1/d stays finite.
__device__ __forceinline__ f3 safe_inv(f3 d) {
    const float tiny = 1e-18f;
    float x = fabsf(d.x) < tiny ? copysignf(tiny, d.x) : d.x;
    float y = fabsf(d.y) < tiny ? copysignf(tiny, d.y) : d.y;
    float z = fabsf(d.z) < tiny ? copysignf(tiny, d.z) : d.z;
    return mk(1.0f / x, 1.0f / y, 1.0f / z);
}

// Three-input max and min (exact, order-independent like fmaxf / fminf).
__device__ __forceinline__ float max3f(float a, float b, float c) {
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

__device__ __forceinline__ DevTri load_tri(const DevTri *tris, uint32_t i) {
    const float4 *p = reinterpret_cast<const float4 *>(tris + i);
    DevTri t;
    t.a = __ldg(p + 0);
    t.b = __ldg(p + 1);
    t.c = __ldg(p + 2);
    return t;
}

enum QueryKind : uint32_t {
    Q_CLOSEST = 0,   // nearest hit
    Q_ANY = 1        // any hit with world t < tmax (early exit)
};

// A valid hierarchy needs far fewer steps; the cap only guards against a
// corrupt one looping forever.  When hit, the query stops and sets *err.
#define AZD_MAX_STEPS (1u << 22)
#define AZD_WSTACK 48

// Stack entries (uint2): .x a base index, .y the kind in its top two bits
//   node group      .y = imask << 8 | hit bits (bit = slot ^ octant)
//   primitive group .y = AZD_E_PRIMS | 24-bit mask of untested primitives after .x
//   BLAS exit       .y = AZD_E_EXIT
//   BLAS entry      .y = AZD_E_GROUP, .x = group index
#define AZD_E_EXIT 0xFFFFFFFFu
#define AZD_E_GROUP 0xFFFFFFFEu
#define AZD_E_PRIMS 0x40000000u

// 8-bit grid value q as the float 2^23 + q: PRMT places the byte in the low
// mantissa bits of 2^23 (exact).  The slab test subtracts the 2^23 inside its
// FMA (see wide_test).
__device__ __forceinline__ float qbyte_biased(uint32_t w, uint32_t k) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7540u | k));
}

struct WideHits {
    uint32_t inner;   // hit inner children, bit = slot ^ octant
    uint32_t prims;   // hit leaf primitives, bit = offset from prim_base
};

// Slab test of the 8 quantised child boxes of a wide node.
__device__ __forceinline__ WideHits wide_test(const uint4 w0, const uint4 w1, const uint4 w2, const uint4 w3,
                                              const uint4 w4, f3 o, f3 inv, uint32_t oct, float tmax) {
    const float px = __uint_as_float(w0.x), py = __uint_as_float(w0.y), pz = __uint_as_float(w0.z);
    const uint32_t ex = w0.w & 0xFFu, ey = (w0.w >> 8) & 0xFFu, ez = (w0.w >> 16) & 0xFFu, imask = w0.w >> 24;
    const float sx = __uint_as_float(ex << 23) * inv.x, sy = __uint_as_float(ey << 23) * inv.y,
                sz = __uint_as_float(ez << 23) * inv.z;
    // Plane distance (p + q * step - o) * inv = q * s + o', computed as
    // fma(2^23 + q, s, o' - 2^23 * s): the 2^23 * s terms cancel exactly (the
    // same rounded s in both), so the only cost of the fold is the rounding of
    // o' - 2^23 * s, at most half a grid step in t; the collapse leaves a full
    // step of slack around every child box (az_wide_bvh.cu).
    const float ox = __fmaf_rn(-8388608.0f, sx, (px - o.x) * inv.x);
    const float oy = __fmaf_rn(-8388608.0f, sy, (py - o.y) * inv.y);
    const float oz = __fmaf_rn(-8388608.0f, sz, (pz - o.z) * inv.z);
    // near/far planes: swap lo and hi when the direction is negative
    const bool nx = inv.x < 0.0f, ny = inv.y < 0.0f, nz = inv.z < 0.0f;
    const uint32_t nx0 = nx ? w3.z : w2.x, nx1 = nx ? w3.w : w2.y, fx0 = nx ? w2.x : w3.z, fx1 = nx ? w2.y : w3.w;
    const uint32_t ny0 = ny ? w4.x : w2.z, ny1 = ny ? w4.y : w2.w, fy0 = ny ? w2.z : w4.x, fy1 = ny ? w2.w : w4.y;
    const uint32_t nz0 = nz ? w4.z : w3.x, nz1 = nz ? w4.w : w3.y, fz0 = nz ? w3.x : w4.z, fz1 = nz ? w3.y : w4.w;
    WideHits h{0u, 0u};
#pragma unroll
    for (int s = 0; s < 8; s++) {
        const uint32_t k = s & 3;
        const float tnx = __fmaf_rn(qbyte_biased(s < 4 ? nx0 : nx1, k), sx, ox);
        const float tfx = __fmaf_rn(qbyte_biased(s < 4 ? fx0 : fx1, k), sx, ox);
        const float tny = __fmaf_rn(qbyte_biased(s < 4 ? ny0 : ny1, k), sy, oy);
        const float tfy = __fmaf_rn(qbyte_biased(s < 4 ? fy0 : fy1, k), sy, oy);
        const float tnz = __fmaf_rn(qbyte_biased(s < 4 ? nz0 : nz1, k), sz, oz);
        const float tfz = __fmaf_rn(qbyte_biased(s < 4 ? fz0 : fz1, k), sz, oz);
        const float tn = fmaxf(max3f(tnx, tny, tnz), 0.0f);
        const float tf = fminf(min3f(tfx, tfy, tfz), tmax) * 1.00000095367431640625f;
        if (tn <= tf) {
            if ((imask >> s) & 1u) {
                h.inner |= 1u << (s ^ oct);
            } else {
                const uint32_t meta = ((s < 4 ? w1.z : w1.w) >> (8 * k)) & 0xFFu;
                h.prims |= ((1u << (meta >> 5)) - 1u) << (meta & 31u);   // empty slot: meta 0, no bits
            }
        }
    }
    return h;
}

// The next child of a node group to visit.  A hit bit is the child's slot
// XOR the ray's direction octant, so the lowest bit is the child nearest the
// ray origin.  Closest-hit queries go near first (pruning by the nearest hit
// so far); any-hit queries go far first: a visibility ray starts on a surface
// whose own neighbourhood seldom blocks it, and its occluders lie between the
// surface and the light (C1 frame 336 -> 330 ms, C3 562 -> 521 ms in the same
// launch configuration; the answer does not depend on the order).
template <QueryKind KIND>
__device__ __forceinline__ uint32_t child_key(uint32_t hits) {
    return KIND == Q_ANY ? 31u - __clz(hits) : __ffs(hits) - 1u;
}

__device__ __forceinline__ uint32_t octant_of(f3 d) {
    return (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
}

// World t of a triangle hit of group g at local t (azimuth's instance path,
// src/azimuth_main.cpp:256-262).
__device__ __forceinline__ float group_world_t(const DevGroup &g, const Ray &wr, const Ray &lr, float t) {
    if (g.raw) return t;
    if (g.identity) {
        // point_xf of the identity returns the point (x * 1 + y * 0 + z * 0 + 0
        // is x) and the motion is zero: the same world t without the products
        const f3 lp = lr.o + (lr.d * t);
        return length(lp - wr.o) / length(wr.d);
    }
    f3 motion = wr.time * mk(g.motion[0], g.motion[1], g.motion[2]);
    f3 o2 = wr.o - motion;
    f3 lp = lr.o + (lr.d * t);
    f3 wp = point_xf(g.xf, lp) + motion;
    return length(wp - o2 - motion) / length(wr.d);
}

// Factor from a world distance along d to the group's local distance
// (|inv * d| / |d|) with a margin of 1e-4 for rounding; exactly 1.0001 for an
// identity group, whose vector transform returns d unchanged.
__device__ __forceinline__ float group_t_scale(const DevGroup &g, f3 d) {
    if (g.identity) return 1.0001f;
    return length(vector_xf(g.inv, d)) / length(d) * 1.0001f;
}

// The traversal loops call the rarely taken paths below out of line, with
// values and global pointers only, so that the loops' own code stays small
// (the instruction cache of an SM holds the hot loop; a scene's spheres,
// transformed instances and entity lights take these calls).

// sphere_test of entity e for the world ray: out of line, or inline (INL)
// in the kernels that serve scenes with spheres at the top level.
struct SphereHit {
    float t_world, t_local;
    uint32_t hit;
};
static __device__ __noinline__ SphereHit sphere_test_call(const DevEntity *e, Ray wr, float eps) {
    SphereHit h;
    h.t_world = h.t_local = FLT_MAX;
    h.hit = sphere_test(*e, wr, eps, h.t_world, h.t_local) ? 1u : 0u;
    return h;
}
template <bool INL>
__device__ __forceinline__ SphereHit sphere_hit(const DevEntity *e, const Ray &wr, float eps) {
    if (!INL) return sphere_test_call(e, wr, eps);
    SphereHit h;
    h.t_world = h.t_local = FLT_MAX;
    h.hit = sphere_test(*e, wr, eps, h.t_world, h.t_local) ? 1u : 0u;
    return h;
}

// The local ray of a transformed, possibly moving group (GetLocalRay of the
// motion-shifted ray) and the group_t_scale of the world direction.
struct GroupRay {
    Ray r;
    float scale;
};
static __device__ __noinline__ GroupRay group_ray_call(const DevGroup *gp, Ray wr) {
    const DevGroup &g = *gp;
    Ray m = wr;
    m.o = wr.o - wr.time * mk(g.motion[0], g.motion[1], g.motion[2]);
    GroupRay out;
    out.r = local_ray(m, g.inv);
    out.scale = group_t_scale(g, wr.d);
    return out;
}

// Two-level traversal of the 8-wide hierarchy, after the node-group /
// primitive-group scheme of Ylitie, Karras, Laine, "Efficient Incoherent Ray
// Traversal on GPUs Through Compressed Wide BVHs" (HPG 2017): each step
// visits the nearest node of the current group, then tests the primitives its
// leaves hit, postponing them onto the stack while few lanes of the warp have
// primitives to test.  The traversal is a resumable state machine (init, then
// step() until it reports the query finished) so that persistent kernels can
// hand a lane a new ray as soon as its query ends.
//
// Q_CLOSEST: nearest hit in `best` (best.ent == 0xFFFFFFFF: none).
// Q_ANY: `hit_any` is set as soon as a primitive's world t < tmax.
// `skip_ent` is an entity whose primitives are ignored (0xFFFFFFFF: none).
template <QueryKind KIND, bool WT = false>
__device__ bool trace(const DevScene &S, const Ray &wr, bool cull, float eps, float tmax, Hit &best,
                      uint32_t *counts = nullptr, uint32_t *err = nullptr, uint32_t skip_ent = 0xFFFFFFFFu);

// POP_FIRST: a step that starts with both current groups empty pops the
// stack until it holds a node or primitive group and visits it in the same
// step (a finished query is reported at the end of its last step); otherwise
// a step ends with the pop and the popped group waits for the next step.
// WT: triangles by the watertight test instead of azimuth's Cramer test.
// SPH: the top-level sphere test inline (scenes with spheres at the top
// level); otherwise it is called out of line.
template <QueryKind KIND, bool POP_FIRST = false, bool WT = false, bool SPH = false>
struct Tracer {
    static constexpr uint32_t kNoNode = 0xFFFFFFFFu;
    Ray wr;                    // world ray
    Ray r;                     // ray in the current space (world or a group's local space)
    f3 inv;
    uint32_t oct;
    float tcur;                // pruning distance in the current space
    float tmax, eps;
    bool cull, in_blas, hit_any;
    uint32_t skip_ent, g_idx;
    float bl_t;                // nearest local hit of this BLAS visit
    uint32_t bl_prim;
    uint32_t ng_base, ng_bits; // current node group
    uint32_t pg_base, pg_mask; // current primitive group
    uint32_t steps, nodes_visited, prims_visited;
    int sp;
    Hit best;
    WtRay wt;                  // WT: shear of the current ray space

    // `stack`: the query's stack (AZD_WSTACK entries), which a scene whose top
    // level is a single group starts with that group's exit marker.
    __device__ __forceinline__ void init(const DevScene &S, const Ray &ray, bool cull_, float eps_, float tmax_,
                                         uint2 *stack, uint32_t skip = 0xFFFFFFFFu) {
        wr = ray;
        r = ray;
        tmax = tmax_;
        eps = eps_;
        cull = cull_;
        tcur = KIND == Q_ANY ? tmax_ : FLT_MAX;
        in_blas = false;
        hit_any = false;
        skip_ent = skip;
        g_idx = 0;
        bl_t = FLT_MAX;
        bl_prim = 0xFFFFFFFFu;
        pg_base = 0;
        pg_mask = 0;
        steps = nodes_visited = prims_visited = 0;
        sp = 0;
        best.t = FLT_MAX;
        best.tl = 0.0f;
        best.prim = 0xFFFFFFFFu;
        best.ent = 0xFFFFFFFFu;
        if (S.tlas_single_group != 0xFFFFFFFFu) {
            // a top level holding one group only: enter its hierarchy directly
            // (the top-level root test and the group's leaf would only lead there)
            inv = mk(0.0f, 0.0f, 0.0f);
            oct = 0u;
            ng_base = 0u;
            ng_bits = 0u;
            enter_group(S, stack, S.tlas_single_group);
        } else {
            // current node group: the root alone (imask bit 0, hit bit 0 ^ oct)
            inv = safe_inv(r.d);
            oct = octant_of(r.d);
            if (WT) wt = wt_setup(r.d);
            ng_base = S.tlas_root;
            ng_bits = S.tlas_root == 0xFFFFFFFFu ? 0u : ((1u << 8) | (1u << oct));
        }
    }

    // Enters group gi's bottom-level hierarchy (azimuth: GetLocalRay of the
    // motion-shifted ray, src/azimuth_main.cpp:246-250); its exit marker goes on
    // the stack (room for it is kept when a group entry is pushed).
    __device__ __forceinline__ void enter_group(const DevScene &S, uint2 *stack, uint32_t gi) {
        g_idx = gi;
        const DevGroup &g = S.groups[g_idx];
        if (g.root == 0xFFFFFFFFu) return;
        stack[sp++] = make_uint2(0u, AZD_E_EXIT);
        const float wlim = KIND == Q_ANY ? tmax : best.t;
        tcur = FLT_MAX;
        if (g.raw) {
            r = wr;
            if (wlim < FLT_MAX) tcur = wlim + 1e-30f;
        } else if (g.identity) {
            r = local_ray_identity(wr);
            if (wlim < FLT_MAX) tcur = wlim * 1.0001f + 1e-30f;
        } else {
            const GroupRay gr = group_ray_call(S.groups + g_idx, wr);
            r = gr.r;
            if (wlim < FLT_MAX) tcur = wlim * gr.scale + 1e-30f;
        }
        inv = safe_inv(r.d);
        oct = octant_of(r.d);
        if (WT) wt = wt_setup(r.d);
        bl_t = FLT_MAX;
        bl_prim = 0xFFFFFFFFu;
        in_blas = true;
        ng_base = g.root;
        ng_bits = (1u << 8) | (1u << oct);
    }

    __device__ __forceinline__ void push(uint2 *stack, uint32_t x, uint32_t y, uint32_t *err) {
        if (sp < AZD_WSTACK) stack[sp++] = make_uint2(x, y);
        else if (err) atomicOr(err, 2u);
    }

    // Takes the top stack entry: leaves or enters a bottom-level hierarchy, or
    // makes the entry the current primitive or node group.
    __device__ __forceinline__ void pop(const DevScene &S, uint2 *stack) {
        const uint2 e = stack[--sp];
        if (e.y == AZD_E_EXIT) {
            // leaving a BLAS: azimuth's instance path keeps the nearest local hit
            // and recomputes its world t (src/azimuth_main.cpp:256-276)
            if (KIND == Q_CLOSEST && bl_prim != 0xFFFFFFFFu) {
                float wt_ = group_world_t(S.groups[g_idx], wr, r, bl_t);
                if (wt_ > eps && wt_ < best.t) {
                    best.t = wt_;
                    best.tl = bl_t;
                    best.prim = bl_prim;
                    best.ent = S.tri_attr[bl_prim].entity;
                }
            }
            in_blas = false;
            if (sp == 0) return;   // the query is done: no world-space traversal follows
            r = wr;
            inv = safe_inv(r.d);
            oct = octant_of(r.d);
            if (WT) wt = wt_setup(r.d);
            tcur = KIND == Q_ANY ? tmax : best.t;
        } else if (e.y == AZD_E_GROUP) {
            enter_group(S, stack, e.x);   // its exit marker reuses the popped entry's slot
        } else if ((e.y & 0xC0000000u) == AZD_E_PRIMS) {
            pg_base = e.x;
            pg_mask = e.y & 0x00FFFFFFu;
        } else {
            ng_base = e.x;
            ng_bits = e.y;
        }
    }

    // One step: visit the nearest node of the current group and test the
    // primitives it hits, and pop the stack when both groups are empty.
    // Returns true when finished.  The stack (AZD_WSTACK entries) is a
    // separate array of the caller so that the state above stays in registers.
    __device__ __forceinline__ bool step(const DevScene &S, uint2 *stack, uint32_t *err) {
        uint32_t node;
        if (begin(S, stack, err, node)) return true;
        uint4 w[5];
        if (node != kNoNode) {
            const uint4 *np = reinterpret_cast<const uint4 *>(S.wnodes + node);
#pragma unroll
            for (int k = 0; k < 5; k++) w[k] = __ldg(np + k);
        }
        return finish(S, stack, err, node, w);
    }

    // The first half of a step: the step count, the pops of a pop-first
    // tracer, and the choice of the node to visit (`node`, kNoNode when the
    // step visits none).  Returns true when the query is finished.  A caller
    // that fetches the node itself (stage_nodes) runs begin, the fetch, then
    // finish.
    __device__ __forceinline__ bool begin(const DevScene &S, uint2 *stack, uint32_t *err, uint32_t &node) {
        node = kNoNode;
        if (++steps > AZD_MAX_STEPS) {
            if (err) atomicOr(err, 1u);
            return true;
        }
        if (POP_FIRST) {
            while (!(ng_bits & 0xFFu) && !pg_mask) {
                if (sp == 0) return true;
                pop(S, stack);
            }
        }
        if (ng_bits & 0xFFu) {
            const uint32_t hits = ng_bits & 0xFFu, imask = (ng_bits >> 8) & 0xFFu;
            const uint32_t key = child_key<KIND>(hits);
            const uint32_t slot = key ^ oct;
            node = ng_base + __popc(imask & ((1u << slot) - 1u));
            ng_bits &= ~(1u << key);
            if (ng_bits & 0xFFu) push(stack, ng_base, ng_bits, err);
        }
        return false;
    }

    // The second half: the eight child tests of `node` (w: its five 16-byte
    // words), the primitives, and the pop of exhausted groups.  Returns true
    // when the query is finished.
    __device__ __forceinline__ bool finish(const DevScene &S, uint2 *stack, uint32_t *err, uint32_t node,
                                           const uint4 (&w)[5]) {
        if (node != kNoNode) {
            nodes_visited++;
            const WideHits h = wide_test(w[0], w[1], w[2], w[3], w[4], r.o, inv, oct, tcur);
            ng_base = w[1].x;
            ng_bits = h.inner | ((w[0].w >> 24) << 8);
            if (h.prims) {
                if (pg_mask) push(stack, pg_base, AZD_E_PRIMS | pg_mask, err);   // keep the older group for later
                pg_base = w[1].y;
                pg_mask = h.prims;
            }
        }
        // primitives, postponed while few lanes of the warp have any
        while (pg_mask) {
            if (__popc(__activemask()) < 6u && (ng_bits & 0xFFu) && sp < AZD_WSTACK) {
                stack[sp++] = make_uint2(pg_base, AZD_E_PRIMS | pg_mask);
                pg_mask = 0;
                break;
            }
            const uint32_t bit = __ffs(pg_mask) - 1u;
            pg_mask &= pg_mask - 1u;
            const uint32_t pi = pg_base + bit;
            prims_visited++;
            if (in_blas) {
                float t, b, gm;
                bool hit;
                if (WT) {
                    hit = tri_test_wt(load_tri_verts(S.tri_verts, pi), r, wt, cull, eps, bl_t, t);
                } else {
                    hit = tri_test(load_tri(S.tris, pi), r, cull, eps, bl_t, t, b, gm);
                }
                if (hit) {
                    // a primitive of the skipped entity is ignored; its owner is
                    // looked up only for the few primitives that are hit
                    if (skip_ent != 0xFFFFFFFFu && __ldg(&S.tri_attr[pi].entity) == skip_ent) continue;
                    bl_t = t;
                    bl_prim = pi;
                    if (KIND == Q_ANY) {
                        // finished as soon as one hit of this group is in range
                        float wt = group_world_t(S.groups[g_idx], wr, r, t);
                        if (wt > eps && wt < tmax) {
                            hit_any = true;
                            return true;
                        }
                    } else {
                        tcur = fminf(tcur, t);
                    }
                }
            } else {
                const uint32_t p = __ldg(S.tlas_prims + pi);
                if (p & AZD_TLAS_GROUP) {
                    push(stack, p & ~AZD_TLAS_GROUP, AZD_E_GROUP, err);   // entered when popped
                } else if (p != skip_ent && S.ents[p].type == ENT_SPHERE) {
                    const SphereHit sh = sphere_hit<SPH>(S.ents + p, wr, eps);
                    if (sh.hit) {
                        if (KIND == Q_ANY) {
                            if (sh.t_world < tmax) {
                                hit_any = true;
                                return true;
                            }
                        } else if (sh.t_world < best.t) {
                            best.t = sh.t_world;
                            best.tl = sh.t_local;
                            best.prim = 0xFFFFFFFFu;
                            best.ent = p;
                            tcur = sh.t_world;
                        }
                    }
                }
            }
        }
        if ((ng_bits & 0xFFu) || pg_mask) return false;
        // nothing left in the current groups: pop (or, popping first, let the
        // next step pop; a leftover BLAS exit marker must still be taken)
        if (sp == 0) return true;
        if (POP_FIRST) return false;
        pop(S, stack);
        return false;
    }

    __device__ __forceinline__ void flush_counts(uint32_t *counts) const {
        if (counts) {
            atomicAdd(counts + 0, nodes_visited);
            atomicAdd(counts + 1, prims_visited);
        }
    }
};

// Node fetch staged through shared memory, called by all 32 lanes of a warp
// between Tracer::begin and Tracer::finish.  The nodes that the lanes visit
// this step (node: kNoNode for none) are loaded together: 16-byte word c of
// the warp's list (word c % 5 of lane c / 5's node) is read by lane c % 32 in
// round c / 32, so five neighbouring lanes read one node's 80 contiguous bytes
// instead of every lane reading 16 bytes of its own node per instruction;
// each lane then takes its node's five words from `stage` (the warp's 160
// words of shared memory).
__device__ __forceinline__ void stage_nodes(const WideNode *nodes, uint32_t node, uint4 *stage, uint4 (&w)[5]) {
    constexpr uint32_t kNone = 0xFFFFFFFFu;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t want = __ballot_sync(0xFFFFFFFFu, node != kNone);
    if (!want) return;
    const uint4 *base = reinterpret_cast<const uint4 *>(nodes);
#pragma unroll
    for (uint32_t it = 0; it < 5; it++) {
        const uint32_t c = 32u * it + lane, j = c / 5u, part = c - 5u * j;
        const uint32_t nj = __shfl_sync(0xFFFFFFFFu, node, j);
        if ((want >> j) & 1u) stage[c] = __ldg(base + (size_t)nj * 5u + part);
    }
    __syncwarp();
    if (node != kNone) {
#pragma unroll
        for (int k = 0; k < 5; k++) w[k] = stage[5u * lane + k];
    }
    __syncwarp();   // the stage is free for the next step
}

// A whole query in one loop: the same traversal as Tracer written as a single
// function, which the compiler schedules better when one thread runs one
// query to its end (grid-stride kernels).  For Q_CLOSEST returns whether
// something was hit and the nearest hit in `best`; for Q_ANY returns whether a
// primitive lies closer than tmax.  `skip_ent` is an entity whose primitives
// are ignored; `counts` accumulates node and primitive visits.
template <QueryKind KIND, bool WT>
__device__ bool trace(const DevScene &S, const Ray &wr, bool cull, float eps, float tmax, Hit &best,
                      uint32_t *counts, uint32_t *err, uint32_t skip_ent) {
    best.t = FLT_MAX;
    best.tl = 0.0f;
    best.prim = 0xFFFFFFFFu;
    best.ent = 0xFFFFFFFFu;
    if (S.tlas_root == 0xFFFFFFFFu) return false;

    uint2 stack[AZD_WSTACK];
    int sp = 0;

    Ray r = wr;                                    // current ray space
    const bool single = S.tlas_single_group != 0xFFFFFFFFu;
    f3 inv = single ? mk(0.0f, 0.0f, 0.0f) : safe_inv(r.d);   // a single group sets its own
    uint32_t oct = single ? 0u : octant_of(r.d);
    WtRay wt;                                      // WT: shear of the current ray space
    if (WT && !single) wt = wt_setup(r.d);
    float tcur = KIND == Q_ANY ? tmax : FLT_MAX;   // pruning distance in the current space
    bool in_blas = false;
    uint32_t g_idx = 0;
    float bl_t = FLT_MAX;                          // nearest local hit of this BLAS visit
    uint32_t bl_prim = 0xFFFFFFFFu;
    uint32_t nodes_visited = 0, prims_visited = 0, steps = 0;
    bool hit_any = false;

    // current node group: the root alone (imask bit 0, hit bit 0 ^ oct)
    uint32_t ng_base = S.tlas_root, ng_bits = (1u << 8) | (1u << oct);
    uint32_t pg_base = 0, pg_mask = 0;             // current primitive group
    if (single) {
        // a top level holding one group only: start with its entry on the stack
        ng_bits = 0u;
        stack[sp++] = make_uint2(S.tlas_single_group, AZD_E_GROUP);
    }

    while (true) {
        if (++steps > AZD_MAX_STEPS) {
            if (err) atomicOr(err, 1u);
            break;
        }
        if (ng_bits & 0xFFu) {
            // visit the nearest node of the group; the rest of the group waits on the stack
            const uint32_t hits = ng_bits & 0xFFu, imask = (ng_bits >> 8) & 0xFFu;
            const uint32_t key = child_key<KIND>(hits);
            const uint32_t slot = key ^ oct;
            const uint32_t node = ng_base + __popc(imask & ((1u << slot) - 1u));
            ng_bits &= ~(1u << key);
            if (ng_bits & 0xFFu) {
                if (sp < AZD_WSTACK) stack[sp++] = make_uint2(ng_base, ng_bits);
                else if (err) atomicOr(err, 2u);
            }
            const uint4 *np = reinterpret_cast<const uint4 *>(S.wnodes + node);
            const uint4 w0 = __ldg(np + 0), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3),
                        w4 = __ldg(np + 4);
            nodes_visited++;
            const WideHits h = wide_test(w0, w1, w2, w3, w4, r.o, inv, oct, tcur);
            ng_base = w1.x;
            ng_bits = h.inner | ((w0.w >> 24) << 8);
            if (h.prims) {
                if (pg_mask) {   // still holding primitives: keep them for later
                    if (sp < AZD_WSTACK) stack[sp++] = make_uint2(pg_base, AZD_E_PRIMS | pg_mask);
                    else if (err) atomicOr(err, 2u);
                }
                pg_base = w1.y;
                pg_mask = h.prims;
            }
        }
        // primitives, postponed while few lanes of the warp have any
        while (pg_mask) {
            if (__popc(__activemask()) < 6u && (ng_bits & 0xFFu) && sp < AZD_WSTACK) {
                stack[sp++] = make_uint2(pg_base, AZD_E_PRIMS | pg_mask);
                pg_mask = 0;
                break;
            }
            const uint32_t bit = __ffs(pg_mask) - 1u;
            pg_mask &= pg_mask - 1u;
            const uint32_t pi = pg_base + bit;
            prims_visited++;
            if (in_blas) {
                float t, b, gm;
                bool hit;
                if (WT) {
                    hit = tri_test_wt(load_tri_verts(S.tri_verts, pi), r, wt, cull, eps, bl_t, t);
                } else {
                    hit = tri_test(load_tri(S.tris, pi), r, cull, eps, bl_t, t, b, gm);
                }
                if (hit) {
                    // a primitive of the skipped entity is ignored; its owner is
                    // looked up only for the few primitives that are hit
                    if (skip_ent != 0xFFFFFFFFu && __ldg(&S.tri_attr[pi].entity) == skip_ent) continue;
                    bl_t = t;
                    bl_prim = pi;
                    if (KIND == Q_ANY) {
                        // exit as soon as one hit of this group is in range
                        float wt = group_world_t(S.groups[g_idx], wr, r, t);
                        if (wt > eps && wt < tmax) {
                            hit_any = true;
                            break;
                        }
                    } else {
                        tcur = fminf(tcur, t);
                    }
                }
            } else {
                const uint32_t p = __ldg(S.tlas_prims + pi);
                if (p & AZD_TLAS_GROUP) {
                    // entered when popped; leave room for its exit marker
                    if (sp + 1 < AZD_WSTACK) stack[sp++] = make_uint2(p & ~AZD_TLAS_GROUP, AZD_E_GROUP);
                    else if (err) atomicOr(err, 2u);
                } else if (p != skip_ent && S.ents[p].type == ENT_SPHERE) {
                    const SphereHit sh = sphere_hit<true>(S.ents + p, wr, eps);
                    if (sh.hit) {
                        if (KIND == Q_ANY) {
                            if (sh.t_world < tmax) {
                                hit_any = true;
                                break;
                            }
                        } else if (sh.t_world < best.t) {
                            best.t = sh.t_world;
                            best.tl = sh.t_local;
                            best.prim = 0xFFFFFFFFu;
                            best.ent = p;
                            tcur = sh.t_world;
                        }
                    }
                }
            }
        }
        if (KIND == Q_ANY && hit_any) break;
        if ((ng_bits & 0xFFu) || pg_mask) continue;
        // nothing left in the current groups: pop
        if (sp == 0) break;
        const uint2 e = stack[--sp];
        if (e.y == AZD_E_EXIT) {
            // leaving a BLAS: azimuth's instance path keeps the nearest local hit
            // and recomputes its world t (src/azimuth_main.cpp:256-276)
            if (KIND == Q_CLOSEST && bl_prim != 0xFFFFFFFFu) {
                float wt = group_world_t(S.groups[g_idx], wr, r, bl_t);
                if (wt > eps && wt < best.t) {
                    best.t = wt;
                    best.tl = bl_t;
                    best.prim = bl_prim;
                    best.ent = S.tri_attr[bl_prim].entity;
                }
            }
            r = wr;
            inv = safe_inv(r.d);
            oct = octant_of(r.d);
            if (WT) wt = wt_setup(r.d);
            tcur = KIND == Q_ANY ? tmax : best.t;
            in_blas = false;
        } else if (e.y == AZD_E_GROUP) {
            // enter the group's BLAS (azimuth: GetLocalRay of the motion-shifted
            // ray, src/azimuth_main.cpp:246-250)
            g_idx = e.x;
            const DevGroup &g = S.groups[g_idx];
            if (g.root == 0xFFFFFFFFu) continue;
            stack[sp++] = make_uint2(0u, AZD_E_EXIT);   // room was kept when the entry was pushed
            const float wlim = KIND == Q_ANY ? tmax : best.t;
            tcur = FLT_MAX;
            if (g.raw) {
                r = wr;
                if (wlim < FLT_MAX) tcur = wlim + 1e-30f;
            } else if (g.identity) {
                r = local_ray_identity(wr);
                if (wlim < FLT_MAX) tcur = wlim * 1.0001f + 1e-30f;
            } else {
                const GroupRay gr = group_ray_call(S.groups + g_idx, wr);
                r = gr.r;
                if (wlim < FLT_MAX) tcur = wlim * gr.scale + 1e-30f;
            }
            inv = safe_inv(r.d);
            oct = octant_of(r.d);
            if (WT) wt = wt_setup(r.d);
            bl_t = FLT_MAX;
            bl_prim = 0xFFFFFFFFu;
            in_blas = true;
            ng_base = g.root;
            ng_bits = (1u << 8) | (1u << oct);
        } else if ((e.y & 0xC0000000u) == AZD_E_PRIMS) {
            pg_base = e.x;
            pg_mask = e.y & 0x00FFFFFFu;
        } else {
            ng_base = e.x;
            ng_bits = e.y;
        }
    }
    if (counts) {
        atomicAdd(counts + 0, nodes_visited);
        atomicAdd(counts + 1, prims_visited);
    }
    if (KIND == Q_ANY) return hit_any;
    return best.ent != 0xFFFFFFFFu;
}

}  // namespace azd
