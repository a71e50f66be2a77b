// Closest-hit and occlusion queries on the device scene.
//
// Primitive tests reproduce azimuth's arithmetic exactly (same operation
// order, IEEE rounding, no contraction): the Cramer triangle test
// (src/azimuth_main.cpp:147-243), the transformed, moving sphere
// (:64-146) and the mesh-instance path (:244-281: motion, GetLocalRay with a
// re-normalised direction, world t recomputed from the local hit point).
// The hierarchy is this library's own BVH, traversed near-first with
// t-pruning on conservative boxes; it finds the same nearest primitive as
// azimuth's exhaustive BVH walk except for exact ties and rays that graze a
// box azimuth's slab test rejects.
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
    float beta = detB / detM;
    if (!(beta > lower && beta <= 1.0f)) return false;
    float detG = (A * M * I) + (D * N * C) + (G * K * F) - (C * M * G) - (F * N * A) - (I * K * D);
    float gamma = detG / detM;
    if (!(gamma > lower && gamma <= 1.0f)) return false;
    float alpha = 1.0f - beta - gamma;
    if (!(alpha > lower)) return false;
    float detT = (A * E * N) + (D * H * K) + (G * B * M) - (K * E * G) - (M * H * A) - (N * B * D);
    float t = detT / detM;
    if (!(t > eps && t < tmax)) return false;
    t_out = t;
    beta_out = beta;
    gamma_out = gamma;
    return true;
}

// Conservative slab test of both children of a node (explicit FMAs; boxes are
// stored slightly enlarged).  Returns a 2-bit mask and the entry distances.
__device__ __forceinline__ uint32_t node_test(const BVHNode &n, f3 oinv, f3 inv, float tmin, float tmax,
                                              float &t0, float &t1) {
    const float l0x = __fmaf_rn(n.bx.x, inv.x, -oinv.x), h0x = __fmaf_rn(n.bx.y, inv.x, -oinv.x);
    const float l1x = __fmaf_rn(n.bx.z, inv.x, -oinv.x), h1x = __fmaf_rn(n.bx.w, inv.x, -oinv.x);
    const float l0y = __fmaf_rn(n.by.x, inv.y, -oinv.y), h0y = __fmaf_rn(n.by.y, inv.y, -oinv.y);
    const float l1y = __fmaf_rn(n.by.z, inv.y, -oinv.y), h1y = __fmaf_rn(n.by.w, inv.y, -oinv.y);
    const float l0z = __fmaf_rn(n.bz.x, inv.z, -oinv.z), h0z = __fmaf_rn(n.bz.y, inv.z, -oinv.z);
    const float l1z = __fmaf_rn(n.bz.z, inv.z, -oinv.z), h1z = __fmaf_rn(n.bz.w, inv.z, -oinv.z);
    float n0 = fmaxf(fmaxf(fminf(l0x, h0x), fminf(l0y, h0y)), fmaxf(fminf(l0z, h0z), tmin));
    float f0 = fminf(fminf(fmaxf(l0x, h0x), fmaxf(l0y, h0y)), fminf(fmaxf(l0z, h0z), tmax));
    float n1 = fmaxf(fmaxf(fminf(l1x, h1x), fminf(l1y, h1y)), fmaxf(fminf(l1z, h1z), tmin));
    float f1 = fminf(fminf(fmaxf(l1x, h1x), fmaxf(l1y, h1y)), fminf(fmaxf(l1z, h1z), tmax));
    // 1 + 2^-20 absorbs the rounding of the slab distances (cf. Ize 2013)
    f0 *= 1.00000095367431640625f;
    f1 *= 1.00000095367431640625f;
    t0 = n0;
    t1 = n1;
    return (n0 <= f0 ? 1u : 0u) | (n1 <= f1 ? 2u : 0u);
}

__device__ __forceinline__ f3 safe_inv(f3 d) {
    const float tiny = 1e-30f;
    float x = fabsf(d.x) < tiny ? copysignf(tiny, d.x) : d.x;
    float y = fabsf(d.y) < tiny ? copysignf(tiny, d.y) : d.y;
    float z = fabsf(d.z) < tiny ? copysignf(tiny, d.z) : d.z;
    return mk(1.0f / x, 1.0f / y, 1.0f / z);
}

__device__ __forceinline__ BVHNode load_node(const BVHNode *nodes, uint32_t i) {
    const float4 *p = reinterpret_cast<const float4 *>(nodes + i);
    BVHNode n;
    n.bx = __ldg(p + 0);
    n.by = __ldg(p + 1);
    n.bz = __ldg(p + 2);
    float4 c = __ldg(p + 3);
    n.ch = make_uint4(__float_as_uint(c.x), __float_as_uint(c.y), __float_as_uint(c.z), __float_as_uint(c.w));
    return n;
}

__device__ __forceinline__ DevTri load_tri(const DevTri *tris, uint32_t i) {
    const float4 *p = reinterpret_cast<const float4 *>(tris + i);
    DevTri t;
    t.a = __ldg(p + 0);
    t.b = __ldg(p + 1);
    t.c = __ldg(p + 2);
    return t;
}

// Stack entries: inner node index, leaf range or the BLAS-exit marker.
#define AZD_ENT_LEAF 0x80000000u
#define AZD_ENT_EXIT 0xFFFFFFFFu
#define AZD_STACK 64

// leaf entry: flag, 3 bits of count-1 (leaves hold at most 8 primitives), 27 bits of start
__device__ __forceinline__ uint32_t leaf_entry(uint32_t start, uint32_t count) {
    return AZD_ENT_LEAF | (((count - 1u) & 7u) << 27) | (start & 0x07FFFFFFu);
}

enum QueryKind : uint32_t {
    Q_CLOSEST = 0,   // nearest hit
    Q_ANY = 1        // any hit with world t < tmax (early exit)
};

// Two-level traversal.  For Q_CLOSEST returns the nearest hit in `best`
// (best.ent == 0xFFFFFFFF: none).  For Q_ANY returns true as soon as a
// primitive's world t < tmax.  `counts` (optional) accumulates node and
// primitive visits.
// A valid BVH needs far fewer steps; the cap only guards against a corrupt
// tree looping forever.  When hit, the query stops and sets *err.
#define AZD_MAX_STEPS (1u << 22)

template <QueryKind KIND>
__device__ bool trace(const DevScene &S, const Ray &wr, bool cull, float eps, float tmax, Hit &best,
                      uint32_t *counts = nullptr, uint32_t *err = nullptr) {
    best.t = FLT_MAX;
    best.tl = 0.0f;
    best.prim = 0xFFFFFFFFu;
    best.ent = 0xFFFFFFFFu;
    if (S.tlas_root == 0xFFFFFFFFu) return false;

    uint32_t stack_node[AZD_STACK];
    float stack_t[AZD_STACK];
    int sp = 0;

    // current ray space
    Ray r = wr;
    f3 inv = safe_inv(r.d);
    f3 oinv = had(r.o, inv);
    float tcur = KIND == Q_ANY ? tmax : FLT_MAX;   // pruning distance in the current space
    bool in_blas = false;
    uint32_t g_idx = 0;
    float blas_scale = 1.0f;                        // local t per world t (upper bound)
    float bl_t = FLT_MAX, bl_b = 0.0f;              // nearest local hit of this BLAS visit
    uint32_t bl_prim = 0xFFFFFFFFu;
    uint32_t nodes_visited = 0, prims_visited = 0;

    uint32_t cur = S.tlas_root;  // inner node index or an entry
    uint32_t steps = 0;
    while (true) {
        if (++steps > AZD_MAX_STEPS) {
            if (err) atomicOr(err, 1u);
            break;
        }
        if (cur == AZD_ENT_EXIT) {
            // leaving a BLAS: azimuth's instance path keeps the nearest local hit
            // and recomputes its world t (src/azimuth_main.cpp:256-276)
            const DevGroup &g = S.groups[g_idx];
            if (bl_prim != 0xFFFFFFFFu) {
                float wt;
                if (g.raw) {
                    wt = bl_t;
                } else {
                    f3 motion = wr.time * mk(g.motion[0], g.motion[1], g.motion[2]);
                    f3 o2 = wr.o - motion;
                    f3 lp = r.o + (r.d * bl_t);
                    f3 wp = point_xf(g.xf, lp) + motion;
                    wt = length(wp - o2 - motion) / length(wr.d);
                }
                if (wt > eps && wt < best.t) {
                    if (KIND == Q_ANY) {
                        if (wt < tmax) return true;
                    } else {
                        best.t = wt;
                        best.tl = bl_t;
                        best.prim = bl_prim;
                        best.ent = S.tri_attr[bl_prim].entity;
                    }
                }
            }
            (void)bl_b;
            r = wr;
            inv = safe_inv(r.d);
            oinv = had(r.o, inv);
            tcur = KIND == Q_ANY ? tmax : best.t;
            in_blas = false;
            cur = 0xFFFFFFFEu;  // pop next
        } else if (cur & AZD_ENT_LEAF) {
            uint32_t start = cur & 0x07FFFFFFu, count = ((cur >> 27) & 7u) + 1u;
            cur = 0xFFFFFFFEu;
            if (in_blas) {
                for (uint32_t i = 0; i < count; i++) {
                    uint32_t pi = start + i;
                    DevTri tr = load_tri(S.tris, pi);
                    float t, b, gm;
                    prims_visited++;
                    if (tri_test(tr, r, cull, eps, bl_t, t, b, gm)) {
                        bl_t = t;
                        bl_b = b;
                        bl_prim = pi;
                        if (KIND == Q_ANY) {
                            // early exit as soon as one hit of this group is in range
                            const DevGroup &g = S.groups[g_idx];
                            float wt;
                            if (g.raw) {
                                wt = t;
                            } else {
                                f3 motion = wr.time * mk(g.motion[0], g.motion[1], g.motion[2]);
                                f3 o2 = wr.o - motion;
                                f3 lp = r.o + (r.d * t);
                                f3 wp = point_xf(g.xf, lp) + motion;
                                wt = length(wp - o2 - motion) / length(wr.d);
                            }
                            if (wt > eps && wt < tmax) return true;
                        } else {
                            tcur = fminf(tcur, t);
                        }
                    }
                }
            } else {
                for (uint32_t i = 0; i < count; i++) {
                    uint32_t p = __ldg(S.tlas_prims + start + i);
                    prims_visited++;
                    if (p & AZD_TLAS_GROUP) {
                        // enter the group's BLAS (azimuth: GetLocalRay of the
                        // motion-shifted ray, src/azimuth_main.cpp:246-250)
                        g_idx = p & ~AZD_TLAS_GROUP;
                        const DevGroup &g = S.groups[g_idx];
                        if (g.root == 0xFFFFFFFFu) continue;
                        if (sp >= AZD_STACK) break;
                        stack_node[sp] = AZD_ENT_EXIT;
                        stack_t[sp] = -FLT_MAX;
                        sp++;
                        if (g.raw) {
                            r = wr;
                            blas_scale = 1.0f;
                        } else {
                            Ray m = wr;
                            m.o = wr.o - wr.time * mk(g.motion[0], g.motion[1], g.motion[2]);
                            r = local_ray(m, g.inv);
                            // local t = world t * |inv * d| / |d| (up to rounding)
                            f3 ld = vector_xf(g.inv, wr.d);
                            blas_scale = length(ld) / length(wr.d) * 1.0001f;
                        }
                        inv = safe_inv(r.d);
                        oinv = had(r.o, inv);
                        float wlim = KIND == Q_ANY ? tmax : best.t;
                        tcur = wlim < FLT_MAX ? wlim * blas_scale + 1e-30f : FLT_MAX;
                        bl_t = FLT_MAX;
                        bl_prim = 0xFFFFFFFFu;
                        in_blas = true;
                        cur = g.root;
                        break;  // TLAS leaves hold one primitive
                    } else {
                        const DevEntity &e = S.ents[p];
                        float wt, tl;
                        if (e.type == ENT_SPHERE && sphere_test(e, wr, eps, wt, tl)) {
                            if (KIND == Q_ANY) {
                                if (wt < tmax) return true;
                            } else if (wt < best.t) {
                                best.t = wt;
                                best.tl = tl;
                                best.prim = 0xFFFFFFFFu;
                                best.ent = p;
                                tcur = wt;
                            }
                        }
                    }
                }
            }
        } else if (cur != 0xFFFFFFFEu) {
            // inner node: test both children, continue with the nearer one
            BVHNode n = load_node(S.nodes, cur);
            nodes_visited++;
            float t0, t1;
            uint32_t mask = node_test(n, oinv, inv, 0.0f, tcur, t0, t1);
            uint32_t e0 = n.ch.z ? leaf_entry(n.ch.x, n.ch.z) : n.ch.x;
            uint32_t e1 = n.ch.w ? leaf_entry(n.ch.y, n.ch.w) : n.ch.y;
            if (mask == 3u) {
                uint32_t nearE = e0, farE = e1;
                float farT = t1;
                if (t1 < t0) { nearE = e1; farE = e0; farT = t0; }
                if (sp < AZD_STACK) {
                    stack_node[sp] = farE;
                    stack_t[sp] = farT;
                    sp++;
                }
                cur = nearE;
            } else if (mask == 1u) {
                cur = e0;
            } else if (mask == 2u) {
                cur = e1;
            } else {
                cur = 0xFFFFFFFEu;
            }
        }
        if (cur == 0xFFFFFFFEu) {
            // pop, skipping entries beyond the current pruning distance
            bool found = false;
            while (sp > 0) {
                sp--;
                uint32_t e = stack_node[sp];
                if (e == AZD_ENT_EXIT || !(stack_t[sp] > tcur)) {
                    cur = e;
                    found = true;
                    break;
                }
            }
            if (!found) break;
        }
    }
    if (counts) {
        atomicAdd(counts + 0, nodes_visited);
        atomicAdd(counts + 1, prims_visited);
    }
    if (KIND == Q_ANY) return false;
    return best.ent != 0xFFFFFFFFu;
}

}  // namespace azd
