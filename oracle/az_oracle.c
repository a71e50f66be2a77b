/*
 * az_oracle.c -- CPU restatement of azimuth's render path (TEST INFRASTRUCTURE).
 *
 * This file is the oracle the GPU kernels are checked against.  It is plain
 * C, written from the reference's algorithm: every function names the
 * azimuth source lines (file:line in ff-k/azimuth) it follows.  It is pinned
 * against azimuth's own code compiled by oracle/build.py
 * (tests/test_oracle_pin.py); it is never linked into the product.
 *
 * Randomness: azimuth's Random01 (src/azimuth_math.cpp:1-8) is replaced by
 * the counter RNG of az_rng_oracle.h.  Each TraceRay activation is one node of
 * the sample's path tree; a draw is keyed by (seed, pixel, sample, node, dim)
 * where node = (level, 2-bit child index per level) and dim counts the draws
 * made by that node.
 *
 * Where azimuth draws twice inside one expression (function arguments or an
 * overloaded operator+), the order is whatever GCC chose for the oracle
 * build; it is a parameter here (AZ_ORDER_*), pinned by the tests.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "az_abi.h"
#include "az_rng_oracle.h"

/* ----------------------------------------------------------------------- */
/* vec3 helpers: src/azimuth_math.cpp:572-1348 (plain IEEE float ops)        */
/* ----------------------------------------------------------------------- */
typedef az_vec3 v3;
static inline v3 mk(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 mul(v3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
static inline v3 smul(float s, v3 a) { return mk(s * a.x, s * a.y, s * a.z); }
static inline v3 had(v3 a, v3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 neg(v3 a) { return mk(-a.x, -a.y, -a.z); }
static inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) {
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float len(v3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
static inline v3 nrm(v3 a) {                              /* :1298-1313 */
    float l = len(a);
    if (l != 0.0f) return mk(a.x / l, a.y / l, a.z / l);
    return mk(0, 0, 0);
}
static inline v3 reflect(v3 v, v3 r) { return sub(smul(2.0f * dot(v, r), r), v); } /* :1335-1348 */
static inline float comp(v3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

static inline v3 point_to_world(v3 v, const az_mat4 *m) {    /* :1775-1800 */
    return mk(m->E[0][0] * v.x + m->E[0][1] * v.y + m->E[0][2] * v.z + m->E[0][3],
              m->E[1][0] * v.x + m->E[1][1] * v.y + m->E[1][2] * v.z + m->E[1][3],
              m->E[2][0] * v.x + m->E[2][1] * v.y + m->E[2][2] * v.z + m->E[2][3]);
}
static inline v3 vector_to_world(v3 v, const az_mat4 *m) {   /* :1803-1826 */
    return mk(m->E[0][0] * v.x + m->E[0][1] * v.y + m->E[0][2] * v.z,
              m->E[1][0] * v.x + m->E[1][1] * v.y + m->E[1][2] * v.z,
              m->E[2][0] * v.x + m->E[2][1] * v.y + m->E[2][2] * v.z);
}
static inline v3 normal_to_world(v3 v, const az_mat4 *inv) { /* :1828-1843 */
    return nrm(mk(inv->E[0][0] * v.x + inv->E[1][0] * v.y + inv->E[2][0] * v.z,
                  inv->E[0][1] * v.x + inv->E[1][1] * v.y + inv->E[2][1] * v.z,
                  inv->E[0][2] * v.x + inv->E[1][2] * v.y + inv->E[2][2] * v.z));
}
static inline void onb(v3 w, v3 *u, v3 *v) {                 /* :1845-1863 */
    if (w.z < 0.0) {
        const float a = 1.0f / (1.0f - w.z);
        const float b = w.x * w.y * a;
        *u = mk(1.0f - w.x * w.x * a, -b, w.x);
        *v = mk(b, w.y * w.y * a - 1.0f, -w.y);
    } else {
        const float a = 1.0f / (1.0f + w.z);
        const float b = -w.x * w.y * a;
        *u = mk(1.0f - w.x * w.x * a, b, -w.x);
        *v = mk(b, 1.0f - w.y * w.y * a, -w.y);
    }
}

#define PI_F32 ((float)3.14159265359)

typedef struct { v3 o, d; float t; } ray;
typedef struct { v3 p, n; az_vec2 uv; const az_entity *e; float t; } hit;

/* GetLocalRay, src/azimuth_ray.h:24-66 */
static ray local_ray(ray r, const az_mat4 *m) {
    ray out = r;
    out.o = mk(m->E[0][0] * r.o.x + m->E[0][1] * r.o.y + m->E[0][2] * r.o.z + m->E[0][3],
               m->E[1][0] * r.o.x + m->E[1][1] * r.o.y + m->E[1][2] * r.o.z + m->E[1][3],
               m->E[2][0] * r.o.x + m->E[2][1] * r.o.y + m->E[2][2] * r.o.z + m->E[2][3]);
    out.d = nrm(mk(m->E[0][0] * r.d.x + m->E[0][1] * r.d.y + m->E[0][2] * r.d.z,
                   m->E[1][0] * r.d.x + m->E[1][1] * r.d.y + m->E[1][2] * r.d.z,
                   m->E[2][0] * r.d.x + m->E[2][1] * r.d.y + m->E[2][2] * r.d.z));
    return out;
}

/* RayAABBIntersection, src/azimuth_ray.h:68-125 */
static int ray_aabb(const az_aabb *b, ray r) {
    v3 inv = mk(1.0f / r.d.x, 1.0f / r.d.y, 1.0f / r.d.z);
    v3 mn = sub(b->Min, r.o), mx = sub(b->Max, r.o);
    float ex, ey, ez, xx, xy, xz;
    if (inv.x > 0.0f) { ex = mn.x * inv.x; xx = mx.x * inv.x; } else { ex = mx.x * inv.x; xx = mn.x * inv.x; }
    if (inv.y > 0.0f) { ey = mn.y * inv.y; xy = mx.y * inv.y; } else { ey = mx.y * inv.y; xy = mn.y * inv.y; }
    if (inv.z > 0.0f) { ez = mn.z * inv.z; xz = mx.z * inv.z; } else { ez = mx.z * inv.z; xz = mn.z * inv.z; }
    float enter = ex > ey ? ex : ey;
    enter = ez > enter ? ez : enter;
    float exit = xx < xy ? xx : xy;
    exit = xz < exit ? xz : exit;
    return enter <= exit && exit > 0.0f;
}

/* ----------------------------------------------------------------------- */
/* RNG context                                                              */
/* ----------------------------------------------------------------------- */
typedef struct {
    uint64_t seed;
    uint32_t pixel, sample;
    uint32_t level, digits, dim, next_child;
} node_ctx;

static inline float rnd(node_ctx *c) {
    return az_oracle_u01(c->seed, c->pixel, c->sample, c->digits, c->level, c->dim++);
}
static node_ctx child_ctx(node_ctx *p) {
    node_ctx c = *p;
    uint32_t k = p->next_child++;
    c.level = p->level + 1;
    if (c.level >= 2 && c.level - 2 < 16) c.digits |= (k & 3u) << (2u * (c.level - 2u));
    c.dim = 0;
    c.next_child = 0;
    return c;
}

/* Evaluation order of paired draws inside one expression (bit set = the
 * second draw in source order is taken first). */
enum { AZ_ORDER_LENS = 1, AZ_ORDER_AREA = 2, AZ_ORDER_GLOSSY = 4 };
static int g_order = 0;
static const float *g_gradients = 0;   /* azimuth's global PerlinGradient[256] */

/* ----------------------------------------------------------------------- */
/* Textures: src/azimuth_texture.h:134-357                                  */
/* ----------------------------------------------------------------------- */
static inline uint32_t perlin_hash(const uint32_t *P, int32_t i, int32_t j, int32_t k) { /* :134-144 */
    /* s32 + u32 is unsigned arithmetic in azimuth, so only the innermost
     * K % 256 is a signed remainder; a negative K indexes before the table
     * there (quirk), so callers stay at non-negative coordinates */
    uint32_t a = P[k % 256];
    uint32_t b = P[((uint32_t)j + a) % 256u];
    return P[((uint32_t)i + b) % 256u];
}
static inline float perlin_weight(float v) {                 /* :146-154 */
    v = fabsf(v);
    return 1.0f - ((((6.0f * v) - 15.0f) * v + 10.0f) * v * v * v);
}
static float sample_perlin(const az_texture *t, v3 p) {      /* :156-195 */
    float r = 0.0f;
    p = mul(p, t->ScalingFactor);
    int32_t I = (int32_t)floorf(p.x), J = (int32_t)floorf(p.y), K = (int32_t)floorf(p.z);
    for (int32_t z = 0; z < 2; z++)
        for (int32_t y = 0; y < 2; y++)
            for (int32_t x = 0; x < 2; x++) {
                uint32_t h = perlin_hash(t->Perm, I + x, J + y, K + z);
                v3 e = mk(g_gradients[3 * h], g_gradients[3 * h + 1], g_gradients[3 * h + 2]);
                v3 v = mk(p.x - (float)(I + x), p.y - (float)(J + y), p.z - (float)(K + z));
                r += dot(e, v) * perlin_weight(v.x) * perlin_weight(v.y) * perlin_weight(v.z);
            }
    if (t->PerlinAppearance == AZ_PerlinAppearance_Patch) r = (r + 1.0f) / 2.0f;
    else r = fabsf(r);
    return r;
}
static v3 fetch(const az_texture *t, uint32_t x, uint32_t y) {  /* :197-237 */
    uint32_t idx = (y * t->Width + x) * 3;
    if (t->PixelFormat == AZ_PixelFormat_RGB_U8) {
        const uint8_t *p = (const uint8_t *)t->Pixels;
        return mk((float)p[idx], (float)p[idx + 1], (float)p[idx + 2]);
    }
    const float *p = (const float *)t->Pixels;
    return mk(p[idx], p[idx + 1], p[idx + 2]);
}
static v3 sample_tex2d(const az_texture *t, az_vec2 uv, int normalize) { /* :239-339 */
    v3 r;
    if (t->WrapMode == AZ_TextureWrap_Clamp) {
        float u = uv.x < 1.0f ? uv.x : 1.0f; uv.x = 0.0f > u ? 0.0f : u;
        float v = uv.y < 1.0f ? uv.y : 1.0f; uv.y = 0.0f > v ? 0.0f : v;
    } else {
        uv.x = uv.x - floorf(uv.x);
        uv.y = uv.y - floorf(uv.y);
    }
    if (t->Filter == AZ_TextureFilter_Nearest) {
        uint32_t fx = (uint32_t)floorf(uv.x * ((float)t->Width - 1.0f) + 0.5f);
        uint32_t fy = (uint32_t)floorf(uv.y * ((float)t->Height - 1.0f) + 0.5f);
        r = fetch(t, fx, fy);
    } else {
        float su = uv.x * (float)t->Width, sv = uv.y * (float)t->Height;
        uint32_t ax = (uint32_t)(su + 0.5f) % t->Width;
        uint32_t ay = (uint32_t)(sv + 0.5f) % t->Height;
        uint32_t bx = (ax - 1) % t->Width, by = ay % t->Height;
        uint32_t cx = (ax - 1) % t->Width, cy = (ay - 1) % t->Height;
        uint32_t dx = ax % t->Width, dy = (ay - 1) % t->Height;
        v3 A = fetch(t, ax, ay), B = fetch(t, bx, by), Cc = fetch(t, cx, cy), D = fetch(t, dx, dy);
        su = floorf(su + 0.5f);
        sv = floorf(sv + 0.5f);
        if (su >= t->Width) su -= t->Width;
        if (sv >= t->Height) sv -= t->Height;
        float fx = su - (float)ax, fy = sv - (float)ay;
        r = add(add(add(mul(mul(A, 1.0f - fx), 1.0f - fy), mul(mul(B, fx), 1.0f - fy)),
                    mul(mul(Cc, fx), fy)), mul(mul(D, 1.0f - fx), fy));
    }
    if (normalize) {
        r.x /= t->Normalizer; r.y /= t->Normalizer; r.z /= t->Normalizer;
    }
    return r;
}
static v3 sample_texture(const az_texture *t, v3 p, az_vec2 uv) {  /* :341-357 */
    if (t->Type == AZ_TextureType_2D) return sample_tex2d(t, uv, 1);
    float n = sample_perlin(t, p);
    return mk(n, n, n);
}

/* ----------------------------------------------------------------------- */
/* Intersection: src/azimuth_main.cpp:53-385                                */
/* ----------------------------------------------------------------------- */
static int isect(hit *h, ray r, const az_entity *e, const az_texture *textures, int cull, float eps) {
    int result = 0;
    const az_texture *tex = 0;
    v3 Pu = mk(0, 0, 0), Pv = mk(0, 0, 0);
    int deferred = 0;
    switch (e->Type) {
    case AZ_Entity_Sphere: {                                   /* :64-146 */
        v3 motion = smul(r.t, e->MotionVector);
        r.o = sub(r.o, motion);
        ray lr = local_ray(r, &e->InvTransformationMatrix);
        float radius = e->Radius;
        v3 c = e->Center;
        v3 dist = sub(lr.o, c);
        float A = dot(lr.d, lr.d), B = dot(dist, lr.d), C = dot(dist, dist) - radius * radius;
        float disc = B * B - (A * C);
        if (disc > 0.0f) {
            float sq = sqrtf(disc);
            float t1 = (-B + sq) / (A), t2 = (-B - sq) / (A);
            float t = FLT_MAX;
            if (t1 > eps && t2 > eps) t = t1 < t2 ? t1 : t2;
            else if (t1 > eps) t = t1;
            else if (t2 > eps) t = t2;
            if (t > eps && t < h->t) {
                v3 hp = add(lr.o, mul(lr.d, t));
                v3 lhp = sub(hp, c);
                v3 hn = nrm(lhp);
                v3 wp = add(point_to_world(hp, &e->TransformationMatrix), motion);
                float wt = len(sub(sub(wp, r.o), motion)) / len(r.d);
                if (wt > eps && wt < h->t) {
                    float theta = acosf(hn.y), phi = atan2f(hn.z, hn.x);
                    float two_pi = PI_F32 * 2.0f;
                    h->p = wp;
                    if (e->TextureIndex) {
                        tex = textures + (e->TextureIndex - 1);
                        if (tex->BumpMap) {
                            float pypi = PI_F32 * lhp.y, rpi = PI_F32 * radius;
                            Pv = mk(cosf(phi) * pypi, -sinf(theta) * rpi, sinf(phi) * pypi);
                            Pu = mk(two_pi * lhp.z, 0.0f, -two_pi * lhp.x);
                        } else {
                            tex = 0;
                        }
                        h->n = hn;
                        deferred = 1;
                    } else {
                        h->n = normal_to_world(hn, &e->InvTransformationMatrix);
                    }
                    h->uv.x = (-phi + PI_F32) / two_pi;
                    h->uv.y = theta / PI_F32;
                    h->e = e;
                    h->t = wt;
                    result = 1;
                }
            }
        }
    } break;
    case AZ_Entity_Triangle: {                                 /* :147-243 */
        v3 P0 = e->P0, P1 = e->P1, P2 = e->P2, FN = e->FaceNormal;
        if (!cull || dot(r.d, FN) < 0.0f) {
            float A = P0.x - P1.x, B = P0.x - P2.x, C = r.d.x;
            float D = P0.y - P1.y, E = P0.y - P2.y, F = r.d.y;
            float G = P0.z - P1.z, H = P0.z - P2.z, I = r.d.z;
            float detM = (A * E * I) + (D * H * C) + (G * B * F) - (C * E * G) - (F * H * A) - (I * B * D);
            float K = P0.x - r.o.x, M = P0.y - r.o.y, N = P0.z - r.o.z;
            float detB = (K * E * I) + (M * H * C) + (N * B * F) - (C * E * N) - (F * H * K) - (I * B * M);
            const float lower = -0.000001f;
            float beta = detB / detM;
            if (beta > lower && beta <= 1.0f) {
                float detG = (A * M * I) + (D * N * C) + (G * K * F) - (C * M * G) - (F * N * A) - (I * K * D);
                float gamma = detG / detM;
                if (gamma > lower && gamma <= 1.0f) {
                    float detT = (A * E * N) + (D * H * K) + (G * B * M) - (K * E * G) - (M * H * A) - (N * B * D);
                    float alpha = 1.0f - beta - gamma;
                    if (alpha > lower) {
                        float t = detT / detM;
                        if (t > eps && t < h->t) {
                            h->p = add(r.o, mul(r.d, t));
                            if (e->ShadingMode == AZ_Shading_Flat) h->n = FN;
                            else h->n = add(add(smul(alpha, e->N0), smul(beta, e->N1)), smul(gamma, e->N2));
                            az_vec2 uv0 = e->UV0, uv1 = e->UV1, uv2 = e->UV2;
                            h->uv.x = ((alpha * uv0.x) + (beta * uv1.x)) + (gamma * uv2.x);
                            h->uv.y = ((alpha * uv0.y) + (beta * uv1.y)) + (gamma * uv2.y);
                            h->e = e;
                            h->t = t;
                            if (e->TextureIndex) {
                                tex = textures + (e->TextureIndex - 1);
                                if (tex->BumpMap) {
                                    float div = ((uv1.x - uv0.x) * (uv2.y - uv0.y)) - ((uv1.y - uv0.y) * (uv2.x - uv0.x));
                                    div = 1.0f / div;
                                    Pu = add(smul(uv2.y - uv0.y, sub(P1, P0)), smul(uv0.y - uv1.y, sub(P2, P0)));
                                    Pu = mul(Pu, div);
                                    Pv = add(smul(uv0.x - uv2.x, sub(P1, P0)), smul(uv1.x - uv0.x, sub(P2, P0)));
                                    Pv = mul(Pv, div);
                                } else {
                                    tex = 0;
                                }
                            }
                            result = 1;
                        }
                    }
                }
            }
        }
    } break;
    case AZ_Entity_MeshInstance: {                             /* :244-281 */
        if (ray_aabb(&e->AABB, r)) {
            v3 motion = smul(r.t, e->MotionVector);
            r.o = sub(r.o, motion);
            ray lr = local_ray(r, &e->InvTransformationMatrix);
            hit lh;
            memset(&lh, 0, sizeof(lh));
            lh.t = FLT_MAX;
            if (isect(&lh, lr, e->Mesh->BVH, textures, cull, eps)) {
                v3 wp = add(point_to_world(lh.p, &e->TransformationMatrix), motion);
                float wt = len(sub(sub(wp, r.o), motion)) / len(r.d);
                if (wt > eps && wt < h->t) {
                    *h = lh;
                    h->p = wp;
                    h->n = normal_to_world(lh.n, &e->InvTransformationMatrix);
                    h->e = e;
                    h->t = wt;
                    result = 1;
                } else {
                    result = 0;
                }
            }
        }
    } break;
    case AZ_Entity_BVHNode: {                                  /* :282-319 */
        if (ray_aabb(&e->AABB, r)) {
            hit lh, rh;
            memset(&lh, 0, sizeof(lh));
            memset(&rh, 0, sizeof(rh));
            lh.t = FLT_MAX;
            rh.t = FLT_MAX;
            int L = isect(&lh, r, e->Left, textures, cull, eps);
            int R = isect(&rh, r, e->Right, textures, cull, eps);
            if (L) {
                result = 1;
                *h = (R && !(lh.t < rh.t)) ? rh : lh;
            } else if (R) {
                result = 1;
                *h = rh;
            }
        }
    } break;
    }

    if (tex) {                                                 /* :321-377 */
        az_vec2 uv = h->uv;
        if (tex->Type == AZ_TextureType_2D) {
            v3 A = sample_tex2d(tex, uv, 0);
            az_vec2 uvu = {uv.x + tex->InvWidth, uv.y}, uvv = {uv.x, uv.y + tex->InvHeight};
            v3 B = sample_tex2d(tex, uvu, 0), C = sample_tex2d(tex, uvv, 0);
            v3 du3 = sub(B, A), dv3 = sub(C, A);
            float du = ((du3.x + du3.y + du3.z) / 3.0f) * tex->BumpMapMultiplier;
            float dv = ((dv3.x + dv3.y + dv3.z) / 3.0f) * tex->BumpMapMultiplier;
            v3 dPu = add(Pu, smul(du, h->n)), dPv = add(Pv, smul(dv, h->n));
            h->n = nrm(cross(dPv, dPu));
        } else {
            const float be = 0.001f;
            v3 p = h->p;
            float d = sample_perlin(tex, p);
            float dx = sample_perlin(tex, mk(p.x + be, p.y, p.z));
            float dy = sample_perlin(tex, mk(p.x, p.y + be, p.z));
            float dz = sample_perlin(tex, mk(p.x, p.y, p.z + be));
            v3 g = mk((dx - d) / be, (dy - d) / be, (dz - d) / be);
            h->n = sub(h->n, mul(g, tex->BumpMapMultiplier));
            h->n = nrm(h->n);
        }
    }
    if (deferred) h->n = normal_to_world(h->n, &e->InvTransformationMatrix);
    return result;
}

/* ----------------------------------------------------------------------- */
/* Lights and BRDFs: src/azimuth_main.cpp:392-779                           */
/* ----------------------------------------------------------------------- */
static void sample_entity_light(const az_entity *le, v3 hp, node_ctx *rc, v3 *dir, float *invpdf) { /* :392-459 */
    v3 hpl = point_to_world(hp, &le->InvTransformationMatrix);
    v3 ldl = mk(0, 0, 0);
    *invpdf = 0.0f;
    if (le->Type == AZ_Entity_Sphere) {
        v3 D = sub(le->Center, hpl);
        float rod = le->Radius / len(D);
        float ctm = sqrtf(1.0f - rod * rod);
        float ct = 1.0f + rnd(rc) * (ctm - 1.0f);
        float st = sqrtf(1.0f - ct * ct);
        float phi = 2.0f * PI_F32 * rnd(rc);
        float cp = cosf(phi), sp = sinf(phi);
        v3 W = nrm(D), U, V;
        onb(W, &U, &V);
        ldl = nrm(add(add(mul(mul(U, st), cp), mul(mul(V, st), sp)), mul(W, ct)));
        *invpdf = 2.0f * PI_F32 * (1.0f - ctm);
    } else if (le->Type == AZ_Entity_MeshInstance) {
        const az_mesh *m = le->Mesh;
        uint32_t idx = (uint32_t)(rnd(rc) * (m->TriangleCount));
        if (idx > m->TriangleCount - 1) idx = m->TriangleCount - 1;
        const az_triangle *T = m->Triangles + idx;
        float r1 = sqrtf(rnd(rc));
        float r2 = rnd(rc);
        v3 Q = add(smul(1.0f - r2, T->P0), smul(r2, T->P1));
        v3 P = add(smul(1.0f - r1, T->P2), smul(r1, Q));
        v3 wi = sub(P, hpl);
        float A = m->TotalArea;
        ldl = nrm(wi);
        float ca = dot(ldl, T->N);
        if (ca < 0.0f) ca *= -1.0f;
        float l = len(wi);
        *invpdf = (A * ca) / (l * l);
    }
    *dir = vector_to_world(ldl, &le->TransformationMatrix);
}

static void eval_brdf(float *diffuse, float *specular, const az_brdf *b, v3 L, v3 N, v3 V, float cti) { /* :461-569 */
    switch (b->Type) {
    case AZ_BRDF_Phong: {
        float ca = dot(neg(V), reflect(L, N));
        *specular = ca > 0.0f ? powf(ca, b->Exponent) / cti : 0.0f;
    } break;
    case AZ_BRDF_ModifiedPhong: {
        float ca = dot(neg(V), reflect(L, N));
        *specular = ca > 0.0f ? powf(ca, b->Exponent) : 0.0f;
    } break;
    case AZ_BRDF_NormalizedModifiedPhong: {
        *diffuse = (float)(1.0 / 3.14159265359);
        float ca = dot(neg(V), reflect(L, N));
        *specular = ca > 0.0f ? ((b->Exponent + 2.0f) / (2.0f * PI_F32)) * powf(ca, b->Exponent) : 0.0f;
    } break;
    case AZ_BRDF_BlinnPhong: {
        float ca = dot(N, nrm(add(neg(V), L)));
        *specular = ca > 0.0f ? powf(ca, b->Exponent) / cti : 0.0f;
    } break;
    case AZ_BRDF_ModifiedBlinnPhong: {
        float ca = dot(N, nrm(add(neg(V), L)));
        *specular = ca > 0.0f ? powf(ca, b->Exponent) : 0.0f;
    } break;
    case AZ_BRDF_NormalizedModifiedBlinnPhong: {
        *diffuse = (float)(1.0 / 3.14159265359);
        float ca = dot(N, nrm(add(neg(V), L)));
        *specular = ca > 0.0f ? ((b->Exponent + 8.0f) / (8.0f * PI_F32)) * powf(ca, b->Exponent) : 0.0f;
    } break;
    case AZ_BRDF_TorranceSparrow: {
        *diffuse = (float)(1.0 / 3.14159265359);
        v3 hv = nrm(add(neg(V), L));
        float ca = dot(N, hv);
        if (ca > 0.0f) {
            float e = b->Exponent;
            float D = ((e + 2.0f) / (2.0f * PI_F32)) * powf(ca, e);
            float nw0 = dot(N, neg(V)), w0wh = dot(neg(V), hv);
            float G = nw0 < cti ? nw0 : cti;
            G = (2.0f * G * ca) / w0wh;
            G = 1.0f < G ? 1.0f : G;
            float ri = b->RefractiveIndex;
            float r0 = ((ri - 1.0f) * (ri - 1.0f)) / ((ri + 1.0f) * (ri + 1.0f));
            float F = r0 + (1.0f - r0) * powf(1.0f - w0wh, 5.0f);
            *specular = (D * F * G) / (4.0f * cti * nw0);
        } else {
            *specular = 0.0f;
        }
    } break;
    }
}

static void light_contribution(v3 *dc, v3 *sc, const az_brdf *b, v3 I, v3 ldir, v3 vdir, v3 n,
                               float ldist, float falloff, float invpdf) { /* :571-603 */
    float d2 = ldist * ldist;
    v3 ln = nrm(ldir);
    v3 li = mul(mk(I.x / d2, I.y / d2, I.z / d2), falloff);
    float cti = dot(n, ln);
    if (cti > 0.0f) {
        float diffuse = 1.0f, specular = 1.0f;
        eval_brdf(&diffuse, &specular, b, ln, n, vdir, cti);
        v3 cm = mul(mul(li, cti), invpdf);
        *dc = add(*dc, mul(cm, diffuse));
        *sc = add(*sc, mul(cm, specular));
    }
}

typedef struct {
    const az_scene *s;
    const az_epsilon_values *eps;
    int cull;
} scene_ctx;

static v3 trace(const scene_ctx *sc, ray r, uint32_t depth, int inside, float *travel, node_ctx *parent);

static void calc_lighting(const scene_ctx *sc, v3 *dc, v3 *spc, ray r, const az_brdf *b, v3 hp, v3 hn,
                          float seps, int inside, node_ctx *rc) { /* :605-779 */
    const az_scene *s = sc->s;
    for (uint32_t li = 0; li < s->LightCount; li++) {
        const az_light *L = s->Lights + li;
        v3 ldir = mk(0, 0, 0), I = L->Intensity;
        int discard_any = 0;
        float falloff = 1.0f, ldist = 1.0f, invpdf = 1.0f;
        switch (L->Type) {
        case AZ_Light_Point:
            ldir = sub(L->Position, hp);
            ldist = len(ldir);
            break;
        case AZ_Light_Area: {
            float u0, u1;
            if (g_order & AZ_ORDER_AREA) { u1 = rnd(rc); u0 = rnd(rc); } else { u0 = rnd(rc); u1 = rnd(rc); }
            v3 lp = add(add(L->Position, mul(L->EdgeVectors[0], u0)), mul(L->EdgeVectors[1], u1));
            falloff = dot(nrm(sub(lp, hp)), L->Normal);
            if (falloff < 0.0f) falloff *= -1.0f;
            ldir = sub(lp, hp);
            ldist = len(ldir);
        } break;
        case AZ_Light_Directional:
            ldir = nrm(neg(L->Direction));
            discard_any = 1;
            break;
        case AZ_Light_Spot: {
            ldir = sub(L->Position, hp);
            ldist = len(ldir);
            float ct = dot(nrm(neg(ldir)), nrm(L->SpotDirection));
            if (ct < L->CosHalfCoverage) falloff = 0.0f;
            else if (ct > L->CosHalfFallOff) falloff = 1.0f;
            else {
                falloff = (ct - L->CosHalfCoverage) / (L->CosHalfFallOff - L->CosHalfCoverage);
                falloff = powf(falloff, 4.0f);
                if (falloff < 0.0f) falloff = 0.0f;
                else if (falloff > 1.0f) falloff = 1.0f;
            }
        } break;
        case AZ_Light_Entity: {
            sample_entity_light(&L->Entity, hp, rc, &ldir, &invpdf);
            I = L->Entity.Radiance;
        } break;
        }
        if (ldist == 0.0f) ldist = 0.001f;
        ray sr;
        sr.o = add(hp, mul(ldir, seps));
        sr.d = ldir;
        sr.t = r.t;
        int reaches = 1;
        hit lh;
        memset(&lh, 0, sizeof(lh));
        lh.t = FLT_MAX;
        if (isect(&lh, sr, s->BVHRoot, s->Textures, 0, 0.0f)) {
            if (L->Type == AZ_Light_Entity) {
                if (lh.e->UniqueEntityID != L->Entity.UniqueEntityID) reaches = 0;
            } else if (discard_any || lh.t < (1.0f - seps)) {
                reaches = 0;
            }
        }
        if (reaches && !inside) light_contribution(dc, spc, b, I, ldir, r.d, hn, ldist, falloff, invpdf);
    }
    if (s->UseEnvironmentMap) {
        float phi = 2.0f * PI_F32 * rnd(rc);
        float cp = cosf(phi), sp = sinf(phi);
        float theta = asinf(sqrtf(rnd(rc)));
        float ct = cosf(theta), st = sinf(theta);
        v3 U, V;
        onb(hn, &U, &V);
        v3 L = nrm(add(add(mul(mul(U, st), cp), mul(mul(V, st), sp)), mul(hn, ct)));
        ray er;
        er.o = add(hp, mul(L, seps));
        er.d = L;
        er.t = r.t;
        hit eh;
        memset(&eh, 0, sizeof(eh));
        eh.t = FLT_MAX;
        if (!isect(&eh, er, s->BVHRoot, s->Textures, 0, 0.0f)) {
            az_vec2 uv = {(-atan2f(L.z, L.x) + PI_F32) / (2.0f * PI_F32), acosf(L.y) / PI_F32};
            v3 I = sample_texture(&s->EnvironmentMap, mk(uv.x, uv.y, 1.0f), uv);
            float ca = dot(L, hn);
            if (ca == 0.0f) ca = 0.000001f;
            light_contribution(dc, spc, b, I, L, r.d, hn, 1.0f, 1.0f, PI_F32 / ca);
        }
    }
}

static v3 mirror_contribution(const scene_ctx *sc, uint32_t depth, const az_material *m, ray r, v3 hp, v3 hn,
                              int inside, float *travel, node_ctx *rc) { /* :781-854 */
    v3 rd = reflect(neg(r.d), hn);
    float g = m->Glossiness;
    if (g != 0.0f) {
        v3 rp = mk(fabsf(rd.x), fabsf(rd.y), fabsf(rd.z));
        if (rp.x < rp.y) {
            if (rp.x < rp.z) { rp = rd; rp.x = rp.x < 0.0f ? -1.0f : 1.0f; }
            else { rp = rd; rp.z = rp.z < 0.0f ? -1.0f : 1.0f; }
        } else {
            if (rp.y < rp.z) { rp = rd; rp.y = rp.y < 0.0f ? -1.0f : 1.0f; }
            else { rp = rd; rp.z = rp.z < 0.0f ? -1.0f : 1.0f; }
        }
        rp = nrm(rp);
        v3 u = cross(rp, rd), v = cross(u, rd);
        float a, bb;
        if (g_order & AZ_ORDER_GLOSSY) { bb = rnd(rc); a = rnd(rc); } else { a = rnd(rc); bb = rnd(rc); }
        rd = add(rd, smul(2.0f * g, add(mul(u, a - 0.5f), mul(v, bb - 0.5f))));
        rd = nrm(rd);
    }
    const float meps = 0.000825f;
    ray mr;
    mr.o = add(hp, mul(rd, meps));
    mr.d = rd;
    mr.t = r.t;
    return had(m->MirrorReflectance, trace(sc, mr, depth + 1, inside, travel, rc));
}

static v3 transparency_contribution(const scene_ctx *sc, const az_material *m, ray r, v3 hp, v3 hn,
                                    uint32_t depth, int inside, node_ctx *rc) { /* :856-964 */
    v3 result = mk(0, 0, 0);
    v3 T = m->Transparency;
    float to = m->RefractionIndex, from = 1.0f;
    if (inside) { from = m->RefractionIndex; to = 1.0f; }
    v3 N = hn;
    float ct = -dot(r.d, N);
    if (ct < 0.0f) { N = neg(hn); ct = -dot(r.d, N); }
    float ratio = from / to;
    float delta = 1.0f - (ratio * ratio) * (1.0f - ct * ct);
    float refl;
    if (delta <= 0.0f) {
        refl = 1.0f;
    } else {
        float cphi = sqrtf(delta);
        float cair = inside ? cphi : ct;
        float icair = 1.0f - cair;
        float q = (from - to) / (from + to);
        float r0 = q * q;
        refl = r0 + (1.0f - r0) * powf(icair, 5);
        v3 td = sub(mul(add(r.d, mul(N, ct)), ratio), mul(N, cphi));
        td = nrm(td);
        ray rr;
        rr.o = add(hp, mul(td, 0.0001f));
        rr.d = td;
        rr.t = r.t;
        float tdist = 0;
        v3 rcontrib = trace(sc, rr, depth + 1, !inside, &tdist, rc);
        v3 att = mk(1, 1, 1);
        if (!inside) att = mk(expf((T.x - 1.0f) * tdist), expf((T.y - 1.0f) * tdist), expf((T.z - 1.0f) * tdist));
        result = add(result, smul(1.0f - refl, had(att, rcontrib)));
    }
    v3 rd = reflect(neg(r.d), N);
    ray lr;
    lr.o = add(hp, mul(rd, 0.0001f));
    lr.d = rd;
    lr.t = r.t;
    float tdist = 0;
    v3 lcontrib = trace(sc, lr, depth + 1, inside, &tdist, rc);
    v3 att = mk(1, 1, 1);
    if (inside) att = mk(expf((T.x - 1.0f) * tdist), expf((T.y - 1.0f) * tdist), expf((T.z - 1.0f) * tdist));
    result = add(result, smul(refl, had(att, lcontrib)));
    return result;
}

/* TraceRay, src/azimuth_main.cpp:966-1133; `parent` is the caller's RNG node */
static v3 trace(const scene_ctx *sc, ray r, uint32_t depth, int inside, float *travel, node_ctx *parent) {
    node_ctx rc = child_ctx(parent);
    const az_scene *s = sc->s;
    v3 result = mk(0, 0, 0);
    if (depth > s->MaxRecursionDepth) return result;
    hit h;
    memset(&h, 0, sizeof(h));
    h.t = FLT_MAX;
    if (!isect(&h, r, s->BVHRoot, s->Textures, sc->cull, sc->eps->Intersection)) return result;
    *travel += h.t;
    const az_entity *e = h.e;
    if (e->IsEmitter) return e->Radiance;
    const az_material *m = s->Materials + e->MaterialIndex;
    const az_brdf *b = &m->BRDF;
    v3 dcol = m->DiffuseReflectance, scol = m->SpecularReflectance;
    v3 dc = mk(0, 0, 0), spc = mk(0, 0, 0);
    v3 hp = h.p, hn = h.n;
    int ignore_ambient = 0;
    if (e->TextureIndex) {
        const az_texture *t = s->Textures + (e->TextureIndex - 1);
        v3 ts = sample_texture(t, hp, h.uv);
        if (t->BlendMode == AZ_TextureBlend_ReplaceAll) {
            dcol = ts;
            dc = mk(1.0f, 1.0f, 1.0f);
            spc = mk(0, 0, 0);
            ignore_ambient = 1;
        } else if (t->BlendMode == AZ_TextureBlend_ReplaceDiffuse) {
            dcol = ts;
        } else {
            dcol = add(dcol, ts);
            dcol = mul(dcol, 0.5f);
        }
    }
    calc_lighting(sc, &dc, &spc, r, b, hp, hn, sc->eps->ShadowRay, inside, &rc);
    if (s->PathTrace) {
        float theta = s->ImportanceSampling ? asinf(sqrtf(rnd(&rc))) : acosf(rnd(&rc));
        float ct = cosf(theta), st = sinf(theta);
        float phi = 2.0f * PI_F32 * rnd(&rc);
        float cp = cosf(phi), sp = sinf(phi);
        v3 U, V;
        onb(hn, &U, &V);
        v3 S = nrm(add(add(mul(mul(U, st), cp), mul(mul(V, st), sp)), mul(hn, ct)));
        ray sr;
        sr.o = add(hp, mul(S, sc->eps->ShadowRay));
        sr.d = S;
        sr.t = r.t;
        float st_travel = 0.0f;
        v3 scol_in = trace(sc, sr, depth + 1, inside, &st_travel, &rc);
        float invpdf;
        if (s->ImportanceSampling) {
            float cs = dot(S, hn);
            if (cs == 0.0f) cs = 0.000001f;
            invpdf = PI_F32 / cs;
        } else {
            invpdf = PI_F32 * 2.0f;
        }
        light_contribution(&dc, &spc, b, scol_in, sr.d, r.d, hn, 1.0f, 1.0f, invpdf);
    }
    result = add(result, had(dcol, dc));
    result = add(result, had(scol, spc));
    uint32_t tb[3], mb[3];
    memcpy(tb, &m->Transparency, 12);
    memcpy(mb, &m->MirrorReflectance, 12);
    int transparent = (tb[0] | tb[1] | tb[2]) != 0;
    if ((!inside || !transparent) && !ignore_ambient) result = add(result, had(m->AmbientReflectance, s->AmbientLight));
    if (mb[0] | mb[1] | mb[2]) result = add(result, mirror_contribution(sc, depth, m, r, hp, hn, inside, travel, &rc));
    if (transparent) result = add(result, transparency_contribution(sc, m, r, hp, hn, depth, inside, &rc));
    return result;
}

/* ----------------------------------------------------------------------- */
/* Camera, background and film: src/azimuth_main.cpp:1135-1397              */
/* ----------------------------------------------------------------------- */
static v3 background(const az_scene *s, v3 d, int32_t w1, int32_t h1, uint32_t row, uint32_t col) { /* :1180-1207 */
    if (s->UseEnvironmentMap) {
        float theta = acosf(d.y), phi = atan2f(d.z, d.x);
        az_vec2 uv = {(-phi + PI_F32) / (2.0f * PI_F32), theta / PI_F32};
        return sample_texture(&s->EnvironmentMap, mk(uv.x, uv.y, 1.0f), uv);
    }
    if (s->UseBackgroundTexture) {
        az_vec2 uv = {(float)col / (float)w1, (float)row / (float)h1};
        return sample_texture(&s->BackgroundTexture, mk(uv.x, uv.y, 1.0f), uv);
    }
    return s->BackgroundColor;
}

static inline void atomic_addf(float *p, float v) {
    uint32_t *bits = (uint32_t *)p;
    for (;;) {
        uint32_t old = __atomic_load_n(bits, __ATOMIC_RELAXED);
        float of, nf;
        memcpy(&of, &old, 4);
        nf = of + v;
        uint32_t nw;
        memcpy(&nw, &nf, 4);
        if (__atomic_compare_exchange_n(bits, &old, nw, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) break;
    }
}

/* Per-sample values for one row range; also used to compute single samples. */
typedef struct {
    v3 base, pos, axx, axy, stepx, stepy;
    float aperture, inv_sqrt;
    uint32_t sqrt_spp, width, height;
    int32_t gk;
    float g_norm, g_neg;
} cam_setup;

static void camera_setup(const az_camera *c, cam_setup *cs) { /* :1265-1347 */
    v3 gaze = c->Gaze;
    if (c->GazeIsPoint) gaze = sub(c->Gaze, c->Position);
    v3 gn = nrm(gaze);
    v3 az = neg(gn), ax, ay;
    if (c->IsLeftHanded) { ax = nrm(cross(nrm(c->Up), gn)); ay = cross(ax, az); }
    else { ax = nrm(cross(gn, nrm(c->Up))); ay = cross(az, ax); }
    float fdn = 1.0f;
    if (c->FocusDistance != 0.0f) fdn = c->FocusDistance / c->NearDistance;
    cs->width = c->Resolution.x;
    cs->height = c->Resolution.y;
    az_vec4 np = c->NearPlane;   /* r,l,b,t stored as x,y,z,w */
    if (c->Type == AZ_Camera_Simple) {
        float hh = c->NearDistance * tanf((c->FovY / 2.0f / 180.0f) * (float)3.14159265359);
        float ar = (float)cs->width / (float)cs->height;
        float wh = ar * hh;
        np.w = +hh; np.z = -hh; np.x = +wh; np.y = -wh;
    }
    float psx = (np.x - np.y) / (float)cs->width, psy = (np.w - np.z) / (float)cs->height;
    cs->stepx = mul(mul(ax, psx), fdn);
    cs->stepy = mul(mul(ay, psy), fdn);
    v3 tl = add(add(add(c->Position, smul(c->NearDistance, gn)), smul(np.y, ax)), smul(np.w, ay));
    cs->base = mul(sub(tl, c->Position), fdn);
    cs->pos = c->Position;
    cs->axx = ax;
    cs->axy = ay;
    cs->aperture = c->ApertureSize;
    cs->sqrt_spp = (uint32_t)sqrtf((float)c->SampleCount);
    cs->inv_sqrt = 1.0f / cs->sqrt_spp;
    float gr = 1.5f, sigma = gr / 3.0f, two = 2.0f * (sigma * sigma);
    cs->g_neg = -1.0f / two;
    cs->g_norm = 1.0f / (two * (float)3.14159265359);
    cs->gk = (int32_t)ceilf(gr - 0.5f);
}

/* One camera sample: GetSampleCoord + GetRayForPixel + TraceRay + background.
 * Returns the sample colour and writes the sample position. */
static v3 render_sample(const scene_ctx *sc, const cam_setup *cs, uint64_t seed, uint32_t row, uint32_t col,
                        uint32_t sx, uint32_t sy, az_vec2 *coord) {
    node_ctx cam;
    memset(&cam, 0, sizeof(cam));
    cam.seed = seed;
    cam.pixel = (row << 16) | col;
    cam.sample = (sy << 16) | sx;
    float ox = 0.5f * cs->inv_sqrt + sx * cs->inv_sqrt;
    float oy = 0.5f * cs->inv_sqrt + sy * cs->inv_sqrt;
    coord->x = col + ox;
    coord->y = row + oy;
    float lx, ly;
    if (g_order & AZ_ORDER_LENS) { ly = rnd(&cam) - 0.5f; lx = rnd(&cam) - 0.5f; }
    else { lx = rnd(&cam) - 0.5f; ly = rnd(&cam) - 0.5f; }
    lx *= cs->aperture;
    ly *= cs->aperture;
    v3 offx = mul(cs->axx, lx), offy = mul(cs->axy, ly);
    v3 dir = nrm(sub(sub(sub(add(cs->base, smul(coord->x, cs->stepx)), smul(coord->y, cs->stepy)), offx), offy));
    ray r;
    r.o = add(add(cs->pos, offx), offy);
    r.d = dir;
    r.t = rnd(&cam);
    float travel = 0.0f;
    v3 c = trace(sc, r, 0, 0, &travel, &cam);
    if (travel == 0.0f)
        c = background(sc->s, r.d, (int32_t)cs->width - 1, (int32_t)cs->height - 1, row, col);
    return c;
}

/* ComputeSampleWeight, src/azimuth_main.cpp:1209-1254 */
static void splat(float *film, const cam_setup *cs, v3 c, az_vec2 coord, uint32_t row, uint32_t col, int filter) {
    if (filter == AZ_Filter_Box) {
        float *p = film + 4 * ((size_t)row * cs->width + col);
        atomic_addf(p + 0, c.x);
        atomic_addf(p + 1, c.y);
        atomic_addf(p + 2, c.z);
        atomic_addf(p + 3, 1.0f);
        return;
    }
    int32_t w1 = (int32_t)cs->width - 1, h1 = (int32_t)cs->height - 1;
    int32_t x0 = (int32_t)col - cs->gk > 0 ? (int32_t)col - cs->gk : 0;
    int32_t x1 = (int32_t)col + cs->gk < w1 ? (int32_t)col + cs->gk : w1;
    int32_t y0 = (int32_t)row - cs->gk > 0 ? (int32_t)row - cs->gk : 0;
    int32_t y1 = (int32_t)row + cs->gk < h1 ? (int32_t)row + cs->gk : h1;
    for (int32_t gy = y0; gy <= y1; gy++)
        for (int32_t gx = x0; gx <= x1; gx++) {
            float dx = coord.x - (gx + 0.5f), dy = coord.y - (gy + 0.5f);
            float d2 = dx * dx + dy * dy;
            float g = cs->g_norm * expf(cs->g_neg * d2);
            float *p = film + 4 * ((size_t)gy * cs->width + gx);
            atomic_addf(p + 0, c.x * g);
            atomic_addf(p + 1, c.y * g);
            atomic_addf(p + 2, c.z * g);
            atomic_addf(p + 3, g);
        }
}

/* ------------------------------- C interface --------------------------- */
void azo_set_order(int order) { g_order = order; }
void azo_set_gradients(const float *g768) { g_gradients = g768; }

/* ProduceImageInLinearSpace (src/azimuth_main.cpp:1256-1397) over a scissor,
 * rows split across OpenMP threads; accumulates into film[W*H*4]. */
void azo_produce_image(float *film, const az_scene *s, const az_camera *c, const az_epsilon_values *eps,
                       az_scissor sc_rect, int filter, int cull, uint64_t seed, int threads) {
    scene_ctx sc = {s, eps, cull};
    cam_setup cs;
    camera_setup(c, &cs);
    uint32_t r0 = sc_rect.Min.y, r1 = sc_rect.Max.y < cs.height ? sc_rect.Max.y : cs.height;
    uint32_t c0 = sc_rect.Min.x, c1 = sc_rect.Max.x < cs.width ? sc_rect.Max.x : cs.width;
    if (threads <= 0) threads = 1;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1)
    for (int64_t row = r0; row < (int64_t)r1; row++)
        for (uint32_t col = c0; col < c1; col++)
            for (uint32_t sy = 0; sy < cs.sqrt_spp; sy++)
                for (uint32_t sx = 0; sx < cs.sqrt_spp; sx++) {
                    az_vec2 coord;
                    v3 v = render_sample(&sc, &cs, seed, (uint32_t)row, col, sx, sy, &coord);
                    splat(film, &cs, v, coord, (uint32_t)row, col, filter);
                }
}

/* Colour of individual camera samples (pixel row/col, sample x/y). */
void azo_render_samples(float *out3, const az_scene *s, const az_camera *c, const az_epsilon_values *eps,
                        const uint32_t *rows, const uint32_t *cols, const uint32_t *sxs, const uint32_t *sys,
                        uint32_t n, int cull, uint64_t seed) {
    scene_ctx sc = {s, eps, cull};
    cam_setup cs;
    camera_setup(c, &cs);
    for (uint32_t i = 0; i < n; i++) {
        az_vec2 coord;
        v3 v = render_sample(&sc, &cs, seed, rows[i], cols[i], sxs[i], sys[i], &coord);
        out3[3 * i] = v.x; out3[3 * i + 1] = v.y; out3[3 * i + 2] = v.z;
    }
}

/* Closest hit on the scene root; same outputs as the reference harness. */
void azo_closest_hit(const az_scene *s, const az_ray3 *rays, uint32_t n, int cull, float eps,
                     uint32_t *out_hit, uint32_t *out_uid, uint32_t *out_face, float *out_t, int threads) {
    if (threads <= 0) threads = 1;
#pragma omp parallel for num_threads(threads) schedule(dynamic, 256)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        ray r;
        r.o = rays[i].Origin; r.d = rays[i].Direction; r.t = rays[i].T;
        hit h;
        memset(&h, 0, sizeof(h));
        h.t = FLT_MAX;
        int ok = isect(&h, r, s->BVHRoot, s->Textures, cull, eps);
        out_hit[i] = (uint32_t)ok;
        out_uid[i] = ok ? h.e->UniqueEntityID : 0xFFFFFFFFu;
        out_face[i] = 0xFFFFFFFFu;
        out_t[i] = ok ? h.t : 0.0f;
        if (ok && h.e->Type == AZ_Entity_MeshInstance) {
            ray rr = r;
            rr.o = sub(rr.o, smul(rr.t, h.e->MotionVector));
            ray lr = local_ray(rr, &h.e->InvTransformationMatrix);
            hit lh;
            memset(&lh, 0, sizeof(lh));
            lh.t = FLT_MAX;
            if (isect(&lh, lr, h.e->Mesh->BVH, s->Textures, cull, eps)) out_face[i] = lh.e->ID;
        } else if (ok && h.e->Type == AZ_Entity_Triangle) {
            out_face[i] = h.e->ID;
        }
    }
}

float azo_u01(uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t digits, uint32_t level, uint32_t dim) {
    return az_oracle_u01(seed, pixel, sample, digits, level, dim);
}

void azo_philox(const uint32_t *ctr4, uint32_t k0, uint32_t k1, uint32_t *out4) {
    az_oracle_philox4x32_10(ctr4, k0, k1, out4);
}

float azo_sample_perlin(const az_texture *t, float x, float y, float z) { return sample_perlin(t, mk(x, y, z)); }

/* OutputPixelsToFile's post-processing (src/azimuth_main.cpp:1620-1760) for an
 * 8-bit file: normalise by TotalWeight; photographic tone mapping with the
 * log-average luminance (f32 running sum of log(L + 1e-5)), the burn-out
 * luminance at index round((1 - burnout/100) (N - 1)) of the sorted
 * luminances, Ld = Ls (1 + Ls / Lwhite^2) / (1 + Ls), colour (C/L)^saturation
 * Ld clamped; then sRGB or 1/gamma; the writers' bytes are
 * (u8)(clamp01(C) * 255) (:1473-1475).  Luminance 0.27 R + 0.67 G + 0.06 B
 * (src/azimuth_math.cpp:1866-1880).  rgb: N x 3 floats out; rgb8: N x 3 bytes out. */
static int cmp_f32(const void *a, const void *b) {
    float x = *(const float *)a, y = *(const float *)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

static float lum3(float r, float g, float b) { return r * 0.27f + g * 0.67f + b * 0.06f; }
static float clamp01(float v) { return v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v); }

int azo_output_pixels(const float *film4, uint32_t w, uint32_t h, const az_tonemap *tm, float inv_gamma,
                      uint32_t srgb, float *rgb, uint8_t *rgb8) {
    const uint32_t n = w * h;
    const int tonemapped = tm->Operator != AZ_Tonemap_None;
    float *lums = tonemapped ? (float *)malloc(sizeof(float) * (n ? n : 1)) : NULL;
    float logavg = 0.0f;
    for (uint32_t i = 0; i < n; i++) {
        const float wt = film4[4 * i + 3];
        float r = film4[4 * i + 0] / wt, g = film4[4 * i + 1] / wt, b = film4[4 * i + 2] / wt;
        rgb[3 * i + 0] = r;
        rgb[3 * i + 1] = g;
        rgb[3 * i + 2] = b;
        if (tonemapped) {
            const float l = lum3(r, g, b);
            lums[i] = l;
            logavg += logf(l + 0.00001f);
        }
    }
    if (tonemapped) {
        logavg = expf(logavg / (float)n);
        const float factor = tm->KeyValue / logavg;
        qsort(lums, n, sizeof(float), cmp_f32);
        const uint32_t li = (uint32_t)((1.0f - tm->BurnoutPercentage * 0.01f) * (float)(n - 1) + 0.5f);
        float lw2 = lums[li] * factor;
        lw2 = lw2 * lw2;
        for (uint32_t i = 0; i < n; i++) {
            const float r = rgb[3 * i + 0], g = rgb[3 * i + 1], b = rgb[3 * i + 2];
            const float l = lum3(r, g, b);
            if (l != 0.0f) {
                const float ls = l * factor;
                const float ld = (ls * (1.0f + (ls / lw2))) / (1.0f + ls);
                rgb[3 * i + 0] = clamp01(powf(r / l, tm->Saturation) * ld);
                rgb[3 * i + 1] = clamp01(powf(g / l, tm->Saturation) * ld);
                rgb[3 * i + 2] = clamp01(powf(b / l, tm->Saturation) * ld);
            }
        }
        free(lums);
    }
    for (uint32_t i = 0; i < 3 * n; i++) {
        float v = rgb[i];
        if (srgb) v = v > 0.0031308f ? 1.055f * powf(v, inv_gamma) - 0.055f : v * 12.92f;
        else v = powf(v, inv_gamma);
        rgb[i] = v;
        if (rgb8) rgb8[i] = (uint8_t)(clamp01(v) * 255.0f);
    }
    return 1;
}
