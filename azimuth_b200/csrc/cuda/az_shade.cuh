// Surface interaction on the device: hit attributes, textures, Perlin noise,
// bump mapping, BRDFs and light sampling, in azimuth's operation order.
#pragma once
#include "az_trace.cuh"

namespace azd {

// ---------------------------------------------------------------------------
// Textures, src/azimuth_texture.h:134-357
// ---------------------------------------------------------------------------
__device__ __forceinline__ float perlin_weight(float v) {  // :146-154
    v = fabsf(v);
    return 1.0f - ((((6.0f * v) - 15.0f) * v + 10.0f) * v * v * v);
}

// PerlinHash (:134-144).  azimuth adds s32 lattice coordinates to u32 table
// entries, so only the innermost K % 256 is a signed remainder; for K < 0 it
// indexes before the table, and the device table holds the 255 words azimuth
// reads there (az_scene_upload.cu, ToDevTexture).
__device__ __forceinline__ uint32_t perlin_hash(const uint32_t *P, int32_t i, int32_t j, int32_t k) {
    uint32_t a = __ldg(P + (k % 256));
    uint32_t b = __ldg(P + (((uint32_t)j + a) & 255u));
    return __ldg(P + (((uint32_t)i + b) & 255u));
}

static __device__ float sample_perlin(const DevScene &S, const DevTexture &t, f3 p) {  // :156-195
    float r = 0.0f;
    p = p * t.scaling;
    int32_t I = (int32_t)floorf(p.x), J = (int32_t)floorf(p.y), K = (int32_t)floorf(p.z);
    const uint32_t *P = S.perlin_perm + t.perm_offset;
    for (int32_t z = 0; z < 2; z++)
        for (int32_t y = 0; y < 2; y++)
            for (int32_t x = 0; x < 2; x++) {
                uint32_t h = perlin_hash(P, I + x, J + y, K + z) & 255u;
                f3 e = mk(__ldg(S.perlin_grad + 3 * h), __ldg(S.perlin_grad + 3 * h + 1), __ldg(S.perlin_grad + 3 * h + 2));
                f3 v = mk(p.x - (float)(I + x), p.y - (float)(J + y), p.z - (float)(K + z));
                r += dot(e, v) * perlin_weight(v.x) * perlin_weight(v.y) * perlin_weight(v.z);
            }
    if (t.appearance == 0) r = (r + 1.0f) / 2.0f;
    else r = fabsf(r);
    return r;
}

__device__ __forceinline__ f3 fetch_texel(const DevScene &S, const DevTexture &t, uint32_t x, uint32_t y) {
    uint32_t idx = (y * t.width + x) * 3u;
    if (t.format == 0) {
        const unsigned char *p = S.texels + t.texel_offset;
        return mk((float)p[idx], (float)p[idx + 1], (float)p[idx + 2]);
    }
    const float *p = reinterpret_cast<const float *>(S.texels + t.texel_offset);
    return mk(__ldg(p + idx), __ldg(p + idx + 1), __ldg(p + idx + 2));
}

static __device__ f3 sample_tex2d(const DevScene &S, const DevTexture &t, float u, float v, bool normalize_) {  // :239-339
    f3 r;
    if (t.wrap == 0) {
        float a = u < 1.0f ? u : 1.0f;
        u = 0.0f > a ? 0.0f : a;
        float b = v < 1.0f ? v : 1.0f;
        v = 0.0f > b ? 0.0f : b;
    } else {
        u = u - floorf(u);
        v = v - floorf(v);
    }
    if (t.filter == 0) {
        uint32_t fx = (uint32_t)floorf(u * ((float)t.width - 1.0f) + 0.5f);
        uint32_t fy = (uint32_t)floorf(v * ((float)t.height - 1.0f) + 0.5f);
        fx = min(fx, t.width - 1u);   // azimuth asserts these bounds (:206-207)
        fy = min(fy, t.height - 1u);
        r = fetch_texel(S, t, fx, fy);
    } else {
        float su = u * (float)t.width, sv = v * (float)t.height;
        uint32_t ax = (uint32_t)(su + 0.5f) % t.width;
        uint32_t ay = (uint32_t)(sv + 0.5f) % t.height;
        uint32_t bx = (ax - 1u) % t.width, by = ay % t.height;
        uint32_t cx = (ax - 1u) % t.width, cy = (ay - 1u) % t.height;
        uint32_t dx = ax % t.width, dy = (ay - 1u) % t.height;
        f3 A = fetch_texel(S, t, ax, ay), B = fetch_texel(S, t, bx, by);
        f3 C = fetch_texel(S, t, cx, cy), D = fetch_texel(S, t, dx, dy);
        su = floorf(su + 0.5f);
        sv = floorf(sv + 0.5f);
        if (su >= (float)t.width) su -= (float)t.width;
        if (sv >= (float)t.height) sv -= (float)t.height;
        float fx = su - (float)ax, fy = sv - (float)ay;
        r = A * (1.0f - fx) * (1.0f - fy) + B * fx * (1.0f - fy) + C * fx * fy + D * (1.0f - fx) * fy;
    }
    if (normalize_) {
        r.x /= t.normalizer;
        r.y /= t.normalizer;
        r.z /= t.normalizer;
    }
    return r;
}

__device__ __forceinline__ f3 sample_texture(const DevScene &S, const DevTexture &t, f3 p, float u, float v) {  // :341-357
    if (t.type == 0) return sample_tex2d(S, t, u, v, true);
    float n = sample_perlin(S, t, p);
    return mk(n, n, n);
}

// ---------------------------------------------------------------------------
// Hit attributes: the shading half of RayEntityIntersection
// (src/azimuth_main.cpp:64-146, :147-243, :244-281, bump :321-382)
// ---------------------------------------------------------------------------
struct Surface {
    f3 p, n;
    float u, v;
    uint32_t ent;
};

__device__ __forceinline__ void apply_bump(const DevScene &S, const DevTexture &tex, f3 pu, f3 pv, Surface &s) {
    if (tex.type == 0) {
        f3 A = sample_tex2d(S, tex, s.u, s.v, false);
        f3 B = sample_tex2d(S, tex, s.u + tex.inv_width, s.v, false);
        f3 C = sample_tex2d(S, tex, s.u, s.v + tex.inv_height, false);
        f3 du3 = B - A, dv3 = C - A;
        float du = ((du3.x + du3.y + du3.z) / 3.0f) * tex.bump_mul;
        float dv = ((dv3.x + dv3.y + dv3.z) / 3.0f) * tex.bump_mul;
        f3 dpu = pu + du * s.n, dpv = pv + dv * s.n;
        s.n = normalize(cross(dpv, dpu));
    } else {
        const float be = 0.001f;
        f3 p = s.p;
        float d = sample_perlin(S, tex, p);
        float dx = sample_perlin(S, tex, mk(p.x + be, p.y, p.z));
        float dy = sample_perlin(S, tex, mk(p.x, p.y + be, p.z));
        float dz = sample_perlin(S, tex, mk(p.x, p.y, p.z + be));
        f3 g = mk((dx - d) / be, (dy - d) / be, (dz - d) / be);
        s.n = s.n - g * tex.bump_mul;
        s.n = normalize(s.n);
    }
}

// Recompute P, normal and UV of a hit exactly as azimuth does when it finds it.
// TEX = false when the scene has no textures (no bump mapping to apply).
template <bool TEX>
__device__ Surface surface_at(const DevScene &S, const Ray &wr, const Hit &h) {
    Surface s;
    s.ent = h.ent;
    const DevEntity &e = S.ents[h.ent];
    if (h.prim == 0xFFFFFFFFu) {
        // sphere, :79-131
        f3 motion = wr.time * mk(e.motion[0], e.motion[1], e.motion[2]);
        Ray r = wr;
        r.o = wr.o - motion;
        Ray lr = local_ray(r, e.inv);
        f3 c = mk(e.center[0], e.center[1], e.center[2]);
        float t = h.tl;
        f3 hp = lr.o + (lr.d * t);
        f3 lhp = hp - c;
        f3 hn = normalize(lhp);
        f3 wp = point_xf(e.xf, hp) + motion;
        float theta = acosf(hn.y), phi = atan2f(hn.z, hn.x);
        const float two_pi = AZD_PI_F32 * 2.0f;
        s.p = wp;
        bool deferred = false;
        if (TEX && e.texture_index) {
            const DevTexture &tex = S.textures[e.texture_index - 1];
            s.n = hn;
            deferred = true;
            s.u = (-phi + AZD_PI_F32) / two_pi;
            s.v = theta / AZD_PI_F32;
            if (tex.bump) {
                float pypi = AZD_PI_F32 * lhp.y, rpi = AZD_PI_F32 * e.radius;
                f3 pv = mk(cosf(phi) * pypi, -sinf(theta) * rpi, sinf(phi) * pypi);
                f3 pu = mk(two_pi * lhp.z, 0.0f, -two_pi * lhp.x);
                apply_bump(S, tex, pu, pv, s);
            }
        } else {
            s.n = normal_xf(e.inv, hn);
            s.u = (-phi + AZD_PI_F32) / two_pi;
            s.v = theta / AZD_PI_F32;
        }
        if (deferred) s.n = normal_xf(e.inv, s.n);
        return s;
    }
    // triangle inside a group (mesh instances or top-level triangles)
    const DevTriAttr &a = S.tri_attr[h.prim];
    const DevGroup &g = S.groups[e.type == ENT_INSTANCE ? e.group : e.group];
    DevTri tr = load_tri(S.tris, h.prim);
    Ray lr = wr;
    f3 motion = mk(0.0f, 0.0f, 0.0f);
    if (!g.raw) {
        motion = wr.time * mk(g.motion[0], g.motion[1], g.motion[2]);
        Ray m = wr;
        m.o = wr.o - motion;
        lr = local_ray(m, g.inv);
    }
    // barycentrics from the same Cramer expressions as the test (:154-186)
    const float A = tr.a.w, D = tr.b.x, G = tr.b.y, B = tr.b.z, E = tr.b.w, H = tr.c.x;
    const float C = lr.d.x, F = lr.d.y, I = lr.d.z;
    float detM = (A * E * I) + (D * H * C) + (G * B * F) - (C * E * G) - (F * H * A) - (I * B * D);
    float K = tr.a.x - lr.o.x, M = tr.a.y - lr.o.y, N = tr.a.z - lr.o.z;
    float detB = (K * E * I) + (M * H * C) + (N * B * F) - (C * E * N) - (F * H * K) - (I * B * M);
    float detG = (A * M * I) + (D * N * C) + (G * K * F) - (C * M * G) - (F * N * A) - (I * K * D);
    float beta = detB / detM, gamma = detG / detM;
    float alpha = 1.0f - beta - gamma;
    float t = h.tl;
    s.p = lr.o + (lr.d * t);
    if (a.shading_mode == 0) {
        s.n = mk(tr.c.y, tr.c.z, tr.c.w);
    } else {
        s.n = alpha * mk(a.n0[0], a.n0[1], a.n0[2]) + beta * mk(a.n1[0], a.n1[1], a.n1[2]) +
              gamma * mk(a.n2[0], a.n2[1], a.n2[2]);
    }
    s.u = ((alpha * a.uv0[0]) + (beta * a.uv1[0])) + (gamma * a.uv2[0]);
    s.v = ((alpha * a.uv0[1]) + (beta * a.uv1[1])) + (gamma * a.uv2[1]);
    if (TEX && a.texture_index) {
        const DevTexture &tex = S.textures[a.texture_index - 1];
        if (tex.bump) {
            float div = ((a.uv1[0] - a.uv0[0]) * (a.uv2[1] - a.uv0[1])) - ((a.uv1[1] - a.uv0[1]) * (a.uv2[0] - a.uv0[0]));
            div = 1.0f / div;
            f3 e1 = mk(-A, -D, -G), e2 = mk(-B, -E, -H);   // P1-P0, P2-P0 (exact negations)
            f3 pu = (a.uv2[1] - a.uv0[1]) * e1 + (a.uv0[1] - a.uv1[1]) * e2;
            pu = pu * div;
            f3 pv = (a.uv0[0] - a.uv2[0]) * e1 + (a.uv1[0] - a.uv0[0]) * e2;
            pv = pv * div;
            apply_bump(S, tex, pu, pv, s);
        }
    }
    if (!g.raw) {
        // instance: world position and normal (:258-272)
        s.p = point_xf(g.xf, s.p) + motion;
        s.n = normal_xf(g.inv, s.n);
    }
    return s;
}

// Density over solid angle of the environment map's luminance CDF
// (DevScene.env_rows / env_cols) at direction d: p(u, v) / (2 pi^2 sin theta)
// with the equirectangular mapping of background().
__device__ __forceinline__ float env_cdf_pdf(const DevScene &S, f3 d) {
    const uint32_t H = S.env_cdf_h, W = S.env_cdf_w;
    const float theta = acosf(fminf(1.0f, fmaxf(-1.0f, d.y)));
    const float u = (-atan2f(d.z, d.x) + AZD_PI_F32) / (2.0f * AZD_PI_F32), v = theta / AZD_PI_F32;
    const uint32_t r = min((uint32_t)fmaxf(0.0f, v * (float)H), H - 1u);
    const uint32_t c = min((uint32_t)fmaxf(0.0f, u * (float)W), W - 1u);
    const float *cc = S.env_cols + (size_t)r * (W + 1);
    const float pdf_uv = (S.env_rows[r + 1] - S.env_rows[r]) * (cc[c + 1] - cc[c]) * (float)H * (float)W;
    const float st = sinf(theta);
    return st > 0.0f ? pdf_uv / (2.0f * AZD_PI_F32 * AZD_PI_F32 * st) : 0.0f;
}

// Environment light direction for AZ_FLAG_ENV_IMPORTANCE: one-sample MIS of
// the map's luminance CDF (row by the marginal over rows, column by the row's
// conditional, uniform within the texel, then the inverse equirectangular
// mapping theta = v pi, phi = pi - 2 pi u) and cosine sampling about n, half
// each (u1 < 1/2 picks the CDF; u1 is then rescaled), so that directions the
// CDF rarely proposes (sky behind an occluded sun) keep the cosine density.
// Returns 1 / (0.5 p_cdf + 0.5 p_cos), or 0 for a degenerate sample.
__device__ __forceinline__ float sample_env_mis(const DevScene &S, f3 n, float u1, float u2, f3 &dir) {
    if (u1 < 0.5f) {
        u1 = 2.0f * u1;
        const uint32_t H = S.env_cdf_h, W = S.env_cdf_w;
        uint32_t lo = 0, hi = H;   // largest r with rows[r] <= u1
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (S.env_rows[mid] <= u1) lo = mid;
            else hi = mid;
        }
        const uint32_t r = lo;
        const float pr = S.env_rows[r + 1] - S.env_rows[r];
        const float fr = pr > 0.0f ? fminf(0.99999994f, fmaxf(0.0f, (u1 - S.env_rows[r]) / pr)) : 0.5f;
        const float *cc = S.env_cols + (size_t)r * (W + 1);
        lo = 0;
        hi = W;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (cc[mid] <= u2) lo = mid;
            else hi = mid;
        }
        const uint32_t c = lo;
        const float pc = cc[c + 1] - cc[c];
        const float fc = pc > 0.0f ? fminf(0.99999994f, fmaxf(0.0f, (u2 - cc[c]) / pc)) : 0.5f;
        const float u = ((float)c + fc) / (float)W, v = ((float)r + fr) / (float)H;
        const float theta = v * AZD_PI_F32, phi = AZD_PI_F32 - 2.0f * AZD_PI_F32 * u;
        const float st = sinf(theta);
        dir = mk(st * cosf(phi), cosf(theta), st * sinf(phi));
    } else {
        u1 = 2.0f * u1 - 1.0f;
        const float theta = asinf(sqrtf(u1)), phi = 2.0f * AZD_PI_F32 * u2;
        f3 U, V;
        onb(n, U, V);
        dir = normalize(U * (sinf(theta) * cosf(phi)) + V * (sinf(theta) * sinf(phi)) + n * cosf(theta));
    }
    const float q = 0.5f * env_cdf_pdf(S, dir) + 0.5f * fmaxf(0.0f, dot(n, dir)) * (1.0f / AZD_PI_F32);
    return q > 0.0f ? 1.0f / q : 0.0f;
}

// Inputs of the path-guiding network at a hit: the world position o + t d
// and the geometric normal (face normal of the triangle, or centre-to-hit
// direction of the sphere), normalised.
__device__ __forceinline__ void guide_query(const DevScene &S, const Ray &wr, const Hit &h, f3 &p, f3 &n) {
    p = wr.o + wr.d * h.t;
    const DevEntity &e = S.ents[h.ent];
    if (h.prim == 0xFFFFFFFFu) {
        const f3 c = point_xf(e.xf, mk(e.center[0], e.center[1], e.center[2])) +
                     wr.time * mk(e.motion[0], e.motion[1], e.motion[2]);
        n = normalize(p - c);
    } else {
        const float4 c4 = S.tris[h.prim].c;
        f3 fn = mk(c4.y, c4.z, c4.w);
        const DevGroup &g = S.groups[e.group];
        if (!g.raw) fn = normal_xf(g.inv, fn);
        n = normalize(fn);
    }
}

// ---------------------------------------------------------------------------
// BRDFs and light contribution, src/azimuth_main.cpp:461-603
// ---------------------------------------------------------------------------
// The seven models share one powf(cos alpha, exponent): Phong-type models take
// cos alpha from the reflected light direction, Blinn-type models and
// Torrance-Sparrow from the half vector.  Each model's expression is azimuth's
// (same operations on the same values), so results are unchanged; warps whose
// lanes hold different models evaluate the power once instead of once per model.
static __device__ void eval_brdf(float &diffuse, float &specular, const DevMaterial &m, f3 L, f3 N, f3 V, float cti) {
    const float e = m.exponent;
    const uint32_t type = m.brdf_type;
    f3 hv = mk(0.0f, 0.0f, 0.0f);
    float ca;
    if (type <= 2) {
        ca = dot(-V, reflect(L, N));
    } else {
        hv = normalize(-V + L);
        ca = dot(N, hv);
    }
    const float p = ca > 0.0f ? powf(ca, e) : 0.0f;
    switch (type) {
        case 0:  // Phong
            specular = ca > 0.0f ? p / cti : 0.0f;
            break;
        case 1:  // Modified Phong
            specular = ca > 0.0f ? p : 0.0f;
            break;
        case 2:  // Normalized Modified Phong
            diffuse = (float)(1.0 / 3.14159265359);
            specular = ca > 0.0f ? ((e + 2.0f) / (2.0f * AZD_PI_F32)) * p : 0.0f;
            break;
        case 3:  // Blinn-Phong
            specular = ca > 0.0f ? p / cti : 0.0f;
            break;
        case 4:  // Modified Blinn-Phong
            specular = ca > 0.0f ? p : 0.0f;
            break;
        case 5:  // Normalized Modified Blinn-Phong
            diffuse = (float)(1.0 / 3.14159265359);
            specular = ca > 0.0f ? ((e + 8.0f) / (8.0f * AZD_PI_F32)) * p : 0.0f;
            break;
        default: {  // Torrance-Sparrow
            diffuse = (float)(1.0 / 3.14159265359);
            if (ca > 0.0f) {
                float D = ((e + 2.0f) / (2.0f * AZD_PI_F32)) * p;
                float nw0 = dot(N, -V), w0wh = dot(-V, hv);
                float G = nw0 < cti ? nw0 : cti;
                G = (2.0f * G * ca) / w0wh;
                G = 1.0f < G ? 1.0f : G;
                float ri = m.brdf_refractive_index;
                float r0 = ((ri - 1.0f) * (ri - 1.0f)) / ((ri + 1.0f) * (ri + 1.0f));
                float F = r0 + (1.0f - r0) * powf(1.0f - w0wh, 5.0f);
                specular = (D * F * G) / (4.0f * cti * nw0);
            } else {
                specular = 0.0f;
            }
        } break;
    }
}

// CalculateLightContribution (:571-603) from zero accumulators.
__device__ __forceinline__ bool light_contribution(f3 &dc, f3 &sc, const DevMaterial &m, f3 I, f3 ldir, f3 vdir,
                                                   f3 n, float ldist, float falloff, float invpdf) {
    float d2 = ldist * ldist;
    f3 ln = normalize(ldir);
    f3 li = mk(I.x / d2, I.y / d2, I.z / d2) * falloff;
    float cti = dot(n, ln);
    if (!(cti > 0.0f)) return false;
    float diffuse = 1.0f, specular = 1.0f;
    eval_brdf(diffuse, specular, m, ln, n, vdir, cti);
    f3 cm = li * cti * invpdf;
    dc = cm * diffuse;
    sc = cm * specular;
    return true;
}

// SampleEntityLight (:392-459): direction and inverse pdf.
static __device__ void sample_entity_light(const DevScene &S, const DevLight &L, f3 hp, NodeRng &rng, f3 &dir, float &invpdf) {
    f3 hpl = point_xf(L.inv, hp);
    f3 ldl = mk(0.0f, 0.0f, 0.0f);
    invpdf = 0.0f;
    if (L.entity_type == ENT_SPHERE) {
        f3 D = mk(L.center[0], L.center[1], L.center[2]) - hpl;
        float rod = L.radius / length(D);
        float ctm = sqrtf(1.0f - rod * rod);
        float ct = 1.0f + rng.next() * (ctm - 1.0f);
        float st = sqrtf(1.0f - ct * ct);
        float phi = 2.0f * AZD_PI_F32 * rng.next();
        float cp = cosf(phi), sp = sinf(phi);
        f3 W = normalize(D), U, V;
        onb(W, U, V);
        ldl = normalize(U * st * cp + V * st * sp + W * ct);
        invpdf = 2.0f * AZD_PI_F32 * (1.0f - ctm);
    } else {
        uint32_t idx = (uint32_t)(rng.next() * (float)L.tri_count);
        idx = min(idx, L.tri_count - 1u);
        const DevLightTri &T = S.light_tris[L.tri_offset + idx];
        float r1 = sqrtf(rng.next());
        float r2 = rng.next();
        f3 p0 = mk(T.p0n.x, T.p0n.y, T.p0n.z), p1 = mk(T.p1n.x, T.p1n.y, T.p1n.z), p2 = mk(T.p2n.x, T.p2n.y, T.p2n.z);
        f3 Q = (1.0f - r2) * p0 + r2 * p1;
        f3 P = (1.0f - r1) * p2 + r1 * Q;
        f3 wi = P - hpl;
        float area = L.total_area;
        ldl = normalize(wi);
        float ca = dot(ldl, mk(T.p0n.w, T.p1n.w, T.p2n.w));
        if (ca < 0.0f) ca *= -1.0f;
        float l = length(wi);
        invpdf = (area * ca) / (l * l);
    }
    dir = vector_xf(L.xf, ldl);
}

// Nearest hit of a ray on an entity light's own primitives, with azimuth's
// arithmetic (sphere :64-146; mesh instance :244-281 over the mesh's
// `triangle` array, whose vertices are the triangle entities' vertices).
// Returns 1 with the world t, 0 if the light is not hit, -1 if the light
// needs a full nearest-hit query instead (entity_light_needs_full_query).
// Called out of line by the visibility kernels (values and global pointers
// only), which keeps their traversal loop small.
struct LightHit {
    int hit;
    float t;   // world t when hit; FLT_MAX otherwise
};
static __device__ int light_entity_hit(const DevEntity *ents, const DevLightTri *light_tris, const DevLight &L,
                                       const Ray &wr, float &t_world);
static __device__ __noinline__ LightHit light_entity_hit_call(const DevEntity *ents, const DevLightTri *light_tris,
                                                             const DevLight *L, Ray wr) {
    LightHit h;
    h.t = FLT_MAX;
    h.hit = light_entity_hit(ents, light_tris, *L, wr, h.t);
    return h;
}
static __device__ int light_entity_hit(const DevEntity *ents, const DevLightTri *light_tris, const DevLight &L,
                                       const Ray &wr, float &t_world) {
    if (entity_light_needs_full_query(L)) return -1;
    if (L.entity_type == ENT_SPHERE) {
        float tl;
        return sphere_test(ents[L.ent_index], wr, 0.0f, t_world, tl) ? 1 : 0;
    }
    f3 motion = wr.time * mk(L.motion[0], L.motion[1], L.motion[2]);
    Ray m = wr;
    m.o = wr.o - motion;
    Ray lr = L.identity ? local_ray_identity(wr) : local_ray(m, L.inv);
    float best = FLT_MAX;
    for (uint32_t k = 0; k < L.tri_count; k++) {
        const DevLightTri &T = light_tris[L.tri_offset + k];
        DevTri tr;
        tr.a = make_float4(T.p0n.x, T.p0n.y, T.p0n.z, T.p0n.x - T.p1n.x);
        tr.b = make_float4(T.p0n.y - T.p1n.y, T.p0n.z - T.p1n.z, T.p0n.x - T.p2n.x, T.p0n.y - T.p2n.y);
        tr.c = make_float4(T.p0n.z - T.p2n.z, T.p0n.w, T.p1n.w, T.p2n.w);
        float t, b, g;
        if (tri_test(tr, lr, false, 0.0f, best, t, b, g)) best = t;
    }
    if (best == FLT_MAX) return 0;
    f3 lp = lr.o + (lr.d * best);
    f3 wp = point_xf(L.xf, lp) + motion;
    float wt = length(wp - m.o - motion) / length(wr.d);
    if (!(wt > 0.0f && wt < FLT_MAX)) return 0;
    t_world = wt;
    return 1;
}

// Background of a primary miss, SampleBackgroundColor (:1180-1207).
static __device__ f3 background(const DevScene &S, f3 d, int32_t w1, int32_t h1, uint32_t row, uint32_t col) {
    if (S.use_env_map) {
        float theta = acosf(d.y), phi = atan2f(d.z, d.x);
        float u = (-phi + AZD_PI_F32) / (2.0f * AZD_PI_F32), v = theta / AZD_PI_F32;
        return sample_texture(S, S.textures[S.env_texture], mk(u, v, 1.0f), u, v);
    }
    if (S.use_bg_texture) {
        float u = (float)col / (float)w1, v = (float)row / (float)h1;
        return sample_texture(S, S.textures[S.bg_texture], mk(u, v, 1.0f), u, v);
    }
    return mk(S.background[0], S.background[1], S.background[2]);
}

}  // namespace azd
