// Shading stage of the wave (TraceRay body, src/azimuth_main.cpp:974-1130),
// in a translation unit of its own (its 48 specialisations compile beside the
// traversal kernels).  Like the traversal it is compiled without FMA
// contraction, so that textures, Perlin noise and the finite differences of
// bump mapping round like azimuth's.
#include <cfloat>

#include "az_render.h"
#include "az_shade.cuh"
#include "az_wave.cuh"

namespace az {
namespace {

using namespace azd;

__device__ __forceinline__ f3 ld3(const float *p) { return mk(p[0], p[1], p[2]); }

// One tree node: direct light, ambient and children (TraceRay body,
// src/azimuth_main.cpp:974-1130).  FEAT (DevScene.features) compiles out the
// parts a scene cannot reach: textures, environment map, mirror/dielectric
// branches, point/area/directional/spot lights.  MULTI: a tile wave of
// several scenes, each entry shaded in the scene its flags name (FEAT then
// covers every scene of the wave).
template <int BLOCK, uint32_t FEAT, bool GUIDED, bool TILES = false, bool MULTI = false>
__global__ void __launch_bounds__(BLOCK) k_shade(DevScene S0, CameraParams cam, WaveQueues Q, uint64_t wave_start,
                                                 uint32_t level) {
    constexpr bool TEX = FEAT & FEAT_TEXTURES, ENV = FEAT & FEAT_ENV, SPECIAL = FEAT & FEAT_SPECIAL,
                   LIGHTS = FEAT & FEAT_ANALYTIC_LIGHTS;
    const int buf = level & 1, nbuf = buf ^ 1;
    const uint32_t n = min(Q.counts[level], Q.cap_q);
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
        const uint32_t sbits = flags & PF_SCENE;   // children and light samples keep the entry's scene
        const DevScene &S = MULTI ? Q.scenes[sbits >> PF_SCENE_SHIFT] : S0;
        const bool can_spawn = level + 1 <= S.max_depth + 1;   // child's RecursionDepth <= MaxRecursionDepth
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
                        kind >= SHADOW_ENTITY ? li : 0u, sbits >> PF_SCENE_SHIFT);
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
                if (!is_zero(c))
                    push_shadow(Q, level, s.p + (Ld * seps), r.time, Ld, FLT_MAX, c, slot, SHADOW_ANY, 0u,
                                sbits >> PF_SCENE_SHIFT);
            }
        }
        uint32_t next_child = 0;
        // a vertex that may spawn more than one child marks its subtree
        const bool multi = SPECIAL && S.path_trace && (m.is_mirror || m.transparent);
        const uint32_t bflag = (((flags & PF_BRANCHED) || multi) ? PF_BRANCHED : 0u) | sbits;
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


constexpr int kBlock = 128;

template <uint32_t F>
void LaunchShadeF(int grid, const DevScene &S, const CameraParams &cam, const WaveQueues &Q, uint64_t start,
                  uint32_t L, cudaStream_t st, bool guided) {
    if (Q.scenes) k_shade<kBlock, F, false, true, true><<<grid, kBlock, 0, st>>>(S, cam, Q, start, L);   // several scenes
    else if (Q.slot_map) k_shade<kBlock, F, false, true><<<grid, kBlock, 0, st>>>(S, cam, Q, start, L);   // tile wave
    else if (guided) k_shade<kBlock, F, true><<<grid, kBlock, 0, st>>>(S, cam, Q, start, L);
    else k_shade<kBlock, F, false><<<grid, kBlock, 0, st>>>(S, cam, Q, start, L);
}


}  // namespace

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

}  // namespace az
