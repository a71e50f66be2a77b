// Seeded procedural scenes in azimuth's structs (see include/azimuth_scenes.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <unordered_map>
#include <vector>

#include "az_scene_build.h"
#include "azimuth_scenes.h"

namespace az {
namespace {

const double kPi = 3.14159265358979323846;

inline az_vec3 V3(float x, float y, float z) { return az_vec3{x, y, z}; }

// SplitMix64 (Steele, Lea, Flood 2014): the generators' own seeded stream.
struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    float uniform(float a, float b) { return (float)(a + (b - a) * uniform()); }
    float loguniform(float a, float b) { return (float)exp(log(a) + (log(b) - log(a)) * uniform()); }
    double normal() {  // Box-Muller
        double u1 = uniform(), u2 = uniform();
        if (u1 < 1e-300) u1 = 1e-300;
        return sqrt(-2.0 * log(u1)) * cos(2.0 * kPi * u2);
    }
};

// Classic 3D gradient noise (Perlin 2002 "improved noise": quintic fade, 12
// edge gradients) with a seeded permutation; used only to displace geometry.
struct GeoNoise {
    int perm[512];
    explicit GeoNoise(uint64_t seed) {
        Rng r(seed ^ 0xA5A5A5A5ull);
        int p[256];
        for (int i = 0; i < 256; i++) p[i] = i;
        for (int i = 255; i > 0; i--) {
            int j = (int)(r.next() % (uint64_t)(i + 1));
            int t = p[i]; p[i] = p[j]; p[j] = t;
        }
        for (int i = 0; i < 512; i++) perm[i] = p[i & 255];
    }
    static double fade(double t) { return t * t * t * (t * (t * 6 - 15) + 10); }
    static double grad(int h, double x, double y, double z) {
        int g = h % 12;
        double u = g < 8 ? x : y, v = g < 4 ? y : (g == 12 || g == 14 ? x : z);
        return ((g & 1) ? -u : u) + ((g & 2) ? -v : v);
    }
    double noise(double x, double y, double z) const {
        double fx = floor(x), fy = floor(y), fz = floor(z);
        int X = (int)fx & 255, Y = (int)fy & 255, Z = (int)fz & 255;
        x -= fx; y -= fy; z -= fz;
        double u = fade(x), v = fade(y), w = fade(z);
        int A = perm[X] + Y, AA = perm[A] + Z, AB = perm[A + 1] + Z;
        int B = perm[X + 1] + Y, BA = perm[B] + Z, BB = perm[B + 1] + Z;
        auto lerp = [](double t, double a, double b) { return a + t * (b - a); };
        return lerp(w, lerp(v, lerp(u, grad(perm[AA], x, y, z), grad(perm[BA], x - 1, y, z)),
                            lerp(u, grad(perm[AB], x, y - 1, z), grad(perm[BB], x - 1, y - 1, z))),
                    lerp(v, lerp(u, grad(perm[AA + 1], x, y, z - 1), grad(perm[BA + 1], x - 1, y, z - 1)),
                         lerp(u, grad(perm[AB + 1], x, y - 1, z - 1), grad(perm[BB + 1], x - 1, y - 1, z - 1))));
    }
    double fbm(double x, double y, double z, int octaves) const {
        double s = 0, a = 1, f = 1;
        for (int o = 0; o < octaves; o++) {
            s += a * noise(x * f, y * f, z * f);
            a *= 0.5;
            f *= 2.0;
        }
        return s;
    }
};

struct Generated {
    SceneBuilder B;
    az_camera Camera;
    az_epsilon_values Eps;
    std::vector<float> Gradients;
    uint64_t Triangles = 0, Spheres = 0;
};

uint32_t AddV(Generated &G, az_vec3 p, az_vec2 uv = az_vec2{0, 0}) {
    G.B.AddUV(uv);
    return G.B.AddVertex(p);
}

// Quad p0..p3 as triangles (p0,p1,p2), (p0,p2,p3); its face normal is
// cross(p1-p0, p2-p0).
void AddQuad(Generated &G, MeshDesc &M, az_vec3 p0, az_vec3 p1, az_vec3 p2, az_vec3 p3,
             bool uv01 = false) {
    uint32_t a = AddV(G, p0, uv01 ? az_vec2{0, 0} : az_vec2{0, 0});
    uint32_t b = AddV(G, p1, uv01 ? az_vec2{0, 1} : az_vec2{0, 0});
    uint32_t c = AddV(G, p2, uv01 ? az_vec2{1, 1} : az_vec2{0, 0});
    uint32_t d = AddV(G, p3, uv01 ? az_vec2{1, 0} : az_vec2{0, 0});
    M.Faces.push_back(az_vec3u{a, b, c});
    M.Faces.push_back(az_vec3u{a, c, d});
}

az_material Lambert(float r, float g, float b) {
    // Lambertian = NormalizedModifiedBlinnPhong with zero specular: Diffuse = 1/pi
    // (src/azimuth_main.cpp:528).
    az_material M = DefaultMaterial();
    M.BRDF.Type = AZ_BRDF_NormalizedModifiedBlinnPhong;
    M.BRDF.Exponent = 1.0f;
    M.DiffuseReflectance = V3(r, g, b);
    return M;
}

struct Box {
    float x0, x1, y0, y1, z0, z1;
};

// Cornell walls with interior-facing normals; the front (z1) stays open.
void CornellWalls(Generated &G, const Box &b, uint32_t white, uint32_t red, uint32_t green,
                  bool floorUV = false, uint32_t floorTex = 0, uint32_t backMat = UINT32_MAX,
                  uint32_t backTex = 0, uint32_t ceilMat = UINT32_MAX) {
    MeshDesc W;
    W.MaterialIndex = white;
    MeshDesc Floor;
    Floor.MaterialIndex = white;
    Floor.TextureIndex = floorTex;
    AddQuad(G, floorTex ? Floor : W, V3(b.x0, b.y0, b.z0), V3(b.x0, b.y0, b.z1), V3(b.x1, b.y0, b.z1),
            V3(b.x1, b.y0, b.z0), floorUV);
    MeshDesc Ceil;
    Ceil.MaterialIndex = ceilMat == UINT32_MAX ? white : ceilMat;
    AddQuad(G, ceilMat == UINT32_MAX ? W : Ceil, V3(b.x0, b.y1, b.z0), V3(b.x1, b.y1, b.z0),
            V3(b.x1, b.y1, b.z1), V3(b.x0, b.y1, b.z1));
    MeshDesc Back;
    Back.MaterialIndex = backMat == UINT32_MAX ? white : backMat;
    Back.TextureIndex = backTex;
    AddQuad(G, backMat == UINT32_MAX ? W : Back, V3(b.x0, b.y0, b.z0), V3(b.x1, b.y0, b.z0),
            V3(b.x1, b.y1, b.z0), V3(b.x0, b.y1, b.z0));
    MeshDesc L;
    L.MaterialIndex = red;
    AddQuad(G, L, V3(b.x0, b.y0, b.z0), V3(b.x0, b.y1, b.z0), V3(b.x0, b.y1, b.z1), V3(b.x0, b.y0, b.z1));
    MeshDesc R;
    R.MaterialIndex = green;
    AddQuad(G, R, V3(b.x1, b.y0, b.z0), V3(b.x1, b.y0, b.z1), V3(b.x1, b.y1, b.z1), V3(b.x1, b.y1, b.z0));
    if (!W.Faces.empty()) G.B.AddMesh(W);
    if (floorTex) G.B.AddMesh(Floor);
    if (ceilMat != UINT32_MAX) G.B.AddMesh(Ceil);
    if (backMat != UINT32_MAX) G.B.AddMesh(Back);
    G.B.AddMesh(L);
    G.B.AddMesh(R);
    G.Triangles += 10;
}

// Emitting quad of size s x s just below the ceiling, facing down; listed as
// an entity light like azimuth's <LightMesh>.
void CeilingLight(Generated &G, float cx, float cz, float s, float y, float radiance, uint32_t mat) {
    MeshDesc M;
    M.MaterialIndex = mat;
    M.IsEmitter = true;
    M.IsLight = true;
    M.Radiance = V3(radiance, radiance, radiance);
    float h = s * 0.5f;
    AddQuad(G, M, V3(cx - h, y, cz - h), V3(cx + h, y, cz - h), V3(cx + h, y, cz + h), V3(cx - h, y, cz + h));
    G.B.AddMesh(M);
    G.Triangles += 2;
}

az_entity Sphere(az_vec3 c, float r, uint32_t mat) {
    az_entity E = DefaultEntity();
    E.Center = c;
    E.Radius = r;
    E.MaterialIndex = mat;
    return E;
}

void SimpleCamera(Generated &G, az_vec3 pos, az_vec3 gaze, float fovy, uint32_t w, uint32_t h, uint32_t spp) {
    G.Camera = DefaultCamera();
    G.Camera.Type = AZ_Camera_Simple;
    G.Camera.FovY = fovy;
    G.Camera.Position = pos;
    G.Camera.Gaze = gaze;
    G.Camera.Up = V3(0, 1, 0);
    G.Camera.NearDistance = 1.0f;
    G.Camera.Resolution = az_vec2u{w, h};
    G.Camera.SampleCount = spp;
}

// Icosahedron subdivided `levels` times onto the unit sphere.
void Icosphere(int levels, std::vector<az_vec3> &V, std::vector<az_vec3u> &F) {
    const double t = (1.0 + sqrt(5.0)) / 2.0;
    const double base[12][3] = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                                {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
    const int faces[20][3] = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11},
                              {1, 5, 9}, {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
                              {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8}, {3, 8, 9},
                              {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
    std::vector<double> P;
    auto push = [&](double x, double y, double z) {
        double l = sqrt(x * x + y * y + z * z);
        P.push_back(x / l); P.push_back(y / l); P.push_back(z / l);
        return (uint32_t)(P.size() / 3 - 1);
    };
    for (auto &b : base) push(b[0], b[1], b[2]);
    std::vector<az_vec3u> cur;
    for (auto &f : faces) cur.push_back(az_vec3u{(uint32_t)f[0], (uint32_t)f[1], (uint32_t)f[2]});
    for (int l = 0; l < levels; l++) {
        std::unordered_map<uint64_t, uint32_t> mid;
        mid.reserve(cur.size() * 2);
        auto midpoint = [&](uint32_t a, uint32_t b) {
            uint64_t key = a < b ? ((uint64_t)a << 32 | b) : ((uint64_t)b << 32 | a);
            auto it = mid.find(key);
            if (it != mid.end()) return it->second;
            uint32_t m = push(P[3 * a] + P[3 * b], P[3 * a + 1] + P[3 * b + 1], P[3 * a + 2] + P[3 * b + 2]);
            mid.emplace(key, m);
            return m;
        };
        std::vector<az_vec3u> nxt;
        nxt.reserve(cur.size() * 4);
        for (auto &f : cur) {
            uint32_t a = midpoint(f.x, f.y), b = midpoint(f.y, f.z), c = midpoint(f.z, f.x);
            nxt.push_back(az_vec3u{f.x, a, c});
            nxt.push_back(az_vec3u{f.y, b, a});
            nxt.push_back(az_vec3u{f.z, c, b});
            nxt.push_back(az_vec3u{a, b, c});
        }
        cur.swap(nxt);
    }
    V.resize(P.size() / 3);
    for (size_t i = 0; i < V.size(); i++) V[i] = V3((float)P[3 * i], (float)P[3 * i + 1], (float)P[3 * i + 2]);
    // outward winding: cross(p1-p0, p2-p0) points away from the centre
    for (auto &f : cur) {
        const az_vec3 &a = V[f.x], &b = V[f.y], &c = V[f.z];
        double ux = b.x - a.x, uy = b.y - a.y, uz = b.z - a.z, vx = c.x - a.x, vy = c.y - a.y, vz = c.z - a.z;
        double nx = uy * vz - uz * vy, ny = uz * vx - ux * vz, nz = ux * vy - uy * vx;
        if (nx * (a.x + b.x + c.x) + ny * (a.y + b.y + c.y) + nz * (a.z + b.z + c.z) < 0) std::swap(f.y, f.z);
    }
    F.swap(cur);
}

// One material per azimuth BRDF model, parameters drawn from `r`.
// Non-normalised models use Diffuse = 1 (src/azimuth_main.cpp:588), so their
// diffuse albedo is kept below 1/pi to keep the path throughput bounded.
az_material RandomBRDFMaterial(Rng &r, uint32_t type) {
    az_material M = DefaultMaterial();
    M.BRDF.Type = type;
    M.BRDF.Exponent = r.loguniform(2.0f, 200.0f);
    M.BRDF.RefractiveIndex = r.uniform(1.2f, 2.5f);
    bool normalized = type == AZ_BRDF_NormalizedModifiedPhong ||
                      type == AZ_BRDF_NormalizedModifiedBlinnPhong || type == AZ_BRDF_TorranceSparrow;
    float dmax = normalized ? 0.8f : 0.25f;
    M.DiffuseReflectance = V3(r.uniform(0.05f, dmax), r.uniform(0.05f, dmax), r.uniform(0.05f, dmax));
    float smax = normalized ? 0.5f : 0.08f;
    M.SpecularReflectance = V3(r.uniform(0.0f, smax), r.uniform(0.0f, smax), r.uniform(0.0f, smax));
    return M;
}

// Equirectangular HDR sky in azimuth's mapping (src/azimuth_main.cpp:1187-1191):
// u = (pi - atan2(z, x)) / 2pi, v = acos(y) / pi; RGB F32, Normalizer 1.
az_texture SkyTexture(Generated &G, uint32_t w, uint32_t h, az_vec3 sunDir, float sunSigmaDeg, float sunPeak) {
    az_texture T = DefaultTexture();
    T.Type = AZ_TextureType_2D;
    T.PixelFormat = AZ_PixelFormat_RGB_F32;
    T.Width = w;
    T.Height = h;
    T.InvWidth = 1.0f / (float)w;
    T.InvHeight = 1.0f / (float)h;
    T.Normalizer = 1.0f;
    T.Loaded = 1;
    T.WrapMode = AZ_TextureWrap_Repeat;
    T.Filter = AZ_TextureFilter_Nearest;
    float *px = (float *)G.B.AllocTexels(sizeof(float) * 3 * (size_t)w * h);
    double sl = sqrt((double)sunDir.x * sunDir.x + (double)sunDir.y * sunDir.y + (double)sunDir.z * sunDir.z);
    double sx = sunDir.x / sl, sy = sunDir.y / sl, sz = sunDir.z / sl;
    double sig = sunSigmaDeg * kPi / 180.0;
    for (uint32_t y = 0; y < h; y++) {
        double theta = kPi * ((double)y + 0.5) / (double)h;
        for (uint32_t x = 0; x < w; x++) {
            double phi = kPi - 2.0 * kPi * ((double)x + 0.5) / (double)w;
            double dx = sin(theta) * cos(phi), dy = cos(theta), dz = sin(theta) * sin(phi);
            double r, g, b;
            if (dy >= 0) {
                double k = pow(dy, 0.4);
                r = 0.9 * (1 - k) + 0.25 * k;
                g = 0.9 * (1 - k) + 0.45 * k;
                b = 0.95 * (1 - k) + 0.95 * k;
            } else {
                r = g = b = 0.18;
            }
            double c = dx * sx + dy * sy + dz * sz;
            double ang = acos(c > 1 ? 1 : (c < -1 ? -1 : c));
            double sun = sunPeak * exp(-ang * ang / (2 * sig * sig));
            float *p = px + 3 * ((size_t)y * w + x);
            p[0] = (float)(r + sun);
            p[1] = (float)(g + sun * 0.95);
            p[2] = (float)(b + sun * 0.85);
        }
    }
    T.Pixels = px;
    return T;
}

az_texture CheckerTexture(Generated &G, uint32_t n, uint32_t filter, uint32_t wrap) {
    az_texture T = DefaultTexture();
    T.Type = AZ_TextureType_2D;
    T.PixelFormat = AZ_PixelFormat_RGB_U8;
    T.Width = n;
    T.Height = n;
    T.InvWidth = 1.0f / (float)n;
    T.InvHeight = 1.0f / (float)n;
    T.Loaded = 1;
    T.Filter = filter;
    T.WrapMode = wrap;
    uint8_t *px = (uint8_t *)G.B.AllocTexels(3 * (size_t)n * n);
    for (uint32_t y = 0; y < n; y++)
        for (uint32_t x = 0; x < n; x++) {
            bool on = ((x / 8) + (y / 8)) & 1;
            uint8_t *p = px + 3 * ((size_t)y * n + x);
            p[0] = on ? 230 : (uint8_t)(20 + 3 * x);
            p[1] = on ? 220 : (uint8_t)(30 + 2 * y);
            p[2] = on ? 200 : 60;
        }
    T.Pixels = px;
    return T;
}

// Perlin texture tables in the form azimuth's InitPerlinNoise leaves them
// (src/azimuth_texture.h:106-132): 256 unit gradients (shared) and a
// per-texture permutation of 0..255 from a Fisher-Yates shuffle.
void PerlinTables(Generated &G, Rng &r, az_texture &T) {
    if (G.Gradients.empty()) {
        G.Gradients.resize(3 * AZ_PERLIN_GRADIENT_SIZE);
        for (int i = 0; i < AZ_PERLIN_GRADIENT_SIZE; i++) {
            float x, y, z, l;
            do {
                x = r.uniform(-1, 1); y = r.uniform(-1, 1); z = r.uniform(-1, 1);
                l = sqrtf(x * x + y * y + z * z);
            } while (l < 1e-3f);
            G.Gradients[3 * i] = x / l; G.Gradients[3 * i + 1] = y / l; G.Gradients[3 * i + 2] = z / l;
        }
    }
    for (uint32_t i = 0; i < AZ_PERLIN_GRADIENT_SIZE; i++) T.Perm[i] = i;
    for (uint32_t i = AZ_PERLIN_GRADIENT_SIZE - 1; i > 0; i--) {
        uint32_t j = (uint32_t)(r.next() % (uint64_t)(i + 1));
        uint32_t t = T.Perm[i]; T.Perm[i] = T.Perm[j]; T.Perm[j] = t;
    }
}

uint32_t Def(uint32_t v, uint32_t d) { return v ? v : d; }

bool GenCornell(Generated &G, const az_gen_params &p, uint64_t seed) {
    (void)seed;
    uint32_t white = G.B.AddMaterial(Lambert(0.73f, 0.73f, 0.73f));
    uint32_t red = G.B.AddMaterial(Lambert(0.65f, 0.05f, 0.05f));
    uint32_t green = G.B.AddMaterial(Lambert(0.12f, 0.45f, 0.15f));
    az_material mirror = DefaultMaterial();
    mirror.BRDF.Type = AZ_BRDF_NormalizedModifiedBlinnPhong;
    mirror.BRDF.Exponent = 1.0f;
    mirror.MirrorReflectance = V3(1, 1, 1);
    uint32_t mir = G.B.AddMaterial(mirror);
    CornellWalls(G, Box{-0.5f, 0.5f, 0.0f, 1.0f, -0.5f, 0.5f}, white, red, green);
    CeilingLight(G, 0.0f, 0.0f, 0.25f, 0.999f, 15.0f, white);
    G.B.AddSphere(Sphere(V3(-0.2f, 0.2f, -0.15f), 0.2f, white), false);
    G.B.AddSphere(Sphere(V3(0.22f, 0.2f, 0.12f), 0.2f, mir), false);
    G.Spheres = 2;
    az_scene &S = G.B.Scene;
    S.MaxRecursionDepth = Def(p.max_depth, 5);
    S.PathTrace = 1;
    S.ImportanceSampling = p.importance_sampling >= 0 ? (uint32_t)p.importance_sampling : 0u;
    uint32_t w = Def(p.width, 256), h = Def(p.height, 256);
    SimpleCamera(G, V3(0.0f, 0.5f, 1.9f), V3(0, 0, -1), 40.0f, w, h, Def(p.spp, 16));
    return true;
}

bool GenDenseMesh(Generated &G, const az_gen_params &p, uint64_t seed) {
    Rng r(seed + 1);
    uint32_t white = G.B.AddMaterial(Lambert(0.73f, 0.73f, 0.73f));
    uint32_t red = G.B.AddMaterial(Lambert(0.65f, 0.05f, 0.05f));
    uint32_t green = G.B.AddMaterial(Lambert(0.12f, 0.45f, 0.15f));
    CornellWalls(G, Box{-0.5f, 0.5f, 0.0f, 1.0f, -0.5f, 0.5f}, white, red, green);
    CeilingLight(G, 0.0f, 0.0f, 0.25f, 0.999f, 15.0f, white);
    uint32_t mats[7];
    for (uint32_t k = 0; k < 7; k++) mats[k] = G.B.AddMaterial(RandomBRDFMaterial(r, k));
    std::vector<az_vec3> V;
    std::vector<az_vec3u> F;
    Icosphere((int)Def(p.detail, 8), V, F);
    GeoNoise noise(seed);
    const az_vec3 c = V3(0.0f, 0.42f, -0.05f);
    const double R = 0.3, A = 0.05, freq = 4.0;
    uint32_t base = (uint32_t)G.B.Vertices.size();
    for (const az_vec3 &n : V) {
        double d = R + A * noise.fbm(n.x * freq + 17.0, n.y * freq + 17.0, n.z * freq + 17.0, 3);
        AddV(G, V3((float)(c.x + n.x * d), (float)(c.y + n.y * d), (float)(c.z + n.z * d)),
             az_vec2{(float)(0.5 + atan2(n.z, n.x) / (2 * kPi)), (float)(acos(n.y) / kPi)});
    }
    MeshDesc M[7];
    for (uint32_t k = 0; k < 7; k++) {
        M[k].MaterialIndex = mats[k];
        M[k].ShadingMode = AZ_Shading_Smooth;
        M[k].Faces.reserve(F.size() / 7 + 1);
    }
    for (size_t f = 0; f < F.size(); f++)
        M[f % 7].Faces.push_back(az_vec3u{base + F[f].x, base + F[f].y, base + F[f].z});
    for (uint32_t k = 0; k < 7; k++)
        if (!M[k].Faces.empty()) G.B.AddMesh(M[k]);
    G.Triangles += F.size();
    az_scene &S = G.B.Scene;
    S.MaxRecursionDepth = Def(p.max_depth, 8);
    S.PathTrace = 1;
    S.ImportanceSampling = p.importance_sampling >= 0 ? (uint32_t)p.importance_sampling : 1u;
    SimpleCamera(G, V3(0.0f, 0.5f, 1.9f), V3(0, 0, -1), 40.0f, Def(p.width, 1024), Def(p.height, 1024),
                 Def(p.spp, 64));
    return true;
}

bool GenMotionEnv(Generated &G, const az_gen_params &p, uint64_t seed) {
    Rng r(seed + 2);
    uint32_t n = Def(p.detail, 10000);
    az_material diel = DefaultMaterial();
    diel.Transparency = V3(1, 1, 1);
    diel.RefractionIndex = 1.5f;
    uint32_t dielMat = G.B.AddMaterial(diel);
    uint32_t mats[7];
    for (uint32_t k = 0; k < 7; k++) mats[k] = G.B.AddMaterial(RandomBRDFMaterial(r, k));
    for (uint32_t i = 0; i < n; i++) {
        float rad = r.loguniform(0.01f, 0.1f);
        az_vec3 c = V3(r.uniform(0, 10), r.uniform(0, 10), r.uniform(0, 10));
        az_entity E = Sphere(c, rad, 0);
        E.MotionVector = V3((float)(0.2 * r.normal()), (float)(0.2 * r.normal()), (float)(0.2 * r.normal()));
        E.MaterialIndex = r.uniform() < 0.3 ? dielMat : mats[r.next() % 7];
        G.B.AddSphere(E, false);
    }
    G.Spheres = n;
    az_scene &S = G.B.Scene;
    S.EnvironmentMap = SkyTexture(G, Def(p.env_width, 2048), Def(p.env_height, 1024), V3(0.4f, 0.7f, 0.35f),
                                  1.0f, 5.0e4f);
    S.UseEnvironmentMap = 1;
    S.MaxRecursionDepth = Def(p.max_depth, 12);
    S.PathTrace = 1;
    S.ImportanceSampling = p.importance_sampling >= 0 ? (uint32_t)p.importance_sampling : 1u;
    SimpleCamera(G, V3(5.0f, 5.0f, 22.0f), V3(0, 0, -1), 40.0f, Def(p.width, 1920), Def(p.height, 1080),
                 Def(p.spp, 32));
    return true;
}

// Tessellated panel: origin o, edge vectors eu (nu cells) and ev (nv cells),
// every interior vertex displaced along nrm by amp * fbm(position * freq);
// faces wound so that the face normal is cross(eu, ev).  Cells whose centre
// lies inside `hole` (fractions of the two edges) are left out (doorways).
struct Hole {
    float u0, u1, v0, v1;   // u0 >= u1: none
};

uint64_t TessPanel(Generated &G, MeshDesc &M, az_vec3 o, az_vec3 eu, az_vec3 ev, uint32_t nu, uint32_t nv,
                   az_vec3 nrm, const GeoNoise &noise, double amp, double freq, Hole hole = Hole{1, 0, 1, 0}) {
    const uint32_t base = (uint32_t)G.B.Vertices.size();
    for (uint32_t j = 0; j <= nv; j++)
        for (uint32_t i = 0; i <= nu; i++) {
            const double fu = (double)i / nu, fv = (double)j / nv;
            double px = o.x + eu.x * fu + ev.x * fv, py = o.y + eu.y * fu + ev.y * fv, pz = o.z + eu.z * fu + ev.z * fv;
            // panel edges stay put so that neighbouring panels meet without cracks
            const bool edge = i == 0 || j == 0 || i == nu || j == nv;
            const double d = edge ? 0.0 : amp * noise.fbm(px * freq + 3.1, py * freq + 7.7, pz * freq + 1.3, 3);
            AddV(G, V3((float)(px + nrm.x * d), (float)(py + nrm.y * d), (float)(pz + nrm.z * d)),
                 az_vec2{(float)fu, (float)fv});
        }
    uint64_t tris = 0;
    for (uint32_t j = 0; j < nv; j++)
        for (uint32_t i = 0; i < nu; i++) {
            const float cu = (i + 0.5f) / nu, cv = (j + 0.5f) / nv;
            if (cu > hole.u0 && cu < hole.u1 && cv > hole.v0 && cv < hole.v1) continue;
            const uint32_t a = base + j * (nu + 1) + i, b = a + 1, c = a + (nu + 1) + 1, d = a + (nu + 1);
            M.Faces.push_back(az_vec3u{a, b, c});
            M.Faces.push_back(az_vec3u{a, c, d});
            tris += 2;
        }
    return tris;
}

// Axis-aligned box with outward faces, each face a panel of n x n cells.
uint64_t TessBox(Generated &G, MeshDesc &M, const Box &b, uint32_t n, const GeoNoise &noise, double amp) {
    const float dx = b.x1 - b.x0, dy = b.y1 - b.y0, dz = b.z1 - b.z0;
    uint64_t t = 0;
    t += TessPanel(G, M, V3(b.x0, b.y1, b.z0), V3(0, 0, dz), V3(dx, 0, 0), n, n, V3(0, 1, 0), noise, amp, 6.0);   // top
    t += TessPanel(G, M, V3(b.x0, b.y0, b.z0), V3(dx, 0, 0), V3(0, 0, dz), n, n, V3(0, -1, 0), noise, amp, 6.0);  // bottom
    t += TessPanel(G, M, V3(b.x0, b.y0, b.z1), V3(dx, 0, 0), V3(0, dy, 0), n, n, V3(0, 0, 1), noise, amp, 6.0);   // +z
    t += TessPanel(G, M, V3(b.x1, b.y0, b.z0), V3(-dx, 0, 0), V3(0, dy, 0), n, n, V3(0, 0, -1), noise, amp, 6.0); // -z
    t += TessPanel(G, M, V3(b.x1, b.y0, b.z1), V3(0, 0, -dz), V3(0, dy, 0), n, n, V3(1, 0, 0), noise, amp, 6.0);  // +x
    t += TessPanel(G, M, V3(b.x0, b.y0, b.z0), V3(0, 0, dz), V3(0, dy, 0), n, n, V3(-1, 0, 0), noise, amp, 6.0);  // -x
    return t;
}

// Interior: three 8 x 4 x 8 rooms in a row along x, joined by 1 x 2 doorways
// in 0.2-thick inner walls, every surface a Perlin-displaced panel tessellated
// at `detail` cells per metre (default 49: about 4 M triangles with the
// clutter), 12 clutter boxes per room, one 1 x 1 area light under the ceiling
// of room 1 and the camera in room 3 looking back through the doorways.
bool GenInterior(Generated &G, const az_gen_params &p, uint64_t seed) {
    Rng r(seed + 3);
    GeoNoise noise(seed + 33);
    const uint32_t cpm = Def(p.detail, 49);
    const double amp = 0.015, freq = 2.5;
    uint32_t wall = G.B.AddMaterial(Lambert(0.75f, 0.73f, 0.70f));
    uint32_t floorm = G.B.AddMaterial(Lambert(0.55f, 0.45f, 0.35f));
    uint32_t ceil = G.B.AddMaterial(Lambert(0.80f, 0.80f, 0.80f));
    uint32_t clutter[4] = {G.B.AddMaterial(Lambert(0.65f, 0.20f, 0.15f)), G.B.AddMaterial(Lambert(0.20f, 0.50f, 0.25f)),
                           G.B.AddMaterial(Lambert(0.20f, 0.30f, 0.65f)), G.B.AddMaterial(Lambert(0.70f, 0.65f, 0.30f))};
    const float W = 8.0f, H = 4.0f, D = 8.0f, T = 0.2f;   // room width (x), height, depth (z); wall thickness
    auto cells = [&](float len) { return std::max<uint32_t>(1u, (uint32_t)std::lround(len * cpm)); };
    uint64_t tris = 0;
    MeshDesc Walls, Floor, Ceil;
    Walls.MaterialIndex = wall;
    Floor.MaterialIndex = floorm;
    Ceil.MaterialIndex = ceil;
    const float X1 = 3 * W + 2 * T;     // total length along x
    // floor (normal +y) and ceiling (normal -y) over the whole length
    tris += TessPanel(G, Floor, V3(0, 0, 0), V3(0, 0, D), V3(X1, 0, 0), cells(D), cells(X1), V3(0, 1, 0), noise, amp, freq);
    tris += TessPanel(G, Ceil, V3(0, H, 0), V3(X1, 0, 0), V3(0, 0, D), cells(X1), cells(D), V3(0, -1, 0), noise, amp, freq);
    // long walls z = 0 (normal +z) and z = D (normal -z)
    tris += TessPanel(G, Walls, V3(0, 0, 0), V3(X1, 0, 0), V3(0, H, 0), cells(X1), cells(H), V3(0, 0, 1), noise, amp, freq);
    tris += TessPanel(G, Walls, V3(X1, 0, D), V3(-X1, 0, 0), V3(0, H, 0), cells(X1), cells(H), V3(0, 0, -1), noise, amp, freq);
    // end walls x = 0 (normal +x) and x = X1 (normal -x)
    tris += TessPanel(G, Walls, V3(0, 0, D), V3(0, 0, -D), V3(0, H, 0), cells(D), cells(H), V3(1, 0, 0), noise, amp, freq);
    tris += TessPanel(G, Walls, V3(X1, 0, 0), V3(0, 0, D), V3(0, H, 0), cells(D), cells(H), V3(-1, 0, 0), noise, amp, freq);
    // inner walls with a 1 x 2 doorway centred in z: two faces, the doorway's jambs and lintel
    const Hole door{(D * 0.5f - 0.5f) / D, (D * 0.5f + 0.5f) / D, 0.0f, 2.0f / H};
    for (int k = 1; k <= 2; k++) {
        const float xa = k * W + (k - 1) * T, xb = xa + T;   // the wall spans x in [xa, xb]
        tris += TessPanel(G, Walls, V3(xa, 0, 0), V3(0, 0, D), V3(0, H, 0), cells(D), cells(H), V3(-1, 0, 0), noise,
                          amp, freq, door);   // face toward room k (normal -x)
        const Hole doorb{1.0f - door.u1, 1.0f - door.u0, door.v0, door.v1};
        tris += TessPanel(G, Walls, V3(xb, 0, D), V3(0, 0, -D), V3(0, H, 0), cells(D), cells(H), V3(1, 0, 0), noise,
                          amp, freq, doorb);  // face toward room k+1 (normal +x)
        const float z0 = D * 0.5f - 0.5f, z1 = D * 0.5f + 0.5f;
        tris += TessPanel(G, Walls, V3(xb, 0, z0), V3(-T, 0, 0), V3(0, 2, 0), cells(T), cells(2), V3(0, 0, 1), noise, 0.0, freq);
        tris += TessPanel(G, Walls, V3(xa, 0, z1), V3(T, 0, 0), V3(0, 2, 0), cells(T), cells(2), V3(0, 0, -1), noise, 0.0, freq);
        tris += TessPanel(G, Walls, V3(xa, 2, z0), V3(T, 0, 0), V3(0, 0, 1), cells(T), cells(1), V3(0, -1, 0), noise, 0.0, freq);
    }
    // clutter boxes on the floor, off the aisle through the doorways
    MeshDesc Clutter[4];
    for (int k = 0; k < 4; k++) Clutter[k].MaterialIndex = clutter[k];
    for (int room = 0; room < 3; room++) {
        const float rx = room * (W + T);
        for (int i = 0; i < 12; i++) {
            const float sx = r.uniform(0.3f, 1.2f), sy = r.uniform(0.2f, 1.5f), sz = r.uniform(0.3f, 1.2f);
            float cx = rx + r.uniform(0.8f, W - 0.8f), cz = r.uniform(0.8f, D - 0.8f);
            if (fabsf(cz - D * 0.5f) < 1.6f) cz = cz < D * 0.5f ? cz - 1.6f : cz + 1.6f;
            const Box b{cx - sx * 0.5f, cx + sx * 0.5f, 0.0f, sy, cz - sz * 0.5f, cz + sz * 0.5f};
            tris += TessBox(G, Clutter[r.next() % 4], b, std::max<uint32_t>(2u, cpm / 2), noise, 0.01);
        }
    }
    G.B.AddMesh(Floor);
    G.B.AddMesh(Ceil);
    G.B.AddMesh(Walls);
    for (int k = 0; k < 4; k++)
        if (!Clutter[k].Faces.empty()) G.B.AddMesh(Clutter[k]);
    G.Triangles += tris;
    // the only light: 1 x 1 under the ceiling of room 1, facing down
    CeilingLight(G, W * 0.5f, D * 0.5f, 1.0f, H - 0.02f, 60.0f, ceil);
    az_scene &S = G.B.Scene;
    S.MaxRecursionDepth = Def(p.max_depth, 10);
    S.PathTrace = 1;
    S.ImportanceSampling = p.importance_sampling >= 0 ? (uint32_t)p.importance_sampling : 1u;
    // room 3, looking toward -x through both doorways
    SimpleCamera(G, V3(X1 - 1.0f, 1.6f, D * 0.5f + 0.6f), V3(-1.0f, -0.08f, -0.12f), 60.0f, Def(p.width, 1920),
                 Def(p.height, 1080), Def(p.spp, 16));
    return true;
}

bool GenFeatures(Generated &G, const az_gen_params &p, uint64_t seed) {
    Rng r(seed + 100);
    az_scene &S = G.B.Scene;
    // materials covering all seven BRDF models
    az_material m;
    m = Lambert(0.7f, 0.7f, 0.7f);
    m.SpecularReflectance = V3(0.1f, 0.1f, 0.1f);
    m.BRDF.Exponent = 20.0f;
    m.AmbientReflectance = V3(0.3f, 0.3f, 0.3f);
    uint32_t white = G.B.AddMaterial(m);
    m = DefaultMaterial(); m.BRDF.Type = AZ_BRDF_Phong; m.BRDF.Exponent = 10.0f;
    m.DiffuseReflectance = V3(0.2f, 0.02f, 0.02f); m.SpecularReflectance = V3(0.05f, 0.05f, 0.05f);
    uint32_t red = G.B.AddMaterial(m);
    m = DefaultMaterial(); m.BRDF.Type = AZ_BRDF_ModifiedPhong; m.BRDF.Exponent = 30.0f;
    m.DiffuseReflectance = V3(0.02f, 0.15f, 0.02f); m.SpecularReflectance = V3(0.05f, 0.05f, 0.05f);
    uint32_t green = G.B.AddMaterial(m);
    m = DefaultMaterial(); m.BRDF.Type = AZ_BRDF_NormalizedModifiedPhong; m.BRDF.Exponent = 50.0f;
    m.DiffuseReflectance = V3(0.6f, 0.55f, 0.5f); m.SpecularReflectance = V3(0.2f, 0.2f, 0.2f);
    uint32_t backMat = G.B.AddMaterial(m);
    m = DefaultMaterial(); m.BRDF.Type = AZ_BRDF_BlinnPhong; m.BRDF.Exponent = 15.0f;
    m.DiffuseReflectance = V3(0.2f, 0.2f, 0.2f); m.SpecularReflectance = V3(0.1f, 0.1f, 0.1f);
    uint32_t ceilMat = G.B.AddMaterial(m);
    m = DefaultMaterial(); m.BRDF.Type = AZ_BRDF_ModifiedBlinnPhong; m.BRDF.Exponent = 40.0f;
    m.DiffuseReflectance = V3(0.05f, 0.05f, 0.05f); m.SpecularReflectance = V3(0.1f, 0.1f, 0.1f);
    m.MirrorReflectance = V3(0.8f, 0.8f, 0.8f); m.Glossiness = 0.05f;
    uint32_t glossy = G.B.AddMaterial(m);
    m = DefaultMaterial(); m.Transparency = V3(0.9f, 0.8f, 0.7f); m.RefractionIndex = 1.5f;
    uint32_t diel = G.B.AddMaterial(m);
    m = DefaultMaterial(); m.BRDF.Type = AZ_BRDF_TorranceSparrow; m.BRDF.Exponent = 60.0f;
    m.BRDF.RefractiveIndex = 1.8f;
    m.DiffuseReflectance = V3(0.5f, 0.4f, 0.3f); m.SpecularReflectance = V3(0.3f, 0.3f, 0.3f);
    uint32_t ts = G.B.AddMaterial(m);
    m = Lambert(0.3f, 0.3f, 0.6f);
    m.SpecularReflectance = V3(0.2f, 0.2f, 0.2f); m.BRDF.Exponent = 80.0f;
    m.AmbientReflectance = V3(0.2f, 0.2f, 0.2f);
    uint32_t boxMat = G.B.AddMaterial(m);

    // textures: checker (nearest, repeat), Perlin patch with bump, bilinear
    // clamp checker with bump, Perlin vein (replace-all)
    az_texture checker = CheckerTexture(G, 64, AZ_TextureFilter_Nearest, AZ_TextureWrap_Repeat);
    checker.BlendMode = AZ_TextureBlend_ReplaceDiffuse;
    uint32_t texChecker = G.B.AddTexture(checker);
    az_texture perlin = DefaultTexture();
    perlin.Type = AZ_TextureType_PerlinNoise;
    perlin.PerlinAppearance = AZ_PerlinAppearance_Patch;
    perlin.BlendMode = AZ_TextureBlend_BlendDiffuse;
    perlin.BumpMap = 1;
    perlin.BumpMapMultiplier = 0.3f;
    PerlinTables(G, r, perlin);
    perlin.ScalingFactor = 6.0f;
    uint32_t texPerlin = G.B.AddTexture(perlin);
    az_texture bil = CheckerTexture(G, 32, AZ_TextureFilter_Bilinear, AZ_TextureWrap_Clamp);
    bil.BlendMode = AZ_TextureBlend_BlendDiffuse;
    bil.BumpMap = 1;
    bil.BumpMapMultiplier = 0.002f;
    uint32_t texBil = G.B.AddTexture(bil);
    az_texture vein = DefaultTexture();
    vein.Type = AZ_TextureType_PerlinNoise;
    vein.PerlinAppearance = AZ_PerlinAppearance_Vein;
    vein.BlendMode = AZ_TextureBlend_ReplaceAll;
    PerlinTables(G, r, vein);
    vein.ScalingFactor = 9.0f;
    uint32_t texVein = G.B.AddTexture(vein);

    CornellWalls(G, Box{0.0f, 1.0f, 0.0f, 1.0f, 0.0f, 1.0f}, white, red, green, true, texChecker, backMat,
                 texPerlin, ceilMat);
    CeilingLight(G, 0.5f, 0.5f, 0.2f, 0.995f, 5.0f, white);

    // transformed, moving, smooth-shaded cube instance
    MeshDesc cube;
    cube.MaterialIndex = boxMat;
    cube.ShadingMode = AZ_Shading_Smooth;
    cube.Motion = V3(0.0f, 0.05f, 0.0f);
    cube.Transform = Mat4Mul(Mat4Translate(V3(0.3f, 0.15f, 0.35f)), Mat4Scale(V3(0.25f, 0.25f, 0.25f)));
    cube.InvTransform = Mat4Mul(Mat4Scale(V3(4.0f, 4.0f, 4.0f)), Mat4Translate(V3(-0.3f, -0.15f, -0.35f)));
    {
        const float h = 0.5f;
        az_vec3 c[8] = {V3(-h, -h, -h), V3(h, -h, -h), V3(h, h, -h), V3(-h, h, -h),
                        V3(-h, -h, h), V3(h, -h, h), V3(h, h, h), V3(-h, h, h)};
        uint32_t vi[8];
        for (int i = 0; i < 8; i++) vi[i] = AddV(G, c[i]);
        const uint32_t q[6][4] = {{0, 3, 2, 1}, {4, 5, 6, 7}, {0, 1, 5, 4}, {3, 7, 6, 2}, {0, 4, 7, 3}, {1, 2, 6, 5}};
        for (auto &f : q) {
            cube.Faces.push_back(az_vec3u{vi[f[0]], vi[f[1]], vi[f[2]]});
            cube.Faces.push_back(az_vec3u{vi[f[0]], vi[f[2]], vi[f[3]]});
        }
        G.B.AddMesh(cube);
        G.Triangles += 12;
    }

    // spheres: glossy mirror with bilinear bump texture, dielectric, moving
    // Torrance-Sparrow with vein texture, a scaled (ellipsoid) sphere, an
    // emitting light sphere
    az_entity e = Sphere(V3(0.25f, 0.2f, 0.65f), 0.15f, glossy);
    e.TextureIndex = texBil;
    G.B.AddSphere(e, false);
    G.B.AddSphere(Sphere(V3(0.72f, 0.2f, 0.5f), 0.15f, diel), false);
    e = Sphere(V3(0.5f, 0.55f, 0.3f), 0.1f, ts);
    e.MotionVector = V3(0.1f, 0.0f, 0.05f);
    e.TextureIndex = texVein;
    G.B.AddSphere(e, false);
    e = Sphere(V3(0, 0, 0), 1.0f, ts);
    e.TransformationMatrix = Mat4Mul(Mat4Translate(V3(0.82f, 0.08f, 0.82f)), Mat4Scale(V3(0.125f, 0.0625f, 0.125f)));
    e.InvTransformationMatrix = Mat4Mul(Mat4Scale(V3(8.0f, 16.0f, 8.0f)), Mat4Translate(V3(-0.82f, -0.08f, -0.82f)));
    G.B.AddSphere(e, false);
    e = Sphere(V3(0.8f, 0.75f, 0.6f), 0.05f, white);
    e.IsEmitter = 1;
    e.Radiance = V3(4.0f, 3.5f, 3.0f);
    G.B.AddSphere(e, true);
    G.Spheres = 5;

    // point, area, directional and spot lights (entity lights are appended by the builder)
    az_light L;
    memset(&L, 0, sizeof(L));
    L.Type = AZ_Light_Point;
    L.Position = V3(0.3f, 0.9f, 0.7f);
    L.Intensity = V3(0.3f, 0.3f, 0.3f);
    G.B.AddLight(L);
    memset(&L, 0, sizeof(L));
    L.Type = AZ_Light_Area;
    L.Position = V3(0.6f, 0.98f, 0.3f);
    L.Intensity = V3(1.0f, 0.9f, 0.8f);
    L.EdgeVectors[0] = V3(0.1f, 0.0f, 0.0f);
    L.EdgeVectors[1] = V3(0.0f, 0.0f, 0.1f);
    L.Normal = V3(0.0f, -1.0f, 0.0f);
    G.B.AddLight(L);
    memset(&L, 0, sizeof(L));
    L.Type = AZ_Light_Directional;
    L.Direction = V3(0.0f, -0.3f, -1.0f);
    L.Intensity = V3(0.2f, 0.2f, 0.25f);
    G.B.AddLight(L);
    memset(&L, 0, sizeof(L));
    L.Type = AZ_Light_Spot;
    L.Position = V3(0.5f, 0.9f, 0.9f);
    L.Intensity = V3(0.5f, 0.5f, 0.4f);
    L.SpotDirection = V3(0.0f, -1.0f, -0.5f);
    L.CoverageAngle = 60.0f;
    L.FallOffAngle = 40.0f;
    L.CosHalfCoverage = cosf(30.0f * (float)kPi / 180.0f);
    L.CosHalfFallOff = cosf(20.0f * (float)kPi / 180.0f);
    G.B.AddLight(L);

    S.AmbientLight = V3(0.05f, 0.05f, 0.05f);
    S.BackgroundColor = V3(0.1f, 0.2f, 0.3f);
    az_texture bg = CheckerTexture(G, 16, AZ_TextureFilter_Nearest, AZ_TextureWrap_Repeat);
    S.BackgroundTexture = bg;
    S.UseBackgroundTexture = 1;
    S.MaxRecursionDepth = Def(p.max_depth, 5);
    S.PathTrace = 1;
    S.ImportanceSampling = p.importance_sampling >= 0 ? (uint32_t)p.importance_sampling : 1u;
    SimpleCamera(G, V3(0.5f, 0.5f, 2.4f), V3(0, 0, -1), 45.0f, Def(p.width, 96), Def(p.height, 96), Def(p.spp, 4));
    G.Camera.ApertureSize = 0.04f;     // thin lens (src/azimuth_main.cpp:1155-1178)
    G.Camera.FocusDistance = 2.0f;
    return true;
}

bool GenEnvSpheres(Generated &G, const az_gen_params &p, uint64_t seed) {
    Rng r(seed + 101);
    uint32_t ground = G.B.AddMaterial(Lambert(0.5f, 0.5f, 0.5f));
    az_material m = DefaultMaterial();
    m.Transparency = V3(0.95f, 0.95f, 1.0f);
    m.RefractionIndex = 1.5f;
    uint32_t diel = G.B.AddMaterial(m);
    m = DefaultMaterial();
    m.MirrorReflectance = V3(0.9f, 0.9f, 0.9f);
    m.Glossiness = 0.02f;
    uint32_t glossy = G.B.AddMaterial(m);
    uint32_t mats[7];
    for (uint32_t k = 0; k < 7; k++) mats[k] = G.B.AddMaterial(RandomBRDFMaterial(r, k));
    MeshDesc floor;
    floor.MaterialIndex = ground;
    AddQuad(G, floor, V3(-4, 0, -4), V3(-4, 0, 4), V3(4, 0, 4), V3(4, 0, -4));
    G.B.AddMesh(floor);
    G.Triangles += 2;
    G.B.AddSphere(Sphere(V3(-1.2f, 0.5f, 0.0f), 0.5f, diel), false);
    G.B.AddSphere(Sphere(V3(0.0f, 0.5f, -0.6f), 0.5f, glossy), false);
    for (int k = 0; k < 7; k++) {
        float a = (float)k / 7.0f * 2.0f * (float)kPi;
        az_entity e = Sphere(V3(1.6f * cosf(a), 0.2f, 1.6f * sinf(a) + 0.6f), 0.2f, mats[k]);
        if (k == 3) e.MotionVector = V3(0.0f, 0.15f, 0.0f);
        G.B.AddSphere(e, false);
    }
    G.Spheres = 9;
    az_scene &S = G.B.Scene;
    S.EnvironmentMap = SkyTexture(G, Def(p.env_width, 256), Def(p.env_height, 128), V3(0.5f, 0.6f, 0.3f), 3.0f,
                                  200.0f);
    S.UseEnvironmentMap = 1;
    S.MaxRecursionDepth = Def(p.max_depth, 6);
    S.PathTrace = 1;
    S.ImportanceSampling = p.importance_sampling >= 0 ? (uint32_t)p.importance_sampling : 1u;
    SimpleCamera(G, V3(0.0f, 1.2f, 4.5f), V3(0.0f, -0.2f, -1.0f), 50.0f, Def(p.width, 96), Def(p.height, 64),
                 Def(p.spp, 4));
    return true;
}

}  // namespace
}  // namespace az

extern "C" int az_scene_generate(int32_t scene_id, uint64_t seed, const az_gen_params *params,
                                 az_generated_scene *out) {
    using namespace az;
    if (!out) return 1;
    memset(out, 0, sizeof(*out));
    az_gen_params p;
    memset(&p, 0, sizeof(p));
    p.filter = -1;
    p.importance_sampling = -1;
    if (params) p = *params;
    Generated *G = new (std::nothrow) Generated();
    if (!G) return 3;
    G->Eps.Intersection = 0.0f;     // azimuth's defaults, src/azimuth_main.cpp:2028-2030
    G->Eps.ShadowRay = 0.000275f;
    int filter = AZ_Filter_Box;
    bool ok = false;
    switch (scene_id) {
        case AZ_SCENE_CORNELL: ok = GenCornell(*G, p, seed); break;
        case AZ_SCENE_DENSE_MESH: ok = GenDenseMesh(*G, p, seed); filter = AZ_Filter_Gaussian; break;
        case AZ_SCENE_MOTION_ENV: ok = GenMotionEnv(*G, p, seed); break;
        case AZ_SCENE_INTERIOR: ok = GenInterior(*G, p, seed); break;
        case AZ_SCENE_FEATURES: ok = GenFeatures(*G, p, seed); filter = AZ_Filter_Gaussian; break;
        case AZ_SCENE_ENV_SPHERES: ok = GenEnvSpheres(*G, p, seed); break;
        default: delete G; return 1;
    }
    if (!ok || !G->B.Finalize((p.flags & AZ_GEN_SOUP_ONLY) != 0)) {
        delete G;
        return 2;
    }
    out->scene = &G->B.Scene;
    out->camera = &G->Camera;
    out->epsilons = &G->Eps;
    out->filter_type = p.filter >= 0 ? p.filter : filter;
    out->backface_culling = 0;
    out->perlin_gradients = G->Gradients.empty() ? nullptr : G->Gradients.data();
    out->triangle_count = G->Triangles;
    out->sphere_count = G->Spheres;
    out->owner = G;
    out->soup = &G->B.Soup;
    return 0;
}

extern "C" void az_scene_release(az_generated_scene *s) {
    if (!s) return;
    delete (az::Generated *)s->owner;
    memset(s, 0, sizeof(*s));
}
