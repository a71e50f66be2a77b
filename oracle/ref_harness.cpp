/*
 * Oracle harness around azimuth's own render code (test infrastructure only).
 *
 * This translation unit #includes azimuth's unity build
 * (src/azimuth_main.cpp, patched by oracle/patch_reference.py) with
 * -Dmain=azimuth_main, so every static routine of the reference is callable
 * here.  It exports a small C interface used by the tests and by the CPU
 * baseline leg of bench.py:
 *
 *   azref_produce_image   ProduceImageInLinearSpace (src/azimuth_main.cpp:1256)
 *                         over N threads with RenderScene's scanline split
 *                         (src/azimuth_main.cpp:1815-1867), any filter
 *   azref_sample_radiance the same loop, recording every camera sample's
 *                         colour before ComputeSampleWeight splats it
 *   azref_closest_hit     RayEntityIntersection on the scene root
 *                         (src/azimuth_main.cpp:53-385), plus the face id of
 *                         a mesh-instance hit (src/azimuth_main.cpp:244-281)
 *   azref_construct_bvh*  ConstructBVH / ConstructBVHTrianglesOnly
 *                         (src/azimuth_bvh.cpp:1-328)
 *   azref_*perlin*, azref_sample_texture, azref_eval_brdf
 *                         per-routine known-answer access
 *   azref_import_xml      ImportXML (src/azimuth_xml.cpp:3021-3930) through
 *                         the reader of include/az_xmlreader.h, with
 *                         azref_scene_summary / azref_mesh_arrays to read
 *                         back what it built
 *
 * It also defines the counter-RNG hooks that the patched Random01,
 * GetSampleCoord and TraceRay call, and the sample hook of the patched
 * ComputeSampleWeight (see oracle/shim/az_oracle_compat.h).
 */
#include "azimuth_main.cpp"

#include <omp.h>
#include <vector>
#include "az_abi.h"
#include "azimuth_gpu.h"
#include "az_rng_oracle.h"

/* ---- the reference structs and the C mirror must share one layout ---- */
#define AZ_SAME(T, AT, F) static_assert(offsetof(T, F) == offsetof(AT, F), #T "." #F)
static_assert(sizeof(entity) == sizeof(az_entity), "entity");
static_assert(sizeof(mesh) == sizeof(az_mesh), "mesh");
static_assert(sizeof(light) == sizeof(az_light), "light");
static_assert(sizeof(material) == sizeof(az_material), "material");
static_assert(sizeof(texture) == sizeof(az_texture), "texture");
static_assert(sizeof(camera) == sizeof(az_camera), "camera");
static_assert(sizeof(scene) == sizeof(az_scene), "scene");
static_assert(sizeof(pixel) == sizeof(az_pixel), "pixel");
static_assert(sizeof(ray_hit) == sizeof(az_ray_hit), "ray_hit");
AZ_SAME(entity, az_entity, Center); AZ_SAME(entity, az_entity, Radius);
AZ_SAME(entity, az_entity, P0); AZ_SAME(entity, az_entity, N2);
AZ_SAME(entity, az_entity, FaceNormal); AZ_SAME(entity, az_entity, UV2);
AZ_SAME(entity, az_entity, ShadingMode); AZ_SAME(entity, az_entity, AABB);
AZ_SAME(entity, az_entity, Mesh); AZ_SAME(entity, az_entity, BaseMeshID);
AZ_SAME(entity, az_entity, Right); AZ_SAME(entity, az_entity, Left);
AZ_SAME(entity, az_entity, InvTransformationMatrix);
AZ_SAME(entity, az_entity, TransformationMatrix);
AZ_SAME(entity, az_entity, MotionVector); AZ_SAME(entity, az_entity, Radiance);
AZ_SAME(entity, az_entity, IsEmitter); AZ_SAME(entity, az_entity, TextureIndex);
AZ_SAME(entity, az_entity, MaterialIndex); AZ_SAME(entity, az_entity, ID);
AZ_SAME(entity, az_entity, UniqueEntityID); AZ_SAME(entity, az_entity, Type);
AZ_SAME(mesh, az_mesh, BVH); AZ_SAME(mesh, az_mesh, Triangles);
AZ_SAME(mesh, az_mesh, TotalArea); AZ_SAME(mesh, az_mesh, TriangleCount);
AZ_SAME(mesh, az_mesh, ShadingMode);
AZ_SAME(light, az_light, Position); AZ_SAME(light, az_light, Intensity);
AZ_SAME(light, az_light, EdgeVectors); AZ_SAME(light, az_light, Normal);
AZ_SAME(light, az_light, Direction); AZ_SAME(light, az_light, SpotDirection);
AZ_SAME(light, az_light, CosHalfFallOff); AZ_SAME(light, az_light, Entity);
AZ_SAME(light, az_light, Type);
AZ_SAME(material, az_material, DiffuseReflectance);
AZ_SAME(material, az_material, Transparency);
AZ_SAME(material, az_material, Glossiness); AZ_SAME(material, az_material, ID);
AZ_SAME(texture, az_texture, Pixels); AZ_SAME(texture, az_texture, Normalizer);
AZ_SAME(texture, az_texture, Perm); AZ_SAME(texture, az_texture, ScalingFactor);
AZ_SAME(texture, az_texture, PerlinAppearance);
AZ_SAME(texture, az_texture, BumpMapMultiplier); AZ_SAME(texture, az_texture, Type);
AZ_SAME(camera, az_camera, NearPlane); AZ_SAME(camera, az_camera, FovY);
AZ_SAME(camera, az_camera, Position); AZ_SAME(camera, az_camera, Resolution);
AZ_SAME(camera, az_camera, ApertureSize); AZ_SAME(camera, az_camera, SampleCount);
AZ_SAME(camera, az_camera, Type);
AZ_SAME(scene, az_scene, BackgroundTexture); AZ_SAME(scene, az_scene, BVHRoot);
AZ_SAME(scene, az_scene, EnvironmentMap); AZ_SAME(scene, az_scene, MaxRecursionDepth);
AZ_SAME(scene, az_scene, ImportanceSampling);

/* ------------------------- counter-RNG hooks -------------------------- */
namespace {
struct NodeCtx {
    uint32_t Level;      /* 0 = camera context, 1 = root TraceRay, ... */
    uint32_t Digits;     /* child index (2 bits) per level >= 2         */
    uint32_t Dim;        /* draws consumed by this node so far          */
    uint32_t NextChild;  /* TraceRay calls made from this node so far   */
};
const int MaxNodeStack = 96;
uint64_t GSeed = 0;
uint32_t GSetupDim = 0;
thread_local NodeCtx TStack[MaxNodeStack];
thread_local int TTop = -1;
thread_local uint32_t TPixel = 0, TSample = 0;
}

extern "C" float AzOracleRandom01(void) {
    if (TTop < 0) {
        /* outside any camera sample: the scene-setup stream (e.g. InitPerlinNoise) */
        return az_oracle_u01(GSeed, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFu, GSetupDim++);
    }
    NodeCtx &C = TStack[TTop];
    return az_oracle_u01(GSeed, TPixel, TSample, C.Digits, C.Level, C.Dim++);
}

extern "C" void AzOracleBeginSample(unsigned Row, unsigned Col, unsigned SampleX, unsigned SampleY) {
    TPixel = (Row << 16) | Col;
    TSample = (SampleY << 16) | SampleX;
    TTop = 0;
    TStack[0] = NodeCtx{0, 0, 0, 0};
}

extern "C" void AzOracleEnterNode(void) {
    if (TTop < 0) {            /* TraceRay outside a sample: give it a context */
        TTop = 0;
        TStack[0] = NodeCtx{0, 0, 0, 0};
    }
    if (TTop + 1 >= MaxNodeStack) { abort(); }
    NodeCtx &P = TStack[TTop];
    uint32_t K = P.NextChild++;
    NodeCtx C;
    C.Level = P.Level + 1;
    C.Digits = P.Digits;
    if (C.Level >= 2 && C.Level - 2 < 16) { C.Digits |= (K & 3u) << (2u * (C.Level - 2u)); }
    C.Dim = 0;
    C.NextChild = 0;
    TStack[++TTop] = C;
}

extern "C" void AzOracleLeaveNode(void) { --TTop; }

/* Per-sample radiance: while GSampleOut is set, every finished camera sample
 * (ComputeSampleWeight's colour) is stored at its index in the scissor's
 * sample order, s = (SampleY * SampleCountSqrt + SampleX) * pixels + pixel,
 * pixel = (Row - RowMin) * Columns + (Col - ColMin); threads write disjoint
 * entries. */
namespace {
float *GSampleOut = nullptr;
uint32_t GSampleRow0 = 0, GSampleCol0 = 0, GSampleCols = 0, GSampleRows = 0, GSampleSqrt = 1;
}

extern "C" void AzOracleSampleDone(float R, float G, float B) {
    if (!GSampleOut) { return; }
    const uint32_t Row = TPixel >> 16, Col = TPixel & 0xFFFFu;
    const uint32_t SX = TSample & 0xFFFFu, SY = TSample >> 16;
    const uint64_t Pixels = (uint64_t)GSampleRows * GSampleCols;
    const uint64_t Pix = (uint64_t)(Row - GSampleRow0) * GSampleCols + (Col - GSampleCol0);
    const uint64_t S = ((uint64_t)SY * GSampleSqrt + SX) * Pixels + Pix;
    float *O = GSampleOut + 4 * S;
    O[0] = R; O[1] = G; O[2] = B; O[3] = 1.0f;
}

/* ------------------------------ C interface ---------------------------- */
extern "C" {

void azref_set_seed(uint64_t Seed) { GSeed = Seed; GSetupDim = 0; }
void azref_end_sample(void) { TTop = -1; }
float azref_random01(void) { return AzOracleRandom01(); }

/* RenderScene's thread split (src/azimuth_main.cpp:1815-1867) without the file
 * output and with the filter as a parameter (RenderScene hard-codes Box). */
void azref_produce_image(az_pixel *Pixels, az_scene *Scene, az_camera *Camera,
                         az_epsilon_values *Epsilons, az_scissor Scissor,
                         int FilterType, int BackfaceCulling, uint32_t ThreadCount) {
    if (ThreadCount == 0) { ThreadCount = 1; }
    uint32_t RowMin = Scissor.Min.y;
    uint32_t RowMax = Scissor.Max.y;
    if (RowMax > Camera->Resolution.y) { RowMax = Camera->Resolution.y; }
    uint32_t Rows = RowMax > RowMin ? RowMax - RowMin : 0;
    if (ThreadCount > Rows && Rows > 0) { ThreadCount = Rows; }

    thread_handle *Handles = (thread_handle *)calloc(ThreadCount, sizeof(thread_handle));
    produce_image_params *Params =
        (produce_image_params *)calloc(ThreadCount, sizeof(produce_image_params));
    uint32_t MinPer = Rows / ThreadCount;
    uint32_t Residual = Rows - MinPer * ThreadCount;
    uint32_t Consumed = RowMin;
    for (uint32_t I = 0; I < ThreadCount; I++) {
        uint32_t Lines = MinPer + (Residual ? 1u : 0u);
        if (Residual) { Residual--; }
        produce_image_params *P = Params + I;
        P->Scissor.Max = Vec2u(Scissor.Max.x, Consumed + Lines);
        P->Scissor.Min = Vec2u(Scissor.Min.x, Consumed);
        P->Pixels = (pixel *)Pixels;
        P->Scene = (scene *)Scene;
        P->Camera = (camera *)Camera;
        P->Epsilons = (epsilon_values *)Epsilons;
        P->FilterType = (filter_type)FilterType;
        P->BackfaceCulling = (b32)BackfaceCulling;
        u32 ThreadID;
        PlatformCreateThread(&Handles[I], ProduceImageInLinearSpaceMT, P, &ThreadID, 0);
        Consumed += Lines;
    }
    PlatformWaitForThreads(ThreadCount, Handles, true, true, 0);
    free(Handles);
    free(Params);
}

/* Each camera sample's colour over the scissor, as ProduceImageInLinearSpace
 * computes it before ComputeSampleWeight splats it: Out holds 4 floats (RGB,
 * 1) per sample in the order of AzOracleSampleDone.  Runs azimuth's own render
 * loop on `ThreadCount` threads (a scratch film takes the splats). */
void azref_sample_radiance(float *Out, az_scene *Scene, az_camera *Camera, az_epsilon_values *Epsilons,
                           az_scissor Scissor, int BackfaceCulling, uint32_t ThreadCount) {
    const uint32_t W = Camera->Resolution.x, H = Camera->Resolution.y;
    const uint32_t R1 = Scissor.Max.y < H ? Scissor.Max.y : H, C1 = Scissor.Max.x < W ? Scissor.Max.x : W;
    GSampleRow0 = Scissor.Min.y;
    GSampleCol0 = Scissor.Min.x;
    GSampleRows = R1 > Scissor.Min.y ? R1 - Scissor.Min.y : 0;
    GSampleCols = C1 > Scissor.Min.x ? C1 - Scissor.Min.x : 0;
    GSampleSqrt = (uint32_t)Sqrt((f32)Camera->SampleCount);
    az_pixel *Film = (az_pixel *)calloc((size_t)W * H, sizeof(az_pixel));
    GSampleOut = Out;
    azref_produce_image(Film, Scene, Camera, Epsilons, Scissor, 0, BackfaceCulling, ThreadCount);
    GSampleOut = nullptr;
    free(Film);
}

/* Closest hit on the scene root for a batch of rays (src/azimuth_main.cpp:53-385).
 * Outputs per ray: hit flag, UniqueEntityID of the top-level entity, face id
 * (entity.ID of the triangle inside a mesh instance; 0xFFFFFFFF otherwise),
 * t, and P/Normal/UV as 8 floats. */
int azref_closest_hit(az_scene *AScene, const az_ray3 *Rays, uint32_t Count, int Cull,
                      float HitEpsilon, uint32_t *OutHit, uint32_t *OutUid,
                      uint32_t *OutFace, float *OutT, float *OutPNUV, int Threads) {
    scene *Scene = (scene *)AScene;
    if (Threads <= 0) { Threads = 1; }
#pragma omp parallel for num_threads(Threads) schedule(dynamic, 256)
    for (int64_t I = 0; I < (int64_t)Count; I++) {
        ray3 Ray;
        memcpy(&Ray, Rays + I, sizeof(ray3));
        ray_hit Hit = {0};
        Hit.t = f32_Max;
        b32 Ok = RayEntityIntersection(&Hit, Ray, Scene->BVHRoot, Scene->Textures,
                                       (b32)Cull, HitEpsilon);
        OutHit[I] = Ok ? 1u : 0u;
        OutUid[I] = 0xFFFFFFFFu;
        OutFace[I] = 0xFFFFFFFFu;
        OutT[I] = Ok ? Hit.t : 0.0f;
        float *Pn = OutPNUV + 8 * I;
        memset(Pn, 0, 8 * sizeof(float));
        if (!Ok) { continue; }
        entity *E = Hit.Entity;
        OutUid[I] = E->UniqueEntityID;
        if (E->Type == EntityType_Triangle) {
            OutFace[I] = E->ID;
        } else if (E->Type == EntityType_MeshInstance) {
            /* the instance path of src/azimuth_main.cpp:246-255, to read the face */
            ray3 R = Ray;
            vec3 Motion = R.T * E->MotionVector;
            R.Origin -= Motion;
            ray3 LocalRay = GetLocalRay(R, E->InvTransformationMatrix);
            ray_hit LocalHit = {0};
            LocalHit.t = f32_Max;
            if (RayEntityIntersection(&LocalHit, LocalRay, E->Mesh->BVH, Scene->Textures,
                                      (b32)Cull, HitEpsilon)) {
                OutFace[I] = LocalHit.Entity->ID;
            }
        }
        Pn[0] = Hit.P.x; Pn[1] = Hit.P.y; Pn[2] = Hit.P.z;
        Pn[3] = Hit.Normal.x; Pn[4] = Hit.Normal.y; Pn[5] = Hit.Normal.z;
        Pn[6] = Hit.UV.u; Pn[7] = Hit.UV.v;
    }
    return 0;
}

int azref_construct_bvh(az_entity **Root, az_entity *Entities, uint32_t Count) {
    return ConstructBVH((entity **)Root, (entity *)Entities, Count) ? 1 : 0;
}

int azref_construct_bvh_triangles(az_entity **Root, az_entity *Triangles, uint32_t Count) {
    return ConstructBVHTrianglesOnly((entity **)Root, (entity *)Triangles, Count) ? 1 : 0;
}

/* InitPerlinNoise (src/azimuth_texture.h:106-132) on the setup RNG stream. */
void azref_init_perlin(az_texture *Texture) { InitPerlinNoise((texture *)Texture); }

void azref_get_perlin_gradients(float *Out768) {
    for (int I = 0; I < PerlinGradientSize; I++) {
        Out768[3 * I + 0] = PerlinGradient[I].x;
        Out768[3 * I + 1] = PerlinGradient[I].y;
        Out768[3 * I + 2] = PerlinGradient[I].z;
    }
}

void azref_set_perlin_gradients(const float *In768) {
    for (int I = 0; I < PerlinGradientSize; I++) {
        PerlinGradient[I] = Vec3(In768[3 * I + 0], In768[3 * I + 1], In768[3 * I + 2]);
    }
    PerlinGradientFilled = true;
}

float azref_sample_perlin(az_texture *Texture, float X, float Y, float Z) {
    return SamplePerlinNoise((texture *)Texture, Vec3(X, Y, Z));
}

void azref_sample_texture(az_texture *Texture, float X, float Y, float Z, float U, float V,
                          float *Out3) {
    vec3 R = SampleTexture((texture *)Texture, Vec3(X, Y, Z), Vec2(U, V));
    Out3[0] = R.x; Out3[1] = R.y; Out3[2] = R.z;
}

/* CalculateLightContribution (src/azimuth_main.cpp:571-603) on zeroed
 * accumulators: returns Diffuse and Specular contributions (3+3 floats). */
void azref_light_contribution(az_brdf *Brdf, const float *Intensity3, const float *LightDir3,
                              const float *ViewDir3, const float *Normal3, float Distance,
                              float FallOff, float InvPdf, float *Out6) {
    vec3 D = Vec3(0.0f, 0.0f, 0.0f), S = Vec3(0.0f, 0.0f, 0.0f);
    CalculateLightContribution(&D, &S, (brdf *)Brdf,
                               Vec3(Intensity3[0], Intensity3[1], Intensity3[2]),
                               Vec3(LightDir3[0], LightDir3[1], LightDir3[2]),
                               Vec3(ViewDir3[0], ViewDir3[1], ViewDir3[2]),
                               Vec3(Normal3[0], Normal3[1], Normal3[2]),
                               Distance, FallOff, InvPdf);
    Out6[0] = D.x; Out6[1] = D.y; Out6[2] = D.z;
    Out6[3] = S.x; Out6[4] = S.y; Out6[5] = S.z;
}

uint32_t azref_sizeof_entity(void) { return (uint32_t)sizeof(entity); }

/* OutputPixelsToFile (src/azimuth_main.cpp:1620-1797) as azimuth calls it for a
 * BMP (SaveFormat BMP, no EXR copy): normalises, tone maps and gamma-corrects
 * `Pixels` in place and writes the file to BmpPath.  The 8-bit values azimuth
 * writes are (u8)(Clamp01(C) * 255.0f) of the resulting colours. */
int azref_output_pixels(az_pixel *Pixels, uint32_t Width, uint32_t Height, const az_tonemap *Tonemap,
                        float InvGamma, uint32_t SRGB, const char *BmpPath) {
    tonemap T;
    memcpy(&T, Tonemap, sizeof(T));
    char Path[256] = {0};
    strncpy(Path, BmpPath, sizeof(Path) - 1);
    return OutputPixelsToFile(Path, (pixel *)Pixels, Vec2u(Width, Height), &T, InvGamma, (b32)SRGB,
                              FileFormat_BMP, false) ? 1 : 0;
}

/* OutputPixelsToFile (src/azimuth_main.cpp:1620-1797) with any of the four
 * 8-bit formats (file_format values, src/azimuth_io.h:1-7); no EXR (OpenEXR
 * is stubbed in this build). */
int azref_output_pixels_fmt(az_pixel *Pixels, uint32_t Width, uint32_t Height, const az_tonemap *Tonemap,
                            float InvGamma, uint32_t SRGB, int32_t Format, const char *FilePath) {
    if (Format < FileFormat_PNG || Format > FileFormat_JPG) return 0;
    tonemap T;
    memcpy(&T, Tonemap, sizeof(T));
    char Path[256] = {0};
    strncpy(Path, FilePath, sizeof(Path) - 1);
    return OutputPixelsToFile(Path, (pixel *)Pixels, Vec2u(Width, Height), &T, InvGamma, (b32)SRGB,
                              (file_format)Format, false) ? 1 : 0;
}

/* OutputPixelsToPNG / BMP / TGA / JPG (src/azimuth_main.cpp:1460-1618)
 * alone, on colours rgb (W*H*3 floats, top row first). */
int azref_write_image(const float *Rgb, uint32_t Width, uint32_t Height, int32_t Format, const char *FilePath) {
    std::vector<pixel> Px((size_t)Width * Height);
    for (size_t i = 0; i < Px.size(); i++) {
        Px[i].Color = Vec3(Rgb[3 * i + 0], Rgb[3 * i + 1], Rgb[3 * i + 2]);
        Px[i].TotalWeight = 1.0f;
    }
    char Path[256] = {0};
    strncpy(Path, FilePath, sizeof(Path) - 1);
    vec2u Size = Vec2u(Width, Height);
    switch (Format) {
        case FileFormat_PNG: return OutputPixelsToPNG(Path, Px.data(), Size) ? 1 : 0;
        case FileFormat_BMP: return OutputPixelsToBMP(Path, Px.data(), Size) ? 1 : 0;
        case FileFormat_TGA: return OutputPixelsToTGA(Path, Px.data(), Size) ? 1 : 0;
        case FileFormat_JPG: return OutputPixelsToJPG(Path, Px.data(), Size) ? 1 : 0;
        default: return 0;
    }
}

/* ImportXML (src/azimuth_xml.cpp:3021-3930) as azimuth's main calls it
 * (src/azimuth_main.cpp:2026-2036): a default scene, epsilons 0 and 0.000275,
 * then the scene file, PLY meshes included.  In this build
 * libxml/xmlreader.h is the header-only reader of include/az_xmlreader.h.
 * Returns 1 on success with heap copies of the scene, the cameras and the
 * epsilons (kept for the life of the process), 0 when ImportXML fails. */
int azref_import_xml(const char *FilePath, az_scene **SceneOut, az_camera **CamerasOut, uint32_t *CameraCount,
                     az_epsilon_values **EpsilonsOut) {
    scene *S = (scene *)calloc(1, sizeof(scene));
    epsilon_values *E = (epsilon_values *)calloc(1, sizeof(epsilon_values));
    if (!S || !E) { free(S); free(E); return 0; }
    *S = DefaultScene();
    E->Intersection = 0.0f;
    E->ShadowRay = 0.000275f;
    camera *Cameras = 0;
    u32 Count = 0;
    std::vector<char> Path(FilePath, FilePath + strlen(FilePath) + 1);
    if (!ImportXML(S, &Cameras, &Count, E, Path.data())) return 0;
    *SceneOut = (az_scene *)S;
    *CamerasOut = (az_camera *)Cameras;
    *CameraCount = Count;
    *EpsilonsOut = (az_epsilon_values *)E;
    return 1;
}

static void CountLeaves(const entity *E, uint32_t *Spheres, uint32_t *Instances) {
    if (!E) return;
    if (E->Type == EntityType_BVHNode) {
        CountLeaves(E->Left, Spheres, Instances);
        CountLeaves(E->Right, Spheres, Instances);
    } else if (E->Type == EntityType_Sphere) {
        (*Spheres)++;
    } else if (E->Type == EntityType_MeshInstance) {
        (*Instances)++;
    }
}

/* Counts of an imported scene: Out[0..8] = meshes, materials, lights,
 * triangles over all meshes, spheres and mesh instances under the top-level
 * BVH, emitting meshes, PathTrace, MaxRecursionDepth. */
void azref_scene_summary(const az_scene *AScene, uint32_t *Out9) {
    const scene *S = (const scene *)AScene;
    uint32_t Tris = 0, Emitters = 0, Spheres = 0, Instances = 0;
    for (u32 M = 0; M < S->MeshCount; M++) {
        Tris += S->Meshes[M].TriangleCount;
        Emitters += S->Meshes[M].IsEmitter ? 1u : 0u;
    }
    CountLeaves(S->BVHRoot, &Spheres, &Instances);
    uint32_t V[9] = {S->MeshCount, S->MaterialCount, S->LightCount, Tris, Spheres, Instances, Emitters,
                     S->PathTrace, S->MaxRecursionDepth};
    memcpy(Out9, V, sizeof(V));
}

static void CollectTriangles(const entity *E, std::vector<const entity *> *Out) {
    if (!E) return;
    if (E->Type == EntityType_BVHNode) {
        CollectTriangles(E->Left, Out);
        CollectTriangles(E->Right, Out);
    } else if (E->Type == EntityType_Triangle) {
        Out->push_back(E);
    }
}

/* What the importer's mesh loop (src/azimuth_xml.cpp:3669-3776) left in mesh
 * M of an imported scene: Tris12 = Mesh->Triangles (P0, P1, P2, N per face,
 * face order), Ents24 = the triangle entities under Mesh->BVH (P0, P1, P2,
 * N0, N1, N2, UV0, UV1, UV2; BVH leaf order), *TotalArea, and the fields of
 * the mesh's az_mesh_desc that come from the mesh itself.  Both arrays hold
 * Mesh->TriangleCount rows; returns that count, or -1 when the BVH holds a
 * different number of triangles. */
int azref_mesh_arrays(const az_scene *AScene, uint32_t M, float *Tris12, float *Ents24, float *TotalArea,
                      az_mesh_desc *Desc) {
    const scene *S = (const scene *)AScene;
    if (M >= S->MeshCount) return -1;
    const mesh *Me = S->Meshes + M;
    memcpy(Tris12, Me->Triangles, sizeof(triangle) * Me->TriangleCount);
    std::vector<const entity *> Leaves;
    CollectTriangles(Me->BVH, &Leaves);
    if (Leaves.size() != Me->TriangleCount) return -1;
    for (size_t I = 0; I < Leaves.size(); I++) {
        const entity *E = Leaves[I];
        const vec3 *V[6] = {&E->P0, &E->P1, &E->P2, &E->N0, &E->N1, &E->N2};
        float *O = Ents24 + 24 * I;
        for (int K = 0; K < 6; K++) { O[3 * K] = V[K]->x; O[3 * K + 1] = V[K]->y; O[3 * K + 2] = V[K]->z; }
        const vec2 *U[3] = {&E->UV0, &E->UV1, &E->UV2};
        for (int K = 0; K < 3; K++) { O[18 + 2 * K] = U[K]->x; O[19 + 2 * K] = U[K]->y; }
    }
    *TotalArea = Me->TotalArea;
    Desc->uv_offset = Me->UVOffset;
    Desc->shading_mode = (uint32_t)Me->ShadingMode;
    Desc->material_index = Me->MaterialIndex;
    Desc->texture_index = Me->TextureIndex;
    Desc->is_emitter = Me->IsEmitter;
    memcpy(&Desc->motion, &Me->MotionVector, sizeof(Desc->motion));
    memcpy(&Desc->radiance, &Me->Radiance, sizeof(Desc->radiance));
    memcpy(&Desc->transform, &Me->TransformationMatrix, sizeof(Desc->transform));
    memcpy(&Desc->inv_transform, &Me->InvTransformationMatrix, sizeof(Desc->inv_transform));
    return (int)Me->TriangleCount;
}

}  /* extern "C" */
