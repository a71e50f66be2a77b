/*
 * az_abi.h -- C mirror of azimuth's scene-model structures (x86-64 layout).
 *
 * The GPU library reads scenes that were built in azimuth's own structs, so
 * every type here has the byte layout of its azimuth counterpart.  Names keep
 * azimuth's field names; azimuth's anonymous unions hold several alias views
 * of the same bytes (e.g. vec3 {x,y,z} / {r,g,b}).  Only one view per offset is
 * kept here, and aliases that would repeat a member name get a different name
 * with the same offset (noted beside each).
 *
 * Reference layouts (file:line in ff-k/azimuth):
 *   vec2/vec3/vec4/mat4/aabb  src/azimuth_math.h:45-430
 *   brdf                      src/azimuth_brdf.h:11-17
 *   texture                   src/azimuth_texture.h:52-86
 *   material                  src/azimuth_material.h:1-19
 *   triangle, mesh, entity    src/azimuth_entity.h:15-102
 *   light                     src/azimuth_light.h:9-42
 *   tonemap, camera           src/azimuth_camera.h:7-56
 *   epsilon_values, scene     src/azimuth_scene.h:1-30
 *   scissor, filter_type,
 *   pixel                     src/azimuth_main.cpp:35-48
 *   ray3, ray_hit             src/azimuth_ray.h:1-13
 */
#ifndef AZ_ABI_H
#define AZ_ABI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct az_vec2  { float x, y; } az_vec2;              /* also u,v   */
typedef struct az_vec2u { uint32_t x, y; } az_vec2u;
typedef struct az_vec3  { float x, y, z; } az_vec3;           /* also r,g,b */
typedef struct az_vec3u { uint32_t x, y, z; } az_vec3u;
typedef struct az_vec4  { float x, y, z, w; } az_vec4;        /* NearPlane: r,l,b,t = x,y,z,w */
typedef struct az_mat4  { float E[4][4]; } az_mat4;           /* row-major E[row][col] */
typedef struct az_aabb  { az_vec3 Min, Max, Center; } az_aabb;

/* src/azimuth_brdf.h:1-9 */
enum {
    AZ_BRDF_Phong = 0,
    AZ_BRDF_ModifiedPhong,
    AZ_BRDF_NormalizedModifiedPhong,
    AZ_BRDF_BlinnPhong,
    AZ_BRDF_ModifiedBlinnPhong,
    AZ_BRDF_NormalizedModifiedBlinnPhong,
    AZ_BRDF_TorranceSparrow
};

typedef struct az_brdf {
    float    Exponent;
    float    RefractiveIndex;
    uint32_t Type;           /* brdf_type */
    uint32_t ID;
} az_brdf;

/* src/azimuth_texture.h:22-50 */
enum { AZ_PerlinAppearance_Patch = 0, AZ_PerlinAppearance_Vein };
enum { AZ_TextureWrap_Clamp = 0, AZ_TextureWrap_Repeat };
enum { AZ_TextureBlend_ReplaceAll = 0, AZ_TextureBlend_ReplaceDiffuse, AZ_TextureBlend_BlendDiffuse };
enum { AZ_TextureFilter_Nearest = 0, AZ_TextureFilter_Bilinear };
enum { AZ_TextureType_2D = 0, AZ_TextureType_PerlinNoise };
enum { AZ_PixelFormat_RGB_U8 = 0, AZ_PixelFormat_RGB_F32 };

#define AZ_PERLIN_GRADIENT_SIZE 256

typedef struct az_texture {
    char ImagePath[256];
    union {
        struct {                       /* 2D image */
            void    *Pixels;
            uint32_t PixelFormat;
            uint32_t Width;
            uint32_t Height;
            float    InvWidth;
            float    InvHeight;
            float    Normalizer;
            uint32_t Loaded;
            uint32_t ImageFileFormat;
        };
        struct {                       /* Perlin noise */
            uint32_t Perm[AZ_PERLIN_GRADIENT_SIZE];
            float    ScalingFactor;
            uint32_t PerlinAppearance;
        };
    };
    float    BumpMapMultiplier;
    uint32_t BumpMap;
    uint32_t Degamma;
    uint32_t ID;
    uint32_t WrapMode;
    uint32_t BlendMode;
    uint32_t Filter;
    uint32_t Type;
} az_texture;

typedef struct az_material {
    az_brdf  BRDF;
    az_vec3  AmbientReflectance;
    az_vec3  DiffuseReflectance;
    az_vec3  SpecularReflectance;
    az_vec3  MirrorReflectance;
    az_vec3  Transparency;
    float    RefractionIndex;
    float    Glossiness;
    uint32_t Degamma;
    uint32_t BRDFID;
    uint32_t ID;
} az_material;

/* src/azimuth_entity.h:1-11 */
enum { AZ_Entity_Sphere = 0, AZ_Entity_Triangle, AZ_Entity_MeshInstance, AZ_Entity_BVHNode };
enum { AZ_Shading_Flat = 0, AZ_Shading_Smooth };

struct az_entity;

typedef struct az_triangle {
    az_vec3 P0, P1, P2, N;
} az_triangle;

typedef struct az_mesh {
    az_mat4  InvTransformationMatrix;
    az_mat4  TransformationMatrix;
    az_vec3  MotionVector;
    az_vec3  Radiance;
    struct az_entity *BVH;
    az_triangle *Triangles;
    float    TotalArea;
    int32_t  UVOffset;
    uint32_t IsEmitter;
    uint32_t TriangleCount;
    uint32_t TextureIndex;
    uint32_t MaterialIndex;
    uint32_t ID;
    uint32_t ShadingMode;
} az_mesh;

typedef struct az_entity {
    union {
        struct {                           /* Sphere */
            az_vec3 Center;
            float   Radius;
        };
        struct {                           /* Triangle */
            az_vec3 P0, P1, P2;
            az_vec3 N0, N1, N2;
            az_vec3 FaceNormal;
            az_vec2 UV0, UV1, UV2;
            uint32_t ShadingMode;
        };
        struct {                           /* MeshInstance */
            az_aabb  AABB;
            az_mesh *Mesh;
            uint32_t BaseMeshID;
            uint32_t ResetTransform;
        };
        struct {                           /* BVHNode: AABB is shared with MeshInstance.AABB */
            az_aabb  NodeAABB;
            struct az_entity *Right;
            struct az_entity *Left;
        };
    };
    az_mat4  InvTransformationMatrix;
    az_mat4  TransformationMatrix;
    az_vec3  MotionVector;
    az_vec3  Radiance;
    uint32_t IsEmitter;
    uint32_t TextureIndex;   /* 0 = untextured, else index+1 into scene.Textures */
    uint32_t MaterialIndex;
    uint32_t ID;
    uint32_t UniqueEntityID;
    uint32_t Type;           /* entity_type */
} az_entity;

/* src/azimuth_light.h:1-7 */
enum { AZ_Light_Point = 0, AZ_Light_Area, AZ_Light_Directional, AZ_Light_Spot, AZ_Light_Entity };

typedef struct az_light {
    union {
        struct {                           /* Point / Area / Spot share Position, Intensity */
            az_vec3 Position;
            az_vec3 Intensity;
            az_vec3 EdgeVectors[2];        /* Area */
            az_vec3 Normal;                /* Area */
        };
        struct {                           /* Directional: Direction aliases Position */
            az_vec3 Direction;
            az_vec3 DirectionalIntensity;  /* alias of Intensity */
        };
        struct {                           /* Spot */
            az_vec3 SpotPosition;          /* alias of Position */
            az_vec3 SpotIntensity;         /* alias of Intensity */
            az_vec3 SpotDirection;
            float   CoverageAngle;
            float   FallOffAngle;
            float   CosHalfCoverage;
            float   CosHalfFallOff;
        };
        struct {
            az_entity Entity;              /* EntityLight: a copy of the emitting entity */
        };
    };
    uint32_t ID;
    uint32_t Type;
} az_light;

/* src/azimuth_camera.h:1-56 */
enum { AZ_Tonemap_None = 0, AZ_Tonemap_Photographic };
enum { AZ_Camera_Detailed = 0, AZ_Camera_Simple };

typedef struct az_tonemap {
    float    KeyValue;
    float    BurnoutPercentage;
    float    Saturation;
    uint32_t Operator;
} az_tonemap;

typedef struct az_camera {
    az_tonemap Tonemap;
    char     ImageName[256];
    uint32_t SaveFormat;
    union {
        az_vec4 NearPlane;                 /* Detailed camera: r,l,b,t */
        float   FovY;                      /* Simple camera, degrees */
    };
    az_vec3  Position;
    az_vec3  Gaze;
    az_vec3  Up;
    az_vec3  BackgroundColor;
    az_vec2u Resolution;
    float    NearDistance;
    float    FocusDistance;
    float    ApertureSize;
    float    Gamma;
    float    InvGamma;
    uint32_t GammaCorrection_sRGB;
    uint32_t GazeIsPoint;
    uint32_t IsLeftHanded;
    uint32_t SaveEXR;
    uint32_t SampleCount;
    uint32_t ID;
    uint32_t Type;
} az_camera;

typedef struct az_epsilon_values {
    float Intersection;
    float ShadowRay;
} az_epsilon_values;

typedef struct az_scene {
    az_vec3     AmbientLight;
    az_vec3     BackgroundColor;
    az_texture  BackgroundTexture;
    az_entity  *BVHRoot;
    az_mesh    *Meshes;
    az_material *Materials;
    az_light   *Lights;
    az_texture *Textures;
    az_texture  EnvironmentMap;
    uint32_t MeshCount;
    uint32_t MaterialCount;
    uint32_t LightCount;
    uint32_t TextureCount;
    uint32_t MaxRecursionDepth;
    uint32_t UseBackgroundTexture;
    uint32_t UseEnvironmentMap;
    uint32_t PathTrace;
    uint32_t ImportanceSampling;
} az_scene;

/* src/azimuth_main.cpp:35-48 */
typedef struct az_scissor { az_vec2u Max; az_vec2u Min; } az_scissor;
enum { AZ_Filter_Box = 0, AZ_Filter_Gaussian = 1 };
typedef struct az_pixel { az_vec3 Color; float TotalWeight; } az_pixel;

/* src/azimuth_ray.h:1-13 */
typedef struct az_ray3 { az_vec3 Origin; az_vec3 Direction; float T; } az_ray3;
typedef struct az_ray_hit {
    az_vec3 P;
    az_vec3 Normal;
    az_vec2 UV;
    az_entity *Entity;
    float t;
} az_ray_hit;

#ifdef __cplusplus
}  /* extern "C" */
#endif

/* Layout checks against the sizes azimuth has on x86-64. */
#ifdef __cplusplus
#define AZ_ABI_STATIC_ASSERT(c, m) static_assert(c, m)
#else
#define AZ_ABI_STATIC_ASSERT(c, m) _Static_assert(c, m)
#endif
AZ_ABI_STATIC_ASSERT(sizeof(az_mat4) == 64, "mat4");
AZ_ABI_STATIC_ASSERT(sizeof(az_aabb) == 36, "aabb");
AZ_ABI_STATIC_ASSERT(sizeof(az_brdf) == 16, "brdf");
AZ_ABI_STATIC_ASSERT(sizeof(az_texture) == 1320, "texture");
AZ_ABI_STATIC_ASSERT(sizeof(az_material) == 96, "material");
AZ_ABI_STATIC_ASSERT(sizeof(az_triangle) == 48, "triangle");
AZ_ABI_STATIC_ASSERT(sizeof(az_mesh) == 200, "mesh");
AZ_ABI_STATIC_ASSERT(sizeof(az_entity) == 288, "entity");
AZ_ABI_STATIC_ASSERT(sizeof(az_light) == 296, "light");
AZ_ABI_STATIC_ASSERT(sizeof(az_camera) == 396, "camera");
AZ_ABI_STATIC_ASSERT(sizeof(az_scene) == 2744, "scene");
AZ_ABI_STATIC_ASSERT(sizeof(az_pixel) == 16, "pixel");
AZ_ABI_STATIC_ASSERT(sizeof(az_scissor) == 16, "scissor");
AZ_ABI_STATIC_ASSERT(sizeof(az_ray3) == 28, "ray3");
AZ_ABI_STATIC_ASSERT(sizeof(az_ray_hit) == 48, "ray_hit");
AZ_ABI_STATIC_ASSERT(offsetof(az_entity, Right) == 40, "entity.Right");
AZ_ABI_STATIC_ASSERT(offsetof(az_entity, Left) == 48, "entity.Left");
AZ_ABI_STATIC_ASSERT(offsetof(az_entity, InvTransformationMatrix) == 112, "entity.Inv");
AZ_ABI_STATIC_ASSERT(offsetof(az_entity, UniqueEntityID) == 280, "entity.UniqueEntityID");
AZ_ABI_STATIC_ASSERT(offsetof(az_texture, Perm) == 256, "texture.Perm");
AZ_ABI_STATIC_ASSERT(offsetof(az_texture, ScalingFactor) == 1280, "texture.ScalingFactor");
AZ_ABI_STATIC_ASSERT(offsetof(az_scene, BVHRoot) == 1344, "scene.BVHRoot");
AZ_ABI_STATIC_ASSERT(offsetof(az_scene, EnvironmentMap) == 1384, "scene.EnvironmentMap");
AZ_ABI_STATIC_ASSERT(offsetof(az_camera, NearPlane) == 276, "camera.NearPlane");
AZ_ABI_STATIC_ASSERT(offsetof(az_light, Type) == 292, "light.Type");

#endif /* AZ_ABI_H */
