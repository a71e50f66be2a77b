// Device-resident scene: flattened from azimuth's pointer graph.
//
// Layout (all arrays in HBM, 16-byte aligned records):
//   tris[]      DevTri, 48 B: P0, P0-P1, P0-P2, face normal -- exactly the
//               operands of azimuth's Cramer test (src/azimuth_main.cpp:154-189)
//   tri_attr[]  DevTriAttr, 80 B: vertex normals, UVs, shading mode,
//               texture, face id, owning entity (only read when shading)
//   ents[]      DevEntity: one per top-level entity (sphere, mesh instance,
//               top-level triangle) with matrices, motion, material, uid
//   groups[]    mesh instances that share bitwise-identical transforms and
//               motion share one bottom-level BVH ("group")
//   tlas_prims[] top-level primitives: sphere entities and groups
//   nodes[]     binary BVH nodes (64 B, both child boxes in one node), TLAS
//               and every group's BLAS in one pool
#pragma once
#include <cstdint>

#include "az_device_math.cuh"

namespace azd {

struct __align__(16) DevTri {
    float4 a;  // P0.x P0.y P0.z E1.x     (E1 = P0 - P1)
    float4 b;  // E1.y E1.z E2.x E2.y     (E2 = P0 - P2)
    float4 c;  // E2.z FN.x FN.y FN.z     (face normal, for back-face culling)
};

// The exact vertices of a triangle: the input of the hierarchy build (boxes)
// and the operands of the watertight test (AZ_FLAG_WATERTIGHT), which needs the
// shared vertices of neighbouring triangles bit for bit.
struct __align__(16) DevTriVerts {
    float4 a;  // P0.x P0.y P0.z P1.x
    float4 b;  // P1.y P1.z P2.x P2.y
    float4 c;  // P2.z FN.x FN.y FN.z     (face normal)
};

struct __align__(16) DevTriAttr {
    float n0[3], n1[3], n2[3];
    float uv0[2], uv1[2], uv2[2];
    uint32_t shading_mode;
    uint32_t texture_index;  // 0 or index+1 into textures (triangle entity's TextureIndex)
    uint32_t face_id;        // azimuth triangle entity ID
    uint32_t entity;         // dense index of the owning top-level entity
};

enum : uint32_t { ENT_SPHERE = 0, ENT_TRIANGLE = 1, ENT_INSTANCE = 2 };

struct __align__(16) DevEntity {
    m34 inv;                 // InvTransformationMatrix (rows 0..2)
    m34 xf;                  // TransformationMatrix (rows 0..2)
    float motion[3];
    float radiance[3];
    float center[3];
    float radius;
    uint32_t type;
    uint32_t is_emitter;
    uint32_t texture_index;
    uint32_t material;
    uint32_t uid;            // UniqueEntityID
    uint32_t group;          // group index of a mesh instance
    uint32_t pad[2];
};

struct __align__(16) DevGroup {
    m34 inv, xf;
    float motion[3];
    uint32_t root;           // BLAS root node, or 0xFFFFFFFF if empty
    uint32_t raw;            // 1: top-level triangles, tested with the world ray as is
    uint32_t tri_begin, tri_end;
    uint32_t identity;       // inv/xf are the identity and motion is zero
};

// TLAS primitive: kind in bit 31 (1 = group), index in the low bits.
#define AZD_TLAS_GROUP 0x80000000u

struct __align__(16) BVHNode {
    float4 bx;   // c0.lo.x c0.hi.x c1.lo.x c1.hi.x
    float4 by;   // c0.lo.y c0.hi.y c1.lo.y c1.hi.y
    float4 bz;   // c0.lo.z c0.hi.z c1.lo.z c1.hi.z
    uint4 ch;    // child0, child1, count0, count1 (count 0: inner node index; else primitive range start)
};

// 8-wide compressed node (80 B = five 16-byte fetches).  Child boxes are
// quantised to 8 bits per bound on a per-node grid: lo = p + q_lo * 2^e,
// hi = p + q_hi * 2^e, rounded outward so the decoded boxes contain the true
// ones.  Slot s holds the child whose centre lies on the side given by the
// bits of s (bit a set: upper half along axis a), so visiting slots in the
// order of (s XOR ray-octant) is near-first.
struct __align__(16) WideNode {
    float px, py, pz;
    uint8_t ex, ey, ez;       // biased float exponents of the grid step per axis
    uint8_t imask;            // bit s: slot s is an inner node
    uint32_t child_base;      // first inner child node; inner children are consecutive in slot order
    uint32_t prim_base;       // first primitive of the leaf children
    uint8_t meta[8];          // inner: 0; leaf: (count << 5) | offset from prim_base; empty: 0 with imask bit clear
    uint8_t qlo_x[8], qlo_y[8], qlo_z[8];
    uint8_t qhi_x[8], qhi_y[8], qhi_z[8];
};
static_assert(sizeof(WideNode) == 80, "wide node is five 16-byte words");

// Textures (src/azimuth_texture.h:52-86), compacted for the device.
struct __align__(16) DevTexture {
    uint32_t type, format, width, height;
    float inv_width, inv_height, normalizer, bump_mul;
    uint32_t wrap, filter, blend, bump;
    float scaling;            // Perlin ScalingFactor
    uint32_t appearance;
    uint32_t perm_offset;     // into perlin_perm (256 entries after the 256 words azimuth reads before them)
    uint32_t pad;
    unsigned long long texel_offset;  // bytes into texels
    unsigned long long pad2;
};

struct __align__(16) DevMaterial {
    float ambient[3], diffuse[3], specular[3], mirror[3], transparency[3];
    float refraction_index, glossiness;
    float exponent, brdf_refractive_index;
    uint32_t brdf_type;
    uint32_t transparent, is_mirror;   // bitwise-nonzero tests of src/azimuth_main.cpp:1091-1104
};

enum : uint32_t { LIGHT_POINT = 0, LIGHT_AREA = 1, LIGHT_DIRECTIONAL = 2, LIGHT_SPOT = 3, LIGHT_ENTITY = 4 };

struct __align__(16) DevLight {
    uint32_t type;
    uint32_t entity_type;     // for entity lights: ENT_SPHERE or ENT_INSTANCE
    uint32_t uid;             // UniqueEntityID of the light's entity
    uint32_t tri_count;
    float position[3];        // also Direction of a directional light
    float intensity[3];       // Radiance for entity lights
    float edge0[3], edge1[3], normal[3];
    float spot_dir[3];
    float cos_half_coverage, cos_half_falloff;
    float center[3], radius;
    float total_area;
    uint32_t tri_offset;      // into light_tris (mesh light's `triangle` array)
    m34 inv, xf;
    float motion[3];          // the light entity's MotionVector
    uint32_t ent_index;       // dense index of the light's entity in ents[], or 0xFFFFFFFF
    uint32_t identity;        // inv/xf are the identity and motion is zero
};

// An entity light whose visibility needs a full nearest-hit query: its entity
// is not among the scene's top-level entities, or its mesh is too large to
// test on its own.
__host__ __device__ __forceinline__ bool entity_light_needs_full_query(const DevLight &L) {
    return L.ent_index == 0xFFFFFFFFu || (L.entity_type != ENT_SPHERE && L.tri_count > 64);
}

struct __align__(16) DevLightTri {
    float4 p0n;  // P0.xyz, N.x
    float4 p1n;  // P1.xyz, N.y
    float4 p2n;  // P2.xyz, N.z
};

// DevScene.features: parts of the shading code a scene can reach.
enum : uint32_t { FEAT_TEXTURES = 1u, FEAT_ENV = 2u, FEAT_SPECIAL = 4u, FEAT_ANALYTIC_LIGHTS = 8u };

// Everything a kernel needs, passed by value.
struct DevScene {
    const DevTri *tris;
    const DevTriVerts *tri_verts;   // the same triangles' exact vertices (watertight test)
    const DevTriAttr *tri_attr;
    const DevEntity *ents;
    const DevGroup *groups;
    const uint32_t *tlas_prims;
    const BVHNode *nodes;           // binary nodes (unused once wide nodes exist)
    const WideNode *wnodes;
    const DevMaterial *materials;
    const DevTexture *textures;     // [0 .. texture_count) = scene.Textures
    const DevLight *lights;
    const DevLightTri *light_tris;
    const uint32_t *perlin_perm;
    const float *perlin_grad;       // 256 * 3
    const unsigned char *texels;
    uint32_t tlas_root;             // 0xFFFFFFFF: empty scene
    uint32_t tlas_single_group;     // the top level's only primitive when it is a group (its hierarchy
                                    // is entered directly), else 0xFFFFFFFF
    float box_lo[3], box_scale[3];  // scene bounds: cell = (p - box_lo) * box_scale in [0, 1)
    uint32_t ent_count, group_count, material_count, texture_count, light_count;
    uint32_t bg_texture, env_texture;  // indices into textures[] (appended after scene.Textures)
    float ambient[3];
    float background[3];
    uint32_t use_bg_texture, use_env_map;
    uint32_t max_depth, path_trace, importance_sampling;
    uint32_t light_draws;           // RNG draws made by the light loop at every vertex
    uint32_t features;              // FEAT_* bits
    uint32_t full_light_queries;    // 1: an entity light needs full nearest-hit visibility queries
    uint32_t top_spheres;           // sphere entities at the top level (the traversal kernels with the
                                    // sphere test inline serve scenes that have any)
    // luminance CDF of a 2D environment map (null when the scene has none):
    // env_rows[0..H] over rows (weighted by sin theta), env_cols[r * (W + 1) + 0..W] within row r
    const float *env_rows;
    const float *env_cols;
    uint32_t env_cdf_w, env_cdf_h;
};

}  // namespace azd
