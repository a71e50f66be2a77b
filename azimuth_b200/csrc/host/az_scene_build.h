// Host-side scene assembly in azimuth's own structs.
//
// SceneBuilder collects what azimuth's XML importer would have parsed
// (spheres, meshes as vertex/face lists, materials, lights, textures) and
// finalises it the way src/azimuth_xml.cpp:3632-3915 does: per-vertex normals,
// triangle entities and `triangle` arrays, TotalArea, one triangle BVH per
// mesh, mesh-instance entities with world AABBs (motion included),
// UniqueEntityID, entity lights and the scene-level BVH.  The two BVH builders
// restate src/azimuth_bvh.cpp so that the resulting pointer graph is the one
// azimuth itself would render.
#pragma once
#include <cstdint>
#include <memory>
#include <vector>

#include "azimuth_gpu.h"

namespace az {

az_mat4 Mat4Identity();
az_mat4 Mat4Mul(const az_mat4 &A, const az_mat4 &B);
az_mat4 Mat4Translate(az_vec3 T);
az_mat4 Mat4Scale(az_vec3 S);
bool Mat4IsIdentity(const az_mat4 &M);

az_entity DefaultEntity();
az_material DefaultMaterial();
az_texture DefaultTexture();
az_camera DefaultCamera();
az_scene DefaultScene();

struct MeshDesc {
    std::vector<az_vec3u> Faces;        // indices into the builder's shared vertex array
    az_mat4 Transform = Mat4Identity();
    az_mat4 InvTransform = Mat4Identity();
    az_vec3 Motion = {0, 0, 0};
    az_vec3 Radiance = {0, 0, 0};
    bool IsEmitter = false;
    bool IsLight = false;               // listed as an entity light (azimuth "LightMesh")
    uint32_t MaterialIndex = 0;
    uint32_t TextureIndex = 0;
    int32_t UVOffset = 0;
    uint32_t ShadingMode = AZ_Shading_Flat;
};

// Owns every array the finished az_scene points into.
class SceneBuilder {
public:
    SceneBuilder();
    ~SceneBuilder();
    SceneBuilder(const SceneBuilder &) = delete;
    SceneBuilder &operator=(const SceneBuilder &) = delete;

    uint32_t AddVertex(az_vec3 P);
    uint32_t AddUV(az_vec2 UV);
    uint32_t AddMaterial(const az_material &M);   // returns its index in Materials[]
    uint32_t AddTexture(const az_texture &T);     // returns TextureIndex (index + 1)
    void AddLight(const az_light &L);             // point/area/directional/spot lights
    // Sphere entity; `IsLight` lists it as an entity light (azimuth "LightSphere").
    void AddSphere(az_entity E, bool IsLight);
    void AddMesh(const MeshDesc &M);
    // Owns texel storage for a 2D texture (kept alive with the scene).
    void *AllocTexels(size_t Bytes);

    // Runs the importer's post-processing and both BVH builds.  Returns false
    // on an empty mesh or a failed allocation.  With `soup_only` the meshes
    // are left as the importer holds them before its post-processing (no
    // triangles, areas or mesh BVHs; BVHRoot over the other entities only).
    bool Finalize(bool soup_only = false);

    az_scene Scene;                  // valid after Finalize()
    az_mesh_soup Soup;               // the meshes before post-processing, valid after Finalize()
    std::vector<az_vec3> Vertices;
    std::vector<az_vec2> UVs;

private:
    struct Storage;
    std::unique_ptr<Storage> S;
};

// Restatements of azimuth's BVH builders (src/azimuth_bvh.cpp:1-221 and
// :223-328): object split at the node AABB centre on axis Depth % 3,
// in-place partition, half split as fallback, one primitive per leaf.
// Nodes are allocated from `Pool`.
struct EntityPool {
    std::vector<std::unique_ptr<az_entity[]>> Blocks;
    size_t Used = 0, Capacity = 0;
    az_entity *Alloc();
};
bool ConstructBVH(az_entity **Node, az_entity *Entities, uint32_t Count, uint32_t Depth,
                  EntityPool &Pool);
bool ConstructBVHTrianglesOnly(az_entity **Node, az_entity *Triangles, uint32_t Count,
                               uint32_t Depth, EntityPool &Pool);

}  // namespace az
