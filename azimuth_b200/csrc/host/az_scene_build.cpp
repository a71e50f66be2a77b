// Host-side scene assembly in azimuth's structs; see az_scene_build.h.
// Compiled with -ffp-contract=off so every sum below rounds like azimuth's.
#include "az_scene_build.h"

#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>

namespace az {

namespace {
inline az_vec3 V3(float x, float y, float z) { return az_vec3{x, y, z}; }
inline az_vec3 Sub(az_vec3 a, az_vec3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline az_vec3 Add(az_vec3 a, az_vec3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline az_vec3 Cross(az_vec3 a, az_vec3 b) {
    return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float Length(az_vec3 v) { return sqrtf(v.x * v.x + v.y * v.y + v.z * v.z); }
inline az_vec3 Normalize(az_vec3 v) {  // src/azimuth_math.cpp:1298-1313
    float L = Length(v);
    if (L != 0.0f) return V3(v.x / L, v.y / L, v.z / L);
    return V3(0, 0, 0);
}
inline float Comp(const az_vec3 &v, uint32_t d) { return d == 0 ? v.x : (d == 1 ? v.y : v.z); }
// mat4 * (x, y, z, 1), src/azimuth_math.cpp:1400-1426 (w row unused here)
inline az_vec3 MulPoint(const az_mat4 &M, az_vec3 v) {
    return V3(M.E[0][0] * v.x + M.E[0][1] * v.y + M.E[0][2] * v.z + M.E[0][3] * 1.0f,
              M.E[1][0] * v.x + M.E[1][1] * v.y + M.E[1][2] * v.z + M.E[1][3] * 1.0f,
              M.E[2][0] * v.x + M.E[2][1] * v.y + M.E[2][2] * v.z + M.E[2][3] * 1.0f);
}
// PointToWorld, src/azimuth_math.cpp:1775-1800
inline az_vec3 PointToWorld(az_vec3 v, const az_mat4 &M) {
    return V3(M.E[0][0] * v.x + M.E[0][1] * v.y + M.E[0][2] * v.z + M.E[0][3],
              M.E[1][0] * v.x + M.E[1][1] * v.y + M.E[1][2] * v.z + M.E[1][3],
              M.E[2][0] * v.x + M.E[2][1] * v.y + M.E[2][2] * v.z + M.E[2][3]);
}
inline void Grow(az_aabb &B, az_vec3 p) {
    if (B.Min.x > p.x) B.Min.x = p.x;
    if (B.Min.y > p.y) B.Min.y = p.y;
    if (B.Min.z > p.z) B.Min.z = p.z;
    if (B.Max.x < p.x) B.Max.x = p.x;
    if (B.Max.y < p.y) B.Max.y = p.y;
    if (B.Max.z < p.z) B.Max.z = p.z;
}
inline az_aabb EmptyBox() {
    az_aabb B;
    B.Min = V3(FLT_MAX, FLT_MAX, FLT_MAX);
    B.Max = V3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    B.Center = V3(0, 0, 0);
    return B;
}
}  // namespace

az_mat4 Mat4Identity() {
    az_mat4 M;
    memset(&M, 0, sizeof(M));
    M.E[0][0] = M.E[1][1] = M.E[2][2] = M.E[3][3] = 1.0f;
    return M;
}

az_mat4 Mat4Mul(const az_mat4 &A, const az_mat4 &B) {  // src/azimuth_math.cpp:1381-1398
    az_mat4 R;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            float v = 0.0f;
            v += A.E[i][0] * B.E[0][j];
            v += A.E[i][1] * B.E[1][j];
            v += A.E[i][2] * B.E[2][j];
            v += A.E[i][3] * B.E[3][j];
            R.E[i][j] = v;
        }
    return R;
}

az_mat4 Mat4Translate(az_vec3 T) {
    az_mat4 M = Mat4Identity();
    M.E[0][3] = T.x; M.E[1][3] = T.y; M.E[2][3] = T.z;
    return M;
}

az_mat4 Mat4Scale(az_vec3 S) {
    az_mat4 M = Mat4Identity();
    M.E[0][0] = S.x; M.E[1][1] = S.y; M.E[2][2] = S.z;
    return M;
}

bool Mat4IsIdentity(const az_mat4 &M) {
    az_mat4 I = Mat4Identity();
    return memcmp(&M, &I, sizeof(M)) == 0;
}

// Defaults of src/azimuth_entity.h:104-114, src/azimuth_material.h:21-30,
// src/azimuth_texture.h:88-104, src/azimuth_camera.h:58-83, src/azimuth_scene.h:32-42.
az_entity DefaultEntity() {
    az_entity E;
    memset(&E, 0, sizeof(E));
    E.Type = AZ_Entity_Sphere;
    E.InvTransformationMatrix = E.TransformationMatrix = Mat4Identity();
    return E;
}

az_material DefaultMaterial() {
    az_material M;
    memset(&M, 0, sizeof(M));
    M.BRDF.Type = AZ_BRDF_BlinnPhong;
    return M;
}

az_texture DefaultTexture() {
    az_texture T;
    memset(&T, 0, sizeof(T));
    T.PixelFormat = AZ_PixelFormat_RGB_U8;
    T.Normalizer = 255.0f;
    T.BumpMapMultiplier = 1.0f;
    T.BumpMap = 0;
    T.WrapMode = AZ_TextureWrap_Repeat;
    T.BlendMode = AZ_TextureBlend_BlendDiffuse;
    T.Filter = AZ_TextureFilter_Nearest;
    T.Type = AZ_TextureType_2D;
    return T;
}

az_camera DefaultCamera() {
    az_camera C;
    memset(&C, 0, sizeof(C));
    memcpy(C.ImageName, "u.png", 5);
    C.NearPlane = az_vec4{1.0f, -1.0f, -1.0f, 1.0f};
    C.Gaze = V3(0, 0, -1);
    C.Up = V3(0, 1, 0);
    C.Resolution = az_vec2u{640, 360};
    C.NearDistance = 1.0f;
    C.Gamma = C.InvGamma = 1.0f;
    C.SampleCount = 1;
    C.Type = AZ_Camera_Detailed;
    return C;
}

az_scene DefaultScene() {
    az_scene S;
    memset(&S, 0, sizeof(S));
    S.BackgroundTexture = DefaultTexture();
    S.EnvironmentMap = DefaultTexture();
    return S;
}

az_entity *EntityPool::Alloc() {
    if (Used == Capacity) {
        size_t n = Capacity ? Capacity : 1024;
        Blocks.emplace_back(new az_entity[n]);
        memset(Blocks.back().get(), 0, n * sizeof(az_entity));
        Used = 0;
        Capacity = n;
    }
    return &Blocks.back()[Used++];
}

// src/azimuth_bvh.cpp:1-221
bool ConstructBVH(az_entity **Node, az_entity *Entities, uint32_t Count, uint32_t Depth,
                  EntityPool &Pool) {
    if (Count == 0) return false;
    if (Count == 1) {
        *Node = Entities;
        return true;
    }
    az_entity *N = Pool.Alloc();
    *Node = N;
    N->Type = AZ_Entity_BVHNode;
    N->Right = nullptr;
    N->Left = nullptr;
    az_aabb B = EmptyBox();
    for (uint32_t i = 0; i < Count; i++) {
        const az_entity *E = Entities + i;
        switch (E->Type) {
            case AZ_Entity_Sphere: {
                az_vec3 Min = V3(E->Center.x - E->Radius, E->Center.y - E->Radius,
                                 E->Center.z - E->Radius);
                az_vec3 Max = V3(E->Center.x + E->Radius, E->Center.y + E->Radius,
                                 E->Center.z + E->Radius);
                const az_vec3 Corners[8] = {
                    V3(Min.x, Min.y, Min.z), V3(Min.x, Min.y, Max.z), V3(Min.x, Max.y, Min.z),
                    V3(Min.x, Max.y, Max.z), V3(Max.x, Min.y, Min.z), V3(Max.x, Min.y, Max.z),
                    V3(Max.x, Max.y, Min.z), V3(Max.x, Max.y, Max.z)};
                for (int c = 0; c < 8; c++) {
                    az_vec3 TV = MulPoint(E->TransformationMatrix, Corners[c]);
                    if (Min.x > TV.x) Min.x = TV.x;
                    if (Min.y > TV.y) Min.y = TV.y;
                    if (Min.z > TV.z) Min.z = TV.z;
                    if (Max.x < TV.x) Max.x = TV.x;
                    if (Max.y < TV.y) Max.y = TV.y;
                    if (Max.z < TV.z) Max.z = TV.z;
                }
                if (Length(E->MotionVector) > 0.0f) {
                    az_vec3 FMin = Add(Min, E->MotionVector);
                    az_vec3 FMax = Add(Max, E->MotionVector);
                    if (Min.x > FMin.x) Min.x = FMin.x;
                    if (Min.y > FMin.y) Min.y = FMin.y;
                    if (Min.z > FMin.z) Min.z = FMin.z;
                    if (Max.x < FMax.x) Max.x = FMax.x;
                    if (Max.y < FMax.y) Max.y = FMax.y;
                    if (Max.z < FMax.z) Max.z = FMax.z;
                }
                Grow(B, Min);
                Grow(B, Max);
            } break;
            case AZ_Entity_Triangle:
                Grow(B, E->P0);
                Grow(B, E->P1);
                Grow(B, E->P2);
                break;
            default:  // mesh instance or BVH node
                Grow(B, E->AABB.Min);
                Grow(B, E->AABB.Max);
                break;
        }
    }
    B.Center = V3(B.Min.x * 0.5f + B.Max.x * 0.5f, B.Min.y * 0.5f + B.Max.y * 0.5f,
                  B.Min.z * 0.5f + B.Max.z * 0.5f);
    N->AABB = B;
    uint32_t Dim = Depth % 3;
    float SplitAt = Comp(B.Center, Dim);
    uint32_t Left = 0;
    for (uint32_t i = 1; i < Count; i++) {
        az_entity *E = Entities + i;
        float Pos = 0.0f;
        switch (E->Type) {
            case AZ_Entity_Sphere: Pos = Comp(PointToWorld(E->Center, E->TransformationMatrix), Dim); break;
            case AZ_Entity_Triangle: Pos = Comp(E->P0, Dim); break;
            default: Pos = Comp(E->AABB.Center, Dim); break;
        }
        if (Pos < SplitAt) {
            az_entity Tmp = Entities[Left];
            Entities[Left] = *E;
            *E = Tmp;
            Left++;
        }
    }
    if (Left == 0 || Left == Count) Left = Count / 2;
    bool Ok = ConstructBVH(&N->Left, Entities, Left, Depth + 1, Pool);
    Ok = ConstructBVH(&N->Right, Entities + Left, Count - Left, Depth + 1, Pool) && Ok;
    return Ok;
}

// src/azimuth_bvh.cpp:223-328
bool ConstructBVHTrianglesOnly(az_entity **Node, az_entity *Tris, uint32_t Count, uint32_t Depth,
                               EntityPool &Pool) {
    if (Count == 0) return false;
    if (Count == 1) {
        *Node = Tris;
        return true;
    }
    az_entity *N = Pool.Alloc();
    *Node = N;
    N->Type = AZ_Entity_BVHNode;
    N->Right = nullptr;
    N->Left = nullptr;
    az_aabb B = EmptyBox();
    for (uint32_t i = 0; i < Count; i++) {
        Grow(B, Tris[i].P0);
        Grow(B, Tris[i].P1);
        Grow(B, Tris[i].P2);
    }
    B.Center = V3(B.Min.x * 0.5f + B.Max.x * 0.5f, B.Min.y * 0.5f + B.Max.y * 0.5f,
                  B.Min.z * 0.5f + B.Max.z * 0.5f);
    N->AABB = B;
    uint32_t Dim = Depth % 3;
    float SplitAt = Comp(B.Center, Dim);
    uint32_t Left = 0;
    for (uint32_t i = 1; i < Count; i++) {
        az_entity *T = Tris + i;
        if (Comp(T->P0, Dim) < SplitAt) {
            az_entity Tmp = Tris[Left];
            Tris[Left] = *T;
            *T = Tmp;
            Left++;
        }
    }
    if (Left == 0 || Left == Count) Left = Count / 2;
    bool Ok = ConstructBVHTrianglesOnly(&N->Left, Tris, Left, Depth + 1, Pool);
    Ok = ConstructBVHTrianglesOnly(&N->Right, Tris + Left, Count - Left, Depth + 1, Pool) && Ok;
    return Ok;
}

struct SceneBuilder::Storage {
    std::vector<az_entity> Spheres;            // with their "is light" flags below
    std::vector<bool> SphereIsLight;
    std::vector<MeshDesc> MeshDescs;
    std::vector<az_material> Materials;
    std::vector<az_texture> Textures;
    std::vector<az_light> Lights;
    std::vector<az_mesh> Meshes;
    std::vector<std::unique_ptr<az_entity[]>> TriEntities;
    std::vector<std::unique_ptr<az_triangle[]>> Triangles;
    std::unique_ptr<az_entity[]> Entities;
    std::unique_ptr<az_entity[]> RootEntities;   // soup-only scenes: the entities other than mesh instances
    std::vector<az_vec3u> SoupFaces;
    std::vector<az_mesh_desc> SoupDescs;
    std::vector<std::unique_ptr<uint8_t[]>> Texels;
    EntityPool Pool;
};

SceneBuilder::SceneBuilder() : Scene(DefaultScene()), S(new Storage) { memset(&Soup, 0, sizeof(Soup)); }
SceneBuilder::~SceneBuilder() = default;

uint32_t SceneBuilder::AddVertex(az_vec3 P) {
    Vertices.push_back(P);
    return (uint32_t)Vertices.size() - 1;
}

uint32_t SceneBuilder::AddUV(az_vec2 UV) {
    UVs.push_back(UV);
    return (uint32_t)UVs.size() - 1;
}

uint32_t SceneBuilder::AddMaterial(const az_material &M) {
    S->Materials.push_back(M);
    return (uint32_t)S->Materials.size() - 1;
}

uint32_t SceneBuilder::AddTexture(const az_texture &T) {
    S->Textures.push_back(T);
    return (uint32_t)S->Textures.size();
}

void SceneBuilder::AddLight(const az_light &L) { S->Lights.push_back(L); }

void SceneBuilder::AddSphere(az_entity E, bool IsLight) {
    E.Type = AZ_Entity_Sphere;
    S->Spheres.push_back(E);
    S->SphereIsLight.push_back(IsLight);
}

void SceneBuilder::AddMesh(const MeshDesc &M) { S->MeshDescs.push_back(M); }

void *SceneBuilder::AllocTexels(size_t Bytes) {
    S->Texels.emplace_back(new uint8_t[Bytes]);
    memset(S->Texels.back().get(), 0, Bytes);
    return S->Texels.back().get();
}

bool SceneBuilder::Finalize(bool soup_only) {
    Storage &St = *S;
    // Entities in importer order: parsed objects first (spheres here), mesh
    // instances appended while meshes are processed (src/azimuth_xml.cpp:3753-3776).
    std::vector<az_entity> Ents(St.Spheres.begin(), St.Spheres.end());
    std::vector<uint32_t> EntityLightIdx;
    for (size_t i = 0; i < St.Spheres.size(); i++)
        if (St.SphereIsLight[i]) EntityLightIdx.push_back((uint32_t)i);

    // The importer's shared arrays before its post-processing: faces of all
    // meshes in mesh order, each mesh a range of them
    St.SoupFaces.clear();
    St.SoupDescs.clear();
    for (size_t mi = 0; mi < St.MeshDescs.size(); mi++) {
        const MeshDesc &D = St.MeshDescs[mi];
        az_mesh_desc d;
        memset(&d, 0, sizeof(d));
        d.face_base = (uint32_t)St.SoupFaces.size();
        d.face_count = (uint32_t)D.Faces.size();
        d.uv_offset = D.UVOffset;
        d.shading_mode = D.ShadingMode;
        d.material_index = D.MaterialIndex;
        d.texture_index = D.TextureIndex;
        d.is_emitter = D.IsEmitter ? 1u : 0u;
        d.unique_entity_id = (uint32_t)(St.Spheres.size() + mi);
        d.motion = D.Motion;
        d.radiance = D.Radiance;
        d.transform = D.Transform;
        d.inv_transform = D.InvTransform;
        St.SoupFaces.insert(St.SoupFaces.end(), D.Faces.begin(), D.Faces.end());
        St.SoupDescs.push_back(d);
    }
    Soup.vertices = Vertices.empty() ? nullptr : Vertices.data();
    Soup.faces = St.SoupFaces.empty() ? nullptr : St.SoupFaces.data();
    Soup.uvs = UVs.empty() ? nullptr : UVs.data();
    Soup.meshes = St.SoupDescs.empty() ? nullptr : St.SoupDescs.data();
    Soup.vertex_count = (uint32_t)Vertices.size();
    Soup.face_count = (uint32_t)St.SoupFaces.size();
    Soup.uv_count = (uint32_t)UVs.size();
    Soup.mesh_count = (uint32_t)St.SoupDescs.size();

    // Per-vertex normals: normalised sum of unnormalised face normals over every
    // face that uses the vertex (src/azimuth_xml.cpp:3632-3667).
    std::vector<az_vec3> VN(soup_only ? 0 : Vertices.size(), V3(0, 0, 0));
    if (!soup_only)
    for (const MeshDesc &M : St.MeshDescs)
        for (const az_vec3u &F : M.Faces) {
            az_vec3 P0 = Vertices[F.x], P1 = Vertices[F.y], P2 = Vertices[F.z];
            az_vec3 FN = Cross(Sub(P1, P0), Sub(P2, P0));
            VN[F.x] = Add(VN[F.x], FN);
            VN[F.y] = Add(VN[F.y], FN);
            VN[F.z] = Add(VN[F.z], FN);
        }
    for (az_vec3 &n : VN) n = Normalize(n);

    St.Meshes.resize(St.MeshDescs.size());
    for (size_t mi = 0; mi < St.MeshDescs.size(); mi++) {
        const MeshDesc &D = St.MeshDescs[mi];
        uint32_t FaceCount = (uint32_t)D.Faces.size();
        if (FaceCount == 0) return false;
        az_mesh &Mesh = St.Meshes[mi];
        memset(&Mesh, 0, sizeof(Mesh));
        Mesh.TransformationMatrix = D.Transform;
        Mesh.InvTransformationMatrix = D.InvTransform;
        Mesh.MotionVector = D.Motion;
        Mesh.Radiance = D.Radiance;
        Mesh.IsEmitter = D.IsEmitter ? 1u : 0u;
        Mesh.TextureIndex = D.TextureIndex;
        Mesh.MaterialIndex = D.MaterialIndex;
        Mesh.UVOffset = D.UVOffset;
        Mesh.ID = (uint32_t)mi + 1;
        Mesh.ShadingMode = D.ShadingMode;
        Mesh.TriangleCount = FaceCount;
        if (soup_only) {
            az_entity Inst = DefaultEntity();
            Inst.BaseMeshID = (uint32_t)mi;
            Inst.ResetTransform = 0;
            Inst.MotionVector = D.Motion;
            Inst.Radiance = D.Radiance;
            Inst.IsEmitter = Mesh.IsEmitter;
            Inst.TextureIndex = D.TextureIndex;
            Inst.MaterialIndex = D.MaterialIndex;
            Inst.Type = AZ_Entity_MeshInstance;
            Ents.push_back(Inst);
            if (D.IsLight) EntityLightIdx.push_back((uint32_t)Ents.size() - 1);
            continue;
        }

        // Triangle entities and the `triangle` array (src/azimuth_xml.cpp:3669-3750).
        // The face index is stamped into the (otherwise unused) entity ID.
        St.TriEntities.emplace_back(new az_entity[FaceCount]);
        St.Triangles.emplace_back(new az_triangle[FaceCount]);
        az_entity *TE = St.TriEntities.back().get();
        az_triangle *Tri = St.Triangles.back().get();
        memset(TE, 0, sizeof(az_entity) * FaceCount);
        float TotalArea = 0.0f;
        for (uint32_t f = 0; f < FaceCount; f++) {
            az_entity &T = TE[f];
            T.ShadingMode = D.ShadingMode;
            T.Radiance = D.Radiance;
            T.IsEmitter = Mesh.IsEmitter;
            T.TextureIndex = D.TextureIndex;
            T.MaterialIndex = D.MaterialIndex;
            T.ID = f;
            T.Type = AZ_Entity_Triangle;
            const az_vec3u F = D.Faces[f];
            az_vec3 P0 = Vertices[F.x], P1 = Vertices[F.y], P2 = Vertices[F.z];
            T.P0 = P0; T.P1 = P1; T.P2 = P2;
            az_vec3 FN = Cross(Sub(P1, P0), Sub(P2, P0));
            float Len = Length(FN);
            TotalArea += Len / 2.0f;
            FN.x /= Len; FN.y /= Len; FN.z /= Len;
            T.FaceNormal = FN;
            T.N0 = VN[F.x]; T.N1 = VN[F.y]; T.N2 = VN[F.z];
            int32_t U0 = (int32_t)F.x + D.UVOffset, U1 = (int32_t)F.y + D.UVOffset,
                    U2 = (int32_t)F.z + D.UVOffset;
            if (U0 >= 0 && (size_t)U0 < UVs.size()) T.UV0 = UVs[U0];
            if (U1 >= 0 && (size_t)U1 < UVs.size()) T.UV1 = UVs[U1];
            if (U2 >= 0 && (size_t)U2 < UVs.size()) T.UV2 = UVs[U2];
            Tri[f].P0 = P0; Tri[f].P1 = P1; Tri[f].P2 = P2; Tri[f].N = FN;
        }
        Mesh.Triangles = Tri;
        Mesh.TotalArea = TotalArea;
        Mesh.TriangleCount = FaceCount;
        if (!ConstructBVHTrianglesOnly(&Mesh.BVH, TE, FaceCount, 0, St.Pool)) return false;

        az_entity Inst = DefaultEntity();
        Inst.BaseMeshID = (uint32_t)mi;
        Inst.ResetTransform = 0;
        Inst.MotionVector = D.Motion;
        Inst.Radiance = D.Radiance;
        Inst.IsEmitter = Mesh.IsEmitter;
        Inst.TextureIndex = D.TextureIndex;
        Inst.MaterialIndex = D.MaterialIndex;
        Inst.Type = AZ_Entity_MeshInstance;
        Ents.push_back(Inst);
        if (D.IsLight) EntityLightIdx.push_back((uint32_t)Ents.size() - 1);
    }

    // Instance transform and world AABB incl. motion (src/azimuth_xml.cpp:3785-3875).
    for (az_entity &E : Ents) {
        if (E.Type != AZ_Entity_MeshInstance) continue;
        E.Mesh = &St.Meshes[E.BaseMeshID];
        if (!E.ResetTransform) {
            E.TransformationMatrix = Mat4Mul(E.TransformationMatrix, E.Mesh->TransformationMatrix);
            E.InvTransformationMatrix = Mat4Mul(E.Mesh->InvTransformationMatrix, E.InvTransformationMatrix);
        }
        if (soup_only) continue;   // no mesh BVH to bound
        E.AABB = E.Mesh->BVH->AABB;  // a 1-triangle mesh reads the triangle's bytes here
        const az_aabb A = E.AABB;
        const az_vec3 Corners[8] = {
            V3(A.Min.x, A.Min.y, A.Min.z), V3(A.Min.x, A.Min.y, A.Max.z), V3(A.Min.x, A.Max.y, A.Min.z),
            V3(A.Min.x, A.Max.y, A.Max.z), V3(A.Max.x, A.Min.y, A.Min.z), V3(A.Max.x, A.Min.y, A.Max.z),
            V3(A.Max.x, A.Max.y, A.Min.z), V3(A.Max.x, A.Max.y, A.Max.z)};
        az_aabb T = EmptyBox();
        for (int c = 0; c < 8; c++) Grow(T, MulPoint(E.TransformationMatrix, Corners[c]));
        if (Length(E.MotionVector) > 0.0f) {
            az_aabb I = T;
            T.Min = Add(T.Min, E.MotionVector);
            T.Max = Add(T.Max, E.MotionVector);
            if (T.Min.x > I.Min.x) T.Min.x = I.Min.x;
            if (T.Min.y > I.Min.y) T.Min.y = I.Min.y;
            if (T.Min.z > I.Min.z) T.Min.z = I.Min.z;
            if (T.Max.x < I.Max.x) T.Max.x = I.Max.x;
            if (T.Max.y < I.Max.y) T.Max.y = I.Max.y;
            if (T.Max.z < I.Max.z) T.Max.z = I.Max.z;
        }
        T.Center = V3(T.Min.x * 0.5f + T.Max.x * 0.5f, T.Min.y * 0.5f + T.Max.y * 0.5f,
                      T.Min.z * 0.5f + T.Max.z * 0.5f);
        E.AABB = T;
    }

    uint32_t EntityCount = (uint32_t)Ents.size();
    if (EntityCount == 0) return false;
    St.Entities.reset(new az_entity[EntityCount]);
    for (uint32_t i = 0; i < EntityCount; i++) {
        St.Entities[i] = Ents[i];
        St.Entities[i].UniqueEntityID = i;
    }
    // Entity lights after the other lights, in importer order (src/azimuth_xml.cpp:3893-3913).
    for (size_t li = 0; li < EntityLightIdx.size(); li++) {
        az_light L;
        memset(&L, 0, sizeof(L));
        L.Entity = St.Entities[EntityLightIdx[li]];
        L.ID = (uint32_t)li;
        L.Type = AZ_Light_Entity;
        St.Lights.push_back(L);
    }

    Scene.Meshes = St.Meshes.empty() ? nullptr : St.Meshes.data();
    Scene.MeshCount = (uint32_t)St.Meshes.size();
    Scene.Materials = St.Materials.empty() ? nullptr : St.Materials.data();
    Scene.MaterialCount = (uint32_t)St.Materials.size();
    Scene.Lights = St.Lights.empty() ? nullptr : St.Lights.data();
    Scene.LightCount = (uint32_t)St.Lights.size();
    Scene.Textures = St.Textures.empty() ? nullptr : St.Textures.data();
    Scene.TextureCount = (uint32_t)St.Textures.size();
    if (soup_only) {
        uint32_t n = 0;
        St.RootEntities.reset(new az_entity[EntityCount]);
        for (uint32_t i = 0; i < EntityCount; i++)
            if (St.Entities[i].Type != AZ_Entity_MeshInstance) St.RootEntities[n++] = St.Entities[i];
        Scene.BVHRoot = nullptr;
        return n == 0 || ConstructBVH(&Scene.BVHRoot, St.RootEntities.get(), n, 0, St.Pool);
    }
    return ConstructBVH(&Scene.BVHRoot, St.Entities.get(), EntityCount, 0, St.Pool);
}

}  // namespace az
