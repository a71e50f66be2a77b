// Flattening azimuth's scene pointer graph into the device layout of
// az_scene_dev.cuh, upload, and BVH construction.
//
// The entity tree under scene.BVHRoot (src/azimuth_bvh.cpp) is only walked to
// find its leaves; the device BVHs are rebuilt on the GPU.  Mesh instances
// (src/azimuth_main.cpp:244-281) whose transformation, inverse and motion are
// bitwise identical are merged into one bottom-level BVH: every per-instance
// quantity azimuth computes (local ray, world t) is then the same for all of
// them, so only the choice between exactly tied hits can differ.
#include <algorithm>
#include <chrono>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <set>
#include <string>

#include "az_internal.h"
#include "az_scene_build.h"

namespace az {

GpuScene::~GpuScene() {
    for (auto &b : bufs)
        if (b.ptr) cudaFree(b.ptr);
    if (host_film_dev) cudaFree(host_film_dev);
}

void *GpuScene::Alloc(size_t bytes) {
    void *p = nullptr;
    if (bytes == 0) bytes = 16;
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    bufs.push_back(DevBuf{p, bytes});
    device_bytes += bytes;
    return p;
}

namespace {

using azd::f3;
using azd::m34;
using azd::mk;

m34 ToM34(const az_mat4 &m) {
    m34 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 4; j++) r.e[4 * i + j] = m.E[i][j];
    return r;
}

bool IsIdentity(const m34 &m) {
    static const float id[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
    return memcmp(m.e, id, sizeof(id)) == 0;
}

struct Box {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void grow(float x, float y, float z) {
        lo[0] = fminf(lo[0], x); lo[1] = fminf(lo[1], y); lo[2] = fminf(lo[2], z);
        hi[0] = fmaxf(hi[0], x); hi[1] = fmaxf(hi[1], y); hi[2] = fmaxf(hi[2], z);
    }
    void grow(const Box &b) {
        grow(b.lo[0], b.lo[1], b.lo[2]);
        grow(b.hi[0], b.hi[1], b.hi[2]);
    }
};

// World box of a local box under an affine transform and linear motion over
// the shutter [0,1] (the bound azimuth's importer uses, src/azimuth_xml.cpp:3791-3875).
Box XformBox(const Box &b, const m34 &m, const float motion[3]) {
    Box r;
    for (int c = 0; c < 8; c++) {
        f3 p = mk(c & 1 ? b.hi[0] : b.lo[0], c & 2 ? b.hi[1] : b.lo[1], c & 4 ? b.hi[2] : b.lo[2]);
        // evaluate in double and round outward so the box stays conservative
        double x = (double)m.e[0] * p.x + (double)m.e[1] * p.y + (double)m.e[2] * p.z + m.e[3];
        double y = (double)m.e[4] * p.x + (double)m.e[5] * p.y + (double)m.e[6] * p.z + m.e[7];
        double z = (double)m.e[8] * p.x + (double)m.e[9] * p.y + (double)m.e[10] * p.z + m.e[11];
        r.grow(nextafterf((float)x, -FLT_MAX), nextafterf((float)y, -FLT_MAX), nextafterf((float)z, -FLT_MAX));
        r.grow(nextafterf((float)x, FLT_MAX), nextafterf((float)y, FLT_MAX), nextafterf((float)z, FLT_MAX));
    }
    if (motion[0] != 0.0f || motion[1] != 0.0f || motion[2] != 0.0f) {
        Box m2 = r;
        for (int k = 0; k < 3; k++) {
            m2.lo[k] += motion[k];
            m2.hi[k] += motion[k];
        }
        r.grow(m2);
    }
    return r;
}

struct GroupKey {
    unsigned char bytes[2 * sizeof(m34) + 12 + 4];
    bool operator<(const GroupKey &o) const { return memcmp(bytes, o.bytes, sizeof(bytes)) < 0; }
};

struct HostGroup {
    azd::DevGroup g{};
    std::vector<azd::DevTriVerts> tris;   // exact vertices; the Cramer operands are made on the GPU
    std::vector<azd::DevTriAttr> attr;
    std::vector<uint32_t> soup_meshes;   // meshes of the soup whose triangles follow `tris` on the device
    std::vector<uint32_t> soup_extra;    // then further placements of soup meshes (Flattener::extra)
    uint32_t soup_tris = 0;
    Box local;
};

struct Flattener {
    const az_scene *s;
    std::vector<azd::DevEntity> ents;
    std::vector<Box> ent_box;            // world boxes of sphere entities
    std::vector<HostGroup> groups;
    std::map<GroupKey, uint32_t> group_of;
    int raw_group = -1;
    bool skip_meshes = false;            // mesh instances come from a soup instead
    const az_mesh_soup *soup = nullptr;
    std::set<uint32_t> soup_uids;        // UniqueEntityIDs of the soup meshes' own instances
    // A mesh instance under BVHRoot that is not a soup mesh's own instance (a
    // MeshInstance element of the scene file): soup mesh `mesh` placed again.
    struct Extra {
        uint32_t mesh, entity, group, out_base;
    };
    std::vector<Extra> extra;
    std::string err;

    // The group of an instance with these matrices and motion (one BLAS per
    // distinct transform).
    uint32_t GroupFor(const azd::DevEntity &d) {
        GroupKey key;
        memcpy(key.bytes, &d.inv, sizeof(m34));
        memcpy(key.bytes + sizeof(m34), &d.xf, sizeof(m34));
        memcpy(key.bytes + 2 * sizeof(m34), d.motion, 12);
        memset(key.bytes + 2 * sizeof(m34) + 12, 0, 4);
        auto it = group_of.find(key);
        if (it != group_of.end()) return it->second;
        const uint32_t gi = (uint32_t)groups.size();
        group_of.emplace(key, gi);
        groups.emplace_back();
        HostGroup &g = groups.back();
        g.g.inv = d.inv;
        g.g.xf = d.xf;
        memcpy(g.g.motion, d.motion, 12);
        g.g.identity = IsIdentity(d.inv) && IsIdentity(d.xf) && d.motion[0] == 0.0f && d.motion[1] == 0.0f &&
                       d.motion[2] == 0.0f;
        return gi;
    }

    azd::DevEntity BaseEntity(const az_entity *e) {
        azd::DevEntity d;
        memset(&d, 0, sizeof(d));
        d.inv = ToM34(e->InvTransformationMatrix);
        d.xf = ToM34(e->TransformationMatrix);
        d.motion[0] = e->MotionVector.x; d.motion[1] = e->MotionVector.y; d.motion[2] = e->MotionVector.z;
        d.radiance[0] = e->Radiance.x; d.radiance[1] = e->Radiance.y; d.radiance[2] = e->Radiance.z;
        d.is_emitter = e->IsEmitter ? 1u : 0u;
        d.texture_index = e->TextureIndex;
        d.material = e->MaterialIndex;
        d.uid = e->UniqueEntityID;
        return d;
    }

    bool AddTriangle(HostGroup &g, const az_entity *t, uint32_t ent) {
        azd::DevTriVerts tr;
        const az_vec3 &p0 = t->P0, &p1 = t->P1, &p2 = t->P2;
        tr.a = make_float4(p0.x, p0.y, p0.z, p1.x);
        tr.b = make_float4(p1.y, p1.z, p2.x, p2.y);
        tr.c = make_float4(p2.z, t->FaceNormal.x, t->FaceNormal.y, t->FaceNormal.z);
        g.tris.push_back(tr);
        azd::DevTriAttr a;
        memset(&a, 0, sizeof(a));
        a.n0[0] = t->N0.x; a.n0[1] = t->N0.y; a.n0[2] = t->N0.z;
        a.n1[0] = t->N1.x; a.n1[1] = t->N1.y; a.n1[2] = t->N1.z;
        a.n2[0] = t->N2.x; a.n2[1] = t->N2.y; a.n2[2] = t->N2.z;
        a.uv0[0] = t->UV0.x; a.uv0[1] = t->UV0.y;
        a.uv1[0] = t->UV1.x; a.uv1[1] = t->UV1.y;
        a.uv2[0] = t->UV2.x; a.uv2[1] = t->UV2.y;
        a.shading_mode = t->ShadingMode;
        a.texture_index = t->TextureIndex;
        a.face_id = t->ID;
        a.entity = ent;
        g.attr.push_back(a);
        g.local.grow(p0.x, p0.y, p0.z);
        g.local.grow(p1.x, p1.y, p1.z);
        g.local.grow(p2.x, p2.y, p2.z);
        return true;
    }

    // Depth-first walk of an entity tree to its leaves.
    template <typename F>
    bool Walk(const az_entity *root, F &&leaf, const char *what) {
        if (!root) {
            err = std::string("null entity in ") + what;
            return false;
        }
        std::vector<const az_entity *> st{root};
        size_t guard = 0;
        while (!st.empty()) {
            const az_entity *e = st.back();
            st.pop_back();
            if (++guard > (size_t)1 << 34) {
                err = std::string("entity tree too large in ") + what;
                return false;
            }
            if (e->Type == AZ_Entity_BVHNode) {
                if (!e->Left || !e->Right) {
                    err = std::string("BVH node without children in ") + what;
                    return false;
                }
                st.push_back(e->Right);
                st.push_back(e->Left);
            } else if (!leaf(e)) {
                return false;
            }
        }
        return true;
    }

    bool Run() {
        if (!s->BVHRoot && skip_meshes) return true;   // every entity is a mesh of the soup
        return Walk(s->BVHRoot, [&](const az_entity *e) -> bool {
            uint32_t idx = (uint32_t)ents.size();
            azd::DevEntity d = BaseEntity(e);
            switch (e->Type) {
                case AZ_Entity_Sphere: {
                    d.type = azd::ENT_SPHERE;
                    d.center[0] = e->Center.x; d.center[1] = e->Center.y; d.center[2] = e->Center.z;
                    d.radius = e->Radius;
                    Box local;
                    float r = fabsf(e->Radius);
                    local.grow(e->Center.x - r, e->Center.y - r, e->Center.z - r);
                    local.grow(e->Center.x + r, e->Center.y + r, e->Center.z + r);
                    ents.push_back(d);
                    ent_box.push_back(XformBox(local, d.xf, d.motion));
                    return true;
                }
                case AZ_Entity_Triangle: {
                    // top-level triangle: tested with the world ray as is
                    d.type = azd::ENT_TRIANGLE;
                    if (raw_group < 0) {
                        raw_group = (int)groups.size();
                        groups.emplace_back();
                        HostGroup &g = groups.back();
                        g.g.inv = ToM34(az_mat4{{{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}}});
                        g.g.xf = g.g.inv;
                        g.g.raw = 1;
                        g.g.identity = 1;
                    }
                    d.group = (uint32_t)raw_group;
                    ents.push_back(d);
                    ent_box.push_back(Box());
                    return AddTriangle(groups[raw_group], e, idx);
                }
                case AZ_Entity_MeshInstance: {
                    if (skip_meshes) {
                        // a soup mesh's own instance is made from the soup; any other
                        // instance places soup mesh BaseMeshID again, with its own
                        // (already composed) transform, motion and material
                        if (soup_uids.count(e->UniqueEntityID)) return true;
                        if (e->BaseMeshID >= soup->mesh_count) {
                            err = "mesh instance's BaseMeshID is not a mesh of the soup";
                            return false;
                        }
                        d.type = azd::ENT_INSTANCE;
                        d.group = GroupFor(d);
                        extra.push_back(Extra{e->BaseMeshID, idx, d.group, 0});
                        ents.push_back(d);
                        ent_box.push_back(Box());
                        return true;
                    }
                    d.type = azd::ENT_INSTANCE;
                    if (!e->Mesh) {
                        err = "mesh instance without mesh";
                        return false;
                    }
                    const uint32_t gi = GroupFor(d);
                    d.group = gi;
                    ents.push_back(d);
                    ent_box.push_back(Box());
                    HostGroup *gp = &groups[gi];
                    return Walk(e->Mesh->BVH, [&](const az_entity *t) -> bool {
                        if (t->Type != AZ_Entity_Triangle) {
                            err = "mesh BVH leaf is not a triangle";
                            return false;
                        }
                        return AddTriangle(*gp, t, idx);
                    }, "mesh BVH");
                }
                default:
                    err = "unexpected entity type";
                    return false;
            }
        }, "scene BVH");
    }
};

// `valid_from`: the first host byte before `t` that may be read (the start of
// the array holding `t`), for the words a Perlin hash reads before the table.
azd::DevTexture ToDevTexture(const az_texture &t, std::vector<unsigned char> &texels, std::vector<uint32_t> &perms,
                             std::string &err, const void *valid_from = nullptr) {
    azd::DevTexture d;
    memset(&d, 0, sizeof(d));
    d.type = t.Type;
    d.format = t.PixelFormat;
    d.width = t.Width;
    d.height = t.Height;
    d.inv_width = t.InvWidth;
    d.inv_height = t.InvHeight;
    d.normalizer = t.Normalizer;
    d.bump_mul = t.BumpMapMultiplier;
    d.wrap = t.WrapMode;
    d.filter = t.Filter;
    d.blend = t.BlendMode;
    d.bump = t.BumpMap;
    if (t.Type == AZ_TextureType_PerlinNoise) {
        d.scaling = t.ScalingFactor;
        d.appearance = t.PerlinAppearance;
        // azimuth's PerlinHash indexes the table with the signed K % 256, so a
        // lattice point with K < 0 reads one of the 255 words in memory before
        // Perm (src/azimuth_texture.h:134-144): the texture's own ImagePath, then
        // the texture before it in the array.  The device table repeats those
        // words before the table itself; words outside the caller's array (the
        // reference reads whatever memory lies there) are 0.
        const unsigned char *perm0 = reinterpret_cast<const unsigned char *>(&t.Perm[0]);
        const unsigned char *lo = valid_from ? static_cast<const unsigned char *>(valid_from)
                                             : reinterpret_cast<const unsigned char *>(&t);
        for (int n = AZ_PERLIN_GRADIENT_SIZE; n >= 1; n--) {
            uint32_t w = 0;
            if (perm0 - lo >= (ptrdiff_t)(4 * n)) memcpy(&w, perm0 - 4 * n, 4);
            perms.push_back(w);
        }
        d.perm_offset = (uint32_t)perms.size();
        for (int i = 0; i < AZ_PERLIN_GRADIENT_SIZE; i++) perms.push_back(t.Perm[i]);
    } else if (t.Pixels && t.Width && t.Height) {
        size_t bpp = t.PixelFormat == AZ_PixelFormat_RGB_F32 ? 12 : 3;
        size_t bytes = (size_t)t.Width * t.Height * bpp;
        size_t off = (texels.size() + 15) & ~(size_t)15;
        texels.resize(off + bytes);
        memcpy(texels.data() + off, t.Pixels, bytes);
        d.texel_offset = off;
    } else {
        d.width = d.height = 0;  // not loaded: sampling it is an error caught at validation
    }
    (void)err;
    return d;
}

template <typename T>
T *Upload(GpuScene &G, const std::vector<T> &v, cudaStream_t st, int &rc) {
    T *p = (T *)G.Alloc(v.size() * sizeof(T));
    if (!p) {
        rc = SetError(AZ_ERR_OUT_OF_MEMORY, "device allocation failed");
        return nullptr;
    }
    if (!v.empty()) {
        cudaError_t e = cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) {
            rc = CudaError(e, "cudaMemcpyAsync(scene)");
            return nullptr;
        }
    }
    return p;
}

// A device buffer that lives only while the scene is built.
template <typename T>
struct TempBuf {
    T *p = nullptr;
    ~TempBuf() {
        if (p) cudaFree(p);
    }
    bool alloc(size_t n) { return cudaMalloc((void **)&p, (n ? n : 1) * sizeof(T)) != cudaSuccess; }   // true on failure
};

// The primitives in wide-leaf order: the exact vertices, and the operands of
// azimuth's Cramer test -- P0, E1 = P0 - P1 and E2 = P0 - P2 in float, the
// A..H of src/azimuth_main.cpp:154-164 (a float subtraction rounds the same
// on the host and here) -- plus the face normal.
__global__ void k_gather_tris(const azd::DevTriVerts *src, const azd::DevTriAttr *src_attr, const uint32_t *perm,
                              uint32_t n, azd::DevTri *dst, azd::DevTriVerts *dst_verts, azd::DevTriAttr *dst_attr) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t s = perm[i];
    const azd::DevTriVerts v = src[s];
    const float p0x = v.a.x, p0y = v.a.y, p0z = v.a.z, p1x = v.a.w, p1y = v.b.x, p1z = v.b.y;
    const float p2x = v.b.z, p2y = v.b.w, p2z = v.c.x;
    azd::DevTri t;
    t.a = make_float4(p0x, p0y, p0z, __fsub_rn(p0x, p1x));
    t.b = make_float4(__fsub_rn(p0y, p1y), __fsub_rn(p0z, p1z), __fsub_rn(p0x, p2x), __fsub_rn(p0y, p2y));
    t.c = make_float4(__fsub_rn(p0z, p2z), v.c.y, v.c.z, v.c.w);
    dst[i] = t;
    dst_verts[i] = v;
    dst_attr[i] = src_attr[s];
}

__global__ void k_gather_u32(const uint32_t *src, const uint32_t *perm, uint32_t n, uint32_t *dst) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[perm[i]];
}

__global__ void k_tri_boxes(const azd::DevTriVerts *t, uint32_t n, float4 *lo, float4 *hi) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const azd::DevTriVerts tr = t[i];
    const float p0x = tr.a.x, p0y = tr.a.y, p0z = tr.a.z, p1x = tr.a.w, p1y = tr.b.x, p1z = tr.b.y;
    const float p2x = tr.b.z, p2y = tr.b.w, p2z = tr.c.x;
    float4 l = make_float4(fminf(p0x, fminf(p1x, p2x)), fminf(p0y, fminf(p1y, p2y)), fminf(p0z, fminf(p1z, p2z)), 0);
    float4 h = make_float4(fmaxf(p0x, fmaxf(p1x, p2x)), fmaxf(p0y, fmaxf(p1y, p2y)), fmaxf(p0z, fmaxf(p1z, p2z)), 0);
    l.x = nextafterf(l.x, -FLT_MAX); l.y = nextafterf(l.y, -FLT_MAX); l.z = nextafterf(l.z, -FLT_MAX);
    h.x = nextafterf(h.x, FLT_MAX); h.y = nextafterf(h.y, FLT_MAX); h.z = nextafterf(h.z, FLT_MAX);
    lo[i] = l;
    hi[i] = h;
}

}  // namespace

int BuildGpuScene(const az_scene *scene, const az_render_opts *opts, cudaStream_t st, GpuScene **out,
                  const az_mesh_soup *soup) {
    if (!scene || !out) return SetError(AZ_ERR_INVALID_ARGUMENT, "null scene");
    *out = nullptr;
    const auto t_start = std::chrono::steady_clock::now();
    std::unique_ptr<GpuScene> G(new GpuScene());
    G->device = opts ? opts->device : 0;
    const uint32_t width = opts && opts->bvh_width ? opts->bvh_width : 8u;
    if (width != 2 && width != 4 && width != 8) return SetError(AZ_ERR_INVALID_ARGUMENT, "bvh_width must be 0, 2, 4 or 8");
    G->bvh_width = width;
    const uint32_t leaf = opts && opts->bvh_leaf ? opts->bvh_leaf : 2u;
    if (leaf < 1 || leaf > 3) return SetError(AZ_ERR_INVALID_ARGUMENT, "bvh_leaf must be 0..3");
    G->bvh_leaf = leaf;
    const uint32_t builder = opts && opts->bvh_builder ? opts->bvh_builder : (uint32_t)AZ_BVH_PLOC;
    if (builder != AZ_BVH_LBVH && builder != AZ_BVH_PLOC)
        return SetError(AZ_ERR_INVALID_ARGUMENT, "bvh_builder must be 0, AZ_BVH_LBVH or AZ_BVH_PLOC");
    G->bvh_builder = builder;
    auto build_binary = builder == AZ_BVH_PLOC ? BuildPLOC : BuildLBVH;
    Flattener F;
    F.s = scene;
    F.skip_meshes = soup != nullptr;
    F.soup = soup;
    if (soup && soup->mesh_count && !soup->meshes)
        return SetError(AZ_ERR_INVALID_ARGUMENT, "mesh soup array missing");
    for (uint32_t m = 0; soup && m < soup->mesh_count; m++) F.soup_uids.insert(soup->meshes[m].unique_entity_id);
    G->from_soup = soup != nullptr;
    if (!scene->BVHRoot && !soup) return SetError(AZ_ERR_INVALID_SCENE, "scene has no BVHRoot");
    if (!F.Run()) return SetError(AZ_ERR_INVALID_SCENE, F.err);

    // ---- meshes of a soup: post-processed on the GPU, one instance entity each ----
    std::unique_ptr<SoupWork, void (*)(SoupWork *)> soupw(nullptr, FreeSoupWork);
    std::vector<IngestMesh> ingest;
    std::vector<float> soup_area;
    if (soup) {
        const auto t_in = std::chrono::steady_clock::now();
        SoupWork *w = nullptr;
        int r = IngestSoup(soup, st, &w);
        if (r != AZ_OK) return r;
        soupw.reset(w);
        if ((r = SoupAreas(*w, soup_area)) != AZ_OK) return r;
        // per-mesh bounds for the top-level boxes of their groups
        std::vector<float> boxes;
        if ((r = SoupBoxes(*w, boxes, st)) != AZ_OK) return r;
        const az_mat4 I = Mat4Identity();
        ingest.resize(soup->mesh_count);
        for (uint32_t m = 0; m < soup->mesh_count; m++) {
            const az_mesh_desc &md = soup->meshes[m];
            if (md.face_count == 0) return SetError(AZ_ERR_INVALID_SCENE, "a mesh of the soup has no faces");
            // the instance entity the importer appends for the mesh
            // (src/azimuth_xml.cpp:3753-3766), transform composed as in :3785-3791
            azd::DevEntity d;
            memset(&d, 0, sizeof(d));
            d.type = azd::ENT_INSTANCE;
            d.xf = ToM34(Mat4Mul(I, md.transform));
            d.inv = ToM34(Mat4Mul(md.inv_transform, I));
            d.motion[0] = md.motion.x; d.motion[1] = md.motion.y; d.motion[2] = md.motion.z;
            d.radiance[0] = md.radiance.x; d.radiance[1] = md.radiance.y; d.radiance[2] = md.radiance.z;
            d.is_emitter = md.is_emitter ? 1u : 0u;
            d.texture_index = md.texture_index;
            d.material = md.material_index;
            d.uid = md.unique_entity_id;
            const uint32_t gi = F.GroupFor(d);
            d.group = gi;
            ingest[m].entity = (uint32_t)F.ents.size();
            ingest[m].shading_mode = md.shading_mode;
            ingest[m].texture_index = md.texture_index;
            F.ents.push_back(d);
            F.ent_box.push_back(Box());
            HostGroup &g = F.groups[gi];
            g.soup_meshes.push_back(m);
            g.soup_tris += md.face_count;
            g.local.grow(boxes[6 * m + 0], boxes[6 * m + 1], boxes[6 * m + 2]);
            g.local.grow(boxes[6 * m + 3], boxes[6 * m + 4], boxes[6 * m + 5]);
        }
        for (uint32_t x = 0; x < F.extra.size(); x++) {
            const uint32_t m = F.extra[x].mesh;
            HostGroup &g = F.groups[F.extra[x].group];
            g.soup_extra.push_back(x);
            g.soup_tris += soup->meshes[m].face_count;
            g.local.grow(boxes[6 * m + 0], boxes[6 * m + 1], boxes[6 * m + 2]);
            g.local.grow(boxes[6 * m + 3], boxes[6 * m + 4], boxes[6 * m + 5]);
        }
        G->ingest_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t_in).count();
    }

    // ---- materials, textures, lights, validation ----
    std::vector<azd::DevMaterial> mats(scene->MaterialCount);
    for (uint32_t i = 0; i < scene->MaterialCount; i++) {
        const az_material &m = scene->Materials[i];
        azd::DevMaterial &d = mats[i];
        memset(&d, 0, sizeof(d));
        memcpy(d.ambient, &m.AmbientReflectance, 12);
        memcpy(d.diffuse, &m.DiffuseReflectance, 12);
        memcpy(d.specular, &m.SpecularReflectance, 12);
        memcpy(d.mirror, &m.MirrorReflectance, 12);
        memcpy(d.transparency, &m.Transparency, 12);
        d.refraction_index = m.RefractionIndex;
        d.glossiness = m.Glossiness;
        d.exponent = m.BRDF.Exponent;
        d.brdf_refractive_index = m.BRDF.RefractiveIndex;
        d.brdf_type = m.BRDF.Type;
        uint32_t tb[3], mb[3];
        memcpy(tb, &m.Transparency, 12);
        memcpy(mb, &m.MirrorReflectance, 12);
        d.transparent = (tb[0] | tb[1] | tb[2]) != 0;
        d.is_mirror = (mb[0] | mb[1] | mb[2]) != 0;
        if (m.BRDF.Type > AZ_BRDF_TorranceSparrow) return SetError(AZ_ERR_INVALID_SCENE, "unknown BRDF type");
    }
    bool uses_perlin = false;
    std::vector<unsigned char> texels;
    std::vector<uint32_t> perms;
    std::vector<azd::DevTexture> texs;
    std::string err;
    for (uint32_t i = 0; i < scene->TextureCount; i++) {
        texs.push_back(ToDevTexture(scene->Textures[i], texels, perms, err, scene->Textures));
        uses_perlin |= scene->Textures[i].Type == AZ_TextureType_PerlinNoise;
    }
    uint32_t bg_idx = (uint32_t)texs.size();
    texs.push_back(ToDevTexture(scene->BackgroundTexture, texels, perms, err));
    uint32_t env_idx = (uint32_t)texs.size();
    texs.push_back(ToDevTexture(scene->EnvironmentMap, texels, perms, err));
    if (scene->UseBackgroundTexture) uses_perlin |= scene->BackgroundTexture.Type == AZ_TextureType_PerlinNoise;
    if (scene->UseEnvironmentMap) uses_perlin |= scene->EnvironmentMap.Type == AZ_TextureType_PerlinNoise;
    if (uses_perlin && (!opts || !opts->perlin_gradients))
        return SetError(AZ_ERR_INVALID_ARGUMENT, "a Perlin texture is used but opts.perlin_gradients is NULL");
    auto tex_ok = [&](uint32_t ti) {
        const azd::DevTexture &t = texs[ti];
        return t.type == AZ_TextureType_PerlinNoise || (t.width > 0 && t.height > 0);
    };
    for (const HostGroup &g : F.groups)
        for (const azd::DevTriAttr &a : g.attr)
            if (a.texture_index && (a.texture_index > scene->TextureCount || !tex_ok(a.texture_index - 1)))
                return SetError(AZ_ERR_INVALID_SCENE, "triangle texture index out of range or texture not loaded");
    for (const IngestMesh &m : ingest)
        if (m.texture_index && (m.texture_index > scene->TextureCount || !tex_ok(m.texture_index - 1)))
            return SetError(AZ_ERR_INVALID_SCENE, "mesh texture index out of range or texture not loaded");
    for (const azd::DevEntity &e : F.ents) {
        if (!e.is_emitter && e.material >= scene->MaterialCount)
            return SetError(AZ_ERR_INVALID_SCENE, "entity material index out of range");
        if (e.texture_index && (e.texture_index > scene->TextureCount || !tex_ok(e.texture_index - 1)))
            return SetError(AZ_ERR_INVALID_SCENE, "entity texture index out of range or texture not loaded");
    }
    if (scene->UseEnvironmentMap && !tex_ok(env_idx))
        return SetError(AZ_ERR_INVALID_SCENE, "environment map not loaded");
    if (scene->UseBackgroundTexture && !scene->UseEnvironmentMap && !tex_ok(bg_idx))
        return SetError(AZ_ERR_INVALID_SCENE, "background texture not loaded");

    std::vector<azd::DevLight> lights;
    std::vector<azd::DevLightTri> light_tris;
    uint32_t light_draws = 0;
    for (uint32_t i = 0; i < scene->LightCount; i++) {
        const az_light &L = scene->Lights[i];
        azd::DevLight d;
        memset(&d, 0, sizeof(d));
        d.type = L.Type;
        memcpy(d.position, &L.Position, 12);
        memcpy(d.intensity, &L.Intensity, 12);
        memcpy(d.edge0, &L.EdgeVectors[0], 12);
        memcpy(d.edge1, &L.EdgeVectors[1], 12);
        memcpy(d.normal, &L.Normal, 12);
        memcpy(d.spot_dir, &L.SpotDirection, 12);
        d.cos_half_coverage = L.CosHalfCoverage;
        d.cos_half_falloff = L.CosHalfFallOff;
        if (L.Type == AZ_Light_Area) light_draws += 2;
        if (L.Type == AZ_Light_Entity) {
            const az_entity &E = L.Entity;
            d.uid = E.UniqueEntityID;
            memcpy(d.motion, &E.MotionVector, 12);
            d.ent_index = 0xFFFFFFFFu;
            for (uint32_t k = 0; k < F.ents.size(); k++)
                if (F.ents[k].uid == E.UniqueEntityID) {
                    d.ent_index = k;
                    break;
                }
            memcpy(d.intensity, &E.Radiance, 12);
            d.inv = ToM34(E.InvTransformationMatrix);
            d.xf = ToM34(E.TransformationMatrix);
            d.identity = IsIdentity(d.inv) && IsIdentity(d.xf) && d.motion[0] == 0.0f && d.motion[1] == 0.0f &&
                         d.motion[2] == 0.0f;
            if (E.Type == AZ_Entity_Sphere) {
                d.entity_type = azd::ENT_SPHERE;
                memcpy(d.center, &E.Center, 12);
                d.radius = E.Radius;
                light_draws += 2;
            } else if (E.Type == AZ_Entity_MeshInstance && soup) {
                // the mesh's triangles and TotalArea from the GPU post-processing
                if (E.BaseMeshID >= soup->mesh_count)
                    return SetError(AZ_ERR_INVALID_SCENE, "entity light's BaseMeshID is not a mesh of the soup");
                const az_mesh_desc &md = soup->meshes[E.BaseMeshID];
                std::vector<az_triangle> tr(md.face_count);
                int r = SoupTriangles(*soupw, md.face_base, md.face_count, tr.data(), st);
                if (r != AZ_OK) return r;
                d.entity_type = azd::ENT_INSTANCE;
                d.tri_offset = (uint32_t)light_tris.size();
                d.tri_count = md.face_count;
                d.total_area = soup_area[E.BaseMeshID];
                for (const az_triangle &T : tr)
                    light_tris.push_back(azd::DevLightTri{make_float4(T.P0.x, T.P0.y, T.P0.z, T.N.x),
                                                          make_float4(T.P1.x, T.P1.y, T.P1.z, T.N.y),
                                                          make_float4(T.P2.x, T.P2.y, T.P2.z, T.N.z)});
                light_draws += 3;
            } else if (E.Type == AZ_Entity_MeshInstance && E.Mesh && E.Mesh->Triangles && E.Mesh->TriangleCount) {
                d.entity_type = azd::ENT_INSTANCE;
                d.tri_offset = (uint32_t)light_tris.size();
                d.tri_count = E.Mesh->TriangleCount;
                d.total_area = E.Mesh->TotalArea;
                for (uint32_t k = 0; k < E.Mesh->TriangleCount; k++) {
                    const az_triangle &T = E.Mesh->Triangles[k];
                    light_tris.push_back(azd::DevLightTri{make_float4(T.P0.x, T.P0.y, T.P0.z, T.N.x),
                                                          make_float4(T.P1.x, T.P1.y, T.P1.z, T.N.y),
                                                          make_float4(T.P2.x, T.P2.y, T.P2.z, T.N.z)});
                }
                light_draws += 3;
            } else {
                return SetError(AZ_ERR_INVALID_SCENE, "entity light is neither a sphere nor a mesh with triangles");
            }
        } else if (L.Type > AZ_Light_Entity) {
            return SetError(AZ_ERR_INVALID_SCENE, "unknown light type");
        }
        lights.push_back(d);
    }

    // ---- upload primitives, build BLAS per group and the TLAS ----
    int rc = AZ_OK;
    uint64_t total_tris = 0;
    for (auto &g : F.groups) total_tris += g.tris.size() + g.soup_tris;
    if (total_tris >= (1ull << 27)) return SetError(AZ_ERR_UNSUPPORTED, "more than 2^27 triangles");
    // per group: the flattened triangles, then those of its soup meshes
    uint32_t cursor = 0;
    for (auto &g : F.groups) {
        g.g.tri_begin = cursor;
        cursor += (uint32_t)g.tris.size();
        for (uint32_t m : g.soup_meshes) {
            ingest[m].out_base = cursor;
            cursor += soup->meshes[m].face_count;
        }
        for (uint32_t x : g.soup_extra) {
            F.extra[x].out_base = cursor;
            cursor += soup->meshes[F.extra[x].mesh].face_count;
        }
        g.g.tri_end = cursor;
    }
    // TLAS primitives: spheres and groups
    std::vector<uint32_t> tlas;
    std::vector<float4> tlo, thi;
    for (uint32_t i = 0; i < F.ents.size(); i++) {
        if (F.ents[i].type != azd::ENT_SPHERE) continue;
        const Box &b = F.ent_box[i];
        tlas.push_back(i);
        tlo.push_back(make_float4(b.lo[0], b.lo[1], b.lo[2], 0));
        thi.push_back(make_float4(b.hi[0], b.hi[1], b.hi[2], 0));
    }
    for (uint32_t gi = 0; gi < F.groups.size(); gi++) {
        HostGroup &g = F.groups[gi];
        if (g.g.tri_end == g.g.tri_begin) continue;
        Box wb = g.g.raw ? g.local : XformBox(g.local, g.g.xf, g.g.motion);
        tlas.push_back(AZD_TLAS_GROUP | gi);
        tlo.push_back(make_float4(wb.lo[0], wb.lo[1], wb.lo[2], 0));
        thi.push_back(make_float4(wb.hi[0], wb.hi[1], wb.hi[2], 0));
    }
    uint32_t node_total = 0;
    for (auto &g : F.groups) {
        uint32_t n = g.g.tri_end - g.g.tri_begin;
        node_total += n > 1 ? n - 1 : (n == 1 ? 1 : 0);
    }
    node_total += tlas.size() > 1 ? (uint32_t)tlas.size() - 1 : (uint32_t)tlas.size();

    G->flatten_ms =
        std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t_start).count() - G->ingest_ms;
    // Build-only buffers are freed when the build ends; the scene keeps the
    // sorted primitives, the wide nodes and the top-level primitive list.
    const size_t nmax = std::max((size_t)total_tris, tlas.size()) + 1;
    TempBuf<azd::DevTriVerts> d_tris_unsorted;
    TempBuf<azd::DevTriAttr> d_attr_unsorted;
    TempBuf<azd::BVHNode> d_nodes;
    TempBuf<uint2> d_range;
    TempBuf<float4> d_lo, d_hi;
    TempBuf<uint32_t> d_perm, d_comp, d_tlas_unsorted;
    TempBuf<azd::WideNode> d_wide_tmp;
    azd::DevTri *d_tris = (azd::DevTri *)G->Alloc(total_tris * sizeof(azd::DevTri));
    azd::DevTriVerts *d_verts = (azd::DevTriVerts *)G->Alloc(total_tris * sizeof(azd::DevTriVerts));
    azd::DevTriAttr *d_attr = (azd::DevTriAttr *)G->Alloc(total_tris * sizeof(azd::DevTriAttr));
    uint32_t *d_tlas = (uint32_t *)G->Alloc((tlas.size() + 1) * sizeof(uint32_t));
    if (!d_tris || !d_verts || !d_attr || !d_tlas || d_tris_unsorted.alloc(total_tris) ||
        d_attr_unsorted.alloc(total_tris) || d_nodes.alloc(node_total) || d_range.alloc(node_total) ||
        d_lo.alloc(nmax) || d_hi.alloc(nmax) || d_perm.alloc(nmax) || d_comp.alloc(nmax) ||
        d_tlas_unsorted.alloc(tlas.size() + 1) || d_wide_tmp.alloc(node_total))
        return SetError(AZ_ERR_OUT_OF_MEMORY, "device allocation failed");
    const auto t_up0 = std::chrono::steady_clock::now();
    for (auto &g : F.groups) {
        if (g.tris.empty()) continue;
        AZ_CUDA_TRY(cudaMemcpyAsync(d_tris_unsorted.p + g.g.tri_begin, g.tris.data(),
                                    g.tris.size() * sizeof(azd::DevTriVerts), cudaMemcpyHostToDevice, st));
        AZ_CUDA_TRY(cudaMemcpyAsync(d_attr_unsorted.p + g.g.tri_begin, g.attr.data(),
                                    g.attr.size() * sizeof(azd::DevTriAttr), cudaMemcpyHostToDevice, st));
    }
    if (soupw) {
        int r = SoupEmitScene(*soupw, ingest, d_tris_unsorted.p, d_attr_unsorted.p, st);
        if (r != AZ_OK) return r;
        std::vector<IngestCopy> copies;
        for (const auto &x : F.extra)
            copies.push_back(IngestCopy{ingest[x.mesh].out_base, x.out_base, soup->meshes[x.mesh].face_count, x.entity});
        if ((r = SoupCopyPlacements(copies, d_tris_unsorted.p, d_attr_unsorted.p, st)) != AZ_OK) return r;
        soupw.reset();   // its device arrays are no longer needed
    }
    if (!tlas.empty())
        AZ_CUDA_TRY(cudaMemcpyAsync(d_tlas_unsorted.p, tlas.data(), tlas.size() * sizeof(uint32_t),
                                    cudaMemcpyHostToDevice, st));
    AZ_CUDA_TRY(cudaStreamSynchronize(st));
    for (auto &g : F.groups) {
        std::vector<azd::DevTriVerts>().swap(g.tris);
        std::vector<azd::DevTriAttr>().swap(g.attr);
    }
    const auto t_up1 = std::chrono::steady_clock::now();
    G->upload_ms += std::chrono::duration<float, std::milli>(t_up1 - t_up0).count();
    // Per hierarchy on the GPU: LBVH, collapse to wide nodes, then the
    // primitives gathered once into wide-leaf order.
    uint32_t wide_count = 0, wide_depth = 0, node_base = 0;
    const int B = 256;
    for (auto &g : F.groups) {
        uint32_t n = g.g.tri_end - g.g.tri_begin;
        if (n == 0) {
            g.g.root = 0xFFFFFFFFu;
            continue;
        }
        k_tri_boxes<<<(n + B - 1) / B, B, 0, st>>>(d_tris_unsorted.p + g.g.tri_begin, n, d_lo.p, d_hi.p);
        AZ_CUDA_TRY(cudaGetLastError());
        uint32_t root, wroot, depth = 0;
        rc = build_binary(d_lo.p, d_hi.p, n, d_nodes.p, d_range.p, node_base, g.g.tri_begin, d_perm.p, st, &root);
        if (rc != AZ_OK) return rc;
        rc = CollapseToWide(d_nodes.p, d_range.p, root, n, g.g.tri_begin, d_perm.p, leaf, width, d_wide_tmp.p,
                            node_total, &wide_count, d_comp.p, st, &wroot, &depth);
        if (rc != AZ_OK) return rc;
        wide_depth = std::max(wide_depth, depth);
        g.g.root = wroot;
        node_base += n > 1 ? n - 1 : 1;
        k_gather_tris<<<(n + B - 1) / B, B, 0, st>>>(d_tris_unsorted.p + g.g.tri_begin,
                                                     d_attr_unsorted.p + g.g.tri_begin, d_comp.p, n,
                                                     d_tris + g.g.tri_begin, d_verts + g.g.tri_begin,
                                                     d_attr + g.g.tri_begin);
        AZ_CUDA_TRY(cudaGetLastError());
        G->hierarchies++;
    }
    uint32_t tlas_root = 0xFFFFFFFFu;
    if (!tlas.empty()) {
        uint32_t n = (uint32_t)tlas.size();
        AZ_CUDA_TRY(cudaMemcpyAsync(d_lo.p, tlo.data(), tlo.size() * sizeof(float4), cudaMemcpyHostToDevice, st));
        AZ_CUDA_TRY(cudaMemcpyAsync(d_hi.p, thi.data(), thi.size() * sizeof(float4), cudaMemcpyHostToDevice, st));
        uint32_t root, depth = 0;
        rc = build_binary(d_lo.p, d_hi.p, n, d_nodes.p, d_range.p, node_base, 0, d_perm.p, st, &root);
        if (rc != AZ_OK) return rc;
        // top-level leaves hold one primitive each (a group is entered from its leaf)
        rc = CollapseToWide(d_nodes.p, d_range.p, root, n, 0, d_perm.p, 1, width, d_wide_tmp.p, node_total,
                            &wide_count, d_comp.p, st, &tlas_root, &depth);
        if (rc != AZ_OK) return rc;
        wide_depth = std::max(wide_depth, depth);
        node_base += n > 1 ? n - 1 : 1;
        k_gather_u32<<<(n + B - 1) / B, B, 0, st>>>(d_tlas_unsorted.p, d_comp.p, n, d_tlas);
        AZ_CUDA_TRY(cudaGetLastError());
        G->hierarchies++;
    }
    azd::WideNode *d_wide = (azd::WideNode *)G->Alloc(((size_t)wide_count + 1) * sizeof(azd::WideNode));
    if (!d_wide) return SetError(AZ_ERR_OUT_OF_MEMORY, "device allocation failed");
    if (wide_count)
        AZ_CUDA_TRY(cudaMemcpyAsync(d_wide, d_wide_tmp.p, (size_t)wide_count * sizeof(azd::WideNode),
                                    cudaMemcpyDeviceToDevice, st));
    AZ_CUDA_TRY(cudaStreamSynchronize(st));
    G->bvh_ms += std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t_up1).count();

    std::vector<azd::DevGroup> dgroups;
    for (auto &g : F.groups) dgroups.push_back(g.g);
    std::vector<float> grad(3 * AZ_PERLIN_GRADIENT_SIZE, 0.0f);
    if (opts && opts->perlin_gradients) memcpy(grad.data(), opts->perlin_gradients, grad.size() * sizeof(float));
    if (perms.empty()) perms.push_back(0);
    if (texels.empty()) texels.resize(16);

    azd::DevScene &D = G->dev;
    D.tris = d_tris;
    D.tri_verts = d_verts;
    D.tri_attr = d_attr;
    D.ents = Upload(*G, F.ents, st, rc);
    D.groups = Upload(*G, dgroups, st, rc);
    D.tlas_prims = d_tlas;
    D.nodes = nullptr;
    D.wnodes = d_wide;
    D.materials = Upload(*G, mats, st, rc);
    D.textures = Upload(*G, texs, st, rc);
    D.lights = Upload(*G, lights, st, rc);
    D.light_tris = Upload(*G, light_tris, st, rc);
    D.perlin_perm = Upload(*G, perms, st, rc);
    D.perlin_grad = Upload(*G, grad, st, rc);
    D.texels = Upload(*G, texels, st, rc);
    if (rc != AZ_OK) return rc;
    D.tlas_root = tlas_root;
    {
        Box sb;
        for (size_t k = 0; k < tlo.size(); k++) {
            sb.grow(tlo[k].x, tlo[k].y, tlo[k].z);
            sb.grow(thi[k].x, thi[k].y, thi[k].z);
        }
        for (int a = 0; a < 3; a++) {
            const float ext = sb.hi[a] > sb.lo[a] ? sb.hi[a] - sb.lo[a] : 1.0f;
            D.box_lo[a] = tlo.empty() ? 0.0f : sb.lo[a];
            D.box_scale[a] = 1.0f / ext;
        }
    }
    D.tlas_single_group = tlas.size() == 1 && (tlas[0] & AZD_TLAS_GROUP) ? (tlas[0] & ~AZD_TLAS_GROUP) : 0xFFFFFFFFu;
    D.ent_count = (uint32_t)F.ents.size();
    D.group_count = (uint32_t)dgroups.size();
    D.material_count = scene->MaterialCount;
    D.texture_count = scene->TextureCount;
    D.light_count = (uint32_t)lights.size();
    D.bg_texture = bg_idx;
    D.env_texture = env_idx;
    // luminance CDF of a 2D environment map for AZ_FLAG_ENV_IMPORTANCE: per
    // texel the largest luminance of its 3 x 3 neighbourhood (the lookup's
    // nearest texel is round(u (W - 1)), up to one texel off this CDF's
    // floor(u W) cells, and a bilinear lookup blends neighbours), times
    // sin(theta) of its row centre, plus a small floor
    D.env_rows = D.env_cols = nullptr;
    D.env_cdf_w = D.env_cdf_h = 0;
    {
        const az_texture &E = scene->EnvironmentMap;
        if (scene->UseEnvironmentMap && E.Type != AZ_TextureType_PerlinNoise && E.Pixels && E.Width && E.Height) {
            const uint32_t W = E.Width, H = E.Height;
            std::vector<double> lum((size_t)W * H);
            double total_l = 0.0;
            for (uint32_t y = 0; y < H; y++)
                for (uint32_t x = 0; x < W; x++) {
                    double rgb[3];
                    const size_t i = (size_t)y * W + x;
                    for (int c = 0; c < 3; c++)
                        rgb[c] = E.PixelFormat == AZ_PixelFormat_RGB_F32 ? (double)((const float *)E.Pixels)[3 * i + c]
                                                                          : (double)((const uint8_t *)E.Pixels)[3 * i + c];
                    const double l = std::max(0.0, 0.2126 * rgb[0] + 0.7152 * rgb[1] + 0.0722 * rgb[2]);
                    lum[i] = l;
                    total_l += l;
                }
            const double floor_l = 1e-3 * total_l / ((double)W * H) + 1e-30;
            {
                std::vector<double> dil(lum.size());
                for (uint32_t y = 0; y < H; y++)
                    for (uint32_t x = 0; x < W; x++) {
                        double m = 0.0;
                        for (int dy = -1; dy <= 1; dy++) {
                            const int yy = std::min<int>((int)H - 1, std::max<int>(0, (int)y + dy));
                            for (int dx = -1; dx <= 1; dx++) {
                                const int xx = ((int)x + dx + (int)W) % (int)W;
                                m = std::max(m, lum[(size_t)yy * W + xx]);
                            }
                        }
                        dil[(size_t)y * W + x] = m;
                    }
                lum.swap(dil);
            }
            std::vector<float> rows(H + 1), cols((size_t)H * (W + 1));
            std::vector<double> row_w(H);
            double tot = 0.0;
            for (uint32_t y = 0; y < H; y++) {
                const double st = std::sin(3.14159265358979323846 * (y + 0.5) / H);
                double acc = 0.0;
                for (uint32_t x = 0; x < W; x++) acc += lum[(size_t)y * W + x] + floor_l;
                double run = 0.0;
                cols[(size_t)y * (W + 1)] = 0.0f;
                for (uint32_t x = 0; x < W; x++) {
                    run += lum[(size_t)y * W + x] + floor_l;
                    cols[(size_t)y * (W + 1) + x + 1] = (float)(run / acc);
                }
                cols[(size_t)y * (W + 1) + W] = 1.0f;
                row_w[y] = acc * st;
                tot += row_w[y];
            }
            double run = 0.0;
            rows[0] = 0.0f;
            for (uint32_t y = 0; y < H; y++) {
                run += row_w[y];
                rows[y + 1] = (float)(run / tot);
            }
            rows[H] = 1.0f;
            int urc = AZ_OK;
            D.env_rows = Upload(*G, rows, st, urc);
            if (urc == AZ_OK) D.env_cols = Upload(*G, cols, st, urc);
            if (urc != AZ_OK) return urc;
            D.env_cdf_w = W;
            D.env_cdf_h = H;
        }
    }
    memcpy(D.ambient, &scene->AmbientLight, 12);
    memcpy(D.background, &scene->BackgroundColor, 12);
    D.use_bg_texture = scene->UseBackgroundTexture ? 1u : 0u;
    D.use_env_map = scene->UseEnvironmentMap ? 1u : 0u;
    D.max_depth = scene->MaxRecursionDepth;
    D.path_trace = scene->PathTrace ? 1u : 0u;
    D.importance_sampling = scene->ImportanceSampling ? 1u : 0u;
    D.light_draws = light_draws;
    D.features = 0;
    if (scene->TextureCount > 0) D.features |= azd::FEAT_TEXTURES;
    if (scene->UseEnvironmentMap) D.features |= azd::FEAT_ENV;
    for (const azd::DevMaterial &m : mats)
        if (m.transparent || m.is_mirror) D.features |= azd::FEAT_SPECIAL;
    D.full_light_queries = 0;
    D.top_spheres = (uint32_t)(tlas.size() - dgroups.size());
    for (const azd::DevLight &l : lights) {
        if (l.type != azd::LIGHT_ENTITY) D.features |= azd::FEAT_ANALYTIC_LIGHTS;
        else if (azd::entity_light_needs_full_query(l)) D.full_light_queries = 1;
    }
    AZ_CUDA_TRY(cudaStreamSynchronize(st));
    G->triangle_count = total_tris;
    G->sphere_count = tlas.size() - dgroups.size();
    G->node_count = wide_count;
    G->max_bvh_depth = wide_depth;
    G->total_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    *out = G.release();
    return AZ_OK;
}

}  // namespace az
