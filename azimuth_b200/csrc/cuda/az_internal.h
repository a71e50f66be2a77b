// Internal host-side declarations shared by the CUDA translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "az_render.h"
#include "az_scene_dev.cuh"
#include "azimuth_gpu.h"

namespace az {

// Status plus message; stored per thread for az_gpu_last_error().
int SetError(int code, const std::string &msg);
int CudaError(cudaError_t e, const char *what);

#define AZ_CUDA_TRY(expr)                                       \
    do {                                                        \
        cudaError_t az_e_ = (expr);                             \
        if (az_e_ != cudaSuccess) return ::az::CudaError(az_e_, #expr); \
    } while (0)

// A device allocation owned by a GpuScene.
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
};

struct GpuScene {
    int device = 0;
    azd::DevScene dev{};
    std::vector<DevBuf> bufs;
    uint64_t triangle_count = 0;
    uint64_t sphere_count = 0;
    uint64_t node_count = 0;
    uint32_t max_bvh_depth = 0;
    uint32_t hierarchies = 0;    // bottom-level hierarchies plus the top level
    float flatten_ms = 0.0f;     // host: azimuth's structs walked into device records
    float upload_ms = 0.0f;      // host-to-device copies of the primitives
    float bvh_ms = 0.0f;         // GPU: LBVH builds, wide collapse, primitive gather
    float total_ms = 0.0f;       // the whole az_gpu_scene_create
    float ingest_ms = 0.0f;      // GPU post-processing of a mesh soup (az_gpu_scene_create_from_meshes)
    uint32_t bvh_width = 8;      // children per wide node (2, 4 or 8)
    uint32_t bvh_leaf = 2;       // triangles per bottom-level leaf at most
    uint32_t bvh_builder = AZ_BVH_PLOC;   // binary hierarchy under the wide collapse
    bool from_soup = false;      // meshes came from az_gpu_scene_create_from_meshes
    size_t device_bytes = 0;
    WaveBuffers waves;           // reused across render calls on this scene
    uint32_t variant = 7;        // traversal launch configuration, 0-based (128 threads, 8 blocks/SM,
                                 // persistent fetching; az_gpu_autotune picks per scene)
    uint32_t shadow_variant = 0xFFFFFFFFu;   // the shadow queries' own configuration (az_gpu_autotune;
                                             // 0xFFFFFFFF: `variant`)
    uint32_t order = 0;          // queue ordering (kOrderShadow | kOrderExtend); az_gpu_autotune picks
    az_pixel *host_film_dev = nullptr;   // device film of az_gpu_render_host
    size_t host_film_bytes = 0;
    ~GpuScene();
    void *Alloc(size_t bytes);   // nullptr on failure
};

// Builds the device scene from azimuth's structs (az_scene_upload.cu); with
// `soup` the meshes come from it instead (post-processed on the GPU).
int BuildGpuScene(const az_scene *scene, const az_render_opts *opts, cudaStream_t stream, GpuScene **out,
                  const az_mesh_soup *soup = nullptr);

// The importer's mesh post-processing on the GPU (az_mesh_ingest.cu).
struct SoupWork;
struct IngestMesh {
    uint32_t out_base;           // first slot of the mesh's triangles in the device primitive arrays
    uint32_t entity;             // dense index of its instance entity
    uint32_t shading_mode, texture_index;
};
int IngestSoup(const az_mesh_soup *soup, cudaStream_t st, SoupWork **out);
void FreeSoupWork(SoupWork *w);
int SoupAreas(const SoupWork &w, std::vector<float> &areas);
// Per mesh (soup order): lo.xyz, hi.xyz of its faces' vertices.
int SoupBoxes(const SoupWork &w, std::vector<float> &boxes, cudaStream_t st);
int SoupRecords(const SoupWork &w, az_triangle *tris, az_face_attr *attrs, az_vec3 *vertex_normals, cudaStream_t st);
int SoupTriangles(const SoupWork &w, uint32_t face_base, uint32_t count, az_triangle *tris, cudaStream_t st);
int SoupEmitScene(const SoupWork &w, const std::vector<IngestMesh> &meshes, azd::DevTriVerts *d_tris,
                  azd::DevTriAttr *d_attr, cudaStream_t st);
// A further placement of a soup mesh (a mesh instance besides the importer's
// own one): `count` primitives copied from slot `src` to slot `dst` of the
// device primitive arrays, with their instance entity set to `entity`.
struct IngestCopy {
    uint32_t src, dst, count, entity;
};
int SoupCopyPlacements(const std::vector<IngestCopy> &copies, azd::DevTriVerts *d_tris, azd::DevTriAttr *d_attr,
                       cudaStream_t st);

// LBVH over `n` boxes (device arrays lo/hi of float4).  Writes nodes into
// `nodes` starting at `node_base` (n-1 nodes, or 1 for n == 1), each inner
// node's primitive range (first sorted position + leaf_base, count) into
// `range` at the same index, and the sorted primitive order into `perm`.  Leaf
// child references are `leaf_base + sorted position`.  Returns the root node
// index.
int BuildLBVH(const float4 *d_lo, const float4 *d_hi, uint32_t n, azd::BVHNode *d_nodes, uint2 *d_range,
              uint32_t node_base, uint32_t leaf_base, uint32_t *d_perm, cudaStream_t stream, uint32_t *root_out);
// The same outputs from PLOC clustering (az_bvh_build.cu); primitive order is
// then the tree's depth-first leaf order, so every node's range is contiguous.
int BuildPLOC(const float4 *d_lo, const float4 *d_hi, uint32_t n, azd::BVHNode *d_nodes, uint2 *d_range,
              uint32_t node_base, uint32_t leaf_base, uint32_t *d_perm, cudaStream_t stream, uint32_t *root_out);

// Collapse, on the GPU, of the binary LBVH of `n` primitives rooted at
// `bin_root` (device nodes and ranges as BuildLBVH writes them) into wide nodes
// of at most `width` (2, 4 or 8) children and leaves of at most `max_leaf`
// primitives, written to d_wide from index *wide_count on (at most wide_cap
// nodes in all; *wide_count is advanced).  Leaf primitives are numbered
// leaf_base + [0, n): d_out_perm[j] receives the unsorted local index of the
// primitive placed at j (d_sorted_perm maps sorted positions to those).
int CollapseToWide(const azd::BVHNode *d_nodes, const uint2 *d_range, uint32_t bin_root, uint32_t n,
                   uint32_t leaf_base, const uint32_t *d_sorted_perm, uint32_t max_leaf, uint32_t width,
                   azd::WideNode *d_wide, uint32_t wide_cap, uint32_t *wide_count, uint32_t *d_out_perm,
                   cudaStream_t st, uint32_t *root_out, uint32_t *depth_out);

int SetupCamera(const az_camera *c, az_scissor sc, int32_t filter, uint32_t cull, const az_epsilon_values *eps,
                uint64_t seed, CameraParams &cam);
// Path guide (az_guide.cu): network state and the hooks of a guided render.
struct GuideState;
int CreateGuide(const GpuScene &G, const az_guide_config *cfg, GuideState **out);
void DestroyGuide(GuideState *g);
// Proposal and training-record buffers (in W) of a wave whose queues hold at
// most `cap_q` entries and `levels` tree levels; sets the guide fields of Q and
// lowers Q.cap_q to the proposals' capacity.
int GuidePrepareWave(GuideState &g, WaveBuffers &W, WaveQueues &Q, uint32_t cap_q, uint32_t levels, cudaStream_t st);
// Proposals for the extension queue of `level` (between extend and shade).
int GuideInfer(GuideState &g, const GpuScene &G, const WaveQueues &Q, uint32_t level, cudaStream_t st);
// Training targets of the finished wave and one Adam step.
int GuideTrainWave(GuideState &g, const WaveQueues &Q, cudaStream_t st);
GuideState *GuideOf(az_guide *g);
// AZ_ERR_CUDA if a tensor-core wait of the proposal kernel gave up since the last check (the flag is cleared).
int GuideCheck(GuideState &g, cudaStream_t st);
// Serialises the renders that use one guide (its proposal and record buffers).
std::mutex &GuideLock(GuideState &g);

// `guide` (may be null) steers the scattering direction; `train` also
// updates the network after every wave.
// `wave_buffers`: the queues to use (null: the scene's own); concurrent
// renders of one scene need their own.
// `sample_out`: instead of splatting into `film` (which may then be null),
// write every camera sample's radiance sum to sample_out[s], s the sample's
// index in the scissor (sample number * scissor pixels + pixel).
int Render(GpuScene &G, az_pixel *film, const az_camera *camera, const az_epsilon_values *eps, az_scissor sc,
           int32_t filter, uint32_t cull, const az_render_opts *opts, cudaStream_t st, az_render_stats *stats,
           GuideState *guide = nullptr, bool train = false, WaveBuffers *wave_buffers = nullptr,
           float4 *sample_out = nullptr);
int Autotune(GpuScene &G, const az_camera *camera, const az_epsilon_values *eps, az_scissor sc, int32_t filter,
             uint32_t cull, const az_render_opts *opts, cudaStream_t st, uint32_t *best_out, float *ms_out);
// One render job of a tile render (az_gpu_render_tiles).
struct TileJob {
    GpuScene *scene = nullptr;   // the job's scene (null: RenderTiles' own); all on one device
    az_pixel *film;              // device film of the job's camera
    const az_camera *camera;
    const az_epsilon_values *eps;
    az_scissor scissor;
    int32_t filter;
    uint32_t cull;
    uint64_t seed;
    uint64_t samples = 0;        // written: the job's camera samples
    float done_ms = 0.0f;        // written: device time from the call's start to its last wave's end
};
// Renders jobs together: their samples are cut into tiles, and every wave
// takes the next tiles of all jobs from a device work queue, so one chain of
// launches serves every job.  Jobs may render different scenes (up to 256,
// one device): every queue entry then carries its scene's index and each
// kernel reads that scene's record.  The jobs must share epsilons and
// culling.  `origin`, when given, is an event recorded earlier on `st` from
// which the jobs' completion times are measured (default: the call's start).
int RenderTiles(GpuScene &G, std::vector<TileJob> &jobs, const az_render_opts *opts, cudaStream_t st,
                az_render_stats *stats, cudaEvent_t origin = nullptr);
// OutputPixelsToFile's post-processing of a device film (az_post.cu).
int PostProcess(const az_pixel *film, uint32_t w, uint32_t h, const az_tonemap *tm, float inv_gamma, uint32_t srgb,
                uint32_t linear, float *rgb_out, uint8_t *rgb8_out, cudaStream_t st);
int ClosestHit(GpuScene &G, const az_ray3 *rays, uint32_t n, int32_t cull, float eps, uint32_t *out_hit,
               uint32_t *out_uid, uint32_t *out_face, float *out_t, cudaStream_t st, bool watertight = false);

}  // namespace az

// The opaque handle of include/azimuth_gpu.h.
struct az_gpu_scene {
    az::GpuScene *impl;
};
