// Wavefront render state shared between the render driver and the C-ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "az_device_math.cuh"
#include "az_guide.cuh"

namespace azd {
struct DevScene;
}

namespace az {

constexpr uint32_t AZ_MAX_LEVELS = 64;                   // tree levels kept in the counters
constexpr uint32_t AZ_COUNT_SHADOW = AZ_MAX_LEVELS;      // shadow-queue sizes per level
constexpr uint32_t AZ_COUNT_OVERFLOW = 2 * AZ_MAX_LEVELS;
constexpr uint32_t AZ_COUNT_NODES = 2 * AZ_MAX_LEVELS + 2;  // node visits, primitive visits
constexpr uint32_t AZ_COUNT_ERROR = 2 * AZ_MAX_LEVELS + 4;  // traversal step limit reached
constexpr uint32_t AZ_COUNT_SNODES = 2 * AZ_MAX_LEVELS + 5; // visibility queries: node visits, primitive visits
constexpr uint32_t AZ_COUNT_FETCH = 2 * AZ_MAX_LEVELS + 8;  // per level: extend, then shadow work counters
constexpr uint32_t AZ_COUNT_TOTAL = 4 * AZ_MAX_LEVELS + 8;

// Camera and film parameters of one render call (ProduceImageInLinearSpace's
// locals, src/azimuth_main.cpp:1265-1347).
struct CameraParams {
    azd::f3 base, pos, axx, axy, stepx, stepy;
    float aperture, inv_sqrt;
    uint32_t sqrt_spp, width, height;
    uint32_t r0, c0, wsc, hsc;     // scissor origin and size
    uint64_t npix;
    int32_t filter;
    float g_norm, g_neg;
    int32_t gk;
    uint64_t seed;
    float eps_isect, eps_shadow;
    uint32_t cull;
    uint32_t count_traversal;
    uint32_t variant;              // launch configuration of the extension queries
    uint32_t shadow_variant;       // launch configuration of the shadow queries
    uint32_t env_importance;       // AZ_FLAG_ENV_IMPORTANCE
    uint32_t order;                // kOrderShadow | kOrderExtend: queues visited in sorted order
    uint32_t serial_levels;        // AZ_FLAG_SERIAL_LEVELS: no overlap of a level's visibility queries
                                   // with the next level's closest-hit queries
    uint32_t watertight;           // AZ_FLAG_WATERTIGHT: triangles by the watertight test
    uint32_t scene;                // a tile wave of several scenes: the job's index in WaveQueues.scenes
    float4 *sample_out;            // per-sample radiance output (az_gpu_render_samples): sample s of the
                                   // scissor at [s] instead of a splat into the film; null: splat
};

constexpr uint32_t kOrderShadow = 1, kOrderExtend = 2;

// Device queues of one wave of camera samples (structure of arrays).
struct WaveQueues {
    float4 *o[2], *d[2], *tp[2], *att[2];   // path nodes, ping-pong by level parity
    uint32_t *digits[2];
    uint4 *hit;
    uint32_t cap_q;
    float4 *so, *sd, *sc;                   // shadow queue
    uint32_t *smeta;
    uint32_t cap_s;
    // visiting orders of the extension and shadow queues (null: queue order);
    // entry k of the stage's work is queue entry order[k]
    const uint32_t *eorder, *sorder;
    float4 *accum;                          // per-sample radiance sums
    uint32_t *counts;                       // see AZ_COUNT_*
    // [first sample, sample count, seed] of the current wave when set: a
    // captured CUDA graph replays the same launches for every wave and reads
    // them here; null: the kernels' arguments and cam.seed
    const uint64_t *wave;
    // path guiding (null when rendering without a guide)
    azd::GuideLobes *lobes;                 // per extension-queue entry of the current level
    azd::GuideRecord *rec;                  // [level][n_rec] training vertices
    uint32_t n_rec, rec_levels;
    float guide_alpha_max;                  // cap on the learned selection probability (1: none)
    // a tile wave (az_gpu_render_tiles) holds samples of several jobs of one
    // scene: per wave slot its (job, sample index in the job), and each job's
    // camera; null: every sample belongs to the kernels' `cam`
    const uint2 *slot_map;
    const CameraParams *job_cams;
    // a tile wave whose jobs render different scenes: the scenes' device
    // records; every path entry carries its scene index in its flags (bits
    // 16-23) and every shadow entry in its meta word (bits 22-29); null: the
    // kernels' own scene argument
    const azd::DevScene *scenes;
};

// One tile of a tile wave: samples [first, first + count) of job `job`, at
// wave slots [slot, slot + count).
struct Tile {
    uint32_t job, first, count, slot;
};

struct WaveBuffers {
    WaveQueues q{};
    uint32_t chunk = 0;
    std::vector<void *> ptrs;
    // the per-wave launches captured as a CUDA graph, with what they were captured for
    uint64_t *wave_dev = nullptr;          // device copy of the wave descriptor
    uint64_t *wave_host = nullptr;         // pinned staging for it
    cudaGraphExec_t graph = nullptr;
    std::vector<unsigned char> graph_key;
    uint64_t graph_launches = 0, graph_extend_launches = 0;   // kernels in the graph
    // scratch of guided waves: proposals per queue entry, training records
    azd::GuideLobes *guide_lobes = nullptr;
    size_t guide_lobes_cap = 0;
    azd::GuideRecord *guide_rec = nullptr;
    size_t guide_rec_cap = 0;
    // queue ordering: cell keys (double-buffered), identity indices, the two
    // visiting orders and the radix sort's scratch
    uint32_t *okey[2] = {nullptr, nullptr}, *oval = nullptr, *oidx_e = nullptr, *oidx_s = nullptr;
    void *otemp = nullptr;
    size_t otemp_bytes = 0;
    uint32_t ocap = 0;
    // second stream of a wave: a level's visibility queries run on it beside
    // the next level's closest-hit queries (fork after shading, join before
    // the next shading)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    ~WaveBuffers();
    int EnsureSide();
    int EnsureOrder(uint32_t cap);
    void DropGraph();
    int Ensure(uint32_t chunk, uint32_t cap_q, uint32_t cap_s);
};

struct RenderCounters {
    uint64_t extend = 0, shadow = 0, nodes = 0, prims = 0, snodes = 0, sprims = 0, launches = 0, extend_launches = 0;
    uint32_t chunks = 0, retries = 0;
};

}  // namespace az
