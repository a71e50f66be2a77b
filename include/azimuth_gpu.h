/*
 * azimuth_gpu.h -- C-ABI of the B200 render path.
 *
 * Drop-in for azimuth's render core: the scene, camera and epsilon structs are
 * azimuth's own (see az_abi.h), and the film is azimuth's `pixel` buffer
 * ({rgb sum, weight sum} per pixel, src/azimuth_main.cpp:45-48).  No function
 * throws, traps the GPU or falls back to the CPU; every call returns an
 * AZ_* status and az_gpu_last_error() describes the last failure of the
 * calling thread.
 *
 * Randomness: azimuth's Random01 (src/azimuth_math.cpp:1-8, libc rand()) is
 * replaced by a counter-based RNG.  Every TraceRay activation of a camera
 * sample is a node of the sample's path tree; draw `dim` of node (level,
 * digits) of sample (SampleX, SampleY) of pixel (Row, Col) is lane dim&3 of
 * Philox-4x32-10 with counter {Row<<16|Col, SampleY<<16|SampleX, digits,
 * level<<24 | dim>>2} and key `seed`, mapped to [0,1) as (x>>8)*2^-24.
 * Level 0 is the camera (lens y, lens x, shutter time), level 1 the primary
 * TraceRay, and child k (0..3, in azimuth's call order: scatter, mirror,
 * refraction, reflection) of a node at level L adds k << 2*(L-1) to digits.
 */
#ifndef AZIMUTH_GPU_H
#define AZIMUTH_GPU_H

#include "az_abi.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
    AZ_OK = 0,
    AZ_ERR_INVALID_ARGUMENT = 1,
    AZ_ERR_INVALID_SCENE = 2,
    AZ_ERR_OUT_OF_MEMORY = 3,
    AZ_ERR_CUDA = 4,
    AZ_ERR_TIMEOUT = 5,
    AZ_ERR_UNSUPPORTED = 6,
    AZ_ERR_NO_DEVICE = 7,
    AZ_ERR_IO = 8
};

/* az_render_opts.flags */
enum {
    AZ_FLAG_NONE = 0,
    AZ_FLAG_COUNT_TRAVERSAL = 1u << 0,  /* fill az_render_stats node/primitive visit counters (waves of at
                                           most 2^22 samples unless chunk_samples is set) */
    AZ_FLAG_NO_GRAPH = 1u << 1,         /* launch the per-bounce stages directly, not as a CUDA graph */
    AZ_FLAG_TIME_STAGES = 1u << 2,      /* time each stage with CUDA events (az_render_stats *_ms) */
    AZ_FLAG_ENV_IMPORTANCE = 1u << 3,   /* environment light samples by one-sample MIS of a luminance CDF of
                                           the 2D environment map and cosine sampling, instead of azimuth's
                                           cosine sampling alone (same estimate, lower variance for peaked
                                           maps; not a parity mode) */
    /* Queue ordering (the results do not change, only which rays share a warp):
     * by default the scene's choice (az_gpu_autotune picks it). */
    AZ_FLAG_ORDER_SHADOW = 1u << 4,     /* visit each level's shadow queue in the order of the rays' origin cells */
    AZ_FLAG_ORDER_EXTEND = 1u << 5,     /* visit each level's extension queue by origin cell and direction octant */
    AZ_FLAG_ORDER_NONE = 1u << 6,       /* queues in the order they were filled */
    AZ_FLAG_SERIAL_LEVELS = 1u << 7,    /* run each tree level's visibility queries before the next level's
                                           closest-hit queries (default: the two run side by side on two
                                           streams, so one's tail overlaps the other's work) */
    AZ_FLAG_WATERTIGHT = 1u << 8        /* production mode: triangles by the watertight test of Woop, Benthin
                                           and Wald (JCGT 2013) on the exact vertices -- no ray passes between
                                           triangles that share an edge or vertex -- instead of azimuth's
                                           Cramer test with its -1e-6 barycentric tolerance (the parity
                                           default); one launch configuration; also az_gpu_closest_hit */
};

/* Number of traversal launch configurations (az_render_opts.variant). */
#define AZ_LAUNCH_VARIANTS 20

typedef struct az_render_opts {
    uint64_t seed;                  /* counter-RNG key */
    const float *perlin_gradients;  /* azimuth's PerlinGradient[256] (src/azimuth_texture.h:17-18),
                                       256*3 floats; required when a Perlin texture is used */
    void *stream;                   /* cudaStream_t to run on, or NULL for the library's own stream */
    int32_t device;                 /* CUDA device ordinal */
    uint32_t flags;                 /* AZ_FLAG_* */
    uint32_t chunk_samples;         /* camera samples in flight per wave; 0 = automatic: the power of two
                                       from 2^22 to 2^26 whose wave queues (~350 bytes a sample) fit in a
                                       quarter of the free device memory; they stay allocated with the
                                       scene for its next render */
    uint32_t bvh_width;             /* az_gpu_scene_create: children per BVH node, 2, 4 or 8 (0 = 8) */
    uint32_t block_size;            /* reserved (0) */
    uint32_t variant;               /* traversal launch configuration 1..AZ_LAUNCH_VARIANTS (threads per
                                       block, register cap, how queries map to threads: one per thread
                                       to its end, warp lockstep per traversal step, or persistent
                                       fetching, with node fetches staged through shared memory in
                                       variants 19 and 20); 0 = the scene's choice: 8 (128 threads, at most 64
                                       registers, persistent fetching) until az_gpu_autotune picks another */
    uint32_t bvh_leaf;              /* az_gpu_scene_create: triangles per bottom-level leaf at most, 1..3 (0 = 2) */
    uint32_t bvh_builder;           /* az_gpu_scene_create: binary hierarchy before the wide collapse,
                                       AZ_BVH_LBVH or AZ_BVH_PLOC (0 = the default, AZ_BVH_PLOC) */
    uint32_t sample_part;           /* with sample_parts > 1: render only part sample_part (0-based) of */
    uint32_t sample_parts;          /* sample_parts equal ranges of the scissor's camera-sample sequence
                                       (sample number x pixels, pixels fastest), i.e. about spp/parts
                                       samples of every pixel; the parts of one frame sum to the whole
                                       frame (one GPU per part); 0 or 1 = every sample */
} az_render_opts;

enum {
    AZ_BVH_LBVH = 1,   /* Morton-order radix tree (Karras 2012): fastest build */
    AZ_BVH_PLOC = 2    /* locally-ordered clustering (Meister, Bittner 2018): fewer nodes visited per ray */
};

typedef struct az_render_stats {
    uint64_t samples;               /* camera samples rendered */
    uint64_t extend_rays;           /* closest-hit queries (path segments) */
    uint64_t shadow_rays;           /* NEE visibility queries */
    uint32_t chunks;
    uint32_t retries;               /* waves re-run with fewer samples after a queue overflow */
    uint64_t kernel_launches;
    float gpu_ms;                   /* device time of the render, CUDA events on the render stream */
    float extend_ms;                /* with AZ_FLAG_TIME_STAGES: closest-hit stage */
    float shade_ms;                 /* with AZ_FLAG_TIME_STAGES: shading stage */
    float shadow_ms;                /* with AZ_FLAG_TIME_STAGES: visibility stage */
    uint64_t node_visits;           /* with AZ_FLAG_COUNT_TRAVERSAL: BVH nodes visited by closest-hit queries */
    uint64_t prim_visits;           /* with AZ_FLAG_COUNT_TRAVERSAL: primitives tested by closest-hit queries */
    uint32_t extend_launches;       /* closest-hit stage launches */
    uint32_t reserved0;
    uint64_t shadow_node_visits;    /* with AZ_FLAG_COUNT_TRAVERSAL: BVH nodes visited by visibility queries */
    uint64_t shadow_prim_visits;    /* with AZ_FLAG_COUNT_TRAVERSAL: primitives tested by visibility queries */
    uint32_t reserved[2];
} az_render_stats;

typedef struct az_gpu_scene az_gpu_scene;

/* Flatten `scene` (walking its BVH trees to the leaves), upload it and build
 * the device BVHs.  The host scene is only read. */
int az_gpu_scene_create(const az_scene *scene, const az_render_opts *opts, az_gpu_scene **out);
void az_gpu_scene_destroy(az_gpu_scene *scene);

/* What az_gpu_scene_create built and how long its parts took (no counterpart
 * in azimuth, whose ImportXML builds its BVHs on the host,
 * src/azimuth_xml.cpp:3632-3875 and src/azimuth_bvh.cpp:1-328). */
typedef struct az_scene_info {
    uint64_t triangles;          /* triangles of all meshes, after flattening */
    uint64_t spheres;
    uint64_t wide_nodes;         /* compressed wide BVH nodes of all hierarchies */
    uint64_t device_bytes;       /* device memory the scene holds */
    uint32_t bvh_width, bvh_leaf;
    uint32_t bvh_depth;          /* deepest wide-node level (root = 0) */
    uint32_t hierarchies;        /* bottom-level hierarchies plus the top level */
    float flatten_ms;            /* host: azimuth's entity trees walked into device records (and the
                                    lights, materials and textures) */
    float upload_ms;             /* host-to-device copies of the primitives */
    float bvh_ms;                /* GPU: LBVH builds, wide collapse and primitive gather */
    float total_ms;              /* the whole az_gpu_scene_create call */
    float ingest_ms;             /* GPU post-processing of a mesh soup (az_gpu_scene_create_from_meshes) */
    uint32_t bvh_builder;        /* AZ_BVH_LBVH or AZ_BVH_PLOC */
    uint32_t queue_order;        /* the scene's queue ordering: AZ_FLAG_ORDER_SHADOW | AZ_FLAG_ORDER_EXTEND bits
                                    (0: queue order); az_gpu_autotune sets it */
    uint32_t variant;            /* the scene's traversal launch configuration, 1-based */
    uint32_t shadow_variant;     /* the shadow queries' launch configuration, 1-based (az_gpu_autotune
                                    times it separately; a variant named in az_render_opts applies to both) */
} az_scene_info;

int az_gpu_scene_info(const az_gpu_scene *scene, az_scene_info *out);

/* Device addresses of a resident scene's hierarchy and triangles (no
 * counterpart in azimuth, whose BVH is a tree of host entities), for callers
 * that run kernels of their own on the scene.  The arrays belong to the scene
 * until az_gpu_scene_destroy; the renderer reads them on every query, so a
 * caller that writes into them changes what later renders see (a damaged
 * hierarchy makes a render fail with AZ_ERR_CUDA once a query exceeds its
 * step limit, never hang).
 *   wide node (80 B): grid origin (3 floats), 3 exponent bytes, an inner-child
 *   mask byte, first inner child, first leaf primitive, 8 leaf-meta bytes
 *   (count << 5 | offset), then the 8 children's quantised low x, y, z and
 *   high x, y, z bytes;
 *   triangle (48 B): P0, P0 - P1, P0 - P2, face normal, in leaf order. */
typedef struct az_scene_arrays {
    void *wide_nodes;
    uint64_t wide_node_count;
    void *triangles;
    uint64_t triangle_count;
    uint32_t tlas_root;          /* top-level root node; 0xFFFFFFFF: empty scene */
    uint32_t single_group_root;  /* when the top level holds one group, the root of its hierarchy, which
                                    queries enter directly; else 0xFFFFFFFF */
    uint32_t reserved[4];
} az_scene_arrays;

int az_gpu_scene_arrays(const az_gpu_scene *scene, az_scene_arrays *out);

/* ---- Scene ingestion on the GPU ----
 * azimuth's importer collects every mesh's vertices, faces and UVs into shared
 * arrays, then post-processes them on the host (src/azimuth_xml.cpp:3632-3776:
 * per-vertex normals as the normalised sum of the unnormalised normals of the
 * faces using the vertex, in face order; face normals; TotalArea; UVs through
 * UVOffset) and builds a 288-byte entity BVH per mesh.  The two calls below
 * take those arrays as they are before the post-processing and do it on the
 * GPU with the same float arithmetic (per-vertex sums in face order, so the
 * results are bit for bit azimuth's). */
typedef struct az_mesh_desc {
    uint32_t face_base, face_count;   /* the mesh's faces: faces[face_base, face_base + face_count) */
    int32_t uv_offset;                /* Mesh->UVOffset: vertex i's UV is uvs[i + uv_offset] when in range */
    uint32_t shading_mode;            /* AZ_Shading_* */
    uint32_t material_index, texture_index;
    uint32_t is_emitter;
    uint32_t unique_entity_id;        /* UniqueEntityID of the mesh's instance entity */
    az_vec3 motion, radiance;
    az_mat4 transform, inv_transform; /* Mesh->TransformationMatrix / InvTransformationMatrix */
} az_mesh_desc;

typedef struct az_mesh_soup {
    const az_vec3 *vertices;          /* host arrays */
    const az_vec3u *faces;            /* vertex indices */
    const az_vec2 *uvs;               /* may be NULL when uv_count is 0 */
    const az_mesh_desc *meshes;       /* face ranges must not overlap */
    uint32_t vertex_count, face_count, uv_count, mesh_count;
} az_mesh_soup;

/* Per-face shading data of the importer's triangle entities (entity.N0-N2, UV0-UV2). */
typedef struct az_face_attr {
    az_vec3 N0, N1, N2;
    az_vec2 UV0, UV1, UV2;
} az_face_attr;

/* The importer's mesh post-processing on the GPU, results copied to the HOST
 * arrays given (any may be NULL): vertex_normals[vertex_count], triangles
 * and attrs[face_count] (azimuth's triangle {P0, P1, P2, unit face normal}
 * and the entity fields, for every face; a face outside every mesh gets UVs
 * 0), total_area[mesh_count] (Mesh->TotalArea: the float sum of |N|/2 over the
 * mesh's faces in order).  Synchronous. */
int az_gpu_mesh_postprocess(const az_mesh_soup *soup, az_vec3 *vertex_normals, az_triangle *triangles,
                            az_face_attr *attrs, float *total_area, const az_render_opts *opts);

/* az_gpu_scene_create for a scene whose meshes come as `soup`: the meshes are
 * post-processed on the GPU and go straight into the device scene, with no
 * host triangles or entity BVHs.  Everything else comes from `scene`:
 * materials, textures, lights, environment and settings, and the other
 * entities found under scene->BVHRoot (BVHRoot may be NULL).  A mesh instance
 * there whose UniqueEntityID is a soup mesh's unique_entity_id is that mesh's
 * own instance and comes from the soup; any other mesh instance (a
 * MeshInstance element, src/azimuth_xml.cpp:2743-2797) places soup mesh
 * BaseMeshID again with the instance's transform, motion and material.  An
 * entity light whose entity is a mesh instance takes its triangles and area
 * from soup mesh Entity.BaseMeshID. */
int az_gpu_scene_create_from_meshes(const az_scene *scene, const az_mesh_soup *soup, const az_render_opts *opts,
                                    az_gpu_scene **out);

/* ProduceImageInLinearSpace (src/azimuth_main.cpp:1256-1263) on the GPU:
 * accumulates every camera sample of the scissor rectangle into the HOST film
 * `pixels` (W*H entries, caller-zeroed or holding earlier sums), with
 * filter_type AZ_Filter_Box or AZ_Filter_Gaussian (src/azimuth_main.cpp:1209-1254).
 * Builds and frees a device scene for this one call. */
int az_gpu_produce_image(az_pixel *pixels, const az_scene *scene, const az_camera *camera,
                         const az_epsilon_values *epsilons, az_scissor scissor, int32_t filter_type,
                         uint32_t backface_culling, const az_render_opts *opts);

/* Same render on a device scene; `film` is a DEVICE pointer to W*H az_pixel
 * that is accumulated into.  Runs on opts->stream; returns after the work is
 * queued unless `stats` is non-NULL (then it synchronises and fills it). */
int az_gpu_render(az_gpu_scene *scene, az_pixel *film, const az_camera *camera,
                  const az_epsilon_values *epsilons, az_scissor scissor, int32_t filter_type,
                  uint32_t backface_culling, const az_render_opts *opts, az_render_stats *stats);

/* Per-sample radiance (the value ProduceImageInLinearSpace hands to
 * ComputeSampleWeight, src/azimuth_main.cpp:1365-1391, before any filter):
 * renders the scissor like az_gpu_render but writes camera sample s's RGB sum
 * to samples[4 s .. 4 s + 2] (DEVICE memory, 16-byte aligned, 4 floats per
 * sample; the 4th is 0) instead of splatting it, with s = (SampleY *
 * SampleCountSqrt + SampleX) * scissor pixels + (Row - Min.y) * scissor width
 * + (Col - Min.x).  For per-path comparisons with azimuth. */
int az_gpu_render_samples(az_gpu_scene *scene, float *samples, const az_camera *camera,
                          const az_epsilon_values *epsilons, az_scissor scissor, uint32_t backface_culling,
                          const az_render_opts *opts, az_render_stats *stats);

/* ProduceImageInLinearSpace on a device scene with a HOST film: copies
 * `pixels` to the device, renders into it and copies it back (synchronous). */
int az_gpu_render_host(az_gpu_scene *scene, az_pixel *pixels, const az_camera *camera,
                       const az_epsilon_values *epsilons, az_scissor scissor, int32_t filter_type,
                       uint32_t backface_culling, const az_render_opts *opts, az_render_stats *stats);

/* Autotuner: renders a band of the frame (the middle rows of the scissor: an
 * eighth of them, or enough for about 2^20 samples) with each traversal launch
 * configuration and keeps the fastest as the scene's default.  Writes the chosen variant (1-based) and its
 * time in ms.  Synchronous. */
int az_gpu_autotune(az_gpu_scene *scene, const az_camera *camera, const az_epsilon_values *epsilons,
                    az_scissor scissor, int32_t filter_type, uint32_t backface_culling,
                    const az_render_opts *opts, uint32_t *variant_out, float *ms_out);

/* Autotuner over the hierarchy's shape as well: rebuilds the device
 * hierarchy of `host_scene` (the scene `scene` was created from) with 8, 4 and
 * 2 children per node and 1 to 3 triangles per bottom-level leaf, runs
 * az_gpu_autotune on each and keeps the fastest build (and its launch
 * configuration) in `scene`; the binary builder stays the scene's.  Writes the
 * width, the variant (1-based) and its time in ms.  Synchronous; `scene` must
 * not be rendering meanwhile.  A scene made by az_gpu_scene_create_from_meshes
 * has no host_scene to rebuild from: AZ_ERR_UNSUPPORTED. */
int az_gpu_autotune_scene(const az_scene *host_scene, az_gpu_scene *scene, const az_camera *camera,
                          const az_epsilon_values *epsilons, az_scissor scissor, int32_t filter_type,
                          uint32_t backface_culling, const az_render_opts *opts, uint32_t *width_out,
                          uint32_t *variant_out, float *ms_out);

/* OutputPixelsToFile's image post-processing (src/azimuth_main.cpp:1620-1760)
 * on the GPU, for a DEVICE film of width x height az_pixel that is left
 * untouched: colour / TotalWeight; with tonemap->Operator == Photographic
 * (and not `linear`) azimuth's photographic operator (log-average luminance,
 * burn-out percentile of the sorted luminances, saturation); then, unless
 * `linear` (azimuth's EXR output), sRGB (`srgb`) or 1/gamma (`inv_gamma`)
 * correction.  Writes the resulting colours (width*height*3 floats) to the
 * DEVICE buffer rgb_out and/or the bytes azimuth's PNG/BMP/TGA/JPG writers
 * store, (uint8)(clamp01(c) * 255), to the DEVICE buffer rgb8_out (either may
 * be NULL).  Synchronous.  The log-average is summed in double (azimuth: a
 * serial float sum), so results can differ from azimuth's in the last bits. */
int az_gpu_postprocess(const az_pixel *film, uint32_t width, uint32_t height, const az_tonemap *tonemap,
                       float inv_gamma, uint32_t srgb, uint32_t linear, float *rgb_out, uint8_t *rgb8_out,
                       const az_render_opts *opts);

/* ---- Batched render jobs (no counterpart in azimuth, which renders one camera per call) ----
 *
 * Many render jobs of uneven size, scene and settings in one call: the jobs
 * run concurrently on `streams` CUDA streams (default 4), shortest first (or
 * largest first), each stream with its own wave queues; a job of several
 * waves replays its wave launches as one CUDA graph.  Each job is az_gpu_render (or, with a guide,
 * az_gpu_render_guided) of its own scene, camera and DEVICE film.  Jobs that
 * share a guide run one after another. */
typedef struct az_job {
    az_gpu_scene *scene;
    struct az_guide *guide;         /* NULL: plain render */
    az_pixel *film;                 /* DEVICE film, W*H of the job's camera, accumulated into */
    const az_camera *camera;
    const az_epsilon_values *epsilons;
    az_scissor scissor;
    int32_t filter_type;
    uint32_t backface_culling;
    uint32_t train;                 /* guided jobs: train the guide while rendering */
    uint32_t reserved0;
    uint64_t seed;
    /* written by az_gpu_render_batch */
    float done_ms;                  /* completion time after the batch started (device clock) */
    int32_t status;                 /* AZ_OK or the job's error */
    uint64_t samples;
} az_job;

typedef struct az_batch_opts {
    int32_t device;
    uint32_t streams;               /* concurrent jobs; 0 = 4 */
    uint32_t flags;                 /* AZ_FLAG_* applied to every job */
    uint32_t chunk_samples;         /* 0 = 2^22 per job in az_gpu_render_batch; az_gpu_render_tiles as
                                       az_render_opts.chunk_samples */
    uint32_t largest_first;         /* 0: shortest jobs first (low completion times); 1: largest first */
    uint32_t tiles;                 /* az_gpu_render_batch: 1 = the plain jobs (guide NULL) render together
                                       in tile waves (az_gpu_render_tiles) on one stream while the other
                                       streams take the guided jobs; 0 = every job on its own */
    uint32_t reserved[2];
} az_batch_opts;

typedef struct az_batch_stats {
    uint64_t samples;               /* camera samples of all jobs */
    float gpu_ms;                   /* batch start to the last job's completion */
    float p50_ms, p99_ms;           /* job completion times */
    uint32_t jobs, failed, streams;
    uint32_t reserved[3];
} az_batch_stats;

/* Returns AZ_OK when every job succeeded, else the first failing job's status
 * (see each job's `status`). Synchronous. */
int az_gpu_render_batch(az_job *jobs, uint32_t n, const az_batch_opts *opts, az_batch_stats *stats);

/* Jobs rendered together: every job's camera samples are cut into tiles of
 * 4096, and each wave of the render takes the next tiles of all jobs from a
 * device work queue (a camera kernel whose blocks pull tiles), so one chain
 * of extend/shade/shadow launches per wave serves every job and small jobs
 * share waves instead of running their own.  The jobs may differ in scene
 * (up to 256 device scenes of one device: every queue entry carries its
 * scene's index, and the kernels trace and shade it in that scene), camera,
 * resolution, spp, depth, scissor, filter, seed and film; they must share the
 * epsilon values and culling, and be plain renders (guide NULL).  Each job's
 * film gets exactly what az_gpu_render with the job's seed would add (up to
 * the order of float atomics).  opts->streams and largest_first are ignored;
 * a job's done_ms is the end of the wave holding its last tile.  Synchronous. */
int az_gpu_render_tiles(az_job *jobs, uint32_t n, const az_batch_opts *opts, az_batch_stats *stats);

/* ---- Neural path guiding (the learned proposal; no counterpart in azimuth) ----
 *
 * A guide belongs to one device scene.  Rendered with az_gpu_render_guided,
 * the scattering direction of every diffuse vertex is drawn by one-sample
 * MIS from a learned mixture of 8 von Mises-Fisher lobes (a hash-grid encoded
 * MLP of position, normal and outgoing direction) and cosine sampling, with a
 * learned selection probability; the mixture density weights the sample, so
 * the estimate stays unbiased.  With `train` set, every wave also trains the
 * network (four Adam steps by default) on the radiance its own paths brought back. */
typedef struct az_guide az_guide;

typedef struct az_guide_config {
    float learning_rate;            /* Adam step size; 0 = 1e-2 */
    uint32_t train_batch;           /* training rows per step at most; 0 = 2^18 */
    uint32_t record_samples;        /* camera samples per wave whose vertices are recorded; 0 = 2^17 */
    uint32_t steps_per_wave;        /* Adam steps on each wave's rows when training; 0 = 4 */
    uint64_t seed;                  /* weight initialisation */
    uint32_t kernels;               /* network kernels (proposals and training): AZ_GUIDE_TCGEN05 (0, the
                                       default) runs the MLP on the 5th-generation tensor cores
                                       (tcgen05.mma, operands in shared memory, accumulators in tensor
                                       memory, 128 rows per CTA); AZ_GUIDE_MMA_SYNC runs it warp by warp
                                       with mma.sync (16 rows per warp) */
    uint32_t queue_order_rows;      /* 1: the tcgen05 proposals visit a level's rows in queue order; 0 (the
                                       default): bucketed by the cell of their hit point first, so a
                                       tile's hash-grid gathers share cells */
    uint32_t reserved[4];
} az_guide_config;

enum { AZ_GUIDE_TCGEN05 = 0, AZ_GUIDE_MMA_SYNC = 1 };

int az_guide_create(az_gpu_scene *scene, const az_guide_config *cfg, az_guide **out);
void az_guide_destroy(az_guide *guide);

/* az_gpu_render with the guide's proposal for the scattering direction;
 * `train` != 0 trains after every wave (waves of 2^20 camera samples unless
 * opts->chunk_samples says otherwise).
 * Pass the scene the guide was created for. */
int az_gpu_render_guided(az_gpu_scene *scene, az_guide *guide, az_pixel *film, const az_camera *camera,
                         const az_epsilon_values *epsilons, az_scissor scissor, int32_t filter_type,
                         uint32_t backface_culling, uint32_t train, const az_render_opts *opts,
                         az_render_stats *stats);

/* Network access for tests and tools (host arrays, synchronous).
 * mlp: 4 x 64 x 64 weights W[layer][input][output]; bias: 64 output-layer
 * biases; grid: 16 x 2^19 x 2 hash-grid features.  NULL skips an array. */
int az_guide_get_params(az_guide *guide, float *mlp, float *bias, float *grid);
int az_guide_set_params(az_guide *guide, const float *mlp, const float *bias, const float *grid);
/* Level resolutions (16), position normalisation (lo, 1/extent) and Adam steps taken. */
int az_guide_info(az_guide *guide, uint32_t *res, float *lo, float *inv_ext, uint32_t *steps);
/* Rows: n x 16 floats (position, weight, normal, 0, outgoing direction, 0,
 * incident direction, 0).  Evaluates the network and the loss
 * sum_i -w_i log q_i(wi_i) without updating it: raw outputs (n x 64), the
 * loss, its gradient with respect to the MLP weights, the output biases and
 * the encoded grid features (n x 32).  Any output may be NULL. */
int az_guide_eval(az_guide *guide, const float *rows, uint32_t n, float *outputs, float *loss, float *mlp_grad,
                  float *bias_grad, float *enc_grad);
/* `steps` Adam steps on the given rows; per-step loss (before the step) in losses. */
int az_guide_train(az_guide *guide, const float *rows, uint32_t n, uint32_t steps, float *losses);
/* Raw network outputs (n x 64) of caller rows (the layout of az_guide_eval)
 * computed by the tcgen05 inference kernel that makes the render's proposals.
 * AZ_ERR_CUDA if a tensor-core wait gave up (the kernel then stops). */
int az_guide_infer(az_guide *guide, const float *rows, uint32_t n, float *outputs);

/* Allocation-free variant of az_gpu_render; it has no counterpart in azimuth.
 *
 * For callers that cannot allocate device memory while they render: hosts
 * whose caching allocator has already reserved the GPU's memory (a cudaMalloc
 * from the library would fail, or fragment the host's pool), plug-in hosts
 * that forbid their plug-ins to allocate, and real-time loops that keep a
 * fixed memory budget.  The scene (created earlier with az_gpu_scene_create)
 * and the DEVICE film are passed in as usual; the wave queues live in one
 * static device array of 9,110,784 bytes (8.7 MiB) that every GPU loading
 * this library holds until the process exits, which caps a wave at 16384
 * camera samples: opts->chunk_samples above 16384 is rejected with
 * AZ_ERR_INVALID_ARGUMENT.  The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress).  All calls share the array and it keeps the last
 * call's contents (the counters are cleared at the start of every wave):
 * calls that overlap on the GPU (other threads or streams) race and must be
 * serialised by the caller.  A wave whose queues overflow the array is run
 * again with half the samples, down to 256.  opts->flags may hold
 * AZ_FLAG_ENV_IMPORTANCE and AZ_FLAG_WATERTIGHT; flags that need allocations
 * or statistics (AZ_FLAG_COUNT_TRAVERSAL, AZ_FLAG_TIME_STAGES,
 * AZ_FLAG_ORDER_SHADOW, AZ_FLAG_ORDER_EXTEND) are rejected with
 * AZ_ERR_INVALID_ARGUMENT, and the scene's own queue ordering is not applied
 * (it never changes the film).  Synchronous: every wave copies its queue
 * counters to the host and synchronises the stream.  Runs on opts->stream, or
 * on the per-thread default stream when that is NULL; never calls cudaMalloc
 * or cudaFree. */
int az_gpu_render_noalloc(az_gpu_scene *scene, az_pixel *film, const az_camera *camera,
                          const az_epsilon_values *epsilons, az_scissor scissor, int32_t filter_type,
                          uint32_t backface_culling, const az_render_opts *opts);

/* Closest hit for `count` HOST rays (azimuth's RayEntityIntersection on the
 * scene root, src/azimuth_main.cpp:53-385).  Per ray: hit flag, UniqueEntityID
 * of the top-level entity, face id (entity.ID of the triangle hit inside a
 * mesh instance, else 0xFFFFFFFF; in a scene built from a mesh soup, the
 * face's index within its mesh, as azimuth's importer keeps no face id of its
 * own, src/azimuth_xml.cpp:3695) and world t.  Synchronous. */
int az_gpu_closest_hit(az_gpu_scene *scene, const az_ray3 *rays, uint32_t count, int32_t cull,
                       float hit_epsilon, uint32_t *out_hit, uint32_t *out_uid, uint32_t *out_face,
                       float *out_t, const az_render_opts *opts);

/* Device name, SM count and memory; returns AZ_ERR_NO_DEVICE without a GPU. */
int az_gpu_device_info(int32_t device, char *name, uint32_t name_len);

/* The counter RNG on the host: draw `dim` of tree node (level, digits) of
 * camera sample `sample` (SampleY<<16|SampleX) of pixel `pixel` (Row<<16|Col),
 * exactly as the kernels draw it; and the raw Philox-4x32-10 block function. */
float az_rng_u01(uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t digits, uint32_t level, uint32_t dim);
void az_rng_philox4x32_10(const uint32_t counter[4], uint32_t key0, uint32_t key1, uint32_t out[4]);

/* Message of the last failed call on this thread ("" if none). */
const char *az_gpu_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
