// extern "C" entry points of include/azimuth_gpu.h.
//
// Each call selects opts->device, runs on opts->stream (or a private stream),
// catches every CUDA error into an AZ_* status and never throws across the ABI.
#include <cfloat>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "az_internal.h"
#include "azimuth_io.h"

namespace az {

namespace {
thread_local std::string t_last_error;
}

int SetError(int code, const std::string &msg) {
    t_last_error = msg;
    return code;
}

int CudaError(cudaError_t e, const char *what) {
    int code = e == cudaErrorMemoryAllocation ? AZ_ERR_OUT_OF_MEMORY
               : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? AZ_ERR_NO_DEVICE
                                                                             : AZ_ERR_CUDA;
    cudaGetLastError();  // clear a sticky non-fatal error state
    return SetError(code, std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

// Picks the device and the stream for one call; owns a private stream when
// the caller passed none.
struct CallContext {
    cudaStream_t stream = nullptr;
    bool own = false;
    int begin(const az_render_opts *opts) {
        int dev = opts ? opts->device : 0;
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess || n == 0) return SetError(AZ_ERR_NO_DEVICE, "no CUDA device available");
        if (dev < 0 || dev >= n) return SetError(AZ_ERR_INVALID_ARGUMENT, "device ordinal out of range");
        AZ_CUDA_TRY(cudaSetDevice(dev));
        if (opts && opts->stream) {
            stream = (cudaStream_t)opts->stream;
        } else {
            // a blocking stream: ordered after earlier work on the legacy default
            // stream (a film zeroed there, for instance)
            AZ_CUDA_TRY(cudaStreamCreate(&stream));
            own = true;
        }
        return AZ_OK;
    }
    ~CallContext() {
        if (own && stream) {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
    }
};

}  // namespace az


using namespace az;

extern "C" const char *az_gpu_last_error(void) { return t_last_error.c_str(); }

extern "C" int az_gpu_device_info(int32_t device, char *name, uint32_t name_len) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return SetError(AZ_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= n) return SetError(AZ_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    cudaDeviceProp p;
    AZ_CUDA_TRY(cudaGetDeviceProperties(&p, device));
    if (name && name_len) {
        snprintf(name, name_len, "%s|sm_%d%d|%d SMs|%zu MiB", p.name, p.major, p.minor, p.multiProcessorCount,
                 (size_t)(p.totalGlobalMem >> 20));
    }
    return AZ_OK;
}

extern "C" int az_gpu_scene_create(const az_scene *scene, const az_render_opts *opts, az_gpu_scene **out) {
    if (!scene || !out) return SetError(AZ_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    CallContext ctx;
    int rc = ctx.begin(opts);
    if (rc != AZ_OK) return rc;
    GpuScene *g = nullptr;
    rc = BuildGpuScene(scene, opts, ctx.stream, &g);
    if (rc != AZ_OK) return rc;
    az_gpu_scene *h = new (std::nothrow) az_gpu_scene{g};
    if (!h) {
        delete g;
        return SetError(AZ_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    *out = h;
    return AZ_OK;
}

extern "C" int az_gpu_scene_create_from_meshes(const az_scene *scene, const az_mesh_soup *soup,
                                               const az_render_opts *opts, az_gpu_scene **out) {
    if (!scene || !soup || !out) return SetError(AZ_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    CallContext ctx;
    int rc = ctx.begin(opts);
    if (rc != AZ_OK) return rc;
    GpuScene *g = nullptr;
    rc = BuildGpuScene(scene, opts, ctx.stream, &g, soup);
    if (rc != AZ_OK) return rc;
    az_gpu_scene *h = new (std::nothrow) az_gpu_scene{g};
    if (!h) {
        delete g;
        return SetError(AZ_ERR_OUT_OF_MEMORY, "host allocation failed");
    }
    *out = h;
    return AZ_OK;
}

extern "C" int az_gpu_mesh_postprocess(const az_mesh_soup *soup, az_vec3 *vertex_normals, az_triangle *triangles,
                                       az_face_attr *attrs, float *total_area, const az_render_opts *opts) {
    if (!soup) return SetError(AZ_ERR_INVALID_ARGUMENT, "null mesh soup");
    CallContext ctx;
    int rc = ctx.begin(opts);
    if (rc != AZ_OK) return rc;
    SoupWork *w = nullptr;
    rc = IngestSoup(soup, ctx.stream, &w);
    if (rc != AZ_OK) return rc;
    std::unique_ptr<SoupWork, void (*)(SoupWork *)> hold(w, FreeSoupWork);
    if (total_area) {
        std::vector<float> a;
        if ((rc = SoupAreas(*w, a)) != AZ_OK) return rc;
        if (!a.empty()) memcpy(total_area, a.data(), a.size() * sizeof(float));
    }
    return SoupRecords(*w, triangles, attrs, vertex_normals, ctx.stream);
}

extern "C" int az_gpu_scene_info(const az_gpu_scene *scene, az_scene_info *out) {
    if (!scene || !scene->impl || !out) return SetError(AZ_ERR_INVALID_ARGUMENT, "null scene or output");
    const GpuScene &G = *scene->impl;
    memset(out, 0, sizeof(*out));
    out->triangles = G.triangle_count;
    out->spheres = G.sphere_count;
    out->wide_nodes = G.node_count;
    out->device_bytes = G.device_bytes;
    out->bvh_width = G.bvh_width;
    out->bvh_leaf = G.bvh_leaf;
    out->bvh_depth = G.max_bvh_depth;
    out->hierarchies = G.hierarchies;
    out->flatten_ms = G.flatten_ms;
    out->upload_ms = G.upload_ms;
    out->bvh_ms = G.bvh_ms;
    out->total_ms = G.total_ms;
    out->ingest_ms = G.ingest_ms;
    out->bvh_builder = G.bvh_builder;
    out->queue_order = ((G.order & kOrderShadow) ? (uint32_t)AZ_FLAG_ORDER_SHADOW : 0u) |
                       ((G.order & kOrderExtend) ? (uint32_t)AZ_FLAG_ORDER_EXTEND : 0u);
    out->variant = G.variant + 1;
    out->shadow_variant = (G.shadow_variant < AZ_LAUNCH_VARIANTS ? G.shadow_variant : G.variant) + 1;
    return AZ_OK;
}

extern "C" int az_gpu_scene_arrays(const az_gpu_scene *scene, az_scene_arrays *out) {
    if (!scene || !scene->impl || !out) return SetError(AZ_ERR_INVALID_ARGUMENT, "null scene or output");
    const GpuScene &G = *scene->impl;
    memset(out, 0, sizeof(*out));
    out->wide_nodes = (void *)G.dev.wnodes;
    out->wide_node_count = G.node_count;
    out->triangles = (void *)G.dev.tris;
    out->triangle_count = G.triangle_count;
    out->tlas_root = G.dev.tlas_root;
    out->single_group_root = 0xFFFFFFFFu;
    if (G.dev.tlas_single_group != 0xFFFFFFFFu) {
        AZ_CUDA_TRY(cudaSetDevice(G.device));
        azd::DevGroup g;
        AZ_CUDA_TRY(cudaMemcpy(&g, G.dev.groups + G.dev.tlas_single_group, sizeof(g), cudaMemcpyDeviceToHost));
        out->single_group_root = g.root;
    }
    return AZ_OK;
}

extern "C" void az_gpu_scene_destroy(az_gpu_scene *s) {
    if (!s) return;
    if (s->impl) {
        cudaSetDevice(s->impl->device);
        cudaDeviceSynchronize();
        delete s->impl;
    }
    delete s;
}

extern "C" int az_gpu_render(az_gpu_scene *scene, az_pixel *film, const az_camera *camera,
                             const az_epsilon_values *epsilons, az_scissor scissor, int32_t filter_type,
                             uint32_t backface_culling, const az_render_opts *opts, az_render_stats *stats) {
    if (!scene || !scene->impl || !film || !camera) return SetError(AZ_ERR_INVALID_ARGUMENT, "null argument");
    CallContext ctx;
    int rc = ctx.begin(opts);
    if (rc != AZ_OK) return rc;
    return Render(*scene->impl, film, camera, epsilons, scissor, filter_type, backface_culling, opts, ctx.stream,
                  stats);
}

extern "C" int az_gpu_render_samples(az_gpu_scene *scene, float *samples, const az_camera *camera,
                                     const az_epsilon_values *epsilons, az_scissor scissor,
                                     uint32_t backface_culling, const az_render_opts *opts,
                                     az_render_stats *stats) {
    if (!scene || !scene->impl || !samples || !camera) return SetError(AZ_ERR_INVALID_ARGUMENT, "null argument");
    if ((uintptr_t)samples % 16 != 0) return SetError(AZ_ERR_INVALID_ARGUMENT, "samples must be 16-byte aligned");
    CallContext ctx;
    int rc = ctx.begin(opts);
    if (rc != AZ_OK) return rc;
    return Render(*scene->impl, nullptr, camera, epsilons, scissor, AZ_Filter_Box, backface_culling, opts, ctx.stream,
                  stats, nullptr, false, nullptr, reinterpret_cast<float4 *>(samples));
}

extern "C" int az_gpu_render_host(az_gpu_scene *scene, az_pixel *pixels, const az_camera *camera,
                                  const az_epsilon_values *epsilons, az_scissor scissor, int32_t filter_type,
                                  uint32_t backface_culling, const az_render_opts *opts, az_render_stats *stats) {
    if (!scene || !scene->impl || !pixels || !camera) return SetError(AZ_ERR_INVALID_ARGUMENT, "null argument");
    CallContext ctx;
    int rc = ctx.begin(opts);
    if (rc != AZ_OK) return rc;
    GpuScene &G = *scene->impl;
    size_t bytes = (size_t)camera->Resolution.x * camera->Resolution.y * sizeof(az_pixel);
    if (G.host_film_bytes < bytes) {
        if (G.host_film_dev) cudaFree(G.host_film_dev);
        G.host_film_dev = nullptr;
        G.host_film_bytes = 0;
        AZ_CUDA_TRY(cudaMalloc((void **)&G.host_film_dev, bytes));
        G.host_film_bytes = bytes;
    }
    AZ_CUDA_TRY(cudaMemcpyAsync(G.host_film_dev, pixels, bytes, cudaMemcpyHostToDevice, ctx.stream));
    rc = Render(G, G.host_film_dev, camera, epsilons, scissor, filter_type, backface_culling, opts, ctx.stream,
                stats);
    if (rc != AZ_OK) return rc;
    AZ_CUDA_TRY(cudaMemcpyAsync(pixels, G.host_film_dev, bytes, cudaMemcpyDeviceToHost, ctx.stream));
    AZ_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
    return AZ_OK;
}

extern "C" int az_gpu_produce_image(az_pixel *pixels, const az_scene *scene, const az_camera *camera,
                                    const az_epsilon_values *epsilons, az_scissor scissor, int32_t filter_type,
                                    uint32_t backface_culling, const az_render_opts *opts) {
    if (!pixels || !scene || !camera) return SetError(AZ_ERR_INVALID_ARGUMENT, "null argument");
    CallContext ctx;
    int rc = ctx.begin(opts);
    if (rc != AZ_OK) return rc;
    GpuScene *g = nullptr;
    rc = BuildGpuScene(scene, opts, ctx.stream, &g);
    if (rc != AZ_OK) return rc;
    std::unique_ptr<GpuScene> hold(g);
    size_t bytes = (size_t)camera->Resolution.x * camera->Resolution.y * sizeof(az_pixel);
    az_pixel *d_film = nullptr;
    AZ_CUDA_TRY(cudaMallocAsync((void **)&d_film, bytes, ctx.stream));
    // the film accumulates: start from the caller's sums
    cudaError_t e = cudaMemcpyAsync(d_film, pixels, bytes, cudaMemcpyHostToDevice, ctx.stream);
    if (e != cudaSuccess) {
        cudaFreeAsync(d_film, ctx.stream);
        return CudaError(e, "film upload");
    }
    rc = Render(*g, d_film, camera, epsilons, scissor, filter_type, backface_culling, opts, ctx.stream, nullptr);
    if (rc == AZ_OK) {
        e = cudaMemcpyAsync(pixels, d_film, bytes, cudaMemcpyDeviceToHost, ctx.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx.stream);
        if (e != cudaSuccess) rc = CudaError(e, "film download");
    }
    cudaFreeAsync(d_film, ctx.stream);
    cudaStreamSynchronize(ctx.stream);
    return rc;
}

extern "C" int az_gpu_autotune(az_gpu_scene *scene, const az_camera *camera, const az_epsilon_values *epsilons,
                               az_scissor scissor, int32_t filter_type, uint32_t backface_culling,
                               const az_render_opts *opts, uint32_t *variant_out, float *ms_out) {
    if (!scene || !scene->impl || !camera) return SetError(AZ_ERR_INVALID_ARGUMENT, "null argument");
    CallContext ctx;
    int rc = ctx.begin(opts);
    if (rc != AZ_OK) return rc;
    return Autotune(*scene->impl, camera, epsilons, scissor, filter_type, backface_culling, opts, ctx.stream,
                    variant_out, ms_out);
}

extern "C" int az_gpu_autotune_scene(const az_scene *host_scene, az_gpu_scene *scene, const az_camera *camera,
                                     const az_epsilon_values *epsilons, az_scissor scissor, int32_t filter_type,
                                     uint32_t backface_culling, const az_render_opts *opts, uint32_t *width_out,
                                     uint32_t *variant_out, float *ms_out) {
    if (!host_scene || !scene || !scene->impl || !camera) return SetError(AZ_ERR_INVALID_ARGUMENT, "null argument");
    CallContext ctx;
    int rc = ctx.begin(opts);
    if (rc != AZ_OK) return rc;
    az_render_opts o;
    if (opts) o = *opts;
    else memset(&o, 0, sizeof(o));
    o.device = scene->impl->device;
    o.bvh_builder = scene->impl->bvh_builder;
    if (scene->impl->from_soup)
        return SetError(AZ_ERR_UNSUPPORTED, "a scene built from a mesh soup cannot be rebuilt from host_scene; "
                                            "use az_gpu_autotune or create it with the shape wanted");
    GpuScene *best = nullptr;
    uint32_t best_v = 0;
    float best_ms = FLT_MAX;
    // hierarchy shapes: children per node x triangles per leaf
    const uint32_t shapes[][2] = {{8, 2}, {8, 1}, {8, 3}, {4, 2}, {4, 3}, {2, 2}};
    for (const auto &shape : shapes) {
        const uint32_t width = shape[0], leaf = shape[1];
        GpuScene *g = scene->impl;
        if (width != g->bvh_width || leaf != g->bvh_leaf) {
            o.bvh_width = width;
            o.bvh_leaf = leaf;
            g = nullptr;
            rc = BuildGpuScene(host_scene, &o, ctx.stream, &g);
            if (rc != AZ_OK) break;
        }
        uint32_t v = 0;
        float ms = FLT_MAX;
        rc = Autotune(*g, camera, epsilons, scissor, filter_type, backface_culling, opts, ctx.stream, &v, &ms);
        if (rc == AZ_OK && ms < best_ms) {
            if (best && best != scene->impl) delete best;
            best = g;
            best_v = v;
            best_ms = ms;
        } else if (g != scene->impl) {
            delete g;
        }
        if (rc != AZ_OK) break;
    }
    if (rc != AZ_OK) {
        if (best && best != scene->impl) delete best;
        return rc;
    }
    if (best != scene->impl) {
        cudaStreamSynchronize(ctx.stream);
        delete scene->impl;
        scene->impl = best;
    }
    if (width_out) *width_out = best->bvh_width;
    if (variant_out) *variant_out = best_v;
    if (ms_out) *ms_out = best_ms;
    return AZ_OK;
}

extern "C" int az_gpu_render_guided(az_gpu_scene *scene, az_guide *guide, az_pixel *film, const az_camera *camera,
                                    const az_epsilon_values *epsilons, az_scissor scissor, int32_t filter_type,
                                    uint32_t backface_culling, uint32_t train, const az_render_opts *opts,
                                    az_render_stats *stats) {
    if (!scene || !scene->impl || !guide || !film || !camera) return SetError(AZ_ERR_INVALID_ARGUMENT, "null argument");
    GuideState *g = GuideOf(guide);
    if (!g) return SetError(AZ_ERR_INVALID_ARGUMENT, "null guide");
    CallContext ctx;
    int rc = ctx.begin(opts);
    if (rc != AZ_OK) return rc;
    std::lock_guard<std::mutex> lock(GuideLock(*g));
    rc = Render(*scene->impl, film, camera, epsilons, scissor, filter_type, backface_culling, opts, ctx.stream, stats,
                g, train != 0);
    if (rc == AZ_OK) rc = GuideCheck(*g, ctx.stream);
    return rc;
}

extern "C" int az_gpu_postprocess(const az_pixel *film, uint32_t width, uint32_t height, const az_tonemap *tonemap,
                                  float inv_gamma, uint32_t srgb, uint32_t linear, float *rgb_out, uint8_t *rgb8_out,
                                  const az_render_opts *opts) {
    if ((width && height) && (!film || (!rgb_out && !rgb8_out)))
        return SetError(AZ_ERR_INVALID_ARGUMENT, "null film or no output");
    if ((uint64_t)width * height > 0x7FFFFFFFull) return SetError(AZ_ERR_INVALID_ARGUMENT, "film too large");
    CallContext ctx;
    int rc = ctx.begin(opts);
    if (rc != AZ_OK) return rc;
    return PostProcess(film, width, height, tonemap, inv_gamma, srgb, linear, rgb_out, rgb8_out, ctx.stream);
}

extern "C" int az_gpu_output_pixels_to_file(const char *path, const az_pixel *film, uint32_t width, uint32_t height,
                                            const az_tonemap *tonemap, float inv_gamma, uint32_t srgb, int32_t format,
                                            uint32_t save_exr, const az_render_opts *opts) {
    if (!path || !film || width == 0 || height == 0) return SetError(AZ_ERR_INVALID_ARGUMENT, "null path or film");
    if (format < AZ_FileFormat_PNG || format > AZ_FileFormat_EXR)
        return SetError(AZ_ERR_INVALID_ARGUMENT, "unknown file format");
    if ((uint64_t)width * height > 0x7FFFFFFFull) return SetError(AZ_ERR_INVALID_ARGUMENT, "film too large");
    CallContext ctx;
    int rc = ctx.begin(opts);
    if (rc != AZ_OK) return rc;
    const size_t n = (size_t)width * height;
    if (format == AZ_FileFormat_EXR || save_exr) {
        // the normalised colours times 255, before tone mapping and gamma
        // (OutputPixelsToEXR, src/azimuth_main.cpp:1426-1458)
        std::string exr_path = path;
        if (format != AZ_FileFormat_EXR) {
            char sib[256];
            exr_path = az_exr_sibling_path(path, sib, sizeof(sib)) == AZ_OK ? std::string(sib) : std::string();
        }
        if (!exr_path.empty()) {
            float *d_rgb = nullptr;
            AZ_CUDA_TRY(cudaMalloc((void **)&d_rgb, n * 3 * sizeof(float)));
            rc = PostProcess(film, width, height, tonemap, inv_gamma, srgb, 1, d_rgb, nullptr, ctx.stream);
            std::vector<float> rgb(n * 3);
            if (rc == AZ_OK) {
                cudaError_t e = cudaMemcpy(rgb.data(), d_rgb, n * 3 * sizeof(float), cudaMemcpyDeviceToHost);
                if (e != cudaSuccess) rc = CudaError(e, "cudaMemcpy(EXR colours)");
            }
            cudaFree(d_rgb);
            if (rc != AZ_OK) return rc;
            for (float &c : rgb) c = c * 255.0f;
            if (az_write_exr(exr_path.c_str(), rgb.data(), width, height) != AZ_OK)
                return SetError(AZ_ERR_IO, "cannot write " + exr_path);
        }
        if (format == AZ_FileFormat_EXR) return AZ_OK;
    }
    uint8_t *d_rgb8 = nullptr;
    AZ_CUDA_TRY(cudaMalloc((void **)&d_rgb8, n * 3));
    rc = PostProcess(film, width, height, tonemap, inv_gamma, srgb, 0, nullptr, d_rgb8, ctx.stream);
    std::vector<uint8_t> rgb8(n * 3);
    if (rc == AZ_OK) {
        cudaError_t e = cudaMemcpy(rgb8.data(), d_rgb8, n * 3, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = CudaError(e, "cudaMemcpy(8-bit colours)");
    }
    cudaFree(d_rgb8);
    if (rc != AZ_OK) return rc;
    if (az_write_image(path, rgb8.data(), width, height, format) != AZ_OK)
        return SetError(AZ_ERR_IO, std::string("cannot write ") + path);
    return AZ_OK;
}

extern "C" int az_gpu_closest_hit(az_gpu_scene *scene, const az_ray3 *rays, uint32_t count, int32_t cull,
                                  float hit_epsilon, uint32_t *out_hit, uint32_t *out_uid, uint32_t *out_face,
                                  float *out_t, const az_render_opts *opts) {
    if (!scene || !scene->impl || (count && (!rays || !out_hit || !out_uid || !out_face || !out_t)))
        return SetError(AZ_ERR_INVALID_ARGUMENT, "null argument");
    CallContext ctx;
    int rc = ctx.begin(opts);
    if (rc != AZ_OK) return rc;
    return ClosestHit(*scene->impl, rays, count, cull, hit_epsilon, out_hit, out_uid, out_face, out_t, ctx.stream,
                      opts && (opts->flags & AZ_FLAG_WATERTIGHT));
}

extern "C" float az_rng_u01(uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t digits, uint32_t level,
                            uint32_t dim) {
    azd::NodeRng r;
    r.init(seed, pixel, sample, digits, level);
    r.skip(dim);
    return r.next();
}

extern "C" void az_rng_philox4x32_10(const uint32_t counter[4], uint32_t key0, uint32_t key1, uint32_t out[4]) {
    azd::philox4x32_10(counter[0], counter[1], counter[2], counter[3], key0, key1, out);
}
