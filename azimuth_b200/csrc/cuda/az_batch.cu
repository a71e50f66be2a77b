// Batched render jobs: many jobs of uneven resolution, sample count, depth
// and scene in one call (az_gpu_render_batch, include/azimuth_gpu.h).
//
// One host worker per CUDA stream pulls the next job from a shared queue
// ordered by estimated cost (samples x tree levels): shortest first by
// default, which minimises the jobs' completion times (a large job's waves
// fill the GPU on their own, so it loses little by starting late), or
// largest first; each worker renders with its own wave queues; the streams run concurrently on the device, so small jobs fill
// the SMs that a large job's waves leave idle.  A job of three or more waves
// replays its per-wave launches as one CUDA graph.  With opts->tiles the
// plain jobs, whatever their scenes, render together in tile waves pulled
// from a device work queue (RenderTiles) on the first stream, while the other
// streams take the guided jobs.  Completion times are device times between an
// event recorded before any job and each job's end event (for tiled jobs, the
// end of the wave holding their last tile).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "az_internal.h"

namespace az {
namespace {

struct Worker {
    cudaStream_t st = nullptr;
    WaveBuffers W;
};

uint64_t JobSamples(const az_job &j) {
    const az_camera *c = j.camera;
    uint32_t x0 = std::min(j.scissor.Min.x, c->Resolution.x), x1 = std::min(j.scissor.Max.x, c->Resolution.x);
    uint32_t y0 = std::min(j.scissor.Min.y, c->Resolution.y), y1 = std::min(j.scissor.Max.y, c->Resolution.y);
    if (x1 <= x0 || y1 <= y0) return 0;
    const uint64_t s = (uint64_t)std::floor(std::sqrt((double)c->SampleCount));
    return (uint64_t)(x1 - x0) * (y1 - y0) * s * s;
}

}  // namespace
}  // namespace az

using namespace az;

extern "C" int az_gpu_render_batch(az_job *jobs, uint32_t n, const az_batch_opts *opts, az_batch_stats *stats) {
    if (stats) memset(stats, 0, sizeof(*stats));
    if (n && !jobs) return SetError(AZ_ERR_INVALID_ARGUMENT, "null job array");
    for (uint32_t i = 0; i < n; i++) {
        const az_job &j = jobs[i];
        if (!j.scene || !j.scene->impl || !j.film || !j.camera)
            return SetError(AZ_ERR_INVALID_ARGUMENT, "job " + std::to_string(i) + ": null scene, film or camera");
        if (j.guide && !GuideOf(j.guide))
            return SetError(AZ_ERR_INVALID_ARGUMENT, "job " + std::to_string(i) + ": null guide");
    }
    if (n == 0) return AZ_OK;
    const int device = opts ? opts->device : 0;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return SetError(AZ_ERR_NO_DEVICE, "no CUDA device available");
    if (device < 0 || device >= count) return SetError(AZ_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    for (uint32_t i = 0; i < n; i++)
        if (jobs[i].scene->impl->device != device)
            return SetError(AZ_ERR_INVALID_ARGUMENT, "job " + std::to_string(i) + ": scene on another device");
    AZ_CUDA_TRY(cudaSetDevice(device));
    const uint32_t S = std::max(1u, std::min(opts && opts->streams ? opts->streams : 4u, n));
    const uint32_t chunk = opts && opts->chunk_samples ? opts->chunk_samples : (1u << 22);

    // with opts->tiles, the plain jobs go to one tile render; the queue holds the rest
    const bool tiles = opts && opts->tiles;
    std::vector<uint32_t> order, tiled;
    const bool largest_first = opts && opts->largest_first;
    std::vector<double> cost(n);
    for (uint32_t i = 0; i < n; i++) {
        if (tiles && !jobs[i].guide) tiled.push_back(i);
        else order.push_back(i);
        jobs[i].samples = JobSamples(jobs[i]);
        cost[i] = (double)jobs[i].samples * (jobs[i].scene->impl->dev.max_depth + 1);
        jobs[i].status = AZ_OK;
        jobs[i].done_ms = 0.0f;
    }
    const uint32_t queued = (uint32_t)order.size();
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return largest_first ? cost[a] > cost[b] : cost[a] < cost[b]; });

    std::vector<std::unique_ptr<Worker>> workers;
    std::vector<cudaEvent_t> done(n, nullptr);
    cudaEvent_t start = nullptr;
    int rc = AZ_OK;
    auto cleanup = [&]() {
        for (auto &w : workers)
            if (w->st) {
                cudaStreamSynchronize(w->st);
                w->W.DropGraph();
                cudaStreamDestroy(w->st);
                w->st = nullptr;
            }
        for (cudaEvent_t e : done)
            if (e) cudaEventDestroy(e);
        if (start) cudaEventDestroy(start);
    };
    for (uint32_t w = 0; w < S && rc == AZ_OK; w++) {
        workers.emplace_back(new Worker());
        // blocking streams: each waits for earlier work on the legacy default
        // stream (films zeroed there) but not for the other workers
        if (cudaStreamCreate(&workers.back()->st) != cudaSuccess)
            rc = SetError(AZ_ERR_CUDA, "stream creation");
    }
    for (uint32_t i = 0; i < n && rc == AZ_OK; i++)
        if (cudaEventCreate(&done[i]) != cudaSuccess) rc = SetError(AZ_ERR_CUDA, "event creation");
    if (rc == AZ_OK && cudaEventCreate(&start) != cudaSuccess) rc = SetError(AZ_ERR_CUDA, "event creation");
    if (rc != AZ_OK) {
        cleanup();
        return rc;
    }
    // every stream starts after `start`
    cudaEventRecord(start, workers[0]->st);
    for (uint32_t w = 1; w < S; w++) cudaStreamWaitEvent(workers[w]->st, start, 0);

    std::atomic<uint32_t> next{0};
    std::vector<std::string> messages(n);
    std::vector<char> tile_done(n, 0);
    auto render_tiled = [&](Worker *wk) {
        std::vector<TileJob> tj(tiled.size());
        for (size_t k = 0; k < tiled.size(); k++) {
            const az_job &j = jobs[tiled[k]];
            tj[k].scene = j.scene->impl;
            tj[k].film = j.film;
            tj[k].camera = j.camera;
            tj[k].eps = j.epsilons;
            tj[k].scissor = j.scissor;
            tj[k].filter = j.filter_type;
            tj[k].cull = j.backface_culling;
            tj[k].seed = j.seed;
        }
        az_render_opts o;
        memset(&o, 0, sizeof(o));
        o.device = device;
        o.flags = opts ? opts->flags : 0u;
        const int trc = RenderTiles(*tj[0].scene, tj, &o, wk->st, nullptr, start);
        const std::string msg = trc != AZ_OK ? az_gpu_last_error() : "";
        for (size_t k = 0; k < tiled.size(); k++) {
            az_job &j = jobs[tiled[k]];
            j.status = trc;
            j.done_ms = tj[k].done_ms;
            if (trc != AZ_OK) messages[tiled[k]] = msg;
            tile_done[tiled[k]] = 1;
        }
    };
    auto work = [&](Worker *wk, bool tile_first) {
        cudaSetDevice(device);
        if (tile_first) render_tiled(wk);
        for (;;) {
            const uint32_t k = next.fetch_add(1);
            if (k >= queued) break;
            az_job &j = jobs[order[k]];
            az_render_opts o;
            memset(&o, 0, sizeof(o));
            o.seed = j.seed;
            o.stream = wk->st;
            o.device = device;
            o.flags = opts ? opts->flags : 0u;
            o.chunk_samples = chunk;
            if ((j.samples + chunk - 1) / chunk < 3) o.flags |= AZ_FLAG_NO_GRAPH;   // capture would not pay
            GuideState *g = j.guide ? GuideOf(j.guide) : nullptr;
            int jrc;
            if (g) {
                std::lock_guard<std::mutex> lock(GuideLock(*g));
                jrc = Render(*j.scene->impl, j.film, j.camera, j.epsilons, j.scissor, j.filter_type,
                             j.backface_culling, &o, wk->st, nullptr, g, j.train != 0, &wk->W);
            } else {
                jrc = Render(*j.scene->impl, j.film, j.camera, j.epsilons, j.scissor, j.filter_type,
                             j.backface_culling, &o, wk->st, nullptr, nullptr, false, &wk->W);
            }
            j.status = jrc;
            if (jrc != AZ_OK) messages[order[k]] = az_gpu_last_error();
            cudaEventRecord(done[order[k]], wk->st);
        }
    };
    std::vector<std::thread> threads;
    for (uint32_t w = 0; w < S; w++) threads.emplace_back(work, workers[w].get(), w == 0 && !tiled.empty());
    for (auto &t : threads) t.join();
    std::vector<float> times;
    uint32_t failed = 0;
    int first_rc = AZ_OK;
    std::string first_msg;
    for (uint32_t i = 0; i < n; i++) {
        float ms = jobs[i].done_ms;   // a tiled job's: set by the tile render
        if (!tile_done[i]) {
            ms = 0.0f;
            if (cudaEventSynchronize(done[i]) == cudaSuccess) cudaEventElapsedTime(&ms, start, done[i]);
        }
        jobs[i].done_ms = ms;
        times.push_back(ms);
        if (jobs[i].status != AZ_OK) {
            failed++;
            if (first_rc == AZ_OK) {
                first_rc = jobs[i].status;
                first_msg = "job " + std::to_string(i) + ": " + messages[i];
            }
        }
    }
    cleanup();
    if (stats) {
        std::vector<float> s = times;
        std::sort(s.begin(), s.end());
        auto pct = [&](double p) { return s[std::min<size_t>(s.size() - 1, (size_t)std::floor(p * (s.size() - 1) + 0.5))]; };
        uint64_t samples = 0;
        for (uint32_t i = 0; i < n; i++) samples += jobs[i].samples;
        stats->samples = samples;
        stats->gpu_ms = s.back();
        stats->p50_ms = pct(0.50);
        stats->p99_ms = pct(0.99);
        stats->jobs = n;
        stats->failed = failed;
        stats->streams = S;
    }
    if (first_rc != AZ_OK) return SetError(first_rc, first_msg);
    return AZ_OK;
}

extern "C" int az_gpu_render_tiles(az_job *jobs, uint32_t n, const az_batch_opts *opts, az_batch_stats *stats) {
    if (stats) memset(stats, 0, sizeof(*stats));
    if (n && !jobs) return SetError(AZ_ERR_INVALID_ARGUMENT, "null job array");
    if (n == 0) return AZ_OK;
    GpuScene *G = jobs[0].scene && jobs[0].scene->impl ? jobs[0].scene->impl : nullptr;
    std::vector<TileJob> tj(n);
    for (uint32_t i = 0; i < n; i++) {
        const az_job &j = jobs[i];
        if (!j.scene || !j.scene->impl)
            return SetError(AZ_ERR_INVALID_ARGUMENT, "job " + std::to_string(i) + ": null scene");
        if (j.scene->impl->device != G->device)
            return SetError(AZ_ERR_INVALID_ARGUMENT, "job " + std::to_string(i) + ": scene on another device");
        tj[i].scene = j.scene->impl;
        if (!j.film || !j.camera)
            return SetError(AZ_ERR_INVALID_ARGUMENT, "job " + std::to_string(i) + ": null film or camera");
        if (j.guide) return SetError(AZ_ERR_UNSUPPORTED, "job " + std::to_string(i) + ": guided jobs are not tiled");
        tj[i].film = j.film;
        tj[i].camera = j.camera;
        tj[i].eps = j.epsilons;
        tj[i].scissor = j.scissor;
        tj[i].filter = j.filter_type;
        tj[i].cull = j.backface_culling;
        tj[i].seed = j.seed;
    }
    const int device = opts ? opts->device : 0;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return SetError(AZ_ERR_NO_DEVICE, "no CUDA device available");
    if (device < 0 || device >= count || G->device != device)
        return SetError(AZ_ERR_INVALID_ARGUMENT, "device ordinal out of range or not the scene's");
    AZ_CUDA_TRY(cudaSetDevice(device));
    az_render_opts ro;
    memset(&ro, 0, sizeof(ro));
    ro.device = device;
    ro.flags = opts ? opts->flags : 0u;
    ro.chunk_samples = opts ? opts->chunk_samples : 0u;
    // a blocking stream: ordered after earlier work on the legacy default stream (films zeroed there)
    cudaStream_t st = nullptr;
    if (cudaStreamCreate(&st) != cudaSuccess) return SetError(AZ_ERR_CUDA, "stream creation");
    az_render_stats rs;
    int rc = RenderTiles(*G, tj, &ro, st, &rs);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    std::vector<float> done;
    for (uint32_t i = 0; i < n; i++) {
        jobs[i].status = rc;
        jobs[i].samples = tj[i].samples;
        jobs[i].done_ms = tj[i].done_ms;
        done.push_back(tj[i].done_ms);
    }
    if (stats) {
        std::sort(done.begin(), done.end());
        stats->samples = rc == AZ_OK ? rs.samples : 0;
        stats->gpu_ms = rc == AZ_OK ? rs.gpu_ms : 0.0f;
        stats->p50_ms = done[(n - 1) / 2];
        stats->p99_ms = done[std::min<size_t>(n - 1, (size_t)(0.99 * n))];
        stats->jobs = n;
        stats->failed = rc == AZ_OK ? 0u : n;
        stats->streams = 1;
    }
    return rc;
}
