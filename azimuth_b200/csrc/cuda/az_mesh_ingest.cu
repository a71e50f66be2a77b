// The importer's mesh post-processing on the GPU (src/azimuth_xml.cpp:3632-3776),
// bit for bit:
//
//   k_ingest_faces     per face: Cross(P1 - P0, P2 - P0), its length, |N| / 2
//                      and the unit face normal (Normalize's divisions), and
//                      the face's three (vertex, corner) incidences
//   radix sort         of the incidences by vertex; the sort is stable, so each
//                      vertex's incidences stay in face order, then corner order
//   k_ingest_vertices  per vertex: the sum of its faces' unnormalised normals in
//                      that order, starting from 0 (azimuth's serial `+=` loop
//                      gives each vertex exactly this sequence of additions),
//                      then Normalize
//   k_ingest_area      per mesh: TotalArea, the float sum of |N| / 2 over its
//                      faces in order (one thread per mesh, serial like azimuth)
//   k_ingest_emit_*    per face: azimuth's triangle {P0, P1, P2, N} and the
//                      entity fields N0-N2 (vertex normals) and UV0-UV2
//                      (UVs[i + UVOffset] when in range), either as host-visible
//                      records or directly as the device scene's primitives.
//
// Arithmetic is plain IEEE float with no contraction (the library is built
// with --fmad=false), as azimuth's own build of these loops is.
#include <cub/cub.cuh>

#include <algorithm>
#include <cfloat>
#include <cstring>

#include "az_internal.h"

namespace az {
namespace {

struct MeshRange {
    uint32_t face_base, face_count;
    int32_t uv_offset;
    uint32_t index;   // position in the soup's mesh array
};

// The mesh owning face f (ranges sorted by face_base), or -1.
__device__ __forceinline__ int mesh_of(const MeshRange *m, uint32_t nm, uint32_t f) {
    int lo = 0, hi = (int)nm - 1, found = -1;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        if (m[mid].face_base <= f) {
            found = mid;
            lo = mid + 1;
        } else {
            hi = mid - 1;
        }
    }
    if (found >= 0 && f - m[found].face_base < m[found].face_count) return found;
    return -1;
}

__global__ void k_ingest_faces(const float *v, uint32_t nv, const uint32_t *faces, uint32_t nf, float *fn_raw,
                               float *half_area, float *fn_unit, uint32_t *inc_key, uint32_t *inc_val,
                               uint32_t *err) {
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const uint32_t i0 = faces[3 * f + 0], i1 = faces[3 * f + 1], i2 = faces[3 * f + 2];
    for (int c = 0; c < 3; c++) {
        inc_key[3 * f + c] = faces[3 * f + c];
        inc_val[3 * f + c] = 3 * f + c;
    }
    if (i0 >= nv || i1 >= nv || i2 >= nv) {
        atomicOr(err, 1u);
        return;
    }
    const float p0x = v[3 * i0], p0y = v[3 * i0 + 1], p0z = v[3 * i0 + 2];
    const float ax = v[3 * i1] - p0x, ay = v[3 * i1 + 1] - p0y, az_ = v[3 * i1 + 2] - p0z;   // P1 - P0
    const float bx = v[3 * i2] - p0x, by = v[3 * i2 + 1] - p0y, bz = v[3 * i2 + 2] - p0z;   // P2 - P0
    // Cross (src/azimuth_math.cpp:1325-1333)
    const float nx = ay * bz - az_ * by, ny = az_ * bx - ax * bz, nz = ax * by - ay * bx;
    fn_raw[3 * f + 0] = nx;
    fn_raw[3 * f + 1] = ny;
    fn_raw[3 * f + 2] = nz;
    const float len = sqrtf(nx * nx + ny * ny + nz * nz);   // Length
    half_area[f] = len / 2.0f;
    fn_unit[3 * f + 0] = nx / len;
    fn_unit[3 * f + 1] = ny / len;
    fn_unit[3 * f + 2] = nz / len;
}

// First and one-past-last position of each vertex's incidences in the sorted list.
__global__ void k_ingest_segments(const uint32_t *sorted_key, uint32_t n, uint32_t *start, uint32_t *end) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t k = sorted_key[i];
    if (i == 0 || sorted_key[i - 1] != k) start[k] = i;
    if (i == n - 1 || sorted_key[i + 1] != k) end[k] = i + 1;
}

__global__ void k_ingest_vertices(const uint32_t *start, const uint32_t *end, const uint32_t *sorted_val,
                                  const float *fn_raw, uint32_t nv, float *vn) {
    const uint32_t vi = blockIdx.x * blockDim.x + threadIdx.x;
    if (vi >= nv) return;
    float x = 0.0f, y = 0.0f, z = 0.0f;
    for (uint32_t i = start[vi]; i < end[vi]; i++) {
        const uint32_t f = sorted_val[i] / 3u;
        x = x + fn_raw[3 * f + 0];
        y = y + fn_raw[3 * f + 1];
        z = z + fn_raw[3 * f + 2];
    }
    // Normalize (src/azimuth_math.cpp:1299-1313)
    const float L = sqrtf(x * x + y * y + z * z);
    if (L != 0.0f) {
        x = x / L;
        y = y / L;
        z = z / L;
    } else {
        x = y = z = 0.0f;
    }
    vn[3 * vi + 0] = x;
    vn[3 * vi + 1] = y;
    vn[3 * vi + 2] = z;
}

__global__ void k_ingest_area(const MeshRange *m, uint32_t nm, const float *half_area, float *total) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nm) return;
    float a = 0.0f;
    const uint32_t b = m[i].face_base, n = m[i].face_count;
    for (uint32_t k = 0; k < n; k++) a += half_area[b + k];
    total[m[i].index] = a;
}

__device__ __forceinline__ void face_uvs(const float *uv, uint32_t nuv, int32_t off, const uint32_t idx[3],
                                         float out[6]) {
    for (int c = 0; c < 3; c++) {
        const int32_t u = (int32_t)idx[c] + off;
        const bool ok = u >= 0 && (uint32_t)u < nuv;
        out[2 * c + 0] = ok ? uv[2 * u + 0] : 0.0f;
        out[2 * c + 1] = ok ? uv[2 * u + 1] : 0.0f;
    }
}

// Host-visible records of faces [f0, f0 + n) in face order: az_triangle and az_face_attr.
__global__ void k_ingest_emit_records(const float *v, const uint32_t *faces, uint32_t f0, uint32_t n,
                                      const float *fn_unit, const float *vn, const float *uv, uint32_t nuv,
                                      const MeshRange *m, uint32_t nm, az_triangle *tris, az_face_attr *attrs) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const uint32_t f = f0 + j;
    const uint32_t idx[3] = {faces[3 * f], faces[3 * f + 1], faces[3 * f + 2]};
    if (tris) {
        az_triangle t;
        t.P0 = az_vec3{v[3 * idx[0]], v[3 * idx[0] + 1], v[3 * idx[0] + 2]};
        t.P1 = az_vec3{v[3 * idx[1]], v[3 * idx[1] + 1], v[3 * idx[1] + 2]};
        t.P2 = az_vec3{v[3 * idx[2]], v[3 * idx[2] + 1], v[3 * idx[2] + 2]};
        t.N = az_vec3{fn_unit[3 * f], fn_unit[3 * f + 1], fn_unit[3 * f + 2]};
        tris[j] = t;
    }
    if (attrs) {
        const int mi = mesh_of(m, nm, f);
        float u[6] = {0, 0, 0, 0, 0, 0};
        if (mi >= 0) face_uvs(uv, nuv, m[mi].uv_offset, idx, u);
        az_face_attr a;
        a.N0 = az_vec3{vn[3 * idx[0]], vn[3 * idx[0] + 1], vn[3 * idx[0] + 2]};
        a.N1 = az_vec3{vn[3 * idx[1]], vn[3 * idx[1] + 1], vn[3 * idx[1] + 2]};
        a.N2 = az_vec3{vn[3 * idx[2]], vn[3 * idx[2] + 1], vn[3 * idx[2] + 2]};
        a.UV0 = az_vec2{u[0], u[1]};
        a.UV1 = az_vec2{u[2], u[3]};
        a.UV2 = az_vec2{u[4], u[5]};
        attrs[j] = a;
    }
}

// Device-scene primitives of every face that belongs to a mesh, at the
// mesh's place in its group (out_base[mesh index] + face offset): the exact
// vertices and face normal and the shading attributes, exactly as the host
// flattening makes them from triangle entities.
__global__ void k_ingest_emit_scene(const float *v, const uint32_t *faces, uint32_t nf, const float *fn_unit,
                                    const float *vn, const float *uv, uint32_t nuv, const MeshRange *m, uint32_t nm,
                                    const IngestMesh *meshes, azd::DevTriVerts *tris, azd::DevTriAttr *attrs) {
    const uint32_t f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const int mi = mesh_of(m, nm, f);
    if (mi < 0) return;
    const IngestMesh &M = meshes[m[mi].index];
    const uint32_t local = f - m[mi].face_base, o = M.out_base + local;
    const uint32_t idx[3] = {faces[3 * f], faces[3 * f + 1], faces[3 * f + 2]};
    const float p0x = v[3 * idx[0]], p0y = v[3 * idx[0] + 1], p0z = v[3 * idx[0] + 2];
    const float p1x = v[3 * idx[1]], p1y = v[3 * idx[1] + 1], p1z = v[3 * idx[1] + 2];
    const float p2x = v[3 * idx[2]], p2y = v[3 * idx[2] + 1], p2z = v[3 * idx[2] + 2];
    azd::DevTriVerts t;
    t.a = make_float4(p0x, p0y, p0z, p1x);
    t.b = make_float4(p1y, p1z, p2x, p2y);
    t.c = make_float4(p2z, fn_unit[3 * f], fn_unit[3 * f + 1], fn_unit[3 * f + 2]);
    tris[o] = t;
    float u[6];
    face_uvs(uv, nuv, m[mi].uv_offset, idx, u);
    azd::DevTriAttr a;
    memset(&a, 0, sizeof(a));
    for (int k = 0; k < 3; k++) {
        a.n0[k] = vn[3 * idx[0] + k];
        a.n1[k] = vn[3 * idx[1] + k];
        a.n2[k] = vn[3 * idx[2] + k];
    }
    a.uv0[0] = u[0]; a.uv0[1] = u[1];
    a.uv1[0] = u[2]; a.uv1[1] = u[3];
    a.uv2[0] = u[4]; a.uv2[1] = u[5];
    a.shading_mode = M.shading_mode;
    a.texture_index = M.texture_index;
    a.face_id = local;
    a.entity = M.entity;
    attrs[o] = a;
}

// One thread per copied primitive; `start` holds each copy's first thread
// (exclusive prefix of the counts), so a thread finds its copy by bisection.
__global__ void k_ingest_copy(const IngestCopy *copies, const uint32_t *start, uint32_t nc, uint32_t total,
                              azd::DevTriVerts *tris, azd::DevTriAttr *attrs) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    int lo = 0, hi = (int)nc - 1, c = 0;
    while (lo <= hi) {
        const int mid = (lo + hi) >> 1;
        if (start[mid] <= t) {
            c = mid;
            lo = mid + 1;
        } else {
            hi = mid - 1;
        }
    }
    const IngestCopy &C = copies[c];
    const uint32_t k = t - start[c];
    if (k >= C.count) return;
    tris[C.dst + k] = tris[C.src + k];
    azd::DevTriAttr a = attrs[C.src + k];
    a.entity = C.entity;
    attrs[C.dst + k] = a;
}

template <typename T>
struct Dev {
    T *p = nullptr;
    ~Dev() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t n) { return cudaMalloc((void **)&p, (n ? n : 1) * sizeof(T)); }
};

}  // namespace

struct SoupWork {
    uint32_t nv = 0, nf = 0, nuv = 0, nm = 0;
    Dev<float> v, uv, fn_raw, fn_unit, half_area, vn, area;
    Dev<uint32_t> faces;
    Dev<MeshRange> ranges;
};

void FreeSoupWork(SoupWork *w) { delete w; }

int IngestSoup(const az_mesh_soup *soup, cudaStream_t st, SoupWork **out) {
    *out = nullptr;
    if (!soup) return SetError(AZ_ERR_INVALID_ARGUMENT, "null mesh soup");
    if ((soup->vertex_count && !soup->vertices) || (soup->face_count && !soup->faces) ||
        (soup->uv_count && !soup->uvs) || (soup->mesh_count && !soup->meshes))
        return SetError(AZ_ERR_INVALID_ARGUMENT, "mesh soup array missing");
    if (soup->face_count >= (1u << 27)) return SetError(AZ_ERR_UNSUPPORTED, "more than 2^27 faces");
    // mesh ranges: inside the face array, not overlapping
    std::vector<MeshRange> ranges(soup->mesh_count);
    for (uint32_t i = 0; i < soup->mesh_count; i++) {
        const az_mesh_desc &d = soup->meshes[i];
        if ((uint64_t)d.face_base + d.face_count > soup->face_count)
            return SetError(AZ_ERR_INVALID_SCENE, "mesh face range outside the face array");
        ranges[i] = MeshRange{d.face_base, d.face_count, d.uv_offset, i};
    }
    std::stable_sort(ranges.begin(), ranges.end(),
                     [](const MeshRange &a, const MeshRange &b) { return a.face_base < b.face_base; });
    for (size_t i = 1; i < ranges.size(); i++)
        if (ranges[i - 1].face_base + ranges[i - 1].face_count > ranges[i].face_base &&
            ranges[i - 1].face_count && ranges[i].face_count)
            return SetError(AZ_ERR_INVALID_SCENE, "mesh face ranges overlap");
    std::unique_ptr<SoupWork> W(new SoupWork());
    W->nv = soup->vertex_count;
    W->nf = soup->face_count;
    W->nuv = soup->uv_count;
    W->nm = soup->mesh_count;
    const uint32_t nv = W->nv, nf = W->nf, n_inc = 3 * nf;
    Dev<uint32_t> key, val, skey, sval, vstart, vend, err;
    AZ_CUDA_TRY(W->v.alloc((size_t)3 * nv));
    AZ_CUDA_TRY(W->uv.alloc((size_t)2 * W->nuv));
    AZ_CUDA_TRY(W->faces.alloc((size_t)3 * nf));
    AZ_CUDA_TRY(W->fn_raw.alloc((size_t)3 * nf));
    AZ_CUDA_TRY(W->fn_unit.alloc((size_t)3 * nf));
    AZ_CUDA_TRY(W->half_area.alloc(nf));
    AZ_CUDA_TRY(W->vn.alloc((size_t)3 * nv));
    AZ_CUDA_TRY(W->area.alloc(W->nm));
    AZ_CUDA_TRY(W->ranges.alloc(W->nm));
    AZ_CUDA_TRY(key.alloc(n_inc));
    AZ_CUDA_TRY(val.alloc(n_inc));
    AZ_CUDA_TRY(skey.alloc(n_inc));
    AZ_CUDA_TRY(sval.alloc(n_inc));
    AZ_CUDA_TRY(vstart.alloc(nv));
    AZ_CUDA_TRY(vend.alloc(nv));
    AZ_CUDA_TRY(err.alloc(1));
    if (nv) AZ_CUDA_TRY(cudaMemcpyAsync(W->v.p, soup->vertices, (size_t)nv * 12, cudaMemcpyHostToDevice, st));
    if (W->nuv) AZ_CUDA_TRY(cudaMemcpyAsync(W->uv.p, soup->uvs, (size_t)W->nuv * 8, cudaMemcpyHostToDevice, st));
    if (nf) AZ_CUDA_TRY(cudaMemcpyAsync(W->faces.p, soup->faces, (size_t)nf * 12, cudaMemcpyHostToDevice, st));
    if (W->nm)
        AZ_CUDA_TRY(cudaMemcpyAsync(W->ranges.p, ranges.data(), ranges.size() * sizeof(MeshRange),
                                    cudaMemcpyHostToDevice, st));
    AZ_CUDA_TRY(cudaMemsetAsync(err.p, 0, sizeof(uint32_t), st));
    AZ_CUDA_TRY(cudaMemsetAsync(vstart.p, 0, (size_t)(nv ? nv : 1) * sizeof(uint32_t), st));
    AZ_CUDA_TRY(cudaMemsetAsync(vend.p, 0, (size_t)(nv ? nv : 1) * sizeof(uint32_t), st));
    const int B = 256;
    if (nf) {
        k_ingest_faces<<<(nf + B - 1) / B, B, 0, st>>>(W->v.p, nv, W->faces.p, nf, W->fn_raw.p, W->half_area.p,
                                                       W->fn_unit.p, key.p, val.p, err.p);
        AZ_CUDA_TRY(cudaGetLastError());
        uint32_t err_h = 0;
        AZ_CUDA_TRY(cudaMemcpyAsync(&err_h, err.p, sizeof(err_h), cudaMemcpyDeviceToHost, st));
        AZ_CUDA_TRY(cudaStreamSynchronize(st));
        if (err_h) return SetError(AZ_ERR_INVALID_SCENE, "a face refers to a vertex past the vertex array");
        int end_bit = 1;
        while (end_bit < 32 && (nv >> end_bit)) end_bit++;
        size_t temp_bytes = 0;
        AZ_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, key.p, skey.p, val.p, sval.p, (int)n_inc, 0,
                                                    end_bit, st));
        Dev<unsigned char> temp;
        AZ_CUDA_TRY(temp.alloc(temp_bytes));
        AZ_CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp.p, temp_bytes, key.p, skey.p, val.p, sval.p, (int)n_inc, 0,
                                                    end_bit, st));
        k_ingest_segments<<<(n_inc + B - 1) / B, B, 0, st>>>(skey.p, n_inc, vstart.p, vend.p);
        AZ_CUDA_TRY(cudaGetLastError());
        AZ_CUDA_TRY(cudaStreamSynchronize(st));   // temp is freed on return
    }
    if (nv) {
        k_ingest_vertices<<<(nv + B - 1) / B, B, 0, st>>>(vstart.p, vend.p, sval.p, W->fn_raw.p, nv, W->vn.p);
        AZ_CUDA_TRY(cudaGetLastError());
    }
    if (W->nm) {
        k_ingest_area<<<(W->nm + 63) / 64, 64, 0, st>>>(W->ranges.p, W->nm, W->half_area.p, W->area.p);
        AZ_CUDA_TRY(cudaGetLastError());
    }
    AZ_CUDA_TRY(cudaStreamSynchronize(st));
    *out = W.release();
    return AZ_OK;
}

int SoupAreas(const SoupWork &w, std::vector<float> &areas) {
    areas.assign(w.nm, 0.0f);
    if (w.nm) AZ_CUDA_TRY(cudaMemcpy(areas.data(), w.area.p, w.nm * sizeof(float), cudaMemcpyDeviceToHost));
    return AZ_OK;
}

int SoupRecords(const SoupWork &w, az_triangle *tris, az_face_attr *attrs, az_vec3 *vertex_normals,
                cudaStream_t st) {
    if (vertex_normals && w.nv)
        AZ_CUDA_TRY(cudaMemcpy(vertex_normals, w.vn.p, (size_t)w.nv * 12, cudaMemcpyDeviceToHost));
    if ((!tris && !attrs) || w.nf == 0) return AZ_OK;
    Dev<az_triangle> dt;
    Dev<az_face_attr> da;
    if (tris) AZ_CUDA_TRY(dt.alloc(w.nf));
    if (attrs) AZ_CUDA_TRY(da.alloc(w.nf));
    k_ingest_emit_records<<<(w.nf + 255) / 256, 256, 0, st>>>(w.v.p, w.faces.p, 0, w.nf, w.fn_unit.p, w.vn.p, w.uv.p,
                                                             w.nuv, w.ranges.p, w.nm, dt.p, da.p);
    AZ_CUDA_TRY(cudaGetLastError());
    AZ_CUDA_TRY(cudaStreamSynchronize(st));
    if (tris) AZ_CUDA_TRY(cudaMemcpy(tris, dt.p, (size_t)w.nf * sizeof(az_triangle), cudaMemcpyDeviceToHost));
    if (attrs) AZ_CUDA_TRY(cudaMemcpy(attrs, da.p, (size_t)w.nf * sizeof(az_face_attr), cudaMemcpyDeviceToHost));
    return AZ_OK;
}

// Per-mesh bounds of the faces' vertices (the min / max of Box::grow in the
// host flattening, order-independent), one block per mesh.
__global__ void k_ingest_boxes(const float *v, const uint32_t *faces, const MeshRange *m, float *boxes) {
    const MeshRange r = m[blockIdx.x];
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t f = r.face_base + threadIdx.x; f < r.face_base + r.face_count; f += blockDim.x)
        for (int c = 0; c < 3; c++) {
            const uint32_t i = faces[3 * f + c];
            for (int a = 0; a < 3; a++) {
                lo[a] = fminf(lo[a], v[3 * i + a]);
                hi[a] = fmaxf(hi[a], v[3 * i + a]);
            }
        }
    __shared__ float s[6][256];
    for (int a = 0; a < 3; a++) {
        s[a][threadIdx.x] = lo[a];
        s[3 + a][threadIdx.x] = hi[a];
    }
    __syncthreads();
    for (uint32_t k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k)
            for (int a = 0; a < 3; a++) {
                s[a][threadIdx.x] = fminf(s[a][threadIdx.x], s[a][threadIdx.x + k]);
                s[3 + a][threadIdx.x] = fmaxf(s[3 + a][threadIdx.x], s[3 + a][threadIdx.x + k]);
            }
        __syncthreads();
    }
    if (threadIdx.x < 6) boxes[6 * r.index + threadIdx.x] = s[threadIdx.x][0];
}

int SoupBoxes(const SoupWork &w, std::vector<float> &boxes, cudaStream_t st) {
    boxes.assign(6 * (size_t)w.nm, 0.0f);
    if (w.nm == 0) return AZ_OK;
    Dev<float> d;
    AZ_CUDA_TRY(d.alloc(boxes.size()));
    k_ingest_boxes<<<w.nm, 256, 0, st>>>(w.v.p, w.faces.p, w.ranges.p, d.p);
    AZ_CUDA_TRY(cudaGetLastError());
    AZ_CUDA_TRY(cudaMemcpyAsync(boxes.data(), d.p, boxes.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
    AZ_CUDA_TRY(cudaStreamSynchronize(st));
    return AZ_OK;
}

int SoupTriangles(const SoupWork &w, uint32_t face_base, uint32_t count, az_triangle *tris, cudaStream_t st) {
    if (count == 0) return AZ_OK;
    if ((uint64_t)face_base + count > w.nf) return SetError(AZ_ERR_INVALID_SCENE, "face range outside the soup");
    Dev<az_triangle> dt;
    AZ_CUDA_TRY(dt.alloc(count));
    k_ingest_emit_records<<<(count + 255) / 256, 256, 0, st>>>(w.v.p, w.faces.p, face_base, count, w.fn_unit.p,
                                                              w.vn.p, w.uv.p, w.nuv, w.ranges.p, w.nm, dt.p, nullptr);
    AZ_CUDA_TRY(cudaGetLastError());
    AZ_CUDA_TRY(cudaStreamSynchronize(st));
    AZ_CUDA_TRY(cudaMemcpy(tris, dt.p, (size_t)count * sizeof(az_triangle), cudaMemcpyDeviceToHost));
    return AZ_OK;
}

int SoupEmitScene(const SoupWork &w, const std::vector<IngestMesh> &meshes, azd::DevTriVerts *d_tris,
                  azd::DevTriAttr *d_attr, cudaStream_t st) {
    if (w.nf == 0 || w.nm == 0) return AZ_OK;
    Dev<IngestMesh> dm;
    AZ_CUDA_TRY(dm.alloc(meshes.size()));
    AZ_CUDA_TRY(cudaMemcpyAsync(dm.p, meshes.data(), meshes.size() * sizeof(IngestMesh), cudaMemcpyHostToDevice, st));
    k_ingest_emit_scene<<<(w.nf + 255) / 256, 256, 0, st>>>(w.v.p, w.faces.p, w.nf, w.fn_unit.p, w.vn.p, w.uv.p, w.nuv,
                                                           w.ranges.p, w.nm, dm.p, d_tris, d_attr);
    AZ_CUDA_TRY(cudaGetLastError());
    AZ_CUDA_TRY(cudaStreamSynchronize(st));
    return AZ_OK;
}

int SoupCopyPlacements(const std::vector<IngestCopy> &copies, azd::DevTriVerts *d_tris, azd::DevTriAttr *d_attr,
                       cudaStream_t st) {
    if (copies.empty()) return AZ_OK;
    std::vector<uint32_t> start(copies.size());
    uint64_t total = 0;
    for (size_t i = 0; i < copies.size(); i++) {
        start[i] = (uint32_t)total;
        total += copies[i].count;
    }
    if (total >= (1ull << 31)) return SetError(AZ_ERR_UNSUPPORTED, "more than 2^31 instanced primitives");
    if (total == 0) return AZ_OK;
    Dev<IngestCopy> dc;
    Dev<uint32_t> ds;
    AZ_CUDA_TRY(dc.alloc(copies.size()));
    AZ_CUDA_TRY(ds.alloc(copies.size()));
    AZ_CUDA_TRY(cudaMemcpyAsync(dc.p, copies.data(), copies.size() * sizeof(IngestCopy), cudaMemcpyHostToDevice, st));
    AZ_CUDA_TRY(cudaMemcpyAsync(ds.p, start.data(), start.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    k_ingest_copy<<<(uint32_t)((total + 255) / 256), 256, 0, st>>>(dc.p, ds.p, (uint32_t)copies.size(),
                                                                    (uint32_t)total, d_tris, d_attr);
    AZ_CUDA_TRY(cudaGetLastError());
    AZ_CUDA_TRY(cudaStreamSynchronize(st));
    return AZ_OK;
}

}  // namespace az
