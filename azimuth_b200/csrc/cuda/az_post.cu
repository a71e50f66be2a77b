// Film post-processing on the GPU: OutputPixelsToFile's normalisation,
// photographic tone mapping and gamma correction (src/azimuth_main.cpp:
// 1620-1760) and the writers' 8-bit conversion (:1473-1475), for a device
// film that stays untouched.
//
//   k_post_normalise  colour / TotalWeight, luminance 0.27 R + 0.67 G + 0.06 B
//                     (src/azimuth_math.cpp:1866-1880), sum of log(L + 1e-5) in
//                     double (azimuth accumulates it serially in float)
//   CUB radix sort    of the luminances, for the burn-out luminance at index
//                     round((1 - burnout / 100) (N - 1)) (azimuth: qsort)
//   k_post_map        Ld = Ls (1 + Ls / Lwhite^2) / (1 + Ls), (C / L)^saturation
//                     Ld clamped, then sRGB or 1/gamma, then (u8)(clamp01(C) 255)
#include <cub/cub.cuh>

#include <cmath>
#include <cstring>

#include "az_internal.h"

namespace az {
namespace {

__device__ __forceinline__ float lum3(float r, float g, float b) { return r * 0.27f + g * 0.67f + b * 0.06f; }
__device__ __forceinline__ float clamp01(float v) { return fminf(1.0f, fmaxf(0.0f, v)); }

__global__ void k_post_normalise(const float4 *film, uint32_t n, float *rgb, float *lums, double *logsum) {
    double part = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = film[i];
        const float r = p.x / p.w, g = p.y / p.w, b = p.z / p.w;
        rgb[3 * i + 0] = r;
        rgb[3 * i + 1] = g;
        rgb[3 * i + 2] = b;
        if (lums) {
            const float l = lum3(r, g, b);
            lums[i] = l;
            part += (double)logf(l + 0.00001f);
        }
    }
    if (!lums) return;
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xFFFFFFFFu, part, o);
    if ((threadIdx.x & 31u) == 0) atomicAdd(logsum, part);
}

struct MapParams {
    uint32_t n;
    int tonemapped;
    float factor, lw2, saturation;
    float inv_gamma;
    uint32_t srgb, linear;
};

__global__ void k_post_map(float *rgb, uint8_t *rgb8, MapParams P) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
        float c[3] = {rgb[3 * i + 0], rgb[3 * i + 1], rgb[3 * i + 2]};
        if (P.tonemapped) {
            const float l = lum3(c[0], c[1], c[2]);
            if (l != 0.0f) {
                const float ls = l * P.factor;
                const float ld = (ls * (1.0f + (ls / P.lw2))) / (1.0f + ls);
                for (int k = 0; k < 3; k++) c[k] = clamp01(powf(c[k] / l, P.saturation) * ld);
            }
        }
        for (int k = 0; k < 3; k++) {
            float v = c[k];
            if (!P.linear) {
                if (P.srgb) v = v > 0.0031308f ? 1.055f * powf(v, P.inv_gamma) - 0.055f : v * 12.92f;
                else v = powf(v, P.inv_gamma);
            }
            rgb[3 * i + k] = v;
            if (rgb8) rgb8[3 * i + k] = (uint8_t)(clamp01(v) * 255.0f);
        }
    }
}

}  // namespace

int PostProcess(const az_pixel *film, uint32_t w, uint32_t h, const az_tonemap *tm, float inv_gamma, uint32_t srgb,
                uint32_t linear, float *rgb_out, uint8_t *rgb8_out, cudaStream_t st) {
    const uint32_t n = w * h;
    if (n == 0) return AZ_OK;
    const bool tonemapped = !linear && tm && tm->Operator != AZ_Tonemap_None;
    if (tm && tm->Operator > AZ_Tonemap_Photographic) return SetError(AZ_ERR_INVALID_ARGUMENT, "unknown tone-mapping operator");
    // scratch: colours (when the caller wants bytes only), luminances, sorted copy, sort temp, log sum
    float *rgb = rgb_out, *lums = nullptr, *sorted = nullptr;
    double *logsum = nullptr;
    void *temp = nullptr;
    size_t temp_bytes = 0;
    int rc = AZ_OK;
    auto fail = [&](cudaError_t e, const char *what) {
        rc = CudaError(e, what);
    };
    cudaError_t e = cudaSuccess;
    if (!rgb && (e = cudaMalloc((void **)&rgb, (size_t)n * 3 * sizeof(float))) != cudaSuccess) fail(e, "post-process colours");
    if (rc == AZ_OK && tonemapped) {
        if ((e = cudaMalloc((void **)&lums, (size_t)n * sizeof(float))) != cudaSuccess) fail(e, "post-process luminances");
        else if ((e = cudaMalloc((void **)&sorted, (size_t)n * sizeof(float))) != cudaSuccess) fail(e, "post-process sort");
        else if ((e = cudaMalloc((void **)&logsum, sizeof(double))) != cudaSuccess) fail(e, "post-process sum");
        else if ((e = cub::DeviceRadixSort::SortKeys(nullptr, temp_bytes, lums, sorted, (int)n, 0, 32, st)) != cudaSuccess)
            fail(e, "post-process sort size");
        else if ((e = cudaMalloc(&temp, temp_bytes)) != cudaSuccess) fail(e, "post-process sort scratch");
    }
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = sms * 8;
    MapParams P;
    memset(&P, 0, sizeof(P));
    P.n = n;
    P.inv_gamma = inv_gamma;
    P.srgb = srgb;
    P.linear = linear;
    if (rc == AZ_OK && tonemapped) {
        if ((e = cudaMemsetAsync(logsum, 0, sizeof(double), st)) != cudaSuccess) fail(e, "post-process");
    }
    if (rc == AZ_OK) {
        k_post_normalise<<<grid, 256, 0, st>>>(reinterpret_cast<const float4 *>(film), n, rgb, tonemapped ? lums : nullptr,
                                               logsum);
        if ((e = cudaGetLastError()) != cudaSuccess) fail(e, "k_post_normalise");
    }
    if (rc == AZ_OK && tonemapped) {
        // luminances are >= 0, so their IEEE bit patterns sort in value order
        if ((e = cub::DeviceRadixSort::SortKeys(temp, temp_bytes, lums, sorted, (int)n, 0, 32, st)) != cudaSuccess)
            fail(e, "post-process sort");
        const uint32_t li = (uint32_t)((1.0f - tm->BurnoutPercentage * 0.01f) * (float)(n - 1) + 0.5f);
        double sum = 0.0;
        float lwhite = 0.0f;
        if (rc == AZ_OK && (e = cudaMemcpyAsync(&sum, logsum, sizeof(double), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            fail(e, "post-process");
        if (rc == AZ_OK && (e = cudaMemcpyAsync(&lwhite, sorted + std::min(li, n - 1), sizeof(float),
                                                cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            fail(e, "post-process");
        if (rc == AZ_OK && (e = cudaStreamSynchronize(st)) != cudaSuccess) fail(e, "post-process");
        if (rc == AZ_OK) {
            const float logavg = expf((float)sum / (float)n);
            P.tonemapped = 1;
            P.factor = tm->KeyValue / logavg;
            P.lw2 = lwhite * P.factor;
            P.lw2 = P.lw2 * P.lw2;
            P.saturation = tm->Saturation;
        }
    }
    if (rc == AZ_OK) {
        k_post_map<<<grid, 256, 0, st>>>(rgb, rgb8_out, P);
        if ((e = cudaGetLastError()) != cudaSuccess) fail(e, "k_post_map");
    }
    if (rc == AZ_OK && (e = cudaStreamSynchronize(st)) != cudaSuccess) fail(e, "post-process");
    if (rgb != rgb_out && rgb) cudaFree(rgb);
    if (lums) cudaFree(lums);
    if (sorted) cudaFree(sorted);
    if (logsum) cudaFree(logsum);
    if (temp) cudaFree(temp);
    return rc;
}

}  // namespace az
