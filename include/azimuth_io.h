/*
 * azimuth_io.h -- image output of the B200 render path.
 *
 * OutputPixelsToFile (src/azimuth_main.cpp:1620-1797) in two parts: the
 * post-process of a device film on the GPU and this library's own image
 * writers in place of azimuth's stb_image_write and OpenEXR calls
 * (OutputPixelsToPNG/BMP/TGA/JPG/EXR, src/azimuth_main.cpp:1426-1618).
 * Every function returns an AZ_* status (azimuth_gpu.h); a file that cannot
 * be written gives AZ_ERR_IO.
 */
#ifndef AZIMUTH_IO_H
#define AZIMUTH_IO_H

#include "azimuth_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* azimuth's file_format (src/azimuth_io.h:1-7), same values. */
enum {
    AZ_FileFormat_PNG = 0,
    AZ_FileFormat_BMP = 1,
    AZ_FileFormat_TGA = 2,
    AZ_FileFormat_JPG = 3,
    AZ_FileFormat_EXR = 4
};

/* 8-bit RGB, W*H*3 bytes, top row first (the Pixels255 buffer of
 * OutputPixelsToPNG/BMP/TGA/JPG), written as PNG, 24-bit BMP, run-length
 * encoded TGA or baseline JPEG of quality 100 (what OutputPixelsToJPG asks
 * of stb_image_write). */
int az_write_image(const char *path, const uint8_t *rgb8, uint32_t width, uint32_t height, int32_t format);
/* Baseline JPEG at another quality (1..100, the usual scaling of the
 * ITU-T T.81 Annex K tables). */
int az_write_jpg_quality(const char *path, const uint8_t *rgb8, uint32_t width, uint32_t height, int32_t quality);
/* Float RGB, W*H*3 values, as an uncompressed scanline OpenEXR file with HALF
 * channels R, G, B holding the values as given (OutputPixelsToEXR writes
 * colour * 255, src/azimuth_main.cpp:1436-1440). */
int az_write_exr(const char *path, const float *rgb, uint32_t width, uint32_t height);
/* The name OutputPixelsToFile gives the EXR written beside another format
 * (src/azimuth_main.cpp:1660-1683): the three characters after the last '.'
 * become "exr".  AZ_ERR_INVALID_ARGUMENT when fewer than three follow it
 * (azimuth then writes no EXR) or the name exceeds 255 characters. */
int az_exr_sibling_path(const char *path, char *out, uint32_t out_len);

/* OutputPixelsToFile for a DEVICE film: normalisation, tone mapping and
 * gamma on the GPU (az_gpu_postprocess), then the file.  format
 * AZ_FileFormat_EXR writes the normalised colours times 255 with no tone
 * mapping or gamma; with save_exr set another format also gets that EXR
 * under az_exr_sibling_path's name.  The device film is left untouched.
 * Runs on opts->stream (NULL: the per-thread default stream). */
int az_gpu_output_pixels_to_file(const char *path, const az_pixel *film, uint32_t width, uint32_t height,
                                 const az_tonemap *tonemap, float inv_gamma, uint32_t srgb, int32_t format,
                                 uint32_t save_exr, const az_render_opts *opts);

#ifdef __cplusplus
}
#endif
#endif
