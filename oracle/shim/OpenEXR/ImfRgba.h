/* Oracle-build stub for OpenEXR's Imf::Rgba (no OpenEXR library in this image).
 * Only the members the azimuth sources name are declared; EXR input and
 * output are unavailable in the oracle build and report failure.          */
#pragma once
namespace Imf {
struct Rgba { float r, g, b, a; };
enum RgbaChannels { WRITE_RGB = 0x7, WRITE_RGBA = 0xf };
}
