/* Oracle-build stub for OpenEXR's RGBA file classes: opening any EXR file
 * yields an empty 1x1 image, and writes are discarded.                     */
#pragma once
#include "ImfRgba.h"
namespace Imath {
struct V2i { int x, y; };
struct Box2i { V2i min, max; };
}
namespace Imf {
struct RgbaOutputFile {
    RgbaOutputFile(const char *, int, int, RgbaChannels) {}
    void setFrameBuffer(const Rgba *, unsigned long, unsigned long) {}
    void writePixels(int) {}
};
struct RgbaInputFile {
    explicit RgbaInputFile(const char *) {}
    Imath::Box2i dataWindow() const { Imath::Box2i b = {{0, 0}, {0, 0}}; return b; }
    void setFrameBuffer(Rgba *p, unsigned long, unsigned long) { Buffer = p; }
    void readPixels(int, int) { if (Buffer) { Buffer->r = Buffer->g = Buffer->b = 0.0f; Buffer->a = 1.0f; } }
    Rgba *Buffer = nullptr;
};
}
