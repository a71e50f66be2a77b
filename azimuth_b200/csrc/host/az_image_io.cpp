// Image writers of OutputPixelsToFile (src/azimuth_main.cpp:1426-1618): 8-bit
// RGB as PNG, BMP, TGA or JPEG, and colours as an OpenEXR file.  azimuth
// writes the first four through the stb_image_write header and EXR through
// OpenEXR; these are this library's own writers, each following its format's
// published specification:
//   BMP   24-bit BI_RGB, bottom-up rows padded to 4 bytes (BITMAPINFOHEADER)
//   TGA   true-colour run-length encoded (image type 10), packets within a row
//   PNG   colour type 2, per-row filter chosen by the smallest sum of absolute
//         residuals (the PNG specification's heuristic), zlib-compressed IDAT
//   JPEG  baseline sequential DCT (ITU-T T.81), JFIF YCbCr, 4:4:4, the Annex K
//         tables scaled by the common quality rule (quality 100 for
//         OutputPixelsToJPG), Annex K Huffman tables
//   EXR   single-part scanline file, NO_COMPRESSION, HALF channels B, G, R
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "azimuth_io.h"

namespace {

struct File {
    FILE *f = nullptr;
    explicit File(const char *path) : f(fopen(path, "wb")) {}
    ~File() {
        if (f) fclose(f);
    }
    bool put(const void *p, size_t n) { return fwrite(p, 1, n, f) == n; }
};

void le16(std::vector<uint8_t> &v, uint32_t x) {
    v.push_back(x & 0xFF);
    v.push_back((x >> 8) & 0xFF);
}
void le32(std::vector<uint8_t> &v, uint32_t x) {
    le16(v, x & 0xFFFF);
    le16(v, x >> 16);
}
void be16(std::vector<uint8_t> &v, uint32_t x) {
    v.push_back((x >> 8) & 0xFF);
    v.push_back(x & 0xFF);
}
void be32(std::vector<uint8_t> &v, uint32_t x) {
    be16(v, x >> 16);
    be16(v, x & 0xFFFF);
}

bool WriteAll(const char *path, const std::vector<uint8_t> &bytes) {
    File f(path);
    return f.f && f.put(bytes.data(), bytes.size());
}

// ---- BMP ----
bool WriteBMP(const char *path, const uint8_t *rgb, uint32_t w, uint32_t h) {
    const uint32_t stride = (3 * w + 3) & ~3u;
    const uint64_t data = (uint64_t)stride * h;
    if (54 + data > 0xFFFFFFFFull) return false;
    std::vector<uint8_t> v;
    v.reserve(54 + data);
    v.push_back('B');
    v.push_back('M');
    le32(v, (uint32_t)(54 + data));   // file size
    le32(v, 0);                       // reserved
    le32(v, 54);                      // pixel data offset
    le32(v, 40);                      // BITMAPINFOHEADER
    le32(v, w);
    le32(v, h);                       // positive: bottom-up rows
    le16(v, 1);                       // planes
    le16(v, 24);                      // bits per pixel
    le32(v, 0);                       // BI_RGB
    le32(v, (uint32_t)data);
    le32(v, 0);                       // pixels per metre, x and y: unspecified
    le32(v, 0);
    le32(v, 0);                       // palette entries
    le32(v, 0);
    for (uint32_t r = 0; r < h; r++) {
        const uint8_t *row = rgb + (size_t)(h - 1 - r) * w * 3;
        for (uint32_t x = 0; x < w; x++) {
            v.push_back(row[3 * x + 2]);
            v.push_back(row[3 * x + 1]);
            v.push_back(row[3 * x + 0]);
        }
        for (uint32_t p = 3 * w; p < stride; p++) v.push_back(0);
    }
    return WriteAll(path, v);
}

// ---- TGA (run-length encoded true colour) ----
bool WriteTGA(const char *path, const uint8_t *rgb, uint32_t w, uint32_t h) {
    if (w > 0xFFFF || h > 0xFFFF) return false;
    std::vector<uint8_t> v;
    v.reserve(18 + (size_t)w * h * 3 + (size_t)h * (w / 128 + 2));
    const uint8_t hdr[18] = {0, 0, 10, 0, 0, 0, 0, 0, 0, 0, 0, 0,
                             (uint8_t)(w & 0xFF), (uint8_t)(w >> 8), (uint8_t)(h & 0xFF), (uint8_t)(h >> 8),
                             24, 0x20};   // 24 bits per pixel; descriptor bit 5: top row first
    v.insert(v.end(), hdr, hdr + 18);
    auto same = [&](const uint8_t *a, const uint8_t *b) { return a[0] == b[0] && a[1] == b[1] && a[2] == b[2]; };
    auto bgr = [&](const uint8_t *p) {
        v.push_back(p[2]);
        v.push_back(p[1]);
        v.push_back(p[0]);
    };
    for (uint32_t y = 0; y < h; y++) {
        const uint8_t *row = rgb + (size_t)y * w * 3;
        uint32_t x = 0;
        while (x < w) {
            uint32_t run = 1;
            while (x + run < w && run < 128 && same(row + 3 * x, row + 3 * (x + run))) run++;
            if (run >= 2) {   // run-length packet
                v.push_back((uint8_t)(0x80 | (run - 1)));
                bgr(row + 3 * x);
                x += run;
                continue;
            }
            // raw packet up to the next pair of equal neighbours
            uint32_t n = 1;
            while (x + n < w && n < 128 && !(x + n + 1 < w && same(row + 3 * (x + n), row + 3 * (x + n + 1)))) n++;
            v.push_back((uint8_t)(n - 1));
            for (uint32_t k = 0; k < n; k++) bgr(row + 3 * (x + k));
            x += n;
        }
    }
    return WriteAll(path, v);
}

// ---- PNG ----
void Chunk(std::vector<uint8_t> &v, const char *type, const uint8_t *data, size_t n) {
    be32(v, (uint32_t)n);
    const size_t start = v.size();
    v.insert(v.end(), type, type + 4);
    if (n) v.insert(v.end(), data, data + n);
    be32(v, (uint32_t)crc32(0L, v.data() + start, (uInt)(n + 4)));
}

uint8_t Paeth(int a, int b, int c) {
    const int p = a + b - c, pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
    if (pa <= pb && pa <= pc) return (uint8_t)a;
    return (uint8_t)(pb <= pc ? b : c);
}

// Byte i of a row under PNG filter f (0 none, 1 sub, 2 up, 3 average, 4 Paeth).
uint8_t Filtered(int f, const uint8_t *cur, const uint8_t *up, size_t i) {
    const int a = i >= 3 ? cur[i - 3] : 0, b = up[i], c = i >= 3 ? up[i - 3] : 0;
    switch (f) {
        case 1: return (uint8_t)(cur[i] - a);
        case 2: return (uint8_t)(cur[i] - b);
        case 3: return (uint8_t)(cur[i] - ((a + b) >> 1));
        case 4: return (uint8_t)(cur[i] - Paeth(a, b, c));
        default: return cur[i];
    }
}

bool WritePNG(const char *path, const uint8_t *rgb, uint32_t w, uint32_t h) {
    const size_t stride = (size_t)w * 3;
    std::vector<uint8_t> raw((stride + 1) * h);
    std::vector<uint8_t> zero(stride, 0);
    for (uint32_t y = 0; y < h; y++) {
        const uint8_t *cur = rgb + y * stride, *up = y ? rgb + (y - 1) * stride : zero.data();
        uint64_t best_sum = UINT64_MAX;
        int best = 0;
        for (int f = 0; f < 5; f++) {
            uint64_t sum = 0;
            for (size_t i = 0; i < stride; i++) sum += (uint64_t)std::abs((int)(int8_t)Filtered(f, cur, up, i));
            if (sum < best_sum) {
                best_sum = sum;
                best = f;
            }
        }
        uint8_t *out = raw.data() + y * (stride + 1);
        out[0] = (uint8_t)best;
        for (size_t i = 0; i < stride; i++) out[1 + i] = Filtered(best, cur, up, i);
    }
    uLongf zn = compressBound((uLong)raw.size());
    std::vector<uint8_t> z(zn);
    if (compress2(z.data(), &zn, raw.data(), (uLong)raw.size(), 6) != Z_OK) return false;
    std::vector<uint8_t> v;
    const uint8_t sig[8] = {0x89, 'P', 'N', 'G', 0x0D, 0x0A, 0x1A, 0x0A};
    v.insert(v.end(), sig, sig + 8);
    std::vector<uint8_t> ihdr;
    be32(ihdr, w);
    be32(ihdr, h);
    ihdr.push_back(8);   // bit depth
    ihdr.push_back(2);   // colour type: RGB
    ihdr.push_back(0);   // deflate
    ihdr.push_back(0);   // adaptive filtering
    ihdr.push_back(0);   // no interlace
    Chunk(v, "IHDR", ihdr.data(), ihdr.size());
    Chunk(v, "IDAT", z.data(), zn);
    Chunk(v, "IEND", nullptr, 0);
    return WriteAll(path, v);
}

// ---- JPEG (baseline, ITU-T T.81) ----
// Annex K.1 / K.2 quantisation tables in natural (row-major) order.
const uint8_t kLumaQ[64] = {16, 11, 10, 16, 24,  40,  51,  61,  12, 12, 14, 19, 26,  58,  60,  55,
                            14, 13, 16, 24, 40,  57,  69,  56,  14, 17, 22, 29, 51,  87,  80,  62,
                            18, 22, 37, 56, 68,  109, 103, 77,  24, 35, 55, 64, 81,  104, 113, 92,
                            49, 64, 78, 87, 103, 121, 120, 101, 72, 92, 95, 98, 112, 100, 103, 99};
const uint8_t kChromaQ[64] = {17, 18, 24, 47, 99, 99, 99, 99, 18, 21, 26, 66, 99, 99, 99, 99,
                              24, 26, 56, 99, 99, 99, 99, 99, 47, 66, 99, 99, 99, 99, 99, 99,
                              99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99,
                              99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99};
// Annex K.3-K.6 Huffman tables: code counts per length 1..16, then symbols.
const uint8_t kDcLumaBits[16] = {0, 1, 5, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0};
const uint8_t kDcChromaBits[16] = {0, 3, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0};
const uint8_t kDcVals[12] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11};
const uint8_t kAcLumaBits[16] = {0, 2, 1, 3, 3, 2, 4, 3, 5, 5, 4, 4, 0, 0, 1, 0x7d};
const uint8_t kAcLumaVals[162] = {
    0x01, 0x02, 0x03, 0x00, 0x04, 0x11, 0x05, 0x12, 0x21, 0x31, 0x41, 0x06, 0x13, 0x51, 0x61, 0x07, 0x22, 0x71,
    0x14, 0x32, 0x81, 0x91, 0xa1, 0x08, 0x23, 0x42, 0xb1, 0xc1, 0x15, 0x52, 0xd1, 0xf0, 0x24, 0x33, 0x62, 0x72,
    0x82, 0x09, 0x0a, 0x16, 0x17, 0x18, 0x19, 0x1a, 0x25, 0x26, 0x27, 0x28, 0x29, 0x2a, 0x34, 0x35, 0x36, 0x37,
    0x38, 0x39, 0x3a, 0x43, 0x44, 0x45, 0x46, 0x47, 0x48, 0x49, 0x4a, 0x53, 0x54, 0x55, 0x56, 0x57, 0x58, 0x59,
    0x5a, 0x63, 0x64, 0x65, 0x66, 0x67, 0x68, 0x69, 0x6a, 0x73, 0x74, 0x75, 0x76, 0x77, 0x78, 0x79, 0x7a, 0x83,
    0x84, 0x85, 0x86, 0x87, 0x88, 0x89, 0x8a, 0x92, 0x93, 0x94, 0x95, 0x96, 0x97, 0x98, 0x99, 0x9a, 0xa2, 0xa3,
    0xa4, 0xa5, 0xa6, 0xa7, 0xa8, 0xa9, 0xaa, 0xb2, 0xb3, 0xb4, 0xb5, 0xb6, 0xb7, 0xb8, 0xb9, 0xba, 0xc2, 0xc3,
    0xc4, 0xc5, 0xc6, 0xc7, 0xc8, 0xc9, 0xca, 0xd2, 0xd3, 0xd4, 0xd5, 0xd6, 0xd7, 0xd8, 0xd9, 0xda, 0xe1, 0xe2,
    0xe3, 0xe4, 0xe5, 0xe6, 0xe7, 0xe8, 0xe9, 0xea, 0xf1, 0xf2, 0xf3, 0xf4, 0xf5, 0xf6, 0xf7, 0xf8, 0xf9, 0xfa};
const uint8_t kAcChromaBits[16] = {0, 2, 1, 2, 4, 4, 3, 4, 7, 5, 4, 4, 0, 1, 2, 0x77};
const uint8_t kAcChromaVals[162] = {
    0x00, 0x01, 0x02, 0x03, 0x11, 0x04, 0x05, 0x21, 0x31, 0x06, 0x12, 0x41, 0x51, 0x07, 0x61, 0x71, 0x13, 0x22,
    0x32, 0x81, 0x08, 0x14, 0x42, 0x91, 0xa1, 0xb1, 0xc1, 0x09, 0x23, 0x33, 0x52, 0xf0, 0x15, 0x62, 0x72, 0xd1,
    0x0a, 0x16, 0x24, 0x34, 0xe1, 0x25, 0xf1, 0x17, 0x18, 0x19, 0x1a, 0x26, 0x27, 0x28, 0x29, 0x2a, 0x35, 0x36,
    0x37, 0x38, 0x39, 0x3a, 0x43, 0x44, 0x45, 0x46, 0x47, 0x48, 0x49, 0x4a, 0x53, 0x54, 0x55, 0x56, 0x57, 0x58,
    0x59, 0x5a, 0x63, 0x64, 0x65, 0x66, 0x67, 0x68, 0x69, 0x6a, 0x73, 0x74, 0x75, 0x76, 0x77, 0x78, 0x79, 0x7a,
    0x82, 0x83, 0x84, 0x85, 0x86, 0x87, 0x88, 0x89, 0x8a, 0x92, 0x93, 0x94, 0x95, 0x96, 0x97, 0x98, 0x99, 0x9a,
    0xa2, 0xa3, 0xa4, 0xa5, 0xa6, 0xa7, 0xa8, 0xa9, 0xaa, 0xb2, 0xb3, 0xb4, 0xb5, 0xb6, 0xb7, 0xb8, 0xb9, 0xba,
    0xc2, 0xc3, 0xc4, 0xc5, 0xc6, 0xc7, 0xc8, 0xc9, 0xca, 0xd2, 0xd3, 0xd4, 0xd5, 0xd6, 0xd7, 0xd8, 0xd9, 0xda,
    0xe2, 0xe3, 0xe4, 0xe5, 0xe6, 0xe7, 0xe8, 0xe9, 0xea, 0xf2, 0xf3, 0xf4, 0xf5, 0xf6, 0xf7, 0xf8, 0xf9, 0xfa};

struct Huff {
    uint16_t code[256];
    uint8_t len[256];
    bool ok;
    // canonical codes from the counts per length (T.81 Annex C)
    Huff(const uint8_t bits[16], const uint8_t *vals, int nvals) : ok(true) {
        memset(code, 0, sizeof(code));
        memset(len, 0, sizeof(len));
        uint32_t c = 0;
        int k = 0;
        for (int l = 1; l <= 16; l++) {
            for (int i = 0; i < bits[l - 1]; i++) {
                if (k >= nvals || c >= (1u << l) - 1u) {   // the all-ones code of a length is reserved
                    ok = false;
                    return;
                }
                code[vals[k]] = (uint16_t)c;
                len[vals[k]] = (uint8_t)l;
                k++;
                c++;
            }
            c <<= 1;
        }
        ok = k == nvals;
    }
};

struct BitWriter {
    std::vector<uint8_t> &v;
    uint32_t acc = 0;
    int n = 0;
    explicit BitWriter(std::vector<uint8_t> &o) : v(o) {}
    void put(uint32_t bits, int count) {
        for (int i = count - 1; i >= 0; i--) {
            acc = (acc << 1) | ((bits >> i) & 1u);
            if (++n == 8) {
                v.push_back((uint8_t)acc);
                if (acc == 0xFF) v.push_back(0);   // byte stuffing
                acc = 0;
                n = 0;
            }
        }
    }
    void flush() {
        while (n) put(1, 1);   // pad with one-bits
    }
};

// zigzag position k -> natural index, by walking the anti-diagonals
void ZigZag(int zz[64]) {
    int k = 0;
    for (int s = 0; s < 15; s++) {
        if (s % 2 == 0) {
            for (int r = s < 8 ? s : 7; r >= 0 && s - r < 8; r--) zz[k++] = r * 8 + (s - r);
        } else {
            for (int c = s < 8 ? s : 7; c >= 0 && s - c < 8; c--) zz[k++] = (s - c) * 8 + c;
        }
    }
}

int Category(int v) {
    int a = v < 0 ? -v : v, n = 0;
    while (a) {
        n++;
        a >>= 1;
    }
    return n;
}

bool WriteJPG(const char *path, const uint8_t *rgb, uint32_t w, uint32_t h, int quality) {
    if (w == 0 || h == 0 || w > 0xFFFF || h > 0xFFFF) return false;
    quality = quality < 1 ? 1 : (quality > 100 ? 100 : quality);
    const int scale = quality < 50 ? 5000 / quality : 200 - 2 * quality;
    uint8_t q[2][64];
    for (int i = 0; i < 64; i++) {
        const int a = (kLumaQ[i] * scale + 50) / 100, b = (kChromaQ[i] * scale + 50) / 100;
        q[0][i] = (uint8_t)(a < 1 ? 1 : (a > 255 ? 255 : a));
        q[1][i] = (uint8_t)(b < 1 ? 1 : (b > 255 ? 255 : b));
    }
    const Huff dc[2] = {Huff(kDcLumaBits, kDcVals, 12), Huff(kDcChromaBits, kDcVals, 12)};
    const Huff ac[2] = {Huff(kAcLumaBits, kAcLumaVals, 162), Huff(kAcChromaBits, kAcChromaVals, 162)};
    if (!dc[0].ok || !dc[1].ok || !ac[0].ok || !ac[1].ok) return false;
    int zz[64];
    ZigZag(zz);
    double cosv[8][8];
    for (int x = 0; x < 8; x++)
        for (int u = 0; u < 8; u++) cosv[x][u] = std::cos((2 * x + 1) * u * M_PI / 16.0);

    std::vector<uint8_t> v;
    auto marker = [&](uint8_t m) {
        v.push_back(0xFF);
        v.push_back(m);
    };
    marker(0xD8);   // SOI
    marker(0xE0);   // APP0 JFIF 1.01, no density units, aspect 1:1
    be16(v, 16);
    const uint8_t jfif[14] = {'J', 'F', 'I', 'F', 0, 1, 1, 0, 0, 1, 0, 1, 0, 0};
    v.insert(v.end(), jfif, jfif + 14);
    for (int t = 0; t < 2; t++) {   // DQT, zigzag order
        marker(0xDB);
        be16(v, 67);
        v.push_back((uint8_t)t);
        for (int k = 0; k < 64; k++) v.push_back(q[t][zz[k]]);
    }
    marker(0xC0);   // SOF0: 8-bit, 3 components, no subsampling
    be16(v, 17);
    v.push_back(8);
    be16(v, h);
    be16(v, w);
    v.push_back(3);
    const uint8_t comps[9] = {1, 0x11, 0, 2, 0x11, 1, 3, 0x11, 1};
    v.insert(v.end(), comps, comps + 9);
    auto dht = [&](uint8_t cls_id, const uint8_t bits[16], const uint8_t *vals, int n) {
        marker(0xC4);
        be16(v, 2 + 1 + 16 + n);
        v.push_back(cls_id);
        v.insert(v.end(), bits, bits + 16);
        v.insert(v.end(), vals, vals + n);
    };
    dht(0x00, kDcLumaBits, kDcVals, 12);
    dht(0x10, kAcLumaBits, kAcLumaVals, 162);
    dht(0x01, kDcChromaBits, kDcVals, 12);
    dht(0x11, kAcChromaBits, kAcChromaVals, 162);
    marker(0xDA);   // SOS
    be16(v, 12);
    v.push_back(3);
    const uint8_t sos[6] = {1, 0x00, 2, 0x11, 3, 0x11};
    v.insert(v.end(), sos, sos + 6);
    v.push_back(0);
    v.push_back(63);
    v.push_back(0);

    BitWriter bw(v);
    int pred[3] = {0, 0, 0};
    double blk[3][64];
    for (uint32_t by = 0; by < h; by += 8)
        for (uint32_t bx = 0; bx < w; bx += 8) {
            // JFIF colour conversion, edge pixels repeated past the image
            for (int y = 0; y < 8; y++)
                for (int x = 0; x < 8; x++) {
                    const uint32_t sx = std::min(bx + x, w - 1), sy = std::min(by + y, h - 1);
                    const uint8_t *p = rgb + ((size_t)sy * w + sx) * 3;
                    const double r = p[0], g = p[1], b = p[2];
                    blk[0][y * 8 + x] = 0.299 * r + 0.587 * g + 0.114 * b - 128.0;
                    blk[1][y * 8 + x] = -0.168736 * r - 0.331264 * g + 0.5 * b;
                    blk[2][y * 8 + x] = 0.5 * r - 0.418688 * g - 0.081312 * b;
                }
            for (int c = 0; c < 3; c++) {
                const int t = c ? 1 : 0;
                int coef[64];
                for (int v8 = 0; v8 < 8; v8++)
                    for (int u = 0; u < 8; u++) {
                        double s = 0.0;
                        for (int y = 0; y < 8; y++)
                            for (int x = 0; x < 8; x++) s += blk[c][y * 8 + x] * cosv[x][u] * cosv[y][v8];
                        const double cu = u ? 1.0 : M_SQRT1_2, cv = v8 ? 1.0 : M_SQRT1_2;
                        const double f = 0.25 * cu * cv * s;
                        coef[v8 * 8 + u] = (int)std::lround(f / q[t][v8 * 8 + u]);
                    }
                // DC difference, then run-length coded AC in zigzag order
                const int diff = coef[0] - pred[c];
                pred[c] = coef[0];
                int cat = Category(diff);
                bw.put(dc[t].code[cat], dc[t].len[cat]);
                if (cat) bw.put((uint32_t)(diff < 0 ? diff + (1 << cat) - 1 : diff), cat);
                int run = 0;
                for (int k = 1; k < 64; k++) {
                    const int a = coef[zz[k]];
                    if (a == 0) {
                        run++;
                        continue;
                    }
                    while (run > 15) {
                        bw.put(ac[t].code[0xF0], ac[t].len[0xF0]);
                        run -= 16;
                    }
                    cat = Category(a);
                    const int sym = (run << 4) | cat;
                    bw.put(ac[t].code[sym], ac[t].len[sym]);
                    bw.put((uint32_t)(a < 0 ? a + (1 << cat) - 1 : a), cat);
                    run = 0;
                }
                if (run) bw.put(ac[t].code[0x00], ac[t].len[0x00]);
            }
        }
    bw.flush();
    marker(0xD9);   // EOI
    return WriteAll(path, v);
}

// ---- OpenEXR ----
// IEEE binary16, round to nearest even (overflow to infinity, subnormals kept).
uint16_t ToHalf(float f) {
    uint32_t x;
    memcpy(&x, &f, 4);
    const uint32_t sign = (x >> 16) & 0x8000u, ax = x & 0x7FFFFFFFu;
    if (ax >= 0x7F800000u) return (uint16_t)(sign | 0x7C00u | (ax > 0x7F800000u ? 0x200u : 0u));   // inf / nan
    if (ax >= 0x477FF000u) return (uint16_t)(sign | 0x7C00u);    // rounds to above 65504
    if (ax < 0x33000001u) return (uint16_t)sign;                 // below half the smallest subnormal
    int e = (int)(ax >> 23) - 127;
    uint32_t m = (ax & 0x7FFFFFu) | 0x800000u;
    int shift;
    uint32_t base;
    if (e < -14) {            // subnormal half: value = m * 2^(e-23) = q * 2^-24
        shift = -1 - e;       // 13 + (-14 - e)
        base = 0;
    } else {
        shift = 13;
        base = (uint32_t)(e + 15) << 10;
        m &= 0x7FFFFFu;
    }
    uint32_t q = m >> shift, rem = m & ((1u << shift) - 1u), half = 1u << (shift - 1);
    if (rem > half || (rem == half && (q & 1u))) q++;
    return (uint16_t)(sign | (base + q));   // a mantissa carry steps the exponent, as it should
}

bool WriteEXR(const char *path, const float *rgb, uint32_t w, uint32_t h) {
    if (w == 0 || h == 0 || w > 0x7FFFFFFF || h > 0x7FFFFFFF) return false;
    std::vector<uint8_t> v;
    le32(v, 20000630u);   // magic
    le32(v, 2u);          // version 2, single-part scanline
    auto attr = [&](const char *name, const char *type, const std::vector<uint8_t> &val) {
        v.insert(v.end(), name, name + strlen(name) + 1);
        v.insert(v.end(), type, type + strlen(type) + 1);
        le32(v, (uint32_t)val.size());
        v.insert(v.end(), val.begin(), val.end());
    };
    std::vector<uint8_t> ch;
    for (const char *c : {"B", "G", "R"}) {   // channels in name order
        ch.push_back((uint8_t)c[0]);
        ch.push_back(0);
        le32(ch, 1);   // HALF
        ch.push_back(0);   // pLinear
        ch.push_back(0);
        ch.push_back(0);
        ch.push_back(0);
        le32(ch, 1);   // x sampling
        le32(ch, 1);   // y sampling
    }
    ch.push_back(0);
    attr("channels", "chlist", ch);
    attr("compression", "compression", std::vector<uint8_t>{0});   // NO_COMPRESSION
    std::vector<uint8_t> box;
    le32(box, 0);
    le32(box, 0);
    le32(box, w - 1);
    le32(box, h - 1);
    attr("dataWindow", "box2i", box);
    attr("displayWindow", "box2i", box);
    attr("lineOrder", "lineOrder", std::vector<uint8_t>{0});   // increasing y
    std::vector<uint8_t> one, v2;
    float f1 = 1.0f, f0 = 0.0f;
    uint32_t b1, b0;
    memcpy(&b1, &f1, 4);
    memcpy(&b0, &f0, 4);
    le32(one, b1);
    le32(v2, b0);
    le32(v2, b0);
    attr("pixelAspectRatio", "float", one);
    attr("screenWindowCenter", "v2f", v2);
    attr("screenWindowWidth", "float", one);
    v.push_back(0);   // end of header
    const uint64_t table = v.size(), line = 8 + (uint64_t)w * 3 * 2;
    const uint64_t first = table + 8ull * h;
    for (uint32_t y = 0; y < h; y++) {
        const uint64_t off = first + y * line;
        le32(v, (uint32_t)(off & 0xFFFFFFFFu));
        le32(v, (uint32_t)(off >> 32));
    }
    for (uint32_t y = 0; y < h; y++) {
        le32(v, y);
        le32(v, (uint32_t)(w * 3 * 2));
        for (int c = 2; c >= 0; c--)   // B, G, R
            for (uint32_t x = 0; x < w; x++) le16(v, ToHalf(rgb[((size_t)y * w + x) * 3 + c]));
    }
    return WriteAll(path, v);
}

}  // namespace

extern "C" int az_write_image(const char *path, const uint8_t *rgb8, uint32_t width, uint32_t height, int32_t format) {
    if (!path || !rgb8 || width == 0 || height == 0) return AZ_ERR_INVALID_ARGUMENT;
    bool ok;
    switch (format) {
        case AZ_FileFormat_PNG: ok = WritePNG(path, rgb8, width, height); break;
        case AZ_FileFormat_BMP: ok = WriteBMP(path, rgb8, width, height); break;
        case AZ_FileFormat_TGA: ok = WriteTGA(path, rgb8, width, height); break;
        case AZ_FileFormat_JPG: ok = WriteJPG(path, rgb8, width, height, 100); break;
        default: return AZ_ERR_INVALID_ARGUMENT;
    }
    return ok ? AZ_OK : AZ_ERR_IO;
}

extern "C" int az_write_exr(const char *path, const float *rgb, uint32_t width, uint32_t height) {
    if (!path || !rgb || width == 0 || height == 0) return AZ_ERR_INVALID_ARGUMENT;
    return WriteEXR(path, rgb, width, height) ? AZ_OK : AZ_ERR_IO;
}

extern "C" int az_write_jpg_quality(const char *path, const uint8_t *rgb8, uint32_t width, uint32_t height,
                                    int32_t quality) {
    if (!path || !rgb8 || width == 0 || height == 0) return AZ_ERR_INVALID_ARGUMENT;
    return WriteJPG(path, rgb8, width, height, quality) ? AZ_OK : AZ_ERR_IO;
}

extern "C" int az_exr_sibling_path(const char *path, char *out, uint32_t out_len) {
    // OutputPixelsToFile's EXR name: the three characters after the last '.'
    // become "exr" (src/azimuth_main.cpp:1660-1683); no EXR when fewer follow it
    if (!path || !out || out_len == 0) return AZ_ERR_INVALID_ARGUMENT;
    const size_t n = strlen(path);
    if (n == 0 || n + 1 > out_len || n + 1 > 256) return AZ_ERR_INVALID_ARGUMENT;
    memcpy(out, path, n + 1);
    size_t dot = n - 1;
    while (dot > 0 && out[dot] != '.') dot--;
    if (n - dot - 1 < 3) return AZ_ERR_INVALID_ARGUMENT;
    memcpy(out + dot + 1, "exr", 3);
    return AZ_OK;
}
