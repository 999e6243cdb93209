// Film -> image conversion and image writers (host C++).
//
// cav_film_to_rgb8 follows the reference's Film::readCurrentResult (Core/Film.cu:20-46):
// sum / weight, clamp to [0,1], sRGB encode (Core/Color.h:53-58), x255 truncated.  PNGs are
// written with stored (uncompressed) deflate blocks, as the reference's svpng does; PFM is
// the float film output.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "../../include/cavalry.h"

namespace {

uint32_t crc_table[256];
bool crc_ready = false;

void crc_init() {
    for (uint32_t n = 0; n < 256; ++n) {
        uint32_t c = n;
        for (int k = 0; k < 8; ++k) c = (c & 1) ? 0xedb88320u ^ (c >> 1) : c >> 1;
        crc_table[n] = c;
    }
    crc_ready = true;
}

uint32_t crc32(const uint8_t* p, size_t n, uint32_t c = 0xffffffffu) {
    if (!crc_ready) crc_init();
    for (size_t i = 0; i < n; ++i) c = crc_table[(c ^ p[i]) & 0xff] ^ (c >> 8);
    return c;
}

void put32(std::vector<uint8_t>& v, uint32_t x) {
    v.push_back((uint8_t)(x >> 24));
    v.push_back((uint8_t)(x >> 16));
    v.push_back((uint8_t)(x >> 8));
    v.push_back((uint8_t)x);
}

void chunk(FILE* f, const char* type, const std::vector<uint8_t>& data) {
    std::vector<uint8_t> buf;
    put32(buf, (uint32_t)data.size());
    buf.insert(buf.end(), type, type + 4);
    buf.insert(buf.end(), data.begin(), data.end());
    uint32_t c = crc32(buf.data() + 4, buf.size() - 4) ^ 0xffffffffu;
    put32(buf, c);
    fwrite(buf.data(), 1, buf.size(), f);
}

float srgb(float v) {
    if (v <= 0.0031308f) return 12.92f * v;
    return 1.055f * std::pow(v, 1.f / 2.4f) - 0.055f;
}

}  // namespace

extern "C" {

cav_status cav_film_to_rgb8(const float* film_sum, const float* film_weight, int width, int height, uint8_t* rgb) {
    if (!film_sum || !film_weight || !rgb || width <= 0 || height <= 0) return CAV_ERR_INVALID_ARGUMENT;
    const int64_t n = (int64_t)width * height;
    for (int64_t i = 0; i < n; ++i) {
        for (int k = 0; k < 3; ++k) {
            float v = film_sum[3 * i + k] / film_weight[i];
            v = std::fmax(0.f, std::fmin(1.f, v));
            rgb[3 * i + k] = (uint8_t)(srgb(v) * 255);
        }
    }
    return CAV_OK;
}

cav_status cav_write_png(const char* path, const uint8_t* rgb, int width, int height) {
    if (!path || !rgb || width <= 0 || height <= 0) return CAV_ERR_INVALID_ARGUMENT;
    FILE* f = std::fopen(path, "wb");
    if (!f) return CAV_ERR_INVALID_ARGUMENT;
    static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    fwrite(sig, 1, 8, f);
    std::vector<uint8_t> ihdr;
    put32(ihdr, (uint32_t)width);
    put32(ihdr, (uint32_t)height);
    ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});  // 8-bit RGB
    chunk(f, "IHDR", ihdr);
    // zlib stream of stored blocks over the filtered scanlines (filter byte 0)
    std::vector<uint8_t> raw;
    raw.reserve((size_t)height * (3 * width + 1));
    for (int y = 0; y < height; ++y) {
        raw.push_back(0);
        raw.insert(raw.end(), rgb + (size_t)y * 3 * width, rgb + (size_t)(y + 1) * 3 * width);
    }
    std::vector<uint8_t> z = {0x78, 0x01};
    size_t pos = 0;
    uint32_t a = 1, b = 0;
    for (uint8_t c : raw) {
        a = (a + c) % 65521;
        b = (b + a) % 65521;
    }
    do {
        size_t len = raw.size() - pos < 65535 ? raw.size() - pos : 65535;
        z.push_back(pos + len == raw.size() ? 1 : 0);
        z.push_back((uint8_t)(len & 0xff));
        z.push_back((uint8_t)(len >> 8));
        z.push_back((uint8_t)(~len & 0xff));
        z.push_back((uint8_t)((~len >> 8) & 0xff));
        z.insert(z.end(), raw.begin() + (long)pos, raw.begin() + (long)(pos + len));
        pos += len;
    } while (pos < raw.size());
    put32(z, (b << 16) | a);
    chunk(f, "IDAT", z);
    chunk(f, "IEND", {});
    std::fclose(f);
    return CAV_OK;
}

cav_status cav_write_pfm(const char* path, const float* film_sum, const float* film_weight, int width, int height) {
    if (!path || !film_sum || !film_weight || width <= 0 || height <= 0) return CAV_ERR_INVALID_ARGUMENT;
    FILE* f = std::fopen(path, "wb");
    if (!f) return CAV_ERR_INVALID_ARGUMENT;
    std::fprintf(f, "PF\n%d %d\n-1.0\n", width, height);
    std::vector<float> row(3 * (size_t)width);
    for (int y = height - 1; y >= 0; --y) {  // PFM rows run bottom to top
        for (int x = 0; x < width; ++x) {
            int64_t i = (int64_t)y * width + x;
            for (int k = 0; k < 3; ++k) row[3 * x + k] = film_sum[3 * i + k] / film_weight[i];
        }
        fwrite(row.data(), sizeof(float), row.size(), f);
    }
    std::fclose(f);
    return CAV_OK;
}

}  // extern "C"
