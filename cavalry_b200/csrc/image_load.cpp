// Host image loading for textures and environment maps: the reference reads them through
// stb_image (Core/Texture.cu:27-83: 8-bit RGBA, flipped vertically on load, and for .png /
// .tga files each colour channel mapped through the inverse sRGB curve and truncated back to
// 8 bits).  This loader reads PNG (8- or 16-bit greyscale, grey+alpha, RGB, RGBA and
// palette images, not interlaced) with zlib's inflate; other formats are refused.
#include <zlib.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

#include "../../include/cavalry.h"
#include "pbrt.h"

namespace cavpbrt {

namespace {

uint32_t be32(const unsigned char* p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }

int paeth(int a, int b, int c) {
    const int p = a + b - c, pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
    if (pa <= pb && pa <= pc) return a;
    return pb <= pc ? b : c;
}

// Color.h inverseGammaCorrect (sRGB to linear), single precision as the reference's host code
float inverse_gamma(float value) {
    if (value <= 0.04045f) return value * 1.f / 12.92f;
    return std::pow((value + 0.055f) * 1.f / 1.055f, (float)2.4f);
}

}  // namespace

TextureImage load_texture_image(const std::string& path) {
    const size_t dot = path.find_last_of('.');
    std::string ext = dot == std::string::npos ? "" : path.substr(dot + 1);
    for (auto& ch : ext) ch = (char)std::tolower((unsigned char)ch);
    if (ext != "png") throw ParseError("texture " + path + ": only PNG images are read (got '" + ext + "')");
    std::ifstream f(path, std::ios::binary);
    if (!f) throw ParseError("texture " + path + ": cannot open");
    const std::string data((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    const unsigned char* d = (const unsigned char*)data.data();
    static const unsigned char sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    if (data.size() < 8 || std::memcmp(d, sig, 8) != 0) throw ParseError("texture " + path + ": not a PNG file");
    uint32_t w = 0, h = 0;
    int depth = 0, ctype = -1, interlace = 0;
    std::vector<unsigned char> idat, plte, trns;
    for (size_t pos = 8; pos + 12 <= data.size();) {
        const uint32_t n = be32(d + pos);
        if (pos + 12 + (size_t)n > data.size()) throw ParseError("texture " + path + ": truncated chunk");
        const std::string type((const char*)d + pos + 4, 4);
        const unsigned char* body = d + pos + 8;
        if (type == "IHDR" && n >= 13) {
            w = be32(body);
            h = be32(body + 4);
            depth = body[8];
            ctype = body[9];
            interlace = body[12];
        } else if (type == "PLTE") {
            plte.assign(body, body + n);
        } else if (type == "tRNS") {
            trns.assign(body, body + n);
        } else if (type == "IDAT") {
            idat.insert(idat.end(), body, body + n);
        } else if (type == "IEND") {
            break;
        }
        pos += 12 + (size_t)n;
    }
    if (w == 0 || h == 0 || w > (1u << 15) || h > (1u << 15)) throw ParseError("texture " + path + ": bad size");
    if (interlace != 0) throw ParseError("texture " + path + ": interlaced PNG images are not read");
    int channels;
    switch (ctype) {
        case 0: channels = 1; break;
        case 2: channels = 3; break;
        case 3: channels = 1; break;
        case 4: channels = 2; break;
        case 6: channels = 4; break;
        default: throw ParseError("texture " + path + ": unknown PNG colour type");
    }
    if (!(depth == 8 || (depth == 16 && ctype != 3))) throw ParseError("texture " + path + ": unsupported bit depth");
    const size_t bpp = (size_t)channels * (depth / 8);
    const size_t stride = bpp * w;
    std::vector<unsigned char> raw((stride + 1) * h);
    uLongf raw_len = (uLongf)raw.size();
    if (uncompress(raw.data(), &raw_len, idat.data(), (uLong)idat.size()) != Z_OK || raw_len != raw.size())
        throw ParseError("texture " + path + ": corrupt image data");
    std::vector<unsigned char> img(stride * h);
    for (uint32_t y = 0; y < h; ++y) {  // reverse the scanline filters
        const unsigned char* src = raw.data() + y * (stride + 1) + 1;
        unsigned char* row = img.data() + y * stride;
        const unsigned char* up = y ? img.data() + (y - 1) * stride : nullptr;
        const int filter = raw[y * (stride + 1)];
        for (size_t x = 0; x < stride; ++x) {
            const int a = x >= bpp ? row[x - bpp] : 0, b = up ? up[x] : 0, c = (up && x >= bpp) ? up[x - bpp] : 0;
            int v = src[x];
            switch (filter) {
                case 0: break;
                case 1: v += a; break;
                case 2: v += b; break;
                case 3: v += (a + b) / 2; break;
                case 4: v += paeth(a, b, c); break;
                default: throw ParseError("texture " + path + ": bad scanline filter");
            }
            row[x] = (unsigned char)v;
        }
    }
    TextureImage t;
    t.width = (int)w;
    t.height = (int)h;
    t.rgba.resize((size_t)4 * w * h);
    for (uint32_t y = 0; y < h; ++y) {
        const unsigned char* row = img.data() + y * stride;
        unsigned char* out = t.rgba.data() + (size_t)4 * w * (h - 1 - y);  // flipped vertically on load
        for (uint32_t x = 0; x < w; ++x) {
            unsigned char px[4];
            auto sample = [&](int ch) { return row[(x * channels + ch) * (depth / 8)]; };  // 16-bit: high byte
            if (ctype == 3) {
                const int k = row[x];
                if ((size_t)(3 * k + 2) >= plte.size()) throw ParseError("texture " + path + ": palette index");
                px[0] = plte[3 * k];
                px[1] = plte[3 * k + 1];
                px[2] = plte[3 * k + 2];
                px[3] = (size_t)k < trns.size() ? trns[k] : 255;
            } else if (channels <= 2) {
                px[0] = px[1] = px[2] = sample(0);
                px[3] = channels == 2 ? sample(1) : 255;
            } else {
                px[0] = sample(0);
                px[1] = sample(1);
                px[2] = sample(2);
                px[3] = channels == 4 ? sample(3) : 255;
            }
            for (int c = 0; c < 3; ++c)  // .png: inverse gamma, truncated to 8 bits
                px[c] = (unsigned char)(255.f * inverse_gamma(px[c] / 255.f));
            std::memcpy(out + 4 * x, px, 4);
        }
    }
    return t;
}

}  // namespace cavpbrt

// Host-only: the texture loader's output for one image (no GPU).
extern "C" cav_status cav_load_texture_png(const char* path, uint8_t* rgba, int64_t capacity_bytes, int* width,
                                           int* height, char* err, int err_len) {
    if (!path || !width || !height) return CAV_ERR_INVALID_ARGUMENT;
    try {
        const cavpbrt::TextureImage t = cavpbrt::load_texture_image(path);
        *width = t.width;
        *height = t.height;
        if (!rgba) return CAV_OK;  // size query
        if (capacity_bytes < (int64_t)t.rgba.size()) {
            if (err && err_len > 0) {
                std::strncpy(err, "cav_load_texture_png: output buffer too small", (size_t)err_len - 1);
                err[err_len - 1] = 0;
            }
            return CAV_ERR_INVALID_ARGUMENT;
        }
        std::memcpy(rgba, t.rgba.data(), t.rgba.size());
    } catch (const std::exception& e) {
        if (err && err_len > 0) {
            std::strncpy(err, e.what(), (size_t)err_len - 1);
            err[err_len - 1] = 0;
        }
        return CAV_ERR_INVALID_ARGUMENT;
    }
    return CAV_OK;
}
