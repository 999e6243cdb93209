// Host image loading for textures and environment maps, as Core/Texture.cu:27-83 loads them:
// a file whose name ends in "exr" (case as written) through tinyexr's LoadEXR (RGBA floats,
// rows as stored, no gamma), anything else through stb_image (8-bit RGBA, flipped vertically
// on load, and for names ending in "png" or "tga" each colour channel mapped through the
// inverse sRGB curve and truncated back to 8 bits).  This loader reads PNG (8- or 16-bit
// greyscale, grey+alpha, RGB, RGBA and palette images, not interlaced) and OpenEXR scanline
// images (NONE, RLE, ZIPS, ZIP compression; HALF and FLOAT channels), both with zlib's
// inflate; other formats, tiled or multi-part EXR and the PIZ / PXR24 / B44 / DWA codecs
// are refused with a message.
#include <zlib.h>

#include <algorithm>
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

// ------------------------------------------------------------------ OpenEXR
namespace {

uint32_t le32(const unsigned char* p) { return (uint32_t)p[0] | (uint32_t)p[1] << 8 | (uint32_t)p[2] << 16 | (uint32_t)p[3] << 24; }

// IEEE half to single precision (exact for every value; NaN payloads kept in the top bits).
float half_to_float(uint16_t h) {
    const uint32_t sign = (uint32_t)(h >> 15) << 31;
    uint32_t exp = (h >> 10) & 0x1f, mant = h & 0x3ff, bits;
    if (exp == 0) {
        if (mant == 0) {
            bits = sign;
        } else {  // subnormal half: normalise into a float
            int e = -1;
            do {
                ++e;
                mant <<= 1;
            } while ((mant & 0x400) == 0);
            bits = sign | (uint32_t)(127 - 15 - e) << 23 | (mant & 0x3ff) << 13;
        }
    } else if (exp == 31) {
        bits = sign | 0x7f800000u | mant << 13;
    } else {
        bits = sign | (exp - 15 + 127) << 23 | mant << 13;
    }
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

// The OpenEXR ZIP / RLE post-processing, undone: the encoder split the bytes into even and
// odd halves and stored the differences between neighbours (+128); decode in reverse.
void undo_predictor_and_split(std::vector<unsigned char>& t) {
    for (size_t i = 1; i < t.size(); ++i) t[i] = (unsigned char)(t[i - 1] + t[i] - 128);
    std::vector<unsigned char> out(t.size());
    const size_t half = (t.size() + 1) / 2;
    for (size_t i = 0; i < t.size(); ++i) out[i] = (i & 1) ? t[half + i / 2] : t[i / 2];
    t.swap(out);
}

struct ExrChannel {
    std::string name;
    int type;  // 0 UINT, 1 HALF, 2 FLOAT
};

}  // namespace

TextureImage load_exr(const std::string& path) {
    auto fail = [&](const std::string& m) { return ParseError("exr " + path + ": " + m); };
    std::ifstream f(path, std::ios::binary);
    if (!f) throw fail("cannot open");
    const std::string data((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    const unsigned char* d = (const unsigned char*)data.data();
    const size_t size = data.size();
    if (size < 8 || le32(d) != 20000630u) throw fail("not an OpenEXR file");
    const uint32_t version = le32(d + 4);
    if ((version & 0xff) != 2) throw fail("unsupported file version");
    if (version & 0x200) throw fail("tiled images are not read");
    if (version & 0x1800) throw fail("multi-part and deep images are not read");
    // header attributes: name, type name, size, value; an empty name ends the header
    size_t pos = 8;
    auto cstr = [&](std::string& out) {
        const size_t e = data.find('\0', pos);
        if (e == std::string::npos) throw fail("truncated header");
        out = data.substr(pos, e - pos);
        pos = e + 1;
    };
    std::vector<ExrChannel> channels;
    int compression = -1, line_order = 0;
    int32_t dw[4] = {0, 0, -1, -1};
    bool have_dw = false;
    for (;;) {
        std::string name, type;
        cstr(name);
        if (name.empty()) break;
        cstr(type);
        if (pos + 4 > size) throw fail("truncated header");
        const uint32_t n = le32(d + pos);
        pos += 4;
        if (pos + n > size) throw fail("truncated attribute " + name);
        const unsigned char* v = d + pos;
        if (name == "channels" && type == "chlist") {
            size_t q = 0;
            while (q < n && v[q] != 0) {
                const size_t e = data.find('\0', pos + q);
                if (e == std::string::npos || e + 17 > pos + n) throw fail("bad channel list");
                ExrChannel c;
                c.name = data.substr(pos + q, e - pos - q);
                const unsigned char* r = d + e + 1;
                c.type = (int)le32(r);
                const int32_t xs = (int32_t)le32(r + 8), ys = (int32_t)le32(r + 12);
                if (xs != 1 || ys != 1) throw fail("subsampled channel " + c.name);
                if (c.type < 0 || c.type > 2) throw fail("bad pixel type");
                channels.push_back(c);
                q = e + 17 - pos;
            }
        } else if (name == "compression" && n >= 1) {
            compression = v[0];
        } else if (name == "dataWindow" && n >= 16) {
            for (int k = 0; k < 4; ++k) dw[k] = (int32_t)le32(v + 4 * k);
            have_dw = true;
        } else if (name == "lineOrder" && n >= 1) {
            line_order = v[0];
        }
        pos += n;
    }
    if (channels.empty() || !have_dw || compression < 0) throw fail("missing channels, dataWindow or compression");
    if (line_order > 1) throw fail("random line order is not read");
    int lines_per_chunk = 0;
    switch (compression) {
        case 0: case 1: case 2: lines_per_chunk = 1; break;
        case 3: lines_per_chunk = 16; break;
        default: throw fail("compression " + std::to_string(compression) + " is not read (NONE, RLE, ZIPS, ZIP are)");
    }
    const int64_t W = (int64_t)dw[2] - dw[0] + 1, H = (int64_t)dw[3] - dw[1] + 1;
    if (W <= 0 || H <= 0 || W * H > ((int64_t)1 << 28)) throw fail("bad data window");
    int bytes_px = 0;
    for (const auto& c : channels) {
        if (c.type == 0) throw fail("UINT channel " + c.name + " is not read");
        bytes_px += c.type == 1 ? 2 : 4;
    }
    // channel planes, one float per pixel, rows in data-window order
    std::vector<std::vector<float>> plane(channels.size(), std::vector<float>((size_t)(W * H)));
    const int64_t chunks = (H + lines_per_chunk - 1) / lines_per_chunk;
    if (pos + 8 * (size_t)chunks > size) throw fail("truncated offset table");
    for (int64_t k = 0; k < chunks; ++k) {
        uint64_t off = 0;
        std::memcpy(&off, d + pos + 8 * k, 8);
        if (off + 8 > size) throw fail("bad chunk offset");
        const int32_t y0 = (int32_t)le32(d + off);
        const uint32_t packed = le32(d + off + 4);
        if (off + 8 + packed > size) throw fail("truncated chunk");
        if (y0 < dw[1] || y0 > dw[3]) throw fail("chunk outside the data window");
        const int64_t lines = std::min<int64_t>(lines_per_chunk, (int64_t)dw[3] - y0 + 1);
        const size_t raw_size = (size_t)(lines * W * bytes_px);
        const unsigned char* src = d + off + 8;
        std::vector<unsigned char> raw;
        if (compression == 0 || packed == raw_size) {  // stored: the codec did not pay
            if (packed != raw_size) throw fail("bad chunk size");
            raw.assign(src, src + packed);
        } else if (compression == 1) {
            raw.reserve(raw_size);
            for (size_t i = 0; i < packed;) {
                const int count = (signed char)src[i++];
                if (count < 0) {
                    if (i + (size_t)(-count) > packed) throw fail("bad RLE data");
                    raw.insert(raw.end(), src + i, src + i - count);
                    i += (size_t)(-count);
                } else {
                    if (i >= packed) throw fail("bad RLE data");
                    raw.insert(raw.end(), (size_t)count + 1, src[i++]);
                }
            }
            if (raw.size() != raw_size) throw fail("bad RLE size");
            undo_predictor_and_split(raw);
        } else {
            raw.resize(raw_size);
            uLongf out_len = (uLongf)raw_size;
            if (uncompress(raw.data(), &out_len, src, packed) != Z_OK || out_len != raw_size)
                throw fail("bad ZIP data");
            undo_predictor_and_split(raw);
        }
        // lines of the chunk; per line, each channel's row of values (little-endian)
        const unsigned char* p = raw.data();
        for (int64_t ln = 0; ln < lines; ++ln) {
            const int64_t row = (int64_t)y0 - dw[1] + ln;
            for (size_t c = 0; c < channels.size(); ++c) {
                float* out = plane[c].data() + row * W;
                if (channels[c].type == 1) {
                    for (int64_t x = 0; x < W; ++x, p += 2) out[x] = half_to_float((uint16_t)(p[0] | p[1] << 8));
                } else {
                    for (int64_t x = 0; x < W; ++x, p += 4) std::memcpy(out + x, p, 4);
                }
            }
        }
    }
    // LoadEXR's channel mapping: names without their layer prefix; R, G, B and A are looked
    // up among the first four channels (header order); one channel fills all four values;
    // otherwise R, G and B are required and a missing A reads 1
    TextureImage t;
    t.width = (int)W;
    t.height = (int)H;
    t.is_float = true;
    t.rgba.clear();
    t.rgbaf.assign((size_t)(4 * W * H), 0.f);
    int idx[4] = {-1, -1, -1, -1};
    const size_t first = std::min<size_t>(channels.size(), 4);
    for (size_t c = 0; c < first; ++c) {
        std::string nm = channels[c].name;
        const size_t dot = nm.find_last_of('.');
        if (dot != std::string::npos) nm = nm.substr(dot + 1);
        if (nm == "R") idx[0] = (int)c;
        else if (nm == "G") idx[1] = (int)c;
        else if (nm == "B") idx[2] = (int)c;
        else if (nm == "A") idx[3] = (int)c;
    }
    for (int64_t i = 0; i < W * H; ++i) {
        float* o = t.rgbaf.data() + 4 * i;
        if (channels.size() == 1) {
            o[0] = o[1] = o[2] = o[3] = plane[0][i];
        } else {
            if (idx[0] < 0 || idx[1] < 0 || idx[2] < 0) throw fail("R, G or B channel not found");
            for (int k = 0; k < 3; ++k) o[k] = plane[idx[k]][i];
            o[3] = idx[3] >= 0 ? plane[idx[3]][i] : 1.f;
        }
    }
    return t;
}

TextureImage load_texture_image(const std::string& path) {
    // the name's text after its last '.', as written (Utils/Utils.h getFileNamePostfix)
    const size_t dot = path.find_last_of('.');
    const std::string postfix = dot == std::string::npos ? "" : path.substr(dot + 1);
    if (postfix == "exr") return load_exr(path);
    const bool invert_gamma = postfix == "png" || postfix == "tga";
    std::string ext = postfix;
    for (auto& ch : ext) ch = (char)std::tolower((unsigned char)ch);
    if (ext != "png") throw ParseError("texture " + path + ": only PNG and OpenEXR images are read (got '" + postfix + "')");
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
            if (invert_gamma)  // names ending in "png": inverse gamma, truncated to 8 bits
                for (int c = 0; c < 3; ++c) px[c] = (unsigned char)(255.f * inverse_gamma(px[c] / 255.f));
            std::memcpy(out + 4 * x, px, 4);
        }
    }
    return t;
}

}  // namespace cavpbrt

// Host-only: an OpenEXR image as the texture loader reads it (RGBA floats, no GPU).
extern "C" cav_status cav_load_texture_exr(const char* path, float* rgba, int64_t capacity_floats, int* width,
                                           int* height, char* err, int err_len) {
    if (!path || !width || !height) return CAV_ERR_INVALID_ARGUMENT;
    try {
        const cavpbrt::TextureImage t = cavpbrt::load_exr(path);
        *width = t.width;
        *height = t.height;
        if (!rgba) return CAV_OK;  // size query
        if (capacity_floats < (int64_t)t.rgbaf.size()) {
            if (err && err_len > 0) {
                std::strncpy(err, "cav_load_texture_exr: output buffer too small", (size_t)err_len - 1);
                err[err_len - 1] = 0;
            }
            return CAV_ERR_INVALID_ARGUMENT;
        }
        std::memcpy(rgba, t.rgbaf.data(), t.rgbaf.size() * sizeof(float));
    } catch (const std::exception& e) {
        if (err && err_len > 0) {
            std::strncpy(err, e.what(), (size_t)err_len - 1);
            err[err_len - 1] = 0;
        }
        return CAV_ERR_INVALID_ARGUMENT;
    }
    return CAV_OK;
}

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
