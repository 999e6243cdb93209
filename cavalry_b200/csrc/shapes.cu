// Host-side shape ingestion for the .pbrt loader: the PLY reader behind "plymesh" /
// "trianglemesh" with a "filename" (Core/TriangleMesh.cu:53-108, which reads through the
// happly library), and the sphere and disk meshes the reference tessellates for those shapes
// (ShapeMesh/Sphere.cu:3-94, ShapeMesh/Disk.cu:4-50).
//
// Host code only; it is a .cu file so that the sphere's vector normalisation calls the CUDA
// toolkit's host rsqrtf, as the reference's Sphere.cu does (its helper_math normalize).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <sstream>
#include <string>
#include <vector>

#include "pbrt.h"

namespace cavpbrt {

namespace {

// ------------------------------------------------------------------ PLY
enum PlyType { kI8, kU8, kI16, kU16, kI32, kU32, kF32, kF64 };

int ply_type(const std::string& t, const std::string& path) {
    if (t == "char" || t == "int8") return kI8;
    if (t == "uchar" || t == "uint8") return kU8;
    if (t == "short" || t == "int16") return kI16;
    if (t == "ushort" || t == "uint16") return kU16;
    if (t == "int" || t == "int32") return kI32;
    if (t == "uint" || t == "uint32") return kU32;
    if (t == "float" || t == "float32") return kF32;
    if (t == "double" || t == "float64") return kF64;
    throw ParseError("read ply file failed, unknown property type '" + t + "' in " + path);
}

int type_size(int t) {
    switch (t) {
        case kI8: case kU8: return 1;
        case kI16: case kU16: return 2;
        case kI32: case kU32: case kF32: return 4;
        default: return 8;
    }
}

struct PlyProp {
    std::string name;
    int type = kF32;
    bool list = false;
    int count_type = kU8;
};

struct PlyElem {
    std::string name;
    int64_t count = 0;
    std::vector<PlyProp> props;
};

// The fewest bytes one row of an element can take: binary, its scalar properties and the
// count of each list; ASCII, one character per scalar or list count.  A header whose element
// count cannot fit in the rest of the file is refused with this before anything is allocated
// for the element (a damaged count would otherwise reserve gigabytes first).
size_t min_row_bytes(const PlyElem& e, int fmt) {
    size_t b = 0;
    for (const PlyProp& p : e.props) b += fmt == 0 ? 1 : (size_t)type_size(p.list ? p.count_type : p.type);
    return b;
}

// Sequential reader over the body: binary (either byte order) or ASCII tokens.
struct PlyBody {
    const std::string& data;
    size_t pos;
    int fmt;  // 0 ascii, 1 binary little endian, 2 binary big endian
    const std::string& path;

    double read(int t) {
        if (fmt == 0) {
            while (pos < data.size() && std::isspace((unsigned char)data[pos])) ++pos;
            if (pos >= data.size()) throw ParseError("read ply file failed, unexpected end of data in " + path);
            const char* b = data.c_str() + pos;
            char* e = nullptr;
            double v = std::strtod(b, &e);
            if (e == b) throw ParseError("read ply file failed, bad number in " + path);
            pos += (size_t)(e - b);
            return v;
        }
        const int n = type_size(t);
        if (pos + n > data.size()) throw ParseError("read ply file failed, unexpected end of data in " + path);
        unsigned char b[8];
        std::memcpy(b, data.data() + pos, n);
        pos += n;
        if (fmt == 2)
            for (int k = 0; k < n / 2; ++k) std::swap(b[k], b[n - 1 - k]);
        switch (t) {
            case kI8: { int8_t v; std::memcpy(&v, b, 1); return v; }
            case kU8: return b[0];
            case kI16: { int16_t v; std::memcpy(&v, b, 2); return v; }
            case kU16: { uint16_t v; std::memcpy(&v, b, 2); return v; }
            case kI32: { int32_t v; std::memcpy(&v, b, 4); return v; }
            case kU32: { uint32_t v; std::memcpy(&v, b, 4); return v; }
            case kF32: { float v; std::memcpy(&v, b, 4); return v; }
            default: { double v; std::memcpy(&v, b, 8); return v; }
        }
    }
};

// ------------------------------------------------------------------ shapes
struct V3 {
    float x, y, z;
};
V3 vadd(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 vscale(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
// helper_math normalize: v * rsqrtf(dot(v, v))
V3 vnormalize(V3 v) {
    const float inv = rsqrtf(v.x * v.x + v.y * v.y + v.z * v.z);
    return vscale(v, inv);
}

}  // namespace

PlyMesh read_ply(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw ParseError("read ply file failed, cannot open " + path);
    const std::string data((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    size_t pos = 0;
    auto next_line = [&]() {
        const size_t e = data.find('\n', pos);
        if (e == std::string::npos) throw ParseError("read ply file failed, header not terminated in " + path);
        std::string l = data.substr(pos, e - pos);
        pos = e + 1;
        if (!l.empty() && l.back() == '\r') l.pop_back();
        return l;
    };
    if (next_line() != "ply") throw ParseError("read ply file failed, not a PLY file: " + path);
    int fmt = -1;
    std::vector<PlyElem> elems;
    for (;;) {
        std::istringstream ss(next_line());
        std::string kw;
        ss >> kw;
        if (kw.empty() || kw == "comment" || kw == "obj_info") continue;
        if (kw == "end_header") break;
        if (kw == "format") {
            std::string name;
            ss >> name;
            if (name == "ascii") fmt = 0;
            else if (name == "binary_little_endian") fmt = 1;
            else if (name == "binary_big_endian") fmt = 2;
            else throw ParseError("read ply file failed, unknown format '" + name + "' in " + path);
        } else if (kw == "element") {
            PlyElem e;
            ss >> e.name >> e.count;
            if (!ss || e.count < 0) throw ParseError("read ply file failed, bad element line in " + path);
            elems.push_back(e);
        } else if (kw == "property") {
            if (elems.empty()) throw ParseError("read ply file failed, property before element in " + path);
            PlyProp p;
            std::string t;
            ss >> t;
            if (t == "list") {
                std::string ct, it;
                ss >> ct >> it >> p.name;
                p.list = true;
                p.count_type = ply_type(ct, path);
                p.type = ply_type(it, path);
            } else {
                p.type = ply_type(t, path);
                ss >> p.name;
            }
            elems.back().props.push_back(p);
        } else {
            throw ParseError("read ply file failed, unexpected header line '" + kw + "' in " + path);
        }
    }
    if (fmt < 0) throw ParseError("read ply file failed, no format line in " + path);
    PlyMesh m;
    bool have_vertex = false, have_face = false;
    PlyBody body{data, pos, fmt, path};
    for (const PlyElem& e : elems) {
        const size_t row = min_row_bytes(e, fmt);
        const size_t left = body.pos <= data.size() ? data.size() - body.pos : 0;
        if (row > 0 && (uint64_t)e.count > left / row)
            throw ParseError("read ply file failed, element '" + e.name + "' count " + std::to_string(e.count) +
                             " exceeds the data in " + path);
        if (e.name == "vertex") {
            have_vertex = true;
            int ix = -1, iy = -1, iz = -1, inx = -1, iny = -1, inz = -1, iu = -1, iv = -1;
            for (size_t k = 0; k < e.props.size(); ++k) {
                const std::string& n = e.props[k].name;
                if (e.props[k].list) continue;
                if (n == "x") ix = (int)k;
                else if (n == "y") iy = (int)k;
                else if (n == "z") iz = (int)k;
                else if (n == "nx") inx = (int)k;
                else if (n == "ny") iny = (int)k;
                else if (n == "nz") inz = (int)k;
                else if (n == "u") iu = (int)k;
                else if (n == "v") iv = (int)k;
            }
            if (ix < 0 || iy < 0 || iz < 0) throw ParseError("read ply file failed, vertex x/y/z missing in " + path);
            const bool normals = inx >= 0 && iny >= 0 && inz >= 0;
            const bool uvs = iu >= 0 && iv >= 0;
            m.positions.resize(3 * (size_t)e.count);
            if (normals) m.normals.resize(3 * (size_t)e.count);
            if (uvs) m.uvs.resize(2 * (size_t)e.count);
            bool all_f32 = fmt == 1;  // binary little endian with float properties only: one block
            for (const PlyProp& p : e.props) all_f32 = all_f32 && !p.list && p.type == kF32;
            if (all_f32) {
                const size_t np = e.props.size(), bytes = 4 * np * (size_t)e.count;
                if (body.pos + bytes > data.size())
                    throw ParseError("read ply file failed, unexpected end of data in " + path);
                const char* base = data.data() + body.pos;
                auto col = [&](int64_t r, int k) {
                    float v;
                    std::memcpy(&v, base + 4 * (np * (size_t)r + (size_t)k), 4);
                    return v;
                };
                for (int64_t r = 0; r < e.count; ++r) {
                    m.positions[3 * r] = col(r, ix);
                    m.positions[3 * r + 1] = col(r, iy);
                    m.positions[3 * r + 2] = col(r, iz);
                    if (normals) {
                        m.normals[3 * r] = col(r, inx);
                        m.normals[3 * r + 1] = col(r, iny);
                        m.normals[3 * r + 2] = col(r, inz);
                    }
                    if (uvs) {
                        m.uvs[2 * r] = col(r, iu);
                        m.uvs[2 * r + 1] = col(r, iv);
                    }
                }
                body.pos += bytes;
                continue;
            }
            std::vector<double> rec(e.props.size());
            for (int64_t r = 0; r < e.count; ++r) {
                for (size_t k = 0; k < e.props.size(); ++k) {
                    const PlyProp& p = e.props[k];
                    if (p.list) {
                        const int64_t c = (int64_t)body.read(p.count_type);
                        for (int64_t q = 0; q < c; ++q) body.read(p.type);
                        rec[k] = 0;
                    } else {
                        rec[k] = body.read(p.type);
                    }
                }
                m.positions[3 * r] = (float)rec[ix];
                m.positions[3 * r + 1] = (float)rec[iy];
                m.positions[3 * r + 2] = (float)rec[iz];
                if (normals) {
                    m.normals[3 * r] = (float)rec[inx];
                    m.normals[3 * r + 1] = (float)rec[iny];
                    m.normals[3 * r + 2] = (float)rec[inz];
                }
                if (uvs) {
                    m.uvs[2 * r] = (float)rec[iu];
                    m.uvs[2 * r + 1] = (float)rec[iv];
                }
            }
        } else if (e.name == "face") {
            have_face = true;
            int il = -1;
            for (size_t k = 0; k < e.props.size(); ++k)
                if (e.props[k].list && e.props[k].name == "vertex_indices") il = (int)k;
            if (il < 0) throw ParseError("read ply file failed, face list 'vertex_indices' missing in " + path);
            m.indices.reserve(3 * (size_t)e.count);
            const PlyProp& lp = e.props[il];
            if (fmt == 1 && e.props.size() == 1 && lp.count_type == kU8 && (lp.type == kI32 || lp.type == kU32)) {
                // binary little endian, the index list alone: read each face's count byte and
                // indices straight from the buffer (the same values the generic path reads)
                size_t pos = body.pos;
                for (int64_t r = 0; r < e.count; ++r) {
                    if (pos + 1 > data.size())
                        throw ParseError("read ply file failed, unexpected end of data in " + path);
                    const int c = (unsigned char)data[pos];
                    if (c < 3) throw ParseError("read ply file failed, a face with fewer than 3 vertices in " + path);
                    if (pos + 1 + 4 * (size_t)c > data.size())
                        throw ParseError("read ply file failed, unexpected end of data in " + path);
                    for (int q = 0; q < 3; ++q) {  // TriangleMesh::createFromPLY keeps the first three
                        int32_t v;
                        std::memcpy(&v, data.data() + pos + 1 + 4 * q, 4);
                        m.indices.push_back(lp.type == kI32 ? (int)v : (int)(double)(uint32_t)v);
                    }
                    pos += 1 + 4 * (size_t)c;
                }
                body.pos = pos;
                continue;
            }
            for (int64_t r = 0; r < e.count; ++r) {
                for (size_t k = 0; k < e.props.size(); ++k) {
                    const PlyProp& p = e.props[k];
                    if (!p.list) {
                        body.read(p.type);
                        continue;
                    }
                    const int64_t c = (int64_t)body.read(p.count_type);
                    if ((int)k == il && c < 3)
                        throw ParseError("read ply file failed, a face with fewer than 3 vertices in " + path);
                    for (int64_t q = 0; q < c; ++q) {
                        const double v = body.read(p.type);
                        // TriangleMesh::createFromPLY keeps each face's first three indices
                        if ((int)k == il && q < 3) m.indices.push_back((int)v);
                    }
                }
            }
        } else {
            for (int64_t r = 0; r < e.count; ++r)
                for (const PlyProp& p : e.props) {
                    if (p.list) {
                        const int64_t c = (int64_t)body.read(p.count_type);
                        for (int64_t q = 0; q < c; ++q) body.read(p.type);
                    } else {
                        body.read(p.type);
                    }
                }
        }
    }
    if (!have_vertex || !have_face) throw ParseError("read ply file failed, vertex or face element missing in " + path);
    const int64_t nv = (int64_t)(m.positions.size() / 3);
    for (int v : m.indices)
        if (v < 0 || v >= nv) throw ParseError("read ply file failed, face index out of range in " + path);
    return m;
}

void sphere_mesh(float radius, std::vector<float>& pos_out, std::vector<float>& nrm_out, std::vector<int>& idx_out) {
    // an octahedron, subdivided four times; every split pushes three new midpoint vertices
    std::vector<V3> p = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    std::vector<int> cur = {0, 2, 4, 0, 2, 5, 0, 3, 4, 0, 3, 5, 1, 2, 4, 1, 2, 5, 1, 3, 4, 1, 3, 5};
    for (int level = 0; level < 4; ++level) {
        std::vector<int> next;
        next.reserve(cur.size() * 4);
        for (size_t t = 0; t < cur.size(); t += 3) {
            const int i0 = cur[t], i1 = cur[t + 1], i2 = cur[t + 2];
            const V3 p0 = p[i0], p1 = p[i1], p2 = p[i2];
            p.push_back(vnormalize(vscale(vadd(p0, p1), 0.5f)));
            const int i01 = (int)p.size() - 1;
            p.push_back(vnormalize(vscale(vadd(p0, p2), 0.5f)));
            const int i02 = (int)p.size() - 1;
            p.push_back(vnormalize(vscale(vadd(p1, p2), 0.5f)));
            const int i12 = (int)p.size() - 1;
            const int tri[12] = {i01, i02, i12, i0, i01, i02, i1, i01, i12, i2, i02, i12};
            next.insert(next.end(), tri, tri + 12);
        }
        cur.swap(next);
    }
    pos_out.resize(3 * p.size());
    nrm_out.resize(3 * p.size());
    for (size_t k = 0; k < p.size(); ++k) {
        nrm_out[3 * k] = p[k].x;  // normal before the normal transform: the unit position
        nrm_out[3 * k + 1] = p[k].y;
        nrm_out[3 * k + 2] = p[k].z;
        const V3 q = vscale(p[k], radius);
        pos_out[3 * k] = q.x;
        pos_out[3 * k + 1] = q.y;
        pos_out[3 * k + 2] = q.z;
    }
    idx_out = cur;
}

void disk_mesh(float radius, float height, std::vector<float>& pos_out, std::vector<int>& idx_out) {
    const int segments = 360;
    pos_out.clear();
    idx_out.clear();
    for (int s = 0; s < segments; ++s) {
        const float theta = (float)(2.f * 3.14159265358979323846 * (float)s / (float)segments);
        pos_out.push_back(sinf(theta) * radius);
        pos_out.push_back(cosf(theta) * radius);
        pos_out.push_back(height);
    }
    pos_out.push_back(0.f);  // the centre, last
    pos_out.push_back(0.f);
    pos_out.push_back(height);
    for (int s = 0; s < segments; ++s) {
        idx_out.push_back((s + 1) % segments);
        idx_out.push_back(s);
        idx_out.push_back(segments);
    }
}

}  // namespace cavpbrt
