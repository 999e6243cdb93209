// .pbrt lexer and parser (host C++17).  Behaviour follows the reference's hand-written
// loader so that every scene it accepts loads to the same flat scene:
//   lexing    SceneLoading/Lexing.cu:8-52 (whitespace, '#' comments, brackets, keywords of
//             letters only and from a fixed set :106-107, quoted strings split on spaces,
//             numbers made of [0-9.-e] only, a leading '.' read as "0.")
//   parsing   SceneLoading/Parsing.cu: object definitions :67-106 (typed parameter names keep
//             their last word), LookAt through lookAtLH :196-204, Translate/Rotate/Scale/
//             Transform :120-173, scene-wide options :175-266 (the --spp/--integrator/--output
//             overrides :208-228, default pixel filter "triangle"), world subsections
//             :270-387 (AttributeBegin/End nesting, Material / MakeNamedMaterial /
//             NamedMaterial, AreaLightSource bound to the next Shape, ReverseOrientation,
//             Include spliced in place).
//   shapes    Core/TriangleMesh.cu:119-186 ("P", "indices", optional "N", or a PLY "filename"
//             read by shapes.cu), ShapeMesh/ShapeMesh.h:8-24 (tessellated sphere and disk).
//   materials Materials/{MatteMaterial,Plastic,Glass,Mirror}.h createFromParams defaults.
#include "pbrt.h"

#include <complex>

#include "../../include/cavalry.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <cfloat>
#include <charconv>
#include <deque>
#include <cstdlib>
#include <cerrno>
#include <filesystem>
#include <fstream>
#include <memory>
#include <map>
#include <set>
#include <sstream>

namespace cavpbrt {

float Params::num(const std::string& k) const {
    auto it = nums.find(k);
    if (it != nums.end()) return it->second;
    auto jt = num_lists.find(k);
    if (jt != num_lists.end() && !jt->second.empty()) return jt->second[0];
    throw ParseError("missing numeric parameter '" + k + "'");
}
const std::vector<float>& Params::list(const std::string& k) const {
    auto it = num_lists.find(k);
    if (it == num_lists.end()) throw ParseError("missing list parameter '" + k + "'");
    return it->second;
}
const std::string& Params::str(const std::string& k) const {
    auto it = strings.find(k);
    if (it != strings.end()) return it->second;
    auto jt = string_lists.find(k);
    if (jt != string_lists.end() && !jt->second.empty()) return jt->second[0];
    throw ParseError("missing string parameter '" + k + "'");
}

// ------------------------------------------------------------------ matrices
Mat4 identity() {
    Mat4 m{};
    m[0] = m[5] = m[10] = m[15] = 1.f;
    return m;
}

Mat4 mul(const Mat4& a, const Mat4& b) {
    Mat4 r{};
    for (int c = 0; c < 4; ++c)
        for (int rr = 0; rr < 4; ++rr) {
            float s = 0.f;
            for (int k = 0; k < 4; ++k) s += a[k * 4 + rr] * b[c * 4 + k];
            r[c * 4 + rr] = s;
        }
    return r;
}

// General 4x4 inverse by Gauss-Jordan elimination in double (column-major in and out).
Mat4 inverse(const Mat4& m) {
    double inv[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 8; ++c) inv[r][c] = c < 4 ? m[c * 4 + r] : (c - 4 == r ? 1.0 : 0.0);
    for (int c = 0; c < 4; ++c) {
        int piv = c;
        for (int r = c + 1; r < 4; ++r)
            if (std::fabs(inv[r][c]) > std::fabs(inv[piv][c])) piv = r;
        if (inv[piv][c] == 0.0) throw ParseError("singular transform");
        if (piv != c)
            for (int k = 0; k < 8; ++k) std::swap(inv[piv][k], inv[c][k]);
        double d = inv[c][c];
        for (int k = 0; k < 8; ++k) inv[c][k] /= d;
        for (int r = 0; r < 4; ++r) {
            if (r == c) continue;
            double f = inv[r][c];
            for (int k = 0; k < 8; ++k) inv[r][k] -= f * inv[c][k];
        }
    }
    Mat4 out{};
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) out[c * 4 + r] = (float)inv[r][c + 4];
    return out;
}

void apply_point(const Mat4& m, const float* v, float* out) {
    float t[4];
    for (int r = 0; r < 4; ++r) t[r] = m[0 * 4 + r] * v[0] + m[1 * 4 + r] * v[1] + m[2 * 4 + r] * v[2] + m[3 * 4 + r];
    out[0] = t[0] / t[3];
    out[1] = t[1] / t[3];
    out[2] = t[2] / t[3];
}

static void apply_vector3(const Mat4& m, const float* v, float* out) {  // glm::mat3(m) * v
    for (int r = 0; r < 3; ++r) out[r] = m[0 * 4 + r] * v[0] + m[1 * 4 + r] * v[1] + m[2 * 4 + r] * v[2];
}

static Mat4 translate(const Mat4& m, float x, float y, float z) {
    Mat4 r = m;
    for (int k = 0; k < 4; ++k) r[12 + k] = m[0 + k] * x + m[4 + k] * y + m[8 + k] * z + m[12 + k];
    return r;
}

static Mat4 scale(const Mat4& m, float x, float y, float z) {
    Mat4 r = m;
    for (int k = 0; k < 4; ++k) {
        r[0 + k] = m[0 + k] * x;
        r[4 + k] = m[4 + k] * y;
        r[8 + k] = m[8 + k] * z;
    }
    return r;
}

// Rotation by `deg` degrees about `axis` (right-multiplied, as glm::rotate does).
static Mat4 rotate(const Mat4& m, float deg, float ax, float ay, float az) {
    const float a = deg * 3.14159265358979323846f / 180.f;
    const float c = std::cos(a), s = std::sin(a);
    float len = std::sqrt(ax * ax + ay * ay + az * az);
    if (len == 0.f) throw ParseError("Rotate about a zero axis");
    ax /= len;
    ay /= len;
    az /= len;
    const float t = 1.f - c;
    Mat4 R = identity();
    R[0] = c + t * ax * ax;
    R[1] = t * ax * ay + s * az;
    R[2] = t * ax * az - s * ay;
    R[4] = t * ay * ax - s * az;
    R[5] = c + t * ay * ay;
    R[6] = t * ay * az + s * ax;
    R[8] = t * az * ax + s * ay;
    R[9] = t * az * ay - s * ax;
    R[10] = c + t * az * az;
    return mul(m, R);
}

// Left-handed look-at view matrix (world -> camera, camera looks down +z).
static Mat4 look_at_lh(const float* eye, const float* center, const float* up) {
    auto norm = [](float* v) {
        float l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        if (l == 0.f) throw ParseError("degenerate LookAt");
        v[0] /= l;
        v[1] /= l;
        v[2] /= l;
    };
    auto cross = [](const float* a, const float* b, float* o) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = a[2] * b[0] - a[0] * b[2];
        o[2] = a[0] * b[1] - a[1] * b[0];
    };
    float f[3] = {center[0] - eye[0], center[1] - eye[1], center[2] - eye[2]};
    norm(f);
    float s[3];
    cross(up, f, s);
    norm(s);
    float u[3];
    cross(f, s, u);
    Mat4 r = identity();
    r[0] = s[0];
    r[4] = s[1];
    r[8] = s[2];
    r[1] = u[0];
    r[5] = u[1];
    r[9] = u[2];
    r[2] = f[0];
    r[6] = f[1];
    r[10] = f[2];
    r[12] = -(s[0] * eye[0] + s[1] * eye[1] + s[2] * eye[2]);
    r[13] = -(u[0] * eye[0] + u[1] * eye[1] + u[2] * eye[2]);
    r[14] = -(f[0] * eye[0] + f[1] * eye[1] + f[2] * eye[2]);
    return r;
}

float roughness_to_alpha(float roughness) {
    roughness = std::max(roughness, 1e-3f);
    float x = std::log(roughness);
    return 1.62142f + 0.819955f * x + 0.1734f * x * x + 0.0171201f * x * x * x + 0.000640711f * x * x * x * x;
}

// -------------------------------------------------------------------- lexer
namespace {

enum class Tok { Keyword, String, Num, LBracket, RBracket };

struct StrRec {
    std::string text;                // keyword word / full string
    std::vector<std::string> words;  // string split on spaces
};

// 16 bytes: a mesh's numbers are most of a large file's tokens.  Keyword and string tokens
// point into the parser's arena (a deque, so the records never move).
struct Token {
    Tok type;
    float num = 0.f;
    const StrRec* s = nullptr;
    const std::string& text() const {
        static const std::string empty;
        return s ? s->text : empty;
    }
    const std::vector<std::string>& words() const {
        static const std::vector<std::string> none;
        return s ? s->words : none;
    }
};

std::string describe(const Token& t) {  // for messages
    if (t.type == Tok::LBracket) return "[";
    if (t.type == Tok::RBracket) return "]";
    if (t.type == Tok::Num) {
        char b[32];
        const auto r = std::to_chars(b, b + sizeof(b), t.num);
        return std::string(b, r.ptr);
    }
    return t.text();
}

const std::set<std::string>& keywords() {
    static const std::set<std::string> k = {
        "ReverseOrientation", "Material", "MakeNamedMedium", "MediumInterface", "NamedMedium", "Include",
        "PixelFilter", "Transform", "NamedMaterial", "TransformBegin", "TransformEnd", "AreaLightSource",
        "MakeNamedMaterial", "Texture", "Scale", "Rotate", "Translate", "LightSource", "LookAt", "Camera", "Film",
        "WorldBegin", "WorldEnd", "AttributeBegin", "AttributeEnd", "Sampler", "Shape", "Integrator"};
    return k;
}

bool is_letter(char c) { return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z'); }
bool is_digit(char c) { return c >= '0' && c <= '9'; }

std::vector<std::string> split_spaces(const std::string& s) {
    std::vector<std::string> out;
    size_t start = 0;
    for (;;) {
        size_t p = s.find(' ', start);
        out.push_back(s.substr(start, p == std::string::npos ? std::string::npos : p - start));
        if (p == std::string::npos) break;
        start = p + 1;
    }
    return out;
}

// NumToken::read (SceneLoading/Lexing.cu:88-103) converts the token's characters with
// std::stof after prefixing "0" to a leading '.'.  This gives std::stof's result and failures
// (no conversion, or ERANGE, which the reference leaves uncaught) on those characters:
// the characters are copied into a terminated buffer so that strtof cannot read past the
// token (it would accept "e+5" or "x1p3" that the lexer leaves for the next token).
float token_number(const char* p, size_t n) {
    char small[64];
    std::string big;
    char* buf = small;
    const bool dot = p[0] == '.';  // the lexer reads ".5" as "0.5"
    const size_t len = n + (dot ? 1 : 0);
    if (len + 1 > sizeof(small)) {
        big.resize(len + 1);
        buf = &big[0];
    }
    size_t k = 0;
    if (dot) buf[k++] = '0';
    std::memcpy(buf + k, p, n);
    buf[len] = 0;
    // std::from_chars and strtof both round correctly, so they agree on every normal result;
    // zero, subnormal, infinite or failed conversions take strtof's path, whose ERANGE rules
    // std::stof follows
    float v = 0.f;
    const std::from_chars_result r = std::from_chars(buf, buf + len, v);
    if (r.ec == std::errc() && r.ptr != buf && std::fabs(v) >= FLT_MIN && std::fabs(v) <= FLT_MAX) return v;
    char* end = nullptr;
    errno = 0;
    v = std::strtof(buf, &end);
    if (end == buf || errno == ERANGE) throw ParseError("Lexing Error: bad number '" + std::string(buf) + "'");
    return v;
}

std::vector<Token> lex(const std::string& input, std::deque<StrRec>& arena) {
    std::vector<Token> toks;
    toks.reserve(input.size() / 10 + 16);  // a mesh number with its separator is about 10 characters
    size_t pos = 0;
    while (pos < input.size()) {
        char c = input[pos];
        if (c == ' ' || c == '\n' || c == '\t' || c == '\r') {
            ++pos;
        } else if (c == '#') {
            while (pos < input.size() && input[pos] != '\n') ++pos;
            ++pos;
        } else if (c == '[') {
            toks.push_back({Tok::LBracket, 0.f, nullptr});
            ++pos;
        } else if (c == ']') {
            toks.push_back({Tok::RBracket, 0.f, nullptr});
            ++pos;
        } else if (is_letter(c)) {
            const size_t start = pos;
            while (pos < input.size() && is_letter(input[pos])) ++pos;
            std::string w = input.substr(start, pos - start);
            if (!keywords().count(w)) throw ParseError("Unrecognized Keyword: " + w);
            arena.push_back(StrRec{std::move(w), {}});
            toks.push_back({Tok::Keyword, 0.f, &arena.back()});
        } else if (c == '"') {
            ++pos;
            const size_t start = pos;
            while (pos < input.size() && input[pos] != '"') ++pos;
            if (pos == input.size()) throw ParseError("Lexing Error: Didn't find ending quotation");
            std::string raw = input.substr(start, pos - start);
            ++pos;
            std::vector<std::string> words = split_spaces(raw);
            arena.push_back(StrRec{std::move(raw), std::move(words)});
            toks.push_back({Tok::String, 0.f, &arena.back()});
        } else if (is_digit(c) || c == '-' || c == '.') {
            const size_t start = pos;
            while (pos < input.size() &&
                   (is_digit(input[pos]) || input[pos] == '-' || input[pos] == '.' || input[pos] == 'e'))
                ++pos;
            toks.push_back({Tok::Num, token_number(input.data() + start, pos - start), nullptr});
        } else {
            throw ParseError(std::string("unrecognized character ") + c);
        }
    }
    return toks;
}

std::string read_text(const std::filesystem::path& p) {
    std::ifstream f(p, std::ios::binary);
    if (!f) throw ParseError("fileNotFound: " + p.string());
    f.seekg(0, std::ios::end);
    const std::streamoff n = f ? (std::streamoff)f.tellg() : (std::streamoff)-1;
    if (n < 0) {
        // not seekable (a FIFO, /dev/stdin, process substitution): read the stream to its end
        f.clear();
        std::ostringstream all;
        all << f.rdbuf();
        if (f.bad()) throw ParseError("cannot read " + p.string());
        return all.str();
    }
    std::string text((size_t)n, '\0');
    f.seekg(0);
    if (n > 0 && !f.read(&text[0], n)) throw ParseError("cannot read " + p.string());
    return text;
}

// ------------------------------------------------------------------- parser
struct Parser {
    std::deque<StrRec> arena;  // keyword and string tokens' text (stable addresses)
    std::vector<Token> toks;
    size_t i = 0;
    std::filesystem::path base;
    Scene& scene;
    std::map<std::string, Material> named;
    // Included files whose spliced tokens are still ahead, innermost last: the file and the
    // index just past its tokens.  A file that includes itself, directly or through others,
    // would splice without end; it is refused instead.
    std::vector<std::pair<std::string, size_t>> includes;

    Parser(const std::string& text, std::filesystem::path b, Scene& s) : base(std::move(b)), scene(s) {
        toks = lex(text, arena);
    }

    const Token& peek(size_t k = 0) {
        if (i + k >= toks.size()) throw ParseError("unexpected end of input");
        return toks[i + k];
    }
    const Token& pop(Tok want, const char* what) {
        const Token& t = peek();
        if (t.type != want)
            throw ParseError(std::string("Parsing Error: ") + what + " expected at token " + std::to_string(i) + ": " +
                             describe(t));
        ++i;
        return t;
    }

    std::vector<float> num_list() {
        pop(Tok::LBracket, "[");
        std::vector<float> r;
        while (peek().type == Tok::Num) r.push_back(pop(Tok::Num, "number").num);
        pop(Tok::RBracket, "]");
        return r;
    }
    std::vector<std::string> string_list() {
        pop(Tok::LBracket, "[");
        std::vector<std::string> r;
        while (peek().type == Tok::String) r.push_back(pop(Tok::String, "string").text());
        pop(Tok::RBracket, "]");
        return r;
    }

    ObjectDef object() {
        ObjectDef d;
        d.keyword = pop(Tok::Keyword, "keyword").text();
        d.name = pop(Tok::String, "object name").words()[0];
        while (i < toks.size() && peek().type == Tok::String) {
            const Token& key = pop(Tok::String, "parameter name");
            std::string field = key.words().back();
            const Token& nx = peek();
            if (nx.type == Tok::String) {
                d.params.strings[field] = pop(Tok::String, "string").text();
            } else if (nx.type == Tok::Num) {
                d.params.nums[field] = pop(Tok::Num, "number").num;
            } else if (nx.type == Tok::LBracket) {
                const Token& el = peek(1);
                if (el.type == Tok::Num || el.type == Tok::RBracket) d.params.num_lists[field] = num_list();
                else if (el.type == Tok::String) d.params.string_lists[field] = string_list();
                else throw ParseError("Unaccepted List Element at token " + std::to_string(i + 1));
            } else {
                throw ParseError("Read Object failed at token " + std::to_string(i));
            }
        }
        d.defined = true;
        return d;
    }

    void skip_object() {  // readUntilNextKeyWorkd
        pop(Tok::Keyword, "keyword");
        while (i < toks.size() && peek().type != Tok::Keyword) ++i;
    }

    bool transform(Mat4& m) {
        const Token& t = peek();
        if (t.type != Tok::Keyword) throw ParseError("Keyword expected at token " + std::to_string(i));
        if (t.text() == "Translate" || t.text() == "Scale") {
            bool tr = t.text() == "Translate";
            ++i;
            float x = pop(Tok::Num, "number").num, y = pop(Tok::Num, "number").num, z = pop(Tok::Num, "number").num;
            m = tr ? translate(m, x, y, z) : scale(m, x, y, z);
            return true;
        }
        if (t.text() == "Rotate") {
            ++i;
            float a = pop(Tok::Num, "number").num;
            float x = pop(Tok::Num, "number").num, y = pop(Tok::Num, "number").num, z = pop(Tok::Num, "number").num;
            m = rotate(m, a, x, y, z);
            return true;
        }
        if (t.text() == "Transform") {
            ++i;
            std::vector<float> v = num_list();
            if (v.size() != 16) throw ParseError("Transform needs 16 numbers");
            Mat4 t4;
            std::memcpy(t4.data(), v.data(), 64);
            m = mul(t4, m);
            return true;
        }
        return false;
    }

    void scene_wide(const Overrides& ov) {
        Mat4 xf = identity();
        ObjectDef camera, film, integrator, sampler, filter;
        filter.defined = true;
        filter.name = "triangle";
        for (;;) {
            const Token& t = peek();
            if (t.type != Tok::Keyword) throw ParseError("Keyword expected at token " + std::to_string(i));
            if (t.text() == "WorldBegin") break;
            if (t.text() == "LookAt") {
                ++i;
                float e[3], c[3], u[3];
                for (float& v : e) v = pop(Tok::Num, "number").num;
                for (float& v : c) v = pop(Tok::Num, "number").num;
                for (float& v : u) v = pop(Tok::Num, "number").num;
                float e2[3], c2[3], u2[3];
                apply_point(xf, e, e2);
                apply_point(xf, c, c2);
                apply_vector3(xf, u, u2);
                xf = mul(look_at_lh(e2, c2, u2), xf);
            } else if (t.text() == "Camera") {
                camera = object();
            } else if (t.text() == "Film") {
                film = object();
            } else if (t.text() == "Sampler") {
                sampler = object();
            } else if (transform(xf)) {
            } else if (t.text() == "Integrator") {
                integrator = object();
            } else if (t.text() == "PixelFilter") {
                filter = object();
            } else {
                skip_object();
            }
        }
        if (!(camera.defined && film.defined && integrator.defined && sampler.defined))
            throw ParseError("incomplete scene-wide options: requires Camera, Film, Integrator, Sampler");
        if (camera.name != "perspective") throw ParseError("unsupported camera: " + camera.name);
        scene.fov_deg = camera.params.num("fov");
        scene.width = (int)film.params.num("xresolution");
        scene.height = (int)film.params.num("yresolution");
        if (film.params.has_string("filename")) scene.output = film.params.str("filename");
        if (!ov.output.empty()) scene.output = ov.output;
        scene.sampler = sampler.name;
        if (scene.sampler != "halton")
            throw ParseError("unsupported sampler: " + sampler.name + " (the time-seeded random sampler is not built)");
        scene.spp = (int)sampler.params.num("pixelsamples");
        if (ov.spp > 0) scene.spp = ov.spp;
        scene.integrator = ov.integrator.empty() ? integrator.name : ov.integrator;
        if (scene.integrator == "path" || scene.integrator == "rlpath") {
            scene.max_depth = (int)integrator.params.num("maxdepth");
        } else if (scene.integrator == "directlighting") {  // one bounce; maxdepth is not read
            scene.max_depth = 1;
        } else {
            scene.integrator = "path";  // CreateIntegrator.cu:23-25
            scene.max_depth = 8;
        }
        scene.filter_xwidth = filter.params.has_num("xwidth") ? filter.params.num("xwidth") : 1.f;
        scene.filter_ywidth = filter.params.has_num("ywidth") ? filter.params.num("ywidth") : 1.f;
        scene.camera_to_world = inverse(xf);
    }

    static void rgb(const Params& p, const char* k, float* out) {
        if (p.has_list(k)) {
            const auto& v = p.list(k);
            if (v.size() < 3) throw ParseError(std::string("parameter ") + k + " needs 3 values");
            out[0] = v[0];
            out[1] = v[1];
            out[2] = v[2];
        }
    }

    Material material(const ObjectDef& d, const std::string& type) {
        Material m;
        const Params& p = d.params;
        if (type == "matte") {
            m.type = kMatte;
            m.kd[0] = m.kd[1] = m.kd[2] = 1.f;
            rgb(p, "Kd", m.kd);
        } else if (type == "plastic") {
            m.type = kPlastic;
            m.kd[0] = m.kd[1] = m.kd[2] = 0.25f;
            rgb(p, "Kd", m.kd);
            rgb(p, "Ks", m.ks);
            float rough = p.has_num("roughness") ? p.num("roughness") : 0.1f;
            bool remap = p.has_string("remaproughness") ? p.str("remaproughness") == "true" : true;
            m.alpha_u = m.alpha_v = remap ? roughness_to_alpha(rough) : rough;
            m.eta = 1.5f;
        } else if (type == "glass") {  // Materials/Glass.h: specular, or microfacet when rough
            m.type = kGlass;
            rgb(p, "Kr", m.kr);
            rgb(p, "Kt", m.kt);
            m.eta = p.has_num("eta") ? p.num("eta") : (p.has_num("index") ? p.num("index") : 1.5f);
            float u = p.has_num("uroughness") ? p.num("uroughness") : 0.f;
            float v = p.has_num("vroughness") ? p.num("vroughness") : 0.f;
            if (p.has_num("roughness")) u = v = p.num("roughness");
            bool remap = p.has_string("remaproughness") ? p.str("remaproughness") == "true" : true;
            if (u != 0.f || v != 0.f) {  // perfectSpecular only when both are exactly 0
                m.alpha_u = remap ? roughness_to_alpha(u) : u;
                m.alpha_v = remap ? roughness_to_alpha(v) : v;
            }
        } else if (type == "mirror") {
            m.type = kMirror;
            m.mirror_kr = p.has_num("Kr") ? p.num("Kr") : 0.9f;
        } else if (type == "metal") {  // Materials/Metal.h
            m.type = kMetal;
            m.has_f0 = true;
            m.f0[0] = 0.955f; m.f0[1] = 0.638f; m.f0[2] = 0.538f;  // the reference's copper f0
            if (p.has_list("eta") && p.has_list("k")) {
                const auto& e = p.list("eta");
                const auto& k = p.list("k");
                if (e.size() < 3 || k.size() < 3) throw ParseError("metal eta / k need 3 values");
                for (int c = 0; c < 3; ++c) {  // |((eta - 1) + ik) / ((eta + 1) + ik)|^2
                    std::complex<float> z((float)e[c], (float)k[c]), one(1.f, 0.f);
                    m.f0[c] = (float)std::abs(std::pow((z - one) / (z + one), 2));
                }
            }
            float u = p.has_num("uroughness") ? p.num("uroughness") : 0.1f;
            float v = p.has_num("vroughness") ? p.num("vroughness") : 0.1f;
            if (p.has_num("roughness")) u = v = p.num("roughness");
            bool remap = p.has_string("remaproughness") ? p.str("remaproughness") == "true" : true;
            m.alpha_u = remap ? roughness_to_alpha(u) : u;
            m.alpha_v = remap ? roughness_to_alpha(v) : v;
        } else if (type == "substrate") {  // Materials/Substrate.h: FresnelBlend
            m.type = kSubstrate;
            m.kd[0] = m.kd[1] = m.kd[2] = 0.5f;
            m.ks[0] = m.ks[1] = m.ks[2] = 0.5f;
            rgb(p, "Kd", m.kd);
            rgb(p, "Ks", m.ks);
            float u = p.has_num("uroughness") ? p.num("uroughness") : 0.1f;
            float v = p.has_num("vroughness") ? p.num("vroughness") : 0.1f;
            if (p.has_num("roughness")) u = v = p.num("roughness");
            bool remap = p.has_string("remaproughness") ? p.str("remaproughness") == "true" : true;
            m.alpha_u = remap ? roughness_to_alpha(u) : u;
            m.alpha_v = remap ? roughness_to_alpha(v) : v;
        } else {
            // MaterialObject::createFromObjectDefinition falls back to matte for an unknown type
            m.type = kMatte;
            m.kd[0] = m.kd[1] = m.kd[2] = 1.f;
            rgb(p, "Kd", m.kd);
        }
        // "texture Kd": MatteMaterial multiplies its colour by the texel, Plastic and Substrate
        // take the texel as their diffuse colour (Materials/*.h createFromParams)
        if ((m.type == kMatte || m.type == kPlastic || m.type == kSubstrate) && p.has_string("Kd")) {
            auto it = texture_names.find(p.str("Kd"));
            if (it == texture_names.end()) throw ParseError("texture not found: " + p.str("Kd"));
            m.kd_texture = it->second;
        }
        return m;
    }
    std::map<std::string, int> texture_names;

    int add_material(const Material& m) {
        scene.materials.push_back(m);
        return (int)scene.materials.size() - 1;
    }

    void world(Mat4 xf, int current_material, bool& next_shape_light, bool top) {
        const Token& begin = pop(Tok::Keyword, "XXXBegin");
        const std::string bw = begin.text();
        if (bw.size() < 5 || bw.compare(bw.size() - 5, 5, "Begin") != 0) throw ParseError("XXXBegin expected");
        std::string name = bw.substr(0, bw.size() - 5);
        bool reverse = false;
        for (;;) {
            if (i >= toks.size()) {
                if (top) return;  // tolerate a missing WorldEnd
                throw ParseError("unterminated " + name + "Begin");
            }
            const Token& t = peek();
            if (t.type != Tok::Keyword) throw ParseError("Keyword expected at token " + std::to_string(i));
            const std::string w = t.text();
            if (w.size() > 3 && w.compare(w.size() - 3, 3, "End") == 0) {
                if (w.substr(0, w.size() - 3) != name) throw ParseError("Mismatching subsection names: " + w);
                break;
            } else if (w.size() > 5 && w.compare(w.size() - 5, 5, "Begin") == 0) {
                world(xf, current_material, next_shape_light, false);
            } else if (w == "Shape") {
                ObjectDef d = object();
                Mesh mesh;
                // positions through the CTM (apply), normals through transpose(inverse) of its
                // upper 3x3 and normalised (getTransformForNormal, Utils/MathsCommons.h:80-82)
                auto put_positions = [&](const std::vector<float>& P) {
                    size_t nv = P.size() / 3;
                    mesh.positions.resize(3 * nv);
                    for (size_t k = 0; k < nv; ++k) apply_point(xf, &P[3 * k], &mesh.positions[3 * k]);
                };
                auto put_normals = [&](const std::vector<float>& N) {
                    size_t nv = mesh.positions.size() / 3;
                    if (N.size() < 3 * nv) throw ParseError("N needs 3 values per vertex");
                    Mat4 inv = inverse(xf);
                    mesh.normals.resize(3 * nv);
                    for (size_t k = 0; k < nv; ++k) {
                        float n[3];
                        for (int r = 0; r < 3; ++r)
                            n[r] = inv[r * 4 + 0] * N[3 * k] + inv[r * 4 + 1] * N[3 * k + 1] + inv[r * 4 + 2] * N[3 * k + 2];
                        float l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
                        for (int r = 0; r < 3; ++r) mesh.normals[3 * k + r] = n[r] / l;
                    }
                };
                auto put_indices = [&](const std::vector<int>& I) {
                    const int nv = (int)(mesh.positions.size() / 3);
                    for (int v : I)
                        if (v < 0 || v >= nv) throw ParseError("triangle index out of range");
                    mesh.indices = I;
                };
                if (d.name == "trianglemesh" || d.name == "plymesh") {  // Core/TriangleMesh.cu:119-186
                    if (d.params.has_string("filename")) {
                        PlyMesh pm = read_ply((base / d.params.str("filename")).string());
                        put_positions(pm.positions);
                        put_indices(pm.indices);
                        if (!pm.normals.empty()) put_normals(pm.normals);
                        mesh.uvs = pm.uvs;
                    } else if (d.params.has_list("P") && d.params.has_list("indices")) {
                        put_positions(d.params.list("P"));
                        const auto& I = d.params.list("indices");
                        std::vector<int> ii(3 * (I.size() / 3));
                        for (size_t k = 0; k < ii.size(); ++k) ii[k] = (int)I[k];
                        put_indices(ii);
                        if (d.params.has_list("N")) put_normals(d.params.list("N"));
                        if (d.params.has_list("uv")) {
                            const auto& uv = d.params.list("uv");
                            if (uv.size() < mesh.positions.size() / 3 * 2) throw ParseError("uv needs 2 values per vertex");
                            mesh.uvs.assign(uv.begin(), uv.begin() + (long)(mesh.positions.size() / 3 * 2));
                        }
                    } else {
                        throw ParseError("No valid inputs for triangle mesh");
                    }
                } else if (d.name == "sphere") {  // ShapeMesh/Sphere.cu:3-94
                    const float radius = d.params.num("radius");
                    std::vector<float> P, N;
                    std::vector<int> I;
                    sphere_mesh(radius, P, N, I);
                    put_positions(P);
                    put_indices(I);
                    put_normals(N);
                    mesh.shape = 1;
                    const float o[3] = {0, 0, 0}, rx[3] = {radius, 0, 0};
                    float c[3], e[3];
                    apply_point(xf, o, c);
                    apply_point(xf, rx, e);
                    const float dx = c[0] - e[0], dy = c[1] - e[1], dz = c[2] - e[2];
                    mesh.sphere[0] = c[0];
                    mesh.sphere[1] = c[1];
                    mesh.sphere[2] = c[2];
                    mesh.sphere[3] = std::sqrt(dx * dx + dy * dy + dz * dz);
                } else if (d.name == "disk") {  // ShapeMesh/Disk.cu:4-50
                    const float radius = d.params.num("radius");
                    const float height = d.params.has_num("height") ? d.params.num("height") : 0.f;
                    std::vector<float> P;
                    std::vector<int> I;
                    disk_mesh(radius, height, P, I);
                    put_positions(P);
                    put_indices(I);
                    mesh.shape = 2;
                } else {
                    throw ParseError("ShapeMesh type not supported: " + d.name);
                }
                mesh.reverse_orientation = reverse;
                if (current_material < 0) {
                    Material gray;
                    gray.type = kMatte;
                    current_material = add_material(gray);
                }
                mesh.material = current_material;
                if (next_shape_light) {
                    mesh.light = (int)scene.lights.size() - 1;
                    scene.lights.back().mesh = (int)scene.meshes.size();
                    next_shape_light = false;
                }
                scene.meshes.push_back(std::move(mesh));
            } else if (w == "AreaLightSource") {
                ObjectDef d = object();
                if (d.name != "diffuse") throw ParseError("unsupported area light: " + d.name);
                Light l;
                if (d.params.has_list("L")) rgb(d.params, "L", l.L);
                else if (d.params.has_list("l")) rgb(d.params, "l", l.L);
                scene.lights.push_back(l);
                next_shape_light = true;
            } else if (w == "LightSource") {  // Lights/LightObject.h:89-127, Parsing.cu:336-342
                ObjectDef d = object();
                Light l;
                l.kind = 1;
                if (d.params.has_list("L")) rgb(d.params, "L", l.L);
                else if (d.params.has_list("l")) rgb(d.params, "l", l.L);
                l.world_to_light = inverse(xf);
                if (d.name == "infinite") {
                    if (d.params.has_list("scale")) rgb(d.params, "scale", l.L);
                    if (d.params.has_string("mapname")) {
                        scene.textures.push_back(load_texture_image((base / d.params.str("mapname")).string()));
                        l.texture = (int)scene.textures.size() - 1;
                    }
                    scene.environment = (int)scene.lights.size();
                } else {  // an unrecognised source stays in the light list as a black environment
                    l.L[0] = l.L[1] = l.L[2] = 0.f;
                }
                scene.lights.push_back(l);
            } else if (transform(xf)) {
            } else if (w == "MakeNamedMaterial") {
                ObjectDef d = object();
                named[d.name] = material(d, d.params.str("type"));
            } else if (w == "Material") {
                ObjectDef d = object();
                current_material = add_material(material(d, d.name));
            } else if (w == "NamedMaterial") {
                ++i;
                std::string n = pop(Tok::String, "material name").text();
                auto it = named.find(n);
                if (it == named.end()) throw ParseError("Named material not found: " + n);
                current_material = add_material(it->second);
            } else if (w == "Include") {
                const size_t at = i;  // the directive's own position decides which includes enclose it
                ++i;
                std::string file = pop(Tok::String, "file name").text();
                while (!includes.empty() && includes.back().second <= at) includes.pop_back();
                std::error_code ec;
                std::string key = std::filesystem::weakly_canonical(base / file, ec).string();
                if (ec) key = (base / file).string();
                for (const auto& open : includes)
                    if (open.first == key) throw ParseError("Include cycle: " + file + " includes itself");
                std::vector<Token> inc = lex(read_text(base / file), arena);
                toks.insert(toks.begin() + (long)i, inc.begin(), inc.end());
                for (auto& open : includes) open.second += inc.size();
                includes.emplace_back(key, i + inc.size());
            } else if (w == "ReverseOrientation") {
                ++i;
                reverse = true;
            } else if (w == "Texture") {  // Core/Texture.cu:12-25: an image, or one black texel
                ObjectDef d = object();
                TextureImage t;
                if (d.params.has_string("filename"))
                    t = load_texture_image((base / d.params.str("filename")).string());
                scene.textures.push_back(std::move(t));
                texture_names[d.name] = (int)scene.textures.size() - 1;
            } else {
                skip_object();
            }
        }
        ++i;  // the XXXEnd keyword
    }
};

}  // namespace

Scene load_string(const std::string& text, const std::string& base_dir, const Overrides& ov) {
    Scene scene;
    Parser p(text, std::filesystem::path(base_dir), scene);
    p.scene_wide(ov);
    bool next_light = false;
    p.world(identity(), -1, next_light, true);
    if (scene.meshes.empty()) throw ParseError("the scene has no shapes");
    if (scene.lights.empty()) throw ParseError("the scene has no lights");
    for (const Light& l : scene.lights)
        if (l.kind == 0 && l.mesh < 0) throw ParseError("AreaLightSource without a following Shape");
    return scene;
}

Scene load_file(const std::string& path, const Overrides& ov) {
    std::filesystem::path p(path);
    return load_string(read_text(p), p.parent_path().string(), ov);
}

}  // namespace cavpbrt

// Host-only parse for tools and CPU tests: fills a cav_scene_info_t and the camera-to-world
// matrix (16 floats, column-major) without touching the GPU.  `err` (or NULL) receives the
// parser's message, truncated to err_len bytes.
extern "C" cav_status cav_pbrt_load_triangles(const char* path, float* positions, int64_t max_vertices,
                                              int32_t* indices, int32_t* mesh_ids, int64_t max_triangles,
                                              int64_t* num_vertices, int64_t* num_triangles, char* err, int err_len) {
    if (!path || !num_vertices || !num_triangles) return CAV_ERR_INVALID_ARGUMENT;
    try {
        cavpbrt::Scene s = cavpbrt::load_file(path, cavpbrt::Overrides{});
        int64_t nv = 0, nt = 0;
        for (const auto& m : s.meshes) {
            nv += (int64_t)m.positions.size() / 3;
            nt += (int64_t)m.indices.size() / 3;
        }
        *num_vertices = nv;
        *num_triangles = nt;
        if (!positions && !indices && !mesh_ids) return CAV_OK;
        if ((positions && max_vertices < nv) || ((indices || mesh_ids) && max_triangles < nt))
            return CAV_ERR_INVALID_ARGUMENT;
        int64_t vb = 0, tb = 0;
        for (size_t mi = 0; mi < s.meshes.size(); ++mi) {
            const auto& m = s.meshes[mi];
            if (positions) std::memcpy(positions + 3 * vb, m.positions.data(), m.positions.size() * sizeof(float));
            const int64_t mt = (int64_t)m.indices.size() / 3;
            for (int64_t t = 0; t < mt; ++t) {
                if (indices)
                    for (int k = 0; k < 3; ++k) indices[3 * (tb + t) + k] = (int32_t)(m.indices[3 * t + k] + vb);
                if (mesh_ids) mesh_ids[tb + t] = (int32_t)mi;
            }
            vb += (int64_t)m.positions.size() / 3;
            tb += mt;
        }
    } catch (const std::exception& e) {
        if (err && err_len > 0) {
            std::strncpy(err, e.what(), (size_t)err_len - 1);
            err[err_len - 1] = 0;
        }
        return CAV_ERR_INVALID_ARGUMENT;
    }
    return CAV_OK;
}

extern "C" cav_status cav_pbrt_parse_info(const char* path, int spp_override, const char* integrator_override,
                                          cav_scene_info_t* info, float* camera_to_world16, char* err,
                                          int err_len) {
    if (!path || !info) return CAV_ERR_INVALID_ARGUMENT;
    cavpbrt::Overrides ov;
    ov.spp = spp_override;
    if (integrator_override) ov.integrator = integrator_override;
    try {
        cavpbrt::Scene s = cavpbrt::load_file(path, ov);
        info->width = s.width;
        info->height = s.height;
        info->spp = s.spp;
        info->max_depth = s.max_depth;
        int64_t tris = 0;
        for (const auto& m : s.meshes) tris += (int64_t)m.indices.size() / 3;
        info->triangles = tris;
        info->meshes = (int)s.meshes.size();
        info->lights = (int)s.lights.size();
        info->bvh_rounds = -1;
        info->integrator = s.integrator == "rlpath" ? 1 : (s.integrator == "directlighting" ? 3 : 0);
        if (camera_to_world16) std::memcpy(camera_to_world16, s.camera_to_world.data(), 64);
    } catch (const std::exception& e) {
        if (err && err_len > 0) {
            std::strncpy(err, e.what(), (size_t)err_len - 1);
            err[err_len - 1] = 0;
        }
        return CAV_ERR_INVALID_ARGUMENT;
    }
    return CAV_OK;
}
