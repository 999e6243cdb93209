// Host-side .pbrt scene loading: the lexer and recursive-descent parser of the pbrt-v3
// subset the reference reads (SceneLoading/Lexing.cu:8-107, SceneLoading/Parsing.cu:67-406),
// producing a flat scene description for the device renderer.  Errors are reported by
// throwing cavpbrt::ParseError (the reference prints and exit()s).
#pragma once

#include <array>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace cavpbrt {

struct ParseError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

using Mat4 = std::array<float, 16>;  // column-major, m[c * 4 + r] (the glm layout)

struct Params {
    std::map<std::string, std::string> strings;
    std::map<std::string, float> nums;
    std::map<std::string, std::vector<float>> num_lists;
    std::map<std::string, std::vector<std::string>> string_lists;
    // Core/Parameters.h:13-49: a number may also be read from the first element of a list,
    // a string from the first element of a string list.
    bool has_num(const std::string& k) const { return nums.count(k) != 0 || num_lists.count(k) != 0; }
    bool has_list(const std::string& k) const { return num_lists.count(k) != 0; }
    bool has_string(const std::string& k) const { return strings.count(k) != 0 || string_lists.count(k) != 0; }
    float num(const std::string& k) const;
    const std::vector<float>& list(const std::string& k) const;
    const std::string& str(const std::string& k) const;
};

struct ObjectDef {
    std::string keyword;
    std::string name;
    Params params;
    bool defined = false;
};

enum MaterialType : int { kMatte = 0, kMirror = 1, kSubstrate = 2, kMetal = 3, kGlass = 4, kPlastic = 5 };

struct Material {
    int type = kMatte;
    float kd[3] = {1, 1, 1};
    float ks[3] = {0.25f, 0.25f, 0.25f};
    float kr[3] = {1, 1, 1};
    float kt[3] = {1, 1, 1};
    float alpha_u = 0, alpha_v = 0;  // GGX alphas after the optional roughness remap
    float eta = 1.5f;
    float mirror_kr = 0.9f;
    bool has_f0 = false;             // metal: Fresnel f0 from a complex IOR (or the copper default)
    float f0[3] = {0, 0, 0};
    int kd_texture = -1;             // matte / plastic / substrate "texture Kd": index into Scene::textures
};

// An image texture as the reference holds it (Core/Texture.h): 8-bit RGBA texels read as
// normalized floats, rows bottom-up after stb_image's load flip (PNG), or FLOAT RGBA texels
// read as they are, rows in the file's order (OpenEXR through tinyexr's LoadEXR, no flip);
// bilinear filtering, wrapped normalized coordinates either way.
struct TextureImage {
    int width = 1, height = 1;
    std::vector<unsigned char> rgba{0, 0, 0, 0};  // 8-bit texels (is_float false)
    bool is_float = false;
    std::vector<float> rgbaf;                     // float texels (is_float true)
};
TextureImage load_texture_image(const std::string& path);
// OpenEXR (scanline, single part; NONE, RLE, ZIPS and ZIP compression; HALF and FLOAT
// channels) to RGBA floats as tinyexr's LoadEXR returns them.
TextureImage load_exr(const std::string& path);

struct Mesh {
    std::vector<float> positions;  // world space (transform applied), 3 per vertex
    std::vector<float> normals;    // 3 per vertex, or empty
    std::vector<float> uvs;        // 2 per vertex ("uv" / PLY u v), or empty
    std::vector<int> indices;      // 3 per triangle
    bool reverse_orientation = false;
    int material = 0;
    int light = -1;  // index into Scene::lights when the mesh is an area light
    int shape = 0;   // 0 triangle mesh, 1 tessellated sphere, 2 tessellated disk
    float sphere[4] = {0, 0, 0, 0};  // sphere: world centre and radius (light sampling)
};

// A PLY file's triangle data as TriangleMesh::createFromPLY reads it (Core/TriangleMesh.cu:53-108):
// float x/y/z (any numeric PLY type), optional nx/ny/nz and u/v, and the first three entries of
// every face's "vertex_indices" list.  ASCII and binary (either byte order) formats.
struct PlyMesh {
    std::vector<float> positions, normals, uvs;
    std::vector<int> indices;
};
PlyMesh read_ply(const std::string& path);

// The reference's shape meshes (ShapeMesh/Sphere.cu:3-94, ShapeMesh/Disk.cu:4-50): positions
// (and for the sphere unit normals before the normal transform) in object space.
void sphere_mesh(float radius, std::vector<float>& pos, std::vector<float>& nrm, std::vector<int>& idx);
void disk_mesh(float radius, float height, std::vector<float>& pos, std::vector<int>& idx);

struct Light {
    float L[3] = {1, 1, 1};
    int mesh = -1;     // diffuse area light: its mesh
    int kind = 0;      // 0 diffuse area light; 1 environment (LightSource "infinite", or an
                       // unrecognised LightSource, which the reference keeps as a black one)
    int texture = -1;  // environment: "mapname" image, index into Scene::textures
    Mat4 world_to_light{};
};

struct Scene {
    // camera
    float fov_deg = 90.f;
    Mat4 camera_to_world{};
    // film / sampler / filter / integrator
    int width = 0, height = 0;
    std::string output = "output.png";
    int spp = 1;
    std::string sampler = "halton";
    float filter_xwidth = 1.f, filter_ywidth = 1.f;
    std::string integrator = "path";
    int max_depth = 8;
    std::vector<Material> materials;
    std::vector<Mesh> meshes;
    std::vector<Light> lights;
    std::vector<TextureImage> textures;
    int environment = -1;  // the light that rays leaving the scene see (the last "infinite")
};

struct Overrides {
    int spp = -1;                 // --spp
    std::string integrator;       // --integrator
    std::string output;           // --output
};

Scene load_file(const std::string& path, const Overrides& ov);
Scene load_string(const std::string& text, const std::string& base_dir, const Overrides& ov);

// GGX roughness remap of the reference (BSDFs/MicrofacetDistribution.h roughnessToAlpha).
float roughness_to_alpha(float roughness);

Mat4 identity();
Mat4 mul(const Mat4& a, const Mat4& b);
Mat4 inverse(const Mat4& m);
void apply_point(const Mat4& m, const float* in, float* out);

}  // namespace cavpbrt
