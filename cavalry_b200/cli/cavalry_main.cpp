// `cavalry` command line: the reference's CLI surface (main.cu:25-96) over the C ABI.
//
//   cavalry --input scene.pbrt [--output out.png] [--spp N] [--integrator path|rlpath]
//           [--bvh-opt-rounds R] [--pfm film.pfm] [--device D]
//
// Loads the scene with the host .pbrt parser, builds the BVH (R treelet rounds; -1 = the
// reference's default), renders on the GPU and writes the 8-bit PNG the reference writes
// (plus, with --pfm, the float film).
#include <cerrno>
#include <chrono>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cavalry.h"

static void usage() {
    std::fprintf(stderr,
                 "usage: cavalry --input scene.pbrt [--output out.png] [--spp N] [--integrator path|rlpath]\n"
                 "               [--bvh-opt-rounds R] [--pfm film.pfm] [--device D]\n");
}

// A whole decimal int or exit 2: the reference reads these flags as ints through cxxopts,
// which refuses anything else (std::atoi would read "abc" as 0 and overflow on long input).
static int int_arg(const char* name, const std::string& v) {
    errno = 0;
    char* end = nullptr;
    const long x = std::strtol(v.c_str(), &end, 10);
    if (v.empty() || end != v.c_str() + v.size() || errno == ERANGE || x < INT_MIN || x > INT_MAX) {
        std::fprintf(stderr, "invalid integer value '%s' for %s\n", v.c_str(), name);
        std::exit(2);
    }
    return (int)x;
}

int main(int argc, char** argv) {
    std::string input, output, integrator, pfm;
    int spp = -1, rounds = -1, device = 0;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        auto next = [&](const char* name) -> std::string {
            if (i + 1 >= argc) {
                std::fprintf(stderr, "missing value for %s\n", name);
                std::exit(2);
            }
            return argv[++i];
        };
        if (a == "--input") input = next("--input");
        else if (a == "--output") output = next("--output");
        else if (a == "--spp") spp = int_arg("--spp", next("--spp"));
        else if (a == "--integrator") integrator = next("--integrator");
        else if (a == "--bvh-opt-rounds") rounds = int_arg("--bvh-opt-rounds", next("--bvh-opt-rounds"));
        else if (a == "--pfm") pfm = next("--pfm");
        else if (a == "--device") device = int_arg("--device", next("--device"));
        else if (a == "--help" || a == "-h") {
            usage();
            return 0;
        } else {
            std::fprintf(stderr, "unknown argument %s\n", a.c_str());
            usage();
            return 2;
        }
    }
    if (input.empty()) {
        usage();
        return 2;
    }
    cav_ctx* ctx = nullptr;
    if (cav_ctx_create(device, &ctx) != CAV_OK) {
        std::fprintf(stderr, "cavalry: no usable CUDA device %d\n", device);
        return 1;
    }
    auto t0 = std::chrono::steady_clock::now();
    cav_scene* scene = nullptr;
    cav_status st = cav_scene_load_pbrt(ctx, input.c_str(), spp, integrator.empty() ? nullptr : integrator.c_str(),
                                        rounds, &scene);
    if (st != CAV_OK) {
        std::fprintf(stderr, "cavalry: %s: %s\n", cav_status_string(st), cav_last_error(ctx));
        cav_ctx_destroy(ctx);
        return 1;
    }
    auto t1 = std::chrono::steady_clock::now();
    cav_scene_info_t info;
    cav_scene_info(scene, &info);
    std::printf("scene: %lld triangles, %d meshes, %d lights, %dx%d, %d spp, depth %d, %d treelet rounds\n",
                (long long)info.triangles, info.meshes, info.lights, info.width, info.height, info.spp,
                info.max_depth, info.bvh_rounds);
    std::vector<float> sum(3 * (size_t)info.width * info.height), weight((size_t)info.width * info.height);
    float ms = 0.f;
    st = cav_render_to_host(ctx, scene, nullptr, sum.data(), weight.data(), &ms);
    if (st != CAV_OK) {
        std::fprintf(stderr, "cavalry: render failed: %s: %s\n", cav_status_string(st), cav_last_error(ctx));
        cav_scene_free(scene);
        cav_ctx_destroy(ctx);
        return 1;
    }
    std::printf("Preparation took %.1f ms\nRendering took %.1f ms\n",
                std::chrono::duration<double, std::milli>(t1 - t0).count(), ms);
    if (output.empty()) output = "output.png";
    std::vector<uint8_t> rgb(3 * (size_t)info.width * info.height);
    cav_film_to_rgb8(sum.data(), weight.data(), info.width, info.height, rgb.data());
    if (cav_write_png(output.c_str(), rgb.data(), info.width, info.height) != CAV_OK)
        std::fprintf(stderr, "cavalry: cannot write %s\n", output.c_str());
    if (!pfm.empty()) cav_write_pfm(pfm.c_str(), sum.data(), weight.data(), info.width, info.height);
    cav_scene_free(scene);
    cav_ctx_destroy(ctx);
    return 0;
}
