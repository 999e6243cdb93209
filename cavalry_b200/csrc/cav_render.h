// Device-side scene records of the wavefront renderer (render.cu).
#pragma once

#include <stdint.h>

namespace cav {

// shape of a mesh (Core/TriangleMesh.h MeshShapeType): a tessellated sphere is sampled as a
// light by the cone it subtends (TriangleMesh::sample :110-116)
enum : int32_t { kShapeMesh = 0, kShapeSphere = 1, kShapeDisk = 2 };

struct RMesh {
    int32_t first_tri, tri_count;
    int32_t has_normals, reverse;
    int32_t material, light;
    float area;  // TriangleMesh::surfaceArea
    int32_t shape;
    float sphere[4];  // kShapeSphere: world centre and radius (TriangleMesh::shapeParams)
};

struct RMaterial {
    int32_t type;
    float kd[3], ks[3], kr[3], kt[3];
    float alpha_u, alpha_v, eta, mirror_kr;
    float f0[3];  // Schlick f0 of Fresnel::createFromIOR, computed on the host as the reference does
    int32_t kd_tex;  // "texture Kd": index into the scene's texture objects, or -1
};

enum : int32_t { kLightArea = 0, kLightEnvironment = 1 };

struct RLight {
    float L[3];
    int32_t mesh;  // area light: its mesh
    int32_t kind;  // kLightArea or kLightEnvironment (EnvironmentMap, Core/Light.h:43-122)
    int32_t tex;   // environment: its image texture, or -1
    float w2l[9];  // environment: mat3(worldToLight), row-major (r * 3 + c)
};

}  // namespace cav
