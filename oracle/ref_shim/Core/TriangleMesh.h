// Test-infrastructure shim (oracle only, never part of the product).
//
// Stands in for the reference's Core/TriangleMesh.h when its BVH sources
// (BVH/BVH.cu, BVH/Optimization.cu, BVH/BVH.h) and Core/Triangle.h are compiled
// verbatim into the golden/timing harness.  The real header drags in the scene
// parameter system, samplers and the variant machinery; the BVH path only touches
// the fields declared here:
//   Core/Triangle.h:173-174, :193-196, :211, :220, :228, :244-246
//   (positions/normals/texCoords/indices .gpu.data/.cpu.data, hasVertexNormals,
//    reverseOrientation, prim).
#pragma once

#include "../Utils/GpuCommons.h"
#include "../Utils/MathsCommons.h"
#include "IntersectionResult.h"
#include "Ray.h"

class Primitive;

template <typename T>
struct ShimBuffer {
    T* data = nullptr;
};

template <typename T>
struct ShimArrayPair {
    ShimBuffer<T> cpu;
    ShimBuffer<T> gpu;
};

class TriangleMesh {
public:
    int trianglesCount = 0;
    int verticesCount = 0;
    bool hasVertexNormals = false;
    bool reverseOrientation = false;
    ShimArrayPair<float3> positions;
    ShimArrayPair<float3> normals;
    ShimArrayPair<float2> texCoords;
    ShimArrayPair<int3> indices;
    int meshIndex = 0;
    Primitive* prim = nullptr;
};
