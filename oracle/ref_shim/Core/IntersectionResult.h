// Test-infrastructure shim (oracle only, never part of the product).
//
// Stands in for the reference's Core/IntersectionResult.h (:8-15) in the golden
// harness.  BVH::intersect (BVH/BVH.h:23-107) and Triangle::fillIntersectionInformation
// (Core/Triangle.h:95-136) write only these fields; the BSDF member and its
// variant dependencies are not on the traversal path.
#pragma once

#include "../Utils/GpuCommons.h"
#include "../Utils/MathsCommons.h"

class Primitive;

struct IntersectionResult {
    bool intersected = false;
    float distance;
    float3 position;
    float3 normal;
    float2 textureCoordinates;
    const Primitive* primitive;
};
