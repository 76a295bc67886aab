// core/scene.h -- triangle scenes and demo inputs of quarry's API (src/core/scene.h:9-45).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "core/geometry.h"

struct Scene {
    std::vector<Tri> tris;
    AABB bounds;
    void updateBounds() {
        bounds = AABB{};
        for (const Tri& t : tris) bounds.extend(t.bounds());
    }
};

struct SceneSpec {
    std::string kind = "terrain";  // terrain | random | mixed | city
    int grid = 256;
    int randomTris = 0;
    uint64_t seed = 1;
    int buildings = 65536;
};

Scene buildScene(const SceneSpec& spec);

enum class RayMode { Down, Random };

std::vector<Ray> makeRays(const AABB& bounds, RayMode mode, int count, uint64_t seed);
const char* rayModeName(RayMode mode);
float terrainHeight(float x, float z);
std::vector<Vec3> makeQueryPoints(const AABB& bounds, int count, uint64_t seed);
