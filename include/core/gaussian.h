// core/gaussian.h -- Gaussian ellipsoid primitives of quarry's API (src/core/gaussian.h:12-20,
// 133-154 of the reference).  Query semantics: the solid ellipsoid (distance 0 inside).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "core/geometry.h"

struct Quat {
    float x = 0.0f, y = 0.0f, z = 0.0f, w = 1.0f;
};

struct Gaussian {
    Vec3 mean;
    Quat rot;    // normalized when used
    Vec3 scale;  // semi-axes, > 0
};

struct GaussianCloud {
    std::vector<Gaussian> gaussians;
    AABB bounds;
    void updateBounds();  // union of the padded ellipsoid boxes (engine arithmetic)
};

struct GaussianCloudSpec {
    std::string kind = "sheet";  // sheet | volume
    int count = 131072;
    uint64_t seed = 1;
    float scaleMin = 0.08f;
    float scaleMax = 0.50f;
    float aspectMin = 0.40f;
};

GaussianCloud buildGaussianCloud(const GaussianCloudSpec& spec);
