// core/point_cloud.h -- point clouds of quarry's API (src/core/point_cloud.h:9-29).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "core/geometry.h"

struct PointCloud {
    std::vector<Vec3> pts;
    AABB bounds;
    void updateBounds() {
        bounds = AABB{};
        for (const Vec3& p : pts) bounds.extend(p);
    }
};

struct PointCloudSpec {
    std::string kind = "sheet";  // sheet | volume
    int count = 131072;
    uint64_t seed = 1;
};

PointCloud buildPointCloud(const PointCloudSpec& spec);
