// Global box, local subdomain, process grid and halo settings of the
// dsDecompX drop-in (same declarations as the reference's include/domain.hpp).
#pragma once

#include <array>

namespace dsdecompx {

using Vec3d = std::array<double, 3>;
using Vec3i = std::array<int, 3>;

struct GlobalDomain {
    Vec3d lower{0.0, 0.0, 0.0};
    Vec3d upper{1.0, 1.0, 1.0};
    std::array<bool, 3> periodic{true, true, true};
};

struct LocalDomain {
    Vec3d lower{0.0, 0.0, 0.0};
    Vec3d upper{1.0, 1.0, 1.0};
};

struct ProcessGrid {
    // zero entries are filled by the planner
    Vec3i dimensions{0, 0, 0};
    bool allow_rank_reorder = false;
};

struct HaloConfig {
    double width = 0.0;
    bool include_edges_and_corners = true;
};

}  // namespace dsdecompx
