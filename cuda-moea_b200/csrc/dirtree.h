// Cone tree over a set of reference directions (host side), used by the
// pruned exact association search.  Built by build_direction_tree
// (directions.cpp) and uploaded into a Workspace by prepare_direction_tree.
#pragma once

#include <vector>

namespace moea {

struct DirectionTreeHost {
    int M = 0, H = 0, nodes = 0, max_depth = 0;
    float delta = 0.0f;           // max | |r|^2 - 1 |
    std::vector<int> order;       // tree position -> direction index
    std::vector<float> dirs;      // (M, H) directions in tree order
    std::vector<float> center;    // (M, nodes) unit cone axes
    std::vector<float> cos_r;     // (nodes) cos of the cone half angle (rounded down)
    std::vector<float> sin_r;     // (nodes) sin of the cone half angle (rounded up)
    std::vector<int> link;        // (nodes, 2) {first child, count} or leaf {first position, -count}
};

int build_direction_tree(const float* refs, int M, int H, DirectionTreeHost& t);

}  // namespace moea
