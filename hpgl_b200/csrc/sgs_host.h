// Host schedule of sequential Gaussian simulation (sgs_host.cpp): the
// reference's random path over the grid, its random draws, and the batches
// of path-consecutive nodes that the GPU can simulate at once.
#pragma once
#include <cstdint>
#include <vector>

namespace hpgl_b200 {

struct SgsSchedule {
    std::vector<int> nodes;         // simulated nodes in path order
    std::vector<double> xp;         // standard normal quantile of each node's draw
    std::vector<long long> batches; // batch b = nodes[batches[b], batches[b+1])
};

// nodes: the path's uninformed nodes inside `sim_mask` (all when null);
// batches: maximal runs in which no node lies inside another's search box
// (|dx| <= rx, |dy| <= ry, |dz| <= rz), so that each node sees exactly the
// nodes simulated before it on the path, at most `max_batch` nodes.
void sgs_schedule(int nx, int ny, int nz, const uint8_t *mask, const uint8_t *sim_mask, long long seed,
                  const int radii[3], long long max_batch, SgsSchedule &out);

}  // namespace hpgl_b200
