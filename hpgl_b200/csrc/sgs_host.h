// Host side of sequential simulation (sgs_host.cpp): the reference's random
// path over the grid, its random draws, and the normal-score transforms of
// sequential Gaussian simulation.
#pragma once
#include <cstdint>
#include <vector>

namespace hpgl_b200 {

struct SimPath {
    std::vector<int> nodes;  // simulated nodes in path order
    std::vector<double> u;   // per simulated node: its draw in [0, 1], or the draw's quantile
};

// The path's uninformed nodes inside `sim_mask` (all when null: a node is
// simulated when sim_mask[node] == 1) in path order, with the generator's
// draws in the same order -- or, with `quantiles`, their standard normal
// quantiles (gaussian_cdf_t::inverse).  Throws std::domain_error above 10^7 nodes and
// std::invalid_argument when the seed, as the int the path takes, is
// negative.
void sim_path(int nx, int ny, int nz, const uint8_t *mask, const uint8_t *sim_mask, long long seed, bool quantiles,
              SimPath &out);

// The checks sim_path makes before any work (same exceptions).
void check_sim_path(long long size, long long seed);

// A caller's non-parametric CDF (hpgl_non_parametric_cdf_t): `size` values in
// increasing order and their cumulative probabilities.
struct NonParametricCdf {
    const float *values;
    const float *probs;
    long long size;
};

// Normal-score transform (cdf_utils.h:12-25 with non_parametric_cdf_2_t as
// the source and the standard normal as the target): out[i] =
// N^-1(F(in[i])) for the nodes with mask[i] != 0 (every node when mask is
// null); out may be in.
void cdf_to_gaussian(const NonParametricCdf &cdf, const float *in, float *out, const uint8_t *mask, long long n,
                     int threads);
// The back transform: values[i] = F^-1(N(values[i])) where mask[i] != 0.
void gaussian_to_cdf(const NonParametricCdf &cdf, float *values, const uint8_t *mask, long long n, int threads);

}  // namespace hpgl_b200
