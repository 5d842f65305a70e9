// Test driver: the host side of sequential simulation (the random path, the
// draws and their quantiles, the CDF transforms of hpgl_b200/csrc/sgs_host.cpp)
// built for the host, so that tests/test_sim_host.py compares it with the
// restatement without a GPU.
#include <cstdint>
#include <cstring>
#include <stdexcept>

#include "../../hpgl_b200/csrc/sgs_host.h"

using namespace hpgl_b200;

extern "C" {

// Fills nodes / u (capacity n) and returns the count, or -1 (domain) / -2
// (invalid seed).
long long shc_path(int nx, int ny, int nz, const uint8_t *mask, const uint8_t *sim_mask, long long seed,
                   int quantiles, int *nodes, double *u) {
    SimPath p;
    try {
        sim_path(nx, ny, nz, mask, sim_mask, seed, quantiles != 0, p);
    } catch (const std::domain_error &) {
        return -1;
    } catch (const std::invalid_argument &) {
        return -2;
    }
    memcpy(nodes, p.nodes.data(), p.nodes.size() * sizeof(int));
    memcpy(u, p.u.data(), p.u.size() * sizeof(double));
    return (long long)p.nodes.size();
}

// direction 0: values through the CDF to the standard normal (mask optional);
// 1: back (mask required).
void shc_cdf(const float *cv, const float *cp, long long cs, float *values, const uint8_t *mask, long long n,
             int direction, int threads) {
    const NonParametricCdf c{cv, cp, cs};
    if (direction == 0) cdf_to_gaussian(c, values, values, mask, n, threads);
    else gaussian_to_cdf(c, values, mask, n, threads);
}
}
