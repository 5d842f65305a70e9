// Host schedule of sequential Gaussian simulation.
//
// Path (path_random_generator.cpp:20-66): a linear congruential walk x ->
// (A x + C) mod size from x0 = seed mod size, A = 1 + the product of the
// distinct primes dividing size (twice that when 4 divides size), C = the
// largest prime <= size / 3 that does not divide size -- full period, so
// every node once.  The reference reads its primes from primes.txt, which its
// checkout lacks; init_rnd's asserts leave one reading of that table (every
// prime in increasing order past the grid size), restated here with a sieve.
//
// Draws (bs_random_generator.cpp, sample.h:14-17): boost::mt11213b seeded
// with the seed, one 32-bit output per simulated node divided by 2^32 - 1,
// turned into the standard normal quantile of Odeh and Evans's rational
// approximation (gaussian_distribution.h:49-66) with the C library's log and
// sqrt -- the GPU multiplies it by the kriging standard deviation and adds the
// kriged mean, as gaussian_cdf_t::inverse does.
//
// Batches: the nodes of one batch are outside each other's search boxes, so
// none can be a neighbour of another and simulating them at once gives the
// sequential result.  A grid of cells of the box's size holds the current
// batch's nodes; a node is checked against the 27 cells around its own.
#include "sgs_host.h"

#include <cmath>
#include <stdexcept>

namespace hpgl_b200 {

namespace {

struct Path {
    long long A = 1, C = 2, M = 1, R = 0;
    Path(long long size, long long seed) {
        M = size;
        const long long lim = (size > 3 ? size : 3) + 1;
        std::vector<char> comp((size_t)lim + 1, 0);
        std::vector<long long> primes;
        for (long long i = 2; i <= lim; ++i) {
            if (comp[(size_t)i]) continue;
            primes.push_back(i);
            for (long long j = i * i; j <= lim; j += i) comp[(size_t)j] = 1;
        }
        for (long long p : primes) {
            if (p > size) break;
            if (size % p == 0) A *= p;
        }
        if (M % 4 == 0) A *= 2;
        A += 1;
        size_t idx = 0;
        while (idx + 1 < primes.size() && primes[idx + 1] <= size / 3) ++idx;
        for (long long k = (long long)idx; k >= 0; k--) {
            C = primes[(size_t)k];
            if (std::floor(double(size) / double(C)) != (double(size) / double(C))) break;
        }
        R = seed % size;
    }
    long long next() {
        const long long r = R;
        R = (A * R + C) % M;
        return r;
    }
};

// The Mersenne Twister (Matsumoto and Nishimura, ACM TOMACS 8(1), 1998) with
// boost's mt11213b parameters: w 32, n 351, m 175, r 19, a 0xccab8ee7,
// tempering (11, 7, 0x31b6ab00, 15, 0xffe50000, 17), seeding with 1812433253.
struct Mt11213b {
    enum { N = 351, M = 175, R = 19 };
    uint32_t x[N];
    int i = N;
    explicit Mt11213b(uint32_t s) {
        x[0] = s;
        for (int k = 1; k < N; ++k) x[k] = 1812433253u * (x[k - 1] ^ (x[k - 1] >> 30)) + (uint32_t)k;
    }
    uint32_t next() {
        if (i >= N) {
            const uint32_t upper = ~((1u << R) - 1u), lower = (1u << R) - 1u;
            for (int k = 0; k < N; ++k) {
                const uint32_t y = (x[k] & upper) | (x[(k + 1) % N] & lower);
                x[k] = x[(k + M) % N] ^ (y >> 1) ^ ((y & 1u) ? 0xccab8ee7u : 0u);
            }
            i = 0;
        }
        uint32_t y = x[i++];
        y ^= y >> 11;
        y ^= (y << 7) & 0x31b6ab00u;
        y ^= (y << 15) & 0xffe50000u;
        y ^= y >> 17;
        return y;
    }
};

double quantile(double p) {
    const double ps[] = {-0.322232431088, -1.0, -0.342242088547, -0.0204231210245, -0.453642210148e-4};
    const double qs[] = {0.0993484626060, 0.588581570495, 0.531103462366, 0.103537752850, 0.38560700634e-2};
    const double p2 = (p > 0.5) ? (1 - p) : p;
    const double y = std::sqrt(std::log(1 / (p2 * p2)));
    double xp = y + ((((ps[4] * y + ps[3]) * y + ps[2]) * y + ps[1]) * y + ps[0]) /
                        ((((qs[4] * y + qs[3]) * y + qs[2]) * y + qs[1]) * y + qs[0]);
    if (p < 0.5) xp = -xp;
    return xp;
}

}  // namespace

void sgs_schedule(int nx, int ny, int nz, const uint8_t *mask, const uint8_t *sim_mask, long long seed,
                  const int radii[3], long long max_batch, SgsSchedule &out) {
    const long long size = (long long)nx * ny * nz;
    out.nodes.clear();
    out.xp.clear();
    out.batches.clear();
    if (size <= 0) return;
    if (size > 10000000LL)
        throw std::domain_error("the simulation path is defined for grids of at most 10^7 nodes");
    Path path(size, seed);
    long long node = path.next();
    for (long long counter = 0; counter < size; ++counter, node = path.next()) {
        if (mask[node]) continue;
        if (sim_mask && sim_mask[node] != 1) continue;
        out.nodes.push_back((int)node);
    }
    Mt11213b gen((uint32_t)seed);
    out.xp.resize(out.nodes.size());
    for (size_t k = 0; k < out.nodes.size(); ++k) out.xp[k] = quantile(double(gen.next()) / double(0xffffffffu));
    // batches
    const int bx = radii[0] + 1, by = radii[1] + 1, bz = radii[2] + 1;
    const int cx = nx / bx + 1, cy = ny / by + 1, cz = nz / bz + 1;
    std::vector<long long> stamp((size_t)cx * cy * cz, -1);
    std::vector<std::vector<int>> cell((size_t)cx * cy * cz);
    long long batch = 0, in_batch = 0;
    out.batches.push_back(0);
    for (size_t k = 0; k < out.nodes.size(); ++k) {
        const int nd = out.nodes[k];
        const int x = nd % nx, y = nd / nx % ny, z = nd / nx / ny;
        const int gx = x / bx, gy = y / by, gz = z / bz;
        bool conflict = in_batch >= max_batch;
        for (int dz = -1; dz <= 1 && !conflict; ++dz)
            for (int dy = -1; dy <= 1 && !conflict; ++dy)
                for (int dx = -1; dx <= 1 && !conflict; ++dx) {
                    const int ax = gx + dx, ay = gy + dy, az = gz + dz;
                    if (ax < 0 || ay < 0 || az < 0 || ax >= cx || ay >= cy || az >= cz) continue;
                    const size_t c = ((size_t)az * cy + ay) * cx + ax;
                    if (stamp[c] != batch) continue;
                    for (int o : cell[c]) {
                        const int ox = o % nx, oy = o / nx % ny, oz = o / nx / ny;
                        if (std::abs(ox - x) <= radii[0] && std::abs(oy - y) <= radii[1] &&
                            std::abs(oz - z) <= radii[2]) {
                            conflict = true;
                            break;
                        }
                    }
                }
        if (conflict) {
            ++batch;
            in_batch = 0;
            out.batches.push_back((long long)k);
        }
        const size_t c = ((size_t)gz * cy + gy) * cx + gx;
        if (stamp[c] != batch) {
            stamp[c] = batch;
            cell[c].clear();
        }
        cell[c].push_back(nd);
        ++in_batch;
    }
    out.batches.push_back((long long)out.nodes.size());
}

}  // namespace hpgl_b200
