// Test driver: the clusterizer's candidate box (Plan::cand_box, plan.cpp)
// against the model itself.  For seeded variograms of every type (ranges,
// anisotropy, rotations, sills and nuggets), every integer offset within a
// margin around the box whose covariance exceeds C(0)/100 -- the clusterizer's
// keep test -- must lie inside the box, and the box must not exceed the
// offsets that pass by more than two cells per axis.  Returns the number of
// failures.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "../../hpgl_b200/csrc/plan.h"

using namespace hpgl_b200;

extern "C" int cbc_run(unsigned seed, int cases) {
    std::mt19937 g(seed);
    int bad = 0;
    for (int t = 0; t < cases; ++t) {
        KrigingParams p{};
        p.cov_type = t % 3;
        p.ranges[0] = 2 + g() % 20 + (g() % 100) * 0.01;
        p.ranges[1] = 2 + g() % 20 + (g() % 100) * 0.01;
        p.ranges[2] = 1 + g() % 8 + (g() % 100) * 0.01;
        p.angles[0] = g() % 360;
        p.angles[1] = (int)(g() % 90) - 45;
        p.angles[2] = (int)(g() % 60) - 30;
        p.sill = 1 + (g() % 5) * 0.25;
        p.nugget = (g() % 3) * 0.05;
        p.radii[0] = p.radii[1] = p.radii[2] = 4;
        p.max_neighbours = 8;
        const int nx = 12, ny = 12, nz = 6;
        std::vector<uint8_t> m((size_t)nx * ny * nz, 0);
        m[0] = 1;
        Plan P;
        build_plan(P, KIND_OK, nx, ny, nz, p, m.data(), 2);
        CovModel cov(p);
        const double thr = cov(0, 0, 0) / 100;
        int ext[3] = {0, 0, 0};
        const int *b = P.cand_box;
        if (b[0] > 200 || b[1] > 200 || b[2] > 200) {
            ++bad;
            continue;
        }
        for (int z = -b[2] - 3; z <= b[2] + 3; ++z)
            for (int y = -b[1] - 3; y <= b[1] + 3; ++y)
                for (int x = -b[0] - 3; x <= b[0] + 3; ++x)
                    if (cov(x, y, z) > thr) {
                        if (std::abs(x) > b[0] || std::abs(y) > b[1] || std::abs(z) > b[2]) {
                            if (bad < 5) fprintf(stderr, "case %d: offset (%d,%d,%d) passes outside box\n", t, x, y, z);
                            ++bad;
                        }
                        ext[0] = std::max(ext[0], std::abs(x));
                        ext[1] = std::max(ext[1], std::abs(y));
                        ext[2] = std::max(ext[2], std::abs(z));
                    }
        for (int a = 0; a < 3; ++a)
            if (b[a] > ext[a] + 2) {
                if (bad < 5) fprintf(stderr, "case %d: box %d wider than needed (%d)\n", t, b[a], ext[a]);
                ++bad;
            }
    }
    return bad;
}
