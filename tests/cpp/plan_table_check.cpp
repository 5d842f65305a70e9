// Test driver: the covariance table of a plan (hpgl_b200/csrc/plan.cpp) --
// taken from the search template's box when the two coincide -- against the
// table evaluated from the model on its own box, bit for bit, over seeded
// grids, variograms and search radii.  Returns the number of mismatches.
#include <cstdio>
#include <cstring>
#include <random>

#include "../../hpgl_b200/csrc/plan.h"

using namespace hpgl_b200;

extern "C" int ptc_run(unsigned seed, int cases) {
    std::mt19937 g(seed);
    int bad = 0;
    for (int t = 0; t < cases; ++t) {
        const int nx = 20 + g() % 100, ny = 20 + g() % 100, nz = 5 + g() % 40;
        std::vector<uint8_t> m((size_t)nx * ny * nz);
        for (auto &x : m) x = (g() % 50) == 0;
        KrigingParams p{};
        p.cov_type = g() % 3;
        p.ranges[0] = 3 + g() % 30;
        p.ranges[1] = 3 + g() % 30;
        p.ranges[2] = 2 + g() % 10;
        p.angles[0] = g() % 360;
        p.angles[1] = (int)(g() % 90) - 45;
        p.angles[2] = (int)(g() % 60) - 30;
        p.sill = 1 + (g() % 5) * 0.25;
        p.nugget = (g() % 3) * 0.05;
        p.radii[0] = 2 + g() % 40;
        p.radii[1] = 2 + g() % 40;
        p.radii[2] = 1 + g() % 15;
        p.max_neighbours = 8 + g() % 24;
        for (int kind : {KIND_SK, KIND_OK}) {
            Plan P;
            build_plan(P, kind, nx, ny, nz, p, m.data(), 4, false);
            std::vector<double> ref;
            fill_cov_table(ref, P.B, p, 4);
            if (ref.size() != P.table.size() || memcmp(ref.data(), P.table.data(), ref.size() * 8)) ++bad;
        }
    }
    return bad;
}
