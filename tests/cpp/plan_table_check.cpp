// Test driver: the covariance table of a plan (hpgl_b200/csrc/plan.cpp) --
// taken from the search template's box when the two coincide -- against the
// table evaluated from the model on its own box, bit for bit, over seeded
// grids, variograms and search radii.  Returns the number of mismatches.
#include <cstdio>
#include <cstring>
#include <random>

#include "../../hpgl_b200/csrc/plan.h"
#include "../../hpgl_b200/csrc/introsort.h"

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

// The plan's search template (sorted on the planning threads, sub-ranges as
// pool tasks) against the template rebuilt here on one thread: C(0 - v) over
// the radius box in z-y-x order, kept above C(0)/100 as the offset -v, ordered
// by the sequential reference sort.  Radii large enough that the sort hands
// sub-ranges to other threads.  Returns the number of differing templates.
extern "C" int ptc_template(unsigned seed, int cases, int threads) {
    std::mt19937 g(seed);
    int bad = 0, large = 0;
    for (int t = 0; t < cases; ++t) {
        const int nx = 40 + g() % 60, ny = 40 + g() % 60, nz = 10 + g() % 20;
        std::vector<uint8_t> m((size_t)nx * ny * nz);
        for (auto &x : m) x = (g() % 50) == 0;
        KrigingParams p{};
        p.cov_type = g() % 3;
        p.ranges[0] = 10 + g() % 30;
        p.ranges[1] = 10 + g() % 30;
        p.ranges[2] = 4 + g() % 10;
        p.angles[0] = (g() % 4) * 30;  // ties between mirrored offsets at some angles
        p.sill = 1;
        p.nugget = (g() % 2) * 0.05;
        p.radii[0] = 15 + g() % 30;
        p.radii[1] = 15 + g() % 30;
        p.radii[2] = 4 + g() % 10;
        p.max_neighbours = 16;
        Plan P;
        build_plan(P, KIND_SK, nx, ny, nz, p, m.data(), threads, false);
        CovModel cov(p);
        const double thr = cov(0.0, 0.0, 0.0) / 100;
        std::vector<double> key;
        std::vector<int> off;
        const int rx = p.radii[0], ry = p.radii[1], rz = p.radii[2];
        for (int z = -rz; z <= rz; ++z)
            for (int y = -ry; y <= ry; ++y)
                for (int x = -rx; x <= rx; ++x) {
                    const double k = cov(0.0 - x, 0.0 - y, 0.0 - z);
                    if (k > thr) {
                        key.push_back(k);
                        off.push_back((int)key.size() - 1);
                    }
                }
        // offsets in collection order, indexed by `off`
        std::vector<int> ox, oy, oz;
        for (int z = -rz; z <= rz; ++z)
            for (int y = -ry; y <= ry; ++y)
                for (int x = -rx; x <= rx; ++x)
                    if (cov(0.0 - x, 0.0 - y, 0.0 - z) > thr) {
                        ox.push_back(-x);
                        oy.push_back(-y);
                        oz.push_back(-z);
                    }
        SortArr a{key.data(), off.data()};
        reference_sort(a, (int)key.size());
        bool same = P.tmpl.size() == key.size();
        for (size_t i = 0; same && i < key.size(); ++i) {
            const int o = off[i];
            same = P.tmpl[i].dx == ox[o] && P.tmpl[i].dy == oy[o] && P.tmpl[i].dz == oz[o];
        }
        if (!same) ++bad;
        if (key.size() >= 8192) ++large;
    }
    return large > 0 ? bad : -1;  // -1: no template large enough to exercise the tasks
}
