// Host planning of a kriging job.  Compiled with -O2 -ffp-contract=off so
// that every covariance value is the one the reference computes (same
// expression order, glibc libm, no fused multiply-adds).  Paths cited are
// relative to the reference's src/geo_bsd/hpgl/.
#include "plan.h"

#include <algorithm>
#include <cstring>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <stdexcept>
#include <mutex>
#include <thread>

#include "introsort.h"
#include "task_pool.h"

namespace hpgl_b200 {



static std::atomic<int> g_threads{0};

int host_threads() {
    int n = g_threads.load();
    if (n > 0) return n;
    unsigned hc = std::thread::hardware_concurrency();
    return hc ? (int)hc : 1;
}

void set_host_threads(int n) { g_threads.store(n > 0 ? n : 0); }

// f(lo, hi) over [0, n) split across up to `threads` threads of the pool, at
// least `grain` items per thread.
template <typename F>
static void parallel_for(long long n, int threads, F f, long long grain = 4096) {
    pool_for(n, threads, f, grain);
}

// C(v) over the box |v_i| <= r_i into out[((z+rz)*(2ry+1) + y+ry)*(2rx+1) + x+rx],
// evaluated as f(x, y, z).  C(v) == C(-v) bit for bit (every transformed
// component only changes sign), so the half with z > 0 or (z == 0, y > 0) or
// (z == y == 0, x >= 0) is evaluated and mirrored.
template <typename F>
static void fill_symmetric(std::vector<double> &out, int rx, int ry, int rz, int threads, F f) {
    const int xd = 2 * rx + 1, yd = 2 * ry + 1;
    out.assign((size_t)xd * yd * (2 * rz + 1), 0.0);
    auto idx = [&](int x, int y, int z) { return ((size_t)(z + rz) * yd + (y + ry)) * xd + (x + rx); };
    // rows (z, y) of the evaluated half, z = 0..rz (y >= 0 at z = 0), a few
    // thousand covariances per thread at least
    const long long rows = (long long)(rz + 1) * yd;
    parallel_for(
        rows, threads,
        [&](long long lo, long long hi) {
            for (long long r = lo; r < hi; ++r) {
                const int z = (int)(r / yd), y = (int)(r % yd) - ry;
                if (z == 0 && y < 0) continue;
                for (int x = (z == 0 && y == 0 ? 0 : -rx); x <= rx; ++x) {
                    const double v = f(x, y, z);
                    out[idx(x, y, z)] = v;
                    out[idx(-x, -y, -z)] = v;
                }
            }
        },
        std::max<long long>(1, 4096 / xd));
}

// Sub-ranges above this many entries may go to another thread.
constexpr int SORT_SPAWN_MIN = 4096;

// The reference's std::sort permutation (introsort.h) with the independent
// right-hand sub-ranges of large partitions sorted as pool tasks: each
// sub-range's processing touches only its own elements, so the result is
// the sequential algorithm's, element for element, whatever runs where.
static void sort_subrange(SortArr a, int lo, int hi, int depth, TaskGroup &g) {
    while (hi - lo > 16) {
        if (depth == 0) {
            sort_heapsort(a, lo, hi);
            return;
        }
        --depth;
        const int mid = lo + (hi - lo) / 2;
        sort_median_to_first(a, lo, lo + 1, mid, hi - 1);
        const int cut = sort_partition(a, lo + 1, hi, lo);
        if (hi - cut > SORT_SPAWN_MIN)
            task_submit(g, [a, cut, hi, depth, &g] { sort_subrange(a, cut, hi, depth, g); });
        else
            sort_subrange(a, cut, hi, depth, g);
        hi = cut;
    }
}

static void parallel_reference_sort(std::vector<double> &key, std::vector<int> &idx, int threads) {
    const int n = (int)key.size();
    if (n <= 1) return;
    SortArr a{key.data(), idx.data()};
    if (threads > 1) task_pool_reserve(threads - 1);
    TaskGroup g;
    std::exception_ptr own;
    try {
        sort_subrange(a, 0, n, 2 * sort_floor_log2(n), g);
    } catch (...) {
        own = std::current_exception();
    }
    task_wait(g);
    if (own) std::rethrow_exception(own);
    if (n > 16) {
        sort_insertion(a, 0, 16);
        for (int i = 16; i < n; ++i) sort_linear_insert(a, i);
    } else {
        sort_insertion(a, 0, n);
    }
}

// 3x3 product summed left to right, as TNT's matmult (tnt_cmat.h:472-498).
static void mat3(const double *a, const double *b, double *c) {
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) {
            double s = 0;
            for (int j = 0; j < 3; ++j) s = s + a[3 * i + j] * b[3 * j + k];
            c[3 * i + k] = s;
        }
}

CovModel::CovModel(const KrigingParams &p) {
    type = p.cov_type;
    sill = p.sill;
    nugget = p.nugget;
    range0 = p.ranges[0];
    // create_transform (cov_model.h:16-61); grad_to_rad is (grad*pi)/180.
    const double pi = 3.14159265358979323846264338327950288419;
    const double a0 = (p.angles[0] * pi) / 180, a1 = (p.angles[1] * pi) / 180, a2 = (p.angles[2] * pi) / 180;
    const double s[9] = {1.0, 0, 0, 0, p.ranges[0] / p.ranges[1], 0, 0, 0, p.ranges[0] / p.ranges[2]};
    const double rz[9] = {cos(a0), sin(a0), 0, -sin(a0), cos(a0), 0, 0, 0, 1};
    const double ry[9] = {cos(a1), 0, -sin(a1), 0, 1, 0, sin(a1), 0, cos(a1)};
    const double rx[9] = {1, 0, 0, 0, cos(a2), sin(a2), 0, -sin(a2), cos(a2)};
    double xy[9], xyz[9];
    mat3(rx, ry, xy);
    mat3(xy, rz, xyz);
    mat3(s, xyz, t);
}

double CovModel::operator()(double vx, double vy, double vz) const {
    const double v[3] = {vx, vy, vz};
    double acc = 0.0;
    for (int i = 0; i < 3; ++i) {
        double d = 0.0;
        for (int j = 0; j < 3; ++j) d += v[j] * t[3 * i + j];
        acc += d * d;
    }
    const double h = sqrt(acc);
    if (h < 0.0001) return sill - nugget;
    switch (type) {
    case 2: return (sill - nugget) * exp(-3 * pow(h / range0, 2));
    case 1: return (sill - nugget) * exp(-3 * h / range0);
    default:
        if (h > range0) return 0;
        return (sill - nugget) * (1 - 1.5 * h / range0 + 0.5 * pow(h / range0, 3));
    }
}

void validate_params(const KrigingParams &p, int kind) {
    if (p.cov_type < 0 || p.cov_type > 2) throw std::invalid_argument("covariance type must be 0, 1 or 2");
    for (int i = 0; i < 3; ++i) {
        // cov_model.h:24-25 raises on a zero range.
        if (p.ranges[i] == 0) throw std::invalid_argument("All covariance ranges should be non-zero");
        if (p.radii[i] <= 0) throw std::invalid_argument("search radiuses must be positive");
    }
    if (p.max_neighbours <= 0) throw std::invalid_argument("max_neighbours must be positive");
    if (p.max_neighbours > 64) throw std::domain_error("max_neighbours > 64 is not supported by this build");
    if (kind == KIND_IK && !(p.marginal_prob == p.marginal_prob))
        throw std::invalid_argument("marginal probability is NaN");
}

bool same_system(const KrigingParams &a, const KrigingParams &b) {
    if (a.cov_type != b.cov_type || a.sill != b.sill || a.nugget != b.nugget || a.max_neighbours != b.max_neighbours)
        return false;
    for (int i = 0; i < 3; ++i)
        if (a.ranges[i] != b.ranges[i] || a.angles[i] != b.angles[i] || a.radii[i] != b.radii[i]) return false;
    return true;
}

double informed_mean(const float *values, const uint8_t *mask, long long size) {
    int count = 0;
    double sum = 0;
    for (long long i = 0; i < size; ++i)
        if (mask[i]) {
            sum += values[i];
            count += 1;
        }
    return count == 0 ? 0 : sum / count;
}

// ---- clusterizer (clusterizer.cpp:52-184) ----
// Boxes of the radii (doubles in the reference: sugarbox_search_ellipsoid_t),
// mx = (int)(nx / rx + 2); a box overflows past limit = |template| / 250
// (sugarbox_indexed_neighbour_lookup.h:58) and then holds no nodes.  Fills
// P's clusterizer fields (P.size and P.clusterizer set).
static void build_buckets(Plan &P, int nx, int ny, int nz, const KrigingParams &p, const uint8_t *mask,
                          long long limit, int threads) {
    for (int i = 0; i < 3; ++i) P.cl_r[i] = (double)p.radii[i];
    P.mx = (int)(nx / P.cl_r[0] + 2);
    P.my = (int)(ny / P.cl_r[1] + 2);
    P.mz = (int)(nz / P.cl_r[2] + 2);
    P.limit = limit;
    const long long nb = (long long)P.mx * P.my * P.mz;
    std::vector<int> count(nb, 0);
    std::vector<uint8_t> exceeded(nb, 0);
    auto bucket_of = [&](long long idx) {
        int x = (int)(idx % nx), y = (int)(idx % ((long long)nx * ny) / nx), z = (int)(idx / ((long long)nx * ny));
        int cx = (int)(x / P.cl_r[0]), cy = (int)(y / P.cl_r[1]), cz = (int)(z / P.cl_r[2]);
        return ((long long)cz * P.my + cy) * P.mx + cx;
    };
    // The informed nodes in index order (stretches of the mask scanned on all
    // threads, eight bytes at a time).  A box takes nodes in that order until
    // it holds `limit`, and the next one makes it overflow: it overflows
    // exactly when it receives more than `limit` nodes.
    std::vector<int> informed;
    {
        const long long chunk = std::max<long long>(1 << 16, (P.size + threads - 1) / std::max(threads, 1));
        const long long parts = (P.size + chunk - 1) / chunk;
        std::vector<std::vector<int>> part((size_t)parts);
        parallel_for(parts, threads, [&](long long lo, long long hi) {
            for (long long c = lo; c < hi; ++c) {
                const long long a = c * chunk, e = std::min(P.size, a + chunk);
                std::vector<int> &v = part[(size_t)c];
                long long i = a;
                for (; i < e && (i & 7); ++i)
                    if (mask[i]) v.push_back((int)i);
                for (; i + 8 <= e; i += 8) {
                    uint64_t w;
                    memcpy(&w, mask + i, 8);
                    if (!w) continue;
                    for (int k = 0; k < 8; ++k)
                        if (mask[i + k]) v.push_back((int)(i + k));
                }
                for (; i < e; ++i)
                    if (mask[i]) v.push_back((int)i);
            }
        });
        size_t total = 0;
        for (auto &v : part) total += v.size();
        informed.reserve(total);
        for (auto &v : part) informed.insert(informed.end(), v.begin(), v.end());
    }
    P.informed = (long long)informed.size();
    std::vector<long long> box_of(informed.size());
    for (size_t k = 0; k < informed.size(); ++k) {
        box_of[k] = bucket_of(informed[k]);
        count[box_of[k]]++;
    }
    for (long long b = 0; b < nb; ++b)
        if (count[b] > P.limit) {
            exceeded[b] = 1;
            count[b] = 0;
        }
    P.bucket_start.assign(nb + 1, 0);
    for (long long b = 0; b < nb; ++b) P.bucket_start[b + 1] = P.bucket_start[b] + count[b];
    P.bucket_nodes.assign(P.bucket_start[nb], 0);
    {
        std::vector<int> fill(P.bucket_start.begin(), P.bucket_start.end() - 1);
        for (size_t k = 0; k < informed.size(); ++k) {
            const long long b = box_of[k];
            if (!exceeded[b]) P.bucket_nodes[fill[b]++] = informed[k];
        }
    }
    P.bucket_clean.assign(nb, 0);
    P.any_clean = false;
    P.max_candidates = 0;
    // Only boxes that hold grid nodes are ever asked (cx < nx/rx + 1 < mx).
    for (int cz = 0; cz < P.mz; ++cz)
        for (int cy = 0; cy < P.my; ++cy)
            for (int cx = 0; cx < P.mx; ++cx) {
                if ((double)cx * P.cl_r[0] >= nx || (double)cy * P.cl_r[1] >= ny || (double)cz * P.cl_r[2] >= nz)
                    continue;
                bool clean = true;
                int cand = 0;
                for (int k = cz - 1; k <= cz + 1; ++k)
                    for (int j = cy - 1; j <= cy + 1; ++j)
                        for (int i = cx - 1; i <= cx + 1; ++i) {
                            if (i < 0 || j < 0 || k < 0 || i > P.mx || j > P.my || k > P.mz) continue;
                            long long b = ((long long)k * P.my + j) * P.mx + i;
                            if (b >= nb) continue;  // the inclusive box edge is never reached by real nodes
                            if (exceeded[b]) clean = false;
                            cand += count[b];
                        }
                long long b = ((long long)cz * P.my + cy) * P.mx + cx;
                if (!P.clusterizer) clean = false;
                P.bucket_clean[b] = clean ? 1 : 0;
                if (clean) {
                    P.any_clean = true;
                    P.max_candidates = std::max(P.max_candidates, cand);
                }
            }

}

void build_plan(Plan &P, int kind, int nx, int ny, int nz, const KrigingParams &p, const uint8_t *mask,
                int threads, bool sequential) {
    static const bool timing = getenv("HPGL_B200_PLAN_TIMING") != nullptr;
    auto t_last = std::chrono::steady_clock::now();
    auto lap = [&](const char *what) {
        if (!timing) return;
        auto now = std::chrono::steady_clock::now();
        fprintf(stderr, "plan %-10s %8.2f ms\n", what, std::chrono::duration<double, std::milli>(now - t_last).count());
        t_last = now;
    };
    validate_params(p, kind);
    CovModel cov(p);
    P.kind = kind;
    P.nx = nx;
    P.ny = ny;
    P.nz = nz;
    P.size = (long long)nx * ny * nz;
    P.nmax = p.max_neighbours;
    // Ordinary kriging and cokriging use the model itself; cokriging searches
    // with neighbour_lookup_t alone (simple_cokriging_markI.cpp:201, no
    // clusterizer).
    P.truncated = (kind != KIND_OK && !kind_is_cokriging(kind)) || sequential;
    P.clusterizer = !kind_is_cokriging(kind) && !sequential;
    for (int i = 0; i < 3; ++i) P.radii[i] = p.radii[i];
    const int rx = p.radii[0], ry = p.radii[1], rz = p.radii[2];

    // ---- search template: calc_cov_field (covariance_field.h:62-106) ----
    // C(0 - v) over the +-radius box in z-y-x order, offsets above C(0)/100
    // kept as the vector -v, sorted descending by std::sort (the same
    // unstable algorithm on the same input order as the reference, hence the
    // same order of equal keys).  Every covariance object the reference can
    // pass here (the model, the precalculated table, covariance_field_t)
    // yields these same values inside the box.
    const int xd = 2 * rx + 1, yd = 2 * ry + 1;
    std::vector<double> data;
    fill_symmetric(data, rx, ry, rz, threads, [&](int x, int y, int z) { return cov(0.0 - x, 0.0 - y, 0.0 - z); });
    lap("box");
    const double c0 = cov(0.0, 0.0, 0.0);
    const double threshold = c0 / 100;
    // Offsets -v in z-y-x order of v, keyed by C(v) (= C(-v)); collected per
    // z-slab in parallel and concatenated in slab order.
    std::vector<double> keys;
    std::vector<int> order;
    // the template's extent: that of the offsets above the threshold,
    // per slab while they are collected
    P.ext[0] = P.ext[1] = P.ext[2] = 0;
    {
        const int zd = 2 * rz + 1;
        std::vector<std::vector<double>> kz(zd);
        std::vector<std::vector<int>> oz(zd);
        std::vector<int> ez((size_t)zd * 3, 0);
        parallel_for(
            zd, threads,
            [&](long long lo, long long hi) {
            for (long long zi = lo; zi < hi; ++zi) {
                const int z = (int)zi - rz;
                int ex = 0, ey = 0;
                for (int y = -ry; y <= ry; ++y)
                    for (int x = -rx; x <= rx; ++x) {
                        const double k = data[((size_t)(z + rz) * yd + (y + ry)) * xd + (x + rx)];
                        if (k > threshold) {
                            kz[zi].push_back(k);
                            oz[zi].push_back((int)((((size_t)(-z + rz) * yd) + (-y + ry)) * xd + (-x + rx)));
                            ex = std::max(ex, std::abs(x));
                            ey = std::max(ey, std::abs(y));
                        }
                    }
                ez[3 * zi] = ex;
                ez[3 * zi + 1] = ey;
                ez[3 * zi + 2] = kz[zi].empty() ? 0 : std::abs(z);
            }
            },
            std::max<long long>(1, 4096 / ((long long)xd * yd)));
        size_t total = 0;
        for (auto &v : kz) total += v.size();
        keys.reserve(total);
        order.reserve(total);
        for (int zi = 0; zi < zd; ++zi) {
            keys.insert(keys.end(), kz[zi].begin(), kz[zi].end());
            order.insert(order.end(), oz[zi].begin(), oz[zi].end());
            for (int a = 0; a < 3; ++a) P.ext[a] = std::max(P.ext[a], ez[3 * zi + a]);
        }
    }
    lap("keys");
    // Every collected key is above the threshold, so the template keeps all
    // of them and the clusterizer's limit (|template| / 250) is known before
    // the sort: the buckets are built as a pool task meanwhile.
    const int bucket_threads = std::max(1, threads / 4);
    TaskGroup bucket_task;
    task_pool_reserve(1);
    task_submit(bucket_task, [&] { build_buckets(P, nx, ny, nz, p, mask, (long long)(keys.size() / 250), bucket_threads); });
    try {
        parallel_reference_sort(keys, order, threads);
    } catch (...) {
        try {
            task_wait(bucket_task);
        } catch (...) {
        }
        throw;
    }
    lap("sort");
    size_t kept = keys.size();
    for (size_t i = 0; i < keys.size(); ++i)
        if (keys[i] < threshold) {
            kept = i;
            break;
        }
    P.tmpl.resize(kept);
    parallel_for((long long)kept, threads, [&](long long lo, long long hi) {
        for (long long i = lo; i < hi; ++i) {
            const int o = order[i];
            TemplateEntry &e = P.tmpl[i];
            e.dx = o % xd - rx;
            e.dy = o / xd % yd - ry;
            e.dz = o / xd / yd - rz;
            e.delta = e.dx + nx * (e.dy + ny * e.dz);
        }
    });
    if (kept < keys.size()) {
        // entries cut after the sort (not reachable with the > threshold
        // filter, kept for the reference's second cut-off) do not widen ext
        P.ext[0] = P.ext[1] = P.ext[2] = 0;
        for (const TemplateEntry &e : P.tmpl) {
            P.ext[0] = std::max(P.ext[0], std::abs(e.dx));
            P.ext[1] = std::max(P.ext[1], std::abs(e.dy));
            P.ext[2] = std::max(P.ext[2], std::abs(e.dz));
        }
    }

    lap("template");
    task_wait(bucket_task);
    if ((long long)(P.tmpl.size() / 250) != P.limit)
        build_buckets(P, nx, ny, nz, p, mask, (long long)(P.tmpl.size() / 250), threads);
    lap("buckets");
    // ---- covariance table ----
    // Truncated kinds read C(v) only for |v| <= radii.  Ordinary kriging uses
    // the untruncated model; the template path needs |v| <= 2*ext (pairs of
    // template offsets), the clusterizer path |v| <= 4r-2 (pairs of
    // candidates from the 3x3x3 boxes).  No offset exceeds the grid.
    const int n3[3] = {nx, ny, nz};
    for (int a = 0; a < 3; ++a) {
        int need;
        if (P.truncated) {
            need = p.radii[a];
        } else {
            need = 2 * P.ext[a];
            if (P.any_clean) need = std::max(need, 4 * p.radii[a] - 2);
        }
        P.B[a] = std::max(0, std::min(need, n3[a] - 1));
        P.trunc[a] = P.truncated ? p.radii[a] : P.B[a];
    }
    if (P.B[0] == rx && P.B[1] == ry && P.B[2] == rz) {
        // the template's box already holds C(-v) at v, which is C(v) bit for
        // bit (the transform of -v is the negated transform of v, and only
        // its squares enter the distance)
        P.table.swap(data);
    } else {
        fill_symmetric(P.table, P.B[0], P.B[1], P.B[2], threads,
                       [&](int x, int y, int z) { return cov((double)x, (double)y, (double)z); });
    }
    P.c0 = c0;
    lap("table");

    // ---- informed-bit rows for the device template search ----
    P.px = 32 * ((P.ext[0] + 31) / 32);
    P.nseg = (nx + 31) / 32;
    P.wpr = P.nseg + 2 * (P.px / 32) + 2;

}


void fill_cov_table(std::vector<double> &table, const int B[3], const KrigingParams &p, int threads) {
    CovModel cov(p);
    fill_symmetric(table, B[0], B[1], B[2], threads,
                   [&](int x, int y, int z) { return cov((double)x, (double)y, (double)z); });
}

}  // namespace hpgl_b200
