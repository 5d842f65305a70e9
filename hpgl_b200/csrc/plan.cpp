// Host planning of a kriging job.  Compiled with -O2 -ffp-contract=off so
// that every covariance value is the one the reference computes (same
// expression order, glibc libm, no fused multiply-adds).  Paths cited are
// relative to the reference's src/geo_bsd/hpgl/.
#include "plan.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <stdexcept>
#include <thread>

namespace hpgl_b200 {

static std::atomic<int> g_threads{0};

int host_threads() {
    int n = g_threads.load();
    if (n > 0) return n;
    unsigned hc = std::thread::hardware_concurrency();
    return hc ? (int)hc : 1;
}

void set_host_threads(int n) { g_threads.store(n > 0 ? n : 0); }

template <typename F>
static void parallel_for(long long n, int threads, F f) {
    threads = (int)std::max<long long>(1, std::min<long long>(threads, n / 4096 + 1));
    if (threads == 1) {
        f(0LL, n);
        return;
    }
    std::vector<std::thread> pool;
    long long chunk = (n + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        long long lo = t * chunk, hi = std::min(n, lo + chunk);
        if (lo >= hi) break;
        pool.emplace_back([=] { f(lo, hi); });
    }
    for (auto &th : pool) th.join();
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

void build_plan(Plan &P, int kind, int nx, int ny, int nz, const KrigingParams &p, const uint8_t *mask,
                int threads) {
    validate_params(p, kind);
    CovModel cov(p);
    P.kind = kind;
    P.nx = nx;
    P.ny = ny;
    P.nz = nz;
    P.size = (long long)nx * ny * nz;
    P.nmax = p.max_neighbours;
    P.truncated = kind != KIND_OK;
    for (int i = 0; i < 3; ++i) P.radii[i] = p.radii[i];
    const int rx = p.radii[0], ry = p.radii[1], rz = p.radii[2];

    // ---- search template: calc_cov_field (covariance_field.h:62-106) ----
    // C(0 - v) over the +-radius box in z-y-x order, offsets above C(0)/100
    // kept as the vector -v, sorted descending by std::sort (the same
    // unstable algorithm on the same input order as the reference, hence the
    // same order of equal keys).  Every covariance object the reference can
    // pass here (the model, the precalculated table, covariance_field_t)
    // yields these same values inside the box.
    const int xd = 2 * rx + 1, yd = 2 * ry + 1, zd = 2 * rz + 1;
    std::vector<double> data((size_t)xd * yd * zd);
    parallel_for(zd, threads, [&](long long lo, long long hi) {
        for (long long zi = lo; zi < hi; ++zi)
            for (int yi = 0; yi < yd; ++yi)
                for (int xi = 0; xi < xd; ++xi) {
                    int x = xi - rx, y = yi - ry, z = (int)zi - rz;
                    data[((size_t)zi * yd + yi) * xd + xi] = cov(0.0 - x, 0.0 - y, 0.0 - z);
                }
    });
    const double c0 = cov(0.0, 0.0, 0.0);
    const double threshold = c0 / 100;
    struct V3 { int c[3]; };
    std::vector<V3> vecs;
    for (int z = -rz; z <= rz; ++z)
        for (int y = -ry; y <= ry; ++y)
            for (int x = -rx; x <= rx; ++x)
                if (data[((size_t)(z + rz) * yd + (y + ry)) * xd + (x + rx)] > threshold) vecs.push_back(V3{{-x, -y, -z}});
    auto key = [&](const V3 &v) { return data[((size_t)(v.c[2] + rz) * yd + (v.c[1] + ry)) * xd + (v.c[0] + rx)]; };
    std::sort(vecs.begin(), vecs.end(), [&](const V3 &a, const V3 &b) { return key(a) > key(b); });
    for (size_t i = 0; i < vecs.size(); ++i)
        if (key(vecs[i]) < threshold) {
            vecs.resize(i);
            break;
        }
    P.tmpl.resize(vecs.size());
    P.ext[0] = P.ext[1] = P.ext[2] = 0;
    for (size_t i = 0; i < vecs.size(); ++i) {
        TemplateEntry &e = P.tmpl[i];
        e.dx = vecs[i].c[0];
        e.dy = vecs[i].c[1];
        e.dz = vecs[i].c[2];
        e.delta = e.dx + nx * (e.dy + ny * e.dz);
        for (int a = 0; a < 3; ++a) P.ext[a] = std::max(P.ext[a], std::abs(vecs[i].c[a]));
    }

    // ---- clusterizer (clusterizer.cpp:52-184) ----
    // Boxes of the radii (doubles in the reference: sugarbox_search_ellipsoid_t),
    // mx = (int)(nx / rx + 2); a box overflows past limit = |template| / 250
    // (sugarbox_indexed_neighbour_lookup.h:58) and then holds no nodes.
    for (int i = 0; i < 3; ++i) P.cl_r[i] = (double)p.radii[i];
    P.mx = (int)(nx / P.cl_r[0] + 2);
    P.my = (int)(ny / P.cl_r[1] + 2);
    P.mz = (int)(nz / P.cl_r[2] + 2);
    P.limit = (long long)(P.tmpl.size() / 250);
    const long long nb = (long long)P.mx * P.my * P.mz;
    std::vector<int> count(nb, 0);
    std::vector<uint8_t> exceeded(nb, 0);
    auto bucket_of = [&](long long idx) {
        int x = (int)(idx % nx), y = (int)(idx % ((long long)nx * ny) / nx), z = (int)(idx / ((long long)nx * ny));
        int cx = (int)(x / P.cl_r[0]), cy = (int)(y / P.cl_r[1]), cz = (int)(z / P.cl_r[2]);
        return ((long long)cz * P.my + cy) * P.mx + cx;
    };
    for (long long i = 0; i < P.size; ++i) {
        if (!mask[i]) continue;
        long long b = bucket_of(i);
        if (exceeded[b]) continue;
        if (count[b] >= P.limit) {
            exceeded[b] = 1;
            count[b] = 0;
            continue;
        }
        count[b]++;
    }
    P.bucket_start.assign(nb + 1, 0);
    for (long long b = 0; b < nb; ++b) P.bucket_start[b + 1] = P.bucket_start[b] + count[b];
    P.bucket_nodes.assign(P.bucket_start[nb], 0);
    {
        std::vector<int> fill(P.bucket_start.begin(), P.bucket_start.end() - 1);
        for (long long i = 0; i < P.size; ++i) {
            if (!mask[i]) continue;
            long long b = bucket_of(i);
            if (exceeded[b]) continue;
            P.bucket_nodes[fill[b]++] = (int)i;
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
                P.bucket_clean[b] = clean ? 1 : 0;
                if (clean) {
                    P.any_clean = true;
                    P.max_candidates = std::max(P.max_candidates, cand);
                }
            }

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
    const int bx = 2 * P.B[0] + 1, by = 2 * P.B[1] + 1, bz = 2 * P.B[2] + 1;
    P.table.assign((size_t)bx * by * bz, 0.0);
    parallel_for(bz, threads, [&](long long lo, long long hi) {
        for (long long zi = lo; zi < hi; ++zi)
            for (int yi = 0; yi < by; ++yi)
                for (int xi = 0; xi < bx; ++xi) {
                    int x = xi - P.B[0], y = yi - P.B[1], z = (int)zi - P.B[2];
                    P.table[((size_t)zi * by + yi) * bx + xi] = cov((double)x, (double)y, (double)z);
                }
    });
    P.c0 = c0;

    // ---- informed-bit rows for the device template search ----
    P.px = 32 * ((P.ext[0] + 31) / 32);
    P.nseg = (nx + 31) / 32;
    P.wpr = P.nseg + 2 * (P.px / 32) + 2;
}

}  // namespace hpgl_b200
