// ORACLE — test infrastructure only.  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline leg load this; the shipped library never links
// or calls it.  It is the checker the GPU results are compared against.
//
// CPU restatement of HPGL 0.9.9's kriging estimation path (ordinary, simple,
// locally-varying-mean, indicator and median-indicator kriging, and colocated
// simple cokriging with the Markov models I and II).  Each piece
// cites the reference file:line it follows (paths relative to the reference's
// src/geo_bsd/hpgl/).  Parity of this restatement is pinned by comparing it
// with the reference's own sources compiled by oracle/build_ref.sh (estimates,
// masks, neighbour lists, weights and variances).
//
// Build with -O2 -ffp-contract=off so that covariance and solver arithmetic
// round exactly like the reference compiled the same way.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#include <omp.h>

extern "C" int oracle_dpotf2_upper(int n, double *a, int lda);
extern "C" void oracle_dpotrs_upper(int n, int nrhs, const double *a, int lda, double *b, int ldb);

namespace {

enum { KIND_OK = 0, KIND_SK = 1, KIND_LVM = 2, KIND_IK = 3, KIND_MEDIAN_IK = 4 };
enum { ST_SUCCESS = 0, ST_NO_NEIGHBOURS = 1, ST_SINGULAR = 2, ST_NOT_KRIGED = -1 };

}  // namespace

extern "C" {
// Per-category kriging parameters, the fields of hpgl_ik_params_t
// (api.h:110-120); `marginal_prob` is ignored for OK/SK/LVM/median IK.
typedef struct {
    int cov_type;
    double ranges[3];
    double angles[3];
    double sill;
    double nugget;
    int radii[3];
    int max_neighbours;
    double marginal_prob;
} oracle_params_t;
}

namespace {

// Anisotropy transform, cov_model.h:16-61: scale * ((Rx * Ry) * Rz), each
// 3x3 product summed left to right (TNT matmult, tnt_cmat.h:472-498).
void mat3_mul(const double *a, const double *b, double *c) {
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) {
            double s = 0;
            for (int j = 0; j < 3; ++j) s = s + a[3 * i + j] * b[3 * j + k];
            c[3 * i + k] = s;
        }
}

struct cov_model {
    int type;
    double sill, nugget, r0;
    double t[9];

    explicit cov_model(const oracle_params_t &p) {
        for (int i = 0; i < 3; ++i)
            if (p.ranges[i] == 0) throw std::runtime_error("All covariance ranges should be non-zero");
        type = p.cov_type;
        sill = p.sill;
        nugget = p.nugget;
        r0 = p.ranges[0];
        const double pi = 3.14159265358979323846264338327950288419;
        double a0 = (p.angles[0] * pi) / 180, a1 = (p.angles[1] * pi) / 180, a2 = (p.angles[2] * pi) / 180;
        double scale[9] = {1.0, 0, 0, 0, p.ranges[0] / p.ranges[1], 0, 0, 0, p.ranges[0] / p.ranges[2]};
        double rz[9] = {cos(a0), sin(a0), 0, -sin(a0), cos(a0), 0, 0, 0, 1};
        double ry[9] = {cos(a1), 0, -sin(a1), 0, 1, 0, sin(a1), 0, cos(a1)};
        double rx[9] = {1, 0, 0, 0, cos(a2), sin(a2), 0, -sin(a2), cos(a2)};
        double xy[9], xyz[9];
        mat3_mul(rx, ry, xy);
        mat3_mul(xy, rz, xyz);
        mat3_mul(scale, xyz, t);
    }

    // cov_model.h:63-77 (transfrom_and_norm) and :144-181 (models).
    double operator()(double v0, double v1, double v2) const {
        double v[3] = {v0, v1, v2};
        double result = 0.0;
        for (int i = 0; i < 3; ++i) {
            double d = 0.0;
            for (int j = 0; j < 3; ++j) d += v[j] * t[3 * i + j];
            result += d * d;
        }
        double h = sqrt(result);
        if (h < 0.0001) return sill - nugget;
        switch (type) {
        case 2: return (sill - nugget) * exp(-3 * pow(h / r0, 2));
        case 1: return (sill - nugget) * exp(-3 * h / r0);
        default:
            if (h > r0) return 0;
            return (sill - nugget) * (1 - 1.5 * h / r0 + 0.5 * pow(h / r0, 3));
        }
    }
    // cov_model.h:131-142: v = c1 - c2 of two grid locations.
    double at(const int *c1, const int *c2) const {
        return (*this)((double)(c1[0] - c2[0]), (double)(c1[1] - c2[1]), (double)(c1[2] - c2[2]));
    }
};

// The covariance seen by the search and the weights.  Ordinary kriging uses
// the model directly (ordinary_kriging.cpp:27-34); SK, LVM and IK use
// precalculated_covariances_t (precalculated_covariance.h:33-75) and median IK
// covariance_field_t (covariance_field.h:144-153): both a table over the
// +-radius box that returns 0 outside it.
struct covariance {
    cov_model model;
    bool truncated;
    int rx, ry, rz, sx, sy;
    std::vector<double> table;

    covariance(const oracle_params_t &p, bool trunc) : model(p), truncated(trunc) {
        rx = p.radii[0];
        ry = p.radii[1];
        rz = p.radii[2];
        sx = 2 * rx + 1;
        sy = 2 * ry + 1;
        if (truncated) {
            table.resize((size_t)sx * sy * (2 * rz + 1));
            for (int z = 0; z < 2 * rz + 1; ++z)
                for (int y = 0; y < sy; ++y)
                    for (int x = 0; x < sx; ++x)
                        table[((size_t)z * sy + y) * sx + x] = model(0.0 - (x - rx), 0.0 - (y - ry), 0.0 - (z - rz));
        }
    }
    // cov(c1, c2); the table path keys the offset c2 - c1.
    double operator()(const int *c1, const int *c2) const {
        if (!truncated) return model.at(c1, c2);
        int vx = c2[0] - c1[0], vy = c2[1] - c1[1], vz = c2[2] - c1[2];
        if (vx < -rx || vx > rx || vy < -ry || vy > ry || vz < -rz || vz > rz) return 0;
        return table[((size_t)(vz + rz) * sy + (vy + ry)) * sx + (vx + rx)];
    }
};

struct grid3 {
    int nx, ny, nz;
    // sugarbox_grid.cpp:70-74 and sugarbox_grid.h:39-57.
    void loc(int idx, int *c) const {
        c[0] = idx % nx;
        c[1] = idx % (nx * ny) / nx;
        c[2] = idx / (nx * ny);
    }
    int index(const int *c) const {
        if ((unsigned)c[0] < (unsigned)nx && (unsigned)c[1] < (unsigned)ny && (unsigned)c[2] < (unsigned)nz)
            return c[2] * nx * ny + c[1] * nx + c[0];
        return -1;
    }
    int size() const { return nx * ny * nz; }
};

// Search template, calc_cov_field (covariance_field.h:62-106): every offset of
// the +-radius box whose covariance exceeds C(0)/100, collected in z-y-x
// order as the vector (0,0,0) - (x,y,z), sorted by std::sort on the
// covariance, descending (same unstable algorithm, same input order, hence
// the same order of ties), then cut at the first entry below the threshold.
std::vector<int> build_template(const covariance &cov, const oracle_params_t &p) {
    int rx = p.radii[0], ry = p.radii[1], rz = p.radii[2];
    int zero[3] = {0, 0, 0};
    double threshold = cov(zero, zero) / 100;
    int xd = 2 * rx + 1, yd = 2 * ry + 1;
    std::vector<double> data;
    struct v3 { int c[3]; };
    std::vector<v3> vecs;
    for (int z = -rz; z <= rz; ++z)
        for (int y = -ry; y <= ry; ++y)
            for (int x = -rx; x <= rx; ++x) {
                int c[3] = {x, y, z};
                double value = cov(zero, c);
                data.push_back(value);
                if (value > threshold) vecs.push_back(v3{{-x, -y, -z}});
            }
    auto key = [&](const v3 &v) { return data[((size_t)(v.c[2] + rz) * yd + (v.c[1] + ry)) * xd + (v.c[0] + rx)]; };
    std::sort(vecs.begin(), vecs.end(), [&](const v3 &a, const v3 &b) { return key(a) > key(b); });
    for (size_t i = 0; i < vecs.size(); ++i) {
        if (cov(zero, vecs[i].c) < threshold) {
            vecs.resize(i);
            break;
        }
    }
    std::vector<int> out;
    for (auto &v : vecs) out.insert(out.end(), v.c, v.c + 3);
    return out;
}

// clusterizer_t (clusterizer.cpp:10-184): boxes of the search radii (the
// radii are doubles, sugarbox_search_ellipsoid_t; division truncates), each
// with a fill limit = template size / 250 (sugarbox_indexed_neighbour_lookup.h:58).
struct clusterizer {
    grid3 g;
    double r[3];
    int mx, my, mz;
    size_t limit;
    std::vector<std::vector<int>> nodes;
    std::vector<char> exceeded;

    clusterizer(const grid3 &grid, const int *radii, size_t lim) : g(grid), limit(lim) {
        for (int i = 0; i < 3; ++i) r[i] = radii[i];
        mx = (int)(g.nx / r[0] + 2);
        my = (int)(g.ny / r[1] + 2);
        mz = (int)(g.nz / r[2] + 2);
        nodes.resize((size_t)mx * my * mz);
        exceeded.assign(nodes.size(), 0);
    }
    void cell(const int *c, int *cc) const {
        cc[0] = (int)(c[0] / r[0]);
        cc[1] = (int)(c[1] / r[1]);
        cc[2] = (int)(c[2] / r[2]);
    }
    // The cluster box is inclusive of mx,my,mz (geometry.h:232-235), which real
    // nodes never reach.
    int index(int cx, int cy, int cz) const {
        if (cx < 0 || cx > mx || cy < 0 || cy > my || cz < 0 || cz > mz) return -1;
        return cz * mx * my + cy * mx + cx;
    }
    void add(int idx) {
        int c[3], cc[3];
        g.loc(idx, c);
        cell(c, cc);
        int ci = index(cc[0], cc[1], cc[2]);
        if (exceeded[ci]) return;
        if (nodes[ci].size() >= limit) {
            exceeded[ci] = 1;
            nodes[ci].clear();
            return;
        }
        nodes[ci].push_back(idx);
    }
    bool limit_exceeded(int idx) const {
        int c[3], cc[3];
        g.loc(idx, c);
        cell(c, cc);
        for (int k = cc[2] - 1; k <= cc[2] + 1; ++k)
            for (int j = cc[1] - 1; j <= cc[1] + 1; ++j)
                for (int i = cc[0] - 1; i <= cc[0] + 1; ++i) {
                    int ci = index(i, j, k);
                    if (ci >= 0 && exceeded[ci]) return true;
                }
        return false;
    }
    void nearby(int idx, std::vector<int> &out) const {
        int c[3], cc[3];
        g.loc(idx, c);
        cell(c, cc);
        out.clear();
        for (int k = cc[2] - 1; k <= cc[2] + 1; ++k)
            for (int j = cc[1] - 1; j <= cc[1] + 1; ++j)
                for (int i = cc[0] - 1; i <= cc[0] + 1; ++i) {
                    int ci = index(i, j, k);
                    if (ci >= 0) out.insert(out.end(), nodes[ci].begin(), nodes[ci].end());
                }
    }
};

// indexed_neighbour_lookup_t (sugarbox_indexed_neighbour_lookup.h:41-130)
// over neighbour_lookup_t (sugarbox_neighbour_lookup.h:23-61).
struct lookup {
    const grid3 &g;
    const covariance &cov;
    std::vector<int> tmpl;  // (dx,dy,dz) triples
    clusterizer cl;
    int max_nb;

    lookup(const grid3 &grid, const covariance &c, const oracle_params_t &p)
        : g(grid), cov(c), tmpl(build_template(c, p)), cl(grid, p.radii, tmpl.size() / 3 / 250),
          max_nb(p.max_neighbours) {}

    void find(int node, const unsigned char *mask, std::vector<int> &out, bool *via_template) const {
        out.clear();
        int center[3];
        g.loc(node, center);
        auto informed = [&](int idx) { return idx >= 0 && idx < g.size() && mask[idx] != 0; };
        if (cl.limit_exceeded(node)) {
            // Template walk: the first max_nb informed in-grid cells in template order.
            *via_template = true;
            int n_t = (int)tmpl.size() / 3;
            for (int t = 0; t < n_t && (int)out.size() < max_nb; ++t) {
                int pt[3] = {center[0] + tmpl[3 * t], center[1] + tmpl[3 * t + 1], center[2] + tmpl[3 * t + 2]};
                int idx = g.index(pt);
                if (informed(idx)) out.push_back(idx);
            }
            return;
        }
        *via_template = false;
        std::vector<int> cand;
        cl.nearby(node, cand);
        struct entry { int index; double cov; };
        std::vector<entry> sorted;
        double threshold = cov(center, center) / 100;
        for (int idx : cand) {
            int c[3];
            g.loc(idx, c);
            double v = cov(center, c);
            if (v > threshold) sorted.push_back(entry{idx, v});
        }
        std::sort(sorted.begin(), sorted.end(), [](const entry &a, const entry &b) { return a.cov > b.cov; });
        for (size_t i = 0; i < sorted.size() && (int)i < max_nb; ++i) out.push_back(sorted[i].index);
    }
};

// sk_kriging_weights_3 / ok_kriging_weights_3 (my_kriging_weights.h:26-255).
// Returns success; writes weights (n) and the variance of the reference's
// formula (ok: including the `- weights[size-1]` term, :246).
bool kriging_weights(bool ordinary, const int *center, const std::vector<int> &coords, const covariance &cov,
                     std::vector<double> &w, double &variance) {
    int n = (int)coords.size() / 3;
    w.assign(n, 0.0);
    if (n <= 0) return false;
    std::vector<double> A((size_t)n * n), b(n);
    for (int i = 0; i < n; ++i) {
        for (int j = i; j < n; ++j) {
            A[(size_t)i * n + j] = cov(&coords[3 * i], &coords[3 * j]);
            A[(size_t)j * n + i] = A[(size_t)i * n + j];
        }
        b[i] = cov(&coords[3 * i], center);
    }
    int info = oracle_dpotf2_upper(n, A.data(), n);
    bool solved = info == 0;
    if (!ordinary) {
        for (int i = 0; i < n; ++i) w[i] = b[i];
        oracle_dpotrs_upper(n, 1, A.data(), n, w.data(), n);
    } else {
        std::vector<double> sk(b), ones(n, 1.0);
        oracle_dpotrs_upper(n, 1, A.data(), n, sk.data(), n);
        oracle_dpotrs_upper(n, 1, A.data(), n, ones.data(), n);
        double sum_sk = 0, sum_ones = 0;
        for (int k = 0; k < n; ++k) {
            sum_sk += sk[k];
            sum_ones += ones[k];
        }
        double mu = (sum_sk - 1) / sum_ones;
        for (int k = 0; k < n; ++k) w[k] = sk[k] - mu * ones[k];
    }
    if (solved) {
        double v = cov(center, center);
        for (int i = 0; i < n; ++i) v -= w[i] * b[i];
        if (ordinary) v -= w[n - 1];
        variance = v;
    } else {
        variance = -1;
    }
    return solved;
}

struct outputs {
    float *out_values;
    unsigned char *out_codes;
    unsigned char *out_mask;
    double *variance;
    signed char *status;
    int *nb_count;
    int *nb_index;
    double *weights;
    float *probs;
    unsigned char *via_template;
    int nb_cap;
};

// calc_mean (calc_mean.cpp:6-30): double sum of informed values / count.
double calc_mean(const float *values, const unsigned char *mask, int size) {
    int count = 0;
    double sum = 0;
    for (int i = 0; i < size; ++i)
        if (mask[i]) {
            sum += values[i];
            count += 1;
        }
    return count == 0 ? 0 : sum / count;
}

void coords_of(const grid3 &g, const std::vector<int> &idx, std::vector<int> &coords) {
    coords.resize(idx.size() * 3);
    for (size_t i = 0; i < idx.size(); ++i) g.loc(idx[i], &coords[3 * i]);
}

void dump_system(const outputs &o, long slot, const std::vector<int> &nb, const std::vector<double> &w,
                 double variance, int status, bool via_t) {
    if (o.nb_count) o.nb_count[slot] = (int)nb.size();
    if (o.via_template) o.via_template[slot] = via_t ? 1 : 0;
    for (size_t i = 0; i < nb.size() && (int)i < o.nb_cap; ++i) {
        if (o.nb_index) o.nb_index[slot * o.nb_cap + i] = nb[i];
        if (o.weights) o.weights[slot * o.nb_cap + i] = i < w.size() ? w[i] : 0.0;
    }
    if (o.variance) o.variance[slot] = variance;
    if (o.status) o.status[slot] = (signed char)status;
}

// cont_kriging (cont_kriging.h:39-121) for OK / SK / LVM.
void cont_kriging(int kind, const grid3 &g, const float *values, const unsigned char *mask, const float *mean_cube,
                  const oracle_params_t &p, double sk_mean, int sk_auto, const outputs &o, const int *list,
                  int n_list) {
    int size = g.size();
    covariance cov(p, kind != KIND_OK);
    lookup nl(g, cov, p);
    for (int n = 0; n < size; ++n)
        if (mask[n]) nl.cl.add(n);
    double mean = 0;
    if (kind == KIND_SK) mean = sk_auto ? calc_mean(values, mask, size) : sk_mean;
    int count = list ? n_list : size;
#pragma omp parallel for schedule(dynamic, 256)
    for (int it = 0; it < count; ++it) {
        int idx = list ? list[it] : it;
        if (mask[idx]) {
            o.out_values[idx] = values[idx];
            o.out_mask[idx] = 1;
            if (o.status) o.status[idx] = ST_NOT_KRIGED;
            continue;
        }
        // Mean provider (mean_provider.h:8-33): 0, a constant, or the mean cube;
        // the combiner takes the centre mean and neighbour means as float.
        auto mean_at = [&](int i) -> float {
            if (kind == KIND_OK) return 0.0f;
            if (kind == KIND_SK) return (float)mean;
            return mean_cube[i];
        };
        std::vector<int> nb, coords;
        bool via_t = false;
        nl.find(idx, mask, nb, &via_t);
        std::vector<double> w;
        double variance = -1;
        int status;
        if (nb.empty()) {
            status = ST_NO_NEIGHBOURS;
        } else {
            coords_of(g, nb, coords);
            int center[3];
            g.loc(idx, center);
            bool ok = kriging_weights(kind == KIND_OK, center, coords, cov, w, variance);
            status = ok ? ST_SUCCESS : ST_SINGULAR;
        }
        dump_system(o, idx, nb, w, variance, status, via_t);
        if (status == ST_SUCCESS) {
            // combine (combiner.h:9-24): float accumulation in neighbour order.
            float result = mean_at(idx);
            for (size_t i = 0; i < nb.size(); ++i)
                result += (float)(w[i] * (values[nb[i]] - mean_at(nb[i])));
            o.out_values[idx] = result;
            o.out_mask[idx] = 1;
        } else if (kind != KIND_OK) {
            // mean_on_failure (cont_kriging.h:87-97); OK leaves the node as is.
            o.out_values[idx] = (kind == KIND_SK) ? (float)mean : mean_cube[idx];
            o.out_mask[idx] = 1;
        }
    }
}

// do_indicator_kriging (indicator_kriging.h:57-124): every node, each category
// k with its own covariance table and lookup, value = (code == k), mean =
// marginal prob (a float, mean_provider.cpp:8-13), failure -> marginal prob;
// output = first most probable category (cdf_utils.cpp:9-24), mask := 1.
void indicator_kriging(const grid3 &g, const unsigned char *codes, const unsigned char *mask,
                       const oracle_params_t *params, int K, const outputs &o, const int *list, int n_list) {
    int size = g.size();
    std::vector<covariance *> covs;
    std::vector<lookup *> lookups;
    for (int k = 0; k < K; ++k) {
        covs.push_back(new covariance(params[k], true));
        lookups.push_back(new lookup(g, *covs[k], params[k]));
    }
    for (int n = 0; n < size; ++n)
        if (mask[n])
            for (int k = 0; k < K; ++k) lookups[k]->cl.add(n);
    int count = list ? n_list : size;
#pragma omp parallel for schedule(dynamic, 256)
    for (int it = 0; it < count; ++it) {
        int idx = list ? list[it] : it;
        std::vector<float> probs(K);
        int center[3];
        g.loc(idx, center);
        for (int k = 0; k < K; ++k) {
            float pk = (float)params[k].marginal_prob;
            std::vector<int> nb, coords;
            bool via_t = false;
            lookups[k]->find(idx, mask, nb, &via_t);
            std::vector<double> w;
            double variance = -1;
            int status;
            if (nb.empty()) {
                status = ST_NO_NEIGHBOURS;
            } else {
                coords_of(g, nb, coords);
                status = kriging_weights(false, center, coords, *covs[k], w, variance) ? ST_SUCCESS : ST_SINGULAR;
            }
            dump_system(o, (long)idx * K + k, nb, w, variance, status, via_t);
            float prob;
            if (status == ST_SUCCESS) {
                prob = pk;
                for (size_t i = 0; i < nb.size(); ++i) {
                    float v = codes[nb[i]] == k ? 1.0f : 0.0f;
                    prob += (float)(w[i] * (v - pk));
                }
            } else {
                prob = pk;
            }
            probs[k] = prob;
            if (o.probs) o.probs[(long)idx * K + k] = prob;
        }
        double max_prob = probs[0];
        int max_idx = 0;
        for (int k = 1; k < K; ++k) {
            double pr = probs[k];
            if (pr > max_prob) {
                max_prob = pr;
                max_idx = k;
            }
        }
        o.out_codes[idx] = (unsigned char)max_idx;
        o.out_mask[idx] = 1;
    }
    for (int k = 0; k < K; ++k) {
        delete lookups[k];
        delete covs[k];
    }
}

// median_ik_for_two_indicators (median_ik.cpp:24-93): one system per node with
// the truncated table, value = (code == 1), centre/neighbour mean =
// (float)marginal_probs[1], estimate accumulated in double (result_t is
// double there), output = prob <= 0.5 ? 0 : 1 after a cast to float.  The
// reference leaves `prob` uninitialised when the system fails; this
// restatement uses the marginal probability for such nodes.
void median_ik(const grid3 &g, const unsigned char *codes, const unsigned char *mask, const oracle_params_t &p,
               double marginal1, const outputs &o, const int *list, int n_list) {
    int size = g.size();
    covariance cov(p, true);
    lookup nl(g, cov, p);
    for (int n = 0; n < size; ++n)
        if (mask[n]) nl.cl.add(n);
    float m = (float)marginal1;
    int count = list ? n_list : size;
#pragma omp parallel for schedule(dynamic, 256)
    for (int it = 0; it < count; ++it) {
        int idx = list ? list[it] : it;
        int center[3];
        g.loc(idx, center);
        std::vector<int> nb, coords;
        bool via_t = false;
        nl.find(idx, mask, nb, &via_t);
        std::vector<double> w;
        double variance = -1;
        int status;
        if (nb.empty()) {
            status = ST_NO_NEIGHBOURS;
        } else {
            coords_of(g, nb, coords);
            status = kriging_weights(false, center, coords, cov, w, variance) ? ST_SUCCESS : ST_SINGULAR;
        }
        dump_system(o, idx, nb, w, variance, status, via_t);
        double prob = m;
        if (status == ST_SUCCESS) {
            for (size_t i = 0; i < nb.size(); ++i) {
                float v = codes[nb[i]] == 1 ? 1.0f : 0.0f;
                prob += (double)(w[i] * (v - m));
            }
        }
        if (o.probs) o.probs[idx] = (float)prob;
        o.out_codes[idx] = ((float)prob <= 0.5) ? 0 : 1;
        o.out_mask[idx] = 1;
    }
}

// gauss_solve (gauss_solver.cpp:5-63): for column i the first row not yet
// used whose entry is non-zero becomes the pivot row (no magnitude
// pivoting); it is divided by its pivot entry from column i on, and
// eliminated from every unused row; back substitution reads B in position
// order (B[i]) with the pivot rows' coefficients, as the reference does.
// A is row-major size x size and is overwritten; returns false when a
// column has no usable pivot.
bool gauss_solve(double *A, double *B, double *X, int size) {
    std::vector<int> flags(size, 0), order(size, 0);
    for (int i = 0; i < size; ++i) {
        int row = -1;
        for (int j = 0; j < size; ++j)
            if (flags[j] == 0 && A[(size_t)j * size + i] != 0) {
                row = j;
                flags[j] = 1;
                order[i] = j;
                break;
            }
        if (row < 0) return false;
        const double coef = A[(size_t)row * size + i];
        for (int j = i; j < size; ++j) A[(size_t)row * size + j] /= coef;
        B[row] /= coef;
        for (int j = 0; j < size; ++j) {
            if (flags[j] == 0) {
                const double c = A[(size_t)j * size + i];
                for (int k = i; k < size; ++k) A[(size_t)j * size + k] -= c * A[(size_t)row * size + k];
                B[j] -= c * B[row];
            }
        }
    }
    for (int i = size - 1; i >= 0; --i) {
        const int row = order[i];
        X[i] = B[i];
        for (int j = size - 1; j > i; --j) X[i] -= A[(size_t)row * size + j] * X[j];
    }
    return true;
}

// simple_cokriging_markI / markII (simple_cokriging_markI.cpp:19-307):
// colocated simple cokriging with the Markov model I or II cross
// covariance.  The search is neighbour_lookup_t over the untruncated primary
// model (no clusterizer); the (N+1)-row system holds the primary covariances,
// the cross covariances coef * C_x(center - x_i) in its last row and column,
// and the secondary variance in the corner; b = (C(x_i - center), coef * C_x(0)).
// Means are floats (mean_t); the estimate is
// m1 + sum (v_i - m1) w_i + w_N (s - m2), each step widened to double and
// rounded back to the float result; failures give m1 + s - m2.
void cokriging(int mark, const grid3 &g, const float *values, const unsigned char *mask, const float *svalues,
               const unsigned char *smask, const oracle_params_t &pp, const oracle_params_t *sp, float m1, float m2,
               double secondary_variance_m1, double corr, const outputs &o, const int *list, int n_list) {
    covariance cov(pp, false);
    const cov_model &model = cov.model;
    cov_model smodel(mark == 2 ? *sp : pp);
    const int zero[3] = {0, 0, 0};
    double coef, secondary_variance;
    if (mark == 1) {
        // cross_cov_model_mark_i_t: p12 * sqrt(d2) / sqrt(C(0))
        coef = corr * sqrt(secondary_variance_m1) / sqrt(model.at(zero, zero));
        secondary_variance = secondary_variance_m1;
    } else {
        // cross_cov_model_mark_ii_t: p12 * sqrt(C2(0) / C1(0))
        const double pv = model.at(zero, zero);
        secondary_variance = smodel.at(zero, zero);
        coef = corr * sqrt(secondary_variance / pv);
    }
    const cov_model &cross = mark == 1 ? model : smodel;
    const std::vector<int> tmpl = build_template(cov, pp);
    const int n_t = (int)tmpl.size() / 3;
    const int size = g.size();
    const int count = list ? n_list : size;
#pragma omp parallel for schedule(dynamic, 256)
    for (int it = 0; it < count; ++it) {
        const int idx = list ? list[it] : it;
        float result;
        std::vector<int> nb;
        std::vector<double> w;
        int status = ST_NOT_KRIGED;
        if (mask[idx]) {
            result = values[idx];
        } else {
            const float sv = smask[idx] ? svalues[idx] : m2;
            int center[3];
            g.loc(idx, center);
            // neighbour_lookup_t::find (sugarbox_neighbour_lookup.h:35-61)
            for (int t = 0; t < n_t && (int)nb.size() < pp.max_neighbours; ++t) {
                int pt[3] = {center[0] + tmpl[3 * t], center[1] + tmpl[3 * t + 1], center[2] + tmpl[3 * t + 2]};
                const int q = g.index(pt);
                if (q >= 0 && mask[q]) nb.push_back(q);
            }
            bool ok = !nb.empty();
            status = ok ? ST_SUCCESS : ST_NO_NEIGHBOURS;
            if (ok) {
                // build_system (simple_cokriging_markI.cpp:19-54)
                const int n = (int)nb.size(), ms = n + 1;
                std::vector<int> coords;
                coords_of(g, nb, coords);
                std::vector<double> A((size_t)ms * ms), b(ms);
                for (int i = 0; i < n; ++i)
                    for (int j = i; j < n; ++j) {
                        A[(size_t)i * ms + j] = model.at(&coords[3 * i], &coords[3 * j]);
                        A[(size_t)j * ms + i] = A[(size_t)i * ms + j];
                    }
                for (int i = 0; i < n; ++i) {
                    A[(size_t)n * ms + i] = coef * cross.at(center, &coords[3 * i]);
                    A[(size_t)i * ms + n] = A[(size_t)n * ms + i];
                    b[i] = model.at(&coords[3 * i], center);
                }
                b[n] = coef * cross.at(zero, zero);
                A[(size_t)ms * ms - 1] = secondary_variance;
                w.resize(ms);
                ok = gauss_solve(A.data(), b.data(), w.data(), ms);
                if (!ok) status = ST_SINGULAR;
            }
            if (ok) {
                // combine (simple_cokriging_markI.cpp:84-105)
                const int n = (int)nb.size();
                result = m1;
                for (int i = 0; i < n; ++i) result += (values[nb[i]] - m1) * w[i];
                result += w[n] * (sv - m2);
            } else {
                result = m1 + sv - m2;
            }
        }
        o.out_values[idx] = result;
        o.out_mask[idx] = 1;
        if (o.status) o.status[idx] = (signed char)status;
        if (o.nb_count) o.nb_count[idx] = (int)nb.size();
        if (o.nb_index)
            for (size_t i = 0; i < nb.size() && (int)i < o.nb_cap; ++i) o.nb_index[(size_t)idx * o.nb_cap + i] = nb[i];
        if (o.weights && status == ST_SUCCESS)
            for (size_t i = 0; i < w.size() && (int)i <= o.nb_cap; ++i)
                o.weights[(size_t)idx * (o.nb_cap + 1) + i] = w[i];
    }
}

}  // namespace

extern "C" {

// Colocated simple cokriging (mark 1 or 2) of a primary cube with a
// secondary cube of the same shape.  `secondary` (Markov model II only) is
// the secondary covariance; `secondary_variance` is Markov model I's d2.
// Optional dumps per node: status, neighbour count and indices (`nb_cap`
// per node), weights (`nb_cap` + 1 per node, the last one the secondary's).
int oracle_cokriging(int mark, int nx, int ny, int nz, const float *values, const unsigned char *mask,
                     const float *svalues, const unsigned char *smask, const oracle_params_t *primary,
                     const oracle_params_t *secondary, double primary_mean, double secondary_mean,
                     double secondary_variance, double corr, float *out_values, unsigned char *out_mask,
                     signed char *status, int *nb_count, int *nb_index, double *weights, int nb_cap,
                     const int *node_list, int n_nodes, int threads, char *err, int err_len) {
    try {
        if (threads > 0) omp_set_num_threads(threads);
        if (mark != 1 && mark != 2) throw std::runtime_error("mark must be 1 or 2");
        for (int i = 0; i < 3; ++i)
            if (primary->radii[i] <= 0) throw std::runtime_error("search radii must be positive");
        grid3 g{nx, ny, nz};
        outputs o{out_values, nullptr, out_mask, nullptr, status, nb_count, nb_index, weights, nullptr, nullptr,
                  nb_cap};
        // the reference passes the means as mean_t (float)
        cokriging(mark, g, values, mask, svalues, smask, *primary, secondary, (float)primary_mean,
                  (float)secondary_mean, secondary_variance, corr, o, node_list, n_nodes);
        return 0;
    } catch (const std::exception &e) {
        if (err && err_len > 0) {
            strncpy(err, e.what(), err_len - 1);
            err[err_len - 1] = 0;
        }
        return 1;
    }
}

// Runs one kriging job.  kind: 0 OK, 1 SK, 2 LVM, 3 IK, 4 median IK.
// Inputs: `values` (OK/SK/LVM) or `codes` (IK/median IK), `mask`,
// `mean_cube` (LVM), `params` (K entries for IK, else 1), `sk_mean` /
// `sk_auto_mean` (SK), `median_marginal1` (median IK marginal_probs[1]).
// Outputs: out_values or out_codes, out_mask (caller pre-fills them like the
// reference's callers do); the optional dumps are per system slot (node for
// OK/SK/LVM/median IK, node*K + k for IK): variance, status (0 success,
// 1 no neighbours, 2 singular, -1 informed node copied), neighbour count,
// neighbour indices and weights (`nb_cap` per slot), probabilities (IK:
// node*K + k; median IK: node) and whether the template path was used.
// With `node_list` non-null only those `n_nodes` nodes are processed (the
// search still sees every informed cell), so large grids can be sampled.
// Returns 0, or 1 with a message in `err` (size `err_len`).
int oracle_krige(int kind, int nx, int ny, int nz, const float *values, const unsigned char *codes,
                 const unsigned char *mask, const float *mean_cube, const oracle_params_t *params, int K,
                 double sk_mean, int sk_auto_mean, double median_marginal1, float *out_values,
                 unsigned char *out_codes, unsigned char *out_mask, double *variance, signed char *status,
                 int *nb_count, int *nb_index, double *weights, float *probs, unsigned char *via_template,
                 int nb_cap, const int *node_list, int n_nodes, int threads, char *err, int err_len) {
    try {
        if (threads > 0) omp_set_num_threads(threads);
        grid3 g{nx, ny, nz};
        outputs o{out_values, out_codes, out_mask, variance, status, nb_count, nb_index, weights, probs,
                  via_template, nb_cap};
        for (int k = 0; k < (kind == KIND_IK ? K : 1); ++k) {
            if (params[k].max_neighbours > 64) throw std::runtime_error("max_neighbours > 64 is not restated");
            for (int i = 0; i < 3; ++i)
                if (params[k].radii[i] <= 0) throw std::runtime_error("search radii must be positive");
        }
        switch (kind) {
        case KIND_OK:
        case KIND_SK:
        case KIND_LVM: cont_kriging(kind, g, values, mask, mean_cube, params[0], sk_mean, sk_auto_mean, o, node_list, n_nodes); break;
        case KIND_IK: indicator_kriging(g, codes, mask, params, K, o, node_list, n_nodes); break;
        case KIND_MEDIAN_IK: median_ik(g, codes, mask, params[0], median_marginal1, o, node_list, n_nodes); break;
        default: throw std::runtime_error("unknown kind");
        }
        return 0;
    } catch (const std::exception &e) {
        if (err && err_len > 0) {
            strncpy(err, e.what(), err_len - 1);
            err[err_len - 1] = 0;
        }
        return 1;
    }
}

// ---- sequential Gaussian simulation --------------------------------------------
}  // extern "C"

namespace {

// path_random_generator.cpp:20-66: a full-period linear congruential walk
// over [0, size).  The reference includes its prime table from primes.txt,
// which its checkout lacks; init_rnd's asserts leave one reading of it, every
// prime in increasing order past the grid size, which this restates.
struct path_walk {
    long long A = 1, C = 2, M = 1, R = 0;
    path_walk(long long size, long long seed) {
        M = size;
        const long long lim = std::max<long long>(size, 3) + 1;
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
        // path_random_generator_t(int size, int seed): the seed arrives as int
        const int s32 = (int)(uint32_t)seed;
        if (s32 < 0) throw std::runtime_error("the path is undefined for a negative seed");
        R = s32 % size;
    }
    long long next() {
        const long long r = R;
        R = (A * R + C) % M;
        return r;
    }
};

// boost::mt11213b: the Mersenne Twister (Matsumoto and Nishimura, 1998) with
// boost's published mt11213b parameters and the usual seeding.
struct mt11213b {
    enum { N = 351, M = 175, R = 19 };
    uint32_t x[N];
    int i = N;
    explicit mt11213b(uint32_t s) {
        x[0] = s;
        for (int k = 1; k < N; ++k) x[k] = 1812433253u * (x[k - 1] ^ (x[k - 1] >> 30)) + (uint32_t)k;
    }
    uint32_t operator()() {
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
    // mt_random_generator_t::operator()() (bs_random_generator.cpp:16-19)
    double uniform() { return double((*this)()) / double(0xffffffffu); }
};

// gaussian_cdf_t::inverse (gaussian_distribution.h:49-66), Odeh and Evans's
// rational approximation: the standard normal quantile of p.
double gaussian_quantile(double p) {
    const double ps[] = {-0.322232431088, -1.0, -0.342242088547, -0.0204231210245, -0.453642210148e-4};
    const double qs[] = {0.0993484626060, 0.588581570495, 0.531103462366, 0.103537752850, 0.38560700634e-2};
    const double p2 = (p > 0.5) ? (1 - p) : p;
    const double y = std::sqrt(std::log(1 / (p2 * p2)));
    double xp = y + ((((ps[4] * y + ps[3]) * y + ps[2]) * y + ps[1]) * y + ps[0]) /
                        ((((qs[4] * y + qs[3]) * y + qs[2]) * y + qs[1]) * y + qs[0]);
    if (p < 0.5) xp = -xp;
    return xp;
}

// non_parametric_cdf_2_t (non_parametric_cdf.h:185-260): a caller's CDF of
// increasing values and cumulative probabilities, read and inverted by float
// linear interpolation between the bracketing entries (the first / last
// entry outside them).
struct np_cdf {
    const float *v, *p;
    long long n;
    float prob(float value) const {
        const float *it = std::lower_bound(v, v + n, value);
        if (it == v + n) return p[n - 1];
        if (it == v) return p[0];
        const long long b = it - v, a = b - 1;
        return p[a] + (p[b] - p[a]) / (v[b] - v[a]) * (value - v[a]);
    }
    float inverse(float prob) const {
        if (n <= 0) return 0;
        const float *it = std::lower_bound(p, p + n, prob);
        if (it == p) return v[0];
        if (it == p + n) return v[n - 1];
        const long long b = it - p, a = b - 1;
        return v[a] + (v[b] - v[a]) / (p[b] - p[a]) * (prob - p[a]);
    }
};

// gaussian_cdf_t::operator() (gaussian_distribution.h:22-41), Abramowitz and
// Stegun 26.2.17, mean 0 and variance 1.
double gaussian_cdf(double x) {
    const double b[] = {0.319381530, -0.356563782, 1.781477937, -1.821255978, 1.330274429};
    double sx = (x - 0.0) / std::sqrt(1.0);
    const bool neg = sx < 0;
    if (neg) sx = -sx;
    const double t = 1 / (1 + 0.2316419 * sx);
    const double zx = 1 / std::sqrt(2 * 3.14159265358) * std::exp(-sx * sx / 2);
    const double r = 1 - zx * ((((b[4] * t + b[3]) * t + b[2]) * t + b[1]) * t + b[0]) * t;
    return neg ? 1 - r : r;
}

// do_sequential_gausian_simulation (sequential_simulation.h:49-122) with
// neighbour_lookup_t over the precalculated (radius-truncated) covariance:
// nodes in the walk's order; each uninformed node inside the simulation mask
// is kriged from the informed cells and the nodes simulated before it (SK with
// mean 0, OK, or SK with the mean cube), and set to the Gaussian quantile of
// the next draw with the kriged mean and variance (N(0, 1) when the kriging
// fails).
void sgs(const grid3 &g, float *values, unsigned char *mask, const oracle_params_t &p, bool ordinary,
         const float *lvm, long long seed, const unsigned char *sim_mask, int *order, int *n_order) {
    covariance cov(p, true);
    const std::vector<int> tmpl = build_template(cov, p);
    const int n_t = (int)tmpl.size() / 3;
    const long long size = g.size();
    path_walk path(size, seed);
    mt11213b gen((uint32_t)seed);
    int count = 0;
    long long node = path.next();
    for (long long counter = 0; counter < size; ++counter, node = path.next()) {
        if (mask[node]) continue;
        if (sim_mask && sim_mask[node] != 1) continue;
        if (order) order[count] = (int)node;
        ++count;
        int center[3];
        g.loc((int)node, center);
        std::vector<int> nb, coords;
        for (int t = 0; t < n_t && (int)nb.size() < p.max_neighbours; ++t) {
            int pt[3] = {center[0] + tmpl[3 * t], center[1] + tmpl[3 * t + 1], center[2] + tmpl[3 * t + 2]};
            const int idx = g.index(pt);
            if (idx >= 0 && mask[idx]) nb.push_back(idx);
        }
        auto mean_at = [&](int i) -> float { return lvm ? lvm[i] : 0.0f; };
        bool ok = false;
        double variance = -1;
        float mean = 0.f;
        if (!nb.empty()) {
            coords_of(g, nb, coords);
            std::vector<double> w;
            ok = kriging_weights(ordinary, center, coords, cov, w, variance);
            if (ok) {
                float result = mean_at((int)node);
                for (size_t i = 0; i < nb.size(); ++i) result += (float)(w[i] * (values[nb[i]] - mean_at(nb[i])));
                mean = result;
            }
        }
        const double u = gen.uniform();
        const double xp = gaussian_quantile(u);
        const double value = ok ? xp * std::sqrt(variance) + (double)mean : xp * std::sqrt(1.0) + 0.0;
        values[node] = (float)value;
        mask[node] = 1;
    }
    if (n_order) *n_order = count;
}

// corellogramed_weights_3 (my_kriging_weights.h:257-363): simple kriging of
// the system scaled by the indicator standard deviations sigma =
// sqrt(m (1 - m)) of the neighbours' and the centre's means (a mean of
// exactly 0 or 1 moved by 1e-5): A(i,j) = C(x_i, x_j) (s_i s_j), b_i =
// C(x_i, x0) (s_i s_c); the weights are not rescaled.
bool correlogram_weights(const int *center, float center_mean, const std::vector<int> &coords,
                         const std::vector<float> &means, const covariance &cov, std::vector<double> &w) {
    const int n = (int)coords.size() / 3;
    w.assign(n, 0.0);
    if (n <= 0) return false;
    auto sigma = [](double m) {
        if (m == 0) m += 0.00001;
        if (m == 1) m -= 0.00001;
        return std::sqrt(m * (1 - m));
    };
    const double sc = sigma(center_mean);
    std::vector<double> sg(n), A((size_t)n * n), b(n);
    for (int i = 0; i < n; ++i) sg[i] = sigma(means[i]);
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) A[(size_t)i * n + j] = cov(&coords[3 * i], &coords[3 * j]) * (sg[i] * sg[j]);
        b[i] = cov(&coords[3 * i], center) * (sg[i] * sc);
    }
    const int info = oracle_dpotf2_upper(n, A.data(), n);
    for (int i = 0; i < n; ++i) w[i] = b[i];
    oracle_dpotrs_upper(n, 1, A.data(), n, w.data(), n);
    return info == 0;
}

// do_sis (sequential_indicator_simulation.cpp:23-116): along the random path
// each uninformed node inside the simulation mask gets, per category k, the
// simple-kriged probability of code k from the informed and already
// simulated nodes (kriging_interpolation.h:228-265 with the category's
// radius-truncated covariance and template search; the estimate
// m_c + sum w_i (ind_i - m_i) accumulated in double; the mean, p_k or the
// category's mean cube, when the kriging fails); two categories krige
// category 0 only and take 1 - p for the other.  The code is drawn from the
// float probabilities (sample.cpp:8-21).
void sis(const grid3 &g, unsigned char *codes, unsigned char *mask, const oracle_params_t *p, int K,
         const float *const *lvm, bool corr, long long seed, const unsigned char *sim_mask) {
    std::vector<covariance> covs;
    std::vector<std::vector<int>> tmpls;
    for (int k = 0; k < K; ++k) {
        covs.emplace_back(p[k], true);
        tmpls.push_back(build_template(covs.back(), p[k]));
    }
    const long long size = g.size();
    path_walk path(size, seed);
    mt11213b gen((uint32_t)seed);
    long long node = path.next();
    for (long long counter = 0; counter < size; ++counter, node = path.next()) {
        if (mask[node]) continue;
        if (sim_mask && sim_mask[node] != 1) continue;
        int center[3];
        g.loc((int)node, center);
        std::vector<float> probs;
        const int cats = K == 2 ? 1 : K;
        for (int k = 0; k < cats; ++k) {
            const std::vector<int> &tm = tmpls[k];
            std::vector<int> nb, coords;
            for (size_t t = 0; t < tm.size() / 3 && (int)nb.size() < p[k].max_neighbours; ++t) {
                int pt[3] = {center[0] + tm[3 * t], center[1] + tm[3 * t + 1], center[2] + tm[3 * t + 2]};
                const int idx = g.index(pt);
                if (idx >= 0 && mask[idx]) nb.push_back(idx);
            }
            const float pk = (float)p[k].marginal_prob;
            auto mean_at = [&](long long i) -> float { return lvm ? lvm[k][i] : pk; };
            double prob = lvm ? (double)lvm[k][node] : (double)pk;
            if (!nb.empty()) {
                coords_of(g, nb, coords);
                std::vector<float> means(nb.size());
                for (size_t i = 0; i < nb.size(); ++i) means[i] = mean_at(nb[i]);
                std::vector<double> w;
                double variance;
                const bool ok = corr ? correlogram_weights(center, mean_at(node), coords, means, covs[k], w)
                                     : kriging_weights(false, center, coords, covs[k], w, variance);
                if (ok) {
                    double r = (float)mean_at(node);
                    for (size_t i = 0; i < nb.size(); ++i)
                        r += w[i] * (float)((codes[nb[i]] == k ? 1 : 0) - means[i]);
                    prob = r;
                }
            }
            probs.push_back((float)prob);
            if (K == 2) probs.push_back((float)(1 - prob));
        }
        double sum = 0.0;
        for (float q : probs) sum += q;
        const double s = gen.uniform() * sum;
        double acc = 0;
        int code = (int)probs.size() - 1;
        for (size_t i = 0; i < probs.size(); ++i) {
            acc += probs[i];
            if (s < acc) {
                code = (int)i;
                break;
            }
        }
        codes[node] = (unsigned char)code;
        mask[node] = 1;
    }
}

}  // namespace

extern "C" {

// Sequential Gaussian simulation in place on values / mask; `order`
// (optional) receives the simulated nodes in simulation order.
int oracle_sgs(int nx, int ny, int nz, float *values, unsigned char *mask, const oracle_params_t *p, int ordinary,
               const float *lvm, long long seed, const unsigned char *sim_mask, int *order, int *n_order, char *err,
               int err_len) {
    try {
        if (p->max_neighbours > 64) throw std::runtime_error("max_neighbours > 64 is not restated");
        sgs(grid3{nx, ny, nz}, values, mask, *p, ordinary != 0, lvm, seed, sim_mask, order, n_order);
        return 0;
    } catch (const std::exception &e) {
        if (err && err_len > 0) {
            strncpy(err, e.what(), err_len - 1);
            err[err_len - 1] = 0;
        }
        return 1;
    }
}

// Normal-score transforms of sequential Gaussian simulation (cdf_utils.h:12-50):
// direction 0 maps values through the CDF to the standard normal quantile
// (transform_cdf_p / transform_cdf_ptr from non_parametric_cdf_2_t to
// gaussian_cdf_t), direction 1 back (gaussian_cdf_t to the CDF's inverse,
// the probability passed as float).  Only nodes with mask != 0 (every node
// when mask is null); out may be in.
void oracle_cdf_transform(const float *in, float *out, const unsigned char *mask, long long n, const float *cdf_values,
                          const float *cdf_probs, long long cdf_size, int direction) {
    const np_cdf c{cdf_values, cdf_probs, cdf_size};
    for (long long i = 0; i < n; ++i) {
        if (mask && !mask[i]) continue;
        if (direction == 0) {
            const double P = c.prob(in[i]);
            out[i] = (float)(gaussian_quantile(P) * std::sqrt(1.0) + 0.0);
        } else {
            const double P = gaussian_cdf(in[i]);
            out[i] = c.inverse((float)P);
        }
    }
}

// Sequential indicator simulation in place on codes / mask; `lvm` (optional)
// holds K mean cubes, `corr` selects the correlogram weights.
int oracle_sis(int nx, int ny, int nz, unsigned char *codes, unsigned char *mask, const oracle_params_t *p, int K,
               const float *const *lvm, int corr, long long seed, const unsigned char *sim_mask, char *err,
               int err_len) {
    try {
        if (K < 2) throw std::runtime_error("at least two categories");
        sis(grid3{nx, ny, nz}, codes, mask, p, K, lvm, corr != 0, seed, sim_mask);
        return 0;
    } catch (const std::exception &e) {
        if (err && err_len > 0) {
            strncpy(err, e.what(), err_len - 1);
            err[err_len - 1] = 0;
        }
        return 1;
    }
}

// The standard normal quantiles of the first n draws of the generator.
void oracle_sgs_draws(long long seed, long long n, double *xp) {
    mt11213b gen((uint32_t)seed);
    for (long long k = 0; k < n; ++k) xp[k] = gaussian_quantile(gen.uniform());
}

// The sorted search template as (dx,dy,dz) triples; returns its length or -1
// when `cap` is too small.
int oracle_template(const oracle_params_t *p, int truncated, int *out_xyz, int cap) {
    covariance cov(*p, truncated != 0);
    std::vector<int> t = build_template(cov, *p);
    int n = (int)t.size() / 3;
    if (n > cap) return -1;
    std::copy(t.begin(), t.end(), out_xyz);
    return n;
}
}

extern "C" {
// Simple-kriging weights of one point from explicit coordinates:
// hpgl_simple_kriging_weights (api.cpp:292-342) over simple_kriging_weights
// (simple_kriging.cpp:15-35): float coordinates widened to double, the
// untruncated model on real-valued offsets, sk_kriging_weights_3
// (my_kriging_weights.h:26-129).  Returns 0, or 1 when the system is not
// positive definite (the reference then reads past an emptied vector).
int oracle_sk_weights(const float *center, const float *xs, const float *ys, const float *zs, int n,
                      const oracle_params_t *p, float *weights) {
    try {
        cov_model model(*p);
        if (n <= 0) return 0;
        double c[3] = {center[0], center[1], center[2]};
        std::vector<double> pts(3 * (size_t)n);
        for (int i = 0; i < n; ++i) {
            pts[3 * i] = xs[i];
            pts[3 * i + 1] = ys[i];
            pts[3 * i + 2] = zs[i];
        }
        std::vector<double> A((size_t)n * n), b(n);
        for (int i = 0; i < n; ++i) {
            for (int j = i; j < n; ++j) {
                A[(size_t)i * n + j] = model(pts[3 * i] - pts[3 * j], pts[3 * i + 1] - pts[3 * j + 1],
                                             pts[3 * i + 2] - pts[3 * j + 2]);
                A[(size_t)j * n + i] = A[(size_t)i * n + j];
            }
            b[i] = model(pts[3 * i] - c[0], pts[3 * i + 1] - c[1], pts[3 * i + 2] - c[2]);
        }
        if (n > 64) return 2;
        int info = oracle_dpotf2_upper(n, A.data(), n);
        std::vector<double> w(b);
        oracle_dpotrs_upper(n, 1, A.data(), n, w.data(), n);
        if (info != 0) return 1;
        for (int i = 0; i < n; ++i) weights[i] = (float)w[i];
        return 0;
    } catch (const std::exception &) {
        return 3;
    }
}
}
