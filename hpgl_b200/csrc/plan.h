// Host-side planning of one kriging job: everything that depends only on the
// variogram, the search parameters and the informed mask, computed once per
// job before the device pipeline runs.  All of it reproduces the reference's
// arithmetic bit for bit (compiled with -ffp-contract=off, glibc libm), so the
// device kernels see exactly the covariance values, search template and
// clusterizer buckets the reference would use.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace hpgl_b200 {

enum Kind { KIND_OK = 0, KIND_SK = 1, KIND_LVM = 2, KIND_IK = 3, KIND_MEDIAN_IK = 4, KIND_COK1 = 5, KIND_COK2 = 6 };
inline bool kind_is_cokriging(int k) { return k == KIND_COK1 || k == KIND_COK2; }
// kinds with a continuous property (values in, values out)
inline bool kind_is_cont(int k) { return k <= KIND_LVM || kind_is_cokriging(k); }

struct KrigingParams {
    int cov_type;
    double ranges[3];
    double angles[3];
    double sill;
    double nugget;
    int radii[3];
    int max_neighbours;
    double marginal_prob;
};

// Variogram model of cov_model_t (cov_model.h:79-182).
struct CovModel {
    int type;
    double sill, nugget, range0;
    double t[9];  // scale * ((Rx * Ry) * Rz), cov_model.h:16-61
    explicit CovModel(const KrigingParams &p);
    // C(v) for an offset v of grid steps (cov_model.h:63-77, 131-181).
    double operator()(double vx, double vy, double vz) const;
};

// Search template entry: the grid offset and the two forms the device search
// needs — the x word offset / bit shift inside the padded informed-bit rows,
// and the linear node-index delta.
struct TemplateEntry {
    int dx, dy, dz;
    int delta;
};

struct Plan {
    int kind = 0;
    int nx = 0, ny = 0, nz = 0;
    long long size = 0;
    int nmax = 0;            // max_neighbours
    bool truncated = false;  // covariance returns 0 outside +-radii (SK, LVM, IK, median IK)
    bool clusterizer = true; // the search may take the clusterizer path (not for cokriging)
    int radii[3] = {0, 0, 0};

    // sorted search template (covariance_field.h:62-106)
    std::vector<TemplateEntry> tmpl;
    int ext[3] = {0, 0, 0};  // largest |offset| of the template per axis

    // covariance table over +-B, C(v) = table[((vz+Bz)*(2By+1) + vy+By)*(2Bx+1) + vx+Bx];
    // entries with |v| > trunc on an axis read as 0.
    int B[3] = {0, 0, 0};
    int trunc[3] = {0, 0, 0};
    std::vector<double> table;
    double c0 = 0;  // C(0)

    // clusterizer (clusterizer.cpp:52-184)
    double cl_r[3] = {0, 0, 0};
    int mx = 0, my = 0, mz = 0;
    long long limit = 0;
    std::vector<int> bucket_start;        // CSR over mx*my*mz buckets
    std::vector<int> bucket_nodes;
    std::vector<uint8_t> bucket_clean;    // no exceeded bucket in the 3x3x3 neighbourhood
    bool any_clean = false;
    int max_candidates = 0;               // largest candidate count of a clean neighbourhood
    long long informed = 0;               // informed nodes of the mask

    // padded informed-bit rows for the template search
    int px = 0;      // x padding in cells, a multiple of 32
    int nseg = 0;    // 32-cell segments per row
    int wpr = 0;     // 32-bit words per padded row

};



// Validates parameters (throws std::invalid_argument / std::domain_error).
void validate_params(const KrigingParams &p, int kind);

// Builds the plan of one kind/params over the informed `mask` (size nx*ny*nz).
// sequential: the covariance of sequential simulation (truncated at the radii
// for every kind, precalculated_covariances_t in sequential_simulation.h:67)
// and the template search alone (neighbour_lookup_t, no clusterizer).
void build_plan(Plan &plan, int kind, int nx, int ny, int nz, const KrigingParams &p, const uint8_t *mask,
                int threads, bool sequential = false);

// C(v) of `p`'s model over the box +-B, laid out like Plan::table.
void fill_cov_table(std::vector<double> &table, const int B[3], const KrigingParams &p, int threads);

// True when two categories' parameters give identical searches and systems.
bool same_system(const KrigingParams &a, const KrigingParams &b);

// calc_mean (calc_mean.cpp:6-30).
double informed_mean(const float *values, const uint8_t *mask, long long size);

int host_threads();
void set_host_threads(int n);

}  // namespace hpgl_b200
