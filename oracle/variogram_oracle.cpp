// ORACLE — test infrastructure only.  Only tests/ and bench.py's CPU-baseline
// leg load this; the shipped library never links or calls it.
//
// CPU restatement of the reference's experimental variograms and layer
// stacking (src/geo_bsd/_cvariogram/):
//   fill_ellipsoid_directions        ellipsoid.cpp:40-72
//   is_in_tunnel                     variograms.cpp:26-40
//   calc_search_template_window      variograms.cpp:85-130
//   init_lag_list / calc_lag_areas   variograms.cpp:140-225
//   update_lags                      variograms.cpp:306-333
//   calc_variograms                  variograms.cpp:335-417
//   calc_variograms_from_point_set   variograms.cpp:419-503
//   stack_layers                     stack_layers.h:5-63
// in the reference's own loop order and arithmetic (double products and sums
// without fused multiply-adds).  Beside the reference's sequential per-lag
// sums it returns the exact sums (every term added into a fixed-point
// accumulator wide enough for any double, then rounded once), which is what
// the GPU's order-independent accumulation is compared with.  Parity of the
// restatement is pinned against the reference's sources compiled by
// oracle/build_ref.sh.
//
// percentToUse < 100: the reference keeps a pair when rand() % 100 <
// percentToUse, a draw from the process's C library generator; this
// restatement (like the GPU) keeps it when a hash of (offset index, cell
// index) taken modulo 100 is below percentToUse.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

struct vec3 {
    double v[3];
};
struct ellipsoid {
    vec3 d1, d2, d3;
    double R1, R2, R3;
};
struct templ_t {
    double lag_width, lag_separation, tol_distance;
    int num_lags;
    double first_lag_distance;
    ellipsoid ell;
};
struct hard_data {
    float *data;
    unsigned char *mask;
    int data_shape[3], data_strides[3], mask_shape[3], mask_strides[3];
};
struct point_set {
    float *xs, *ys, *zs, *values;
    int size;
};
struct float_data {
    float *data;
    int shape[3], strides[3];
};

double dot(const vec3 &a, const vec3 &b) {
    double r = 0.0;
    for (int i = 0; i < 3; ++i) r += a.v[i] * b.v[i];
    return r;
}

bool in_tunnel(const templ_t &t, const vec3 &v) {
    const double ss1 = dot(v, t.ell.d1), ss2 = dot(v, t.ell.d2), ss3 = dot(v, t.ell.d3);
    const double s2 = ss2 / t.ell.R2, s3 = ss3 / t.ell.R3;
    const double dist = std::sqrt(s2 * s2 + s3 * s3);
    return dist <= 1.0 && t.tol_distance * dist <= ss1;
}

void window(const templ_t &t, double w[6]) {
    double mini = 1e10, minj = 1e10, mink = 1e10, maxi = -1e10, maxj = -1e10, maxk = -1e10;
    for (int i = 0; i < 2; ++i)
        for (int j = -1; j < 3; j += 2)
            for (int k = -1; k < 3; k += 2) {
                vec3 DI, DJ, DK, V;
                for (int c = 0; c < 3; ++c) {
                    DI.v[c] = t.ell.d1.v[c] * t.lag_separation;
                    DI.v[c] = DI.v[c] * t.num_lags;
                    DI.v[c] = DI.v[c] * i;
                    DJ.v[c] = t.ell.d2.v[c] * t.ell.R2;
                    DJ.v[c] = DJ.v[c] * j;
                    DK.v[c] = t.ell.d3.v[c] * t.ell.R3;
                    DK.v[c] = DK.v[c] * k;
                    V.v[c] = DI.v[c] + DJ.v[c];
                    V.v[c] = V.v[c] + DK.v[c];
                }
                if (V.v[0] < mini) mini = V.v[0];
                if (V.v[0] > maxi) maxi = V.v[0];
                if (V.v[1] < minj) minj = V.v[1];
                if (V.v[1] > maxj) maxj = V.v[1];
                if (V.v[2] < mink) mink = V.v[2];
                if (V.v[2] > maxk) maxk = V.v[2];
            }
    w[0] = mini;
    w[1] = minj;
    w[2] = mink;
    w[3] = maxi;
    w[4] = maxj;
    w[5] = maxk;
}

// Exact sum of non-negative doubles: 2^-1074 .. 2^1152 in 64-bit limbs.
struct ExactSum {
    enum { LIMBS = 36 };
    uint64_t l[LIMBS];
    ExactSum() { memset(l, 0, sizeof l); }
    void add(double x) {
        if (!(x > 0.0)) return;  // terms are squares: 0 adds nothing
        int e;
        const double fr = std::frexp(x, &e);            // x = fr * 2^e, fr in [0.5, 1)
        const uint64_t m = (uint64_t)std::ldexp(fr, 53);  // x = m * 2^(e-53)
        int pos = e - 53 + 1074;                         // bit position of m's bit 0
        if (pos < 0) return;                             // not reached for doubles
        const int li = pos / 64, sh = pos % 64;
        unsigned __int128 acc = (unsigned __int128)m << sh;
        for (int k = li; k < LIMBS && acc; ++k) {
            acc += l[k];
            l[k] = (uint64_t)acc;
            acc >>= 64;
        }
    }
    void add(const ExactSum &o) {
        unsigned __int128 c = 0;
        for (int k = 0; k < LIMBS; ++k) {
            c += (unsigned __int128)l[k] + o.l[k];
            l[k] = (uint64_t)c;
            c >>= 64;
        }
    }
    // correctly rounded (nearest-even) double
    double value() const {
        int top = -1;
        for (int k = LIMBS - 1; k >= 0 && top < 0; --k)
            if (l[k]) top = k * 64 + 63 - __builtin_clzll(l[k]);
        if (top < 0) return 0.0;
        auto bit = [&](int p) { return p >= 0 ? (int)((l[p / 64] >> (p % 64)) & 1u) : 0; };
        // 53 bits from top down
        uint64_t m = 0;
        for (int p = top; p > top - 53; --p) m = (m << 1) | (uint64_t)bit(p);
        const int lowest = top - 52;
        bool round = bit(lowest - 1), sticky = false;
        for (int p = lowest - 2; p >= 0 && !sticky; --p) sticky = bit(p);
        if (round && (sticky || (m & 1))) ++m;
        return std::ldexp((double)m, lowest - 1074);
    }
};

uint32_t mix(uint64_t a, uint64_t b) {
    uint64_t z = a * 0x9E3779B97F4A7C15ull ^ (b + 0x632BE59BD9B4E019ull);
    z ^= z >> 31;
    z *= 0xBF58476D1CE4E5B9ull;
    z ^= z >> 29;
    z *= 0x94D049BB133111EBull;
    z ^= z >> 32;
    return (uint32_t)z;
}

}  // namespace

extern "C" {

void oracle_fill_ellipsoid_directions(double *d, double azimuth, double dip, double rotation) {
    const double coef = 3.14159265358 / 180.0;
    const double ra = azimuth * coef, rd = dip * coef, rr = rotation * coef;
    const double A[9] = {cos(ra), -sin(ra), 0, sin(ra), cos(ra), 0, 0, 0, 1};
    const double B[9] = {cos(rd), 0, -sin(rd), 0, 1, 0, sin(rd), 0, cos(rd)};
    const double C[9] = {1, 0, 0, 0, cos(rr), -sin(rr), 0, sin(rr), cos(rr)};
    double M[9], M2[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double s = 0.0;
            for (int i = 0; i < 3; ++i) s += A[r * 3 + i] * B[i * 3 + c];
            M[r * 3 + c] = s;
        }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double s = 0.0;
            for (int i = 0; i < 3; ++i) s += M[r * 3 + i] * C[i * 3 + c];
            M2[r * 3 + c] = s;
        }
    for (int col = 0; col < 3; ++col)
        for (int i = 0; i < 3; ++i) d[col * 3 + i] = M2[i * 3 + col];
}

void oracle_template_window(const templ_t *t, double *w) { window(*t, w); }

int oracle_in_tunnel(const templ_t *t, double x, double y, double z) {
    const vec3 v{{x, y, z}};
    return in_tunnel(*t, v) ? 1 : 0;
}

// calc_lag_areas: number of integer offsets of each lag's shell inside the
// tunnel (variograms.cpp:157-225)
long long oracle_lag_areas(const templ_t *t) {
    double w[6];
    window(*t, w);
    const int mini = (int)std::floor(w[0]), minj = (int)std::floor(w[1]), mink = (int)std::floor(w[2]);
    const int maxi = (int)std::ceil(w[3]), maxj = (int)std::ceil(w[4]), maxk = (int)std::ceil(w[5]);
    long long n = 0;
    for (int lag = 0; lag < t->num_lags; ++lag) {
        const double d = lag * t->lag_separation + t->first_lag_distance;
        const double start = d - t->lag_width / 2, end = d + t->lag_width / 2;
        for (int i = mini; i <= maxi; ++i)
            for (int j = minj; j <= maxj; ++j)
                for (int k = mink; k <= maxk; ++k) {
                    const vec3 v{{(double)i, (double)j, (double)k}};
                    const double dist = std::sqrt((double)(i * i + j * j + k * k));
                    if (in_tunnel(*t, v) && start <= dist && dist < end) ++n;
                }
    }
    return n;
}

// calc_variograms.  result: the reference's per-lag floats; seq_sums: its
// sequential double sums; exact_sums: the exact sums rounded once; counts.
void oracle_calc_variograms(const templ_t *t, const hard_data *data, float *result, double *seq_sums,
                            double *exact_sums, long long *counts, int result_length, int percent) {
    const int lag_count = t->num_lags <= result_length ? t->num_lags : result_length;
    std::vector<double> sum(lag_count, 0.0);
    std::vector<long long> cnt(lag_count, 0);
    std::vector<ExactSum> ex(lag_count);
    double w[6];
    window(*t, w);
    long long offset_index = 0;
    for (int i2 = (int)w[0]; i2 <= w[3]; ++i2)
        for (int j2 = (int)w[1]; j2 <= w[4]; ++j2)
            for (int k2 = (int)w[2]; k2 <= w[5]; ++k2) {
                const vec3 v{{(double)i2, (double)j2, (double)k2}};
                const int doffset = (int)(0 + (double)i2 * data->data_strides[0]);
                const int doff = (int)((double)doffset + (double)j2 * data->data_strides[1]);
                const int dof = (int)((double)doff + (double)k2 * data->data_strides[2]);
                const int mo0 = (int)(0 + (double)i2 * data->mask_strides[0]);
                const int mo1 = (int)((double)mo0 + (double)j2 * data->mask_strides[1]);
                const int moffset = (int)((double)mo1 + (double)k2 * data->mask_strides[2]);
                const long long oi = offset_index++;
                if (!in_tunnel(*t, v)) continue;
                const double dist = std::sqrt(((0.0 + v.v[0] * v.v[0]) + v.v[1] * v.v[1]) + v.v[2] * v.v[2]);
                int lmin = (int)std::ceil((dist - (t->lag_width / 2) - t->first_lag_distance) / t->lag_separation);
                int lmax = (int)std::floor((dist + (t->lag_width / 2) - t->first_lag_distance) / t->lag_separation);
                for (int z1 = 0; z1 < data->data_shape[2]; ++z1)
                    for (int y1 = 0; y1 < data->data_shape[1]; ++y1)
                        for (int x1 = 0; x1 < data->data_shape[0]; ++x1) {
                            const long long mi = (long long)x1 * data->mask_strides[0] +
                                                 (long long)y1 * data->mask_strides[1] +
                                                 (long long)z1 * data->mask_strides[2];
                            if (!data->mask[mi]) continue;
                            const int x = x1 + i2, y = y1 + j2, z = z1 + k2;
                            if (x < 0 || y < 0 || z < 0 || x >= data->mask_shape[0] || y >= data->mask_shape[1] ||
                                z >= data->mask_shape[2])
                                continue;
                            if (!data->mask[mi + moffset]) continue;
                            const long long di = (long long)x1 * data->data_strides[0] +
                                                 (long long)y1 * data->data_strides[1] +
                                                 (long long)z1 * data->data_strides[2];
                            if (percent < 100 && (int)(mix((uint64_t)oi, (uint64_t)mi) % 100u) >= percent) continue;
                            double var = (double)data->data[di] - (double)data->data[di + dof];
                            var = var * var;
                            if (lmin >= lag_count) continue;
                            if (lmax < 0) continue;
                            const int hi = lmax >= lag_count ? lag_count - 1 : lmax;
                            const int lo = lmin < 0 ? 0 : lmin;
                            for (int l = lo; l <= hi; ++l) {
                                sum[l] += var;
                                cnt[l] += 1;
                                ex[l].add(var);
                            }
                        }
            }
    for (int l = 0; l < lag_count; ++l) {
        result[l] = (float)(sum[l] / (double)cnt[l] / 2);
        if (seq_sums) seq_sums[l] = sum[l];
        if (exact_sums) exact_sums[l] = ex[l].value();
        if (counts) counts[l] = cnt[l];
    }
}

// calc_variograms_from_point_set (every ordered pair, a point with itself
// included).
void oracle_calc_variograms_points(const templ_t *t, const point_set *ps, float *result, double *seq_sums,
                                   double *exact_sums, long long *counts, int result_length) {
    const int lag_count = t->num_lags <= result_length ? t->num_lags : result_length;
    std::vector<double> sum(lag_count, 0.0), start(lag_count), end(lag_count);
    std::vector<long long> cnt(lag_count, 0);
    std::vector<ExactSum> ex(lag_count);
    for (int l = 0; l < lag_count; ++l) {
        const double d = l * t->lag_separation + t->first_lag_distance;
        start[l] = d - t->lag_width / 2;
        end[l] = d + t->lag_width / 2;
    }
    for (int a = 0; a < ps->size; ++a)
        for (int b = 0; b < ps->size; ++b) {
            const vec3 v{{(double)(ps->xs[a] - ps->xs[b]), (double)(ps->ys[a] - ps->ys[b]),
                          (double)(ps->zs[a] - ps->zs[b])}};
            if (!in_tunnel(*t, v)) continue;
            const double dist = std::sqrt(((0.0 + v.v[0] * v.v[0]) + v.v[1] * v.v[1]) + v.v[2] * v.v[2]);
            const double dv = (double)(ps->values[a] - ps->values[b]);
            const double var = dv * dv;
            for (int l = 0; l < lag_count; ++l)
                if (start[l] <= dist && dist < end[l]) {
                    sum[l] += var;
                    cnt[l] += 1;
                    ex[l].add(var);
                }
        }
    for (int l = 0; l < lag_count; ++l) {
        result[l] = (float)(sum[l] / (double)cnt[l] / 2);
        if (cnt[l] == 0) result[l] = 0;
        if (seq_sums) seq_sums[l] = sum[l];
        if (exact_sums) exact_sums[l] = ex[l].value();
        if (counts) counts[l] = cnt[l];
    }
}

// stack_layers (stack_layers.h:5-63).  Layer indices below 0 (a column
// whose cumulative thickness went negative) are skipped; the reference writes
// before the start of the result array there.
void oracle_stack_layers(const float_data *layers, const int *markers, int layers_count, int nz, float scalez,
                         int blank_value, float_data *result) {
    const int nx = layers[0].shape[0], ny = layers[0].shape[1];
    std::vector<double> cum((size_t)nx * ny, 0.0);
    for (int layer = 0; layer < layers_count; ++layer)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                const int mi = layers[layer].strides[0] * i + layers[layer].strides[1] * j;
                const float th = layers[layer].data[mi];
                if (th > 0) {
                    const float old_k = (float)cum[mi];
                    cum[mi] += th / scalez;
                    const float new_k = (float)cum[mi];
                    int k_next = (int)std::floor(new_k) + 1;
                    if (k_next > nz) k_next = nz;
                    for (int k = (int)std::ceil(old_k); k < k_next; ++k)
                        if (k >= 0)  // the reference writes before the array here
                            result->data[result->strides[0] * i + result->strides[1] * j + result->strides[2] * k] =
                            (float)markers[layer];
                } else {
                    const int k_start = (int)std::ceil(cum[mi] + (th / scalez));
                    for (int k = k_start; k < nz; ++k)
                        if (k >= 0)
                            result->data[result->strides[0] * i + result->strides[1] * j + result->strides[2] * k] =
                            (float)blank_value;
                    cum[mi] += th / scalez;
                }
            }
}
}
