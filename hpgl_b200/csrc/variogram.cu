// Experimental variograms and layer stacking on the GPU (the reference's
// _cvariogram library: variograms.cpp, ellipsoid.cpp, stack_layers.h).
//
// Grid variograms (calc_variograms, variograms.cpp:335-417).  The reference
// walks every integer offset of the template's bounding window, keeps those in
// the tunnel, and for each adds (v1 - v2)^2 of every pair of informed cells
// at that offset to the lags whose window holds the offset's length.  Here:
//   k_cv_offsets   one thread per window offset: tunnel test and lag range in
//                  the reference's double arithmetic (no fused multiply-add);
//                  the host keeps the offsets with a non-empty range;
//   k_cv_flags / k_cv_emit   the informed cells as a compact list;
//   k_cv_pairs     one block per (offset, slice of the cell list): each thread
//                  accumulates its pairs' squared differences in double-double
//                  and counts them, the block combines in a fixed order;
//   k_cv_offset_sums, k_cv_lag_sums   fixed-order sums over slices, then over
//                  the offsets of each lag.
// The per-lag sums are exact to about 2^-100 relative and independent of the
// launch shape (the reference's sequential double sum differs from the exact
// sum in its last bits); the pair counts are exact.
//
// Point-set variograms (calc_variograms_from_point_set, :419-503): every
// ordered pair (a point with itself included); threads own points a, the
// block stages points b in shared memory; a warp aggregates its lanes' pairs
// per lag in lane order into per-warp accumulators in shared memory.
//
// Layer stacking (stack_layers.h:5-63): one thread per map column, layers in
// order, the reference's float/double mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cvariogram.h"
#include "../../include/hpgl.h"
#include "engine.h"
#include "textio.h"
#include "variogram.h"

namespace hpgl_b200 {

#define CV_CHECK(expr)                                                                               \
    do {                                                                                             \
        cudaError_t e__ = (expr);                                                                    \
        if (e__ != cudaSuccess)                                                                      \
            throw HpglError{HPGL_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e__)};     \
    } while (0)

namespace {

constexpr unsigned FULL_MASK = 0xffffffffu;
constexpr int NT = 256;

// Template values the kernels use.
struct CvT {
    double d1[3], d2[3], d3[3];
    double R2, R3, tol, width, sep, first;
    double R2m, R3m;  // quick-reject bounds: |ss2| above R2m means s2 > 1 after rounding
    int lags;
};

CvT cv_t(const variogram_search_template_t &t, int lags) {
    CvT c;
    for (int i = 0; i < 3; ++i) {
        c.d1[i] = t.m_ellipsoid.m_direction1.m_data[i];
        c.d2[i] = t.m_ellipsoid.m_direction2.m_data[i];
        c.d3[i] = t.m_ellipsoid.m_direction3.m_data[i];
    }
    c.R2 = t.m_ellipsoid.m_R2;
    c.R3 = t.m_ellipsoid.m_R3;
    c.tol = t.m_tol_distance;
    c.width = t.m_lag_width;
    c.sep = t.m_lag_separation;
    c.first = t.m_first_lag_distance;
    // |ss2| >= R2 (1 + 2^-20) makes the rounded quotient ss2 / R2 exceed 1,
    // so the tunnel test fails whatever s3 is
    c.R2m = c.R2 > 0 ? c.R2 * (1.0 + 1.0 / 1048576.0) : HUGE_VAL;
    c.R3m = c.R3 > 0 ? c.R3 * (1.0 + 1.0 / 1048576.0) : HUGE_VAL;
    c.lags = lags;
    return c;
}

// dot_product (variograms.cpp:9-17): 0.0 + v0 d0 + v1 d1 + v2 d2
__device__ __forceinline__ double dot3(const double *d, double x, double y, double z) {
    double r = __dadd_rn(0.0, __dmul_rn(x, d[0]));
    r = __dadd_rn(r, __dmul_rn(y, d[1]));
    return __dadd_rn(r, __dmul_rn(z, d[2]));
}

// is_in_tunnel (variograms.cpp:26-40).  Vectors far outside the tunnel's
// cross-section, or behind it (ss1 < 0 with a non-negative tolerance), fail
// before the divisions and the square root: the exact test would fail them
// too (dist > 1, or tol * dist >= 0 > ss1).
__device__ __forceinline__ bool in_tunnel(const CvT &T, double x, double y, double z) {
    const double ss1 = dot3(T.d1, x, y, z), ss2 = dot3(T.d2, x, y, z), ss3 = dot3(T.d3, x, y, z);
    if (fabs(ss2) > T.R2m || fabs(ss3) > T.R3m || (T.tol >= 0.0 && ss1 < 0.0)) return false;
    const double s2 = __ddiv_rn(ss2, T.R2), s3 = __ddiv_rn(ss3, T.R3);
    const double dist = __dsqrt_rn(__dadd_rn(__dmul_rn(s2, s2), __dmul_rn(s3, s3)));
    return dist <= 1.0 && __dmul_rn(T.tol, dist) <= ss1;
}

// calc_dist (variograms.cpp:279-287)
__device__ __forceinline__ double length3(double x, double y, double z) {
    double r = __dadd_rn(0.0, __dmul_rn(x, x));
    r = __dadd_rn(r, __dmul_rn(y, y));
    return __dsqrt_rn(__dadd_rn(r, __dmul_rn(z, z)));
}

// Double-double accumulation (Knuth's two-sum, then a fast renormalisation).
struct DD {
    double hi, lo;
};
__device__ __forceinline__ DD dd_add(DD a, double b_hi, double b_lo) {
    const double s = __dadd_rn(a.hi, b_hi);
    const double bb = __dsub_rn(s, a.hi);
    double err = __dadd_rn(__dsub_rn(a.hi, __dsub_rn(s, bb)), __dsub_rn(b_hi, bb));
    err = __dadd_rn(err, __dadd_rn(a.lo, b_lo));
    const double hi = __dadd_rn(s, err);
    return DD{hi, __dsub_rn(err, __dsub_rn(hi, s))};
}

// xor-tree over the warp (the same order on every run)
__device__ __forceinline__ void warp_reduce(DD &a, unsigned long long &n) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double h = __shfl_xor_sync(FULL_MASK, a.hi, o), l = __shfl_xor_sync(FULL_MASK, a.lo, o);
        const unsigned long long m = __shfl_xor_sync(FULL_MASK, n, o);
        // combine in lane order: the lower lane's value first
        const bool low = ((threadIdx.x & 31) & o) == 0;
        a = low ? dd_add(a, h, l) : dd_add(DD{h, l}, a.hi, a.lo);
        n += m;
    }
}

// block of NT threads: fixed-order combination of the warps' results on thread 0
__device__ __forceinline__ void block_reduce(DD &a, unsigned long long &n) {
    __shared__ double sh[NT / 32], sl[NT / 32];
    __shared__ unsigned long long sn[NT / 32];
    warp_reduce(a, n);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        sh[w] = a.hi;
        sl[w] = a.lo;
        sn[w] = n;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        a = DD{sh[0], sl[0]};
        n = sn[0];
        for (int i = 1; i < NT / 32; ++i) {
            a = dd_add(a, sh[i], sl[i]);
            n += sn[i];
        }
    }
    __syncthreads();
}

struct Partial {
    double hi, lo;
    unsigned long long n;
};

// lag range of an offset of length dist (update_lags, variograms.cpp:306-333)
__device__ __forceinline__ bool lag_range(const CvT &T, double dist, int &lo, int &hi) {
    const double half = __ddiv_rn(T.width, 2.0);
    const int lmin = (int)ceil(__ddiv_rn(__dsub_rn(__dsub_rn(dist, half), T.first), T.sep));
    if (lmin >= T.lags) return false;
    const int lmax = (int)floor(__ddiv_rn(__dsub_rn(__dadd_rn(dist, half), T.first), T.sep));
    if (lmax < 0) return false;
    lo = lmin < 0 ? 0 : lmin;
    hi = lmax >= T.lags ? T.lags - 1 : lmax;
    return true;
}

__global__ void k_cv_offsets(CvT T, int i0, int j0, int k0, int nj, int nk, long long total, int2 *range) {
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int c = (int)(idx % nk), b = (int)((idx / nk) % nj), a = (int)(idx / ((long long)nk * nj));
    const double x = i0 + a, y = j0 + b, z = k0 + c;
    int lo = -1, hi = -1;
    if (in_tunnel(T, x, y, z)) {
        if (!lag_range(T, length3(x, y, z), lo, hi)) lo = hi = -1;
    }
    range[idx] = make_int2(lo, hi);
}

struct Grid {
    const float *data;
    const unsigned char *mask;
    int nx, ny, nz;        // data shape (the cells walked)
    int mx, my, mz;        // mask shape (the bounds of the paired cell)
    int ds0, ds1, ds2;     // data strides (elements)
    int ms0, ms1, ms2;     // mask strides
};

// informed-cell flags per block of NT logical cells (x fastest)
__global__ void k_cv_flags(Grid G, long long total, long long *block_counts) {
    const long long i = blockIdx.x * (long long)NT + threadIdx.x;
    bool inf = false;
    if (i < total) {
        const int x = (int)(i % G.nx), y = (int)((i / G.nx) % G.ny), z = (int)(i / ((long long)G.nx * G.ny));
        inf = G.mask[(long long)x * G.ms0 + (long long)y * G.ms1 + (long long)z * G.ms2] != 0;
    }
    const int n = __syncthreads_count(inf);
    if (threadIdx.x == 0) block_counts[blockIdx.x] = n;
}

__global__ void __launch_bounds__(1024) k_cv_scan(long long *v, long long n, long long *total) {
    __shared__ long long ws[32];
    const long long per = (n + 1023) / 1024;
    const long long a = threadIdx.x * per, b = min(n, a + per);
    long long s = 0;
    for (long long i = a; i < b; ++i) s += v[i];
    // inclusive warp scan, then across warps
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    long long x = s;
    for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(FULL_MASK, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) ws[w] = x;
    __syncthreads();
    long long base = 0, tot = 0;
    for (int i = 0; i < 32; ++i) {
        if (i < w) base += ws[i];
        tot += ws[i];
    }
    long long r = base + x - s;
    for (long long i = a; i < b; ++i) {
        const long long c = v[i];
        v[i] = r;
        r += c;
    }
    if (threadIdx.x == 0) *total = tot;
}

__global__ void k_cv_emit(Grid G, long long total, const long long *block_base, int4 *cells) {
    __shared__ int wc[NT / 32];
    const long long i = blockIdx.x * (long long)NT + threadIdx.x;
    bool inf = false;
    int x = 0, y = 0, z = 0;
    if (i < total) {
        x = (int)(i % G.nx);
        y = (int)((i / G.nx) % G.ny);
        z = (int)(i / ((long long)G.nx * G.ny));
        inf = G.mask[(long long)x * G.ms0 + (long long)y * G.ms1 + (long long)z * G.ms2] != 0;
    }
    const unsigned b = __ballot_sync(FULL_MASK, inf);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) wc[w] = __popc(b);
    __syncthreads();
    int base = 0;
    for (int k = 0; k < w; ++k) base += wc[k];
    if (inf) {
        const long long pos = block_base[blockIdx.x] + base + __popc(b & ((1u << lane) - 1u));
        cells[pos] = make_int4(x, y, z, 0);
    }
}

// hash of (offset index, cell index) for percentToUse < 100
__device__ __forceinline__ unsigned mix2(unsigned long long a, unsigned long long b) {
    unsigned long long z = a * 0x9E3779B97F4A7C15ull ^ (b + 0x632BE59BD9B4E019ull);
    z ^= z >> 31;
    z *= 0xBF58476D1CE4E5B9ull;
    z ^= z >> 29;
    z *= 0x94D049BB133111EBull;
    z ^= z >> 32;
    return (unsigned)z;
}

struct Offset {
    int x, y, z;
    int lo, hi;
    long long index;  // position in the window walk (sampling hash)
};

__global__ void __launch_bounds__(NT) k_cv_pairs(Grid G, const Offset *offs, const int4 *cells, long long ncells,
                                                 int nchunks, long long chunk, int percent, Partial *part) {
    const long long o = blockIdx.x / nchunks;
    const int ch = (int)(blockIdx.x % nchunks);
    const Offset f = offs[o];
    const long long moff = (long long)f.x * G.ms0 + (long long)f.y * G.ms1 + (long long)f.z * G.ms2;
    const long long doff = (long long)f.x * G.ds0 + (long long)f.y * G.ds1 + (long long)f.z * G.ds2;
    DD acc{0.0, 0.0};
    unsigned long long n = 0;
    const long long c0 = ch * chunk, c1 = min(ncells, c0 + chunk);
    for (long long c = c0 + threadIdx.x; c < c1; c += NT) {
        const int4 q = cells[c];
        const int x = q.x + f.x, y = q.y + f.y, z = q.z + f.z;
        if (x < 0 || y < 0 || z < 0 || x >= G.mx || y >= G.my || z >= G.mz) continue;
        const long long mi = (long long)q.x * G.ms0 + (long long)q.y * G.ms1 + (long long)q.z * G.ms2;
        if (!G.mask[mi + moff]) continue;
        if (percent < 100 && (int)(mix2((unsigned long long)f.index, (unsigned long long)mi) % 100u) >= percent)
            continue;
        const long long di = (long long)q.x * G.ds0 + (long long)q.y * G.ds1 + (long long)q.z * G.ds2;
        const double d = __dsub_rn((double)G.data[di], (double)G.data[di + doff]);
        acc = dd_add(acc, __dmul_rn(d, d), 0.0);
        ++n;
    }
    block_reduce(acc, n);
    if (threadIdx.x == 0) part[blockIdx.x] = Partial{acc.hi, acc.lo, n};
}

// one warp per offset: its slices in order
__global__ void k_cv_offset_sums(const Partial *part, long long noff, int nchunks, Partial *sums) {
    const long long o = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (o >= noff) return;
    DD a{0.0, 0.0};
    unsigned long long n = 0;
    for (int c = lane; c < nchunks; c += 32) {
        const Partial p = part[o * nchunks + c];
        a = dd_add(a, p.hi, p.lo);
        n += p.n;
    }
    warp_reduce(a, n);
    if (lane == 0) sums[o] = Partial{a.hi, a.lo, n};
}

// one block per lag: the offsets whose lag range holds it
__global__ void __launch_bounds__(NT) k_cv_lag_sums(const Offset *offs, const Partial *sums, long long noff,
                                                    double *lag_sum, unsigned long long *lag_n) {
    const int lag = blockIdx.x;
    DD a{0.0, 0.0};
    unsigned long long n = 0;
    for (long long o = threadIdx.x; o < noff; o += NT) {
        if (offs[o].lo <= lag && lag <= offs[o].hi) {
            a = dd_add(a, sums[o].hi, sums[o].lo);
            n += sums[o].n;
        }
    }
    block_reduce(a, n);
    if (threadIdx.x == 0) {
        lag_sum[lag] = __dadd_rn(a.hi, a.lo);
        lag_n[lag] = n;
    }
}

// ---- point sets ----------------------------------------------------------

constexpr int PT_TILE = 256;

struct Points {
    const float *x, *y, *z, *v;
    int n;
};

// Threads own points a; points b come through shared memory in tiles of 256,
// blockIdx.y picks a share of the tiles.  Each warp keeps per-lag
// accumulators in shared memory (laid out after the staging tiles) and adds
// its lanes' pairs of a lag in lane order.
__global__ void __launch_bounds__(NT) k_cv_points(CvT T, Points P, const double *lag_start, const double *lag_end,
                                                  int tiles_per_y, Partial *part) {
    extern __shared__ __align__(16) unsigned char smem[];
    float *bx = reinterpret_cast<float *>(smem);
    float *by = bx + PT_TILE, *bz = by + PT_TILE, *bv = bz + PT_TILE;
    double *slot = reinterpret_cast<double *>(bv + PT_TILE);      // [NT] staged values
    double *acc_hi = slot + NT;                                    // [warps][lags]
    double *acc_lo = acc_hi + (NT / 32) * T.lags;
    unsigned long long *acc_n = reinterpret_cast<unsigned long long *>(acc_lo + (NT / 32) * T.lags);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < (NT / 32) * T.lags; i += NT) {
        acc_hi[i] = 0.0;
        acc_lo[i] = 0.0;
        acc_n[i] = 0;
    }
    const int a = blockIdx.x * NT + threadIdx.x;
    const bool has_a = a < P.n;
    const float ax = has_a ? P.x[a] : 0.f, ay = has_a ? P.y[a] : 0.f, az = has_a ? P.z[a] : 0.f,
                av = has_a ? P.v[a] : 0.f;
    const int ntiles = (P.n + PT_TILE - 1) / PT_TILE;
    const int t0 = blockIdx.y * tiles_per_y, t1 = min(ntiles, t0 + tiles_per_y);
    for (int t = t0; t < t1; ++t) {
        __syncthreads();
        const int bi = t * PT_TILE + threadIdx.x;
        if (threadIdx.x < PT_TILE && bi < P.n) {
            bx[threadIdx.x] = P.x[bi];
            by[threadIdx.x] = P.y[bi];
            bz[threadIdx.x] = P.z[bi];
            bv[threadIdx.x] = P.v[bi];
        }
        __syncthreads();
        const int nb = min(PT_TILE, P.n - t * PT_TILE);
        for (int j = 0; j < nb; ++j) {
            // vec = x_a - x_b in float, then double (variograms.cpp:441-444)
            const double vx = (double)__fsub_rn(ax, bx[j]), vy = (double)__fsub_rn(ay, by[j]),
                         vz = (double)__fsub_rn(az, bz[j]);
            int lo = 0, hi = -1;
            double var = 0.0;
            if (has_a && in_tunnel(T, vx, vy, vz)) {
                const double dist = length3(vx, vy, vz);
                const double dv = (double)__fsub_rn(av, bv[j]);
                var = __dmul_rn(dv, dv);
                // candidate lags from the centres, each confirmed with the
                // reference's comparisons start <= dist < end
                const double c = (dist - T.first) / T.sep;
                const double h = T.width / T.sep;
                lo = max(0, (int)floor(c - 0.5 * h) - 1);
                hi = min(T.lags - 1, (int)ceil(c + 0.5 * h) + 1);
                while (lo <= hi && !(lag_start[lo] <= dist && dist < lag_end[lo])) ++lo;
                while (hi >= lo && !(lag_start[hi] <= dist && dist < lag_end[hi])) --hi;
            }
            // lags lo..hi of this lane (contiguous: the windows' starts and
            // ends both increase with the lag)
            for (;;) {
                const bool want = lo <= hi;
                unsigned pending = __ballot_sync(FULL_MASK, want);
                if (!pending) break;
                slot[threadIdx.x] = var;
                __syncwarp();
                while (pending) {
                    const int leader = __ffs(pending) - 1;
                    const int l = __shfl_sync(FULL_MASK, lo, leader);
                    const unsigned grp = __ballot_sync(FULL_MASK, want && lo == l);
                    if (lane == leader) {
                        DD s{acc_hi[w * T.lags + l], acc_lo[w * T.lags + l]};
                        for (unsigned g = grp; g; g &= g - 1) s = dd_add(s, slot[w * 32 + __ffs(g) - 1], 0.0);
                        acc_hi[w * T.lags + l] = s.hi;
                        acc_lo[w * T.lags + l] = s.lo;
                        acc_n[w * T.lags + l] += (unsigned long long)__popc(grp);
                    }
                    pending &= ~grp;
                    __syncwarp();
                }
                if (want) ++lo;
            }
        }
    }
    __syncthreads();
    // the block's warps in order, per lag
    for (int l = threadIdx.x; l < T.lags; l += NT) {
        DD s{0.0, 0.0};
        unsigned long long n = 0;
        for (int k = 0; k < NT / 32; ++k) {
            s = dd_add(s, acc_hi[k * T.lags + l], acc_lo[k * T.lags + l]);
            n += acc_n[k * T.lags + l];
        }
        part[((long long)blockIdx.y * gridDim.x + blockIdx.x) * T.lags + l] = Partial{s.hi, s.lo, n};
    }
}

// one warp per lag: the blocks' partials, lanes strided, then the xor tree
__global__ void k_cv_points_sum(const Partial *part, long long nparts, int lags, double *lag_sum,
                                unsigned long long *lag_n) {
    const int l = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (l >= lags) return;
    DD s{0.0, 0.0};
    unsigned long long n = 0;
    for (long long p = lane; p < nparts; p += 32) {
        s = dd_add(s, part[p * lags + l].hi, part[p * lags + l].lo);
        n += part[p * lags + l].n;
    }
    warp_reduce(s, n);
    if (lane == 0) {
        lag_sum[l] = __dadd_rn(s.hi, s.lo);
        lag_n[l] = n;
    }
}

// ---- layer stacking --------------------------------------------------------

struct Layer {
    const float *data;
    int s0, s1;
};

__global__ void k_stack_layers(const Layer *layers, const int *markers, int nlayers, int nx, int ny, int nz,
                               float scalez, int blank, float *out, int r0, int r1, int r2) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nx * ny) return;
    const int i = idx % nx, j = idx / nx;
    double cum = 0.0;
    for (int l = 0; l < nlayers; ++l) {
        const float th = layers[l].data[layers[l].s0 * i + layers[l].s1 * j];
        const float step = __fdiv_rn(th, scalez);
        if (th > 0) {
            const float old_k = __double2float_rn(cum);
            cum = __dadd_rn(cum, (double)step);
            const float new_k = __double2float_rn(cum);
            int k_next = (int)floorf(new_k) + 1;
            if (k_next > nz) k_next = nz;
            for (int k = (int)ceilf(old_k); k < k_next; ++k)
                if (k >= 0) out[(long long)r0 * i + (long long)r1 * j + (long long)r2 * k] = (float)markers[l];
        } else {
            const int k_start = (int)ceil(__dadd_rn(cum, (double)step));
            for (int k = k_start; k < nz; ++k)
                if (k >= 0) out[(long long)r0 * i + (long long)r1 * j + (long long)r2 * k] = (float)blank;
            cum = __dadd_rn(cum, (double)step);
        }
    }
}

// ---- host ------------------------------------------------------------------

std::mutex g_cv_mutex;

// CUDA events around a call's kernels, and its wall time
struct CallTiming {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    TextIoTiming t;
    CallTiming() {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
    }
    ~CallTiming() {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }
    void done(long long units) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) t.ms_device = ms;
        t.ms_total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        t.tokens = units;
        set_last_io_timing(t);
    }
};

cudaStream_t cv_stream() {
    static cudaStream_t s = nullptr;
    if (!s) {
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e == cudaSuccess && n == 0) e = cudaErrorNoDevice;
        if (e != cudaSuccess)
            throw HpglError{HPGL_E_CUDA, std::string("no CUDA device available: ") + cudaGetErrorString(e)};
        CV_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    }
    return s;
}

// device allocations freed at scope exit
struct DevMem {
    std::vector<void *> p;
    template <typename T>
    T *alloc(size_t n) {
        void *q = nullptr;
        CV_CHECK(cudaMalloc(&q, std::max<size_t>(n * sizeof(T), 16)));
        p.push_back(q);
        return static_cast<T *>(q);
    }
    ~DevMem() {
        for (void *q : p) cudaFree(q);
    }
};

// elements spanned by a strided 3-D array (non-negative strides)
long long span(const int *shape, const int *strides) {
    long long s = 1;
    for (int i = 0; i < 3; ++i) {
        if (shape[i] <= 0) return 0;
        if (strides[i] < 0) throw HpglError{HPGL_E_UNSUPPORTED, "negative strides are not supported"};
        s += (long long)strides[i] * (shape[i] - 1);
    }
    return s;
}

void window_of(const variogram_search_template_t &t, double w[6]) {
    // calc_search_template_window (variograms.cpp:85-130), same operation order
    double mini = 1e10, minj = 1e10, mink = 1e10, maxi = -1e10, maxj = -1e10, maxk = -1e10;
    const ellipsoid_t &e = t.m_ellipsoid;
    for (int i = 0; i < 2; ++i)
        for (int j = -1; j < 3; j += 2)
            for (int k = -1; k < 3; k += 2) {
                double V[3];
                for (int c = 0; c < 3; ++c) {
                    double di = e.m_direction1.m_data[c] * t.m_lag_separation;
                    di = di * t.m_num_lags;
                    di = di * i;
                    double dj = e.m_direction2.m_data[c] * e.m_R2;
                    dj = dj * j;
                    double dk = e.m_direction3.m_data[c] * e.m_R3;
                    dk = dk * k;
                    V[c] = di + dj;
                    V[c] = V[c] + dk;
                }
                if (V[0] < mini) mini = V[0];
                if (V[0] > maxi) maxi = V[0];
                if (V[1] < minj) minj = V[1];
                if (V[1] > maxj) maxj = V[1];
                if (V[2] < mink) mink = V[2];
                if (V[2] > maxk) maxk = V[2];
            }
    w[0] = mini;
    w[1] = minj;
    w[2] = mink;
    w[3] = maxi;
    w[4] = maxj;
    w[5] = maxk;
}

}  // namespace

void cv_fill_ellipsoid(ellipsoid_t *ell, double azimuth, double dip, double rotation) {
    // ellipsoid.cpp:40-72: M = (A B) C with the reference's value of pi
    const double coef = 3.14159265358 / 180.0;
    const double ra = azimuth * coef, rd = dip * coef, rr = rotation * coef;
    const double A[9] = {std::cos(ra), -std::sin(ra), 0, std::sin(ra), std::cos(ra), 0, 0, 0, 1};
    const double B[9] = {std::cos(rd), 0, -std::sin(rd), 0, 1, 0, std::sin(rd), 0, std::cos(rd)};
    const double C[9] = {1, 0, 0, 0, std::cos(rr), -std::sin(rr), 0, std::sin(rr), std::cos(rr)};
    double M[9], N[9];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += A[r * 3 + k] * B[k * 3 + c];
            M[r * 3 + c] = s;
        }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += M[r * 3 + k] * C[k * 3 + c];
            N[r * 3 + c] = s;
        }
    vector_t *dst[3] = {&ell->m_direction1, &ell->m_direction2, &ell->m_direction3};
    for (int col = 0; col < 3; ++col)
        for (int i = 0; i < 3; ++i) dst[col]->m_data[i] = N[i * 3 + col];
}

void cv_grid(const variogram_search_template_t &t, const hard_data_t &hd, int result_length, int percent,
             double *sums, unsigned long long *counts) {
    const int lags = std::min(t.m_num_lags, result_length);
    if (lags <= 0) return;
    if (!(t.m_lag_separation > 0)) throw HpglError{HPGL_E_INVALID, "the lag separation must be positive"};
    for (int l = 0; l < lags; ++l) {
        sums[l] = 0.0;
        counts[l] = 0;
    }
    if (!hd.m_data || !hd.m_mask) throw HpglError{HPGL_E_INVALID, "data or mask is null"};
    std::lock_guard<std::mutex> lock(g_cv_mutex);
    cudaStream_t s = cv_stream();
    DevMem M;
    CallTiming timing;
    double w[6];
    window_of(t, w);
    // loop bounds of the reference: int i2 = (int)min; i2 <= max
    const int i0 = (int)w[0], j0 = (int)w[1], k0 = (int)w[2];
    auto count = [](int from, double to) { return to < from ? 0 : (int)std::floor(to - from) + 1; };
    const int ni = count(i0, w[3]), nj = count(j0, w[4]), nk = count(k0, w[5]);
    const long long nwin = (long long)ni * nj * nk;
    const long long ncell_all = (long long)hd.m_data_shape[0] * hd.m_data_shape[1] * hd.m_data_shape[2];
    if (nwin <= 0 || ncell_all <= 0) return;
    const CvT T = cv_t(t, lags);
    // offsets in the tunnel with a non-empty lag range, in the walk's order
    int2 *d_range = M.alloc<int2>((size_t)nwin);
    k_cv_offsets<<<(unsigned)((nwin + NT - 1) / NT), NT, 0, s>>>(T, i0, j0, k0, nj, nk, nwin, d_range);
    std::vector<int2> range((size_t)nwin);
    CV_CHECK(cudaMemcpyAsync(range.data(), d_range, (size_t)nwin * sizeof(int2), cudaMemcpyDeviceToHost, s));
    CV_CHECK(cudaStreamSynchronize(s));
    std::vector<Offset> offs;
    for (long long idx = 0; idx < nwin; ++idx) {
        if (range[idx].x < 0) continue;
        const int c = (int)(idx % nk), b = (int)((idx / nk) % nj), a = (int)(idx / ((long long)nk * nj));
        offs.push_back(Offset{i0 + a, j0 + b, k0 + c, range[idx].x, range[idx].y, idx});
    }
    if (offs.empty()) return;
    // data and mask on the device
    const long long dspan = span(hd.m_data_shape, hd.m_data_strides), mspan = span(hd.m_mask_shape, hd.m_mask_strides);
    float *d_data = M.alloc<float>((size_t)dspan);
    unsigned char *d_mask = M.alloc<unsigned char>((size_t)mspan);
    CV_CHECK(cudaMemcpyAsync(d_data, hd.m_data, (size_t)dspan * 4, cudaMemcpyHostToDevice, s));
    CV_CHECK(cudaMemcpyAsync(d_mask, hd.m_mask, (size_t)mspan, cudaMemcpyHostToDevice, s));
    Grid G{d_data, d_mask, hd.m_data_shape[0], hd.m_data_shape[1], hd.m_data_shape[2], hd.m_mask_shape[0],
           hd.m_mask_shape[1], hd.m_mask_shape[2], hd.m_data_strides[0], hd.m_data_strides[1],
           hd.m_data_strides[2], hd.m_mask_strides[0], hd.m_mask_strides[1], hd.m_mask_strides[2]};
    // the walked cells must lie in the mask too (the reference reads both at
    // the same coordinates)
    for (int i = 0; i < 3; ++i)
        if (hd.m_data_shape[i] > hd.m_mask_shape[i])
            throw HpglError{HPGL_E_INVALID, "the mask is smaller than the data"};
    // informed cells
    const long long nb = (ncell_all + NT - 1) / NT;
    long long *d_bc = M.alloc<long long>((size_t)nb);
    long long *d_tot = M.alloc<long long>(1);
    k_cv_flags<<<(unsigned)nb, NT, 0, s>>>(G, ncell_all, d_bc);
    k_cv_scan<<<1, 1024, 0, s>>>(d_bc, nb, d_tot);
    long long ncells = 0;
    CV_CHECK(cudaMemcpyAsync(&ncells, d_tot, sizeof(long long), cudaMemcpyDeviceToHost, s));
    CV_CHECK(cudaStreamSynchronize(s));
    if (ncells == 0) return;
    int4 *d_cells = M.alloc<int4>((size_t)ncells);
    k_cv_emit<<<(unsigned)nb, NT, 0, s>>>(G, ncell_all, d_bc, d_cells);
    // (offset, slice) blocks: enough blocks to fill the GPU, slices of whole
    // thread rows
    const long long noff = (long long)offs.size();
    const long long want_blocks = 148LL * 16;
    long long nchunks = std::max<long long>(1, (want_blocks + noff - 1) / noff);
    nchunks = std::min<long long>(nchunks, (ncells + NT - 1) / NT);
    const long long chunk = ((ncells + nchunks - 1) / nchunks + NT - 1) / NT * NT;
    nchunks = (ncells + chunk - 1) / chunk;
    Offset *d_offs = M.alloc<Offset>((size_t)noff);
    CV_CHECK(cudaMemcpyAsync(d_offs, offs.data(), (size_t)noff * sizeof(Offset), cudaMemcpyHostToDevice, s));
    Partial *d_part = M.alloc<Partial>((size_t)(noff * nchunks));
    Partial *d_osum = M.alloc<Partial>((size_t)noff);
    double *d_lsum = M.alloc<double>((size_t)lags);
    unsigned long long *d_ln = M.alloc<unsigned long long>((size_t)lags);
    const long long blocks = noff * nchunks;
    if (blocks > 0x7fffffffLL) throw HpglError{HPGL_E_CAPACITY, "too many offsets for one launch"};
    CV_CHECK(cudaEventRecord(timing.e0, s));
    k_cv_pairs<<<(unsigned)blocks, NT, 0, s>>>(G, d_offs, d_cells, ncells, (int)nchunks, chunk,
                                               std::max(0, percent), d_part);
    k_cv_offset_sums<<<(unsigned)((noff * 32 + NT - 1) / NT), NT, 0, s>>>(d_part, noff, (int)nchunks, d_osum);
    k_cv_lag_sums<<<lags, NT, 0, s>>>(d_offs, d_osum, noff, d_lsum, d_ln);
    CV_CHECK(cudaEventRecord(timing.e1, s));
    CV_CHECK(cudaMemcpyAsync(sums, d_lsum, (size_t)lags * sizeof(double), cudaMemcpyDeviceToHost, s));
    CV_CHECK(cudaMemcpyAsync(counts, d_ln, (size_t)lags * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    CV_CHECK(cudaStreamSynchronize(s));
    CV_CHECK(cudaGetLastError());
    timing.done(noff * ncells);
}

void cv_points(const variogram_search_template_t &t, const cont_point_set_t &ps, int result_length, double *sums,
               unsigned long long *counts) {
    const int lags = std::min(t.m_num_lags, result_length);
    if (lags <= 0) return;
    for (int l = 0; l < lags; ++l) {
        sums[l] = 0.0;
        counts[l] = 0;
    }
    if (!(t.m_lag_separation > 0)) throw HpglError{HPGL_E_INVALID, "the lag separation must be positive"};
    const int n = ps.size;
    if (n <= 0) return;
    if (!ps.xs || !ps.ys || !ps.zs || !ps.values) throw HpglError{HPGL_E_INVALID, "point arrays are null"};
    std::lock_guard<std::mutex> lock(g_cv_mutex);
    cudaStream_t s = cv_stream();
    DevMem M;
    CallTiming timing;
    // lag windows (init_lag_list, variograms.cpp:140-151)
    std::vector<double> st(lags), en(lags);
    for (int l = 0; l < lags; ++l) {
        const double d = l * t.m_lag_separation + t.m_first_lag_distance;
        st[l] = d - t.m_lag_width / 2;
        en[l] = d + t.m_lag_width / 2;
    }
    float *d_pts = M.alloc<float>((size_t)n * 4);
    CV_CHECK(cudaMemcpyAsync(d_pts, ps.xs, (size_t)n * 4, cudaMemcpyHostToDevice, s));
    CV_CHECK(cudaMemcpyAsync(d_pts + n, ps.ys, (size_t)n * 4, cudaMemcpyHostToDevice, s));
    CV_CHECK(cudaMemcpyAsync(d_pts + 2 * (size_t)n, ps.zs, (size_t)n * 4, cudaMemcpyHostToDevice, s));
    CV_CHECK(cudaMemcpyAsync(d_pts + 3 * (size_t)n, ps.values, (size_t)n * 4, cudaMemcpyHostToDevice, s));
    double *d_st = M.alloc<double>((size_t)lags), *d_en = M.alloc<double>((size_t)lags);
    CV_CHECK(cudaMemcpyAsync(d_st, st.data(), (size_t)lags * 8, cudaMemcpyHostToDevice, s));
    CV_CHECK(cudaMemcpyAsync(d_en, en.data(), (size_t)lags * 8, cudaMemcpyHostToDevice, s));
    const Points P{d_pts, d_pts + n, d_pts + 2 * (size_t)n, d_pts + 3 * (size_t)n, n};
    const int gx = (n + NT - 1) / NT;
    const int ntiles = (n + PT_TILE - 1) / PT_TILE;
    const int gy_want = std::max(1, std::min(ntiles, (148 * 8 + gx - 1) / gx));
    const int tiles_per_y = (ntiles + gy_want - 1) / gy_want;
    const int gy = (ntiles + tiles_per_y - 1) / tiles_per_y;
    const size_t smem = 4 * PT_TILE * sizeof(float) + NT * sizeof(double) + (size_t)(NT / 32) * lags * 24;
    if (smem > 200 * 1024) throw HpglError{HPGL_E_UNSUPPORTED, "too many lags for the point-set variogram"};
    CV_CHECK(cudaFuncSetAttribute(k_cv_points, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const CvT T = cv_t(t, lags);
    Partial *d_part = M.alloc<Partial>((size_t)gx * gy * lags);
    double *d_lsum = M.alloc<double>((size_t)lags);
    unsigned long long *d_ln = M.alloc<unsigned long long>((size_t)lags);
    CV_CHECK(cudaEventRecord(timing.e0, s));
    k_cv_points<<<dim3(gx, gy), NT, smem, s>>>(T, P, d_st, d_en, tiles_per_y, d_part);
    k_cv_points_sum<<<(lags * 32 + NT - 1) / NT, NT, 0, s>>>(d_part, (long long)gx * gy, lags, d_lsum, d_ln);
    CV_CHECK(cudaEventRecord(timing.e1, s));
    CV_CHECK(cudaMemcpyAsync(sums, d_lsum, (size_t)lags * 8, cudaMemcpyDeviceToHost, s));
    CV_CHECK(cudaMemcpyAsync(counts, d_ln, (size_t)lags * 8, cudaMemcpyDeviceToHost, s));
    CV_CHECK(cudaStreamSynchronize(s));
    CV_CHECK(cudaGetLastError());
    timing.done((long long)n * n);
}

void cv_stack_layers(const float_data_t *layers, const int *markers, int nlayers, int nz, float scalez, int blank,
                     float_data_t *result) {
    if (nlayers <= 0) return;
    if (!layers || !markers || !result || !result->m_data) throw HpglError{HPGL_E_INVALID, "null argument"};
    const int nx = layers[0].m_data_shape[0], ny = layers[0].m_data_shape[1];
    if (nx <= 0 || ny <= 0) return;
    // the reference keeps one running depth per layer-0 map index; every
    // layer must address the map the same way
    for (int l = 0; l < nlayers; ++l) {
        if (!layers[l].m_data) throw HpglError{HPGL_E_INVALID, "a layer is null"};
        if (layers[l].m_data_strides[0] != layers[0].m_data_strides[0] ||
            layers[l].m_data_strides[1] != layers[0].m_data_strides[1] || layers[l].m_data_shape[0] < nx ||
            layers[l].m_data_shape[1] < ny)
            throw HpglError{HPGL_E_UNSUPPORTED, "layers with different shapes or strides"};
    }
    const int s0 = layers[0].m_data_strides[0], s1 = layers[0].m_data_strides[1];
    {
        // distinct map indices inside the running-depth array (nx * ny)
        const long long a = (long long)s0 * (nx - 1) + (long long)s1 * (ny - 1);
        if (s0 < 0 || s1 < 0 || a >= (long long)nx * ny || (nx > 1 && ny > 1 && s0 == 0) || (ny > 1 && s1 == 0))
            throw HpglError{HPGL_E_UNSUPPORTED, "layer strides outside a contiguous map"};
    }
    std::lock_guard<std::mutex> lock(g_cv_mutex);
    cudaStream_t s = cv_stream();
    DevMem M;
    const long long lspan = span(layers[0].m_data_shape, layers[0].m_data_strides);
    std::vector<Layer> hl(nlayers);
    for (int l = 0; l < nlayers; ++l) {
        float *d = M.alloc<float>((size_t)lspan);
        CV_CHECK(cudaMemcpyAsync(d, layers[l].m_data, (size_t)lspan * 4, cudaMemcpyHostToDevice, s));
        hl[l] = Layer{d, s0, s1};
    }
    Layer *d_layers = M.alloc<Layer>((size_t)nlayers);
    int *d_markers = M.alloc<int>((size_t)nlayers);
    CV_CHECK(cudaMemcpyAsync(d_layers, hl.data(), (size_t)nlayers * sizeof(Layer), cudaMemcpyHostToDevice, s));
    CV_CHECK(cudaMemcpyAsync(d_markers, markers, (size_t)nlayers * 4, cudaMemcpyHostToDevice, s));
    const long long rspan = span(result->m_data_shape, result->m_data_strides);
    float *d_out = M.alloc<float>((size_t)rspan);
    CV_CHECK(cudaMemcpyAsync(d_out, result->m_data, (size_t)rspan * 4, cudaMemcpyHostToDevice, s));
    if (nz > result->m_data_shape[2]) throw HpglError{HPGL_E_INVALID, "nz exceeds the result's depth"};
    k_stack_layers<<<(nx * ny + NT - 1) / NT, NT, 0, s>>>(d_layers, d_markers, nlayers, nx, ny, nz, scalez, blank,
                                                         d_out, result->m_data_strides[0], result->m_data_strides[1],
                                                         result->m_data_strides[2]);
    CV_CHECK(cudaMemcpyAsync(result->m_data, d_out, (size_t)rspan * 4, cudaMemcpyDeviceToHost, s));
    CV_CHECK(cudaStreamSynchronize(s));
    CV_CHECK(cudaGetLastError());
}

}  // namespace hpgl_b200
