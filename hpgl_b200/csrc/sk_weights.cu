// Simple-kriging weights of one point from explicit neighbour coordinates
// (the reference's hpgl_simple_kriging_weights, api.cpp:292-342, over
// simple_kriging_weights, simple_kriging.cpp:15-35, and
// sk_kriging_weights_3, my_kriging_weights.h:26-129).
//
// One warp builds the covariance system of the n neighbours in global
// scratch (column-major, leading dimension n; n is the caller's and may be
// large), factors it with the reference DPOTRF 'U' operation order (the
// unblocked DPOTF2 that LAPACK runs for n <= 64; above 64 LAPACK switches to
// its blocked variant and results agree to rounding) and solves with the
// DPOTRS order.  The covariance of continuous coordinates is
// evaluated on the device (transform and norm in the reference's expression
// order without fused multiply-adds; exp/pow from CUDA's libm), so weights
// agree with the reference to rounding.
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/hpgl.h"
#include "engine.h"

namespace hpgl_b200 {

// Largest system the entry point accepts (one warp factors it).
constexpr int SK_WEIGHTS_MAX = 1024;

struct WeightsScratchLayout {
    // doubles: coords 3n | center 3 | A n*n | b n | x n ; then an int status
    static constexpr size_t doubles(int n) { return (size_t)3 * n + 3 + (size_t)n * n + 2 * (size_t)n; }
    static constexpr size_t bytes(int n) { return doubles(n) * sizeof(double) + 2 * sizeof(int); }
};

struct CovDev {
    int type;
    double sill, nugget, r0;
    double t[9];
};

// cov_model.h:63-77, 144-181, without fused multiply-adds.
__device__ double cov_dev(const CovDev &c, double v0, double v1, double v2) {
    const double v[3] = {v0, v1, v2};
    double acc = 0.0;
    for (int i = 0; i < 3; ++i) {
        double d = 0.0;
        for (int j = 0; j < 3; ++j) d = __dadd_rn(d, __dmul_rn(v[j], c.t[3 * i + j]));
        acc = __dadd_rn(acc, __dmul_rn(d, d));
    }
    const double h = __dsqrt_rn(acc);
    const double s = __dsub_rn(c.sill, c.nugget);
    if (h < 0.0001) return s;
    if (c.type == 2) {
        const double q = __ddiv_rn(h, c.r0);
        return __dmul_rn(s, exp(__dmul_rn(-3.0, __dmul_rn(q, q))));
    }
    if (c.type == 1) return __dmul_rn(s, exp(__ddiv_rn(__dmul_rn(-3.0, h), c.r0)));
    if (h > c.r0) return 0.0;
    const double q = __ddiv_rn(h, c.r0);
    const double a = __dsub_rn(1.0, __ddiv_rn(__dmul_rn(1.5, h), c.r0));
    return __dmul_rn(s, __dadd_rn(a, __dmul_rn(0.5, pow(q, 3.0))));
}

// Scratch layout as WeightsScratchLayout; coords and center filled by the
// caller (host copy), weights read back from x.
__global__ void k_sk_weights(CovDev cov, int n, double *scratch) {
    const int lane = threadIdx.x & 31;
    double *xyz = scratch;
    double *ctr = xyz + 3 * (size_t)n;
    double *A = ctr + 3;
    double *b = A + (size_t)n * n;
    double *x = b + n;
    int *status = (int *)(x + n);
    // A(r,c) = C(p_r - p_c), r <= c; b_r = C(p_r - center).
    for (int c = 0; c < n; ++c)
        for (int r = lane; r <= c; r += 32)
            A[r + (size_t)c * n] = cov_dev(cov, __dsub_rn(xyz[3 * r], xyz[3 * c]), __dsub_rn(xyz[3 * r + 1], xyz[3 * c + 1]),
                                           __dsub_rn(xyz[3 * r + 2], xyz[3 * c + 2]));
    for (int r = lane; r < n; r += 32)
        b[r] = cov_dev(cov, __dsub_rn(xyz[3 * r], ctr[0]), __dsub_rn(xyz[3 * r + 1], ctr[1]),
                       __dsub_rn(xyz[3 * r + 2], ctr[2]));
    __syncwarp();
    // DPOTF2 'U'
    int info = 0;
    for (int j = 0; j < n && !info; ++j) {
        double ajj = 0.0;
        for (int k = j + lane; k < n; k += 32) {
            double t = 0.0;
            for (int i = 0; i < j; ++i) t = __dadd_rn(t, __dmul_rn(A[i + (size_t)k * n], A[i + (size_t)j * n]));
            if (k == j) ajj = __dsub_rn(A[j + (size_t)j * n], t);
            else if (j > 0) A[j + (size_t)k * n] = __dadd_rn(A[j + (size_t)k * n], -t);
        }
        ajj = __shfl_sync(0xffffffffu, ajj, 0);
        __syncwarp();
        if (!(ajj > 0.0)) {
            if (lane == 0) A[j + (size_t)j * n] = ajj;
            info = j + 1;
            break;
        }
        ajj = __dsqrt_rn(ajj);
        const double rinv = __ddiv_rn(1.0, ajj);
        if (lane == 0) A[j + (size_t)j * n] = ajj;
        for (int k = j + 1 + lane; k < n; k += 32) A[j + (size_t)k * n] = __dmul_rn(rinv, A[j + (size_t)k * n]);
        __syncwarp();
    }
    // DPOTRS 'U' (sequential: one lane, the reference's loop order)
    if (lane == 0) {
        for (int i = 0; i < n; ++i) x[i] = b[i];
        for (int i = 0; i < n; ++i) {
            double t = x[i];
            for (int k = 0; k < i; ++k) t = __dsub_rn(t, __dmul_rn(A[k + (size_t)i * n], x[k]));
            x[i] = __ddiv_rn(t, A[i + (size_t)i * n]);
        }
        for (int k = n - 1; k >= 0; --k) {
            if (x[k] != 0.0) {
                x[k] = __ddiv_rn(x[k], A[k + (size_t)k * n]);
                for (int i = 0; i < k; ++i) x[i] = __dsub_rn(x[i], __dmul_rn(x[k], A[i + (size_t)k * n]));
            }
        }
        status[0] = info;
    }
}

static CovDev make_cov(const hpgl_cov_params_t *p) {
    KrigingParams kp;
    memset(&kp, 0, sizeof(kp));
    kp.cov_type = p->m_covariance_type;
    for (int i = 0; i < 3; ++i) {
        kp.ranges[i] = p->m_ranges[i];
        kp.angles[i] = p->m_angles[i];
        kp.radii[i] = 1;
    }
    kp.sill = p->m_sill;
    kp.nugget = p->m_nugget;
    kp.max_neighbours = 1;
    if (kp.cov_type < 0 || kp.cov_type > 2) throw HpglError{HPGL_E_INVALID, "covariance type must be 0, 1 or 2"};
    for (int i = 0; i < 3; ++i)
        if (kp.ranges[i] == 0) throw HpglError{HPGL_E_INVALID, "All covariance ranges should be non-zero"};
    CovModel m(kp);
    CovDev c;
    c.type = m.type;
    c.sill = m.sill;
    c.nugget = m.nugget;
    c.r0 = m.range0;
    for (int i = 0; i < 9; ++i) c.t[i] = m.t[i];
    return c;
}

#define WCHECK(expr)                                                                             \
    do {                                                                                         \
        cudaError_t e__ = (expr);                                                                \
        if (e__ != cudaSuccess)                                                                  \
            throw HpglError{HPGL_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e__)}; \
    } while (0)

static void check_inputs(const float *c, const float *x, const float *y, const float *z, int n,
                         const hpgl_cov_params_t *p, const float *w) {
    if (!c || !p || !w || (n > 0 && (!x || !y || !z))) throw HpglError{HPGL_E_INVALID, "null argument"};
    if (n < 0) throw HpglError{HPGL_E_INVALID, "negative neighbour count"};
}

// Host side shared by both entry points: stage the coordinates into
// `scratch` (device), run the kernel, read back status and weights.
static void weights_on_device(double *scratch, const float *center, const float *xs, const float *ys,
                              const float *zs, int n, const CovDev &cov, float *weights) {
    std::vector<double> h(3 * (size_t)n + 3);
    for (int i = 0; i < n; ++i) {
        h[3 * i] = xs[i];
        h[3 * i + 1] = ys[i];
        h[3 * i + 2] = zs[i];
    }
    for (int i = 0; i < 3; ++i) h[3 * (size_t)n + i] = center[i];
    WCHECK(cudaMemcpy(scratch, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    k_sk_weights<<<1, 32>>>(cov, n, scratch);
    WCHECK(cudaGetLastError());
    std::vector<double> x(n);
    int status = 0;
    double *dx = scratch + 3 * (size_t)n + 3 + (size_t)n * n + n;
    if (n > 0) WCHECK(cudaMemcpy(x.data(), dx, n * sizeof(double), cudaMemcpyDeviceToHost));
    WCHECK(cudaMemcpy(&status, dx + n, sizeof(int), cudaMemcpyDeviceToHost));
    // sk_kriging_weights_3 fails on a non-positive pivot; the reference's
    // wrapper then reads past its emptied weight vector (api.cpp:337-340).
    if (status != 0) throw HpglError{HPGL_E_INVALID, "kriging system is not positive definite"};
    for (int i = 0; i < n; ++i) weights[i] = (float)x[i];
}

static std::mutex g_weights_mutex;

void sk_weights_alloc(const float *center, const float *xs, const float *ys, const float *zs, int n,
                      const hpgl_cov_params_t *p, float *weights) {
    check_inputs(center, xs, ys, zs, n, p, weights);
    if (n > SK_WEIGHTS_MAX)
        throw HpglError{HPGL_E_UNSUPPORTED, "neighbours_count above " + std::to_string(SK_WEIGHTS_MAX)};
    const CovDev cov = make_cov(p);
    if (n == 0) return;
    std::lock_guard<std::mutex> lock(g_weights_mutex);
    double *scratch = nullptr;
    WCHECK(cudaMalloc(&scratch, WeightsScratchLayout::bytes(n)));
    try {
        weights_on_device(scratch, center, xs, ys, zs, n, cov, weights);
    } catch (...) {
        cudaFree(scratch);
        throw;
    }
    WCHECK(cudaFree(scratch));
}

// ---- the same kernel without any device allocation -------------------------
//
// hpgl_b200_simple_kriging_weights_static (include/hpgl.h) serves callers that
// must not allocate device memory: cudaMalloc/cudaFree synchronise the whole
// device (stalling the caller's other streams), and a host application that
// has reserved the GPU's memory for its own pool leaves nothing to allocate.
// Its scratch is this file-scope array: every GPU that loads the library
// holds it until the process exits.  Every call shares it and leaves the last
// call's contents behind; k_sk_weights writes each word of its layout before
// reading it (coordinates by the host copy, then A, b, x and the status word
// by the kernel), so nothing needs clearing between calls.  Calls that
// overlapped on the GPU would race on the array; the static entry point's
// calls are serialised with each other by g_static_mutex (the allocating
// entry point has its own scratch and lock).  The copies and the kernel run
// on the calling thread's per-thread default stream, which does not wait for
// the caller's other (blocking) streams as the legacy stream 0 would.
constexpr int STATIC_WEIGHTS_MAX = HPGL_B200_STATIC_WEIGHTS_MAX;
constexpr size_t STATIC_WEIGHTS_BYTES = (WeightsScratchLayout::bytes(STATIC_WEIGHTS_MAX) + 255) / 256 * 256;
static __device__ __align__(256) unsigned char g_weights_scratch[STATIC_WEIGHTS_BYTES];

static std::mutex g_static_mutex;

// Device address of g_weights_scratch on the current device.  In host code
// the array's name is only a stand-in, never a device address.  The address
// is looked up on every call, with the calling device current: the lookup
// allocates nothing, and a context that was reset and re-created (which
// reloads the library's module, possibly elsewhere) is followed.  The first
// lookup on a device also loads the module there, so that first call should
// come before any stream capture.
static double *static_scratch() {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_weights_scratch);
    if (e != cudaSuccess || !ptr)
        throw HpglError{HPGL_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e)};
    return (double *)ptr;
}

void sk_weights_static(const float *center, const float *xs, const float *ys, const float *zs, int n,
                       const hpgl_cov_params_t *p, float *weights) {
    check_inputs(center, xs, ys, zs, n, p, weights);
    if (n > STATIC_WEIGHTS_MAX)
        throw HpglError{HPGL_E_CAPACITY, "neighbours_count above the static scratch limit of " +
                                             std::to_string(STATIC_WEIGHTS_MAX)};
    const CovDev cov = make_cov(p);
    if (n == 0) return;
    std::lock_guard<std::mutex> lock(g_static_mutex);
    double *scratch = static_scratch();
    const cudaStream_t s = cudaStreamPerThread;
    double coords[3 * STATIC_WEIGHTS_MAX + 3];
    for (int i = 0; i < n; ++i) {
        coords[3 * i] = xs[i];
        coords[3 * i + 1] = ys[i];
        coords[3 * i + 2] = zs[i];
    }
    for (int i = 0; i < 3; ++i) coords[3 * n + i] = center[i];
    WCHECK(cudaMemcpyAsync(scratch, coords, (3 * (size_t)n + 3) * sizeof(double), cudaMemcpyHostToDevice, s));
    k_sk_weights<<<1, 32, 0, s>>>(cov, n, scratch);
    WCHECK(cudaGetLastError());
    double x[STATIC_WEIGHTS_MAX + 1];
    const double *dx = scratch + 3 * (size_t)n + 3 + (size_t)n * n + n;
    int status = 0;
    WCHECK(cudaMemcpyAsync(x, dx, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    WCHECK(cudaMemcpyAsync(&status, dx + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    WCHECK(cudaStreamSynchronize(s));
    if (status != 0) throw HpglError{HPGL_E_INVALID, "kriging system is not positive definite"};
    for (int i = 0; i < n; ++i) weights[i] = (float)x[i];
}

}  // namespace hpgl_b200
