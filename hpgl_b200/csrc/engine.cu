// Job execution on the GPU.  One CUDA stream, device buffers cached and grown
// across calls; every call is synchronous at the C ABI.
#include <algorithm>
#include <chrono>
#include <climits>
#include <functional>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>

#include "engine.h"
#include "kernels.cuh"

namespace hpgl_b200 {

#define CUDA_CHECK(expr)                                                                              \
    do {                                                                                              \
        cudaError_t e__ = (expr);                                                                     \
        if (e__ != cudaSuccess)                                                                       \
            throw HpglError{HPGL_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e__)};      \
    } while (0)

static int env_precision() {
    const char *e = getenv("HPGL_B200_PRECISION");
    if (e && (strcmp(e, "mixed") == 0 || strcmp(e, "1") == 0)) return HPGL_PRECISION_MIXED;
    return HPGL_PRECISION_FP64;
}
static int g_precision = env_precision();
int default_precision() { return g_precision; }
void set_default_precision(int p) { g_precision = p; }

template <typename T>
struct DBuf {
    T *p = nullptr;
    size_t cap = 0;
    void ensure(size_t n) {
        if (n == 0) n = 1;
        if (n <= cap) return;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        CUDA_CHECK(cudaMalloc(&p, n * sizeof(T)));
        cap = n;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

struct Counters {
    int n_untouched;
    int n_routed;
    int err;
    int pad;
    unsigned long long n_fp64;
};

struct PlanBuffers {
    DBuf<int4> tmpl;
    DBuf<double> table;
    DBuf<int> bucket_start, bucket_nodes;
    DBuf<uint8_t> bucket_clean;
    DBuf<uint32_t> bits;
    ~PlanBuffers() {
        tmpl.release();
        table.release();
        bucket_start.release();
        bucket_nodes.release();
        bucket_clean.release();
        bits.release();
    }
};

struct Context {
    cudaStream_t stream = nullptr;
    DBuf<float> values, mean, out_values, probs, pk;
    DBuf<uint8_t> codes, mask, out_codes, out_mask;
    DBuf<int8_t> status;
    DBuf<double> variance, weights, skey;
    DBuf<int> nb, nbcount, untouched, routed, sidx;
    DBuf<Counters> counters;
    DBuf<char> flush;
};

static std::mutex g_mutex;

static Context &ctx() {
    static Context *c = nullptr;
    if (!c) {
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e != cudaSuccess || n == 0)
            throw HpglError{HPGL_E_CUDA, std::string("no CUDA device available: ") + cudaGetErrorString(e)};
        auto *nc = new Context();
        CUDA_CHECK(cudaStreamCreateWithFlags(&nc->stream, cudaStreamNonBlocking));
        c = nc;
    }
    return *c;
}

static double ms_since(std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

// ---- job state -------------------------------------------------------------

struct Group {
    int k0, k1;
    Plan plan;
    std::unique_ptr<PlanBuffers> buf;
    DevPlan dp;
};

struct JobState {
    hpgl_b200_job_t job;
    int precision;
    long long size;
    int K;            // categories (IK), else 1
    bool per_category;
    int status_stride;
    std::vector<Group> groups;
    std::vector<float> pk;
    double sk_mean;
    int nmax_all;
};

static KrigingParams to_params(const hpgl_ik_params_t &p) {
    KrigingParams k;
    k.cov_type = p.m_covariance_type;
    for (int i = 0; i < 3; ++i) {
        k.ranges[i] = p.m_ranges[i];
        k.angles[i] = p.m_angles[i];
        k.radii[i] = p.m_radiuses[i];
    }
    k.sill = p.m_sill;
    k.nugget = p.m_nugget;
    k.max_neighbours = p.m_max_neighbours;
    k.marginal_prob = p.m_marginal_prob;
    return k;
}

static void invalid(const std::string &m) { throw HpglError{HPGL_E_INVALID, m}; }

static void prepare(JobState &S, const hpgl_b200_job_t &job) {
    S.job = job;
    if (job.kind < 0 || job.kind > 4) invalid("unknown kriging kind");
    if (job.nx <= 0 || job.ny <= 0 || job.nz <= 0) invalid("grid dimensions must be positive");
    S.size = (long long)job.nx * job.ny * job.nz;
    if (S.size > 2147483647LL) invalid("grid larger than 2^31-1 nodes (node indices are int, typedefs.h:112)");
    if (!job.mask) invalid("mask is null");
    if (!job.params || job.n_params < 1) invalid("params missing");
    const bool cont = job.kind <= KIND_LVM;
    if (cont && !job.values) invalid("values are null");
    if (!cont && !job.codes) invalid("codes are null");
    if (job.kind == KIND_LVM && !job.mean) invalid("mean cube is null");
    if (job.kind != KIND_IK && job.n_params != 1) invalid("exactly one params entry expected");
    if (job.kind == KIND_IK && job.n_params > 255) invalid("too many categories");
    S.precision = job.precision >= 0 ? job.precision : g_precision;
    if (S.precision != HPGL_PRECISION_FP64 && S.precision != HPGL_PRECISION_MIXED) invalid("unknown precision");
    S.K = job.kind == KIND_IK ? job.n_params : 1;
    std::vector<KrigingParams> kp;
    for (int k = 0; k < S.K; ++k) kp.push_back(to_params(job.params[k]));
    S.per_category = false;
    for (int k = 1; k < S.K; ++k)
        if (!same_system(kp[0], kp[k])) S.per_category = true;
    S.status_stride = S.per_category ? S.K : 1;
    S.nmax_all = 0;
    const int threads = host_threads();
    if (S.per_category) {
        S.groups.resize(S.K);
        for (int k = 0; k < S.K; ++k) {
            S.groups[k].k0 = k;
            S.groups[k].k1 = k + 1;
        }
    } else {
        S.groups.resize(1);
        S.groups[0].k0 = 0;
        S.groups[0].k1 = S.K;
    }
    try {
        for (auto &g : S.groups) {
            build_plan(g.plan, job.kind, job.nx, job.ny, job.nz, kp[g.k0], job.mask, threads);
            S.nmax_all = std::max(S.nmax_all, g.plan.nmax);
        }
    } catch (const std::domain_error &e) {
        throw HpglError{HPGL_E_UNSUPPORTED, e.what()};
    } catch (const std::invalid_argument &e) {
        throw HpglError{HPGL_E_INVALID, e.what()};
    }
    // The reference keeps marginal probabilities as float (ik_params.h:41,
    // mean_provider.cpp:8-13) and hands every mean to the combiner as float.
    S.pk.resize(S.K);
    for (int k = 0; k < S.K; ++k) S.pk[k] = (float)kp[k].marginal_prob;
    S.sk_mean = 0;
    if (job.kind == KIND_SK)
        S.sk_mean = job.sk_automatic_mean ? informed_mean(job.values, job.mask, S.size) : job.sk_mean;
}

static void upload_plan(Group &g, cudaStream_t s) {
    const Plan &P = g.plan;
    g.buf.reset(new PlanBuffers());
    PlanBuffers &B = *g.buf;
    std::vector<int4> t(P.tmpl.size());
    for (size_t i = 0; i < t.size(); ++i)
        t[i] = make_int4(P.px + P.tmpl[i].dx, P.tmpl[i].dy, P.tmpl[i].dz, P.tmpl[i].delta);
    B.tmpl.ensure(t.size());
    B.table.ensure(P.table.size());
    B.bucket_start.ensure(P.bucket_start.size());
    B.bucket_nodes.ensure(P.bucket_nodes.size());
    B.bucket_clean.ensure(P.bucket_clean.size());
    B.bits.ensure((size_t)P.wpr * P.ny * P.nz + 2);
    if (!t.empty()) CUDA_CHECK(cudaMemcpyAsync(B.tmpl.p, t.data(), t.size() * sizeof(int4), cudaMemcpyHostToDevice, s));
    CUDA_CHECK(cudaMemcpyAsync(B.table.p, P.table.data(), P.table.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    CUDA_CHECK(cudaMemcpyAsync(B.bucket_start.p, P.bucket_start.data(), P.bucket_start.size() * sizeof(int),
                               cudaMemcpyHostToDevice, s));
    if (!P.bucket_nodes.empty())
        CUDA_CHECK(cudaMemcpyAsync(B.bucket_nodes.p, P.bucket_nodes.data(), P.bucket_nodes.size() * sizeof(int),
                                   cudaMemcpyHostToDevice, s));
    CUDA_CHECK(cudaMemcpyAsync(B.bucket_clean.p, P.bucket_clean.data(), P.bucket_clean.size(), cudaMemcpyHostToDevice, s));
    DevPlan &d = g.dp;
    d.nmax = P.nmax;
    d.tmpl = B.tmpl.p;
    d.tmpl_len = (int)P.tmpl.size();
    d.px = P.px;
    d.nseg = P.nseg;
    d.wpr = P.wpr;
    d.table = B.table.p;
    d.Bx = P.B[0];
    d.By = P.B[1];
    d.Bz = P.B[2];
    d.Tx = std::min(P.trunc[0], P.B[0]);
    d.Ty = std::min(P.trunc[1], P.B[1]);
    d.Tz = std::min(P.trunc[2], P.B[2]);
    d.sx = 2 * P.B[0] + 1;
    d.syx = d.sx * (2 * P.B[1] + 1);
    d.center = P.B[2] * d.syx + P.B[1] * d.sx + P.B[0];
    d.truncated = P.truncated ? 1 : 0;
    d.c0 = P.c0;
    d.bucket_start = B.bucket_start.p;
    d.bucket_nodes = B.bucket_nodes.p;
    d.bucket_clean = B.bucket_clean.p;
    d.crx = P.cl_r[0];
    d.cry = P.cl_r[1];
    d.crz = P.cl_r[2];
    d.mx = P.mx;
    d.my = P.my;
    d.mz = P.mz;
    d.max_candidates = std::max(1, P.max_candidates);
}

static void upload_inputs(JobState &S, Context &C, const hpgl_b200_result_t *res) {
    cudaStream_t s = C.stream;
    const hpgl_b200_job_t &job = S.job;
    const size_t n = (size_t)S.size;
    C.mask.ensure(n);
    CUDA_CHECK(cudaMemcpyAsync(C.mask.p, job.mask, n, cudaMemcpyHostToDevice, s));
    if (job.kind <= KIND_LVM) {
        C.values.ensure(n);
        CUDA_CHECK(cudaMemcpyAsync(C.values.p, job.values, n * sizeof(float), cudaMemcpyHostToDevice, s));
        C.out_values.ensure(n);
    } else {
        C.codes.ensure(n);
        CUDA_CHECK(cudaMemcpyAsync(C.codes.p, job.codes, n, cudaMemcpyHostToDevice, s));
        C.out_codes.ensure(n);
        C.probs.ensure(n * S.K);
    }
    if (job.kind == KIND_LVM) {
        C.mean.ensure(n);
        CUDA_CHECK(cudaMemcpyAsync(C.mean.p, job.mean, n * sizeof(float), cudaMemcpyHostToDevice, s));
    }
    C.out_mask.ensure(n);
    C.status.ensure(n * S.status_stride);
    C.nb.ensure(n * (size_t)S.nmax_all);
    C.nbcount.ensure(n);
    C.untouched.ensure(n);
    C.routed.ensure(n);
    C.counters.ensure(1);
    C.pk.ensure(S.K);
    CUDA_CHECK(cudaMemcpyAsync(C.pk.p, S.pk.data(), S.K * sizeof(float), cudaMemcpyHostToDevice, s));
    if (res && res->variance) C.variance.ensure(n * S.status_stride);
    if (res && res->weights) C.weights.ensure(n * S.status_stride * (size_t)S.nmax_all);
    int max_cand = 1;
    for (auto &g : S.groups) {
        upload_plan(g, s);
        if (g.plan.any_clean) max_cand = std::max(max_cand, g.plan.max_candidates);
    }
    // clusterizer scratch: one candidate list per resident warp
    bool any_clean = false;
    for (auto &g : S.groups) any_clean |= g.plan.any_clean;
    if (any_clean) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        long long warps = std::min<long long>((long long)sms * 32, (S.size + 31) / 32 * 32);
        C.skey.ensure((size_t)warps * max_cand);
        C.sidx.ensure((size_t)warps * max_cand);
    }
}

static DevJob make_devjob(JobState &S, Context &C, const Group &g, const hpgl_b200_result_t *res) {
    const hpgl_b200_job_t &job = S.job;
    DevJob J;
    memset(&J, 0, sizeof(J));
    J.kind = job.kind;
    J.nx = job.nx;
    J.ny = job.ny;
    J.nz = job.nz;
    J.size = S.size;
    J.values = job.kind <= KIND_LVM ? C.values.p : nullptr;
    J.codes = job.kind <= KIND_LVM ? nullptr : C.codes.p;
    J.mask = C.mask.p;
    J.mean = job.kind == KIND_LVM ? C.mean.p : nullptr;
    J.bits = g.buf->bits.p;
    J.K = S.K;
    J.k0 = g.k0;
    J.k1 = g.k1;
    J.pk = C.pk.p;
    J.sk_mean_f = (float)S.sk_mean;
    J.median_m = (float)job.median_marginal1;
    J.nb = C.nb.p;
    J.nbcount = C.nbcount.p;
    J.out_values = job.kind <= KIND_LVM ? C.out_values.p : nullptr;
    J.out_codes = job.kind <= KIND_LVM ? nullptr : C.out_codes.p;
    J.out_mask = C.out_mask.p;
    J.variance = (res && res->variance) ? C.variance.p : nullptr;
    J.status = C.status.p;
    J.probs = job.kind <= KIND_LVM ? nullptr : C.probs.p;
    J.weights = (res && res->weights) ? C.weights.p : nullptr;
    J.status_stride = S.status_stride;
    J.status_offset = S.per_category ? g.k0 : 0;
    J.untouched = C.untouched.p;
    J.n_untouched = &C.counters.p->n_untouched;
    J.routed = C.routed.p;
    J.n_routed = &C.counters.p->n_routed;
    J.n_fp64 = &C.counters.p->n_fp64;
    J.err = &C.counters.p->err;
    return J;
}

struct PassTiming {
    cudaEvent_t top0 = nullptr, top1 = nullptr;
    int launches = 0;
};

// One device pass over all groups: bits, searches, solve(s), argmax.
static void device_pass(JobState &S, Context &C, const hpgl_b200_result_t *res, PassTiming *pt,
                        const std::function<void(const Group &)> &after_group) {
    cudaStream_t s = C.stream;
    CUDA_CHECK(cudaMemsetAsync(C.counters.p, 0, sizeof(Counters), s));
    int launches = 0;
    for (size_t gi = 0; gi < S.groups.size(); ++gi) {
        Group &g = S.groups[gi];
        DevJob J = make_devjob(S, C, g, res);
        CUDA_CHECK(cudaMemsetAsync(C.nbcount.p, 0, (size_t)S.size * sizeof(int), s));
        launch_build_bits(J, g.dp, g.buf->bits.p, s);
        launch_search_template(J, g.dp, s);
        launches += 2;
        if (g.plan.any_clean) {
            long long warps = C.skey.cap / g.dp.max_candidates;
            int dev = 0, sms = 148;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            warps = std::min<long long>(warps, (long long)sms * 32);
            launch_search_cluster(J, g.dp, C.skey.p, C.sidx.p, (int)std::max<long long>(1, warps), s);
            ++launches;
        }
        if (pt && gi == 0) CUDA_CHECK(cudaEventRecord(pt->top0, s));
        launch_solve(J, g.dp, S.precision, nullptr, nullptr, 0, s);
        ++launches;
        if (pt && gi == 0) CUDA_CHECK(cudaEventRecord(pt->top1, s));
        if (S.precision == HPGL_PRECISION_MIXED) {
            launch_solve(J, g.dp, HPGL_PRECISION_FP64, C.routed.p, J.n_routed, (int)S.size, s);
            ++launches;
        }
        CUDA_CHECK(cudaGetLastError());
        if (after_group) after_group(g);
        if (S.precision == HPGL_PRECISION_MIXED && gi + 1 < S.groups.size())
            CUDA_CHECK(cudaMemsetAsync(&C.counters.p->n_routed, 0, sizeof(int), s));
    }
    if (S.per_category) {
        DevJob J = make_devjob(S, C, S.groups[0], res);
        launch_ik_argmax(J, s);
        ++launches;
    }
    CUDA_CHECK(cudaGetLastError());
    if (pt) pt->launches = launches;
}

static void download(JobState &S, Context &C, hpgl_b200_result_t &res, const Counters &cnt) {
    cudaStream_t s = C.stream;
    const hpgl_b200_job_t &job = S.job;
    const size_t n = (size_t)S.size;
    if (cnt.err)
        throw HpglError{HPGL_E_INTERNAL, "device invariant violated (error bits " + std::to_string(cnt.err) + ")"};
    // Ordinary-kriging failures keep the caller's output content.
    std::vector<int> untouched(cnt.n_untouched);
    std::vector<float> saved_v(cnt.n_untouched);
    std::vector<uint8_t> saved_m(cnt.n_untouched);
    if (cnt.n_untouched > 0) {
        CUDA_CHECK(cudaMemcpyAsync(untouched.data(), C.untouched.p, cnt.n_untouched * sizeof(int), cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaStreamSynchronize(s));
        for (int i = 0; i < cnt.n_untouched; ++i) {
            saved_v[i] = res.out_values[untouched[i]];
            saved_m[i] = res.out_mask[untouched[i]];
        }
    }
    if (job.kind <= KIND_LVM)
        CUDA_CHECK(cudaMemcpyAsync(res.out_values, C.out_values.p, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    else
        CUDA_CHECK(cudaMemcpyAsync(res.out_codes, C.out_codes.p, n, cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaMemcpyAsync(res.out_mask, C.out_mask.p, n, cudaMemcpyDeviceToHost, s));
    const size_t slots = n * S.status_stride;
    if (res.status) CUDA_CHECK(cudaMemcpyAsync(res.status, C.status.p, slots, cudaMemcpyDeviceToHost, s));
    if (res.variance) CUDA_CHECK(cudaMemcpyAsync(res.variance, C.variance.p, slots * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (res.probs && job.kind >= KIND_IK)
        CUDA_CHECK(cudaMemcpyAsync(res.probs, C.probs.p, n * (job.kind == KIND_IK ? S.K : 1) * sizeof(float),
                                   cudaMemcpyDeviceToHost, s));
    if (res.weights)
        CUDA_CHECK(cudaMemcpy2DAsync(res.weights, (size_t)res.nb_stride * sizeof(double), C.weights.p,
                                     (size_t)S.nmax_all * sizeof(double), (size_t)S.nmax_all * sizeof(double), slots,
                                     cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    for (int i = 0; i < cnt.n_untouched; ++i) {
        res.out_values[untouched[i]] = saved_v[i];
        res.out_mask[untouched[i]] = saved_m[i];
    }
}

// Neighbour lists of the group just searched, into slot node*stride + offset.
static void download_neighbours(JobState &S, Context &C, const Group &g, hpgl_b200_result_t &res) {
    cudaStream_t s = C.stream;
    const size_t n = (size_t)S.size;
    const int off = S.per_category ? g.k0 : 0;
    if (res.nb_count)
        CUDA_CHECK(cudaMemcpy2DAsync(res.nb_count + off, (size_t)S.status_stride * sizeof(int), C.nbcount.p, sizeof(int),
                                     sizeof(int), n, cudaMemcpyDeviceToHost, s));
    if (res.nb_index)
        CUDA_CHECK(cudaMemcpy2DAsync(res.nb_index + (size_t)off * res.nb_stride,
                                     (size_t)S.status_stride * res.nb_stride * sizeof(int), C.nb.p,
                                     (size_t)g.plan.nmax * sizeof(int), (size_t)g.plan.nmax * sizeof(int), n,
                                     cudaMemcpyDeviceToHost, s));
}

static void check_result(const JobState &S, const hpgl_b200_result_t &res) {
    if (S.job.kind <= KIND_LVM && !res.out_values) invalid("out_values is null");
    if (S.job.kind > KIND_LVM && !res.out_codes) invalid("out_codes is null");
    if (!res.out_mask) invalid("out_mask is null");
    if ((res.nb_index || res.weights) && res.nb_stride < S.nmax_all) invalid("nb_stride smaller than max_neighbours");
}

void run_job(const hpgl_b200_job_t &job, hpgl_b200_result_t &res) {
    std::lock_guard<std::mutex> lock(g_mutex);
    auto t0 = std::chrono::steady_clock::now();
    JobState S;
    prepare(S, job);
    check_result(S, res);
    res.ms_plan = ms_since(t0);
    Context &C = ctx();
    auto t1 = std::chrono::steady_clock::now();
    upload_inputs(S, C, &res);
    CUDA_CHECK(cudaStreamSynchronize(C.stream));
    res.ms_h2d = ms_since(t1);
    cudaEvent_t e0, e1;
    CUDA_CHECK(cudaEventCreate(&e0));
    CUDA_CHECK(cudaEventCreate(&e1));
    CUDA_CHECK(cudaEventRecord(e0, C.stream));
    const bool want_nb = res.nb_count || res.nb_index;
    device_pass(S, C, &res, nullptr, [&](const Group &g) {
        if (want_nb) download_neighbours(S, C, g, res);
    });
    CUDA_CHECK(cudaEventRecord(e1, C.stream));
    Counters cnt;
    CUDA_CHECK(cudaMemcpyAsync(&cnt, C.counters.p, sizeof(Counters), cudaMemcpyDeviceToHost, C.stream));
    CUDA_CHECK(cudaStreamSynchronize(C.stream));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    res.ms_device = ms;
    auto t2 = std::chrono::steady_clock::now();
    download(S, C, res, cnt);
    res.ms_d2h = ms_since(t2);
    // systems attempted: kriged nodes (uninformed for OK/SK/LVM, all for IK)
    // times categories solved separately
    long long kriged = 0;
    if (job.kind <= KIND_LVM) {
        for (long long i = 0; i < S.size; ++i) kriged += job.mask[i] == 0;
    } else {
        kriged = S.size;
    }
    res.systems = kriged * (long long)S.groups.size();
    res.systems_fp64 = (long long)cnt.n_fp64;
    res.failures = 0;
    res.ms_total = ms_since(t0);
}

void bench_job(const hpgl_b200_job_t &job, hpgl_b200_result_t &res, hpgl_b200_bench_t &bench) {
    std::lock_guard<std::mutex> lock(g_mutex);
    auto t0 = std::chrono::steady_clock::now();
    JobState S;
    prepare(S, job);
    check_result(S, res);
    bench.ms_plan = ms_since(t0);
    Context &C = ctx();
    upload_inputs(S, C, &res);
    if (bench.flush_bytes > 0) C.flush.ensure((size_t)bench.flush_bytes);
    CUDA_CHECK(cudaStreamSynchronize(C.stream));
    PassTiming pt;
    CUDA_CHECK(cudaEventCreate(&pt.top0));
    CUDA_CHECK(cudaEventCreate(&pt.top1));
    cudaEvent_t e0, e1;
    CUDA_CHECK(cudaEventCreate(&e0));
    CUDA_CHECK(cudaEventCreate(&e1));
    double top_sum = 0;
    Counters cnt{};
    for (int it = 0; it < bench.warmup + bench.iters; ++it) {
        if (bench.flush_bytes > 0)
            CUDA_CHECK(cudaMemsetAsync(C.flush.p, it & 0xff, (size_t)bench.flush_bytes, C.stream));
        CUDA_CHECK(cudaEventRecord(e0, C.stream));
        device_pass(S, C, &res, &pt, nullptr);
        CUDA_CHECK(cudaEventRecord(e1, C.stream));
        CUDA_CHECK(cudaMemcpyAsync(&cnt, C.counters.p, sizeof(Counters), cudaMemcpyDeviceToHost, C.stream));
        CUDA_CHECK(cudaStreamSynchronize(C.stream));
        if (it >= bench.warmup) {
            float ms = 0, tms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            cudaEventElapsedTime(&tms, pt.top0, pt.top1);
            if (bench.ms_per_iter) bench.ms_per_iter[it - bench.warmup] = ms;
            top_sum += tms;
        }
    }
    bench.ms_top_kernel = bench.iters > 0 ? top_sum / bench.iters : 0;
    snprintf(bench.top_kernel, sizeof(bench.top_kernel), "k_solve<%d,%d>", S.nmax_all <= 32 ? 32 : 64,
             S.precision);
    bench.launches_per_iter = pt.launches;
    cudaEventDestroy(pt.top0);
    cudaEventDestroy(pt.top1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    download(S, C, res, cnt);
    long long kriged = 0;
    if (job.kind <= KIND_LVM) {
        for (long long i = 0; i < S.size; ++i) kriged += job.mask[i] == 0;
    } else {
        kriged = S.size;
    }
    bench.systems = kriged * (long long)S.groups.size();
    bench.systems_fp64 = (long long)cnt.n_fp64;
    res.systems = bench.systems;
    res.systems_fp64 = bench.systems_fp64;
}

}  // namespace hpgl_b200
