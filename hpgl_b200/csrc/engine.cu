// Job execution on the GPU.
//
// Every job gets one device arena holding its inputs, plan (template,
// covariance table, clusterizer buckets, informed-bit rows), neighbour lists,
// scratch and outputs.  The synchronous C-ABI calls run on one stream with a
// cached, grow-only arena; the server (server section below) runs several jobs
// at once, each on its own stream with an arena from the stream-ordered pool
// (cudaMallocAsync), admitted against an HBM budget.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <thread>

#include "engine.h"
#include "sgs_host.h"
#include "task_pool.h"
#include "kernels.cuh"

namespace hpgl_b200 {

// jobs of at most this many neighbours take the exact path when mixed is asked for
constexpr int MIXED_MIN_NEIGHBOURS = 12;

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
static std::atomic<int> g_sim_window{1 << 18};
void set_sim_window(int window) { g_sim_window = window; }

static double ms_since(std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

static void ensure_device() {
    static const cudaError_t probe = [] {
        int n = 0;
        cudaError_t e = cudaGetDeviceCount(&n);
        if (e == cudaSuccess && n == 0) e = cudaErrorNoDevice;
        return e;
    }();
    if (probe != cudaSuccess)
        throw HpglError{HPGL_E_CUDA, std::string("no CUDA device available: ") + cudaGetErrorString(probe)};
}

static int sm_count_host() {
    static const int n = [] {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        return sms > 0 ? sms : 148;
    }();
    return n;
}

struct Counters {
    int n_untouched;
    int n_routed;
    int err;
    int n_attempt;         // mixed path: systems attempted in FP32
    int n_attempt_routed;  // and of those routed
    int abandon;           // the job was abandoned to the plain FP64 pass
    int seg_next;          // template search: the next segment (reset per launch)
    int node_next;         // clusterizer search: the next chunk of nodes (reset per launch)
    unsigned long long n_fp64;
};

// ---- job state ---------------------------------------------------------------

struct Group {
    int k0, k1;
    Plan plan;
    std::vector<int4> tmpl_dev;  // device form of the template
    DevPlan dp;
    // arena offsets
    size_t o_tmpl, o_table, o_bstart, o_bnodes, o_bclean, o_bits;
};

struct Arena {
    size_t o_values, o_codes, o_mask, o_mean, o_out_values, o_out_codes, o_out_mask, o_probs, o_pk, o_status,
        o_variance, o_weights, o_nb, o_nbcount, o_untouched, o_routed, o_counters, o_skey, o_sidx, o_svalues,
        o_smask, o_cross;
    size_t in_total;  // the inputs (mask, values or codes, mean cubes) come first: [0, in_total)
    size_t total;
    long long cluster_warps;
};

struct JobState {
    hpgl_b200_job_t job;
    int precision;
    long long size;
    int K;
    bool per_category;
    int status_stride;
    std::vector<Group> groups;
    std::vector<float> pk;
    double sk_mean;
    int nmax_all;
    bool want_variance, want_weights;
    bool sis_lvm = false;
    long long kriged;
    // cokriging
    bool cok = false;
    double cok_coef = 0, cok_svar = 0;
    std::vector<double> cross_table;  // Markov model II: the secondary model's table
    Arena ar;
    // Device addresses: offsets below ar.in_total from in_base (the inputs),
    // the others from rest + (off - in_total).  One arena: in_base = the
    // arena, rest = arena + in_total (set_arena); inputs uploaded on their
    // own (the synchronous calls): in_base = that buffer, rest = the arena.
    char *in_base = nullptr;
    char *rest = nullptr;
};

static void set_arena(JobState &S, char *arena) {
    S.in_base = arena;
    S.rest = arena + S.ar.in_total;
}

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

static void check_result(const JobState &S, const hpgl_b200_result_t &res) {
    if (kind_is_cont(S.job.kind) && !res.out_values) invalid("out_values is null");
    if (!kind_is_cont(S.job.kind) && !res.out_codes) invalid("out_codes is null");
    if (S.cok && res.weights && res.nb_stride < S.nmax_all + 1)
        invalid("nb_stride smaller than max_neighbours + 1 (cokriging weights)");
    if (!res.out_mask) invalid("out_mask is null");
    if ((res.nb_index || res.weights) && res.nb_stride < S.nmax_all) invalid("nb_stride smaller than max_neighbours");
}

static size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

// The arena's first part, the job's inputs: mask, values or codes, mean
// cubes (from S.job, S.size, S.K); returns its size.
static size_t layout_inputs(JobState &S) {
    const hpgl_b200_job_t &job = S.job;
    const bool cont = kind_is_cont(job.kind);
    const size_t n = (size_t)S.size;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += align_up(bytes ? bytes : 1);
        return o;
    };
    Arena &A = S.ar;
    A.o_mask = take(n);
    A.o_values = cont ? take(n * 4) : 0;
    A.o_codes = cont ? 0 : take(n);
    S.sis_lvm = job.sequential && job.kind == KIND_IK && job.category_means;
    A.o_mean = job.kind == KIND_LVM ? take(n * 4) : (S.sis_lvm ? take(n * S.K * 4) : 0);
    A.in_total = off;
    return off;
}

// Host planning and arena layout (no device work).
// plan_threads: host threads for the planning (0: host_threads()).
static void prepare(JobState &S, const hpgl_b200_job_t &job, const hpgl_b200_result_t &res, int plan_threads = 0) {
    S.job = job;
    if (job.kind < 0 || job.kind > 6) invalid("unknown kriging kind");
    if (job.nx <= 0 || job.ny <= 0 || job.nz <= 0) invalid("grid dimensions must be positive");
    S.size = (long long)job.nx * job.ny * job.nz;
    if (S.size > 2147483647LL) invalid("grid larger than 2^31-1 nodes (node indices are int, typedefs.h:112)");
    if (!job.mask) invalid("mask is null");
    if (!job.params || job.n_params < 1) invalid("params missing");
    const bool cont = kind_is_cont(job.kind);
    S.cok = kind_is_cokriging(job.kind);
    if (cont && !job.values) invalid("values are null");
    if (S.cok && (!job.secondary_values || !job.secondary_mask)) invalid("secondary property is null");
    if (job.kind == KIND_COK2 && !job.secondary_cov) invalid("secondary covariance is null");
    if (!cont && !job.codes) invalid("codes are null");
    if (job.kind == KIND_LVM && !job.mean) invalid("mean cube is null");
    if (job.kind != KIND_IK && job.n_params != 1) invalid("exactly one params entry expected");
    if (job.kind == KIND_IK && job.n_params > 255) invalid("too many categories");
    S.precision = job.precision >= 0 ? job.precision : g_precision;
    if (S.cok) S.precision = HPGL_PRECISION_FP64;  // cokriging is solved in the reference's order only
    if (job.sequential) {
        if (job.kind != KIND_OK && job.kind != KIND_SK && job.kind != KIND_LVM && job.kind != KIND_IK)
            invalid("sequential simulation takes the kinds OK, SK, LVM and IK");
        S.precision = HPGL_PRECISION_FP64;  // each node's draw depends on its exact kriging
        if (job.kind == KIND_IK && job.category_means)
            for (int k = 0; k < job.n_params; ++k)
                if (!job.category_means[k]) invalid("category mean cube is null");
    }
    if (S.precision != HPGL_PRECISION_FP64 && S.precision != HPGL_PRECISION_MIXED) invalid("unknown precision");
    S.K = job.kind == KIND_IK ? job.n_params : 1;
    std::vector<KrigingParams> kp;
    for (int k = 0; k < S.K; ++k) kp.push_back(to_params(job.params[k]));
    S.per_category = false;
    for (int k = 1; k < S.K; ++k)
        if (!same_system(kp[0], kp[k])) S.per_category = true;
    S.status_stride = S.per_category ? S.K : 1;
    S.nmax_all = 0;
    const int threads = plan_threads > 0 ? plan_threads : host_threads();
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
            build_plan(g.plan, job.kind, job.nx, job.ny, job.nz, kp[g.k0], job.mask, threads, job.sequential != 0);
            S.nmax_all = std::max(S.nmax_all, g.plan.nmax);
        }
        if (job.sequential && job.kind == KIND_IK) {
            // indicator simulation searches every category's template over
            // one set of informed bits: one padding for all
            int px = 0;
            for (auto &g : S.groups) px = std::max(px, g.plan.px);
            for (auto &g : S.groups) {
                g.plan.px = px;
                g.plan.wpr = g.plan.nseg + 2 * (px / 32) + 2;
            }
        }
    } catch (const std::domain_error &e) {
        throw HpglError{HPGL_E_UNSUPPORTED, e.what()};
    } catch (const std::invalid_argument &e) {
        throw HpglError{HPGL_E_INVALID, e.what()};
    }
    // Up to MIXED_MIN_NEIGHBOURS neighbours the exact solve is the faster one
    // (its factorisation stops at n, the FP32 sweep always runs 32 rows: the
    // mixed solve takes 1.25-1.33x the exact one at 8-9 neighbours and 0.69x
    // at 19), so a mixed request takes the exact path, whose results are the
    // FP64 ones.
    if (S.precision == HPGL_PRECISION_MIXED && S.nmax_all <= MIXED_MIN_NEIGHBOURS) S.precision = HPGL_PRECISION_FP64;
    if (S.cok) {
        // cross covariance models (simple_cokriging_markI.cpp:140-181); the
        // means are mean_t (float) in the reference
        const Plan &P = S.groups[0].plan;
        const double pv = P.c0;  // C(0) of the primary model
        if (job.kind == KIND_COK1) {
            S.cok_coef = job.correlation * sqrt(job.secondary_variance) / sqrt(pv);
            S.cok_svar = job.secondary_variance;
        } else {
            KrigingParams sp = kp[0];
            sp.cov_type = job.secondary_cov->m_covariance_type;
            for (int i = 0; i < 3; ++i) {
                sp.ranges[i] = job.secondary_cov->m_ranges[i];
                sp.angles[i] = job.secondary_cov->m_angles[i];
            }
            sp.sill = job.secondary_cov->m_sill;
            sp.nugget = job.secondary_cov->m_nugget;
            try {
                validate_params(sp, KIND_OK);
            } catch (const std::invalid_argument &e) {
                throw HpglError{HPGL_E_INVALID, std::string("secondary covariance: ") + e.what()};
            }
            S.cok_svar = CovModel(sp)(0.0, 0.0, 0.0);
            S.cok_coef = job.correlation * sqrt(S.cok_svar / pv);
            fill_cov_table(S.cross_table, P.B, sp, threads);
        }
    }
    check_result(S, res);
    // The reference keeps marginal probabilities as float (ik_params.h:41,
    // mean_provider.cpp:8-13) and hands every mean to the combiner as float.
    S.pk.resize(S.K);
    for (int k = 0; k < S.K; ++k) S.pk[k] = (float)kp[k].marginal_prob;
    S.sk_mean = 0;
    // sequential simulation krigs with mean 0 (sequential_gaussian_simulation.cpp:39-41)
    if (job.kind == KIND_SK && !job.sequential)
        S.sk_mean = job.sk_automatic_mean ? informed_mean(job.values, job.mask, S.size) : job.sk_mean;
    S.want_variance = res.variance != nullptr || (job.sequential && cont);
    S.want_weights = res.weights != nullptr;
    // the plan counted the informed cells (every plan of the job reads the same mask)
    S.kriged = cont ? S.size - S.groups[0].plan.informed : S.size;

    // arena layout
    const size_t n = (size_t)S.size, slots = n * S.status_stride;
    size_t off = layout_inputs(S);
    auto take = [&](size_t bytes) {
        size_t o = off;
        off += align_up(bytes ? bytes : 1);
        return o;
    };
    Arena &A = S.ar;
    A.o_out_values = cont ? take(n * 4) : 0;
    A.o_out_codes = cont ? 0 : take(n);
    A.o_out_mask = take(n);
    A.o_probs = cont ? 0 : take(n * S.K * 4);
    A.o_pk = take(S.K * 4);
    A.o_status = take(slots);
    A.o_variance = S.want_variance ? take(slots * 8) : 0;
    A.o_weights = S.want_weights ? take(slots * (S.nmax_all + (S.cok ? 1 : 0)) * 8) : 0;
    A.o_svalues = S.cok ? take(n * 4) : 0;
    A.o_smask = S.cok ? take(n) : 0;
    A.o_cross = S.cross_table.empty() ? 0 : take(S.cross_table.size() * 8);
    A.o_nb = take(n * (size_t)S.nmax_all * 4);
    A.o_nbcount = take(n * 4);
    A.o_untouched = take(n * 4);
    A.o_routed = take(n);  // per-node routed flags
    A.o_counters = take(sizeof(Counters));
    int max_cand = 1;
    bool any_clean = false;
    for (auto &g : S.groups) {
        const Plan &P = g.plan;
        g.tmpl_dev.resize(P.tmpl.size());
        for (size_t i = 0; i < P.tmpl.size(); ++i)
            g.tmpl_dev[i] = make_int4(P.px + P.tmpl[i].dx, P.tmpl[i].dy, P.tmpl[i].dz, P.tmpl[i].delta);
        g.o_tmpl = take(g.tmpl_dev.size() * sizeof(int4));
        g.o_table = take(P.table.size() * 8);
        g.o_bstart = take(P.bucket_start.size() * 4);
        g.o_bnodes = take(P.bucket_nodes.size() * 4);
        g.o_bclean = take(P.bucket_clean.size());
        g.o_bits = take(((size_t)P.wpr * P.ny * P.nz + 2) * 4);
        if (P.any_clean) {
            any_clean = true;
            max_cand = std::max(max_cand, P.max_candidates);
        }
    }
    A.cluster_warps = 0;
    if (any_clean) {
        // 64 warps a SM (the kernel's 16 blocks of 4: the search waits on
        // memory, and more warps hide more of it), fewer where the candidate
        // scratch (12 bytes a candidate a warp) would pass 4 GiB
        const long long sms = sm_count_host();
        const long long by_scratch = (4LL << 30) / std::max<long long>(1, (long long)max_cand * 12);
        const long long warps = std::min(sms * 64, std::max(sms * 8, by_scratch));
        A.cluster_warps = std::min<long long>(warps, (S.size + 31) / 32 * 32);
        A.o_skey = take((size_t)A.cluster_warps * max_cand * 8);
        A.o_sidx = take((size_t)A.cluster_warps * max_cand * 4);
    } else {
        A.o_skey = A.o_sidx = 0;
    }
    A.total = off;
}

template <typename T>
static T *at(const JobState &S, size_t off) {
    return reinterpret_cast<T *>(off < S.ar.in_total ? S.in_base + off : S.rest + (off - S.ar.in_total));
}

// The job's input arrays, in the arena's input layout: (offset, host
// address, bytes).
struct InputPart {
    size_t off;
    const void *src;
    size_t bytes;
};
static std::vector<InputPart> input_parts(const JobState &S) {
    const hpgl_b200_job_t &job = S.job;
    const size_t n = (size_t)S.size;
    const Arena &A = S.ar;
    std::vector<InputPart> v;
    v.push_back({A.o_mask, job.mask, n});
    if (kind_is_cont(job.kind)) v.push_back({A.o_values, job.values, n * 4});
    else v.push_back({A.o_codes, job.codes, n});
    if (job.kind == KIND_LVM) v.push_back({A.o_mean, job.mean, n * 4});
    if (S.sis_lvm)
        for (int k = 0; k < S.K; ++k) v.push_back({A.o_mean + (size_t)k * n * 4, job.category_means[k], n * 4});
    return v;
}

static void upload_inputs(JobState &S, cudaStream_t s) {
    for (const InputPart &p : input_parts(S))
        CUDA_CHECK(cudaMemcpyAsync(at<char>(S, p.off), p.src, p.bytes, cudaMemcpyHostToDevice, s));
}

// Everything but the inputs: marginal probabilities, cokriging data, the
// plans (template, table, clusterizer buckets); fills the device plans.
static void upload_rest(JobState &S, cudaStream_t s) {
    const hpgl_b200_job_t &job = S.job;
    const size_t n = (size_t)S.size;
    const Arena &A = S.ar;
    CUDA_CHECK(cudaMemcpyAsync(at<float>(S, A.o_pk), S.pk.data(), S.K * 4, cudaMemcpyHostToDevice, s));
    if (S.cok) {
        CUDA_CHECK(cudaMemcpyAsync(at<float>(S, A.o_svalues), job.secondary_values, n * 4, cudaMemcpyHostToDevice, s));
        CUDA_CHECK(cudaMemcpyAsync(at<uint8_t>(S, A.o_smask), job.secondary_mask, n, cudaMemcpyHostToDevice, s));
        if (!S.cross_table.empty())
            CUDA_CHECK(cudaMemcpyAsync(at<double>(S, A.o_cross), S.cross_table.data(), S.cross_table.size() * 8,
                                       cudaMemcpyHostToDevice, s));
    }
    for (auto &g : S.groups) {
        const Plan &P = g.plan;
        if (!g.tmpl_dev.empty())
            CUDA_CHECK(cudaMemcpyAsync(at<int4>(S, g.o_tmpl), g.tmpl_dev.data(), g.tmpl_dev.size() * sizeof(int4),
                                       cudaMemcpyHostToDevice, s));
        CUDA_CHECK(cudaMemcpyAsync(at<double>(S, g.o_table), P.table.data(), P.table.size() * 8,
                                   cudaMemcpyHostToDevice, s));
        CUDA_CHECK(cudaMemcpyAsync(at<int>(S, g.o_bstart), P.bucket_start.data(), P.bucket_start.size() * 4,
                                   cudaMemcpyHostToDevice, s));
        if (!P.bucket_nodes.empty())
            CUDA_CHECK(cudaMemcpyAsync(at<int>(S, g.o_bnodes), P.bucket_nodes.data(), P.bucket_nodes.size() * 4,
                                       cudaMemcpyHostToDevice, s));
        CUDA_CHECK(cudaMemcpyAsync(at<uint8_t>(S, g.o_bclean), P.bucket_clean.data(), P.bucket_clean.size(),
                                   cudaMemcpyHostToDevice, s));
        DevPlan &d = g.dp;
        d.nmax = P.nmax;
        d.tmpl = at<int4>(S, g.o_tmpl);
        d.tmpl_len = (int)P.tmpl.size();
        d.px = P.px;
        d.nseg = P.nseg;
        d.wpr = P.wpr;
        d.table = at<double>(S, g.o_table);
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
        d.bucket_start = at<int>(S, g.o_bstart);
        d.bucket_nodes = at<int>(S, g.o_bnodes);
        d.bucket_clean = at<uint8_t>(S, g.o_bclean);
        d.crx = P.cl_r[0];
        d.cry = P.cl_r[1];
        d.crz = P.cl_r[2];
        d.mx = P.mx;
        d.my = P.my;
        d.mz = P.mz;
        d.max_candidates = std::max(1, P.max_candidates);
    }
}

static void upload(JobState &S, cudaStream_t s) {
    upload_inputs(S, s);
    upload_rest(S, s);
}

static DevJob make_devjob(const JobState &S, const Group &g) {
    const hpgl_b200_job_t &job = S.job;
    const Arena &A = S.ar;
    const bool cont = kind_is_cont(job.kind);
    DevJob J;
    memset(&J, 0, sizeof(J));
    J.kind = job.kind;
    J.nx = job.nx;
    J.ny = job.ny;
    J.nz = job.nz;
    J.div_nx = FastDiv((unsigned)job.nx);
    J.div_ny = FastDiv((unsigned)job.ny);
    J.size = S.size;
    J.values = cont ? at<float>(S, A.o_values) : nullptr;
    J.codes = cont ? nullptr : at<uint8_t>(S, A.o_codes);
    J.mask = at<uint8_t>(S, A.o_mask);
    J.mean = (job.kind == KIND_LVM || S.sis_lvm) ? at<float>(S, A.o_mean) : nullptr;
    J.bits = at<uint32_t>(S, g.o_bits);
    J.K = S.K;
    J.k0 = g.k0;
    J.k1 = g.k1;
    J.pk = at<float>(S, A.o_pk);
    J.sk_mean_f = (float)S.sk_mean;
    J.median_m = (float)job.median_marginal1;
    J.nb = at<int>(S, A.o_nb);
    J.nbcount = at<int>(S, A.o_nbcount);
    J.out_values = cont ? at<float>(S, A.o_out_values) : nullptr;
    J.out_codes = cont ? nullptr : at<uint8_t>(S, A.o_out_codes);
    J.out_mask = at<uint8_t>(S, A.o_out_mask);
    J.variance = S.want_variance ? at<double>(S, A.o_variance) : nullptr;
    J.sim_values = cont ? at<float>(S, A.o_values) : nullptr;
    J.sim_mask = at<uint8_t>(S, A.o_mask);
    J.sim_bits = at<uint32_t>(S, g.o_bits);
    J.sim_codes = cont ? nullptr : at<uint8_t>(S, A.o_codes);
    J.sis_lvm = S.sis_lvm ? 1 : 0;
    J.sis_corr = job.correlogram ? 1 : 0;
    J.nb_stride = S.nmax_all;
    J.status = at<int8_t>(S, A.o_status);
    J.probs = cont ? nullptr : at<float>(S, A.o_probs);
    J.weights = S.want_weights ? at<double>(S, A.o_weights) : nullptr;
    J.status_stride = S.status_stride;
    J.status_offset = S.per_category ? g.k0 : 0;
    Counters *cnt = at<Counters>(S, A.o_counters);
    J.untouched = at<int>(S, A.o_untouched);
    J.n_untouched = &cnt->n_untouched;
    J.routed = at<uint8_t>(S, A.o_routed);
    J.n_routed = &cnt->n_routed;
    J.n_attempt = &cnt->n_attempt;
    J.n_attempt_routed = &cnt->n_attempt_routed;
    J.abandon = &cnt->abandon;
    J.seg_next = &cnt->seg_next;
    J.node_next = &cnt->node_next;
    J.n_fp64 = &cnt->n_fp64;
    J.err = &cnt->err;
    if (S.cok) {
        J.svalues = at<float>(S, A.o_svalues);
        J.smask = at<uint8_t>(S, A.o_smask);
        J.cross_table = S.cross_table.empty() ? g.dp.table : at<double>(S, A.o_cross);
        J.cok_coef = S.cok_coef;
        J.cok_svar = S.cok_svar;
        J.cok_m1 = (float)job.primary_mean;
        J.cok_m2 = (float)job.secondary_mean;
    }
    return J;
}

// Events around the first group's phases: search start, solve start, solve
// end (top kernel), re-solve end.
struct PassTiming {
    cudaEvent_t search0 = nullptr, top0 = nullptr, top1 = nullptr, resolve1 = nullptr;
    int launches = 0;
};

// One device pass over all groups: bits, searches, solve(s), argmax.  The
// per-node kernels follow the launch tuning of the group's family: either
// the template search then the solve, or the clusterizer search then the
// fused search+solve kernel.
static void device_pass(JobState &S, cudaStream_t s, PassTiming *pt,
                        const std::function<void(const Group &)> &after_group) {
    const Arena &A = S.ar;
    Counters *cnt = at<Counters>(S, A.o_counters);
    CUDA_CHECK(cudaMemsetAsync(cnt, 0, sizeof(Counters), s));
    int launches = 0;
    for (size_t gi = 0; gi < S.groups.size(); ++gi) {
        Group &g = S.groups[gi];
        DevJob J = make_devjob(S, g);
        const LaunchTuning tune = tuning_get(tuning_family(g.plan.nmax), S.precision);
        const LaunchTuning tune64 = tuning_get(tuning_family(g.plan.nmax), HPGL_PRECISION_FP64);
        if (pt && gi == 0) CUDA_CHECK(cudaEventRecord(pt->search0, s));
        CUDA_CHECK(cudaMemsetAsync(J.nbcount, 0, (size_t)S.size * sizeof(int), s));
        if (S.precision == HPGL_PRECISION_MIXED) CUDA_CHECK(cudaMemsetAsync(J.routed, 0, (size_t)S.size, s));
        launch_build_bits(J, g.dp, at<uint32_t>(S, g.o_bits), s);
        ++launches;
        if (S.cok) {
            // template search, then the cokriging systems (FP64, reference order)
            CUDA_CHECK(cudaMemsetAsync(J.seg_next, 0, sizeof(int), s));
            launch_search_template(J, g.dp, s);
            if (pt && gi == 0) CUDA_CHECK(cudaEventRecord(pt->top0, s));
            launch_cokriging(J, g.dp, s);
            if (pt && gi == 0) {
                CUDA_CHECK(cudaEventRecord(pt->top1, s));
                CUDA_CHECK(cudaEventRecord(pt->resolve1, s));
            }
            launches += 2;
            CUDA_CHECK(cudaGetLastError());
            if (after_group) after_group(g);
            continue;
        }
        if (tune.schedule == SCHED_SPLIT) {
            CUDA_CHECK(cudaMemsetAsync(J.seg_next, 0, sizeof(int), s));
            launch_search_template(J, g.dp, s);
            ++launches;
        }
        if (g.plan.any_clean) {
            CUDA_CHECK(cudaMemsetAsync(J.node_next, 0, sizeof(int), s));
            launch_search_cluster(J, g.dp, at<double>(S, A.o_skey), at<int>(S, A.o_sidx), (int)A.cluster_warps, s);
            ++launches;
        }
        if (pt && gi == 0) CUDA_CHECK(cudaEventRecord(pt->top0, s));
        if (tune.schedule == SCHED_FUSED) {
            if (g.plan.nmax <= 32) launch_fused32(J, g.dp, S.precision, s, tune.blocks_per_sm);
            else launch_fused64(J, g.dp, S.precision, s, tune.blocks_per_sm);
        } else {
            CUDA_CHECK(cudaMemsetAsync(J.node_next, 0, sizeof(int), s));  // the mixed kernel's chunk counter
            launch_solve(J, g.dp, S.precision, nullptr, s, tune.blocks_per_sm);
        }
        ++launches;
        if (pt && gi == 0) CUDA_CHECK(cudaEventRecord(pt->top1, s));
        if (S.precision == HPGL_PRECISION_MIXED) {
            CUDA_CHECK(cudaMemsetAsync(J.node_next, 0, sizeof(int), s));  // an abandoned job's full FP64 pass
            launch_solve(J, g.dp, HPGL_PRECISION_FP64, J.routed, s, tune64.blocks_per_sm);
            ++launches;
        }
        if (pt && gi == 0) CUDA_CHECK(cudaEventRecord(pt->resolve1, s));
        CUDA_CHECK(cudaGetLastError());
        if (after_group) after_group(g);
        if (S.precision == HPGL_PRECISION_MIXED && gi + 1 < S.groups.size()) {
            // the routed count and the job-level tally start over per group
            CUDA_CHECK(cudaMemsetAsync(&cnt->n_routed, 0, sizeof(int), s));
            CUDA_CHECK(cudaMemsetAsync(&cnt->n_attempt, 0, 3 * sizeof(int), s));
        }
    }
    if (S.per_category) {
        DevJob J = make_devjob(S, S.groups[0]);
        launch_ik_argmax(J, s);
        ++launches;
    }
    CUDA_CHECK(cudaGetLastError());
    if (pt) pt->launches = launches;
}

// Neighbour lists of the group just searched, into slot node*stride + offset.
static void download_neighbours(const JobState &S, const Group &g, hpgl_b200_result_t &res, cudaStream_t s) {
    const size_t n = (size_t)S.size;
    const int off = S.per_category ? g.k0 : 0;
    if (res.nb_count)
        CUDA_CHECK(cudaMemcpy2DAsync(res.nb_count + off, (size_t)S.status_stride * sizeof(int),
                                     at<int>(S, S.ar.o_nbcount), sizeof(int), sizeof(int), n, cudaMemcpyDeviceToHost,
                                     s));
    if (res.nb_index)
        CUDA_CHECK(cudaMemcpy2DAsync(res.nb_index + (size_t)off * res.nb_stride,
                                     (size_t)S.status_stride * res.nb_stride * sizeof(int), at<int>(S, S.ar.o_nb),
                                     (size_t)g.plan.nmax * sizeof(int), (size_t)g.plan.nmax * sizeof(int), n,
                                     cudaMemcpyDeviceToHost, s));
}

static Counters read_counters(const JobState &S, cudaStream_t s) {
    Counters c;
    CUDA_CHECK(cudaMemcpyAsync(&c, at<Counters>(S, S.ar.o_counters), sizeof(Counters), cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    return c;
}

// memcpy on up to host_threads() pool threads, at least 4 MiB each.
static void parallel_copy(void *dst, const void *src, size_t bytes) {
    pool_for((long long)bytes, host_threads(), [=](long long lo, long long hi) {
        memcpy((char *)dst + lo, (const char *)src + lo, (size_t)(hi - lo));
    }, 4LL << 20);
}

// staging: pinned host memory of at least the main outputs' size (the
// estimate or codes and the mask), or null for direct copies.
static void download(const JobState &S, hpgl_b200_result_t &res, const Counters &cnt, cudaStream_t s,
                     char *staging = nullptr) {
    const hpgl_b200_job_t &job = S.job;
    const Arena &A = S.ar;
    const size_t n = (size_t)S.size;
    if (cnt.err)
        throw HpglError{HPGL_E_INTERNAL, "device invariant violated (error bits " + std::to_string(cnt.err) + ")"};
    // Ordinary-kriging failures keep the caller's output content.
    std::vector<int> untouched(cnt.n_untouched);
    std::vector<float> saved_v(cnt.n_untouched);
    std::vector<uint8_t> saved_m(cnt.n_untouched);
    if (cnt.n_untouched > 0) {
        CUDA_CHECK(cudaMemcpyAsync(untouched.data(), at<int>(S, A.o_untouched), cnt.n_untouched * sizeof(int),
                                   cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaStreamSynchronize(s));
        for (int i = 0; i < cnt.n_untouched; ++i) {
            saved_v[i] = res.out_values[untouched[i]];
            saved_m[i] = res.out_mask[untouched[i]];
        }
    }
    const bool cont = kind_is_cont(job.kind);
    void *out_main = cont ? (void *)res.out_values : (void *)res.out_codes;
    const size_t main_bytes = cont ? n * 4 : n;
    const void *dev_main = cont ? (const void *)at<float>(S, A.o_out_values) : (const void *)at<uint8_t>(S, A.o_out_codes);
    if (staging) {
        CUDA_CHECK(cudaMemcpyAsync(staging, dev_main, main_bytes, cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaMemcpyAsync(staging + main_bytes, at<uint8_t>(S, A.o_out_mask), n, cudaMemcpyDeviceToHost, s));
    } else {
        CUDA_CHECK(cudaMemcpyAsync(out_main, dev_main, main_bytes, cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaMemcpyAsync(res.out_mask, at<uint8_t>(S, A.o_out_mask), n, cudaMemcpyDeviceToHost, s));
    }
    const size_t slots = n * S.status_stride;
    if (res.status) CUDA_CHECK(cudaMemcpyAsync(res.status, at<int8_t>(S, A.o_status), slots, cudaMemcpyDeviceToHost, s));
    if (res.variance)
        CUDA_CHECK(cudaMemcpyAsync(res.variance, at<double>(S, A.o_variance), slots * 8, cudaMemcpyDeviceToHost, s));
    if (res.probs && job.kind >= KIND_IK)
        CUDA_CHECK(cudaMemcpyAsync(res.probs, at<float>(S, A.o_probs), n * (job.kind == KIND_IK ? S.K : 1) * 4,
                                   cudaMemcpyDeviceToHost, s));
    if (res.weights) {
        const size_t wn = (size_t)S.nmax_all + (S.cok ? 1 : 0);
        CUDA_CHECK(cudaMemcpy2DAsync(res.weights, (size_t)res.nb_stride * 8, at<double>(S, A.o_weights), wn * 8,
                                     wn * 8, slots, cudaMemcpyDeviceToHost, s));
    }
    CUDA_CHECK(cudaStreamSynchronize(s));
    if (staging) {
        parallel_copy(out_main, staging, main_bytes);
        parallel_copy(res.out_mask, staging + main_bytes, n);
    }
    for (int i = 0; i < cnt.n_untouched; ++i) {
        res.out_values[untouched[i]] = saved_v[i];
        res.out_mask[untouched[i]] = saved_m[i];
    }
    res.systems = S.kriged * (long long)S.groups.size();
    res.systems_fp64 = (long long)cnt.n_fp64;
    res.failures = 0;
}

// ---- synchronous calls ---------------------------------------------------------

struct SyncContext {
    cudaStream_t stream = nullptr;
    char *arena = nullptr;
    size_t cap = 0;
    char *inputs = nullptr;   // the job's inputs, uploaded while it is planned
    size_t in_cap = 0;
    char *pinned = nullptr;   // host staging of the inputs and the main outputs
    size_t pinned_cap = 0;
    unsigned char *sim = nullptr;  // sequential simulation's scratch (grows, kept)
    size_t sim_cap = 0;
    char *flush = nullptr;
    size_t flush_cap = 0;
};

static std::mutex g_sync_mutex;

static SyncContext &sync_ctx() {
    static SyncContext *c = nullptr;
    if (!c) {
        ensure_device();
        auto *nc = new SyncContext();
        CUDA_CHECK(cudaStreamCreateWithFlags(&nc->stream, cudaStreamNonBlocking));
        c = nc;
    }
    return *c;
}

static void sync_arena(SyncContext &C, size_t bytes) {
    if (bytes <= C.cap) return;
    if (C.arena) cudaFree(C.arena);
    C.arena = nullptr;
    C.cap = 0;
    CUDA_CHECK(cudaMalloc(&C.arena, bytes));
    C.cap = bytes;
}

static void sync_inputs(SyncContext &C, size_t bytes) {
    if (bytes <= C.in_cap) return;
    if (C.inputs) cudaFree(C.inputs);
    C.inputs = nullptr;
    C.in_cap = 0;
    CUDA_CHECK(cudaMalloc(&C.inputs, bytes));
    C.in_cap = bytes;
}

static void sync_pinned(SyncContext &C, size_t bytes) {
    if (bytes <= C.pinned_cap) return;
    if (C.pinned) cudaFreeHost(C.pinned);
    C.pinned = nullptr;
    C.pinned_cap = 0;
    CUDA_CHECK(cudaMallocHost(&C.pinned, bytes));
    C.pinned_cap = bytes;
}

static void sync_sim(SyncContext &C, size_t bytes) {
    if (bytes <= C.sim_cap) return;
    if (C.sim) cudaFree(C.sim);
    C.sim = nullptr;
    C.sim_cap = 0;
    CUDA_CHECK(cudaMalloc(&C.sim, bytes));
    C.sim_cap = bytes;
}

// Sequential simulation (sequential_simulation.h:49-122,
// sequential_indicator_simulation.cpp:23-116): the host path and draws, then
// speculative rounds on the device; the property in the arena is simulated in
// place and copied out.
static void sgs_run(JobState &S, hpgl_b200_result_t &res, SyncContext &C, std::chrono::steady_clock::time_point t0);

// The inputs of a kriging job can be uploaded before it is planned: its
// arrays are present and its grid is valid (prepare() reports anything else).
static bool early_inputs(const hpgl_b200_job_t &job) {
    if (job.sequential || job.kind < 0 || job.kind > 6 || kind_is_cokriging(job.kind)) return false;
    if (job.nx <= 0 || job.ny <= 0 || job.nz <= 0) return false;
    if ((long long)job.nx * job.ny * job.nz > 2147483647LL) return false;
    if (!job.mask || !job.params || job.n_params < 1) return false;
    if (kind_is_cont(job.kind) ? !job.values : !job.codes) return false;
    if (job.kind == KIND_LVM && !job.mean) return false;
    if (job.kind != KIND_IK && job.n_params != 1) return false;
    if (job.kind == KIND_IK && job.n_params > 255) return false;
    try {
        for (int k = 0; k < job.n_params; ++k) validate_params(to_params(job.params[k]), job.kind);
    } catch (const std::exception &) {
        return false;
    }
    return true;
}

void run_job(const hpgl_b200_job_t &job, hpgl_b200_result_t &res) {
    auto t0 = std::chrono::steady_clock::now();
    JobState S;
    if (job.sequential || !early_inputs(job)) {
        prepare(S, job, res);
        res.ms_plan = ms_since(t0);
        if (job.sequential) {
            std::lock_guard<std::mutex> lock(g_sync_mutex);
            sgs_run(S, res, sync_ctx(), t0);
            return;
        }
    }
    std::lock_guard<std::mutex> lock(g_sync_mutex);
    SyncContext &C = sync_ctx();
    char *staging = nullptr;
    if (early_inputs(job)) {
        // The inputs go to pinned staging and on to the device on a helper
        // thread while this one plans the job; the same layout function
        // places them in both.
        S.job = job;
        S.size = (long long)job.nx * job.ny * job.nz;
        S.K = job.kind == KIND_IK ? job.n_params : 1;
        const size_t in_total = layout_inputs(S);
        const size_t n = (size_t)S.size;
        const size_t out_bytes = (kind_is_cont(job.kind) ? n * 4 : n) + n;
        sync_inputs(C, in_total);
        sync_pinned(C, std::max(in_total, out_bytes));
        staging = C.pinned;
        const std::vector<InputPart> parts = input_parts(S);
        std::exception_ptr copy_error;
        std::thread copier([&] {
            try {
                for (const InputPart &p : parts) parallel_copy(C.pinned + p.off, p.src, p.bytes);
                CUDA_CHECK(cudaMemcpyAsync(C.inputs, C.pinned, in_total, cudaMemcpyHostToDevice, C.stream));
            } catch (...) {
                copy_error = std::current_exception();
            }
        });
        try {
            prepare(S, job, res);
        } catch (...) {
            copier.join();
            cudaStreamSynchronize(C.stream);
            throw;
        }
        res.ms_plan = ms_since(t0);
        copier.join();
        if (copy_error) {
            cudaStreamSynchronize(C.stream);
            std::rethrow_exception(copy_error);
        }
        if (S.ar.in_total != in_total) throw HpglError{HPGL_E_INTERNAL, "input layout changed while planning"};
        auto t1 = std::chrono::steady_clock::now();
        sync_arena(C, S.ar.total - in_total);
        S.in_base = C.inputs;
        S.rest = C.arena;
        upload_rest(S, C.stream);
        CUDA_CHECK(cudaStreamSynchronize(C.stream));
        res.ms_h2d = ms_since(t1);
    } else {
        auto t1 = std::chrono::steady_clock::now();
        sync_arena(C, S.ar.total);
        set_arena(S, C.arena);
        upload(S, C.stream);
        CUDA_CHECK(cudaStreamSynchronize(C.stream));
        res.ms_h2d = ms_since(t1);
    }
    cudaEvent_t e0, e1;
    CUDA_CHECK(cudaEventCreate(&e0));
    CUDA_CHECK(cudaEventCreate(&e1));
    CUDA_CHECK(cudaEventRecord(e0, C.stream));
    const bool want_nb = res.nb_count || res.nb_index;
    device_pass(S, C.stream, nullptr, [&](const Group &g) {
        if (want_nb) download_neighbours(S, g, res, C.stream);
    });
    CUDA_CHECK(cudaEventRecord(e1, C.stream));
    Counters cnt = read_counters(S, C.stream);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    res.ms_device = ms;
    auto t2 = std::chrono::steady_clock::now();
    download(S, res, cnt, C.stream, staging);
    res.ms_d2h = ms_since(t2);
    res.ms_total = ms_since(t0);
}

static void sgs_run(JobState &S, hpgl_b200_result_t &res, SyncContext &C, std::chrono::steady_clock::time_point t0) {
    const hpgl_b200_job_t &job = S.job;
    Group &g = S.groups[0];
    const Plan &P = g.plan;
    SimPath path;
    try {
        sim_path(job.nx, job.ny, job.nz, job.mask, job.simulation_mask, job.seed, job.kind != KIND_IK, path);
    } catch (const std::domain_error &e) {
        throw HpglError{HPGL_E_UNSUPPORTED, e.what()};
    } catch (const std::invalid_argument &e) {
        throw HpglError{HPGL_E_INVALID, e.what()};
    }
    const bool indicator = job.kind == KIND_IK;
    // per path rank: the draw itself (sample() compares it) or its normal
    // quantile
    const double *draws = path.u.data();
    res.ms_plan = ms_since(t0);
    auto t1 = std::chrono::steady_clock::now();
    cudaStream_t s = C.stream;
    sync_arena(C, S.ar.total);
    set_arena(S, C.arena);
    upload(S, s);
    const long long nsim = (long long)path.nodes.size();
    const int window = g_sim_window.load();
    const size_t bits_bytes = ((size_t)P.wpr * P.ny * P.nz + 2) * 4;
    // scratch: control, path, quantiles, ranks, pending bits, window buffers, flags
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += align_up(bytes ? bytes : 1);
        return o;
    };
    const size_t o_ctl = take(sizeof(SgsCtl)), o_nodes = take((size_t)nsim * 4), o_xp = take((size_t)nsim * 8),
                 o_rank = take((size_t)S.size * 4), o_pend = take(bits_bytes), o_blocker = take((size_t)nsim * 4),
                 o_done = take((size_t)nsim), o_w0 = take((size_t)window * 4), o_w1 = take((size_t)window * 4),
                 o_ok = take((size_t)window), o_try = take((size_t)window * 4);
    std::vector<DevPlan> cat_plans;  // indicator simulation: every category's plan (its group's)
    if (indicator)
        for (auto &gr : S.groups)
            for (int k = gr.k0; k < gr.k1; ++k) cat_plans.push_back(gr.dp);
    const size_t o_plans = take(cat_plans.size() * sizeof(DevPlan));
    sync_sim(C, off);
    unsigned char *scratch = C.sim;
    SgsState G;
    G.ctl = reinterpret_cast<SgsCtl *>(scratch + o_ctl);
    G.nodes = reinterpret_cast<const int *>(scratch + o_nodes);
    G.xp = reinterpret_cast<const double *>(scratch + o_xp);
    G.rank_of = reinterpret_cast<const int *>(scratch + o_rank);
    G.pend = reinterpret_cast<uint32_t *>(scratch + o_pend);
    G.blocker = reinterpret_cast<int *>(scratch + o_blocker);
    G.done = scratch + o_done;
    G.win0 = reinterpret_cast<int *>(scratch + o_w0);
    G.win1 = reinterpret_cast<int *>(scratch + o_w1);
    G.ok = scratch + o_ok;
    G.trylist = reinterpret_cast<int *>(scratch + o_try);
    DevPlan *d_plans = reinterpret_cast<DevPlan *>(scratch + o_plans);
    SgsCtl hc;
    memset(&hc, 0, sizeof(hc));
    hc.window = window;
    hc.total = nsim;
    CUDA_CHECK(cudaMemcpyAsync(G.ctl, &hc, sizeof(hc), cudaMemcpyHostToDevice, s));
    if (indicator)
        CUDA_CHECK(cudaMemcpyAsync(d_plans, cat_plans.data(), cat_plans.size() * sizeof(DevPlan),
                                   cudaMemcpyHostToDevice, s));
    if (nsim > 0) {
        CUDA_CHECK(cudaMemcpyAsync(scratch + o_nodes, path.nodes.data(), (size_t)nsim * 4, cudaMemcpyHostToDevice, s));
        CUDA_CHECK(cudaMemcpyAsync(scratch + o_xp, draws, (size_t)nsim * 8, cudaMemcpyHostToDevice, s));
    }
    CUDA_CHECK(cudaMemsetAsync(G.pend, 0, bits_bytes, s));
    CUDA_CHECK(cudaMemsetAsync(G.blocker, 0xff, (size_t)nsim * 4, s));
    CUDA_CHECK(cudaMemsetAsync(G.done, 0, (size_t)nsim, s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    res.ms_h2d = ms_since(t1);
    struct Events {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        ~Events() {
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        }
    } ev;
    CUDA_CHECK(cudaEventCreate(&ev.e0));
    CUDA_CHECK(cudaEventCreate(&ev.e1));
    CUDA_CHECK(cudaEventRecord(ev.e0, s));
    DevJob J = make_devjob(S, g);
    Counters *cnt = at<Counters>(S, S.ar.o_counters);
    CUDA_CHECK(cudaMemsetAsync(cnt, 0, sizeof(Counters), s));
    CUDA_CHECK(cudaMemsetAsync(J.nbcount, 0, (size_t)S.size * sizeof(int), s));
    launch_build_bits(J, g.dp, at<uint32_t>(S, g.o_bits), s);
    launch_sgs_ranks(J, G, nsim, s);
    long long round = 0;
    if (nsim > 0) {
        // every round commits at least the pending node of lowest rank
        launch_sgs_admit(J, g.dp, G, 1, s);
        int chunk = 4;
        long long committed = 0;
        for (;;) {
            for (int c = 0; c < chunk; ++c, ++round) {
                if (indicator) launch_sis_round(J, g.dp, d_plans, S.nmax_all <= 32 ? 0 : 1, G, (int)(round & 1), s);
                else launch_sgs_round(J, g.dp, G, (int)(round & 1), s);
            }
            CUDA_CHECK(cudaGetLastError());
            CUDA_CHECK(cudaMemcpyAsync(&hc, G.ctl, sizeof(hc), cudaMemcpyDeviceToHost, s));
            CUDA_CHECK(cudaStreamSynchronize(s));
            if (hc.next >= hc.total && hc.count[round & 1] == 0) break;
            // a round with pending nodes commits at least one of them
            if (hc.commits <= committed)
                throw HpglError{HPGL_E_INTERNAL, "sequential simulation made no progress in " +
                                                     std::to_string(chunk) + " rounds"};
            committed = hc.commits;
            chunk = std::min(chunk * 2, 64);
        }
    }
    CUDA_CHECK(cudaEventRecord(ev.e1, s));
    Counters hcnt;
    CUDA_CHECK(cudaMemcpyAsync(&hcnt, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    float ms = 0;
    cudaEventElapsedTime(&ms, ev.e0, ev.e1);
    res.ms_device = ms;
    if (hcnt.err)
        throw HpglError{HPGL_E_INTERNAL, "device invariant violated (error bits " + std::to_string(hcnt.err) + ")"};
    if (nsim > 0 && hc.commits != nsim)
        throw HpglError{HPGL_E_INTERNAL, "sequential simulation committed " + std::to_string(hc.commits) + " of " +
                                             std::to_string(nsim) + " nodes"};
    auto t2 = std::chrono::steady_clock::now();
    const size_t n = (size_t)S.size;
    if (indicator)
        CUDA_CHECK(cudaMemcpyAsync(res.out_codes, at<uint8_t>(S, S.ar.o_codes), n, cudaMemcpyDeviceToHost, s));
    else
        CUDA_CHECK(cudaMemcpyAsync(res.out_values, at<float>(S, S.ar.o_values), n * 4, cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaMemcpyAsync(res.out_mask, at<uint8_t>(S, S.ar.o_mask), n, cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    res.ms_d2h = ms_since(t2);
    res.systems = hc.tries;
    res.systems_fp64 = hc.tries;
    res.failures = 0;
    res.ms_total = ms_since(t0);
    res.rounds = hc.rounds;
}

static const char *top_kernel_name(int nmax, int precision, int schedule, const DevPlan &dp) {
    if (schedule == SCHED_FUSED) {
        if (nmax <= 32) return precision ? "k_fused32<1>" : "k_fused32<0>";
        return precision ? "k_fused64<1>" : "k_fused64<0>";
    }
    if (nmax <= 32) return precision ? mixed32_kernel_name(dp) : "k_solve_exact32";
    return precision ? "k_solve_mixed64" : "k_solve_exact64";
}

// The job's device pass captured once as a CUDA graph and replayed for every
// timed iteration: one launch per pass instead of one per kernel and memset.
struct PassGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~PassGraph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

static void capture_pass(JobState &S, cudaStream_t s, PassGraph &G) {
    CUDA_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    device_pass(S, s, nullptr, nullptr);
    CUDA_CHECK(cudaStreamEndCapture(s, &G.graph));
    CUDA_CHECK(cudaGraphInstantiate(&G.exec, G.graph, 0));
}

void bench_job(const hpgl_b200_job_t &job, hpgl_b200_result_t &res, hpgl_b200_bench_t &bench) {
    auto t0 = std::chrono::steady_clock::now();
    JobState S;
    prepare(S, job, res);
    bench.ms_plan = ms_since(t0);
    std::lock_guard<std::mutex> lock(g_sync_mutex);
    SyncContext &C = sync_ctx();
    sync_arena(C, S.ar.total);
    set_arena(S, C.arena);
    upload(S, C.stream);
    if (bench.flush_bytes > (long long)C.flush_cap) {
        if (C.flush) cudaFree(C.flush);
        C.flush = nullptr;
        C.flush_cap = 0;
        CUDA_CHECK(cudaMalloc(&C.flush, (size_t)bench.flush_bytes));
        C.flush_cap = (size_t)bench.flush_bytes;
    }
    CUDA_CHECK(cudaStreamSynchronize(C.stream));
    PassTiming pt;
    CUDA_CHECK(cudaEventCreate(&pt.search0));
    CUDA_CHECK(cudaEventCreate(&pt.top0));
    CUDA_CHECK(cudaEventCreate(&pt.top1));
    CUDA_CHECK(cudaEventCreate(&pt.resolve1));
    cudaEvent_t e0, e1;
    CUDA_CHECK(cudaEventCreate(&e0));
    CUDA_CHECK(cudaEventCreate(&e1));
    // Phase times from eager passes (events between the launches), then the
    // timed iterations as graph replays.
    double top_sum = 0, search_sum = 0, resolve_sum = 0;
    const int phase_runs = std::max(1, std::min(bench.iters, 3));
    for (int it = 0; it < 1 + phase_runs; ++it) {
        if (bench.flush_bytes > 0)
            CUDA_CHECK(cudaMemsetAsync(C.flush, it & 0xff, (size_t)bench.flush_bytes, C.stream));
        device_pass(S, C.stream, &pt, nullptr);
        read_counters(S, C.stream);
        if (it == 0) continue;  // first use of every kernel
        float tms = 0, sms = 0, rms = 0;
        cudaEventElapsedTime(&tms, pt.top0, pt.top1);
        cudaEventElapsedTime(&sms, pt.search0, pt.top0);
        cudaEventElapsedTime(&rms, pt.top1, pt.resolve1);
        top_sum += tms;
        search_sum += sms;
        resolve_sum += rms;
    }
    PassGraph G;
    capture_pass(S, C.stream, G);
    Counters cnt{};
    for (int it = 0; it < bench.warmup + bench.iters; ++it) {
        if (bench.flush_bytes > 0)
            CUDA_CHECK(cudaMemsetAsync(C.flush, it & 0xff, (size_t)bench.flush_bytes, C.stream));
        CUDA_CHECK(cudaEventRecord(e0, C.stream));
        CUDA_CHECK(cudaGraphLaunch(G.exec, C.stream));
        CUDA_CHECK(cudaEventRecord(e1, C.stream));
        cnt = read_counters(S, C.stream);
        if (it >= bench.warmup) {
            float ms = 0;
            cudaEventElapsedTime(&ms, e0, e1);
            if (bench.ms_per_iter) bench.ms_per_iter[it - bench.warmup] = ms;
        }
    }
    bench.ms_top_kernel = top_sum / phase_runs;
    bench.ms_search = search_sum / phase_runs;
    bench.ms_resolve = resolve_sum / phase_runs;
    snprintf(bench.top_kernel, sizeof(bench.top_kernel), "%s",
             S.cok ? "k_cokriging"
                   : top_kernel_name(S.nmax_all, S.precision,
                                     tuning_get(tuning_family(S.nmax_all), S.precision).schedule, S.groups[0].dp));
    bench.launches_per_iter = pt.launches;
    cudaEventDestroy(pt.search0);
    cudaEventDestroy(pt.top0);
    cudaEventDestroy(pt.top1);
    cudaEventDestroy(pt.resolve1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    download(S, res, cnt, C.stream);
    bench.systems = res.systems;
    bench.systems_fp64 = res.systems_fp64;
}

// Autotuner: times the job's device pass (after an L2 flush, median of
// three) under each candidate launch setting of the job's family and
// precision -- separate or fused schedule, persistent blocks per SM from
// "as many as fit" down -- and keeps the fastest in the tuning table, which
// every later pass of that family and precision uses.
void autotune_job(const hpgl_b200_job_t &job, hpgl_b200_tune_t &rep) {
    hpgl_b200_result_t res;
    memset(&res, 0, sizeof(res));
    std::vector<float> outv;
    std::vector<uint8_t> outc, outm;
    const size_t size = (size_t)job.nx * job.ny * job.nz;
    outm.assign(job.mask, job.mask + size);
    if (kind_is_cont(job.kind)) {
        outv.assign(job.values, job.values + size);
        res.out_values = outv.data();
    } else {
        outc.assign(job.codes, job.codes + size);
        res.out_codes = outc.data();
    }
    res.out_mask = outm.data();
    JobState S;
    prepare(S, job, res);
    std::lock_guard<std::mutex> lock(g_sync_mutex);
    SyncContext &C = sync_ctx();
    sync_arena(C, S.ar.total);
    set_arena(S, C.arena);
    upload(S, C.stream);
    const size_t flush = 256u << 20;
    if (C.flush_cap < flush) {
        if (C.flush) cudaFree(C.flush);
        C.flush = nullptr;
        C.flush_cap = 0;
        CUDA_CHECK(cudaMalloc(&C.flush, flush));
        C.flush_cap = flush;
    }
    const int family = tuning_family(S.nmax_all), precision = S.precision;
    const LaunchTuning before = tuning_get(family, precision);
    const int sched[] = {SCHED_FUSED, SCHED_SPLIT};
    const int bps[] = {0, 4, 3, 2};
    cudaEvent_t e0, e1;
    CUDA_CHECK(cudaEventCreate(&e0));
    CUDA_CHECK(cudaEventCreate(&e1));
    rep.candidates = 0;
    rep.chosen = -1;
    double best = 1e300;
    try {
        for (int sc : sched) {
            for (int b : bps) {
                if (rep.candidates >= HPGL_B200_TUNE_MAX) break;
                LaunchTuning t;
                t.schedule = sc;
                t.blocks_per_sm = b;
                tuning_set(family, precision, t);
                device_pass(S, C.stream, nullptr, nullptr);  // warm-up
                read_counters(S, C.stream);
                float runs[3];
                for (float &r : runs) {
                    CUDA_CHECK(cudaMemsetAsync(C.flush, 0, flush, C.stream));
                    CUDA_CHECK(cudaEventRecord(e0, C.stream));
                    device_pass(S, C.stream, nullptr, nullptr);
                    CUDA_CHECK(cudaEventRecord(e1, C.stream));
                    read_counters(S, C.stream);
                    cudaEventElapsedTime(&r, e0, e1);
                }
                std::sort(runs, runs + 3);
                const int i = rep.candidates++;
                rep.schedule[i] = sc;
                rep.blocks_per_sm[i] = b;
                rep.ms[i] = runs[1];
                if (runs[1] < best) {
                    best = runs[1];
                    rep.chosen = i;
                }
            }
        }
    } catch (...) {
        tuning_set(family, precision, before);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    LaunchTuning t;
    t.schedule = rep.schedule[rep.chosen];
    t.blocks_per_sm = rep.blocks_per_sm[rep.chosen];
    tuning_set(family, precision, t);
    rep.family = family;
    rep.precision = precision;
}

// ---- server: continuous batching ----------------------------------------------
//
// Each submitted job is planned on a host worker, then waits for admission:
// a free stream slot and room in the HBM budget for its arena.  Admitted jobs
// run concurrently, each on its own stream with an arena from the
// stream-ordered pool, so work from jobs that arrive while others are on the
// GPU overlaps on the device; finishing jobs return their memory and slot and
// the next waiting job is admitted at once.  Results are exactly those of
// hpgl_b200_krige on the same job (the kernels share nothing across jobs).

struct ServerJob {
    long long ticket;
    hpgl_b200_job_t job;
    std::vector<hpgl_ik_params_t> params;
    hpgl_b200_result_t *result;
    std::chrono::steady_clock::time_point submitted;
    bool done = false;
    int code = HPGL_OK;
    std::string message;
    double latency_ms = 0;
    double plan_ms = 0, wait_ms = 0, run_ms = 0;
};

struct Server {
    long long budget;
    int max_inflight;
    std::vector<cudaStream_t> streams;
    std::vector<int> free_slots;
    long long in_use = 0;
    long long peak_bytes = 0;
    int inflight = 0;
    int peak_inflight = 0;
    std::mutex mu;
    std::condition_variable cv_admit;
    std::condition_variable cv_done;
    std::deque<std::shared_ptr<ServerJob>> queue;
    std::vector<std::shared_ptr<ServerJob>> all;
    std::vector<std::thread> workers;
    bool stopping = false;
    long long next_ticket = 0;
    long long systems_done = 0;
    std::chrono::steady_clock::time_point first_submit, last_done;
    bool any_submit = false;
    int device = 0;
    std::atomic<int> planners{0};  // jobs being planned on the host right now

    // Planned jobs waiting for admission.  Among those that fit (a free slot,
    // room in the budget) the one with the least estimated device work goes
    // first -- small jobs do not queue behind large ones, which keeps the
    // median latency low when jobs arrive faster than the GPU finishes
    // them -- except that a job waiting longer than AGE_MS goes before all
    // younger ones (oldest first), so large jobs are not held back for good.
    struct Waiter {
        long long ticket;
        double cost;
        std::chrono::steady_clock::time_point since;
        long long bytes;
    };
    static constexpr double AGE_MS = 2000.0;
    std::vector<Waiter *> waiting;
    bool first_to_admit(const Waiter &w) const {
        const auto now = std::chrono::steady_clock::now();
        auto aged = [&](const Waiter *x) {
            return std::chrono::duration<double, std::milli>(now - x->since).count() >= AGE_MS;
        };
        for (const Waiter *o : waiting) {
            if (o == &w || in_use + o->bytes > budget) continue;
            const bool ao = aged(o), aw = aged(&w);
            if (ao != aw) {
                if (ao) return false;
                continue;
            }
            if (ao ? (o->since < w.since || (o->since == w.since && o->ticket < w.ticket))
                   : (o->cost < w.cost || (o->cost == w.cost && o->ticket < w.ticket)))
                return false;
        }
        return true;
    }

    void worker_loop();
    void run_one(const std::shared_ptr<ServerJob> &sj);
};

// Estimated device work of a planned job: its systems times the square of
// the neighbour count (the solves' cost grows with N^2 to N^3, the searches
// with N), per category group.
static double job_cost(const JobState &S) {
    double c = 0;
    for (const auto &g : S.groups) c += (double)S.kriged * (double)g.plan.nmax * (double)g.plan.nmax;
    return c;
}

void Server::run_one(const std::shared_ptr<ServerJob> &sj) {
    JobState S;
    int slot = -1;
    long long bytes = 0;
    try {
        CUDA_CHECK(cudaSetDevice(device));
        const auto t_plan = std::chrono::steady_clock::now();
        // the jobs planning at the same time share the host threads
        {
            const int planning = ++planners;
            struct Leave {
                std::atomic<int> &n;
                ~Leave() { --n; }
            } leave{planners};
            prepare(S, sj->job, *sj->result, std::max(1, host_threads() / planning));
        }
        sj->plan_ms = ms_since(t_plan);
        bytes = (long long)S.ar.total;
        if (bytes > budget)
            throw HpglError{HPGL_E_CAPACITY, "job needs " + std::to_string(bytes) +
                                                 " bytes of device memory, above the server's budget of " +
                                                 std::to_string(budget)};
        const auto t_wait = std::chrono::steady_clock::now();
        {
            std::unique_lock<std::mutex> l(mu);
            Waiter w{sj->ticket, job_cost(S), t_wait, bytes};
            waiting.push_back(&w);
            cv_admit.wait(l, [&] {
                return stopping || (!free_slots.empty() && in_use + bytes <= budget && first_to_admit(w));
            });
            waiting.erase(std::find(waiting.begin(), waiting.end(), &w));
            if (stopping) throw HpglError{HPGL_E_INTERNAL, "server stopped"};
            slot = free_slots.back();
            free_slots.pop_back();
            in_use += bytes;
            peak_bytes = std::max(peak_bytes, in_use);
            ++inflight;
            peak_inflight = std::max(peak_inflight, inflight);
            cv_admit.notify_all();  // the next waiter may fit too
        }
        sj->wait_ms = ms_since(t_wait);
        const auto t_run = std::chrono::steady_clock::now();
        cudaStream_t s = streams[slot];
        void *arena = nullptr;
        CUDA_CHECK(cudaMallocAsync(&arena, S.ar.total, s));
        set_arena(S, (char *)arena);
        try {
            upload(S, s);
            hpgl_b200_result_t &res = *sj->result;
            const bool want_nb = res.nb_count || res.nb_index;
            device_pass(S, s, nullptr, [&](const Group &g) {
                if (want_nb) download_neighbours(S, g, res, s);
            });
            Counters cnt = read_counters(S, s);
            download(S, *sj->result, cnt, s);
        } catch (...) {
            cudaFreeAsync(arena, s);
            cudaStreamSynchronize(s);
            throw;
        }
        CUDA_CHECK(cudaFreeAsync(arena, s));
        CUDA_CHECK(cudaStreamSynchronize(s));
        sj->run_ms = ms_since(t_run);
    } catch (const HpglError &e) {
        sj->code = e.code;
        sj->message = e.message;
    } catch (const std::exception &e) {
        sj->code = HPGL_E_INTERNAL;
        sj->message = e.what();
    }
    std::lock_guard<std::mutex> l(mu);
    if (slot >= 0) {
        free_slots.push_back(slot);
        in_use -= bytes;
        --inflight;
    }
    sj->done = true;
    sj->latency_ms = ms_since(sj->submitted);
    if (sj->code == HPGL_OK) systems_done += sj->result->systems;
    last_done = std::chrono::steady_clock::now();
    cv_admit.notify_all();
    cv_done.notify_all();
}

void Server::worker_loop() {
    while (true) {
        std::shared_ptr<ServerJob> sj;
        {
            std::unique_lock<std::mutex> l(mu);
            cv_admit.wait(l, [&] { return stopping || !queue.empty(); });
            if (queue.empty()) return;
            sj = queue.front();
            queue.pop_front();
        }
        run_one(sj);
    }
}

void *server_create(const hpgl_b200_server_config_t &cfg) {
    ensure_device();
    if (cfg.hbm_budget_bytes <= 0) invalid("hbm_budget_bytes must be positive");
    if (cfg.max_inflight < 1 || cfg.max_inflight > 64) invalid("max_inflight must be in [1, 64]");
    auto *sv = new Server();
    sv->budget = cfg.hbm_budget_bytes;
    sv->max_inflight = cfg.max_inflight;
    cudaGetDevice(&sv->device);
    // Keep freed arenas in the pool up to the budget, so admission does not
    // return memory to the driver and fetch it again.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, sv->device) == cudaSuccess) {
        unsigned long long thr = (unsigned long long)cfg.hbm_budget_bytes;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    for (int i = 0; i < cfg.max_inflight; ++i) {
        cudaStream_t s;
        CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        sv->streams.push_back(s);
        sv->free_slots.push_back(i);
    }
    int workers = cfg.worker_threads > 0 ? cfg.worker_threads : cfg.max_inflight * 2;
    for (int i = 0; i < workers; ++i) sv->workers.emplace_back([sv] { sv->worker_loop(); });
    return sv;
}

long long server_submit(void *h, const hpgl_b200_job_t &job, hpgl_b200_result_t *result) {
    auto *sv = (Server *)h;
    if (!result) invalid("result is null");
    if (!job.params || job.n_params < 1 || job.n_params > 255) invalid("params missing");
    auto sj = std::make_shared<ServerJob>();
    sj->job = job;
    sj->params.assign(job.params, job.params + job.n_params);
    sj->job.params = sj->params.data();
    sj->result = result;
    sj->submitted = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> l(sv->mu);
    if (!sv->any_submit) {
        sv->any_submit = true;
        sv->first_submit = sj->submitted;
    }
    sj->ticket = sv->next_ticket++;
    sv->all.push_back(sj);
    sv->queue.push_back(sj);
    sv->cv_admit.notify_all();
    return sj->ticket;
}

int server_wait(void *h, long long ticket, int timeout_ms, std::string &message) {
    auto *sv = (Server *)h;
    std::unique_lock<std::mutex> l(sv->mu);
    if (ticket < 0 || ticket >= (long long)sv->all.size()) invalid("unknown ticket");
    auto sj = sv->all[ticket];
    auto ready = [&] { return sj->done; };
    if (timeout_ms < 0) sv->cv_done.wait(l, ready);
    else if (!sv->cv_done.wait_for(l, std::chrono::milliseconds(timeout_ms), ready)) return -1;
    message = sj->message;
    return sj->code;
}

void server_stats(void *h, hpgl_b200_server_stats_t &st) {
    auto *sv = (Server *)h;
    std::lock_guard<std::mutex> l(sv->mu);
    std::vector<double> lat;
    long long failed = 0, completed = 0;
    double plan = 0, wait = 0, run = 0;
    for (auto &sj : sv->all) {
        if (!sj->done) continue;
        ++completed;
        if (sj->code != HPGL_OK) {
            ++failed;
        } else {
            lat.push_back(sj->latency_ms);
            plan += sj->plan_ms;
            wait += sj->wait_ms;
            run += sj->run_ms;
        }
    }
    std::sort(lat.begin(), lat.end());
    auto pct = [&](double q) {
        if (lat.empty()) return 0.0;
        long long i = (long long)std::ceil(q * (double)lat.size()) - 1;
        if (i < 0) i = 0;
        if (i >= (long long)lat.size()) i = (long long)lat.size() - 1;
        return lat[i];
    };
    double sum = 0;
    for (double v : lat) sum += v;
    st.submitted = (long long)sv->all.size();
    st.completed = completed;
    st.failed = failed;
    st.systems = sv->systems_done;
    st.p50_ms = pct(0.50);
    st.p99_ms = pct(0.99);
    st.mean_ms = lat.empty() ? 0 : sum / lat.size();
    st.wall_s = sv->any_submit && completed ? std::chrono::duration<double>(sv->last_done - sv->first_submit).count()
                                            : 0;
    st.systems_per_s = st.wall_s > 0 ? sv->systems_done / st.wall_s : 0;
    st.peak_inflight = sv->peak_inflight;
    st.peak_bytes = sv->peak_bytes;
    const double nok = lat.empty() ? 1.0 : (double)lat.size();
    st.mean_plan_ms = plan / nok;
    st.mean_wait_ms = wait / nok;
    st.mean_run_ms = run / nok;
}

void server_destroy(void *h) {
    auto *sv = (Server *)h;
    {
        std::unique_lock<std::mutex> l(sv->mu);
        sv->cv_done.wait(l, [&] {
            for (auto &sj : sv->all)
                if (!sj->done) return false;
            return true;
        });
        sv->stopping = true;
        sv->cv_admit.notify_all();
    }
    for (auto &t : sv->workers) t.join();
    for (auto s : sv->streams) cudaStreamDestroy(s);
    delete sv;
}

}  // namespace hpgl_b200
