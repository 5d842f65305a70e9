// Device-side data of one kriging pass and the kernel launchers.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace hpgl_b200 {

enum Status : int8_t { ST_SUCCESS = 0, ST_NO_NEIGHBOURS = 1, ST_SINGULAR = 2, ST_NOT_KRIGED = -1 };

// Error bits raised by kernels (never expected; each names a broken
// invariant so the host can report it instead of returning wrong results).
enum DevError : int {
    DERR_TABLE_RANGE = 1,      // a covariance offset fell outside the table
    DERR_CAND_CAPACITY = 2,    // clusterizer candidates exceeded the scratch
    DERR_SORT_STACK = 4,
};

struct DevPlan {
    int nmax;
    // template
    const int4 *tmpl;        // (packed window offset, dy, dz, node delta)
    int tmpl_len;
    int px, nseg, wpr;
    // covariance table
    const double *table;
    int Bx, By, Bz;
    int Tx, Ty, Tz;          // half extents read from the table (beyond: 0)
    int sx, syx;             // table strides (x, then y*x)
    int center;              // table index of offset 0
    int truncated;           // beyond T is the model's 0 (else a broken invariant)
    double c0;
    // clusterizer
    const int *bucket_start;
    const int *bucket_nodes;
    const uint8_t *bucket_clean;
    double crx, cry, crz;
    int mx, my, mz;
    int max_candidates;
};

// Division by a runtime-invariant divisor d >= 1 of any n < 2^32 with one
// multiply-high: t = umulhi(m, n), n / d = (t + ((n - t) >> 1)) >> (l - 1),
// where l = ceil(log2 d) and m = floor(2^32 (2^l - d) / d) + 1 (Granlund and
// Montgomery, "Division by invariant integers using multiplication", PLDI
// 1994, the variant with the 33-bit multiplier's top bit folded into the
// add).  d = 1 (l = 0) returns n.  tests/cpp/fastdiv_check.cpp checks it
// against integer division.
struct FastDiv {
    unsigned d = 1, m = 0;
    int l = 0;
    FastDiv() = default;
    explicit FastDiv(unsigned dv) : d(dv) {
        while ((1ull << l) < dv) ++l;
        m = (unsigned)((((unsigned long long)1 << 32) * (((unsigned long long)1 << l) - dv)) / dv + 1);
    }
#ifdef __CUDACC__
    __host__ __device__ __forceinline__ unsigned div(unsigned n) const {
#ifdef __CUDA_ARCH__
        const unsigned t = __umulhi(m, n);
#else
        const unsigned t = (unsigned)(((unsigned long long)m * n) >> 32);
#endif
        return l == 0 ? n : (t + ((n - t) >> 1)) >> (l - 1);
    }
#else
    unsigned div(unsigned n) const {
        const unsigned t = (unsigned)(((unsigned long long)m * n) >> 32);
        return l == 0 ? n : (t + ((n - t) >> 1)) >> (l - 1);
    }
#endif
};

struct DevJob {
    int kind;
    int nx, ny, nz;
    FastDiv div_nx, div_ny;  // node index -> (x, y, z)
    long long size;
    const float *values;
    const uint8_t *codes;
    const uint8_t *mask;
    const float *mean;
    const uint32_t *bits;    // padded informed-bit rows
    // categories: this pass computes probabilities of categories [k0, k1)
    int K, k0, k1;
    const float *pk;         // IK marginal probabilities (float) per category
    float sk_mean_f;         // SK mean as the float the combiner sees
    float median_m;          // median IK (float)marginal_probs[1]
    // neighbour lists
    int *nb;                 // [size][nmax]
    int *nbcount;            // [size]
    // outputs
    float *out_values;
    uint8_t *out_codes;
    uint8_t *out_mask;
    double *variance;        // optional
    int8_t *status;          // [size] (or [size*K] for per-category IK)
    float *probs;            // IK [size*K], median IK [size]
    double *weights;         // optional [size][nmax]
    int status_stride;       // 1, or K for per-category IK
    int status_offset;       // category for per-category IK
    // untouched nodes (ordinary kriging failures keep the caller's content)
    int *untouched;
    int *n_untouched;
    // mixed precision routing; the job-level tally of attempts (AttemptTally)
    uint8_t *routed;         // per node: routed to the FP64 re-solve
    int *n_routed;
    int *n_attempt;
    int *n_attempt_routed;
    int *abandon;            // set: the re-solve runs the plain FP64 pass
    int *seg_next;           // template search: the next 32-node segment to take
    int *node_next;          // clusterizer search: the next chunk of nodes to take
    // counters
    unsigned long long *n_fp64;
    int *err;
    // colocated cokriging (kinds 5, 6)
    const float *svalues;        // secondary property
    const uint8_t *smask;
    const double *cross_table;   // covariance of the cross model, laid out like DevPlan::table
    double cok_coef;             // cross covariance = coef * cross_table
    double cok_svar;             // secondary variance (the system's corner)
    float cok_m1, cok_m2;        // primary and secondary means (float, mean_t)
    // sequential simulation: the property, its mask and the informed bits,
    // written as nodes are simulated (the same buffers as values / mask /
    // bits)
    float *sim_values;
    uint8_t *sim_mask;
    uint32_t *sim_bits;
    // sequential indicator simulation: the codes written as nodes are
    // simulated (the same buffer as codes), per-category mean cubes in
    // `mean` (K x size) instead of pk, the correlogram weights, and the
    // stride of the neighbour lists (the largest max_neighbours)
    uint8_t *sim_codes;
    int sis_lvm;
    int sis_corr;
    int nb_stride;
};

// Launch tuning of the per-node kernels: the schedule (separate template
// search and solve, or the fused kernel) and the number of persistent blocks
// per SM (0 = as many as fit).  One setting per (family, precision), family
// 0 for max_neighbours <= 32 and 1 above; the autotuner (engine.cu) fills
// the table, the launchers read it.
enum Schedule : int { SCHED_SPLIT = 0, SCHED_FUSED = 1 };
struct LaunchTuning {
    int schedule = SCHED_SPLIT;
    int blocks_per_sm = 0;
};
LaunchTuning tuning_get(int family, int precision);
void tuning_set(int family, int precision, const LaunchTuning &t);
inline int tuning_family(int nmax) { return nmax <= 32 ? 0 : 1; }
// grid for a persistent kernel: min(units, SMs x min(blocks_per_sm, occupancy))
long long persistent_grid(const void *fn, int threads, size_t smem, int blocks_per_sm, long long units);

// Launchers (stream-ordered, no synchronisation).
void launch_build_bits(const DevJob &J, const DevPlan &P, uint32_t *bits, cudaStream_t s);
void launch_search_template(const DevJob &J, const DevPlan &P, cudaStream_t s);
void launch_search_cluster(const DevJob &J, const DevPlan &P, double *scratch_key, int *scratch_idx,
                           int n_warps, cudaStream_t s);
// precision: 0 exact FP64, 1 FP32 + FP64 refinement (flags J.routed).
// routed: optional per-node flags (the routed re-solve: the flagged nodes in
// node order, every node once the job is abandoned); else every node.
void launch_solve(const DevJob &J, const DevPlan &P, int precision, const uint8_t *routed, cudaStream_t s,
                  int blocks_per_sm = 0);
void launch_ik_argmax(const DevJob &J, cudaStream_t s);
// cokriging.cu: colocated simple cokriging of every node (after the template search)
void launch_cokriging(const DevJob &J, const DevPlan &P, cudaStream_t s);
// Sequential simulation in speculative rounds.  The path's nodes enter, in
// path order, a window of pending nodes.  Each round krigs pending nodes
// from the committed nodes of lower path rank (informed bits, rank_of); a
// node commits unless the part of its search template that the search read
// holds a pending node of lower rank -- a committed node has then seen
// exactly the nodes the sequential order gives it, so the result is the
// sequential one.  A node that did not commit records that pending node
// (its blocker) and is not tried again before the blocker commits.  The
// pending node of lowest rank always commits, so every round makes progress.
struct SgsCtl {
    int count[2];           // pending nodes in window buffer 0 / 1
    int window;             // window size (pending nodes per round)
    unsigned blocks_done;   // commit kernel: blocks finished
    unsigned cursor;        // try kernels: next entry of the try list to hand out
    int ntry;               // entries of this round's try list
    long long next;         // next path rank to admit
    long long total;        // path length
    long long admit_base;   // window slot of the first admitted node
    long long admit;        // nodes admitted by the pending admission
    long long rounds, tries, commits;
};
struct SgsState {
    SgsCtl *ctl;
    const int *nodes;       // path order
    const double *xp;       // per path rank: the draw's standard normal quantile
    const int *rank_of;     // per node: -1 informed, path rank, or INT_MAX
    uint32_t *pend;         // pending bits, laid out like the informed bits
    int *blocker;           // per path rank: the pending rank that blocked it, or -1
    uint8_t *done;          // per path rank: committed
    int *win0, *win1;       // window buffers (path ranks)
    uint8_t *ok;            // per window slot: the node committed this round
    int *trylist;           // window slots tried this round (blocker committed or none)
};
// rank_of from the mask and the path
void launch_sgs_ranks(const DevJob &J, const SgsState &G, long long nsim, cudaStream_t s);
// one round: list the pending nodes of window buffer `cur` to try, try them,
// commit, admit
void launch_sgs_round(const DevJob &J, const DevPlan &P, const SgsState &G, int cur, cudaStream_t s);
void launch_sgs_try32(const DevJob &J, const DevPlan &P, const SgsState &G, int cur, cudaStream_t s);
void launch_sgs_try64(const DevJob &J, const DevPlan &P, const SgsState &G, int cur, cudaStream_t s);
// the first admission (window buffer 0 from an empty buffer 1)
void launch_sgs_admit(const DevJob &J, const DevPlan &P, const SgsState &G, int cur, cudaStream_t s);
// sequential indicator simulation: one round over window buffer `cur` with
// the categories' plans (device array of K); family 0 when every category
// has at most 32 neighbours
void launch_sis_round(const DevJob &J, const DevPlan &P0, const DevPlan *plans, int family, const SgsState &G,
                      int cur, cudaStream_t s);
void launch_sis_try32(const DevJob &J, const DevPlan *plans, const SgsState &G, int cur, cudaStream_t s);
void launch_sis_try64(const DevJob &J, const DevPlan *plans, const SgsState &G, int cur, cudaStream_t s);
// solve32.cu: the mixed-precision kernel launch_solve32 runs for plan P
const char *mixed32_kernel_name(const DevPlan &P);
// solve32.cu: register-resident solves for max_neighbours <= 32
void launch_solve32(const DevJob &J, const DevPlan &P, int precision, const uint8_t *routed, cudaStream_t s,
                    int blocks_per_sm);
// solve64.cu: solves for 33..64 neighbours (exact FP64; FP32 inverse + FP64
// refinement, routing to `routed`)
void launch_solve64_exact(const DevJob &J, const DevPlan &P, const uint8_t *routed, cudaStream_t s,
                          int blocks_per_sm);
void launch_solve64_mixed(const DevJob &J, const DevPlan &P, cudaStream_t s, int blocks_per_sm);
// Fused template search + solve of every node (the clusterizer search runs
// first); precision 0 exact FP64, 1 mixed.
void launch_fused32(const DevJob &J, const DevPlan &P, int precision, cudaStream_t s, int blocks_per_sm);
void launch_fused64(const DevJob &J, const DevPlan &P, int precision, cudaStream_t s, int blocks_per_sm);

}  // namespace hpgl_b200
