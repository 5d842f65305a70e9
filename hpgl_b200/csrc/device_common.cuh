// Device helpers shared by the kernel files.
#pragma once
#include <cstdint>

#include "kernels.cuh"

namespace hpgl_b200 {

#define FULL_MASK 0xffffffffu

// kinds with a continuous property: OK, SK, LVM and the two cokriging kinds
__device__ __forceinline__ bool is_cont(int kind) { return kind <= 2 || kind == 5 || kind == 6; }

// Covariance of offset v (grid steps) from the plan's table.  Truncated kinds
// read 0 beyond the search radii (precalculated_covariance.h:60-75,
// covariance_field.h:144-153); the table box covers every offset the search
// can produce, anything else is a broken invariant.
// For truncated kinds T = min(radii, B) and every |v| <= n-1 <= B, so the
// table covers all in-radius offsets; for ordinary kriging T = B covers
// every offset the search produces (an offset beyond it raises an error bit).
__device__ __forceinline__ bool cov_in_range(const DevPlan &P, int vx, int vy, int vz) {
    return (unsigned)(vx + P.Tx) <= (unsigned)(2 * P.Tx) && (unsigned)(vy + P.Ty) <= (unsigned)(2 * P.Ty) &&
           (unsigned)(vz + P.Tz) <= (unsigned)(2 * P.Tz);
}

// lin = vz*syx + vy*sx + vx, the table offset of v relative to its centre.
__device__ __forceinline__ double cov_lin(const DevPlan &P, int vx, int vy, int vz, int lin, int *err) {
    if (!cov_in_range(P, vx, vy, vz)) {
        if (!P.truncated) atomicOr(err, DERR_TABLE_RANGE);
        return 0.0;
    }
    return __ldg(P.table + (P.center + lin));
}

__device__ __forceinline__ double cov_at(const DevPlan &P, int vx, int vy, int vz, int *err) {
    return cov_lin(P, vx, vy, vz, vz * P.syx + vy * P.sx + vx, err);
}

// Node coordinates, sugarbox_grid.cpp:70-74 (x = idx % nx, y = idx % (nx ny) / nx,
// z = idx / (nx ny)), with the two divisions by multiply-high.
__device__ __forceinline__ void node_xyz(const DevJob &J, int idx, int &x, int &y, int &z) {
    const unsigned r = J.div_nx.div((unsigned)idx);
    const unsigned q = J.div_ny.div(r);
    x = idx - (int)r * J.nx;
    y = (int)r - (int)q * J.ny;
    z = (int)q;
}

// A node takes the template walk when any of its 27 neighbouring clusterizer
// boxes overflowed (sugarbox_indexed_neighbour_lookup.h:68-71).
__device__ __forceinline__ bool node_clean(const DevPlan &P, int x, int y, int z) {
    int cx = (int)(x / P.crx), cy = (int)(y / P.cry), cz = (int)(z / P.crz);
    return P.bucket_clean[((long long)cz * P.my + cy) * P.mx + cx] != 0;
}

__device__ __forceinline__ bool node_needs_kriging(const DevJob &J, int node) {
    return is_cont(J.kind) ? J.mask[node] == 0 : true;
}

// Correctly rounded quotient a / b from y = RN(1/b): q = RN(a*y) is within
// one ulp of a/b, r = a - b*q is exact in one fused multiply-add, and
// RN(q + r*y) is the correctly rounded quotient (Markstein's theorem, IBM J.
// Res. Dev. 34(1), 1990, for round-to-nearest binary arithmetic away from
// overflow and the subnormal range).  Bit-identical to __ddiv_rn on the
// kriging systems' magnitudes; tests/test_division.py checks it against
// __ddiv_rn on the GPU.
__device__ __forceinline__ double div_by_rcp(double a, double b, double y) {
    const double q = __dmul_rn(a, y);
    const double r = __fma_rn(-q, b, a);
    return __fma_rn(r, y, q);
}

// The first loads of a node, issued one node ahead by the persistent loops
// (the neighbour count, the lane's neighbour cells -- rows lane and lane + 32
// -- and the informed flag start a chain of dependent loads; issuing them
// while the previous system is solved hides that latency).  Plain loads: the
// fused kernels read lists their own warp has just written.
struct NodeFetch {
    int node;  // -1: past the end
    int n;
    int cell, cell2;
    bool informed;
};

__device__ __forceinline__ NodeFetch fetch_node(const DevJob &J, const DevPlan &P, int node, int lane) {
    NodeFetch f;
    f.node = node;
    f.n = 0;
    f.cell = 0;
    f.cell2 = 0;
    f.informed = false;
    if (node >= 0) {
        f.n = J.nbcount[node];
        const int *lst = J.nb + (long long)node * P.nmax;
        if (lane < P.nmax) f.cell = lst[lane];
        if (lane + 32 < P.nmax) f.cell2 = lst[lane + 32];
        f.informed = is_cont(J.kind) && __ldg(J.mask + node) != 0;
    }
    return f;
}

// Acceptance of an iterative refinement x <- x + d.  After a correction d_k
// the remaining error is about rho_k |d_k|, with the contraction rho_k =
// |d_k| / |d_{k-1}| (for the first correction |d_0| / |x|, the error it
// removed being about |x|).  A solution is accepted once that estimate is
// below REFINE_TOL |x| (max norms), so what is accepted is converged to near
// FP64 accuracy; a refinement that contracts by less than REFINE_RHO_MAX per
// step is not going to get there and is routed at once.
constexpr double REFINE_TOL = 1e-13;
constexpr double REFINE_RHO_MAX = 0.5;

struct RefineGate {
    double prev = -1.0;
    // +1 accept, -1 route, 0 correct again
    __device__ __forceinline__ int step(double dmax, double xmax) {
        const double rho = prev < 0.0 ? dmax / xmax : dmax / prev;
        prev = dmax;
        if (!(xmax > 0.0)) return dmax == 0.0 ? 1 : -1;
        if (rho * dmax <= REFINE_TOL * xmax) return 1;
        if (!(rho <= REFINE_RHO_MAX)) return -1;
        return 0;
    }
};

// Per-warp guess of whether the mixed path will route a system.  A system
// the FP32 factorisation or the refinement cannot take costs the FP32
// attempt and then the FP64 re-solve, so where most systems are routed
// (ill-conditioned models, clustered data) attempting loses to the FP64
// path alone.  A warp keeps an average of its recent attempts' outcomes
// (weight 1/4 for the newest); below `keep` it stops attempting and routes its
// systems straight to the FP64 re-solve, attempting every 8th again to
// notice when its nodes become well conditioned.  A kernel that hands out
// its nodes dynamically restarts the guess with every chunk of consecutive
// nodes, so the choice depends on the chunk's nodes only and is the same on
// every run; routed systems get the FP64 path's results, which the mixed
// results match within their tolerance either way.
// A kernel passes the success share below which attempting stops paying:
// an attempt costs about c of an FP64 solve and saves one when it succeeds,
// so it pays while the share of successes exceeds c.
struct RouteGuess {
    float ok = 1.f;
    int skipped = 0;
    float keep;  // attempt while the recent success share is at least this
    __device__ explicit RouteGuess(float keep_) : keep(keep_) {}
    __device__ __forceinline__ bool attempt() {
        if (ok >= keep || skipped >= 7) {
            skipped = 0;
            return true;
        }
        ++skipped;
        return false;
    }
    // outcome: -1 no system, 0 solved, 1 routed
    __device__ __forceinline__ void record(bool attempted, int outcome) {
        if (attempted && outcome >= 0) ok = 0.75f * ok + (outcome == 0 ? 0.25f : 0.f);
    }
};

// Nodes a solve warp takes from the per-job counter at a time: up to `cap`,
// fewer on small jobs so that every warp of the grid still gets about 8
// chunks (the size depends only on the job and the launch).
__device__ __forceinline__ int chunk_nodes(const DevJob &J, int cap, int warps_per_block) {
    const long long c = J.size / ((long long)gridDim.x * warps_per_block * 8);
    return (int)(c < 1 ? 1 : (c > cap ? cap : c));
}

// Sends a node's system to the FP64 re-solve (one lane).
__device__ __forceinline__ void route(const DevJob &J, int node) {
    J.routed[node] = 1;
    atomicAdd(J.n_routed, 1);
}

// Job-level decision of the mixed path.  When most systems of a job are
// routed (an ill-conditioned model over the whole grid), the FP32 attempts
// are wasted and the re-solve is nearly the plain FP64 pass anyway.  The
// warps therefore add up their attempts and routed attempts every 16
// nodes; once at least ABANDON_MIN systems have been
// attempted and more than the kernel's `fraction` of them routed, the job is
// abandoned: the mixed kernel stops, and the re-solve kernel runs the plain
// FP64 pass over every node instead of the flagged ones (results of nodes
// the mixed kernel already solved are recomputed, so every result is the
// FP64 one).
//
// The break-even points, measured: a 32-row FP32 attempt costs about 0.42 of
// the exact 32-row solve (23.2 vs 54.8 ms over the SK 256x256x64 job), so
// attempts pay above 42 % successes (keep 0.5, abandon above 60 % routed);
// a 64-row attempt costs about 0.82 of the exact 64-row solve (the median
// over serving jobs of 38-60 neighbours with nothing routed), so they pay
// only above about 82 % successes (keep 0.85, abandon above 15 % routed).
constexpr int ABANDON_MIN = 4096;
constexpr float ROUTE_KEEP32 = 0.5f, ABANDON_FRACTION32 = 0.6f;
constexpr float ROUTE_KEEP64 = 0.85f, ABANDON_FRACTION64 = 0.15f;

struct AttemptTally {
    int att = 0, routed = 0, since = 0;
    float fraction;
    __device__ explicit AttemptTally(float fraction_) : fraction(fraction_) {}
    // after each node (outcome of mixed*_node, attempted or not); true once
    // the job is abandoned
    __device__ __forceinline__ bool step(const DevJob &J, bool attempted, int outcome, int lane) {
        if (attempted && outcome >= 0) {
            ++att;
            routed += outcome;
        }
        if (++since < 16) return false;
        since = 0;
        int flag = 0;
        if (lane == 0) {
            if (att) {
                const int a = atomicAdd(J.n_attempt, att) + att;
                const int r = atomicAdd(J.n_attempt_routed, routed) + routed;
                if (a >= ABANDON_MIN && (float)r > fraction * (float)a) atomicExch(J.abandon, 1);
            }
            flag = *reinterpret_cast<volatile int *>(J.abandon);
        }
        att = routed = 0;
        return __shfl_sync(FULL_MASK, flag, 0) != 0;
    }
};

}  // namespace hpgl_b200
