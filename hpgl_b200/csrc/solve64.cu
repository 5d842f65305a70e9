// Per-node solves for systems of 33 to 64 neighbours (one warp per system,
// persistent over the node list; lane l owns rows and columns l and l + 32).
//
//   k_solve_exact64  FP64 in the reference's exact operation order
//                    (my_kriging_weights.h:26-255 over LAPACK DPOTF2/DPOTRS,
//                    the same arithmetic as the 32-neighbour kernel).  The
//                    system and its factor live in a skewed packed upper
//                    triangle in shared memory: every lane reads its own
//                    columns as conflict-free 16-byte pairs while the column
//                    of the step is broadcast, and the forward substitution
//                    U^T y = b runs inside the factorisation (row j of U is
//                    final at step j, which is all the dot-product form of
//                    DTRSM needs).  The step loop is a plain runtime loop, so
//                    the kernel stays small for the instruction caches.
#include <algorithm>

#include "device_common.cuh"
#include "search_common.cuh"

namespace hpgl_b200 {

namespace {

constexpr int N64 = 64;

constexpr int WARPS64_BLOCK = 1;

// At most this many nodes a 64-row solve warp takes from the per-job counter at a time, and the
// taking itself (lane 0's atomic, broadcast).
constexpr int CHUNK64 = 16;
__device__ __forceinline__ int take_chunk64(const DevJob &J, int lane, int csize) {
    int c = 0;
    if (lane == 0) c = atomicAdd(J.node_next, csize);
    return __shfl_sync(FULL_MASK, c, 0);
}

// The factor lives in shared memory as a skewed packed upper triangle:
// column k starts at col_start(k), holds rows 0..k (padded to an even count)
// and col_start(k) = 2k (mod 16) doubles, so when every lane reads a 16-byte
// pair of its own column at the same row, the 32 addresses fall on 8
// different 16-byte bank groups, 4 each: conflict-free.  Column k is the
// matrix column A(., k) until its rows are overwritten, one per step, by the
// factor's row; its diagonal slot stays zero until step k.
// (col_start_c runs a loop: device code reads the starts from a table the
// kernels fill once per block.)
__host__ __device__ constexpr int col_start_c(int k) {
    int start = 0, end = 0;
    for (int c = 0; c <= k; ++c) {
        start = end;
        while ((start & 15) != ((2 * c) & 15)) ++start;
        end = start + ((c + 2) & ~1);
    }
    return start;
}
constexpr int U64_SIZE = col_start_c(N64 - 1) + N64;  // 2558 doubles
static_assert(col_start_c(3) == 22 && U64_SIZE == 2558, "skewed layout");

struct Exact64Smem {
    double U[U64_SIZE];
    int4 nb[N64];     // neighbour offsets from the node (x, y, z, table offset)
};

__device__ __noinline__ double dsqrt64(double a) { return __dsqrt_rn(a); }
__device__ __noinline__ double drcp64(double a) { return __drcp_rn(a); }

struct Node64 {
    int n;
    float dv[2];  // cont: value - mean (float, combiner.h:18-22)
    int code[2];  // IK: category code
    double b[2];  // C(x_row - x0)
};

__device__ __forceinline__ Node64 load_node64(const DevJob &J, const DevPlan &P, int4 *nb, const NodeFetch &f,
                                              int lane) {
    Node64 d;
    const int node = f.node;
    d.n = f.n;
    int x0, y0, z0;
    node_xyz(J, node, x0, y0, z0);
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int row = lane + 32 * r;
        d.dv[r] = 0.f;
        d.code[r] = -1;
        d.b[r] = 0.0;
        int4 o = make_int4(0, 0, 0, 0);
        if (row < d.n) {
            const int cell = r ? f.cell2 : f.cell;
            int qx, qy, qz;
            node_xyz(J, cell, qx, qy, qz);
            o.x = qx - x0;
            o.y = qy - y0;
            o.z = qz - z0;
            o.w = o.z * P.syx + o.y * P.sx + o.x;
            if (is_cont(J.kind)) {
                const float m = J.kind == 1 ? J.sk_mean_f : (J.kind == 2 ? J.mean[cell] : 0.f);
                d.dv[r] = __fsub_rn(J.values[cell], m);
            } else {
                d.code[r] = J.codes[cell];
            }
            d.b[r] = cov_lin(P, o.x, o.y, o.z, o.w, J.err);
        }
        nb[row] = o;
    }
    __syncwarp();
    return d;
}

// Value of row i (0..63) held as (v0 in lane i) / (v1 in lane i - 32).
template <typename T>
__device__ __forceinline__ T row_val(T v0, T v1, int i) {
    return i < 32 ? __shfl_sync(FULL_MASK, v0, i) : __shfl_sync(FULL_MASK, v1, i - 32);
}

// init + v_0 + v_1 + ... + v_{n-1} in row order (v_i held as v0 in lane i
// for i < 32, v1 in lane i - 32 above), float or double.
__device__ __forceinline__ float rows_fsum(float acc, float v0, float v1, int n) {
    const int n0 = n < 32 ? n : 32;
    for (int i = 0; i < n0; ++i) acc = __fadd_rn(acc, __shfl_sync(FULL_MASK, v0, i));
    for (int i = 32; i < n; ++i) acc = __fadd_rn(acc, __shfl_sync(FULL_MASK, v1, i - 32));
    return acc;
}
__device__ __forceinline__ double rows_dsum(double acc, double v0, double v1, int n) {
    const int n0 = n < 32 ? n : 32;
    for (int i = 0; i < n0; ++i) acc = __dadd_rn(acc, __shfl_sync(FULL_MASK, v0, i));
    for (int i = 32; i < n; ++i) acc = __dadd_rn(acc, __shfl_sync(FULL_MASK, v1, i - 32));
    return acc;
}

// Outputs of one solved (or failed) system, weights w0/w1 of rows lane and
// lane + 32; the same combination rules as the 32-neighbour kernels.
__device__ __forceinline__ void write_outputs64(const DevJob &J, const DevPlan &P, int node, int lane,
                                                const Node64 &d, int status, double w0, double w1,
                                                double variance) {
    const long long slot = (long long)node * J.status_stride + J.status_offset;
    const bool success = status == ST_SUCCESS;
    const int n = d.n;
    if (J.weights && n > 0) {
        if (lane < n) J.weights[slot * P.nmax + lane] = w0;
        if (lane + 32 < n) J.weights[slot * P.nmax + lane + 32] = w1;
    }
    if (J.variance && lane == 0) J.variance[slot] = success ? variance : -1.0;
    if (lane == 0) J.status[slot] = (int8_t)status;
    if (is_cont(J.kind)) {
        if (success) {
            // combine (combiner.h:9-24): float sum in neighbour order.
            const float t0 = __double2float_rn(__dmul_rn(w0, (double)d.dv[0]));
            const float t1 = __double2float_rn(__dmul_rn(w1, (double)d.dv[1]));
            float res = J.kind == 1 ? J.sk_mean_f : (J.kind == 2 ? J.mean[node] : 0.f);
            res = rows_fsum(res, t0, t1, n);
            if (lane == 0) {
                J.out_values[node] = res;
                J.out_mask[node] = 1;
            }
        } else if (lane == 0) {
            if (J.kind == 0) {
                const int pos = atomicAdd(J.n_untouched, 1);
                J.untouched[pos] = node;
            } else {
                J.out_values[node] = J.kind == 1 ? J.sk_mean_f : J.mean[node];
                J.out_mask[node] = 1;
            }
        }
    } else if (J.kind == 3) {
        int best = 0;
        double best_p = 0;
        for (int k = J.k0; k < J.k1; ++k) {
            const float pk = J.pk[k];
            float prob = pk;
            if (success) {
                const float t0 =
                    __double2float_rn(__dmul_rn(w0, (double)__fsub_rn(d.code[0] == k ? 1.f : 0.f, pk)));
                const float t1 =
                    __double2float_rn(__dmul_rn(w1, (double)__fsub_rn(d.code[1] == k ? 1.f : 0.f, pk)));
                prob = rows_fsum(prob, t0, t1, n);
            }
            if (lane == 0) J.probs[(long long)node * J.K + k] = prob;
            if (k == J.k0 || (double)prob > best_p) {
                best_p = prob;
                best = k;
            }
        }
        if (J.k0 == 0 && J.k1 == J.K && lane == 0) {
            J.out_codes[node] = (uint8_t)best;
            J.out_mask[node] = 1;
        }
    } else {
        const float m = J.median_m;
        double prob = (double)m;
        if (success) {
            const double t0 = __dmul_rn(w0, (double)__fsub_rn(d.code[0] == 1 ? 1.f : 0.f, m));
            const double t1 = __dmul_rn(w1, (double)__fsub_rn(d.code[1] == 1 ? 1.f : 0.f, m));
            prob = rows_dsum(prob, t0, t1, n);
        }
        if (lane == 0) {
            J.probs[node] = (float)prob;
            J.out_codes[node] = ((float)prob <= 0.5f) ? 0 : 1;
            J.out_mask[node] = 1;
        }
    }
}

__device__ __forceinline__ bool copy_informed64(const DevJob &J, const NodeFetch &f, int lane) {
    const int node = f.node;
    if (f.informed) {
        if (lane == 0) {
            J.out_values[node] = J.values[node];
            J.out_mask[node] = 1;
            J.status[(long long)node * J.status_stride + J.status_offset] = ST_NOT_KRIGED;
        }
        return true;
    }
    return false;
}

__device__ __forceinline__ double pair_cov64(const DevJob &J, const DevPlan &P, const int4 &a, const int4 &b) {
    // C(x_a - x_b) (my_kriging_weights.h:53, 160)
    return cov_lin(P, a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w, J.err);
}

// Build: the n(n-1)/2 entries A(i, k) = C(x_i - x_k), i < k, of the upper
// triangle into the skewed packed layout (my_kriging_weights.h:49-58; the
// tables are exactly symmetric, C(v) = C(-v) bit for bit, so either
// orientation gives the reference's value).  Lane l takes the pairs
// (r, r + d mod 64) of its rows r = l, l + 32 for d = 1..31, and (l, l + 32):
// every pair once, 63 a lane, 16 gathers in flight per trip.  Columns from n
// on are left as they are.
template <bool CORR>
__device__ __forceinline__ void build_packed(const DevJob &J, const DevPlan &P, double *U, const int4 *nb,
                                             const int *cs, int n, int lane, const double *sg) {
    const int4 own[2] = {nb[lane], nb[lane + 32]};
#pragma unroll 1
    for (int d0 = 1; d0 <= 32; d0 += 8) {
        double v[16];
        int dst[16];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            const int d = d0 + (e >> 1), h = e & 1;
            const int r = lane + 32 * h, k = (r + d) & 63;
            dst[e] = -1;
            v[e] = 0.0;
            if (r < n && k < n && (d < 32 || h == 0)) {
                v[e] = pair_cov64(J, P, own[h], nb[k]);
                const int lo = r < k ? r : k, hi = r < k ? k : r;
                if (CORR) v[e] = __dmul_rn(v[e], __dmul_rn(sg[hi], sg[lo]));
                dst[e] = cs[hi] + lo;
            }
        }
#pragma unroll
        for (int e = 0; e < 16; ++e)
            if (dst[e] >= 0) U[dst[e]] = v[e];
    }
    __syncwarp();
}

// Factorises and solves one system (weights of rows lane, lane + 32 in w0,
// w1); returns the status.  CORR scales entry (i, k) by sg[k] sg[i]
// (corellogramed_weights_3, my_kriging_weights.h:308-317; b is scaled by
// the caller).
template <bool CORR>
__device__ int exact64_core(const DevJob &J, const DevPlan &P, Exact64Smem &S, const int *cs,
                            int lane, const Node64 &d, const double *sg, double &w0_out, double &w1_out) {
    const int n = d.n;
    const bool ordinary = J.kind == 0;
    double *U = S.U;
    build_packed<CORR>(J, P, U, S.nb, cs, n, lane, sg);
    const int k0 = lane, k1 = lane + 32;  // the lane's columns in the factorisation
    const double a_diag = __ldg(P.table + P.center);  // A(k,k) = C(0), the table's centre
    // diagonal slots and pads of the lane's columns are zero until their step
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int k = lane + 32 * h;
        U[cs[k] + k] = 0.0;
        if (!(k & 1)) U[cs[k] + k + 1] = 0.0;
    }
    __syncwarp();
    const double *c0 = U + cs[k0];
    const double *c1 = U + cs[k1];
    int info = 0;
    double dg0 = 0.0, rc0 = 0.0, dg1 = 0.0, rc1 = 0.0;  // U(k,k) and RN(1/U(k,k)) of the lane's columns
    double xa0 = d.b[0], xa1 = d.b[1], xb0 = 1.0, xb1 = 1.0;
    // DPOTF2 'U' step j, left-looking like the reference: the sums
    // t = sum_{i<j} U(i,k) U(i,j) (DDOT for k = j, DGEMV for k > j) run over i in
    // ascending order from +0, each lane over its own columns while column j
    // is broadcast; an odd j pairs row j, whose slot in column j is still
    // zero.  Every lane runs every instruction of a step: the pivot's square
    // root and reciprocal and the forward division are computed by all lanes
    // from broadcast values (the same operations the owner would do), which
    // keeps the warp converged.
    for (int j = 0; j < n; ++j) {
        const bool lo = j < 32;  // the lane's first column is still open
        const int owner = j & 31;
        const bool mine = lane == owner;
        const double2 *uj = reinterpret_cast<const double2 *>(U + cs[j]);
        const double2 *a0p = reinterpret_cast<const double2 *>(c0);
        const double2 *a1p = reinterpret_cast<const double2 *>(c1);
        double t0 = 0.0, t1 = 0.0;
        const int pairs = (j + 1) >> 1;
        if (lo) {
            for (int q = 0; q < pairs; ++q) {
                const double2 u = uj[q], a0 = a0p[q], a1 = a1p[q];
                t0 = __dadd_rn(t0, __dmul_rn(a0.x, u.x));
                t1 = __dadd_rn(t1, __dmul_rn(a1.x, u.x));
                t0 = __dadd_rn(t0, __dmul_rn(a0.y, u.y));
                t1 = __dadd_rn(t1, __dmul_rn(a1.y, u.y));
            }
        } else {
            for (int q = 0; q < pairs; ++q) {
                const double2 u = uj[q], a1 = a1p[q];
                t1 = __dadd_rn(t1, __dmul_rn(a1.x, u.x));
                t1 = __dadd_rn(t1, __dmul_rn(a1.y, u.y));
            }
        }
        // every lane has read column j's diagonal slot before it is written
        __syncwarp();
        const double tj = __shfl_sync(FULL_MASK, lo ? t0 : t1, owner);
        const double ajj = __dsub_rn(CORR ? __dmul_rn(a_diag, __dmul_rn(sg[j], sg[j])) : a_diag, tj);
        if (!(ajj > 0.0)) {
            info = j + 1;
            break;
        }
        const double ujj = dsqrt64(ajj);
        const double rinv = drcp64(ujj);
        if (mine) {
            U[cs[j] + j] = ujj;
            if (lo) {
                dg0 = ujj;
                rc0 = rinv;
            } else {
                dg1 = ujj;
                rc1 = rinv;
            }
        }
        // forward substitution U^T y = b, row j final: y_j = x_j / u_jj
        const double xaj = __shfl_sync(FULL_MASK, lo ? xa0 : xa1, owner);
        const double ya = div_by_rcp(xaj, ujj, rinv);
        double yb = 0.0;
        if (ordinary) yb = div_by_rcp(__shfl_sync(FULL_MASK, lo ? xb0 : xb1, owner), ujj, rinv);
        if (mine) {
            if (lo) {
                xa0 = ya;
                xb0 = yb;
            } else {
                xa1 = ya;
                xb1 = yb;
            }
        }
        // row j of U: u_jk = (a_jk - t) / u_jj for the lane's columns k > j,
        // then x_k -= u_jk y_j
        if (lo && k0 > j) {
            double v = U[cs[k0] + j];
            if (j > 0) v = __dadd_rn(v, -t0);
            const double v0 = __dmul_rn(rinv, v);
            U[cs[k0] + j] = v0;
            xa0 = __dsub_rn(xa0, __dmul_rn(v0, ya));
            if (ordinary) xb0 = __dsub_rn(xb0, __dmul_rn(v0, yb));
        }
        if (k1 > j) {
            double v = U[cs[k1] + j];
            if (j > 0) v = __dadd_rn(v, -t1);
            const double v1 = __dmul_rn(rinv, v);
            U[cs[k1] + j] = v1;
            xa1 = __dsub_rn(xa1, __dmul_rn(v1, ya));
            if (ordinary) xb1 = __dsub_rn(xb1, __dmul_rn(v1, yb));
        }
        __syncwarp();
    }
    double w0 = 0.0, w1 = 0.0;
    int status = ST_SUCCESS;
    const int n0 = n < 32 ? n : 32;  // rows held in the lanes' first halves
    if (info != 0) {
        status = ST_SINGULAR;
    } else {
        // DPOTRS back substitution U x = y (DTRSM column form, k descending):
        // x_k /= u_kk where x_k != 0, then x_i -= x_k u_ik for i < k.
        for (int k = n - 1; k >= 0; --k) {
            const int owner = k & 31;
            const bool hi = k >= 32;
            const double ukk = __shfl_sync(FULL_MASK, hi ? dg1 : dg0, owner);
            const double rk = __shfl_sync(FULL_MASK, hi ? rc1 : rc0, owner);
            double va = __shfl_sync(FULL_MASK, hi ? xa1 : xa0, owner);
            double vb = ordinary ? __shfl_sync(FULL_MASK, hi ? xb1 : xb0, owner) : 0.0;
            const bool nza = va != 0.0, nzb = vb != 0.0;
            if (nza) va = div_by_rcp(va, ukk, rk);
            if (nzb) vb = div_by_rcp(vb, ukk, rk);
            if (lane == owner) {
                if (hi) {
                    xa1 = va;
                    xb1 = vb;
                } else {
                    xa0 = va;
                    xb0 = vb;
                }
            }
            const double *uk = U + cs[k];
            if (k0 < k) {
                const double u = uk[k0];
                if (nza) xa0 = __dsub_rn(xa0, __dmul_rn(va, u));
                if (nzb) xb0 = __dsub_rn(xb0, __dmul_rn(vb, u));
            }
            if (k1 < k) {
                const double u = uk[k1];
                if (nza) xa1 = __dsub_rn(xa1, __dmul_rn(va, u));
                if (nzb) xb1 = __dsub_rn(xb1, __dmul_rn(vb, u));
            }
        }
        if (ordinary) {
            // SumSK, SumOnes in row order (my_kriging_weights.h), then
            // mu = (SumSK - 1) / SumOnes and w = x_sk - mu x_ones
            double ssk = 0.0, son = 0.0;
            for (int i = 0; i < n0; ++i) {
                ssk = __dadd_rn(ssk, __shfl_sync(FULL_MASK, xa0, i));
                son = __dadd_rn(son, __shfl_sync(FULL_MASK, xb0, i));
            }
            for (int i = 32; i < n; ++i) {
                ssk = __dadd_rn(ssk, __shfl_sync(FULL_MASK, xa1, i - 32));
                son = __dadd_rn(son, __shfl_sync(FULL_MASK, xb1, i - 32));
            }
            const double mu = __ddiv_rn(__dsub_rn(ssk, 1.0), son);
            w0 = __dsub_rn(xa0, __dmul_rn(mu, xb0));
            w1 = __dsub_rn(xa1, __dmul_rn(mu, xb1));
        } else {
            w0 = xa0;
            w1 = xa1;
        }
    }
    w0_out = w0;
    w1_out = w1;
    return status;
}

__device__ void exact64_system(const DevJob &J, const DevPlan &P, Exact64Smem &S, const int *cs, int node,
                               int lane, const Node64 &d) {
    const int n = d.n;
    const bool ordinary = J.kind == 0;
    const int n0 = n < 32 ? n : 32;
    double w0, w1;
    const int status = exact64_core<false>(J, P, S, cs, lane, d, nullptr, w0, w1);
    double variance = -1.0;
    if (J.variance && status == ST_SUCCESS) {
        double v = P.c0;
        const double p0 = __dmul_rn(w0, d.b[0]), p1 = __dmul_rn(w1, d.b[1]);
        for (int i = 0; i < n0; ++i) v = __dsub_rn(v, __shfl_sync(FULL_MASK, p0, i));
        for (int i = 32; i < n; ++i) v = __dsub_rn(v, __shfl_sync(FULL_MASK, p1, i - 32));
        if (ordinary) v = __dsub_rn(v, row_val(w0, w1, n - 1));
        variance = v;
    }
    write_outputs64(J, P, node, lane, d, status, w0, w1, variance);
}

// One node of the exact path; returns whether a system was solved.
__device__ __forceinline__ bool exact64_node(const DevJob &J, const DevPlan &P, Exact64Smem &S, const int *cs,
                                             const NodeFetch &cur, int lane) {
    if (copy_informed64(J, cur, lane)) return false;
    const Node64 d = load_node64(J, P, S.nb, cur, lane);
    if (d.n <= 0) {
        write_outputs64(J, P, cur.node, lane, d, ST_NO_NEIGHBOURS, 0.0, 0.0, -1.0);
        return false;
    }
    exact64_system(J, P, S, cs, cur.node, lane, d);
    return true;
}

// One speculative round of sequential simulation (33-64 neighbours): one
// warp per pending node of window buffer `cur`.
__global__ void __launch_bounds__(WARPS64_BLOCK * 32) k_sgs_try64(DevJob J, DevPlan P, SgsState G, int cur) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    __shared__ int s_cs[N64];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int k = threadIdx.x; k < N64; k += blockDim.x) s_cs[k] = col_start_c(k);
    __syncthreads();
    Exact64Smem &S = reinterpret_cast<Exact64Smem *>(dyn_smem)[warp];
    const int ntry = G.ctl->ntry;
    const int *win = cur ? G.win1 : G.win0;
    // the round's tries are handed out one at a time as warps free up
    int slot, rank;
    while (sgs_next_try(G, win, ntry, lane, slot, rank)) {
        const int node = G.nodes[rank];
        int cnt;
        const int blocker = template_node_spec(J, P, G, node, rank, lane, J.nb + (long long)node * P.nmax, cnt);
        if (lane == 0 && blocker < 0) J.nbcount[node] = cnt;
        __syncwarp();
        if (blocker < 0) {
            const NodeFetch f = fetch_node(J, P, node, lane);
            exact64_node(J, P, S, s_cs, f, lane);
            __syncwarp();
            if (lane == 0) sgs_value(J, node, G.xp[rank]);
        }
        if (lane == 0) {
            G.ok[slot] = blocker < 0;
            if (blocker >= 0) G.blocker[rank] = blocker;
        }
        __syncwarp();
    }
}

// routed: per-node flags of the mixed pass -- the flagged nodes are solved,
// 32 flags read at a time and taken in node order (every node once the job
// was abandoned); null: every node.
__global__ void __launch_bounds__(WARPS64_BLOCK * 32) k_solve_exact64(DevJob J, DevPlan P, const uint8_t *routed) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    __shared__ int s_cs[N64];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int k = threadIdx.x; k < N64; k += blockDim.x) s_cs[k] = col_start_c(k);
    __syncthreads();
    Exact64Smem &S = reinterpret_cast<Exact64Smem *>(dyn_smem)[warp];
    const long long stride = (long long)gridDim.x * WARPS64_BLOCK;
    unsigned long long solved = 0;
    long long it = (long long)blockIdx.x * WARPS64_BLOCK + warp;
    if (routed && !*J.abandon) {
        for (long long base = it * 32; base < J.size; base += stride * 32) {
            const long long i = base + lane;
            unsigned m = __ballot_sync(FULL_MASK, i < J.size && routed[i]);
            while (m) {
                const int k = __ffs(m) - 1;
                m &= m - 1;
                const NodeFetch f = fetch_node(J, P, (int)(base + k), lane);
                solved += exact64_node(J, P, S, s_cs, f, lane);
                __syncwarp();
            }
        }
    } else {
        // warps take up to CHUNK64 consecutive nodes at a time from a per-job
        // counter (the next chunk taken while the current one's last node is
        // solved), so none waits on a fixed share at the end
        const int csize = chunk_nodes(J, CHUNK64, WARPS64_BLOCK);
        int chunk = take_chunk64(J, lane, csize);
        it = chunk;
        NodeFetch cur = fetch_node(J, P, it < J.size ? (int)it : -1, lane);
        while (it < J.size) {
            long long nx = it + 1;
            int nchunk = chunk;
            if (nx == (long long)chunk + csize) {
                nchunk = take_chunk64(J, lane, csize);
                nx = nchunk;
            }
            const NodeFetch next = fetch_node(J, P, nx < J.size ? (int)nx : -1, lane);
            solved += exact64_node(J, P, S, s_cs, cur, lane);
            __syncwarp();
            cur = next;
            it = nx;
            chunk = nchunk;
        }
    }
    if (lane == 0 && solved) atomicAdd(J.n_fp64, solved);
}

// ---------------------------------------------------------------------------
// Mixed path: FP32 Gauss-Jordan inverse + FP64 refinement.

constexpr float MIXED64_PIVOT_MIN = 1e-3f;  // on the unit-diagonal scaled system
constexpr int MIXED64_MAX_CORR = 6;

struct Mixed64Smem {
    double U[U64_SIZE];  // exact FP64 system, skewed packed upper triangle (diagonal = C(0))
    double xv[2][N64];   // FP64 vectors broadcast for the residuals
    float row[N64];      // pivot row of the sweep
    float vf[2][N64];    // FP32 vectors broadcast for the inverse's products
    int4 nb[N64];
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

__device__ __forceinline__ double warp_sum64(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
    return v;
}
__device__ __forceinline__ double warp_max64(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL_MASK, v, o));
    return v;
}

// (y0, y1) = rows lane and lane + 32 of M v with M's diagonal offset removed
// (the sweep leaves every swept diagonal entry 2 above the sweep operator's
// value; see the sweep below).
__device__ __forceinline__ void apply64(const float2 (&m0)[32], const float2 (&m1)[32], float v0, float v1,
                                        float *buf, int lane, float &y0, float &y1) {
    buf[lane] = v0;
    buf[lane + 32] = v1;
    __syncwarp();
    float2 a0 = f2(0.f, 0.f), a1 = f2(0.f, 0.f);
    const float4 *b4 = reinterpret_cast<const float4 *>(buf);
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const float4 u = b4[q];
        a0 = __ffma2_rn(m0[2 * q], f2(u.x, u.y), a0);
        a1 = __ffma2_rn(m1[2 * q], f2(u.x, u.y), a1);
        a0 = __ffma2_rn(m0[2 * q + 1], f2(u.z, u.w), a0);
        a1 = __ffma2_rn(m1[2 * q + 1], f2(u.z, u.w), a1);
    }
    __syncwarp();
    y0 = (a0.x + a0.y) - 2.f * v0;
    y1 = (a1.x + a1.y) - 2.f * v1;
}

// Rows lane and lane + 32 of r = b - A x in FP64 for one or two right-hand
// sides; A from the packed triangle (entries of columns below n only).
__device__ __forceinline__ void residual64(const Mixed64Smem &S, const int *cs, double a_diag, int n, int lane,
                                           bool two, double xa0, double xa1, double xb0, double xb1,
                                           double &ra0, double &ra1, double &rb0, double &rb1) {
    double *xa = const_cast<double *>(S.xv[0]), *xb = const_cast<double *>(S.xv[1]);
    xa[lane] = xa0;
    xa[lane + 32] = xa1;
    if (two) {
        xb[lane] = xb0;
        xb[lane + 32] = xb1;
    }
    __syncwarp();
    const int r0 = lane, r1 = lane + 32;
    const int cs0 = cs[r0], cs1 = cs[r1];
    double sa0 = 0.0, sa1 = 0.0, sb0 = 0.0, sb1 = 0.0;
    for (int k = 0; k < n; ++k) {
        const int ck = cs[k];
        const double a = xa[k];
        const double b = two ? xb[k] : 0.0;
        // A(r, k): column k at row r above the diagonal, column r at row k below
        const double e0 = k == r0 ? a_diag : S.U[k > r0 ? ck + r0 : cs0 + k];
        const double e1 = k == r1 ? a_diag : S.U[k > r1 ? ck + r1 : cs1 + k];
        sa0 = fma(e0, a, sa0);
        sa1 = fma(e1, a, sa1);
        if (two) {
            sb0 = fma(e0, b, sb0);
            sb1 = fma(e1, b, sb1);
        }
    }
    __syncwarp();
    // rows from n on are padding: their residual is zero (their stale
    // columns must not reach the inverse's products)
    ra0 = r0 < n ? -sa0 : 0.0;
    ra1 = r1 < n ? -sa1 : 0.0;
    rb0 = r0 < n ? -sb0 : 0.0;
    rb1 = r1 < n ? -sb1 : 0.0;
}

// One node of the mixed path; systems that do not qualify are appended to
// J.routed.  skip: a system is appended at once, without the FP32 attempt.
// Returns -1 when the node needs no system, 0 when solved here, 1 when
// routed.
__device__ __forceinline__ int mixed64_node(const DevJob &J, const DevPlan &P, Mixed64Smem &S, const int *cs,
                                            const NodeFetch &cur, int lane, bool skip = false) {
    const bool ordinary = J.kind == 0;
    const double a_diag = __ldg(P.table + P.center);  // A(k,k) = C(0)
    const double inv_c0 = 1.0 / P.c0;
    const int r0 = lane, r1 = lane + 32;
    const int cs0 = cs[r0], cs1 = cs[r1];
    const int node = cur.node;
    if (copy_informed64(J, cur, lane)) return -1;
    if (skip && cur.n > 0) {
        if (lane == 0) route(J, node);
        __syncwarp();
        return 1;
    }
    const Node64 d = load_node64(J, P, S.nb, cur, lane);
    if (d.n <= 0) {
        write_outputs64(J, P, node, lane, d, ST_NO_NEIGHBOURS, 0.0, 0.0, -1.0);
        return -1;
    }
    const int n = d.n;
    build_packed<false>(J, P, S.U, S.nb, cs, n, lane, nullptr);
    // Rows lane and lane + 32 of the unit-diagonal system A / C(0),
    // identity beyond n.
    float2 m0[32], m1[32];
#pragma unroll
    for (int c = 0; c < N64; c += 2) {
        float e[2][2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = h ? r1 : r0, csr = h ? cs1 : cs0;
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                const int cc = c + t;
                float v;
                if (r < n && cc < n) {
                    const double a = cc == r ? a_diag : S.U[cc > r ? cs[cc] + r : csr + cc];
                    v = (float)(a * inv_c0);
                } else {
                    v = cc == r ? 1.f : 0.f;
                }
                e[h][t] = v;
            }
        }
        m0[c / 2] = f2(e[0][0], e[0][1]);
        m1[c / 2] = f2(e[1][0], e[1][1]);
    }
    // Symmetric Gauss-Jordan sweeps over the n live rows: the matrix stays
    // symmetric, so pivot row p (broadcast by its owner lane) is also
    // column p and every lane reads its rows' multipliers from it.  The
    // broadcast entry at p is set to piv - 1, which turns the same fused
    // update into the sweep's column p (g = m_rp / piv) on every other row
    // and leaves 2 - 1/piv in place of -1/piv on the pivot itself; swept
    // diagonal entries are never read again, so the constant offset is
    // removed when the inverse is applied.  After all sweeps M holds
    // -(A/C(0))^-1 (+2 on the diagonal).
    bool low = false;
    for (int p = 0; p < n; ++p) {
        const int owner = p & 31;
        if (lane == owner) {
            float4 *dst = reinterpret_cast<float4 *>(S.row);
            if (p < 32) {
#pragma unroll
                for (int q = 0; q < 16; ++q)
                    dst[q] = make_float4(m0[2 * q].x, m0[2 * q].y, m0[2 * q + 1].x, m0[2 * q + 1].y);
            } else {
#pragma unroll
                for (int q = 0; q < 16; ++q)
                    dst[q] = make_float4(m1[2 * q].x, m1[2 * q].y, m1[2 * q + 1].x, m1[2 * q + 1].y);
            }
        }
        __syncwarp();
        const float piv = S.row[p];
        if (!(piv > MIXED64_PIVOT_MIN)) {  // uniform: every lane read the same pivot
            low = true;
            break;
        }
        const float dinv = __fdividef(1.f, piv);  // approximate: the refinement absorbs it
        const float g0 = (S.row[r0] - (r0 == p ? 1.f : 0.f)) * dinv;
        const float g1 = (S.row[r1] - (r1 == p ? 1.f : 0.f)) * dinv;
        __syncwarp();
        if (lane == 0) S.row[p] = piv - 1.f;
        __syncwarp();
        const float2 ng0 = f2(-g0, -g0), ng1 = f2(-g1, -g1);
        const float4 *r4 = reinterpret_cast<const float4 *>(S.row);
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const float4 u = r4[q];
            m0[2 * q] = __ffma2_rn(ng0, f2(u.x, u.y), m0[2 * q]);
            m1[2 * q] = __ffma2_rn(ng1, f2(u.x, u.y), m1[2 * q]);
            m0[2 * q + 1] = __ffma2_rn(ng0, f2(u.z, u.w), m0[2 * q + 1]);
            m1[2 * q + 1] = __ffma2_rn(ng1, f2(u.z, u.w), m1[2 * q + 1]);
        }
        __syncwarp();
    }
    if (low) {
        if (lane == 0) route(J, node);
        __syncwarp();
        return 1;
    }
    // A^-1 v = -(M v) / C(0); solutions for b (and the ones vector for OK)
    // refined with FP64 residuals.
    const double sc = -inv_c0;
    const double ba0 = d.b[0], ba1 = d.b[1];
    const double bb0 = r0 < n ? 1.0 : 0.0, bb1 = r1 < n ? 1.0 : 0.0;
    float y0, y1;
    apply64(m0, m1, (float)ba0, (float)ba1, S.vf[0], lane, y0, y1);
    double xa0 = (double)y0 * sc, xa1 = (double)y1 * sc, xb0 = 0.0, xb1 = 0.0;
    if (ordinary) {
        apply64(m0, m1, (float)bb0, (float)bb1, S.vf[1], lane, y0, y1);
        xb0 = (double)y0 * sc;
        xb1 = (double)y1 * sc;
    }
    RefineGate gate;
    bool converged = false;
    for (int corr = 0; corr < MIXED64_MAX_CORR; ++corr) {
        double ra0, ra1, rb0, rb1;
        residual64(S, cs, a_diag, n, lane, ordinary, xa0, xa1, xb0, xb1, ra0, ra1, rb0, rb1);
        ra0 += ba0;
        ra1 += ba1;
        apply64(m0, m1, (float)ra0, (float)ra1, S.vf[0], lane, y0, y1);
        const double da0 = (double)y0 * sc, da1 = (double)y1 * sc;
        xa0 += da0;
        xa1 += da1;
        double dmax = fmax(fabs(da0), fabs(da1)), xmax = fmax(fabs(xa0), fabs(xa1));
        if (ordinary) {
            rb0 += bb0;
            rb1 += bb1;
            apply64(m0, m1, (float)rb0, (float)rb1, S.vf[1], lane, y0, y1);
            const double db0 = (double)y0 * sc, db1 = (double)y1 * sc;
            xb0 += db0;
            xb1 += db1;
            dmax = fmax(dmax, fmax(fabs(db0), fabs(db1)));
            xmax = fmax(xmax, fmax(fabs(xb0), fabs(xb1)));
        }
        const int decision = gate.step(warp_max64(dmax), warp_max64(xmax));
        if (decision != 0) {
            converged = decision > 0;
            break;
        }
    }
    if (!converged) {
        if (lane == 0) route(J, node);
        __syncwarp();
        return 1;
    }
    if (r0 >= n) xa0 = xb0 = 0.0;
    if (r1 >= n) xa1 = xb1 = 0.0;
    double w0, w1;
    if (ordinary) {
        const double mu = (warp_sum64(xa0 + xa1) - 1.0) / warp_sum64(xb0 + xb1);
        w0 = xa0 - mu * xb0;
        w1 = xa1 - mu * xb1;
    } else {
        w0 = xa0;
        w1 = xa1;
    }
    double variance = -1.0;
    if (J.variance) {
        // b.x* = b.x + x*.r to second order in the solution's error, with r
        // = b - A x one more FP64 residual of the accepted solution (likewise
        // for the ordinary-kriging sums), as residual_corrected_variance in
        // solve32.cu
        double qa0, qa1, qb0, qb1;
        residual64(S, cs, a_diag, n, lane, ordinary, xa0, xa1, xb0, xb1, qa0, qa1, qb0, qb1);
        qa0 += ba0;
        qa1 += ba1;
        const double bxa = warp_sum64(d.b[0] * xa0 + xa0 * qa0 + d.b[1] * xa1 + xa1 * qa1);
        if (!ordinary) {
            variance = P.c0 - bxa;
        } else {
            qb0 += bb0;
            qb1 += bb1;
            const double bxb = warp_sum64(d.b[0] * xb0 + xa0 * qb0 + d.b[1] * xb1 + xa1 * qb1);
            const double oxa = warp_sum64(xa0 + xb0 * qa0 + xa1 + xb1 * qa1);
            const double oxb = warp_sum64(xb0 + xb0 * qb0 + xb1 + xb1 * qb1);
            const double mu = (oxa - 1.0) / oxb;
            variance = P.c0 - (bxa - mu * bxb) - row_val(xa0 - mu * xb0, xa1 - mu * xb1, n - 1);
        }
    }
    write_outputs64(J, P, node, lane, d, ST_SUCCESS, w0, w1, variance);
    __syncwarp();
    return 0;
}

__global__ void __launch_bounds__(32) k_solve_mixed64(DevJob J, DevPlan P) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    __shared__ int s_cs[N64];
    const int lane = threadIdx.x & 31;
    for (int k = threadIdx.x; k < N64; k += blockDim.x) s_cs[k] = col_start_c(k);
    __syncthreads();
    Mixed64Smem &S = *reinterpret_cast<Mixed64Smem *>(dyn_smem);
    // chunks of up to CHUNK64 nodes from the per-job counter, as the exact kernel;
    // the routing guess restarts with each chunk, so its choices depend on
    // the chunk's nodes only
    const int csize = chunk_nodes(J, CHUNK64, 1);
    int chunk = take_chunk64(J, lane, csize);
    long long it = chunk;
    NodeFetch next = fetch_node(J, P, it < J.size ? (int)it : -1, lane);
    RouteGuess guess(ROUTE_KEEP64);
    AttemptTally tally(ABANDON_FRACTION64);
    while (it < J.size) {
        const NodeFetch cur = next;
        if (it == chunk) guess = RouteGuess(ROUTE_KEEP64);
        long long nx = it + 1;
        int nchunk = chunk;
        if (nx == (long long)chunk + csize) {
            nchunk = take_chunk64(J, lane, csize);
            nx = nchunk;
        }
        next = fetch_node(J, P, nx < J.size ? (int)nx : -1, lane);
        const bool attempt = guess.attempt();
        const int outcome = mixed64_node(J, P, S, s_cs, cur, lane, !attempt);
        guess.record(attempt, outcome);
        __syncwarp();
        if (tally.step(J, attempt, outcome, lane)) break;
        it = nx;
        chunk = nchunk;
    }
}

// Fused search + solve (one warp per block): template search of a 32-node
// segment, then the segment's systems, as in the 32-neighbour fused kernel.
template <int MODE>
__global__ void __launch_bounds__(32) k_fused64(DevJob J, DevPlan P) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    __shared__ int s_cs[N64];
    __shared__ int delta_sm[32];
    const int lane = threadIdx.x & 31;
    for (int k = threadIdx.x; k < N64; k += blockDim.x) s_cs[k] = col_start_c(k);
    __syncthreads();
    const long long total = (long long)P.nseg * J.ny * J.nz;
    unsigned long long solved = 0;
    for (long long segi = blockIdx.x; segi < total; segi += gridDim.x) {
        const int base = template_segment(J, P, segi, lane, delta_sm);
        __syncwarp();
        const int x0 = (int)(segi % P.nseg) * 32;
        const int cnt = min(32, J.nx - x0);
        NodeFetch next = fetch_node(J, P, base, lane);
        for (int b = 0; b < cnt; ++b) {
            const NodeFetch cur = next;
            next = fetch_node(J, P, b + 1 < cnt ? base + b + 1 : -1, lane);
            if (MODE == 0) solved += exact64_node(J, P, *reinterpret_cast<Exact64Smem *>(dyn_smem), s_cs, cur, lane);
            else mixed64_node(J, P, *reinterpret_cast<Mixed64Smem *>(dyn_smem), s_cs, cur, lane);
            __syncwarp();
        }
    }
    if (MODE == 0 && lane == 0 && solved) atomicAdd(J.n_fp64, solved);
}

constexpr size_t SMEM64_EXACT = sizeof(Exact64Smem) * WARPS64_BLOCK;
constexpr size_t SMEM64_MIXED = sizeof(Mixed64Smem);

// ---------------------------------------------------------------------------
// Sequential indicator simulation with categories of up to 64 neighbours
// (the 32-neighbour kernel's rules, k_sis_try32 in solve32.cu).

struct Sis64Smem {
    Exact64Smem e;
    double sg[N64];  // the rows' sigma (correlogram weights)
};

__device__ __forceinline__ Node64 sis_load64(const DevJob &J, const DevPlan &P, Sis64Smem &S, int node,
                                             const int *list, int n, int k, double sgc, int lane) {
    Node64 d;
    d.n = n;
    int x0, y0, z0;
    node_xyz(J, node, x0, y0, z0);
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int row = lane + 32 * r;
        d.dv[r] = 0.f;
        d.code[r] = -1;
        d.b[r] = 0.0;
        double sg = 0.0;
        int4 o = make_int4(0, 0, 0, 0);
        if (row < n) {
            const int cell = list[row];
            int qx, qy, qz;
            node_xyz(J, cell, qx, qy, qz);
            o.x = qx - x0;
            o.y = qy - y0;
            o.z = qz - z0;
            o.w = o.z * P.syx + o.y * P.sx + o.x;
            const float m = sis_mean(J, k, cell);
            d.dv[r] = __fsub_rn(J.codes[cell] == k ? 1.f : 0.f, m);
            d.b[r] = cov_lin(P, o.x, o.y, o.z, o.w, J.err);
            if (J.sis_corr) {
                sg = sis_sigma(m);
                d.b[r] = __dmul_rn(d.b[r], __dmul_rn(sg, sgc));
            }
        }
        S.e.nb[row] = o;
        S.sg[row] = sg;
    }
    __syncwarp();
    return d;
}

__global__ void __launch_bounds__(WARPS64_BLOCK * 32) k_sis_try64(DevJob J, const DevPlan *plans, SgsState G, int cur) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    __shared__ int s_cs[N64];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int k = threadIdx.x; k < N64; k += blockDim.x) s_cs[k] = col_start_c(k);
    __syncthreads();
    Sis64Smem &S = reinterpret_cast<Sis64Smem *>(dyn_smem)[warp];
    const int ntry = G.ctl->ntry;
    const int *win = cur ? G.win1 : G.win0;
    const int cats = J.K == 2 ? 1 : J.K;
    // the round's tries are handed out one at a time as warps free up
    int slot, rank;
    while (sgs_next_try(G, win, ntry, lane, slot, rank)) {
        const int node = G.nodes[rank];
        int *list = J.nb + (long long)node * J.nb_stride;
        float *probs = J.probs + (long long)node * J.K;
        int blocker = -1;
        for (int k = 0; k < cats; ++k) {
            const DevPlan &P = plans[k];
            int cnt;
            blocker = template_node_spec(J, P, G, node, rank, lane, list, cnt);
            if (blocker >= 0) break;
            __syncwarp();
            const float mc = sis_mean(J, k, node);
            double prob = (double)mc;
            if (cnt > 0) {
                const double sgc = J.sis_corr ? sis_sigma(mc) : 0.0;
                const Node64 d = sis_load64(J, P, S, node, list, cnt, k, sgc, lane);
                double w0, w1;
                const int status =
                    J.sis_corr ? exact64_core<true>(J, P, S.e, s_cs, lane, d, S.sg, w0, w1)
                               : exact64_core<false>(J, P, S.e, s_cs, lane, d, nullptr, w0, w1);
                if (status == ST_SUCCESS) {
                    const double t0 = __dmul_rn(w0, (double)d.dv[0]), t1 = __dmul_rn(w1, (double)d.dv[1]);
                    prob = rows_dsum((double)mc, t0, t1, cnt);
                }
            }
            if (lane == 0) {
                probs[k] = __double2float_rn(prob);
                if (J.K == 2) probs[1] = __double2float_rn(__dsub_rn(1.0, prob));
            }
            __syncwarp();
        }
        if (lane == 0) sis_finish(J, G, node, rank, slot, blocker);
        __syncwarp();
    }
}

}  // namespace

void launch_solve64_exact(const DevJob &J, const DevPlan &P, const uint8_t *routed, cudaStream_t s,
                          int blocks_per_sm) {
    const long long g = persistent_grid((const void *)k_solve_exact64, WARPS64_BLOCK * 32, SMEM64_EXACT,
                                        blocks_per_sm, (J.size + WARPS64_BLOCK - 1) / WARPS64_BLOCK);
    k_solve_exact64<<<(unsigned)g, WARPS64_BLOCK * 32, SMEM64_EXACT, s>>>(J, P, routed);
}

void launch_sgs_try64(const DevJob &J, const DevPlan &P, const SgsState &G, int cur, cudaStream_t s) {
    const long long g = persistent_grid((const void *)k_sgs_try64, WARPS64_BLOCK * 32, SMEM64_EXACT, 0, 1LL << 30);
    k_sgs_try64<<<(unsigned)g, WARPS64_BLOCK * 32, SMEM64_EXACT, s>>>(J, P, G, cur);
}

void launch_sis_try64(const DevJob &J, const DevPlan *plans, const SgsState &G, int cur, cudaStream_t s) {
    const size_t smem = sizeof(Sis64Smem) * WARPS64_BLOCK;
    const long long g = persistent_grid((const void *)k_sis_try64, WARPS64_BLOCK * 32, smem, 0, 1LL << 30);
    k_sis_try64<<<(unsigned)g, WARPS64_BLOCK * 32, smem, s>>>(J, plans, G, cur);
}

void launch_solve64_mixed(const DevJob &J, const DevPlan &P, cudaStream_t s, int blocks_per_sm) {
    if (J.size <= 0) return;
    const long long g = persistent_grid((const void *)k_solve_mixed64, 32, SMEM64_MIXED, blocks_per_sm, J.size);
    k_solve_mixed64<<<(unsigned)g, 32, SMEM64_MIXED, s>>>(J, P);
}

void launch_fused64(const DevJob &J, const DevPlan &P, int precision, cudaStream_t s, int blocks_per_sm) {
    const long long segs = (long long)P.nseg * J.ny * J.nz;
    if (segs <= 0) return;
    if (precision == 0) {
        const long long g = persistent_grid((const void *)k_fused64<0>, 32, sizeof(Exact64Smem), blocks_per_sm, segs);
        k_fused64<0><<<(unsigned)g, 32, sizeof(Exact64Smem), s>>>(J, P);
    } else {
        const long long g = persistent_grid((const void *)k_fused64<1>, 32, SMEM64_MIXED, blocks_per_sm, segs);
        k_fused64<1><<<(unsigned)g, 32, SMEM64_MIXED, s>>>(J, P);
    }
}

}  // namespace hpgl_b200
