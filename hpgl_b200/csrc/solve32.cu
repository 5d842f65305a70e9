// Register-resident per-node solves for systems of at most 32 neighbours
// (one warp per system, persistent over the grid's nodes).
//
//   k_solve_exact32  FP64 in the reference's exact operation order
//                    (my_kriging_weights.h:26-255 over LAPACK DPOTF2/DPOTRS):
//                    lane k holds column k of the system in registers; the
//                    finished part of column j is broadcast through shared
//                    memory as 16-byte pairs for the dot products of step j.
//   k_solve_mixed32  FP32 Gauss-Jordan inverse of the (unit-diagonal scaled)
//                    system, lane r holding row r, every solve a parallel
//                    matrix-vector product; FP64 residuals against the exact
//                    FP64 system refine the solution.  Systems whose FP32
//                    pivots fall below 1e-3 (the FP64 factorisation cannot
//                    fail above that), or whose refinement stalls, are routed
//                    to the exact kernel.
//
// Both start from the same system: neighbour offsets from the search lists
// and covariances gathered from the plan's table (my_kriging_weights.h:49-58,
// 156-165), padded to 32x32 with the identity.
#include "device_common.cuh"
#include "search_common.cuh"

namespace hpgl_b200 {

namespace {

constexpr int N32 = 32;
constexpr int WARPS32 = 4;
constexpr int MIXED_CHUNK = 32;  // at most this many nodes a warp takes from the counter at a time
constexpr float MIXED_PIVOT_MIN = 1e-3f;  // on the unit-diagonal scaled system
constexpr int MIXED_MAX_CORR = 4;

// Per-warp shared memory; NA doubles of system storage (the exact path uses
// columns of 34: NC * 34 for systems of at most NC neighbours).
template <int NA>
struct SysSmemN {
    double A[NA];           // exact: in-place factor (column k at k*34); mixed: full system (LD 32, msw)
    double vd[N32];         // double vector broadcast
    float vf[2][N32];       // float vector broadcast
    float row[2][N32];      // mixed: pivot row broadcast (double buffered)
    int4 nb[N32];           // neighbour offsets from the node (x, y, z, table offset)
};
using SysSmem = SysSmemN<N32 * 34>;
// systems of at most 16 neighbours (sequential simulation): half the
// registers and shared memory, twice the warps per SM
constexpr int N16 = 16;
using SysSmem16 = SysSmemN<N16 * 34>;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL_MASK, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL_MASK, v, o));
    return v;
}

// Per-node prologue shared by both kernels.  Returns n (neighbour count) and
// fills the lane's neighbour data; the system itself is built separately.
struct NodeData {
    int n;
    float dv;   // cont: value - mean of row `lane` (float, combiner.h:18-22)
    int code;   // IK: category code of row `lane`
    double b;   // b_lane = C(x_lane - x0)
    int ox, oy, oz, lin;  // offset of neighbour `lane` from the node, and its table offset
};

template <typename SM>
__device__ __forceinline__ NodeData load_node(const DevJob &J, const DevPlan &P, SM &S, const NodeFetch &f,
                                              int lane) {
    NodeData d;
    const int node = f.node;
    d.n = f.n;
    int x0, y0, z0;
    node_xyz(J, node, x0, y0, z0);
    d.dv = 0.f;
    d.code = -1;
    d.b = 0.0;
    int ox = 0, oy = 0, oz = 0;
    if (lane < d.n) {
        const int cell = f.cell;
        int qx, qy, qz;
        node_xyz(J, cell, qx, qy, qz);
        ox = qx - x0;
        oy = qy - y0;
        oz = qz - z0;
        if (is_cont(J.kind)) {
            const float m = J.kind == 1 ? J.sk_mean_f : (J.kind == 2 ? J.mean[cell] : 0.f);
            d.dv = __fsub_rn(J.values[cell], m);
        } else {
            d.code = J.codes[cell];
        }
        d.b = cov_at(P, ox, oy, oz, J.err);
    }
    d.ox = ox;
    d.oy = oy;
    d.oz = oz;
    d.lin = oz * P.syx + oy * P.sx + ox;
    S.nb[lane] = make_int4(ox, oy, oz, d.lin);
    __syncwarp();
    return d;
}

// Position of A(i, j) in the mixed kernel's FP64 system: column j at j*32,
// row i XOR-swizzled by j/4 within it.  A lane reading its row (the FP64
// residuals, lane = row) and the lanes reading 8x4 tiles (the FP32 copy,
// rows 8 (lane/8) .. +7, columns 4 (lane%8) .. +3) both hit every
// shared-memory bank at most twice per 32 doubles, the minimum; the build's
// stores along the cyclic diagonals (l, l+d) and (l+d, l) take 86
// wavefronts a system against 62 at best (128 with a column stride of 33).
__device__ __forceinline__ int msw(int i, int j) { return j * 32 + (i ^ (j >> 2)); }

// The full symmetric system into S.A (column k at k*32, msw): the entries
// A(i,k) = C(x_i - x_k) (my_kriging_weights.h:49-58, 156-165; the tables
// are exactly symmetric, C(v) = C(-v) bit for bit, so either orientation
// gives the reference's value); diagonal C(0); the identity beyond n.
// Lane l takes the pairs (l, l+d mod 32), d = 1..16 (d = 16 on lanes 0-15
// only): every off-diagonal pair once, all 16 gathers of a lane in flight
// together, and the zero padding written by the same stores.
__device__ __forceinline__ void build_full32(const DevJob &J, const DevPlan &P, SysSmem &S, int n, int lane) {
    const int4 a = S.nb[lane];
    double v[16];
#pragma unroll
    for (int d = 1; d <= 16; ++d) {
        const int k = (lane + d) & 31;
        v[d - 1] = 0.0;
        if (lane < n && k < n && (d < 16 || lane < 16)) {
            const int4 b = S.nb[k];
            v[d - 1] = cov_lin(P, a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w, J.err);
        }
    }
#pragma unroll
    for (int d = 1; d <= 16; ++d) {
        const int k = (lane + d) & 31;
        if (d < 16 || lane < 16) {
            S.A[msw(lane, k)] = v[d - 1];
            S.A[msw(k, lane)] = v[d - 1];
        }
    }
    S.A[msw(lane, lane)] = lane < n ? __ldg(P.table + P.center) : 1.0;
    __syncwarp();
}

// init + t_0 + t_1 + ... + t_{n-1} in that order, t_i = `term` of lane i,
// computed by lane 0 from 16-byte reads of a shared buffer (valid on lane 0).
__device__ __forceinline__ float seq_fsum(float init, float term, int n, float *buf, int lane) {
    buf[lane] = term;
    __syncwarp();
    float r = init;
    if (lane == 0) {
        const float4 *b4 = reinterpret_cast<const float4 *>(buf);
#pragma unroll
        for (int q = 0; q < N32 / 4; ++q) {
            if (4 * q < n) {
                const float4 v = b4[q];
                r = __fadd_rn(r, v.x);
                if (4 * q + 1 < n) r = __fadd_rn(r, v.y);
                if (4 * q + 2 < n) r = __fadd_rn(r, v.z);
                if (4 * q + 3 < n) r = __fadd_rn(r, v.w);
            }
        }
    }
    __syncwarp();
    return r;
}
__device__ __forceinline__ double seq_dsum(double init, double term, int n, double *buf, int lane) {
    buf[lane] = term;
    __syncwarp();
    double r = init;
    if (lane == 0) {
        const double2 *b2 = reinterpret_cast<const double2 *>(buf);
#pragma unroll
        for (int q = 0; q < N32 / 2; ++q) {
            if (2 * q < n) {
                const double2 v = b2[q];
                r = __dadd_rn(r, v.x);
                if (2 * q + 1 < n) r = __dadd_rn(r, v.y);
            }
        }
    }
    __syncwarp();
    return r;
}

// Outputs of one solved (or failed) system: weights w (row `lane`), status.
// The estimate sums run on lane 0 in neighbour order (combiner.h:9-24:
// float terms summed in float; median IK in double), which is also the only
// lane that stores them.
template <typename SM>
__device__ __forceinline__ void write_outputs(const DevJob &J, const DevPlan &P, SM &S, int node, int lane,
                                              const NodeData &d, int status, double w, double variance) {
    const long long slot = (long long)node * J.status_stride + J.status_offset;
    const bool success = status == ST_SUCCESS;
    const int n = d.n;
    if (J.weights && n > 0 && lane < n) J.weights[slot * P.nmax + lane] = w;
    if (J.variance && lane == 0) J.variance[slot] = success ? variance : -1.0;
    if (lane == 0) J.status[slot] = (int8_t)status;
    if (is_cont(J.kind)) {
        if (success) {
            const float term = __double2float_rn(__dmul_rn(w, (double)d.dv));
            const float m0 = J.kind == 1 ? J.sk_mean_f : (J.kind == 2 ? J.mean[node] : 0.f);
            const float res = seq_fsum(m0, term, n, S.vf[0], lane);
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
                const float term = __double2float_rn(__dmul_rn(w, (double)__fsub_rn(d.code == k ? 1.f : 0.f, pk)));
                prob = seq_fsum(pk, term, n, S.vf[0], lane);
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
            const double term = __dmul_rn(w, (double)__fsub_rn(d.code == 1 ? 1.f : 0.f, m));
            prob = seq_dsum(prob, term, n, S.vd, lane);
        }
        if (lane == 0) {
            J.probs[node] = (float)prob;
            J.out_codes[node] = ((float)prob <= 0.5f) ? 0 : 1;
            J.out_mask[node] = 1;
        }
    }
}

__device__ __forceinline__ bool copy_informed(const DevJob &J, const NodeFetch &f, int lane) {
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

// ---------------------------------------------------------------------------
// Exact FP64 path.

// IEEE square root and reciprocal (one lane per factorisation step).
__device__ __noinline__ double dsqrt_rn(double a) { return __dsqrt_rn(a); }
__device__ __noinline__ double drcp_rn(double a) { return __drcp_rn(a); }

// Factorises and solves one system (weights of row `lane` in w); returns the
// status.  Lane k gathers column k of the upper triangle straight into
// registers.  CORR scales entry (i, k) by sg_k sg_i, sg the lanes' sigma
// (corellogramed_weights_3, my_kriging_weights.h:308-317; b is scaled by the
// caller).
template <bool CORR, int NC = N32, typename SM>
__device__ __forceinline__ int exact_core(const DevJob &J, const DevPlan &P, SM &S, int lane, const NodeData &d,
                                          double sg, double &w_out) {
    constexpr int LD = 34;
    const int n = d.n;
    const bool ordinary = J.kind == 0;
    double c[NC];
#pragma unroll
    for (int i = 0; i < NC; ++i) {
        // A(i, lane) = C(x_i - x_lane) for i <= lane (my_kriging_weights.h:53);
        // neighbour i's offsets are one broadcast read of S.nb
        const int4 q = S.nb[i];
        const double si = CORR ? __shfl_sync(FULL_MASK, sg, i) : 0.0;
        c[i] = 0.0;
        if (i <= lane && lane < n) {
            c[i] = cov_lin(P, q.x - d.ox, q.y - d.oy, q.z - d.oz, q.w - d.lin, J.err);
            if (CORR) c[i] = __dmul_rn(c[i], __dmul_rn(sg, si));
        }
    }
    // DPOTF2 'U': column j, ajj = a_jj - sum_{i<j} a_ij^2; a_jk += -sum a_ij a_ik;
    // a_jk *= 1/ajj.  Finished entries U(j,k) go to S.A (column k at k*34)
    // for the broadcasts and for the transposed reads of the back substitution.
    int info = 0;
    double my_rcp = 0.0;  // RN(1/U(lane,lane))
#pragma unroll
    for (int j = 0; j < NC; ++j) {
        if (j >= n) break;
        double t = 0.0;
        const double2 *cj = reinterpret_cast<const double2 *>(S.A + j * LD);
#pragma unroll
        for (int q = 0; q < (j + 1) / 2; ++q) {
            const double2 u = cj[q];
            t = __dadd_rn(t, __dmul_rn(c[2 * q], u.x));
            if (2 * q + 1 < j) t = __dadd_rn(t, __dmul_rn(c[2 * q + 1], u.y));
        }
        int fail = 0;
        double rinv = 0.0;
        if (lane == j) {
            double ajj = __dsub_rn(c[j], t);
            if (!(ajj > 0.0)) {
                fail = 1;
            } else {
                ajj = dsqrt_rn(ajj);
                rinv = drcp_rn(ajj);
            }
            c[j] = ajj;
            S.A[j * LD + j] = ajj;
            my_rcp = rinv;
        }
        fail = __shfl_sync(FULL_MASK, fail, j);
        if (fail) {
            info = j + 1;
            break;
        }
        rinv = __shfl_sync(FULL_MASK, rinv, j);
        if (lane > j && lane < NC) {  // the lane's column exists (NC * 34 doubles of S.A)
            double v = c[j];
            if (j > 0) v = __dadd_rn(v, -t);
            v = __dmul_rn(rinv, v);
            c[j] = v;
            S.A[lane * LD + j] = v;
        }
        __syncwarp();
    }
    double w = 0.0;
    int status = ST_SUCCESS;
    if (info != 0) {
        status = ST_SINGULAR;
    } else {
        // DPOTRS 'U': U^T y = b (dot form, k ascending), then U x = y (column form).
        double xa = d.b, xb = 1.0;
#pragma unroll
        for (int i = 0; i < NC; ++i) {
            if (i >= n) break;
            double ya = 0.0, yb = 0.0;
            if (lane == i) {
                ya = div_by_rcp(xa, c[i], my_rcp);
                xa = ya;
                if (ordinary) {
                    yb = div_by_rcp(xb, c[i], my_rcp);
                    xb = yb;
                }
            }
            ya = __shfl_sync(FULL_MASK, ya, i);
            if (ordinary) yb = __shfl_sync(FULL_MASK, yb, i);
            if (lane > i) {
                xa = __dsub_rn(xa, __dmul_rn(c[i], ya));
                if (ordinary) xb = __dsub_rn(xb, __dmul_rn(c[i], yb));
            }
        }
        __syncwarp();
        for (int k = n - 1; k >= 0; --k) {
            double va = __shfl_sync(FULL_MASK, xa, k);
            double vb = ordinary ? __shfl_sync(FULL_MASK, xb, k) : 0.0;
            const bool nza = va != 0.0, nzb = vb != 0.0;
            if (lane == k) {
                const double ukk = S.A[k * LD + k];
                if (nza) xa = div_by_rcp(xa, ukk, my_rcp);
                if (ordinary && nzb) xb = div_by_rcp(xb, ukk, my_rcp);
            }
            va = __shfl_sync(FULL_MASK, xa, k);
            if (ordinary) vb = __shfl_sync(FULL_MASK, xb, k);
            if (lane < k) {
                const double u = S.A[k * LD + lane];
                if (nza) xa = __dsub_rn(xa, __dmul_rn(va, u));
                if (ordinary && nzb) xb = __dsub_rn(xb, __dmul_rn(vb, u));
            }
        }
        if (ordinary) {
            const double ssk = __shfl_sync(FULL_MASK, seq_dsum(0.0, lane < n ? xa : 0.0, n, S.vd, lane), 0);
            const double son = __shfl_sync(FULL_MASK, seq_dsum(0.0, lane < n ? xb : 0.0, n, S.vd, lane), 0);
            const double mu = __ddiv_rn(__dsub_rn(ssk, 1.0), son);
            w = __dsub_rn(xa, __dmul_rn(mu, xb));
        } else {
            w = xa;
        }
    }
    w_out = w;
    return status;
}

// Solves and writes the outputs of one system.
template <int NC = N32, typename SM>
__device__ __forceinline__ void exact_system(const DevJob &J, const DevPlan &P, SM &S, int node, int lane,
                                             const NodeData &d) {
    const int n = d.n;
    const bool ordinary = J.kind == 0;
    double w;
    const int status = exact_core<false, NC>(J, P, S, lane, d, 0.0, w);
    double variance = -1.0;
    if (J.variance && status == ST_SUCCESS) {
        // c0 - p_0 - p_1 - ... (my_kriging_weights.h): subtracting p is adding -p
        double v = seq_dsum(P.c0, -__dmul_rn(w, d.b), n, S.vd, lane);
        if (ordinary) v = __dsub_rn(v, __shfl_sync(FULL_MASK, w, n - 1));
        variance = v;
    }
    write_outputs(J, P, S, node, lane, d, status, w, variance);
}

// One node of the exact path; returns whether a system was solved.
template <int NC = N32, typename SM>
__device__ __forceinline__ bool exact32_node(const DevJob &J, const DevPlan &P, SM &S, const NodeFetch &cur,
                                             int lane) {
    if (copy_informed(J, cur, lane)) return false;
    const NodeData d = load_node(J, P, S, cur, lane);
    if (d.n <= 0) {
        write_outputs(J, P, S, cur.node, lane, d, ST_NO_NEIGHBOURS, 0.0, -1.0);
        return false;
    }
    exact_system<NC>(J, P, S, cur.node, lane, d);
    return true;
}

// routed: per-node flags of the mixed pass -- the flagged nodes are solved,
// 32 flags read at a time and taken in node order (every node once the job
// was abandoned); null: every node.
__global__ void __launch_bounds__(WARPS32 * 32) k_solve_exact32(DevJob J, DevPlan P, const uint8_t *routed) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    SysSmem &S = reinterpret_cast<SysSmem *>(dyn_smem)[warp];
    const long long stride = (long long)gridDim.x * WARPS32;
    unsigned long long solved = 0;
    long long it = (long long)blockIdx.x * WARPS32 + warp;
    if (routed && !*J.abandon) {
        for (long long base = it * 32; base < J.size; base += stride * 32) {
            const long long i = base + lane;
            unsigned m = __ballot_sync(FULL_MASK, i < J.size && routed[i]);
            while (m) {
                const int k = __ffs(m) - 1;
                m &= m - 1;
                const NodeFetch f = fetch_node(J, P, (int)(base + k), lane);
                solved += exact32_node(J, P, S, f, lane);
                __syncwarp();
            }
        }
    } else {
        // warps take up to MIXED_CHUNK consecutive nodes at a time from the per-job
        // counter, as the mixed kernel
        const int csize = chunk_nodes(J, MIXED_CHUNK, WARPS32);
        int chunk = 0;
        if (lane == 0) chunk = atomicAdd(J.node_next, csize);
        chunk = __shfl_sync(FULL_MASK, chunk, 0);
        it = chunk;
        NodeFetch cur = fetch_node(J, P, it < J.size ? (int)it : -1, lane);
        while (it < J.size) {
            long long nx = it + 1;
            int nchunk = chunk;
            if (nx == (long long)chunk + csize) {
                int c = 0;
                if (lane == 0) c = atomicAdd(J.node_next, csize);
                nchunk = __shfl_sync(FULL_MASK, c, 0);
                nx = nchunk;
            }
            const NodeFetch next = fetch_node(J, P, nx < J.size ? (int)nx : -1, lane);
            solved += exact32_node(J, P, S, cur, lane);
            __syncwarp();
            cur = next;
            it = nx;
            chunk = nchunk;
        }
    }
    if (lane == 0 && solved) atomicAdd(J.n_fp64, solved);
}

// ---------------------------------------------------------------------------
// Mixed path.

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

// The FP32 inverse is held in 8x4 tiles: lane l owns rows 8 (l/8) .. +7 and
// columns 4 (l%8) .. +3, t[r][h] = (M(row r, col 2h), M(row r, col 2h+1)).
// Per sweep step a lane needs the pivot row's 4 values at its columns and 8
// at its rows (the pivot column, by symmetry): three 16-byte broadcast reads
// and one store by the 8 lanes of the pivot row, half the shared-memory
// traffic of a lane holding a whole row.
struct Tile {
    float2 t[8][2];
};

// y = (T - 2 I) v for v given row by row (v of row `lane`); returns y of row
// `lane`.
// Each lane forms its columns' partial sums over its rows (M is symmetric),
// the four lanes of a column group add them up while scattering the four
// columns among themselves (lane (g, c) ends with column 4c + g), and one
// shuffle brings each row its value.
__device__ __forceinline__ float apply_inverse(const Tile &T, float v, float *buf, int lane) {
    buf[lane] = v;
    __syncwarp();
    const int rg = lane >> 3;
    const float4 v0 = *reinterpret_cast<const float4 *>(buf + 8 * rg);
    const float4 v1 = *reinterpret_cast<const float4 *>(buf + 8 * rg + 4);
    const float vr[8] = {v0.x, v0.y, v0.z, v0.w, v1.x, v1.y, v1.z, v1.w};
    float2 a01 = f2(0.f, 0.f), a23 = f2(0.f, 0.f);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        a01 = __ffma2_rn(T.t[r][0], f2(vr[r], vr[r]), a01);
        a23 = __ffma2_rn(T.t[r][1], f2(vr[r], vr[r]), a23);
    }
    __syncwarp();
    const bool hi2 = (rg & 2) != 0, hi1 = (rg & 1) != 0;
    float2 keep = hi2 ? a23 : a01;
    const float2 send = hi2 ? a01 : a23;
    keep.x += __shfl_xor_sync(FULL_MASK, send.x, 16);
    keep.y += __shfl_xor_sync(FULL_MASK, send.y, 16);
    float k = hi1 ? keep.y : keep.x;
    k += __shfl_xor_sync(FULL_MASK, hi1 ? keep.x : keep.y, 8);
    // the sweep leaves +2 on the diagonal
    return __shfl_sync(FULL_MASK, k, 8 * (lane & 3) + (lane >> 2)) - 2.f * v;
}

// r = b - A x in FP64 (row `lane`; S.A holds the full symmetric system, msw).
template <typename SM>
__device__ __forceinline__ double residual(const SM &S, double *vd, double x, double b, int lane) {
    vd[lane] = x;
    __syncwarp();
    // four independent accumulation chains (the dot product's order is free
    // on the refinement path)
    double acc0 = 0.0, acc1 = 0.0, acc2 = 0.0, acc3 = 0.0;
    const double2 *x2 = reinterpret_cast<const double2 *>(vd);
#pragma unroll
    for (int q = 0; q < N32 / 4; ++q) {
        const double2 u = x2[2 * q], w = x2[2 * q + 1];
        acc0 = fma(S.A[msw(lane, 4 * q)], u.x, acc0);
        acc1 = fma(S.A[msw(lane, 4 * q + 1)], u.y, acc1);
        acc2 = fma(S.A[msw(lane, 4 * q + 2)], w.x, acc2);
        acc3 = fma(S.A[msw(lane, 4 * q + 3)], w.y, acc3);
    }
    __syncwarp();
    return b - ((acc0 + acc1) + (acc2 + acc3));
}

// The kriging variance of a refined solution, c0 - b.w (ordinary kriging:
// c0 - b.w - w_{n-1}, my_kriging_weights.h:246), accurate to second order in
// the solution's error.  With x the accepted solution and r = b - A x its
// FP64 residual (A symmetric, A x* = b): b.x* = b.x + x*.r, taken as
// b.x + x.r, whose error (x - x*).r is the product of two tiny quantities;
// the same holds for the ordinary-kriging sums b.xb*, 1.xa*, 1.xb*
// (A xb* = 1, its residual rb), from which mu and w_{n-1} are formed.
// Where the variance is a small difference of c0 and b.w (nodes next to or
// on informed cells), the plain sum would carry the refinement's relative
// error of w (up to about 1e-13) straight into it.  One more residual per
// right-hand side, only when variances are asked for.
template <typename SM>
__device__ __forceinline__ double residual_corrected_variance(const SM &S, double c0, double b, double ba,
                                                              double bb, bool ordinary, int n, double xa,
                                                              double xb, int lane) {
    const double ra = residual(S, const_cast<double *>(S.vd), xa, ba, lane);
    const double bxa = warp_sum(b * xa + xa * ra);
    if (!ordinary) return c0 - bxa;
    const double rb = residual(S, const_cast<double *>(S.vd), xb, bb, lane);
    const double bxb = warp_sum(b * xb + xa * rb);
    const double oxa = warp_sum(xa + xb * ra);
    const double oxb = warp_sum(xb + xb * rb);
    const double mu = (oxa - 1.0) / oxb;
    const double wl = __shfl_sync(FULL_MASK, xa - mu * xb, n - 1);
    return c0 - (bxa - mu * bxb) - wl;
}

// One node of the mixed path (FP32 inverse + FP64 refinement); systems that
// do not qualify are appended to J.routed.  skip: a system is appended to
// J.routed at once, without the FP32 attempt.  Returns -1 when the node
// needs no system, 0 when it was solved here, 1 when routed.
// STEPS: the sweep's pivots, at least the job's largest neighbour count (a
// multiple of 8): rows from n on are identity padding, decoupled from the
// live block, with zero right-hand sides, so their solutions stay zero
// whether or not their pivots are swept; a job of at most 24 neighbours
// sweeps 24 pivots, and the steps stay fully unrolled.
template <int STEPS = N32>
__device__ __forceinline__ int mixed32_node(const DevJob &J, const DevPlan &P, SysSmem &S, const NodeFetch &cur,
                                            int lane, bool skip = false) {
    const bool ordinary = J.kind == 0;
    const double inv_c0 = 1.0 / P.c0;
    const int node = cur.node;
    if (copy_informed(J, cur, lane)) return -1;
    if (skip && cur.n > 0) {
        if (lane == 0) route(J, node);
        __syncwarp();
        return 1;
    }
    const NodeData d = load_node(J, P, S, cur, lane);
    if (d.n <= 0) {
        write_outputs(J, P, S, node, lane, d, ST_NO_NEIGHBOURS, 0.0, -1.0);
        return -1;
    }
    const int n = d.n;
    build_full32(J, P, S, n, lane);
    // The lane's tile of the unit-diagonal system A / C(0) (identity padding).
    const int rg = lane >> 3, cg = lane & 7;
    Tile T;
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int h = 0; h < 2; ++h)
            T.t[r][h] = f2((float)(S.A[msw(8 * rg + r, 4 * cg + 2 * h)] * inv_c0),
                           (float)(S.A[msw(8 * rg + r, 4 * cg + 2 * h + 1)] * inv_c0));
    // Symmetric Gauss-Jordan sweeps (the sweep operator): the matrix stays
    // symmetric, so row p is column p; the lanes holding row p publish it,
    // every lane reads it at its columns (the update's right factor) and at
    // its rows (its rows' multipliers).  The pivot's own entry of the right
    // factor is taken as piv - 1, which turns the same fused update into the
    // swept column p (m_rp / piv) on every other row and leaves 2 - 1/piv
    // in place of -1/piv on the pivot itself; a swept diagonal entry is never
    // read again, so after all sweeps T holds -(A/C(0))^-1 + 2 I and the
    // products subtract the 2 v (apply_inverse).
    bool low = false;
#pragma unroll
    for (int p = 0; p < STEPS; ++p) {
        float *rb = S.row[p & 1];
        const int rgp = p >> 3, rp = p & 7, cgp = p >> 2, cp = p & 3;
        const bool prow = rg == rgp;
        if (prow)
            *reinterpret_cast<float4 *>(rb + 4 * cg) =
                make_float4(T.t[rp][0].x, T.t[rp][0].y, T.t[rp][1].x, T.t[rp][1].y);
        __syncwarp();
        float4 cv = *reinterpret_cast<const float4 *>(rb + 4 * cg);
        const float4 r0 = *reinterpret_cast<const float4 *>(rb + 8 * rg);
        const float4 r1 = *reinterpret_cast<const float4 *>(rb + 8 * rg + 4);
        const float piv = rb[p];
        low |= !(piv > MIXED_PIVOT_MIN);
        const float dinv = __fdividef(1.f, piv);  // approximate: the refinement absorbs it
        if (cg == cgp) {
            if (cp == 0) cv.x = piv - 1.f;
            else if (cp == 1) cv.y = piv - 1.f;
            else if (cp == 2) cv.z = piv - 1.f;
            else cv.w = piv - 1.f;
        }
        const float rv[8] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w};
        const float2 nd = f2(-dinv, -dinv);
        // the pivot row's multiplier is (m_pp - 1) / piv
        const float dp = prow ? dinv : 0.f;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const float2 ng = __ffma2_rn(f2(rv[r], rv[r]), nd, r == rp ? f2(dp, dp) : f2(0.f, 0.f));
            T.t[r][0] = __ffma2_rn(ng, f2(cv.x, cv.y), T.t[r][0]);
            T.t[r][1] = __ffma2_rn(ng, f2(cv.z, cv.w), T.t[r][1]);
        }
        __syncwarp();
    }
    if (__any_sync(FULL_MASK, low)) {
        if (lane == 0) route(J, node);
        __syncwarp();
        return 1;
    }
    // A^-1 v = -(M v) / C(0); solutions for b (and the ones vector for OK)
    // refined with FP64 residuals.
    const double sc = -inv_c0;
    double xa = (double)apply_inverse(T, (float)d.b, S.vf[0], lane) * sc;
    double xb = ordinary ? (double)apply_inverse(T, lane < n ? 1.f : 0.f, S.vf[1], lane) * sc : 0.0;
    const double ba = d.b, bb = lane < n ? 1.0 : 0.0;
    RefineGate gate;
    bool converged = false;
    for (int corr = 0; corr < MIXED_MAX_CORR; ++corr) {
        const double ra = residual(S, S.vd, xa, ba, lane);
        const double da = (double)apply_inverse(T, (float)ra, S.vf[0], lane) * sc;
        xa += da;
        double dmax = fabs(da), xmax = fabs(xa);
        if (ordinary) {
            const double rbv = residual(S, S.vd, xb, bb, lane);
            const double db = (double)apply_inverse(T, (float)rbv, S.vf[1], lane) * sc;
            xb += db;
            dmax = fmax(dmax, fabs(db));
            xmax = fmax(xmax, fabs(xb));
        }
        const int decision = gate.step(warp_max(dmax), warp_max(xmax));
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
    if (lane >= n) {
        xa = 0.0;
        xb = 0.0;
    }
    double w;
    if (ordinary) {
        const double mu = (warp_sum(xa) - 1.0) / warp_sum(xb);
        w = xa - mu * xb;
    } else {
        w = xa;
    }
    double variance = -1.0;
    if (J.variance) variance = residual_corrected_variance(S, P.c0, d.b, ba, bb, ordinary, n, xa, xb, lane);
    write_outputs(J, P, S, node, lane, d, ST_SUCCESS, w, variance);
    __syncwarp();
    return 0;
}

template <int STEPS>
__device__ __forceinline__ void mixed32_warps(const DevJob &J, const DevPlan &P) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    SysSmem &S = reinterpret_cast<SysSmem *>(dyn_smem)[warp];
    // Warps take MIXED_CHUNK consecutive nodes at a time from a per-job
    // counter (the next chunk is taken while the current chunk's last node is
    // solved), so none waits on a fixed share at the end.  The routing guess
    // starts afresh with every chunk: its choices depend on the chunk's nodes
    // only, whichever warp takes it.
    int chunk = 0;
    if (lane == 0) chunk = atomicAdd(J.node_next, MIXED_CHUNK);
    chunk = __shfl_sync(FULL_MASK, chunk, 0);
    long long it = chunk;
    NodeFetch next = fetch_node(J, P, it < J.size ? (int)it : -1, lane);
    RouteGuess guess(ROUTE_KEEP32);
    AttemptTally tally(ABANDON_FRACTION32);
    while (it < J.size) {
        const NodeFetch cur = next;
        if (it == chunk) guess = RouteGuess(ROUTE_KEEP32);
        long long nit = it + 1;
        int nchunk = chunk;
        if (nit == (long long)chunk + MIXED_CHUNK) {
            int c = 0;
            if (lane == 0) c = atomicAdd(J.node_next, MIXED_CHUNK);
            nchunk = __shfl_sync(FULL_MASK, c, 0);
            nit = nchunk;
        }
        next = fetch_node(J, P, nit < J.size ? (int)nit : -1, lane);
        const bool attempt = guess.attempt();
        const int outcome = mixed32_node<STEPS>(J, P, S, cur, lane, !attempt);
        guess.record(attempt, outcome);
        __syncwarp();
        if (tally.step(J, attempt, outcome, lane)) break;
        it = nit;
        chunk = nchunk;
    }
}

__global__ void __launch_bounds__(WARPS32 * 32) k_solve_mixed32(DevJob J, DevPlan P) { mixed32_warps<N32>(J, P); }

// jobs of at most 16 or 24 neighbours: the sweep stops there (held to 4
// blocks a SM, the 128 registers the full sweep compiles to by itself)
template <int STEPS>
__global__ void __launch_bounds__(WARPS32 * 32, 4) k_solve_mixed32_short(DevJob J, DevPlan P) {
    mixed32_warps<STEPS>(J, P);
}

// Fused search + solve: each warp takes 32-node x-segments, runs the template
// search for the segment's template-path nodes (lists to J.nb, still in L2),
// then solves the segment's nodes one after the other -- the clusterizer-path
// nodes' lists come from the clusterizer search launched before.  Warps in
// the search phase (memory latency) and in the solve phase (FP pipes)
// overlap on every SM.
template <int MODE>
__global__ void __launch_bounds__(WARPS32 * 32) k_fused32(DevJob J, DevPlan P) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    __shared__ int delta_sm[WARPS32][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    SysSmem &S = reinterpret_cast<SysSmem *>(dyn_smem)[warp];
    const long long total = (long long)P.nseg * J.ny * J.nz;
    const long long stride = (long long)gridDim.x * WARPS32;
    unsigned long long solved = 0;
    for (long long segi = (long long)blockIdx.x * WARPS32 + warp; segi < total; segi += stride) {
        const int base = template_segment(J, P, segi, lane, delta_sm[warp]);
        __syncwarp();
        const int x0 = (int)(segi % P.nseg) * 32;
        const int cnt = min(32, J.nx - x0);
        NodeFetch next = fetch_node(J, P, base, lane);
        for (int b = 0; b < cnt; ++b) {
            const NodeFetch cur = next;
            next = fetch_node(J, P, b + 1 < cnt ? base + b + 1 : -1, lane);
            if (MODE == 0) solved += exact32_node(J, P, S, cur, lane);
            else mixed32_node(J, P, S, cur, lane);
            __syncwarp();
        }
    }
    if (MODE == 0 && lane == 0 && solved) atomicAdd(J.n_fp64, solved);
}

constexpr size_t SMEM32 = sizeof(SysSmem) * WARPS32;

// The simulated value of one node of sequential Gaussian simulation from its
// neighbour list (`list`, `n` entries, in shared memory): the exact system,
// the estimate and variance by exact_system's and write_outputs' rules,
// and the value xp sqrt(variance) + estimate (sgs_value's rule), kept in
// registers instead of going through the status / variance / estimate
// arrays.  Written to the property and its mask by lane 0.
template <int NC, typename SM>
__device__ __forceinline__ void sgs_node32(const DevJob &J, const DevPlan &P, SM &S, int node, const int *list, int n,
                                           double xp, int lane) {
    NodeFetch f;
    f.node = node;
    f.n = n;
    f.cell = lane < n ? list[lane] : 0;
    f.cell2 = 0;
    f.informed = false;
    const NodeData d = load_node(J, P, S, f, lane);
    const bool ordinary = J.kind == 0;
    int status = ST_NO_NEIGHBOURS;
    double variance = 0.0;
    float est = 0.f;
    if (n > 0) {
        double w;
        status = exact_core<false, NC>(J, P, S, lane, d, 0.0, w);
        if (status == ST_SUCCESS) {
            double v = seq_dsum(P.c0, -__dmul_rn(w, d.b), n, S.vd, lane);
            if (ordinary) v = __dsub_rn(v, __shfl_sync(FULL_MASK, w, n - 1));
            variance = v;
            const float term = __double2float_rn(__dmul_rn(w, (double)d.dv));
            const float m0 = J.kind == 1 ? J.sk_mean_f : (J.kind == 2 ? J.mean[node] : 0.f);
            est = seq_fsum(m0, term, n, S.vf[0], lane);
        }
    }
    if (lane == 0) {
        const double value = status == ST_SUCCESS ? __dadd_rn(__dmul_rn(xp, __dsqrt_rn(variance)), (double)est)
                                                  : __dadd_rn(__dmul_rn(xp, 1.0), 0.0);
        J.sim_values[node] = __double2float_rn(value);
        J.sim_mask[node] = 1;
    }
}

// One speculative round of sequential simulation (at most 32 neighbours):
// one warp per pending node of window buffer `cur`: the template search with
// conflict detection (the list in shared memory), the exact FP64 system and
// the simulated value.
template <int NC>
__global__ void __launch_bounds__(WARPS32 * 32) k_sgs_try32(DevJob J, DevPlan P, SgsState G, int cur) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    using SM = SysSmemN<NC * 34>;
    SM &S = reinterpret_cast<SM *>(dyn_smem)[warp];
    const int ntry = G.ctl->ntry;
    const int *win = cur ? G.win1 : G.win0;
    // the round's tries are handed out one at a time as warps free up
    int slot, rank;
    int *list = reinterpret_cast<int *>(S.row);  // 64 ints, unused by the exact path
    while (sgs_next_try(G, win, ntry, lane, slot, rank)) {
        const int node = G.nodes[rank];
        int cnt;
        const int blocker = template_node_spec(J, P, G, node, rank, lane, list, cnt);
        __syncwarp();
        if (blocker < 0) {
            sgs_node32<NC>(J, P, S, node, list, cnt, G.xp[rank], lane);
            __syncwarp();
        }
        if (lane == 0) {
            G.ok[slot] = blocker < 0;
            if (blocker >= 0) G.blocker[rank] = blocker;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Sequential indicator simulation (do_sis, sequential_indicator_simulation.cpp:23-116).

// Row `lane` of category k's system: dv = indicator - mean of the neighbour
// (float, combiner.h:18-22), b = C(x_lane - x0), scaled by sg sgc with the
// correlogram weights (sg: the neighbour's sigma).
template <typename SM>
__device__ __forceinline__ NodeData sis_load32(const DevJob &J, const DevPlan &P, SM &S, int node,
                                               const int *list, int n, int k, double sgc, int lane, double &sg) {
    NodeData d;
    d.n = n;
    int x0, y0, z0;
    node_xyz(J, node, x0, y0, z0);
    d.dv = 0.f;
    d.code = -1;
    d.b = 0.0;
    sg = 0.0;
    int ox = 0, oy = 0, oz = 0;
    if (lane < n) {
        const int cell = list[lane];
        int qx, qy, qz;
        node_xyz(J, cell, qx, qy, qz);
        ox = qx - x0;
        oy = qy - y0;
        oz = qz - z0;
        const float m = sis_mean(J, k, cell);
        d.dv = __fsub_rn(J.codes[cell] == k ? 1.f : 0.f, m);
        d.b = cov_at(P, ox, oy, oz, J.err);
        if (J.sis_corr) {
            sg = sis_sigma(m);
            d.b = __dmul_rn(d.b, __dmul_rn(sg, sgc));
        }
    }
    d.ox = ox;
    d.oy = oy;
    d.oz = oz;
    d.lin = oz * P.syx + oy * P.sx + ox;
    S.nb[lane] = make_int4(ox, oy, oz, d.lin);
    __syncwarp();
    return d;
}

// One speculative round of sequential indicator simulation (every category
// at most 32 neighbours): one warp per pending node, the categories in
// order; per category the template search with conflict detection, the
// simple kriging system (correlogram-scaled with the mean cubes when asked)
// and the probability m_c + sum w_i (ind_i - m_i) accumulated in double
// (kriging_interpolation.h:228-265 with a double result), the mean when the
// kriging fails.  Two categories krige category 0 only and take 1 - p for
// the other (median SIS).  The code is drawn from the float probabilities.
template <int NC>
__global__ void __launch_bounds__(WARPS32 * 32) k_sis_try32(DevJob J, const DevPlan *plans, SgsState G, int cur) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    using SM = SysSmemN<NC * 34>;
    SM &S = reinterpret_cast<SM *>(dyn_smem)[warp];
    const int ntry = G.ctl->ntry;
    const int *win = cur ? G.win1 : G.win0;
    const int cats = J.K == 2 ? 1 : J.K;
    // the round's tries are handed out one at a time as warps free up
    int slot, rank;
    while (sgs_next_try(G, win, ntry, lane, slot, rank)) {
        const int node = G.nodes[rank];
        int *list = reinterpret_cast<int *>(S.row);  // 64 ints, unused by the exact path
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
                double sg, w;
                const NodeData d = sis_load32(J, P, S, node, list, cnt, k, sgc, lane, sg);
                const int status = J.sis_corr ? exact_core<true, NC>(J, P, S, lane, d, sg, w)
                                              : exact_core<false, NC>(J, P, S, lane, d, 0.0, w);
                if (status == ST_SUCCESS)
                    prob = seq_dsum((double)mc, __dmul_rn(w, (double)d.dv), cnt, S.vd, lane);
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

void launch_sgs_try32(const DevJob &J, const DevPlan &P, const SgsState &G, int cur, cudaStream_t s) {
    if (P.nmax <= N16) {
        constexpr size_t smem = sizeof(SysSmem16) * WARPS32;
        const long long g = persistent_grid((const void *)k_sgs_try32<N16>, WARPS32 * 32, smem, 0, 1LL << 30);
        k_sgs_try32<N16><<<(unsigned)g, WARPS32 * 32, smem, s>>>(J, P, G, cur);
        return;
    }
    const long long g = persistent_grid((const void *)k_sgs_try32<N32>, WARPS32 * 32, SMEM32, 0, 1LL << 30);
    k_sgs_try32<N32><<<(unsigned)g, WARPS32 * 32, SMEM32, s>>>(J, P, G, cur);
}

void launch_sis_try32(const DevJob &J, const DevPlan *plans, const SgsState &G, int cur, cudaStream_t s) {
    if (J.nb_stride <= N16) {
        constexpr size_t smem = sizeof(SysSmem16) * WARPS32;
        const long long g = persistent_grid((const void *)k_sis_try32<N16>, WARPS32 * 32, smem, 0, 1LL << 30);
        k_sis_try32<N16><<<(unsigned)g, WARPS32 * 32, smem, s>>>(J, plans, G, cur);
        return;
    }
    const long long g = persistent_grid((const void *)k_sis_try32<N32>, WARPS32 * 32, SMEM32, 0, 1LL << 30);
    k_sis_try32<N32><<<(unsigned)g, WARPS32 * 32, SMEM32, s>>>(J, plans, G, cur);
}

void launch_fused32(const DevJob &J, const DevPlan &P, int precision, cudaStream_t s, int blocks_per_sm) {
    const long long segs = (long long)P.nseg * J.ny * J.nz;
    if (segs <= 0) return;
    const int threads = WARPS32 * 32;
    if (precision == 0) {
        const long long g = persistent_grid((const void *)k_fused32<0>, threads, SMEM32, blocks_per_sm,
                                            (segs + WARPS32 - 1) / WARPS32);
        k_fused32<0><<<(unsigned)g, threads, SMEM32, s>>>(J, P);
    } else {
        const long long g = persistent_grid((const void *)k_fused32<1>, threads, SMEM32, blocks_per_sm,
                                            (segs + WARPS32 - 1) / WARPS32);
        k_fused32<1><<<(unsigned)g, threads, SMEM32, s>>>(J, P);
    }
}

const char *mixed32_kernel_name(const DevPlan &P) { return P.nmax <= 24 ? "k_solve_mixed32_short" : "k_solve_mixed32"; }

void launch_solve32(const DevJob &J, const DevPlan &P, int precision, const uint8_t *routed, cudaStream_t s,
                    int blocks_per_sm) {
    const int threads = WARPS32 * 32;
    const long long units = (J.size + WARPS32 - 1) / WARPS32;
    if (precision == 0 || routed) {
        const long long g = persistent_grid((const void *)k_solve_exact32, threads, SMEM32, blocks_per_sm, units);
        k_solve_exact32<<<(unsigned)g, threads, SMEM32, s>>>(J, P, routed);
    } else {
        // the sweep's length: the job's largest neighbour count rounded up to 8
        const int steps = P.nmax <= 16 ? 16 : (P.nmax <= 24 ? 24 : 32);
        const void *k = steps == 16 ? (const void *)k_solve_mixed32_short<16>
                                    : (steps == 24 ? (const void *)k_solve_mixed32_short<24> : (const void *)k_solve_mixed32);
        const long long g = persistent_grid(k, threads, SMEM32, blocks_per_sm, units);
        if (steps == 16) k_solve_mixed32_short<16><<<(unsigned)g, threads, SMEM32, s>>>(J, P);
        else if (steps == 24) k_solve_mixed32_short<24><<<(unsigned)g, threads, SMEM32, s>>>(J, P);
        else k_solve_mixed32<<<(unsigned)g, threads, SMEM32, s>>>(J, P);
    }
}

}  // namespace hpgl_b200
