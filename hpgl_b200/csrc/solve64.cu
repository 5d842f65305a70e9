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
#include "device_common.cuh"

namespace hpgl_b200 {

namespace {

constexpr int N64 = 64;

constexpr int WARPS64_BLOCK = 1;

// The factor lives in shared memory as a skewed packed upper triangle:
// column k starts at col_start(k), holds rows 0..k (padded to an even count)
// and col_start(k) = 2k (mod 16) doubles, so when every lane reads a 16-byte
// pair of its own column at the same row, the 32 addresses fall on 8
// different 16-byte bank groups, 4 each: conflict-free.  Column k is the
// matrix column A(., k) until its rows are overwritten, one per step, by the
// factor's row; its diagonal slot stays zero until step k.
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

// The upper triangle's (row, column) pairs in column order, i | k << 8.
struct PairTable64 {
    uint16_t v[N64 * (N64 - 1) / 2];
    constexpr PairTable64() : v() {
        for (int k = 1, p = 0; k < N64; ++k)
            for (int i = 0; i < k; ++i) v[p++] = (uint16_t)(i | k << 8);
    }
};
__device__ const PairTable64 g_pairs64;

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

__device__ __forceinline__ Node64 load_node64(const DevJob &J, const DevPlan &P, int4 *nb, int node, int lane) {
    Node64 d;
    d.n = J.nbcount[node];
    int x0, y0, z0;
    node_xyz(node, J.nx, J.ny, x0, y0, z0);
#pragma unroll
    for (int r = 0; r < 2; ++r) {
        const int row = lane + 32 * r;
        d.dv[r] = 0.f;
        d.code[r] = -1;
        d.b[r] = 0.0;
        int4 o = make_int4(0, 0, 0, 0);
        if (row < d.n) {
            const int cell = J.nb[(long long)node * P.nmax + row];
            int qx, qy, qz;
            node_xyz(cell, J.nx, J.ny, qx, qy, qz);
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

__device__ __forceinline__ bool copy_informed64(const DevJob &J, int node, int lane) {
    if (is_cont(J.kind) && J.mask[node]) {
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

__device__ void exact64_system(const DevJob &J, const DevPlan &P, Exact64Smem &S, const int *cs,
                               const uint16_t *pairs, int node, int lane, const Node64 &d) {
    const int n = d.n;
    const bool ordinary = J.kind == 0;
    double *U = S.U;
    // Build: the n(n-1)/2 entries A(i, k) = C(x_i - x_k), i < k, of the upper
    // triangle in column order, 32 at a time (pairs[p] = i | k << 8); lanes
    // stay converged and the gathers of 8 pairs are issued together.
    {
        const int npairs = n * (n - 1) / 2;
        for (int p0 = 0; p0 < npairs; p0 += 256) {
            double v[8];
            int dst[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const int p = p0 + 32 * e + lane;
                dst[e] = -1;
                v[e] = 0.0;
                if (p < npairs) {
                    const int ik = __ldg(pairs + p);
                    const int i = ik & 0xff, k = ik >> 8;
                    v[e] = pair_cov64(J, P, S.nb[i], S.nb[k]);
                    dst[e] = cs[k] + i;
                }
            }
#pragma unroll
            for (int e = 0; e < 8; ++e)
                if (dst[e] >= 0) U[dst[e]] = v[e];
        }
    }
    __syncwarp();
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
        const double ajj = __dsub_rn(a_diag, tj);
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

__global__ void __launch_bounds__(WARPS64_BLOCK * 32) k_solve_exact64(DevJob J, DevPlan P, const int *list,
                                                                      const int *n_list) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    __shared__ int s_cs[N64];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int k = threadIdx.x; k < N64; k += blockDim.x) s_cs[k] = col_start_c(k);
    __syncthreads();
    Exact64Smem &S = reinterpret_cast<Exact64Smem *>(dyn_smem)[warp];
    const long long count = list ? (long long)*n_list : J.size;
    unsigned long long solved = 0;
    for (long long it = (long long)blockIdx.x * WARPS64_BLOCK + warp; it < count;
         it += (long long)gridDim.x * WARPS64_BLOCK) {
        const int node = list ? list[it] : (int)it;
        if (copy_informed64(J, node, lane)) continue;
        const Node64 d = load_node64(J, P, S.nb, node, lane);
        if (d.n <= 0) {
            write_outputs64(J, P, node, lane, d, ST_NO_NEIGHBOURS, 0.0, 0.0, -1.0);
            continue;
        }
        exact64_system(J, P, S, s_cs, g_pairs64.v, node, lane, d);
        ++solved;
        __syncwarp();
    }
    if (lane == 0 && solved) atomicAdd(J.n_fp64, solved);
}

constexpr size_t SMEM64_EXACT = sizeof(Exact64Smem) * WARPS64_BLOCK;

int grid64_for(const void *fn, size_t smem) {
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0, dev = 0, sms = 148;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, WARPS64_BLOCK * 32, smem);
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (per_sm < 1 ? 1 : per_sm) * sms;
}

}  // namespace

void launch_solve64_exact(const DevJob &J, const DevPlan &P, const int *node_list, const int *n_list,
                          long long n_max, cudaStream_t s) {
    if (n_max <= 0) return;
    static const int grid = grid64_for((const void *)k_solve_exact64, SMEM64_EXACT);
    long long blocks = (n_max + WARPS64_BLOCK - 1) / WARPS64_BLOCK;
    if (blocks > grid) blocks = grid;
    k_solve_exact64<<<(unsigned)blocks, WARPS64_BLOCK * 32, SMEM64_EXACT, s>>>(J, P, node_list, n_list);
}

}  // namespace hpgl_b200
