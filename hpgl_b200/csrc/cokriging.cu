// Colocated simple cokriging, Markov models I and II
// (simple_cokriging_markI.cpp:19-307), one warp per node, FP64 in the
// reference's exact operation order.
//
// The neighbours come from the template search (neighbour_lookup_t over the
// untruncated primary model; the reference uses no clusterizer here).  The
// (N+1)-row system -- primary covariances, the cross covariances
// coef * C_x(center - x_i) in its last row and column, the secondary variance
// in the corner -- is solved by the reference's gauss_solve
// (gauss_solver.cpp:5-63): for column i the first row not yet used whose
// entry is non-zero is the pivot row, it is divided by its pivot entry (here
// with the correctly rounded reciprocal and one fused correction, which is
// the IEEE quotient), and eliminated from every unused row; the back
// substitution starts each unknown from B at its own position (B[i], as the
// reference does) and subtracts the pivot rows' terms from the last column
// down.  The system lives row-major in shared memory; lane l owns rows l,
// l + 32 and l + 64 (the last only for lane 0).
#include <algorithm>

#include "device_common.cuh"

namespace hpgl_b200 {

namespace {


// The shared area of one warp, sized for the job's largest system (rows =
// max_neighbours + 1): the row-major system with an odd row stride (the
// lanes' own-row accesses spread over the banks), B, the neighbour offsets
// and the pivot order.
struct CokSmem {
    double *A;
    double *B;
    int4 *nb;
    int *order;
    int ld;
};

__host__ __device__ inline int cok_ld(int nmax) { return (nmax + 1) | 1; }
__host__ __device__ inline size_t cok_smem_bytes(int nmax) {
    const int rows = nmax + 1, ld = cok_ld(nmax);
    return (size_t)rows * ld * 8 + (size_t)rows * 8 + 64 * 16 + (size_t)rows * 4 + 16;
}

__device__ __noinline__ double crcp(double a) { return __drcp_rn(a); }

// Value of position i (0..64) held by lane i % 32 in slot i / 32.
__device__ __forceinline__ double slot_val(double v0, double v1, double v2, int i) {
    const double v = i < 32 ? v0 : (i < 64 ? v1 : v2);
    return __shfl_sync(FULL_MASK, v, i & 31);
}

__device__ void cok_node(const DevJob &J, const DevPlan &P, CokSmem &S, int node, int lane,
                         unsigned long long &solved) {
    const long long slot = node;
    const int LD = S.ld;
    const float m1 = J.cok_m1, m2 = J.cok_m2;
    if (J.mask[node]) {
        // informed primary: copied (set_at, simple_cokriging_markI.cpp:245-248)
        if (lane == 0) {
            J.out_values[node] = J.values[node];
            J.out_mask[node] = 1;
            J.status[slot] = ST_NOT_KRIGED;
        }
        return;
    }
    const float sv = J.smask[node] ? J.svalues[node] : m2;
    const int n = J.nbcount[node];
    const int ms = n + 1;
    int status = ST_NO_NEIGHBOURS;
    float result = 0.f;
    double w0 = 0.0, w1 = 0.0, w2 = 0.0;
    if (n > 0) {
        int x0, y0, z0;
        node_xyz(J, node, x0, y0, z0);
        float v0 = 0.f, v1 = 0.f;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = lane + 32 * h;
            int4 o = make_int4(0, 0, 0, 0);
            if (r < n) {
                const int cell = J.nb[(long long)node * P.nmax + r];
                int qx, qy, qz;
                node_xyz(J, cell, qx, qy, qz);
                o = make_int4(qx - x0, qy - y0, qz - z0, 0);
                o.w = o.z * P.syx + o.y * P.sx + o.x;
                (h ? v1 : v0) = J.values[cell];
            }
            S.nb[r] = o;
        }
        __syncwarp();
        // build_system (simple_cokriging_markI.cpp:19-54): A(i,k) = C(x_i - x_k)
        // for i != k < n; the table is exactly symmetric (C(v) = C(-v) bit for
        // bit), so either orientation gives the reference's value.  Pairs
        // (r, r + d) along cyclic diagonals, all of a lane's gathers of a trip
        // in flight: for n <= 32, lane l takes (l, l+d mod 32), d = 1..16 (d = 16
        // on lanes 0-15 only); above, the pairs of its rows l and l+32 with
        // d = 1..31 mod 64 and (l, l+32).
        if (n <= 32) {
            const int4 a = S.nb[lane];
            double v[16];
#pragma unroll
            for (int d = 1; d <= 16; ++d) {
                const int k = (lane + d) & 31;
                v[d - 1] = 0.0;
                if (lane < n && k < n && (d < 16 || lane < 16)) {
                    const int4 c = S.nb[k];
                    v[d - 1] = cov_lin(P, a.x - c.x, a.y - c.y, a.z - c.z, a.w - c.w, J.err);
                }
            }
#pragma unroll
            for (int d = 1; d <= 16; ++d) {
                const int k = (lane + d) & 31;
                if (lane < n && k < n && (d < 16 || lane < 16)) {
                    S.A[lane * LD + k] = v[d - 1];
                    S.A[k * LD + lane] = v[d - 1];
                }
            }
        } else {
            const int4 own[2] = {S.nb[lane], S.nb[lane + 32]};
#pragma unroll 1
            for (int d0 = 1; d0 <= 32; d0 += 8) {
                double v[16];
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    const int d = d0 + (e >> 1), h = e & 1;
                    const int r = lane + 32 * h, k = (r + d) & 63;
                    v[e] = 0.0;
                    if (r < n && k < n && (d < 32 || h == 0)) {
                        const int4 c = S.nb[k];
                        v[e] = cov_lin(P, own[h].x - c.x, own[h].y - c.y, own[h].z - c.z, own[h].w - c.w, J.err);
                    }
                }
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    const int d = d0 + (e >> 1), h = e & 1;
                    const int r = lane + 32 * h, k = (r + d) & 63;
                    if (r < n && k < n && (d < 32 || h == 0)) {
                        S.A[r * LD + k] = v[e];
                        S.A[k * LD + r] = v[e];
                    }
                }
            }
        }
        const double c0 = __ldg(P.table + P.center);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = lane + 32 * h;
            if (r < n) {
                const int4 a = S.nb[r];
                S.A[r * LD + r] = c0;
                // cross_cov(center, x_r) = coef * C_x(center - x_r); C_x(-v) = C_x(v)
                double cx = 0.0;
                if (cov_in_range(P, a.x, a.y, a.z)) cx = __ldg(J.cross_table + (P.center + a.w));
                else if (!P.truncated) atomicOr(J.err, DERR_TABLE_RANGE);
                const double x = __dmul_rn(J.cok_coef, cx);
                S.A[n * LD + r] = x;
                S.A[r * LD + n] = x;
                S.B[r] = cov_lin(P, a.x, a.y, a.z, a.w, J.err);  // primary_cov(x_r, center)
            }
        }
        if (lane == 0) {
            S.B[n] = __dmul_rn(J.cok_coef, __ldg(J.cross_table + P.center));
            S.A[n * LD + n] = J.cok_svar;
        }
        __syncwarp();
        // gauss_solve (gauss_solver.cpp:5-63)
        bool used0 = false, used1 = false, used2 = false;  // flags of the lane's rows
        bool singular = false;
        for (int i = 0; i < ms; ++i) {
            const int r0 = lane, r1 = lane + 32, r2 = lane + 64;
            const bool c0ok = r0 < ms && !used0 && S.A[r0 * LD + i] != 0.0;
            const bool c1ok = r1 < ms && !used1 && S.A[r1 * LD + i] != 0.0;
            const bool c2ok = r2 < ms && !used2 && S.A[r2 * LD + i] != 0.0;
            const unsigned b0 = __ballot_sync(FULL_MASK, c0ok), b1 = __ballot_sync(FULL_MASK, c1ok),
                           b2 = __ballot_sync(FULL_MASK, c2ok);
            int row;
            if (b0) row = __ffs(b0) - 1;
            else if (b1) row = 32 + __ffs(b1) - 1;
            else if (b2) row = 64 + __ffs(b2) - 1;
            else {
                singular = true;
                break;
            }
            if (row == r0) used0 = true;
            if (row == r1) used1 = true;
            if (row == r2) used2 = true;
            if (lane == 0) S.order[i] = row;
            const double coef = S.A[row * LD + i];
            const double y = crcp(coef);
            __syncwarp();
            // normalise the pivot row from column i on, and its B
            for (int j = i + lane; j < ms; j += 32) S.A[row * LD + j] = div_by_rcp(S.A[row * LD + j], coef, y);
            if (lane == 0) S.B[row] = div_by_rcp(S.B[row], coef, y);
            __syncwarp();
            // eliminate column i from every unused row.  The unused rows are
            // listed (in shared memory; the neighbour offsets are no longer
            // needed) and dealt out to the lanes in turn, so that no lane
            // takes two rows while another is idle (a 33-row system would
            // otherwise leave lane 0 two rows per step).
            const double *pr = S.A + row * LD;
            const double bp = S.B[row];
            int *live = reinterpret_cast<int *>(S.nb);
            const bool l0 = lane < ms && !used0, l1 = lane + 32 < ms && !used1, l2 = lane + 64 < ms && !used2;
            const unsigned lb0 = __ballot_sync(FULL_MASK, l0), lb1 = __ballot_sync(FULL_MASK, l1),
                           lb2 = __ballot_sync(FULL_MASK, l2);
            const unsigned below = (1u << lane) - 1u;
            if (l0) live[__popc(lb0 & below)] = lane;
            if (l1) live[__popc(lb0) + __popc(lb1 & below)] = lane + 32;
            if (l2) live[__popc(lb0) + __popc(lb1) + __popc(lb2 & below)] = lane + 64;
            const int nlive = __popc(lb0) + __popc(lb1) + __popc(lb2);
            __syncwarp();
            for (int t = lane; t < nlive; t += 32) {
                const int r = live[t];
                double *ar = S.A + r * LD;
                const double c = ar[i];
                for (int k = i; k < ms; ++k) ar[k] = __dsub_rn(ar[k], __dmul_rn(c, pr[k]));
                S.B[r] = __dsub_rn(S.B[r], __dmul_rn(c, bp));
            }
            __syncwarp();
        }
        if (!singular) {
            // back substitution: X[i] = B[i] - sum_{j>i, j descending} A[order[i]][j] X[j]
            double x0 = lane < ms ? S.B[lane] : 0.0;
            double x1 = lane + 32 < ms ? S.B[lane + 32] : 0.0;
            double x2 = lane + 64 < ms ? S.B[lane + 64] : 0.0;
            const int o0 = lane < ms ? S.order[lane] : 0;
            const int o1 = lane + 32 < ms ? S.order[lane + 32] : 0;
            const int o2 = lane + 64 < ms ? S.order[lane + 64] : 0;
            for (int j = ms - 1; j > 0; --j) {
                const double xj = slot_val(x0, x1, x2, j);
                if (lane < j) x0 = __dsub_rn(x0, __dmul_rn(S.A[o0 * LD + j], xj));
                if (lane + 32 < j) x1 = __dsub_rn(x1, __dmul_rn(S.A[o1 * LD + j], xj));
                if (lane + 64 < j) x2 = __dsub_rn(x2, __dmul_rn(S.A[o2 * LD + j], xj));
            }
            w0 = x0;
            w1 = x1;
            w2 = x2;
            // combine (simple_cokriging_markI.cpp:84-105): float result, each
            // step widened to double and rounded back
            const float t0 = __fsub_rn(v0, m1), t1 = __fsub_rn(v1, m1);
            float res = m1;
            for (int i = 0; i < n; ++i) {
                const float ti = __shfl_sync(FULL_MASK, i < 32 ? t0 : t1, i & 31);
                const double wi = slot_val(w0, w1, w2, i);
                res = __double2float_rn(__dadd_rn((double)res, __dmul_rn((double)ti, wi)));
            }
            const double wn = slot_val(w0, w1, w2, n);
            res = __double2float_rn(__dadd_rn((double)res, __dmul_rn(wn, (double)__fsub_rn(sv, m2))));
            result = res;
            status = ST_SUCCESS;
        } else {
            status = ST_SINGULAR;
        }
        ++solved;
    }
    if (status != ST_SUCCESS) result = __fsub_rn(__fadd_rn(m1, sv), m2);  // failure estimate
    if (lane == 0) {
        J.out_values[node] = result;
        J.out_mask[node] = 1;
        J.status[slot] = (int8_t)status;
    }
    if (J.weights && status == ST_SUCCESS) {
        double *wdst = J.weights + slot * (P.nmax + 1);
        if (lane < ms) wdst[lane] = w0;
        if (lane + 32 < ms) wdst[lane + 32] = w1;
        if (lane + 64 < ms) wdst[lane + 64] = w2;
    }
}

__global__ void __launch_bounds__(32) k_cokriging(DevJob J, DevPlan P) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    CokSmem S;
    {
        const int rows = P.nmax + 1;
        S.ld = cok_ld(P.nmax);
        S.nb = reinterpret_cast<int4 *>(dyn_smem);  // 16-byte aligned first
        S.A = reinterpret_cast<double *>(dyn_smem + 64 * 16);
        S.B = S.A + (size_t)rows * S.ld;
        S.order = reinterpret_cast<int *>(S.B + rows);
    }
    const int lane = threadIdx.x & 31;
    unsigned long long solved = 0;
    for (long long node = blockIdx.x; node < J.size; node += gridDim.x) {
        cok_node(J, P, S, (int)node, lane, solved);
        __syncwarp();
    }
    if (lane == 0 && solved) atomicAdd(J.n_fp64, solved);
}

}  // namespace

void launch_cokriging(const DevJob &J, const DevPlan &P, cudaStream_t s) {
    if (J.size <= 0) return;
    // the occupancy lookup is cached per kernel: ask it for the largest area,
    // and size this grid from the job's own area
    const size_t smem = cok_smem_bytes(P.nmax);
    const long long cap = persistent_grid((const void *)k_cokriging, 32, cok_smem_bytes(64), 0, J.size);
    int per_sm = 0, dev = 0, sms = 148;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cokriging, 32, smem);
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    long long g = (long long)std::max(1, per_sm) * sms;
    g = std::max<long long>(cap, std::min<long long>(g, J.size));
    k_cokriging<<<(unsigned)g, 32, smem, s>>>(J, P);
}

}  // namespace hpgl_b200
