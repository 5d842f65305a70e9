// CUDA kernels of the kriging pipeline for sm_100a:
//   k_build_bits       informed mask -> padded bit rows
//   k_search_template  bit-sliced walk of the sorted search template
//   k_search_cluster   clusterizer gather, covariance filter, reference sort
//   k_solve<NMAX,MODE> covariance build + Cholesky solve + estimate/variance
//   k_ik_argmax        most probable category
// Paths cited are relative to the reference's src/geo_bsd/hpgl/.
#include <algorithm>
#include <climits>
#include <cstdio>

#include "device_common.cuh"
#include "introsort.h"
#include "kernels.cuh"

namespace hpgl_b200 {

// ---------------------------------------------------------------------------
// informed-bit rows: bit j of word w of row (z*ny + y) is padded x = 32w + j,
// i.e. grid x = 32w + j - px.
__global__ void k_build_bits(DevJob J, DevPlan P, uint32_t *bits) {
    long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    long long rows = (long long)J.ny * J.nz;
    if (t >= rows * P.wpr) return;
    long long row = t / P.wpr;
    int w = (int)(t % P.wpr);
    uint32_t word = 0;
    const uint8_t *m = J.mask + row * J.nx;
    for (int j = 0; j < 32; ++j) {
        int x = 32 * w + j - P.px;
        if (x >= 0 && x < J.nx && m[x]) word |= 1u << j;
    }
    bits[t] = word;
}

// ---------------------------------------------------------------------------
// Template search (neighbour_lookup_t::find, sugarbox_neighbour_lookup.h:35-61).
// One warp per 32-node x-segment of a grid row walks the sorted template 32
// entries at a time: lane t loads entry base+t and forms the 32-bit window of
// informed flags of the segment's 32 target cells at that offset (one
// funnel shift of two words of bit row (y+dy, z+dz); out-of-grid cells are 0
// bits, matching is_informed(-1) == false).  A 32x32 bit transpose across
// the lanes turns the windows into, for node b (lane b), the mask of chunk
// entries that hit it; lane b appends them in template order until it holds
// max_neighbours.  Nodes that do not take the template path (clean
// clusterizer neighbourhoods) or need no kriging never become active.
__device__ __forceinline__ uint32_t transpose32(uint32_t x, int lane) {
    const uint32_t lo_masks[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
    for (int st = 0; st < 5; ++st) {
        const int j = 16 >> st;
        const uint32_t m = lo_masks[st];
        const uint32_t y = __shfl_xor_sync(FULL_MASK, x, j);
        x = (lane & j) ? ((x & ~m) | ((y >> j) & m)) : ((x & m) | ((y & m) << j));
    }
    return x;
}

__global__ void __launch_bounds__(256) k_search_template(DevJob J, DevPlan P) {
    __shared__ int delta_sm[8][32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const long long total = (long long)P.nseg * J.ny * J.nz;
    const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
    int *dsm = delta_sm[wib];
    for (long long segi = (long long)blockIdx.x * (blockDim.x >> 5) + wib; segi < total; segi += nwarps) {
        const int seg = (int)(segi % P.nseg);
        const long long row = segi / P.nseg;
        const int y = (int)(row % J.ny), z = (int)(row / J.ny);
        const int x0 = seg * 32;
        const int base = (int)(row * J.nx) + x0;
        const int node = base + lane;
        const bool act = x0 + lane < J.nx && node_needs_kriging(J, node) && !node_clean(P, x0 + lane, y, z);
        uint32_t active = __ballot_sync(FULL_MASK, act);
        if (!active) continue;
        const int nmax = P.nmax;
        int cnt = 0;
        int *out = J.nb + (long long)node * nmax;
        const uint32_t *bits = J.bits;
        for (int tb = 0; tb < P.tmpl_len && active; tb += 32) {
            const int t = tb + lane;
            uint32_t w = 0;
            int delta = 0;
            if (t < P.tmpl_len) {
                const int4 e = __ldg(&P.tmpl[t]);
                delta = e.w;
                const int yy = y + e.y, zz = z + e.z;
                if ((unsigned)yy < (unsigned)J.ny && (unsigned)zz < (unsigned)J.nz) {
                    const uint32_t *rp = bits + ((long long)zz * J.ny + yy) * P.wpr + seg + (e.x >> 5);
                    w = __funnelshift_r(__ldg(rp), __ldg(rp + 1), e.x & 31);
                }
            }
            w &= active;
            dsm[lane] = delta;
            uint32_t hits = transpose32(w, lane);
            __syncwarp();
            while (hits && cnt < nmax) {
                const int tt = __ffs(hits) - 1;
                hits &= hits - 1;
                out[cnt++] = node + dsm[tt];
            }
            __syncwarp();
            active = __ballot_sync(FULL_MASK, act && cnt < nmax);
        }
        if (act) J.nbcount[node] = cnt;
    }
}

// ---------------------------------------------------------------------------
// Warp form of the reference sort's partition (sort_partition_pairs): each
// round collects the next 32 left stoppers and 32 right stoppers with
// ballots, lane k holds the pair (L_k, R_k), the pairs with L_k < R_k (a
// prefix of the lanes) swap at once, and the first failing pair gives the
// cut.  Each round scans left from L_{b-1}+1 up to R_{b-1} and right from
// R_{b-1}-1 down to L_{b-1}; earlier rounds' swaps only ever turn positions
// at or beyond those bounds into stoppers, which yields the same
// min(L_m, R_{m-1}).  Ranges up to PAR_PARTITION_MIN elements partition on
// lane 0.
constexpr int PAR_PARTITION_MIN = 64;
constexpr int SORT_STACK = 72;

__device__ int warp_partition(SortArr &a, int lo, int hi, int pivot, int *lbuf, int *rbuf, int lane) {
    const double pk = a.key[pivot];
    const uint32_t below = (1u << lane) - 1;
    int lp = lo, lend = hi - 1;      // left scan window [lp, lend], upwards
    int rp = hi - 1, rend = pivot;   // right scan window [rend, rp], downwards
    int rprev = INT_MAX;             // R_{b-1}
    while (true) {
        int cnt = 0;
        for (int p0 = lp; cnt < 32 && p0 <= lend; p0 += 32) {
            const int p = p0 + lane;
            const bool st = p <= lend && !(a.key[p] > pk);
            const uint32_t bal = __ballot_sync(FULL_MASK, st);
            const int r = cnt + __popc(bal & below);
            if (st && r < 32) lbuf[r] = p;
            cnt += __popc(bal);
        }
        __syncwarp();
        const int my_l = lane < cnt ? lbuf[lane] : INT_MAX;
        cnt = 0;
        for (int q0 = rp; cnt < 32 && q0 >= rend; q0 -= 32) {
            const int q = q0 - lane;
            const bool st = q >= rend && !(pk > a.key[q]);
            const uint32_t bal = __ballot_sync(FULL_MASK, st);
            const int r = cnt + __popc(bal & below);
            if (st && r < 32) rbuf[r] = q;
            cnt += __popc(bal);
        }
        __syncwarp();
        const int my_r = lane < cnt ? rbuf[lane] : INT_MIN;
        const bool pair = my_l < my_r;
        const int m = __popc(__ballot_sync(FULL_MASK, pair));
        if (pair) a.swap(my_l, my_r);
        __syncwarp();
        if (m < 32) {
            const int lm = __shfl_sync(FULL_MASK, my_l, m);
            const int rl = __shfl_sync(FULL_MASK, my_r, (m + 31) & 31);
            const int rm = m > 0 ? rl : rprev;
            return lm < rm ? lm : rm;
        }
        const int l31 = __shfl_sync(FULL_MASK, my_l, 31), r31 = __shfl_sync(FULL_MASK, my_r, 31);
        lp = l31 + 1;
        lend = r31;
        rp = r31 - 1;
        rend = l31;
        rprev = r31;
    }
}

struct SortFrame {
    int lo, hi, depth;
};

// reference_sort_prefix driven by a whole warp: control flow is uniform,
// lane 0 does the median-of-three, small partitions, heap sorts and the final
// insertion sort, the warp does the long partitions.  `stack` holds
// SORT_STACK frames, `lbuf`/`rbuf` 32 positions each (shared memory).
__device__ bool warp_reference_sort_prefix(SortArr &a, int n, int k, int lane, SortFrame *stack, int *lbuf,
                                           int *rbuf) {
    if (n <= 1) return true;
    if (k > n) k = n;
    int sp = 0;
    if (lane == 0) stack[0] = SortFrame{0, n, 2 * sort_floor_log2(n)};
    ++sp;
    bool ok = true;
    while (sp > 0) {
        __syncwarp();
        const SortFrame f = stack[--sp];
        int lo = f.lo, hi = f.hi, depth = f.depth;
        if (lo >= k) continue;
        while (hi - lo > 16) {
            if (depth == 0) {
                if (lane == 0) sort_heapsort(a, lo, hi);
                break;
            }
            --depth;
            const int mid = lo + (hi - lo) / 2;
            if (lane == 0) sort_median_to_first(a, lo, lo + 1, mid, hi - 1);
            __syncwarp();
            int cut;
            if (hi - lo > PAR_PARTITION_MIN) {
                cut = warp_partition(a, lo + 1, hi, lo, lbuf, rbuf, lane);
            } else {
                int c0 = 0;
                if (lane == 0) c0 = sort_partition(a, lo + 1, hi, lo);
                cut = __shfl_sync(FULL_MASK, c0, 0);
            }
            if (cut < k) {
                if (sp >= SORT_STACK) {
                    ok = false;
                    sp = 0;
                    break;
                }
                __syncwarp();
                if (lane == 0) stack[sp] = SortFrame{cut, hi, depth};
                ++sp;
            }
            hi = cut;
        }
    }
    __syncwarp();
    if (!ok) return false;
    if (lane == 0) {
        const int end = (k + 16 < n) ? k + 16 : n;
        if (n > 16) {
            sort_insertion(a, 0, 16);
            for (int i = 16; i < end; ++i) sort_linear_insert(a, i);
        } else {
            sort_insertion(a, 0, n);
        }
    }
    __syncwarp();
    return true;
}

// ---------------------------------------------------------------------------
// Clusterizer search (sugarbox_indexed_neighbour_lookup.h:72-121): one warp
// per node whose 27 boxes are all within their fill limit.  The warp gathers
// the boxes' informed nodes in the reference's k-j-i / insertion order,
// keeps those with covariance above C(0)/100 (order-preserving ballot
// compaction), then the warp orders them exactly as the reference's
// std::sort does — as far as the first max_neighbours positions, which become
// the list.
constexpr int CLUSTER_WARPS = 4;

__global__ void __launch_bounds__(CLUSTER_WARPS * 32) k_search_cluster(DevJob J, DevPlan P, double *scratch_key,
                                                                      int *scratch_idx, int n_warps_total) {
    __shared__ SortFrame s_stack[CLUSTER_WARPS][SORT_STACK];
    __shared__ int s_lbuf[CLUSTER_WARPS][32], s_rbuf[CLUSTER_WARPS][32];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (gw >= n_warps_total) return;
    const int cap = P.max_candidates;
    double *keys = scratch_key + (long long)gw * cap;
    int *idxs = scratch_idx + (long long)gw * cap;
    const double thr = P.c0 / 100;
    for (long long node_l = gw; node_l < J.size; node_l += n_warps_total) {
        const int node = (int)node_l;
        if (!node_needs_kriging(J, node)) continue;
        int x, y, z;
        node_xyz(node, J.nx, J.ny, x, y, z);
        if (!node_clean(P, x, y, z)) continue;
        const int cx = (int)(x / P.crx), cy = (int)(y / P.cry), cz = (int)(z / P.crz);
        int n = 0;
        for (int k = cz - 1; k <= cz + 1; ++k)
            for (int j = cy - 1; j <= cy + 1; ++j)
                for (int i = cx - 1; i <= cx + 1; ++i) {
                    if (i < 0 || j < 0 || k < 0 || i > P.mx || j > P.my || k > P.mz) continue;
                    const long long bi = ((long long)k * P.my + j) * P.mx + i;
                    const int s0 = P.bucket_start[bi], s1 = P.bucket_start[bi + 1];
                    for (int base = s0; base < s1; base += 32) {
                        const int p = base + lane;
                        bool keep = false;
                        double key = 0;
                        int cand = 0;
                        if (p < s1) {
                            cand = P.bucket_nodes[p];
                            int qx, qy, qz;
                            node_xyz(cand, J.nx, J.ny, qx, qy, qz);
                            key = cov_at(P, qx - x, qy - y, qz - z, J.err);
                            keep = key > thr;
                        }
                        const uint32_t bal = __ballot_sync(FULL_MASK, keep);
                        const int pos = n + __popc(bal & ((1u << lane) - 1));
                        if (keep) {
                            if (pos < cap) {
                                keys[pos] = key;
                                idxs[pos] = cand;
                            } else {
                                atomicOr(J.err, DERR_CAND_CAPACITY);
                            }
                        }
                        n += __popc(bal);
                    }
                }
        if (n > cap) n = cap;
        __syncwarp();
        {
            // only the first max_neighbours positions of the reference's sort are used
            SortArr a{keys, idxs};
            if (!warp_reference_sort_prefix(a, n, P.nmax, lane, s_stack[wib], s_lbuf[wib], s_rbuf[wib]) && lane == 0)
                atomicOr(J.err, DERR_SORT_STACK);
        }
        const int cnt = n < P.nmax ? n : P.nmax;
        for (int i = lane; i < cnt; i += 32) J.nb[(long long)node * P.nmax + i] = idxs[i];
        if (lane == 0) J.nbcount[node] = cnt;
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Per-node solve.  One warp per kriging system; the system lives in shared
// memory (column-major upper triangle, column c at A[c*LD]), lane l owns the
// columns / rows l and l+32.
//
// MODE 0 — the reference's FP64 arithmetic in its exact operation order:
// sk/ok_kriging_weights_3 (my_kriging_weights.h:26-255) over LAPACK DPOTRF
// 'U' (unblocked DPOTF2 for N <= 64: ajj = a_jj - sum a_ij^2, row update
// a_jk += -sum a_ij a_ik, scaling by 1/ajj) and DPOTRS 'U' (DTRSM transposed
// dot-product form, then DTRSM column form).  Every product and sum uses
// explicit round-to-nearest intrinsics (no fused multiply-add) and every sum
// runs in the reference's index order, so weights, variance and estimate are
// bit-identical to the reference's.
//
// MODE 1 — FP32 Cholesky (fused multiply-adds) with FP64 iterative
// refinement: x <- x + A32^-1 (b - A x) with the residual in FP64 against the
// exact FP64 matrix.  A system is routed to the MODE 0 path (appended to
// J.routed) when an FP32 pivot falls below 1e-3 of its diagonal entry (the
// reference's FP64 factorisation cannot fail above that) or refinement does
// not reach 1e-13 relative within 4 steps.
constexpr float ROUTE_PIVOT_RATIO = 1e-3f;
constexpr double REFINE_TOL = 1e-13;
constexpr int REFINE_MAX = 4;

template <int NMAX, int MODE>
struct SolveCfg {
    static constexpr int S = NMAX / 32;
    static constexpr int LD = NMAX + 1;
    static constexpr int WARPS = NMAX <= 32 ? 8 : 4;
    static constexpr int A_D = NMAX * LD;                    // doubles
    static constexpr int B_D = NMAX;                         // doubles
    static constexpr int OFS_D = (3 * NMAX + 1) / 2;         // 3*NMAX ints
    static constexpr int A32_D = MODE ? (NMAX * LD + 1) / 2 : 0;
    static constexpr int PER_WARP = A_D + B_D + OFS_D + A32_D;
    static constexpr size_t SMEM = (size_t)PER_WARP * WARPS * sizeof(double);
};

template <int S>
__device__ __forceinline__ double pick(const double (&v)[S], int s) {
    double r = v[0];
#pragma unroll
    for (int i = 1; i < S; ++i)
        if (s == i) r = v[i];
    return r;
}
template <int S>
__device__ __forceinline__ void put(double (&v)[S], int s, double x) {
#pragma unroll
    for (int i = 0; i < S; ++i)
        if (s == i) v[i] = x;
}
template <int S>
__device__ __forceinline__ float pickf(const float (&v)[S], int s) {
    float r = v[0];
#pragma unroll
    for (int i = 1; i < S; ++i)
        if (s == i) r = v[i];
    return r;
}
template <int S>
__device__ __forceinline__ void putf(float (&v)[S], int s, float x) {
#pragma unroll
    for (int i = 0; i < S; ++i)
        if (s == i) v[i] = x;
}

// value of row k held by lane k&31 in slot k>>5
template <int S>
__device__ __forceinline__ double bcast(const double (&v)[S], int k) {
    return __shfl_sync(FULL_MASK, pick<S>(v, k >> 5), k & 31);
}
template <int S>
__device__ __forceinline__ float bcastf(const float (&v)[S], int k) {
    return __shfl_sync(FULL_MASK, pickf<S>(v, k >> 5), k & 31);
}

// Exact DPOTF2 'U' on A (n x n).  Returns LAPACK's INFO.
template <int NMAX>
__device__ int exact_potrf(double *A, int n, int lane) {
    constexpr int S = NMAX / 32, LD = NMAX + 1;
    for (int j = 0; j < n; ++j) {
        double t[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int k = lane + 32 * s;
            double acc = 0.0;
            if (k >= j && k < n) {
                const double *ck = A + k * LD, *cj = A + j * LD;
                for (int i = 0; i < j; ++i) acc = __dadd_rn(acc, __dmul_rn(ck[i], cj[i]));
            }
            t[s] = acc;
        }
        const int owner = j & 31;
        int fail = 0;
        double rinv = 0.0;
        if (lane == owner) {
            double ajj = __dsub_rn(A[j * LD + j], pick<S>(t, j >> 5));
            if (!(ajj > 0.0)) {
                fail = 1;
                A[j * LD + j] = ajj;
            } else {
                ajj = __dsqrt_rn(ajj);
                A[j * LD + j] = ajj;
                rinv = __ddiv_rn(1.0, ajj);
            }
        }
        fail = __shfl_sync(FULL_MASK, fail, owner);
        if (fail) {
            __syncwarp();
            return j + 1;
        }
        rinv = __shfl_sync(FULL_MASK, rinv, owner);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int k = lane + 32 * s;
            if (k > j && k < n) {
                double v = A[k * LD + j];
                if (j > 0) v = __dadd_rn(v, -t[s]);
                A[k * LD + j] = __dmul_rn(rinv, v);
            }
        }
        __syncwarp();
    }
    return 0;
}

// Exact DPOTRS 'U' for one or two right-hand sides held per row in xa / xb.
template <int NMAX, bool TWO>
__device__ void exact_potrs(const double *A, int n, int lane, double (&xa)[NMAX / 32], double (&xb)[NMAX / 32]) {
    constexpr int S = NMAX / 32, LD = NMAX + 1;
    // U^T y = b: y_i = (b_i - sum_{k<i} U(k,i) y_k) / U(i,i), k ascending.
    for (int i = 0; i < n; ++i) {
        const int owner = i & 31, so = i >> 5;
        double ya = 0.0, yb = 0.0;
        if (lane == owner) {
            const double d = A[i * LD + i];
            ya = __ddiv_rn(pick<S>(xa, so), d);
            put<S>(xa, so, ya);
            if (TWO) {
                yb = __ddiv_rn(pick<S>(xb, so), d);
                put<S>(xb, so, yb);
            }
        }
        ya = __shfl_sync(FULL_MASK, ya, owner);
        if (TWO) yb = __shfl_sync(FULL_MASK, yb, owner);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int r = lane + 32 * s;
            if (r > i && r < n) {
                const double a = A[r * LD + i];
                xa[s] = __dsub_rn(xa[s], __dmul_rn(a, ya));
                if (TWO) xb[s] = __dsub_rn(xb[s], __dmul_rn(a, yb));
            }
        }
    }
    // U x = y, column form: for k = n-1..0, if x_k != 0: x_k /= U(k,k);
    // x_i -= x_k U(i,k) for i < k.
    for (int k = n - 1; k >= 0; --k) {
        const int owner = k & 31, so = k >> 5;
        double va = 0.0, vb = 0.0;
        int nza = 0, nzb = 0;
        if (lane == owner) {
            const double d = A[k * LD + k];
            va = pick<S>(xa, so);
            nza = va != 0.0;
            if (nza) {
                va = __ddiv_rn(va, d);
                put<S>(xa, so, va);
            }
            if (TWO) {
                vb = pick<S>(xb, so);
                nzb = vb != 0.0;
                if (nzb) {
                    vb = __ddiv_rn(vb, d);
                    put<S>(xb, so, vb);
                }
            }
        }
        nza = __shfl_sync(FULL_MASK, nza, owner);
        va = __shfl_sync(FULL_MASK, va, owner);
        if (TWO) {
            nzb = __shfl_sync(FULL_MASK, nzb, owner);
            vb = __shfl_sync(FULL_MASK, vb, owner);
        }
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int r = lane + 32 * s;
            if (r < k) {
                const double a = A[k * LD + r];
                if (nza) xa[s] = __dsub_rn(xa[s], __dmul_rn(va, a));
                if (TWO && nzb) xb[s] = __dsub_rn(xb[s], __dmul_rn(vb, a));
            }
        }
    }
}

// FP32 Cholesky of A32 (left-looking, fused multiply-adds).  Returns false
// when a pivot is below ROUTE_PIVOT_RATIO of the FP64 diagonal entry.
template <int NMAX>
__device__ bool f32_potrf(float *A32, const double *A, int n, int lane) {
    constexpr int S = NMAX / 32, LD = NMAX + 1;
    for (int j = 0; j < n; ++j) {
        float t[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int k = lane + 32 * s;
            float acc = 0.f;
            if (k >= j && k < n) {
                const float *ck = A32 + k * LD, *cj = A32 + j * LD;
                for (int i = 0; i < j; ++i) acc = fmaf(ck[i], cj[i], acc);
            }
            t[s] = acc;
        }
        const int owner = j & 31;
        int ok = 1;
        float rinv = 0.f;
        if (lane == owner) {
            float ajj = A32[j * LD + j] - pickf<S>(t, j >> 5);
            ok = ajj > ROUTE_PIVOT_RATIO * (float)A[j * LD + j];
            if (ok) {
                ajj = sqrtf(ajj);
                A32[j * LD + j] = ajj;
                rinv = 1.0f / ajj;
            }
        }
        ok = __shfl_sync(FULL_MASK, ok, owner);
        if (!ok) {
            __syncwarp();
            return false;
        }
        rinv = __shfl_sync(FULL_MASK, rinv, owner);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int k = lane + 32 * s;
            if (k > j && k < n) A32[k * LD + j] = (A32[k * LD + j] - t[s]) * rinv;
        }
        __syncwarp();
    }
    return true;
}

// Solve (U^T U) y = r in FP32, rows held per lane.
template <int NMAX>
__device__ void f32_potrs(const float *A32, int n, int lane, float (&x)[NMAX / 32]) {
    constexpr int S = NMAX / 32, LD = NMAX + 1;
    for (int i = 0; i < n; ++i) {
        const int owner = i & 31, so = i >> 5;
        float y = 0.f;
        if (lane == owner) {
            y = pickf<S>(x, so) / A32[i * LD + i];
            putf<S>(x, so, y);
        }
        y = __shfl_sync(FULL_MASK, y, owner);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int r = lane + 32 * s;
            if (r > i && r < n) x[s] = fmaf(-A32[r * LD + i], y, x[s]);
        }
    }
    for (int k = n - 1; k >= 0; --k) {
        const int owner = k & 31, so = k >> 5;
        float v = 0.f;
        if (lane == owner) {
            v = pickf<S>(x, so) / A32[k * LD + k];
            putf<S>(x, so, v);
        }
        v = __shfl_sync(FULL_MASK, v, owner);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int r = lane + 32 * s;
            if (r < k) x[s] = fmaf(-v, A32[k * LD + r], x[s]);
        }
    }
}

// residual r = b - A x (FP64), row per lane, A symmetric from its upper triangle.
template <int NMAX>
__device__ void residual(const double *A, int n, int lane, const double (&b)[NMAX / 32], const double (&x)[NMAX / 32],
                         double (&r)[NMAX / 32]) {
    constexpr int S = NMAX / 32, LD = NMAX + 1;
    double acc[S];
#pragma unroll
    for (int s = 0; s < S; ++s) acc[s] = 0.0;
    for (int k = 0; k < n; ++k) {
        const double xk = bcast<S>(x, k);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int row = lane + 32 * s;
            if (row < n) {
                const double a = k >= row ? A[k * LD + row] : A[row * LD + k];
                acc[s] = fma(a, xk, acc[s]);
            }
        }
    }
#pragma unroll
    for (int s = 0; s < S; ++s) r[s] = (lane + 32 * s < n) ? b[s] - acc[s] : 0.0;
}

template <int NMAX, bool TWO>
__device__ bool refine(const double *A, const float *A32, int n, int lane, const double (&b)[NMAX / 32],
                       double (&xa)[NMAX / 32], double (&xb)[NMAX / 32]) {
    constexpr int S = NMAX / 32;
    float ya[S], yb[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        ya[s] = (float)b[s];
        yb[s] = 1.0f;
    }
    f32_potrs<NMAX>(A32, n, lane, ya);
    if (TWO) f32_potrs<NMAX>(A32, n, lane, yb);
    double ones[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        xa[s] = ya[s];
        xb[s] = TWO ? (double)yb[s] : 0.0;
        ones[s] = 1.0;
    }
    for (int it = 0; it < REFINE_MAX; ++it) {
        double ra[S], rb[S];
        residual<NMAX>(A, n, lane, b, xa, ra);
        if (TWO) residual<NMAX>(A, n, lane, ones, xb, rb);
        float da[S], db[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            da[s] = (float)ra[s];
            db[s] = TWO ? (float)rb[s] : 0.f;
        }
        f32_potrs<NMAX>(A32, n, lane, da);
        if (TWO) f32_potrs<NMAX>(A32, n, lane, db);
        double dmax = 0.0, xmax = 0.0;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            if (lane + 32 * s < n) {
                xa[s] += (double)da[s];
                dmax = fmax(dmax, fabs((double)da[s]));
                xmax = fmax(xmax, fabs(xa[s]));
                if (TWO) {
                    xb[s] += (double)db[s];
                    dmax = fmax(dmax, fabs((double)db[s]));
                    xmax = fmax(xmax, fabs(xb[s]));
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            dmax = fmax(dmax, __shfl_xor_sync(FULL_MASK, dmax, o));
            xmax = fmax(xmax, __shfl_xor_sync(FULL_MASK, xmax, o));
        }
        if (it > 0 && dmax <= REFINE_TOL * xmax) return true;
    }
    return false;
}

template <int NMAX, int MODE>
__global__ void __launch_bounds__(SolveCfg<NMAX, MODE>::WARPS * 32)
    k_solve(DevJob J, DevPlan P, const int *list, const int *n_list) {
    using C = SolveCfg<NMAX, MODE>;
    constexpr int S = C::S, LD = C::LD;
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *A = smem + (size_t)warp * C::PER_WARP;
    double *bsm = A + C::A_D;
    int *ox = (int *)(bsm + C::B_D);
    int *oy = ox + NMAX, *oz = oy + NMAX;
    float *A32 = (float *)(A + C::A_D + C::B_D + C::OFS_D);
    const long long count = list ? (long long)*n_list : J.size;
    const bool cont = is_cont(J.kind);
    const int nmax = P.nmax;
    unsigned long long solved64 = 0;
    for (long long it = (long long)blockIdx.x * C::WARPS + warp; it < count; it += (long long)gridDim.x * C::WARPS) {
        const int node = list ? list[it] : (int)it;
        const long long slot = (long long)node * J.status_stride + J.status_offset;
        if (cont && J.mask[node]) {
            // cont_kriging.h:103-106: informed nodes are copied.
            if (lane == 0) {
                J.out_values[node] = J.values[node];
                J.out_mask[node] = 1;
                J.status[slot] = ST_NOT_KRIGED;
            }
            continue;
        }
        const int n = J.nbcount[node];
        int x0, y0, z0;
        node_xyz(node, J.nx, J.ny, x0, y0, z0);
        // Neighbour data, row r held by lane r & 31 (slot r >> 5).
        float dv[S];   // cont: value - mean (float, as combiner.h:18-22)
        int code[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int r = lane + 32 * s;
            dv[s] = 0.f;
            code[s] = -1;
            if (r < n) {
                const int cell = J.nb[(long long)node * nmax + r];
                int qx, qy, qz;
                node_xyz(cell, J.nx, J.ny, qx, qy, qz);
                ox[r] = qx - x0;
                oy[r] = qy - y0;
                oz[r] = qz - z0;
                if (cont) {
                    const float m = J.kind == 1 ? J.sk_mean_f : (J.kind == 2 ? J.mean[cell] : 0.f);
                    dv[s] = __fsub_rn(J.values[cell], m);
                } else {
                    code[s] = J.codes[cell];
                }
            }
        }
        __syncwarp();
        int status = ST_SUCCESS;
        double w[S], bsave[S];
        if (n <= 0) {
            status = ST_NO_NEIGHBOURS;
        } else {
            // A(r,c) = C(x_r - x_c) for r <= c; b_r = C(x_r - x0)
            // (my_kriging_weights.h:49-58, 156-165).
            for (int c = 0; c < n; ++c) {
                const int cxo = ox[c], cyo = oy[c], czo = oz[c];
                for (int r = lane; r <= c; r += 32)
                    A[c * LD + r] = cov_at(P, ox[r] - cxo, oy[r] - cyo, oz[r] - czo, J.err);
            }
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int r = lane + 32 * s;
                bsave[s] = r < n ? cov_at(P, ox[r], oy[r], oz[r], J.err) : 0.0;
            }
            __syncwarp();
            const bool ordinary = J.kind == 0;
            double xa[S], xb[S];
            bool exact = MODE == 0;
            if (MODE == 1) {
                for (int c = 0; c < n; ++c)
                    for (int r = lane; r <= c; r += 32) A32[c * LD + r] = (float)A[c * LD + r];
                __syncwarp();
                bool ok = f32_potrf<NMAX>(A32, A, n, lane);
                if (ok) ok = ordinary ? refine<NMAX, true>(A, A32, n, lane, bsave, xa, xb)
                                      : refine<NMAX, false>(A, A32, n, lane, bsave, xa, xb);
                if (!ok) {
                    if (lane == 0) {
                        const int pos = atomicAdd(J.n_routed, 1);
                        J.routed[pos] = node;
                    }
                    __syncwarp();
                    continue;
                }
            }
            if (exact) {
                const int info = exact_potrf<NMAX>(A, n, lane);
#pragma unroll
                for (int s = 0; s < S; ++s) {
                    xa[s] = bsave[s];
                    xb[s] = 1.0;
                }
                if (ordinary) exact_potrs<NMAX, true>(A, n, lane, xa, xb);
                else exact_potrs<NMAX, false>(A, n, lane, xa, xb);
                if (info != 0) status = ST_SINGULAR;
                ++solved64;
            }
            if (ordinary) {
                // mu = (sum sk - 1) / sum ones; w = sk - mu * ones (:217-231)
                double ssk = 0.0, son = 0.0;
                for (int k = 0; k < n; ++k) {
                    ssk = __dadd_rn(ssk, bcast<S>(xa, k));
                    son = __dadd_rn(son, bcast<S>(xb, k));
                }
                const double mu = __ddiv_rn(__dsub_rn(ssk, 1.0), son);
#pragma unroll
                for (int s = 0; s < S; ++s) w[s] = __dsub_rn(xa[s], __dmul_rn(mu, xb[s]));
            } else {
#pragma unroll
                for (int s = 0; s < S; ++s) w[s] = xa[s];
            }
        }
        const bool success = status == ST_SUCCESS;
        if (J.weights && n > 0) {
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const int r = lane + 32 * s;
                if (r < n) J.weights[slot * nmax + r] = w[s];
            }
        }
        if (J.variance) {
            // variance = C(0) - sum w_i b_i  (- w_{n-1} for OK, :246)
            double v = -1.0;
            if (success) {
                v = P.c0;
                for (int i = 0; i < n; ++i) {
                    const int owner = i & 31, so = i >> 5;
                    const double p = __shfl_sync(FULL_MASK, __dmul_rn(pick<S>(w, so), pick<S>(bsave, so)), owner);
                    v = __dsub_rn(v, p);
                }
                if (J.kind == 0) v = __dsub_rn(v, bcast<S>(w, n - 1));
            }
            if (lane == 0) J.variance[slot] = v;
        }
        if (lane == 0) J.status[slot] = (int8_t)status;
        if (cont) {
            // combine (combiner.h:9-24): float sum in neighbour order.
            if (success) {
                float term[S];
#pragma unroll
                for (int s = 0; s < S; ++s) term[s] = __double2float_rn(__dmul_rn(w[s], (double)dv[s]));
                float res = J.kind == 1 ? J.sk_mean_f : (J.kind == 2 ? J.mean[node] : 0.f);
                for (int i = 0; i < n; ++i) res = __fadd_rn(res, __shfl_sync(FULL_MASK, pickf<S>(term, i >> 5), i & 31));
                if (lane == 0) {
                    J.out_values[node] = res;
                    J.out_mask[node] = 1;
                }
            } else if (lane == 0) {
                if (J.kind == 0) {
                    // undefined_on_failure: the caller's content stays.
                    const int pos = atomicAdd(J.n_untouched, 1);
                    J.untouched[pos] = node;
                } else {
                    J.out_values[node] = J.kind == 1 ? J.sk_mean_f : J.mean[node];
                    J.out_mask[node] = 1;
                }
            }
        } else if (J.kind == 3) {
            // do_indicator_kriging (indicator_kriging.h:98-114)
            int best = 0;
            double best_p = 0;
            for (int k = J.k0; k < J.k1; ++k) {
                const float pk = J.pk[k];
                float prob = pk;
                if (success) {
                    float term[S];
#pragma unroll
                    for (int s = 0; s < S; ++s)
                        term[s] = __double2float_rn(__dmul_rn(w[s], (double)__fsub_rn(code[s] == k ? 1.f : 0.f, pk)));
                    for (int i = 0; i < n; ++i) prob = __fadd_rn(prob, __shfl_sync(FULL_MASK, pickf<S>(term, i >> 5), i & 31));
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
            // median_ik_for_two_indicators (median_ik.cpp:65-81): double sum.
            const float m = J.median_m;
            double prob = (double)m;
            if (success) {
                double term[S];
#pragma unroll
                for (int s = 0; s < S; ++s)
                    term[s] = __dmul_rn(w[s], (double)__fsub_rn(code[s] == 1 ? 1.f : 0.f, m));
                for (int i = 0; i < n; ++i) prob = __dadd_rn(prob, bcast<S>(term, i));
            }
            if (lane == 0) {
                J.probs[node] = (float)prob;
                J.out_codes[node] = ((float)prob <= 0.5f) ? 0 : 1;
                J.out_mask[node] = 1;
            }
        }
        __syncwarp();
    }
    if (MODE == 0 && lane == 0 && solved64) atomicAdd(J.n_fp64, solved64);
}

// most_probable_category (cdf_utils.cpp:9-24): first maximum wins.
__global__ void k_ik_argmax(DevJob J) {
    long long node = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (node >= J.size) return;
    const float *p = J.probs + node * J.K;
    double best = p[0];
    int bi = 0;
    for (int k = 1; k < J.K; ++k)
        if ((double)p[k] > best) {
            best = p[k];
            bi = k;
        }
    J.out_codes[node] = (uint8_t)bi;
    J.out_mask[node] = 1;
}

// ---------------------------------------------------------------------------
static int sm_count() {
    static const int n = [] {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        return sms > 0 ? sms : 148;
    }();
    return n;
}

void launch_build_bits(const DevJob &J, const DevPlan &P, uint32_t *bits, cudaStream_t s) {
    long long n = (long long)J.ny * J.nz * P.wpr;
    k_build_bits<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(J, P, bits);
}

void launch_search_template(const DevJob &J, const DevPlan &P, cudaStream_t s) {
    const long long segs = (long long)P.nseg * J.ny * J.nz;
    long long blocks = (segs + 7) / 8;
    const long long cap = (long long)sm_count() * 8;  // 8 blocks of 8 warps per SM
    if (blocks > cap) blocks = cap;
    k_search_template<<<(unsigned)std::max<long long>(1, blocks), 256, 0, s>>>(J, P);
}

void launch_search_cluster(const DevJob &J, const DevPlan &P, double *sk, int *si, int n_warps, cudaStream_t s) {
    const int threads = CLUSTER_WARPS * 32;
    k_search_cluster<<<(unsigned)((n_warps * 32 + threads - 1) / threads), threads, 0, s>>>(J, P, sk, si, n_warps);
}

template <int NMAX, int MODE>
static void launch_solve_t(const DevJob &J, const DevPlan &P, const int *list, const int *n_list, long long n_max,
                           cudaStream_t s) {
    using C = SolveCfg<NMAX, MODE>;
    static const int per_sm = [] {
        cudaFuncSetAttribute(k_solve<NMAX, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
        int v = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_solve<NMAX, MODE>, C::WARPS * 32, C::SMEM);
        return v < 1 ? 1 : v;
    }();
    long long blocks = (n_max + C::WARPS - 1) / C::WARPS;
    long long cap = (long long)sm_count() * per_sm * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    k_solve<NMAX, MODE><<<(unsigned)blocks, C::WARPS * 32, C::SMEM, s>>>(J, P, list, n_list);
}

void launch_solve(const DevJob &J, const DevPlan &P, int precision, const int *node_list, const int *n_list,
                  int n_list_max, cudaStream_t s) {
    long long n_max = node_list ? (long long)n_list_max : J.size;
    if (n_max <= 0) return;
    if (P.nmax <= 32) {
        launch_solve32(J, P, precision, node_list, n_list, n_max, s);
        return;
    }
    if (precision == 0 || node_list) launch_solve64_exact(J, P, node_list, n_list, n_max, s);
    else launch_solve_t<64, 1>(J, P, node_list, n_list, n_max, s);
}

void launch_ik_argmax(const DevJob &J, cudaStream_t s) {
    k_ik_argmax<<<(unsigned)((J.size + 255) / 256), 256, 0, s>>>(J);
}

}  // namespace hpgl_b200
