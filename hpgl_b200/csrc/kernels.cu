// CUDA kernels of the kriging pipeline for sm_100a (the per-node solves are
// in solve32.cu and solve64.cu):
//   k_build_bits       informed mask -> padded bit rows
//   k_search_template  bit-sliced walk of the sorted search template
//   k_search_cluster   clusterizer gather, covariance filter, reference sort
//   k_ik_argmax        most probable category
//   k_sgs_*            bookkeeping of the speculative simulation rounds
// Paths cited are relative to the reference's src/geo_bsd/hpgl/.
#include <algorithm>
#include <climits>
#include <cstdio>
#include <map>
#include <mutex>

#include "device_common.cuh"
#include "introsort.h"
#include "search_common.cuh"
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
// Template search: one warp per 32-node x-segment (template_segment in
// search_common.cuh), persistent: each warp takes the next segment from a
// counter, so warps whose segments end early (dense regions) take more and
// none waits on a fixed share at the end.
__global__ void __launch_bounds__(256) k_search_template(DevJob J, DevPlan P) {
    __shared__ int delta_sm[8][32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const long long total = (long long)P.nseg * J.ny * J.nz;
    while (true) {
        int segi = 0;
        if (lane == 0) segi = atomicAdd(J.seg_next, 1);
        segi = __shfl_sync(FULL_MASK, segi, 0);
        if (segi >= total) break;
        template_segment(J, P, segi, lane, delta_sm[wib]);
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
constexpr int CLUSTER_CHUNK = 16;  // nodes a warp takes from the counter at a time

// 16 blocks a SM (32 registers): the engine launches 64 warps a SM
__global__ void __launch_bounds__(CLUSTER_WARPS * 32, 16) k_search_cluster(DevJob J, DevPlan P, double *scratch_key,
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
    // warps take CLUSTER_CHUNK consecutive nodes at a time from a counter:
    // clusterizer-path nodes sit in sparse regions, so a fixed share would
    // leave some warps most of them
    while (true) {
        int chunk = 0;
        if (lane == 0) chunk = atomicAdd(J.node_next, CLUSTER_CHUNK);
        chunk = __shfl_sync(FULL_MASK, chunk, 0);
        if (chunk >= J.size) break;
        const int chunk_end = (int)min((long long)chunk + CLUSTER_CHUNK, (long long)J.size);
        for (int node = chunk; node < chunk_end; ++node) {
            if (!node_needs_kriging(J, node)) continue;
            int x, y, z;
            node_xyz(J, node, x, y, z);
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
                                node_xyz(J, cand, qx, qy, qz);
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

void launch_solve(const DevJob &J, const DevPlan &P, int precision, const uint8_t *routed, cudaStream_t s,
                  int blocks_per_sm) {
    if (J.size <= 0) return;
    if (P.nmax <= 32) {
        launch_solve32(J, P, precision, routed, s, blocks_per_sm);
        return;
    }
    if (precision == 0 || routed) launch_solve64_exact(J, P, routed, s, blocks_per_sm);
    else launch_solve64_mixed(J, P, s, blocks_per_sm);
}

// ---------------------------------------------------------------------------
// Speculative sequential simulation: path ranks, commits and admissions (the
// rounds' kriging is k_sgs_try32 / k_sgs_try64).

__global__ void k_sgs_rank_init(DevJob J, int *rank_of) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < J.size) rank_of[i] = J.mask[i] ? -1 : INT_MAX;
}

__global__ void k_sgs_rank_path(const int *nodes, int *rank_of, long long nsim) {
    const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (r < nsim) rank_of[nodes[r]] = (int)r;
}

__device__ __forceinline__ void sgs_bit(const DevJob &J, const DevPlan &P, int node, long long &w, uint32_t &bit) {
    int x, y, z;
    node_xyz(J, node, x, y, z);
    const int px = x + P.px;
    w = ((long long)z * J.ny + y) * P.wpr + (px >> 5);
    bit = 1u << (px & 31);
}

// The round's try list: the pending nodes of window buffer `cur` without a
// blocker or whose blocker has committed (one counter update per warp); the
// others stay pending untried.
__global__ void __launch_bounds__(256) k_sgs_list(SgsState G, int cur) {
    SgsCtl *ctl = G.ctl;
    const int count = ctl->count[cur];
    const int *win = cur ? G.win1 : G.win0;
    const int lane = threadIdx.x & 31;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < count; base += stride) {
        const int i = base + lane;
        bool tr = false;
        if (i < count) {
            const int b = G.blocker[win[i]];
            tr = b < 0 || G.done[b];
            if (!tr) G.ok[i] = 0;
        }
        const unsigned m = __ballot_sync(FULL_MASK, tr);
        int slot0 = 0;
        if (lane == 0 && m) slot0 = atomicAdd(&ctl->ntry, __popc(m));
        slot0 = __shfl_sync(FULL_MASK, slot0, 0);
        if (tr) G.trylist[slot0 + __popc(m & ((1u << lane) - 1u))] = i;
    }
}

// Commits the nodes of window buffer `cur` that the round kept (informed bit
// set, pending bit cleared, done) and moves the others to the other buffer
// (one counter update per warp).  The last block to finish (a ticket
// counter, no waiting) tops the window up to its size and records the
// admission that k_sgs_admit carries out.
__global__ void __launch_bounds__(256) k_sgs_commit(DevJob J, DevPlan P, SgsState G, int cur) {
    SgsCtl *ctl = G.ctl;
    const int count = *(volatile int *)&ctl->count[cur];
    const int *win = cur ? G.win1 : G.win0;
    int *nxt = cur ? G.win0 : G.win1;
    const int lane = threadIdx.x & 31;
    const int stride = gridDim.x * blockDim.x;
    for (int base = blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < count; base += stride) {
        const int i = base + lane;
        int rank = -1;
        bool keep = false;
        if (i < count) {
            rank = win[i];
            if (G.ok[i]) {
                long long w;
                uint32_t bit;
                sgs_bit(J, P, G.nodes[rank], w, bit);
                atomicOr(J.sim_bits + w, bit);
                atomicAnd(G.pend + w, ~bit);
                G.done[rank] = 1;
            } else {
                keep = true;
            }
        }
        const unsigned km = __ballot_sync(FULL_MASK, keep);
        int slot0 = 0;
        if (lane == 0 && km) slot0 = atomicAdd(&ctl->count[cur ^ 1], __popc(km));
        slot0 = __shfl_sync(FULL_MASK, slot0, 0);
        if (keep) nxt[slot0 + __popc(km & ((1u << lane) - 1u))] = rank;
    }
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&ctl->blocks_done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    const int kept = atomicAdd(&ctl->count[cur ^ 1], 0);
    long long add = (long long)ctl->window - kept;
    if (add < 0) add = 0;
    if (add > ctl->total - ctl->next) add = ctl->total - ctl->next;
    ctl->admit_base = kept;
    ctl->admit = add;
    ctl->next += add;
    ctl->count[cur ^ 1] = kept + (int)add;
    ctl->count[cur] = 0;
    if (count > 0) {
        ctl->rounds += 1;
        ctl->commits += count - kept;
    }
    ctl->tries += ctl->ntry;
    ctl->ntry = 0;
    ctl->blocks_done = 0;
    ctl->cursor = 0;
}

// Appends the admitted path ranks to window buffer `buf` and marks them
// pending.
__global__ void __launch_bounds__(256) k_sgs_admit(DevJob J, DevPlan P, SgsState G, int buf) {
    const SgsCtl *ctl = G.ctl;
    const long long add = ctl->admit, base = ctl->admit_base, first = ctl->next - add;
    int *win = buf ? G.win1 : G.win0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < add;
         k += (long long)gridDim.x * blockDim.x) {
        const int rank = (int)(first + k);
        win[base + k] = rank;
        long long w;
        uint32_t bit;
        sgs_bit(J, P, G.nodes[rank], w, bit);
        atomicOr(G.pend + w, bit);
    }
}

void launch_sgs_ranks(const DevJob &J, const SgsState &G, long long nsim, cudaStream_t s) {
    int *rank_of = const_cast<int *>(G.rank_of);
    k_sgs_rank_init<<<(unsigned)((J.size + 255) / 256), 256, 0, s>>>(J, rank_of);
    if (nsim > 0) k_sgs_rank_path<<<(unsigned)((nsim + 255) / 256), 256, 0, s>>>(G.nodes, rank_of, nsim);
}

static void sgs_commit_admit(const DevJob &J, const DevPlan &P, const SgsState &G, int cur, cudaStream_t s) {
    const unsigned blocks = (unsigned)sm_count() * 4;
    k_sgs_commit<<<blocks, 256, 0, s>>>(J, P, G, cur);
    k_sgs_admit<<<blocks, 256, 0, s>>>(J, P, G, cur ^ 1);
}

void launch_sgs_admit(const DevJob &J, const DevPlan &P, const SgsState &G, int cur, cudaStream_t s) {
    sgs_commit_admit(J, P, G, cur, s);
}

static void sgs_list(const SgsState &G, int cur, cudaStream_t s) {
    k_sgs_list<<<(unsigned)sm_count() * 4, 256, 0, s>>>(G, cur);
}

void launch_sis_round(const DevJob &J, const DevPlan &P0, const DevPlan *plans, int family, const SgsState &G,
                      int cur, cudaStream_t s) {
    sgs_list(G, cur, s);
    if (family == 0) launch_sis_try32(J, plans, G, cur, s);
    else launch_sis_try64(J, plans, G, cur, s);
    sgs_commit_admit(J, P0, G, cur, s);
}

void launch_sgs_round(const DevJob &J, const DevPlan &P, const SgsState &G, int cur, cudaStream_t s) {
    sgs_list(G, cur, s);
    if (P.nmax <= 32) launch_sgs_try32(J, P, G, cur, s);
    else launch_sgs_try64(J, P, G, cur, s);
    sgs_commit_admit(J, P, G, cur, s);
}

long long persistent_grid(const void *fn, int threads, size_t smem, int blocks_per_sm, long long units) {
    // occupancy of each kernel is looked up once
    static std::mutex mu;
    static std::map<const void *, int> occ;
    int per_sm;
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = occ.find(fn);
        if (it == occ.end()) {
            cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            int v = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, fn, threads, smem);
            it = occ.emplace(fn, v < 1 ? 1 : v).first;
        }
        per_sm = it->second;
    }
    if (blocks_per_sm > 0 && blocks_per_sm < per_sm) per_sm = blocks_per_sm;
    const long long cap = (long long)per_sm * sm_count();
    return std::max<long long>(1, std::min(units, cap));
}

namespace {
std::mutex g_tuning_mu;
LaunchTuning g_tuning[2][2];
}  // namespace

LaunchTuning tuning_get(int family, int precision) {
    std::lock_guard<std::mutex> lock(g_tuning_mu);
    return g_tuning[family & 1][precision & 1];
}

void tuning_set(int family, int precision, const LaunchTuning &t) {
    std::lock_guard<std::mutex> lock(g_tuning_mu);
    g_tuning[family & 1][precision & 1] = t;
}

void launch_ik_argmax(const DevJob &J, cudaStream_t s) {
    k_ik_argmax<<<(unsigned)((J.size + 255) / 256), 256, 0, s>>>(J);
}

}  // namespace hpgl_b200
