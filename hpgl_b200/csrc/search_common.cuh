// Template search of one 32-node x-segment, shared by the search kernel and
// the fused search+solve kernels.
#pragma once
#include "device_common.cuh"

namespace hpgl_b200 {

// neighbour_lookup_t::find (sugarbox_neighbour_lookup.h:35-61) for the 32
// nodes of segment `segi` (grid row (y, z), x in [32 seg, 32 seg + 32)): the
// warp walks the sorted template 32 entries at a time; lane t loads entry
// base+t and forms the 32-bit window of informed flags of the segment's 32
// target cells at that offset (one funnel shift of two words of bit row
// (y+dy, z+dz); out-of-grid cells are 0 bits, matching is_informed(-1) ==
// false).  A 32x32 bit transpose across the lanes turns the windows into, for
// node b (lane b), the mask of chunk entries that hit it; lane b appends them
// in template order until it holds max_neighbours.  Nodes that do not take
// the template path (clean clusterizer neighbourhoods) or need no kriging
// never become active.  Lists and counts go to J.nb / J.nbcount.
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

// Returns the segment's first node; dsm is a 32-int per-warp scratch.
__device__ __forceinline__ int template_segment(const DevJob &J, const DevPlan &P, long long segi, int lane,
                                                int *dsm) {
    const int seg = (int)(segi % P.nseg);
    const long long row = segi / P.nseg;
    const int y = (int)(row % J.ny), z = (int)(row / J.ny);
    const int x0 = seg * 32;
    const int base = (int)(row * J.nx) + x0;
    const int node = base + lane;
    const bool act = x0 + lane < J.nx && node_needs_kriging(J, node) && !node_clean(P, x0 + lane, y, z);
    uint32_t active = __ballot_sync(FULL_MASK, act);
    if (!active) return base;
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
    return base;
}

// neighbour_lookup_t::find (sugarbox_neighbour_lookup.h:35-61) for one node:
// the warp tests 32 template entries at a time against the informed-bit rows
// (lane t entry base + t, lanes in template order) and keeps the first
// max_neighbours hits.  List and count go to J.nb / J.nbcount.
__device__ __forceinline__ void template_node(const DevJob &J, const DevPlan &P, int node, int lane) {
    int x, y, z;
    node_xyz(J, node, x, y, z);
    const int nmax = P.nmax;
    int *out = J.nb + (long long)node * nmax;
    int cnt = 0;
    for (int tb = 0; tb < P.tmpl_len && cnt < nmax; tb += 32) {
        const int t = tb + lane;
        bool hit = false;
        int delta = 0;
        if (t < P.tmpl_len) {
            const int4 e = __ldg(&P.tmpl[t]);
            delta = e.w;
            const int yy = y + e.y, zz = z + e.z;
            if ((unsigned)yy < (unsigned)J.ny && (unsigned)zz < (unsigned)J.nz) {
                const int px = x + e.x;  // padded x of the target cell
                hit = (J.bits[((long long)zz * J.ny + yy) * P.wpr + (px >> 5)] >> (px & 31)) & 1u;
            }
        }
        const unsigned b = __ballot_sync(FULL_MASK, hit);
        const int rank = __popc(b & ((1u << lane) - 1u));
        if (hit && cnt + rank < nmax) out[cnt + rank] = node + delta;
        cnt += __popc(b);
    }
    if (lane == 0) J.nbcount[node] = min(cnt, nmax);
}

// One lane's template entry of a speculative search: the informed and
// pending words of its target cell, loaded ahead of their use.
struct SpecProbe {
    int delta;
    uint32_t bit, inf, pen;  // bit == 0: past the template or outside the grid
};

__device__ __forceinline__ SpecProbe spec_probe(const DevJob &J, const DevPlan &P, const SgsState &G, int x, int y,
                                                int z, int t) {
    SpecProbe q{0, 0u, 0u, 0u};
    if (t < P.tmpl_len) {
        const int4 e = __ldg(&P.tmpl[t]);
        q.delta = e.w;
        const int yy = y + e.y, zz = z + e.z;
        if ((unsigned)yy < (unsigned)J.ny && (unsigned)zz < (unsigned)J.nz) {
            const int px = x + e.x;  // padded x of the target cell
            const long long w = ((long long)zz * J.ny + yy) * P.wpr + (px >> 5);
            q.bit = 1u << (px & 31);
            q.inf = __ldg(J.bits + w);
            q.pen = __ldg(G.pend + w);
        }
    }
    return q;
}

// neighbour_lookup_t::find for one node of a speculative simulation round
// (path rank `rank`): as template_node, over the committed nodes of lower
// rank (informed bit set and rank_of below `rank`; informed data have rank
// -1); the list goes to `out`, its length to `count`.  Returns -1 when the
// search completed, else the rank of the first pending node of lower rank met
// before the point where the search would stop: in the sequential order that
// node would have been simulated and seen, so nothing of this search is kept.
// The bits and ranks are read-only while a round's nodes are tried.
__device__ __forceinline__ int template_node_spec(const DevJob &J, const DevPlan &P, const SgsState &G, int node,
                                                  int rank, int lane, int *out, int &count) {
    int x, y, z;
    node_xyz(J, node, x, y, z);
    const int nmax = P.nmax;
    int cnt = 0;
    count = 0;
    // the next chunk's entries and words are loaded while this chunk's ranks
    // are read and its hits counted
    SpecProbe q = spec_probe(J, P, G, x, y, z, lane);
    for (int tb = 0; tb < P.tmpl_len && cnt < nmax; tb += 32) {
        const SpecProbe nq = spec_probe(J, P, G, x, y, z, tb + 32 + lane);
        bool hit = false, conflict = false;
        int r = -1;
        const bool inf = (q.inf & q.bit) != 0, pen = (q.pen & q.bit) != 0;
        if (inf || pen) {  // set bits only inside the grid
            r = __ldg(G.rank_of + node + q.delta);
            hit = inf && r < rank;
            conflict = pen && r < rank;
        }
        const unsigned b = __ballot_sync(FULL_MASK, hit);
        const unsigned c = __ballot_sync(FULL_MASK, conflict);
        if (c) {
            const int first = __ffs(c) - 1;
            const int blocker = __shfl_sync(FULL_MASK, r, first);
            if (cnt + __popc(b & ((1u << first) - 1u)) < nmax) return blocker;
        }
        const int pos = __popc(b & ((1u << lane) - 1u));
        if (hit && cnt + pos < nmax) out[cnt + pos] = node + q.delta;
        cnt += __popc(b);
        q = nq;
    }
    count = min(cnt, nmax);
    return -1;
}

// The next node to try this round, handed out one at a time from the round's
// try list: its window slot and path rank; false once the list is used up.
__device__ __forceinline__ bool sgs_next_try(const SgsState &G, const int *win, int ntry, int lane, int &slot,
                                             int &rank) {
    int k = 0;
    if (lane == 0) k = (int)atomicAdd(&G.ctl->cursor, 1u);
    k = __shfl_sync(FULL_MASK, k, 0);
    if (k >= ntry) return false;
    slot = G.trylist[k];
    rank = win[slot];
    return true;
}

// The simulated value of a kriged node (sequential_simulation.h:106-110,
// gaussian_cdf_t::inverse in gaussian_distribution.h:49-66): xp, the
// standard normal quantile of the node's draw, times sqrt(variance) plus the
// kriged estimate; N(0, 1) when the kriging failed.  The node joins the
// informed set when its round commits.
__device__ __forceinline__ void sgs_value(const DevJob &J, int node, double xp) {
    double v;
    if (J.status[node] == ST_SUCCESS)
        v = __dadd_rn(__dmul_rn(xp, __dsqrt_rn(J.variance[node])), (double)J.out_values[node]);
    else
        v = __dadd_rn(__dmul_rn(xp, 1.0), 0.0);
    J.sim_values[node] = __double2float_rn(v);
    J.sim_mask[node] = 1;
}

// Sequential indicator simulation helpers (sequential_indicator_simulation.cpp).

// The mean of category k at a node: the category's mean cube, or its
// marginal probability (mean_t, float).
__device__ __forceinline__ float sis_mean(const DevJob &J, int k, long long node) {
    return J.sis_lvm ? J.mean[(long long)k * J.size + node] : J.pk[k];
}

// sigma = sqrt(m (1 - m)) of an indicator mean, a mean of exactly 0 or 1
// moved by 1e-5 (corellogramed_weights_3, my_kriging_weights.h:275-305).
__device__ __forceinline__ double sis_sigma(float mean) {
    double m = (double)mean;
    if (m == 0) m = __dadd_rn(m, 0.00001);
    if (m == 1) m = __dsub_rn(m, 0.00001);
    return __dsqrt_rn(__dmul_rn(m, __dsub_rn(1.0, m)));
}

// sample (sample.cpp:8-21): the first category whose running sum of the
// float probabilities (in double) exceeds u times their total; the last one
// otherwise.
__device__ __forceinline__ int sis_sample(const float *probs, int n, double u) {
    double sum = 0.0;
    for (int i = 0; i < n; ++i) sum = __dadd_rn(sum, (double)probs[i]);
    const double s = __dmul_rn(u, sum);
    double p = 0.0;
    for (int i = 0; i < n; ++i) {
        p = __dadd_rn(p, (double)probs[i]);
        if (s < p) return i;
    }
    return n - 1;
}

// Records the outcome of one tried node: its code (and mask) once every
// category's search completed, else its blocker.
__device__ __forceinline__ void sis_finish(const DevJob &J, const SgsState &G, int node, int rank, int slot,
                                           int blocker) {
    if (blocker < 0) {
        J.sim_codes[node] = (uint8_t)sis_sample(J.probs + (long long)node * J.K, J.K, G.xp[rank]);
        J.sim_mask[node] = 1;
    } else {
        G.blocker[rank] = blocker;
    }
    G.ok[slot] = blocker < 0;
}

}  // namespace hpgl_b200
