// Order of equal keys under the reference's std::sort.
//
// The reference ranks clusterizer candidates with std::sort on entries
// ordered by covariance, descending (sugarbox_indexed_neighbour_lookup.h:13-37,
// :99).  std::sort is not stable, so which of several equally-covariant
// candidates come first — and therefore which of them make the cut at
// max_neighbours — is decided by the sort algorithm itself.  The reference
// is built with GCC's libstdc++, whose std::sort is an introsort:
//   * an introspective quicksort loop on ranges longer than 16 elements with
//     a depth budget of 2*floor(log2 n); each step moves the median of
//     (first+1, middle, last-1) to `first` and Hoare-partitions the rest
//     around it without bounds checks; the right part is sorted recursively,
//     the loop continues on the left part; an exhausted budget heap-sorts
//     the range (make_heap + sort_heap);
//   * a final insertion sort: guarded over the first 16 elements, unguarded
//     linear insertion for the rest.
// This header restates those published steps for a key/index array pair so
// the device can reproduce the exact permutation.  It is compiled for host
// and device; a CPU test compares it with std::sort on tie-heavy inputs.
#pragma once

#ifdef __CUDACC__
#define HPGL_HD __host__ __device__ __forceinline__
#else
#define HPGL_HD inline
#endif

namespace hpgl_b200 {

struct SortArr {
    double *key;
    int *idx;
    // "a before b": larger covariance first.
    HPGL_HD bool before(int a, int b) const { return key[a] > key[b]; }
    HPGL_HD bool before_val(double ka, int b) const { return ka > key[b]; }
    HPGL_HD bool val_before(int a, double kb) const { return key[a] > kb; }
    HPGL_HD void swap(int a, int b) {
        double tk = key[a];
        key[a] = key[b];
        key[b] = tk;
        int ti = idx[a];
        idx[a] = idx[b];
        idx[b] = ti;
    }
    HPGL_HD void copy(int dst, int src) {
        key[dst] = key[src];
        idx[dst] = idx[src];
    }
};

HPGL_HD int sort_floor_log2(int n) {
    int r = 0;
    while (n > 1) {
        n >>= 1;
        ++r;
    }
    return r;
}

HPGL_HD void sort_median_to_first(SortArr &a, int result, int x, int y, int z) {
    if (a.before(x, y)) {
        if (a.before(y, z)) a.swap(result, y);
        else if (a.before(x, z)) a.swap(result, z);
        else a.swap(result, x);
    } else if (a.before(x, z)) {
        a.swap(result, x);
    } else if (a.before(y, z)) {
        a.swap(result, z);
    } else {
        a.swap(result, y);
    }
}

// Hoare partition of [lo, hi) around the element at `pivot` (outside the
// range), scanning without bounds checks: the median-of-three guarantees a
// stopper on each side.
HPGL_HD int sort_partition(SortArr &a, int lo, int hi, int pivot) {
    while (true) {
        while (a.before(lo, pivot)) ++lo;
        --hi;
        while (a.before(pivot, hi)) --hi;
        if (!(lo < hi)) return lo;
        a.swap(lo, hi);
        ++lo;
    }
}

// The same partition computed from its stoppers, the form a warp evaluates
// in parallel.  Left stoppers L_0 < L_1 < ... are the positions of
// [lo, hi) whose element is not before the pivot, right stoppers
// R_0 > R_1 > ... the positions of [pivot, hi) the pivot is not before.  The
// scans of sort_partition meet stopper k on each side at step k while
// L_k < R_k, and every such step swaps the pair (L_k, R_k), which no other
// step touches; with m the first k where L_k >= R_k, the left scan of the
// last step stops at L_m or, if that lies past R_{m-1}, at R_{m-1} (which
// holds the swapped-in element of L_{m-1}, a left stopper).  So the result is
// m disjoint swaps and cut = min(L_m, R_{m-1}).  `lbuf`/`rbuf` hold up to
// hi - pivot positions each.
HPGL_HD int sort_partition_pairs(SortArr &a, int lo, int hi, int pivot, int *lbuf, int *rbuf) {
    int nl = 0, nr = 0;
    for (int p = lo; p < hi; ++p)
        if (!a.before(p, pivot)) lbuf[nl++] = p;
    for (int q = hi - 1; q >= pivot; --q)
        if (!a.before(pivot, q)) rbuf[nr++] = q;
    int m = 0;
    while (m < nl && m < nr && lbuf[m] < rbuf[m]) ++m;
    for (int k = 0; k < m; ++k) a.swap(lbuf[k], rbuf[k]);
    const int lm = m < nl ? lbuf[m] : 0x7fffffff;
    const int rm = m > 0 ? rbuf[m - 1] : 0x7fffffff;
    return lm < rm ? lm : rm;
}

// Sift the value (vk, vi) down from `hole` in the heap [first, first+len),
// then up towards `top`.
HPGL_HD void sort_adjust_heap(SortArr &a, int first, int hole, int len, double vk, int vi) {
    const int top = hole;
    int child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (a.before(first + child, first + child - 1)) child--;
        a.copy(first + hole, first + child);
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        a.copy(first + hole, first + child - 1);
        hole = child - 1;
    }
    int parent = (hole - 1) / 2;
    while (hole > top && a.val_before(first + parent, vk)) {
        a.copy(first + hole, first + parent);
        hole = parent;
        parent = (hole - 1) / 2;
    }
    a.key[first + hole] = vk;
    a.idx[first + hole] = vi;
}

HPGL_HD void sort_heapsort(SortArr &a, int first, int last) {
    int len = last - first;
    if (len >= 2) {
        for (int parent = (len - 2) / 2;; --parent) {
            double vk = a.key[first + parent];
            int vi = a.idx[first + parent];
            sort_adjust_heap(a, first, parent, len, vk, vi);
            if (parent == 0) break;
        }
    }
    while (last - first > 1) {
        --last;
        double vk = a.key[last];
        int vi = a.idx[last];
        a.copy(last, first);
        sort_adjust_heap(a, first, 0, last - first, vk, vi);
    }
}

HPGL_HD void sort_linear_insert(SortArr &a, int pos) {
    double vk = a.key[pos];
    int vi = a.idx[pos];
    int next = pos - 1;
    while (a.before_val(vk, next)) {
        a.copy(pos, next);
        pos = next;
        --next;
    }
    a.key[pos] = vk;
    a.idx[pos] = vi;
}

HPGL_HD void sort_insertion(SortArr &a, int first, int last) {
    if (first == last) return;
    for (int i = first + 1; i < last; ++i) {
        if (a.before(i, first)) {
            double vk = a.key[i];
            int vi = a.idx[i];
            for (int j = i; j > first; --j) a.copy(j, j - 1);
            a.key[first] = vk;
            a.idx[first] = vi;
        } else {
            sort_linear_insert(a, i);
        }
    }
}

// Sorts [0, n) like the reference's std::sort.  Returns false only if the
// explicit stack would overflow (it cannot for n < 2^31: the depth budget
// bounds the pending right-hand parts).
HPGL_HD bool reference_sort(SortArr &a, int n) {
    if (n <= 1) return true;
    struct Frame { int lo, hi, depth; };
    Frame stack[72];
    int sp = 0;
    stack[sp++] = Frame{0, n, 2 * sort_floor_log2(n)};
    while (sp > 0) {
        Frame f = stack[--sp];
        int lo = f.lo, hi = f.hi, depth = f.depth;
        while (hi - lo > 16) {
            if (depth == 0) {
                sort_heapsort(a, lo, hi);
                break;
            }
            --depth;
            int mid = lo + (hi - lo) / 2;
            sort_median_to_first(a, lo, lo + 1, mid, hi - 1);
            int cut = sort_partition(a, lo + 1, hi, lo);
            if (sp >= 72) return false;
            stack[sp++] = Frame{cut, hi, depth};  // ranges are disjoint: order of processing is free
            hi = cut;
        }
    }
    if (n > 16) {
        sort_insertion(a, 0, 16);
        for (int i = 16; i < n; ++i) sort_linear_insert(a, i);
    } else {
        sort_insertion(a, 0, n);
    }
    return true;
}

// The first `k` positions of reference_sort's result, without sorting the
// rest.  Sub-ranges are processed independently and the final insertion sort
// only moves elements within runs of at most 16, so a right-hand part that
// starts at or beyond k, and insertions of elements at or beyond k + 16,
// cannot change positions below k: skipping them leaves [0, k) exactly as
// the full sort would.
HPGL_HD bool reference_sort_prefix(SortArr &a, int n, int k) {
    if (n <= 1) return true;
    if (k >= n) return reference_sort(a, n);
    struct Frame { int lo, hi, depth; };
    Frame stack[72];
    int sp = 0;
    stack[sp++] = Frame{0, n, 2 * sort_floor_log2(n)};
    while (sp > 0) {
        Frame f = stack[--sp];
        int lo = f.lo, hi = f.hi, depth = f.depth;
        if (lo >= k) continue;
        while (hi - lo > 16) {
            if (depth == 0) {
                sort_heapsort(a, lo, hi);
                break;
            }
            --depth;
            int mid = lo + (hi - lo) / 2;
            sort_median_to_first(a, lo, lo + 1, mid, hi - 1);
            int cut = sort_partition(a, lo + 1, hi, lo);
            if (cut < k) {
                if (sp >= 72) return false;
                stack[sp++] = Frame{cut, hi, depth};
            }
            hi = cut;
        }
    }
    const int end = (k + 16 < n) ? k + 16 : n;
    if (n > 16) {
        sort_insertion(a, 0, 16);
        for (int i = 16; i < end; ++i) sort_linear_insert(a, i);
    } else {
        sort_insertion(a, 0, n);
    }
    return true;
}

}  // namespace hpgl_b200
