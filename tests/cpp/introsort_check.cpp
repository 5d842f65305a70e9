// Compares the device introsort restatement (hpgl_b200/csrc/introsort.h),
// compiled here for the host, with std::sort on tie-heavy inputs: the
// permutation of equal keys must be identical.  Prints "ok <cases>" or the
// first mismatch and exits non-zero.
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <random>
#include <vector>
#include "../../hpgl_b200/csrc/introsort.h"

// Lane-by-lane emulation of the warp partition of the clusterizer kernel
// (warp_partition in hpgl_b200/csrc/kernels.cu): every ballot, buffer write
// and shuffle of the device code, with the 32 lanes run in a loop.
static int warp_partition_emulated(hpgl_b200::SortArr &a, int lo, int hi, int pivot) {
    const double pk = a.key[pivot];
    int lp = lo, lend = hi - 1, rp = hi - 1, rend = pivot, rprev = INT_MAX;
    while (true) {
        int lbuf[32], rbuf[32], my_l[32], my_r[32];
        int cnt = 0;
        for (int p0 = lp; cnt < 32 && p0 <= lend; p0 += 32) {
            bool st[32];
            uint32_t bal = 0;
            for (int lane = 0; lane < 32; ++lane) {
                const int p = p0 + lane;
                st[lane] = p <= lend && !(a.key[p] > pk);
                if (st[lane]) bal |= 1u << lane;
            }
            for (int lane = 0; lane < 32; ++lane) {
                const int r = cnt + __builtin_popcount(bal & ((1u << lane) - 1));
                if (st[lane] && r < 32) lbuf[r] = p0 + lane;
            }
            cnt += __builtin_popcount(bal);
        }
        for (int lane = 0; lane < 32; ++lane) my_l[lane] = lane < cnt ? lbuf[lane] : INT_MAX;
        cnt = 0;
        for (int q0 = rp; cnt < 32 && q0 >= rend; q0 -= 32) {
            bool st[32];
            uint32_t bal = 0;
            for (int lane = 0; lane < 32; ++lane) {
                const int q = q0 - lane;
                st[lane] = q >= rend && !(pk > a.key[q]);
                if (st[lane]) bal |= 1u << lane;
            }
            for (int lane = 0; lane < 32; ++lane) {
                const int r = cnt + __builtin_popcount(bal & ((1u << lane) - 1));
                if (st[lane] && r < 32) rbuf[r] = q0 - lane;
            }
            cnt += __builtin_popcount(bal);
        }
        for (int lane = 0; lane < 32; ++lane) my_r[lane] = lane < cnt ? rbuf[lane] : INT_MIN;
        uint32_t pairs = 0;
        for (int lane = 0; lane < 32; ++lane)
            if (my_l[lane] < my_r[lane]) pairs |= 1u << lane;
        const int m = __builtin_popcount(pairs);
        for (int lane = 0; lane < 32; ++lane)
            if (pairs >> lane & 1) a.swap(my_l[lane], my_r[lane]);
        if (m < 32) {
            const int lm = my_l[m];
            const int rm = m > 0 ? my_r[m - 1] : rprev;
            return lm < rm ? lm : rm;
        }
        lp = my_l[31] + 1;
        lend = my_r[31];
        rp = my_r[31] - 1;
        rend = my_l[31];
        rprev = my_r[31];
    }
}

int main(int argc, char **argv) {
    int cases = argc > 1 ? atoi(argv[1]) : 20000;
    std::mt19937_64 rng(12345);
    for (int c = 0; c < cases; ++c) {
        int n = (int)(rng() % (c % 10 == 0 ? 6000 : 400));
        int distinct = 1 + (int)(rng() % (c % 3 == 0 ? 4 : (c % 3 == 1 ? 40 : 100000)));
        struct E { int index; double cov; };
        std::vector<E> ref(n);
        std::vector<double> key(n);
        std::vector<int> idx(n);
        for (int i = 0; i < n; ++i) {
            double k = (double)(rng() % distinct) * 0.125;
            if (c % 7 == 0) k = (double)((n - i) / 3);        // descending runs
            if (c % 11 == 0) k = (double)(i / 5);             // ascending runs
            ref[i] = E{i, k};
            key[i] = k;
            idx[i] = i;
        }
        std::sort(ref.begin(), ref.end(), [](const E &a, const E &b) { return a.cov > b.cov; });
        hpgl_b200::SortArr a{key.data(), idx.data()};
        if (!hpgl_b200::reference_sort(a, n)) { printf("stack overflow n=%d\n", n); return 2; }
        for (int i = 0; i < n; ++i)
            if (ref[i].index != idx[i] || ref[i].cov != key[i]) {
                printf("mismatch case %d n=%d at %d: ref %d got %d\n", c, n, i, ref[i].index, idx[i]);
                return 1;
            }
    }
    // The stopper-pair form of the partition: same array, same cut.
    for (int c = 0; c < cases; ++c) {
        int n = 17 + (int)(rng() % (c % 10 == 0 ? 5000 : 300));
        int distinct = 1 + (int)(rng() % (c % 3 == 0 ? 3 : (c % 3 == 1 ? 30 : 100000)));
        std::vector<double> k1(n), k2;
        std::vector<int> i1(n), i2;
        for (int i = 0; i < n; ++i) {
            k1[i] = (double)(rng() % distinct);
            i1[i] = i;
        }
        hpgl_b200::SortArr a1{k1.data(), i1.data()};
        hpgl_b200::sort_median_to_first(a1, 0, 1, n / 2, n - 1);
        k2 = k1;
        i2 = i1;
        hpgl_b200::SortArr a2{k2.data(), i2.data()};
        std::vector<int> lb(n), rb(n);
        const int c1 = hpgl_b200::sort_partition(a1, 1, n, 0);
        const int c2 = hpgl_b200::sort_partition_pairs(a2, 1, n, 0, lb.data(), rb.data());
        if (c1 != c2 || i1 != i2) {
            printf("partition mismatch case %d n=%d cut %d vs %d\n", c, n, c1, c2);
            return 1;
        }
    }
    // The warp partition: same array, same cut, on ranges long enough for
    // several rounds of 32 pairs.
    for (int c = 0; c < cases; ++c) {
        int n = 17 + (int)(rng() % (c % 10 == 0 ? 8000 : 700));
        int distinct = 1 + (int)(rng() % (c % 4 == 0 ? 2 : (c % 4 == 1 ? 5 : (c % 4 == 2 ? 60 : 100000))));
        std::vector<double> k1(n), k2;
        std::vector<int> i1(n), i2;
        for (int i = 0; i < n; ++i) {
            k1[i] = (double)(rng() % distinct);
            if (c % 9 == 0) k1[i] = (double)((n - i) / 4);
            if (c % 13 == 0) k1[i] = (double)(i / 6);
            i1[i] = i;
        }
        hpgl_b200::SortArr a1{k1.data(), i1.data()};
        hpgl_b200::sort_median_to_first(a1, 0, 1, n / 2, n - 1);
        k2 = k1;
        i2 = i1;
        hpgl_b200::SortArr a2{k2.data(), i2.data()};
        const int c1 = hpgl_b200::sort_partition(a1, 1, n, 0);
        const int c2 = warp_partition_emulated(a2, 1, n, 0);
        if (c1 != c2 || i1 != i2) {
            printf("warp partition mismatch case %d n=%d cut %d vs %d\n", c, n, c1, c2);
            return 1;
        }
    }
    // The prefix variant: first k positions equal to the full sort's.
    for (int c = 0; c < cases; ++c) {
        int n = (int)(rng() % (c % 10 == 0 ? 6000 : 600));
        int k = 1 + (int)(rng() % 70);
        int distinct = 1 + (int)(rng() % (c % 3 == 0 ? 4 : (c % 3 == 1 ? 40 : 100000)));
        struct E { int index; double cov; };
        std::vector<E> ref(n);
        std::vector<double> key(n);
        std::vector<int> idx(n);
        for (int i = 0; i < n; ++i) {
            double kk = (double)(rng() % distinct) * 0.25;
            if (c % 7 == 0) kk = (double)((n - i) / 3);
            ref[i] = E{i, kk};
            key[i] = kk;
            idx[i] = i;
        }
        std::sort(ref.begin(), ref.end(), [](const E &a, const E &b) { return a.cov > b.cov; });
        hpgl_b200::SortArr a{key.data(), idx.data()};
        if (!hpgl_b200::reference_sort_prefix(a, n, k)) { printf("stack overflow\n"); return 2; }
        for (int i = 0; i < k && i < n; ++i)
            if (ref[i].index != idx[i]) {
                printf("prefix mismatch case %d n=%d k=%d at %d\n", c, n, k, i);
                return 1;
            }
    }
    // The depth-budget fallback: heap sort of a range, as std::partial_sort
    // over the whole range (heap_select + sort_heap).
    for (int c = 0; c < cases / 10; ++c) {
        int n = (int)(rng() % 300);
        int distinct = 1 + (int)(rng() % 20);
        struct E { int index; double cov; };
        std::vector<E> ref(n);
        std::vector<double> key(n);
        std::vector<int> idx(n);
        for (int i = 0; i < n; ++i) {
            double k = (double)(rng() % distinct);
            ref[i] = E{i, k};
            key[i] = k;
            idx[i] = i;
        }
        std::partial_sort(ref.begin(), ref.end(), ref.end(), [](const E &a, const E &b) { return a.cov > b.cov; });
        hpgl_b200::SortArr a{key.data(), idx.data()};
        hpgl_b200::sort_heapsort(a, 0, n);
        for (int i = 0; i < n; ++i)
            if (ref[i].index != idx[i]) {
                printf("heap mismatch case %d n=%d at %d\n", c, n, i);
                return 1;
            }
    }
    printf("ok %d\n", cases);
    return 0;
}
