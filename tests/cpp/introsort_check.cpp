// Compares the device introsort restatement (hpgl_b200/csrc/introsort.h),
// compiled here for the host, with std::sort on tie-heavy inputs: the
// permutation of equal keys must be identical.  Prints "ok <cases>" or the
// first mismatch and exits non-zero.
#include <algorithm>
#include <cstdio>
#include <random>
#include <vector>
#include "../../hpgl_b200/csrc/introsort.h"

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
