// Checks FastDiv (hpgl_b200/csrc/kernels.cuh), compiled here for the host,
// against integer division: every divisor 1..4096 and the grid extents up
// to 2^16 with edge and random numerators, plus all numerators below 2^22
// for a few divisors.  Prints "ok <checks>" or the first mismatch.
#include <cstdio>
#include <random>
#include "../../hpgl_b200/csrc/kernels.cuh"

using hpgl_b200::FastDiv;

static bool check(unsigned d, unsigned n, long long &count) {
    ++count;
    const FastDiv f(d);
    if (f.div(n) != n / d) {
        printf("mismatch d=%u n=%u got %u want %u\n", d, n, f.div(n), n / d);
        return false;
    }
    return true;
}

int main() {
    std::mt19937 rng(7);
    long long count = 0;
    for (unsigned d = 1; d <= 65536; d = d <= 4096 ? d + 1 : d * 3 / 2 + 1) {
        const unsigned edges[] = {0u, 1u, d - 1, d, d + 1, 2 * d - 1, 2 * d, 0x7fffffffu, 0xfffffffeu, 0xffffffffu};
        for (unsigned n : edges)
            if (!check(d, n, count)) return 1;
        for (int i = 0; i < 2000; ++i)
            if (!check(d, rng(), count)) return 1;
        const unsigned long long top = 0xffffffffull / d;
        for (int i = 0; i < 200; ++i) {
            const unsigned long long q = rng() % (top + 1);
            for (long long dn = -1; dn <= 1; ++dn) {
                const long long n = (long long)(q * d) + dn;
                if (n >= 0 && n <= 0xffffffffll && !check(d, (unsigned)n, count)) return 1;
            }
        }
    }
    const unsigned ds[] = {3u, 7u, 48u, 50u, 200u, 256u, 512u, 641u};
    for (unsigned d : ds)
        for (unsigned n = 0; n < (1u << 22); ++n)
            if (!check(d, n, count)) return 1;
    printf("ok %lld\n", count);
    return 0;
}
