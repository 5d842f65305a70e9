// Host side of sequential simulation.
//
// Path (path_random_generator.cpp:20-66): a linear congruential walk x ->
// (A x + C) mod size from x0 = seed mod size, A = 1 + the product of the
// distinct primes dividing size (twice that when 4 divides size), C = the
// largest prime <= size / 3 that does not divide size -- full period, so
// every node once.  The reference reads its primes from primes.txt, which its
// checkout lacks; init_rnd's asserts leave one reading of that table (every
// prime in increasing order past the grid size), restated here with a sieve.
//
// Draws (bs_random_generator.cpp, sample.h:14-17, sample.cpp:8-21):
// boost::mt11213b seeded with the seed, one 32-bit output per simulated node
// divided by 2^32 - 1.  Gaussian simulation turns it into the standard
// normal quantile of Odeh and Evans's rational approximation
// (gaussian_distribution.h:49-66) with the C library's log and sqrt -- the GPU
// multiplies it by the kriging standard deviation and adds the kriged mean,
// as gaussian_cdf_t::inverse does; indicator simulation compares it with the
// cumulative category probabilities.
//
// Normal-score transforms (sequential_gaussian_simulation.cpp:32-35, 72-73,
// 97-103, 119-123): the caller's CDF interpolated in float
// (non_parametric_cdf.h:185-260) and the standard normal CDF of Abramowitz and
// Stegun 26.2.17 (gaussian_distribution.h:22-47).  They run here, over the
// host threads, because the C library's log and exp define their bits.
#include "sgs_host.h"

#include "plan.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <stdexcept>
#include <thread>

namespace hpgl_b200 {

namespace {

bool is_prime(long long v) {
    if (v < 2) return false;
    for (long long d = 2; d * d <= v; ++d)
        if (v % d == 0) return false;
    return true;
}

// The walk x -> (A x + C) mod M and its jumps: an affine map composed with
// itself (a, c) -> (a a, a c + c) by doubling, all terms below 2^50 for
// M <= 10^7.
struct Path {
    long long A = 1, C = 2, M = 1, R = 0;
    Path(long long size, long long seed) {
        M = size;
        // A: 1 + the product of the distinct primes dividing size (times 2
        // when 4 divides it)
        long long rest = size;
        for (long long d = 2; d * d <= rest; ++d) {
            if (rest % d) continue;
            A *= d;
            while (rest % d == 0) rest /= d;
        }
        if (rest > 1) A *= rest;
        if (M % 4 == 0) A *= 2;
        A += 1;
        // C: the largest prime <= size / 3 that does not divide size; 2 when
        // there is none (the table's first prime)
        C = 2;
        for (long long c = size / 3; c >= 2; --c) {
            if (size % c != 0 && is_prime(c)) {
                C = c;
                break;
            }
        }
        // path_random_generator_t(int size, int seed) takes the seed as int;
        // a negative one makes the walk leave the grid
        const int s32 = (int)(uint32_t)seed;
        if (s32 < 0) throw std::invalid_argument("the simulation path is undefined for a negative seed");
        R = s32 % size;
    }
    long long step(long long x) const { return (A * x + C) % M; }
    // the position `j` steps after x
    long long jump(long long x, long long j) const {
        long long a = A % M, c = C % M;  // the map of 2^i steps
        long long ja = 1, jc = 0;          // the map of the steps taken so far
        while (j > 0) {
            if (j & 1) {
                ja = ja * a % M;
                jc = (a * jc + c) % M;
            }
            c = (a * c + c) % M;
            a = a * a % M;
            j >>= 1;
        }
        return (ja * x + jc) % M;
    }
};

// The Mersenne Twister (Matsumoto and Nishimura, ACM TOMACS 8(1), 1998) with
// boost's mt11213b parameters: w 32, n 351, m 175, r 19, a 0xccab8ee7,
// tempering (11, 7, 0x31b6ab00, 15, 0xffe50000, 17), seeding with 1812433253.
struct Mt11213b {
    enum { N = 351, M = 175, R = 19 };
    uint32_t x[N];
    int i = N;
    explicit Mt11213b(uint32_t s) {
        x[0] = s;
        for (int k = 1; k < N; ++k) x[k] = 1812433253u * (x[k - 1] ^ (x[k - 1] >> 30)) + (uint32_t)k;
    }
    uint32_t next() {
        if (i >= N) {
            // the in-place twist, its index wrap-around split into three runs
            const uint32_t upper = ~((1u << R) - 1u), lower = (1u << R) - 1u;
            auto twist = [&](int k, int k1, int km) {
                const uint32_t y = (x[k] & upper) | (x[k1] & lower);
                x[k] = x[km] ^ (y >> 1) ^ ((y & 1u) ? 0xccab8ee7u : 0u);
            };
            int k = 0;
            for (; k < N - M; ++k) twist(k, k + 1, k + M);
            for (; k < N - 1; ++k) twist(k, k + 1, k + M - N);
            twist(N - 1, 0, M - 1);
            i = 0;
        }
        uint32_t y = x[i++];
        y ^= y >> 11;
        y ^= (y << 7) & 0x31b6ab00u;
        y ^= (y << 15) & 0xffe50000u;
        y ^= y >> 17;
        return y;
    }
};

double quantile(double p) {
    const double ps[] = {-0.322232431088, -1.0, -0.342242088547, -0.0204231210245, -0.453642210148e-4};
    const double qs[] = {0.0993484626060, 0.588581570495, 0.531103462366, 0.103537752850, 0.38560700634e-2};
    const double p2 = (p > 0.5) ? (1 - p) : p;
    const double y = std::sqrt(std::log(1 / (p2 * p2)));
    double xp = y + ((((ps[4] * y + ps[3]) * y + ps[2]) * y + ps[1]) * y + ps[0]) /
                        ((((qs[4] * y + qs[3]) * y + qs[2]) * y + qs[1]) * y + qs[0]);
    if (p < 0.5) xp = -xp;
    return xp;
}

}  // namespace

namespace {

template <typename F>
void parallel_for(long long n, int threads, F f) {
    const long long chunk = 1 << 16;
    const int t = (int)std::max<long long>(1, std::min<long long>(threads, (n + chunk - 1) / chunk));
    if (t <= 1) {
        f(0, n);
        return;
    }
    std::vector<std::thread> pool;
    const long long per = (n + t - 1) / t;
    for (int k = 0; k < t; ++k) {
        const long long a = k * per, b = std::min(n, a + per);
        if (a < b) pool.emplace_back([=] { f(a, b); });
    }
    for (auto &th : pool) th.join();
}

// std::lower_bound over a sorted float array, narrowed by buckets of its
// range: thresholds t[0] <= ... <= t[nb] (floats) and lo[b] = lower_bound(t[b]).
// A query v with t[b] <= v < t[b + 1] has its lower bound in [lo[b], lo[b + 1]]:
// everything before lo[b] is below t[b] <= v, and the element at lo[b + 1] is
// >= t[b + 1] > v.  Queries outside [t[0], t[nb]), NaN, and arrays holding a
// NaN take the whole range.  The result is std::lower_bound's.
struct SortedIndex {
    const float *a;
    long long n;
    int nb = 0;
    double base = 0, scale = 0;
    std::vector<float> t;
    std::vector<int> lo;
    SortedIndex(const float *arr, long long count, int buckets) : a(arr), n(count) {
        if (n < 2 || n > 0x7fffffffLL) return;
        for (long long i = 0; i < n; ++i)
            if (!std::isfinite(a[i])) return;
        const double v0 = a[0], v1 = a[n - 1];
        if (!(v1 > v0)) return;
        nb = buckets;
        base = v0;
        scale = nb / (v1 - v0);
        t.resize((size_t)nb + 1);
        lo.resize((size_t)nb + 1);
        for (int b = 0; b <= nb; ++b) {
            t[b] = (float)(v0 + b / scale);
            if (b > 0 && t[b] < t[b - 1]) t[b] = t[b - 1];
            lo[b] = (int)(std::lower_bound(a, a + n, t[b]) - a);
        }
    }
    const float *lower_bound(float v) const {
        if (nb == 0 || !(v >= t[0] && v < t[nb])) return std::lower_bound(a, a + n, v);
        int b = (int)((v - base) * scale);
        b = std::min(std::max(b, 0), nb - 1);
        while (b > 0 && v < t[b]) --b;
        while (b + 1 < nb && v >= t[b + 1]) ++b;
        return std::lower_bound(a + lo[b], a + lo[b + 1], v);
    }
};

// non_parametric_cdf_2_t::operator() (non_parametric_cdf.h:202-228): float
// interpolation between the bracketing values; it = lower_bound(values, value).
float npcdf_prob_at(const NonParametricCdf &c, float value, const float *it) {
    if (it == c.values + c.size) return c.probs[c.size - 1];
    if (it == c.values) return c.probs[0];
    const long long i2 = it - c.values, i1 = i2 - 1;
    const float x1 = c.values[i1], x2 = c.values[i2], y1 = c.probs[i1], y2 = c.probs[i2];
    return y1 + (y2 - y1) / (x2 - x1) * (value - x1);
}

// non_parametric_cdf_2_t::inverse (non_parametric_cdf.h:230-257), given
// it = lower_bound(probs, prob).
float npcdf_inverse_at(const NonParametricCdf &c, float prob, const float *it) {
    if (c.size <= 0) return 0;
    if (it == c.probs) return c.values[0];
    if (it == c.probs + c.size) return c.values[c.size - 1];
    const long long i2 = it - c.probs, i1 = i2 - 1;
    const float x1 = c.values[i1], x2 = c.values[i2], y1 = c.probs[i1], y2 = c.probs[i2];
    return x1 + (x2 - x1) / (y2 - y1) * (prob - y1);
}

// gaussian_cdf_t::operator() with mean 0 and variance 1
// (gaussian_distribution.h:22-41).
double gaussian_prob(double x) {
    const double p = 0.2316419;
    const double b[] = {0.319381530, -0.356563782, 1.781477937, -1.821255978, 1.330274429};
    double sx = (x - 0.0) / std::sqrt(1.0);
    const bool neg = sx < 0;
    if (neg) sx = -sx;
    const double t = 1 / (1 + p * sx);
    const double zx = 1 / std::sqrt(2 * 3.14159265358) * std::exp(-sx * sx / 2);
    double result = 1 - zx * ((((b[4] * t + b[3]) * t + b[2]) * t + b[1]) * t + b[0]) * t;
    if (neg) result = 1 - result;
    return result;
}

}  // namespace

void check_sim_path(long long size, long long seed) {
    if (size > 10000000LL)
        throw std::domain_error("the simulation path is defined for grids of at most 10^7 nodes");
    if ((int)(uint32_t)seed < 0)
        throw std::invalid_argument("the simulation path is undefined for a negative seed");
}

void sim_path(int nx, int ny, int nz, const uint8_t *mask, const uint8_t *sim_mask, long long seed, bool quantiles,
              SimPath &out) {
    const long long size = (long long)nx * ny * nz;
    out.nodes.clear();
    out.u.clear();
    if (size <= 0) return;
    check_sim_path(size, seed);
    const Path path(size, seed);
    // The draws do not depend on the walk: one thread runs the generator
    // while the others walk their stretches of the path (from jumps) and then
    // turn the finished stretches of draws into quantiles, in place, behind
    // the generator (`produced` publishes its progress).
    std::vector<double> u;
    u.reserve((size_t)size);
    double *const ud = u.data();
    std::atomic<long long> needed{size}, produced{0};
    std::thread draws([&] {
        Mt11213b gen((uint32_t)seed);
        long long k = 0;
        for (; k < needed.load(std::memory_order_relaxed); ++k) {
            u.push_back(double(gen.next()) / double(0xffffffffu));
            if ((k & 4095) == 4095) produced.store(k + 1, std::memory_order_release);
        }
        produced.store(k, std::memory_order_release);
    });
    // A - 1 holds every prime factor of the size (and 4 when 4 divides it),
    // so the walk visits every node once exactly when gcd(C, size) = 1
    // (Hull and Dobell).  The fallback C = 2 of sizes 2, 4, 6, 8 and 12
    // divides the size: that walk repeats nodes, and the reference skips a
    // repeated node as already simulated -- done here by a single thread.
    long long g = path.C, h = size;
    while (h) {
        const long long r = g % h;
        g = h;
        h = r;
    }
    const bool full_period = g == 1;
    const int t = full_period ? (int)std::max<long long>(1, std::min<long long>(host_threads(), size / (1 << 16))) : 1;
    std::vector<std::vector<int>> part((size_t)t);
    const long long per = (size + t - 1) / t;
    std::vector<std::thread> pool;
    for (int i = 0; i < t; ++i) {
        pool.emplace_back([&, i] {
            const long long a = i * per, b = std::min(size, a + per);
            long long x = path.jump(path.R, a);
            std::vector<int> &v = part[(size_t)i];
            std::vector<char> seen(full_period ? 0 : (size_t)size, 0);
            for (long long k = a; k < b; ++k, x = path.step(x)) {
                if (mask[x]) continue;
                if (sim_mask && sim_mask[x] != 1) continue;
                if (!full_period) {
                    if (seen[(size_t)x]) continue;
                    seen[(size_t)x] = 1;
                }
                v.push_back((int)x);
            }
        });
    }
    for (auto &th : pool) th.join();
    pool.clear();
    size_t count = 0;
    for (auto &v : part) count += v.size();
    needed = (long long)count;
    if (quantiles) {
        constexpr long long CH = 1 << 15;
        std::atomic<long long> next{0};
        const long long n = (long long)count;
        const int w = std::max(1, host_threads() - 1);
        for (int i = 0; i < w; ++i) {
            pool.emplace_back([&] {
                for (long long c = next.fetch_add(1); c * CH < n; c = next.fetch_add(1)) {
                    const long long a = c * CH, b = std::min(n, a + CH);
                    while (produced.load(std::memory_order_acquire) < b) std::this_thread::yield();
                    for (long long k = a; k < b; ++k) ud[k] = quantile(ud[k]);
                }
            });
        }
    }
    out.nodes.reserve(count);
    for (auto &v : part) out.nodes.insert(out.nodes.end(), v.begin(), v.end());
    for (auto &th : pool) th.join();
    draws.join();
    u.resize(count);
    out.u.swap(u);
}

void cdf_to_gaussian(const NonParametricCdf &cdf, const float *in, float *out, const uint8_t *mask, long long n,
                     int threads) {
    const SortedIndex index(cdf.values, cdf.size, 1 << 16);
    parallel_for(n, threads, [&](long long a, long long b) {
        for (long long i = a; i < b; ++i) {
            if (mask && !mask[i]) continue;
            const double P = npcdf_prob_at(cdf, in[i], index.lower_bound(in[i]));
            out[i] = (float)(quantile(P) * std::sqrt(1.0) + 0.0);
        }
    });
}

void gaussian_to_cdf(const NonParametricCdf &cdf, float *values, const uint8_t *mask, long long n, int threads) {
    const SortedIndex index(cdf.probs, cdf.size, 1 << 16);
    parallel_for(n, threads, [&](long long a, long long b) {
        for (long long i = a; i < b; ++i) {
            if (!mask[i]) continue;
            const float p = (float)gaussian_prob(values[i]);
            values[i] = npcdf_inverse_at(cdf, p, index.lower_bound(p));
        }
    });
}

}  // namespace hpgl_b200
