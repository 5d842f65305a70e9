// ORACLE shim — test infrastructure only.  Stands in for boost::random's
// mersenne_twister so that the reference's sequential-simulation sources
// compile here: the Mersenne Twister of Matsumoto and Nishimura (ACM TOMACS
// 8(1), 1998) with boost's published mt11213b parameters (w = 32, n = 351,
// m = 175, r = 19, a = 0xccab8ee7, u = 11, s = 7, b = 0x31b6ab00, t = 15,
// c = 0xffe50000, l = 17) and the usual seeding x[i] = 1812433253 (x[i-1] ^
// (x[i-1] >> 30)) + i; default seed 5489.
#ifndef ORACLE_SHIM_BOOST_MERSENNE_TWISTER_HPP
#define ORACLE_SHIM_BOOST_MERSENNE_TWISTER_HPP
#include <cstdint>

#ifndef BOOST_PREVENT_MACRO_SUBSTITUTION
#define BOOST_PREVENT_MACRO_SUBSTITUTION
#endif

namespace boost {
namespace random {

template <int N, int M, int R, uint32_t A, int U, int S, uint32_t B, int T, uint32_t C, int L>
class mt32 {
    uint32_t x[N];
    int i;

    void twist() {
        const uint32_t upper = ~((1u << R) - 1u), lower = (1u << R) - 1u;
        for (int k = 0; k < N; ++k) {
            const uint32_t y = (x[k] & upper) | (x[(k + 1) % N] & lower);
            x[k] = x[(k + M) % N] ^ (y >> 1) ^ ((y & 1u) ? A : 0u);
        }
        i = 0;
    }

public:
    typedef uint32_t result_type;
    mt32() { seed(5489u); }
    explicit mt32(uint32_t v) { seed(v); }
    void seed(uint32_t v) {
        x[0] = v;
        for (int k = 1; k < N; ++k) x[k] = 1812433253u * (x[k - 1] ^ (x[k - 1] >> 30)) + (uint32_t)k;
        i = N;
    }
    static uint32_t min BOOST_PREVENT_MACRO_SUBSTITUTION() { return 0u; }
    static uint32_t max BOOST_PREVENT_MACRO_SUBSTITUTION() { return 0xffffffffu; }
    uint32_t operator()() {
        if (i >= N) twist();
        uint32_t y = x[i++];
        y ^= y >> U;
        y ^= (y << S) & B;
        y ^= (y << T) & C;
        y ^= y >> L;
        return y;
    }
};

}  // namespace random

typedef random::mt32<351, 175, 19, 0xccab8ee7u, 11, 7, 0x31b6ab00u, 15, 0xffe50000u, 17> mt11213b;

}  // namespace boost
#endif
