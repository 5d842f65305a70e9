// Number <-> text conversions of the Eclipse INC and GSLIB readers and
// writers (read_inc_file.cpp:54-122, property_writer.cpp:18-26), written once
// for the device kernels of textio.cu and for a host build that the tests
// compare against the C library.
//
// The reference reads each value token with sscanf("%f") or sscanf("%d") and
// writes each value with fprintf("%E\n") of the value widened to double, or
// fprintf("%d\n") of (int)(char)byte.  These functions give the same results
// for every token of at most 255 characters:
//
//  scan_f32  the "%f" conversion: optional sign; "inf" / "infinity" (a token
//            that starts "infi" must spell "infinity", else no match); "nan"
//            followed by anything; "0x" hex significands (a digit or '.' must
//            follow the "0x"; an optional 'p' exponent); decimal significands
//            with at least one digit and an optional 'e' exponent, which is
//            ignored when no digit follows it.  Decimal strings are rounded
//            to nearest-even exactly: a double-precision fast path (Clinger,
//            "How to Read Floating Point Numbers Accurately", PLDI 1990, with
//            a check that the double is not a binary32 halfway point), and
//            otherwise a big-integer comparison of the decimal value with the
//            halfway points next to a candidate (Clinger's Algorithm R
//            idea).  Hex strings are rounded to nearest-even as glibc 2.39
//            does, including its treatment of subnormal results, where the
//            bit 24 places below the leading bit does not count as sticky.
//  scan_int  the "%d" conversion: optional sign, at least one digit, the
//            value saturated to the 64-bit range and then truncated to int.
//  format_E  "%E" of a binary32 value widened to double: exact decimal digits
//            rounded to nearest-even, "INF", "NAN", sign of NaN kept.
//  format_d  "%d".
#pragma once
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define NT_FN __host__ __device__ inline
#define NT_SLOW __host__ __device__ __noinline__
#else
#define NT_FN inline
#define NT_SLOW inline
#endif

namespace hpgl_b200 {
namespace numtext {

typedef unsigned __int128 u128;

NT_FN bool is_ws(unsigned c) { return c == ' ' || (c - 9u) <= 4u; }  // " \t\n\v\f\r"
NT_FN bool is_dig(unsigned c) { return (c - '0') <= 9u; }
NT_FN unsigned lower(unsigned c) { return (c - 'A') <= 25u ? c + 32u : c; }
NT_FN int hex_val(unsigned c) {
    if (is_dig(c)) return (int)(c - '0');
    const unsigned l = lower(c);
    return (l - 'a') <= 5u ? (int)(l - 'a' + 10) : -1;
}

NT_FN float u2f(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, 4);
    return f;
#endif
}
NT_FN uint32_t f2u(float f) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
#endif
}
NT_FN uint64_t d2u(double d) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(d);
#else
    uint64_t u;
    memcpy(&u, &d, 8);
    return u;
#endif
}
NT_FN int clz64(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return __clzll((long long)x);
#else
    return x ? __builtin_clzll(x) : 64;
#endif
}
NT_FN int clz32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __clz((int)x);
#else
    return x ? __builtin_clz(x) : 32;
#endif
}

// Bytes of one token: positions at or past len read as 0.  With
// Bounded = false the bytes are read as they lie, for a token that a blank
// follows: no rule of the grammar accepts a blank (nor a 0 byte), so the
// result is the same and the per-byte bound check is gone.
template <bool Bounded = true>
struct TokT {
    const unsigned char *s;
    int len;
    NT_FN unsigned at(int i) const { return (!Bounded || i < len) ? s[i] : 0u; }
};

// ---- exact slow path: little-endian 32-bit limbs ---------------------------
// Capacity: the largest operand is a 255-digit significand (848 bits) or a
// 53-bit halfway point times 5^300, shifted by at most 400 bits: < 1300 bits.
struct BigU {
    enum { CAP = 48 };
    uint32_t v[CAP];
    int n;
    NT_FN void set(uint64_t x) {
        v[0] = (uint32_t)x;
        v[1] = (uint32_t)(x >> 32);
        n = v[1] ? 2 : (v[0] ? 1 : 0);
    }
    NT_FN void mul_small(uint32_t m) {
        uint64_t carry = 0;
        for (int i = 0; i < n; ++i) {
            const uint64_t t = (uint64_t)v[i] * m + carry;
            v[i] = (uint32_t)t;
            carry = t >> 32;
        }
        if (carry && n < CAP) v[n++] = (uint32_t)carry;
    }
    NT_FN void add_small(uint32_t a) {
        uint64_t carry = a;
        for (int i = 0; i < n && carry; ++i) {
            const uint64_t t = (uint64_t)v[i] + carry;
            v[i] = (uint32_t)t;
            carry = t >> 32;
        }
        if (carry && n < CAP) v[n++] = (uint32_t)carry;
    }
    NT_FN void mul_pow5(int k) {
        while (k >= 13) {
            mul_small(1220703125u);  // 5^13
            k -= 13;
        }
        uint32_t p = 1;
        while (k-- > 0) p *= 5u;
        if (p != 1) mul_small(p);
    }
    NT_FN void shl(int s) {
        if (n == 0 || s <= 0) return;
        const int limbs = s >> 5, bits = s & 31;
        int nn = n + limbs + 1;
        if (nn > CAP) nn = CAP;
        for (int i = nn - 1; i >= 0; --i) {
            const int src = i - limbs;
            uint32_t hi = (src >= 0 && src < n) ? v[src] : 0u;
            uint32_t lo = (src - 1 >= 0 && src - 1 < n) ? v[src - 1] : 0u;
            v[i] = bits ? (hi << bits) | (lo >> (32 - bits)) : hi;
        }
        n = nn;
        while (n > 0 && v[n - 1] == 0) --n;
    }
};

NT_FN int big_cmp(const BigU &a, const BigU &b) {
    if (a.n != b.n) return a.n < b.n ? -1 : 1;
    for (int i = a.n - 1; i >= 0; --i)
        if (a.v[i] != b.v[i]) return a.v[i] < b.v[i] ? -1 : 1;
    return 0;
}

// Sign of (D * 10^q - mid), D = the significant digits in [sig, end) (a '.'
// among them is skipped), mid a positive normal double.  Kept out of line:
// it holds two big integers and runs only for rare tokens.
template <bool B>
NT_SLOW int cmp_decimal_mid(const TokT<B> &t, int sig, int end, int q, double mid) {
    BigU L, R;
    L.n = 0;
    uint32_t acc = 0, scale = 1;
    for (int i = sig; i < end; ++i) {
        const unsigned c = t.at(i);
        if (!is_dig(c)) continue;
        acc = acc * 10u + (c - '0');
        scale *= 10u;
        if (scale == 1000000000u) {
            if (L.n == 0) L.set(acc);
            else {
                L.mul_small(scale);
                L.add_small(acc);
            }
            acc = 0;
            scale = 1;
        }
    }
    if (scale != 1) {
        if (L.n == 0) L.set(acc);
        else {
            L.mul_small(scale);
            L.add_small(acc);
        }
    }
    const uint64_t mb = d2u(mid);
    const int ex = (int)((mb >> 52) & 0x7ff);
    R.set((mb & ((1ull << 52) - 1)) | (1ull << 52));
    const int he = ex - 1075;
    // D * 2^q * 5^q  vs  R * 2^he
    if (q >= 0) L.mul_pow5(q);
    else R.mul_pow5(-q);
    const int d = q - he;
    if (d >= 0) L.shl(d);
    else R.shl(-d);
    return big_cmp(L, R);
}

// ---- binary rounding (hex significands) -------------------------------------
// m * 2^e2 (+ something below when sticky) to binary32 bits, nearest-even,
// with glibc's subnormal behaviour for hex input.
NT_FN uint32_t round_binary(uint64_t m, bool sticky, int e2) {
    if (m == 0) return 0;
    const int nb = 64 - clz64(m);
    const int E = e2 + nb - 1;
    if (E > 127) return 0x7f800000u;
    const int keep = E >= -126 ? 24 : 24 - (-126 - E);
    if (keep < 0) return 0;
    const int sh = nb - keep;
    uint64_t mant;
    if (sh <= 0) {
        mant = m << (-sh);
    } else {
        mant = sh >= 64 ? 0 : (m >> sh);
        uint64_t rem = sh >= 64 ? m : (m & ((1ull << sh) - 1));
        const uint64_t half = 1ull << (sh - 1);
        if (keep < 24) {
            const int p24 = nb - 25;
            if (p24 >= 0 && p24 < sh - 1) rem &= ~(1ull << p24);
        }
        if (rem > half || (rem == half && (sticky || (mant & 1)))) ++mant;
    }
    uint64_t bits = keep == 24 ? ((uint64_t)(E + 126) << 23) + mant : mant;
    if (bits >= 0x7f800000ull) bits = 0x7f800000ull;
    return (uint32_t)bits;
}

template <bool B>
NT_FN bool scan_hex(const TokT<B> &t, int i, uint32_t sign, float &out) {
    unsigned c = t.at(i);
    if (!(hex_val(c) >= 0 || c == '.')) return false;
    uint64_t m = 0;
    int e2 = 0;
    bool sticky = false;
    int d;
    while ((d = hex_val(t.at(i))) >= 0) {
        if ((m >> 60) == 0) m = m * 16 + (uint64_t)d;
        else {
            e2 += 4;
            sticky |= d != 0;
        }
        ++i;
    }
    if (t.at(i) == '.') {
        ++i;
        while ((d = hex_val(t.at(i))) >= 0) {
            if ((m >> 60) == 0) {
                m = m * 16 + (uint64_t)d;
                e2 -= 4;
            } else {
                sticky |= d != 0;
            }
            ++i;
        }
    }
    if (lower(t.at(i)) == 'p') {
        int j = i + 1;
        bool neg = false;
        if (t.at(j) == '+' || t.at(j) == '-') {
            neg = t.at(j) == '-';
            ++j;
        }
        if (is_dig(t.at(j))) {
            long long ev = 0;
            while (is_dig(t.at(j))) {
                if (ev < 100000000) ev = ev * 10 + (t.at(j) - '0');
                ++j;
            }
            e2 += (int)(neg ? -ev : ev);
        }
    }
    out = u2f(sign | round_binary(m, sticky, e2));
    return true;
}

// 10^k for 0 <= k <= 22, exact (every partial product is a power of ten
// that a double holds exactly).
NT_FN double exact_pow10(int k) {
    double r = 1.0, b = 10.0;
    while (k) {
        if (k & 1) r *= b;
        b *= b;
        k >>= 1;
    }
    return r;
}

template <bool B>
NT_FN bool scan_dec(const TokT<B> &t, int i, uint32_t sign, float &out) {
    int ndig = 0, nfrac = 0, nsig = 0, nw = 0, sig = -1;
    uint64_t w = 0;
    bool trunc = false;
    unsigned c;
    bool frac = false;
    for (;;) {
        c = t.at(i);
        if (is_dig(c)) {
            ++ndig;
            if (frac) ++nfrac;
            const unsigned dv = c - '0';
            if (nsig > 0 || dv != 0) {
                if (nsig == 0) sig = i;
                ++nsig;
                if (nw < 19) {
                    w = w * 10 + dv;
                    ++nw;
                } else if (dv) {
                    trunc = true;
                }
            }
            ++i;
        } else if (c == '.' && !frac) {
            frac = true;
            ++i;
        } else {
            break;
        }
    }
    if (ndig == 0) return false;
    const int mant_end = i;
    long long ev = 0;
    if (lower(t.at(i)) == 'e') {
        int j = i + 1;
        bool neg = false;
        if (t.at(j) == '+' || t.at(j) == '-') {
            neg = t.at(j) == '-';
            ++j;
        }
        if (is_dig(t.at(j))) {
            while (is_dig(t.at(j))) {
                if (ev < 100000000) ev = ev * 10 + (t.at(j) - '0');
                ++j;
            }
            if (neg) ev = -ev;
        }
    }
    if (nsig == 0) {
        out = u2f(sign);
        return true;
    }
    const int q_full = (int)ev - nfrac;  // value = D * 10^q_full
    const int mag = nsig + q_full;       // value in [10^(mag-1), 10^mag)
    if (mag > 39) {
        out = u2f(sign | 0x7f800000u);
        return true;
    }
    if (mag < -45) {
        out = u2f(sign);
        return true;
    }
    const int q = q_full + (nsig - nw);  // value ~ w * 10^q
    if (!trunc && w < (1ull << 53) && q >= -22 && q <= 22) {
        const double p = exact_pow10(q >= 0 ? q : -q);
        const double dv = q >= 0 ? (double)w * p : (double)w / p;
        const float f = (float)dv;
        const double fd = (double)f;
        if (fd == dv) {
            out = u2f(sign | f2u(f));
            return true;
        }
        const uint32_t fb = f2u(f);
        const double gd = (double)u2f(dv > fd ? fb + 1 : fb - 1);
        if (dv * 2.0 != fd + gd) {
            out = u2f(sign | fb);
            return true;
        }
    }
    // slow path: a candidate from double arithmetic, then exact comparisons
    // with the halfway points on either side
    double dv = (double)w;
    {
        int k = q < 0 ? -q : q;
        double p = 1.0, b = 10.0;
        while (k) {
            if (k & 1) p *= b;
            b *= b;
            k >>= 1;
        }
        dv = q < 0 ? dv / p : dv * p;
    }
    const double flt_max = (double)u2f(0x7f7fffffu);
    const double two128 = 18446744073709551616.0 * 18446744073709551616.0;
    uint32_t u = dv < flt_max ? f2u((float)dv) : 0x7f7fffffu;
    for (int it = 0; it < 64; ++it) {
        const double fd = (double)u2f(u);
        const double up = u == 0x7f7fffffu ? two128 : (double)u2f(u + 1);
        const int c_up = cmp_decimal_mid(t, sig, mant_end, q_full, (fd + up) * 0.5);
        if (c_up > 0) {
            ++u;
            if (u >= 0x7f800000u) break;
            continue;
        }
        if (c_up == 0) {
            if (u & 1) ++u;
            break;
        }
        if (u == 0) break;
        const double dn = (double)u2f(u - 1);
        const int c_dn = cmp_decimal_mid(t, sig, mant_end, q_full, (dn + fd) * 0.5);
        if (c_dn < 0) {
            --u;
            continue;
        }
        if (c_dn == 0 && (u & 1)) --u;
        break;
    }
    if (u > 0x7f800000u) u = 0x7f800000u;
    out = u2f(sign | u);
    return true;
}

// sscanf(token, "%f", &out) == 1
template <bool Bounded = true>
NT_FN bool scan_f32(const unsigned char *s, int len, float &out) {
    const TokT<Bounded> t{s, len};
    int i = 0;
    uint32_t sign = 0;
    unsigned c = t.at(0);
    if (c == '+' || c == '-') {
        sign = c == '-' ? 0x80000000u : 0u;
        c = t.at(++i);
    }
    const unsigned lc = lower(c);
    if (lc == 'i') {
        if (lower(t.at(i + 1)) != 'n' || lower(t.at(i + 2)) != 'f') return false;
        if (lower(t.at(i + 3)) == 'i' &&
            (lower(t.at(i + 4)) != 'n' || lower(t.at(i + 5)) != 'i' || lower(t.at(i + 6)) != 't' ||
             lower(t.at(i + 7)) != 'y'))
            return false;
        out = u2f(sign | 0x7f800000u);
        return true;
    }
    if (lc == 'n') {
        if (lower(t.at(i + 1)) != 'a' || lower(t.at(i + 2)) != 'n') return false;
        out = u2f(sign | 0x7fc00000u);
        return true;
    }
    if (c == '0' && lower(t.at(i + 1)) == 'x') return scan_hex(t, i + 2, sign, out);
    return scan_dec(t, i, sign, out);
}

// sscanf(token, "%d", &out) == 1
template <bool Bounded = true>
NT_FN bool scan_int(const unsigned char *s, int len, int &out) {
    const TokT<Bounded> t{s, len};
    int i = 0;
    bool neg = false;
    unsigned c = t.at(0);
    if (c == '+' || c == '-') {
        neg = c == '-';
        ++i;
    }
    if (!is_dig(t.at(i))) return false;
    uint64_t mag = 0;
    bool ovf = false;
    while (is_dig(c = t.at(i))) {
        if (!ovf) {
            const uint64_t d = c - '0';
            if (mag > (0xffffffffffffffffull - d) / 10) ovf = true;
            else mag = mag * 10 + d;
        }
        ++i;
    }
    int64_t v;
    if (!neg) v = (ovf || mag > 0x7fffffffffffffffull) ? (int64_t)0x7fffffffffffffffll : (int64_t)mag;
    else v = (ovf || mag > 0x8000000000000000ull) ? (int64_t)(-0x7fffffffffffffffll - 1) : (int64_t)(0 - mag);
    out = (int)(uint32_t)(uint64_t)v;
    return true;
}

// ---- formatting -------------------------------------------------------------

// 5^k for 0 <= k <= 27
NT_FN uint64_t pow5_u64_small(int k) {
    uint64_t r = 1, b = 5;
    while (k) {
        if (k & 1) r *= b;
        b *= b;
        k >>= 1;
    }
    return r;
}

// 5^k for 0 <= k <= 55 (< 2^128)
NT_FN u128 pow5_u128(int k) {
    u128 r = pow5_u64_small(k < 27 ? k : 27);
    if (k > 27) r *= (u128)pow5_u64_small(k - 27);
    return r;
}

// snprintf("%E", (double)x) without the terminating zero; returns the length
// (at most 13).
NT_FN int format_E(float x, char *o) {
    const uint32_t b = f2u(x);
    int n = 0;
    if (b >> 31) o[n++] = '-';
    const uint32_t a = b & 0x7fffffffu;
    if (a >= 0x7f800000u) {
        const char *w = a > 0x7f800000u ? "NAN" : "INF";
        o[n++] = w[0];
        o[n++] = w[1];
        o[n++] = w[2];
        return n;
    }
    uint32_t digits = 0;
    int E = 0;
    if (a != 0) {
        const int ef = (int)(a >> 23);
        const uint32_t M = ef ? ((a & 0x7fffffu) | 0x800000u) : a;
        const int e = ef ? ef - 150 : -149;
        const int bexp = e + (32 - clz32(M)) - 1;  // x in [2^bexp, 2^(bexp+1))
        E = ((bexp + 1) * 78913) >> 18;             // floor((bexp+1) log10 2): E10 or E10 + 1
        // Fast path: y = |x| * 10^(6-E) with an exact power of ten, one
        // rounding (error < 2^-30 for y < 2^24); its integer part and the
        // side of .5 are those of the exact product unless y lies within
        // 2^-26 of a half, where the exact path below decides.  Exponents
        // near a power of ten resolve to the same digits either way (a
        // rounded 10^6 or 10^7 carries as the exact value would).
        bool done = false;
        {
            const double xa = (double)u2f(a);
            int Ef = E;
            for (int it = 0; it < 3; ++it) {
                const int k = 6 - Ef;
                if (k < -22 || k > 22) break;
                const double y = k >= 0 ? xa * exact_pow10(k) : xa / exact_pow10(-k);
                if (y < 1e6) {
                    --Ef;
                    continue;
                }
                if (y >= 1e7) {
                    ++Ef;
                    continue;
                }
                const uint32_t fl = (uint32_t)y;
                const double fr = y - (double)fl;
                const double dh = fr - 0.5;
                if (dh < 1.0 / 67108864.0 && dh > -1.0 / 67108864.0) break;
                digits = fl + (fr > 0.5 ? 1u : 0u);
                E = Ef;
                done = true;
                break;
            }
        }
        // exact path: floor(|x| / 10^(E-6)) and the rounding bit in 128-bit
        // integers (|x| = M * 2^e; every intermediate < 2^128 for E = E10
        // or E10 + 1)
        for (int it = 0; it < 4 && !done; ++it) {
            const int k = E - 6;
            u128 qq;
            bool up;
            if (k >= 0) {
                const int tt = e - k;
                u128 N, D;
                if (tt >= 0) {
                    N = (u128)M << tt;
                    D = pow5_u128(k);
                } else {
                    N = M;
                    D = pow5_u128(k) << (-tt);
                }
                qq = N / D;
                const u128 r2 = (N - qq * D) << 1;
                up = r2 > D || (r2 == D && (qq & 1));
            } else {
                const int p = -k;
                const u128 X = (u128)M * pow5_u128(p);
                const int s = e + p;
                if (s >= 0) {
                    qq = X << s;
                    up = false;
                } else {
                    const int rs = -s;
                    qq = X >> rs;
                    const u128 rem = X & (((u128)1 << rs) - 1);
                    const u128 half = (u128)1 << (rs - 1);
                    up = rem > half || (rem == half && (qq & 1));
                }
            }
            if (qq < 1000000u) {
                --E;
                continue;
            }
            if (qq >= 10000000u) {
                ++E;
                continue;
            }
            digits = (uint32_t)qq + (up ? 1u : 0u);
            break;
        }
        if (digits == 10000000u) {
            digits = 1000000u;
            ++E;
        }
    }
    char d[7];
    for (int i = 6; i >= 0; --i) {
        d[i] = (char)('0' + digits % 10u);
        digits /= 10u;
    }
    o[n++] = d[0];
    o[n++] = '.';
    for (int i = 1; i < 7; ++i) o[n++] = d[i];
    o[n++] = 'E';
    o[n++] = E < 0 ? '-' : '+';
    const int ae = E < 0 ? -E : E;
    o[n++] = (char)('0' + ae / 10);
    o[n++] = (char)('0' + ae % 10);
    return n;
}

// snprintf("%d", v); returns the length (at most 11)
NT_FN int format_d(int v, char *o) {
    int n = 0;
    uint32_t u = (uint32_t)v;
    if (v < 0) {
        o[n++] = '-';
        u = 0u - u;
    }
    char tmp[10];
    int k = 0;
    do {
        tmp[k++] = (char)('0' + u % 10u);
        u /= 10u;
    } while (u);
    while (k) o[n++] = tmp[--k];
    return n;
}

}  // namespace numtext
}  // namespace hpgl_b200
