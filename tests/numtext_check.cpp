// Test-only host build of hpgl_b200/csrc/numtext.cuh (the number <-> text
// conversions that the INC/GSLIB kernels run on the device), with generators
// that compare it against the C library's sscanf("%f"), sscanf("%d") and
// snprintf("%E"), the calls the reference's readers and writers make
// (read_inc_file.cpp:54-122, property_writer.cpp:18-26).  Built and loaded by
// tests/test_numtext.py.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "../hpgl_b200/csrc/numtext.cuh"

using namespace hpgl_b200::numtext;

namespace {

struct Rng {
    uint64_t s;
    uint64_t next() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return s;
    }
    int below(int n) { return (int)(next() % (uint64_t)n); }
};

std::string random_chars(Rng &r) {
    static const char alphabet[] = "0123456789.eE+-xXpPaAbBcCdDfFiInNtTyY()_/,*";
    const int len = 1 + r.below(24);
    std::string s;
    for (int i = 0; i < len; ++i) s += alphabet[r.below((int)sizeof(alphabet) - 1)];
    return s;
}

std::string random_digits(Rng &r, int n) {
    std::string s;
    for (int i = 0; i < n; ++i) s += (char)('0' + r.below(10));
    return s;
}

std::string random_decimal(Rng &r) {
    std::string s;
    const int sg = r.below(4);
    if (sg == 1) s += '-';
    if (sg == 2) s += '+';
    const int nint = r.below(4) == 0 ? r.below(40) : r.below(8);
    const int nfrac = r.below(3) == 0 ? r.below(40) : r.below(10);
    if (r.below(5) == 0) s += std::string(r.below(30), '0');
    s += random_digits(r, nint);
    if (r.below(4)) s += '.';
    s += random_digits(r, nfrac);
    if (r.below(2)) {
        s += r.below(2) ? 'e' : 'E';
        const int es = r.below(3);
        if (es == 1) s += '-';
        if (es == 2) s += '+';
        s += std::to_string(r.below(4) == 0 ? r.below(400) : r.below(60));
    }
    if (s.empty() || s == "-" || s == "+") s += '0';
    return s;
}

float random_float(Rng &r) {
    uint32_t b = (uint32_t)r.next();
    if (r.below(8) == 0) b &= 0x807fffffu;  // subnormals
    return u2f(b);
}

std::string float_text(Rng &r) {
    const float f = random_float(r);
    char buf[128];
    switch (r.below(5)) {
        case 0: snprintf(buf, sizeof buf, "%.*g", 1 + r.below(12), (double)f); break;
        case 1: snprintf(buf, sizeof buf, "%.9e", (double)f); break;
        case 2: snprintf(buf, sizeof buf, "%E", (double)f); break;
        case 3: snprintf(buf, sizeof buf, "%.17g", (double)f); break;
        default: snprintf(buf, sizeof buf, "%.*f", r.below(50), (double)f); break;
    }
    std::string s(buf);
    if (s.size() > 255) s.resize(255);
    return s;
}

// Decimal text of (or near) the halfway point between two adjacent floats.
std::string near_midpoint(Rng &r, bool long_form) {
    uint32_t b = (uint32_t)r.next() & 0x7fffffffu;
    if (r.below(4) == 0) b &= 0x007fffffu;
    if (b >= 0x7f7fffffu) b = 0x7f7ffffeu;
    const double m = ((double)u2f(b) + (double)u2f(b + 1)) * 0.5;
    char buf[512];
    snprintf(buf, sizeof buf, "%.*e", long_form ? 60 + r.below(140) : 8 + r.below(30), m);
    std::string s(buf);
    const size_t epos = s.find('e');
    std::string mant = s.substr(0, epos), ex = s.substr(epos);
    switch (r.below(4)) {
        case 0: break;
        case 1: mant += std::string(r.below(20), '0') + "1"; break;
        case 2: {
            // nudge the last digit
            char &c = mant.back();
            if (c > '0') --c; else c = '1';
            break;
        }
        default: mant += random_digits(r, 1 + r.below(10)); break;
    }
    s = mant + ex;
    if (s.size() > 255) s = mant.substr(0, 255 - ex.size()) + ex;
    return s;
}

std::string random_hex(Rng &r) {
    char buf[96];
    uint64_t m = r.next() & ((r.below(2) ? ~0ull : (1ull << (1 + r.below(63))) - 1));
    if (r.below(3) == 0) {
        const int nb = m ? 64 - __builtin_clzll(m) : 1;
        m = (1ull << (nb - 1)) | (1ull << r.below(nb));
    }
    const int e = -230 + r.below(380);
    switch (r.below(4)) {
        case 0: snprintf(buf, sizeof buf, "0x%llxp%d", (unsigned long long)m, e); break;
        case 1: snprintf(buf, sizeof buf, "0X%llx.%llxP%+d", (unsigned long long)(m >> 40), (unsigned long long)m, e); break;
        case 2: snprintf(buf, sizeof buf, "-0x.%016llx%llxp%d", (unsigned long long)m, (unsigned long long)r.next(), e); break;
        default: snprintf(buf, sizeof buf, "0x%llx%016llxp%d", (unsigned long long)m, (unsigned long long)r.next(), e - 64); break;
    }
    return buf;
}

std::string long_digits(Rng &r) {
    std::string s = random_digits(r, 100 + r.below(150));
    const int point = r.below((int)s.size());
    if (r.below(2)) s.insert(s.begin() + point, '.');
    if (r.below(2)) s = "0." + std::string(r.below(60), '0') + s.substr(0, 200);
    if (r.below(2)) s += "e" + std::to_string(-120 + r.below(160));
    if (s.size() > 255) s.resize(255);
    return s;
}

std::string float_token(Rng &r, int mode) {
    switch (mode) {
        case 0: return random_chars(r);
        case 1: return random_decimal(r);
        case 2: return float_text(r);
        case 3: return near_midpoint(r, false);
        case 4: return near_midpoint(r, true);
        case 5: return random_hex(r);
        default: return long_digits(r);
    }
}

std::string int_token(Rng &r) {
    switch (r.below(4)) {
        case 0: return random_chars(r);
        case 1: return std::to_string((long long)(int32_t)(uint32_t)r.next());
        case 2: {
            std::string s = (r.below(2) ? "-" : (r.below(2) ? "+" : "")) + std::string(r.below(5), '0');
            return s + random_digits(r, 1 + r.below(25));
        }
        default: return std::to_string((long long)r.below(600) - 300) + random_chars(r);
    }
}

void note(char *report, int cap, int &used, const std::string &line) {
    if (!report || used + (int)line.size() + 2 >= cap) return;
    memcpy(report + used, line.c_str(), line.size());
    used += (int)line.size();
    report[used++] = '\n';
    report[used] = 0;
}

}  // namespace

extern "C" {

int nt_scan_f32(const char *s, int len, float *out) { return scan_f32((const unsigned char *)s, len, *out) ? 1 : 0; }
int nt_scan_int(const char *s, int len, int *out) { return scan_int((const unsigned char *)s, len, *out) ? 1 : 0; }
int nt_format_E(float x, char *out) {
    const int n = format_E(x, out);
    out[n] = 0;
    return n;
}

// Tokens of one kind (mode 0..6) through scan_f32 and sscanf("%f"); returns
// the number of disagreements and lists the first ones in report.
long nt_fuzz_f32(unsigned long long seed, long count, int mode, char *report, int cap) {
    Rng r{seed * 2654435761ull + 12345};
    long bad = 0;
    int used = 0;
    if (report && cap) report[0] = 0;
    for (long i = 0; i < count; ++i) {
        const std::string tok = float_token(r, mode);
        float a = -777.f, b = -777.f;
        const int ra = sscanf(tok.c_str(), "%f", &a) == 1 ? 1 : 0;
        const int rb = scan_f32((const unsigned char *)tok.data(), (int)tok.size(), b) ? 1 : 0;
        // the unbounded variant, on the zero-terminated copy
        float c = -777.f;
        const int rc = scan_f32<false>((const unsigned char *)tok.c_str(), 0, c) ? 1 : 0;
        if (ra != rb || (ra && f2u(a) != f2u(b)) || rc != rb || (rc && f2u(c) != f2u(b))) {
            char buf[400];
            snprintf(buf, sizeof buf, "'%s' libc=%d:%08x mine=%d:%08x unbounded=%d:%08x", tok.c_str(), ra, f2u(a), rb,
                     f2u(b), rc, f2u(c));
            if (bad < 10) note(report, cap, used, buf);
            ++bad;
        }
    }
    return bad;
}

long nt_fuzz_int(unsigned long long seed, long count, char *report, int cap) {
    Rng r{seed * 2654435761ull + 777};
    long bad = 0;
    int used = 0;
    if (report && cap) report[0] = 0;
    for (long i = 0; i < count; ++i) {
        const std::string tok = int_token(r);
        int a = -777, b = -777;
        const int ra = sscanf(tok.c_str(), "%d", &a) == 1 ? 1 : 0;
        const int rb = scan_int((const unsigned char *)tok.data(), (int)tok.size(), b) ? 1 : 0;
        int c = -777;
        const int rc = scan_int<false>((const unsigned char *)tok.c_str(), 0, c) ? 1 : 0;
        if (ra != rb || (ra && a != b) || rc != rb || (rc && c != b)) {
            char buf[400];
            snprintf(buf, sizeof buf, "'%s' libc=%d:%d mine=%d:%d", tok.c_str(), ra, a, rb, b);
            if (bad < 10) note(report, cap, used, buf);
            ++bad;
        }
    }
    return bad;
}

// format_E against snprintf("%E") for the bit patterns lo, lo+step, ... < hi
// (step 0: count random patterns from seed lo instead).
long nt_check_format(unsigned long long lo, unsigned long long hi, unsigned long long step, long count,
                     char *report, int cap) {
    long bad = 0;
    int used = 0;
    if (report && cap) report[0] = 0;
    Rng r{lo * 2654435761ull + 99};
    char want[64], got[64];
    unsigned long long b = lo;
    for (long i = 0;; ++i) {
        uint32_t bits;
        if (step) {
            if (b >= hi) break;
            bits = (uint32_t)b;
            b += step;
        } else {
            if (i >= count) break;
            bits = (uint32_t)r.next();
            if ((i & 7) == 0) bits &= 0x807fffffu;
        }
        const float f = u2f(bits);
        snprintf(want, sizeof want, "%E", (double)f);
        const int n = format_E(f, got);
        got[n] = 0;
        if (strcmp(want, got) != 0) {
            char buf[200];
            snprintf(buf, sizeof buf, "%08x libc=%s mine=%s", bits, want, got);
            if (bad < 10) note(report, cap, used, buf);
            ++bad;
        }
    }
    return bad;
}

// format_d against snprintf("%d") for (int)(char)b, b = 0..255, and a few
// int extremes.
long nt_check_format_d(char *report, int cap) {
    long bad = 0;
    int used = 0;
    if (report && cap) report[0] = 0;
    char want[32], got[32];
    const int extra[] = {0, -1, 1, 2147483647, -2147483647 - 1, 1000000000, -99};
    for (int i = 0; i < 256 + 7; ++i) {
        const int v = i < 256 ? (int)(signed char)(unsigned char)i : extra[i - 256];
        snprintf(want, sizeof want, "%d", v);
        const int n = format_d(v, got);
        got[n] = 0;
        if (strcmp(want, got) != 0) {
            if (bad < 10) note(report, cap, used, std::string(want) + " vs " + got);
            ++bad;
        }
    }
    return bad;
}
}
