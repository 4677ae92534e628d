// Number parsing shared by the device text converters (text.cu) and their host-side
// check. Every function is __host__ __device__ so that the same code runs in a
// kernel and in a plain host test.
//
// The grammar is what std::istream's operator>> accepts for the types the reference's
// converters read (converters/simple.cpp:61-160, matrix-market.cpp:65-241,
// snap.cpp:65-196): leading blanks are skipped, then an optional sign and digits for
// an integer; an optional sign, digits with an optional decimal point and an
// optional exponent for a double. Decimal-to-double conversion must round correctly
// (as strtod does): the device takes the exact fast path of Clinger ("How to read
// floating point numbers accurately", PLDI 1990) -- at most 19 significant digits
// forming an integer m <= 2^53 and a power of ten 10^k with |k| <= 22, both exact in
// binary64, so one correctly rounded multiplication or division gives the correctly
// rounded value -- and reports every other token for a conversion on the host.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define VG_HD __host__ __device__ __forceinline__
#else
#define VG_HD inline
#endif

namespace vgtext {

VG_HD bool is_blank(unsigned char c) {
    return c == ' ' || c == '\t' || c == '\r' || c == '\v' || c == '\f';
}
VG_HD bool is_space(unsigned char c) { return is_blank(c) || c == '\n'; }
VG_HD bool is_digit(unsigned char c) { return c >= '0' && c <= '9'; }

// exact powers of ten representable in binary64 (10^0 .. 10^22)
VG_HD double pow10_exact(int k) {
    double p = 1.0;
    for (int i = 0; i < k; i++) p *= 10.0; // every partial product is exact for k <= 22
    return p;
}

// skips blanks from s[i] (stops at a newline or at end)
VG_HD int64_t skip_blanks(const char *s, int64_t i, int64_t end) {
    while (i < end && is_blank((unsigned char)s[i])) i++;
    return i;
}

// operator>>(long long&): returns 1 and advances *pos on success; 0 when there is no
// number (nothing consumed); -1 on overflow
VG_HD int parse_i64(const char *s, int64_t *pos, int64_t end, int64_t *out, bool cross_lines) {
    int64_t i = *pos;
    while (i < end && (cross_lines ? is_space((unsigned char)s[i]) : is_blank((unsigned char)s[i])))
        i++;
    bool neg = false;
    if (i < end && (s[i] == '+' || s[i] == '-')) {
        neg = s[i] == '-';
        i++;
    }
    if (i >= end || !is_digit((unsigned char)s[i])) return 0;
    uint64_t v = 0;
    bool over = false;
    while (i < end && is_digit((unsigned char)s[i])) {
        const uint64_t d = (uint64_t)(s[i] - '0');
        if (v > (UINT64_MAX - d) / 10) over = true;
        else v = v * 10 + d;
        i++;
    }
    if (over || v > (neg ? (uint64_t)INT64_MAX + 1 : (uint64_t)INT64_MAX)) return -1;
    *out = neg ? (int64_t)(0 - v) : (int64_t)v;
    *pos = i;
    return 1;
}

enum { F_NONE = 0, F_OK = 1, F_HOST = 2 };

// operator>>(double&) on the exact fast path: F_OK with *out set, F_NONE when no
// number starts here (nothing consumed; the stream's value would be 0.0), F_HOST
// when the token is a number that needs the host's conversion (*pos advanced past
// it, *tok_start set to where it starts)
VG_HD int parse_f64(const char *s, int64_t *pos, int64_t end, double *out, int64_t *tok_start) {
    int64_t i = skip_blanks(s, *pos, end);
    const int64_t start = i;
    bool neg = false;
    if (i < end && (s[i] == '+' || s[i] == '-')) {
        neg = s[i] == '-';
        i++;
    }
    uint64_t m = 0;
    int nd = 0;        // significant digits kept in m
    bool lost = false; // a nonzero digit did not fit
    int exp10 = 0;
    bool any = false;
    while (i < end && is_digit((unsigned char)s[i])) {
        any = true;
        const int d = s[i] - '0';
        if (nd < 19) {
            if (m || d) {
                m = m * 10 + (uint64_t)d;
                nd++;
            }
        } else {
            exp10++;
            if (d) lost = true;
        }
        i++;
    }
    if (i < end && s[i] == '.') {
        i++;
        while (i < end && is_digit((unsigned char)s[i])) {
            any = true;
            const int d = s[i] - '0';
            if (nd < 19) {
                if (m || d) {
                    m = m * 10 + (uint64_t)d;
                    nd++;
                }
                exp10--;
            } else if (d) {
                lost = true;
            }
            i++;
        }
    }
    if (!any) return F_NONE;
    if (i < end && (s[i] == 'e' || s[i] == 'E')) {
        int64_t j = i + 1;
        bool eneg = false;
        if (j < end && (s[j] == '+' || s[j] == '-')) {
            eneg = s[j] == '-';
            j++;
        }
        if (j < end && is_digit((unsigned char)s[j])) {
            int e = 0;
            while (j < end && is_digit((unsigned char)s[j])) {
                if (e < 100000) e = e * 10 + (s[j] - '0');
                j++;
            }
            exp10 += eneg ? -e : e;
            i = j;
        }
    }
    *pos = i;
    *tok_start = start;
    if (m == 0 && !lost) {
        *out = neg ? -0.0 : 0.0;
        return F_OK;
    }
    if (lost || m > (1ULL << 53) || exp10 > 22 || exp10 < -22) return F_HOST;
    double v = (double)m; // exact: m <= 2^53
#if defined(__CUDA_ARCH__)
    v = exp10 >= 0 ? __dmul_rn(v, pow10_exact(exp10)) : __ddiv_rn(v, pow10_exact(-exp10));
#else
    v = exp10 >= 0 ? v * pow10_exact(exp10) : v / pow10_exact(-exp10);
#endif
    *out = neg ? -v : v;
    return F_OK;
}

} // namespace vgtext
