// story_num.h -- number fields of Starlab story text, converted exactly as
// the C library converts them when the reference reads a snapshot:
//   * reals with strtod (m: node_io.C:88 / dyn_io.C:196; r and v:
//     set_vector_from_string, util_io.C:145-157; system_time: dyn_io.C:192),
//   * the particle index with strtol(val, NULL, 10) (tree_io.C:330).
// Host and device: the same code runs in the story kernels and, compiled by
// the host compiler, in the CPU tests that compare it with the C library.
//
// Decimal to double.  The digits give w (up to 40 significant digits) and
// a decimal exponent q, value V = w * 10^q.  Then:
//   1. w < 2^53 and |q| <= 22: one IEEE multiply or divide of two exact
//      doubles, which rounds V correctly (Clinger 1990, "How to read
//      floating point numbers accurately", the fast path);
//   2. otherwise a candidate c within a few units in the last place is
//      refined as in Clinger's AlgorithmR: V is compared EXACTLY, in integer
//      arithmetic, with the midpoints between c and its two neighbours, and
//      c steps one unit up or down until V lies between them (ties to even).
//      The comparison of w * 5^q * 2^q with K * 2^k needs no division: the
//      side with the negative exponent is moved across.  Three 64-bit words
//      (registers) cover |q| <= 27 with up to 19 digits (every number the
//      reference writes at its default 18 digits); larger exponents or more
//      digits use 20 words.
// Before step 2, up to 19 digits (w < 2^64) go through the Eisel-Lemire
// conversion: w normalised times a 128-bit approximation of 5^q
// (pow5_table.h), whose leading bits are the rounded significand -- exact
// for every w < 2^64 and every q of the table (Lemire 2021, "Number parsing
// at a gigabyte per second"; Mushtak and Lemire 2023, "Fast number parsing
// without fallback"), with the exact ties-to-even test for the q where a
// decimal can lie halfway between two doubles (-4 <= q <= 23).  Step 2
// then only sees more than 19 digits.
// Forms the reference never writes -- hexadecimal floats, NaN payloads
// "nan(...)", more than 40 significant digits -- are reported, not guessed.
#pragma once
#include <stdint.h>
#include "pow5_table.h"

#if defined(__CUDACC__)
#define SN_HD __host__ __device__ __forceinline__
#else
#define SN_HD inline
#endif

namespace story {

SN_HD uint64_t mul_hi64(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

SN_HD uint64_t dbits(double x) {
#if defined(__CUDA_ARCH__)
    return (uint64_t)__double_as_longlong(x);
#else
    uint64_t u;
    __builtin_memcpy(&u, &x, 8);
    return u;
#endif
}

SN_HD double from_bits(uint64_t u) {
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    double x;
    __builtin_memcpy(&x, &u, 8);
    return x;
#endif
}

// Unsigned integer of up to NL 64-bit words (least significant first).
template <int NL>
struct Big {
    uint64_t w[NL];
    int n;     // words in use (no leading zero word)
    bool ovf;  // a result did not fit

    SN_HD void set(uint64_t x) {
        for (int i = 0; i < NL; ++i) w[i] = 0;
        w[0] = x;
        n = x ? 1 : 0;
        ovf = false;
    }
    SN_HD void mul_add(uint64_t m, uint64_t a) {  // this = this * m + a
        uint64_t carry = a;
        for (int i = 0; i < n; ++i) {
            uint64_t lo = w[i] * m;
            uint64_t hi = mul_hi64(w[i], m);
            lo += carry;
            hi += lo < carry;
            w[i] = lo;
            carry = hi;
        }
        if (carry) {
            if (n < NL)
                w[n++] = carry;
            else
                ovf = true;
        }
    }
    SN_HD void shl(int s) {
        if (n == 0 || s == 0) return;
        const int words = s >> 6, bits = s & 63;
        const uint64_t top = bits ? (w[n - 1] >> (64 - bits)) : 0;
        const int nn = n + words + (top ? 1 : 0);
        if (nn > NL) {
            ovf = true;
            return;
        }
        for (int i = nn - 1; i >= 0; --i) {
            const int j = i - words;
            const uint64_t hi = (j >= 0 && j < n) ? w[j] : 0;
            const uint64_t lo = (j - 1 >= 0 && j - 1 < n) ? w[j - 1] : 0;
            w[i] = bits ? (hi << bits) | (lo >> (64 - bits)) : hi;
        }
        n = nn;
    }
    SN_HD void mul_pow5(int e) {  // this *= 5^e, e >= 0
        const uint64_t p27 = 7450580596923828125ull;  // 5^27, the largest power of 5 below 2^63
        while (e >= 27) {
            mul_add(p27, 0);
            e -= 27;
        }
        uint64_t p = 1;
        while (e-- > 0) p *= 5;
        if (p > 1) mul_add(p, 0);
    }
};

template <int NL>
SN_HD int big_cmp(const Big<NL> &a, const Big<NL> &b) {
    if (a.n != b.n) return a.n < b.n ? -1 : 1;
    for (int i = a.n - 1; i >= 0; --i)
        if (a.w[i] != b.w[i]) return a.w[i] < b.w[i] ? -1 : 1;
    return 0;
}

SN_HD double pow10_exact(int k) {  // 10^k for 0 <= k <= 22, exact
    double r = 1.0;
    if (k & 1) r *= 10.0;
    if (k & 2) r *= 100.0;
    if (k & 4) r *= 1e4;
    if (k & 8) r *= 1e8;
    if (k & 16) r *= 1e16;
    return r;
}

#if defined(__CUDACC__)
__device__ static const uint64_t kPow5Dev[] = SN_POW5_TABLE;
#endif
static const uint64_t kPow5Host[] = SN_POW5_TABLE;

SN_HD uint64_t pow5_word(int k) {
#if defined(__CUDA_ARCH__)
    return __ldg(&kPow5Dev[k]);
#else
    return kPow5Host[k];
#endif
}

SN_HD int clz64(uint64_t x) {
#if defined(__CUDA_ARCH__)
    return __clzll((long long)x);
#else
    return __builtin_clzll(x);
#endif
}

// Eisel-Lemire: the bits of the double nearest w * 10^q (w < 2^64, w > 0,
// SN_POW5_MIN_Q <= q <= SN_POW5_MAX_Q), sign not included.
SN_HD uint64_t eisel_lemire(uint64_t w, int q) {
    const int lz = clz64(w);
    w <<= lz;
    const int idx = 2 * (q - SN_POW5_MIN_Q);
    // 128-bit product of w with the table's high word; the low word only
    // when the product's bits below the 55 kept ones are all ones
    uint64_t lo = w * pow5_word(idx), hi = mul_hi64(w, pow5_word(idx));
    if ((hi & 0x1ffu) == 0x1ffu) {
        const uint64_t lo2 = mul_hi64(w, pow5_word(idx + 1));
        lo += lo2;
        hi += lo < lo2;
    }
    const int upper = (int)(hi >> 63);
    const int shift = upper + 9;
    uint64_t m = hi >> shift;
    // binary exponent: floor(q log2 10) + 63, + the product's top bit, - lz, + the bias 1023
    int p2 = (((152170 + 65536) * q) >> 16) + 63 + upper - lz + 1023;
    if (p2 <= 0) {  // subnormal
        if (-p2 + 1 >= 64) return 0;
        m >>= -p2 + 1;
        m += m & 1;
        m >>= 1;
        return m;  // 2^52 when it rounded up to the smallest normal: the same bits
    }
    if (lo <= 1 && q >= -4 && q <= 23 && (m & 3) == 1 && (m << shift) == hi) m &= ~(uint64_t)1;  // exact tie: to even
    m += m & 1;
    m >>= 1;
    if (m >= (2ull << 52)) {
        m = 1ull << 52;
        ++p2;
    }
    m &= ~(1ull << 52);
    if (p2 >= 0x7ff) return 0x7ff0000000000000ull;
    return m | ((uint64_t)p2 << 52);
}

SN_HD bool is_space(char c) { return c == ' ' || (c >= '\t' && c <= '\r'); }
SN_HD bool is_digit(char c) { return c >= '0' && c <= '9'; }
SN_HD char lower(char c) { return (c >= 'A' && c <= 'Z') ? (char)(c + 32) : c; }
SN_HD bool is_hex(char c) { return is_digit(c) || (lower(c) >= 'a' && lower(c) <= 'f'); }

SN_HD bool match_ci(const char *s, const char *e, const char *lit) {
    for (; *lit; ++lit, ++s)
        if (s >= e || lower(*s) != *lit) return false;
    return true;
}

// V = w * 10^q compared with K * 2^k: -1, 0, 1.  A0 = w * 5^q when q >= 0,
// P = 5^-q when q < 0 (computed once per number by the caller).
template <int NL>
SN_HD int cmp_mid(const Big<NL> &w, const Big<NL> &A0, const Big<NL> &P, int q, uint64_t K, int k, bool &ovf) {
    Big<NL> A, B;
    int a, b;
    if (q >= 0) {
        A = A0;
        a = q;
        B.set(K);
        b = k;
    } else {
        A = w;
        a = 0;
        B = P;
        B.mul_add(K, 0);
        b = k - q;
    }
    const int s = a < b ? a : b;
    A.shl(a - s);
    B.shl(b - s);
    if (A.ovf || B.ovf) {
        ovf = true;
        return 0;
    }
    return big_cmp(A, B);
}

// Steps the candidate c (> 0, finite) to the double nearest V.  Returns
// false if an integer did not fit or it did not settle.
template <int NL>
SN_HD bool refine(const Big<NL> &w, int q, double &c) {
    Big<NL> A0, P;
    if (q >= 0) {
        A0 = w;
        A0.mul_pow5(q);
        P.set(1);
    } else {
        P.set(1);
        P.mul_pow5(-q);
        A0.set(0);
    }
    if (A0.ovf || P.ovf) return false;
    for (int it = 0; it < 96; ++it) {
        const uint64_t bits = dbits(c);
        const int ex = (int)(bits >> 52);
        uint64_t M = bits & ((1ull << 52) - 1);
        int E;
        if (ex == 0) {
            E = -1074;
        } else {
            M |= 1ull << 52;
            E = ex - 1075;
        }
        bool ovf = false;
        const int up = cmp_mid(w, A0, P, q, 2 * M + 1, E - 1, ovf);
        if (ovf) return false;
        if (up > 0 || (up == 0 && (M & 1))) {
            c = from_bits(bits + 1);  // DBL_MAX + 1 unit is +inf
            if (bits + 1 == 0x7ff0000000000000ull) return true;
            continue;
        }
        uint64_t Kd;
        int kd;
        if (M == (1ull << 52) && E > -1074) {  // c a power of two: the lower neighbour is half a unit away
            Kd = 4 * M - 1;
            kd = E - 2;
        } else {
            Kd = 2 * M - 1;
            kd = E - 1;
        }
        const int dn = cmp_mid(w, A0, P, q, Kd, kd, ovf);
        if (ovf) return false;
        if (dn < 0 || (dn == 0 && (M & 1))) {
            c = from_bits(bits - 1);
            if (bits == 1) return true;  // below half the smallest subnormal: zero
            continue;
        }
        return true;
    }
    return false;
}

// The same refinement in three fixed 64-bit words (registers) for w < 2^64
// and |q| <= 27, where every integer of the comparison stays below 2^192.
struct U192 {
    uint64_t a, b, c;  // least significant first
};

SN_HD U192 mul64x64(uint64_t x, uint64_t y) { return U192{x * y, mul_hi64(x, y), 0}; }

SN_HD U192 mul192x64(U192 x, uint64_t y, bool &ovf) {
    U192 r;
    r.a = x.a * y;
    uint64_t h = mul_hi64(x.a, y);
    uint64_t lo = x.b * y, hi = mul_hi64(x.b, y);
    r.b = lo + h;
    hi += r.b < lo;
    lo = x.c * y;
    uint64_t top = mul_hi64(x.c, y);
    r.c = lo + hi;
    top += r.c < lo;
    if (top) ovf = true;
    return r;
}

SN_HD U192 shl192(U192 x, int s, bool &ovf) {
    if (s <= 0) return x;
    if (s >= 192) {
        if (x.a | x.b | x.c) ovf = true;
        return U192{0, 0, 0};
    }
    while (s >= 64) {
        if (x.c) ovf = true;
        x = U192{0, x.a, x.b};
        s -= 64;
    }
    if (s) {
        if (x.c >> (64 - s)) ovf = true;
        x = U192{x.a << s, (x.b << s) | (x.a >> (64 - s)), (x.c << s) | (x.b >> (64 - s))};
    }
    return x;
}

SN_HD int cmp192(U192 x, U192 y) {
    if (x.c != y.c) return x.c < y.c ? -1 : 1;
    if (x.b != y.b) return x.b < y.b ? -1 : 1;
    if (x.a != y.a) return x.a < y.a ? -1 : 1;
    return 0;
}

SN_HD uint64_t pow5_64(int e) {  // 5^e, e <= 27
    uint64_t p = 1;
    for (int i = 0; i < e; ++i) p *= 5;
    return p;
}

SN_HD bool refine192(uint64_t w, int q, double &c) {
    const uint64_t p5 = pow5_64(q >= 0 ? q : -q);
    const U192 A0 = q >= 0 ? mul64x64(w, p5) : U192{w, 0, 0};
    auto cmp = [&](uint64_t K, int k, bool &ovf) -> int {
        U192 A = A0, B;
        int a, b;
        if (q >= 0) {
            a = q;
            B = U192{K, 0, 0};
            b = k;
        } else {
            a = 0;
            B = mul64x64(K, p5);
            b = k - q;
        }
        const int s = a < b ? a : b;
        A = shl192(A, a - s, ovf);
        B = shl192(B, b - s, ovf);
        return cmp192(A, B);
    };
    for (int it = 0; it < 96; ++it) {
        const uint64_t bits = dbits(c);
        const int ex = (int)(bits >> 52);
        uint64_t M = bits & ((1ull << 52) - 1);
        int E;
        if (ex == 0) {
            E = -1074;
        } else {
            M |= 1ull << 52;
            E = ex - 1075;
        }
        bool ovf = false;
        const int up = cmp(2 * M + 1, E - 1, ovf);
        if (ovf) return false;
        if (up > 0 || (up == 0 && (M & 1))) {
            c = from_bits(bits + 1);
            if (bits + 1 == 0x7ff0000000000000ull) return true;
            continue;
        }
        uint64_t Kd;
        int kd;
        if (M == (1ull << 52) && E > -1074) {
            Kd = 4 * M - 1;
            kd = E - 2;
        } else {
            Kd = 2 * M - 1;
            kd = E - 1;
        }
        const int dn = cmp(Kd, kd, ovf);
        if (ovf) return false;
        if (dn < 0 || (dn == 0 && (M & 1))) {
            c = from_bits(bits - 1);
            if (bits == 1) return true;
            continue;
        }
        return true;
    }
    return false;
}

struct Real {
    double v;
    int n;    // characters used (0: no conversion, v = 0)
    int err;  // 1: a form this reader does not convert
};

// strtod over [p, e): the text ends at e as at a terminating NUL.
SN_HD Real parse_real(const char *p, const char *e) {
    Real r{0.0, 0, 0};
    const char *s = p;
    while (s < e && is_space(*s)) ++s;
    bool neg = false;
    if (s < e && (*s == '+' || *s == '-')) {
        neg = *s == '-';
        ++s;
    }
    if (s < e && lower(*s) == 'i') {
        if (!match_ci(s, e, "inf")) return r;
        const char *t = s + 3;
        if (match_ci(t, e, "inity")) t += 5;
        r.v = from_bits(0x7ff0000000000000ull | (neg ? 0x8000000000000000ull : 0));
        r.n = (int)(t - p);
        return r;
    }
    if (s < e && lower(*s) == 'n') {
        if (!match_ci(s, e, "nan")) return r;
        const char *t = s + 3;
        if (t < e && *t == '(') r.err = 1;
        r.v = from_bits(0x7ff8000000000000ull | (neg ? 0x8000000000000000ull : 0));
        r.n = (int)(t - p);
        return r;
    }
    if (s + 1 < e && s[0] == '0' && lower(s[1]) == 'x' &&
        ((s + 2 < e && is_hex(s[2])) || (s + 3 < e && s[2] == '.' && is_hex(s[3])))) {
        r.err = 1;
        return r;
    }
    uint64_t w0 = 0;
    Big<20> wb;  // set when a 20th significant digit appears
    bool big = false, any = false, dropped = false;
    int nd = 0;
    long long q = 0;
    auto digit = [&](int d, bool frac) {
        any = true;
        if (nd == 0 && d == 0) {
            if (frac) --q;
            return;
        }
        if (nd < 19) {
            w0 = w0 * 10 + (uint64_t)d;
            ++nd;
            if (frac) --q;
        } else if (nd < 40) {
            if (!big) {
                wb.set(w0);
                big = true;
            }
            wb.mul_add(10, (uint64_t)d);
            ++nd;
            if (frac) --q;
        } else {
            if (d) dropped = true;
            if (!frac) ++q;
        }
    };
    for (; s < e && is_digit(*s); ++s) digit(*s - '0', false);
    if (s < e && *s == '.') {
        const char *t = s + 1;
        bool fd = false;
        for (; t < e && is_digit(*t); ++t) {
            digit(*t - '0', true);
            fd = true;
        }
        if (any || fd) s = t;
    }
    if (!any) return r;
    if (s < e && lower(*s) == 'e') {
        const char *t = s + 1;
        bool eneg = false;
        if (t < e && (*t == '+' || *t == '-')) {
            eneg = *t == '-';
            ++t;
        }
        if (t < e && is_digit(*t)) {
            long long ev = 0;
            for (; t < e && is_digit(*t); ++t)
                if (ev < 100000000) ev = ev * 10 + (*t - '0');
            q += eneg ? -ev : ev;
            s = t;
        }
    }
    r.n = (int)(s - p);
    if (dropped) {
        r.err = 1;
        return r;
    }
    const uint64_t sign = neg ? 0x8000000000000000ull : 0;
    if (nd == 0 || q + nd < -324) {  // zero, or below 10^-325 < half the smallest subnormal
        r.v = from_bits(sign);
        return r;
    }
    if (q + nd - 1 > 308) {  // at least 10^309
        r.v = from_bits(sign | 0x7ff0000000000000ull);
        return r;
    }
    const int qi = (int)q;
    if (!big && w0 < (1ull << 53) && qi >= -22 && qi <= 22) {
        const double wd = (double)w0;
        r.v = qi >= 0 ? wd * pow10_exact(qi) : wd / pow10_exact(-qi);
        if (neg) r.v = -r.v;
        return r;
    }
    if (!big) {
        // q + nd in [-324, 309] with nd <= 19: q <= 308; below the table
        // (q = -343) w * 10^q < 10^-324, under half the smallest subnormal
        r.v = from_bits((qi < SN_POW5_MIN_Q ? 0 : eisel_lemire(w0, qi)) | sign);
        return r;
    }
    // Candidate: w as a double, scaled by powers of ten in steps of at most
    // 10^22, with a binary pre-scale near the ends of the range so that no
    // step overflows or loses precision to underflow.
    double c = big ? ((double)wb.w[2] * from_bits((uint64_t)(1023 + 128) << 52) + (double)wb.w[1] * 18446744073709551616.0) +
                         (double)wb.w[0]
                   : (double)w0;
    int pre = 0;
    if (q + nd < -290) pre = 600;
    if (q + nd > 290) pre = -600;
    const double two600 = from_bits((uint64_t)(1023 + 600) << 52), two_600 = from_bits((uint64_t)(1023 - 600) << 52);
    if (pre > 0) c *= two600;
    if (pre < 0) c *= two_600;
    for (int qq = qi; qq != 0;) {
        const int k = qq > 22 ? 22 : (qq < -22 ? -22 : qq);
        c = k > 0 ? c * pow10_exact(k) : c / pow10_exact(-k);
        qq -= k;
    }
    if (pre > 0) c *= two_600;
    if (pre < 0) c *= two600;
    if (!(c < 1.7976931348623157e308)) c = 1.7976931348623157e308;
    if (c == 0.0) c = from_bits(1);
    bool ok = false;
    if (!big && qi >= -27 && qi <= 27) {
        double c3 = c;
        ok = refine192(w0, qi, c3);
        if (ok) c = c3;
    }
    if (!ok) {
        if (!big) wb.set(w0);
        ok = refine(wb, qi, c);
    }
    if (!ok) {
        r.err = 1;
        return r;
    }
    r.v = from_bits(dbits(c) | sign);
    return r;
}

struct Long {
    long long v;
    int n;  // characters used (0: no conversion)
};

// strtol(p, NULL, 10) over [p, e) with a 64-bit long: saturates at the
// limits of long on overflow.
SN_HD Long parse_long(const char *p, const char *e) {
    Long r{0, 0};
    const char *s = p;
    while (s < e && is_space(*s)) ++s;
    bool neg = false;
    if (s < e && (*s == '+' || *s == '-')) {
        neg = *s == '-';
        ++s;
    }
    if (!(s < e && is_digit(*s))) return r;
    const uint64_t lim = neg ? 9223372036854775808ull : 9223372036854775807ull;
    uint64_t v = 0;
    bool sat = false;
    for (; s < e && is_digit(*s); ++s) {
        const uint64_t d = (uint64_t)(*s - '0');
        if (sat || v > (lim - d) / 10)
            sat = true;
        else
            v = v * 10 + d;
    }
    if (sat) v = lim;
    r.v = neg ? (long long)(0 - v) : (long long)v;
    r.n = (int)(s - p);
    return r;
}

}  // namespace story
