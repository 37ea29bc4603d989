// parse.cuh -- the MULTICUT text format read on the device
// (src/multicut_text_parser.cpp:6-31 of the reference).
//
// Format: a first line "MULTICUT", then whitespace-separated triples "i j
// cost" until the first token that does not read as a number of its kind
// (the reference's `while (f >> i >> j >> cost)`); a trailing incomplete
// triple is dropped.  Here every token is read in parallel: token starts are
// compacted, each token is converted on its own, and the first failing token
// ends the input.  A token must be a number as a whole (the reference would
// also accept a numeric prefix of a malformed token; no well-formed file has
// one).
//
// Integers: [+-]digits, within int32 (overflow fails, as for operator>>).
// Costs: [+-](digits[.digits] | .digits)[(e|E)[+-]digits], converted to the
// nearest float with ties to even, as strtof; a value beyond FLT_MAX fails
// (operator>> sets failbit), tiny values round to subnormals or zero.
//
// Decimal -> float: with at most 19 significant digits M and x = M * 10^E,
// M <= 2^53 and |E| <= 22, one IEEE double multiplication or division gives
// r = RN_double(x) (both operands exact: Clinger's fast path).  Rounding r to
// float is exact unless r lies on a float midpoint.  In that case, and when
// the fast path does not apply, an approximation r within a few double ulps
// picks the candidate float and its neighbouring midpoints are compared with
// x exactly, with big integers: Mb * 5^max(E,0) * 2^(E-s) against
// m * 5^max(-E,0) * 2^(q-s) for a midpoint m * 2^q and s = min(E, q), where
// Mb holds the first 120 significant digits (every float midpoint has fewer)
// and a sticky flag records non-zero digits beyond them.
#pragma once
#include "prims.cuh"

namespace rama {

__device__ __forceinline__ bool is_space_char(char c)
{
    return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

// ---------------------------------------------------------------------------
// small unsigned big integers (little-endian 32-bit limbs)
// ---------------------------------------------------------------------------
constexpr int BIG_LIMBS = 28;  // 896 bits: 19-digit M times 5^64 times 2^(<=600)

struct Big {
    uint32_t w[BIG_LIMBS];
    int n;  // limbs in use
    bool overflow;
};

__device__ __forceinline__ void big_set(Big &b, uint64_t v)
{
    b.n = 0;
    b.overflow = false;
    while (v) {
        b.w[b.n++] = (uint32_t)v;
        v >>= 32;
    }
}

__device__ __forceinline__ void big_mul_small(Big &b, uint32_t m)
{
    uint64_t carry = 0;
    for (int k = 0; k < b.n; ++k) {
        uint64_t t = (uint64_t)b.w[k] * m + carry;
        b.w[k] = (uint32_t)t;
        carry = t >> 32;
    }
    if (carry) {
        if (b.n < BIG_LIMBS)
            b.w[b.n++] = (uint32_t)carry;
        else
            b.overflow = true;
    }
}

__device__ __forceinline__ void big_mul_pow5(Big &b, int e)
{
    // 5^13 = 1220703125 < 2^31
    while (e >= 13) {
        big_mul_small(b, 1220703125u);
        e -= 13;
    }
    uint32_t m = 1;
    while (e-- > 0) m *= 5;
    if (m > 1) big_mul_small(b, m);
}

__device__ __forceinline__ void big_shl(Big &b, int s)
{
    if (b.n == 0 || s <= 0) return;
    const int limbs = s >> 5, bits = s & 31;
    if (b.n + limbs + 1 > BIG_LIMBS) {
        b.overflow = true;
        return;
    }
    if (bits) {
        uint32_t carry = 0;
        for (int k = 0; k < b.n; ++k) {
            uint32_t v = b.w[k];
            b.w[k] = (v << bits) | carry;
            carry = v >> (32 - bits);
        }
        if (carry) b.w[b.n++] = carry;
    }
    if (limbs) {
        for (int k = b.n - 1; k >= 0; --k) b.w[k + limbs] = b.w[k];
        for (int k = 0; k < limbs; ++k) b.w[k] = 0;
        b.n += limbs;
    }
}

__device__ __forceinline__ int big_cmp(const Big &a, const Big &b)
{
    if (a.n != b.n) return a.n < b.n ? -1 : 1;
    for (int k = a.n - 1; k >= 0; --k)
        if (a.w[k] != b.w[k]) return a.w[k] < b.w[k] ? -1 : 1;
    return 0;
}

// sign of x - m for x = Mb * 10^E (plus a little when `sticky`) and the
// positive double m (a float midpoint, or any double with <= 53 bits)
__device__ int cmp_dec_double(const Big &Mb, int E, bool sticky, double m, bool &fail)
{
    int q;
    double fr = frexp(m, &q);               // m = fr * 2^q, fr in [0.5, 1)
    uint64_t mm = (uint64_t)ldexp(fr, 53);  // exact: m has <= 53 significant bits
    q -= 53;
    while (mm && !(mm & 1)) {
        mm >>= 1;
        ++q;
    }
    const int s = E < q ? E : q;
    Big a = Mb, b;
    big_set(b, mm);
    big_mul_pow5(a, E > 0 ? E : 0);
    big_mul_pow5(b, E < 0 ? -E : 0);
    big_shl(a, E - s);
    big_shl(b, q - s);
    if (a.overflow || b.overflow) {
        fail = true;
        return 0;
    }
    const int c = big_cmp(a, b);
    return (c == 0 && sticky) ? 1 : c;
}

__device__ __forceinline__ float next_up(float f) { return __uint_as_float(__float_as_uint(f) + 1u); }
__device__ __forceinline__ float next_down(float f) { return __uint_as_float(__float_as_uint(f) - 1u); }

// A decimal x > 0: its first significant digits as M19 (up to 19 digits, x ~
// M19 * 10^E19, `inexact19` when more digits follow) and, exactly enough for
// every float midpoint, Mb = the first 120 significant digits with x = Mb *
// 10^Eb (+ a little when `sticky`).  A float midpoint has at most 113
// significant decimal digits, so the comparison with 120 digits and the
// sticky flag decides exactly.
struct Dec {
    uint64_t M19;
    int E19;
    bool inexact19;
    Big Mb;
    int Eb;
    bool sticky;
};

// |x| rounded to float (ties to even).  Sets `overflow` when the value rounds
// beyond FLT_MAX.
__device__ float dec_to_float_abs(const Dec &d, bool &overflow, bool &fail)
{
    overflow = false;
    // magnitude screen: x < 10^-46 is below half the smallest subnormal; x >=
    // 10^39 is above FLT_MAX
    int digits = 0;
    for (uint64_t t = d.M19; t; t /= 10) ++digits;
    if (digits + d.E19 <= -46) return 0.0f;
    if (digits + d.E19 > 39) {
        overflow = true;
        return 0.0f;
    }
    const uint64_t M = d.M19;
    const int E = d.E19;
    double r;
    const bool fast = !d.inexact19 && M <= (uint64_t(1) << 53) && E >= -22 && E <= 22;
    if (fast) {
        double p = 1.0;
        for (int k = 0; k < (E < 0 ? -E : E); ++k) p = __dmul_rn(p, 10.0);  // exact up to 10^22
        r = E < 0 ? __ddiv_rn((double)M, p) : __dmul_rn((double)M, p);
    } else {
        // an approximation within a few double ulps, then the exact checks
        const double tens[] = {1e1, 1e2, 1e4, 1e8, 1e16, 1e32, 1e64, 1e128, 1e256};
        int e = E < 0 ? -E : E;
        double p = 1.0;
        for (int k = 0; e && k < 9; ++k, e >>= 1)
            if (e & 1) p *= tens[k];
        r = E < 0 ? (double)M / p : (double)M * p;
    }
    if (!(r < 3.5e38)) r = 3.4028234663852886e38;  // near or above FLT_MAX: the exact check decides
    float f = __double2float_rn(r);
    if (isinf(f)) f = 3.40282347e38f;
    // r exactly on a float midpoint, or r itself inexact: check the
    // neighbouring midpoints exactly.  Above FLT_MAX the "midpoint" is the
    // overflow threshold 2^128 - 2^103.
    const double up_mid =
        f == 3.40282347e38f ? 3.4028235677973366e38 : ((double)f + (double)next_up(f)) * 0.5;
    const double dn_mid = f > 0.0f ? ((double)next_down(f) + (double)f) * 0.5 : 0.0;
    if (fast && r != up_mid && r != dn_mid) return f;
    const int cu = cmp_dec_double(d.Mb, d.Eb, d.sticky, up_mid, fail);
    if (cu > 0 || (cu == 0 && (__float_as_uint(f) & 1u))) {
        if (f == 3.40282347e38f) {
            overflow = true;
            return f;
        }
        return next_up(f);
    }
    if (f > 0.0f) {
        const int cd = cmp_dec_double(d.Mb, d.Eb, d.sticky, dn_mid, fail);
        if (cd < 0 || (cd == 0 && (__float_as_uint(f) & 1u))) return next_down(f);
    }
    return f;
}

// One token [p, e): an int32 (kind 0) or a float (kind 1).  Returns false
// when the token is not a number of that kind.
__device__ bool parse_int_token(const char *p, const char *e, int32_t &out)
{
    bool neg = false;
    if (p < e && (*p == '+' || *p == '-')) {
        neg = *p == '-';
        ++p;
    }
    if (p == e) return false;
    int64_t v = 0;
    for (; p < e; ++p) {
        const char c = *p;
        if (c < '0' || c > '9') return false;
        v = v * 10 + (c - '0');
        if (v > 2147483648ll) return false;
    }
    if (!neg && v > 2147483647ll) return false;
    out = (int32_t)(neg ? -v : v);
    return true;
}

__device__ bool parse_float_token(const char *p, const char *e, float &out)
{
    bool neg = false;
    if (p < e && (*p == '+' || *p == '-')) {
        neg = *p == '-';
        ++p;
    }
    // mantissa [m0, m1): digits with at most one point
    const char *m0 = p;
    int ndig = 0, nfrac = 0, nsig = 0;
    bool seen_point = false;
    for (; p < e; ++p) {
        const char c = *p;
        if (c == '.') {
            if (seen_point) return false;
            seen_point = true;
            continue;
        }
        if (c < '0' || c > '9') break;
        ++ndig;
        if (seen_point) ++nfrac;
        if (nsig || c != '0') ++nsig;  // leading zeros are not significant
    }
    const char *m1 = p;
    if (ndig == 0) return false;
    int64_t ex = 0;
    if (p < e && (*p == 'e' || *p == 'E')) {
        ++p;
        bool eneg = false;
        if (p < e && (*p == '+' || *p == '-')) {
            eneg = *p == '-';
            ++p;
        }
        if (p == e) return false;
        for (; p < e; ++p) {
            const char c = *p;
            if (c < '0' || c > '9') return false;
            if (ex < 100000) ex = ex * 10 + (c - '0');
        }
        if (eneg) ex = -ex;
    }
    if (p != e) return false;
    if (nsig == 0) {
        out = neg ? -0.0f : 0.0f;
        return true;
    }
    // value = (significant digits as an integer) * 10^(ex - nfrac)
    Dec d;
    d.M19 = 0;
    d.sticky = false;
    d.inexact19 = false;
    big_set(d.Mb, 0);
    const int k19 = nsig < 19 ? nsig : 19, kb = nsig < 120 ? nsig : 120;
    int seen = 0;
    for (const char *q = m0; q < m1; ++q) {
        const char c = *q;
        if (c == '.') continue;
        if (seen == 0 && c == '0') continue;
        const uint32_t dg = (uint32_t)(c - '0');
        if (seen < k19) d.M19 = d.M19 * 10 + dg;
        else if (dg) d.inexact19 = true;
        if (nsig > 19) {
            if (seen < kb) {
                big_mul_small(d.Mb, 10);
                if (dg) {
                    // add the digit
                    uint64_t carry = dg;
                    for (int k = 0; carry && k < BIG_LIMBS; ++k) {
                        if (k == d.Mb.n) d.Mb.w[d.Mb.n++] = 0;
                        const uint64_t t = (uint64_t)d.Mb.w[k] + carry;
                        d.Mb.w[k] = (uint32_t)t;
                        carry = t >> 32;
                    }
                }
            } else if (dg) {
                d.sticky = true;
            }
        }
        ++seen;
    }
    const int64_t base = ex - nfrac;
    d.E19 = (int)(base + (nsig - k19));
    if (nsig > 19) {
        d.Eb = (int)(base + (nsig - kb));
    } else {
        big_set(d.Mb, d.M19);
        d.Eb = d.E19;
    }
    bool overflow = false, fail = false;
    const float a = dec_to_float_abs(d, overflow, fail);
    if (overflow || fail) return false;
    out = neg ? -a : a;
    return true;
}

// Parses text[0, len).  Writes up to `cap` triples; returns their count, or
// -1 when the first line is not "MULTICUT" (one trailing '\r' allowed).
template <class Team>
__device__ int64_t parse_multicut(const Team &t, Scratch &sc, char *sm, const char *text, int64_t len, int32_t *oi,
                                  int32_t *oj, float *oc, int64_t cap)
{
    const int64_t nl = team_min<Team, int64_t>(t, sc, sm, len, len,
                                               [&](int64_t p) -> int64_t { return text[p] == '\n' ? p : len; });
    int64_t fl = nl;
    if (fl > 0 && text[fl - 1] == '\r') --fl;
    const char head[] = "MULTICUT";
    bool ok = fl == 8;
    for (int k = 0; ok && k < 8; ++k) ok = text[k] == head[k];
    if (!ok) return -1;
    const int64_t s0 = nl + 1 < len ? nl + 1 : len;
    const int64_t body = len - s0;
    uint64_t mark = sc.arena.mark();
    int64_t *tpos = sc.arena.take<int64_t>(body / 2 + 2);
    uint32_t *tval = sc.arena.take<uint32_t>(body / 2 + 2);
    if (!sc.arena.ok()) return 0;
    // token starts: a non-space byte after a space (or at the body's start)
    const int64_t ntok = team_compact(
        t, sc, sm, body,
        [&](int64_t q) { return !is_space_char(text[s0 + q]) && (q == 0 || is_space_char(text[s0 + q - 1])); },
        [&](int64_t q, int64_t k) { tpos[k] = s0 + q; });
    // convert every token; the first one that fails ends the input
    const int64_t first_bad = team_min<Team, int64_t>(t, sc, sm, ntok, ntok, [&](int64_t k) -> int64_t {
        const char *p = text + tpos[k];
        const char *e = p;
        const char *end = text + len;
        while (e < end && !is_space_char(*e)) ++e;
        bool good;
        if (k % 3 == 2) {
            float f = 0.0f;
            good = parse_float_token(p, e, f);
            tval[k] = __float_as_uint(f);
        } else {
            int32_t v = 0;
            good = parse_int_token(p, e, v);
            tval[k] = (uint32_t)v;
        }
        return good ? ntok : k;
    });
    int64_t n = first_bad / 3;
    if (n > cap) n = cap;
    for (int64_t r = t.rank(); r < n; r += t.size()) {
        oi[r] = (int32_t)tval[3 * r];
        oj[r] = (int32_t)tval[3 * r + 1];
        oc[r] = __uint_as_float(tval[3 * r + 2]);
    }
    t.sync();
    sc.arena.release(mark);
    sc.alg_bytes += (double)len + 12.0 * (double)n;
    return n;
}

}  // namespace rama
