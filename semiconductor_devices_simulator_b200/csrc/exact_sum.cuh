// Order-independent sums of doubles for kernels whose threads add into shared totals.
//
// A floating-point atomicAdd makes a total depend on the order in which threads arrive, so
// two runs of the same solve can differ in the last bits.  Here every term is added exactly
// into a fixed-point accumulator instead: the term's 53-bit significand, shifted to its
// binary exponent, is split into 32-bit digits, and each digit is added with an integer
// atomic into a 64-bit word (integer additions commute, and 2^32 additions fit a word before
// it could wrap).  Positive and negative terms have accumulators of their own.  The total is
// read back once by xs_value: the same for any order of the terms.
//
// The accumulator covers bit weights 2^XS_LO .. 2^(XS_LO + 32 XS_DIGITS); the bits of a term
// below 2^XS_LO are dropped (deterministically), and a term too large to fit sets the
// accumulator's flag word, which makes xs_value return NaN, as does a NaN term.
#pragma once
#include <cstdint>

namespace ss {

constexpr int XS_DIGITS = 42;                 // 32-bit digits per sign
constexpr int XS_LO = -600;                   // weight of bit 0: 2^-600
constexpr int XS_WORDS = 2 * XS_DIGITS + 1;   // [sign][digit], then the flag word

// add v to the accumulator acc[XS_WORDS]
__device__ __forceinline__ void xs_add(unsigned long long *acc, double v) {
    if (v == 0.0) return;
    if (!(v == v)) { atomicOr(acc + 2 * XS_DIGITS, 1ull); return; }
    const unsigned long long bits = (unsigned long long)__double_as_longlong(v);
    const int neg = (int)(bits >> 63);
    const int ex = (int)((bits >> 52) & 0x7ff);
    unsigned long long mant = bits & ((1ull << 52) - 1);
    int e2;                                   // |v| = mant * 2^e2
    if (ex == 0) e2 = -1074;
    else { mant |= 1ull << 52; e2 = ex - 1075; }
    if (ex == 0x7ff) { atomicOr(acc + 2 * XS_DIGITS, 1ull); return; }
    int p = e2 - XS_LO;                       // bit position of mant's lowest bit
    if (p < 0) {
        if (p <= -53) return;
        mant >>= -p;
        p = 0;
        if (!mant) return;
    }
    if (p + 53 > 32 * (XS_DIGITS - 1)) { atomicOr(acc + 2 * XS_DIGITS, 1ull); return; }
    const int q = p >> 5, o = p & 31;
    const unsigned long long lo = mant << o, hi = o ? mant >> (64 - o) : 0ull;
    unsigned long long *d = acc + neg * XS_DIGITS + q;
    if (lo & 0xffffffffull) atomicAdd(d, lo & 0xffffffffull);
    if (lo >> 32) atomicAdd(d + 1, lo >> 32);
    if (hi) atomicAdd(d + 2, hi);
}

// the accumulator's total (pos - neg): both sides carry-propagated to 32-bit digits, their
// difference taken exactly, then rounded to a double from its top 96 bits
__device__ __forceinline__ double xs_value(const unsigned long long *acc) {
    if (acc[2 * XS_DIGITS]) return __longlong_as_double(0x7ff8000000000000ll);
    unsigned int dig[2][XS_DIGITS];
    for (int s = 0; s < 2; s++) {
        unsigned long long carry = 0;
        for (int q = 0; q < XS_DIGITS; q++) {
            const unsigned long long t = acc[s * XS_DIGITS + q] + carry;
            dig[s][q] = (unsigned int)(t & 0xffffffffull);
            carry = t >> 32;
        }
    }
    int big = 0;                              // the side with the larger magnitude
    for (int q = XS_DIGITS - 1; q >= 0; q--)
        if (dig[0][q] != dig[1][q]) { big = dig[0][q] > dig[1][q] ? 0 : 1; break; }
    unsigned int dif[XS_DIGITS];
    long long borrow = 0;
    for (int q = 0; q < XS_DIGITS; q++) {
        long long t = (long long)dig[big][q] - (long long)dig[1 - big][q] - borrow;
        borrow = t < 0;
        if (t < 0) t += 4294967296ll;
        dif[q] = (unsigned int)t;
    }
    int h = XS_DIGITS - 1;
    while (h >= 0 && dif[h] == 0) h--;
    if (h < 0) return 0.0;
    double v = 0.0;
    const int lo = h >= 2 ? h - 2 : 0;
    for (int q = h; q >= lo; q--) v = v * 4294967296.0 + (double)dif[q];
    v = scalbn(v, 32 * lo + XS_LO);
    return big ? -v : v;
}

}  // namespace ss
