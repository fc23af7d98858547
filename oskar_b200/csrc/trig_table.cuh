// Table-driven phase factors e^{i ph} in FP64 for the element loops of the
// station beam and the weighted DFT, where one sincos per element-direction
// bounds the kernel on the FP64 pipe.
//
// Method: P. T. P. Tang's table-driven scheme ("Table-lookup algorithms for
// elementary functions and their error analysis", ARITH 1991) with
// Cody-Waite argument reduction (W. J. Cody and W. Waite, "Software Manual
// for the Elementary Functions", 1980):
//
//   ph = n h + r,  h = 2 pi / 128,  |r| <= h / 2 (plus rounding),
//   e^{i ph} = T[n mod 128] * e^{i r},  T[j] = e^{2 pi i j / 128},
//
// with e^{i r} from its Taylor series: sin r to r^7 and cos r - 1 to r^6;
// the first omitted terms, r^9/9! and r^8/8!, are below 4e-18 for
// |r| <= pi / 128. h is carried as a head (the double nearest pi, over 64)
// and a tail ((pi - that double) / 64), applied with fused multiply-adds,
// so r is accurate to about one ulp of r for |ph| < 2^40; larger phases,
// infinities and NaN take sincos(). n comes from adding 1.5 x 2^52, which
// leaves round(ph / h) in the low bits of the sum.
//
// The table sits in shared memory as 8 copies interleaved entry by entry:
// entry j of copy c is element 8 j + c. A 16-byte shared load is served a
// quarter-warp (8 lanes) at a time, and lane l reads copy l mod 8, which
// lies in bank group l mod 8 whatever the index, so the random lookups of a
// warp take four wavefronts and never conflict. 16 KB per CTA.
//
// Cost per phase factor: 16 FP64 operations, one 16-byte shared load and
// two integer operations, against one library sincos.
#pragma once

#include "common.cuh"

namespace oskb {

constexpr int kTrigEntries = 128;
constexpr int kTrigCopies = 8;
constexpr int kTrigTableSize = kTrigEntries * kTrigCopies;  // double2 slots

// Fills the table; all threads of the CTA take part and must reach a
// __syncthreads() before the first lookup.
__device__ __forceinline__ void trig_table_fill(double2* table)
{
    for (int j = threadIdx.x; j < kTrigEntries; j += blockDim.x)
    {
        double s, c;
        sincospi((double) j / (kTrigEntries / 2), &s, &c);
#pragma unroll
        for (int k = 0; k < kTrigCopies; ++k)
            table[j * kTrigCopies + k] = make_double2(c, s);
    }
}

// Whether the table method covers ph (false for |ph| >= 2^40 and NaN).
__device__ __forceinline__ bool trig_table_covers(double ph)
{
    return fabs(ph) < 1.0995116277760000e12;
}

// e^{i ph} as (*c, *s), reading the copy of this lane; no range check (a
// phase outside trig_table_covers gives a wrong but finite-index result).
// Hot loops call this and redo the rare uncovered case with sincos, so
// that the unrolled loop body has no branch.
__device__ __forceinline__ void trig_table_sincos_unchecked(
        const double2* table, double ph, double* s, double* c)
{
    // 64 / pi and the head/tail split of pi / 64.
    constexpr double kInvStep = 20.371832715762604;
    constexpr double kStepHi = 3.141592653589793 / 64.0;
    constexpr double kStepLo = 1.2246467991473532e-16 / 64.0;
    constexpr double kShift = 6755399441055744.0;  // 1.5 x 2^52
    const double t = fma(ph, kInvStep, kShift);
    const int n = __double2loint(t);
    const double nd = t - kShift;
    double r = fma(-nd, kStepHi, ph);
    r = fma(-nd, kStepLo, r);
    const double r2 = r * r;
    // sin r = r + r^3 (-1/6 + r^2 (1/120 - r^2 / 5040))
    const double ps = fma(r2, fma(r2, -1.0 / 5040.0, 1.0 / 120.0),
            -1.0 / 6.0);
    const double sr = fma(r * r2, ps, r);
    // cos r - 1 = r^2 (-1/2 + r^2 (1/24 - r^2 / 720))
    const double cm = r2 * fma(r2, fma(r2, -1.0 / 720.0, 1.0 / 24.0), -0.5);
    const double2 e = table[((n & (kTrigEntries - 1)) * kTrigCopies) |
            (threadIdx.x & (kTrigCopies - 1))];
    // (e.x + i e.y)(1 + cm + i sr), the small terms added to e last
    *c = fma(e.x, cm, fma(-e.y, sr, e.x));
    *s = fma(e.y, cm, fma(e.x, sr, e.y));
}

// e^{i ph} as (*c, *s) for any ph: the table where it covers ph, else
// sincos().
__device__ __forceinline__ void trig_table_sincos(const double2* table,
        double ph, double* s, double* c)
{
    if (!trig_table_covers(ph))
    {
        sincos(ph, s, c);
        return;
    }
    trig_table_sincos_unchecked(table, ph, s, c);
}

}  // namespace oskb
