// Table-driven phase factors e^{i ph} in FP64 for the element loops of the
// station beam and the weighted DFT, where one sincos per element-direction
// bounds the kernel on the FP64 pipe.
//
// Method: P. T. P. Tang's table-driven scheme ("Table-lookup algorithms for
// elementary functions and their error analysis", ARITH 1991). The loops
// carry the phase in table steps, u = ph / h with h = 2 pi / 128 (the
// per-direction factors are pre-scaled by 1 / h, so u costs the same
// multiply-adds as ph would), and
//
//   u = n + f,  n = round(u),  |f| <= 1/2 (f = u - n exactly),
//   e^{i h u} = T[n mod 128] * e^{i h f},  T[j] = e^{2 pi i j / 128},
//
// with e^{i h f} from the Taylor series of sin and cos in x = h f,
// |x| <= pi / 128, written as polynomials in f: sin to x^7 and cos - 1 to
// x^6; the first omitted terms, x^9/9! and x^8/8!, are below 4e-18. n comes
// from adding 1.5 x 2^52, which leaves round(u) in the low bits of the
// sum; the high word of that sum is one of two values exactly when
// -2^32 <= n < 2^32 (|ph| below 2.1e8 rad), which is the range the table
// path covers. Other phases, infinities and NaN are flagged for sincospi().
//
// The table sits in shared memory as 8 copies interleaved entry by entry:
// entry j of copy c is element 8 j + c. A 16-byte shared load is served a
// quarter-warp (8 lanes) at a time, and lane l reads copy l mod 8, which
// lies in bank group l mod 8 whatever the index, so the random lookups of a
// warp take four wavefronts and never conflict. 16 KB per CTA.
//
// Cost per phase factor: 15 FP64 operations (3 for the reduction, 8 for the
// polynomials, 4 to rotate the table entry), one 16-byte shared load and
// three integer operations, against one library sincos.
#pragma once

#include "common.cuh"

namespace oskb {

constexpr int kTrigEntries = 128;
constexpr int kTrigCopies = 8;
constexpr int kTrigTableSize = kTrigEntries * kTrigCopies;  // double2 slots

// 1 / h = 64 / pi: multiplies a phase in radians into table steps.
constexpr double kTrigStepsPerRadian = 20.371832715762604;

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

// e^{i h u} as (*c, *s) from the copy of this lane. Clears *covered when u
// is outside the table's range (the result is then wrong but the lookup
// stays inside the table): hot loops accumulate the flag and redo the rare
// uncovered case with trig_steps_exact, so the unrolled body has no branch.
__device__ __forceinline__ void trig_steps_sincos(const double2* table,
        double u, double* s, double* c, bool& covered)
{
    constexpr double kShift = 6755399441055744.0;  // 1.5 x 2^52
    constexpr double h = 3.141592653589793 / 64.0;
    constexpr double s1 = h, s3 = -h * h * h / 6.0,
            s5 = h * h * h * h * h / 120.0,
            s7 = -h * h * h * h * h * h * h / 5040.0;
    constexpr double c2 = -h * h / 2.0, c4 = h * h * h * h / 24.0,
            c6 = -h * h * h * h * h * h / 720.0;
    const double t = u + kShift;
    const int n = __double2loint(t);
    covered &= (unsigned) (__double2hiint(t) - 0x4337FFFF) <= 1u;
    const double f = u - (t - kShift);
    const double f2 = f * f;
    // sin(h f) = f (s1 + f^2 (s3 + f^2 (s5 + f^2 s7)))
    const double sr = f * fma(f2, fma(f2, fma(f2, s7, s5), s3), s1);
    // cos(h f) - 1 = f^2 (c2 + f^2 (c4 + f^2 c6))
    const double cm = f2 * fma(f2, fma(f2, c6, c4), c2);
    const double2 e = table[((n & (kTrigEntries - 1)) * kTrigCopies) |
            (threadIdx.x & (kTrigCopies - 1))];
    // (e.x + i e.y)(1 + cm + i sr), the small terms added to e last
    *c = fma(e.x, cm, fma(-e.y, sr, e.x));
    *s = fma(e.y, cm, fma(e.x, sr, e.y));
}

// e^{i h u} for any u, through the library: sincospi(u / 64) (u / 64 is
// exact).
__device__ __forceinline__ void trig_steps_exact(double u, double* s,
        double* c)
{
    sincospi(u * (1.0 / (kTrigEntries / 2)), s, c);
}

// e^{i h u} for any u: the table where it covers u, else the library.
__device__ __forceinline__ void trig_steps_checked(const double2* table,
        double u, double* s, double* c)
{
    bool covered = true;
    trig_steps_sincos(table, u, s, c, covered);
    if (!covered) trig_steps_exact(u, s, c);
}

}  // namespace oskb
