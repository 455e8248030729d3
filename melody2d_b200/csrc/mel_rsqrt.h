/* Correctly rounded x^(-1/2) for host and device.
 *
 * The reference evaluates pow(d2, -0.5) for inverse lengths in its projections
 * (Code/Tools.h:108-110,152,187) and border loads (Code/Body.h:733-734).  glibc's pow is not
 * correctly rounded for this exponent: for about 8 arguments in 10,000 it returns the neighbour of
 * the nearest double.  CUDA has no bit-compatible pow, so the device computes the double nearest
 * to 1/sqrt(x) instead, and the oracle can run in either mode (glibc's pow, pinned to the
 * reference; or this function, which the GPU path must then match bit for bit):
 *
 *   y  = 1 / sqrt(x)                      two correctly rounded IEEE operations, |y/t - 1| < 2^-52
 *   r  = 1 - x*y*y                        evaluated with error-free products (fma), |r| < 2^-51
 *   t ~= y + y*r/2                        one Newton step for x^(-1/2); the dropped 3r^2/8 term and
 *                                         the rounding of r leave |y + y*r/2 - t| < 2^-103 t
 *
 * so rounding y + y*r/2 to double gives the correctly rounded result unless 1/sqrt(x) lies within
 * 2^-103 (relative) of the midpoint between two doubles.  tests/test_rsqrt.py checks it against a
 * 60-digit decimal evaluation and counts glibc's misrounded cases.
 * Arguments outside [1e-289, 1e289] are scaled by exact powers of two first. */
#ifndef MEL_RSQRT_H
#define MEL_RSQRT_H

#include <math.h>

#if defined(__CUDACC__)
#define MEL_HD __host__ __device__ __forceinline__
#else
#define MEL_HD static inline
#endif

MEL_HD double mel_rsqrt_core(double x)
{
    double y = 1.0 / sqrt(x);
    double p = y * y;
    double pe = fma(y, y, -p);          /* y*y = p + pe exactly          */
    double q = x * p;
    double qe = fma(x, p, -q);          /* x*p = q + qe exactly          */
    double r = (1.0 - q) - qe;          /* 1 - q is exact (q close to 1) */
    r = r - x * pe;
    double d = 0.5 * y;
    d = d * r;
    return y + d;
}

MEL_HD double mel_rsqrt(double x)
{
    if (x != x) return x;                           /* NaN                              */
    if (x == 0.0) return HUGE_VAL;                  /* pow(+-0, -0.5) = +inf            */
    if (x < 0.0) return sqrt(x);                    /* NaN, as pow(negative, -0.5)      */
    if (x == HUGE_VAL) return 0.0;
    const double two500 = 3.2733906078961419e150;   /* 2^500  */
    const double twom500 = 3.0549363634996047e-151; /* 2^-500 */
    if (x < 1.0e-289) return mel_rsqrt_core((x * two500) * two500) * two500;
    if (x > 1.0e289) return mel_rsqrt_core((x * twom500) * twom500) * twom500;
    return mel_rsqrt_core(x);
}

#endif
