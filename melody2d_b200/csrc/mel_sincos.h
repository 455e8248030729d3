/* Correctly rounded sine and cosine for host and device.
 *
 * Rigid bodies turn their nodes by the angle rd - r0 of the body (Code/Body.h:2284-2300, and the
 * temporary kinematics of the adaptive schemes, Code/Body.h:2235-2264), with the C library's cos and
 * sin.  CUDA's cos and sin are accurate to a few units in the last place but are not the same
 * functions (and glibc's miss the nearest double for a few arguments in ten thousand), so the device
 * evaluates the double nearest to the exact value instead, and the oracle's correctly-rounded mode
 * uses this same header; tests/test_sincos.py checks it against an 80-digit evaluation.
 *
 * Method (double-double arithmetic, every product made exact with fma):
 *   n = nearest integer to x * 2/pi,  r = x - n * pi/2 with pi/2 = P1 + P2 + P3 (Cody-Waite: P1 and
 *   P2 carry 33 significant bits, so n*P1 and n*P2 are exact for |n| < 2^20, and n*P3 is split
 *   exactly), kept as a double-double r = rh + rl;
 *   sin r = r * sum_k (-1)^k r^2k / (2k+1)!  (k <= 14),  cos r = sum_k (-1)^k r^2k / (2k)!  (k <= 15),
 *   Horner in double-double with the coefficients 1/k! as double-double constants; for |r| <= pi/4
 *   the dropped terms are below 2^-107 of the result;
 *   the quadrant n mod 4 selects +-sin r or +-cos r, and the double-double result is rounded once.
 * The result is the double nearest to sin x (cos x) unless the exact value lies within about 2^-100
 * (relative) of a midpoint between two doubles.  Beyond |x| = 2^19 pi/2 the reduction would lose its
 * exactness, and there (and for non-finite x) the functions return the platform's own sin and cos. */
#ifndef MEL_SINCOS_H
#define MEL_SINCOS_H

#include <math.h>

#if defined(__CUDACC__)
#define MEL_SC_HD __host__ __device__ __forceinline__
#else
#define MEL_SC_HD static inline
#endif

typedef struct { double h, l; } mel_dd;

MEL_SC_HD mel_dd mel_dd_two_sum(double a, double b)
{
    mel_dd r;
    r.h = a + b;
    double v = r.h - a;
    r.l = (a - (r.h - v)) + (b - v);
    return r;
}

MEL_SC_HD mel_dd mel_dd_quick(double a, double b)   /* |a| >= |b| */
{
    mel_dd r;
    r.h = a + b;
    r.l = b - (r.h - a);
    return r;
}

MEL_SC_HD mel_dd mel_dd_mul(mel_dd a, mel_dd b)
{
    double p = a.h * b.h;
    double e = fma(a.h, b.h, -p);
    e = e + (a.h * b.l + a.l * b.h);
    return mel_dd_quick(p, e);
}

MEL_SC_HD mel_dd mel_dd_add(mel_dd a, mel_dd b)
{
    mel_dd s = mel_dd_two_sum(a.h, b.h);
    mel_dd t = mel_dd_two_sum(a.l, b.l);
    s.l = s.l + t.h;
    s = mel_dd_quick(s.h, s.l);
    s.l = s.l + t.l;
    return mel_dd_quick(s.h, s.l);
}

/* 1/k! as double-double (k = 0..30), exact to about 2^-106 */
MEL_SC_HD mel_dd mel_invfact(int k)
{
    /* high parts */
    const double H[31] = {
        1.0, 1.0, 0x1.0000000000000p-1, 0x1.5555555555555p-3, 0x1.5555555555555p-5, 0x1.1111111111111p-7,
        0x1.6c16c16c16c17p-10, 0x1.a01a01a01a01ap-13, 0x1.a01a01a01a01ap-16, 0x1.71de3a556c734p-19,
        0x1.27e4fb7789f5cp-22, 0x1.ae64567f544e4p-26, 0x1.1eed8eff8d898p-29, 0x1.6124613a86d09p-33,
        0x1.93974a8c07c9dp-37, 0x1.ae7f3e733b81fp-41, 0x1.ae7f3e733b81fp-45, 0x1.952c77030ad4ap-49,
        0x1.6827863b97d97p-53, 0x1.2f49b46814157p-57, 0x1.e542ba4020225p-62, 0x1.71b8ef6dcf572p-66,
        0x1.0ce396db7f853p-70, 0x1.761b41316381ap-75, 0x1.f2cf01972f578p-80, 0x1.3f3ccdd165fa9p-84,
        0x1.88e85fc6a4e5ap-89, 0x1.d1ab1c2dccea3p-94, 0x1.0a18a2635085dp-98, 0x1.259f98b4358adp-103,
        0x1.3932c5047d60ep-108 };
    /* low parts */
    const double L[31] = {
        0.0, 0.0, 0.0, 0x1.5555555555555p-57, 0x1.5555555555555p-59, 0x1.1111111111111p-63,
        -0x1.f49f49f49f49fp-65, 0x1.a01a01a01a01ap-73, 0x1.a01a01a01a01ap-76, -0x1.c154f8ddc6c00p-73,
        0x1.cbbc05b4fa99ap-76, -0x1.c062e06d1f209p-80, -0x1.2aec959e14c06p-83, 0x1.f28e0cc748ebep-87,
        0x1.05d6f8a2efd1fp-92, 0x1.1d8656b0ee8cbp-97, 0x1.1d8656b0ee8cbp-101, 0x1.ac981465ddc6cp-103,
        0x1.eec01221a8b0bp-107, 0x1.2650f61dbdcb4p-112, 0x1.ea72b4afe3c2fp-120, -0x1.d043ae40c4647p-120,
        -0x1.aebcdbd20331cp-124, -0x1.3423c7d91404fp-130, -0x1.9ada5fcc1ab14p-135, -0x1.58ddadf344487p-139,
        -0x1.71c37ebd16540p-143, 0x1.054d0c78aea14p-149, 0x1.b9e2e28e1aa54p-153, 0x1.eaf8c39dd9bc5p-157,
        0x1.832b7b530a627p-162 };
    mel_dd r;
    r.h = H[k];
    r.l = L[k];
    return r;
}

/* sum_{k=0..K} (-1)^k r2^k c(k0 + 2k), Horner from the last term */
MEL_SC_HD mel_dd mel_dd_series(mel_dd r2, int k0, int K)
{
    mel_dd s = mel_invfact(k0 + 2 * K);
    if (K & 1) { s.h = -s.h; s.l = -s.l; }
    for (int k = K - 1; k >= 0; k--) {
        mel_dd c = mel_invfact(k0 + 2 * k);
        if (k & 1) { c.h = -c.h; c.l = -c.l; }
        s = mel_dd_add(c, mel_dd_mul(r2, s));
    }
    return s;
}

/* sin (which = 0) or cos (which = 1) of x, correctly rounded as described above */
MEL_SC_HD double mel_sincos_eval(double x, int which)
{
    const double two_over_pi = 0x1.45f306dc9c883p-1;
    const double P1 = 0x1.921fb54400000p+0, P2 = 0x1.0b4611a600000p-34, P3 = 0x1.3198a2e037073p-69;
    if (!(fabs(x) <= 823550.0)) return which ? cos(x) : sin(x);   /* 2^19 pi/2, NaN, inf */
    if (x == 0.0) return which ? 1.0 : x;                          /* keeps the sign of zero */
    const double n = rint(x * two_over_pi);
    /* r = x - n P1 - n P2 - n P3 as a double-double (the first subtraction is exact) */
    mel_dd a = mel_dd_two_sum(x, -(n * P1));
    mel_dd b = mel_dd_two_sum(a.h, -(n * P2));
    double p3 = n * P3;
    double e3 = fma(n, P3, -p3);
    double lo = ((a.l + b.l) - p3) - e3;
    mel_dd r = mel_dd_two_sum(b.h, lo);
    mel_dd r2 = mel_dd_mul(r, r);
    const int q = (int)((long long)n & 3);
    const int use_cos = (q & 1) ^ which;         /* cos(x) = sin(x + pi/2) */
    mel_dd v;
    if (use_cos) v = mel_dd_series(r2, 0, 15);
    else v = mel_dd_mul(r, mel_dd_series(r2, 1, 14));
    /* sin: quadrants 2, 3 negate; cos: quadrants 1, 2 negate */
    const int neg = which ? (q == 1 || q == 2) : (q >= 2);
    double out = v.h + v.l;
    return neg ? -out : out;
}

MEL_SC_HD double mel_sin(double x) { return mel_sincos_eval(x, 0); }
MEL_SC_HD double mel_cos(double x) { return mel_sincos_eval(x, 1); }

#endif
