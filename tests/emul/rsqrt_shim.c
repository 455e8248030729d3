/* Test shim: mel_rsqrt (the device's x^(-1/2)) and glibc's pow(x, -0.5) over arrays. */
#include <math.h>
#include "mel_rsqrt.h"

void rsqrt_batch(const double* x, double* y, int n)
{
    for (int i = 0; i < n; i++) y[i] = mel_rsqrt(x[i]);
}

void pow_batch(const double* x, double* y, int n)
{
    for (int i = 0; i < n; i++) y[i] = pow(x[i], -0.5);
}
