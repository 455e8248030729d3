/* Test shim: mel_sin / mel_cos (the device's rigid-rotation sine and cosine) and glibc's sin / cos
 * over arrays. */
#include <math.h>
#include "mel_sincos.h"

void mel_sincos_batch(const double* x, double* s, double* c, int n)
{
    for (int i = 0; i < n; i++) { s[i] = mel_sin(x[i]); c[i] = mel_cos(x[i]); }
}

void libm_sincos_batch(const double* x, double* s, double* c, int n)
{
    for (int i = 0; i < n; i++) { s[i] = sin(x[i]); c[i] = cos(x[i]); }
}
