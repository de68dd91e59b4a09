/* gxfft: double-precision DFT for the oracle (test infrastructure only).
 * See gxfft.h for the convention it follows. */
#include "gxfft.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

static const double GX_PI = 3.14159265358979323846264338327950288;

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

void gxfft_c2c_f64(double *d, int n, int sign)
{
  if (n <= 1) return;
  if (!is_pow2(n)) {
    double *t = (double *)malloc(sizeof(double) * 2 * n);
    for (int k = 0; k < n; k++) {
      double sr = 0, si = 0;
      for (int j = 0; j < n; j++) {
        long long m = ((long long)j * k) % n;
        double a = sign * 2.0 * GX_PI * (double)m / (double)n;
        double c = cos(a), s = sin(a);
        sr += d[2*j] * c - d[2*j+1] * s;
        si += d[2*j] * s + d[2*j+1] * c;
      }
      t[2*k] = sr; t[2*k+1] = si;
    }
    memcpy(d, t, sizeof(double) * 2 * n);
    free(t);
    return;
  }
  /* bit reversal */
  for (int i = 1, j = 0; i < n; i++) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      double tr = d[2*i], ti = d[2*i+1];
      d[2*i] = d[2*j]; d[2*i+1] = d[2*j+1];
      d[2*j] = tr; d[2*j+1] = ti;
    }
  }
  for (int len = 2; len <= n; len <<= 1) {
    int half = len >> 1;
    for (int k = 0; k < half; k++) {
      /* twiddle evaluated directly (no recurrence) for accuracy */
      double a = sign * 2.0 * GX_PI * (double)k / (double)len;
      double wr = cos(a), wi = sin(a);
      for (int s = 0; s < n; s += len) {
        int p = s + k, q = p + half;
        double xr = d[2*q] * wr - d[2*q+1] * wi;
        double xi = d[2*q] * wi + d[2*q+1] * wr;
        d[2*q] = d[2*p] - xr; d[2*q+1] = d[2*p+1] - xi;
        d[2*p] += xr; d[2*p+1] += xi;
      }
    }
  }
}

void gxfft_c2c_f32(const float *in, float *out, int n, int sign)
{
  double *t = (double *)malloc(sizeof(double) * 2 * (n > 0 ? n : 1));
  for (int i = 0; i < 2 * n; i++) t[i] = in[i];
  gxfft_c2c_f64(t, n, sign);
  for (int i = 0; i < 2 * n; i++) out[i] = (float)t[i];
  free(t);
}
