/* Oracle build shim (test infrastructure only): FFTW plan API over gxfft. */
#include "fftw3.h"
#include "../gxfft.h"
#include <stdlib.h>
#include <string.h>

enum { K_C2C = 0, K_R2C = 1, K_C2R = 2, K_C2C_2D = 3 };
struct gx_fftwf_plan_s { int kind, n, n1, sign; void *in, *out; };

void *fftwf_malloc(size_t n) { void *p = 0; if (posix_memalign(&p, 64, n ? n : 16)) return 0; return p; }
void fftwf_free(void *p) { free(p); }

static fftwf_plan mk(int kind, int n, int n1, int sign, void *in, void *out)
{
  fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
  p->kind = kind; p->n = n; p->n1 = n1; p->sign = sign; p->in = in; p->out = out;
  return p;
}
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned f)
{ (void)f; return mk(K_C2C, n, 1, sign, in, out); }
fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in, fftwf_complex *out, int sign, unsigned f)
{ (void)f; return mk(K_C2C_2D, n0, n1, sign, in, out); }
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out, unsigned f)
{ (void)f; return mk(K_R2C, n, 1, -1, in, out); }
fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex *in, float *out, unsigned f)
{ (void)f; return mk(K_C2R, n, 1, +1, in, out); }
void fftwf_destroy_plan(fftwf_plan p) { free(p); }

void fftwf_execute(const fftwf_plan p)
{
  int n = p->n;
  if (p->kind == K_C2C) {
    gxfft_c2c_f32((const float *)p->in, (float *)p->out, n, p->sign);
  } else if (p->kind == K_R2C) {
    double *t = (double *)malloc(sizeof(double) * 2 * n);
    const float *x = (const float *)p->in;
    for (int i = 0; i < n; i++) { t[2*i] = x[i]; t[2*i+1] = 0.0; }
    gxfft_c2c_f64(t, n, -1);
    float *o = (float *)p->out;
    for (int i = 0; i < 2 * (n / 2 + 1); i++) o[i] = (float)t[i];
    free(t);
  } else if (p->kind == K_C2R) {
    double *t = (double *)malloc(sizeof(double) * 2 * n);
    const float *x = (const float *)p->in;
    for (int i = 0; i <= n / 2; i++) { t[2*i] = x[2*i]; t[2*i+1] = x[2*i+1]; }
    for (int i = n / 2 + 1; i < n; i++) { t[2*i] = x[2*(n-i)]; t[2*i+1] = -x[2*(n-i)+1]; }
    gxfft_c2c_f64(t, n, +1);
    float *o = (float *)p->out;
    for (int i = 0; i < n; i++) o[i] = (float)t[2*i];
    free(t);
  } else {
    /* 2-D: rows then columns, in double */
    int n0 = p->n, n1 = p->n1;
    double *t = (double *)malloc(sizeof(double) * 2 * n0 * n1);
    double *col = (double *)malloc(sizeof(double) * 2 * n0);
    const float *x = (const float *)p->in;
    for (int i = 0; i < 2 * n0 * n1; i++) t[i] = x[i];
    for (int r = 0; r < n0; r++) gxfft_c2c_f64(t + 2 * r * n1, n1, p->sign);
    for (int c = 0; c < n1; c++) {
      for (int r = 0; r < n0; r++) { col[2*r] = t[2*(r*n1+c)]; col[2*r+1] = t[2*(r*n1+c)+1]; }
      gxfft_c2c_f64(col, n0, p->sign);
      for (int r = 0; r < n0; r++) { t[2*(r*n1+c)] = col[2*r]; t[2*(r*n1+c)+1] = col[2*r+1]; }
    }
    float *o = (float *)p->out;
    for (int i = 0; i < 2 * n0 * n1; i++) o[i] = (float)t[i];
    free(col); free(t);
  }
}
