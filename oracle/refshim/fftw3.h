/* Oracle build shim (test infrastructure only): the handful of FFTW entry
 * points the reference's GENERIC architecture path calls
 * (mpifxcorr/src/architecture.h.in:798-845, 1014-1046), implemented on the
 * oracle's own double-precision DFT (gxfft.c), because FFTW is not
 * installed.  Plans are forward/backward un-normalised like FFTW's. */
#ifndef GX_ORACLE_FFTW3_SHIM_H
#define GX_ORACLE_FFTW3_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef float fftwf_complex[2];
typedef double fftw_complex[2];
typedef struct gx_fftwf_plan_s *fftwf_plan;
typedef struct gx_fftwf_plan_s *fftw_plan;
#define FFTW_FORWARD  (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MEASURE  0U
void *fftwf_malloc(size_t n);
void fftwf_free(void *p);
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex *in, float *out, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
#ifdef __cplusplus
}
#endif
#endif
