/* gxfft: the oracle's discrete Fourier transform (test infrastructure only).
 *
 * Evaluates the un-normalised forward DFT X[k] = sum_j x[j] exp(-2 pi i jk/n)
 * (the convention of the reference's FFT calls, mpifxcorr/src/architecture.h.in:
 * 824-836 FFTW_FORWARD plans, and IPP's ippsFFTFwd_CToC_32fc with
 * IPP_FFT_NODIV_BY_ANY) in double precision and rounds once to float, so the
 * float result is within ~1 ulp of the exact transform of the float input.
 * Power-of-two lengths use an iterative radix-2 transform; other lengths a
 * direct O(n^2) sum.  Used by the oracle C restatement and by the fftw3.h
 * shim that lets the reference sources compile without FFTW. */
#ifndef GXFFT_H
#define GXFFT_H
#ifdef __cplusplus
extern "C" {
#endif
/* in/out: n interleaved (re, im) float pairs; out may alias in. sign=-1 forward, +1 backward. */
void gxfft_c2c_f32(const float *in, float *out, int n, int sign);
/* same in double, in place on n interleaved pairs */
void gxfft_c2c_f64(double *data, int n, int sign);
#ifdef __cplusplus
}
#endif
#endif
