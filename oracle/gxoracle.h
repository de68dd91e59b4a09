/*
 * gxoracle -- CPU restatement of DiFX's FX-correlation hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the gxcorr CUDA path.  Nothing
 * in the product links, loads or calls this code.
 *
 * It restates, for the configurations gxcorr supports (single-thread VDIF,
 * real or complex single-sideband sampling, fringe rotation order 1, one
 * phase centre, no pulsar binning, zoom bands, phase cal or channel
 * averaging), the algorithm of:
 *   Mk5Mode::unpack           mpifxcorr/src/mk5mode.cpp:94-174 with the VDIF
 *                             decode/validate/blank of libraries/mark5access
 *                             (format_vdif.c:66-146, 7619-7667;
 *                             mark5_stream.c:144-191; blanker_mark5.c:272-306;
 *                             mark5_stream_unpacker.c:119-183)
 *   Mode::process             mpifxcorr/src/mode.cpp:634-1374
 *   Core::processdata XMAC    mpifxcorr/src/core.cpp:657-1129
 *   result layout             mpifxcorr/src/configuration.cpp:2348-2630
 *
 * Two precisions:
 *   GXO_FP32_REF  the reference's FP32 operation order (GENERIC
 *                 architecture, architecture.h.in:512-880), including the
 *                 thread block split and the shift/average flush intervals,
 *                 so a single-threaded reference run is reproduced exactly;
 *   GXO_FP64      every step in double (exact sincos, double DFT, double
 *                 accumulation): the precision oracle for the tensor-core form.
 */
#ifndef GXORACLE_H
#define GXORACLE_H
#include "../include/gxcorr.h"
#ifdef __cplusplus
extern "C" {
#endif

enum { GXO_FP32_REF = 0, GXO_FP64 = 1 };

typedef struct gxo_params {
  int precision;            /* GXO_FP32_REF or GXO_FP64 */
  int nthreads;             /* reference process threads (block split, core.cpp:2162-2166) */
  int num_buffered_ffts;    /* NUM BUFFERED FFTS */
  long long xc_avg_ns;      /* UVSHIFT INTERVAL (NS): cross-correlation flush interval */
  long long ac_avg_ns;      /* AC AVG INTERVAL (NS): autocorrelation flush interval */
} gxo_params;

/* Length of the Core result array (complex floats) and the offsets
   (complex-float units; [nfreqs*nbaselines], [nstations]). */
long long gxo_layout(const gx_job_desc *d, int *blofs, int *bwofs, int *acofs, int *acwofs);

/* Unpack nsamp time samples of every band starting at sample `offset`.
   out: nbands x nsamp floats (real) or nbands x 2*nsamp (complex, interleaved).
   Returns the good-sample count (nsamp minus blanked samples). */
int gxo_unpack(const gx_station_desc *st, int framesamples, const unsigned char *data, long long datalen,
               int offset, int nsamp, float *out);

/* One FFT block of one station (Mode::process): nbands x nchan complex
   values (double, interleaved) and the block's data weight. */
int gxo_station_block(const gx_job_desc *d, const gx_subint_desc *s, int station, int block,
                      const gxo_params *p, double *spectra, double *weight);

/* Whole subint -> Core result array as doubles (2*result_length values). */
int gxo_subint(const gx_job_desc *d, const gx_subint_desc *s, const gxo_params *p, double *results);

#ifdef __cplusplus
}
#endif
#endif
