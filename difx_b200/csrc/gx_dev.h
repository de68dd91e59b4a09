// Device-side job and subint descriptions shared by the gxcorr kernels and
// the host driver.  All stations of one job share the sampling setup (bits,
// sampling type, frame size, bands, channels); the per-station parts are the
// recorded-frequency tables and the data buffers.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/gxcorr.h"

namespace gx {

constexpr int kMaxFramesPerBlock = 64;   // frames one FFT block may span (bits of BlockParam::validmask)
constexpr int kFThreads = 256;           // threads per F-step CTA
constexpr int kMaxFreqsPerStation = GX_MAX_LOCAL_FREQS;

// Per-station constants (device copy lives in global memory).
struct DevStation {
  int nrecfreqs;
  int fractional_lo;      // Mode::fractionalLoFreq (mode.cpp:86-102)
  int deltapol;           // any CLK OFFSET delta != 0 (mode.cpp:335-343)
  int interlaced;         // INTERLACEDVDIF: EDV4 per-band validity and weights (mk5mode.cpp:142-163)
  int wrow0;              // interlaced: weight row of band 0 (rows wrow0 .. wrow0 + nbands - 1)
  int pad_;
  double lofreq[kMaxFreqsPerStation];      // LO used for fringe rotation (mode.cpp:872-880)
  int lsb[kMaxFreqsPerStation];
  int freq_index[kMaxFreqsPerStation];     // job freq table index
  double clk[kMaxFreqsPerStation];
  double clkdelta[kMaxFreqsPerStation];
  double looff[kMaxFreqsPerStation];       // Hz
  int band_localfreq[GX_MAX_BANDS];
  int band_input[GX_MAX_BANDS];            // row of this band in its freq's spectra block
  int band_polb[GX_MAX_BANDS];             // uses fracsamprotatorB (mode.cpp:1257-1261)
};

// Job-wide constants (passed by value to kernels).
struct DevJob {
  int nstations;
  int nbands;             // recorded bands per station
  int nbits, cplx;
  int framebytes, framesamples;
  int bps_num, bps_den;   // bytes per time sample = bps_num / bps_den (mode.cpp:131-143)
  int nchan;              // N: channels per band
  int fftlen;             // F: fftchannels (2N real, N complex)
  int stride;             // S: arraystridelength
  int nfr;                // F / S
  int half;               // numfracstrides / 2
  int unpacksamples;
  int ninputs;            // NI: padded spectra rows per freq
  int nfreqs;
  int blocks_per_send;
  int sb_items;           // station-block F-step: FFT blocks per group and CTA (0: 4)
  int flaglen;
  int lgstride;           // log2(stride): FFT length, channels and stride are powers of two
  int fringe_order;       // FRINGE ROTN ORDER: 1 pre-F linear, 2 pre-F quadratic, 0 post-F (real data)
  int deltapol_any;       // some station has a second (polarisation B) fractional-sample rotator
  double sampletime;      // us
  double bw;              // MHz
  const float2 *twiddle;  // exp(-2 pi i m / F), m in [0, F), then the pass rows of r16::tw_pass_offset
  float lut[256];         // level of each sample code (VDIF decode table), staged to shared memory
  double lut_offset, lut_div;   // 8-bit codes: level = (code - lut_offset) / lut_div
  // 8-bit codes by arithmetic: level = fma(x, lut_hi, x * lut_lo) with
  // x = float(2^23 + code) - lut_bias; set only when the host has checked that
  // this equals lut[code] for all 256 codes (lut_affine = 1)
  int lut_affine;
  float lut_bias, lut_hi, lut_lo;
};

// Offset of (input row, channel c) inside the spectra of one (freq, block):
// spec[freq][block][row][channel].
__host__ __device__ __forceinline__ size_t spec_offset(const DevJob &J, int row, int c)
{
  return (size_t)row * J.nchan + c;
}

// Per (station, FFT block) parameters, computed in FP64 by blockparams_kernel
// (mode.cpp:656-757, 782-799; mk5mode.cpp:94-174) and read by the F-step.
struct __align__(16) BlockParam {
  double a, b;                    // linear delay interpolation over the block (us), b without integer part;
                                  // post-F rotation: a = 0, b = block-centre delay without its integer part;
                                  // quadratic: a = first-stride slope, b = delay at the block start
  double qa, qb;                  // quadratic: curvature and slope of the delay at the block start
  double fracwalltime;
  unsigned long long validmask;   // bit q: frame fr0+q is valid
  int nearestsample, fr0, integerdelay, intwalltime;
  float fracsampleerror, weight;
  int state, nframes;             // state 0: zeroed block
};

// Start of the subint (read from device memory, so that a replayed CUDA
// graph sees each call's value).
struct SubintClock {
  int sec, ns;
  double scan_start_sec;
};

// One subint: device pointers to its buffers.
struct SubintArrays {
  const SubintClock *clock;
  const uint8_t *const *data;    // [nstations] device pointers
  const int64_t *datalen;        // [nstations]
  const int32_t *control;        // [nstations][controlstride]
  int controlstride;
  const double *interp;          // [nstations][3]
  // [nstations][nblk][nbands] frames (bit q: frame fr0 + q) whose samples of
  // that band an EDV4 validity mask blanks; null when no station is interlaced
  const unsigned long long *bandmask;
};

// One recorded band with phase-cal extraction (the reference's implicit-shift
// extractors, pcal.cpp:1032-1222 real, 1419-1600 complex): sample n of a block
// whose absolute sample number is S goes to bin (S + n) mod nbins; tone t is
// bin offset_bin + t * step of the bins' forward DFT (0 past nbins).
// Shifting extractors (rotlen > 0): each sample is first multiplied by
// rot[rot0 + (S mod rotlen) + (n mod rotlen)], the FP32 oscillator of the
// reference (2 rotlen entries).  Tones t >= nextract stay zero.
struct PcalBand {
  int station, band, nbins, ntones, offset_bin, step;
  long long result_offset;   // first tone in the full-resolution result array
  int nextract, rotlen;
  long long rot0;
};

// Phase-cal bin sums formed inside the station-block F-step (the block's
// samples are decoded there anyway) instead of by a second read of the VDIF.
// Taken when every station with phase-cal has one implicit-shift band per
// recorded band, all with nbins bins, and nbins divides the transform's
// threads per group (F / 16): the 16 samples a thread decodes then share one
// bin.  Group g of F-step CTA x adds its sums into partial[x G + g][band][bin]
// (slots partial slots in all); first[s] is station s's first band in the
// phase-cal band list (-1: none).
struct PcalFuse {
  float2 *partial;
  const int *first;
  int nbins, maxbins, nbands_total, slots;
};

// Raises `kernel`'s dynamic shared-memory limit on the current device to at
// least `bytes`.  Safe from several host threads at once: the limit only ever
// grows, so a launch that opted in for its size cannot be undercut by another
// thread opting in for a smaller one.
cudaError_t smem_opt_in(const void *kernel, size_t bytes);

// Phase-cal: bin sums of one pass of blocks (added into partial[chunk][band][bin]),
// then the tones of all bands into the result array.
cudaError_t pcal_bins_launch(const DevJob &J, const SubintArrays &S, const BlockParam *bp, int nblk,
                             const PcalBand *bands, const float2 *rot, int nbands, int per_station, int chunks,
                             int maxbins,
                             float2 *partial, cudaStream_t st);
cudaError_t pcal_tones_launch(const PcalBand *bands, int nbands, int chunks, int maxbins, const float2 *partial,
                              float2 *results, cudaStream_t st);
// Adds chunks 1 .. chunks-1 of partial ([chunk][n]) into chunk 0, in chunk
// order, so that the tones can be formed from one chunk.
cudaError_t pcal_fold_launch(float2 *partial, int chunks, long long n, cudaStream_t st);

}  // namespace gx
