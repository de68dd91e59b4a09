// Kernel entry points and tables shared between the gxcorr kernels and the host driver.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>
#include "gx_dev.h"

namespace gx {

// One visibility row of the Core result array: result_offset + c <- acc[acc_index + c] (conj if set).
struct ProdEntry {
  long long result_offset;  // complex-float index into the result array
  long long acc_index;      // complex-float index into the ks = 0 accumulator slice
  int conj;
  int pad_;
};

// One float slot of the result array that holds a weight.
struct WeightEntry {
  long long float_index;    // float index into the result array
  int source;               // index into the weight accumulators (-1: zero)
  int pad_;
};

// One visibility row for the tensor-core X-step: input pair (a, b) of freq.
struct TcProdEntry {
  long long result_offset;  // complex-float index into the result array
  int freq, a, b;
  int pad_;
};

struct XmacShape {
  int T, ST, CT;
  int nsuper, npairs;
};

XmacShape xmac_shape(int NI);

// 4-D FP32 tensor map over a dense array (dims innermost first), box `box`.
cudaError_t tma_map_f32_4d(CUtensorMap *map, const void *base, const cuuint64_t dims[4], const cuuint32_t box[4]);

size_t fstep_smem_bytes(const DevJob &J, int nrf, int nslots);
// Whether the station-block F-step (gx_fstep_sb.cu) takes this job.
bool fstep_sb_eligible(const DevJob &J, bool interlaced);
// F-step of one pass of blocks.  With pf, the station-block kernel also forms
// the phase-cal bin sums when it takes the job; *pcal_done (if given) tells
// whether it did (else the caller runs pcal_bins_launch).
cudaError_t fstep_launch(const DevJob &J, const DevStation *stations, int maxnrf, const SubintArrays &S,
                         int blk0, int nblk, int nslots, float2 *spec, float *weights, BlockParam *bp,
                         cudaStream_t st, const PcalFuse *pf = nullptr, bool *pcal_done = nullptr);
// FP32 X-step over one pass of blocks; *err (may be null) receives a nonzero
// status if a wait of the kernel expired.  variant: the launch shape (0: the
// default channel tile and stage depth; 1: the other one of the shape class,
// kXmacVariants in all); the sums are the same for every variant.
constexpr int kXmacVariants = 2;
cudaError_t xmac_fp32_launch(const float2 *spec, int nblk, int NI, int N, int nfreqs, int ks, float2 *acc, int *err,
                             cudaStream_t st, int variant = 0);
cudaError_t weights_launch(const float *w, int nblk, int nstations, const int2 *pairs, int npairs, float *wacc,
                           cudaStream_t st);
// Entries [start, end) of the tensor-core product table (sorted by freq, then a)
// share row a of freq; bmin is their smallest b.
struct TcRowEntry {
  int freq, a, bmin, start, end;
};

// Tensor-core X-step over spectra [freq][block][ninputs][N] (ninputs <= 128,
// the MMA tile's M; missing rows are zeros); acc holds, per K-split slice,
// [freq][N/2][128][128] float4 = (Re, Im) of both channels of a channel pair,
// unscaled, of which rows and columns below ninputs are written.
size_t xmac_tc_smem_bytes(bool hilo);
cudaError_t xmac_tc_launch(const float2 *spec, int nblk, int N, int nfreqs, int ninputs, int ks, bool hilo,
                           const float *scale, float4 *acc, int accumulate, int *err, cudaStream_t st);
cudaError_t finalise_tc_launch(const TcProdEntry *prods, const TcRowEntry *rows, int nrows, const float4 *acc,
                               int nfreqs, int N, int ninputs, int ks, float2 *results, cudaStream_t st);
// One record of channel averaging (CHANS TO AVG): n output values at dst, each
// the mean of L consecutive values from src (L = 1: a copy, for weights).
// One spectra row of a zoom freq (Mode, mode.cpp:184-196: a zoom band's
// spectrum is its parent recorded band's from a channel offset on): row `zrow`
// of zoom freq `zf` takes input `mrow` of freq `mf` from channel `off`.
struct ZoomRow {
  int zf, zrow, mf, mrow, off;
};
// specz[zf][block][zrow][0 .. Nz) = spec[mf][block][mrow][off .. off + Nz)
// for the nblk blocks of a pass (rows not in the table are left as they are).
cudaError_t zoom_gather_launch(const ZoomRow *rows, int nrows, const float2 *spec, int NIm, int Nm, float2 *specz,
                               int NIz, int Nz, int nblk, cudaStream_t st);

// Multiple phase centres (Core::uvshiftAndAverageBaselineFreq,
// core.cpp:1605-1938): one product row of the FP32 accumulators.  A cross
// product (stride > 0) is rotated by each phase centre's differential delay
// and added at result offset ro + s * stride; an autocorrelation (stride 0)
// is added once.
struct UvEntry {
  long long ro;          // result offset of phase centre 0
  long long acc_index;   // accumulator index (ks = 0 slice)
  int conj;
  int baseline, freq;
  int stride;            // complex floats between phase centres' records; 0: autocorrelation
};
// Per freq: band edge (MHz), channel width (MHz), sideband, channels.
struct UvFreq {
  double lofreq, chanbw;
  int lsb, nchan;
};
// Adds one interval's accumulators into the result array.  delays[bl][s]
// (us): the differential delay of phase centre s on baseline bl; rsl: the
// rotate stride length (the two-level rotator of core.cpp:1690-1766).
cudaError_t uvshift_launch(const UvEntry *ents, int nents, const float2 *acc, int ks, size_t ks_stride, int N,
                           const double *delays, int npc, int maxpc, const UvFreq *freqs, int rsl, float2 *results,
                           cudaStream_t st);
// results_f[first + i] = vals[i], i < n (floats)
cudaError_t copy_floats_launch(const float *vals, long long n, float *results_f, long long first, cudaStream_t st);

// Pulsar binning (core.cpp:803-811, 913-958; Polyco::getBins,
// polyco.cpp:177-224).  One cross product row: inputs a x conj(b) of freq f,
// product p of npol; its bin-b record starts at ro + (b * npol + p) * N
// (scrunched: ro + p * N); fj indexes its (freq, baseline) weight sums.
struct BinEntry {
  long long ro;
  int f, a, b, p, npol, fj;
};
// (freq, baseline stations) of a binned weight sum
struct BinWeightItem {
  int f, s1, s2;
};
// result float index <- the weight sum of item fj, bin b
struct BinWeightOut {
  long long float_index;
  int fj, bin;
};
// One pass of nblk blocks starting at subint block b0: acc[e][bin][c] +=
// spec[f][blk][a][c] * conj(spec[f][blk][b][c]) in block order, the bin of
// (block, channel) from the block's mean pulse phase and the channel's
// dispersion phase offset (dmoff[f][c]).
cudaError_t binned_xmac_launch(const BinEntry *ents, int nents, const float2 *spec, int NI, int N, int nblk, int b0,
                               const double *avgphase, const double *dmoff, const double *binphases, int nbins,
                               float2 *acc, cudaStream_t st);
// The binned baseline weights of one pass, in the reference's order
// (buffered FFT groups, xmac strides, blocks, channels): per bin the sum of
// w1 w2 / nchan over the channels in the bin; scrunched (scrunch != 0), one
// sum of w1 w2 / nchan x the bin's weight over channels of positive-weight bins.
cudaError_t binned_weights_launch(const BinWeightItem *items, int nitems, const float *w, int nblk, int b0, int N,
                                  int nbuf, int xmacstride, const double *avgphase, const double *dmoff,
                                  const double *binphases, const double *binweights, int nbins, int scrunch,
                                  float *wbins, cudaStream_t st);
// The binned records (or their weighted sum when scrunched) and weights into the result array.
cudaError_t binned_finalise_launch(const BinEntry *ents, int nents, const float2 *acc, int N, int nbins, int scrunch,
                                   const double *binweights, const BinWeightOut *wout, int nwout, const float *wbins,
                                   float2 *results, cudaStream_t st);

struct AvgEntry {
  long long src, dst;
  int n, L;
};
cudaError_t average_launch(const AvgEntry *tab, int nent, const float2 *full, float2 *out, cudaStream_t st);
constexpr int kTcInputs = 128;   // inputs per frequency of the tensor-core X-step (the MMA M)

cudaError_t finalise_launch(const ProdEntry *prods, int nprods, const float2 *acc, int ks, size_t ks_stride, int N,
                            const WeightEntry *we, int nw, const float *wacc, float2 *results, cudaStream_t st);

}  // namespace gx
