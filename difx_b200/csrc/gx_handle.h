// The gx_handle behind the C ABI of include/gxcorr.h (host driver state),
// shared by the translation units of the host driver.
#pragma once
#include <cstdint>
#include <deque>
#include <memory>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/gxcorr.h"
#include "gx_dev.h"
#include "gx_host.h"
#include "gx_xstep.h"

struct gx_handle {
  std::string err;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = true;

  std::vector<gx_station_desc> st;
  std::vector<gx_freq_desc> fr;
  std::vector<gx_baseline_desc> bl;
  gx_job_desc jd{};

  gx::DevJob J{};
  int maxnrf = 1, nslots = 1, chunk = 0, ks = 1, xmac_stride = 0, maxprod = 0;
  gx::XmacShape xs{};
  long long rl = 0;                          // result length (averaged layout)
  std::vector<int> blofs, bwofs, acofs, acwofs;
  int avg = 1;                               // CHANS TO AVG
  long long rl_full = 0;                     // the layout at full resolution (the kernels' target)
  std::vector<int> blofs_full, bwofs_full, acofs_full, acwofs_full;
  std::vector<gx::AvgEntry> avgtab;          // full -> averaged records
  gx::AvgEntry *d_avgtab = nullptr;
  float2 *d_full = nullptr;
  std::vector<gx::PcalBand> pcal;            // recorded bands with phase-cal extraction
  gx::PcalBand *d_pcal = nullptr;
  std::vector<float2> pcal_rot;              // shifting extractors' oscillator tables (2 rotlen each)
  float2 *d_pcalrot = nullptr;
  float2 *d_pcalbins = nullptr;              // [chunk][pcal band][bin] partial bin sums
  int pcal_chunks = 0, pcal_maxbins = 0, pcal_per_station = 0;
  // bin sums formed inside the station-block F-step (gx::PcalFuse): station
  // -> first phase-cal band (-1: none), on the device; 0 bins when not offered
  int *d_pcalfirst = nullptr;
  int pcal_fuse_bins = 0;
  std::vector<int> pc_off, pc_ntones;        // [station * GX_MAX_BANDS + band]: result index / tones
  std::vector<std::vector<double>> pc_tone_hz;   // [station * GX_MAX_BANDS + band]: tone frequencies (Hz)
  std::vector<int> pc_maxtones;              // [station]: most tones of a band (0: phase-cal off)
  std::vector<std::vector<int>> band_input;  // [station][band]
  // Zoom freqs (zoom bands, mode.cpp:184-196): every pass gathers their
  // spectra rows from the parent freqs' rows, and the FP32 X-step
  // cross-multiplies them into accumulators of their own.
  int nfmain = 0;                            // freqs [0, nfmain) hold the recorded bands
  std::vector<int> zfreq;                    // zoom ordinal -> freq table index
  int nzchan = 0, nzrows = 0, zks = 1;       // zoom channels, rows per zoom freq (padded), K-split
  gx::XmacShape zxs{};
  std::vector<gx::ZoomRow> zrows;
  std::vector<gx::ProdEntry> zprods;
  size_t zacc_slice = 0;                     // float2 per zoom K-split slice
  // Multiple phase centres (Core::uvshiftAndAverage, core.cpp:1431-1938): the
  // subint runs in uv-shift intervals of blocks; after each, the FP32
  // accumulators are rotated per phase centre and added into the results.
  int maxpc = 1;                             // most phase centres of a scan: records per baseline-freq
  std::vector<gx::UvEntry> uvents;
  std::vector<gx::UvFreq> uvfreqs;
  gx::UvEntry *d_uvents = nullptr;
  gx::UvFreq *d_uvfreqs = nullptr;
  int uv_nint = 0, rsl = 1;                  // intervals per subint at most; rotate stride length
  std::vector<int> bsdofs, bsdofs_full;      // [freq * nbaselines + baseline] shift-decorrelation offsets
  long long bsd_first = 0, bsd_count = 0;    // complex-float range of that section (full layout)
  size_t o_uvdelay = 0, o_bsd = 0;           // in the per-subint table block
  int cur_npc[2] = {1, 1}, cur_M[2] = {0, 0};   // per slot: phase centres of the staged subint's scan, interval blocks
  // Pulsar binning (core.cpp:803-811, 913-958): cross products accumulated
  // per pulse-phase bin by their own kernel, the autocorrelations through the
  // FP32 X-step as usual.
  int nbins = 0, binloop = 1;                // bins (0: no binning); records per baseline-freq
  bool scrunch = false;
  std::vector<gx::BinEntry> binents;
  std::vector<gx::BinWeightItem> binitems;
  std::vector<gx::BinWeightOut> binwout;
  std::vector<gx::ProdEntry> autoprods;      // the autocorrelation rows of prods
  std::vector<gx::WeightEntry> autowents;    // and their weight entries
  gx::BinEntry *d_binents = nullptr;
  gx::BinWeightItem *d_binitems = nullptr;
  gx::BinWeightOut *d_binwout = nullptr;
  gx::ProdEntry *d_autoprods = nullptr;
  gx::WeightEntry *d_autowents = nullptr;
  double *d_binphase = nullptr, *d_binweight = nullptr;
  float2 *d_accb = nullptr;                  // [entry][bin][chan]
  float *d_wbins = nullptr;                  // [item][bin]
  size_t o_avgphase = 0, o_dmoff = 0;        // per-subint tables: mean phase per block, dispersion phase offsets
  std::vector<std::vector<int>> zparent;     // [station][zoom band] parent recorded band
  std::vector<std::vector<int>> acbands;     // [station] total bands (recorded, then zoom) with autocorrelations
  gx::ZoomRow *d_zrows = nullptr;
  gx::ProdEntry *d_zprods = nullptr;
  float2 *d_specz = nullptr, *d_accz = nullptr;
  std::vector<gx::ProdEntry> prods;
  std::vector<gx::TcProdEntry> tcprods;   // sorted by (freq, a)
  std::vector<gx::TcRowEntry> tcrows;
  std::vector<gx::WeightEntry> wents;
  std::vector<int2> pairs;
  int xstep = 0;                   // X-step form in use (GX_XSTEP_AUTO resolved at open)
  bool tc = false, hilo = false;   // tensor-core X-step (split FP16 product)
  float tc_scale0 = 1.0f;          // default power-of-two operand scale
  float *d_scale = nullptr;        // [freq][128][nchan] operand scales
  gx::TcProdEntry *d_tcprods = nullptr;
  gx::TcRowEntry *d_tcrows = nullptr;
  int *d_err = nullptr;            // kernel status (bounded waits that expired)
  int *h_err = nullptr;            // pinned copies of *d_err after each subint, one per slot
  cudaStream_t last_stream = nullptr;  // stream of the last gx_subint_device

  gx::DevStation *d_st = nullptr;
  float2 *d_tw = nullptr, *d_spec = nullptr, *d_acc = nullptr, *d_results = nullptr, *d_spec1 = nullptr;
  float *d_w = nullptr, *d_wacc = nullptr, *d_w1 = nullptr;
  gx::BlockParam *d_bp = nullptr, *d_bp1 = nullptr;
  size_t acc_slice = 0;  // float2 per K-split slice
  int2 *d_pairs = nullptr;
  // INTERLACEDVDIF stations: per-band weight rows after the station rows, and
  // the per-(station, block, band) frames their EDV4 masks blank
  bool interlaced_any = false;
  int nwrows = 0;
  unsigned long long *d_bandmask = nullptr;
  gx::ProdEntry *d_prods = nullptr;
  gx::WeightEntry *d_went = nullptr;
  // Per-subint tables, one block written on the host (pinned) and copied to
  // the device with one copy per subint:
  //   SubintClock | datalen[nst] (int64) | data pointers[nst] | interp[nst][3]
  //   (double) | control words[nst][ctrlstride] (int32)
  // Two slots, so that gx_subint_async can stage and upload one subint while
  // the previous one computes; every other entry point uses slot 0.
  static constexpr int kSlots = 2;
  int slot = 0;                    // slot of the subint being staged and enqueued
  unsigned char *h_sub[kSlots] = {}, *d_sub = nullptr;
  size_t sub_bytes = 0, o_len = 0, o_ptr = 0, o_interp = 0, o_ctrl = 0;
  // data ring subints (gx_ring_subint_device): [nstations][3] span delays in
  // the block, and the ring whose walk runs right after the block's copy
  size_t o_ring = 0;
  struct gx_ring *ring_req = nullptr;
  int ring_scan = 0, ring_sec = 0, ring_ns = 0;
  cudaEvent_t ev_sub[kSlots] = {}; // recorded after a block's copy (host may rewrite it once passed)
  bool ev_sub_pending[kSlots] = {};
  int ctrlstride = 0;
  bool untimed = false;            // no events recorded (batch runs, CUDA-graph capture)
  std::vector<uint8_t *> d_data[kSlots];     // host-buffer entry points: device copies of the station data
  std::vector<int64_t> data_cap[kSlots];     // usable bytes of d_data[k][s]
  std::vector<long long> data_alloc[kSlots]; // allocated bytes of d_data[k][s]
  cudaStream_t copy_stream = nullptr;        // uploads of gx_subint_async
  cudaEvent_t ev_copied[kSlots] = {}, ev_done[kSlots] = {};
  std::deque<int> inflight;                  // slots of gx_subint_async calls not yet waited for

  gx::SubintArrays last{};
  bool have_last = false;
  std::vector<cudaEvent_t> evs;  // pairs per launch: [start, end]
  std::vector<int> ev_stage;
  int launches = 0;

  std::vector<int> sta_acoff, sta_acw;   // [station * GX_MAX_BANDS + recorded band]: autocorrelation record, weight (-1: none)
  struct gx_kurtosis_state *kurt = nullptr;   // gx_set_kurtosis
  int xvar = 0;                              // FP32 X-step launch variant (gx_set_tiles)
  std::unique_ptr<HostModel> model;  // only for gx_open_input
  std::unique_ptr<gx::JobMeta> meta; // only for gx_open_input
  std::vector<gx::DevStation> dst;   // host copy of the per-station device constants

  long long dev_bytes = 0;           // device memory held by the handle

  template <typename T>
  cudaError_t dalloc(T **p, size_t bytes)
  {
    cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), bytes);
    if (e == cudaSuccess) dev_bytes += (long long)bytes;
    return e;
  }

  gx_status fail(gx_status s, const std::string &m)
  {
    err = m;
    return s;
  }
  gx_status cuda(cudaError_t e, const char *what)
  {
    if (e == cudaSuccess) return GX_OK;
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return GX_ERR_CUDA;
  }
};

#define CKR(h, call)                                         \
  do {                                                       \
    gx_status _s = (h)->cuda((call), #call);                 \
    if (_s != GX_OK) return _s;                              \
  } while (0)

// local freq index of job freq f on baseline b (-1: not correlated)
int gx_bl_localfreq(const gx_baseline_desc &b, int f);

// The two halves of one subint, shared with the batch runner: the host half
// writes the subint's tables into the handle's pinned block; the device half
// enqueues the tables' copy and all kernels on `st` without waiting on the
// host (capturable into a CUDA graph when h->untimed is set).
gx_status gx_stage_subint(gx_handle *h, const gx_subint_desc *sub, const uint8_t *const *devdata);
gx_status gx_enqueue_subint(gx_handle *h, float2 *dev_results, cudaStream_t st);
// The ring walk of h->ring_req over the copied tables (gx_ring.cu).
gx_status gx_ring_enqueue_control(struct gx_ring *r, gx_handle *h, cudaStream_t st);
// Spectral kurtosis of the recorded bands (gx_monitor.cu): zero the sums,
// add one pass of spectra, finish the subint.
gx_status gx_kurtosis_begin(gx_handle *h, cudaStream_t st);
gx_status gx_kurtosis_pass(gx_handle *h, int nblk, cudaStream_t st);
gx_status gx_kurtosis_end(gx_handle *h, cudaStream_t st);
void gx_kurtosis_free(struct gx_kurtosis_state *k);
