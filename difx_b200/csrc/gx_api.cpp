// gxcorr host driver: the C ABI of include/gxcorr.h.
//
// gx_open derives, from a gx_job_desc, what Configuration::getMode and
// Configuration::populateResultLengths derive from the .input tables
// (mpifxcorr/src/configuration.cpp:932-998, 2348-2630, setStrides 2701-2734,
// calcstridelength 38-50, calcgoodxmacstridelength 2653-2698), allocates the
// device buffers once, and precomputes the tables that map the X-step
// accumulators onto the Core result array.  gx_subint[_device] then runs one
// Core slot: F-step and X-step over chunks of FFT blocks, then one
// finalising pass writing the result array.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/gxcorr.h"
#include "gx_dev.h"
#include "gx_xstep.h"
#include "gx_host.h"
#include "gx_plan.h"
#include "gx_handle.h"
#include "gx_fft16.h"

using namespace gx;

namespace {

constexpr double kTwoPi = 6.283185307179586476925286766559;   // TWO_PI of the generic architecture

int stride_length(int n)  // calcstridelength, configuration.cpp:38-50
{
  if (n <= 16) return n;
  for (unsigned int g = (unsigned int)std::sqrt(n + 0.1);; --g)
    if (n % g == 0) return n / (int)g;
}


long gcdl(long a, long b)
{
  while (b) { long t = a % b; a = b; b = t; }
  return a;
}

}  // namespace


static void free_all(gx_handle *h)
{
  if (h->device < 0) return;
  void *ptrs[] = {h->d_st, h->d_tw, h->d_spec, h->d_acc, h->d_results, h->d_spec1, h->d_w, h->d_wacc, h->d_w1,
                  h->d_pairs, h->d_prods, h->d_went, h->d_sub, h->d_bp, h->d_bp1, h->d_scale, h->d_tcprods,
                  h->d_tcrows, h->d_err, h->d_full, h->d_avgtab, h->d_pcal, h->d_pcalbins, h->d_zrows,
                  h->d_zprods, h->d_specz, h->d_accz, h->d_uvents, h->d_uvfreqs, h->d_binents, h->d_binitems,
                  h->d_binwout, h->d_autoprods, h->d_autowents, h->d_binphase, h->d_binweight, h->d_accb,
                  h->d_wbins, h->d_pcalrot, h->d_pcalfirst};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (h->h_err) cudaFreeHost(h->h_err);
  h->h_err = nullptr;
  for (int k = 0; k < gx_handle::kSlots; k++) {
    if (h->h_sub[k]) cudaFreeHost(h->h_sub[k]);
    h->h_sub[k] = nullptr;
    if (h->ev_sub[k]) cudaEventDestroy(h->ev_sub[k]);
    if (h->ev_copied[k]) cudaEventDestroy(h->ev_copied[k]);
    if (h->ev_done[k]) cudaEventDestroy(h->ev_done[k]);
    h->ev_sub[k] = h->ev_copied[k] = h->ev_done[k] = nullptr;
    for (auto p : h->d_data[k])
      if (p) cudaFree(p);
  }
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  h->copy_stream = nullptr;
  for (auto e : h->evs) cudaEventDestroy(e);
  h->evs.clear();
  if (h->stream && h->own_stream) cudaStreamDestroy(h->stream);
}

int gx_bl_localfreq(const gx_baseline_desc &b, int f)
{
  int r = -1;
  for (int j = 0; j < b.nfreqs; j++)
    if (b.freq[j] == f) r = j;
  return r;
}

static int bl_localfreq(const gx_baseline_desc &b, int f) { return gx_bl_localfreq(b, f); }

static gx_status setup(gx_handle *h)
{
  const gx_job_desc &d = h->jd;
  if (d.nstations < 1 || !d.stations || d.nfreqs < 1 || !d.freqs || d.nbaselines < 0)
    return h->fail(GX_ERR_ARG, "job descriptor: missing stations or freqs");
  if (d.fringe_rotation_order < 0 || d.fringe_rotation_order > 2)
    return h->fail(GX_ERR_UNSUPPORTED, "FRINGE ROTN ORDER must be 0, 1 or 2");
  const gx_station_desc &s0 = d.stations[0];
  if (d.fringe_rotation_order == 0 && s0.is_complex)   // as the reference (mode.cpp:1131-1134)
    return h->fail(GX_ERR_UNSUPPORTED, "post-F (0th order) fringe rotation is not supported for complex sampled data");
  for (int s = 0; s < d.nstations; s++) {
    const gx_station_desc &x = d.stations[s];
    if (x.nbits != s0.nbits || x.is_complex != s0.is_complex || x.framebytes != s0.framebytes ||
        x.nbands != s0.nbands)
      return h->fail(GX_ERR_UNSUPPORTED, "all datastreams must share bits, sampling, frame size and band count");
    if (x.nrecfreqs < 1 || x.nrecfreqs > GX_MAX_LOCAL_FREQS || x.nbands < 1 || x.nbands > GX_MAX_BANDS)
      return h->fail(GX_ERR_ARG, "datastream freq/band count out of range");
    for (int i = 0; i < x.nrecfreqs; i++)
      if (x.recfreq[i] < 0 || x.recfreq[i] >= d.nfreqs) return h->fail(GX_ERR_ARG, "REC FREQ INDEX out of range");
    for (int b = 0; b < x.nbands; b++)
      if (x.band_localfreq[b] < 0 || x.band_localfreq[b] >= x.nrecfreqs)
        return h->fail(GX_ERR_ARG, "REC BAND INDEX out of range");
    if (x.nzoomfreqs < 0 || x.nzoomfreqs > GX_MAX_LOCAL_FREQS || x.nzoombands < 0 ||
        x.nbands + x.nzoombands > GX_MAX_BANDS)
      return h->fail(GX_ERR_ARG, "datastream zoom freq/band count out of range");
    for (int i = 0; i < x.nzoomfreqs; i++)
      if (x.zoomfreq[i] < 0 || x.zoomfreq[i] >= d.nfreqs) return h->fail(GX_ERR_ARG, "ZOOM FREQ INDEX out of range");
    for (int b = 0; b < x.nzoombands; b++)
      if (x.zoomband_localfreq[b] < 0 || x.zoomband_localfreq[b] >= x.nzoomfreqs)
        return h->fail(GX_ERR_ARG, "ZOOM BAND INDEX out of range");
  }
  if (s0.nbits != 1 && s0.nbits != 2 && s0.nbits != 4 && s0.nbits != 8)
    return h->fail(GX_ERR_UNSUPPORTED, "QUANTISATION BITS must be 1, 2, 4 or 8");
  // phase centres: the result records of a baseline-freq are repeated for the
  // most phase centres of any scan (configuration.cpp:2366-2373)
  h->maxpc = 1;
  if (h->model)
    for (const auto &sc : h->model->scans) h->maxpc = std::max(h->maxpc, sc.numphasecentres);
  // pulsar binning: records per bin unless scrunched (configuration.cpp:2455-2470)
  h->nbins = 0;
  h->binloop = 1;
  h->scrunch = false;
  if (h->meta && h->meta->pulsar) {
    h->nbins = h->meta->pulsar->nbins;
    h->scrunch = h->meta->pulsar->scrunch;
    h->binloop = h->scrunch ? 1 : h->nbins;
  }
  // the recorded freqs share bandwidth and channel count and come first in the
  // freq table: their spectra and accumulators are slabs [0, nfmain)
  const gx_freq_desc &f0 = d.freqs[s0.recfreq[0]];
  h->nfmain = 0;
  for (int s = 0; s < d.nstations; s++)
    for (int i = 0; i < d.stations[s].nrecfreqs; i++) {
      const gx_freq_desc &fq = d.freqs[d.stations[s].recfreq[i]];
      if (fq.nchan != f0.nchan || fq.bw_mhz != f0.bw_mhz)
        return h->fail(GX_ERR_UNSUPPORTED, "all recorded freqs must share bandwidth and channel count");
      h->nfmain = std::max(h->nfmain, d.stations[s].recfreq[i] + 1);
    }
  const int cplx = s0.is_complex ? 1 : 0;
  const int bits_ts = s0.nbands * s0.nbits * (cplx ? 2 : 1);
  // whole bytes per time sample, or a whole number of time samples per byte
  // (mark5access sample granularity 8 / bits, mk5mode.cpp:100, 118-141)
  if (bits_ts % 8 != 0 && 8 % bits_ts != 0)
    return h->fail(GX_ERR_UNSUPPORTED, "a time sample must fill whole bytes or divide a byte");
  // complex samples narrower than a byte: the reference's granularity erase
  // indexes its complex unpack arrays as floats (mk5mode.cpp:118-141 over the
  // aliased arrays of mode.cpp:152-154) and zeroes components inside the window
  if (bits_ts < 8 && cplx)
    return h->fail(GX_ERR_UNSUPPORTED, "complex time samples narrower than a byte are not implemented");
  const int payload = s0.framebytes - 32;
  if (payload <= 0 || (payload * 8) % bits_ts != 0 || payload % 8 != 0)
    return h->fail(GX_ERR_ARG, "DATA FRAME SIZE is not a whole number of time samples");

  DevJob &J = h->J;
  J.deltapol_any = 0;
  J.nstations = d.nstations;
  J.nbands = s0.nbands;
  J.nbits = s0.nbits;
  J.cplx = cplx;
  J.framebytes = s0.framebytes;
  J.framesamples = payload * 8 / (s0.nbits * s0.nbands);
  if (cplx) J.framesamples /= 2;
  J.bps_num = bits_ts >= 8 ? bits_ts / 8 : 1;
  J.bps_den = bits_ts >= 8 ? 1 : 8 / bits_ts;
  J.nchan = f0.nchan;
  J.fftlen = cplx ? f0.nchan : 2 * f0.nchan;
  if (J.fftlen & (J.fftlen - 1)) return h->fail(GX_ERR_UNSUPPORTED, "FFT length must be a power of two");
  if (J.fftlen < 16 || J.fftlen > 8192) return h->fail(GX_ERR_UNSUPPORTED, "FFT length must be in [16, 8192]");
  J.stride = d.array_stride > 0 ? d.array_stride : stride_length(f0.nchan);
  if (J.fftlen % J.stride) return h->fail(GX_ERR_ARG, "array stride does not divide the FFT length");
  J.nfr = J.fftlen / J.stride;
  if (J.stride & (J.stride - 1)) return h->fail(GX_ERR_UNSUPPORTED, "array stride must be a power of two");
  J.fringe_order = d.fringe_rotation_order;
  J.lgstride = 0;
  while ((1 << J.lgstride) < J.stride) J.lgstride++;
  J.half = (cplx ? 2 * J.nfr : J.nfr) / 2;
  J.unpacksamples = cplx ? f0.nchan : 2 * f0.nchan;
  J.sampletime = 1.0 / (2.0 * f0.bw_mhz);
  if (cplx) J.sampletime *= 2.0;
  J.bw = f0.bw_mhz;
  J.nfreqs = h->nfmain;
  {
    double ffttime = 1000.0 * f0.nchan / f0.bw_mhz;
    double b = d.subint_ns / ffttime;
    J.blocks_per_send = (int)(b + 0.5);
    if (std::fabs(b - J.blocks_per_send) > 1e-9 || J.blocks_per_send < 1)
      return h->fail(GX_ERR_ARG, "SUBINT NANOSECONDS is not a whole number of FFT blocks");
  }
  J.flaglen = J.blocks_per_send / 30 + (J.blocks_per_send % 30 ? 1 : 0);
  if ((J.unpacksamples + J.framesamples - 1) / J.framesamples + 1 > kMaxFramesPerBlock)
    return h->fail(GX_ERR_UNSUPPORTED, "an FFT block spans too many frames");

  // xmac stride (does not change results; reported for layout parity)
  {
    int g = 0;
    for (int j = 0; j < d.nbaselines; j++)
      for (int k = 0; k < d.baselines[j].nfreqs; k++) {
        int n = d.freqs[d.baselines[j].freq[k]].nchan;
        g = g ? (int)gcdl(g, n) : n;
      }
    if (d.xmac_stride > 0) h->xmac_stride = d.xmac_stride;
    else {
      double err = 1e12;
      for (int guess = g; guess > 0; --guess) {
        if (g % guess) continue;
        double e = std::fabs((double)guess - 150);
        if (e < err) { err = e; h->xmac_stride = guess; }
      }
    }
  }

  // spectra rows: every (station, band) of a freq gets one input row
  std::vector<int> count(d.nfreqs, 0);
  h->band_input.assign(d.nstations, std::vector<int>(s0.nbands, -1));
  h->maxnrf = 1;
  std::vector<DevStation> dst(d.nstations);
  for (int s = 0; s < d.nstations; s++) {
    const gx_station_desc &x = d.stations[s];
    DevStation &D = dst[s];
    memset(&D, 0, sizeof(D));
    D.nrecfreqs = x.nrecfreqs;
    if (x.nrecfreqs > h->maxnrf) h->maxnrf = x.nrecfreqs;
    for (int i = 0; i < x.nrecfreqs; i++) {
      const gx_freq_desc &fq = d.freqs[x.recfreq[i]];
      double lo = fq.freq_mhz;
      if (std::fabs(lo - (int)(lo + 0.5)) > (double)0.000000001f) D.fractional_lo = 1;
      if (x.clock_offset_delta_us[i] != 0.0) D.deltapol = 1;
      D.lofreq[i] = (cplx && fq.lower_sideband) ? -lo : lo;
      D.lsb[i] = fq.lower_sideband ? 1 : 0;
      D.freq_index[i] = x.recfreq[i];
      D.clk[i] = x.clock_offset_us[i];
      D.clkdelta[i] = x.clock_offset_delta_us[i];
      D.looff[i] = x.lo_offset_hz[i];
    }
    for (int b = 0; b < x.nbands; b++) {
      int f = x.recfreq[x.band_localfreq[b]];
      D.band_localfreq[b] = x.band_localfreq[b];
      D.band_input[b] = count[f]++;
      h->band_input[s][b] = D.band_input[b];
    }
    for (int b = 0; b < x.nbands; b++) D.band_polb[b] = (D.deltapol && x.band_pol[b] != 'R') ? 1 : 0;
    if (D.deltapol) J.deltapol_any = 1;
  }
  // INTERLACEDVDIF stations: one weight row per band after the station rows
  h->interlaced_any = false;
  h->nwrows = d.nstations;
  for (int s = 0; s < d.nstations; s++) {
    if (!d.stations[s].interlaced) continue;
    if (d.stations[s].nbands > 30)   // the blanker's int-width thread masks (format_vdif.c:8509, 8530)
      return h->fail(GX_ERR_UNSUPPORTED, "INTERLACEDVDIF with more than 30 bands is not implemented");
    h->interlaced_any = true;
    dst[s].interlaced = 1;
    dst[s].wrow0 = h->nwrows;
    h->nwrows += d.stations[s].nbands;
  }
  int ni = 0;
  for (int f = 0; f < d.nfreqs; f++) ni = count[f] > ni ? count[f] : ni;
  if (d.xstep < GX_XSTEP_FP32 || d.xstep > GX_XSTEP_AUTO) return h->fail(GX_ERR_ARG, "unknown xstep");
  h->xstep = d.xstep;
  if (d.xstep == GX_XSTEP_AUTO) {
    const char *e = getenv("GX_XSTEP_AUTO_MIN_INPUTS");
    const int nmin = e ? atoi(e) : 48;
    h->xstep = (ni >= nmin && ni <= kTcInputs && J.nchan >= 2 && h->maxpc == 1 && h->nbins == 0)
                   ? GX_XSTEP_TC_FP16_HILO : GX_XSTEP_FP32;
  }
  if (h->maxpc > 1 && h->xstep != GX_XSTEP_FP32)
    return h->fail(GX_ERR_UNSUPPORTED, "multiple phase centres are implemented with the FP32 X-step only");
  if (h->nbins > 0) {
    if (h->xstep != GX_XSTEP_FP32)
      return h->fail(GX_ERR_UNSUPPORTED, "pulsar binning is implemented with the FP32 X-step only");
    if (h->maxpc > 1) return h->fail(GX_ERR_UNSUPPORTED, "pulsar binning with multiple phase centres is not implemented");
    if (h->interlaced_any) return h->fail(GX_ERR_UNSUPPORTED, "pulsar binning of INTERLACEDVDIF is not implemented");
  }
  h->tc = h->xstep != GX_XSTEP_FP32;
  h->hilo = h->xstep == GX_XSTEP_TC_FP16_HILO;
  if (h->tc) {
    if (ni > kTcInputs)
      return h->fail(GX_ERR_UNSUPPORTED, "the tensor-core X-step takes at most 128 inputs (station bands) per freq");
    if (J.nchan < 2) return h->fail(GX_ERR_UNSUPPORTED, "the tensor-core X-step needs at least 2 channels");
    J.ninputs = ni;   // the X-step reads the rows up to 128 beyond these as zeros
  } else {
    h->xs = xmac_shape(ni);
    J.ninputs = h->xs.nsuper * h->xs.ST;
  }
  h->xs = xmac_shape(J.ninputs);
  h->dst = dst;

  // Core result layout (populateResultLengths, one phase centre, no bins, no averaging)
  const int nbl = d.nbaselines;
  auto freq_used = [&](int f) {
    for (int j = 0; j < nbl; j++)
      if (bl_localfreq(d.baselines[j], f) >= 0) return true;
    return false;
  };
  h->maxprod = 0;
  for (int j = 0; j < nbl; j++)
    for (int k = 0; k < d.baselines[j].nfreqs; k++) {
      if (d.baselines[j].npolprod[k] > h->maxprod) h->maxprod = d.baselines[j].npolprod[k];
      if (d.baselines[j].npolprod[k] < 1 || d.baselines[j].npolprod[k] > GX_MAX_POLPRODUCTS)
        return h->fail(GX_ERR_ARG, "POL PRODUCTS out of range");
    }
  const int bpa = h->maxprod > 2 ? 2 : 1;
  const bool writecross = d.write_autocorrs && h->maxprod > 2;

  // Zoom freqs (configuration.cpp:1701-1753, 2774-2880; mode.cpp:184-196,
  // 379-391): a station's zoom freq is a channel range of the recorded freq
  // that contains it (the last one, as Configuration's search leaves it), from
  // the channel offset Configuration computes with the first recorded freq's
  // channel width; a zoom band takes the parent band of its polarisation.
  // Each zoom freq gets spectra rows of its own: one per zoom band, plus the
  // parent's cross-polarisation partner where the zoom freq lacks it (its
  // cross-pol autocorrelation is a slice of the parent's).  Zoom freqs follow
  // the recorded freqs in the freq table and share one channel count.
  h->zfreq.clear();
  h->zrows.clear();
  h->nzchan = 0;
  std::vector<int> zord(d.nfreqs, -1), zcount;
  // [station][zoom band]: parent recorded band, row, row of the cross-pol partner (-1: none)
  std::vector<std::vector<int>> zparent(d.nstations), zrow(d.nstations), zpartner(d.nstations);
  auto partner_of = [&](const gx_station_desc &x, int b, int *i0p = nullptr, int *i1p = nullptr) {
    // the two bands of b's local freq in band order (mode.cpp:1124-1129, 1333-1351)
    int i0 = -1, i1 = -1;
    for (int q = 0; q < x.nbands; q++)
      if (x.band_localfreq[q] == x.band_localfreq[b]) {
        if (i0 < 0) i0 = q;
        else if (i1 < 0) i1 = q;
      }
    if (i0p) *i0p = i0;
    if (i1p) *i1p = i1;
    return (b == i0) ? i1 : ((b == i1) ? i0 : -1);
  };
  for (int s = 0; s < d.nstations; s++) {
    const gx_station_desc &x = d.stations[s];
    zparent[s].assign(x.nzoombands, -1);
    zrow[s].assign(x.nzoombands, -1);
    zpartner[s].assign(x.nzoombands, -1);
    if (x.nzoombands == 0) continue;
    std::vector<int> zpar(x.nzoomfreqs, -1), zoff(x.nzoomfreqs, 0);
    const gx_freq_desc &r0 = d.freqs[x.recfreq[0]];
    for (int j = 0; j < x.nzoomfreqs; j++) {
      const int fz = x.zoomfreq[j];
      if (fz < h->nfmain)
        return h->fail(GX_ERR_UNSUPPORTED, "zoom freqs must follow every recorded freq in the freq table");
      const gx_freq_desc &zq = d.freqs[fz];
      double zlo = zq.freq_mhz, zhi = zq.freq_mhz + zq.bw_mhz;
      if (zq.lower_sideband) { zlo -= zq.bw_mhz; zhi -= zq.bw_mhz; }
      for (int k = 0; k < x.nrecfreqs; k++) {
        const gx_freq_desc &pq = d.freqs[x.recfreq[k]];
        double plo = pq.freq_mhz, phi = pq.freq_mhz + pq.bw_mhz;
        if (pq.lower_sideband) { plo -= pq.bw_mhz; phi -= pq.bw_mhz; }
        if (zhi <= phi && zlo >= plo) {
          zpar[j] = k;
          zoff[j] = (int)(((zlo - plo) / r0.bw_mhz) * r0.nchan + 0.5);
        }
      }
      if (zpar[j] < 0) return h->fail(GX_ERR_ARG, "a zoom freq does not fit into any recorded freq");
      const gx_freq_desc &pq = d.freqs[x.recfreq[zpar[j]]];
      if (std::fabs(zq.bw_mhz / zq.nchan - pq.bw_mhz / pq.nchan) > 0.000000001)   // Mode::TINY
        return h->fail(GX_ERR_ARG, "a zoom freq's channel width differs from its parent's");
      if (zq.lower_sideband != pq.lower_sideband)
        return h->fail(GX_ERR_UNSUPPORTED, "a zoom freq of the other sideband than its parent");
      if (zoff[j] < 0 || zoff[j] + zq.nchan > pq.nchan)
        return h->fail(GX_ERR_UNSUPPORTED, "a zoom freq's channels run past its parent's");
      if (zq.nchan < 2 || zq.nchan % 2) return h->fail(GX_ERR_UNSUPPORTED, "zoom freqs need an even channel count");
      if (h->nzchan == 0) h->nzchan = zq.nchan;
      else if (zq.nchan != h->nzchan) return h->fail(GX_ERR_UNSUPPORTED, "zoom freqs with different channel counts");
      if (zord[fz] < 0) {
        zord[fz] = (int)h->zfreq.size();
        h->zfreq.push_back(fz);
        zcount.push_back(0);
      }
    }
    for (int b = 0; b < x.nzoombands; b++) {
      const int j = x.zoomband_localfreq[b];
      int parent = -1, nmatch = 0;
      for (int l = 0; l < x.nbands; l++)
        if (x.band_localfreq[l] == zpar[j] && x.band_pol[l] == x.zoomband_pol[b]) { parent = l; nmatch++; }
      if (nmatch == 0) return h->fail(GX_ERR_ARG, "a zoom band's polarisation is not recorded in its parent freq");
      if (nmatch > 1) return h->fail(GX_ERR_UNSUPPORTED, "a zoom band's parent freq records its polarisation twice");
      const int z = zord[x.zoomfreq[j]];
      zparent[s][b] = parent;
      zrow[s][b] = zcount[z]++;
      h->zrows.push_back(ZoomRow{z, zrow[s][b], x.recfreq[zpar[j]], h->band_input[s][parent], zoff[j]});
    }
    if (writecross)
      for (int b = 0; b < x.nzoombands; b++) {
        const int pp = partner_of(x, zparent[s][b]);
        if (pp < 0) continue;
        const int j = x.zoomband_localfreq[b];
        for (int b2 = 0; b2 < x.nzoombands; b2++)
          if (x.zoomband_localfreq[b2] == j && zparent[s][b2] == pp) zpartner[s][b] = zrow[s][b2];
        if (zpartner[s][b] < 0) {   // the partner's channels as a row of their own
          const int z = zord[x.zoomfreq[j]];
          zpartner[s][b] = zcount[z]++;
          h->zrows.push_back(ZoomRow{z, zpartner[s][b], x.recfreq[zpar[j]], h->band_input[s][pp], zoff[j]});
        }
      }
  }
  if (!h->zfreq.empty() && h->maxpc > 1)
    return h->fail(GX_ERR_UNSUPPORTED, "zoom bands with multiple phase centres are not implemented");
  if (!h->zfreq.empty() && h->nbins > 0)
    return h->fail(GX_ERR_UNSUPPORTED, "zoom bands with pulsar binning are not implemented");
  {
    int nzi = 0;
    for (int c : zcount) nzi = std::max(nzi, c);
    h->zxs = xmac_shape(std::max(1, nzi));
    h->nzrows = h->zxs.nsuper * h->zxs.ST;
  }
  // freq of total band k of a station (recorded bands, then zoom bands: getDTotalFreqIndex)
  auto total_freq = [&](const gx_station_desc &x, int k) {
    return k < x.nbands ? x.recfreq[x.band_localfreq[k]] : x.zoomfreq[x.zoomband_localfreq[k - x.nbands]];
  };
  // Autocorrelations are kept for bands whose freq, or an equivalent one (same
  // band edge, bandwidth, sideband-adjusted, and channel count), a baseline
  // correlates (configuration.cpp:2299-2325; core.cpp:1273-1301)
  auto ac_used = [&](int f) {
    if (freq_used(f)) return true;
    const gx_freq_desc &a = d.freqs[f];
    for (int k = 0; k < d.nfreqs; k++) {
      const gx_freq_desc &b = d.freqs[k];
      double fd = a.freq_mhz - b.freq_mhz;
      if (a.lower_sideband) fd -= a.bw_mhz;
      if (b.lower_sideband) fd += b.bw_mhz;
      const int aa = a.chans_to_average > 1 ? a.chans_to_average : 1, ba = b.chans_to_average > 1 ? b.chans_to_average : 1;
      if (std::fabs(a.bw_mhz - b.bw_mhz) < 0.000000001 && std::fabs(fd) < 0.000000001 && a.nchan == b.nchan &&
          aa == ba && freq_used(k))
        return true;
    }
    return false;
  };
  // the total bands of a station with autocorrelations in the result, in order
  auto ac_bands = [&](int s) {
    const gx_station_desc &x = d.stations[s];
    std::vector<int> v;
    for (int k = 0; k < x.nbands + x.nzoombands; k++)
      if (ac_used(total_freq(x, k))) v.push_back(k);
    return v;
  };
  h->zparent = zparent;
  h->acbands.resize(d.nstations);
  for (int s = 0; s < d.nstations; s++) h->acbands[s] = ac_bands(s);
  // CHANS TO AVG (core.cpp:1819-1869, mode.cpp:1376-1401): one averaging length
  // per job, dividing the channel count
  int avg = 1;
  for (int f = 0; f < d.nfreqs; f++) {
    const int a = d.freqs[f].chans_to_average > 1 ? d.freqs[f].chans_to_average : 1;
    if (f == 0) avg = a;
    else if (a != avg) return h->fail(GX_ERR_UNSUPPORTED, "freqs with different CHANS TO AVG");
    if (d.freqs[f].nchan % a) return h->fail(GX_ERR_UNSUPPORTED, "CHANS TO AVG does not divide NUM CHANNELS");
  }
  h->avg = avg;
  // Phase-cal tones per recorded band (configuration.cpp:1754-1835: integer
  // Hz, PHASE CAL DIVISOR 1) and the extractor the reference would pick
  // (PCal::getNew, pcal.cpp:191-260; the implicit-shift ones are built)
  std::vector<std::vector<int>> pc_ntones(d.nstations);
  h->pcal.clear();
  h->pcal_rot.clear();
  h->pc_tone_hz.assign((size_t)d.nstations * GX_MAX_BANDS, {});
  h->pc_maxtones.assign(d.nstations, 0);
  for (int s = 0; s < d.nstations; s++) {
    const gx_station_desc &x = d.stations[s];
    if (x.phase_cal_interval_hz <= 0) continue;
    const long long interval = x.phase_cal_interval_hz, base = x.phase_cal_base_hz;
    pc_ntones[s].assign(x.nbands, 0);
    for (int b = 0; b < x.nbands; b++) {
      const gx_freq_desc &fq = d.freqs[x.recfreq[x.band_localfreq[b]]];
      const double lofreq = fq.freq_mhz, bw = fq.bw_mhz;
      const double stepmhz = interval * 1e-6;
      long long harmonic = (long long)((lofreq - base * 1e-6) / stepmhz);
      double tonefreq = harmonic * stepmhz + base * 1e-6;
      int n = 0;
      long long offset = -1;
      if (fq.lower_sideband) {
        if (tonefreq >= lofreq) { tonefreq -= stepmhz; harmonic -= 1; }
        if (tonefreq >= lofreq - bw)
          while (tonefreq - n * stepmhz >= lofreq - bw) n++;
        if (n > 0) offset = (long long)(1e6 * lofreq) - harmonic * interval;
      } else {
        if (tonefreq <= lofreq) { tonefreq += stepmhz; harmonic += 1; }
        if (tonefreq <= lofreq + bw)
          while (tonefreq + n * stepmhz <= lofreq + bw) n++;
        if (n > 0) offset = harmonic * interval - (long long)(1e6 * lofreq);
      }
      // tone frequencies (configuration.cpp:1784-1786, 1818-1820) and the most per band
      std::vector<double> &tf = h->pc_tone_hz[(size_t)s * GX_MAX_BANDS + b];
      for (int k = 0; k < n; k++)
        tf.push_back((double)((fq.lower_sideband ? harmonic - k : harmonic + k) * interval) + (double)base);
      h->pc_maxtones[s] = std::max(h->pc_maxtones[s], n);
      if (n == 0) {        // no tone in the band: one zero placeholder at 0 Hz
        n = 1;
        tf.push_back(0.0);
      }
      pc_ntones[s][b] = n;
      PcalBand P{};
      P.station = s;
      P.band = b;
      P.ntones = n;
      P.nbins = 0;
      P.nextract = n;
      if (offset >= 0) {
        // the extractor PCal::getNew picks (pcal.cpp:191-260): offset and
        // spacing periods No and Np (No at least the 1 MHz resolution,
        // PCal::setMinFrequencyResolution, mode.cpp:403), tones per PCal::calcNumTones
        const long long bwhz = (long long)(1e6 * bw);
        const long long fs = cplx ? bwhz : 2 * bwhz;
        long long No = fs / gcdl(fs, offset);
        const long long Np = fs / gcdl(fs, interval);
        while (fs / (2 * No) > 1000000) No *= 2;
        int nt = 0;   // PCal::calcNumTones (pcal.cpp:317-335): tones in [offset, bw], a DC tone and a top-edge one counted once
        long long ftone = offset;
        while (ftone <= bwhz) {
          nt++;
          ftone += interval;
        }
        if (offset == 0 && ftone - interval == bwhz) nt--;
        long long nb = 0;
        if (nt == 0) {
          nb = 0;   // PCalExtractorDummy: zeros
        } else if (!cplx && offset == 0) {
          // PCalExtractorTrivial (pcal.cpp:427-575): bins of the spacing period, tone i at bin (i + 1) step
          nb = fs / gcdl(fs, interval);
          P.step = (int)(interval / gcdl(fs, interval));
          P.offset_bin = P.step;
          P.nextract = nt - 1;
        } else if (No % Np == 0) {
          // the implicit-shift extractors (pcal.cpp:1032-1222, 1419-1600)
          nb = fs / gcdl(fs, offset);
          while (fs / (2 * nb) > 1000000) nb *= 2;
          P.step = (int)std::floor((double)nb * (double)interval / (double)fs);
          P.offset_bin = (int)std::floor((double)nb * (double)offset / (double)fs);
          P.nextract = nt;
        } else {
          // the shifting extractors (pcal.cpp:583-800 real, 806-1025 complex): the
          // samples mixed down by the offset with an FP32 oscillator table, bins
          // of the spacing period, tone i at bin i step
          nb = fs / gcdl(fs, interval);
          if (cplx)
            while (fs / (2 * nb) > 1000000) nb *= 2;
          const long long lo = fs / gcdl(fs, offset);
          const long long L = nb * lo / gcdl(lo, nb);
          if (L > (1LL << 22)) return h->fail(GX_ERR_UNSUPPORTED, "phase-cal oscillator period above 4M samples");
          P.step = (int)std::floor((double)nb * (double)interval / (double)fs);
          P.offset_bin = 0;
          P.nextract = nt;
          P.rotlen = (int)L;
          P.rot0 = (long long)h->pcal_rot.size();
          const double dphi = -2 * M_PI * (double)offset / (double)fs;
          for (long long m = 0; m < 2 * L; m++) {
            const double arg = dphi * double(m);
            h->pcal_rot.push_back(make_float2((float)std::cos(arg), (float)std::sin(arg)));
          }
        }
        if (nb > 65536) return h->fail(GX_ERR_UNSUPPORTED, "more than 65536 phase-cal bins");
        P.nbins = (int)nb;
      }
      h->pcal.push_back(P);
    }
  }
  // Core result layout for records of 1 / div of the channels: crosses by
  // freq and baseline, baseline weights, autocorrelations, their weights
  auto build = [&](int div, std::vector<int> &blofs, std::vector<int> &bwofs, std::vector<int> &acofs,
                   std::vector<int> &acwofs, std::vector<int> &bsdofs) -> long long {
    blofs.assign(d.nfreqs * (nbl ? nbl : 1), -1);
    bwofs.assign(d.nfreqs * (nbl ? nbl : 1), -1);
    bsdofs.assign(d.nfreqs * (nbl ? nbl : 1), -1);
    acofs.assign(d.nstations, 0);
    acwofs.assign(d.nstations, 0);
    long long idx = 0;
    for (int f = 0; f < d.nfreqs; f++) {
      if (!freq_used(f)) continue;
      for (int j = 0; j < nbl; j++) {
        int lf = bl_localfreq(d.baselines[j], f);
        if (lf < 0) continue;
        blofs[f * nbl + j] = (int)idx;
        idx += (long long)h->maxpc * h->binloop * d.baselines[j].npolprod[lf] * (d.freqs[f].nchan / div);
      }
    }
    for (int f = 0; f < d.nfreqs; f++) {
      if (!freq_used(f)) continue;
      for (int j = 0; j < nbl; j++) {
        int lf = bl_localfreq(d.baselines[j], f);
        if (lf < 0) continue;
        bwofs[f * nbl + j] = (int)idx;
        int np = h->binloop * d.baselines[j].npolprod[lf];   // a weight per bin and product
        idx += np / 2 + np % 2;
      }
    }
    if (h->maxpc > 1)   // shift decorrelation factors, one float per phase centre (configuration.cpp:2548-2566)
      for (int f = 0; f < d.nfreqs; f++) {
        if (!freq_used(f)) continue;
        for (int j = 0; j < nbl; j++) {
          if (bl_localfreq(d.baselines[j], f) < 0) continue;
          bsdofs[f * nbl + j] = (int)idx;
          idx += h->maxpc / 2 + h->maxpc % 2;
        }
      }
    for (int s = 0; s < d.nstations; s++) {
      acofs[s] = (int)idx;
      const gx_station_desc &x = d.stations[s];
      for (int k : ac_bands(s)) idx += (long long)bpa * (d.freqs[total_freq(x, k)].nchan / div);
    }
    for (int s = 0; s < d.nstations; s++) {
      acwofs[s] = (int)idx;
      int add = bpa * (int)ac_bands(s).size();
      add = (add + 1) / 2;
      if (add == 0) add = 1;
      idx += add;
    }
    for (int s = 0; s < d.nstations; s++)   // and finally the phase-cal tones
      for (int n : pc_ntones[s]) idx += n;
    return idx;
  };
  // the kernels fill the full-resolution array; the averaged one is the result
  h->rl_full = build(1, h->blofs_full, h->bwofs_full, h->acofs_full, h->acwofs_full, h->bsdofs_full);
  h->rl = build(avg, h->blofs, h->bwofs, h->acofs, h->acwofs, h->bsdofs);
  // each recorded band's autocorrelation record and weight (for gx_sta)
  h->sta_acoff.assign((size_t)d.nstations * GX_MAX_BANDS, -1);
  h->sta_acw.assign((size_t)d.nstations * GX_MAX_BANDS, -1);
  for (int s = 0; s < d.nstations; s++) {
    long long o = h->acofs[s];
    int p = 0;
    for (int k : ac_bands(s)) {
      if (k < d.stations[s].nbands) {
        h->sta_acoff[(size_t)s * GX_MAX_BANDS + k] = (int)o;
        h->sta_acw[(size_t)s * GX_MAX_BANDS + k] = p;
      }
      o += d.freqs[total_freq(d.stations[s], k)].nchan / avg;
      p++;
    }
  }
  h->bsd_first = h->bsd_count = 0;
  if (h->maxpc > 1) {
    long long lo = -1, hi = -1;
    for (int x : h->bsdofs_full)
      if (x >= 0) {
        lo = lo < 0 ? x : std::min<long long>(lo, x);
        hi = std::max<long long>(hi, x + h->maxpc / 2 + h->maxpc % 2);
      }
    if (lo >= 0) { h->bsd_first = lo; h->bsd_count = hi - lo; }
  }
  // phase-cal section: after the autocorrelation weights, datastream by datastream, band by band
  h->pc_off.assign((size_t)d.nstations * GX_MAX_BANDS, -1);
  h->pc_ntones.assign((size_t)d.nstations * GX_MAX_BANDS, 0);
  {
    long long pos_full = h->rl_full, pos = h->rl;
    for (int s = 0; s < d.nstations; s++)
      for (int n : pc_ntones[s]) pos_full -= n, pos -= n;
    size_t k = 0;
    for (int s = 0; s < d.nstations; s++)
      for (int b = 0; b < (int)pc_ntones[s].size(); b++) {
        h->pcal[k++].result_offset = pos_full;
        h->pc_off[(size_t)s * GX_MAX_BANDS + b] = (int)pos;
        h->pc_ntones[(size_t)s * GX_MAX_BANDS + b] = pc_ntones[s][b];
        pos_full += pc_ntones[s][b];
        pos += pc_ntones[s][b];
      }
  }
  h->avgtab.clear();
  if (avg > 1) {
    auto add = [&](long long src, long long dst, int n, int L) { h->avgtab.push_back(AvgEntry{src, dst, n, L}); };
    for (int f = 0; f < d.nfreqs; f++)
      for (int j = 0; j < nbl; j++) {
        const int lf = bl_localfreq(d.baselines[j], f);
        if (lf < 0 || h->blofs[f * nbl + j] < 0) continue;
        const int nf = d.freqs[f].nchan, np = d.baselines[j].npolprod[lf];
        for (int p = 0; p < h->maxpc * h->binloop * np; p++)   // records of every phase centre and bin
          add(h->blofs_full[f * nbl + j] + (long long)p * nf, h->blofs[f * nbl + j] + (long long)p * (nf / avg),
              nf / avg, avg);
        const int nw = h->binloop * np;
        add(h->bwofs_full[f * nbl + j], h->bwofs[f * nbl + j], nw / 2 + nw % 2, 1);
        if (h->maxpc > 1) add(h->bsdofs_full[f * nbl + j], h->bsdofs[f * nbl + j], h->maxpc / 2 + h->maxpc % 2, 1);
      }
    long long total_pc = 0;   // the phase-cal section follows the autocorrelation weights
    for (int q = 0; q < d.nstations; q++)
      for (int n : pc_ntones[q]) total_pc += n;
    for (int s = 0; s < d.nstations; s++) {
      // parallel-hand rows of the station's bands, then (with cross-pol) the cross-hand rows
      long long src = h->acofs_full[s], dst = h->acofs[s];
      const std::vector<int> acb = ac_bands(s);
      for (int rep = 0; rep < bpa; rep++)
        for (int k : acb) {
          const int nf = d.freqs[total_freq(d.stations[s], k)].nchan;
          add(src, dst, nf / avg, avg);
          src += nf;
          dst += nf / avg;
        }
      const long long wend_full = s + 1 < d.nstations ? h->acwofs_full[s + 1] : h->rl_full - total_pc;
      add(h->acwofs_full[s], h->acwofs[s], (int)(wend_full - h->acwofs_full[s]), 1);
    }
    for (const PcalBand &P : h->pcal)   // phase-cal tones are copied
      add(P.result_offset, h->pc_off[(size_t)P.station * GX_MAX_BANDS + P.band], P.ntones, 1);
  }

  // FP32 accumulator index of the Hermitian entry (a, b) of freq slab f (shape
  // xs, N channels)
  const XmacShape &xs = h->xs;
  auto shape_index = [](const XmacShape &xs, int N, int f, int a, int b, int &conj) -> long long {
    conj = 0;
    if (a / xs.T > b / xs.T) { int t = a; a = b; b = t; conj = 1; }
    int SI = a / xs.ST, SJ = b / xs.ST;
    long long stp = 0;
    for (int i = 0; i < SI; i++) stp += xs.nsuper - i;
    stp += SJ - SI;
    return (((long long)f * xs.npairs + stp) * xs.ST * xs.ST + (long long)(a % xs.ST) * xs.ST + (b % xs.ST)) * N;
  };
  auto acc_index = [&](int f, int a, int b, int &conj) { return shape_index(xs, J.nchan, f, a, b, conj); };
  h->zprods.clear();
  // one zoom visibility row: result offset ro <- rows (a, b) of zoom freq z
  auto add_zprod = [&](long long ro, int z, int a, int b) {
    ProdEntry e{};
    e.result_offset = ro;
    e.acc_index = shape_index(h->zxs, h->nzchan, z, a, b, e.conj);
    h->zprods.push_back(e);
  };
  h->prods.clear();
  h->uvents.clear();
  h->binents.clear();
  h->binitems.clear();
  h->binwout.clear();
  h->autoprods.clear();
  h->autowents.clear();
  h->tcprods.clear();
  h->wents.clear();
  h->pairs.clear();
  // one visibility row: result offset ro <- input pair (a, b) of freq f
  auto add_prod = [&](long long ro, int f, int a, int b) {
    ProdEntry e{};
    e.result_offset = ro;
    e.acc_index = acc_index(f, a, b, e.conj);
    h->prods.push_back(e);
    TcProdEntry t{};
    t.result_offset = ro;
    t.freq = f;
    t.a = a;
    t.b = b;
    h->tcprods.push_back(t);
  };
  for (int j = 0; j < nbl; j++) {
    const gx_baseline_desc &B = d.baselines[j];
    if (B.ds1 < 0 || B.ds1 >= d.nstations || B.ds2 < 0 || B.ds2 >= d.nstations)
      return h->fail(GX_ERR_ARG, "baseline datastream index out of range");
    if (!h->interlaced_any) h->pairs.push_back(make_int2(B.ds1, B.ds2));
  }
  // Weight sums: item i < nstations sums station row i; item nstations + k
  // is pairs[k]: the product of rows (x, y) summed over blocks, or row x
  // alone when y < 0.  Rows of interlaced stations are per band: the
  // reference's getDataWeight(band) and perbandweights (core.cpp:911-912,
  // 1039-1044; mode.cpp:1277-1284, 1342-1351).
  std::map<std::pair<int, int>, int> witem;
  auto wrow = [&](int s, int b) { return d.stations[s].interlaced ? dst[s].wrow0 + b : s; };
  auto item = [&](int r1, int r2) -> int {
    if (r2 < 0 && r1 < d.nstations) return r1;
    auto it = witem.find({r1, r2});
    if (it != witem.end()) return it->second;
    const int idx = d.nstations + (int)h->pairs.size();
    h->pairs.push_back(make_int2(r1, r2));
    witem[{r1, r2}] = idx;
    return idx;
  };
  for (int f = 0; f < d.nfreqs; f++) {
    for (int j = 0; j < nbl; j++) {
      const gx_baseline_desc &B = d.baselines[j];
      int lf = bl_localfreq(B, f);
      if (lf < 0) continue;
      const gx_station_desc &x1 = d.stations[B.ds1], &x2 = d.stations[B.ds2];
      const int z = zord[f];
      for (int p = 0; p < B.npolprod[lf]; p++) {
        int b1 = B.band1[lf][p], b2 = B.band2[lf][p];
        WeightEntry w{};
        w.float_index = 2LL * h->bwofs_full[f * nbl + j] + p;
        if (z < 0) {
          if (b1 < 0 || b1 >= x1.nbands || b2 < 0 || b2 >= x2.nbands)
            return h->fail(GX_ERR_ARG, "baseline band index out of range");
          int a = h->band_input[B.ds1][b1], bb = h->band_input[B.ds2][b2];
          add_prod(h->blofs_full[f * nbl + j] + (long long)p * J.nchan, f, a, bb);
          const ProdEntry &pe = h->prods.back();
          h->uvents.push_back(UvEntry{pe.result_offset, pe.acc_index, pe.conj, j, f, B.npolprod[lf] * J.nchan});
          w.source = h->interlaced_any ? item(wrow(B.ds1, b1), wrow(B.ds2, b2)) : d.nstations + j;
          if (h->nbins > 0) {
            // binned: one weight sum per (freq, baseline), the same for its products
            if (p == 0) h->binitems.push_back(BinWeightItem{f, B.ds1, B.ds2});
            const int fj = (int)h->binitems.size() - 1;
            h->binents.push_back(BinEntry{h->blofs_full[f * nbl + j], f, a, bb, p, B.npolprod[lf], fj});
            for (int b = 0; b < h->binloop; b++)
              h->binwout.push_back(BinWeightOut{2LL * h->bwofs_full[f * nbl + j] + b * B.npolprod[lf] + p, fj, b});
            continue;   // no unbinned weight entry
          }
        } else {
          // zoom bands: the products of their rows; weights of their parent
          // recorded bands (datastream record band index, configuration.cpp:1203-1260)
          const int z1 = b1 - x1.nbands, z2 = b2 - x2.nbands;
          if (z1 < 0 || z1 >= x1.nzoombands || z2 < 0 || z2 >= x2.nzoombands || total_freq(x1, b1) != f ||
              total_freq(x2, b2) != f)
            return h->fail(GX_ERR_ARG, "a baseline's zoom freq product names a band of another freq");
          add_zprod(h->blofs_full[f * nbl + j] + (long long)p * h->nzchan, z, zrow[B.ds1][z1], zrow[B.ds2][z2]);
          w.source = h->interlaced_any ? item(wrow(B.ds1, zparent[B.ds1][z1]), wrow(B.ds2, zparent[B.ds2][z2]))
                                       : d.nstations + j;
        }
        h->wents.push_back(w);
      }
    }
  }
  const size_t ncross_prods = h->prods.size();   // the autocorrelation rows follow
  for (int s = 0; s < d.nstations; s++) {
    const gx_station_desc &x = d.stations[s];
    long long ro = h->acofs_full[s];
    long long wo = 2LL * h->acwofs_full[s];
    // total bands: recorded, then zoom (their autocorrelations are slices of
    // the parent band's, mode.cpp:379-391; weights the parent's, core.cpp:1317-1370)
    const std::vector<int> used = ac_bands(s);
    for (int k : used) {
      const int f = total_freq(x, k);
      WeightEntry w{};
      w.float_index = wo++;
      if (k < x.nbands) {
        const int a = h->band_input[s][k];
        add_prod(ro, f, a, a);
        const ProdEntry &pe = h->prods.back();
        h->uvents.push_back(UvEntry{pe.result_offset, pe.acc_index, pe.conj, -1, f, 0});
        w.source = item(wrow(s, k), -1);
      } else {
        const int zb = k - x.nbands;
        add_zprod(ro, zord[f], zrow[s][zb], zrow[s][zb]);
        w.source = item(wrow(s, zparent[s][zb]), -1);
      }
      ro += d.freqs[f].nchan;
      h->wents.push_back(w);
    }
    if (writecross) {
      for (int k : used) {
        const int f = total_freq(x, k);
        const int bp = k < x.nbands ? k : zparent[s][k - x.nbands];   // the recorded band
        int i0, i1;
        const int partner = partner_of(x, bp, &i0, &i1);
        WeightEntry w{};
        w.float_index = wo++;
        w.source = partner < 0 ? -1 : x.interlaced ? item(wrow(s, i0), wrow(s, i1)) : s;
        h->wents.push_back(w);
        if (partner >= 0) {
          if (k < x.nbands) {
            add_prod(ro, f, h->band_input[s][k], h->band_input[s][partner]);
            const ProdEntry &pe = h->prods.back();
            h->uvents.push_back(UvEntry{pe.result_offset, pe.acc_index, pe.conj, -1, f, 0});
          } else {
            add_zprod(ro, zord[f], zrow[s][k - x.nbands], zpartner[s][k - x.nbands]);
          }
        }
        ro += d.freqs[f].nchan;
      }
    }
  }

  if (h->nbins > 0) h->autoprods.assign(h->prods.begin() + ncross_prods, h->prods.end());

  // tensor-core finalising pass: entries grouped by (freq, a) row
  h->tcrows.clear();
  if (h->tc) {
    std::stable_sort(h->tcprods.begin(), h->tcprods.end(), [](const TcProdEntry &x, const TcProdEntry &y) {
      return x.freq != y.freq ? x.freq < y.freq : x.a < y.a;
    });
    for (size_t i = 0; i < h->tcprods.size();) {
      TcRowEntry r{h->tcprods[i].freq, h->tcprods[i].a, kTcInputs, (int)i, (int)i};
      while (i < h->tcprods.size() && h->tcprods[i].freq == r.freq && h->tcprods[i].a == r.a) {
        r.bmin = std::min(r.bmin, h->tcprods[i].b);
        i++;
      }
      r.end = (int)i;
      h->tcrows.push_back(r);
    }
  }

  // uv-shift intervals of multi-phase-centre scans (Core::processdata,
  // core.cpp:768-776, 984-991): maxxcblocks blocks each, a multiple of the
  // buffered FFTs, the last one what remains of the subint
  h->uv_nint = 0;
  h->uvfreqs.clear();
  if (h->maxpc > 1) {
    const int nbuf = h->meta ? h->meta->num_buffered_ffts : 1;
    const double blockns = (double)d.subint_ns / (double)J.blocks_per_send;
    for (const auto &sc : h->model->scans) {
      if (sc.numphasecentres < 2) continue;
      int M = (int)(sc.maxns_xc / blockns);
      M -= M % nbuf;
      if (M == 0) M = nbuf;
      h->uv_nint = std::max(h->uv_nint, (J.blocks_per_send + M - 1) / M);
    }
    h->rsl = stride_length(h->xmac_stride);   // rotatestridelen = calcstridelength(xmacstridelen)
    if (h->rsl < 1 || h->xmac_stride % h->rsl || J.nchan % h->xmac_stride)
      return h->fail(GX_ERR_UNSUPPORTED, "rotate stride length does not divide the xmac stride");
    for (int f = 0; f < d.nfreqs; f++)
      h->uvfreqs.push_back(UvFreq{d.freqs[f].freq_mhz, d.freqs[f].bw_mhz / (double)d.freqs[f].nchan,
                                  d.freqs[f].lower_sideband ? 1 : 0, d.freqs[f].nchan});
  }

  // chunking and K-split
  const size_t per_block = ((size_t)h->nfmain * J.ninputs * J.nchan +
                           h->zfreq.size() * (size_t)h->nzrows * h->nzchan) * sizeof(float2);
  // Every pass reads and writes the accumulators once; the spectra of a block
  // are written and read once.  Passes of at least `efficient` blocks keep the
  // accumulator traffic under a quarter of the spectra traffic.
  size_t acc_pass;
  if (h->tc) {
    const size_t cols = (size_t)(ni + 7) / 8 * 8;   // written in 8-column slices
    acc_pass = 2 * (size_t)h->nfmain * (J.nchan / 2) * ni * cols * sizeof(float4);
  } else {
    acc_pass = 2 * (size_t)h->nfmain * xs.npairs * xs.ST * xs.ST * J.nchan * sizeof(float2);
  }
  const size_t efficient = std::max<size_t>(64, (4 * acc_pass + 2 * per_block - 1) / (2 * per_block));
  int chunk;
  if (d.block_chunk > 0) {
    chunk = d.block_chunk;
  } else if (d.spectra_budget_bytes > 0) {
    // memory is shared with other jobs: the efficient length, within the budget
    chunk = (int)std::min<size_t>({8192, efficient, std::max<size_t>(16, (size_t)d.spectra_budget_bytes / per_block)});
  } else {
    // Both X-steps move their accumulators through HBM once per pass (the
    // tensor-core form 128 x 128 complex per channel, the FP32 form its upper
    // super-tiles), so passes are long: up to 40 GB of spectra, at most 30% of
    // the device memory free at open.
    size_t spec_budget = size_t(40) << 30;
    {
      size_t fr = 0, tot = 0;
      if (h->device >= 0 && cudaSetDevice(h->device) == cudaSuccess && cudaMemGetInfo(&fr, &tot) == cudaSuccess)
        spec_budget = std::max(size_t(1) << 30, std::min(spec_budget, fr / 10 * 3));
    }
    chunk = (int)std::min<size_t>(4096, std::max<size_t>(64, spec_budget / per_block));
  }
  if (chunk > J.blocks_per_send) chunk = J.blocks_per_send;
  chunk = std::max(1, chunk);
  if (d.block_chunk <= 0) {
    // equal chunks: no short tail pass
    const int nch = (J.blocks_per_send + chunk - 1) / chunk;
    chunk = (J.blocks_per_send + nch - 1) / nch;
  }
  if (h->nbins > 0) {
    // passes of whole buffered-FFT groups: the binned weights are summed in
    // the reference's group order (core.cpp:784-800, 943-950)
    const int nbuf = h->meta ? h->meta->num_buffered_ffts : 1;
    chunk = std::min(J.blocks_per_send, (chunk + nbuf - 1) / nbuf * nbuf);
  }
  h->chunk = chunk;
  if (h->tc) {
    // One CTA per SM (all 512 tensor-memory columns).  Every K-split slice
    // adds a full accumulator write and finalise read, so the K dimension is
    // split only while the grid is under two waves of 148 SMs (at least 4
    // K-tiles per slice).
    const long long base = (long long)(J.nchan / 2) * h->nfmain;
    const int kmax = std::max(1, std::min(16, chunk / 64));
    int best = 1;
    while (best < kmax && base * best < 2 * 148) best++;
    h->ks = best;
  } else {
    long long base = (long long)((J.nchan + xs.CT - 1) / xs.CT) * xs.npairs * h->nfmain;
    // K-split: enough CTAs for at least two per SM, rounded to whole waves of
    // 148 SMs where possible, keeping at least 64 blocks per slice
    const int kmax = std::max(1, std::min(16, chunk / 64));
    int best = 1;
    double best_score = -1;
    for (int ks = 1; ks <= kmax; ks++) {
      const long long ctas = base * ks;
      const double waves = std::ceil(ctas / 148.0);
      const double eff = ctas / (waves * 148.0);
      const double score = eff * std::min(1.0, ctas / 296.0);
      if (score > best_score + 1e-9) { best_score = score; best = ks; }
    }
    h->ks = best;
  }
  // zoom X-step K-split: as the FP32 X-step's, over the zoom freqs
  h->zks = 1;
  if (!h->zfreq.empty()) {
    const XmacShape &zx = h->zxs;
    const long long base = (long long)((h->nzchan + zx.CT - 1) / zx.CT) * zx.npairs * (long long)h->zfreq.size();
    const int kmax = std::max(1, std::min(16, chunk / 64));
    double best_score = -1;
    for (int ks = 1; ks <= kmax; ks++) {
      const long long ctas = base * ks;
      const double waves = std::ceil(ctas / 148.0);
      const double score = ctas / (waves * 148.0) * std::min(1.0, ctas / 296.0);
      if (score > best_score + 1e-9) { best_score = score; h->zks = ks; }
    }
    h->zacc_slice = h->zfreq.size() * (size_t)zx.npairs * zx.ST * zx.ST * h->nzchan;
  }
  // F-step concurrency: FFT slots per CTA
  {
    int ns = std::min(J.nbands, 32);
    while (ns > 1 && (fstep_smem_bytes(J, h->maxnrf, ns) > 200 * 1024 || kFThreads % ns)) ns--;
    h->nslots = ns;
    if (fstep_smem_bytes(J, h->maxnrf, ns) > 227 * 1024)
      return h->fail(GX_ERR_UNSUPPORTED, "F-step shared memory exceeds 227 KB");
  }

  {
    // decode tables (format_vdif.c:66-146): 2-bit {-HiMag,-1,1,HiMag}, 1-bit {-1,1},
    // 4-bit (l-7.5)/2.95, 8-bit (b-128)/3.3 or (b-127.5)/3.3 with SYMMETRIC_8_BIT_VDIF
    float *lut = J.lut;
    memset(lut, 0, sizeof(J.lut));
    const float himag = 3.3359f;
    if (J.nbits == 1) { lut[0] = -1.0f; lut[1] = 1.0f; }
    else if (J.nbits == 2) { lut[0] = -himag; lut[1] = -1.0f; lut[2] = 1.0f; lut[3] = himag; }
    else if (J.nbits == 4) { for (int l = 0; l < 16; l++) lut[l] = (float)((l - 7.5) / (double)2.95f); }
    else {
      double off = getenv("SYMMETRIC_8_BIT_VDIF") ? 127.5 : 128.0;
      for (int b = 0; b < 256; b++) lut[b] = (float)((b - off) / 3.3);
      J.lut_offset = off;
      J.lut_div = 3.3;
      // The same levels without a table lookup: 1 / 3.3 as a two-float sum and
      // one fused multiply-add, used only if it reproduces every entry.
      const double bias = 8388608.0 + off;
      const float hi = (float)(1.0 / 3.3), lo = (float)(1.0 / 3.3 - (double)hi);
      bool ok = (double)(float)bias == bias;
      for (int b = 0; ok && b < 256; b++) {
        const float x = (float)(8388608.0 + b) - (float)bias;
        ok = std::fma(x, hi, x * lo) == lut[b];
      }
      J.lut_affine = ok ? 1 : 0;
      J.lut_bias = (float)bias;
      J.lut_hi = hi;
      J.lut_lo = lo;
    }
    // Tensor-core operands: a power-of-two scale that brings the spectrum of
    // noise with the r.m.s. level of the decode table to an r.m.s. near 8, so
    // that the FP16 values and their split remainders stay in the normal range.
    double ms = 0;
    const int ncode = 1 << J.nbits;
    for (int l = 0; l < ncode; l++) ms += (double)lut[l] * lut[l];
    ms /= ncode;
    const double rms_spec = std::sqrt(ms * J.fftlen * (J.cplx ? 2.0 : 1.0));
    h->tc_scale0 = (float)std::ldexp(1.0, (int)std::lround(std::log2(8.0 / rms_spec)));
  }

  // ---------------------------------------------------------- device state
  if (h->device < 0) return GX_OK;  // host-only handle: layout and model queries
  CKR(h, cudaSetDevice(h->device));
  if (!h->stream) CKR(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  CKR(h, h->dalloc(&h->d_st, sizeof(DevStation) * d.nstations));
  CKR(h, cudaMemcpy(h->d_st, dst.data(), sizeof(DevStation) * d.nstations, cudaMemcpyHostToDevice));
  {
    const std::vector<float2> tw = twiddle_table(J.fftlen);
    CKR(h, h->dalloc(&h->d_tw, sizeof(float2) * tw.size()));
    CKR(h, cudaMemcpy(h->d_tw, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice));
    J.twiddle = h->d_tw;
  }
  const size_t spec_elems = (size_t)h->nfmain * chunk * J.ninputs * J.nchan;
  CKR(h, h->dalloc(&h->d_spec, sizeof(float2) * spec_elems));
  CKR(h, cudaMemsetAsync(h->d_spec, 0, sizeof(float2) * spec_elems, h->stream));
  CKR(h, h->dalloc(&h->d_spec1, sizeof(float2) * (size_t)h->nfmain * J.ninputs * J.nchan));
  CKR(h, cudaMemsetAsync(h->d_spec1, 0, sizeof(float2) * (size_t)h->nfmain * J.ninputs * J.nchan, h->stream));
  CKR(h, h->dalloc(&h->d_w, sizeof(float) * (size_t)h->nwrows * chunk));
  CKR(h, h->dalloc(&h->d_w1, sizeof(float) * (size_t)h->nwrows));
  if (h->interlaced_any)
    CKR(h, h->dalloc(&h->d_bandmask, sizeof(unsigned long long) * (size_t)d.nstations * chunk * J.nbands));
  CKR(h, h->dalloc(&h->d_bp, sizeof(BlockParam) * (size_t)d.nstations * chunk));
  CKR(h, h->dalloc(&h->d_bp1, sizeof(BlockParam) * (size_t)d.nstations));
  if (h->tc) {
    // [freq][chan/2][128][128] float4 (both channels of a pair) per K-split slice
    h->acc_slice = (size_t)h->nfmain * J.nchan * kTcInputs * kTcInputs;
    const size_t nsc = (size_t)h->nfmain * kTcInputs * J.nchan;
    std::vector<float> sc(nsc, h->tc_scale0);
    CKR(h, h->dalloc(&h->d_scale, sizeof(float) * nsc));
    CKR(h, cudaMemcpy(h->d_scale, sc.data(), sizeof(float) * nsc, cudaMemcpyHostToDevice));
    CKR(h, h->dalloc(&h->d_tcprods, sizeof(TcProdEntry) * std::max<size_t>(1, h->tcprods.size())));
    if (!h->tcprods.empty())
      CKR(h, cudaMemcpy(h->d_tcprods, h->tcprods.data(), sizeof(TcProdEntry) * h->tcprods.size(),
                        cudaMemcpyHostToDevice));
    CKR(h, h->dalloc(&h->d_tcrows, sizeof(TcRowEntry) * std::max<size_t>(1, h->tcrows.size())));
    if (!h->tcrows.empty())
      CKR(h, cudaMemcpy(h->d_tcrows, h->tcrows.data(), sizeof(TcRowEntry) * h->tcrows.size(),
                        cudaMemcpyHostToDevice));
  } else {
    h->acc_slice = (size_t)h->nfmain * xs.npairs * xs.ST * xs.ST * J.nchan;
  }
  CKR(h, h->dalloc(&h->d_acc, sizeof(float2) * h->acc_slice * h->ks));
  if (!h->zfreq.empty()) {
    // zoom spectra rows beyond the table's stay zero
    const size_t nz = h->zfreq.size() * (size_t)chunk * h->nzrows * h->nzchan;
    CKR(h, h->dalloc(&h->d_specz, sizeof(float2) * nz));
    CKR(h, cudaMemsetAsync(h->d_specz, 0, sizeof(float2) * nz, h->stream));
    CKR(h, h->dalloc(&h->d_accz, sizeof(float2) * h->zacc_slice * h->zks));
    CKR(h, h->dalloc(&h->d_zrows, sizeof(ZoomRow) * h->zrows.size()));
    CKR(h, cudaMemcpy(h->d_zrows, h->zrows.data(), sizeof(ZoomRow) * h->zrows.size(), cudaMemcpyHostToDevice));
    CKR(h, h->dalloc(&h->d_zprods, sizeof(ProdEntry) * std::max<size_t>(1, h->zprods.size())));
    if (!h->zprods.empty())
      CKR(h, cudaMemcpy(h->d_zprods, h->zprods.data(), sizeof(ProdEntry) * h->zprods.size(), cudaMemcpyHostToDevice));
  }
  CKR(h, h->dalloc(&h->d_err, sizeof(int)));
  CKR(h, cudaMemset(h->d_err, 0, sizeof(int)));
  CKR(h, cudaMallocHost(&h->h_err, sizeof(int) * gx_handle::kSlots));
  for (int k = 0; k < gx_handle::kSlots; k++) h->h_err[k] = 0;
  const size_t npairs = h->pairs.size();
  CKR(h, h->dalloc(&h->d_wacc, sizeof(float) * (d.nstations + npairs)));
  if (npairs) {
    CKR(h, h->dalloc(&h->d_pairs, sizeof(int2) * npairs));
    CKR(h, cudaMemcpy(h->d_pairs, h->pairs.data(), sizeof(int2) * npairs, cudaMemcpyHostToDevice));
  }
  CKR(h, h->dalloc(&h->d_prods, sizeof(ProdEntry) * std::max<size_t>(1, h->prods.size())));
  if (!h->prods.empty())
    CKR(h, cudaMemcpy(h->d_prods, h->prods.data(), sizeof(ProdEntry) * h->prods.size(), cudaMemcpyHostToDevice));
  CKR(h, h->dalloc(&h->d_went, sizeof(WeightEntry) * std::max<size_t>(1, h->wents.size())));
  if (!h->wents.empty())
    CKR(h, cudaMemcpy(h->d_went, h->wents.data(), sizeof(WeightEntry) * h->wents.size(), cudaMemcpyHostToDevice));
  CKR(h, h->dalloc(&h->d_results, sizeof(float2) * h->rl));
  if (h->nbins > 0) {
    const PulsarConfig &P = *h->meta->pulsar;
    auto up = [&](auto **dst, const auto &vec) -> gx_status {
      using T = typename std::remove_reference<decltype(vec)>::type::value_type;
      CKR(h, h->dalloc(dst, sizeof(T) * std::max<size_t>(1, vec.size())));
      if (!vec.empty()) CKR(h, cudaMemcpy(*dst, vec.data(), sizeof(T) * vec.size(), cudaMemcpyHostToDevice));
      return GX_OK;
    };
    gx_status r;
    if ((r = up(&h->d_binents, h->binents)) != GX_OK) return r;
    if ((r = up(&h->d_binitems, h->binitems)) != GX_OK) return r;
    if ((r = up(&h->d_binwout, h->binwout)) != GX_OK) return r;
    if ((r = up(&h->d_autoprods, h->autoprods)) != GX_OK) return r;
    if ((r = up(&h->d_binphase, P.binphaseends)) != GX_OK) return r;
    if ((r = up(&h->d_binweight, P.binweights)) != GX_OK) return r;
    CKR(h, h->dalloc(&h->d_accb, sizeof(float2) * std::max<size_t>(1, h->binents.size()) * h->nbins * J.nchan));
    CKR(h, h->dalloc(&h->d_wbins, sizeof(float) * std::max<size_t>(1, h->binitems.size()) * h->nbins));
  }
  if (h->maxpc > 1) {
    CKR(h, h->dalloc(&h->d_uvents, sizeof(UvEntry) * std::max<size_t>(1, h->uvents.size())));
    if (!h->uvents.empty())
      CKR(h, cudaMemcpy(h->d_uvents, h->uvents.data(), sizeof(UvEntry) * h->uvents.size(), cudaMemcpyHostToDevice));
    CKR(h, h->dalloc(&h->d_uvfreqs, sizeof(UvFreq) * h->uvfreqs.size()));
    CKR(h, cudaMemcpy(h->d_uvfreqs, h->uvfreqs.data(), sizeof(UvFreq) * h->uvfreqs.size(), cudaMemcpyHostToDevice));
  }
  if (!h->pcal.empty()) {
    h->pcal_maxbins = 1;
    for (const PcalBand &P : h->pcal) h->pcal_maxbins = std::max(h->pcal_maxbins, P.nbins);
    // enough CTAs for four waves of the SMs: chunks of blocks per band, at least 8 blocks a chunk
    h->pcal_chunks = (int)std::max<long long>(1, std::min<long long>(std::max(1, h->chunk / 8),
                                                                      (4 * 148 + (long long)h->pcal.size() - 1) /
                                                                          (long long)h->pcal.size()));
    // one CTA per station when every station with phase-cal has the same bands
    // and bin count (the usual case), else one per band
    h->pcal_per_station = J.nbands;
    for (size_t i = 0; i < h->pcal.size(); i++)
      if (h->pcal.size() % J.nbands || h->pcal[i].nbins != h->pcal[0].nbins || h->pcal[i].nbins <= 0 ||
          h->pcal[i].rotlen > 0 ||
          h->pcal[i].station != h->pcal[i - i % J.nbands].station || h->pcal[i].band != (int)(i % J.nbands))
        h->pcal_per_station = 0;
    if (h->pcal_per_station) {   // chunks for about eight 256-thread CTAs per SM
      const long long ng = (long long)h->pcal.size() / J.nbands;
      h->pcal_chunks = (int)std::max<long long>(1, std::min<long long>(std::max(1, h->chunk / 8), (8 * 148 + ng - 1) / ng));
    }
    CKR(h, h->dalloc(&h->d_pcal, sizeof(PcalBand) * h->pcal.size()));
    CKR(h, cudaMemcpy(h->d_pcal, h->pcal.data(), sizeof(PcalBand) * h->pcal.size(), cudaMemcpyHostToDevice));
    if (!h->pcal_rot.empty()) {
      CKR(h, h->dalloc(&h->d_pcalrot, sizeof(float2) * h->pcal_rot.size()));
      CKR(h, cudaMemcpy(h->d_pcalrot, h->pcal_rot.data(), sizeof(float2) * h->pcal_rot.size(), cudaMemcpyHostToDevice));
    }
    // The station-block F-step forms the bin sums itself when each thread's
    // samples share a bin (nbins divides F / 16); it then needs one slot of
    // partial sums per CTA group of the longest pass.
    h->pcal_fuse_bins = 0;
    if (h->pcal_per_station && fstep_sb_eligible(J, false)) {
      const int NT = J.fftlen / 16, G = (NT >= 256 ? NT : 256) / NT, nbins = h->pcal[0].nbins;
      if (nbins <= NT && NT % nbins == 0) {
        const int bpc = (J.sb_items > 0 ? J.sb_items : 4) * G;
        const long long slots = (long long)((h->chunk + bpc - 1) / bpc) * G;
        if (slots * (long long)h->pcal.size() * h->pcal_maxbins <= (64ll << 20)) {   // at most 512 MB of sums
          std::vector<int> first(d.nstations, -1);
          for (size_t i = 0; i < h->pcal.size(); i += J.nbands) first[h->pcal[i].station] = (int)i;
          CKR(h, h->dalloc(&h->d_pcalfirst, sizeof(int) * first.size()));
          CKR(h, cudaMemcpy(h->d_pcalfirst, first.data(), sizeof(int) * first.size(), cudaMemcpyHostToDevice));
          h->pcal_chunks = (int)std::max<long long>(h->pcal_chunks, slots);
          h->pcal_fuse_bins = nbins;
        }
      }
    }
    CKR(h, h->dalloc(&h->d_pcalbins, sizeof(float2) * (size_t)h->pcal_chunks * h->pcal.size() * h->pcal_maxbins));
  }
  if (h->avg > 1) {
    CKR(h, h->dalloc(&h->d_full, sizeof(float2) * h->rl_full));
    CKR(h, h->dalloc(&h->d_avgtab, sizeof(AvgEntry) * h->avgtab.size()));
    CKR(h, cudaMemcpy(h->d_avgtab, h->avgtab.data(), sizeof(AvgEntry) * h->avgtab.size(), cudaMemcpyHostToDevice));
  }
  h->ctrlstride = 3 + J.flaglen;
  h->o_len = sizeof(SubintClock);
  h->o_ptr = h->o_len + sizeof(int64_t) * d.nstations;
  h->o_interp = h->o_ptr + sizeof(uint8_t *) * d.nstations;
  h->o_ctrl = h->o_interp + sizeof(double) * 3 * d.nstations;
  // multiple phase centres: the intervals' differential delays [interval][baseline][centre]
  // (doubles) and the shift-decorrelation section of the result (floats)
  h->o_uvdelay = (h->o_ctrl + sizeof(int32_t) * h->ctrlstride * d.nstations + 15) & ~(size_t)15;
  h->o_bsd = h->o_uvdelay + sizeof(double) * (size_t)h->uv_nint * d.nbaselines * h->maxpc;
  // pulsar binning: the mean pulse phase of every block and the dispersion
  // phase offset of every channel (doubles)
  h->o_avgphase = (h->o_bsd + sizeof(float2) * (size_t)h->bsd_count + 15) & ~(size_t)15;
  h->o_dmoff = h->o_avgphase + (h->nbins > 0 ? sizeof(double) * (size_t)J.blocks_per_send : 0);
  h->o_ring = (h->o_dmoff + (h->nbins > 0 ? sizeof(double) * (size_t)h->nfmain * J.nchan : 0) + 15) & ~(size_t)15;
  h->sub_bytes = h->o_ring + sizeof(double) * 3 * d.nstations;
  CKR(h, h->dalloc(&h->d_sub, h->sub_bytes));
  for (int k = 0; k < gx_handle::kSlots; k++) {
    CKR(h, cudaMallocHost(&h->h_sub[k], h->sub_bytes));
    memset(h->h_sub[k], 0, h->sub_bytes);
    CKR(h, cudaEventCreateWithFlags(&h->ev_sub[k], cudaEventDisableTiming));
    CKR(h, cudaEventCreateWithFlags(&h->ev_copied[k], cudaEventDisableTiming));
    CKR(h, cudaEventCreateWithFlags(&h->ev_done[k], cudaEventDisableTiming));
    h->d_data[k].assign(d.nstations, nullptr);
    h->data_cap[k].assign(d.nstations, 0);
    h->data_alloc[k].assign(d.nstations, 0);
  }
  if (d.max_data_bytes > 0) {   // slot 0 only; slot 1 grows on the first gx_subint_async
    for (int s = 0; s < d.nstations; s++) {
      CKR(h, h->dalloc(&h->d_data[0][s], d.max_data_bytes));
      h->data_cap[0][s] = d.max_data_bytes;
      h->data_alloc[0][s] = d.max_data_bytes;
    }
  }
  CKR(h, cudaStreamSynchronize(h->stream));
  return GX_OK;
}

namespace gx {

// Twiddle table of an F-point transform (F a power of two) in the layout of
// r16::tw_pass_offset: W_F^m, m < F, then the rows of each radix-16 pass of
// stride 16^p and of the final radix pass.  Entries are formed in double and
// rounded once.
std::vector<float2> twiddle_table(int F)
{
  auto w = [F](long long e) {
    const double a = -2.0 * M_PI * (double)(e % F) / (double)F;
    return make_float2((float)std::cos(a), (float)std::sin(a));
  };
  std::vector<float2> tw(F >= 16 ? r16::tw_table_size(F) : F);
  for (int m = 0; m < F; m++) tw[m] = w(m);
  if (F < 16) return tw;
  const int L = r16::log16_floor(F), R0 = F / r16::pow16(L);
  for (int p = 1; p < L; p++) {
    const int Ns = r16::pow16(p), off = r16::tw_pass_offset(F, p);
    for (int r = 1; r < 16; r++)
      for (int m = 0; m < Ns; m++) tw[off + (r - 1) * Ns + m] = w((long long)r * m * (F / (16 * Ns)));
  }
  if (R0 > 1) {
    const int FR = F / R0, off = r16::tw_final_offset(F);
    for (int r = 1; r < R0; r++)
      for (int g = 0; g < FR; g++) tw[off + (r - 1) * FR + g] = w((long long)g * r);
  }
  return tw;
}

// The tables of a host-only open (device -1), handed to callers that place
// them in their own device memory.
gx_status plan_job(const gx_job_desc *desc, JobPlan *plan, std::string &err)
{
  if (!desc || !plan) { err = "null descriptor or plan"; return GX_ERR_ARG; }
  gx_handle h;
  h.device = -1;
  h.jd = *desc;
  if (desc->stations && desc->nstations > 0) h.st.assign(desc->stations, desc->stations + desc->nstations);
  if (desc->freqs && desc->nfreqs > 0) h.fr.assign(desc->freqs, desc->freqs + desc->nfreqs);
  if (desc->baselines && desc->nbaselines > 0) h.bl.assign(desc->baselines, desc->baselines + desc->nbaselines);
  h.jd.stations = h.st.data();
  h.jd.freqs = h.fr.data();
  h.jd.baselines = h.bl.data();
  gx_status s = setup(&h);
  if (s != GX_OK) { err = h.err; return s; }
  if (h.avg > 1) { err = "channel averaging is not implemented by the allocation-free entry point"; return GX_ERR_UNSUPPORTED; }
  if (!h.pcal.empty()) { err = "phase-cal extraction is not implemented by the allocation-free entry point"; return GX_ERR_UNSUPPORTED; }
  if (h.interlaced_any) { err = "INTERLACEDVDIF is not implemented by the allocation-free entry point"; return GX_ERR_UNSUPPORTED; }
  if (!h.zfreq.empty()) { err = "zoom bands are not implemented by the allocation-free entry point"; return GX_ERR_UNSUPPORTED; }
  plan->J = h.J;
  plan->J.twiddle = nullptr;
  plan->maxnrf = h.maxnrf;
  plan->nslots = h.nslots;
  plan->ks = h.ks;
  plan->xs = h.xs;
  plan->result_length = h.rl;
  plan->ctrlstride = 3 + h.J.flaglen;
  plan->stations = h.dst;
  plan->prods = h.prods;
  plan->wents = h.wents;
  plan->pairs = h.pairs;
  plan->twiddle = twiddle_table(h.J.fftlen);
  return GX_OK;
}

}  // namespace gx

extern "C" {

const char *gx_status_string(gx_status s)
{
  switch (s) {
    case GX_OK: return "ok";
    case GX_ERR_ARG: return "invalid argument";
    case GX_ERR_UNSUPPORTED: return "unsupported configuration";
    case GX_ERR_CUDA: return "CUDA error";
    case GX_ERR_NOMEM: return "out of memory";
    case GX_ERR_IO: return "I/O or parse error";
    case GX_ERR_MODEL: return "no delay model";
    case GX_ERR_TIMEOUT: return "device wait timed out";
    case GX_ERR_STATE: return "call out of order";
  }
  return "unknown";
}

// A handle for desc; model and meta (from the .input job) are in place before
// the setup, which takes the phase centres and uv-shift intervals from them.
static gx_status open_handle(const gx_job_desc *desc, int device, std::unique_ptr<HostModel> model,
                             std::unique_ptr<gx::JobMeta> meta, gx_handle **out)
{
  if (!desc || !out) return GX_ERR_ARG;
  *out = nullptr;
  gx_handle *h = new gx_handle();
  h->device = device;
  h->model = std::move(model);
  h->meta = std::move(meta);
  h->jd = *desc;
  if (desc->stations && desc->nstations > 0) h->st.assign(desc->stations, desc->stations + desc->nstations);
  if (desc->freqs && desc->nfreqs > 0) h->fr.assign(desc->freqs, desc->freqs + desc->nfreqs);
  if (desc->baselines && desc->nbaselines > 0)
    h->bl.assign(desc->baselines, desc->baselines + desc->nbaselines);
  h->jd.stations = h->st.data();
  h->jd.freqs = h->fr.data();
  h->jd.baselines = h->bl.data();
  gx_status s = setup(h);
  if (s != GX_OK) {
    fprintf(stderr, "gx_open: %s\n", h->err.c_str());
    free_all(h);
    delete h;
    return s;
  }
  *out = h;
  return GX_OK;
}

gx_status gx_open(const gx_job_desc *desc, int device, gx_handle **out)
{
  return open_handle(desc, device, nullptr, nullptr, out);
}

gx_status gx_close(gx_handle *h)
{
  if (!h) return GX_ERR_ARG;
  if (h->device >= 0) {
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
  }
  free_all(h);
  if (h->kurt) gx_kurtosis_free(h->kurt);
  delete h;
  return GX_OK;
}

const char *gx_last_error(const gx_handle *h) { return h ? h->err.c_str() : "null handle"; }

gx_status gx_get_layout(const gx_handle *h, gx_layout_info *info)
{
  if (!h || !info) return GX_ERR_ARG;
  info->result_length = h->rl;
  info->nfreqs = h->jd.nfreqs;
  info->nbaselines = h->jd.nbaselines;
  info->nstations = h->jd.nstations;
  info->blocks_per_send = h->J.blocks_per_send;
  info->xmac_stride = h->xmac_stride;
  info->array_stride = h->J.stride;
  info->fftchannels = h->J.fftlen;
  info->nchan = h->J.nchan;
  info->xstep = h->xstep;
  info->block_chunk = h->chunk;
  info->chans_to_average = h->avg;
  return GX_OK;
}

gx_status gx_get_pcal_layout(const gx_handle *h, int *offsets, int *ntones)
{
  if (!h) return GX_ERR_ARG;
  if (offsets) memcpy(offsets, h->pc_off.data(), sizeof(int) * h->pc_off.size());
  if (ntones) memcpy(ntones, h->pc_ntones.data(), sizeof(int) * h->pc_ntones.size());
  return GX_OK;
}

gx_status gx_set_tiles(gx_handle *h, int xmac_variant, int fstep_items)
{
  if (!h) return GX_ERR_ARG;
  if (xmac_variant < 0 || xmac_variant >= kXmacVariants || fstep_items < 0 || fstep_items > 64)
    return h->fail(GX_ERR_ARG, "tile choice out of range");
  h->xvar = xmac_variant;
  h->J.sb_items = fstep_items;
  return GX_OK;
}

gx_status gx_get_tiles(const gx_handle *h, int *xmac_variant, int *fstep_items)
{
  if (!h) return GX_ERR_ARG;
  if (xmac_variant) *xmac_variant = h->xvar;
  if (fstep_items) *fstep_items = h->J.sb_items > 0 ? h->J.sb_items : 4;
  return GX_OK;
}

gx_status gx_get_offsets(const gx_handle *h, int *blofs, int *bwofs, int *acofs, int *acwofs)
{
  if (!h) return GX_ERR_ARG;
  if (blofs) memcpy(blofs, h->blofs.data(), sizeof(int) * h->blofs.size());
  if (bwofs) memcpy(bwofs, h->bwofs.data(), sizeof(int) * h->bwofs.size());
  if (acofs) memcpy(acofs, h->acofs.data(), sizeof(int) * h->acofs.size());
  if (acwofs) memcpy(acwofs, h->acwofs.data(), sizeof(int) * h->acwofs.size());
  return GX_OK;
}

static gx_status record(gx_handle *h, cudaStream_t st, int stage, bool start)
{
  cudaEvent_t e;
  CKR(h, cudaEventCreate(&e));
  CKR(h, cudaEventRecord(e, st));
  h->evs.push_back(e);
  if (start) h->ev_stage.push_back(stage);
  return GX_OK;
}

}  // extern "C"

// Writes the per-subint tables of `sub` (data in device buffers `devdata`)
// into the handle's pinned block.
static gx_status stage_subint(gx_handle *h, const gx_subint_desc *sub, const uint8_t *const *devdata)
{
  const gx_job_desc &d = h->jd;
  if (sub->controllen < h->ctrlstride) return h->fail(GX_ERR_ARG, "control buffer shorter than 3 + flag words");
  for (int s = 0; s < d.nstations; s++)
    if (!sub->control[s]) return h->fail(GX_ERR_ARG, "missing control buffer");
  if (!sub->interp && !h->model)
    return h->fail(GX_ERR_ARG, "no interpolators given and the handle has no delay model");
  // the previous copy of this slot's block must have left it
  const int k = h->slot;
  if (h->ev_sub_pending[k]) {
    CKR(h, cudaEventSynchronize(h->ev_sub[k]));
    h->ev_sub_pending[k] = false;
  }
  unsigned char *b = h->h_sub[k];
  *reinterpret_cast<SubintClock *>(b) = SubintClock{sub->sec, sub->ns, sub->scan_start_sec};
  int64_t *lens = reinterpret_cast<int64_t *>(b + h->o_len);
  const uint8_t **ptrs = reinterpret_cast<const uint8_t **>(b + h->o_ptr);
  double *interp = reinterpret_cast<double *>(b + h->o_interp);
  int32_t *ctrl = reinterpret_cast<int32_t *>(b + h->o_ctrl);
  for (int s = 0; s < d.nstations; s++) {
    memcpy(ctrl + (size_t)s * h->ctrlstride, sub->control[s], sizeof(int32_t) * h->ctrlstride);
    lens[s] = sub->datalen[s];
    ptrs[s] = devdata[s];
  }
  if (sub->interp) {
    memcpy(interp, sub->interp, sizeof(double) * 3 * d.nstations);
  } else {
    for (int s = 0; s < d.nstations; s++) {
      gx_status r = h->model->interpolator(s, sub->scan, sub->sec, sub->ns, &interp[3 * s]);
      if (r != GX_OK) return h->fail(r, "no delay model for this subint");
    }
  }
  if (h->nbins > 0) {
    // Pulsar binning: the polyco covering the subint start (Core::loopprocess,
    // core.cpp:496-507; Polyco::setTime and calculateDMPhaseOffsets,
    // polyco.cpp:291-342, 368-387), the dispersion phase offset of every
    // channel (setFrequencyValues, polyco.cpp:226-251, with the FP32 band
    // edges and widths it keeps) and the mean phase of every block
    // (getBins, polyco.cpp:177-190)
    const PulsarConfig &P = *h->meta->pulsar;
    const JobMeta &M = *h->meta;
    const double sec = double(M.start_seconds + (int)h->model->scan_start_sec(sub->scan) + sub->sec) +
                       ((double)sub->ns) / 1000000000.0;
    const int pi = P.current(M.start_mjd, sec / 86400.0);
    if (pi < 0) return h->fail(GX_ERR_MODEL, "no polyco covers this subint");
    const PolycoEntry &Q = P.polycos[pi];
    const int nco = (int)Q.phasecoef.size();
    const double dt0 = (M.start_mjd - Q.mjd) * 1440 + (sec / 86400.0 - Q.mjdfraction) * 1440.0;
    const double calclengthmins = double(d.subint_ns) / 60000000000.0;
    double tp[64];
    tp[0] = 1.0;
    auto dot = [&](double dt, const std::vector<double> &c) {
      for (int i = 1; i < nco; i++) tp[i] = dt * tp[i - 1];
      double acc = 0;
      for (int i = 0; i < nco; i++) acc += tp[i] * c[i];
      return acc;
    };
    const double currentfreq = dot(dt0 + calclengthmins / 2, Q.freqcoef);
    const double DMC = 1.0 / 0.000241;   // Polyco::DM_CONSTANT_SECS
    double *dmoff = reinterpret_cast<double *>(b + h->o_dmoff);
    const int N = h->J.nchan;
    for (int f = 0; f < h->nfmain; f++) {
      const gx_freq_desc &fq = d.freqs[f];
      double lo = fq.freq_mhz;
      if (fq.lower_sideband) lo -= ((double)(fq.nchan - 1)) * fq.bw_mhz / ((double)fq.nchan);
      const float lof = (float)lo, bwf = (float)fq.bw_mhz;
      for (int c = 0; c < N; c++) {
        const double cf = lof + ((float)c * bwf) / double(fq.nchan);
        const double dmdelay = -Q.dm * DMC / (cf * cf) + Q.dm * DMC / (Q.obsfreq * Q.obsfreq);
        dmoff[(size_t)f * N + c] = dmdelay * currentfreq;
      }
    }
    double *avgphase = reinterpret_cast<double *>(b + h->o_avgphase);
    const double blockns = ((double)d.subint_ns) / ((double)h->J.blocks_per_send);
    for (int i = 0; i < h->J.blocks_per_send; i++)
      avgphase[i] = dot(dt0 + ((double)i) * blockns / 60000000000.0, Q.phasecoef);
  }
  h->cur_npc[k] = 1;
  h->cur_M[k] = 0;
  if (h->maxpc > 1) {
    if (sub->scan < 0 || sub->scan >= (int)h->model->scans.size()) return h->fail(GX_ERR_MODEL, "scan out of range");
    const auto &sc = h->model->scans[sub->scan];
    float *bsd = reinterpret_cast<float *>(b + h->o_bsd);
    memset(bsd, 0, sizeof(float2) * h->bsd_count);
    if (sc.numphasecentres > 1) {
      // per uv-shift interval (its centre and width, core.cpp:984-991, 1055-1057),
      // baseline and phase centre: the differential delay and rate against the
      // pointing centre (core.cpp:1641-1673), and the shift decorrelation
      // sum nswidth * time-smearing * delay-window factor (core.cpp:1894-1923)
      const int nph = sc.numphasecentres, bps = h->J.blocks_per_send, nbl = d.nbaselines;
      const int nbuf = h->meta ? h->meta->num_buffered_ffts : 1;
      const double blockns = (double)d.subint_ns / (double)bps;
      int M = (int)(sc.maxns_xc / blockns);
      M -= M % nbuf;
      if (M == 0) M = nbuf;
      double *uvd = reinterpret_cast<double *>(b + h->o_uvdelay);
      const HostModel &mdl = *h->model;
      for (int iv = 0; iv * M < bps; iv++) {
        const int cnt = std::min(M, bps - iv * M);
        const double nsoffset = (iv * M + ((double)cnt) / 2.0) * blockns, nswidth = cnt * blockns;
        const double t = sub->sec + double(sub->ns + nsoffset) / 1000000000.0;
        for (int j = 0; j < nbl; j++) {
          const gx_baseline_desc &B = d.baselines[j];
          const int a1 = mdl.station_of_datastream[B.ds1], a2 = mdl.station_of_datastream[B.ds2];
          double pc1[2], pc2[2];
          if (!mdl.linear(sub->scan, t, a1, 0, pc1) || !mdl.linear(sub->scan, t, a2, 0, pc2))
            return h->fail(GX_ERR_MODEL, "no delay model for a uv-shift interval");
          for (int ph = 0; ph < nph; ph++) {
            double p1[2], p2[2];
            if (!mdl.linear(sub->scan, t, a1, ph + 1, p1) || !mdl.linear(sub->scan, t, a2, ph + 1, p2))
              return h->fail(GX_ERR_MODEL, "no delay model for a phase centre");
            double ad1 = p1[1] - pc1[1], ad2 = p2[1] - pc2[1];
            ad1 += ad1 * pc1[0];   // the geometric rate over the shifted sample range
            ad2 += ad2 * pc2[0];
            const double dd1 = ad2 - ad1;
            const double dd0 = p2[0] + pc1[0] - (p1[0] + pc2[0]);
            uvd[((size_t)iv * nbl + j) * h->maxpc + ph] = dd1;
            for (int f = 0; f < d.nfreqs; f++) {
              const int o = h->bsdofs_full[f * nbl + j];
              if (o < 0) continue;
              double timesmeardecorr = 1.0, delaydecorr = 1.0;
              if (std::fabs(dd0) > 1e-18) {
                const double maxphasechange = kTwoPi * dd0 * (nswidth / 1000.0) * d.freqs[f].freq_mhz;
                timesmeardecorr = std::sin(maxphasechange / 2.0) / (maxphasechange / 2.0);
                if (timesmeardecorr < 0.0) timesmeardecorr = 0;
              }
              if (std::fabs(dd1) > 1e-18) {
                const double delaywindow = d.freqs[f].nchan / d.freqs[f].bw_mhz;   // max lag, plus and minus
                delaydecorr = 1.0 - std::fabs(dd1 / delaywindow);
                if (delaydecorr < 0.0) delaydecorr = 0;
              }
              float &acc = bsd[2 * (o - h->bsd_first) + ph];
              acc += nswidth * timesmeardecorr * delaydecorr;
            }
          }
        }
      }
      h->cur_npc[k] = nph;
      h->cur_M[k] = M;
    }
  }
  return GX_OK;
}

// Enqueues the device work of the staged subint on `st`: the tables' copy,
// F-step, X-step and finalisation into dev_results.  Nothing here waits on
// the host, so the sequence can be captured into a CUDA graph (h->untimed:
// no events recorded; the graph's copy reads the pinned block at replay).
gx_status gx_enqueue_subint(gx_handle *h, float2 *dev_results, cudaStream_t st)
{
  const gx_job_desc &d = h->jd;
  const DevJob &J = h->J;
  const bool timed = !h->untimed;
  if (timed) {
    for (auto e : h->evs) cudaEventDestroy(e);
    h->evs.clear();
    h->ev_stage.clear();
  }
  h->launches = 0;
  const int k = h->slot;
  CKR(h, cudaMemcpyAsync(h->d_sub, h->h_sub[k], h->sub_bytes, cudaMemcpyHostToDevice, st));
  if (timed) {
    CKR(h, cudaEventRecord(h->ev_sub[k], st));
    h->ev_sub_pending[k] = true;
  }
  if (h->ring_req) {
    // station data from the rings: the walk fills in the data pointers,
    // lengths and control words of the tables just copied
    gx_status rr = gx_ring_enqueue_control(h->ring_req, h, st);
    if (rr != GX_OK) return rr;
  }
  SubintArrays S{};
  S.clock = reinterpret_cast<const SubintClock *>(h->d_sub);
  S.data = reinterpret_cast<const uint8_t *const *>(h->d_sub + h->o_ptr);
  S.datalen = reinterpret_cast<const int64_t *>(h->d_sub + h->o_len);
  S.control = reinterpret_cast<const int32_t *>(h->d_sub + h->o_ctrl);
  S.controlstride = h->ctrlstride;
  S.interp = reinterpret_cast<const double *>(h->d_sub + h->o_interp);
  S.bandmask = h->d_bandmask;
  h->last = S;
  h->have_last = true;

  const int nbl = d.nbaselines;
  float4 *acc4 = reinterpret_cast<float4 *>(h->d_acc);
  auto mark = [&](int stage, bool start) -> gx_status { return timed ? record(h, st, stage, start) : GX_OK; };
  // the tensor-core X-step stores its first chunk instead of adding to it
  if (!h->tc) CKR(h, cudaMemsetAsync(h->d_acc, 0, sizeof(float2) * h->acc_slice * h->ks, st));
  const int nzr = (int)h->zrows.size(), nzf = (int)h->zfreq.size();
  if (nzf) CKR(h, cudaMemsetAsync(h->d_accz, 0, sizeof(float2) * h->zacc_slice * h->zks, st));
  if (h->nbins > 0) {
    CKR(h, cudaMemsetAsync(h->d_accb, 0, sizeof(float2) * h->binents.size() * h->nbins * J.nchan, st));
    CKR(h, cudaMemsetAsync(h->d_wbins, 0, sizeof(float) * h->binitems.size() * h->nbins, st));
  }
  const int npairs = (int)h->pairs.size();
  CKR(h, cudaMemsetAsync(h->d_wacc, 0, sizeof(float) * (d.nstations + npairs), st));
  CKR(h, cudaMemsetAsync(h->d_err, 0, sizeof(int), st));
  const int npc = (int)h->pcal.size();
  if (npc)
    CKR(h, cudaMemsetAsync(h->d_pcalbins, 0, sizeof(float2) * (size_t)h->pcal_chunks * npc * h->pcal_maxbins, st));
  gx_status r;
  // with channel averaging the finalise fills the full-resolution array first
  float2 *fin = h->avg > 1 ? h->d_full : dev_results;
  // one pass of nb blocks from block b0: F-step (and phase-cal bins), X-step, weights
  auto pass = [&](int b0, int nb) -> gx_status {
    gx_status r;
    if ((r = mark(0, true)) != GX_OK) return r;
    const PcalFuse pf{h->d_pcalbins, h->d_pcalfirst, h->pcal_fuse_bins, h->pcal_maxbins, npc, h->pcal_chunks};
    bool pcal_done = false;
    CKR(h, fstep_launch(J, h->d_st, h->maxnrf, S, b0, nb, h->nslots, h->d_spec, h->d_w, h->d_bp, st,
                        npc && h->pcal_fuse_bins ? &pf : nullptr, &pcal_done));
    if (h->kurt && (r = gx_kurtosis_pass(h, nb, st)) != GX_OK) return r;
    if (npc && !pcal_done) {
      CKR(h, pcal_bins_launch(J, S, h->d_bp, nb, h->d_pcal, h->d_pcalrot, npc, h->pcal_per_station, h->pcal_chunks,
                              h->pcal_maxbins, h->d_pcalbins, st));
      h->launches += 1;
    }
    if ((r = mark(0, false)) != GX_OK) return r;
    if ((r = mark(1, true)) != GX_OK) return r;
    if (h->tc)
      CKR(h, xmac_tc_launch(h->d_spec, nb, J.nchan, h->nfmain, J.ninputs, h->ks, h->hilo, h->d_scale, acc4,
                            b0 > 0 ? 1 : 0, h->d_err, st));
    else
      CKR(h, xmac_fp32_launch(h->d_spec, nb, J.ninputs, J.nchan, h->nfmain, h->ks, h->d_acc, h->d_err, st, h->xvar));
    if (h->nbins > 0) {   // pulsar binning: the binned cross products and weights of this pass
      const double *avgphase = reinterpret_cast<const double *>(h->d_sub + h->o_avgphase);
      const double *dmoff = reinterpret_cast<const double *>(h->d_sub + h->o_dmoff);
      CKR(h, binned_xmac_launch(h->d_binents, (int)h->binents.size(), h->d_spec, J.ninputs, J.nchan, nb, b0, avgphase,
                                dmoff, h->d_binphase, h->nbins, h->d_accb, st));
      CKR(h, binned_weights_launch(h->d_binitems, (int)h->binitems.size(), h->d_w, nb, b0, J.nchan,
                                   h->meta->num_buffered_ffts, h->xmac_stride, avgphase, dmoff, h->d_binphase,
                                   h->d_binweight, h->nbins, h->scrunch ? 1 : 0, h->d_wbins, st));
      h->launches += 2;
    }
    if (nzf) {   // zoom freqs: their rows of this pass's spectra, then their cross products
      CKR(h, zoom_gather_launch(h->d_zrows, nzr, h->d_spec, J.ninputs, J.nchan, h->d_specz, h->nzrows, h->nzchan, nb,
                                st));
      CKR(h, xmac_fp32_launch(h->d_specz, nb, h->nzrows, h->nzchan, nzf, h->zks, h->d_accz, h->d_err, st));
      h->launches += 2;
    }
    CKR(h, weights_launch(h->d_w, nb, d.nstations, h->d_pairs, npairs, h->d_wacc, st));
    if ((r = mark(1, false)) != GX_OK) return r;
    h->launches += 3;
    return GX_OK;
  };
  const int nph = h->cur_npc[k];
  if (h->kurt && (r = gx_kurtosis_begin(h, st)) != GX_OK) return r;
  if (nph > 1) {
    // Multiple phase centres (Core::processdata / uvshiftAndAverage,
    // core.cpp:984-991, 1431-1938): the accumulators of each uv-shift interval
    // are rotated per phase centre and added into the result array, the
    // autocorrelations added as they are
    CKR(h, cudaMemsetAsync(fin, 0, sizeof(float2) * h->rl_full, st));
    const int M = h->cur_M[k];
    const double *uvd = reinterpret_cast<const double *>(h->d_sub + h->o_uvdelay);
    for (int iv = 0; iv * M < J.blocks_per_send; iv++) {
      const int i0 = iv * M, i1 = std::min(J.blocks_per_send, i0 + M);
      if (iv > 0) CKR(h, cudaMemsetAsync(h->d_acc, 0, sizeof(float2) * h->acc_slice * h->ks, st));
      for (int b0 = i0; b0 < i1; b0 += h->chunk)
        if ((r = pass(b0, std::min(h->chunk, i1 - b0))) != GX_OK) return r;
      if ((r = mark(2, true)) != GX_OK) return r;
      CKR(h, uvshift_launch(h->d_uvents, (int)h->uvents.size(), h->d_acc, h->ks, h->acc_slice, J.nchan,
                            uvd + (size_t)iv * nbl * h->maxpc, nph, h->maxpc, h->d_uvfreqs, h->rsl, fin, st));
      if ((r = mark(2, false)) != GX_OK) return r;
      h->launches += 1;
    }
  } else {
    for (int b0 = 0; b0 < J.blocks_per_send; b0 += h->chunk)
      if ((r = pass(b0, std::min(h->chunk, J.blocks_per_send - b0))) != GX_OK) return r;
  }
  if (h->kurt && (r = gx_kurtosis_end(h, st)) != GX_OK) return r;
  if ((r = mark(2, true)) != GX_OK) return r;
  if (nph > 1) {
    // baseline and autocorrelation weights; the shift decorrelation factors
    CKR(h, finalise_launch(nullptr, 0, h->d_acc, h->ks, h->acc_slice, J.nchan, h->d_went, (int)h->wents.size(),
                           h->d_wacc, fin, st));
    CKR(h, copy_floats_launch(reinterpret_cast<const float *>(h->d_sub + h->o_bsd), 2 * h->bsd_count,
                              reinterpret_cast<float *>(fin), 2 * h->bsd_first, st));
    h->launches += 2;
  } else if (h->tc) {
    CKR(h, cudaMemsetAsync(fin, 0, sizeof(float2) * h->rl_full, st));
    CKR(h, finalise_tc_launch(h->d_tcprods, h->d_tcrows, (int)h->tcrows.size(), acc4, h->nfmain, J.nchan,
                              J.ninputs, h->ks, fin, st));
    CKR(h, finalise_launch(nullptr, 0, h->d_acc, h->ks, h->acc_slice, J.nchan, h->d_went, (int)h->wents.size(),
                           h->d_wacc, fin, st));
  } else if (h->nbins > 0) {
    // the autocorrelations and their weights as usual, the crosses from the bins
    CKR(h, cudaMemsetAsync(fin, 0, sizeof(float2) * h->rl_full, st));
    CKR(h, finalise_launch(h->d_autoprods, (int)h->autoprods.size(), h->d_acc, h->ks, h->acc_slice, J.nchan,
                           h->d_went, (int)h->wents.size(), h->d_wacc, fin, st));
    CKR(h, binned_finalise_launch(h->d_binents, (int)h->binents.size(), h->d_accb, J.nchan, h->nbins,
                                  h->scrunch ? 1 : 0, h->d_binweight, h->d_binwout, (int)h->binwout.size(), h->d_wbins,
                                  fin, st));
    h->launches += 1;
  } else {
    CKR(h, cudaMemsetAsync(fin, 0, sizeof(float2) * h->rl_full, st));
    CKR(h, finalise_launch(h->d_prods, (int)h->prods.size(), h->d_acc, h->ks, h->acc_slice, J.nchan, h->d_went,
                           (int)h->wents.size(), h->d_wacc, fin, st));
  }
  if (nph == 1) h->launches += (h->prods.empty() ? 0 : 1) + (h->wents.empty() ? 0 : 1);
  if (!h->zprods.empty()) {
    CKR(h, finalise_launch(h->d_zprods, (int)h->zprods.size(), h->d_accz, h->zks, h->zacc_slice, h->nzchan, nullptr,
                           0, nullptr, fin, st));
    h->launches += 1;
  }
  if (npc) {
    CKR(h, pcal_fold_launch(h->d_pcalbins, h->pcal_chunks, (long long)npc * h->pcal_maxbins, st));
    CKR(h, pcal_tones_launch(h->d_pcal, npc, 1, h->pcal_maxbins, h->d_pcalbins, fin, st));
    h->launches += h->pcal_chunks > 1 ? 2 : 1;
  }
  if (h->avg > 1) {
    CKR(h, cudaMemsetAsync(dev_results, 0, sizeof(float2) * h->rl, st));
    CKR(h, average_launch(h->d_avgtab, (int)h->avgtab.size(), h->d_full, dev_results, st));
    h->launches += 1;
  }
  if ((r = mark(2, false)) != GX_OK) return r;
  CKR(h, cudaMemcpyAsync(h->h_err + k, h->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  return GX_OK;
}

gx_status gx_stage_subint(gx_handle *h, const gx_subint_desc *sub, const uint8_t *const *devdata)
{
  return stage_subint(h, sub, devdata);
}

extern "C" {

// Runs one subint whose data buffers are already device pointers.
static gx_status run_device(gx_handle *h, const gx_subint_desc *sub, const uint8_t *const *devdata,
                            float2 *dev_results, cudaStream_t st)
{
  gx_status r = stage_subint(h, sub, devdata);
  if (r != GX_OK) return r;
  return gx_enqueue_subint(h, dev_results, st);
}

// Status the kernels of the last subint left in *d_err (read after a synchronise).
static gx_status kernel_status(gx_handle *h, int k = 0)
{
  if (h->h_err && h->h_err[k] != 0)
    return h->fail(GX_ERR_TIMEOUT, "an X-step wait expired (status " + std::to_string(h->h_err[k]) + ")");
  return GX_OK;
}

gx_status gx_subint_device(gx_handle *h, const gx_subint_desc *sub, float *dev_results, void *stream)
{
  if (!h || !sub || !dev_results || !sub->data || !sub->datalen || !sub->control) return GX_ERR_ARG;
  if (h->device < 0) return h->fail(GX_ERR_STATE, "host-only handle (opened with device -1)");
  if (!h->inflight.empty()) return h->fail(GX_ERR_STATE, "subints of gx_subint_async not yet waited for");
  CKR(h, cudaSetDevice(h->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
  h->last_stream = st;
  h->slot = 0;
  return run_device(h, sub, sub->data, reinterpret_cast<float2 *>(dev_results), st);
}

// Device buffers of slot k large enough for the subint's station data.
static gx_status ensure_data(gx_handle *h, int k, const gx_subint_desc *sub)
{
  for (int s = 0; s < h->jd.nstations; s++) {
    if (sub->datalen[s] < 0) return h->fail(GX_ERR_ARG, "negative data length");
    if (sub->datalen[s] > h->data_cap[k][s]) {
      if (h->d_data[k][s]) {
        CKR(h, cudaFree(h->d_data[k][s]));
        h->dev_bytes -= h->data_alloc[k][s];
      }
      h->d_data[k][s] = nullptr;
      CKR(h, h->dalloc(&h->d_data[k][s], sub->datalen[s] + 64));
      h->data_alloc[k][s] = sub->datalen[s] + 64;
      h->data_cap[k][s] = sub->datalen[s];
    }
  }
  return GX_OK;
}

gx_status gx_subint(gx_handle *h, const gx_subint_desc *sub, float *results)
{
  if (!h || !sub || !results || !sub->data || !sub->datalen || !sub->control) return GX_ERR_ARG;
  if (h->device < 0) return h->fail(GX_ERR_STATE, "host-only handle (opened with device -1)");
  if (!h->inflight.empty()) return h->fail(GX_ERR_STATE, "subints of gx_subint_async not yet waited for");
  CKR(h, cudaSetDevice(h->device));
  gx_status r = ensure_data(h, 0, sub);
  if (r != GX_OK) return r;
  const gx_job_desc &d = h->jd;
  for (int s = 0; s < d.nstations; s++)
    if (sub->datalen[s] > 0)
      CKR(h, cudaMemcpyAsync(h->d_data[0][s], sub->data[s], sub->datalen[s], cudaMemcpyHostToDevice, h->stream));
  h->slot = 0;
  r = run_device(h, sub, h->d_data[0].data(), h->d_results, h->stream);
  if (r != GX_OK) return r;
  CKR(h, cudaMemcpyAsync(results, h->d_results, sizeof(float2) * h->rl, cudaMemcpyDeviceToHost, h->stream));
  CKR(h, cudaStreamSynchronize(h->stream));
  return kernel_status(h);
}

gx_status gx_subint_async(gx_handle *h, const gx_subint_desc *sub, float *results)
{
  if (!h || !sub || !results || !sub->data || !sub->datalen || !sub->control) return GX_ERR_ARG;
  if (h->device < 0) return h->fail(GX_ERR_STATE, "host-only handle (opened with device -1)");
  if ((int)h->inflight.size() >= gx_handle::kSlots)
    return h->fail(GX_ERR_STATE, "two subints in flight: gx_subint_wait for one first");
  CKR(h, cudaSetDevice(h->device));
  if (!h->copy_stream) CKR(h, cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
  // the other slot than the one in flight; its last subint has been waited for,
  // so its kernels no longer read its data buffers
  const int k = h->inflight.empty() ? 0 : 1 - h->inflight.back();
  gx_status r = ensure_data(h, k, sub);
  if (r != GX_OK) return r;
  const gx_job_desc &d = h->jd;
  for (int s = 0; s < d.nstations; s++)
    if (sub->datalen[s] > 0)
      CKR(h, cudaMemcpyAsync(h->d_data[k][s], sub->data[s], sub->datalen[s], cudaMemcpyHostToDevice,
                             h->copy_stream));
  CKR(h, cudaEventRecord(h->ev_copied[k], h->copy_stream));
  h->slot = k;
  r = stage_subint(h, sub, h->d_data[k].data());
  if (r == GX_OK) {
    // the kernels start once this subint's data is in and the previous subint's work is done
    r = h->cuda(cudaStreamWaitEvent(h->stream, h->ev_copied[k], 0), "cudaStreamWaitEvent");
    if (r == GX_OK) r = gx_enqueue_subint(h, h->d_results, h->stream);
  }
  h->slot = 0;
  if (r != GX_OK) return r;
  CKR(h, cudaMemcpyAsync(results, h->d_results, sizeof(float2) * h->rl, cudaMemcpyDeviceToHost, h->stream));
  CKR(h, cudaEventRecord(h->ev_done[k], h->stream));
  h->last_stream = h->stream;
  h->inflight.push_back(k);
  return GX_OK;
}

gx_status gx_subint_wait(gx_handle *h)
{
  if (!h) return GX_ERR_ARG;
  if (h->inflight.empty()) return h->fail(GX_ERR_STATE, "no subint of gx_subint_async in flight");
  const int k = h->inflight.front();
  h->inflight.pop_front();
  CKR(h, cudaSetDevice(h->device));
  CKR(h, cudaEventSynchronize(h->ev_done[k]));
  return kernel_status(h, k);
}

gx_status gx_synchronize(gx_handle *h)
{
  if (!h) return GX_ERR_ARG;
  if (h->device < 0) return GX_OK;
  CKR(h, cudaStreamSynchronize(h->stream));
  if (h->last_stream && h->last_stream != h->stream) CKR(h, cudaStreamSynchronize(h->last_stream));
  return kernel_status(h);
}

gx_status gx_stage_times(gx_handle *h, float ms[3])
{
  if (!h || !ms) return GX_ERR_ARG;
  ms[0] = ms[1] = ms[2] = 0.f;
  for (size_t i = 0; i + 1 < h->evs.size(); i += 2) {
    CKR(h, cudaEventSynchronize(h->evs[i + 1]));
    float t = 0;
    CKR(h, cudaEventElapsedTime(&t, h->evs[i], h->evs[i + 1]));
    int stg = h->ev_stage[i / 2];
    if (stg >= 0 && stg < 3) ms[stg] += t;
  }
  return GX_OK;
}

gx_status gx_launch_count(const gx_handle *h, int *count)
{
  if (!h || !count) return GX_ERR_ARG;
  *count = h->launches;
  return GX_OK;
}

gx_status gx_spectra(gx_handle *h, int station, int block, float *out, float *weight)
{
  if (!h || !out || !weight) return GX_ERR_ARG;
  if (h->device < 0 || !h->have_last) return h->fail(GX_ERR_STATE, "no subint has been processed yet");
  const DevJob &J = h->J;
  if (station < 0 || station >= J.nstations || block < 0 || block >= J.blocks_per_send)
    return h->fail(GX_ERR_ARG, "station or block out of range");
  CKR(h, cudaSetDevice(h->device));
  CKR(h, fstep_launch(J, h->d_st, h->maxnrf, h->last, block, 1, h->nslots, h->d_spec1, h->d_w1, h->d_bp1,
                      h->stream));
  const gx_station_desc &x = h->jd.stations[station];
  for (int b = 0; b < x.nbands; b++) {
    int f = x.recfreq[x.band_localfreq[b]];
    const float2 *src = h->d_spec1 + ((size_t)f * J.ninputs + h->band_input[station][b]) * J.nchan;
    CKR(h, cudaMemcpyAsync(out + 2 * (size_t)b * J.nchan, src, sizeof(float2) * J.nchan, cudaMemcpyDeviceToHost,
                           h->stream));
  }
  CKR(h, cudaMemcpyAsync(weight, h->d_w1 + station, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
  CKR(h, cudaStreamSynchronize(h->stream));
  return GX_OK;
}

gx_status gx_interpolator(gx_handle *h, int station, int scan, int sec, int ns, double out[3])
{
  if (!h || !out) return GX_ERR_ARG;
  if (!h->model) return h->fail(GX_ERR_STATE, "handle has no delay model (open it with gx_open_input)");
  return h->model->interpolator(station, scan, sec, ns, out);
}

gx_status gx_scan_start_sec(gx_handle *h, int scan, double *out)
{
  if (!h || !out) return GX_ERR_ARG;
  if (!h->model) return h->fail(GX_ERR_STATE, "handle has no delay model");
  *out = h->model->scan_start_sec(scan);
  return GX_OK;
}

gx_status gx_open_input(const char *inputfile, int device, int xstep, gx_handle **out)
{
  if (!inputfile || !out) return GX_ERR_ARG;
  *out = nullptr;
  std::string err;
  std::unique_ptr<InputJob> job(read_input_job(inputfile, err));
  if (!job) {
    fprintf(stderr, "gx_open_input: %s\n", err.c_str());
    return GX_ERR_IO;
  }
  job->desc.xstep = xstep;
  return open_handle(&job->desc, device, std::move(job->model),
                     std::unique_ptr<gx::JobMeta>(new gx::JobMeta(job->meta)), out);
}

}  // extern "C"

gx_status gx_set_tc_scales(gx_handle *h, int station, int band, const float *scales)
{
  if (!h || !scales) return GX_ERR_ARG;
  if (!h->tc || h->device < 0) return h->fail(GX_ERR_STATE, "handle has no tensor-core X-step on a device");
  if (station < 0 || station >= h->jd.nstations || band < 0 || band >= h->jd.stations[station].nbands)
    return h->fail(GX_ERR_ARG, "station or band out of range");
  const int N = h->J.nchan;
  std::vector<float> row(N);
  for (int c = 0; c < N; c++) {
    const float s = scales[c];
    if (!(s > 0.0f) || !std::isfinite(s)) return h->fail(GX_ERR_ARG, "scales must be finite and positive");
    row[c] = (float)std::ldexp(1.0, (int)std::lround(std::log2((double)s)));
  }
  const gx_station_desc &x = h->jd.stations[station];
  const int f = x.recfreq[x.band_localfreq[band]];
  const size_t off = ((size_t)f * kTcInputs + h->band_input[station][band]) * N;
  CKR(h, cudaSetDevice(h->device));
  CKR(h, cudaMemcpyAsync(h->d_scale + off, row.data(), sizeof(float) * N, cudaMemcpyHostToDevice, h->stream));
  CKR(h, cudaStreamSynchronize(h->stream));
  return GX_OK;
}
