// GpuMode (see gpumode.h): Mode's arrays filled from gx_spectra.
#include "gpumode.h"

#include <cstring>

GpuMode::GpuMode(gx_handle *h, Configuration *conf, int confindex, int dsindex, int recordedbandchan, int chanstoavg,
                 int bpersend, int gsamples, int nrecordedfreqs, double recordedbw, double *recordedfreqclkoffs,
                 double *recordedfreqclkoffsdelta, double *recordedfreqphaseoffs, double *recordedfreqlooffs,
                 int nrecordedbands, int nzoombands, int nbits, Configuration::datasampling sampling,
                 Configuration::complextype tcomplex, bool fbank, bool linear2circular, int fringerotorder,
                 int arraystridelen, bool cacorrs, int framebytes, int framesamples, Configuration::dataformat format)
    : Mk5Mode(conf, confindex, dsindex, recordedbandchan, chanstoavg, bpersend, gsamples, nrecordedfreqs, recordedbw,
              recordedfreqclkoffs, recordedfreqclkoffsdelta, recordedfreqphaseoffs, recordedfreqlooffs,
              nrecordedbands, nzoombands, nbits, sampling, tcomplex, fbank, linear2circular, fringerotorder,
              arraystridelen, cacorrs, framebytes, framesamples, format),
      gx(h), buf(2 * (size_t)nrecordedbands * recordedbandchan)
{
}

GpuMode *GpuMode::create(Configuration *c, int ci, int ds, gx_handle *h)
{
  // the arguments of Configuration::getMode's VDIF branch (configuration.cpp:932-998)
  const Configuration::configdata &conf = c->configs[ci];
  const Configuration::datastreamdata &stream = c->datastreamtable[conf.datastreamindices[ds]];
  if (stream.format != Configuration::VDIF || stream.linear2circular || stream.filterbank) return nullptr;
  const Configuration::freqdata &f0 = c->freqtable[stream.recordedfreqtableindices[0]];
  const int guardsamples = (int)(conf.guardns / (1000.0 / (f0.bandwidth * 2.0)) + 0.5);
  int framesamples = c->getFramePayloadBytes(ci, ds) * 8 /
                     (c->getDNumBits(ci, ds) * c->getDNumRecordedBands(ci, ds) * f0.decimationfactor);
  const int framebytes = c->getFrameBytes(ci, ds);
  if (stream.sampling == Configuration::COMPLEX) framesamples /= 2;
  return new GpuMode(h, c, ci, ds, f0.numchannels, f0.channelstoaverage, conf.blockspersend, guardsamples,
                     stream.numrecordedfreqs, f0.bandwidth, stream.recordedfreqclockoffsets,
                     stream.recordedfreqclockoffsetsdelta, stream.recordedfreqphaseoffset,
                     stream.recordedfreqlooffsets, stream.numrecordedbands, stream.numzoombands, stream.numbits,
                     stream.sampling, stream.tcomplex, stream.filterbank, stream.linear2circular,
                     conf.fringerotationorder, conf.arraystridelen[ds], conf.writeautocorrs, framebytes,
                     framesamples, stream.format);
}

void GpuMode::process(int index, int subloopindex)
{
  const int nc = recordedbandchannels;
  float w = 0.0f;
  if (gx_spectra(gx, datastreamindex, index, buf.data(), &w) != GX_OK) {
    w = 0.0f;   // a block the device could not produce counts as invalid (zeroed, weight 0)
    std::fill(buf.begin(), buf.end(), 0.0f);
  }
  dataweight[subloopindex] = w;
  for (int j = 0; j < numrecordedbands; j++) {
    cf32 *f = fftoutputs[j][subloopindex];
    cf32 *cj = conjfftoutputs[j][subloopindex];
    memcpy(f, buf.data() + 2 * (size_t)j * nc, sizeof(cf32) * nc);
    for (int c = 0; c < nc; c++) {   // vectorConj_cf32
      cj[c].re = f[c].re;
      cj[c].im = -f[c].im;
    }
  }
  if (w <= 0.0f) return;   // zeroed block: no autocorrelation, no weight (mode.cpp:743-754)
  for (int j = 0; j < numrecordedbands; j++) {
    // autocorrelation f conj(f) and its weight (mode.cpp:1270-1284)
    const cf32 *f = fftoutputs[j][subloopindex], *cj = conjfftoutputs[j][subloopindex];
    cf32 *a = autocorrelations[0][j];
    for (int c = 0; c < nc; c++) {
      a[c].re += f[c].re * cj[c].re - f[c].im * cj[c].im;
      a[c].im += f[c].re * cj[c].im + f[c].im * cj[c].re;
    }
    weights[0][j] += w;
  }
  if (!calccrosspolautocorrs) return;
  for (int i = 0; i < numrecordedfreqs; i++) {
    // the first two recorded bands of local freq i (mode.cpp:1138-1150, 1333-1351)
    int idx[2], count = 0;
    for (int j = 0; j < numrecordedbands && count < 2; j++)
      if (config->getDLocalRecordedFreqIndex(configindex, datastreamindex, j) == i) idx[count++] = j;
    if (count < 2) continue;
    for (int k = 0; k < 2; k++) {
      const cf32 *f = fftoutputs[idx[k]][subloopindex], *cj = conjfftoutputs[idx[1 - k]][subloopindex];
      cf32 *a = autocorrelations[1][idx[k]];
      for (int c = 0; c < nc; c++) {
        a[c].re += f[c].re * cj[c].re - f[c].im * cj[c].im;
        a[c].im += f[c].re * cj[c].im + f[c].im * cj[c].re;
      }
      weights[1][idx[k]] += w;
    }
  }
}
