// GpuMode: the per-FFT compatibility path of gxcorr inside mpifxcorr.
//
// What a DiFX maintainer adds to mpifxcorr/src beside gpucore.h, for code
// that keeps reading spectra block by block through the Mode interface
// (mode.h:40-197) -- the reference's own XMAC loop in Core::processdata, or
// any other consumer of Mode::getFreqs.  A GpuMode is the Mk5Mode that
// Configuration::getMode builds for a VDIF datastream (configuration.cpp:
// 932-998), so getFreqs, getConjugatedFreqs, getDataWeight,
// getAutocorrelation and getWeight are Mode's own accessors over Mode's own
// arrays; process() fills those arrays from the GPU instead of unpacking and
// transforming on the host: the block's spectra and data weight come from the
// gxcorr handle that correlated the current slot (gx_spectra), then the
// conjugates, autocorrelations, cross-polarisation autocorrelations and
// weights are formed as Mode::process forms them (mode.cpp:1262-1351).
//
// Edit this needs in mode.h: `virtual` before `void process(int index, int
// subloopindex)` (mode.h:81), so that Core's calls through Mode* reach it
// (and configuration.h's `friend class GpuMode;` for create()).  Not covered:
// INTERLACEDVDIF per-band weights, linear-to-circular conversion, kurtosis,
// phase-cal (gxcorr forms phase-cal tones in its own result array).
#pragma once
#include <vector>
#include "configuration.h"
#include "gxcorr.h"
#include "mk5mode.h"

class GpuMode : public Mk5Mode {
 public:
  // The Mode of VDIF datastream dsindex of configuration configindex, its
  // spectra read from handle h (NULL if the datastream is not plain VDIF).
  static GpuMode *create(Configuration *conf, int configindex, int dsindex, gx_handle *h);

  // Mode::process (mode.cpp:634-1374) for FFT block index of the slot h last
  // correlated, into subloop slot subloopindex.
  void process(int index, int subloopindex);

 private:
  GpuMode(gx_handle *h, Configuration *conf, int confindex, int dsindex, int recordedbandchan, int chanstoavg,
          int bpersend, int gsamples, int nrecordedfreqs, double recordedbw, double *recordedfreqclkoffs,
          double *recordedfreqclkoffsdelta, double *recordedfreqphaseoffs, double *recordedfreqlooffs,
          int nrecordedbands, int nzoombands, int nbits, Configuration::datasampling sampling,
          Configuration::complextype tcomplex, bool fbank, bool linear2circular, int fringerotorder,
          int arraystridelen, bool cacorrs, int framebytes, int framesamples, Configuration::dataformat format);
  gx_handle *gx;
  std::vector<float> buf;   // [nbands][nchan] complex
};
