// Host-side setup readers: .input / .calc / .im and the delay model.
#pragma once
#include <memory>
#include <string>
#include <vector>
#include "../../include/gxcorr.h"

namespace gx {

// Per-scan delay polynomials (Model's scantable, mpifxcorr/src/model.h).
struct ModelScan {
  int offsetseconds = 0;      // SCAN n START (S)
  int durationseconds = 0;
  int numphasecentres = 1;
  int nsamples = 0;
  int polystartmjd = 0, polystartseconds = 0;
  int phase_centre_source = 0;   // .calc SCAN n PHS CTR 0: source table index of the phase centre
  int maxns_xc = 0;              // SCAN n UVSHIFT INTERVAL (NS): cross-correlation shift/average time
  int pointing_source = 0;       // SCAN n POINTING SRC
  std::vector<int> phase_centre_sources;   // SCAN n PHS CTR j: source table index of phase centre j
  // delay[sample][source][station][order+1], us; source 0 = pointing centre
  std::vector<double> delay;
  std::vector<double> u, v, w;   // same indexing, metres
};

// Model::calculateDelayInterpolator and Mode::setOffsets (model.cpp:219-289,
// mode.cpp:1502-1532), with the clock terms folded in as Model::addClockTerms
// does (model.cpp:291-352).
class HostModel {
 public:
  int polyorder = 0, modelincsecs = 0;
  int modelmjd = 0, modelstartseconds = 0;
  int jobmjd = 0, jobseconds = 0;
  int nstations = 0;
  std::vector<ModelScan> scans;
  std::vector<int> station_of_datastream;   // model antenna index per datastream
  std::vector<int> intclockseconds;         // per datastream
  std::vector<double> maxrate;              // per model antenna: Model::getMaxRate (us/s)
  double timespan_s = 0;                    // blockspersend * fftchannels * sampletime / 1e6
  int blocks_per_send = 0;

  double delay_at(const ModelScan &sc, int sample, int src, int ant, int l) const
  {
    return sc.delay[(((size_t)sample * (sc.numphasecentres + 1) + src) * nstations + ant) * (polyorder + 1) + l];
  }
  gx_status interpolator(int datastream, int scan, int sec, int ns, double out[3]) const;
  // Model::calculateDelayInterpolator of order 1 over 1 us with one increment
  // (the uv-shift's delay and rate of model antenna ant, source src of the
  // scan's table, at offsettime seconds after the scan start; core.cpp:1652-1657)
  bool linear(int scan, double offsettime, int ant, int src, double out[2]) const;
  double scan_start_sec(int scan) const;
  // Model::calculateDelayInterpolator of order 0 (model.cpp:232-248): the
  // delay (us, clock included) of datastream ds at offsettime seconds after
  // the scan start, for the source DataStream::calculateControlParams asks
  // for (datastream.cpp:375-377); false outside the scan's model samples.
  bool delay0(int ds, int scan, double offsettime, double *out) const;
  // Model::interpolateUVW (model.cpp:177-217): baseline (u, v, w) of model
  // antennas ant1 - ant2 at offsettime seconds after the scan start, source
  // src of the scan's table (1: first phase centre).
  bool uvw(int scan, double offsettime, int ant1, int ant2, int src, double out[3]) const;
};

// One polyco (Polyco::loadPolycoFile, polyco.cpp:399-524): pulse phase and
// frequency as polynomials in minutes from its centre time.
struct PolycoEntry {
  int mjd = 0;
  double mjdfraction = 0, dm = 0, f0 = 0, refphase = 0, obsfreq = 0;
  int timespan = 0;                     // minutes
  std::vector<double> phasecoef, freqcoef;
};

// PULSAR CONFIG FILE of a configuration (Configuration::processPulsarConfig,
// configuration.cpp:3400-3498) and the polycos of its files.
struct PulsarConfig {
  int nbins = 0;
  bool scrunch = false;
  std::vector<double> binphaseends, binweights;
  std::vector<PolycoEntry> polycos;
  // Polyco::getCurrentPolyco (polyco.cpp:349-366): the first whose span
  // (plus a second) covers mjd + mjdfraction; -1: none
  int current(int mjd, double mjdfraction) const;
};

// Job-level .input facts the visibility writer needs (Configuration).
struct JobMeta {
  int start_mjd = 0, start_seconds = 0, execute_seconds = 0;
  double int_time = 0;                 // INT TIME (SEC)
  std::vector<int> telescope;          // TELESCOPE INDEX per datastream
  std::vector<double> tsys;            // TSYS per datastream
  std::vector<std::string> telescope_name;   // TELESCOPE NAME per telescope
  int num_buffered_ffts = 1;           // NUM BUFFERED FFTS
  int data_buffer_factor = 0, num_data_segments = 0;   // DATA BUFFER FACTOR, NUM DATA SEGMENTS
  std::shared_ptr<PulsarConfig> pulsar;   // PULSAR BINNING: the bins and polycos
};

struct InputJob {
  gx_job_desc desc{};
  std::vector<gx_station_desc> stations;
  std::vector<gx_freq_desc> freqs;
  std::vector<gx_baseline_desc> baselines;
  std::unique_ptr<HostModel> model;
  int start_mjd = 0, start_seconds = 0, execute_seconds = 0;
  double int_time = 0;
  std::vector<std::string> datafiles;   // first file of each datastream
  JobMeta meta;
};

InputJob *read_input_job(const char *inputfile, std::string &err);

}  // namespace gx

using gx::HostModel;
using gx::InputJob;
using gx::read_input_job;
