// Readers for the DiFX job setup files and the host delay model.
//
//   .input  -- the tables Configuration parses (mpifxcorr/src/configuration.cpp:
//              parseConfiguration 198-345, processCommon 1271, processConfig 1315,
//              processFreqTable 1970, processTelescopeTable 2025,
//              processDatastreamTable 1397-1885, processBaselineTable 1033-1180,
//              processDataTable 1956).  A "KEY: value" line has its value from
//              column 20 or after the colon, whichever is later
//              (getinputkeyval, configuration.cpp:3640-3655); '@' starts a comment.
//   .calc   -- Model::readCommonData/readStationData/readScanData (model.cpp:391-527).
//   .im     -- Model::readPolynomialSamples (model.cpp:596-837).
//
// Only the first configuration is read, and the features the device path does
// not implement (pulsar binning, phased array, multiple phase centres,
// PHASE CAL DIVISOR other than 1) are rejected with a message.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>
#include <string>
#include <utility>
#include <vector>
#include "gx_host.h"

namespace gx {

namespace {

struct KVFile {
  struct Item { std::string key, val; int section; };
  std::vector<Item> items;
  std::vector<std::string> sections;
  size_t pos = 0;
  std::string err;

  static std::string rtrim(std::string s)
  {
    while (!s.empty() && (s.back() == '\r' || s.back() == '\n' || s.back() == ' ' || s.back() == '\t')) s.pop_back();
    return s;
  }

  bool load(const std::string &path)
  {
    std::ifstream in(path);
    if (!in) { err = "cannot open " + path; return false; }
    std::string line;
    int sec = -1;
    while (std::getline(in, line)) {
      line = rtrim(line);
      if (line.empty()) continue;
      if (line[0] == '#') { sections.push_back(line); sec = (int)sections.size() - 1; continue; }
      if (line[0] == '@') continue;
      size_t colon = line.find(':');
      if (colon == std::string::npos) { items.push_back({line, "", sec}); continue; }
      size_t vstart = colon + 1 < 20 ? 20 : colon + 1;
      std::string val = vstart < line.size() ? line.substr(vstart) : std::string();
      items.push_back({line.substr(0, colon), val, sec});
    }
    return true;
  }

  // next item whose key starts with prefix; the reference reads strictly in order
  bool get(const std::string &prefix, std::string &val)
  {
    if (pos >= items.size()) { err = "end of file looking for '" + prefix + "'"; return false; }
    const Item &it = items[pos];
    if (it.key.compare(0, prefix.size(), prefix) != 0) {
      err = "expected '" + prefix + "', found '" + it.key + "'";
      return false;
    }
    val = it.val;
    pos++;
    return true;
  }
  bool peek(const std::string &prefix) const
  {
    return pos < items.size() && items[pos].key.compare(0, prefix.size(), prefix) == 0;
  }
  bool seek_section(const std::string &title)
  {
    for (size_t i = 0; i < items.size(); i++)
      if (items[i].section >= 0 && sections[items[i].section].compare(0, title.size(), title) == 0) {
        pos = i;
        return true;
      }
    err = "section '" + title + "' not found";
    return false;
  }
  const std::string *find(const std::string &key) const
  {
    for (const auto &it : items)
      if (it.key == key) return &it.val;
    return nullptr;
  }
};

bool truthy(const std::string &v)
{
  std::string s = KVFile::rtrim(v);
  size_t a = s.find_first_not_of(' ');
  s = a == std::string::npos ? "" : s.substr(a);
  return s == "TRUE" || s == "T" || s == "true" || s == "t";
}

std::string strip(const std::string &v)
{
  size_t a = v.find_first_not_of(" \t");
  if (a == std::string::npos) return "";
  return KVFile::rtrim(v.substr(a));
}

int get_mjd(int year, int month, int day)  // Configuration::getMJD, configuration.cpp:3721-3726
{
  return year * 367 - int(7 * (year + int((month + 9) / 12)) / 4) + int(275 * month / 9) + day - 678987;
}

std::string dir_of(const std::string &path)
{
  size_t p = path.find_last_of('/');
  return p == std::string::npos ? std::string() : path.substr(0, p + 1);
}

std::string resolve(const std::string &file, const std::string &relto)
{
  std::string f = strip(file);
  if (f.empty() || f[0] == '/') return f;
  std::ifstream t(f);
  if (t) return f;
  return dir_of(relto) + f;
}

// Polycos of one file, in order (Polyco::loadPolycoFile, polyco.cpp:399-524):
// two header lines, then the coefficients three to a line, D exponents allowed.
bool read_polycos(const std::string &path, std::vector<PolycoEntry> &out, std::string &err)
{
  std::ifstream in(path);
  if (!in) { err = "cannot open polyco file " + path; return false; }
  std::vector<std::string> lines;
  std::string line;
  while (std::getline(in, line))
    if (line.find_first_not_of(" \t\r\n") != std::string::npos) lines.push_back(line);
  size_t i = 0;
  while (i + 2 <= lines.size()) {
    PolycoEntry P;
    std::istringstream a(lines[i]), b(lines[i + 1]);
    std::string name, date, utc;
    double mjdd = 0;
    if (!(a >> name >> date >> utc >> mjdd >> P.dm)) { err = "polyco header line 1: " + path; return false; }
    P.mjd = int(mjdd);
    P.mjdfraction = mjdd - P.mjd;
    std::string obs;
    int ncoef = 0;
    if (!(b >> P.refphase >> P.f0 >> obs >> P.timespan >> ncoef >> P.obsfreq) || ncoef < 2 || ncoef > 64) {
      err = "polyco header line 2: " + path;
      return false;
    }
    P.refphase = P.refphase - std::floor(P.refphase);
    i += 2;
    std::vector<double> c;
    while ((int)c.size() < ncoef) {
      if (i >= lines.size()) { err = "polyco coefficients: " + path; return false; }
      std::istringstream cs(lines[i++]);
      std::string tok;
      while ((int)c.size() < ncoef && cs >> tok) {
        for (char &ch : tok)
          if (ch == 'D' || ch == 'd') ch = 'E';
        c.push_back(atof(tok.c_str()));
      }
    }
    // frequency and phase coefficients (polyco.cpp:506-515)
    P.freqcoef.assign(ncoef, 0.0);
    P.freqcoef[0] = P.f0 + c[1] / 60.0;
    P.freqcoef[ncoef - 1] = 0.0;
    for (int k = 1; k < ncoef - 1; k++) P.freqcoef[k] = (k + 1) * c[k + 1] / 60.0;
    P.phasecoef.assign(ncoef, 0.0);
    P.phasecoef[0] = P.refphase + c[0];
    P.phasecoef[1] = 60.0 * P.f0 + c[1];
    for (int k = 2; k < ncoef; k++) P.phasecoef[k] = c[k];
    out.push_back(P);
  }
  if (out.empty()) { err = "no polycos in " + path; return false; }
  return true;
}

#define NEED(kv, key, var)          \
  do {                              \
    if (!(kv).get((key), (var))) {  \
      err = (kv).err;               \
      return nullptr;               \
    }                               \
  } while (0)

}  // namespace

double HostModel::scan_start_sec(int scan) const
{
  // Model::getScanStartSec (model.h:115)
  return (double)((modelmjd - jobmjd) * 86400 + (modelstartseconds - jobseconds) + scans[scan].offsetseconds);
}

bool HostModel::uvw(int scanindex, double offsettime, int ant1, int ant2, int src, double out[3]) const
{
  if (scanindex < 0 || scanindex >= (int)scans.size()) return false;
  const ModelScan &sc = scans[scanindex];
  if (sc.u.empty() || ant1 < 0 || ant2 < 0 || ant1 >= nstations || ant2 >= nstations || src < 0 ||
      src > sc.numphasecentres)
    return false;
  const int polyoffset = (modelmjd - sc.polystartmjd) * 86400 + modelstartseconds + sc.offsetseconds - sc.polystartseconds;
  int scansample = int((offsettime + polyoffset) / double(modelincsecs));
  if (scansample == sc.nsamples && ((offsettime + polyoffset - scansample * modelincsecs) < modelincsecs / 1000000.0))
    scansample--;
  if (scansample < 0 || scansample >= sc.nsamples) return false;
  const double deltat = offsettime + polyoffset - scansample * modelincsecs;
  double tp[16];
  tp[0] = 1.0;
  for (int i = 0; i < polyorder; i++) tp[i + 1] = tp[i] * deltat;
  const std::vector<double> *tabs[3] = {&sc.u, &sc.v, &sc.w};
  for (int c = 0; c < 3; c++) {
    const double *c1 = &(*tabs[c])[(((size_t)scansample * (sc.numphasecentres + 1) + src) * nstations + ant1) *
                                    (polyorder + 1)];
    const double *c2 = &(*tabs[c])[(((size_t)scansample * (sc.numphasecentres + 1) + src) * nstations + ant2) *
                                    (polyorder + 1)];
    double a = 0, b = 0;   // dot products in index order (genericDotProduct_64f)
    for (int i = 0; i <= polyorder; i++) a += tp[i] * c1[i];
    for (int i = 0; i <= polyorder; i++) b += tp[i] * c2[i];
    out[c] = a - b;
  }
  return true;
}

int PulsarConfig::current(int mjd, double mjdfraction) const
{
  for (size_t i = 0; i < polycos.size(); i++) {
    const PolycoEntry &P = polycos[i];
    const double differencemins = (mjd - P.mjd) * 1440 + (mjdfraction - P.mjdfraction) * 1440;
    const double rangemins = double(P.timespan) / 2.0 + 1.0 / 60.0;   // an extra second against roundoff
    if (differencemins <= rangemins && differencemins >= -rangemins) return (int)i;
  }
  return -1;
}

bool HostModel::linear(int scanindex, double offsettime, int ant, int src, double out[2]) const
{
  if (scanindex < 0 || scanindex >= (int)scans.size()) return false;
  const ModelScan &sc = scans[scanindex];
  if (ant < 0 || ant >= nstations || src < 0 || src > sc.numphasecentres) return false;
  const double timespan = 0.000001;
  // Model::calculateDelayInterpolator, order 1 (model.cpp:232-281)
  const int polyoffset = (modelmjd - sc.polystartmjd) * 86400 + modelstartseconds + sc.offsetseconds - sc.polystartseconds;
  int scansample = int((offsettime + polyoffset) / double(modelincsecs));
  if (scansample == sc.nsamples && ((offsettime + polyoffset - scansample * modelincsecs) < 1e-6)) scansample--;
  if (scansample < 0 || scansample >= sc.nsamples) return false;
  double tp[16];
  double samples[3];
  // the block-centre sample first, then the start and the end, as the reference forms them
  const double deltas[3] = {offsettime + polyoffset - scansample * modelincsecs,
                            offsettime + polyoffset + timespan / 2.0 - scansample * modelincsecs,
                            offsettime + polyoffset + timespan - scansample * modelincsecs};
  for (int q = 0; q < 3; q++) {
    tp[0] = 1.0;
    for (int i = 0; i < polyorder; i++) tp[i + 1] = tp[i] * deltas[q];
    double acc = 0;
    for (int i = 0; i < polyorder + 1; i++) acc += tp[i] * delay_at(sc, scansample, src, ant, i);
    samples[q] = acc;
  }
  const int numincrements = 1;
  out[0] = (samples[2] - samples[0]) / numincrements;
  out[1] = samples[0] + (samples[1] - (out[0] * numincrements / 2.0 + samples[0])) / 3.0;
  return true;
}

bool HostModel::delay0(int ds, int scanindex, double offsettime, double *out) const
{
  if (scanindex < 0 || scanindex >= (int)scans.size()) return false;
  const ModelScan &sc = scans[scanindex];
  const int ant = station_of_datastream[ds];
  const int srcindex = (sc.numphasecentres == 1) ? 1 : 0;
  const int polyoffset = (modelmjd - sc.polystartmjd) * 86400 + modelstartseconds + sc.offsetseconds - sc.polystartseconds;
  int scansample = int((offsettime + polyoffset) / double(modelincsecs));
  if (scansample == sc.nsamples && ((offsettime + polyoffset - scansample * modelincsecs) < 1e-6)) scansample--;
  if (scansample < 0 || scansample >= sc.nsamples) return false;
  // a zero time span: the polynomial at offsettime itself
  const double dt = offsettime + polyoffset + 0.0 / 2.0 - scansample * modelincsecs;
  double tp[16];
  tp[0] = 1.0;
  for (int i = 0; i < polyorder; i++) tp[i + 1] = tp[i] * dt;
  double acc = 0;
  for (int i = 0; i < polyorder + 1; i++) acc += tp[i] * delay_at(sc, scansample, srcindex, ant, i);
  *out = acc;
  return true;
}

gx_status HostModel::interpolator(int ds, int scanindex, int sec, int ns, double out[3]) const
{
  if (scanindex < 0 || scanindex >= (int)scans.size()) return GX_ERR_MODEL;
  const ModelScan &sc = scans[scanindex];
  const int ant = station_of_datastream[ds];
  const int srcindex = (sc.numphasecentres == 1) ? 1 : 0;   // Mode::setOffsets, mode.cpp:1518-1521
  const double offsettime = (double)sec + ((double)ns) / 1000000000.0;
  const double timespan = timespan_s;
  const long long numincrements = blocks_per_send;
  // Model::calculateDelayInterpolator, order 2 (model.cpp:219-289)
  const int polyoffset = (modelmjd - sc.polystartmjd) * 86400 + modelstartseconds + sc.offsetseconds - sc.polystartseconds;
  int scansample = int((offsettime + polyoffset) / double(modelincsecs));
  if (scansample == sc.nsamples && ((offsettime + polyoffset - scansample * modelincsecs) < 1e-6)) scansample--;
  if (scansample < 0 || scansample >= sc.nsamples) return GX_ERR_MODEL;
  double tp[16];
  double samples[3];
  const double deltas[3] = {offsettime + polyoffset - scansample * modelincsecs,
                            offsettime + polyoffset + timespan / 2.0 - scansample * modelincsecs,
                            offsettime + polyoffset + timespan - scansample * modelincsecs};
  for (int q = 0; q < 3; q++) {
    tp[0] = 1.0;
    for (int i = 0; i < polyorder; i++) tp[i + 1] = tp[i] * deltas[q];
    double acc = 0;
    for (int i = 0; i < polyorder + 1; i++) acc += tp[i] * delay_at(sc, scansample, srcindex, ant, i);
    samples[q] = acc;
  }
  // The reference forms numincrements*numincrements in int; this keeps it in 64 bits
  // (identical whenever blockspersend <= 46340).
  out[0] = (2.0 * samples[0] - 4.0 * samples[1] + 2.0 * samples[2]) / (double)(numincrements * numincrements);
  out[1] = (-3.0 * samples[0] + 4.0 * samples[1] - samples[2]) / numincrements;
  out[2] = samples[0];
  out[2] -= 1000000 * intclockseconds[ds];   // mode.cpp:1526
  return GX_OK;
}

InputJob *read_input_job(const char *inputfile, std::string &err)
{
  KVFile in;
  if (!in.load(inputfile)) { err = in.err; return nullptr; }
  std::unique_ptr<InputJob> job(new InputJob());
  std::string v;

  // ------------------------------------------------------------- COMMON
  if (!in.seek_section("# COMMON SETTINGS")) { err = in.err; return nullptr; }
  std::string calcfile;
  NEED(in, "CALC FILENAME", calcfile);
  NEED(in, "CORE CONF FILENAME", v);
  NEED(in, "EXECUTE TIME (SEC)", v); job->execute_seconds = atoi(v.c_str());
  NEED(in, "START MJD", v); job->start_mjd = atoi(v.c_str());
  NEED(in, "START SECONDS", v); job->start_seconds = atoi(v.c_str());
  NEED(in, "ACTIVE DATASTREAMS", v); const int numds = atoi(v.c_str());
  NEED(in, "ACTIVE BASELINES", v); const int numbl = atoi(v.c_str());

  // ------------------------------------------------------------- CONFIGURATIONS
  if (!in.seek_section("# CONFIGURATIONS")) { err = in.err; return nullptr; }
  NEED(in, "NUM CONFIGURATIONS", v);
  if (atoi(v.c_str()) < 1) { err = "no configurations"; return nullptr; }
  gx_job_desc &d = job->desc;
  memset(&d, 0, sizeof(d));
  NEED(in, "CONFIG NAME", v);
  NEED(in, "INT TIME (SEC)", v); job->int_time = atof(v.c_str());
  NEED(in, "SUBINT NANOSECONDS", v); d.subint_ns = atoi(v.c_str());
  NEED(in, "GUARD NANOSECONDS", v); d.guard_ns = atoi(v.c_str());
  NEED(in, "FRINGE ROTN ORDER", v); d.fringe_rotation_order = atoi(v.c_str());
  NEED(in, "ARRAY STRIDE LEN", v); d.array_stride = atoi(v.c_str());
  NEED(in, "XMAC STRIDE LEN", v); d.xmac_stride = atoi(v.c_str());
  NEED(in, "NUM BUFFERED FFTS", v); job->meta.num_buffered_ffts = std::max(1, atoi(v.c_str()));
  NEED(in, "WRITE AUTOCORRS", v); d.write_autocorrs = truthy(v) ? 1 : 0;
  NEED(in, "PULSAR BINNING", v);
  if (truthy(v)) {
    // the bin configuration and its polycos (configuration.cpp:1368-1372, 3400-3498)
    NEED(in, "PULSAR CONFIG FILE", v);
    KVFile bc;
    if (!bc.load(resolve(v, inputfile))) { err = bc.err; return nullptr; }
    std::shared_ptr<PulsarConfig> pc(new PulsarConfig());
    std::string w;
    if (!bc.get("NUM POLYCO FILES", w)) { err = bc.err; return nullptr; }
    const int nfiles = atoi(w.c_str());
    for (int i = 0; i < nfiles; i++) {
      if (!bc.get("POLYCO FILE", w)) { err = bc.err; return nullptr; }
      if (!read_polycos(resolve(w, inputfile), pc->polycos, err)) return nullptr;
    }
    if (!bc.get("NUM PULSAR BINS", w)) { err = bc.err; return nullptr; }
    pc->nbins = atoi(w.c_str());
    if (pc->nbins < 1 || pc->nbins > 1024) { err = "NUM PULSAR BINS out of range"; return nullptr; }
    if (!bc.get("SCRUNCH OUTPUT", w)) { err = bc.err; return nullptr; }
    pc->scrunch = truthy(w);
    for (int i = 0; i < pc->nbins; i++) {
      if (!bc.get("BIN PHASE END", w)) { err = bc.err; return nullptr; }
      pc->binphaseends.push_back(atof(w.c_str()));
      if (!bc.get("BIN WEIGHT", w)) { err = bc.err; return nullptr; }
      pc->binweights.push_back(atof(w.c_str()));
    }
    for (int i = 1; i < pc->nbins; i++)
      if (pc->binphaseends[i] < pc->binphaseends[i - 1]) { err = "bin phase ends not ascending"; return nullptr; }
    job->meta.pulsar = pc;
  }
  NEED(in, "PHASED ARRAY", v);
  if (truthy(v)) { err = "phased-array mode is not implemented"; return nullptr; }
  std::vector<int> dsidx(numds), blidx(numbl);
  for (int i = 0; i < numds; i++) { NEED(in, "DATASTREAM ", v); dsidx[i] = atoi(v.c_str()); }
  for (int i = 0; i < numbl; i++) { NEED(in, "BASELINE ", v); blidx[i] = atoi(v.c_str()); }

  // ------------------------------------------------------------- FREQ TABLE
  if (!in.seek_section("# FREQ TABLE")) { err = in.err; return nullptr; }
  NEED(in, "FREQ ENTRIES", v);
  const int nfreq = atoi(v.c_str());
  for (int i = 0; i < nfreq; i++) {
    gx_freq_desc f{};
    NEED(in, "FREQ (MHZ) ", v); f.freq_mhz = atof(v.c_str());
    NEED(in, "BW (MHZ) ", v); f.bw_mhz = atof(v.c_str());
    NEED(in, "SIDEBAND ", v);
    std::string sb = strip(v);
    f.lower_sideband = (sb == "L" || sb == "l" || sb == "LOWER" || sb == "lower") ? 1 : 0;
    if (in.peek("RX NAME ")) NEED(in, "RX NAME ", v);
    NEED(in, "NUM CHANNELS ", v); f.nchan = atoi(v.c_str());
    NEED(in, "CHANS TO AVG ", v); f.chans_to_average = atoi(v.c_str());
    NEED(in, "OVERSAMPLE FAC. ", v);
    NEED(in, "DECIMATION FAC. ", v);
    if (atoi(v.c_str()) != 1) { err = "decimation is not implemented"; return nullptr; }
    NEED(in, "PHASE CALS ", v);
    int npc = atoi(v.c_str());
    for (int j = 0; j < npc; j++) NEED(in, "PHASE CAL ", v);
    job->freqs.push_back(f);
  }

  // ------------------------------------------------------------- TELESCOPE TABLE
  if (!in.seek_section("# TELESCOPE TABLE")) { err = in.err; return nullptr; }
  NEED(in, "TELESCOPE ENTRIES", v);
  const int ntel = atoi(v.c_str());
  std::vector<std::string> telname(ntel);
  std::vector<double> clockref(ntel);
  std::vector<std::vector<double>> clockpoly(ntel);
  for (int i = 0; i < ntel; i++) {
    NEED(in, "TELESCOPE NAME ", v); telname[i] = strip(v);
    NEED(in, "CLOCK REF MJD ", v); clockref[i] = atof(v.c_str());
    NEED(in, "CLOCK POLY ORDER ", v);
    int order = atoi(v.c_str());
    for (int j = 0; j <= order; j++) { NEED(in, "CLOCK COEFF ", v); clockpoly[i].push_back(atof(v.c_str())); }
  }

  // ------------------------------------------------------------- DATASTREAM TABLE
  if (!in.seek_section("# DATASTREAM TABLE")) { err = in.err; return nullptr; }
  NEED(in, "DATASTREAM ENTRIES", v);
  const int nds_table = atoi(v.c_str());
  NEED(in, "DATA BUFFER FACTOR", v); job->meta.data_buffer_factor = atoi(v.c_str());
  NEED(in, "NUM DATA SEGMENTS", v); job->meta.num_data_segments = atoi(v.c_str());
  std::vector<gx_station_desc> dstab(nds_table);
  std::vector<int> dstel(nds_table);
  std::vector<double> dstsys(nds_table, 0.0);
  for (int i = 0; i < nds_table; i++) {
    gx_station_desc &s = dstab[i];
    memset(&s, 0, sizeof(s));
    NEED(in, "TELESCOPE INDEX", v); dstel[i] = atoi(v.c_str());
    NEED(in, "TSYS", v); dstsys[i] = atof(v.c_str());
    NEED(in, "DATA FORMAT", v);
    const std::string fmt = strip(v);
    int muxthreads = 0;   // INTERLACEDVDIF/<thread>:<thread>:... (configuration.cpp:1491-1498, 2632-2651)
    if (fmt.compare(0, 15, "INTERLACEDVDIF/") == 0 && fmt.size() > 15) {
      // the thread ids, read with atoi per ':'-separated field
      size_t a = 15;
      while (true) {
        const size_t e = fmt.find(':', a);
        if (muxthreads == GX_MAX_MUX_THREADS) { err = "more than 64 VDIF threads"; return nullptr; }
        s.muxthread[muxthreads++] = atoi(fmt.substr(a, e == std::string::npos ? std::string::npos : e - a).c_str());
        if (e == std::string::npos) break;
        a = e + 1;
      }
      s.nmuxthreads = muxthreads;
      s.interlaced = 1;
    } else if (fmt != "VDIF") {
      err = "DATA FORMAT " + fmt + " is not implemented (VDIF and INTERLACEDVDIF only)";
      return nullptr;
    }
    NEED(in, "QUANTISATION BITS", v); s.nbits = atoi(v.c_str());
    NEED(in, "DATA FRAME SIZE", v); s.framebytes = atoi(v.c_str());
    // the Core sees multiplexed frames: one header, every thread's payload (configuration.cpp:1686-1696)
    if (muxthreads) s.framebytes = (s.framebytes - 32) * muxthreads + 32;
    NEED(in, "DATA SAMPLING", v);
    std::string samp = strip(v);
    if (samp == "REAL") s.is_complex = 0;
    else if (samp == "COMPLEX" || samp == "COMPLEX_IQ" || samp == "COMPLEX_SSB") s.is_complex = 1;
    else { err = "DATA SAMPLING " + samp + " is not implemented"; return nullptr; }
    NEED(in, "DATA SOURCE", v);
    if (in.peek("FILTERBANK USED")) NEED(in, "FILTERBANK USED", v);
    else if (in.peek("PROCESSING METHOD")) {
      NEED(in, "PROCESSING METHOD", v);
      if (strip(v) != "NONE") { err = "PROCESSING METHOD " + strip(v) + " is not implemented"; return nullptr; }
    }
    if (in.peek("TCAL FREQUENCY")) NEED(in, "TCAL FREQUENCY", v);
    NEED(in, "PHASE CAL INT (MHZ)", v); s.phase_cal_interval_hz = (long long)(1e6 * atof(v.c_str()));
    if (in.peek("PHASE CAL DIVISOR")) {
      NEED(in, "PHASE CAL DIVISOR", v);
      if (atol(v.c_str()) != 1) { err = "PHASE CAL DIVISOR other than 1 is not implemented"; return nullptr; }
    }
    if (in.peek("PHASE CAL BASE(MHZ)")) {
      NEED(in, "PHASE CAL BASE(MHZ)", v); s.phase_cal_base_hz = (long long)(1e6 * atof(v.c_str()));
    }
    NEED(in, "NUM RECORDED FREQS", v); s.nrecfreqs = atoi(v.c_str());
    if (s.nrecfreqs > GX_MAX_LOCAL_FREQS) { err = "too many recorded freqs"; return nullptr; }
    int nb = 0;
    for (int j = 0; j < s.nrecfreqs; j++) {
      NEED(in, "REC FREQ INDEX ", v); s.recfreq[j] = atoi(v.c_str());
      NEED(in, "CLK OFFSET ", v);
      {
        // "offset" or "offset:lcpoffset[:phase]" (configuration.cpp:1606-1630)
        std::string cv = strip(v);
        size_t c1 = cv.find(':');
        s.clock_offset_us[j] = atof(cv.substr(0, c1).c_str());
        if (c1 != std::string::npos) {
          std::string rest = cv.substr(c1 + 1);
          size_t c2 = rest.find(':');
          s.clock_offset_delta_us[j] = atof(rest.substr(0, c2).c_str());
          if (c2 != std::string::npos && atof(rest.substr(c2 + 1).c_str()) != 0.0) {
            err = "per-freq phase offsets are not implemented";
            return nullptr;
          }
        }
      }
      NEED(in, "FREQ OFFSET ", v); s.lo_offset_hz[j] = atof(v.c_str());
      NEED(in, "NUM REC POLS ", v); nb += atoi(v.c_str());
    }
    s.nbands = nb;
    if (nb > GX_MAX_BANDS) { err = "too many recorded bands"; return nullptr; }
    for (int j = 0; j < nb; j++) {
      NEED(in, "REC BAND ", v); s.band_pol[j] = strip(v).empty() ? 'R' : strip(v)[0];
      NEED(in, "REC BAND ", v); s.band_localfreq[j] = atoi(v.c_str());
    }
    // zoom freqs and bands (configuration.cpp:1701-1753)
    NEED(in, "NUM ZOOM FREQS", v); s.nzoomfreqs = atoi(v.c_str());
    if (s.nzoomfreqs < 0 || s.nzoomfreqs > GX_MAX_LOCAL_FREQS) { err = "too many zoom freqs"; return nullptr; }
    int nzb = 0;
    for (int j = 0; j < s.nzoomfreqs; j++) {
      NEED(in, "ZOOM FREQ INDEX ", v); s.zoomfreq[j] = atoi(v.c_str());
      NEED(in, "NUM ZOOM POLS ", v); nzb += atoi(v.c_str());
    }
    if (nzb < 0 || nzb > GX_MAX_BANDS) { err = "too many zoom bands"; return nullptr; }
    s.nzoombands = nzb;
    for (int j = 0; j < nzb; j++) {
      NEED(in, "ZOOM BAND ", v); s.zoomband_pol[j] = strip(v).empty() ? 'R' : strip(v)[0];
      NEED(in, "ZOOM BAND ", v); s.zoomband_localfreq[j] = atoi(v.c_str());
    }
    const std::vector<double> &cp = clockpoly[dstel[i]];
    s.clock_int_seconds = int(std::floor((cp.empty() ? 0.0 : cp[0]) / 1000000.0 + 0.5));
  }

  // ------------------------------------------------------------- BASELINE TABLE
  if (!in.seek_section("# BASELINE TABLE")) { err = in.err; return nullptr; }
  NEED(in, "BASELINE ENTRIES", v);
  const int nbl_table = atoi(v.c_str());
  std::vector<gx_baseline_desc> bltab(nbl_table);
  for (int i = 0; i < nbl_table; i++) {
    gx_baseline_desc &b = bltab[i];
    memset(&b, 0, sizeof(b));
    NEED(in, "D/STREAM A INDEX ", v); b.ds1 = atoi(v.c_str());
    NEED(in, "D/STREAM B INDEX ", v); b.ds2 = atoi(v.c_str());
    NEED(in, "NUM FREQS ", v); b.nfreqs = atoi(v.c_str());
    if (b.nfreqs > GX_MAX_LOCAL_FREQS) { err = "too many baseline freqs"; return nullptr; }
    for (int j = 0; j < b.nfreqs; j++) {
      NEED(in, "TARGET FREQ ", v);
      NEED(in, "POL PRODUCTS ", v); b.npolprod[j] = atoi(v.c_str());
      if (b.npolprod[j] > GX_MAX_POLPRODUCTS) { err = "too many pol products"; return nullptr; }
      for (int k = 0; k < b.npolprod[j]; k++) {
        NEED(in, "D/STREAM A BAND ", v); b.band1[j][k] = atoi(v.c_str());
        NEED(in, "D/STREAM B BAND ", v); b.band2[j][k] = atoi(v.c_str());
      }
      // the freq of the first product's band of datastream A; band indices
      // from the recorded band count on name zoom bands (configuration.cpp:1095-1100)
      const gx_station_desc &s1 = dstab[b.ds1];
      const int b1 = b.band1[j][0];
      if (b1 < 0 || b1 >= s1.nbands + s1.nzoombands) { err = "baseline band index out of range"; return nullptr; }
      if (b1 < s1.nbands) {
        b.freq[j] = s1.recfreq[s1.band_localfreq[b1]];
      } else {
        const int zl = s1.zoomband_localfreq[b1 - s1.nbands];
        if (zl < 0 || zl >= s1.nzoomfreqs) { err = "ZOOM BAND INDEX out of range"; return nullptr; }
        b.freq[j] = s1.zoomfreq[zl];
      }
    }
  }

  // ------------------------------------------------------------- DATA TABLE
  if (in.seek_section("# DATA TABLE")) {
    for (int i = 0; i < nds_table; i++) {
      if (!in.get("D/STREAM ", v)) break;
      int nf = atoi(v.c_str());
      std::string first;
      for (int j = 0; j < nf; j++) {
        if (!in.get("FILE ", v)) break;
        if (j == 0) first = strip(v);
      }
      job->datafiles.push_back(first);
    }
  }

  // configuration 0's datastreams and baselines, in config order
  for (int i = 0; i < numds; i++) job->stations.push_back(dstab[dsidx[i]]);
  std::vector<int> tel_of_cfgds(numds);
  for (int i = 0; i < numds; i++) tel_of_cfgds[i] = dstel[dsidx[i]];
  for (int i = 0; i < numbl; i++) {
    gx_baseline_desc b = bltab[blidx[i]];
    int a1 = -1, a2 = -1;
    for (int k = 0; k < numds; k++) {
      if (dsidx[k] == b.ds1) a1 = k;
      if (dsidx[k] == b.ds2) a2 = k;
    }
    if (a1 < 0 || a2 < 0) { err = "baseline refers to an inactive datastream"; return nullptr; }
    b.ds1 = a1;
    b.ds2 = a2;
    job->baselines.push_back(b);
  }
  d.nstations = numds;
  d.stations = job->stations.data();
  d.nfreqs = nfreq;
  d.freqs = job->freqs.data();
  d.nbaselines = numbl;
  d.baselines = job->baselines.data();

  // ------------------------------------------------------------- .calc
  std::string calcpath = resolve(calcfile, inputfile);
  KVFile calc;
  if (!calc.load(calcpath)) { err = calc.err; return nullptr; }
  std::unique_ptr<HostModel> m(new HostModel());
  auto cget = [&](const std::string &k, std::string &out) {
    const std::string *p = calc.find(k);
    if (!p) { err = calcpath + ": missing '" + k + "'"; return false; }
    out = *p;
    return true;
  };
  int Y, Mo, D, H, Mi, Se;
  if (!cget("START YEAR", v)) return nullptr; Y = atoi(v.c_str());
  if (!cget("START MONTH", v)) return nullptr; Mo = atoi(v.c_str());
  if (!cget("START DAY", v)) return nullptr; D = atoi(v.c_str());
  if (!cget("START HOUR", v)) return nullptr; H = atoi(v.c_str());
  if (!cget("START MINUTE", v)) return nullptr; Mi = atoi(v.c_str());
  if (!cget("START SECOND", v)) return nullptr; Se = atoi(v.c_str());
  m->modelmjd = get_mjd(Y, Mo, D);
  m->modelstartseconds = 3600 * H + 60 * Mi + Se;
  m->jobmjd = job->start_mjd;
  m->jobseconds = job->start_seconds;
  if (!cget("NUM TELESCOPES", v)) return nullptr;
  m->nstations = atoi(v.c_str());
  std::vector<std::string> mname(m->nstations);
  for (int i = 0; i < m->nstations; i++) {
    if (!cget("TELESCOPE " + std::to_string(i) + " NAME", v)) return nullptr;
    mname[i] = strip(v);
  }
  if (!cget("NUM SCANS", v)) return nullptr;
  int nscans = atoi(v.c_str());
  m->scans.resize(nscans);
  for (int i = 0; i < nscans; i++) {
    std::string pre = "SCAN " + std::to_string(i) + " ";
    if (!cget(pre + "START (S)", v)) return nullptr; m->scans[i].offsetseconds = atoi(v.c_str());
    if (!cget(pre + "DUR (S)", v)) return nullptr; m->scans[i].durationseconds = atoi(v.c_str());
    if (!cget(pre + "UVSHIFT INTERVAL (NS)", v)) return nullptr; m->scans[i].maxns_xc = atoi(v.c_str());
    if (!cget(pre + "POINTING SRC", v)) return nullptr; m->scans[i].pointing_source = atoi(v.c_str());
    if (!cget(pre + "NUM PHS CTRS", v)) return nullptr; m->scans[i].numphasecentres = atoi(v.c_str());
    if (m->scans[i].numphasecentres < 1 || m->scans[i].numphasecentres > 64) {
      err = "NUM PHS CTRS out of range";
      return nullptr;
    }
    for (int j = 0; j < m->scans[i].numphasecentres; j++) {
      if (!cget(pre + "PHS CTR " + std::to_string(j), v)) return nullptr;
      m->scans[i].phase_centre_sources.push_back(atoi(v.c_str()));
    }
    m->scans[i].phase_centre_source = m->scans[i].phase_centre_sources[0];
  }
  if (!cget("NUM SPACECRAFT", v)) return nullptr;
  if (atoi(v.c_str()) != 0) { err = "spacecraft models are not implemented"; return nullptr; }
  if (!cget("IM FILENAME", v)) return nullptr;
  std::string impath = resolve(v, inputfile);

  // ------------------------------------------------------------- .im
  KVFile im;
  if (!im.load(impath)) { err = im.err; return nullptr; }
  {
    const std::string *p;
    if (!(p = im.find("POLYNOMIAL ORDER"))) { err = "IM: no POLYNOMIAL ORDER"; return nullptr; }
    m->polyorder = atoi(p->c_str());
    if (m->polyorder > 14) { err = "IM: polynomial order too high"; return nullptr; }
    if (!(p = im.find("INTERVAL (SECS)"))) { err = "IM: no INTERVAL"; return nullptr; }
    m->modelincsecs = atoi(p->c_str());
  }
  // walk the file in order: SCAN i NUM POLY, SCAN i POLY k MJD/SEC, SRC s ANT a DELAY (us)
  {
    int curscan = -1, curpoly = -1;
    const int np1 = m->polyorder + 1;
    for (const auto &it : im.items) {
      const std::string &k = it.key;
      int a = -1, b = -1;
      char tail[64];
      if (sscanf(k.c_str(), "SCAN %d NUM POLY", &a) == 1 && k.find("NUM POLY") != std::string::npos) {
        if (a < 0 || a >= nscans) { err = "IM: scan index"; return nullptr; }
        curscan = a;
        ModelScan &sc = m->scans[a];
        sc.nsamples = atoi(it.val.c_str());
        sc.delay.assign((size_t)sc.nsamples * (sc.numphasecentres + 1) * m->nstations * np1, 0.0);
        sc.u = sc.v = sc.w = sc.delay;
      } else if (sscanf(k.c_str(), "SCAN %d POLY %d %63s", &a, &b, tail) == 3) {
        if (a != curscan) { err = "IM: polynomial outside its scan"; return nullptr; }
        curpoly = b;
        if (!strcmp(tail, "MJD") && b == 0) m->scans[a].polystartmjd = atoi(it.val.c_str());
        if (!strcmp(tail, "SEC") && b == 0) m->scans[a].polystartseconds = atoi(it.val.c_str());
      } else if (sscanf(k.c_str(), "SRC %d ANT %d", &a, &b) == 2) {
        int which = -1;   // 0 delay, 1-3 u, v, w
        if (k.find("DELAY (us)") != std::string::npos) which = 0;
        else if (k.find("U (m)") != std::string::npos) which = 1;
        else if (k.find("V (m)") != std::string::npos) which = 2;
        else if (k.find("W (m)") != std::string::npos) which = 3;
        if (which < 0) continue;
        if (curscan < 0 || curpoly < 0) { err = "IM: polynomial row before its scan/poly"; return nullptr; }
        ModelScan &sc = m->scans[curscan];
        std::vector<double> *tab = which == 0 ? &sc.delay : which == 1 ? &sc.u : which == 2 ? &sc.v : &sc.w;
        if (curpoly >= sc.nsamples || a > sc.numphasecentres || b >= m->nstations) { err = "IM: index"; return nullptr; }
        std::istringstream iss(it.val);
        for (int i = 0; i < np1; i++) {
          std::string tok;
          if (!(iss >> tok)) { err = "IM: short polynomial row"; return nullptr; }
          (*tab)[(((size_t)curpoly * (sc.numphasecentres + 1) + a) * m->nstations + b) * np1 + i] = atof(tok.c_str());
        }
      }
    }
  }
  // the largest delay rate of every antenna over the polynomials as read
  // (before the clock terms), skipping rows of negative delay (model.cpp:762-765)
  m->maxrate.assign(m->nstations, 0.0);
  if (m->polyorder >= 1) {
    for (const auto &sc : m->scans)
      for (int k = 0; k < sc.nsamples; k++)
        for (int p = 0; p < sc.numphasecentres + 1; p++)
          for (int a = 0; a < m->nstations; a++) {
            const double *d = &sc.delay[(((size_t)k * (sc.numphasecentres + 1) + p) * m->nstations + a) * (m->polyorder + 1)];
            if (std::fabs(d[1]) > std::fabs(m->maxrate[a]) && d[0] > 0.0) m->maxrate[a] = std::fabs(d[1]);
          }
  }
  // clock terms (Model::addClockTerms, model.cpp:291-352, with isupdate = false)
  std::vector<std::vector<double>> binom(m->polyorder + 1);
  for (int i = 0; i <= m->polyorder; i++) {
    binom[i].assign(i + 1, 0.0);
    binom[i][0] = 1;
    binom[i][i] = 1;
    for (int j = 1; j < i; j++) binom[i][j] = binom[i - 1][j - 1] + binom[i - 1][j];
  }
  for (int t = 0; t < ntel; t++) {
    int ant = -1;
    for (int i = 0; i < m->nstations; i++)
      if (mname[i] == telname[t]) ant = i;
    if (ant < 0) continue;
    const int order = (int)clockpoly[t].size() - 1;
    if (order > m->polyorder) { err = "clock order above the model polynomial order"; return nullptr; }
    for (auto &sc : m->scans) {
      for (int k = 0; k < sc.nsamples; k++) {
        double clockdistance = 86400.0 * (sc.polystartmjd + ((double)sc.polystartseconds) / 86400.0 - clockref[t]) +
                               k * double(m->modelincsecs);
        std::vector<double> dt(order + 1), clk(m->polyorder + 1, 0.0);
        dt[0] = 1.0;
        for (int l = 1; l <= order; l++) dt[l] = dt[l - 1] * clockdistance;
        for (int l = 0; l <= order; l++)
          for (int mm = l; mm <= order; mm++) clk[l] += clockpoly[t][mm] * dt[mm - l] * binom[mm][mm - l];
        for (int p = 0; p < sc.numphasecentres + 1; p++)
          for (int l = 0; l <= m->polyorder; l++)
            sc.delay[(((size_t)k * (sc.numphasecentres + 1) + p) * m->nstations + ant) * (m->polyorder + 1) + l] += clk[l];
      }
    }
  }
  // datastream -> model antenna (by telescope name), clocks, timespan
  for (int i = 0; i < numds; i++) {
    int ant = -1;
    for (int a = 0; a < m->nstations; a++)
      if (mname[a] == telname[tel_of_cfgds[i]]) ant = a;
    if (ant < 0) { err = "telescope " + telname[tel_of_cfgds[i]] + " missing from the model"; return nullptr; }
    m->station_of_datastream.push_back(ant);
    m->intclockseconds.push_back(job->stations[i].clock_int_seconds);
  }
  {
    const gx_freq_desc &f0 = job->freqs[job->stations[0].recfreq[0]];
    const double bw = f0.bw_mhz;
    double sampletime = 1.0 / (2.0 * bw);
    if (job->stations[0].is_complex) sampletime *= 2.0;
    const double ffttime = 1000.0 * f0.nchan / bw;
    m->blocks_per_send = int(d.subint_ns / ffttime + 0.5);
    // Mode::setOffsets timespan (mode.cpp:1523-1524)
    double timespan = m->blocks_per_send * 2 * f0.nchan * sampletime / 1e6;
    if (job->stations[0].is_complex) timespan /= 2;
    m->timespan_s = timespan;
  }
  job->model = std::move(m);
  job->meta.start_mjd = job->start_mjd;
  job->meta.start_seconds = job->start_seconds;
  job->meta.execute_seconds = job->execute_seconds;
  job->meta.int_time = job->int_time;
  job->meta.telescope_name = telname;
  for (int i = 0; i < numds; i++) {
    job->meta.telescope.push_back(tel_of_cfgds[i]);
    job->meta.tsys.push_back(dstsys[dsidx[i]]);
  }
  return job.release();
}

}  // namespace gx
