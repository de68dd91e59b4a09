// Reference harness (test infrastructure only).
//
// Drives the reference correlator's own hot path -- Configuration (non-MPI
// constructor, mpifxcorr/src/configuration.cpp:98), the Mode objects it
// builds (Configuration::getMode, configuration.cpp:932), Mode::process /
// Mk5Mode::unpack (mode.cpp:634, mk5mode.cpp:94) and Core::processdata
// (core.cpp:657) -- on one Core slot, the way Core::loopprocess
// (core.cpp:388-470) prepares each process thread.  The reference sources
// are compiled unmodified, with the GENERIC architecture header and the
// oracle's FFT/MPI/difxmessage shims; this harness alone is compiled with
// refshim/openaccess.h so it can call Core::processdata without the MPI
// receive loop.  Exposes a small C API for the Python tests and the CPU
// baseline.
#include <mpi.h>
#include <pthread.h>
#include <cstring>
#include <cstdio>
#include <vector>
#include "architecture.h"
#include "configuration.h"
#include "core.h"
#include "mode.h"
#include "mk5mode.h"
#include "model.h"
#include "visibility.h"

namespace {
struct RefJob {
  Configuration *config;
  Core *core;
  int nthreads;
  int nds;
  std::vector<Mode **> modes;
  std::vector<void *> scratch;  // Core::threadscratchspace*
  std::vector<int> startblock, numblocks;
  std::vector<u8 *> origbuffers;
  std::vector<std::vector<double>> interp_override;  // per datastream; empty: the model's
  std::vector<Polyco **> polycos;      // per thread (pulsar binning), as Core::updateconfig gives them
  std::vector<int> npolycos;
  std::vector<Polyco *> curpolyco;     // per thread, set for the slot being processed
};

struct ThreadArg {
  RefJob *job;
  int t;
};

void *worker(void *p)
{
  ThreadArg *a = (ThreadArg *)p;
  RefJob *j = a->job;
  Core *c = j->core;
  pthread_mutex_lock(&(c->procslots[0].slotlocks[a->t]));
  c->processdata(0, a->t, j->startblock[a->t], j->numblocks[a->t], j->modes[a->t], j->curpolyco[a->t],
                 (Core::threadscratchspace *)j->scratch[a->t]);
  pthread_mutex_unlock(&(c->procslots[1].slotlocks[a->t]));
  return 0;
}
}  // namespace

extern "C" {

void *ref_open(const char *inputfile)
{
  Configuration *config = new Configuration(inputfile, 0, 0.0);
  if (!config->consistencyOK()) {
    fprintf(stderr, "ref_open: configuration inconsistent\n");
    return 0;
  }
  // mpifxcorr's main() sets this flag (default off) right after constructing
  // the Configuration (mpifxcorr.cpp:262, 370); the constructor leaves it unset.
  config->setVGOSComplexVDIFHack(false);
  RefJob *j = new RefJob();
  j->config = config;
  j->nds = config->getNumDataStreams();
  int *dids = new int[j->nds];
  for (int i = 0; i < j->nds; i++) dids[i] = i + 1;
  // Core id: the first core process (manager 0, datastreams 1..nds)
  j->core = new Core(j->nds + fxcorr::FIRSTTELESCOPEID, config, dids, MPI_COMM_WORLD);
  delete[] dids;
  Core *c = j->core;
  j->nthreads = c->numprocessthreads;
  for (int i = 0; i < j->nds; i++) j->origbuffers.push_back(c->procslots[0].databuffer[i]);
  for (int t = 0; t < j->nthreads; t++) {
    // per-thread scratch, as Core::loopprocess prepares it (core.cpp:397-462)
    Core::threadscratchspace *s = new Core::threadscratchspace;
    s->shifterrorcount = 0;
    s->threadcrosscorrs = vectorAlloc_cf32(c->maxthreadresultlength);
    s->baselineweight = new f32 ***[config->getFreqTableLength()]();
    s->baselineshiftdecorr = new f32 **[config->getFreqTableLength()]();
    s->pulsarscratchspace = 0;
    s->pulsaraccumspace = 0;
    s->starecordbuffer = 0;
    s->bins = 0;
    s->dumpsta = false;
    s->dumpkurtosis = false;
    int maxchan = config->getMaxNumChannels();
    int slen = config->getRotateStrideLength(0);
    int maxrot = slen + maxchan / slen;
    s->chanfreqs = vectorAlloc_f64(maxrot);
    s->rotator = vectorAlloc_cf32(maxrot);
    s->rotated = vectorAlloc_cf32(maxchan);
    s->channelsums = vectorAlloc_cf32(maxchan);
    s->argument = vectorAlloc_f32(3 * maxrot);
    // pulsar binning scratch (core.cpp:437-458)
    const bool psr = config->pulsarBinOn(0);
    if (psr) {
      s->pulsarscratchspace = vectorAlloc_cf32(config->getXmacStrideLength(0));
      if (config->scrunchOutputOn(0)) s->pulsaraccumspace = new cf32 ******[config->getFreqTableLength()]();
      c->createPulsarVaryingSpace(s->pulsaraccumspace, &(s->bins), 0, -1, t);
    }
    c->allocateConfigSpecificThreadArrays(s->baselineweight, s->baselineshiftdecorr, 0, -1, t);
    Mode **modes = new Mode *[j->nds];
    int sb = 0, nb = 0, npoly = 0;
    bool pb = false;
    Polyco **polys = psr ? new Polyco *[config->getNumPolycos(0)] : 0;
    c->updateconfig(0, 0, t, sb, nb, npoly, pb, modes, polys, true);
    j->polycos.push_back(polys);
    j->npolycos.push_back(npoly);
    j->curpolyco.push_back(0);
    j->modes.push_back(modes);
    j->scratch.push_back(s);
    j->startblock.push_back(sb);
    j->numblocks.push_back(nb);
  }
  return j;
}

Configuration *ref_job_config(void *h) { return ((RefJob *)h)->config; }

int gx_stub_binary_take(char *out, int max);

// STA and kurtosis dumps on or off for the following slots, as an operator
// message sets them (Configuration's flags) and Core::loopprocess hands them
// to each thread's scratch space with a record buffer of one MTU
// (core.cpp:510-525).
void ref_set_monitor(void *h, int sta, int kurtosis, int channels)
{
  RefJob *j = (RefJob *)h;
  j->config->dumpsta = sta != 0;
  j->config->dumpkurtosis = kurtosis != 0;
  j->config->stadumpchannels = channels;
  for (void *p : j->scratch) {
    Core::threadscratchspace *s = (Core::threadscratchspace *)p;
    s->dumpsta = sta != 0;
    s->dumpkurtosis = kurtosis != 0;
    if ((sta || kurtosis) && !s->starecordbuffer) s->starecordbuffer = (DifxMessageSTARecord *)malloc(j->config->getMTU());
  }
}

// The binary messages the reference sent since the last call.
int ref_take_messages(void *h, char *out, int max)
{
  (void)h;
  return gx_stub_binary_take(out, max);
}
int ref_num_threads(void *h) { return ((RefJob *)h)->nthreads; }
int ref_result_length(void *h) { return ((RefJob *)h)->config->getCoreResultLength(0); }
int ref_blocks_per_send(void *h) { return ((RefJob *)h)->config->getBlocksPerSend(0); }
int ref_xmac_stride(void *h) { return ((RefJob *)h)->config->getXmacStrideLength(0); }
int ref_array_stride(void *h) { return ((RefJob *)h)->config->getArrayStrideLength(0, 0); }
int ref_num_baselines(void *h) { return ((RefJob *)h)->config->getNumBaselines(); }
int ref_freq_table_length(void *h) { return ((RefJob *)h)->config->getFreqTableLength(); }

// Core result layout offsets (in cf32 units, as configuration.cpp:2348-2630):
// baseline offsets [freq][baseline] (-1 if unused), bweight offsets
// [freq][baseline], autocorr offsets [ds], acweight offsets [ds].
int ref_layout(void *h, int *blofs, int *bwofs, int *acofs, int *acwofs)
{
  RefJob *j = (RefJob *)h;
  Configuration *cf = j->config;
  int nf = cf->getFreqTableLength(), nb = cf->getNumBaselines();
  for (int f = 0; f < nf; f++)
    for (int b = 0; b < nb; b++) {
      bool used = cf->isFrequencyUsed(0, f) && cf->getBLocalFreqIndex(0, b, f) >= 0;
      blofs[f * nb + b] = used ? cf->getCoreResultBaselineOffset(0, f, b) : -1;
      bwofs[f * nb + b] = used ? cf->getCoreResultBWeightOffset(0, f, b) : -1;
    }
  for (int d = 0; d < j->nds; d++) {
    acofs[d] = cf->getCoreResultAutocorrOffset(0, d);
    acwofs[d] = cf->getCoreResultACWeightOffset(0, d);
  }
  return 0;
}

// Delay interpolator exactly as Mode::setOffsets computes it (mode.cpp:1502-1532).
int ref_interpolator(void *h, int station, int scan, int sec, int ns, double *out3)
{
  RefJob *j = (RefJob *)h;
  Mode *m = j->modes[0][station];
  m->datasec = 0;
  m->datascan = scan;
  m->setOffsets(scan, sec, ns);
  for (int i = 0; i < 3; i++) out3[i] = m->interpolator[i];
  return m->offsetseconds == Mode::INVALID_SUBINT ? -1 : 0;
}

// One whole subint through Core::processdata on every process thread.
int ref_process(void *h, int scan, int sec, int ns, const unsigned char **data, const int *datalen,
                const int **control, int controllen, float *results)
{
  RefJob *j = (RefJob *)h;
  Core *c = j->core;
  Core::processslot *slot = &(c->procslots[0]);
  slot->offsets[0] = scan;
  slot->offsets[1] = sec;
  slot->offsets[2] = ns;
  for (int d = 0; d < j->nds; d++) {
    slot->databuffer[d] = (u8 *)data[d];
    slot->datalengthbytes[d] = datalen[d];
    int cl = controllen < c->controllength ? controllen : c->controllength;
    memset(slot->controlbuffer[d], 0, sizeof(s32) * c->controllength);
    memcpy(slot->controlbuffer[d], control[d], sizeof(s32) * cl);
  }
  int rl = j->config->getCoreResultLength(0);
  vectorZero_cf32(slot->results, rl);
  if (j->config->pulsarBinOn(0)) {
    // the polyco of the slot's time (Core::loopprocess, core.cpp:496-507)
    Configuration *cf = j->config;
    const int startmjd = cf->getStartMJD(), startseconds = cf->getStartSeconds();
    const double secs = double(startseconds + c->model->getScanStartSec(scan, startmjd, startseconds) + sec) +
                        ((double)ns) / 1000000000.0;
    for (int t = 0; t < j->nthreads; t++) {
      Polyco *p = Polyco::getCurrentPolyco(0, startmjd, secs / 86400.0, j->polycos[t], j->npolycos[t], false);
      if (!p) return -2;
      p->setTime(startmjd, secs / 86400.0);
      j->curpolyco[t] = p;
    }
  }
  std::vector<pthread_t> th(j->nthreads);
  std::vector<ThreadArg> args(j->nthreads);
  for (int t = 0; t < j->nthreads; t++) {
    args[t].job = j;
    args[t].t = t;
    pthread_create(&th[t], 0, worker, &args[t]);
  }
  for (int t = 0; t < j->nthreads; t++) pthread_join(th[t], 0);
  memcpy(results, slot->results, sizeof(cf32) * rl);
  for (int d = 0; d < j->nds; d++) slot->databuffer[d] = j->origbuffers[d];
  return 0;
}

// One FFT block of one station through Mode::process, returning the spectra of
// every recorded band (nbands x nchan cf32, after the fractional-sample
// rotation) and the block's data weight.  Used to pin the station-based stage.
int ref_mode_block(void *h, int station, const unsigned char *data, int datalen, const int *control,
                   int controllen, int scan, int sec, int ns, int block, float *spectra, float *weight)
{
  RefJob *j = (RefJob *)h;
  Mode *m = j->modes[0][station];
  std::vector<s32> flags(controllen > 3 ? controllen - 3 : 1, 0);
  for (int i = 3; i < controllen; i++) flags[i - 3] = control[i];
  m->zeroAutocorrelations();
  m->setValidFlags(flags.data());
  m->setData((u8 *)data, datalen, control[0], control[1], control[2]);
  m->setOffsets(scan, sec, ns);
  m->process(block, 0);
  int nb = m->numrecordedbands, nc = m->recordedbandchannels;
  for (int b = 0; b < nb; b++) memcpy(spectra + 2 * b * nc, m->fftoutputs[b][0], sizeof(cf32) * nc);
  *weight = m->dataweight[0];
  return 0;
}

// Mode::process of datastream `station` over FFT blocks 0 .. nblocks-1 of
// one subint (data, control words, slot start): per block its spectra
// (nbands x nchan cf32) and data weight, then the autocorrelations
// [2][nbands][nchan] cf32 and weights [2][nbands] accumulated over the blocks.
int ref_mode_blocks(void *h, int station, const unsigned char *data, int datalen, const int *control, int controllen,
                    int scan, int sec, int ns, int nblocks, float *spectra, float *dataweights, float *autos,
                    float *weights)
{
  RefJob *j = (RefJob *)h;
  Mode *m = j->modes[0][station];
  std::vector<s32> flags(controllen > 3 ? controllen - 3 : 1, 0);
  for (int i = 3; i < controllen; i++) flags[i - 3] = control[i];
  m->zeroAutocorrelations();
  m->setValidFlags(flags.data());
  m->setData((u8 *)data, datalen, control[0], control[1], control[2]);
  m->setOffsets(scan, sec, ns);
  if (station < (int)j->interp_override.size() && j->interp_override[station].size() == 3)
    for (int i = 0; i < 3; i++) m->interpolator[i] = j->interp_override[station][i];
  const int nb = m->numrecordedbands, nc = m->recordedbandchannels;
  for (int b = 0; b < nblocks; b++) {
    m->process(b, 0);
    for (int k = 0; k < nb; k++)
      memcpy(spectra + 2 * ((size_t)b * nb + k) * nc, m->getFreqs(k, 0), sizeof(cf32) * nc);
    dataweights[b] = m->getDataWeight(0, 0);
  }
  for (int x = 0; x < 2; x++)
    for (int k = 0; k < nb; k++) {
      memcpy(autos + 2 * ((size_t)x * nb + k) * nc, m->getAutocorrelation(x == 1, k), sizeof(cf32) * nc);
      weights[x * nb + k] = m->getWeight(x == 1, k);
    }
  return 0;
}

// Replaces the delay interpolator that setOffsets computes for `station` in
// later ref_mode_blocks calls (interp3 = null: the model's again).
int ref_set_interpolator(void *h, int station, const double *interp3)
{
  RefJob *j = (RefJob *)h;
  if (station < 0 || station >= j->nds) return -1;
  if ((int)j->interp_override.size() < j->nds) j->interp_override.resize(j->nds);
  j->interp_override[station].clear();
  if (interp3) j->interp_override[station].assign(interp3, interp3 + 3);
  return 0;
}

// Mk5Mode::unpack on its own: unpacked samples (nbands x unpacksamples f32,
// or cf32 for complex data) and the returned weight.
int ref_unpack(void *h, int station, const unsigned char *data, int datalen, int sampleoffset,
               float *out, float *weight, int *unpackstart)
{
  RefJob *j = (RefJob *)h;
  Mode *m = j->modes[0][station];
  m->setData((u8 *)data, datalen, 0, 0, 0);
  *weight = m->unpack(sampleoffset, 0);
  *unpackstart = m->unpackstartsamples;
  int per = m->unpacksamples * (m->usecomplex ? 2 : 1);
  for (int b = 0; b < m->numrecordedbands; b++) memcpy(out + b * per, m->unpackedarrays[b], sizeof(f32) * per);
  return m->unpacksamples;
}

// Visibility (visibility.cpp:33-103, addData 192-205, writedata 353-690,
// writeSWIN 781-960) integrating nsub Core result arrays (host, each of the
// configuration's result length) into the integration that started at scan,
// sec (seconds after the scan start), ns; the records go to
// <outdir>/DIFX_<mjd>_<sec>.s0000.b0000 (the .input's OUTPUT FILENAME is
// replaced by outdir, which must exist).
int ref_vis_write(void *h, int nsub, const float *const *results, int scan, int sec, int ns, const char *outdir)
{
  RefJob *j = (RefJob *)h;
  Configuration *config = j->config;
  config->outputfilename = outdir;
  const long long maxlen = config->getMaxCoreResultLength();
  const long long rl = config->getCoreResultLength(0);
  const long long buflen = maxlen * 8 + (64LL << 20);
  if (buflen > 0x7fffffffLL) return -1;
  char *buf = new char[buflen];
  static const string polnames[] = {"R", "L", "X", "Y"};
  Visibility *v = new Visibility(config, 0, 1, buf, (int)buflen, config->getExecuteSeconds(), scan, sec, ns, polnames);
  cf32 *tmp = vectorAlloc_cf32(maxlen);
  for (int i = 0; i < nsub; i++) {
    vectorZero_cf32(tmp, maxlen);
    memcpy(tmp, results[i], sizeof(cf32) * rl);
    v->addData(tmp);
  }
  v->writedata();
  delete v;
  vectorFree(tmp);
  delete[] buf;
  return 0;
}

// Model::interpolateUVW (model.cpp:177-217) for datastreams ds1, ds2.
int ref_uvw(void *h, int scan, double offset, int ds1, int ds2, double *out3)
{
  RefJob *j = (RefJob *)h;
  Configuration *config = j->config;
  const int a1 = config->getDModelFileIndex(0, ds1), a2 = config->getDModelFileIndex(0, ds2);
  return config->getModel()->interpolateUVW(scan, offset, a1, a2, 1, out3) ? 0 : -1;
}

// Frees everything ref_open made: per thread what Core::loopprocess frees on
// exit (core.cpp:551-581: the Modes and the scratch vectors), the per-freq
// baseline weight rows allocated by allocateConfigSpecificThreadArrays
// (core.cpp:2110-2125; freed here directly, one delete per row array), then
// the Core (core.cpp:159-186) and the Configuration.  A Core holds
// RECEIVE_RING_LENGTH full result slots and every thread a full cross-
// correlation accumulator, so a handle of a large job is many GB of host
// memory.
void ref_close(void *h)
{
  RefJob *j = (RefJob *)h;
  if (!j) return;
  Configuration *cf = j->config;
  Core *c = j->core;
  const int nf = cf->getFreqTableLength(), nb = cf->getNumBaselines();
  for (int t = 0; t < j->nthreads; t++) {
    Mode **modes = j->modes[t];
    for (int d = 0; d < j->nds; d++) delete modes[d];
    delete[] modes;
    Core::threadscratchspace *s = (Core::threadscratchspace *)j->scratch[t];
    for (int f = 0; f < nf; f++) {
      if (!cf->isFrequencyUsed(0, f) || !s->baselineweight[f]) continue;
      for (int b = 0; b < nb; b++)
        if (cf->getBLocalFreqIndex(0, b, f) >= 0) vectorFree(s->baselineweight[f][0][b]);
      delete[] s->baselineweight[f][0];
      delete[] s->baselineweight[f];
    }
    delete[] s->baselineweight;
    delete[] s->baselineshiftdecorr;
    vectorFree(s->threadcrosscorrs);
    vectorFree(s->chanfreqs);
    vectorFree(s->rotator);
    vectorFree(s->rotated);
    vectorFree(s->channelsums);
    vectorFree(s->argument);
    delete s;
  }
  for (int d = 0; d < j->nds; d++) c->procslots[0].databuffer[d] = j->origbuffers[d];
  delete c;
  delete cf;
  delete j;
}
}
