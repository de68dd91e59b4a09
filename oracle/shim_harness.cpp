// Harness for the DiFX-side binding (test infrastructure only): builds the
// reference's Configuration and the GpuCore / GpuMode of
// difx_b200/mpifxcorr from an .input file, fills a Core slot as
// Core::receivedata would (core.cpp:589-656) and runs the binding on it, the
// way ref_harness.cpp runs Core::processdata on the same slot.  Compiled with
// refshim/openaccess.h, which stands in for the friend declarations and the
// `virtual` keywords gpucore.h and gpumode.h ask a maintainer to add to
// core.h, configuration.h and mode.h: here the harness calls
// GpuCore::processdata and GpuMode::process directly.
#include <mpi.h>
#include <cstring>
#include <vector>
#include "architecture.h"
#include "configuration.h"
#include "core.h"
#include "gpucore.h"
#include "gpumode.h"

namespace {
struct ShimJob {
  Configuration *config;
  GpuCore *core;
  std::vector<u8 *> origbuffers;
};
}  // namespace

extern "C" {

void *shim_open(const char *inputfile, int device, int xstep)
{
  Configuration *config = new Configuration(inputfile, 0, 0.0);
  if (!config->consistencyOK()) return 0;
  config->setVGOSComplexVDIFHack(false);   // as mpifxcorr's main() (mpifxcorr.cpp:370)
  const int nds = config->getNumDataStreams();
  std::vector<int> dids(nds);
  for (int i = 0; i < nds; i++) dids[i] = i + 1;
  ShimJob *j = new ShimJob();
  j->config = config;
  j->core = new GpuCore(nds + fxcorr::FIRSTTELESCOPEID, config, dids.data(), MPI_COMM_WORLD, device, xstep);
  for (int i = 0; i < nds; i++) j->origbuffers.push_back(j->core->procslots[0].databuffer[i]);
  return j;
}

const char *shim_last_error(void *h) { return ((ShimJob *)h)->core->lasterror().c_str(); }

// One whole subint through GpuCore::processdata (thread 0) on slot 0; the
// slot's result array is copied to results.  Returns the gx status of the slot.
int shim_process(void *h, int scan, int sec, int ns, const unsigned char **data, const int *datalen,
                 const int **control, int controllen, float *results)
{
  ShimJob *j = (ShimJob *)h;
  GpuCore *c = j->core;
  Core::processslot *slot = &(c->procslots[0]);
  slot->offsets[0] = scan;
  slot->offsets[1] = sec;
  slot->offsets[2] = ns;
  slot->configindex = 0;
  const int nds = j->config->getNumDataStreams();
  for (int d = 0; d < nds; d++) {
    slot->databuffer[d] = (u8 *)data[d];
    slot->datalengthbytes[d] = datalen[d];
    const int cl = controllen < c->controllength ? controllen : c->controllength;
    memset(slot->controlbuffer[d], 0, sizeof(s32) * c->controllength);
    memcpy(slot->controlbuffer[d], control[d], sizeof(s32) * cl);
  }
  const int st = c->correlateslot(0);
  memcpy(results, slot->results, sizeof(cf32) * j->config->getCoreResultLength(0));
  for (int d = 0; d < nds; d++) slot->databuffer[d] = j->origbuffers[d];
  return st;
}

// GpuMode of datastream `station` over FFT blocks 0 .. nblocks-1 of the slot
// shim_process last correlated: per block its spectra (nbands x nchan cf32)
// and data weight, then the autocorrelations [2][nbands][nchan] cf32 and the
// weights [2][nbands] accumulated over the blocks.
int shim_mode_blocks(void *h, int station, int nblocks, float *spectra, float *dataweights, float *autos,
                     float *weights)
{
  ShimJob *j = (ShimJob *)h;
  GpuMode *m = GpuMode::create(j->config, 0, station, j->core->handle(0));
  if (!m) return -1;
  m->zeroAutocorrelations();
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
  delete m;
  return 0;
}

void shim_close(void *h)
{
  ShimJob *j = (ShimJob *)h;
  if (!j) return;
  for (size_t d = 0; d < j->origbuffers.size(); d++) j->core->procslots[0].databuffer[d] = j->origbuffers[d];
  delete j->core;
  delete j->config;
  delete j;
}
}
