// Reference DataStream harness (test infrastructure only).
//
// Drives the reference's VDIF DataStream bookkeeping -- DataStream::initialise
// (datastream.cpp:116-230), VDIFDataStream::dataRead (vdiffile.cpp:668-860,
// the multiplexing of raw VDIF into one buffer segment and the segment's
// time) and DataStream/VDIFDataStream::calculateControlParams
// (datastream.cpp:368-627, vdiffile.cpp:348-470) -- on raw frames handed in
// from Python, single-threaded:
//   * the reader thread is not started; the raw bytes are placed in the read
//     buffer's slots 1.. as that thread leaves them at the end of a file
//     (vdiffile.cpp:293-330: lastslot / endindex), and dataRead is called for
//     the segments in the order the test chooses;
//   * the multiplexer set-up of VDIFDataStream::initialiseFile (vdiffile.cpp:
//     510-546) is made with the same vdifio calls, without opening a file;
//   * vdiffile.cpp is compiled with vdifmux renamed to gx_ref_vdifmux_spy,
//     which records the window each dataRead hands the multiplexer and calls
//     the real vdifmux, so that the device ring can be fed the same windows;
//   * calculateControlParams is followed by the wrap copy of
//     DataStream::execute (datastream.cpp:296-305); nothing is sent.
#include <mpi.h>
#include <cstdio>
#include <cstring>
#include <vector>
#include "architecture.h"
#include "configuration.h"
#include "datastream.h"
#include "mode.h"
#include "vdiffile.h"
#include "vdifio.h"

extern "C" Configuration *ref_job_config(void *h);

namespace {
struct Spy {
  const unsigned char *src = nullptr;
  long long srcsize = 0, destsize = 0, start = 0;
};
Spy g_spy;

struct RefDs {
  VDIFDataStream *ds = nullptr;
  long long rawlen = 0;
};
}  // namespace

extern "C" {

int gx_ref_vdifmux_spy(unsigned char *dest, int destSize, const unsigned char *src, int srcSize,
                       const struct vdif_mux *vm, int64_t startOutputFrameNumber, struct vdif_mux_statistics *stats)
{
  g_spy.src = src;
  g_spy.srcsize = srcSize;
  g_spy.destsize = destSize;
  g_spy.start = startOutputFrameNumber;
  return vdifmux(dest, destSize, src, srcSize, vm, startOutputFrameNumber, stats);
}

// A VDIF DataStream of datastream ds holding the raw bytes [raw, raw + rawlen)
// of one scan file; NULL if they do not fit in read slots 1..(slots - 3).
void *ref_ds_open(void *job, int ds, const unsigned char *raw, long long rawlen)
{
  Configuration *config = ref_job_config(job);
  int cid = 0;
  VDIFDataStream *d = new VDIFDataStream(config, ds, ds + 1, 1, &cid, config->getDDataBufferFactor(),
                                         config->getDNumDataSegments());
  d->initialise();
  // DataStream::execute's starting segments (datastream.cpp:258-259)
  d->waitsegment = 0;
  d->atsegment = 0;
  // VDIFDataStream::initialiseFile's multiplexer and frame rate (vdiffile.cpp:510-546, 576)
  const int ci = 0;
  d->nbits = config->getDNumBits(ci, ds);
  const int nrecordedbands = config->getDNumRecordedBands(ci, ds);
  d->inputframebytes = config->getFrameBytes(ci, ds);
  d->framespersecond = config->getFramesPerSecond(ci, ds) / config->getDNumMuxThreads(ci, ds);
  d->nGap = d->framespersecond / 4;
  d->startOutputFrameNumber = -1;
  d->minleftoverdata = 4 * d->inputframebytes;
  d->nthreads = config->getDNumMuxThreads(ci, ds);
  d->threads = config->getDMuxThreadMap(ci, ds);
  int muxFlags = VDIF_MUX_FLAG_RESPECTGRANULARITY | VDIF_MUX_FLAG_PROPAGATEVALIDITY;
  if (config->getDSampling(ci, ds) == Configuration::COMPLEX) muxFlags |= VDIF_MUX_FLAG_COMPLEX;
  if (configurevdifmux(&d->vm, d->inputframebytes, d->framespersecond, d->nbits, d->nthreads, d->threads, d->nSort,
                       d->nGap, muxFlags) < 0) {
    delete d;
    return 0;
  }
  if (nrecordedbands > d->nthreads) setvdifmuxinputchannels(&d->vm, nrecordedbands / d->nthreads);
  else if (nrecordedbands < d->nthreads) setvdifmuxfanoutfactor(&d->vm, d->nthreads / nrecordedbands);
  // the reader thread's state once the file has been read into slots 1..
  const long long slot = d->readbufferslotsize;
  if (rawlen > (long long)(d->readbufferslots - 3) * slot) {
    delete d;
    return 0;
  }
  // zeros around the data: a window that runs past the end of the data sees
  // no stale bytes (the reader thread would leave earlier reads there)
  memset(d->readbuffer, 0, d->readbuffersize);
  memcpy(d->readbuffer + slot, raw, rawlen);
  d->lastslot = (int)(1 + rawlen / slot);
  d->endindex = slot + rawlen;
  d->lockstart = d->lockend = -1;
  d->dataremaining = true;
  RefDs *r = new RefDs();
  r->ds = d;
  r->rawlen = rawlen;
  return r;
}

// geom: bufferbytes, readbytes, numsegments, overflow (allocated past the
// buffer), sendbytes, blockspersend, controllength, bytespersamplenum,
// bytespersampledenom, bytesbetweenintegerns, nsinc, framegranularity,
// read slot size, frames per second; dbl: sampletimens
void ref_ds_geometry(void *p, long long *geom, double *dbl)
{
  VDIFDataStream *d = ((RefDs *)p)->ds;
  const DataStream::readinfo &b = d->bufferinfo[0];
  geom[0] = d->bufferbytes;
  geom[1] = d->readbytes;
  geom[2] = d->numdatasegments;
  geom[3] = int((((long long)d->config->getDataBytes(0, d->streamnum)) *
                 ((long long)(d->config->getSubintNS(0) + d->config->getGuardNS(0)))) / d->config->getSubintNS(0));
  geom[4] = b.sendbytes;
  geom[5] = b.blockspersend;
  geom[6] = b.controllength;
  geom[7] = b.bytespersamplenum;
  geom[8] = b.bytespersampledenom;
  geom[9] = b.bytesbetweenintegerns;
  geom[10] = b.nsinc;
  geom[11] = d->vm.frameGranularity;
  geom[12] = d->readbufferslotsize;
  geom[13] = d->framespersecond;
  dbl[0] = b.sampletimens;
}

// dataRead(segment).  win: raw offset and size of the window the
// multiplexer saw, the destination size, the start frame it was given;
// seg: scan, scanseconds, scanns, validbytes, readto of the segment.
// Returns 0, or -1 if dataRead stopped (end of the data).
int ref_ds_read(void *p, int segment, long long *win, int *seg)
{
  RefDs *r = (RefDs *)p;
  VDIFDataStream *d = r->ds;
  if (!d->dataremaining) return -1;
  g_spy = Spy();
  d->dataRead(segment);
  win[0] = g_spy.src ? (long long)(g_spy.src - (d->readbuffer + d->readbufferslotsize)) : -1;
  win[1] = g_spy.srcsize;
  win[2] = g_spy.destsize;
  win[3] = g_spy.start;
  const DataStream::readinfo &b = d->bufferinfo[segment];
  seg[0] = b.scan;
  seg[1] = b.scanseconds;
  seg[2] = b.scanns;
  seg[3] = b.validbytes;
  seg[4] = b.readto ? 1 : 0;
  return 0;
}

// Overwrites a segment's description (for walks over made-up segment tables).
void ref_ds_set_segment(void *p, int segment, const int *seg)
{
  VDIFDataStream *d = ((RefDs *)p)->ds;
  DataStream::readinfo &b = d->bufferinfo[segment];
  b.scan = seg[0];
  b.scanseconds = seg[1];
  b.scanns = seg[2];
  b.validbytes = seg[3];
  b.readto = seg[4] != 0;
}

// calculateControlParams for one subint, then the wrap copy of execute.
// ctrl: the control words (controllength); info: send start, segment,
// bytes sent (1 for an invalid subint).
int ref_ds_control(void *p, int scan, int sec, int ns, int *ctrl, int *info)
{
  VDIFDataStream *d = ((RefDs *)p)->ds;
  const int startpos = d->calculateControlParams(scan, sec, ns);
  DataStream::readinfo &b = d->bufferinfo[d->atsegment];
  const int bufferremaining = d->bufferbytes - startpos;
  if (bufferremaining < b.sendbytes)
    memcpy(&d->databuffer[d->bufferbytes], d->databuffer, b.sendbytes - bufferremaining);
  const s32 *cw = b.controlbuffer[b.numsent];
  memcpy(ctrl, cw, sizeof(int) * b.controllength);
  info[0] = startpos;
  info[1] = d->atsegment;
  info[2] = cw[1] == Mode::INVALID_SUBINT ? 1 : b.sendbytes;
  return b.controllength;
}

const unsigned char *ref_ds_buffer(void *p) { return ((RefDs *)p)->ds->databuffer; }

void ref_ds_close(void *p)
{
  RefDs *r = (RefDs *)p;
  if (!r) return;
  VDIFDataStream *d = r->ds;
  d->unlockAllSlots();
  delete d;
  delete r;
}

}  // extern "C"
