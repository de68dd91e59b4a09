// Station data rings in device memory and the control words of every subint
// computed on the device from their segment tables.
//
// The reference's DataStream keeps, per station, a data buffer of DATA BUFFER
// FACTOR x (largest data bytes of a subint) cut into NUM DATA SEGMENTS
// segments (DataStream::initialise, datastream.cpp:116-230).  A reader thread
// fills segments in order (VDIFDataStream::dataRead multiplexes raw VDIF into
// one segment and stamps it with the time of its first output frame,
// vdiffile.cpp:668-860); for each subint the main thread walks the segments
// to the one holding the subint's first sample, works out the byte offset and
// the 30-bit valid-flag words of the FFT blocks (calculateControlParams,
// datastream.cpp:368-627), snaps the offset back to a whole multiplexed frame
// (the VDIF override, vdiffile.cpp:348-470), and sends the bytes from there,
// first copying the start of the buffer past its end when the send wraps
// (DataStream::execute, datastream.cpp:296-305).
//
// Here the buffer is a device allocation per station, the segment table sits
// in device memory beside it, and that walk runs in a kernel -- one thread per
// station -- which writes the control words, the data pointer and the data
// length straight into the subint tables the F-step reads.  A second kernel
// copies the wrapped part of a send.  The only per-subint host inputs are the
// two order-0 delays at the ends of the data span, which come from the delay
// model (they do not depend on the data).  The same walk compiled for the
// host (gx_ring_control_host) serves callers without a device and the tests.
#include <cuda_runtime.h>
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/gxcorr.h"
#include "gx_handle.h"
#include "gx_host.h"

namespace {

constexpr int kFlagsPerInt = 30;            // FLAGS_PER_INT (mpifxcorr.h)
constexpr int kInvalidSubint = -99999999;   // Mode::INVALID_SUBINT (mode.h)

struct RingSeg {
  int scan, scanseconds, scanns, validbytes, readto, configindex;
};

// What one station's walk keeps between subints.
struct RingPos {
  int atsegment;
  int startpos;     // last send start
  int sendlen;      // last send length (1 for an invalid subint)
  int exhausted;    // the last subint lay past every segment
};

// Per-station constants of the walk (gx_ring_geometry plus the bytes the
// frame alignment uses).
struct RingGeom {
  int bufferbytes, readbytes, numsegments, overflowbytes;
  int sendbytes, blockspersend, controllength, blockbytes;
  int bpsnum, bpsden, bbin, nsinc;
  int framebytes, payloadbytes, fps_ctrl, granularity;
  int intclockseconds;
  double sampletimens;
  long long dataspanns;
};

__host__ __device__ inline long long segtime_ns(const RingSeg &a, const RingSeg &b)
{
  // nanoseconds from segment a's first frame to segment b's
  return (long long)(b.scanseconds - a.scanseconds) * 1000000000LL + (long long)b.scanns - (long long)a.scanns;
}

// The walk for one station and one subint (scan, offsetsec, offsetns):
// writes cw[0..controllength) and returns the send start (bytes into the
// buffer).  d1 / d2: the order-0 delays (us, clock included) at the subint
// start and at the end of the data span; ok: both were found.  Returns -1
// (and an invalid subint) when no segment at or after the subint's start
// exists within one lap of the ring -- where the reference's main thread
// would wait for its reader.
__host__ __device__ int ring_walk(const RingGeom &g, const RingSeg *seg, RingPos &pos, int scan, int offsetsec,
                                  int offsetns, double d1, double d2, bool ok, int *cw)
{
  const int nseg = g.numsegments;
  auto invalid = [&](int ret) {
    cw[1] = kInvalidSubint;
    return ret;
  };
  cw[0] = scan;
  // -- the data span's first and last sample times, corrected for the delays
  //    (datastream.cpp:375-397)
  double delayus1 = d1 - g.intclockseconds * 1000000;
  long long firstoffsetns = ((long long)offsetns) - (long long)(delayus1 * 1000);
  double delayus2 = d2 - g.intclockseconds * 1000000;
  if (!ok) return invalid(0);
  long long lastoffsetns = (long long)offsetns + g.dataspanns + (long long)(-1000 * delayus2 + 0.5);
  for (int k = 0; k < 2; k++) {
    if (lastoffsetns < 0) {   // the span starts in the previous second
      offsetsec -= 1;
      firstoffsetns += 1000000000LL;
      lastoffsetns += 1000000000LL;
    }
  }
  int at = pos.atsegment;
  if (scan < seg[at].scan) return invalid(0);
  if (!seg[at].readto) return invalid(0);
  if (scan == seg[at].scan && offsetsec < seg[at].scanseconds - 3) return invalid(0);
  // -- forward to the segment that holds the first sample (datastream.cpp:440-463)
  auto nsdiff_of = [&](const RingSeg &s) {
    return (long long)(offsetsec - s.scanseconds) * 1000000000LL + firstoffsetns - (long long)s.scanns;
  };
  auto validns_of = [&](const RingSeg &s) { return ((long long)s.validbytes * (long long)g.nsinc) / g.readbytes; };
  long long nsdifference = nsdiff_of(seg[at]);
  long long validns = validns_of(seg[at]);
  int steps = 0;
  while (scan > seg[at].scan || (scan == seg[at].scan && nsdifference >= validns)) {
    if (++steps > nseg) {
      pos.atsegment = at;
      pos.exhausted = 1;
      return invalid(-1);
    }
    at = (at + 1) % nseg;
    nsdifference = nsdiff_of(seg[at]);
    validns = validns_of(seg[at]);
  }
  pos.atsegment = at;
  const RingSeg &S = seg[at];
  const RingSeg &N = seg[(at + 1) % nseg];
  cw[0] = scan;
  if (scan < S.scan || nsdifference < -g.nsinc) return invalid(0);
  if (scan > S.scan) return invalid(0);
  const int segbase = at * g.readbytes;
  // the subint's start as a fractional byte offset (datastream.cpp:488, 586)
  auto dbufferindex = [&]() {
    return segbase + ((((offsetsec - S.scanseconds) * 1.0e9 + (firstoffsetns - (long long)S.scanns)) / g.sampletimens) *
                      g.bpsnum) / g.bpsden;
  };
  const double curtime = S.scanseconds + S.scanns / 1.0e9;
  const double nexttime = N.scanseconds + N.scanns / 1.0e9;
  if (S.validbytes < g.readbytes || N.scanseconds - S.scanseconds > 2 || nexttime < curtime) {
    const double db = dbufferindex();
    const int segoff = int(db - segbase);
    if (nexttime < curtime && segoff > S.validbytes) return invalid(0);
    if (db < -g.blockbytes * g.blockspersend || db > g.bufferbytes) return invalid(0);
  }
  const int nwords = g.controllength - 3;
  for (int w = 0; w < nwords; w++) cw[3 + w] = 0;
  cw[1] = S.scanseconds;
  // -- the send start: nearest sample, on a 16-bit boundary (datastream.cpp:500-527)
  int bufferindex = segbase + (int(((offsetsec - S.scanseconds) * 1000000000LL + (firstoffsetns - (long long)S.scanns)) /
                                       g.sampletimens + 0.5) * g.bpsnum) / g.bpsden;
  if (bufferindex % 2 != 0) bufferindex--;
  if (bufferindex == g.bufferbytes) {
    if (S.scan != N.scan || segtime_ns(S, N) - (long long)g.nsinc != 0) return invalid(0);
  }
  // -- skip whole FFT blocks that start before this segment, then allow for the
  //    delay change over the skipped blocks (datastream.cpp:529-560)
  int count = 0;
  while (bufferindex < segbase && count < g.blockspersend) {
    bufferindex += g.blockbytes;
    count++;
  }
  if (bufferindex < segbase) return invalid(0);
  if (count > 0) {
    auto shift = [&](int c) {
      return (int(c * 1000.0 * (delayus2 - delayus1) / (g.sampletimens * g.blockspersend) + 0.5) * g.bpsnum) / g.bpsden;
    };
    int tosubtract = shift(count);
    if (bufferindex - tosubtract < segbase) {
      count++;
      bufferindex += g.blockbytes;
      if (count == g.blockspersend) return invalid(0);
      tosubtract = shift(count);
      bufferindex -= tosubtract;
    }
    bufferindex -= bufferindex % 2;
  }
  // -- back to a byte where the time is a whole nanosecond; the first sample's time
  //    (datastream.cpp:562-574)
  int segoffbytes = bufferindex - segbase;
  bufferindex -= segoffbytes % g.bbin;
  segoffbytes -= segoffbytes % g.bbin;
  const long long segoffns = (long long)(double(segoffbytes * g.bpsden / g.bpsnum) * g.sampletimens + 0.5);
  long long a = (long long)cw[1] + segoffns / 1000000000LL;
  long long b = (long long)S.scanns + segoffns % 1000000000LL;
  a += b / 1000000000LL;
  b %= 1000000000LL;
  cw[1] = (int)a;
  cw[2] = (int)b;
  // -- valid flags: every block whose bytes the segment (or a contiguous next
  //    segment) holds (datastream.cpp:576-619)
  const bool contiguous = S.validbytes == g.readbytes && segtime_ns(S, N) == (long long)g.nsinc;
  if ((S.validbytes - segoffbytes >= g.sendbytes) ||
      (contiguous && (S.validbytes - segoffbytes + N.validbytes) > g.sendbytes)) {
    for (int i = count; i < g.blockspersend; i++) cw[3 + i / kFlagsPerInt] |= 1 << (i % kFlagsPerInt);
  } else {
    const double db = dbufferindex();
    if (db < -g.blockbytes * g.blockspersend || db > g.bufferbytes) return invalid(0);
    for (int i = count; i < g.blockspersend; i++) {
      if (bufferindex + i * g.blockbytes - segbase < S.validbytes)
        cw[3 + i / kFlagsPerInt] |= 1 << (i % kFlagsPerInt);
      else if (contiguous && (S.validbytes - segoffbytes + N.validbytes) > i * g.blockbytes)
        cw[3 + i / kFlagsPerInt] |= 1 << (i % kFlagsPerInt);
    }
    // only whole flag words are looked at here (datastream.cpp:606-614)
    bool somegood = false;
    for (int w = 0; w < g.blockspersend / kFlagsPerInt; w++)
      if (cw[3 + w] > 0) somegood = true;
    if (!somegood) return invalid(0);
  }
  // -- the VDIF form: back to the start of a whole multiplexed frame
  //    (vdiffile.cpp:348-470)
  int look = at;
  if (S.configindex < 0) {
    look = (at + 1) % nseg;   // every segment here shares the one configuration's nsinc
  }
  if (seg[look].configindex < 0) {
    look = (look + 1) % nseg;
    if (seg[look].configindex < 0) return invalid(bufferindex);
  }
  const int vlbaoffset = bufferindex - segbase;
  if (vlbaoffset < 0) return invalid(0);
  int framesin = vlbaoffset / g.payloadbytes;
  framesin -= framesin % g.granularity;
  const long long fns = (long long)S.scanns + (long long)((1000000000.0 * framesin) / g.fps_ctrl);
  cw[1] = S.scanseconds + (int)(fns / 1000000000);
  cw[2] = (int)(fns % 1000000000);
  bufferindex = segbase + framesin * g.framebytes;
  if (bufferindex == g.bufferbytes) {
    // this comparison is made in 32-bit arithmetic (vdiffile.cpp:448-450)
    const unsigned int d = (unsigned)(N.scanseconds - S.scanseconds) * 1000000000u + (unsigned)N.scanns -
                           (unsigned)S.scanns - (unsigned)g.nsinc;
    if (S.scan != N.scan || d != 0u) return invalid(0);
  }
  if (bufferindex > g.bufferbytes) return invalid(0);
  return bufferindex;
}

// One thread per station: the walk, then the subint tables the F-step reads.
__global__ void ring_control_kernel(int nst, const RingGeom *__restrict__ geom, const RingSeg *__restrict__ seg,
                                    RingPos *__restrict__ pos, const double *__restrict__ req, uint8_t *const *base,
                                    int scan, int sec, int ns, int64_t *datalen, const uint8_t **dataptr,
                                    int32_t *control, int ctrlstride)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nst) return;
  const RingGeom g = geom[s];
  RingPos p = pos[s];
  p.exhausted = 0;
  // the staged placeholder words are zero; the walk writes them in place
  int *cw = reinterpret_cast<int *>(control + (size_t)s * ctrlstride);
  const double *r = req + 3 * s;
  int start = ring_walk(g, seg + (size_t)s * g.numsegments, p, scan, sec, ns, r[0], r[1], r[2] != 0.0, cw);
  if (start < 0) start = 0;
  const bool valid = cw[1] != kInvalidSubint;
  p.startpos = start;
  p.sendlen = valid ? g.sendbytes : 1;
  pos[s] = p;
  dataptr[s] = base[s] + start;
  datalen[s] = p.sendlen;
}

// The part of a send past the buffer's end: the buffer's first bytes, copied
// behind it (DataStream::execute, datastream.cpp:296-305).
__global__ void ring_wrap_kernel(int nst, const RingGeom *__restrict__ geom, const RingPos *__restrict__ pos,
                                 uint8_t *const *base)
{
  const int s = blockIdx.y;
  if (s >= nst) return;
  // at most the overflow region (a send start never passes the buffer's end)
  const int n = min(geom[s].sendbytes - (geom[s].bufferbytes - pos[s].startpos), geom[s].overflowbytes);
  if (n <= 0) return;
  uint8_t *b = base[s];
  const int bb = geom[s].bufferbytes;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[bb + i] = b[i];
}

long long gcd_ll(long long a, long long b)
{
  while (b) {
    const long long t = a % b;
    a = b;
    b = t;
  }
  return a;
}

}  // namespace

struct gx_ring {
  std::string err;
  gx_handle *h = nullptr;
  int device = -1;
  int nst = 0, nseg = 0;
  std::vector<RingGeom> geom;
  std::vector<gx_ring_geometry> pub;
  std::vector<RingSeg> segs;              // host copy [station][segment]
  std::vector<RingPos> hpos;              // the host walk's positions
  std::vector<gx_vdifmux *> mux;          // per station (null: this station's form is not multiplexed here)
  std::vector<gx_status> mux_status;
  std::vector<long long> next_frame;      // per station: first output frame number of the next read (-1: any)
  std::vector<uint8_t *> d_buf;           // per station: bufferbytes + overflow + 4
  uint8_t **d_base = nullptr;
  RingGeom *d_geom = nullptr;
  RingSeg *d_segs = nullptr;
  RingPos *d_pos = nullptr;
  cudaStream_t last_stream = nullptr;
  bool pending = false;                   // a device walk was enqueued since the last read-back

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

// Enqueued by gx_enqueue_subint right after the subint tables reach the
// device: the walk writes each station's control words, data pointer and
// length over the staged placeholders, then the wrapped sends are copied.
gx_status gx_ring_enqueue_control(gx_ring *r, gx_handle *h, cudaStream_t st)
{
  uint8_t *sub = h->d_sub;
  const int nst = r->nst;
  ring_control_kernel<<<(nst + 63) / 64, 64, 0, st>>>(
      nst, r->d_geom, r->d_segs, r->d_pos, reinterpret_cast<const double *>(sub + h->o_ring), r->d_base,
      h->ring_scan, h->ring_sec, h->ring_ns, reinterpret_cast<int64_t *>(sub + h->o_len),
      reinterpret_cast<const uint8_t **>(sub + h->o_ptr), reinterpret_cast<int32_t *>(sub + h->o_ctrl), h->ctrlstride);
  int maxsend = 0;
  for (const RingGeom &g : r->geom) maxsend = std::max(maxsend, g.sendbytes);
  const int blocks = std::max(1, std::min(148 * 4, (maxsend + 255) / 256));
  ring_wrap_kernel<<<dim3(blocks, nst), 256, 0, st>>>(nst, r->d_geom, r->d_pos, r->d_base);
  r->last_stream = st;
  r->pending = true;
  return r->cuda(cudaGetLastError(), "ring kernels");
}

extern "C" {

gx_status gx_ring_open(gx_handle *h, int databufferfactor, int numdatasegments, gx_ring **out)
{
  if (!h || !out) return GX_ERR_ARG;
  if (!h->model || !h->meta) return h->fail(GX_ERR_STATE, "gx_ring needs a handle opened with a delay model (gx_open_input)");
  if (databufferfactor <= 0) databufferfactor = h->meta->data_buffer_factor;
  if (numdatasegments <= 0) numdatasegments = h->meta->num_data_segments;
  if (databufferfactor <= 0 || numdatasegments <= 0) return h->fail(GX_ERR_ARG, "no DATA BUFFER FACTOR / NUM DATA SEGMENTS");
  std::unique_ptr<gx_ring> r(new gx_ring());
  r->h = h;
  r->device = h->device;
  const gx_job_desc &d = h->jd;
  r->nst = d.nstations;
  r->nseg = numdatasegments;
  const int subint = d.subint_ns;
  const int bps = h->J.blocks_per_send;
  // GUARD NANOSECONDS 0 is replaced by the largest slip of any datastream: the
  // time to a whole nanosecond plus the delay change over a subint at the
  // model's largest rate (configuration.cpp:2941-2981)
  int guard = d.guard_ns;
  if (guard == 0) {
    int maxslip = 0;
    for (int s = 0; s < d.nstations; s++) {
      const gx_station_desc &st = h->st[s];
      double samplens = 500.0 / h->fr[st.recfreq[0]].bw_mhz;
      if (st.is_complex) samplens *= 2;
      const int nsb = st.nbits * (st.is_complex ? 2 : 1);
      const int den = (st.nbands * nsb) / 8 == 0 ? 8 / (st.nbands * nsb) : 1;
      double nsacc = 0.0;
      const float tiny = 0.000000001f;   // Mode::TINY
      do {
        nsacc += den * samplens;
      } while (!(std::fabs(nsacc - int(nsacc + 0.5)) < 50 * tiny));
      nsacc += h->model->maxrate[h->model->station_of_datastream[s]] * subint * 0.000001;
      const int slip = nsacc > 0 ? int(nsacc + 0.99) : 0;
      maxslip = std::max(maxslip, slip);
    }
    guard = maxslip;
  }
  for (int s = 0; s < d.nstations; s++) {
    const gx_station_desc &st = h->st[s];
    const gx_freq_desc &f0 = h->fr[st.recfreq[0]];
    const int nrb = st.nbands, nbits = st.nbits, decim = 1;
    const int nmux = st.nmuxthreads > 0 ? st.nmuxthreads : 1;
    const int fb_mux = st.framebytes;                                         // getMultiplexedFrameBytes
    const int fb_in = st.nmuxthreads > 0 ? (st.framebytes - 32) / nmux + 32 : st.framebytes;   // getFrameBytes
    const int payload_in = fb_in - 32;                                        // getFramePayloadBytes
    const int payload_mux = fb_mux - 32;
    const double bw = f0.bw_mhz;
    const int numchannels = f0.nchan;
    // Configuration::getFramesPerSecond (configuration.cpp:654-668)
    const double fpsd = 2.0e6 * bw * nrb * nbits * decim / (8 * payload_in);
    // bytes per time sample (configuration.cpp:1655-1664)
    const int nsb = nbits * (st.is_complex ? 2 : 1);
    int bpsnum = (nrb * nsb * decim) / 8, bpsden = 1;
    if (bpsnum == 0) {
      bpsnum = 1;
      bpsden = 8 / (nrb * nsb * decim);
    }
    // Configuration::getDataBytes (configuration.cpp:790-818)
    int validlength = (decim * bps * nrb * 2 * nbits * numchannels) / 8;
    validlength += (decim * (int)(guard / (1000.0 / (bw * 2.0)) + 1.0) * nrb * nbits) / 8;
    const int numframes = validlength / payload_mux + 2;
    const long long databytes = (long long)numframes * fb_mux;
    if ((unsigned long long)databytes * (unsigned long long)databufferfactor > 2147483647ULL)
      return h->fail(GX_ERR_ARG, "station " + std::to_string(s) + ": ring buffer past 2^31 bytes");
    RingGeom g{};
    g.bufferbytes = (int)(databufferfactor * databytes);
    g.readbytes = g.bufferbytes / numdatasegments;
    g.numsegments = numdatasegments;
    const int overflow = int(((long long)databytes * (long long)(subint + guard)) / subint);
    g.overflowbytes = overflow;
    // DataStream::updateConfig then its VDIF form (datastream.cpp:745, vdiffile.cpp:491)
    g.sendbytes = int((((double)overflow) * ((double)subint)) / (subint + guard) + 0.5);
    g.blockspersend = bps;
    g.controllength = bps / kFlagsPerInt + 3 + (bps % kFlagsPerInt > 0 ? 1 : 0);
    g.bpsnum = bpsnum;
    g.bpsden = bpsden;
    g.sampletimens = 500.0 / bw;
    if (st.is_complex) g.sampletimens *= 2;
    int bbin = 0;
    double nsacc = 0.0;
    const float tiny = 0.000000001f;   // Mode::TINY
    do {
      nsacc += bpsden * g.sampletimens;
      bbin += bpsnum;
    } while (!(std::fabs(nsacc - int(nsacc + 0.5)) < 50 * tiny));
    g.bbin = bbin;
    const int ofps = (int)(fpsd / nmux);
    g.nsinc = int(((g.bufferbytes / numdatasegments) / fb_mux) * (1000000000.0 / double(ofps)) + 0.5);
    const int fftchannels = st.is_complex ? numchannels : numchannels * 2;
    g.blockbytes = (fftchannels * bpsnum) / bpsden;
    g.framebytes = fb_mux;
    g.payloadbytes = payload_in * nmux;
    g.fps_ctrl = ((int)fpsd) / nmux;
    g.granularity = (int)(ofps / gcd_ll(ofps, 1000000000LL));
    g.intclockseconds = st.clock_int_seconds;
    long long span = (long long)(numchannels * bps * 2 * g.sampletimens + 0.5);
    if (st.is_complex) span /= 2;
    g.dataspanns = span;
    if (g.readbytes <= 0 || g.payloadbytes <= 0 || ofps <= 0 || g.granularity <= 0)
      return h->fail(GX_ERR_ARG, "station " + std::to_string(s) + ": degenerate ring geometry");
    r->geom.push_back(g);
    gx_ring_geometry P{};
    P.bufferbytes = g.bufferbytes;
    P.readbytes = g.readbytes;
    P.numsegments = numdatasegments;
    P.overflowbytes = overflow;
    P.sendbytes = g.sendbytes;
    P.blockspersend = bps;
    P.controllength = g.controllength;
    P.blockbytes = g.blockbytes;
    P.bytespersamplenum = bpsnum;
    P.bytespersampledenom = bpsden;
    P.bytesbetweenintegerns = bbin;
    P.nsinc = g.nsinc;
    P.framebytes = fb_mux;
    P.payloadbytes = g.payloadbytes;
    P.framespersecond = ofps;
    P.framegranularity = g.granularity;
    P.intclockseconds = g.intclockseconds;
    P.sampletimens = g.sampletimens;
    P.dataspanns = g.dataspanns;
    r->pub.push_back(P);
    // the multiplexer as VDIFDataStream::initialiseFile configures it (vdiffile.cpp:510-546)
    std::vector<int> ids(nmux, 0);
    for (int t = 0; t < st.nmuxthreads; t++) ids[t] = st.muxthread[t];
    gx_vdifmux *m = nullptr;
    gx_status ms = GX_ERR_UNSUPPORTED;
    if (nrb >= nmux && nrb % nmux == 0) {
      int flags = GX_VDIFMUX_RESPECTGRANULARITY | GX_VDIFMUX_PROPAGATEVALIDITY;
      if (st.is_complex) flags |= GX_VDIFMUX_COMPLEX;
      ms = gx_vdifmux_open(fb_in, ofps, nbits, nmux, ids.data(), nrb / nmux, 32, ofps / 4, flags, h->device, &m);
      if (ms == GX_OK) {
        int ofb = 0;
        gx_vdifmux_info(m, &ofb, nullptr, nullptr);
        if (ofb != fb_mux) {
          gx_vdifmux_close(m);
          m = nullptr;
          ms = GX_ERR_ARG;
        }
      }
    }
    r->mux.push_back(m);
    r->mux_status.push_back(ms);
    r->next_frame.push_back(-1);
  }
  // segments as DataStream::initialise leaves them (datastream.cpp:197-207)
  r->segs.assign((size_t)r->nst * r->nseg, RingSeg{0, 0, 0, 0, 0, 0});
  r->hpos.assign(r->nst, RingPos{0, 0, 1, 0});
  if (h->device >= 0) {
    gx_status e;
    if ((e = r->cuda(cudaSetDevice(h->device), "cudaSetDevice")) != GX_OK) return h->fail(e, r->err);
    r->d_buf.assign(r->nst, nullptr);
    for (int s = 0; s < r->nst; s++) {
      const size_t bytes = (size_t)r->geom[s].bufferbytes + r->pub[s].overflowbytes + 4;
      if ((e = r->cuda(cudaMalloc(&r->d_buf[s], bytes), "cudaMalloc")) != GX_OK) return h->fail(GX_ERR_NOMEM, r->err);
      if ((e = r->cuda(cudaMemset(r->d_buf[s], 0, bytes), "cudaMemset")) != GX_OK) return h->fail(e, r->err);
    }
    if ((e = r->cuda(cudaMalloc(&r->d_base, sizeof(uint8_t *) * r->nst), "cudaMalloc")) != GX_OK ||
        (e = r->cuda(cudaMalloc(&r->d_geom, sizeof(RingGeom) * r->nst), "cudaMalloc")) != GX_OK ||
        (e = r->cuda(cudaMalloc(&r->d_segs, sizeof(RingSeg) * r->segs.size()), "cudaMalloc")) != GX_OK ||
        (e = r->cuda(cudaMalloc(&r->d_pos, sizeof(RingPos) * r->nst), "cudaMalloc")) != GX_OK)
      return h->fail(GX_ERR_NOMEM, r->err);
    if ((e = r->cuda(cudaMemcpy(r->d_base, r->d_buf.data(), sizeof(uint8_t *) * r->nst, cudaMemcpyHostToDevice),
                     "cudaMemcpy")) != GX_OK ||
        (e = r->cuda(cudaMemcpy(r->d_geom, r->geom.data(), sizeof(RingGeom) * r->nst, cudaMemcpyHostToDevice),
                     "cudaMemcpy")) != GX_OK ||
        (e = r->cuda(cudaMemcpy(r->d_segs, r->segs.data(), sizeof(RingSeg) * r->segs.size(), cudaMemcpyHostToDevice),
                     "cudaMemcpy")) != GX_OK ||
        (e = r->cuda(cudaMemcpy(r->d_pos, r->hpos.data(), sizeof(RingPos) * r->nst, cudaMemcpyHostToDevice),
                     "cudaMemcpy")) != GX_OK)
      return h->fail(e, r->err);
  }
  *out = r.release();
  return GX_OK;
}

gx_status gx_ring_geometry_get(const gx_ring *r, int station, gx_ring_geometry *g)
{
  if (!r || !g || station < 0 || station >= r->nst) return GX_ERR_ARG;
  *g = r->pub[station];
  return GX_OK;
}

gx_status gx_ring_buffer(const gx_ring *r, int station, uint8_t **dev_buffer)
{
  if (!r || !dev_buffer || station < 0 || station >= r->nst) return GX_ERR_ARG;
  if (r->device < 0) return GX_ERR_STATE;
  *dev_buffer = r->d_buf[station];
  return GX_OK;
}

static gx_status put_segment(gx_ring *r, int station, int segment, cudaStream_t st)
{
  if (r->device < 0) return GX_OK;
  const size_t i = (size_t)station * r->nseg + segment;
  // from pageable memory: the source may be reused as soon as the call returns
  return r->cuda(cudaMemcpyAsync(r->d_segs + i, &r->segs[i], sizeof(RingSeg), cudaMemcpyHostToDevice, st),
                 "cudaMemcpyAsync");
}

gx_status gx_ring_read(gx_ring *r, int station, int segment, int scan, const uint8_t *dev_raw, long long raw_bytes,
                       long long *consumed, void *stream)
{
  if (!r || !dev_raw || station < 0 || station >= r->nst || segment < 0 || segment >= r->nseg || raw_bytes < 0)
    return GX_ERR_ARG;
  if (r->device < 0) return r->fail(GX_ERR_STATE, "host-only ring");
  if (!r->mux[station])
    return r->fail(r->mux_status[station] == GX_ERR_UNSUPPORTED ? GX_ERR_UNSUPPORTED : GX_ERR_ARG,
                   "this station's frames are not multiplexed by the device multiplexer");
  gx_handle *h = r->h;
  if (scan < 0 || scan >= (int)h->model->scans.size()) return r->fail(GX_ERR_ARG, "scan out of range");
  cudaStream_t st = (cudaStream_t)stream;
  gx_status e;
  if ((e = r->cuda(cudaSetDevice(r->device), "cudaSetDevice")) != GX_OK) return e;
  const RingGeom &g = r->geom[station];
  uint8_t *dest = r->d_buf[station] + (size_t)segment * g.readbytes;
  gx_vdifmux_stats stats{};
  e = gx_vdifmux_run(r->mux[station], dev_raw, raw_bytes, dest, g.readbytes, r->next_frame[station], &stats, st);
  if (e != GX_OK) return r->fail(e, std::string("multiplexer: ") + gx_vdifmux_last_error(r->mux[station]));
  RingSeg &S = r->segs[(size_t)station * r->nseg + segment];
  if (consumed) *consumed = stats.src_used;
  if (stats.returned_bytes <= 0) {
    // no data: the segment holds nothing (vdiffile.cpp:748-764)
    S.validbytes = 0;
    return put_segment(r, station, segment, st);
  }
  S.validbytes = (int)stats.dest_used;
  S.readto = 1;
  if (S.validbytes > 0) {
    // the segment's time from its first output frame (vdiffile.cpp:771-790)
    const int fps = r->pub[station].framespersecond;
    const long long sf = stats.start_frame;
    S.scanns = (int)(((sf % fps) * 1000000000LL) / fps);
    S.scan = scan;
    const HostModel &M = *h->model;
    const int scanstart = (M.modelmjd - M.jobmjd) * 86400 + (M.modelstartseconds - M.jobseconds) +
                          M.scans[scan].offsetseconds;
    int ss = (int)((sf / fps) % 86400) + g.intclockseconds - h->meta->start_seconds - scanstart;
    if (ss > 86400 / 2) ss -= 86400;
    else if (ss < -86400 / 2) ss += 86400;
    S.scanseconds = ss;
    r->next_frame[station] = sf + stats.output_frames;
  } else {
    r->next_frame[station] = -1;
  }
  return put_segment(r, station, segment, st);
}

gx_status gx_ring_set_segment(gx_ring *r, int station, int segment, const gx_ring_segment *seg)
{
  if (!r || !seg || station < 0 || station >= r->nst || segment < 0 || segment >= r->nseg) return GX_ERR_ARG;
  if (seg->validbytes < 0 || seg->validbytes > r->geom[station].readbytes) return r->fail(GX_ERR_ARG, "validbytes out of range");
  RingSeg &S = r->segs[(size_t)station * r->nseg + segment];
  S = RingSeg{seg->scan, seg->scanseconds, seg->scanns, seg->validbytes, seg->readto ? 1 : 0, seg->configindex};
  if (r->device >= 0) {
    gx_status e;
    if ((e = r->cuda(cudaSetDevice(r->device), "cudaSetDevice")) != GX_OK) return e;
    if ((e = put_segment(r, station, segment, r->h->stream)) != GX_OK) return e;
    return r->cuda(cudaStreamSynchronize(r->h->stream), "cudaStreamSynchronize");
  }
  return GX_OK;
}

gx_status gx_ring_get_segment(const gx_ring *r, int station, int segment, gx_ring_segment *seg)
{
  if (!r || !seg || station < 0 || station >= r->nst || segment < 0 || segment >= r->nseg) return GX_ERR_ARG;
  const RingSeg &S = r->segs[(size_t)station * r->nseg + segment];
  *seg = gx_ring_segment{S.scan, S.scanseconds, S.scanns, S.validbytes, S.readto, S.configindex};
  return GX_OK;
}

// The order-0 delays at both ends of a station's data span for a subint
// (datastream.cpp:375-383); out[2] = 1 when both exist.
static void span_delays(const gx_ring *r, int station, int scan, int sec, int ns, double out[3])
{
  const HostModel &M = *r->h->model;
  const double t1 = (double)sec + ((double)ns) / 1.0e9;
  const double t2 = (double)sec + ((double)ns + r->geom[station].dataspanns) / 1.0e9;
  out[0] = out[1] = 0.0;
  bool ok = M.delay0(station, scan, t1, &out[0]);
  ok = ok && M.delay0(station, scan, t2, &out[1]);
  out[2] = ok ? 1.0 : 0.0;
}

gx_status gx_ring_control_host(gx_ring *r, int station, int scan, int sec, int ns, int32_t *control, int *startpos)
{
  if (!r || !control || station < 0 || station >= r->nst) return GX_ERR_ARG;
  double dl[3];
  span_delays(r, station, scan, sec, ns, dl);
  const RingGeom &g = r->geom[station];
  std::vector<int> cw(g.controllength, 0);
  RingPos &p = r->hpos[station];
  p.exhausted = 0;
  int start = ring_walk(g, &r->segs[(size_t)station * r->nseg], p, scan, sec, ns, dl[0], dl[1], dl[2] != 0.0, cw.data());
  const bool exhausted = start < 0;
  if (start < 0) start = 0;
  p.startpos = start;
  memcpy(control, cw.data(), sizeof(int32_t) * g.controllength);
  if (startpos) *startpos = start;
  return exhausted ? r->fail(GX_ERR_STATE, "the subint lies past every filled segment") : GX_OK;
}

gx_status gx_ring_subint_device(gx_handle *h, gx_ring *r, int scan, int sec, int ns, double scan_start_sec,
                                float *dev_results, void *stream)
{
  if (!h || !r || !dev_results || r->h != h) return GX_ERR_ARG;
  if (h->device < 0) return h->fail(GX_ERR_STATE, "host-only handle (opened with device -1)");
  if (!h->inflight.empty()) return h->fail(GX_ERR_STATE, "subints of gx_subint_async not yet waited for");
  for (const RingGeom &g : r->geom)
    if (g.controllength != h->ctrlstride) return h->fail(GX_ERR_STATE, "control word count differs from the handle's");
  CKR(h, cudaSetDevice(h->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : h->stream;
  h->last_stream = st;
  h->slot = 0;
  const int nst = r->nst;
  // placeholders the device walk overwrites: empty data, zero control words
  std::vector<int32_t> zero((size_t)h->ctrlstride, 0);
  std::vector<const int32_t *> ctrl(nst, zero.data());
  std::vector<int64_t> lens(nst, 0);
  std::vector<const uint8_t *> data(r->d_buf.begin(), r->d_buf.end());
  gx_subint_desc sd{};
  sd.scan = scan;
  sd.sec = sec;
  sd.ns = ns;
  sd.scan_start_sec = scan_start_sec;
  sd.interp = nullptr;
  sd.data = data.data();
  sd.datalen = lens.data();
  sd.control = ctrl.data();
  sd.controllen = h->ctrlstride;
  gx_status e = gx_stage_subint(h, &sd, data.data());
  if (e != GX_OK) return e;
  double *req = reinterpret_cast<double *>(h->h_sub[0] + h->o_ring);
  for (int s = 0; s < nst; s++) span_delays(r, s, scan, sec, ns, req + 3 * s);
  h->ring_req = r;
  h->ring_scan = scan;
  h->ring_sec = sec;
  h->ring_ns = ns;
  e = gx_enqueue_subint(h, reinterpret_cast<float2 *>(dev_results), st);
  h->ring_req = nullptr;
  return e;
}

gx_status gx_ring_last_control(gx_ring *r, int32_t *control, int *startpos)
{
  if (!r) return GX_ERR_ARG;
  if (r->device < 0 || !r->pending) return r->fail(GX_ERR_STATE, "no device subint from this ring");
  gx_handle *h = r->h;
  gx_status e;
  if ((e = r->cuda(cudaSetDevice(r->device), "cudaSetDevice")) != GX_OK) return e;
  if ((e = r->cuda(cudaStreamSynchronize(r->last_stream), "cudaStreamSynchronize")) != GX_OK) return e;
  std::vector<RingPos> pos(r->nst);
  if ((e = r->cuda(cudaMemcpy(pos.data(), r->d_pos, sizeof(RingPos) * r->nst, cudaMemcpyDeviceToHost), "cudaMemcpy")) !=
      GX_OK)
    return e;
  if (control &&
      (e = r->cuda(cudaMemcpy(control, h->d_sub + h->o_ctrl, sizeof(int32_t) * h->ctrlstride * r->nst,
                              cudaMemcpyDeviceToHost),
                   "cudaMemcpy")) != GX_OK)
    return e;
  bool exhausted = false;
  for (int s = 0; s < r->nst; s++) {
    if (startpos) startpos[s] = pos[s].startpos;
    exhausted = exhausted || pos[s].exhausted;
  }
  return exhausted ? r->fail(GX_ERR_STATE, "a station's subint lay past every filled segment") : GX_OK;
}

gx_status gx_ring_reset(gx_ring *r)
{
  if (!r) return GX_ERR_ARG;
  r->hpos.assign(r->nst, RingPos{0, 0, 1, 0});
  std::fill(r->next_frame.begin(), r->next_frame.end(), -1LL);
  if (r->device >= 0) {
    gx_status e;
    if ((e = r->cuda(cudaSetDevice(r->device), "cudaSetDevice")) != GX_OK) return e;
    if ((e = r->cuda(cudaMemcpy(r->d_pos, r->hpos.data(), sizeof(RingPos) * r->nst, cudaMemcpyHostToDevice),
                     "cudaMemcpy")) != GX_OK)
      return e;
  }
  for (gx_vdifmux *m : r->mux)
    if (m) gx_vdifmux_reset_stats(m);
  return GX_OK;
}

const char *gx_ring_last_error(const gx_ring *r) { return r ? r->err.c_str() : "null ring"; }

gx_status gx_ring_close(gx_ring *r)
{
  if (!r) return GX_ERR_ARG;
  if (r->device >= 0) {
    cudaSetDevice(r->device);
    for (uint8_t *b : r->d_buf) cudaFree(b);
    cudaFree(r->d_base);
    cudaFree(r->d_geom);
    cudaFree(r->d_segs);
    cudaFree(r->d_pos);
  }
  for (gx_vdifmux *m : r->mux)
    if (m) gx_vdifmux_close(m);
  delete r;
  return GX_OK;
}

}  // extern "C"
