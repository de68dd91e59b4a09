// Multi-thread VDIF to single-thread multi-channel VDIF on the device (the
// reference's vdifmux, vdifio/src/vdifmux.c:496-1033, as the VDIF DataStream
// calls it, vdiffile.cpp:495-565, 700-760).
//
// The raw bytes never leave the GPU:
//   1. vmux_classify_kernel: one thread per input frame slot (the input is
//      frame-aligned: frame k starts at byte k x input frame size) writes a
//      16-byte record: what the slot is (fill, foreign frame, invalid, wrong
//      thread, usable), its output channel and its frame number.
//   2. The host copies the records back (16 bytes per frame) and replays the
//      reference's sequential decisions over them -- first-seen wins for
//      duplicates, the out-of-order window (nSort), the gap limit (nGap), the
//      end-of-buffer back-off, the prototype header -- producing the source
//      slot of every (output frame, thread) and the statistics.
//   3. vmux_turn_kernel<P, B>: one thread per (output frame, input payload
//      word) writes the output headers and corner-turns the threads' samples:
//      output time sample s holds, at slot k of P = nThread rounded up to a
//      power of two, the B = bits x (1|2) bits of thread k's sample s (zeros
//      in the slots past nThread); the transpose runs in registers with
//      constant shifts, reads and writes are coalesced.  vmux_output_kernel
//      (one thread per output word) covers the other (P, B).
// A slot the reference would scan byte by byte (a frame that starts with the
// fill pattern but does not end with it, or a header of another frame size,
// channel count or bit depth) is skipped whole here; on frame-aligned input
// without such corrupt frames the output and the statistics are the same.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/gxcorr.h"

namespace {

constexpr uint32_t kFill = 0x11223344u;   // MARK5 fill word as little-endian memory holds it
constexpr int kHeader = 32;
constexpr int kMaxThreadId = 1023;

enum SlotCode : int32_t { kGood = 0, kFillEnd = 1, kFillStart = 2, kForeign = 3, kInvalid = 4, kWrongThread = 5 };

struct SlotRecord {
  int32_t code;
  int32_t chan;
  int64_t frame;   // seconds x frames per second + frame number
};

__global__ void vmux_classify_kernel(const uint8_t *__restrict__ src, long long nslots, int ifb, int fps, int nbits,
                                     int cpt, int enable_validity, const uint16_t *__restrict__ chan_of_thread,
                                     SlotRecord *__restrict__ rec)
{
  const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (k >= nslots) return;
  const uint8_t *f = src + k * (long long)ifb;
  const uint32_t *w = reinterpret_cast<const uint32_t *>(f);
  SlotRecord r{kGood, -1, 0};
  const uint32_t last = *reinterpret_cast<const uint32_t *>(f + ifb - 4);
  const uint32_t w0 = w[0], w1 = w[1], w2 = w[2], w3 = w[3];
  if (last == kFill) {
    r.code = kFillEnd;
  } else if (w0 == kFill) {
    r.code = kFillStart;
  } else if ((int)(w2 & 0xFFFFFFu) * 8 != ifb || (1 << ((w2 >> 24) & 31u)) != cpt ||
             (int)((w3 >> 26) & 31u) + 1 != nbits) {
    r.code = kForeign;
  } else if (enable_validity && (w0 >> 31)) {
    r.code = kInvalid;
  } else {
    const int tid = (int)((w3 >> 16) & 1023u);
    const int chan = chan_of_thread[tid];
    r.frame = (long long)(w0 & 0x3FFFFFFFu) * fps + (long long)(w1 & 0xFFFFFFu);
    if (chan == 0xFFFF) r.code = kWrongThread;
    else r.chan = chan;
  }
  rec[k] = r;
}

// Output frame f: header words from the prototype with the frame's time and
// validity, payload words corner-turned from the source slots of its threads
// (slot < 0: the thread is absent).
__global__ void vmux_output_kernel(const uint8_t *__restrict__ src, uint8_t *__restrict__ dest, int nout, int ofb,
                                   int ifb, int nthreads, int P, int B, const int32_t *__restrict__ slot,
                                   const uint32_t *__restrict__ hdr, int copy_missing_from_src)
{
  const int words = ofb / 4;
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= (long long)nout * words) return;
  const int f = (int)(g / words), w = (int)(g % words);
  uint32_t *out = reinterpret_cast<uint32_t *>(dest + (long long)f * ofb);
  if (w < kHeader / 4) {
    out[w] = hdr[(long long)f * 8 + w];
    return;
  }
  if (hdr[(long long)f * 8] >> 31) return;   // filler frame: payload left as it is
  const int32_t *sl = slot + (long long)f * nthreads;
  const int gpw = 32 / B;                        // B-bit groups per output word
  const long long g0 = (long long)(w - kHeader / 4) * gpw;
  int lgP = 0;
  while ((1 << lgP) < P) lgP++;
  uint32_t v = 0;
  for (int i = 0; i < gpw; i++) {
    const long long gi = g0 + i;
    const long long s = gi >> lgP;               // time sample
    const int k = (int)(gi & (P - 1));           // thread slot within the sample
    if (k >= nthreads) continue;                 // padding slot: zeros
    const int32_t sk = sl[k];
    if (sk < 0 && !copy_missing_from_src) continue;
    const uint8_t *payload = sk >= 0 ? src + (long long)sk * ifb + kHeader : src;   // absent: the reference reads the buffer start
    const long long bit = s * B;
    const uint32_t word = reinterpret_cast<const uint32_t *>(payload)[bit >> 5];
    const uint32_t bits = B == 32 ? word : (word >> (bit & 31)) & ((1u << B) - 1u);
    v |= bits << (i * B);
  }
  out[w] = v;
}

// The same corner turn for compile-time P (threads rounded up to a power of
// two) and B (bits of a thread's time sample): one thread per (output frame,
// input word q) loads word q of each of the P threads' payloads (coalesced
// across the warp) and writes the P output words those 32 / B samples make;
// every shift is a constant after unrolling, so the transpose stays in
// registers.  Header words are written by the threads of q < 8.
template <int P, int B>
__global__ void __launch_bounds__(256) vmux_turn_kernel(const uint8_t *__restrict__ src, uint8_t *__restrict__ dest,
                                                        int nout, int ofb, int ifb, int nthreads,
                                                        const int32_t *__restrict__ slot,
                                                        const uint32_t *__restrict__ hdr, int copy_missing_from_src)
{
  constexpr int G = 32 / B;                       // samples per input word
  constexpr uint32_t M = B == 32 ? 0xFFFFFFFFu : ((1u << B) - 1u);
  const int qwords = (ifb - kHeader) / 4;        // input payload words
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= (long long)nout * qwords) return;
  const int f = (int)(t / qwords), q = (int)(t % qwords);
  uint32_t *out = reinterpret_cast<uint32_t *>(dest + (long long)f * ofb);
  const uint32_t h0 = hdr[(long long)f * 8];
  if (q < kHeader / 4) out[q] = hdr[(long long)f * 8 + q];
  if (h0 >> 31) return;                          // filler frame: payload left as it is
  const int32_t *sl = slot + (long long)f * nthreads;
  uint32_t in[P];
#pragma unroll
  for (int k = 0; k < P; k++) {
    in[k] = 0u;
    if (k < nthreads) {
      const int32_t sk = sl[k];
      if (sk >= 0)
        in[k] = reinterpret_cast<const uint32_t *>(src + (long long)sk * ifb + kHeader)[q];
      else if (copy_missing_from_src)
        in[k] = reinterpret_cast<const uint32_t *>(src)[q];   // absent thread: the reference reads the buffer start
    }
  }
  uint32_t *o = out + kHeader / 4 + (long long)q * P;
  // output group n = s * P + k (sample s of this word, thread k) sits at bits n * B
#pragma unroll
  for (int j = 0; j < P; j++) {                 // output word j of this input word
    uint32_t v = 0u;
#pragma unroll
    for (int i = 0; i < G; i++) {
      const int n = j * G + i;
      const int s = n / P, k = n % P;
      v |= ((in[k] >> (s * B)) & M) << (i * B);
    }
    o[j] = v;
  }
}

}  // namespace

struct gx_vdifmux {
  int device = 0;
  int ifb = 0, fps = 0, nbits = 0, nthreads = 0, cpt = 1, nsort = 0, ngap = 0, flags = 0, cf = 1;
  int ids[64] = {};
  int P = 1, B = 1, nout_chan = 1, ofb = 0, ids_bytes = 0, granularity = 1;
  uint16_t *d_chan = nullptr;
  SlotRecord *d_rec = nullptr;
  long long rec_cap = 0;
  int32_t *d_slot = nullptr;
  uint32_t *d_hdr = nullptr;
  long long out_cap = 0;
  std::string err;
  gx_vdifmux_stats acc{};   // the accumulating counters

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

namespace {

long long gcdll(long long a, long long b)
{
  while (b) {
    const long long t = a % b;
    a = b;
    b = t;
  }
  return a;
}

// The reference's getLowestFrameNumber / getHighestFrameNumber over the slot
// records: the extreme frame number among the first nSort usable frames.
long long extreme_frame(const std::vector<SlotRecord> &rec, int nsort, bool highest)
{
  long long best = -1;
  int n = 0;
  for (const SlotRecord &r : rec) {
    if (r.code == kFillEnd || r.code == kFillStart || r.code == kForeign || r.code == kInvalid) continue;
    // frames of other threads count here: this scan does not look at threads
    const long long fn = r.frame;
    if (best < 0 || (highest ? fn > best : fn < best)) best = fn;
    if (++n >= nsort) break;
  }
  return best;
}

}  // namespace

extern "C" {

gx_status gx_vdifmux_open(int input_frame_bytes, int frames_per_second, int bits_per_sample, int nthreads,
                          const int *thread_ids, int channels_per_thread, int nsort, int ngap, int flags, int device,
                          gx_vdifmux **out)
{
  if (!out || !thread_ids || input_frame_bytes <= kHeader || input_frame_bytes % 8 || frames_per_second <= 0 ||
      nthreads < 1 || nthreads > 64 || channels_per_thread < 1 || nsort < 1 || bits_per_sample < 1 ||
      bits_per_sample > 32)
    return GX_ERR_ARG;
  if (flags & ~(GX_VDIFMUX_GOTOEND | GX_VDIFMUX_RESPECTGRANULARITY | GX_VDIFMUX_ENABLEVALIDITY | GX_VDIFMUX_COMPLEX |
                GX_VDIFMUX_PROPAGATEVALIDITY))
    return GX_ERR_UNSUPPORTED;   // legacy headers are not implemented by the reference either
  std::unique_ptr<gx_vdifmux> m(new gx_vdifmux());
  m->device = device;
  m->ifb = input_frame_bytes;
  m->fps = frames_per_second;
  m->nbits = bits_per_sample;
  m->nthreads = nthreads;
  m->cpt = channels_per_thread;
  m->nsort = nsort;
  m->ngap = std::max(ngap, nsort);
  m->flags = flags;
  m->cf = (flags & GX_VDIFMUX_COMPLEX) ? 2 : 1;
  std::vector<uint16_t> chan(kMaxThreadId + 1, 0xFFFF);
  for (int i = 0; i < nthreads; i++) {
    if (thread_ids[i] < 0 || thread_ids[i] > kMaxThreadId) return GX_ERR_ARG;
    chan[thread_ids[i]] = (uint16_t)i;
    m->ids[i] = thread_ids[i];
  }
  while (m->P < nthreads) m->P *= 2;
  // Several channels per thread (setvdifmuxinputchannels, vdifmux.c:202-242):
  // a thread's time sample holds all its channels, the header counts P x
  // channels, and the output payload stays P input payloads (outputDataSize
  // is fixed at configuration, vdifmux.c:167-171).  One thread: a plain copy.
  m->B = m->P == 1 ? 32 : bits_per_sample * m->cf * channels_per_thread;
  if (32 % m->B) return GX_ERR_UNSUPPORTED;   // a thread's time sample must pack into 32-bit words
  m->nout_chan = m->P * channels_per_thread;
  m->ids_bytes = input_frame_bytes - kHeader;
  if (m->ids_bytes % 4) return GX_ERR_ARG;
  m->ofb = m->ids_bytes * m->P + kHeader;
  m->granularity = (int)(frames_per_second / gcdll(frames_per_second, 1000000000LL));
  if (device >= 0) {
    if (cudaSetDevice(device) != cudaSuccess) return GX_ERR_CUDA;
    if (cudaMalloc(&m->d_chan, sizeof(uint16_t) * chan.size()) != cudaSuccess) return GX_ERR_NOMEM;
    if (cudaMemcpy(m->d_chan, chan.data(), sizeof(uint16_t) * chan.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return GX_ERR_CUDA;
  }
  *out = m.release();
  return GX_OK;
}

gx_status gx_vdifmux_info(const gx_vdifmux *m, int *output_frame_bytes, int *output_channels, int *frame_granularity)
{
  if (!m) return GX_ERR_ARG;
  if (output_frame_bytes) *output_frame_bytes = m->ofb;
  if (output_channels) *output_channels = m->nout_chan;
  if (frame_granularity) *frame_granularity = m->granularity;
  return GX_OK;
}

gx_status gx_vdifmux_run(gx_vdifmux *m, const uint8_t *src, long long src_bytes, uint8_t *dest, long long dest_bytes,
                         long long start_frame, gx_vdifmux_stats *stats, void *stream)
{
  if (!m || !src || !dest || src_bytes < 0 || dest_bytes < 0) return GX_ERR_ARG;
  if (m->device < 0) return m->fail(GX_ERR_STATE, "host-only multiplexer (opened with device -1)");
  if (((uintptr_t)src | (uintptr_t)dest) & 3) return m->fail(GX_ERR_ARG, "buffers must be 4-byte aligned");
  gx_status r;
  if ((r = m->cuda(cudaSetDevice(m->device), "cudaSetDevice")) != GX_OK) return r;
  cudaStream_t st = (cudaStream_t)stream;
  const int ifb = m->ifb;
  // ---- 1. classify every whole frame slot on the device
  const long long nslots = src_bytes >= ifb ? src_bytes / ifb : 0;
  std::vector<SlotRecord> rec(nslots);
  if (nslots > 0) {
    if (nslots > m->rec_cap) {
      cudaFree(m->d_rec);
      m->d_rec = nullptr;
      if ((r = m->cuda(cudaMalloc(&m->d_rec, sizeof(SlotRecord) * nslots), "cudaMalloc")) != GX_OK) return r;
      m->rec_cap = nslots;
    }
    const int tpb = 256;
    vmux_classify_kernel<<<(unsigned)((nslots + tpb - 1) / tpb), tpb, 0, st>>>(
        src, nslots, ifb, m->fps, m->nbits, m->cpt, (m->flags & GX_VDIFMUX_ENABLEVALIDITY) ? 1 : 0, m->d_chan, m->d_rec);
    if ((r = m->cuda(cudaGetLastError(), "vmux_classify_kernel")) != GX_OK) return r;
    if ((r = m->cuda(cudaMemcpyAsync(rec.data(), m->d_rec, sizeof(SlotRecord) * nslots, cudaMemcpyDeviceToHost, st),
                     "cudaMemcpyAsync")) != GX_OK)
      return r;
    if ((r = m->cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize")) != GX_OK) return r;
  }

  // ---- 2. the reference's sequential decisions over the records
  const int nthr = m->nthreads;
  const long long goodmask = nthr == 64 ? ~0ull : ((1ull << nthr) - 1);
  const bool propagate = (m->flags & GX_VDIFMUX_PROPAGATEVALIDITY) != 0;
  int nsort = m->nsort;
  long long N = src_bytes - ifb;
  if (3 * src_bytes <= 4LL * nsort * ifb) nsort = (int)((3 * src_bytes) / (4LL * ifb));
  const long long maxSrcIndex = (m->flags & GX_VDIFMUX_GOTOEND) ? src_bytes - ifb : src_bytes - (long long)nsort * ifb;
  if ((m->flags & GX_VDIFMUX_RESPECTGRANULARITY) && start_frame > 0) {
    const long long q = start_frame % m->granularity;
    if (q) start_frame += m->granularity - q;
  }
  const long long maxDest = dest_bytes / m->ofb - 1;
  long long startFrame = start_frame;
  if (startFrame < 0) {
    startFrame = extreme_frame(rec, m->nsort, false);
    if (startFrame < 0) return m->fail(GX_ERR_IO, "no usable VDIF frame found");
  }
  const long long ntab = maxDest + 1 > 0 ? maxDest + 1 : 0;
  std::vector<uint64_t> mask(ntab, 0);
  std::vector<int32_t> slot((size_t)ntab * nthr, -1);
  long long nValid = 0, nSkip = 0, nFill = 0, nDup = 0, nInvalid = 0, nDiscard = 0, nSeqUnproc = 0, nWrong = 0;
  long long highest = 0, bytesProcessed = -1, firstGoodByte = -1, nEnd = 0, highestSorted = -1;
  long long framesIn = 0;
  int protoSlot = -1;
  long long i = 0;
  for (; i <= N;) {
    const long long k = i / ifb;
    const SlotRecord &rc = rec[k];
    if (rc.code == kFillEnd || rc.code == kFillStart) { i += ifb; nFill += ifb; continue; }
    if (rc.code == kForeign) { i += ifb; nSkip += ifb; continue; }
    if (rc.code == kInvalid) { i += ifb; nInvalid++; continue; }
    if (firstGoodByte < 0) firstGoodByte = i;
    if (rc.code == kWrongThread) { i += ifb; nWrong++; continue; }
    if (protoSlot < 0) protoSlot = (int)k;
    framesIn++;
    const long long di = rc.frame - startFrame;
    if (di < 0) { i += ifb; nDiscard++; continue; }
    if (i > maxSrcIndex && highestSorted < 0) highestSorted = highest;
    if (di > maxDest) {
      nSeqUnproc++;
      if (framesIn < nsort) { i += ifb; nDiscard++; continue; }
      if (bytesProcessed == -1) bytesProcessed = i;
      i += ifb;
      if (++nEnd >= nsort) break;
      continue;
    }
    nSeqUnproc--;
    if (di > highest + m->ngap && m->ngap > 0 && nValid > nsort) {
      if (bytesProcessed == -1) bytesProcessed = i;
      if (++nEnd >= nsort) break;
    }
    const uint64_t bit = 1ull << rc.chan;
    if (mask[di] & bit) {
      nDup++;
    } else {
      mask[di] |= bit;
      slot[(size_t)di * nthr + rc.chan] = (int32_t)k;
      nValid++;
      if (di > highest) highest = di;
    }
    i += ifb;
  }
  if (bytesProcessed == -1) bytesProcessed = i;
  if (highestSorted >= 0) {
    for (long long f = highest; f > highestSorted; --f) {
      if (propagate) {
        if (mask[f] == 0) highest = f - 1;
      } else if (mask[f] != goodmask) {
        highest = f - 1;
        for (int t = 0; t < nthr; t++)
          if (mask[f] & (1ull << t)) {
            const long long d = (long long)slot[(size_t)f * nthr + t] * ifb;
            if (d < bytesProcessed) bytesProcessed = d;
            nValid--;
          }
      }
    }
  } else {
    const long long minDest = highest - nsort / nthr;
    if (minDest >= 0)
      for (long long f = highest; f >= minDest; --f) {
        if (propagate) {
          if (mask[f] == 0) highest = f - 1;
        } else if (mask[f] != goodmask) {
          highest = f - 1;
          for (int t = 0; t < nthr; t++)
            if (mask[f] & (1ull << t)) {
              const long long d = (long long)slot[(size_t)f * nthr + t] * ifb;
              if (d < bytesProcessed) bytesProcessed = d;
              nValid--;
            }
        }
      }
  }
  if (i < N && highest < maxDest && (highest > maxDest - m->ngap || m->ngap == 0)) highest = maxDest;
  if (ntab == 0) highest = -1;

  // output headers: the prototype (first usable frame) with this mux's
  // channel count, thread 0, frame size and each frame's time and validity
  uint32_t proto[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (protoSlot >= 0 &&
      (r = m->cuda(cudaMemcpy(proto, src + (long long)protoSlot * ifb, 16, cudaMemcpyDeviceToHost), "cudaMemcpy")) !=
          GX_OK)
    return r;
  if (propagate) {   // EDV4 words: mask length (bits 16-23), extension version 4, sync word, validity mask
    proto[4] = (((uint32_t)nthr & 0xFFu) << 16) | (4u << 24);
    proto[5] = 0xACABFEEDu;
    proto[6] = proto[7] = 0;
  }
  int lg = 0;
  while ((1 << lg) < m->nout_chan) lg++;
  proto[0] &= ~(1u << 31);                                        // valid
  proto[2] = ((uint32_t)(m->ofb / 8) & 0xFFFFFFu) | ((uint32_t)lg << 24) | (proto[2] & 0xE0000000u);
  proto[3] &= ~(1023u << 16);                                     // thread 0
  const int epoch = protoSlot >= 0 ? (int)((proto[1] >> 24) & 63u) : -1;
  const long long nout = highest + 1;
  std::vector<uint32_t> hdr((size_t)std::max(0LL, nout) * 8);
  long long nGood = 0, nPartial = 0, nBad = 0;
  long long secs = startFrame / m->fps, fnum = startFrame % m->fps;
  for (long long f = 0; f < nout; f++) {
    uint32_t *h = &hdr[(size_t)f * 8];
    memcpy(h, proto, sizeof(proto));
    h[0] = (h[0] & ~0x3FFFFFFFu) | ((uint32_t)secs & 0x3FFFFFFFu);
    h[1] = (h[1] & ~0xFFFFFFu) | ((uint32_t)fnum & 0xFFFFFFu);
    const uint64_t mk = mask[f];
    if (propagate) {
      if (mk != 0) {
        h[6] = (uint32_t)(mk & 0xFFFFFFFFu);
        h[7] = (uint32_t)(mk >> 32);
        if (mk == (uint64_t)goodmask) nGood++;
        else nPartial++;
      } else {
        h[0] |= 1u << 31;
        nBad++;
      }
    } else if (mk == (uint64_t)goodmask) {
      nGood++;
    } else {
      h[0] |= 1u << 31;
      nBad++;
      for (int t = 0; t < nthr; t++) slot[(size_t)f * nthr + t] = -1;
    }
    if (++fnum >= m->fps) {
      secs++;
      fnum -= m->fps;
    }
  }

  // ---- 3. headers and corner turn on the device
  if (nout > 0) {
    if (nout > m->out_cap) {
      cudaFree(m->d_slot);
      cudaFree(m->d_hdr);
      m->d_slot = nullptr;
      m->d_hdr = nullptr;
      if ((r = m->cuda(cudaMalloc(&m->d_slot, sizeof(int32_t) * nout * nthr), "cudaMalloc")) != GX_OK) return r;
      if ((r = m->cuda(cudaMalloc(&m->d_hdr, sizeof(uint32_t) * 8 * nout), "cudaMalloc")) != GX_OK) return r;
      m->out_cap = nout;
    }
    if ((r = m->cuda(cudaMemcpyAsync(m->d_slot, slot.data(), sizeof(int32_t) * nout * nthr, cudaMemcpyHostToDevice, st),
                     "cudaMemcpyAsync")) != GX_OK)
      return r;
    if ((r = m->cuda(cudaMemcpyAsync(m->d_hdr, hdr.data(), sizeof(uint32_t) * 8 * nout, cudaMemcpyHostToDevice, st),
                     "cudaMemcpyAsync")) != GX_OK)
      return r;
    const int tpb = 256;
    const long long turns = nout * (long long)((ifb - kHeader) / 4);
    const unsigned tgrid = (unsigned)((turns + tpb - 1) / tpb);
    bool done = false;
#define GX_TURN(PP, BB)                                                                                     \
    if (!done && m->P == PP && m->B == BB) {                                                                \
      vmux_turn_kernel<PP, BB><<<tgrid, tpb, 0, st>>>(src, dest, (int)nout, m->ofb, ifb, nthr, m->d_slot,   \
                                                     m->d_hdr, propagate ? 1 : 0);                          \
      done = true;                                                                                          \
    }
    // every payload has at least 8 words, so the threads q < 8 cover the header
    if ((ifb - kHeader) / 4 >= kHeader / 4) {
      GX_TURN(1, 1) GX_TURN(2, 1) GX_TURN(4, 1) GX_TURN(8, 1) GX_TURN(16, 1)
      GX_TURN(1, 2) GX_TURN(2, 2) GX_TURN(4, 2) GX_TURN(8, 2) GX_TURN(16, 2) GX_TURN(32, 2)
      GX_TURN(1, 4) GX_TURN(2, 4) GX_TURN(4, 4) GX_TURN(8, 4) GX_TURN(16, 4) GX_TURN(32, 4)
      GX_TURN(1, 8) GX_TURN(2, 8) GX_TURN(4, 8) GX_TURN(8, 8) GX_TURN(16, 8) GX_TURN(32, 8)
      GX_TURN(1, 16) GX_TURN(2, 16) GX_TURN(4, 16) GX_TURN(8, 16) GX_TURN(16, 16)
      GX_TURN(1, 32)
    }
#undef GX_TURN
    if (!done) {   // other thread counts and sample widths: one thread per output word
      const long long words = nout * (long long)(m->ofb / 4);
      vmux_output_kernel<<<(unsigned)((words + tpb - 1) / tpb), tpb, 0, st>>>(src, dest, (int)nout, m->ofb, ifb, nthr,
                                                                             m->P, m->B, m->d_slot, m->d_hdr,
                                                                             propagate ? 1 : 0);
    }
    if ((r = m->cuda(cudaGetLastError(), "vmux corner turn")) != GX_OK) return r;
    if ((r = m->cuda(cudaStreamSynchronize(st), "cudaStreamSynchronize")) != GX_OK) return r;
  }

  gx_vdifmux_stats &a = m->acc;
  a.valid_frames += nValid;
  a.invalid_frames += nInvalid;
  a.discarded_frames += nDiscard;
  a.wrong_thread_frames += nWrong;
  a.skipped_bytes += nSkip;
  a.fill_bytes += nFill;
  a.duplicate_frames += nDup;
  a.bytes_processed += bytesProcessed;
  a.good_output_frames += nGood;
  a.partial_output_frames += nPartial;
  a.filler_output_frames += nBad;
  a.calls++;
  a.src_bytes = src_bytes;
  a.src_used = bytesProcessed;
  a.dest_bytes = dest_bytes;
  a.dest_used = (nGood + nBad + nPartial) * m->ofb;
  a.output_frames = nGood + nBad + nPartial;
  a.epoch = epoch;
  a.start_frame = startFrame;
  long long ret = bytesProcessed > firstGoodByte ? bytesProcessed : firstGoodByte;
  if (a.output_frames == 0 || bytesProcessed == 0 || firstGoodByte < 0 || nSeqUnproc >= nsort) {
    const long long hi = extreme_frame(rec, m->nsort, true);
    if (hi < 0) a.start_frame += (src_bytes / ifb) / nthr + 1;
    else a.start_frame = hi + 1;
    a.output_frames = 0;
    a.src_used = src_bytes - src_bytes % ifb;
    ret = a.src_used > firstGoodByte ? a.src_used : firstGoodByte;
  }
  a.returned_bytes = ret;
  if (stats) *stats = a;
  return GX_OK;
}

gx_status gx_vdifmux_reset_stats(gx_vdifmux *m)
{
  if (!m) return GX_ERR_ARG;
  memset(&m->acc, 0, sizeof(m->acc));
  return GX_OK;
}

const char *gx_vdifmux_last_error(const gx_vdifmux *m) { return m ? m->err.c_str() : "null multiplexer"; }

gx_status gx_vdifmux_close(gx_vdifmux *m)
{
  if (!m) return GX_ERR_ARG;
  if (m->device >= 0) {
    cudaSetDevice(m->device);
    cudaFree(m->d_chan);
    cudaFree(m->d_rec);
    cudaFree(m->d_slot);
    cudaFree(m->d_hdr);
  }
  delete m;
  return GX_OK;
}

}  // extern "C"
