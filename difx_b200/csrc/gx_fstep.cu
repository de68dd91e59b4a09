// F-step: VDIF unpack + validity/weights, FP64 per-block delay evaluation,
// FP32 fringe rotation, shared-memory Stockham FFT, sideband selection and
// fractional-sample correction, writing spectra in the layout both X-steps
// read: spec[freq][block][input][channel] (float2).
//
// Two kernels per pass of blocks:
//   blockparams_kernel  one thread per (station, block): FP64 delay, nearest
//                       sample, fractional-sample error, linear interpolation
//                       coefficients, frame-validity mask and data weight.
//   fstep_r16_kernel    (FFT length 512-8192) a group of F / 16 threads per
//                       (block, band), 16 samples per thread in registers,
//                       radix-16 passes with padded shared-memory exchanges.
//   fstep_warp_kernel   (FFT length 128-256) one warp per (block, band): the
//                       warp builds its rotator tables, decodes and rotates
//                       its samples into warp-private shared memory, runs the
//                       FFT with warp-level synchronisation only and writes
//                       the corrected spectrum row.
//   fstep_cta_kernel    (longer FFTs not covered above) the bands of a block
//                       are transformed concurrently in slots of one CTA.
//
// Reference semantics followed (mpifxcorr/src):
//   block validity / delay / nearest sample      mode.cpp:656-701
//   unpack weight = good samples / unpacksamples  mk5mode.cpp:94-174
//   VDIF validity + fill-pattern blanking         mark5access format_vdif.c:7619-7667,
//                                                 blanker_mark5.c:272-306
//   linear delay interpolation, integer delay     mode.cpp:782-799
//   fringe rotator (two-level arraystride)        mode.cpp:882-955
//   fractional-sample rotator (two-level)         mode.cpp:1029-1073
//   real->complex, rotate, FFT, sideband copy     mode.cpp:1160-1217
//   fractional-sample correction                  mode.cpp:1256-1261
#include <cstdint>
#include <cstdlib>
#include <map>
#include <mutex>
#include <utility>
#include "gx_dev.h"
#include "gx_fcommon.cuh"
#include "gx_fft16.h"

namespace gx {


__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// forward DFT of 4 points in place (natural order)
__device__ __forceinline__ void dft4(float2 &b0, float2 &b1, float2 &b2, float2 &b3)
{
  float2 s02 = cadd(b0, b2), d02 = csub(b0, b2), s13 = cadd(b1, b3), d13 = csub(b1, b3);
  b0 = cadd(s02, s13);
  b2 = csub(s02, s13);
  b1 = make_float2(d02.x + d13.y, d02.y - d13.x);   // d02 - i d13
  b3 = make_float2(d02.x - d13.y, d02.y + d13.x);   // d02 + i d13
}

// forward DFT of 8 points in place (natural order)
__device__ __forceinline__ void dft8(float2 *v)
{
  const float r = 0.70710678118654752440f;
  dft4(v[0], v[2], v[4], v[6]);   // E0..E3 at 0,2,4,6
  dft4(v[1], v[3], v[5], v[7]);   // O0..O3 at 1,3,5,7
  float2 o1 = make_float2((v[3].x + v[3].y) * r, (v[3].y - v[3].x) * r);    // * W8^1
  float2 o2 = make_float2(v[5].y, -v[5].x);                               // * W8^2 = -i
  float2 o3 = make_float2((v[7].y - v[7].x) * r, -(v[7].x + v[7].y) * r); // * W8^3
  float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1];
  v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

// One Stockham radix-R pass: in -> out, butterflies j = lt, lt+nt, ...
template <int R>
__device__ __forceinline__ void stockham_pass(const float2 *in, float2 *out, int F, int Ns,
                                              const float2 *__restrict__ tw, int lt, int nt)
{
  const int nb = F / R;
  const int twstep = F / (Ns * R);
  for (int j = lt; j < nb; j += nt) {
    float2 v[R];
    const int k = j % Ns;
#pragma unroll
    for (int r = 0; r < R; r++) {
      float2 x = in[j + r * nb];
      if (r > 0 && k > 0) x = cmul(x, __ldg(&tw[r * k * twstep]));
      v[r] = x;
    }
    if (R == 8) dft8(v);
    else if (R == 4) dft4(v[0], v[1], v[2], v[3]);
    else {
      float2 t = v[0];
      v[0] = cadd(t, v[1]);
      v[1] = csub(t, v[1]);
    }
    const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) out[idxD + r * Ns] = v[r];
  }
}

__device__ __forceinline__ int frame_ok(const uint8_t *frame, int framebytes, int check_header)
{
  const uint32_t *h = reinterpret_cast<const uint32_t *>(frame);
  if (check_header) {
    if (h[2] == 0u) return 0;
    if ((h[0] >> 31) & 1u) return 0;
  }
  const uint32_t *p0 = reinterpret_cast<const uint32_t *>(frame + 32);
  const uint32_t *p1 = reinterpret_cast<const uint32_t *>(frame + framebytes - 8);
  // MARK5_FILL_WORD64 on a little-endian host = 0x1122334411223344 (blanker_mark5.c:35):
  // two 32-bit words of 0x11223344
  if (p0[0] == 0x11223344u && p0[1] == 0x11223344u) return 0;
  if (p1[0] == 0x11223344u && p1[1] == 0x11223344u) return 0;
  return 1;
}

// --------------------------------------------------------------------------
// Per-block parameters (FP64): mode.cpp:656-757 and 782-799, mk5mode.cpp:94-174.
__global__ void blockparams_kernel(DevJob J, SubintArrays S, int blk0, int nblk, BlockParam *__restrict__ bp,
                                   float *__restrict__ weights)
{
  const int bi = blockIdx.x * blockDim.x + threadIdx.x;
  const int s = blockIdx.y;
  if (bi >= nblk) return;
  const int blk = blk0 + bi;
  const int F = J.fftlen;
  BlockParam P;
  P.state = 0;
  P.weight = 0.0f;
  P.a = P.b = P.qa = P.qb = P.fracwalltime = 0.0;
  P.validmask = 0ull;
  P.nearestsample = P.fr0 = P.integerdelay = P.intwalltime = P.nframes = 0;
  P.fracsampleerror = 0.0f;
  const uint8_t *data = S.data[s];
  const int64_t datalen = S.datalen[s];
  const int32_t *ctrl = S.control + (size_t)s * S.controlstride;
  const double *ip = S.interp + 3 * s;
  const int datasec = ctrl[1], datans = ctrl[2];
  const int flagword = ctrl[3 + blk / 30];
  if (datalen > 1 && ((flagword >> (blk % 30)) & 1) != 0) {
    const double fftcentre = blk + 0.5;
    const double averagedelay = ip[0] * fftcentre * fftcentre + ip[1] * fftcentre + ip[2];
    const double fftstartmicrosec = (blk * F) * J.sampletime;
    const SubintClock clk = *S.clock;
    const double starttime = (clk.sec - datasec) * 1000000.0 +
                             ((long long)clk.ns - (long long)datans) / 1000.0 + fftstartmicrosec - averagedelay;
    int ns = (int)(starttime / J.sampletime + 0.5);
    const double walltimesecs = (double)((long long)clk.scan_start_sec + clk.sec) + clk.ns / 1.0e9 +
                                fftstartmicrosec / 1.0e6;
    P.intwalltime = (int)walltimesecs;
    P.fracwalltime = walltimesecs - P.intwalltime;
    if (!(ns < -1 || ((long long)(ns + F) * J.bps_num) / J.bps_den > datalen)) {
      if (ns == -1) ns = 0;
      P.nearestsample = ns;
      P.fr0 = ns / J.framesamples;
      P.nframes = (ns + J.unpacksamples - 1) / J.framesamples - P.fr0 + 1;
      if (P.nframes <= kMaxFramesPerBlock) {
        int good = 0;
        for (int q = 0; q < P.nframes; q++) {
          const long long fr = (long long)P.fr0 + q;
          int ok = 0;
          if ((fr + 1) * J.framebytes <= datalen)
            ok = frame_ok(data + fr * J.framebytes, J.framebytes, !(J.cplx && q == 0));
          if (ok) {
            P.validmask |= (1ull << q);
            const long long lo = max((long long)ns, fr * J.framesamples);
            const long long hi = min((long long)ns + J.unpacksamples, (fr + 1) * J.framesamples);
            good += (int)(hi - lo);
          }
        }
        P.weight = (float)good / (float)J.unpacksamples;
        if (P.weight > 0.0f) {
          P.state = 1;
          P.fracsampleerror = (float)(starttime - ns * J.sampletime);
        }
        if (P.weight > 0.0f && J.fringe_order == 0) {
          // post-F: the integer part of the block-centre delay (mode.cpp:778-780)
          P.integerdelay = (int)averagedelay;
          P.b = averagedelay - P.integerdelay;
        } else if (P.weight > 0.0f && J.fringe_order == 2) {
          // quadratic (mode.cpp:800-825): delay, slope and curvature at the block start
          const double qa = ip[0];
          const double qb = ip[1] + blk * ip[0] * 2.0;
          double c = ip[2] + blk * ip[1] + blk * blk * ip[0];
          const int idelay = int(c);
          c -= idelay;
          const double stepxoff1 = double(J.stride) / double(F);
          P.a = qb + qa * stepxoff1;
          P.b = c;
          P.qa = qa;
          P.qb = qb;
          P.integerdelay = idelay;
        } else if (P.weight > 0.0f) {
          const double d0 = ip[0] * blk * blk + ip[1] * blk + ip[2];
          const double d1 = ip[0] * (blk + 0.5) * (blk + 0.5) + ip[1] * (blk + 0.5) + ip[2];
          const double d2 = ip[0] * (blk + 1) * (blk + 1) + ip[1] * (blk + 1) + ip[2];
          const double a = d2 - d0;
          double b = d0 + (d1 - (a * 0.5 + d0)) / 3.0;
          const int idelay = (int)b;
          b -= idelay;
          P.a = a;
          P.b = b;
          P.integerdelay = idelay;
        } else {
          P.weight = 0.0f;
        }
      }
    }
  }
  bp[(size_t)s * nblk + bi] = P;
  weights[(size_t)s * nblk + bi] = P.state ? P.weight : 0.0f;
}

// EDV4 per-band validity of multiplexed VDIF (INTERLACEDVDIF; Mk5Mode::unpack,
// mk5mode.cpp:142-163, and blank_vdif_EDV4 / _complex, format_vdif.c:8486-8660).
// The frame geometry comes from the first frame's header in the buffer, as the
// reference reads it: samples per header frame sph = payload bits / (channels x
// bits), which for complex data is twice the frame's complex samples, so header
// frame k then covers data frames [k m, (k+1) m) with m = sph / framesamples.
// A header frame with its invalid bit clear and a validity mask other than all
// channels blanks the samples of every band whose thread bit (band / (channels /
// mask length)) is clear; a blanked sample counts as invalid when its decoded
// value is not zero.  Band weight = (good - invalid[b]) / unpacksamples; block
// weight = (good - sum invalid / nbands) / unpacksamples.  One warp per
// (station, block); bandmask gets, per band, the data frames it blanks.
__global__ void edv4_kernel(DevJob J, const DevStation *__restrict__ stations, SubintArrays S, int nblk,
                            BlockParam *__restrict__ bp, float *__restrict__ weights)
{
  __shared__ float s_lut[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) s_lut[i] = J.lut[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int bi = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int s = blockIdx.y;
  if (bi >= nblk) return;
  const DevStation &st = stations[s];
  const int nb = J.nbands;
  unsigned long long *bm = const_cast<unsigned long long *>(S.bandmask) + ((size_t)s * nblk + bi) * nb;
  if (!st.interlaced) {
    for (int b = lane; b < nb; b += 32) bm[b] = 0ull;
    return;
  }
  BlockParam P = bp[(size_t)s * nblk + bi];
  float *wb = weights + (size_t)st.wrow0 * nblk + bi;   // band b at wb[b * nblk]
  unsigned long long mymask = 0ull;   // lane b < nb: frames blanked for band b
  int inv = 0;                        // lane b: blanked samples with a non-zero value
  const uint8_t *data = S.data[s];
  const int64_t datalen = S.datalen[s];
  if (P.state != 0 && datalen >= 32) {
    const uint32_t *h0 = reinterpret_cast<const uint32_t *>(data);
    const int ever = (int)(h0[4] >> 24), mlen = (int)((h0[4] >> 16) & 0xffu);
    const int nchan = 1 << ((h0[2] >> 24) & 0x1fu);
    const long long flen = (long long)(h0[2] & 0xffffffu) * 8;
    const int hbits = (int)((h0[3] >> 26) & 0x1fu) + 1;
    const long long sph = flen > 32 ? (flen - 32) * 8 / ((long long)nchan * hbits) : 0;
    const int fs = J.framesamples;
    const int dch = mlen > 0 ? nchan / mlen : 0;
    if (ever == 4 && mlen >= 1 && mlen <= 64 && dch > 0 && nchan <= 62 && sph > 0 && sph % fs == 0) {
      const int m = (int)(sph / fs);
      const unsigned long long good_mask = (1ull << nchan) - 1ull;
      // header frames over the window [nearestsample, + fftlen)
      const long long k0 = (long long)P.nearestsample / sph;
      const long long k1 = ((long long)P.nearestsample + J.fftlen - 1) / sph;
      for (long long k = k0; k <= k1; k++) {
        if ((k + 1) * flen > datalen) break;
        const uint32_t *hk = reinterpret_cast<const uint32_t *>(data + k * flen);
        const unsigned long long vmask = (unsigned long long)hk[6] | ((unsigned long long)hk[7] << 32);
        if ((hk[0] >> 31) != 0u || vmask == good_mask) continue;
        if (lane < nb && !((vmask >> (lane / dch)) & 1ull)) {
          for (long long q = k * m; q < (k + 1) * m; q++) {
            const long long rel = q - P.fr0;
            if (rel >= 0 && rel < P.nframes) mymask |= 1ull << rel;
          }
        }
      }
      // count the non-zero samples the masks blank (decoder-valid frames only)
      for (int b = 0; b < nb; b++) {
        const unsigned long long bmask = __shfl_sync(0xffffffffu, mymask, b) & P.validmask;
        if (!bmask) continue;
        int cnt = 0;
        for (int n = lane; n < J.fftlen; n += 32) {
          const int smp = P.nearestsample + n;
          const int q = smp / fs - P.fr0;
          if (!((bmask >> q) & 1ull)) continue;
          const int sub = J.cplx ? 2 : 1;
          const uint8_t *payload = data + ((long long)P.fr0 + q) * J.framebytes + 32;
          const long long bit0 = (long long)(smp % fs) * (nb * J.nbits * sub) + (long long)b * sub * J.nbits;
          const int mask = (1 << J.nbits) - 1;
          const float re = s_lut[(payload[bit0 >> 3] >> (bit0 & 7)) & mask];
          float im = 0.f;
          if (J.cplx) {
            const long long bit1 = bit0 + J.nbits;
            im = s_lut[(payload[bit1 >> 3] >> (bit1 & 7)) & mask];
          }
          if (re != 0.f || im != 0.f) cnt++;
        }
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        if (lane == b) inv = cnt;
      }
    }
  }
  // good samples of the window (as blockparams_kernel counts them)
  int good = 0;
  if (P.state != 0) {
    for (int q = 0; q < P.nframes; q++) {
      if (!((P.validmask >> q) & 1ull)) continue;
      const long long fr = (long long)P.fr0 + q;
      const long long lo = max((long long)P.nearestsample, fr * J.framesamples);
      const long long hi = min((long long)P.nearestsample + J.unpacksamples, (fr + 1) * J.framesamples);
      good += (int)(hi - lo);
    }
  }
  int totalinv = inv;
  for (int o = 16; o > 0; o >>= 1) totalinv += __shfl_xor_sync(0xffffffffu, totalinv, o);
  if (lane < nb) {
    bm[lane] = mymask;
    wb[(size_t)lane * nblk] = P.state != 0 ? ((float)good - (float)inv) / (float)J.unpacksamples : 0.0f;
  }
  if (lane == 0 && P.state != 0 && totalinv > 0) {
    float g = (float)good - (float)totalinv / (float)nb;
    if (g < 0.f) g = 0.f;
    P.weight = g / (float)J.unpacksamples;
    if (!(P.weight > 0.0f)) {
      P.state = 0;
      P.weight = 0.0f;
    }
    bp[(size_t)s * nblk + bi] = P;
    weights[(size_t)s * nblk + bi] = P.weight;
  }
}

// Parameters of block bi as band bd of station s decodes it: frames an EDV4
// validity mask blanks for this band count as invalid.
__device__ __forceinline__ BlockParam band_param(const BlockParam *__restrict__ bp, const SubintArrays &S, int s,
                                                 int nblk, int bi, int nbands, int bd)
{
  BlockParam P = bp[(size_t)s * nblk + bi];
  if (S.bandmask) P.validmask &= ~S.bandmask[((size_t)s * nblk + bi) * nbands + bd];
  return P;
}


// Decoded sample n of band bd (real in .x, imaginary in .y for complex data).
__device__ __forceinline__ float2 decode_sample(const DevJob &J, const uint8_t *__restrict__ data,
                                                const BlockParam &P, int bd, int n, const float *lut)
{
  const int smp = P.nearestsample + n;
  const int q = smp / J.framesamples - P.fr0;
  float2 u = make_float2(0.f, 0.f);
  if ((P.validmask >> q) & 1ull) {
    const int sub = J.cplx ? 2 : 1;
    const int mask = (1 << J.nbits) - 1;
    const uint8_t *payload = data + ((long long)P.fr0 + q) * J.framebytes + 32;
    const long long bit0 = (long long)(smp % J.framesamples) * (J.nbands * J.nbits * sub) +
                           (long long)bd * sub * J.nbits;
    u.x = lut[(__ldg(payload + (bit0 >> 3)) >> (bit0 & 7)) & mask];
    if (J.cplx) {
      const long long bit1 = bit0 + J.nbits;
      u.y = lut[(__ldg(payload + (bit1 >> 3)) >> (bit1 & 7)) & mask];
    }
  }
  return u;
}

// Sideband selection (mode.cpp:1185-1217) of output channel c from FFT result res.
__device__ __forceinline__ float2 select_channel(const DevJob &J, const float2 *res, int lsb, int c)
{
  const int N = J.nchan, F = J.fftlen;
  if (!J.cplx) return res[lsb ? N + c : c];
  if (!lsb) return res[c];
  if (c == 0) return res[0];
  float2 v = res[F - c];
  v.y = -v.y;
  return v;
}

// --------------------------------------------------------------------------
// Warp-private FFT buffers are padded by one element every eight so that the
// strided Stockham stores spread over the shared-memory banks.
__device__ __forceinline__ int pidx(int i) { return i + (i >> 3); }

// One compile-time Stockham pass (FL points, stride NS, radix R), in place in
// one warp's buffer: every lane loads all of its butterflies' inputs, the warp
// synchronises, then every lane stores its outputs.  Indices are shifts/masks.
template <int FL, int NS, int R>
__device__ __forceinline__ void warp_pass(float2 *buf, const float2 *tw, int lane)
{
  constexpr int NB = FL / R;
  constexpr int PER = (NB + 31) / 32;
  constexpr int TWSTEP = FL / (NS * R);
  float2 v[PER][R];
#pragma unroll
  for (int p = 0; p < PER; p++) {
    const int j = lane + 32 * p;
    if (NB % 32 == 0 || j < NB) {
      const int k = j & (NS - 1);
#pragma unroll
      for (int r = 0; r < R; r++) {
        float2 x = buf[pidx(j + r * NB)];
        if (r > 0 && NS > 1) x = cmul(x, tw[r * k * TWSTEP]);
        v[p][r] = x;
      }
      if (R == 8) dft8(v[p]);
      else if (R == 4) dft4(v[p][0], v[p][1], v[p][2], v[p][3]);
      else {
        float2 t = v[p][0];
        v[p][0] = cadd(t, v[p][1]);
        v[p][1] = csub(t, v[p][1]);
      }
    }
  }
  __syncwarp();
#pragma unroll
  for (int p = 0; p < PER; p++) {
    const int j = lane + 32 * p;
    if (NB % 32 == 0 || j < NB) {
      const int k = j & (NS - 1);
      const int idxD = (j - k) * R + k;   // (j / NS) * NS * R + k
#pragma unroll
      for (int r = 0; r < R; r++) buf[pidx(idxD + r * NS)] = v[p][r];
    }
  }
  __syncwarp();
}

// All passes of an FL-point forward FFT in place: radix 8 while it fits, then 4 or 2.
template <int FL, int NS>
__device__ __forceinline__ void warp_fft(float2 *buf, const float2 *tw, int lane)
{
  if constexpr (NS < FL) {
    constexpr int R = (NS * 8 <= FL) ? 8 : ((NS * 4 <= FL) ? 4 : 2);
    warp_pass<FL, NS, R>(buf, tw, lane);
    warp_fft<FL, NS * R>(buf, tw, lane);
  }
}

// Warp-per-(block, band) F-step for FFT lengths up to 1024 (FL points,
// complex sampling CPLX).
constexpr int kWarpKernelThreads = 128;

template <int FL, int CPLX>
__global__ void __launch_bounds__(kWarpKernelThreads)
fstep_warp_kernel(DevJob J, const DevStation *__restrict__ stations, SubintArrays S,
                  const BlockParam *__restrict__ bp, int nblk, int blocks_per_cta, int wstride,
                  float2 *__restrict__ spec)
{
  constexpr int NCH = CPLX ? FL : FL / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ float s_lut[256];
  __shared__ float2 s_tw[FL];
  const int s = blockIdx.y;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  const DevStation &st = stations[s];
  const int Sd = J.stride, lgS = J.lgstride, nfr = J.nfr, half = J.half;
  for (int i = tid; i < 256; i += blockDim.x) s_lut[i] = J.lut[i];
  for (int i = tid; i < FL; i += blockDim.x) s_tw[i] = J.twiddle[i];
  __syncthreads();

  float2 *A = reinterpret_cast<float2 *>(smem_raw) + (size_t)warp * wstride;   // FL + FL/8 (padded)
  float2 *rs = A + FL + FL / 8;   // S
  float2 *rp = rs + Sd;        // nfr
  float2 *fs = rp + nfr;       // S
  float2 *fp = fs + Sd;        // half

  const uint8_t *data = S.data[s];
  const int fsamp = J.framesamples;
  const int bits_ts = J.nbands * J.nbits * (CPLX ? 2 : 1);
  const int cmask = (1 << J.nbits) - 1;
  const int b0 = blockIdx.x * blocks_per_cta;
  const int nbk = min(blocks_per_cta, nblk - b0);
  const int nitems = nbk * J.nbands;
  for (int it = warp; it < nitems; it += nwarps) {
    const int bi = b0 + it / J.nbands;
    const int bd = it % J.nbands;
    const BlockParam P = band_param(bp, S, s, nblk, bi, J.nbands, bd);
    const int lf = st.band_localfreq[bd];
    const int f = st.freq_index[lf];
    float2 *dst = spec + ((size_t)f * nblk + bi) * J.ninputs * NCH;
    const int row = st.band_input[bd];
    if (P.state == 0) {
#pragma unroll
      for (int c = lane; c < NCH; c += 32) dst[spec_offset(J, row, c)] = make_float2(0.f, 0.f);
      continue;
    }
    const int ps = st.band_polb[bd] ? 1 : 0;
    for (int e = lane; e < Sd + nfr; e += 32) {
      const float2 v = fringe_entry(J, st, lf, e, P);
      if (e < Sd) rs[e] = v;
      else rp[e - Sd] = v;
    }
    for (int e = lane; e < Sd + half; e += 32) {
      const float2 v = frac_entry(J, st, lf, ps, e, P);
      if (e < Sd) fs[e] = v;
      else fp[e - Sd] = v;
    }
    __syncwarp();
    // decode + rotate: frame q and in-frame sample r advance incrementally
    {
      const int smp0 = P.nearestsample + lane;
      int q = smp0 / fsamp;
      int r = smp0 - q * fsamp;
      q -= P.fr0;
      const int bitband = bd * (CPLX ? 2 : 1) * J.nbits;
#pragma unroll 4
      for (int n = lane; n < FL; n += 32) {
        float2 u = make_float2(0.f, 0.f);
        if ((P.validmask >> q) & 1ull) {
          const uint8_t *payload = data + ((long long)P.fr0 + q) * J.framebytes + 32;
          const int bit0 = r * bits_ts + bitband;   // < 8 * payload bytes
          u.x = s_lut[(__ldg(payload + (bit0 >> 3)) >> (bit0 & 7)) & cmask];
          if (CPLX) {
            const int bit1 = bit0 + J.nbits;
            u.y = s_lut[(__ldg(payload + (bit1 >> 3)) >> (bit1 & 7)) & cmask];
          }
        }
        const int k = n & (Sd - 1), j = n >> lgS;
        const float2 rot = (j == 0) ? rs[k] : cmul_exact(rs[k], rp[j]);
        A[pidx(n)] = CPLX ? cmul(rot, u) : make_float2(u.x * rot.x, u.x * rot.y);
        r += 32;
        while (r >= fsamp) { r -= fsamp; q++; }
      }
    }
    __syncwarp();
    warp_fft<FL, 1>(A, s_tw, lane);
    const int lsb = st.lsb[lf];
#pragma unroll 4
    for (int c = lane; c < NCH; c += 32) {
      float2 v;
      if (!CPLX) v = A[pidx(lsb ? NCH + c : c)];
      else if (!lsb) v = A[pidx(c)];
      else if (c == 0) v = A[0];
      else { v = A[pidx(FL - c)]; v.y = -v.y; }
      dst[spec_offset(J, row, c)] = cmul(v, cmul_exact(fs[c & (Sd - 1)], fp[c >> lgS]));
    }
    __syncwarp();
  }
}

// --------------------------------------------------------------------------
// Slot-per-band F-step for long FFTs: the bands of a block in waves of
// nslots concurrent FFTs, each over kFThreads / nslots threads.
__global__ void __launch_bounds__(kFThreads)
fstep_cta_kernel(DevJob J, const DevStation *__restrict__ stations, SubintArrays S,
                 const BlockParam *__restrict__ bp, int nblk, int blocks_per_cta, int nslots,
                 float2 *__restrict__ spec)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ float s_lut[256];
  __shared__ BlockParam P;
  const int s = blockIdx.y;
  const int tid = threadIdx.x;
  const DevStation &st = stations[s];
  const int F = J.fftlen, N = J.nchan, Sd = J.stride, nfr = J.nfr, half = J.half;
  const int nrf = st.nrecfreqs;
  for (int i = tid; i < 256; i += blockDim.x) s_lut[i] = J.lut[i];

  float2 *slotbuf = reinterpret_cast<float2 *>(smem_raw);   // nslots * 2F
  float2 *rsub = slotbuf + (size_t)nslots * 2 * F;          // nrf * S
  float2 *rstep = rsub + nrf * Sd;                           // nrf * nfr
  float2 *fsub = rstep + nrf * nfr;                          // 2 * nrf * S
  float2 *fstep = fsub + 2 * nrf * Sd;                       // 2 * nrf * half
  float2 *rquad = fstep + 2 * nrf * (half > 0 ? half : 1);  // nrf * S (quadratic order)
  const bool quad = J.fringe_order == 2;

  const int tps = kFThreads / nslots;
  const int myslot = tid / tps;
  const int lt = (myslot < nslots) ? (tid % tps) : -1;
  const uint8_t *data = S.data[s];

  for (int bi = blockIdx.x * blocks_per_cta; bi < min(nblk, (blockIdx.x + 1) * blocks_per_cta); bi++) {
    __syncthreads();
    if (tid == 0) P = bp[(size_t)s * nblk + bi];
    __syncthreads();
    if (P.state == 0) {
      for (int bd = 0; bd < J.nbands; bd++) {
        const int f = st.freq_index[st.band_localfreq[bd]];
        float2 *dst = spec + ((size_t)f * nblk + bi) * J.ninputs * N;
        const int row = st.band_input[bd];
        for (int c = tid; c < N; c += blockDim.x) dst[spec_offset(J, row, c)] = make_float2(0.f, 0.f);
      }
      continue;
    }
    const int nfe = Sd + nfr + (quad ? Sd : 0);
    for (int idx = tid; idx < nrf * nfe; idx += blockDim.x) {
      const int fi = idx / nfe, e = idx % nfe;
      const float2 v = fringe_entry(J, st, fi, e, P);
      if (e < Sd) rsub[fi * Sd + e] = v;
      else if (e < Sd + nfr) rstep[fi * nfr + e - Sd] = v;
      else rquad[fi * Sd + e - Sd - nfr] = v;
    }
    const int npolsets = st.deltapol ? 2 : 1;
    for (int idx = tid; idx < npolsets * nrf * (Sd + half); idx += blockDim.x) {
      const int ps = idx / (nrf * (Sd + half));
      const int r = idx % (nrf * (Sd + half));
      const int fi = r / (Sd + half), e = r % (Sd + half);
      const float2 v = frac_entry(J, st, fi, ps, e, P);
      if (e < Sd) fsub[(ps * nrf + fi) * Sd + e] = v;
      else fstep[(ps * nrf + fi) * half + (e - Sd)] = v;
    }
    __syncthreads();
    for (int wave0 = 0; wave0 < J.nbands; wave0 += nslots) {
      const int bd = wave0 + myslot;
      const bool active = (lt >= 0) && (bd < J.nbands);
      float2 *bufA = slotbuf + (size_t)myslot * 2 * F;
      float2 *bufB = bufA + F;
      int lf = 0;
      if (active) {
        lf = st.band_localfreq[bd];
        const float2 *rs = rsub + lf * Sd;
        const float2 *rp = rstep + lf * nfr;
        if (quad) {
          // quadratic rotator (mode.cpp:996-1005) into bufB: stride j of entry k is
          // sub[k] quad[k]^j step[j], the powers formed by repeated FP32 products
          const float2 *rq = rquad + lf * Sd;
          for (int k = lt; k < Sd; k += tps) {
            float2 pw = rs[k];
            for (int j = 0; j < nfr; j++) {
              bufB[j * Sd + k] = cmul_exact(pw, rp[j]);
              pw = cmul_exact(rq[k], pw);
            }
          }
        }
      }
      __syncthreads();
      if (active) {
        const float2 *rs = rsub + lf * Sd;
        const float2 *rp = rstep + lf * nfr;
        BlockParam Pb = P;   // this band's frames
        if (S.bandmask) Pb.validmask &= ~S.bandmask[((size_t)s * nblk + bi) * J.nbands + bd];
        for (int n = lt; n < F; n += tps) {
          const float2 u = decode_sample(J, data, Pb, bd, n, s_lut);
          const int k = n % Sd, j = n / Sd;
          const float2 rot = quad ? bufB[n] : (j == 0) ? rs[k] : cmul_exact(rs[k], rp[j]);
          bufA[n] = J.cplx ? cmul(rot, u) : make_float2(u.x * rot.x, u.x * rot.y);
        }
      }
      __syncthreads();
      float2 *in = bufA, *out = bufB;
      for (int Ns = 1; Ns < F;) {
        const int R = (Ns * 8 <= F) ? 8 : ((Ns * 4 <= F) ? 4 : 2);
        if (active) {
          if (R == 8) stockham_pass<8>(in, out, F, Ns, J.twiddle, lt, tps);
          else if (R == 4) stockham_pass<4>(in, out, F, Ns, J.twiddle, lt, tps);
          else stockham_pass<2>(in, out, F, Ns, J.twiddle, lt, tps);
        }
        __syncthreads();
        float2 *t = in; in = out; out = t;
        Ns *= R;
      }
      if (active) {
        const int f = st.freq_index[lf];
        const int lsb = st.lsb[lf];
        const int ps = st.band_polb[bd] ? 1 : 0;
        const float2 *fs = fsub + (ps * nrf + lf) * Sd;
        const float2 *fp = fstep + (ps * nrf + lf) * half;
        float2 *dst = spec + ((size_t)f * nblk + bi) * J.ninputs * N;
        const int row = st.band_input[bd];
        for (int c = lt; c < N; c += tps) {
          const float2 v = select_channel(J, in, lsb, c);
          dst[spec_offset(J, row, c)] = cmul(v, cmul_exact(fs[c % Sd], fp[c / Sd]));
        }
      }
      __syncthreads();
    }
  }
}

// --------------------------------------------------------------------------
// Register-resident F-step for long transforms: a group of NT = F / 16 threads
// per (block, band) item, 16 samples per thread (x[j + NT t]) decoded and
// fringe-rotated straight into registers, transformed by the radix-16 passes of
// gx_fft16.h with padded shared-memory exchanges, and written from registers
// after the sideband selection and fractional-sample correction.  A CTA holds
// G = CTA / NT groups; groups synchronise on their own named barrier.
#ifndef GX_R16_MINB
#define GX_R16_MINB 4
#endif
template <int F>
struct R16Launch {
  static constexpr int NT = F / 16;
  static constexpr int CTA = NT >= 256 ? NT : 256;
  static constexpr int G = CTA / NT;
  static constexpr int MINB = GX_R16_MINB * 256 / CTA;   // resident CTAs per SM the registers are sized for
};


// Samples x[j + NT t] (t = 0..15) of band bd of the block described by P,
// decoded and fringe-rotated (mode.cpp:1160-1183): frame q and in-frame
// sample r advance incrementally; all 16 raw loads are issued before use.
// When a time sample of all bands is whole bytes and a step of NT samples
// crosses at most one frame boundary (NT <= samples per frame), the byte
// offset advances by a constant with one predicated correction per boundary;
// otherwise each sample's bit offset is formed from (q, r).
template <int F, int CPLX>
__device__ __forceinline__ void r16_decode_rotate(const DevJob &J, const uint8_t *__restrict__ data,
                                                  const BlockParam &P, int bd, int j, const float2 *rs,
                                                  const float2 *rp, const float *s_lut, float2 (&v)[16])
{
  constexpr int NT = F / 16;
  const int fsamp = J.framesamples;
  const int bits_ts = J.nbands * J.nbits * (CPLX ? 2 : 1);
  const int cmask = (1 << J.nbits) - 1;
  const bool byte_pairs = CPLX && J.nbits == 8;   // (re, im) = one 16-bit word
  const int smp0 = P.nearestsample + j;
  int q = smp0 / fsamp;
  int r = smp0 - q * fsamp;
  q -= P.fr0;
  const int bitband = bd * (CPLX ? 2 : 1) * J.nbits;
  unsigned int raw[16];
  if ((bits_ts & 7) == 0 && NT <= fsamp && (byte_pairs || !CPLX)) {
    const int bpts = bits_ts >> 3, sh = bitband & 7;
    const uint8_t *fr = data + ((long long)P.fr0 + q) * J.framebytes + 32 + (bitband >> 3);
    int off = r * bpts;
    bool ok = (P.validmask >> q) & 1ull;
#pragma unroll
    for (int t = 0; t < 16; t++) {
      if (byte_pairs)
        raw[t] = ok ? (unsigned int)__ldg(reinterpret_cast<const unsigned short *>(fr + off)) : 0xFFFFFFFFu;
      else
        raw[t] = ok ? ((unsigned int)(__ldg(fr + off) >> sh) & cmask) : 0xFFFFFFFFu;
      r += NT;
      off += NT * bpts;
      if (r >= fsamp) {   // next frame: skip its header
        r -= fsamp;
        off -= fsamp * bpts;
        q++;
        fr += J.framebytes;
        ok = (P.validmask >> q) & 1ull;
      }
    }
  } else {
#pragma unroll
    for (int t = 0; t < 16; t++) {
      raw[t] = 0xFFFFFFFFu;   // invalid frame: decodes to zero
      if ((P.validmask >> q) & 1ull) {
        const uint8_t *payload = data + ((long long)P.fr0 + q) * J.framebytes + 32;
        const int bit0 = r * bits_ts + bitband;   // < 8 * payload bytes
        if (byte_pairs) {
          raw[t] = __ldg(reinterpret_cast<const unsigned short *>(payload + (bit0 >> 3)));
        } else {
          unsigned int w = (__ldg(payload + (bit0 >> 3)) >> (bit0 & 7)) & cmask;
          if (CPLX) {
            const int bit1 = bit0 + J.nbits;
            w |= ((__ldg(payload + (bit1 >> 3)) >> (bit1 & 7)) & cmask) << 8;
          }
          raw[t] = w;
        }
      }
      r += NT;
      while (r >= fsamp) { r -= fsamp; q++; }
    }
  }
  // rotator x[n] = sub[n mod S] * step[n / S]; with S dividing NT the sub entry
  // is the same for all 16 samples of the thread
  const int Sd = J.stride, lgS = J.lgstride;
  const bool kfix = (NT & (Sd - 1)) == 0;
  const float2 rsk = rs[j & (Sd - 1)];
  const int jj0 = j >> lgS, jstep = NT >> lgS;
#pragma unroll
  for (int t = 0; t < 16; t++) {
    float2 u = make_float2(0.f, 0.f);
    if (raw[t] != 0xFFFFFFFFu) {
      u.x = s_lut[raw[t] & 255u];
      if (CPLX) u.y = s_lut[(raw[t] >> 8) & 255u];
    }
    float2 rot;
    if (kfix) {
      const int jj = jj0 + jstep * t;
      rot = (jj == 0) ? rsk : cmul_exact(rsk, rp[jj]);
    } else {
      const int n = j + NT * t;
      const int k = n & (Sd - 1), jj = n >> lgS;
      rot = (jj == 0) ? rs[k] : cmul_exact(rs[k], rp[jj]);
    }
    v[t] = CPLX ? cmul(rot, u) : make_float2(u.x * rot.x, u.x * rot.y);
  }
}

// Forward FFT of the group's transform: radix-16 passes with exchanges through
// the padded buffer sm, then the final radix; register t ends with bin j + NT t.
template <int F, int CTA, typename TW>
__device__ __forceinline__ void r16_fft(float2 (&v)[16], int j, int g, float2 *sm, TW tw)
{
  using Pl = r16::Plan<F>;
  constexpr int NT = Pl::NT;
  int Ns = 1;
#pragma unroll
  for (int pass = 0; pass < Pl::L; pass++) {
    r16::pass16<F>(v, j, Ns, tw);
    if (!(pass == Pl::L - 1 && Pl::R0 == 1)) {
      group_sync<NT, CTA>(g);
      r16::store16(v, j, Ns, sm);
      group_sync<NT, CTA>(g);
      r16::load16<F>(v, j, sm);
    }
    Ns *= 16;
  }
  if constexpr (Pl::R0 > 1) r16::final_pass<F, Pl::R0>(v, j, tw);
}


template <int F, int CPLX>
__global__ void __launch_bounds__(R16Launch<F>::CTA, R16Launch<F>::MINB)
fstep_r16_kernel(DevJob J, const DevStation *__restrict__ stations, SubintArrays S,
                 const BlockParam *__restrict__ bp, int nblk, int blocks_per_cta, int tabstride,
                 float2 *__restrict__ spec)
{
  using Pl = r16::Plan<F>;
  constexpr int NT = Pl::NT, CTA = R16Launch<F>::CTA, G = R16Launch<F>::G;
  constexpr int NCH = CPLX ? F : F / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ float s_lut[256];
  const int s = blockIdx.y;
  const int tid = threadIdx.x, g = tid / NT, j = tid % NT;
  const DevStation &st = stations[s];
  const int Sd = J.stride, lgS = J.lgstride, nfr = J.nfr, half = J.half;
  for (int i = tid; i < 256; i += CTA) s_lut[i] = J.lut[i];
  __syncthreads();

  float2 *sm = reinterpret_cast<float2 *>(smem_raw) + (size_t)g * (Pl::SMEM + tabstride);
  float2 *rs = sm + Pl::SMEM;  // S
  float2 *rp = rs + Sd;        // nfr
  float2 *fs = rp + nfr;       // S
  float2 *fp = fs + Sd;        // half
  const float2 *__restrict__ twg = J.twiddle;
  auto tw = [twg](int m) { return __ldg(&twg[m]); };

  const uint8_t *data = S.data[s];
  const int b0 = blockIdx.x * blocks_per_cta;
  const int nbk = min(blocks_per_cta, nblk - b0);
  const int nitems = nbk * J.nbands;
  for (int it = g; it < nitems; it += G) {
    const int bi = b0 + it / J.nbands;
    const int bd = it % J.nbands;
    const BlockParam P = band_param(bp, S, s, nblk, bi, J.nbands, bd);
    const int lf = st.band_localfreq[bd];
    const int f = st.freq_index[lf];
    const int row = st.band_input[bd];
    float2 *dst = spec + ((size_t)f * nblk + bi) * J.ninputs * NCH;
    if (P.state == 0) {
      for (int c = j; c < NCH; c += NT) dst[spec_offset(J, row, c)] = make_float2(0.f, 0.f);
      continue;
    }
    const int ps = st.band_polb[bd] ? 1 : 0;
    group_sync<NT, CTA>(g);   // the group's previous item is done with the tables and the exchange buffer
    for (int e = j; e < Sd + nfr; e += NT) {
      const float2 v = fringe_entry(J, st, lf, e, P);
      if (e < Sd) rs[e] = v;
      else rp[e - Sd] = v;
    }
    for (int e = j; e < Sd + half; e += NT) {
      const float2 v = frac_entry(J, st, lf, ps, e, P);
      if (e < Sd) fs[e] = v;
      else fp[e - Sd] = v;
    }
    group_sync<NT, CTA>(g);

    float2 v[16];
    r16_decode_rotate<F, CPLX>(J, data, P, bd, j, rs, rp, s_lut, v);
    r16_fft<F, CTA>(v, j, g, sm, tw);
    // register t holds bin j + NT t: sideband selection and fractional-sample correction
    // (with S dividing NT, channel c mod S is the same for all the thread's bins:
    // j mod S, or -j mod S for complex lower sideband)
    const int lsb = st.lsb[lf];
    const bool kfix = (NT & (Sd - 1)) == 0;
    const float2 fsk = fs[((CPLX && lsb) ? -j : j) & (Sd - 1)];
    float2 *drow = dst + spec_offset(J, row, 0);
    auto emit = [&](int c, float2 val) {
      drow[c] = cmul(val, cmul_exact(kfix ? fsk : fs[c & (Sd - 1)], fp[c >> lgS]));
    };
    // one unrolled loop per sideband, so that every channel index is j plus a constant
    if (lsb) {
#pragma unroll
      for (int t = 0; t < 16; t++) {
        float2 val = v[t];
        int c;
        if (r16_channel<F, CPLX>(t, j, 1, val, c)) emit(c, val);
      }
    } else {
#pragma unroll
      for (int t = 0; t < 16; t++) {
        float2 val = v[t];
        int c;
        if (r16_channel<F, CPLX>(t, j, 0, val, c)) emit(c, val);
      }
    }
  }
}

// --------------------------------------------------------------------------
// The warp and radix-16 kernels hold the fringe rotator as two tables
// (sub[k] step[j]); the quadratic order needs the full table of the CTA kernel.
static bool use_warp_kernel(const DevJob &J) { return J.fftlen >= 128 && J.fftlen <= 1024 && J.fringe_order != 2; }

static int warp_stride(const DevJob &J)
{
  int w = J.fftlen + J.fftlen / 8 + 2 * J.stride + J.nfr + (J.half > 0 ? J.half : 1);
  return (w + 1) & ~1;   // keep each warp's region 16-byte aligned
}

// Register-resident radix-16 kernel for the transform lengths it is built for.
static bool use_r16_kernel(const DevJob &J)
{
  const char *e = getenv("GX_FSTEP_R16_MIN");   // smallest length routed to it (tuning runs)
  const int fmin = e ? atoi(e) : 512;
  return J.fftlen >= fmin && J.fftlen >= 512 && J.fftlen <= 8192 && J.fringe_order != 2;
}

// Station-block kernel (gx_fstep_sb.cu) for the jobs it takes; GX_FSTEP_SB=0
// selects the per-band kernels instead (comparison runs).
bool fstep_sb_eligible(const DevJob &J, bool interlaced);
cudaError_t fstep_sb_launch(const DevJob &J, const DevStation *stations, int maxnrf, int deltapol,
                            const SubintArrays &S, int nblk, const BlockParam *bp, float2 *spec, cudaStream_t st,
                            const PcalFuse *pf, bool *pcal_done);

static bool use_sb_kernel(const DevJob &J, bool interlaced)
{
  const char *e = getenv("GX_FSTEP_SB");
  if (e && atoi(e) == 0) return false;
  return fstep_sb_eligible(J, interlaced);
}

static int r16_tabstride(const DevJob &J)
{
  return (2 * J.stride + J.nfr + (J.half > 0 ? J.half : 1) + 1) & ~1;
}

static int r16_groups(const DevJob &J)
{
  const int nt = J.fftlen / 16;
  return nt >= 256 ? 1 : 256 / nt;
}

size_t fstep_smem_bytes(const DevJob &J, int nrf, int nslots)
{
  if (use_r16_kernel(J))
    return (size_t)r16_groups(J) * (J.fftlen + J.fftlen / 16 + r16_tabstride(J)) * sizeof(float2);
  if (use_warp_kernel(J)) return (size_t)(kWarpKernelThreads / 32) * warp_stride(J) * sizeof(float2);
  size_t b = (size_t)nslots * 2 * J.fftlen * sizeof(float2);
  b += (size_t)nrf * (J.stride + J.nfr) * sizeof(float2);
  b += (size_t)2 * nrf * (J.stride + (J.half > 0 ? J.half : 1)) * sizeof(float2);
  b += (size_t)nrf * J.stride * sizeof(float2);   // quadratic per-stride steps
  return b;
}

// ---------------------------------------------------------------------------
// Phase-cal extraction (Mode::process, mode.cpp:759-774; the implicit-shift
// extractors of pcal.cpp).  Every processed block adds its F decoded samples
// (before any rotation, as the reference's unpacked arrays) into nbins bins
// by absolute sample number; thread k of a CTA owns bin k (and k + 256, ...)
// of its chunk of blocks, so every bin sum is formed in a fixed order.
// The samples are decoded as decode_sample (above) and the reference's unpacker do.

// Sum of the decoded samples n = n0, n0 + step, ... < F of band bd of a
// processed block, walking frame q and in-frame sample r incrementally (one
// division per call, not per sample).
__device__ __forceinline__ float2 sum_samples(const DevJob &J, const uint8_t *__restrict__ data,
                                              const BlockParam &P, int bd, int n0, int step, const float *lut)
{
  float2 acc = make_float2(0.f, 0.f);
  if (n0 >= J.fftlen) return acc;
  const int fsamp = J.framesamples;
  const int bits_ts = J.nbands * J.nbits * (J.cplx ? 2 : 1);
  const int cmask = (1 << J.nbits) - 1;
  const int bitband = bd * (J.cplx ? 2 : 1) * J.nbits;
  const int smp0 = P.nearestsample + n0;
  int q = smp0 / fsamp;
  int r = smp0 - q * fsamp;
  q -= P.fr0;
  const int qstep = step / fsamp, rstep = step - qstep * fsamp;
  for (int n = n0; n < J.fftlen; n += step) {
    if ((P.validmask >> q) & 1ull) {
      const uint8_t *payload = data + ((long long)P.fr0 + q) * J.framebytes + 32;
      const int bit0 = r * bits_ts + bitband;
      acc.x += lut[(__ldg(payload + (bit0 >> 3)) >> (bit0 & 7)) & cmask];
      if (J.cplx) {
        const int bit1 = bit0 + J.nbits;
        acc.y += lut[(__ldg(payload + (bit1 >> 3)) >> (bit1 & 7)) & cmask];
      }
    }
    q += qstep;
    r += rstep;
    if (r >= fsamp) {
      r -= fsamp;
      q++;
    }
  }
  return acc;
}

// The shifting extractors' form (pcal.cpp:692-740, 906-955): every sample
// times the oscillator entry (S mod L) + (n mod L) of the reference's table of
// 2 L FP32 values, then summed; S: the block's absolute sample number.
__device__ __forceinline__ float2 sum_samples_rot(const DevJob &J, const uint8_t *__restrict__ data,
                                                  const BlockParam &P, int bd, int n0, int step, const float *lut,
                                                  const float2 *__restrict__ rot, int L, int sl)
{
  float2 acc = make_float2(0.f, 0.f);
  if (n0 >= J.fftlen) return acc;
  const int fsamp = J.framesamples;
  const int bits_ts = J.nbands * J.nbits * (J.cplx ? 2 : 1);
  const int cmask = (1 << J.nbits) - 1;
  const int bitband = bd * (J.cplx ? 2 : 1) * J.nbits;
  const int smp0 = P.nearestsample + n0;
  int q = smp0 / fsamp;
  int r = smp0 - q * fsamp;
  q -= P.fr0;
  const int qstep = step / fsamp, rstep = step - qstep * fsamp;
  const int lstep = step % L;
  int nl = n0 % L;
  for (int n = n0; n < J.fftlen; n += step) {
    if ((P.validmask >> q) & 1ull) {
      const uint8_t *payload = data + ((long long)P.fr0 + q) * J.framebytes + 32;
      const int bit0 = r * bits_ts + bitband;
      const float xr = lut[(__ldg(payload + (bit0 >> 3)) >> (bit0 & 7)) & cmask];
      const float2 o = __ldg(rot + sl + nl);
      if (J.cplx) {
        const int bit1 = bit0 + J.nbits;
        const float xi = lut[(__ldg(payload + (bit1 >> 3)) >> (bit1 & 7)) & cmask];
        acc.x += xr * o.x - xi * o.y;
        acc.y += xr * o.y + xi * o.x;
      } else {
        acc.x += xr * o.x;
        acc.y += xr * o.y;
      }
    }
    q += qstep;
    r += rstep;
    if (r >= fsamp) {
      r -= fsamp;
      q++;
    }
    nl += lstep;
    if (nl >= L) nl -= L;
  }
  return acc;
}

__global__ void __launch_bounds__(256) pcal_bins_kernel(DevJob J, SubintArrays S, const BlockParam *__restrict__ bp,
                                                        int nblk, const PcalBand *__restrict__ bands,
                                                        const float2 *__restrict__ rot, int chunks, int maxbins,
                                                        float2 *__restrict__ partial)
{
  __shared__ float s_lut[256];
  __shared__ float2 s_red[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) s_lut[i] = J.lut[i];
  __syncthreads();
  const int c = blockIdx.x, pb = blockIdx.y;
  const PcalBand B = bands[pb];
  const int s = B.station, N = B.nbins;
  if (N <= 0) return;
  const uint8_t *data = S.data[s];
  const int32_t *ctrl = S.control + (size_t)s * S.controlstride;
  // sample number of the data buffer's start (mode.cpp:761)
  const unsigned long long s0 =
      (unsigned long long)(((double)ctrl[1] * 1e9 + (double)ctrl[2]) / (J.sampletime * 1e3) + 0.5);
  const int per = (nblk + chunks - 1) / chunks;
  const int b0 = c * per, b1 = min(nblk, b0 + per);
  float2 *out = partial + ((size_t)c * gridDim.y + pb) * maxbins;
  const int tid = threadIdx.x, nth = blockDim.x;
  if (N <= nth) {
    // R threads per bin: thread (r, k) takes samples n = n0(k) + (r + R m) N; consecutive
    // threads read consecutive samples
    const int R = nth / N;
    const int k = tid % N, r = tid / N;
    float2 acc = make_float2(0.f, 0.f);
    if (r < R) {
      for (int bi = b0; bi < b1; bi++) {
        const BlockParam P = band_param(bp, S, s, nblk, bi, J.nbands, B.band);
        if (P.state == 0) continue;
        const unsigned long long sb = s0 + (unsigned long long)P.nearestsample;
        const int idx0 = (int)(sb % (unsigned long long)N);
        const float2 v =
            B.rotlen > 0
                ? sum_samples_rot(J, data, P, B.band, (k - idx0 + N) % N + r * N, R * N, s_lut, rot + B.rot0, B.rotlen,
                                  (int)(sb % (unsigned long long)B.rotlen))
                : sum_samples(J, data, P, B.band, (k - idx0 + N) % N + r * N, R * N, s_lut);
        acc.x += v.x;
        acc.y += v.y;
      }
    }
    s_red[tid] = acc;
    __syncthreads();
    if (tid < N) {   // the R partial sums of bin k, in order
      float2 sum = s_red[tid];
      for (int q = 1; q < R; q++) {
        sum.x += s_red[tid + q * N].x;
        sum.y += s_red[tid + q * N].y;
      }
      out[tid].x += sum.x;
      out[tid].y += sum.y;
    }
  } else {
    for (int k = tid; k < N; k += nth) {   // more bins than threads: one thread per bin
      float2 acc = make_float2(0.f, 0.f);
      for (int bi = b0; bi < b1; bi++) {
        const BlockParam P = band_param(bp, S, s, nblk, bi, J.nbands, B.band);
        if (P.state == 0) continue;
        const unsigned long long sb = s0 + (unsigned long long)P.nearestsample;
        const int idx0 = (int)(sb % (unsigned long long)N);
        const float2 v = B.rotlen > 0 ? sum_samples_rot(J, data, P, B.band, (k - idx0 + N) % N, N, s_lut, rot + B.rot0,
                                                        B.rotlen, (int)(sb % (unsigned long long)B.rotlen))
                                      : sum_samples(J, data, P, B.band, (k - idx0 + N) % N, N, s_lut);
        acc.x += v.x;
        acc.y += v.y;
      }
      out[k].x += acc.x;
      out[k].y += acc.y;
    }
  }
}

// The same bin sums for all nb bands of one station at once, for time samples
// of W 32-bit words (W = 1: 8, 16 or 32 bits) holding bands 0..nb-1 in order.
// Thread (r, k) reads whole time samples -- the threads of a warp read
// consecutive ones, one wide load each -- and bins every band from registers.
// 8-bit codes (NBITS 8; level = (code - offset) / div, an affine table) are
// summed as integers: the fields of each word in two 16-bit lanes per
// register (even and odd bytes), moved into 32-bit totals after each block
// (at most 256 samples of a thread, so that no lane overflows), then
// (sum - offset * count) / div in double once per bin.  Integer sums make the
// result independent of the summation order.  Other widths look the level up
// in a per-lane copy of the table (NBITS 0: width read at run time).
constexpr int kPcalMaxBands = 16;

template <int W>
__device__ __forceinline__ uint4 load_timesample(const uint8_t *p, int align)
{
  if (W == 4 && align >= 16) return __ldg(reinterpret_cast<const uint4 *>(p));
  if (W == 2 && align >= 8) {
    const uint2 h = __ldg(reinterpret_cast<const uint2 *>(p));
    return make_uint4(h.x, h.y, 0u, 0u);
  }
  uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
  for (int i = 0; i < W; i++)
    w[i] = align >= 4 ? __ldg(reinterpret_cast<const uint32_t *>(p) + i)
                      : (uint32_t)__ldg(p + 4 * i) | ((uint32_t)__ldg(p + 4 * i + 1) << 8) |
                            ((uint32_t)__ldg(p + 4 * i + 2) << 16) | ((uint32_t)__ldg(p + 4 * i + 3) << 24);
  return make_uint4(w[0], w[1], w[2], w[3]);
}

template <int W>
__device__ __forceinline__ uint32_t word(const uint4 &w, int i)
{
  return (W > 3 && i == 3) ? w.w : (W > 2 && i == 2) ? w.z : (W > 1 && i == 1) ? w.y : w.x;
}

template <int W>
__device__ __forceinline__ uint32_t field(const uint4 &w, int pos)
{
  return word<W>(w, pos >> 5) >> (pos & 31);
}

template <int W, int NBITS, int CPLX>
__global__ void __launch_bounds__(256) pcal_station_kernel(DevJob J, SubintArrays S, const BlockParam *__restrict__ bp,
                                                           int nblk, const PcalBand *__restrict__ bands, int nb,
                                                           int chunks, int maxbins, int nbands_total,
                                                           float2 *__restrict__ partial)
{
  constexpr bool kInt = NBITS == 8;
  // one copy of the decode table per lane, so that a warp's lookups of random
  // codes never share a bank: entry v of lane l at v * 32 + l
  extern __shared__ float s_lut32[];
  __shared__ float2 s_red[256];
  __shared__ int s_cnt[256];
  const int nbits = NBITS ? NBITS : J.nbits;
  const int cplx = NBITS ? CPLX : J.cplx;
  if (!kInt) {
    for (int i = threadIdx.x; i < (32 << nbits); i += blockDim.x) s_lut32[i] = J.lut[i >> 5];
    __syncthreads();
  }
  const float *s_lut = s_lut32 + (threadIdx.x & 31);
  const int c = blockIdx.x, first = blockIdx.y * nb;
  const PcalBand B0 = bands[first];
  const int s = B0.station, N = B0.nbins;
  const uint8_t *data = S.data[s];
  const int32_t *ctrl = S.control + (size_t)s * S.controlstride;
  const unsigned long long s0 =
      (unsigned long long)(((double)ctrl[1] * 1e9 + (double)ctrl[2]) / (J.sampletime * 1e3) + 0.5);
  const int per = (nblk + chunks - 1) / chunks;
  const int b0 = c * per, b1 = min(nblk, b0 + per);
  const int tid = threadIdx.x, nth = blockDim.x;
  const int fsamp = J.framesamples, fb = J.framebytes;
  const int bandbits = nbits * (cplx ? 2 : 1);
  const int bits_ts = nb * bandbits;
  const uint32_t cmask = (1u << nbits) - 1u;
  const uint32_t tsmask = bits_ts >= 32 ? 0xffffffffu : (1u << bits_ts) - 1u;
  // widest load every time sample start allows: the frame stride, the data
  // base and the sample size all keep the alignment
  int align = 16;
  while (align > 1 && (((uintptr_t)data | (uintptr_t)fb | (uintptr_t)32) & (align - 1))) align >>= 1;
  align = min(align, max(4, W * 4));
  if (bits_ts < 32) align = ((uintptr_t)data & 3) || (fb & 3) ? 1 : 4;
  for (int kb = 0; kb < N; kb += nth) {   // bins kb .. kb+nk-1 in this pass
    const int nk = min(nth, N - kb);
    const int R = nth / nk;
    const int k = kb + tid % nk, r = tid / nk;
    float ax[kPcalMaxBands], ay[kPcalMaxBands];
    int tot[4 * W];   // 8-bit: per field (band-major, real then imaginary)
    int cnt = 0;
#pragma unroll
    for (int b = 0; b < kPcalMaxBands; b++) ax[b] = ay[b] = 0.f;
#pragma unroll
    for (int f = 0; f < 4 * W; f++) tot[f] = 0;
    if (r < R) {
      const int step = R * N;
      const int qstep = step / fsamp, rstep = step - qstep * fsamp;
      for (int bi = b0; bi < b1; bi++) {
        const BlockParam P = bp[(size_t)s * nblk + bi];
        if (P.state == 0) continue;
        const int idx0 = (int)((s0 + (unsigned long long)P.nearestsample) % (unsigned long long)N);
        const int n0 = (k - idx0 + N) % N + r * N;
        const int smp0 = P.nearestsample + n0;
        int q = smp0 / fsamp;
        int rr = smp0 - q * fsamp;
        q -= P.fr0;
        uint32_t pe[W], po[W];   // 8-bit: even / odd bytes of word i in 16-bit lanes
#pragma unroll
        for (int i = 0; i < W; i++) pe[i] = po[i] = 0u;
        for (int n = n0; n < J.fftlen; n += step) {
          if ((P.validmask >> q) & 1ull) {
            const uint8_t *payload = data + ((long long)P.fr0 + q) * fb + 32;
            uint4 w;
            int sh = 0;
            if (bits_ts < 32) {
              const int bit = rr * bits_ts;
              w = load_timesample<W>(payload + ((bit >> 5) << 2), align);
              sh = bit & 31;
            } else {
              w = load_timesample<W>(payload + (size_t)rr * (W * 4), align);
            }
            if constexpr (kInt) {
              cnt++;
#pragma unroll
              for (int i = 0; i < W; i++) {
                const uint32_t x = W == 1 ? (w.x >> sh) & tsmask : word<W>(w, i);
                pe[i] += x & 0x00ff00ffu;
                po[i] += (x >> 8) & 0x00ff00ffu;
              }
            } else {
#pragma unroll
              for (int b = 0; b < kPcalMaxBands; b++) {
                if (b < nb) {
                  const int pos = b * bandbits + sh;
                  ax[b] += s_lut[(field<W>(w, pos) & cmask) << 5];
                  if (cplx) ay[b] += s_lut[(field<W>(w, pos + nbits) & cmask) << 5];
                }
              }
            }
          }
          q += qstep;
          rr += rstep;
          if (rr >= fsamp) {
            rr -= fsamp;
            q++;
          }
        }
        if constexpr (kInt) {   // fields 4i, 4i+2 in pe[i]; 4i+1, 4i+3 in po[i]
#pragma unroll
          for (int i = 0; i < W; i++) {
            tot[4 * i] += (int)(pe[i] & 0xffffu);
            tot[4 * i + 2] += (int)(pe[i] >> 16);
            tot[4 * i + 1] += (int)(po[i] & 0xffffu);
            tot[4 * i + 3] += (int)(po[i] >> 16);
          }
        }
      }
    }
    if constexpr (kInt) s_cnt[tid] = cnt;
#pragma unroll
    for (int b = 0; b < kPcalMaxBands; b++) {
      if (b < nb) {
        if constexpr (kInt) {
          const int fr = b * (CPLX ? 2 : 1);   // this band's real field
          int re = 0, im = 0;
#pragma unroll
          for (int f = 0; f < 4 * W; f++) {
            if (f == fr) re = tot[f];
            if (CPLX && f == fr + 1) im = tot[f];
          }
          s_red[tid] = make_float2(__int_as_float(re), __int_as_float(im));
        } else {
          s_red[tid] = make_float2(ax[b], ay[b]);
        }
        __syncthreads();
        if (tid < nk) {   // the R partial sums of (band b, bin k), in order
          float2 sum;
          if constexpr (kInt) {
            long long re = 0, im = 0, n = 0;
            for (int qq = 0; qq < R; qq++) {
              re += __float_as_int(s_red[tid + qq * nk].x);
              im += __float_as_int(s_red[tid + qq * nk].y);
              n += s_cnt[tid + qq * nk];
            }
            sum.x = (float)(((double)re - J.lut_offset * (double)n) / J.lut_div);
            sum.y = CPLX ? (float)(((double)im - J.lut_offset * (double)n) / J.lut_div) : 0.f;
          } else {
            sum = s_red[tid];
            for (int qq = 1; qq < R; qq++) {
              sum.x += s_red[tid + qq * nk].x;
              sum.y += s_red[tid + qq * nk].y;
            }
          }
          float2 &o = partial[((size_t)c * nbands_total + first + b) * maxbins + k];
          o.x += sum.x;
          o.y += sum.y;
        }
        __syncthreads();
      }
    }
  }
}

// Tone t of band pb: the forward DFT of the bins at bin offset_bin + t step,
// summed in double and rounded once (the reference's DFT of its bins).
__global__ void __launch_bounds__(128) pcal_tones_kernel(const PcalBand *__restrict__ bands, int chunks, int maxbins,
                                                         const float2 *__restrict__ partial, float2 *__restrict__ results)
{
  const int pb = blockIdx.x;
  const PcalBand B = bands[pb];
  for (int t = threadIdx.x; t < B.ntones; t += blockDim.x) {
    const long long bin = (long long)B.offset_bin + (long long)t * B.step;
    double re = 0.0, im = 0.0;
    if (B.nbins > 0 && bin < B.nbins && t < B.nextract) {
      for (int k = 0; k < B.nbins; k++) {
        float bx = 0.f, by = 0.f;   // the bin, summed over the chunks in order
        for (int c = 0; c < chunks; c++) {
          const float2 v = partial[((size_t)c * gridDim.x + pb) * maxbins + k];
          bx += v.x;
          by += v.y;
        }
        const long long m = ((long long)k * bin) % B.nbins;
        double sn, cs;
        sincospi(-2.0 * (double)m / (double)B.nbins, &sn, &cs);
        re += (double)bx * cs - (double)by * sn;
        im += (double)bx * sn + (double)by * cs;
      }
    }
    results[B.result_offset + t] = make_float2((float)re, (float)im);
  }
}

cudaError_t pcal_bins_launch(const DevJob &J, const SubintArrays &S, const BlockParam *bp, int nblk,
                             const PcalBand *bands, const float2 *rot, int nbands, int per_station, int chunks,
                             int maxbins,
                             float2 *partial, cudaStream_t st)
{
  if (nbands <= 0 || nblk <= 0) return cudaSuccess;
  const int bits_ts = J.nbands * J.nbits * (J.cplx ? 2 : 1);
  const dim3 grid(chunks, per_station > 0 ? nbands / per_station : 1);
  const size_t lut_bytes = sizeof(float) * 32 * ((size_t)1 << J.nbits);   // at most 32 KB
  // every station has per_station bands (0..per_station-1, in order) with the
  // same bin count, and a time sample is 1, 2 or 4 words or divides a word;
  // the 8-bit integer sums need at most 256 samples of a thread per block
  // (the FFT length over the sample step R N, which is above 128)
  const int W = bits_ts == 128 ? 4 : bits_ts == 64 ? 2 : (bits_ts <= 32 && 32 % bits_ts == 0) ? 1 : 0;
  const bool station = per_station > 0 && per_station <= kPcalMaxBands && W > 0 && !S.bandmask;
  const bool i8 = J.nbits == 8 && J.fftlen <= 256 * 128;
#define GX_PCAL_STATION(w, nbits, cplx)                                                                       \
  pcal_station_kernel<w, nbits, cplx><<<grid, 256, nbits == 8 ? 0 : lut_bytes, st>>>(                         \
      J, S, bp, nblk, bands, per_station, chunks, maxbins, nbands, partial)
  if (station && i8) {
    if (W == 4) { if (J.cplx) GX_PCAL_STATION(4, 8, 1); else GX_PCAL_STATION(4, 8, 0); }
    else if (W == 2) { if (J.cplx) GX_PCAL_STATION(2, 8, 1); else GX_PCAL_STATION(2, 8, 0); }
    else { if (J.cplx) GX_PCAL_STATION(1, 8, 1); else GX_PCAL_STATION(1, 8, 0); }
  } else if (station && J.nbits == 2 && !J.cplx) {
    if (W == 4) GX_PCAL_STATION(4, 2, 0);
    else if (W == 2) GX_PCAL_STATION(2, 2, 0);
    else GX_PCAL_STATION(1, 2, 0);
  } else if (station && J.nbits != 8) {
    if (W == 4) GX_PCAL_STATION(4, 0, 0);
    else if (W == 2) GX_PCAL_STATION(2, 0, 0);
    else GX_PCAL_STATION(1, 0, 0);
  } else {
    pcal_bins_kernel<<<dim3(chunks, nbands), 256, 0, st>>>(J, S, bp, nblk, bands, rot, chunks, maxbins, partial);
  }
#undef GX_PCAL_STATION
  return cudaGetLastError();
}

// Sum of the chunks' partial bin sums into chunk 0, in chunk order (the order
// the tones kernel would add them in): one thread per (band, bin), loads
// coalesced across threads.
__global__ void __launch_bounds__(256) pcal_fold_kernel(float2 *__restrict__ partial, int chunks, long long n)
{
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float bx = 0.f, by = 0.f;
#pragma unroll 8
  for (int c = 0; c < chunks; c++) {
    const float2 v = partial[(size_t)c * n + i];
    bx += v.x;
    by += v.y;
  }
  partial[i] = make_float2(bx, by);
}

cudaError_t pcal_fold_launch(float2 *partial, int chunks, long long n, cudaStream_t st)
{
  if (chunks <= 1 || n <= 0) return cudaSuccess;
  pcal_fold_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(partial, chunks, n);
  return cudaGetLastError();
}

cudaError_t pcal_tones_launch(const PcalBand *bands, int nbands, int chunks, int maxbins, const float2 *partial,
                              float2 *results, cudaStream_t st)
{
  if (nbands <= 0) return cudaSuccess;
  pcal_tones_kernel<<<nbands, 128, 0, st>>>(bands, chunks, maxbins, partial, results);
  return cudaGetLastError();
}

cudaError_t smem_opt_in(const void *kernel, size_t bytes)
{
  if (bytes <= 48 * 1024) return cudaSuccess;
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, size_t> limits;   // (kernel, device) -> limit set
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  size_t &have = limits[{kernel, dev}];
  if (bytes <= have) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) have = bytes;
  return e;
}

cudaError_t fstep_launch(const DevJob &J, const DevStation *stations, int maxnrf, const SubintArrays &S,
                         int blk0, int nblk, int nslots, float2 *spec, float *weights, BlockParam *bp,
                         cudaStream_t st, const PcalFuse *pf, bool *pcal_done)
{
  if (pcal_done) *pcal_done = false;
  {
    dim3 grid((nblk + 127) / 128, J.nstations);
    blockparams_kernel<<<grid, 128, 0, st>>>(J, S, blk0, nblk, bp, weights);
  }
  if (S.bandmask) {   // INTERLACEDVDIF: EDV4 per-band validity, one warp per (station, block)
    dim3 grid((nblk + 7) / 8, J.nstations);
    edv4_kernel<<<grid, 256, 0, st>>>(J, stations, S, nblk, bp, weights);
  }
  if (use_sb_kernel(J, S.bandmask != nullptr)) {
    cudaError_t e = fstep_sb_launch(J, stations, maxnrf, J.deltapol_any, S, nblk, bp, spec, st, pf, pcal_done);
    if (e != cudaErrorNotSupported) return e;
    if (pcal_done) *pcal_done = false;
  }
  const size_t sm = fstep_smem_bytes(J, maxnrf, nslots);
  if (use_r16_kernel(J)) {
    const int G = r16_groups(J);
    // at least four items per group, so that groups overlap their barriers
    const int bpc = std::max(1, (4 * G + J.nbands - 1) / J.nbands);
    dim3 grid((nblk + bpc - 1) / bpc, J.nstations);
    const int ts = r16_tabstride(J);
#define GX_R16_CASE(FLV, CX)                                                                          \
    if (J.fftlen == FLV && J.cplx == CX) {                                                            \
      cudaError_t e = smem_opt_in((const void *)fstep_r16_kernel<FLV, CX>, sm);                       \
      if (e != cudaSuccess) return e;                                                                 \
      fstep_r16_kernel<FLV, CX><<<grid, R16Launch<FLV>::CTA, sm, st>>>(J, stations, S, bp, nblk, bpc, ts, spec); \
      return cudaGetLastError();                                                                      \
    }
    GX_R16_CASE(512, 0) GX_R16_CASE(1024, 0) GX_R16_CASE(2048, 0) GX_R16_CASE(4096, 0) GX_R16_CASE(8192, 0)
    GX_R16_CASE(512, 1) GX_R16_CASE(1024, 1) GX_R16_CASE(2048, 1) GX_R16_CASE(4096, 1) GX_R16_CASE(8192, 1)
#undef GX_R16_CASE
  }
  if (use_warp_kernel(J)) {
    // enough items per CTA that each warp has several (block, band) items
    const int bpc = (J.nbands >= 8) ? 2 : 8;
    dim3 grid((nblk + bpc - 1) / bpc, J.nstations);
    const int ws = warp_stride(J);
#define GX_WARP_CASE(FLV, CX)                                                                         \
    if (J.fftlen == FLV && J.cplx == CX) {                                                            \
      cudaError_t e = smem_opt_in((const void *)fstep_warp_kernel<FLV, CX>, sm);                      \
      if (e != cudaSuccess) return e;                                                                 \
      fstep_warp_kernel<FLV, CX><<<grid, kWarpKernelThreads, sm, st>>>(J, stations, S, bp, nblk, bpc, ws, spec); \
      return cudaGetLastError();                                                                      \
    }
    GX_WARP_CASE(128, 0) GX_WARP_CASE(256, 0) GX_WARP_CASE(512, 0) GX_WARP_CASE(1024, 0)
    GX_WARP_CASE(128, 1) GX_WARP_CASE(256, 1) GX_WARP_CASE(512, 1) GX_WARP_CASE(1024, 1)
#undef GX_WARP_CASE
  }
  {
    cudaError_t e = smem_opt_in((const void *)fstep_cta_kernel, sm);
    if (e != cudaSuccess) return e;
    const int bpc = 2;
    dim3 grid((nblk + bpc - 1) / bpc, J.nstations);
    fstep_cta_kernel<<<grid, kFThreads, sm, st>>>(J, stations, S, bp, nblk, bpc, nslots, spec);
  }
  return cudaGetLastError();
}

}  // namespace gx
