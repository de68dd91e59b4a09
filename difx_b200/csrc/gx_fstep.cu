// F-step: VDIF unpack + validity/weights, FP64 per-block delay evaluation,
// FP32 fringe rotation, shared-memory Stockham FFT, sideband selection and
// fractional-sample correction, writing spectra in the layout the X-step
// reads: spec[freq][block][input][channel] (float2).
//
// One CTA processes a run of consecutive FFT blocks of one station; the
// recorded bands of a block are transformed concurrently in "slots" (one
// FFT per slot, ping-pong buffers in shared memory).
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
#include "gx_dev.h"

namespace gx {

#define GX_TWO_PI 6.283185307179586476925286766559

struct BlockParams {
  int state;             // 0 zero block, 1 process
  int nearestsample;
  int fr0, nframes;
  int integerdelay;
  int intwalltime;
  float fracsampleerror;
  float weight;
  double a, b;
  double fracwalltime;
  int good;
};

__device__ __forceinline__ float2 cmul_exact(float2 a, float2 b)
{
  // no contraction: same rounding as the reference's separate multiplies/adds
  float2 r;
  r.x = __fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y));
  r.y = __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x));
  return r;
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

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

// One Stockham radix-R pass over one slot's buffer: in -> out.
template <int R>
__device__ __forceinline__ void stockham_pass(const float2 *in, float2 *out, int F, int Ns,
                                              const float2 *tw, int lt, int nt)
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

// Whole forward FFT of one slot (bufA holds the input); returns the buffer holding the result.
__device__ float2 *slot_fft(float2 *bufA, float2 *bufB, int F, const float2 *tw, int lt, int nt,
                            int slot_threads_first, int nslots_active)
{
  float2 *in = bufA, *out = bufB;
  int Ns = 1;
  while (Ns < F) {
    int R = (Ns * 8 <= F) ? 8 : ((Ns * 4 <= F) ? 4 : 2);
    if (lt >= 0) {
      if (R == 8) stockham_pass<8>(in, out, F, Ns, tw, lt, nt);
      else if (R == 4) stockham_pass<4>(in, out, F, Ns, tw, lt, nt);
      else stockham_pass<2>(in, out, F, Ns, tw, lt, nt);
    }
    __syncthreads();
    float2 *t = in; in = out; out = t;
    Ns *= R;
  }
  return in;
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

__global__ void __launch_bounds__(kFThreads)
fstep_kernel(DevJob J, const DevStation *__restrict__ stations, SubintArrays S,
             int blk0, int nblk, int blocks_per_cta, int nslots,
             float2 *__restrict__ spec, float *__restrict__ weights)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int s = blockIdx.y;
  const int tid = threadIdx.x;
  const DevStation &st = stations[s];
  const int F = J.fftlen, N = J.nchan, Sd = J.stride, nfr = J.nfr, half = J.half;
  const int nrf = st.nrecfreqs;

  // shared memory carve-up
  float2 *slotbuf = reinterpret_cast<float2 *>(smem_raw);                 // nslots * 2F
  float2 *rsub = slotbuf + (size_t)nslots * 2 * F;                        // nrf * S
  float2 *rstep = rsub + nrf * Sd;                                         // nrf * nfr
  float2 *fsub = rstep + nrf * nfr;                                        // 2 * nrf * S
  float2 *fstep = fsub + 2 * nrf * Sd;                                     // 2 * nrf * half
  int *fvalid = reinterpret_cast<int *>(fstep + 2 * nrf * (half > 0 ? half : 1));  // kMaxFramesPerBlock
  __shared__ BlockParams P;
  __shared__ int good_acc;
  __shared__ float s_lut[256];   // decode table

  const int tps = kFThreads / nslots;
  const int myslot = tid / tps;
  const int lt = (myslot < nslots) ? (tid % tps) : -1;

  const uint8_t *data = S.data[s];
  const int64_t datalen = S.datalen[s];
  const int32_t *ctrl = S.control + (size_t)s * S.controlstride;
  const double *ip = S.interp + 3 * s;
  for (int i = tid; i < 256; i += blockDim.x) s_lut[i] = J.lut[i];
  __syncthreads();

  for (int bi = blockIdx.x * blocks_per_cta; bi < min(nblk, (blockIdx.x + 1) * blocks_per_cta); bi++) {
    const int blk = blk0 + bi;
    if (tid == 0) {
      P.state = 0;
      P.weight = 0.0f;
      good_acc = 0;
      const int datasec = ctrl[1], datans = ctrl[2];
      const int flagword = ctrl[3 + blk / 30];
      if (datalen > 1 && ((flagword >> (blk % 30)) & 1) != 0) {
        const double fftcentre = blk + 0.5;
        const double averagedelay = ip[0] * fftcentre * fftcentre + ip[1] * fftcentre + ip[2];
        const double fftstartmicrosec = (blk * F) * J.sampletime;
        const double starttime = (S.sec - datasec) * 1000000.0 +
                                 ((long long)S.ns - (long long)datans) / 1000.0 + fftstartmicrosec - averagedelay;
        int ns = (int)(starttime / J.sampletime + 0.5);
        const double walltimesecs = (double)((long long)S.scan_start_sec + S.sec) + S.ns / 1.0e9 +
                                    fftstartmicrosec / 1.0e6;
        P.intwalltime = (int)walltimesecs;
        P.fracwalltime = walltimesecs - P.intwalltime;
        if (!(ns < -1 || (long long)(ns + F) * J.bytespersample > datalen)) {
          if (ns == -1) ns = 0;
          P.nearestsample = ns;
          P.fr0 = ns / J.framesamples;
          P.nframes = (ns + J.unpacksamples - 1) / J.framesamples - P.fr0 + 1;
          if (P.nframes <= kMaxFramesPerBlock) {
            P.state = 1;
            P.fracsampleerror = (float)(starttime - ns * J.sampletime);
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
          }
        }
      }
    }
    __syncthreads();
    if (P.state == 1) {
      // frame validity and good-sample count
      for (int q = tid; q < P.nframes; q += blockDim.x) {
        const long long fr = (long long)P.fr0 + q;
        int ok = 0;
        if ((fr + 1) * J.framebytes <= datalen)
          ok = frame_ok(data + fr * J.framebytes, J.framebytes, !(J.cplx && q == 0));
        fvalid[q] = ok;
        if (ok) {
          const long long lo = max((long long)P.nearestsample, fr * J.framesamples);
          const long long hi = min((long long)P.nearestsample + J.unpacksamples, (fr + 1) * J.framesamples);
          atomicAdd(&good_acc, (int)(hi - lo));
        }
      }
      __syncthreads();
      if (tid == 0) {
        P.good = good_acc;
        P.weight = (float)good_acc / (float)J.unpacksamples;
        if (!(P.weight > 0.0f)) P.state = 0;
      }
      __syncthreads();
    }
    if (P.state == 0) {
      // zeroed block (mode.cpp:656-669, 688-701, 743-754)
      for (int bd = 0; bd < J.nbands; bd++) {
        const int lf = st.band_localfreq[bd];
        const int f = st.freq_index[lf];
        float2 *dst = spec + (((size_t)f * nblk + bi) * J.ninputs + st.band_input[bd]) * N;
        for (int c = tid; c < N; c += blockDim.x) dst[c] = make_float2(0.f, 0.f);
      }
      if (tid == 0) weights[(size_t)s * nblk + bi] = 0.0f;
      __syncthreads();
      continue;
    }

    // fringe-rotator and fractional-sample tables for every recorded freq (FP64 phases -> FP32 sincos)
    for (int idx = tid; idx < nrf * (Sd + nfr); idx += blockDim.x) {
      const int fi = idx / (Sd + nfr);
      const int e = idx % (Sd + nfr);
      const double lofreq = st.lofreq[fi];
      const double looffset = st.looff[fi];
      const bool looff = (looffset > 0.0 || looffset < 0.0);
      double ph;
      if (e < Sd) {
        const int k = e;
        double x = ((double)k / (double)F) * P.a;
        x += P.b;
        ph = x * lofreq;
        if (st.fractional_lo) ph += (lofreq - (int)lofreq) * (double)P.integerdelay;
        if (looff) {
          ph += ((k * J.sampletime) / 1e6) * -looffset;
          ph += -looffset * P.fracwalltime;
          double fl = fabs(looffset) - (int)fabs(looffset);
          const bool isfrac = fl > (double)0.000000001f;
          if (looffset < 0) fl = -fl;
          if (isfrac) ph += -fl * P.intwalltime;
        }
        const float arg = (float)(-GX_TWO_PI * (ph - (int)ph));
        float sn, cs;
        sincosf(arg, &sn, &cs);
        rsub[fi * Sd + k] = make_float2(cs, sn);
      } else {
        const int j = e - Sd;
        const double x = ((double)(j * Sd) / (double)F) * P.a;
        ph = x * lofreq;
        if (looff) ph += ((j * Sd * J.sampletime) / 1e6) * -looffset;
        const float arg = (float)(-GX_TWO_PI * (ph - (int)ph));
        float sn, cs;
        sincosf(arg, &sn, &cs);
        rstep[fi * nfr + j] = make_float2(cs, sn);
      }
    }
    const int npolsets = st.deltapol ? 2 : 1;
    for (int idx = tid; idx < npolsets * nrf * (Sd + half); idx += blockDim.x) {
      const int ps = idx / (nrf * (Sd + half));
      const int r = idx % (nrf * (Sd + half));
      const int fi = r / (Sd + half);
      const int e = r % (Sd + half);
      const double sgn = ps == 0 ? 1.0 : -1.0;
      const float val = (float)((double)P.fracsampleerror - st.clk[fi] + sgn * st.clkdelta[fi] / 2);
      float cfreq;
      if (e < Sd) {
        cfreq = (float)((GX_TWO_PI * (e) * J.bw) / N);
      } else {
        const int j = e - Sd;
        cfreq = st.lsb[fi] ? (float)((-GX_TWO_PI * ((half - j) * Sd) * J.bw) / N)
                           : (float)((GX_TWO_PI * j * Sd * J.bw) / N);
      }
      const float arg = __fmul_rn(cfreq, val);
      float sn, cs;
      sincosf(arg, &sn, &cs);
      if (e < Sd) fsub[(ps * nrf + fi) * Sd + e] = make_float2(cs, sn);
      else fstep[(ps * nrf + fi) * half + (e - Sd)] = make_float2(cs, sn);
    }
    __syncthreads();

    // bands in waves of nslots concurrent FFTs
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
        const int sub = J.cplx ? 2 : 1;
        const int bits_per_ts = J.nbands * J.nbits * sub;
        const int mask = (1 << J.nbits) - 1;
        for (int n = lt; n < F; n += tps) {
          const int smp = P.nearestsample + n;
          const int q = smp / J.framesamples - P.fr0;
          float2 u = make_float2(0.f, 0.f);
          if (fvalid[q]) {
            const uint8_t *payload = data + ((long long)P.fr0 + q) * J.framebytes + 32;
            const long long bit0 = (long long)(smp % J.framesamples) * bits_per_ts + (long long)bd * sub * J.nbits;
            const int c0 = (payload[bit0 >> 3] >> (bit0 & 7)) & mask;
            u.x = s_lut[c0];
            if (J.cplx) {
              const long long bit1 = bit0 + J.nbits;
              const int c1 = (payload[bit1 >> 3] >> (bit1 & 7)) & mask;
              u.y = s_lut[c1];
            }
          }
          const int k = n % Sd, j = n / Sd;
          const float2 rot = (j == 0) ? rs[k] : cmul_exact(rs[k], rp[j]);
          float2 v;
          if (J.cplx) v = cmul(rot, u);
          else v = make_float2(u.x * rot.x, u.x * rot.y);
          bufA[n] = v;
        }
      }
      __syncthreads();
      float2 *res = slot_fft(bufA, bufB, F, J.twiddle, active ? lt : -1, tps, 0, nslots);
      if (active) {
        const int f = st.freq_index[lf];
        const int lsb = st.lsb[lf];
        const int ps = st.band_polb[bd] ? 1 : 0;
        const float2 *fs = fsub + (ps * nrf + lf) * Sd;
        const float2 *fp = fstep + (ps * nrf + lf) * half;
        float2 *dst = spec + (((size_t)f * nblk + bi) * J.ninputs + st.band_input[bd]) * N;
        for (int c = lt; c < N; c += tps) {
          float2 v;
          if (!J.cplx) {
            v = res[lsb ? N + c : c];
          } else if (!lsb) {
            v = res[c];
          } else {
            v = (c == 0) ? res[0] : res[F - c];
            if (c != 0) v.y = -v.y;
          }
          const float2 fr = cmul_exact(fs[c % Sd], fp[c / Sd]);
          dst[c] = cmul(v, fr);
        }
      }
      __syncthreads();
    }
    if (tid == 0) weights[(size_t)s * nblk + bi] = P.weight;
    __syncthreads();
  }
}

size_t fstep_smem_bytes(const DevJob &J, int nrf, int nslots)
{
  size_t b = (size_t)nslots * 2 * J.fftlen * sizeof(float2);
  b += (size_t)nrf * (J.stride + J.nfr) * sizeof(float2);
  b += (size_t)2 * nrf * (J.stride + (J.half > 0 ? J.half : 1)) * sizeof(float2);
  b += kMaxFramesPerBlock * sizeof(int);
  return b;
}

cudaError_t fstep_launch(const DevJob &J, const DevStation *stations, int maxnrf, const SubintArrays &S,
                         int blk0, int nblk, int nslots, float2 *spec, float *weights, cudaStream_t st)
{
  const int bpc = 4;
  dim3 grid((nblk + bpc - 1) / bpc, J.nstations);
  size_t sm = fstep_smem_bytes(J, maxnrf, nslots);
  // opt in to the dynamic shared memory this launch needs (the kernel's
  // static shared memory counts against the same 227 KB per block)
  static size_t attr_bytes = 48 * 1024;
  if (sm > attr_bytes) {
    cudaError_t e = cudaFuncSetAttribute(fstep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    attr_bytes = sm;
  }
  fstep_kernel<<<grid, kFThreads, sm, st>>>(J, stations, S, blk0, nblk, bpc, nslots, spec, weights);
  return cudaGetLastError();
}

}  // namespace gx
