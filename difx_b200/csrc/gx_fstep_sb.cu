// Station-block F-step: one group of F / 16 threads per (station, FFT block)
// transforms every recorded band of that block.
//
// The per-band kernels read each band's bit field of every VDIF time sample
// with its own gather, so a time sample of B bands crosses from L2 B times,
// and they build the fringe rotator once per band although both
// polarisations of a frequency share it.  Here a group
//   1. computes the rotator tables of every local frequency of the station
//      once (fringe: mode.cpp:882-955; fractional sample: mode.cpp:1029-1122),
//   2. reads each of its time samples once, CHB bytes at a time with one
//      coalesced load per time sample (consecutive threads, consecutive time
//      samples), into registers,
//   3. for every band held in those bytes: decodes its field through the
//      shared-memory level table (format_vdif.c:66-146), rotates
//      (mode.cpp:1160-1183), transforms (16 points per thread, radix-16
//      passes of gx_fft16.h with twiddle rows read from a contiguous table),
//      selects the sideband, applies the fractional-sample correction
//      (mode.cpp:1185-1261) and writes the channels with coalesced stores.
// Frames a block spans are checked against the block's validity mask only
// when one of them is invalid (samples of invalid frames decode to zero and
// are not read).  Jobs outside this kernel's domain (other transform
// lengths, a non-default array stride, quadratic fringe rotation,
// INTERLACEDVDIF, time samples that are not whole bytes) use the per-band
// kernels of gx_fstep.cu.
#include <cstdint>
#include "gx_dev.h"
#include "gx_fcommon.cuh"
#include "gx_fft16.h"

namespace gx {

cudaError_t smem_opt_in(const void *kernel, size_t bytes);

namespace sb {

// Array stride the reference derives from a channel count when the .input
// leaves it 0 (calcstridelength, configuration.cpp:37-50).
__host__ __device__ constexpr int default_stride(int n)
{
  if (n <= 16) return n;
  int g = 1;
  while ((g + 1) * (g + 1) <= n) g++;
  while (n % g != 0) g--;
  return n / g;
}

__host__ __device__ constexpr int ilog2(int x) { return x <= 1 ? 0 : 1 + ilog2(x >> 1); }

template <int F, int CPLX, int CHB>
struct Cfg {
  static constexpr int NT = F / 16;                    // threads per transform
  static constexpr int CTA = NT >= 256 ? NT : 256;
  static constexpr int G = CTA / NT;                   // groups (items in flight) per CTA
  static constexpr int N = CPLX ? F : F / 2;           // channels
  static constexpr int S = default_stride(N);          // rotator stride
  static constexpr int LGS = ilog2(S);
  static constexpr int NFR = F / S;                    // fringe steps
  static constexpr int HALF = N / S;                   // fractional-sample steps
  static constexpr int JSTEP = NT / S;                 // rotator step index advance per register
  static constexpr int MINB = CTA == 256 ? 2 : 1;      // resident CTAs per SM the registers are sized for
  static_assert((S & (S - 1)) == 0 && NT % S == 0, "the stride must be a power of two dividing F / 16");
};

template <int CHB>
struct RawWord { using T = uint32_t; };
template <>
struct RawWord<8> { using T = uint2; };

// CHB bytes at p: one load when p is aligned, bytes otherwise.
template <int CHB>
__device__ __forceinline__ typename RawWord<CHB>::T load_raw(const uint8_t *p, bool aligned)
{
  if constexpr (CHB == 8) {
    if (aligned) return __ldg(reinterpret_cast<const uint2 *>(p));
    uint2 w = make_uint2(0u, 0u);
#pragma unroll
    for (int b = 0; b < 4; b++) {
      w.x |= (uint32_t)__ldg(p + b) << (8 * b);
      w.y |= (uint32_t)__ldg(p + 4 + b) << (8 * b);
    }
    return w;
  } else {
    if (aligned) {
      if constexpr (CHB == 4) return __ldg(reinterpret_cast<const uint32_t *>(p));
      else if constexpr (CHB == 2) return (uint32_t)__ldg(reinterpret_cast<const unsigned short *>(p));
      else return (uint32_t)__ldg(p);
    }
    uint32_t w = 0u;
#pragma unroll
    for (int b = 0; b < CHB; b++) w |= (uint32_t)__ldg(p + b) << (8 * b);
    return w;
  }
}

template <int CHB>
__device__ __forceinline__ uint32_t pick_word(const typename RawWord<CHB>::T &w, int hi)
{
  if constexpr (CHB == 8) return hi ? w.y : w.x;
  else return w;
}

// Radix-16 pass of stride Ns > 1 with its twiddle row from the table section
// at `sec` (entry (r - 1) Ns + m), then the 16-point transform.
template <int F>
__device__ __forceinline__ void pass16_tab(float2 (&v)[16], int j, int Ns, const float2 *__restrict__ sec)
{
  const float2 *row = sec + (j & (Ns - 1));
#pragma unroll
  for (int r = 1; r < 16; r++) v[r] = r16::mul(v[r], __ldg(row + (r - 1) * Ns));
  r16::dft16(v);
}

// Final radix-R0 pass (stride F / R0) with twiddles from the final section
// (entry (r - 1) (F / R0) + g, g = j + NT mm).
template <int F, int R0>
__device__ __forceinline__ void final_pass_tab(float2 (&v)[16], int j, const float2 *__restrict__ sec)
{
  constexpr int M = 16 / R0, NT = F / 16, FR = F / R0;
  const float2 *row = sec + j;
#pragma unroll
  for (int mm = 0; mm < M; mm++) {
    float2 u[R0];
#pragma unroll
    for (int r = 0; r < R0; r++) u[r] = (r == 0) ? v[mm] : r16::mul(v[mm + M * r], __ldg(row + (r - 1) * FR + NT * mm));
    if constexpr (R0 == 2) r16::dft2(u[0], u[1]);
    else if constexpr (R0 == 4) r16::dft4(u[0], u[1], u[2], u[3]);
    else r16::dft8(u);
#pragma unroll
    for (int r = 0; r < R0; r++) v[mm + M * r] = u[r];
  }
}

// Forward transform of the group's F points (16 per thread): register t ends
// holding bin j + NT t.
template <int F, int CTA>
__device__ __forceinline__ void fft(float2 (&v)[16], int j, int g, float2 *xb, const float2 *__restrict__ tw)
{
  using Pl = r16::Plan<F>;
  constexpr int NT = Pl::NT;
  r16::dft16(v);   // stride-1 pass: no twiddles
#pragma unroll
  for (int p = 1; p < Pl::L; p++) {
    const int Ns = r16::pow16(p - 1);
    group_sync<NT, CTA>(g);
    r16::store16(v, j, Ns, xb);
    group_sync<NT, CTA>(g);
    r16::load16<F>(v, j, xb);
    pass16_tab<F>(v, j, r16::pow16(p), tw + r16::tw_pass_offset(F, p));
  }
  if constexpr (Pl::R0 > 1) {
    // the last radix-16 pass leaves its outputs for a pass of stride F / R0
    group_sync<NT, CTA>(g);
    r16::store16(v, j, r16::pow16(Pl::L - 1), xb);
    group_sync<NT, CTA>(g);
    r16::load16<F>(v, j, xb);
    final_pass_tab<F, Pl::R0>(v, j, tw + r16::tw_final_offset(F));
  }
}

template <int F, int CPLX, int CHB>
__global__ void __launch_bounds__(Cfg<F, CPLX, CHB>::CTA, Cfg<F, CPLX, CHB>::MINB)
fstep_sb_kernel(DevJob J, const DevStation *__restrict__ stations, SubintArrays S, const BlockParam *__restrict__ bp,
                int nblk, int blocks_per_cta, int tabstride, float2 *__restrict__ spec)
{
  using C = Cfg<F, CPLX, CHB>;
  using Pl = r16::Plan<F>;
  constexpr int NT = C::NT, CTA = C::CTA, G = C::G, N = C::N, SD = C::S, LGS = C::LGS, NFR = C::NFR,
                HALF = C::HALF;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ float s_lut[256];
  const int s = blockIdx.y;
  const int tid = threadIdx.x, g = tid / NT, j = tid % NT;
  const DevStation &st = stations[s];
  for (int i = tid; i < 256; i += CTA) s_lut[i] = J.lut[i];
  __syncthreads();

  float2 *xb = reinterpret_cast<float2 *>(smem_raw) + (size_t)g * (Pl::SMEM + tabstride);
  float2 *tab = xb + Pl::SMEM;
  const int nlf = st.nrecfreqs, nps = st.deltapol ? 2 : 1;
  const int lfstride = SD + NFR + nps * (SD + HALF);
  const float2 *__restrict__ tw = J.twiddle;

  const uint8_t *data = S.data[s];
  const int fsamp = J.framesamples, fbytes = J.framebytes;
  const int bpts = J.bps_num / J.bps_den;                  // bytes per time sample (whole bytes here)
  const int nchunk = bpts / CHB, bpc = J.nbands / nchunk;  // chunks of CHB bytes; bands per chunk
  const int fbits = J.nbits * (CPLX ? 2 : 1);
  const uint32_t cmask = (1u << J.nbits) - 1u;
  const bool aligned = ((reinterpret_cast<uintptr_t>(data) | (uintptr_t)fbytes | (uintptr_t)bpts) & (CHB - 1)) == 0;

  const int b0 = blockIdx.x * blocks_per_cta;
  const int nbk = min(blocks_per_cta, nblk - b0);
  for (int it = g; it < nbk; it += G) {
    const int bi = b0 + it;
    const BlockParam P = bp[(size_t)s * nblk + bi];
    if (P.state == 0) {
      for (int bd = 0; bd < J.nbands; bd++) {
        const int f = st.freq_index[st.band_localfreq[bd]];
        float2 *dst = spec + (((size_t)f * nblk + bi) * J.ninputs + st.band_input[bd]) * N;
        for (int c = j; c < N; c += NT) dst[c] = make_float2(0.f, 0.f);
      }
      continue;
    }
    group_sync<NT, CTA>(g);   // the previous item is done with the tables and the exchange buffer
    for (int lf = 0; lf < nlf; lf++) {
      float2 *tl = tab + lf * lfstride;
      for (int e = j; e < SD + NFR; e += NT) tl[e] = fringe_entry(J, st, lf, e, P);
      for (int ps = 0; ps < nps; ps++)
        for (int e = j; e < SD + HALF; e += NT) tl[SD + NFR + ps * (SD + HALF) + e] = frac_entry(J, st, lf, ps, e, P);
    }
    group_sync<NT, CTA>(g);

    const bool allvalid = P.nframes >= 64 ? P.validmask == ~0ull : P.validmask == ((1ull << P.nframes) - 1ull);
    int q0, r0;
    {
      const int smp0 = P.nearestsample + j;
      q0 = smp0 / fsamp;
      r0 = smp0 - q0 * fsamp;
      q0 -= P.fr0;
    }
    for (int ch = 0; ch < nchunk; ch++) {
      // time samples j + NT t of this chunk's bytes; NT <= samples per frame, so
      // a step crosses at most one frame boundary
      typename RawWord<CHB>::T raw[16];
      unsigned int vmask = 0xFFFFu;
      {
        int q = q0, r = r0;
        const uint8_t *fr = data + ((long long)P.fr0 + q) * fbytes + 32 + ch * CHB;
        bool ok = allvalid || ((P.validmask >> q) & 1ull);
#pragma unroll
        for (int t = 0; t < 16; t++) {
          if (ok) raw[t] = load_raw<CHB>(fr + r * bpts, aligned);
          else {
            raw[t] = typename RawWord<CHB>::T{};
            vmask &= ~(1u << t);
          }
          r += NT;
          if (r >= fsamp) {
            r -= fsamp;
            q++;
            fr += fbytes;
            ok = allvalid || (q < 64 && ((P.validmask >> q) & 1ull));
          }
        }
      }
#pragma unroll 1
      for (int kb = 0; kb < bpc; kb++) {
        const int bd = ch * bpc + kb;
        const int bit0 = kb * fbits, hi = bit0 >> 5, sh = bit0 & 31;
        const int lf = st.band_localfreq[bd];
        const float2 *rs = tab + lf * lfstride;
        const float2 *rp = rs + SD;
        const float2 *fs = rp + NFR + (st.band_polb[bd] ? SD + HALF : 0);
        const float2 *fp = fs + SD;
        float2 v[16];
        {
          // decode and fringe-rotate: x[n] sub[n mod S] step[n / S]; S divides NT,
          // so the sub entry is the same for all 16 samples of the thread
          const float2 rsk = rs[j & (SD - 1)];
          const float2 *rpj = rp + (j >> LGS);
#pragma unroll
          for (int t = 0; t < 16; t++) {
            const uint32_t w = pick_word<CHB>(raw[t], hi);
            float2 u;
            u.x = s_lut[(w >> sh) & cmask];
            u.y = CPLX ? s_lut[(w >> (sh + J.nbits)) & cmask] : 0.f;
            const float2 rot = cmul(rsk, rpj[C::JSTEP * t]);
            v[t] = CPLX ? cmul(rot, u) : make_float2(u.x * rot.x, u.x * rot.y);
          }
          if (!allvalid) {
#pragma unroll
            for (int t = 0; t < 16; t++)
              if (!((vmask >> t) & 1u)) v[t] = make_float2(0.f, 0.f);
          }
        }
        fft<F, CTA>(v, j, g, xb, tw);
        // register t holds bin j + NT t: sideband selection, fractional-sample
        // correction sub[c mod S] step[c / S] (c mod S fixed per thread), store
        const int lsb = st.lsb[lf];
        const int f = st.freq_index[lf];
        float2 *drow = spec + (((size_t)f * nblk + bi) * J.ninputs + st.band_input[bd]) * N;
        const float2 fsk = fs[((CPLX && lsb) ? -j : j) & (SD - 1)];
        auto emit = [&](int c, float2 val) { drow[c] = cmul(val, cmul(fsk, fp[c >> LGS])); };
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
  }
}

}  // namespace sb

// Whether the station-block kernel takes this job (see the file comment).
bool fstep_sb_eligible(const DevJob &J, bool interlaced)
{
  const int F = J.fftlen;
  if (F < 512 || F > 8192 || (F & (F - 1))) return false;
  if (J.fringe_order == 2 || interlaced) return false;
  if (J.stride != sb::default_stride(J.nchan)) return false;
  const int bits_ts = J.nbands * J.nbits * (J.cplx ? 2 : 1);
  if (bits_ts % 8 || J.bps_num != bits_ts / 8 * J.bps_den) return false;
  const int bpts = bits_ts / 8;
  const int chb = bpts >= 4 ? 4 : bpts;
  if (bpts < chb || bpts % chb) return false;
  const int nchunk = bpts / chb;
  if (J.nbands % nchunk) return false;
  const int fbits = J.nbits * (J.cplx ? 2 : 1);
  if ((J.nbands / nchunk) * fbits != chb * 8) return false;   // the chunk's bands fill its bytes
  if (F / 16 > J.framesamples) return false;
  if (J.framebytes < 32) return false;
  return true;
}

size_t fstep_sb_smem_bytes(const DevJob &J, int maxnrf, int deltapol)
{
  const int F = J.fftlen, NT = F / 16, G = (NT >= 256 ? NT : 256) / NT;
  const int S = J.stride, nfr = F / S, half = J.nchan / S;
  const int tab = maxnrf * (S + nfr + (deltapol ? 2 : 1) * (S + half));
  return (size_t)G * (F + F / 16 + ((tab + 1) & ~1)) * sizeof(float2);
}

cudaError_t fstep_sb_launch(const DevJob &J, const DevStation *stations, int maxnrf, int deltapol,
                            const SubintArrays &S, int nblk, const BlockParam *bp, float2 *spec, cudaStream_t st)
{
  const int F = J.fftlen, NT = F / 16, G = (NT >= 256 ? NT : 256) / NT;
  const int S_ = J.stride, nfr = F / S_, half = J.nchan / S_;
  const int tab = maxnrf * (S_ + nfr + (deltapol ? 2 : 1) * (S_ + half));
  const int tabstride = (tab + 1) & ~1;
  const size_t sm = fstep_sb_smem_bytes(J, maxnrf, deltapol);
  const int bpts = J.nbands * J.nbits * (J.cplx ? 2 : 1) / 8;
  const int chb = bpts >= 4 ? 4 : bpts;
  const int bpc = 4 * G;   // four items per group
  dim3 grid((nblk + bpc - 1) / bpc, J.nstations);
#define GX_SB_CASE(FLV, CX, CB)                                                                         \
  if (F == FLV && J.cplx == CX && chb == CB) {                                                          \
    using K = sb::Cfg<FLV, CX, CB>;                                                                     \
    cudaError_t e = smem_opt_in((const void *)sb::fstep_sb_kernel<FLV, CX, CB>, sm);                    \
    if (e != cudaSuccess) return e;                                                                     \
    sb::fstep_sb_kernel<FLV, CX, CB><<<grid, K::CTA, sm, st>>>(J, stations, S, bp, nblk, bpc, tabstride, spec); \
    return cudaGetLastError();                                                                          \
  }
  GX_SB_CASE(512, 0, 1) GX_SB_CASE(1024, 0, 1) GX_SB_CASE(2048, 0, 1) GX_SB_CASE(4096, 0, 1) GX_SB_CASE(8192, 0, 1)
  GX_SB_CASE(512, 0, 2) GX_SB_CASE(1024, 0, 2) GX_SB_CASE(2048, 0, 2) GX_SB_CASE(4096, 0, 2) GX_SB_CASE(8192, 0, 2)
  GX_SB_CASE(512, 0, 4) GX_SB_CASE(1024, 0, 4) GX_SB_CASE(2048, 0, 4) GX_SB_CASE(4096, 0, 4) GX_SB_CASE(8192, 0, 4)
  GX_SB_CASE(512, 1, 4) GX_SB_CASE(1024, 1, 4) GX_SB_CASE(2048, 1, 4) GX_SB_CASE(4096, 1, 4) GX_SB_CASE(8192, 1, 4)
#undef GX_SB_CASE
  return cudaErrorNotSupported;
}

}  // namespace gx
