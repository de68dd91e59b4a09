// Station-block F-step: one group of F / 16 threads per (station, FFT block)
// transforms every recorded band of that block.
//
// The per-band kernels read each band's bit field of every VDIF time sample
// with its own gather, so a time sample of B bands crosses from L2 B times,
// and they build the fringe rotator once per band although both
// polarisations of a frequency share it.  Here a group
//   1. stages the block's time samples into shared memory with 16-byte
//      asynchronous copies (frame headers skipped; consecutive threads copy
//      consecutive pieces), so the VDIF crosses from L2 once,
//   2. meanwhile computes the rotator tables of every local frequency of the
//      station once (fringe: mode.cpp:882-955; fractional sample:
//      mode.cpp:1029-1122),
//   3. for every band: decodes its field of the staged samples (8-bit codes
//      by an exact two-term FMA, other widths through the shared-memory level
//      table; format_vdif.c:66-146), rotates
//      (mode.cpp:1160-1183), transforms (16 points per thread, radix-16
//      passes of gx_fft16.h with the twiddle rows of the stride-16 and
//      stride-256 passes in shared memory),
//      selects the sideband, applies the fractional-sample correction
//      (mode.cpp:1185-1261) and writes the channels with coalesced stores;
//   4. with phase-cal (PC, gx::PcalFuse), also adds the decoded samples of
//      each band into their phase-cal bins (mode.cpp:759-774; the
//      implicit-shift extractors of pcal.cpp:1032-1222 and 1419-1600), so
//      the samples are not read and decoded a second time.
// Frames a block spans are checked against the block's validity mask only
// when one of them is invalid (samples of invalid frames decode to zero and
// are not read).  Jobs outside this kernel's domain (other transform
// lengths, a non-default array stride, quadratic fringe rotation,
// INTERLACEDVDIF, frames whose payload is not a whole number of 16-byte
// pieces, time samples that are not whole bytes) use the per-band kernels of
// gx_fstep.cu.
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

template <int F, int CPLX, int BPTS>
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
  static constexpr int RAWB = F * BPTS + 32;           // staged time samples (16-byte rounding at both ends)
  // two resident CTAs per SM: 128 registers a thread up to 4096 points, 64 at 8192
  static constexpr int MINB = 2;
  static_assert((S & (S - 1)) == 0 && NT % S == 0, "the stride must be a power of two dividing F / 16");
};

// 16-byte copy global -> shared that completes asynchronously (cp.async, L2 only).
__device__ __forceinline__ void cp_async16(void *sdst, const void *gsrc)
{
  const unsigned int d = (unsigned int)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
// Waits for this thread's outstanding cp.async copies.
__device__ __forceinline__ void cp_async_wait_all()
{
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
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

// Twiddle rows of the radix-16 passes held in shared memory, 15 x 16 entries
// each, entry (r - 1) 16 + m:
//   A: W_256^(r m)  -- the stride-16 pass's whole table,
//   B: W_4096^(r m) -- the low digit of the stride-256 pass, whose twiddle
//      W_4096^(r m) for m < 256 is B[r][m mod 16] A[r][m / 16].
// The full stride-256 table (3840 entries, 30 KB) is larger than what L1 keeps
// beside two CTAs' shared memory, so reading it per pass went to L2.
constexpr int kTwRow = 16 * 15;

// Fills A and B from the device twiddle table (group-independent; the caller
// synchronises before the first transform).
template <int F>
__device__ __forceinline__ void load_tw_rows(float2 *twA, float2 *twB, const float2 *__restrict__ tw, int tid, int nthr)
{
  using Pl = r16::Plan<F>;
  const float2 *s1 = tw + r16::tw_pass_offset(F, 1);
  for (int i = tid; i < kTwRow; i += nthr) twA[i] = s1[i];
  if constexpr (Pl::L >= 3) {
    const float2 *s2 = tw + r16::tw_pass_offset(F, 2);
    for (int i = tid; i < kTwRow; i += nthr) twB[i] = s2[(i >> 4) * 256 + (i & 15)];
  }
}

// Radix-16 pass of stride 16 (p = 1) or 256 (p = 2) with twiddles from the rows.
template <int P>
__device__ __forceinline__ void pass16_rows(float2 (&v)[16], int j, const float2 *twA, const float2 *twB)
{
  if constexpr (P == 1) {
    const float2 *a = twA + (j & 15);
#pragma unroll
    for (int r = 1; r < 16; r++) v[r] = r16::mul(v[r], a[(r - 1) * 16]);
  } else {
    const float2 *a = twA + ((j >> 4) & 15);
    const float2 *b = twB + (j & 15);
#pragma unroll
    for (int r = 1; r < 16; r++) v[r] = r16::mul(v[r], r16::mul(b[(r - 1) * 16], a[(r - 1) * 16]));
  }
  r16::dft16(v);
}

// Forward transform of the group's F points (16 per thread): register t ends
// holding bin j + NT t.  `mid` runs once, after the group's first barrier
// (everything the group wrote to shared memory before the call is visible).
template <int F, int CTA, typename Mid>
__device__ __forceinline__ void fft(float2 (&v)[16], int j, int g, float2 *xb, const float2 *__restrict__ tw,
                                    const float2 *twA, const float2 *twB, Mid &&mid)
{
  using Pl = r16::Plan<F>;
  constexpr int NT = Pl::NT;
  static_assert(Pl::L <= 3, "shared twiddle rows cover strides 16 and 256");
  r16::dft16(v);   // stride-1 pass: no twiddles
#pragma unroll
  for (int p = 1; p < Pl::L; p++) {
    const int Ns = r16::pow16(p - 1);
    group_sync<NT, CTA>(g);
    if (p == 1) mid();
    r16::store16(v, j, Ns, xb);
    group_sync<NT, CTA>(g);
    r16::load16<F>(v, j, xb);
    if (p == 1) pass16_rows<1>(v, j, twA, twB);
    else pass16_rows<2>(v, j, twA, twB);
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

// Pad slot of thread j in the exchange buffer: position 17 k + 16 is never an
// element (pad(i) = i + i / 16 skips it), so a thread's phase-cal sum parks
// there while the transform uses the buffer.
__device__ __forceinline__ int pc_slot(int j) { return 17 * j + 16; }

template <int F, int CPLX, int BPTS, bool PC>
__global__ void __launch_bounds__(Cfg<F, CPLX, BPTS>::CTA, Cfg<F, CPLX, BPTS>::MINB)
fstep_sb_kernel(DevJob J, const DevStation *__restrict__ stations, SubintArrays S, const BlockParam *__restrict__ bp,
                int nblk, int blocks_per_cta, int tabstride, float2 *__restrict__ spec, PcalFuse pf)
{
  using C = Cfg<F, CPLX, BPTS>;
  using Pl = r16::Plan<F>;
  constexpr int NT = C::NT, CTA = C::CTA, G = C::G, N = C::N, SD = C::S, LGS = C::LGS, NFR = C::NFR,
                HALF = C::HALF, JSTEP = C::JSTEP;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ float s_lut[256];
  const int s = blockIdx.y;
  const int tid = threadIdx.x, g = tid / NT, j = tid % NT;
  const DevStation &st = stations[s];
  // CTA-wide twiddle rows, then per group: exchange buffer, rotator tables,
  // staged time samples
  float2 *twA = reinterpret_cast<float2 *>(smem_raw);
  float2 *twB = twA + kTwRow;
  for (int i = tid; i < 256; i += CTA) s_lut[i] = J.lut[i];
  load_tw_rows<F>(twA, twB, J.twiddle, tid, CTA);
  __syncthreads();

  float2 *xb = reinterpret_cast<float2 *>(smem_raw + 2 * kTwRow * sizeof(float2) +
                                          (size_t)g * ((Pl::SMEM + tabstride) * sizeof(float2) + C::RAWB));
  float2 *tab = xb + Pl::SMEM;
  unsigned char *raw = reinterpret_cast<unsigned char *>(tab + tabstride);
  const int nlf = st.nrecfreqs, nps = st.deltapol ? 2 : 1;
  const int lfstride = SD + NFR + nps * (SD + HALF);
  const float2 *__restrict__ tw = J.twiddle;

  const uint8_t *data = S.data[s];
  const int fsamp = J.framesamples, fbytes = J.framebytes, paybytes = fsamp * BPTS;
  const int fbits = J.nbits * (CPLX ? 2 : 1);
  const uint32_t cmask = (1u << J.nbits) - 1u;
  // 16-byte copies need a 16-byte aligned buffer (the frame layout is checked on the host)
  const bool aligned = (reinterpret_cast<uintptr_t>(data) & 15) == 0;
  // phase-cal (PC): this station's first band in the phase-cal list, the
  // absolute sample number of the subint start (as the binning kernels form
  // it) and this group's slot of partial sums
  const int pcfirst = PC ? pf.first[s] : -1;
  unsigned long long pcs0 = 0;
  if (PC && pcfirst >= 0) {
    const int32_t *ctrl = S.control + (size_t)s * S.controlstride;
    pcs0 = (unsigned long long)(((double)ctrl[1] * 1e9 + (double)ctrl[2]) / (J.sampletime * 1e3) + 0.5);
  }
  float2 *pcout = PC && pcfirst >= 0
                      ? pf.partial + ((size_t)(blockIdx.x * G + g) * pf.nbands_total + pcfirst) * pf.maxbins
                      : nullptr;

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
    const bool allvalid = P.nframes >= 64 ? P.validmask == ~0ull : P.validmask == ((1ull << P.nframes) - 1ull);
    group_sync<NT, CTA>(g);   // the previous item is done with the tables, samples and exchange buffer
    // Stage the block's time samples: payload bytes [p0, pend) of the frames,
    // headers skipped, in 16-byte pieces (a payload is whole pieces, so none
    // straddles a frame); pieces of invalid frames are not read.
    const long long pstart = (long long)P.nearestsample * BPTS;
    const long long p0 = pstart & ~15ll;
    const int off0 = (int)(pstart - p0);   // staged position of the block's first time sample
    const int npieces = (int)(((((long long)(P.nearestsample + F) * BPTS + 15) & ~15ll) - p0) >> 4);
    {
      const long long pos = p0 + 16 * j;
      int q = (int)(pos / paybytes);
      int within = (int)(pos - (long long)q * paybytes);
      for (int k = j; k < npieces; k += NT) {
        if (allvalid || ((P.validmask >> (q - P.fr0)) & 1ull)) {
          const uint8_t *src = data + (long long)q * fbytes + 32 + within;
          if (aligned) {
            cp_async16(raw + 16 * k, src);
          } else {
#pragma unroll
            for (int b = 0; b < 16; b++) raw[16 * k + b] = __ldg(src + b);
          }
        }
        within += 16 * NT;
        while (within >= paybytes) {
          within -= paybytes;
          q++;
        }
      }
    }
    // rotator tables of every local frequency while the copies are in flight
    for (int lf = 0; lf < nlf; lf++) {
      float2 *tl = tab + lf * lfstride;
      for (int e = j; e < SD + NFR; e += NT) tl[e] = fringe_entry(J, st, lf, e, P);
      for (int ps = 0; ps < nps; ps++)
        for (int e = j; e < SD + HALF; e += NT) tl[SD + NFR + ps * (SD + HALF) + e] = frac_entry(J, st, lf, ps, e, P);
    }
    cp_async_wait_all();
    group_sync<NT, CTA>(g);

    // samples j + NT t of invalid frames decode to zero
    unsigned int vmask = 0xFFFFu;
    if (!allvalid) {
      const int smp0 = P.nearestsample + j;
      int q = smp0 / fsamp, r = smp0 - q * fsamp;
      q -= P.fr0;
#pragma unroll
      for (int t = 0; t < 16; t++) {
        if (!((P.validmask >> q) & 1ull)) vmask &= ~(1u << t);
        r += NT;
        while (r >= fsamp) {
          r -= fsamp;
          q++;
        }
        if (q > 63) q = 63;
      }
    }
    const unsigned char *rj = raw + off0 + j * BPTS;   // time sample j of the block
    uint32_t wpair[16];   // 8-bit complex: the words of the current band pair
    // phase-cal: sample n of the block is absolute sample pcs0 + nearestsample + n,
    // bin (that) mod nbins; nbins divides NT, so thread j's samples j + NT t
    // all fall in bin pcbin, and threads j < nbins own one bin each
    const int pcn = PC ? pf.nbins : 1;
    const int pcbin = PC ? (int)((pcs0 + (unsigned long long)P.nearestsample + (unsigned long long)j) %
                                 (unsigned long long)pcn)
                         : 0;
#pragma unroll 1
    for (int bd = 0; bd < J.nbands; bd++) {
      const int bit0 = bd * fbits, sh = bit0 & 7;
      const unsigned char *rb = rj + (bit0 >> 3);
      const int lf = st.band_localfreq[bd];
      const float2 *rs = tab + lf * lfstride;
      const float2 *rp = rs + SD;
      const float2 *fs = rp + NFR + (st.band_polb[bd] ? SD + HALF : 0);
      const float2 *fp = fs + SD;
      float2 v[16];
      float2 ps = make_float2(0.f, 0.f);   // phase-cal: sum of this thread's valid samples
      {
        // decode and fringe-rotate: x[n] sub[n mod S] step[n / S]; S divides NT,
        // so the sub entry is the same for all 16 samples of the thread
        const float2 rsk = rs[j & (SD - 1)];
        const float2 *rpj = rp + (j >> LGS);
        if (CPLX && fbits == 16 && J.lut_affine) {   // 8-bit complex, levels by arithmetic
          // Bands 2k and 2k + 1 share a 4-byte word of the time sample (the
          // complex 8-bit domain has 2, 4 or 8 bands); it is read once for the
          // pair, halving the bank-conflicted reads of the 16-byte-stride samples.
          const unsigned int h = bd & 1;
          if (h == 0) {
#pragma unroll
            for (int t = 0; t < 16; t++) wpair[t] = *reinterpret_cast<const uint32_t *>(rb + NT * BPTS * t);
          }
          const unsigned int sre = 0x7650u + 2u * h, sim = sre + 1u;
          const float bias = J.lut_bias, hi = J.lut_hi, lo = J.lut_lo;
#pragma unroll
          for (int t = 0; t < 16; t++) {
            // code c as the float 2^23 + c (byte placed under the exponent 0x4B)
            const float xr = __uint_as_float(__byte_perm(wpair[t], 0x4B000000u, sre)) - bias;
            const float xi = __uint_as_float(__byte_perm(wpair[t], 0x4B000000u, sim)) - bias;
            const float2 u = make_float2(fmaf(xr, hi, xr * lo), fmaf(xi, hi, xi * lo));
            v[t] = cmul(cmul(rsk, rpj[JSTEP * t]), u);
            if (PC && (allvalid || ((vmask >> t) & 1u))) ps = make_float2(ps.x + u.x, ps.y + u.y);
          }
        } else if (CPLX && fbits == 16) {   // 8-bit complex: one (re, im) byte pair
#pragma unroll
          for (int t = 0; t < 16; t++) {
            const uint32_t w = *reinterpret_cast<const unsigned short *>(rb + NT * BPTS * t);
            const float2 u = make_float2(s_lut[w & 255u], s_lut[w >> 8]);
            v[t] = cmul(cmul(rsk, rpj[JSTEP * t]), u);
            if (PC && (allvalid || ((vmask >> t) & 1u))) ps = make_float2(ps.x + u.x, ps.y + u.y);
          }
        } else {
#pragma unroll
          for (int t = 0; t < 16; t++) {
            const uint32_t w = rb[NT * BPTS * t];
            const float2 rot = cmul(rsk, rpj[JSTEP * t]);
            const float ux = s_lut[(w >> sh) & cmask];
            const float uy = CPLX ? s_lut[(w >> (sh + J.nbits)) & cmask] : 0.f;
            if (CPLX) v[t] = cmul(rot, make_float2(ux, uy));
            else v[t] = make_float2(ux * rot.x, ux * rot.y);
            if (PC && (allvalid || ((vmask >> t) & 1u))) ps = make_float2(ps.x + ux, ps.y + uy);
          }
        }
        if (!allvalid) {
#pragma unroll
          for (int t = 0; t < 16; t++)
            if (!((vmask >> t) & 1u)) v[t] = make_float2(0.f, 0.f);
        }
      }
      if (PC) xb[pc_slot(j)] = ps;
      fft<F, CTA>(v, j, g, xb, tw, twA, twB, [&]() {
        if (PC && pcout && j < pcn) {
          // bin (pcbin of thread j) collects threads j, j + nbins, ...: fixed
          // order; one thread per bin and item, items ordered by the group's
          // barriers, so the sums do not depend on timing
          float2 a = make_float2(0.f, 0.f);
          for (int m = j; m < NT; m += pcn) {
            const float2 q = xb[pc_slot(m)];
            a = make_float2(a.x + q.x, a.y + q.y);
          }
          float2 *o = pcout + (size_t)bd * pf.maxbins + pcbin;
          atomicAdd(&o->x, a.x);
          if (CPLX) atomicAdd(&o->y, a.y);
        }
      });
      // register t holds bin j + NT t: sideband selection, fractional-sample
      // correction sub[c mod S] step[c / S] (c mod S fixed per thread), store
      const int lsb = st.lsb[lf];
      const int f = st.freq_index[lf];
      float2 *drow = spec + (((size_t)f * nblk + bi) * J.ninputs + st.band_input[bd]) * N;
      if (CPLX && lsb) {
        const float2 fsk = fs[(-j) & (SD - 1)];
#pragma unroll
        for (int t = 0; t < 16; t++) {
          float2 val = v[t];
          int c;
          r16_channel<F, CPLX>(t, j, 1, val, c);
          drow[c] = cmul(val, cmul(fsk, fp[c >> LGS]));
        }
      } else {
        // channel c = j + NT t' with t' = t (upper sideband), t - 8 (real lower sideband)
        const float2 fsk = fs[j & (SD - 1)];
        const float2 *fpj = fp + (j >> LGS);
        float2 *dj = drow + j;
#pragma unroll
        for (int t = 0; t < (CPLX ? 16 : 8); t++) {
          const float2 val = (!CPLX && lsb) ? v[t + 8] : v[t];
          dj[NT * t] = cmul(val, cmul(fsk, fpj[JSTEP * t]));
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
  if (J.cplx ? (bpts != 4 && bpts != 8 && bpts != 16) : (bpts != 1 && bpts != 2 && bpts != 4 && bpts != 8))
    return false;
  const int fbits = J.nbits * (J.cplx ? 2 : 1);
  if (fbits > 8 && fbits != 16) return false;   // fields within a byte, or one (re, im) byte pair
  const int paybytes = J.framesamples * bpts;
  if (J.framebytes != 32 + paybytes || paybytes % 16) return false;
  return true;
}

static size_t sb_tab(const DevJob &J, int maxnrf, int deltapol)
{
  const int S = J.stride, nfr = J.fftlen / S, half = J.nchan / S;
  return (size_t)((maxnrf * (S + nfr + (deltapol ? 2 : 1) * (S + half)) + 1) & ~1);
}

size_t fstep_sb_smem_bytes(const DevJob &J, int maxnrf, int deltapol)
{
  const int F = J.fftlen, NT = F / 16, G = (NT >= 256 ? NT : 256) / NT;
  const int bpts = J.nbands * J.nbits * (J.cplx ? 2 : 1) / 8;
  return 2 * sb::kTwRow * sizeof(float2) +
         (size_t)G * ((F + F / 16 + sb_tab(J, maxnrf, deltapol)) * sizeof(float2) + (size_t)(F * bpts + 32));
}

// Whether the kernel can form the phase-cal sums of pf for this job and
// launch shape: bins dividing the threads of a transform, one slot per group.
bool fstep_sb_pcal_fits(const DevJob &J, const PcalFuse &pf, int nblk)
{
  const int F = J.fftlen, NT = F / 16, G = (NT >= 256 ? NT : 256) / NT;
  const int bpc = (J.sb_items > 0 ? J.sb_items : 4) * G;
  return pf.partial && pf.first && pf.nbins > 0 && pf.nbins <= NT && NT % pf.nbins == 0 &&
         (long long)((nblk + bpc - 1) / bpc) * G <= pf.slots;
}

cudaError_t fstep_sb_launch(const DevJob &J, const DevStation *stations, int maxnrf, int deltapol,
                            const SubintArrays &S, int nblk, const BlockParam *bp, float2 *spec, cudaStream_t st,
                            const PcalFuse *pf, bool *pcal_done)
{
  const int F = J.fftlen, NT = F / 16, G = (NT >= 256 ? NT : 256) / NT;
  const int tabstride = (int)sb_tab(J, maxnrf, deltapol);
  const size_t sm = fstep_sb_smem_bytes(J, maxnrf, deltapol);
  if (sm > 227 * 1024) return cudaErrorNotSupported;
  const int bpts = J.nbands * J.nbits * (J.cplx ? 2 : 1) / 8;
  const int bpc = (J.sb_items > 0 ? J.sb_items : 4) * G;   // items per group (four unless tuned)
  dim3 grid((nblk + bpc - 1) / bpc, J.nstations);
  const bool pc = pf && fstep_sb_pcal_fits(J, *pf, nblk);
  const PcalFuse pfv = pc ? *pf : PcalFuse{};
#define GX_SB_CASE(FLV, CX, BP)                                                                          \
  if (F == FLV && J.cplx == CX && bpts == BP) {                                                          \
    using K = sb::Cfg<FLV, CX, BP>;                                                                      \
    const void *kf = pc ? (const void *)sb::fstep_sb_kernel<FLV, CX, BP, true>                           \
                        : (const void *)sb::fstep_sb_kernel<FLV, CX, BP, false>;                         \
    cudaError_t e = smem_opt_in(kf, sm);                                                                 \
    if (e != cudaSuccess) return e;                                                                      \
    if (pc)                                                                                              \
      sb::fstep_sb_kernel<FLV, CX, BP, true><<<grid, K::CTA, sm, st>>>(J, stations, S, bp, nblk, bpc,     \
                                                                        tabstride, spec, pfv);           \
    else                                                                                                 \
      sb::fstep_sb_kernel<FLV, CX, BP, false><<<grid, K::CTA, sm, st>>>(J, stations, S, bp, nblk, bpc,    \
                                                                         tabstride, spec, pfv);          \
    e = cudaGetLastError();                                                                              \
    if (e == cudaSuccess && pcal_done) *pcal_done = pc;                                                  \
    return e;                                                                                            \
  }
#define GX_SB_SIZES(CX, BP) \
  GX_SB_CASE(512, CX, BP) GX_SB_CASE(1024, CX, BP) GX_SB_CASE(2048, CX, BP) GX_SB_CASE(4096, CX, BP) GX_SB_CASE(8192, CX, BP)
  GX_SB_SIZES(0, 1) GX_SB_SIZES(0, 2) GX_SB_SIZES(0, 4) GX_SB_SIZES(0, 8)
  GX_SB_SIZES(1, 4) GX_SB_SIZES(1, 8) GX_SB_SIZES(1, 16)
#undef GX_SB_SIZES
#undef GX_SB_CASE
  return cudaErrorNotSupported;
}

}  // namespace gx
