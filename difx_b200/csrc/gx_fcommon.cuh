// Device helpers shared by the F-step kernels (gx_fstep.cu, gx_fstep_sb.cu):
// complex products, the per-block rotator table entries (FP64 phases, FP32
// sincos; mode.cpp:882-955, 1029-1122), group barriers and the sideband
// selection of the register-resident transforms.
#pragma once
#include <cstdint>
#include "gx_dev.h"

namespace gx {

#define GX_TWO_PI 6.283185307179586476925286766559

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

// Fringe-rotator table entry e of local freq fi: e < S -> sub[e], else step[e - S]
// (mode.cpp:882-955: FP64 phases, FP32 argument, sincos).
__device__ __forceinline__ float2 fringe_entry(const DevJob &J, const DevStation &st, int fi, int e,
                                               const BlockParam &P)
{
  if (J.fringe_order == 0) return make_float2(1.0f, 0.0f);   // post-F: no rotation before the FFT
  const int Sd = J.stride, F = J.fftlen;
  const double lofreq = st.lofreq[fi];
  const double looffset = st.looff[fi];
  const bool looff = (looffset > 0.0 || looffset < 0.0);
  double ph;
  if (e < Sd) {
    double x = ((double)e / (double)F) * P.a;
    x += P.b;
    ph = x * lofreq;
    if (st.fractional_lo) ph += (lofreq - (int)lofreq) * (double)P.integerdelay;
    if (looff) {
      ph += ((e * J.sampletime) / 1e6) * -looffset;
      ph += -looffset * P.fracwalltime;
      double fl = fabs(looffset) - (int)fabs(looffset);
      const bool isfrac = fl > (double)0.000000001f;
      if (looffset < 0) fl = -fl;
      if (isfrac) ph += -fl * P.intwalltime;
    }
  } else if (e < Sd + J.nfr) {
    const int j = e - Sd;
    const double xoff = (double)(j * Sd) / (double)F;
    // quadratic: stepxoff b + stepxoff^2 a (mode.cpp:813-819)
    const double x = J.fringe_order == 2 ? xoff * P.qb + (xoff * xoff) * P.qa : xoff * P.a;
    ph = x * lofreq;
    if (looff) ph += ((j * Sd * J.sampletime) / 1e6) * -looffset;
  } else {
    // quadratic only: the per-stride phase step of sub entry k (mode.cpp:810-812)
    const int k = e - Sd - J.nfr;
    const double x = ((double)k / (double)F) * (2 * P.qa * ((double)Sd / (double)F));
    ph = x * lofreq;
  }
  const float arg = (float)(-GX_TWO_PI * (ph - (int)ph));
  float sn, cs;
  sincosf(arg, &sn, &cs);
  return make_float2(cs, sn);
}

// Fractional-sample rotator entry e of local freq fi, polarisation set ps
// (0: A, 1: B): e < S -> sub[e], else step[e - S] (mode.cpp:1029-1122).
__device__ __forceinline__ float2 frac_entry(const DevJob &J, const DevStation &st, int fi, int ps, int e,
                                             const BlockParam &P)
{
  const int Sd = J.stride, N = J.nchan, half = J.half;
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
  float arg = __fmul_rn(cfreq, val);
  if (J.fringe_order == 0 && e < Sd) {
    // post-F fringe rotation (and LO offset) at the block centre, added to
    // the first stride's argument for both polarisation sets (mode.cpp:1038-1049, 1085-1096)
    const double lofreq = st.lofreq[fi];
    double ph = P.b * lofreq;
    if (st.fractional_lo) ph += P.integerdelay * (lofreq - (int)lofreq);
    ph -= ((double)P.intwalltime + P.fracwalltime) * st.looff[fi];
    arg = __fadd_rn(arg, (float)(-GX_TWO_PI * (ph - (int)ph)));
  }
  float sn, cs;
  sincosf(arg, &sn, &cs);
  return make_float2(cs, sn);
}

template <int NT, int CTA>
__device__ __forceinline__ void group_sync(int g)
{
  if constexpr (NT == 32) __syncwarp();
  else if constexpr (NT == CTA) __syncthreads();
  else asm volatile("bar.sync %0, %1;" ::"r"(g + 1), "r"(NT) : "memory");
}

// Sideband selection (mode.cpp:1185-1217) for bin j + NT t: false when the bin
// is not kept; otherwise its channel c (val conjugated for complex LSB).
template <int F, int CPLX>
__device__ __forceinline__ bool r16_channel(int t, int j, int lsb, float2 &val, int &c)
{
  constexpr int NT = F / 16, NCH = CPLX ? F : F / 2;
  const int bin = j + NT * t;
  if (!CPLX) {
    if (lsb ? (t < 8) : (t >= 8)) return false;   // NT * 8 = F / 2 = NCH
    c = lsb ? bin - NCH : bin;
  } else if (!lsb) {
    c = bin;
  } else {
    c = bin == 0 ? 0 : F - bin;
    if (bin != 0) val.y = -val.y;
  }
  return true;
}

}  // namespace gx
