// Register-resident forward FFT of F points spread over NT = F / 16 threads
// (16 points per thread), the building block of the long-transform F-step.
//
// Stockham formulation: every pass reads the 16 points x[j + NT t] of thread j
// (t = 0..15).  A radix-16 pass of stride Ns twiddles them by W_{16 Ns}^{(j mod Ns) r},
// transforms them in registers (16 = 4 x 4) and writes them to
// out[(j - j mod Ns) * 16 + j mod Ns + Ns r] in shared memory, padded by one
// element every 16 so that the strided stores and loads spread over the banks.
// With F = 16^L * R0 (R0 in {1, 2, 4, 8}) the last radix-16 pass (R0 = 1) or a
// final radix-R0 pass (16 / R0 transforms per thread, done in registers) leaves
// X[j + NT t] in register t of thread j: no exchange after the last pass.
//
// Everything here is __host__ __device__ so that the index arithmetic can be
// exercised on the CPU.
#pragma once
#include <cuda_runtime.h>

namespace gx {
namespace r16 {

__host__ __device__ __forceinline__ float2 add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 mul(float2 a, float2 b)
{
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }   // * (-i)

// shared-memory position of element i: one pad element per 16
__host__ __device__ __forceinline__ int pad(int i) { return i + (i >> 4); }

// Paired FP32 add and subtract (one f32x2 instruction on sm_100, same
// rounding as the two scalar operations); plain float2 arithmetic on the host.
__host__ __device__ __forceinline__ float2 add2(float2 a, float2 b)
{
#ifdef __CUDA_ARCH__
  return __fadd2_rn(a, b);
#else
  return add(a, b);
#endif
}
__host__ __device__ __forceinline__ float2 sub2(float2 a, float2 b)
{
#ifdef __CUDA_ARCH__
  float2 r;
  asm("{\n\t.reg .b64 pa, pb, pd;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "sub.rn.f32x2 pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
#else
  return sub(a, b);
#endif
}

// 4-point forward DFT in place, natural order (the +-i terms stay scalar:
// their operands are swapped lanes)
__host__ __device__ __forceinline__ void dft4(float2 &a, float2 &b, float2 &c, float2 &d)
{
  const float2 s0 = add2(a, c), s1 = sub2(a, c), s2 = add2(b, d), s3 = mul_mi(sub2(b, d));
  a = add2(s0, s2);
  c = sub2(s0, s2);
  b = add(s1, s3);
  d = sub(s1, s3);
}

// 2-point forward DFT in place
__host__ __device__ __forceinline__ void dft2(float2 &a, float2 &b)
{
  const float2 t = a;
  a = add(t, b);
  b = sub(t, b);
}

// 8-point forward DFT in place, natural order: n = 2 n1 + n2, k = k1 + 4 k2
__host__ __device__ __forceinline__ void dft8(float2 *u)
{
  const float h = 0.70710678118654752440f;
  dft4(u[0], u[2], u[4], u[6]);   // even samples: E[k1] at 0, 2, 4, 6
  dft4(u[1], u[3], u[5], u[7]);   // odd samples:  O[k1] at 1, 3, 5, 7
  const float2 o0 = u[1];
  const float2 o1 = make_float2((u[3].x + u[3].y) * h, (u[3].y - u[3].x) * h);    // * W8^1
  const float2 o2 = mul_mi(u[5]);                                                   // * W8^2
  const float2 o3 = make_float2((u[7].y - u[7].x) * h, -(u[7].x + u[7].y) * h);    // * W8^3
  const float2 e0 = u[0], e1 = u[2], e2 = u[4], e3 = u[6];
  u[0] = add(e0, o0);
  u[4] = sub(e0, o0);
  u[1] = add(e1, o1);
  u[5] = sub(e1, o1);
  u[2] = add(e2, o2);
  u[6] = sub(e2, o2);
  u[3] = add(e3, o3);
  u[7] = sub(e3, o3);
}

// 16-point forward DFT in place, natural order: n = 4 n1 + n2, k = k1 + 4 k2,
// X[k1 + 4 k2] = sum_n2 W4^(n2 k2) W16^(n2 k1) sum_n1 x[4 n1 + n2] W4^(n1 k1).
__host__ __device__ __forceinline__ void dft16(float2 (&v)[16])
{
  const float c1 = 0.92387953251128675613f;   // cos(pi / 8)
  const float s1 = 0.38268343236508977173f;   // sin(pi / 8)
  const float h = 0.70710678118654752440f;
#pragma unroll
  for (int n2 = 0; n2 < 4; n2++) dft4(v[n2], v[4 + n2], v[8 + n2], v[12 + n2]);
  // y[n2][k1] sits at v[4 k1 + n2]; multiply by W16^(n2 k1)
  v[5] = mul(v[5], make_float2(c1, -s1));     // W^1
  v[9] = mul(v[9], make_float2(h, -h));       // W^2
  v[13] = mul(v[13], make_float2(s1, -c1));   // W^3
  v[6] = mul(v[6], make_float2(h, -h));       // W^2
  v[10] = mul_mi(v[10]);                      // W^4
  v[14] = mul(v[14], make_float2(-h, -h));    // W^6
  v[7] = mul(v[7], make_float2(s1, -c1));     // W^3
  v[11] = mul(v[11], make_float2(-h, -h));    // W^6
  v[15] = mul(v[15], make_float2(-c1, s1));   // W^9
#pragma unroll
  for (int k1 = 0; k1 < 4; k1++) dft4(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
  // v[4 k1 + k2] = X[k1 + 4 k2]: transpose the 4 x 4 to natural order
#pragma unroll
  for (int a = 0; a < 4; a++)
#pragma unroll
    for (int b = a + 1; b < 4; b++) {
      const float2 t = v[4 * a + b];
      v[4 * a + b] = v[4 * b + a];
      v[4 * b + a] = t;
    }
}

__host__ __device__ constexpr int log16_floor(int f) { return f >= 65536 ? 4 : (f >= 4096 ? 3 : (f >= 256 ? 2 : (f >= 16 ? 1 : 0))); }
__host__ __device__ constexpr int pow16(int l) { return l == 0 ? 1 : 16 * pow16(l - 1); }

// Twiddle table of an F-point transform as the device holds it: W_F^m for m
// in [0, F); then one section per radix-16 pass of stride Ns = 16^p
// (p = 1 .. L - 1), entry (r - 1) Ns + m = W_F^(r m F / (16 Ns)); then, for a
// final radix R0 > 1, entry (r - 1) (F / R0) + g = W_F^(g r).  Each row holds
// consecutive m (or g), so the loads of one r by a warp are contiguous.
__host__ __device__ constexpr int tw_pass_offset(int F, int p)
{
  int o = F;
  for (int q = 1; q < p; q++) o += 15 * pow16(q);
  return o;
}
__host__ __device__ constexpr int tw_final_offset(int F) { return tw_pass_offset(F, log16_floor(F)); }
__host__ __device__ constexpr int tw_table_size(int F)
{
  return tw_final_offset(F) + (F / pow16(log16_floor(F)) > 1 ? (F / pow16(log16_floor(F)) - 1) * pow16(log16_floor(F)) : 0);
}

template <int F>
struct Plan {
  static constexpr int NT = F / 16;               // threads per transform
  static constexpr int L = log16_floor(F);        // radix-16 passes
  static constexpr int R0 = F / pow16(L);         // final radix (1: none)
  static constexpr int SMEM = F + F / 16;         // padded exchange buffer, float2
  static_assert(F >= 256 && F <= 16384 && (F & (F - 1)) == 0, "F must be a power of two in [256, 16384]");
};

// Radix-16 pass of stride Ns: twiddle (Ns > 1) and transform in registers.
// tw[m] = exp(-2 pi i m / F).  The twiddles w^r, r = 1..15, of a thread come
// from four table entries (w, w^2, w^4, w^8) and at most three products each:
// the table gathers of a warp touch many cache lines, so fifteen loads per
// pass cost more L1 throughput than eleven products cost issue slots.
template <int F, typename TW>
__host__ __device__ __forceinline__ void pass16(float2 (&v)[16], int j, int Ns, TW tw)
{
  if (Ns > 1) {
    const int m = j & (Ns - 1);
    const int step = m * (F / (16 * Ns));
    float2 w[16];
    w[1] = tw(step);
    w[2] = tw(2 * step);
    w[4] = tw(4 * step);
    w[8] = tw(8 * step);
    w[3] = mul(w[2], w[1]);
    w[5] = mul(w[4], w[1]);
    w[6] = mul(w[4], w[2]);
    w[7] = mul(w[4], w[3]);
    w[9] = mul(w[8], w[1]);
    w[10] = mul(w[8], w[2]);
    w[11] = mul(w[8], w[3]);
    w[12] = mul(w[8], w[4]);
    w[13] = mul(w[8], w[5]);
    w[14] = mul(w[8], w[6]);
    w[15] = mul(w[8], w[7]);
#pragma unroll
    for (int r = 1; r < 16; r++) v[r] = mul(v[r], w[r]);
  }
  dft16(v);
}

// Outputs of a radix-16 pass of stride Ns (a power of 16) into the padded
// exchange buffer: element base + Ns r sits at pad(base) + r (Ns + Ns / 16)
// (Ns r is a multiple of 16, so the pad of the sum is the sum of the pads), and
// for Ns = 1 (base = 16 j) at 17 j + r: one base index, then constant offsets.
__host__ __device__ __forceinline__ void store16(const float2 (&v)[16], int j, int Ns, float2 *sm)
{
  const int m = j & (Ns - 1);
  const int p0 = Ns == 1 ? 17 * j : pad((j - m) * 16 + m);
  const int step = Ns == 1 ? 1 : Ns + (Ns >> 4);
#pragma unroll
  for (int r = 0; r < 16; r++) sm[p0 + step * r] = v[r];
}

// Inputs x[j + NT t] of the next pass from the padded exchange buffer
// (NT = F / 16 is a multiple of 16: pad(j + NT t) = pad(j) + t (NT + NT / 16)).
template <int F>
__host__ __device__ __forceinline__ void load16(float2 (&v)[16], int j, const float2 *sm)
{
  constexpr int NT = F / 16, step = NT + NT / 16;
  const int p0 = pad(j);
#pragma unroll
  for (int t = 0; t < 16; t++) v[t] = sm[p0 + step * t];
}

// Final radix-R0 pass (stride F / R0) in registers: 16 / R0 transforms per thread.
template <int F, int R0, typename TW>
__host__ __device__ __forceinline__ void final_pass(float2 (&v)[16], int j, TW tw)
{
  constexpr int M = 16 / R0, NT = F / 16;
#pragma unroll
  for (int mm = 0; mm < M; mm++) {
    const int g = j + NT * mm;
    float2 u[R0];
#pragma unroll
    for (int r = 0; r < R0; r++) u[r] = (r == 0) ? v[mm] : mul(v[mm + M * r], tw(g * r));
    if constexpr (R0 == 2) dft2(u[0], u[1]);
    else if constexpr (R0 == 4) dft4(u[0], u[1], u[2], u[3]);
    else dft8(u);
#pragma unroll
    for (int r = 0; r < R0; r++) v[mm + M * r] = u[r];
  }
}

}  // namespace r16
}  // namespace gx
