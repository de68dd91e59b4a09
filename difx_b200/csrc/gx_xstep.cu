// X-step (plain FP32 form): Hermitian cross-multiply-accumulate of the
// spectra of every input (station x band) of a frequency, per channel,
// summed over FFT blocks -- the work of Core::processdata's XMAC loop
// (mpifxcorr/src/core.cpp:884-968, vectorAddProduct_cf32 ->
// genericAddProduct_32fc, architecture.h.in:575-580) and of the station
// autocorrelations (mode.cpp:1270-1285, 1333-1352), which are the diagonal
// and same-station entries of the same Hermitian product.
//
// Work decomposition: the NI x NI input matrix of a frequency is split into
// ST x ST super-tiles; only super-tiles on or above the diagonal are
// computed.  A CTA owns one super-tile for CT channels and a slice of the
// blocks; each thread owns a T x T register tile of accumulators for one
// channel.  Spectra rows of the super-tile are staged in shared memory.
//
// Accumulators: acc[ks][freq][stpair][ST][ST][N] (float2), summed over the
// chunk passes of a subint; finalise_kernel maps them to the Core result
// layout (configuration.cpp:2348-2630) and sums the K-split slices.
#include <cstdint>
#include "gx_dev.h"
#include "gx_xstep.h"

namespace gx {

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int src_bytes)
{
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <int T, int ST, int CT, int KB, int NSTAGE>
__global__ void __launch_bounds__(CT *(ST / T) * (ST / T))
xmac_fp32_kernel(const float2 *__restrict__ spec, int nblk, int NI, int N, int nsuper,
                 int ks_count, float2 *__restrict__ acc)
{
  constexpr int NT = ST / T;            // register tiles per super-tile side
  constexpr int NTHREADS = CT * NT * NT;
  constexpr int STAGE = KB * ST * CT;   // float2 per stage per operand
  extern __shared__ __align__(16) float2 xsm[];
  float2 *sI = xsm;                     // [NSTAGE][KB][ST][CT]
  float2 *sJ = xsm + NSTAGE * STAGE;    // [NSTAGE][KB][ST][CT]

  const int tid = threadIdx.x;
  const int c = tid % CT;
  const int p = tid / CT;
  const int ti = p / NT, tj = p % NT;
  const int c0 = blockIdx.x * CT;
  const int stp = blockIdx.y;           // super-tile pair index (upper triangle, row-major)
  const int f = blockIdx.z / ks_count;
  const int ks = blockIdx.z % ks_count;
  int SI = 0, rem = stp;
  while (rem >= nsuper - SI) { rem -= nsuper - SI; SI++; }
  const int SJ = SI + rem;
  const int I0 = SI * ST, J0 = SJ * ST;
  const bool diag = (SI == SJ);
  const float2 *sJread = diag ? sI : sJ;

  const int kper = (nblk + ks_count - 1) / ks_count;
  const int kb0 = ks * kper, kb1 = min(nblk, kb0 + kper);
  const int nstages = (kb1 > kb0) ? (kb1 - kb0 + KB - 1) / KB : 0;

  // one stage: rows [I0, I0+ST) (and [J0, J0+ST) off the diagonal) x CT channels x KB blocks,
  // 16-byte (two-channel) pieces; missing blocks/channels are zero-filled
  auto load_stage = [&](int st, int buf) {
    const int k = kb0 + st * KB;
    constexpr int PIECES = KB * ST * (CT / 2);
    for (int e = tid; e < PIECES * (diag ? 1 : 2); e += NTHREADS) {
      const int opnd = e / PIECES;
      const int q = e % PIECES;
      const int kk = q / (ST * (CT / 2));
      const int r = (q / (CT / 2)) % ST;
      const int cc = (q % (CT / 2)) * 2;
      const int row = (opnd ? J0 : I0) + r;
      const bool ok = (k + kk < kb1) && (c0 + cc < N) && (row < NI);
      const float2 *src = ok ? spec + (((size_t)f * nblk + (k + kk)) * NI + row) * N + c0 + cc : spec;
      float2 *dst = (opnd ? sJ : sI) + buf * STAGE + (kk * ST + r) * CT + cc;
      cp_async16(dst, src, ok ? 16 : 0);
    }
    cp_async_commit();
  };

  float ar[T][T], ai[T][T];
#pragma unroll
  for (int a = 0; a < T; a++)
#pragma unroll
    for (int b = 0; b < T; b++) { ar[a][b] = 0.f; ai[a][b] = 0.f; }

  const bool compute = !diag || (ti <= tj);   // lower tiles of diagonal super-tiles are redundant

  // NSTAGE-deep cp.async pipeline (one commit group per stage, empty groups at the tail)
#pragma unroll
  for (int s0 = 0; s0 < NSTAGE - 1; s0++) {
    if (s0 < nstages) load_stage(s0, s0);
    else cp_async_commit();
  }
  for (int st = 0; st < nstages; st++) {
    const int buf = st % NSTAGE;
    if (st + NSTAGE - 1 < nstages) load_stage(st + NSTAGE - 1, (st + NSTAGE - 1) % NSTAGE);
    else cp_async_commit();
    cp_async_wait<NSTAGE - 1>();
    __syncthreads();
    if (compute) {
      const float2 *bi_ = sI + buf * STAGE;
      const float2 *bj_ = sJread + buf * STAGE;
#pragma unroll 2
      for (int kk = 0; kk < KB; kk++) {
        float2 xi[T], xj[T];
#pragma unroll
        for (int r = 0; r < T; r++) {
          xi[r] = bi_[(kk * ST + ti * T + r) * CT + c];
          xj[r] = bj_[(kk * ST + tj * T + r) * CT + c];
        }
#pragma unroll
        for (int a = 0; a < T; a++)
#pragma unroll
          for (int b = 0; b < T; b++) {
            // xi * conj(xj)
            ar[a][b] = fmaf(xi[a].x, xj[b].x, ar[a][b]);
            ar[a][b] = fmaf(xi[a].y, xj[b].y, ar[a][b]);
            ai[a][b] = fmaf(xi[a].y, xj[b].x, ai[a][b]);
            ai[a][b] = fmaf(-xi[a].x, xj[b].y, ai[a][b]);
          }
      }
    }
    __syncthreads();
  }
  if (!compute || c0 + c >= N) return;
  const int nfreqs = gridDim.z / ks_count;
  const size_t base = (((size_t)ks * nfreqs + f) * gridDim.y + stp) * (size_t)ST * ST;
#pragma unroll
  for (int a = 0; a < T; a++)
#pragma unroll
    for (int b = 0; b < T; b++) {
      const int ii = ti * T + a, jj = tj * T + b;
      float2 *dst = acc + (base + (size_t)ii * ST + jj) * N + c0 + c;
      float2 v = *dst;
      v.x += ar[a][b];
      v.y += ai[a][b];
      *dst = v;
    }
}

// Sum of weights over the blocks of one chunk (Core::processdata baseline
// weights core.cpp:1005-1052; Mode autocorrelation weights mode.cpp:1277-1284).
// Weight sums over a pass of blocks: item i < nstations sums station row i;
// item nstations + k sums the products of rows pairs[k] (or row pairs[k].x
// alone when pairs[k].y < 0).
__global__ void weights_kernel(const float *__restrict__ w, int nblk, int nstations,
                               const int2 *__restrict__ pairs, int npairs, float *__restrict__ wacc)
{
  __shared__ float red[256];
  const int item = blockIdx.x;  // [0, nstations): station sums; then baseline products
  float sum = 0.f;
  if (item < nstations) {
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) sum += w[(size_t)item * nblk + b];
  } else {
    const int2 pr = pairs[item - nstations];
    if (pr.y < 0) {   // one row alone (a per-band weight row)
      for (int b = threadIdx.x; b < nblk; b += blockDim.x) sum += w[(size_t)pr.x * nblk + b];
    } else {
      for (int b = threadIdx.x; b < nblk; b += blockDim.x)
        sum += w[(size_t)pr.x * nblk + b] * w[(size_t)pr.y * nblk + b];
    }
  }
  red[threadIdx.x] = sum;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) wacc[item] += red[0];
}

// Result array assembly (Core result layout).
__global__ void finalise_vis_kernel(const ProdEntry *__restrict__ prods, int nprods, const float2 *__restrict__ acc,
                                    int ks_count, size_t ks_stride, int N, float2 *__restrict__ results)
{
  const int e = blockIdx.y;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nprods || c >= N) return;
  const ProdEntry pe = prods[e];
  float2 s = make_float2(0.f, 0.f);
  for (int k = 0; k < ks_count; k++) {
    const float2 v = acc[(size_t)k * ks_stride + pe.acc_index + c];
    s.x += v.x;
    s.y += v.y;
  }
  if (pe.conj) s.y = -s.y;
  results[pe.result_offset + c] = s;
}

__global__ void finalise_weights_kernel(const WeightEntry *__restrict__ we, int nw, const float *__restrict__ wacc,
                                        float *__restrict__ results_f)
{
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nw) return;
  const WeightEntry x = we[e];
  results_f[x.float_index] = x.source >= 0 ? wacc[x.source] : 0.0f;
}

// ------------------------------------------------------------------ launchers

template <int T, int ST, int CT, int KB, int NSTAGE>
static cudaError_t launch_t(const float2 *spec, int nblk, int NI, int N, int nfreqs, int ks, float2 *acc,
                            cudaStream_t st)
{
  const int nsuper = (NI + ST - 1) / ST;
  const int npairs = nsuper * (nsuper + 1) / 2;
  const size_t sm = sizeof(float2) * 2 * NSTAGE * KB * ST * CT;
  cudaError_t e = smem_opt_in((const void *)xmac_fp32_kernel<T, ST, CT, KB, NSTAGE>, sm);
  if (e != cudaSuccess) return e;
  dim3 grid((N + CT - 1) / CT, npairs, nfreqs * ks);
  xmac_fp32_kernel<T, ST, CT, KB, NSTAGE>
      <<<grid, CT *(ST / T) * (ST / T), sm, st>>>(spec, nblk, NI, N, nsuper, ks, acc);
  return cudaGetLastError();
}

XmacShape xmac_shape(int NI)
{
  XmacShape s;
  if (NI <= 8) { s.T = 4; s.ST = 8; s.CT = 32; }
  else if (NI <= 16) { s.T = 4; s.ST = 16; s.CT = 16; }
  else { s.T = 8; s.ST = 32; s.CT = 16; }
  s.nsuper = (NI + s.ST - 1) / s.ST;
  s.npairs = s.nsuper * (s.nsuper + 1) / 2;
  return s;
}

cudaError_t xmac_fp32_launch(const float2 *spec, int nblk, int NI, int N, int nfreqs, int ks, float2 *acc,
                             cudaStream_t st)
{
  XmacShape s = xmac_shape(NI);
  if (s.ST == 8) return launch_t<4, 8, 32, 8, 3>(spec, nblk, NI, N, nfreqs, ks, acc, st);
  if (s.ST == 16) return launch_t<4, 16, 16, 8, 3>(spec, nblk, NI, N, nfreqs, ks, acc, st);
  return launch_t<8, 32, 16, 8, 3>(spec, nblk, NI, N, nfreqs, ks, acc, st);
}

cudaError_t weights_launch(const float *w, int nblk, int nstations, const int2 *pairs, int npairs, float *wacc,
                           cudaStream_t st)
{
  weights_kernel<<<nstations + npairs, 256, 0, st>>>(w, nblk, nstations, pairs, npairs, wacc);
  return cudaGetLastError();
}

cudaError_t finalise_launch(const ProdEntry *prods, int nprods, const float2 *acc, int ks, size_t ks_stride, int N,
                            const WeightEntry *we, int nw, const float *wacc, float2 *results, cudaStream_t st)
{
  if (nprods > 0) {
    dim3 grid((N + 127) / 128, nprods);
    finalise_vis_kernel<<<grid, 128, 0, st>>>(prods, nprods, acc, ks, ks_stride, N, results);
  }
  if (nw > 0)
    finalise_weights_kernel<<<(nw + 255) / 256, 256, 0, st>>>(we, nw, wacc, reinterpret_cast<float *>(results));
  return cudaGetLastError();
}

// Channel averaging of the finished result array (Mode::averageFrequency,
// mode.cpp:1376-1401, for autocorrelations; Core's averaged copy,
// core.cpp:1819-1869, for cross products): one CTA per record.
__global__ void average_kernel(const AvgEntry *__restrict__ tab, const float2 *__restrict__ full,
                               float2 *__restrict__ out)
{
  const AvgEntry e = tab[blockIdx.x];
  for (int c = threadIdx.x; c < e.n; c += blockDim.x) {
    const float2 *p = full + e.src + (long long)c * e.L;
    float2 acc = p[0];
    for (int i = 1; i < e.L; i++) {
      acc.x += p[i].x;
      acc.y += p[i].y;
    }
    out[e.dst + c] = e.L == 1 ? acc : make_float2(acc.x / (float)e.L, acc.y / (float)e.L);   // the mean
  }
}

cudaError_t average_launch(const AvgEntry *tab, int nent, const float2 *full, float2 *out, cudaStream_t st)
{
  if (nent <= 0) return cudaSuccess;
  average_kernel<<<nent, 128, 0, st>>>(tab, full, out);
  return cudaGetLastError();
}

}  // namespace gx
