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
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include "gx_dev.h"
#include "gx_xstep.h"
#include "gx_mbar.cuh"
#include "gx_fcommon.cuh"

namespace gx {

template <int T, int ST, int CT>
__host__ __device__ constexpr int xmac_consumers() { return CT * (ST / T) * (ST / T); }

// One CTA: super-tile pair blockIdx.x (upper triangle, row-major) of frequency
// f for CT channels from c0 = blockIdx.y CT, over the blocks of K-split slice
// ks.  One producer warp (the last) loads each stage -- KB blocks x ST rows x
// CT channels of the I and (off the diagonal) J rows -- with one TMA tile per
// operand into an NSTAGE ring; the consumer warps multiply from shared memory
// and free each stage with one arrival per warp, so no CTA-wide barrier
// separates the stages.  Every wait is bounded (kWaitLimitNs): on expiry the
// CTA records a status in *err (when given), drains the copies it issued and
// adds nothing.
template <int T, int ST, int CT, int KB, int NSTAGE, int UNR = 1>
__global__ void __launch_bounds__(xmac_consumers<T, ST, CT>() + 32, 1)
xmac_fp32_kernel(const __grid_constant__ CUtensorMap spec_map, int nblk, int N, int nsuper, int ks_count,
                 int kper, float2 *__restrict__ acc, int *__restrict__ err)
{
  constexpr int NT = ST / T;            // register tiles per super-tile side
  constexpr int NC = xmac_consumers<T, ST, CT>();
  constexpr int NCW = NC / 32;          // consumer warps
  constexpr int STAGE = KB * ST * CT;   // float2 per stage per operand
  extern __shared__ __align__(128) float2 xsm[];
  float2 *sI = xsm;                     // [NSTAGE][KB][ST][CT]
  float2 *sJ = xsm + NSTAGE * STAGE;    // [NSTAGE][KB][ST][CT]
  uint64_t *full = reinterpret_cast<uint64_t *>(sJ + NSTAGE * STAGE);
  uint64_t *empty = full + NSTAGE;
  volatile int *s_abort = reinterpret_cast<volatile int *>(empty + NSTAGE);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int stp = blockIdx.x;           // super-tile pair index
  const int c0 = blockIdx.y * CT;
  const int f = blockIdx.z / ks_count;
  const int ks = blockIdx.z % ks_count;
  int SI = 0, rem = stp;
  while (rem >= nsuper - SI) { rem -= nsuper - SI; SI++; }
  const int SJ = SI + rem;
  const int I0 = SI * ST, J0 = SJ * ST;
  const bool diag = (SI == SJ);

  // slices start on stage boundaries (kper is a multiple of KB); the last
  // stage may reach past nblk, where the copies read zeros
  const int kb0 = ks * kper, kb1 = min(nblk, kb0 + kper);
  const int nstages = (kb1 > kb0) ? (kb1 - kb0 + KB - 1) / KB : 0;

  if (tid == 0) {
    for (int i = 0; i < NSTAGE; i++) {
      mbar_init(smem_u32(full + i), 1);
      mbar_init(smem_u32(empty + i), NCW);
    }
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto abort_with = [&](int code) {
    *s_abort = 1;
    if (err) atomicExch(err, code);
  };

  if (warp == NCW) {
    // ---- producer
    if (lane == 0) {
      const uint32_t bytes = (diag ? 1u : 2u) * (uint32_t)(STAGE * sizeof(float2));
      int issued = 0;
      for (int st = 0; st < nstages; st++) {
        if (*s_abort) break;
        const int b = st % NSTAGE;
        if (st >= NSTAGE && !mbar_wait(smem_u32(empty + b), (uint32_t)(st / NSTAGE - 1) & 1u)) {
          abort_with(13);
          break;
        }
        const uint32_t bar = smem_u32(full + b);
        mbar_expect_tx(bar, bytes);
        const int k = kb0 + st * KB;
        tma_load_4d(smem_u32(sI + b * STAGE), &spec_map, 2 * c0, I0, k, f, bar);
        if (!diag) tma_load_4d(smem_u32(sJ + b * STAGE), &spec_map, 2 * c0, J0, k, f, bar);
        issued = st + 1;
      }
      if (*s_abort) {
        // drain: the copies this CTA issued land before it exits (bounded)
        for (int b = 0; b < NSTAGE && b < issued; b++) {
          const int ulast = b + ((issued - 1 - b) / NSTAGE) * NSTAGE;
          mbar_wait(smem_u32(full + b), (uint32_t)(ulast / NSTAGE) & 1u);
        }
      }
    }
    return;
  }

  // ---- consumers: a T x T register tile of one channel
  const int c = tid % CT;
  const int p = tid / CT;
  const int ti = p / NT, tj = p % NT;
  const float2 *sJread = diag ? sI : sJ;
  float2 acc2[T][T];   // (Re, Im) of each product sum, one register pair for the f32x2 FMAs
#pragma unroll
  for (int a = 0; a < T; a++)
#pragma unroll
    for (int b = 0; b < T; b++) acc2[a][b] = make_float2(0.f, 0.f);
  const bool compute = !diag || (ti <= tj);   // lower tiles of diagonal super-tiles are redundant
  bool ok = true;
  for (int st = 0; st < nstages; st++) {
    const int buf = st % NSTAGE;
    if (!mbar_wait(smem_u32(full + buf), (uint32_t)(st / NSTAGE) & 1u) || *s_abort) {
      abort_with(14);
      ok = false;
      break;
    }
    if (compute) {
      const float2 *bi_ = sI + buf * STAGE;
      const float2 *bj_ = sJread + buf * STAGE;
#pragma unroll UNR
      for (int kk = 0; kk < KB; kk++) {
        float2 xi[T], xj[T];
#pragma unroll
        for (int r = 0; r < T; r++) {
          xi[r] = bi_[(kk * ST + ti * T + r) * CT + c];
          xj[r] = bj_[(kk * ST + tj * T + r) * CT + c];
        }
        // xi * conj(xj) as two paired FMAs (one f32x2 instruction each on
        // sm_100): Re += xi.x xj.x then xi.y xj.y; Im += xi.y xj.x then -xi.x xj.y,
        // the same operations in the same order as four scalar FMAs.
        float2 xs[T], bx[T], by[T];
#pragma unroll
        for (int r = 0; r < T; r++) {
          xs[r] = make_float2(xi[r].y, -xi[r].x);
          bx[r] = make_float2(xj[r].x, xj[r].x);
          by[r] = make_float2(xj[r].y, xj[r].y);
        }
#pragma unroll
        for (int a = 0; a < T; a++)
#pragma unroll
          for (int b = 0; b < T; b++) {
            acc2[a][b] = __ffma2_rn(xi[a], bx[b], acc2[a][b]);
            acc2[a][b] = __ffma2_rn(xs[a], by[b], acc2[a][b]);
          }
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(smem_u32(empty + buf));   // the stage may be reloaded
  }
  if (!ok || !compute || c0 + c >= N) return;
  const int nfreqs = gridDim.z / ks_count;
  const size_t base = (((size_t)ks * nfreqs + f) * gridDim.x + stp) * (size_t)ST * ST;
#pragma unroll
  for (int a = 0; a < T; a++)
#pragma unroll
    for (int b = 0; b < T; b++) {
      const int ii = ti * T + a, jj = tj * T + b;
      float2 *dst = acc + (base + (size_t)ii * ST + jj) * N + c0 + c;
      float2 v = *dst;
      v.x += acc2[a][b].x;
      v.y += acc2[a][b].y;
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

template <int T, int ST, int CT, int KB, int NSTAGE, int UNR = 1>
static cudaError_t launch_t(const float2 *spec, int nblk, int NI, int N, int nfreqs, int ks, float2 *acc, int *err,
                            cudaStream_t st)
{
  const int nsuper = (NI + ST - 1) / ST;
  const int npairs = nsuper * (nsuper + 1) / 2;
  const size_t sm = sizeof(float2) * 2 * NSTAGE * KB * ST * CT + 2 * NSTAGE * sizeof(uint64_t) + 16;
  // spec[freq][block][row][channel] float2 as a 4-D FP32 tensor: {2N floats,
  // NI rows, nblk blocks, nfreqs}; one box = KB blocks x ST rows x CT channels
  CUtensorMap map;
  const cuuint64_t dims[4] = {(cuuint64_t)(2 * N), (cuuint64_t)NI, (cuuint64_t)nblk, (cuuint64_t)nfreqs};
  const cuuint32_t box[4] = {(cuuint32_t)(2 * CT), (cuuint32_t)ST, (cuuint32_t)KB, 1};
  cudaError_t e = tma_map_f32_4d(&map, spec, dims, box);
  if (e != cudaSuccess) return e;
  e = smem_opt_in((const void *)xmac_fp32_kernel<T, ST, CT, KB, NSTAGE, UNR>, sm);
  if (e != cudaSuccess) return e;
  // slices of whole stages, on 16-block boundaries for every variant (KB 8
  // or 16), so that the variants add the same blocks into each slice
  static_assert(16 % KB == 0, "slice boundaries must be whole stages");
  const int kper = ((nblk + ks - 1) / ks + 15) / 16 * 16;
  // super-tile pairs fastest: the pairs that share a channel group's spectra run together
  dim3 grid(npairs, (N + CT - 1) / CT, nfreqs * ks);
  xmac_fp32_kernel<T, ST, CT, KB, NSTAGE, UNR>
      <<<grid, xmac_consumers<T, ST, CT>() + 32, sm, st>>>(map, nblk, N, nsuper, ks, kper, acc, err);
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

cudaError_t xmac_fp32_launch(const float2 *spec, int nblk, int NI, int N, int nfreqs, int ks, float2 *acc, int *err,
                             cudaStream_t st, int variant)
{
  // every variant keeps the register tile T and super-tile ST of the shape
  // (the accumulator layout) and 192 KB of stages; variant 1 trades channels
  // per CTA against blocks per stage (or doubles the channels)
  XmacShape s = xmac_shape(NI);
  if (s.ST == 8)
    return variant == 1 ? launch_t<4, 8, 64, 8, 3>(spec, nblk, NI, N, nfreqs, ks, acc, err, st)
                        : launch_t<4, 8, 32, 8, 3>(spec, nblk, NI, N, nfreqs, ks, acc, err, st);
  if (s.ST == 16)
    return variant == 1 ? launch_t<4, 16, 32, 8, 3>(spec, nblk, NI, N, nfreqs, ks, acc, err, st)
                        : launch_t<4, 16, 16, 8, 3>(spec, nblk, NI, N, nfreqs, ks, acc, err, st);
  // 8 x 8 register tiles of 32-row super-tiles, 16 channels per CTA; the
  // block loop is not unrolled (unrolled by 2 or 4 it measured 3-9% slower)
  return variant == 1 ? launch_t<8, 32, 8, 16, 3>(spec, nblk, NI, N, nfreqs, ks, acc, err, st)
                      : launch_t<8, 32, 16, 8, 3>(spec, nblk, NI, N, nfreqs, ks, acc, err, st);
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

// Zoom spectra rows: one thread per channel of one row of one block.
__global__ void zoom_gather_kernel(const ZoomRow *__restrict__ rows, const float2 *__restrict__ spec, int NIm, int Nm,
                                   float2 *__restrict__ specz, int NIz, int Nz, int nblk)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= Nz) return;
  const ZoomRow r = rows[blockIdx.y];
  const int b = blockIdx.z;
  specz[(((size_t)r.zf * nblk + b) * NIz + r.zrow) * Nz + k] = spec[(((size_t)r.mf * nblk + b) * NIm + r.mrow) * Nm + r.off + k];
}

cudaError_t zoom_gather_launch(const ZoomRow *rows, int nrows, const float2 *spec, int NIm, int Nm, float2 *specz,
                               int NIz, int Nz, int nblk, cudaStream_t st)
{
  if (nrows <= 0 || nblk <= 0) return cudaSuccess;
  if (nrows > 65535 || nblk > 65535) return cudaErrorInvalidConfiguration;
  dim3 grid((Nz + 127) / 128, nrows, nblk);
  zoom_gather_kernel<<<grid, 128, 0, st>>>(rows, spec, NIm, Nm, specz, NIz, Nz, nblk);
  return cudaGetLastError();
}

// One interval of a multi-phase-centre subint: each thread one channel of
// one product row.  The rotator of channel c is the reference's two-level
// one: sub[c mod rsl] (band-edge turns included) times step[c / rsl], FP64
// turns, FP32 arguments and sincos, FP32 products in the reference's order.
__global__ void uvshift_kernel(const UvEntry *__restrict__ ents, const float2 *__restrict__ acc, int ks,
                               size_t ks_stride, int N, const double *__restrict__ delays, int npc, int maxpc,
                               const UvFreq *__restrict__ freqs, int rsl, float2 *__restrict__ results)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const UvEntry e = ents[blockIdx.y];
  float2 v = make_float2(0.f, 0.f);
  for (int k = 0; k < ks; k++) {
    const float2 a = acc[(size_t)k * ks_stride + e.acc_index + c];
    v.x += a.x;
    v.y += a.y;
  }
  if (e.conj) v.y = -v.y;
  if (e.stride == 0) {
    float2 &r = results[e.ro + c];
    r.x += v.x;
    r.y += v.y;
    return;
  }
  const UvFreq F = freqs[e.freq];
  const double stepbw = rsl * F.chanbw;
  const int cr = c % rsl, cs = c / rsl, nsteps = F.nchan / rsl;
  const double f1 = F.lsb ? -(double)(rsl - (cr + 1)) * F.chanbw : cr * F.chanbw;
  const double f2 = F.lsb ? -(double)(nsteps - (cs + 1)) * stepbw : cs * stepbw;
  for (int s = 0; s < npc; s++) {
    const double d = delays[(size_t)e.baseline * maxpc + s];
    float2 out = v;
    if (fabs(d) > 1.0e-20) {
      double edgeturns = d * F.lofreq;
      edgeturns -= floor(edgeturns);
      const double t1 = d * f1 + edgeturns, t2 = d * f2;
      const float a1 = (float)((t1 - floor(t1)) * GX_TWO_PI), a2 = (float)((t2 - floor(t2)) * GX_TWO_PI);
      float s1, c1, s2, c2;
      sincosf(a1, &s1, &c1);
      sincosf(a2, &s2, &c2);
      out = cmul_exact(make_float2(c1, s1), v);      // rotator x data
      out = cmul_exact(out, make_float2(c2, s2));    // times the step rotator
    }
    float2 &r = results[e.ro + (size_t)s * e.stride + c];
    r.x += out.x;
    r.y += out.y;
  }
}

cudaError_t uvshift_launch(const UvEntry *ents, int nents, const float2 *acc, int ks, size_t ks_stride, int N,
                           const double *delays, int npc, int maxpc, const UvFreq *freqs, int rsl, float2 *results,
                           cudaStream_t st)
{
  if (nents <= 0) return cudaSuccess;
  if (nents > 65535) return cudaErrorInvalidConfiguration;
  dim3 grid((N + 127) / 128, nents);
  uvshift_kernel<<<grid, 128, 0, st>>>(ents, acc, ks, ks_stride, N, delays, npc, maxpc, freqs, rsl, results);
  return cudaGetLastError();
}

__global__ void copy_floats_kernel(const float *__restrict__ vals, long long n, float *__restrict__ out)
{
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = vals[i];
}

cudaError_t copy_floats_launch(const float *vals, long long n, float *results_f, long long first, cudaStream_t st)
{
  if (n <= 0) return cudaSuccess;
  copy_floats_kernel<<<(unsigned)std::min<long long>((n + 255) / 256, 1024), 256, 0, st>>>(vals, n, results_f + first);
  return cudaGetLastError();
}

// The pulsar bin of a channel (Polyco::getBins, polyco.cpp:196-222): the
// fractional part of the mean phase plus the channel's dispersion offset,
// bin 0 outside [first end, last end), else the bin whose phase range holds it.
__device__ __forceinline__ int pulsar_bin(double avgphase, double dmoff, const double *__restrict__ bp, int nbins)
{
  const double ap = dmoff + avgphase;
  const double m = ap - floor(ap);
  if (m < bp[0] || m >= bp[nbins - 1]) return 0;
  int bin = 0;
  for (int k = nbins - 1; k > 0; k--)
    if (m < bp[k] && m >= bp[k - 1]) bin = k;
  return bin;
}

__global__ void binned_xmac_kernel(const BinEntry *__restrict__ ents, const float2 *__restrict__ spec, int NI, int N,
                                   int nblk, int b0, const double *__restrict__ avgphase,
                                   const double *__restrict__ dmoff, const double *__restrict__ bp, int nbins,
                                   float2 *__restrict__ acc)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const BinEntry e = ents[blockIdx.y];
  const size_t bstride = (size_t)NI * N;
  const float2 *xa = spec + ((size_t)e.f * nblk * NI + e.a) * N + c;
  const float2 *xb = spec + ((size_t)e.f * nblk * NI + e.b) * N + c;
  const double dm = dmoff[(size_t)e.f * N + c];
  float2 *row = acc + (size_t)blockIdx.y * nbins * N + c;
  // the current bin's accumulator is carried in registers: the same additions,
  // in block order, as adding into it in memory block by block (core.cpp:943-950)
  int cur = -1;
  float2 sum = make_float2(0.f, 0.f);
  for (int k = 0; k < nblk; k++) {
    const int bin = pulsar_bin(avgphase[b0 + k], dm, bp, nbins);
    if (bin != cur) {
      if (cur >= 0) row[(size_t)cur * N] = sum;
      cur = bin;
      sum = row[(size_t)cur * N];
    }
    const float2 x1 = xa[k * bstride], x2 = xb[k * bstride];
    const float2 p = cmul_exact(x1, make_float2(x2.x, -x2.y));   // vis1 x conj(vis2) (vectorMul_cf32)
    sum.x = __fadd_rn(sum.x, p.x);
    sum.y = __fadd_rn(sum.y, p.y);
  }
  if (cur >= 0) row[(size_t)cur * N] = sum;
}

cudaError_t binned_xmac_launch(const BinEntry *ents, int nents, const float2 *spec, int NI, int N, int nblk, int b0,
                               const double *avgphase, const double *dmoff, const double *binphases, int nbins,
                               float2 *acc, cudaStream_t st)
{
  if (nents <= 0 || nblk <= 0) return cudaSuccess;
  if (nents > 65535) return cudaErrorInvalidConfiguration;
  dim3 grid((N + 127) / 128, nents);
  binned_xmac_kernel<<<grid, 128, 0, st>>>(ents, spec, NI, N, nblk, b0, avgphase, dmoff, binphases, nbins, acc);
  return cudaGetLastError();
}

// One thread per (item, bin); the scrunched sum is bin 0's thread.
__global__ void binned_weights_kernel(const BinWeightItem *__restrict__ items, int nitems, const float *__restrict__ w,
                                      int nblk, int b0, int N, int nbuf, int xstride, const double *__restrict__ avgphase,
                                      const double *__restrict__ dmoff, const double *__restrict__ bp,
                                      const double *__restrict__ bw, int nbins, int scrunch, float *__restrict__ wbins)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int fj = t / nbins, mybin = t % nbins;
  if (fj >= nitems || (scrunch && mybin != 0)) return;
  const BinWeightItem it = items[fj];
  const double *dm = dmoff + (size_t)it.f * N;
  float acc = wbins[t];
  const int nstr = (N + xstride - 1) / xstride;
  // buffered-FFT groups of the subint (core.cpp:784-800), xmac strides, blocks, channels
  for (int g0 = 0; g0 < nblk; g0 += nbuf) {
    const int g1 = min(nblk, g0 + nbuf);
    for (int x = 0; x < nstr; x++) {
      const int c0 = x * xstride, c1 = min(N, c0 + xstride);
      for (int k = g0; k < g1; k++) {
        const float bweight = w[(size_t)it.s1 * nblk + k] * w[(size_t)it.s2 * nblk + k] / N;
        const double ap = avgphase[b0 + k];
        for (int c = c0; c < c1; c++) {
          const int bin = pulsar_bin(ap, dm[c], bp, nbins);
          if (scrunch) {
            if (bw[bin] > 0.0) acc = (float)((double)acc + bweight * bw[bin]);
          } else if (bin == mybin) {
            acc = __fadd_rn(acc, bweight);
          }
        }
      }
    }
  }
  wbins[t] = acc;
}

cudaError_t binned_weights_launch(const BinWeightItem *items, int nitems, const float *w, int nblk, int b0, int N,
                                  int nbuf, int xmacstride, const double *avgphase, const double *dmoff,
                                  const double *binphases, const double *binweights, int nbins, int scrunch,
                                  float *wbins, cudaStream_t st)
{
  if (nitems <= 0 || nblk <= 0) return cudaSuccess;
  const int n = nitems * nbins;
  binned_weights_kernel<<<(n + 63) / 64, 64, 0, st>>>(items, nitems, w, nblk, b0, N, nbuf, xmacstride, avgphase, dmoff,
                                                      binphases, binweights, nbins, scrunch, wbins);
  return cudaGetLastError();
}

__global__ void binned_finalise_kernel(const BinEntry *__restrict__ ents, const float2 *__restrict__ acc, int N,
                                       int nbins, int scrunch, const double *__restrict__ bw,
                                       float2 *__restrict__ results)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const BinEntry e = ents[blockIdx.y];
  const float2 *row = acc + (size_t)blockIdx.y * nbins * N + c;
  if (!scrunch) {
    for (int b = 0; b < nbins; b++) results[e.ro + (size_t)(b * e.npol + e.p) * N + c] = row[(size_t)b * N];
    return;
  }
  // each bin scaled by its (FP32) weight, then added in bin order (core.cpp:1439-1470, 1808-1823)
  float2 s = make_float2(0.f, 0.f);
  for (int b = 0; b < nbins; b++) {
    const float wf = (float)bw[b];
    const float2 v = row[(size_t)b * N];
    s.x = __fadd_rn(s.x, __fmul_rn(v.x, wf));
    s.y = __fadd_rn(s.y, __fmul_rn(v.y, wf));
  }
  results[e.ro + (size_t)e.p * N + c] = s;
}

__global__ void binned_weights_out_kernel(const BinWeightOut *__restrict__ wo, int n, const float *__restrict__ wbins,
                                          int nbins, float *__restrict__ results_f)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const BinWeightOut x = wo[i];
  results_f[x.float_index] = wbins[(size_t)x.fj * nbins + x.bin];
}

cudaError_t binned_finalise_launch(const BinEntry *ents, int nents, const float2 *acc, int N, int nbins, int scrunch,
                                   const double *binweights, const BinWeightOut *wout, int nwout, const float *wbins,
                                   float2 *results, cudaStream_t st)
{
  if (nents > 65535) return cudaErrorInvalidConfiguration;
  if (nents > 0) {
    dim3 grid((N + 127) / 128, nents);
    binned_finalise_kernel<<<grid, 128, 0, st>>>(ents, acc, N, nbins, scrunch, binweights, results);
  }
  if (nwout > 0)
    binned_weights_out_kernel<<<(nwout + 255) / 256, 256, 0, st>>>(wout, nwout, wbins, nbins,
                                                                   reinterpret_cast<float *>(results));
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
