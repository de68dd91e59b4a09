// Tensor-core X-step: the cross-multiply-accumulate of Core::processdata
// (mpifxcorr/src/core.cpp:784-1053; the product vis1 * conj(vis2) of
// vectorAddProduct_cf32 at core.cpp:963, summed over the FFT blocks of a
// subint) on the 5th-generation tensor cores: tcgen05.mma with FP16 operands
// and FP32 accumulators in tensor memory.
//
// For one frequency and one channel the blocks of a chunk form the NI x K
// complex matrix X = Xr + i Xi (row a: input a, column k: FFT block k), and the
// visibilities of every input pair are V = X X^H:
//     Re V = Xr Xr^T + Xi Xi^T,    Im V(a, b) = P(a, b) - P(b, a),  P = Xi Xr^T.
// Each CTA owns one frequency and one pair of channels and keeps, per channel, a
// 128-lane x 256-column FP32 accumulator in tensor memory: columns 0..127 hold
// Re V, columns 128..255 hold P.  Per step of 16 FFT blocks and channel:
//     D[:, 0:256) += Xi [Xi ; Xr]^T      (M = 128, N = 256, K = 16)
//     D[:, 0:128) += Xr Xr^T             (M = 128, N = 128, K = 16)
// i.e. three 128x128x16 real products per complex 128x128 Hermitian update
// (the fourth, Xr Xi^T, is P transposed and is formed in the finalising pass).
//
// Data path per CTA: the spectra spec[freq][block][input][chan] (float2, as the
// F-step writes them) are read as a 4-D FP32 tensor; one TMA tile load (no
// multicast) per 16 blocks fetches the 4 floats of the CTA's channel pair for
// all 128 inputs ([block][input][16 bytes], blocks past the chunk and rows
// past the job's inputs read as zeros) into a 4-stage FP32 ring.  The CTA's
// warps have roles joined only by mbarriers: one lane of warp 0 issues the
// tile loads as stages free up; eight converter warps scale each value by a
// power of two per (input, channel), round it to FP16 and store it, transposed
// to K-major, into the canonical no-swizzle core-matrix layout of the MMA
// operand [Xi ; Xr] (256 rows x 16 blocks) of a 2-stage operand ring; one lane
// of warp 1 issues the MMAs of a stage and commits them to the mbarrier that
// frees it.  Loads, conversion and MMAs of neighbouring tiles overlap.  In the split form the FP16
// remainder lo = fp16(x*s - hi) is kept too and the products hi*hi + hi*lo +
// lo*hi are accumulated (lo*lo, below 2^-22 relative, is dropped).
//
// The accumulators leave tensor memory once per chunk.  P of both channels is
// parked in shared memory (rows padded to 129 floats, conflict-free by row and
// by column), so that each thread, holding row a of Re, forms
// Im V(a, b) = P(a, b) - P(b, a), divides out the operand scales and adds the
// complex visibilities of both channels, one float4 per (a, b), into
// acc[freq][chan/2][a][b]; partial sums across chunks and K-split slices stay
// FP32 and the finalising pass reads whole rows.
//
// Every wait on an mbarrier is bounded in time; on expiry the kernel records a
// nonzero status in *err, drains its own copies and MMAs (again bounded),
// releases its tensor memory and returns.
#include <cstdint>
#include <cstdlib>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include "gx_xstep.h"
#include "gx_mbar.cuh"

namespace gx {
namespace {

constexpr int kNI = 128;                     // inputs per frequency = MMA M
constexpr int kKT = 16;                      // FFT blocks per K-tile = one MMA K step for FP16
constexpr int kOpStages = 2;                 // FP16 operand stages
constexpr uint32_t kTmemCols = 512;          // 2 channels x (128 Re + 128 P) FP32 columns
constexpr uint32_t kRowBytes = kNI * 16;     // one block of a channel pair: 128 inputs x 2 channels x float2
constexpr uint32_t kLBO = 128;               // byte step between the two 8-block core matrices of a row group
constexpr uint32_t kSBO = (kKT / 8) * 128;   // byte step between 8-row groups
constexpr uint32_t kOpChanBytes = 2 * kNI * kKT * 2;      // [Xi ; Xr]: 256 rows x 16 FP16 = 8 KB
constexpr uint32_t kXrOffset = (kNI / 8) * kSBO;          // rows 128.. (Xr) start here
constexpr int kPRow = kNI + 1;               // padded row of the P matrices parked in shared memory
constexpr int kVCols = 8;                    // columns of V per epilogue slice (one 128-byte line per row)
constexpr int kVRow = kVCols + 1;            // padded slice row, float4
// FP32 staging ring: RP channel pairs per tile row (RP = 2: whole 32-byte
// sectors, half the row requests of RP = 1), as many stages as fit beside the
// operand stages.
template <bool HILO, int RP>
struct TcRing {
  static constexpr uint32_t kStageBytes = kKT * kRowBytes * RP;   // 32 or 64 KB
  static constexpr int kStages = RP == 1 ? 4 : (HILO ? 2 : 3);
  static constexpr uint32_t kOpStageBytes = (HILO ? 2 : 1) * 2 * kOpChanBytes;
  static_assert((2 * kNI * kPRow + 2 * kNI) * 4 + kNI * kVRow * 16 <= kStages * kStageBytes + kOpStages * kOpStageBytes,
                "epilogue tables must fit in the staging ring and operand stages");
};
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
               : "memory");
}

__device__ __forceinline__ void tmem_relinquish()
{
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, FP16 operands, FP32 accumulator.
__device__ __forceinline__ void mma_f16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// 32 lanes x 16 consecutive FP32 columns: thread i of the warp gets lane (base lane + i).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// 32 lanes x 4 consecutive FP32 columns.
__device__ __forceinline__ void tmem_ld4(uint32_t taddr, float (&v)[4])
{
  uint32_t r[4];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 4; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory operand descriptor, K-major without swizzle: 8-row x 16-byte
// core matrices, kLBO between the two core matrices of a K step, kSBO between
// 8-row groups; version 1 (bits 46-47) as tcgen05 requires.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr)
{
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(kLBO >> 4) << 16) | ((uint64_t)(kSBO >> 4) << 32) |
         (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), FP16 A
// and B (formats 0), both K-major, N >> 3 at bit 17, M >> 4 at bit 24 (M = 128).
__host__ __device__ constexpr uint32_t idesc_f16(int n)
{
  return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kNI >> 4) << 24);
}

__device__ __forceinline__ uint32_t pack_half2(float a, float b)
{
  const __half2 h = __floats2half2_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&h);
}

// hi = fp16(a), lo = fp16(a - hi): a - hi is exact in FP32.
__device__ __forceinline__ void split2(float a, float b, uint32_t &hi, uint32_t &lo)
{
  const __half2 h = __floats2half2_rn(a, b);
  const float2 hf = __half22float2(h);
  const __half2 l = __floats2half2_rn(a - hf.x, b - hf.y);
  hi = *reinterpret_cast<const uint32_t *>(&h);
  lo = *reinterpret_cast<const uint32_t *>(&l);
}


// Warp roles: warp 0 lane 0 issues the tile loads, warp 1 lane 0 issues the
// MMAs, warps 2..9 (kConvThreads threads) convert the staged FP32 tiles to FP16
// operands and later run the epilogue.  The roles hand stages to each other
// through mbarriers only, so a tile's load, conversion and MMAs overlap those
// of its neighbours.
constexpr int kConvThreads = 256;            // converter threads that also run the epilogue
constexpr int kConvWarp0 = 2;
// threads of a CTA with CW converter warps: 1 load warp, 1 MMA warp, CW converters
__host__ __device__ constexpr int tc_threads(int cw) { return 32 * (kConvWarp0 + cw); }
constexpr int kMaxStages = 4;
constexpr int kNumBars = 2 * kMaxStages + 2 * kOpStages + 1;   // full, empty, opfull, opempty, done

template <bool HILO, int RP, int CW>
__global__ void __launch_bounds__(tc_threads(CW), 1)
xmac_tc_kernel(const __grid_constant__ CUtensorMap spec_map, int nblk, int NP, int nfreqs, int ks, int ninputs,
               const float *__restrict__ scale, float4 *__restrict__ acc, int accumulate, int *__restrict__ err)
{
  constexpr int kStages = TcRing<HILO, RP>::kStages;
  constexpr uint32_t kStageBytes = TcRing<HILO, RP>::kStageBytes;
  constexpr uint32_t kOpStageBytes = TcRing<HILO, RP>::kOpStageBytes;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char *staging = smem;
  unsigned char *ops = smem + kStages * kStageBytes;
  uint64_t *bars = reinterpret_cast<uint64_t *>(ops + kOpStages * kOpStageBytes);
  uint64_t *full = bars, *empty = bars + kMaxStages, *opfull = bars + 2 * kMaxStages;
  uint64_t *opempty = opfull + kOpStages, *done = opempty + kOpStages;
  uint32_t *s_tmem = reinterpret_cast<uint32_t *>(bars + kNumBars);
  volatile int *s_abort = reinterpret_cast<volatile int *>(s_tmem + 1);

  const int p = blockIdx.x, f = blockIdx.y, z = blockIdx.z;
  const int N = 2 * NP;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntile_all = (nblk + kKT - 1) / kKT;
  const int t0 = (int)((long long)ntile_all * z / ks);
  const int nt = (int)((long long)ntile_all * (z + 1) / ks) - t0;
  const int nconv_warps = CW;

  if (tid == 0) {
    for (int i = 0; i < kStages; i++) {
      mbar_init(smem_u32(full + i), 1);
      mbar_init(smem_u32(empty + i), nconv_warps);
    }
    for (int i = 0; i < kOpStages; i++) {
      mbar_init(smem_u32(opfull + i), nconv_warps);
      mbar_init(smem_u32(opempty + i), 1);
    }
    mbar_init(smem_u32(done), 1);
    *s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    tmem_alloc(smem_u32(s_tmem), kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *s_tmem;
  auto abort_with = [&](int code) {
    *s_abort = 1;
    atomicExch(err, code);
  };

  int issued = 0, mmas = 0;
  if (warp == 0 && lane == 0) {
    // ---- producer: tile u into stage u % kStages once its previous tile was converted
    for (int u = 0; u < nt; u++) {
      if (*s_abort) break;
      const int st = u % kStages;
      if (u >= kStages && !mbar_wait(smem_u32(empty + st), (uint32_t)(u / kStages - 1) & 1u)) {
        abort_with(3);
        break;
      }
      const uint32_t bar = smem_u32(full + st);
      mbar_expect_tx(bar, kStageBytes);
      tma_load_4d(smem_u32(staging + st * kStageBytes), &spec_map, 4 * RP * (p / RP), 0, (t0 + u) * kKT, f, bar);
      issued = u + 1;
    }
  } else if (warp == 1 && lane == 0) {
    // ---- MMA issuer: operand stage t % kOpStages once converted; its commit frees the stage
    for (int t = 0; t < nt; t++) {
      if (*s_abort) break;
      const int o = t % kOpStages;
      if (!mbar_wait(smem_u32(opfull + o), (uint32_t)(t / kOpStages) & 1u)) {
        abort_with(4);
        break;
      }
      tc_fence_after();
      const uint32_t opb = smem_u32(ops + o * kOpStageBytes);
#pragma unroll
      for (int e = 0; e < 2; e++) {
        const uint32_t d = tmem + (uint32_t)e * 256u;
        const uint32_t hb = opb + (uint32_t)e * kOpChanBytes;
        const uint64_t xi = smem_desc(hb), xr = smem_desc(hb + kXrOffset);
        mma_f16(d, xi, xi, idesc_f16(256), t > 0 ? 1u : 0u);
        mma_f16(d, xr, xr, idesc_f16(128), 1u);
        if (HILO) {
          const uint32_t lb = opb + (2u + (uint32_t)e) * kOpChanBytes;
          const uint64_t li = smem_desc(lb), lr = smem_desc(lb + kXrOffset);
          mma_f16(d, xi, li, idesc_f16(256), 1u);
          mma_f16(d, li, xi, idesc_f16(256), 1u);
          mma_f16(d, xr, lr, idesc_f16(128), 1u);
          mma_f16(d, lr, xr, idesc_f16(128), 1u);
        }
      }
      mma_commit(smem_u32(opempty + o));
      mmas = t + 1;
    }
    if (!*s_abort && mmas == nt && nt > 0) mma_commit(smem_u32(done));
  } else if (warp >= kConvWarp0) {
    // ---- converters: row r, blocks k0 .. k0 + BPT - 1 of each tile
    constexpr int BPT = 64 / CW;   // blocks per thread: 8 (8 warps) or 4 (16 warps)
    constexpr int NW = BPT / 2;    // half2 words per quantity
    const int ct = tid - kConvWarp0 * 32;
    const int r = ct & (kNI - 1), k0 = (ct >> 7) * BPT;
    const float s0 = scale[((size_t)f * kNI + r) * N + 2 * p];
    const float s1 = scale[((size_t)f * kNI + r) * N + 2 * p + 1];
    const uint32_t row_off = (uint32_t)(r >> 3) * kSBO + (uint32_t)(k0 >> 3) * kLBO + (uint32_t)(r & 7) * 16 +
                             (uint32_t)(k0 & 7) * 2;
    for (int t = 0; t < nt; t++) {
      if (*s_abort) break;
      const int st = t % kStages, o = t % kOpStages;
      if (!mbar_wait(smem_u32(full + st), (uint32_t)(t / kStages) & 1u)) {
        abort_with(1);
        break;
      }
      const int kv = min(kKT, nblk - (t0 + t) * kKT);
      // row (k, r) of the stage holds RP channel pairs; this CTA's is pair p % RP
      const float4 *stg = reinterpret_cast<const float4 *>(staging + st * kStageBytes) + (p % RP);
      uint32_t re0[NW], im0[NW], re1[NW], im1[NW];
      uint32_t lre0[NW], lim0[NW], lre1[NW], lim1[NW];
#pragma unroll
      for (int j = 0; j < NW; j++) {
        const int k = k0 + 2 * j;
        const float4 zero = make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 a = (k < kv) ? stg[(k * kNI + r) * RP] : zero;   // (c0.re, c0.im, c1.re, c1.im) at block k
        const float4 b = (k + 1 < kv) ? stg[((k + 1) * kNI + r) * RP] : zero;
        if (HILO) {
          split2(a.x * s0, b.x * s0, re0[j], lre0[j]);
          split2(a.y * s0, b.y * s0, im0[j], lim0[j]);
          split2(a.z * s1, b.z * s1, re1[j], lre1[j]);
          split2(a.w * s1, b.w * s1, im1[j], lim1[j]);
        } else {
          re0[j] = pack_half2(a.x * s0, b.x * s0);
          im0[j] = pack_half2(a.y * s0, b.y * s0);
          re1[j] = pack_half2(a.z * s1, b.z * s1);
          im1[j] = pack_half2(a.w * s1, b.w * s1);
        }
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(empty + st));   // the staging stage may be reloaded
      if (t >= kOpStages && !mbar_wait(smem_u32(opempty + o), (uint32_t)(t / kOpStages - 1) & 1u)) {
        abort_with(2);
        break;
      }
      unsigned char *op = ops + o * kOpStageBytes;
      // channel e, part q at op + (q * 2 + e) * kOpChanBytes; Xi rows 0..127, Xr rows 128..255
      auto put = [&](unsigned char *dst, const uint32_t (&w)[NW]) {
        if constexpr (NW == 4) *reinterpret_cast<uint4 *>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
        else *reinterpret_cast<uint2 *>(dst) = make_uint2(w[0], w[1]);
      };
      put(op + row_off, im0);
      put(op + row_off + kXrOffset, re0);
      put(op + kOpChanBytes + row_off, im1);
      put(op + kOpChanBytes + row_off + kXrOffset, re1);
      if (HILO) {
        unsigned char *lo = op + 2 * kOpChanBytes;
        put(lo + row_off, lim0);
        put(lo + row_off + kXrOffset, lre0);
        put(lo + kOpChanBytes + row_off, lim1);
        put(lo + kOpChanBytes + row_off + kXrOffset, lre1);
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(opfull + o));   // the operand stage may be multiplied
    }
  }
  __syncthreads();
  // all MMAs of the slice have completed once the last commit has arrived
  if (!*s_abort && nt > 0 && tid == 0 && !mbar_wait(smem_u32(done), 0u)) abort_with(5);
  if (*s_abort) {
    // drain: the loads this CTA issued, then the MMAs it committed (bounded)
    if (warp == 0 && lane == 0)
      for (int st = 0; st < kStages && st < issued; st++) {
        const int ulast = st + ((issued - 1 - st) / kStages) * kStages;
        mbar_wait(smem_u32(full + st), (uint32_t)(ulast / kStages) & 1u);
      }
    if (warp == 1 && lane == 0 && mmas > 0)
      mbar_wait(smem_u32(opempty + (mmas - 1) % kOpStages), (uint32_t)((mmas - 1) / kOpStages) & 1u);
  }
  __syncthreads();
  tc_fence_after();

  // the first eight converter warps run the epilogue
  const bool ep = warp >= kConvWarp0 && warp < kConvWarp0 + kConvThreads / 32;
  const int ct = tid - kConvWarp0 * 32;
  if (!*s_abort && !(nt == 0 && accumulate)) {   // an empty slice adds nothing
    // a warp reads tensor-memory lanes 32 (warp % 4) .. +31 (its quadrant), i.e. row a of both accumulators
    const int q = warp & 3, h = (warp - kConvWarp0) >> 2;
    const int a = 32 * q + lane;
    const uint32_t lane_addr = tmem + ((uint32_t)(32 * q) << 16);
    float4 *oblk = acc + (((size_t)z * nfreqs + f) * NP + p) * kNI * kNI;   // [a][b]
    // the staging ring and operand stages are idle now: P of both channels,
    // 1 / scale per (b, channel), and one 8-column slice of V
    float *sP = reinterpret_cast<float *>(staging);                 // [2][128][kPRow]
    float *sInv = sP + 2 * kNI * kPRow;                              // [2][128]
    float4 *sV = reinterpret_cast<float4 *>(sInv + 2 * kNI);         // [128][kVRow]
    const float s0 = ep ? scale[((size_t)f * kNI + a) * N + 2 * p] : 1.0f;
    const float s1 = ep ? scale[((size_t)f * kNI + a) * N + 2 * p + 1] : 1.0f;
    if (nt > 0 && ep) {
      if (h == 1) {
#pragma unroll 1
        for (int cb = 0; cb < kNI / 16; cb++) {
          float v0[16], v1[16];
          tmem_ld16(lane_addr + 128u + (uint32_t)cb * 16u, v0);
          tmem_ld16(lane_addr + 384u + (uint32_t)cb * 16u, v1);
          tmem_ld_wait();
#pragma unroll
          for (int i = 0; i < 16; i++) {
            sP[a * kPRow + cb * 16 + i] = v0[i];
            sP[(kNI + a) * kPRow + cb * 16 + i] = v1[i];
          }
        }
      } else {
        sInv[a] = 1.0f / s0;          // operand scales are powers of two: exact
        sInv[kNI + a] = 1.0f / s1;
      }
    }
    __syncthreads();
    const float ia0 = 1.0f / s0, ia1 = 1.0f / s1;
    // only the job's inputs: rows and 8-column slices beyond them are never read
    const int ncb = (ninputs + kVCols - 1) / kVCols;
#pragma unroll 1
    for (int cb = 0; cb < ncb; cb++) {
      if (ep) {
        // thread (a, h) forms columns b = 8 cb + 4 h + i of row a
        const int b0 = cb * kVCols + h * 4;
        float r0[4] = {0.f, 0.f, 0.f, 0.f}, r1[4] = {0.f, 0.f, 0.f, 0.f};
        if (nt > 0) {
          tmem_ld4(lane_addr + (uint32_t)b0, r0);
          tmem_ld4(lane_addr + 256u + (uint32_t)b0, r1);
          tmem_ld_wait();
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const int b = b0 + i;
          float4 w = make_float4(0.f, 0.f, 0.f, 0.f);
          if (nt > 0) {
            const float i0 = ia0 * sInv[b], i1 = ia1 * sInv[kNI + b];
            const float im0 = sP[a * kPRow + b] - sP[b * kPRow + a];
            const float im1 = sP[(kNI + a) * kPRow + b] - sP[(kNI + b) * kPRow + a];
            w = make_float4(r0[i] * i0, im0 * i0, r1[i] * i1, im1 * i1);
          }
          sV[a * kVRow + h * 4 + i] = w;
        }
      }
      __syncthreads();
      // write the slice back as whole 128-byte lines: 8 consecutive threads per row
      if (ep) {
#pragma unroll
        for (int m = 0; m < kNI * kVCols / kConvThreads; m++) {
          const int i = ct + kConvThreads * m;
          const int row = i / kVCols, col = i % kVCols;
          if (row >= ninputs) continue;
          float4 w = sV[row * kVRow + col];
          float4 *dst = oblk + (size_t)row * kNI + cb * kVCols + col;
          if (accumulate) {
            const float4 old = *dst;
            w.x += old.x;
            w.y += old.y;
            w.z += old.z;
            w.w += old.w;
          }
          *dst = w;
        }
      }
      __syncthreads();
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kTmemCols);
}

// One CTA per (freq, a) row that has visibility rows: passes of kFinPairs
// channel pairs stage acc[z][freq][p][a][bmin..127] (contiguous, summed over
// the K-split slices) in shared memory, then every entry (a, b) of the row
// writes its 2 kFinPairs channels as one contiguous run of the result array.
constexpr int kFinPairs = 16;

__global__ void __launch_bounds__(256)
finalise_tc_kernel(const TcProdEntry *__restrict__ prods, const TcRowEntry *__restrict__ rows,
                   const float4 *__restrict__ acc, int nfreqs, int NP, int ks, int ninputs,
                   float2 *__restrict__ results)
{
  __shared__ float4 sV[kFinPairs][kNI];
  const TcRowEntry R = rows[blockIdx.x];
  const size_t slice = (size_t)nfreqs * NP * kNI * kNI;
  const int nb = ninputs - R.bmin;
  const int ne = R.end - R.start;
  // channel pairs [pb, pe) of this CTA (blockIdx.y of gridDim.y slices)
  const int per = ((NP + gridDim.y - 1) / gridDim.y + kFinPairs - 1) / kFinPairs * kFinPairs;
  const int pb = blockIdx.y * per, pe = min(NP, pb + per);
  for (int p0 = pb; p0 < pe; p0 += kFinPairs) {
    const int np = min(kFinPairs, pe - p0);
    for (int i = threadIdx.x; i < np * nb; i += blockDim.x) {
      const int pp = i / nb, b = R.bmin + i % nb;
      const size_t off = (((size_t)R.freq * NP + p0 + pp) * kNI + R.a) * kNI + b;
      float4 v = acc[off];
      for (int z = 1; z < ks; z++) {
        const float4 u = acc[z * slice + off];
        v.x += u.x;
        v.y += u.y;
        v.z += u.z;
        v.w += u.w;
      }
      sV[pp][b] = v;
    }
    __syncthreads();
    const int nc = 2 * np;
    for (int i = threadIdx.x; i < ne * nc; i += blockDim.x) {
      const TcProdEntry P = prods[R.start + i / nc];
      const int cc = i % nc;
      const float4 v = sV[cc >> 1][P.b];
      results[P.result_offset + 2 * p0 + cc] = (cc & 1) ? make_float2(v.z, v.w) : make_float2(v.x, v.y);
    }
    __syncthreads();
  }
}

}  // namespace


// 4-D FP32 tensor map over a dense row-major array (innermost dimension
// first, strides implied by the dimensions), box `box`, no swizzle, no
// interleave; out-of-bounds elements read as zeros.
cudaError_t tma_map_f32_4d(CUtensorMap *map, const void *base, const cuuint64_t dims[4], const cuuint32_t box[4])
{
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess) return e;
    if (q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const cuuint64_t strides[3] = {dims[0] * 4, dims[0] * 4 * dims[1], dims[0] * 4 * dims[1] * dims[2]};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult cr = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<void *>(base), dims, strides, box, estr,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return cr == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// Channel pairs per staged tile row: 1 (16-byte rows, four stages) unless
// GX_TC_ROW_PAIRS=2 (32-byte rows, fewer stages; measured no faster on C3).
static int tc_row_pairs()
{
  const char *e = getenv("GX_TC_ROW_PAIRS");
  return (e && atoi(e) == 2) ? 2 : 1;
}

size_t xmac_tc_smem_bytes(bool hilo)
{
  const int rp = tc_row_pairs();
  const size_t ring = rp == 1 ? (size_t)TcRing<true, 1>::kStages * TcRing<true, 1>::kStageBytes
                              : (hilo ? (size_t)TcRing<true, 2>::kStages * TcRing<true, 2>::kStageBytes
                                      : (size_t)TcRing<false, 2>::kStages * TcRing<false, 2>::kStageBytes);
  const size_t ops = (size_t)kOpStages * (hilo ? 2 : 1) * 2 * kOpChanBytes;
  return ring + ops + kNumBars * 8 + 16;
}

cudaError_t xmac_tc_launch(const float2 *spec, int nblk, int N, int nfreqs, int ninputs, int ks, bool hilo,
                           const float *scale, float4 *acc, int accumulate, int *err, cudaStream_t st)
{
  if (nblk <= 0) return cudaSuccess;
  if (ninputs < 1 || ninputs > kNI) return cudaErrorInvalidValue;
  // spec[freq][block][row][channel] float2 as a 4-D FP32 tensor (innermost first):
  // {2N floats, ninputs rows, nblk blocks, nfreqs}; box {4 floats, 128 rows, kKT
  // blocks, 1}: the rows beyond the job's inputs (and blocks beyond nblk) are
  // out of bounds, so the copy fills them with zeros without reading memory
  CUtensorMap map;
  const cuuint64_t dims[4] = {(cuuint64_t)(2 * N), (cuuint64_t)ninputs, (cuuint64_t)nblk, (cuuint64_t)nfreqs};
  const int rp = tc_row_pairs();
  const cuuint32_t box[4] = {(cuuint32_t)(4 * rp), (cuuint32_t)kNI, (cuuint32_t)kKT, 1};
  {
    cudaError_t e = tma_map_f32_4d(&map, spec, dims, box);
    if (e != cudaSuccess) return e;
  }
  const size_t sm = xmac_tc_smem_bytes(hilo);
  // converter warps: 8 unless GX_TC_CONV_WARPS=16 (measured no faster on C3)
  const char *ce = getenv("GX_TC_CONV_WARPS");
  const int cw = (ce && atoi(ce) == 16) ? 16 : 8;
  dim3 grid(N / 2, nfreqs, ks);
#define GX_TC_CASE(H, RPV, CWV)                                                                             \
  if (hilo == H && rp == RPV && cw == CWV) {                                                                \
    cudaError_t e = smem_opt_in((const void *)xmac_tc_kernel<H, RPV, CWV>, sm);                             \
    if (e != cudaSuccess) return e;                                                                         \
    xmac_tc_kernel<H, RPV, CWV><<<grid, tc_threads(CWV), sm, st>>>(map, nblk, N / 2, nfreqs, ks, ninputs,   \
                                                                    scale, acc, accumulate, err);           \
    return cudaGetLastError();                                                                              \
  }
  GX_TC_CASE(true, 1, 16) GX_TC_CASE(false, 1, 16) GX_TC_CASE(true, 1, 8) GX_TC_CASE(false, 1, 8)
  GX_TC_CASE(true, 2, 16) GX_TC_CASE(false, 2, 16) GX_TC_CASE(true, 2, 8) GX_TC_CASE(false, 2, 8)
#undef GX_TC_CASE
  return cudaErrorInvalidValue;
}

cudaError_t finalise_tc_launch(const TcProdEntry *prods, const TcRowEntry *rows, int nrows, const float4 *acc,
                               int nfreqs, int N, int ninputs, int ks, float2 *results, cudaStream_t st)
{
  if (nrows <= 0) return cudaSuccess;
  // enough CTAs for several waves: slices of the channel pairs per row
  const int NP = N / 2;
  int slices = 1;
  while ((long long)nrows * slices < 8 * 148 && (slices * 2) * kFinPairs <= NP) slices *= 2;
  finalise_tc_kernel<<<dim3(nrows, slices), 256, 0, st>>>(prods, rows, acc, nfreqs, NP, ks, ninputs, results);
  return cudaGetLastError();
}

}  // namespace gx
