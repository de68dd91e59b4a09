// gx_subint_device_noalloc: one subint through the same F-step / X-step /
// finalise kernels as gx_subint_device, for callers that cannot allocate
// device memory.
//
// Who needs this: host frameworks that hand every byte of device memory to
// their own allocator and only pass buffers in, and threads that must not
// call cudaMalloc/cudaFree because those calls can wait for the whole device
// (every stream), not only for the caller's own work.  Such a caller passes
// device inputs and a device result buffer; everything else this path needs
// -- the per-station tables, twiddles, control words, spectra, accumulators
// and weights -- lives in one fixed scratch array in device global memory,
// declared below.
//
// The scratch array is GX_NOALLOC_SCRATCH_BYTES (64 MiB).  Every GPU on which
// this library's device code is loaded holds that array until the process
// exits.  Jobs whose tables and accumulators do not fit are rejected with
// GX_ERR_UNSUPPORTED and a message giving the bytes needed; the spectra
// buffer is sized down (fewer FFT blocks per pass) to fit what is left.
//
// Set-up: the first call on a device asks the runtime for the array's device
// address on that device (cudaGetSymbolAddress, with the device current) and
// keeps it for later calls; make that first call before any stream capture
// begins on the device.  The kept address is not looked up again, so the
// device must not be reset (cudaDeviceReset) while this library is in use.
//
// The per-call tables are copied from pageable host memory, so a call may
// wait for work already queued on `stream` before it returns.
//
// All calls share the one array and each call leaves its contents behind;
// every region that must start at zero is cleared on the caller's stream at
// the start of the call.  Two calls whose work overlaps on the GPU (on
// different streams, or from different host threads without ordering) race
// on the array and corrupt each other's results: order them on one stream.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "../../include/gxcorr.h"
#include "gx_dev.h"
#include "gx_plan.h"
#include "gx_xstep.h"

namespace {

constexpr size_t kScratchBytes = GX_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void *g_scratch[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device.  The host-side
// symbol is only a stand-in, so the address is asked of the runtime once per
// device, with that device current (the first call on the device).
cudaError_t scratch_address(int dev, unsigned char **out)
{
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch[dev] = p;
  }
  *out = static_cast<unsigned char *>(g_scratch[dev]);
  return cudaSuccess;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

void set_err(char *err, int errlen, const std::string &m)
{
  if (err && errlen > 0) {
    strncpy(err, m.c_str(), (size_t)errlen - 1);
    err[errlen - 1] = '\0';
  }
}

}  // namespace

using namespace gx;

extern "C" gx_status gx_subint_device_noalloc(const gx_job_desc *desc, const gx_subint_desc *sub, float *dev_results,
                                              void *stream, char *err, int errlen)
{
  if (!desc || !sub || !dev_results || !sub->data || !sub->datalen || !sub->control) {
    set_err(err, errlen, "null descriptor or buffer");
    return GX_ERR_ARG;
  }
  if (!sub->interp) {
    set_err(err, errlen, "interpolators are required (there is no delay model without a handle)");
    return GX_ERR_ARG;
  }
  if (desc->xstep != GX_XSTEP_FP32) {
    set_err(err, errlen, "the no-allocation entry point runs the FP32 X-step only");
    return GX_ERR_UNSUPPORTED;
  }
  JobPlan plan;
  std::string perr;
  gx_status ps = plan_job(desc, &plan, perr);
  if (ps != GX_OK) {
    set_err(err, errlen, perr);
    return ps;
  }
  const DevJob &J0 = plan.J;
  const int nst = J0.nstations, nbl = desc->nbaselines;
  if (sub->controllen < plan.ctrlstride) {
    set_err(err, errlen, "control buffer shorter than 3 + flag words");
    return GX_ERR_ARG;
  }

  // carve the scratch array: fixed tables first, then the per-block buffers
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off = align256(off + bytes); return o; };
  const size_t o_st = take(sizeof(DevStation) * nst);
  const size_t o_tw = take(sizeof(float2) * plan.twiddle.size());
  const size_t o_ctrl = take(sizeof(int32_t) * plan.ctrlstride * nst);
  const size_t o_len = take(sizeof(int64_t) * nst);
  const size_t o_ptr = take(sizeof(uint8_t *) * nst);
  const size_t o_interp = take(sizeof(double) * 3 * nst);
  const size_t o_clock = take(sizeof(SubintClock));
  const size_t o_pairs = take(sizeof(int2) * (nbl > 0 ? nbl : 1));
  const size_t o_prods = take(sizeof(ProdEntry) * (plan.prods.empty() ? 1 : plan.prods.size()));
  const size_t o_went = take(sizeof(WeightEntry) * (plan.wents.empty() ? 1 : plan.wents.size()));
  const size_t o_wacc = take(sizeof(float) * (nst + nbl));
  const size_t acc_slice = (size_t)J0.nfreqs * plan.xs.npairs * plan.xs.ST * plan.xs.ST * J0.nchan;
  int ks = plan.ks;
  const size_t per_block = sizeof(float2) * (size_t)J0.nfreqs * J0.ninputs * J0.nchan +
                           (sizeof(float) + sizeof(BlockParam)) * nst + 512;
  size_t fixed = off + align256(sizeof(float2) * acc_slice * ks);
  if (fixed + per_block + 512 > kScratchBytes && ks > 1) {
    ks = 1;
    fixed = off + align256(sizeof(float2) * acc_slice);
  }
  if (fixed + per_block + 512 > kScratchBytes) {
    char m[256];
    snprintf(m, sizeof(m), "job needs at least %zu bytes of scratch; the no-allocation limit is %zu bytes",
             fixed + per_block + 512, kScratchBytes);
    set_err(err, errlen, m);
    return GX_ERR_UNSUPPORTED;
  }
  int chunk = (int)std::min<size_t>((size_t)J0.blocks_per_send, (kScratchBytes - fixed - 512) / per_block);
  if (chunk > 4096) chunk = 4096;
  ks = std::max(1, std::min(ks, chunk / 16 > 0 ? chunk / 16 : 1));
  const size_t o_acc = take(sizeof(float2) * acc_slice * ks);
  const size_t o_w = take(sizeof(float) * (size_t)nst * chunk);
  const size_t o_bp = take(sizeof(BlockParam) * (size_t)nst * chunk);
  const size_t spec_bytes = sizeof(float2) * (size_t)J0.nfreqs * chunk * J0.ninputs * J0.nchan;
  const size_t o_spec = take(spec_bytes);
  if (off > kScratchBytes) {
    set_err(err, errlen, "scratch layout exceeds the no-allocation limit");
    return GX_ERR_UNSUPPORTED;
  }

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  unsigned char *base = nullptr;
  if (e == cudaSuccess) e = scratch_address(dev, &base);
  if (e != cudaSuccess) {
    set_err(err, errlen, std::string("scratch address: ") + cudaGetErrorString(e));
    return GX_ERR_CUDA;
  }
  cudaStream_t st = (cudaStream_t)stream;
  DevJob J = J0;
  J.twiddle = reinterpret_cast<const float2 *>(base + o_tw);
  DevStation *d_st = reinterpret_cast<DevStation *>(base + o_st);
  int32_t *d_ctrl = reinterpret_cast<int32_t *>(base + o_ctrl);
  int64_t *d_len = reinterpret_cast<int64_t *>(base + o_len);
  const uint8_t **d_ptr = reinterpret_cast<const uint8_t **>(base + o_ptr);
  double *d_interp = reinterpret_cast<double *>(base + o_interp);
  SubintClock *d_clock = reinterpret_cast<SubintClock *>(base + o_clock);
  int2 *d_pairs = reinterpret_cast<int2 *>(base + o_pairs);
  ProdEntry *d_prods = reinterpret_cast<ProdEntry *>(base + o_prods);
  WeightEntry *d_went = reinterpret_cast<WeightEntry *>(base + o_went);
  float *d_wacc = reinterpret_cast<float *>(base + o_wacc);
  float2 *d_acc = reinterpret_cast<float2 *>(base + o_acc);
  float *d_w = reinterpret_cast<float *>(base + o_w);
  BlockParam *d_bp = reinterpret_cast<BlockParam *>(base + o_bp);
  float2 *d_spec = reinterpret_cast<float2 *>(base + o_spec);

  // per-call tables (host sources are staged by the copy calls before they return)
  std::vector<int32_t> ctrl((size_t)plan.ctrlstride * nst, 0);
  std::vector<int64_t> lens(nst);
  for (int s = 0; s < nst; s++) {
    memcpy(&ctrl[(size_t)s * plan.ctrlstride], sub->control[s], sizeof(int32_t) * plan.ctrlstride);
    lens[s] = sub->datalen[s];
  }
#define NA_CK(call)                                                        \
  do {                                                                     \
    cudaError_t _e = (call);                                               \
    if (_e != cudaSuccess) {                                               \
      set_err(err, errlen, std::string(#call ": ") + cudaGetErrorString(_e)); \
      return GX_ERR_CUDA;                                                  \
    }                                                                      \
  } while (0)
  NA_CK(cudaMemcpyAsync(d_st, plan.stations.data(), sizeof(DevStation) * nst, cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemcpyAsync((void *)J.twiddle, plan.twiddle.data(), sizeof(float2) * plan.twiddle.size(),
                        cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemcpyAsync(d_ctrl, ctrl.data(), sizeof(int32_t) * ctrl.size(), cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemcpyAsync(d_len, lens.data(), sizeof(int64_t) * nst, cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemcpyAsync(d_ptr, sub->data, sizeof(uint8_t *) * nst, cudaMemcpyHostToDevice, st));
  NA_CK(cudaMemcpyAsync(d_interp, sub->interp, sizeof(double) * 3 * nst, cudaMemcpyHostToDevice, st));
  const SubintClock clock{sub->sec, sub->ns, sub->scan_start_sec};
  NA_CK(cudaMemcpyAsync(d_clock, &clock, sizeof(clock), cudaMemcpyHostToDevice, st));
  if (nbl > 0) NA_CK(cudaMemcpyAsync(d_pairs, plan.pairs.data(), sizeof(int2) * nbl, cudaMemcpyHostToDevice, st));
  if (!plan.prods.empty())
    NA_CK(cudaMemcpyAsync(d_prods, plan.prods.data(), sizeof(ProdEntry) * plan.prods.size(), cudaMemcpyHostToDevice, st));
  if (!plan.wents.empty())
    NA_CK(cudaMemcpyAsync(d_went, plan.wents.data(), sizeof(WeightEntry) * plan.wents.size(), cudaMemcpyHostToDevice, st));
  // regions that must start at zero: accumulators, weight sums, the spectra
  // (its padding rows are never written by the F-step) and the results
  NA_CK(cudaMemsetAsync(d_acc, 0, sizeof(float2) * acc_slice * ks, st));
  NA_CK(cudaMemsetAsync(d_wacc, 0, sizeof(float) * (nst + nbl), st));
  NA_CK(cudaMemsetAsync(d_spec, 0, spec_bytes, st));
  NA_CK(cudaMemsetAsync(dev_results, 0, sizeof(float2) * plan.result_length, st));

  SubintArrays S{};
  S.clock = d_clock;
  S.data = d_ptr;
  S.datalen = d_len;
  S.control = d_ctrl;
  S.controlstride = plan.ctrlstride;
  S.interp = d_interp;
  for (int b0 = 0; b0 < J.blocks_per_send; b0 += chunk) {
    const int nb = std::min(chunk, J.blocks_per_send - b0);
    NA_CK(fstep_launch(J, d_st, plan.maxnrf, S, b0, nb, plan.nslots, d_spec, d_w, d_bp, st));
    NA_CK(xmac_fp32_launch(d_spec, nb, J.ninputs, J.nchan, J.nfreqs, ks, d_acc, nullptr, st));
    NA_CK(weights_launch(d_w, nb, nst, d_pairs, nbl, d_wacc, st));
  }
  NA_CK(finalise_launch(d_prods, (int)plan.prods.size(), d_acc, ks, acc_slice, J.nchan, d_went,
                        (int)plan.wents.size(), d_wacc, reinterpret_cast<float2 *>(dev_results), st));
#undef NA_CK
  set_err(err, errlen, "");
  return GX_OK;
}
