// Monitoring spectra: spectral kurtosis and the STA (autocorrelation) dumps.
//
// With kurtosis dumping on, the reference's Mode adds, for every processed
// FFT block and recorded band, |X|^2 and |X|^4 of every channel of the
// band's spectrum into s1 and s2 (mode.cpp:1237-1254: the FP32 magnitude,
// squared, then squared again), and after its block range turns them into
// the spectral kurtosis n s2 / s1^2 - 1, debiased and averaged down to the
// STA dump channel count (Mode::calculateAndAverageKurtosis,
// mode.cpp:1403-1454), which Core sends on the message bus
// (Core::averageAndSendKurtosis, core.cpp:1378-1430).  The STA dump is the
// band's autocorrelation over the same range, normalised to power spectral
// density and averaged down to the dump channels (core.cpp:1180-1255).
//
// Here the accumulation reads the spectra the F-step left in HBM, one
// thread per (band row, channel), blocks in order within the thread as the
// reference adds them; the spectra carry the fractional-sample correction
// the reference applies after taking the magnitudes, a unit-modulus FP32
// rotation that moves a magnitude by a few units in the last place.  The
// finish runs per band on the device in the reference's FP32 operation
// order.  The STA dump needs no device work: it is formed on the host from
// a Core result array (the autocorrelations and their weights).
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "../../include/gxcorr.h"
#include "gx_handle.h"
#include "gx_host.h"

namespace {

// One recorded band of a station: its spectra row.
struct KurtBand {
  int f, row, nchan;
};

__global__ void kurtosis_accum_kernel(const KurtBand *__restrict__ bands, const float2 *__restrict__ spec, int NI,
                                      int N, int nblk, float *__restrict__ s1, float *__restrict__ s2)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const KurtBand B = bands[blockIdx.y];
  if (c >= B.nchan) return;
  const size_t o = (size_t)blockIdx.y * N + c;
  float a = s1[o], b = s2[o];
  for (int k = 0; k < nblk; k++) {
    const float2 x = spec[(((size_t)B.f * nblk + k) * NI + B.row) * N + c];
    const float m = __fsqrt_rn(__fadd_rn(__fmul_rn(x.x, x.x), __fmul_rn(x.y, x.y)));
    const float m2 = __fmul_rn(m, m);
    a = __fadd_rn(a, m2);
    b = __fadd_rn(b, __fmul_rn(m2, m2));
  }
  s1[o] = a;
  s2[o] = b;
}

// Per band: skipped when no channel of s1 is positive (its previous result
// stays); otherwise sk = s2 n / s1^2 - 1, times n / (n - 1), minus 1, then
// kchanavg channels averaged into each dump channel.  out: [band][dump].
__global__ void kurtosis_finish_kernel(const KurtBand *__restrict__ bands, int nb, const float *__restrict__ s1,
                                       const float *__restrict__ s2, int N, int numblocks, int dump,
                                       float *__restrict__ sk, float *__restrict__ out, int *__restrict__ nonzero)
{
  const int bd = blockIdx.x;
  if (bd >= nb) return;
  const int n = bands[bd].nchan;
  const float *a = s1 + (size_t)bd * N;
  const float *b = s2 + (size_t)bd * N;
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int c = threadIdx.x; c < n; c += blockDim.x)
    if (a[c] > 0.0f) any = 1;
  __syncthreads();
  if (threadIdx.x == 0) nonzero[bd] = any;
  if (!any) return;
  const float fn = (float)numblocks;
  const float debias = (float)((double)fn / (numblocks - 1.0));
  const int kavg = dump < n ? n / dump : 1;
  const float inv = (float)(1.0 / ((float)kavg));
  float *k = sk + (size_t)bd * N;
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    const float sq = __fmul_rn(a[c], a[c]);
    const float t = __fmul_rn(b[c], fn);
    float v = __fdiv_rn(t, sq);
    v = __fadd_rn(v, -1.0f);
    v = __fmul_rn(v, debias);
    v = __fadd_rn(v, -1.0f);
    if (dump < n) v = __fmul_rn(v, inv);
    k[c] = v;
  }
  __syncthreads();
  const int nout = min(dump, n);
  for (int j = threadIdx.x; j < nout; j += blockDim.x) {
    float v = k[(size_t)j * kavg];
    for (int q = 1; q < kavg; q++) v = __fadd_rn(v, k[(size_t)j * kavg + q]);
    out[(size_t)bd * dump + j] = v;
  }
}

}  // namespace

// Kurtosis state of a handle (gx_set_kurtosis).
struct gx_kurtosis_state {
  int dump = 0;
  std::vector<KurtBand> bands;            // [station][recorded band], flattened
  std::vector<int> first;                 // first entry of each station
  KurtBand *d_bands = nullptr;
  float *d_s1 = nullptr, *d_s2 = nullptr, *d_sk = nullptr, *d_out = nullptr;
  int *d_nonzero = nullptr;
  bool have = false;                      // a subint has been finished
};

void gx_kurtosis_free(gx_kurtosis_state *k)
{
  if (!k) return;
  cudaFree(k->d_bands);
  cudaFree(k->d_s1);
  cudaFree(k->d_s2);
  cudaFree(k->d_sk);
  cudaFree(k->d_out);
  cudaFree(k->d_nonzero);
  delete k;
}

gx_status gx_kurtosis_begin(gx_handle *h, cudaStream_t st)
{
  gx_kurtosis_state *k = h->kurt;
  const size_t n = k->bands.size() * (size_t)h->J.nchan;
  CKR(h, cudaMemsetAsync(k->d_s1, 0, sizeof(float) * n, st));
  CKR(h, cudaMemsetAsync(k->d_s2, 0, sizeof(float) * n, st));
  return GX_OK;
}

gx_status gx_kurtosis_pass(gx_handle *h, int nblk, cudaStream_t st)
{
  gx_kurtosis_state *k = h->kurt;
  const int N = h->J.nchan;
  const dim3 grid((N + 127) / 128, (unsigned)k->bands.size());
  kurtosis_accum_kernel<<<grid, 128, 0, st>>>(k->d_bands, h->d_spec, h->J.ninputs, N, nblk, k->d_s1, k->d_s2);
  h->launches += 1;
  return h->cuda(cudaGetLastError(), "kurtosis_accum_kernel");
}

gx_status gx_kurtosis_end(gx_handle *h, cudaStream_t st)
{
  gx_kurtosis_state *k = h->kurt;
  kurtosis_finish_kernel<<<(unsigned)k->bands.size(), 256, 0, st>>>(k->d_bands, (int)k->bands.size(), k->d_s1, k->d_s2,
                                                                    h->J.nchan, h->J.blocks_per_send, k->dump, k->d_sk,
                                                                    k->d_out, k->d_nonzero);
  h->launches += 1;
  k->have = true;
  return h->cuda(cudaGetLastError(), "kurtosis_finish_kernel");
}

extern "C" {

gx_status gx_set_kurtosis(gx_handle *h, int dump_channels)
{
  if (!h) return GX_ERR_ARG;
  if (h->device < 0) return h->fail(GX_ERR_STATE, "host-only handle");
  if (!h->inflight.empty()) return h->fail(GX_ERR_STATE, "subints in flight");
  CKR(h, cudaSetDevice(h->device));
  if (h->kurt) {
    CKR(h, cudaStreamSynchronize(h->stream));
    gx_kurtosis_free(h->kurt);
    h->kurt = nullptr;
  }
  if (dump_channels <= 0) return GX_OK;
  std::unique_ptr<gx_kurtosis_state> k(new gx_kurtosis_state());
  k->dump = dump_channels;
  const gx_job_desc &d = h->jd;
  for (int s = 0; s < d.nstations; s++) {
    const gx_station_desc &x = d.stations[s];
    k->first.push_back((int)k->bands.size());
    for (int b = 0; b < x.nbands; b++) {
      const int f = x.recfreq[x.band_localfreq[b]];
      k->bands.push_back(KurtBand{f, h->band_input[s][b], d.freqs[f].nchan});
    }
  }
  k->first.push_back((int)k->bands.size());
  const size_t nb = k->bands.size(), N = (size_t)h->J.nchan;
  if (cudaMalloc(&k->d_bands, sizeof(KurtBand) * nb) != cudaSuccess ||
      cudaMalloc(&k->d_s1, sizeof(float) * nb * N) != cudaSuccess ||
      cudaMalloc(&k->d_s2, sizeof(float) * nb * N) != cudaSuccess ||
      cudaMalloc(&k->d_sk, sizeof(float) * nb * N) != cudaSuccess ||
      cudaMalloc(&k->d_out, sizeof(float) * nb * dump_channels) != cudaSuccess ||
      cudaMalloc(&k->d_nonzero, sizeof(int) * nb) != cudaSuccess) {
    gx_kurtosis_free(k.release());
    return h->fail(GX_ERR_NOMEM, "kurtosis buffers");
  }
  CKR(h, cudaMemcpy(k->d_bands, k->bands.data(), sizeof(KurtBand) * nb, cudaMemcpyHostToDevice));
  CKR(h, cudaMemset(k->d_out, 0, sizeof(float) * nb * dump_channels));
  CKR(h, cudaMemset(k->d_nonzero, 0, sizeof(int) * nb));
  h->kurt = k.release();
  return GX_OK;
}

gx_status gx_kurtosis(gx_handle *h, float *sk, int *nchan, int *valid)
{
  if (!h || !sk) return GX_ERR_ARG;
  gx_kurtosis_state *k = h->kurt;
  if (!k || !k->have) return h->fail(GX_ERR_STATE, "no kurtosis: gx_set_kurtosis, then a subint");
  CKR(h, cudaSetDevice(h->device));
  CKR(h, cudaStreamSynchronize(h->last_stream ? h->last_stream : h->stream));
  const size_t nb = k->bands.size();
  std::vector<float> out(nb * k->dump);
  std::vector<int> nz(nb);
  CKR(h, cudaMemcpy(out.data(), k->d_out, sizeof(float) * out.size(), cudaMemcpyDeviceToHost));
  CKR(h, cudaMemcpy(nz.data(), k->d_nonzero, sizeof(int) * nb, cudaMemcpyDeviceToHost));
  const gx_job_desc &d = h->jd;
  for (int s = 0; s < d.nstations; s++) {
    const int b0 = k->first[s], b1 = k->first[s + 1];
    for (int b = b0; b < b1; b++) {
      const int bl = b - b0;
      memcpy(sk + ((size_t)s * GX_MAX_BANDS + bl) * k->dump, &out[(size_t)b * k->dump], sizeof(float) * k->dump);
      if (nchan) nchan[s * GX_MAX_BANDS + bl] = std::min(k->dump, k->bands[b].nchan);
    }
    // the reference sends a station's records when its last band had data
    if (valid) valid[s] = b1 > b0 ? nz[b1 - 1] : 0;
  }
  return GX_OK;
}

gx_status gx_sta(const gx_handle *h, const float *results, int dump_channels, float *sta, int *nchan, int *sent)
{
  if (!h || !results || !sta || dump_channels <= 0) return GX_ERR_ARG;
  const gx_job_desc &d = h->jd;
  const double blockns = (double)d.subint_ns / (double)h->J.blocks_per_send;
  const double nswidth = h->J.blocks_per_send * blockns;
  // post-average channel counts: averaged records are used when every freq
  // keeps at least the dump channels (core.cpp:1180-1187)
  int minpost = INT32_MAX;
  for (int f = 0; f < d.nfreqs; f++) minpost = std::min(minpost, d.freqs[f].nchan / std::max(1, d.freqs[f].chans_to_average));
  const bool averaged = minpost >= dump_channels;
  if (!averaged && h->avg > 1) return GX_ERR_UNSUPPORTED;   // the full-resolution autocorrelations are not in the array
  for (int s = 0; s < d.nstations; s++) {
    const gx_station_desc &x = d.stations[s];
    const float *w = results + 2 * (size_t)h->acwofs[s];
    for (int b = 0; b < x.nbands; b++) {
      const int f = x.recfreq[x.band_localfreq[b]];
      const gx_freq_desc &fq = d.freqs[f];
      const int ao = h->sta_acoff.empty() ? -1 : h->sta_acoff[(size_t)s * GX_MAX_BANDS + b];
      const int wi = h->sta_acoff.empty() ? -1 : h->sta_acw[(size_t)s * GX_MAX_BANDS + b];
      float *out = sta + ((size_t)s * GX_MAX_BANDS + b) * dump_channels;
      if (sent) sent[s * GX_MAX_BANDS + b] = 0;
      if (ao < 0 || wi < 0) continue;
      int freqchannels = fq.nchan;
      const double stasamples = 0.001 * nswidth * 2 * fq.bw_mhz;
      const double minimumweight = 0.333 * stasamples / (2 * freqchannels);   // Core::MINIMUM_FILTERBANK_WEIGHT
      const float weight = w[wi];
      if (weight < minimumweight) continue;
      float renorm = (float)(1.0 / (2 * freqchannels * weight));
      const int cta = averaged ? std::max(1, fq.chans_to_average) : 1;
      if (averaged) {
        renorm /= cta;
        freqchannels /= cta;
      }
      const int n = std::min(dump_channels, freqchannels);
      const int avg = freqchannels / n;
      const float *ac = results + 2 * (size_t)ao;
      for (int k = 0; k < n; k++) {
        float v = ac[2 * k * avg];
        for (int l = 1; l < avg; l++) v += ac[2 * (k * avg + l)];
        out[k] = v * renorm;
      }
      if (nchan) nchan[s * GX_MAX_BANDS + b] = n;
      if (sent) sent[s * GX_MAX_BANDS + b] = 1;
    }
  }
  return GX_OK;
}

}  // extern "C"
