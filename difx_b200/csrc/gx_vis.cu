// Visibility output: the integration and SWIN writing of mpifxcorr's
// Visibility (mpifxcorr/src/visibility.cpp) for one job handle.
//
//   gx_vis_add    Visibility::addData (visibility.cpp:192-205): the subint's
//                 Core result array is added into a device-resident
//                 integration buffer (results[i] += subint[i], FP32).
//   gx_vis_write  Visibility::writedata (353-690) + writeSWIN (781-960):
//                 baseline and autocorrelation weights are read back (a few
//                 KB), each record's normalisation 1 / (weight * subints per
//                 integration * blocks per send * 2 * nchan) is formed with the
//                 reference's float/double expression, the records are scaled
//                 on the device, the buffer comes back once, and every record
//                 with a positive weight is appended as a 74-byte SWIN header
//                 (appendSWINHeaderBuffered, 1205-1234) plus nchan complex
//                 floats to <outdir>/DIFX_<mjd>_<sec>.s0000.b0000
//                 (flushBuffersToDisk, 1056-1091): cross-correlations first in
//                 baseline / freq / polarisation-product order, then the
//                 autocorrelations per datastream.
//
// Covered: one configuration, phase centres, pulsar bins, no output
// bands; TSYS 0 (normalised correlation coefficients) or TSYS > 0
// (a-priori calibration by the band-mean autocorrelations).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>
#include "gx_handle.h"

using namespace gx;

namespace {

struct VisScale {
  long long offset;   // complex-float index of the record's first channel
  float scale;
  int nchan;          // the record's channels
};

__global__ void vis_add4_kernel(float4 *__restrict__ acc, const float4 *__restrict__ r, size_t n)
{
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float4 a = acc[i];
    const float4 b = r[i];
    a.x += b.x;
    a.y += b.y;
    a.z += b.z;
    a.w += b.w;
    acc[i] = a;
  }
}

__global__ void vis_add_kernel(float *__restrict__ acc, const float *__restrict__ r, size_t n)
{
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    acc[i] += r[i];
}

__global__ void vis_scale_kernel(float2 *__restrict__ acc, const VisScale *__restrict__ recs)
{
  const VisScale R = recs[blockIdx.y];
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < R.nchan; c += gridDim.x * blockDim.x) {
    float2 v = acc[R.offset + c];
    v.x *= R.scale;
    v.y *= R.scale;
    acc[R.offset + c] = v;
  }
}

char opposite_pol(char p)
{
  switch (p) {
    case 'R': return 'L';
    case 'L': return 'R';
    case 'X': return 'Y';
    case 'Y': return 'X';
    default: return p;
  }
}

template <typename T>
void put(std::vector<char> &b, const T &v)
{
  const char *p = reinterpret_cast<const char *>(&v);
  b.insert(b.end(), p, p + sizeof(T));
}

}  // namespace

struct gx_vis {
  gx_handle *h = nullptr;
  std::string outdir;
  float2 *d_int = nullptr;   // integration buffer, result_length complex floats
  float2 *h_buf = nullptr;   // pinned copy for the writer
  VisScale *d_rec = nullptr;
  int maxrec = 0;
  int nsub = 0;
  cudaStream_t st = nullptr;
};

extern "C" {

gx_status gx_vis_open(gx_handle *h, const char *outdir, gx_vis **out)
{
  if (!h || !outdir || !out) return GX_ERR_ARG;
  *out = nullptr;
  if (h->device < 0) return h->fail(GX_ERR_STATE, "host-only handle (opened with device -1)");
  if (!h->model || !h->meta) return h->fail(GX_ERR_STATE, "the visibility writer needs a handle opened with gx_open_input");
  if (!h->zfreq.empty() && h->meta)
    for (double t : h->meta->tsys)   // Configuration::getDMatchingBand reads zoom bands out of range
      if (t > 0.0) return h->fail(GX_ERR_UNSUPPORTED, "a-priori calibration (TSYS > 0) of zoom bands is not implemented");
  std::unique_ptr<gx_vis> v(new gx_vis());
  v->h = h;
  v->outdir = outdir;
  v->st = h->stream;
  const gx_job_desc &d = h->jd;
  int nrec = 0;
  for (int i = 0; i < d.nbaselines; i++)
    for (int k = 0; k < d.baselines[i].nfreqs; k++) nrec += h->maxpc * h->binloop * d.baselines[i].npolprod[k];
  for (int s = 0; s < d.nstations; s++) nrec += 2 * (d.stations[s].nbands + d.stations[s].nzoombands);
  v->maxrec = nrec > 0 ? nrec : 1;
  CKR(h, cudaSetDevice(h->device));
  CKR(h, cudaMalloc(&v->d_int, sizeof(float2) * h->rl));
  CKR(h, cudaMemsetAsync(v->d_int, 0, sizeof(float2) * h->rl, v->st));
  CKR(h, cudaMallocHost(&v->h_buf, sizeof(float2) * h->rl));
  CKR(h, cudaMalloc(&v->d_rec, sizeof(VisScale) * v->maxrec));
  CKR(h, cudaStreamSynchronize(v->st));
  *out = v.release();
  return GX_OK;
}

gx_status gx_vis_add(gx_vis *v, const float *dev_results, void *stream)
{
  if (!v || !dev_results) return GX_ERR_ARG;
  gx_handle *h = v->h;
  CKR(h, cudaSetDevice(h->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : v->st;
  const size_t nfl = 2 * (size_t)h->rl;
  const int blocks = 148 * 8;
  if (((uintptr_t)dev_results & 15) == 0 && nfl % 4 == 0)
    vis_add4_kernel<<<blocks, 256, 0, st>>>(reinterpret_cast<float4 *>(v->d_int),
                                            reinterpret_cast<const float4 *>(dev_results), nfl / 4);
  else
    vis_add_kernel<<<blocks, 256, 0, st>>>(reinterpret_cast<float *>(v->d_int), dev_results, nfl);
  CKR(h, cudaGetLastError());
  if (st != v->st) {   // later work on the handle's stream sees the sum
    cudaEvent_t e;
    CKR(h, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CKR(h, cudaEventRecord(e, st));
    CKR(h, cudaStreamWaitEvent(v->st, e, 0));
    CKR(h, cudaEventDestroy(e));
  }
  v->nsub++;
  return GX_OK;
}

gx_status gx_vis_write(gx_vis *v, int scan, int sec, int ns, int *nrecords)
{
  if (!v) return GX_ERR_ARG;
  if (nrecords) *nrecords = 0;
  gx_handle *h = v->h;
  const gx_job_desc &d = h->jd;
  const JobMeta &M = *h->meta;
  const HostModel &model = *h->model;
  CKR(h, cudaSetDevice(h->device));
  if (scan < 0 || scan >= (int)model.scans.size()) return GX_OK;               // past the last scan
  const int scanstart = (int)model.scan_start_sec(scan);
  if (sec + scanstart >= M.execute_seconds || v->nsub == 0) return GX_OK;      // writedata's early exits
  const int nbl = d.nbaselines;
  auto nout = [&](int f) { return d.freqs[f].nchan / h->avg; };   // output channels of freq f's records

  // weights: the baseline-weight and autocorrelation-weight regions of the summed array
  std::vector<float> fr(2 * (size_t)h->rl);
  {
    long long bw0 = h->rl, bw1 = 0, aw0 = h->rl;
    for (int f = 0; f < d.nfreqs; f++)   // each baseline-freq's weights: bins x products floats
      for (int i = 0; i < nbl; i++) {
        const int x = h->bwofs[f * nbl + i], lf = gx_bl_localfreq(d.baselines[i], f);
        if (x < 0 || lf < 0) continue;
        bw0 = std::min<long long>(bw0, x);
        bw1 = std::max<long long>(bw1, x + (h->binloop * d.baselines[i].npolprod[lf] + 1) / 2);
      }
    for (int x : h->bsdofs)   // and the shift decorrelation factors that follow them
      if (x >= 0) bw1 = std::max<long long>(bw1, x + h->maxpc / 2 + h->maxpc % 2);
    for (int x : h->acwofs) aw0 = std::min<long long>(aw0, x);
    // TSYS > 0: the autocorrelations too (their band means calibrate, visibility.cpp:463-484)
    for (double t : M.tsys)
      if (t > 0.0)
        for (int x : h->acofs) aw0 = std::min<long long>(aw0, x);
    if (bw1 > bw0)
      CKR(h, cudaMemcpyAsync(&fr[2 * bw0], v->d_int + bw0, sizeof(float2) * (bw1 - bw0), cudaMemcpyDeviceToHost,
                             v->st));
    if (h->rl > aw0)
      CKR(h, cudaMemcpyAsync(&fr[2 * aw0], v->d_int + aw0, sizeof(float2) * (h->rl - aw0), cudaMemcpyDeviceToHost,
                             v->st));
    CKR(h, cudaStreamSynchronize(v->st));
  }
  // Visibility::changeConfig (visibility.cpp:1314-1316)
  const double meansub = M.int_time / (((double)d.subint_ns) / 1000000000.0);
  const double ffts = meansub * h->J.blocks_per_send;
  // blocks per send * 2 * nchan * chanavg of freq f
  auto chanfactor = [&](int f) { return (float)(h->J.blocks_per_send * 2 * nout(f) * h->avg); };
  // pulsar binning (visibility.cpp:402-415, 1376-1393): a bin's baseline
  // weights over the bin's phase width, scrunched ones over the FP32 sum of
  // weight x width of every bin
  const int binloop = h->binloop;
  std::vector<double> binwidth(binloop, 1.0);
  float scrunchdiv = 0.0f;
  if (h->nbins > 0) {
    const PulsarConfig &P = *M.pulsar;
    const int nb = (int)P.binphaseends.size();
    auto width = [&](int b) {
      const double w = P.binphaseends[b] - P.binphaseends[(b + nb - 1) % nb];
      return w < 0.0 ? 1.0 + w : w;
    };
    if (binloop > 1)
      for (int b = 0; b < binloop; b++) binwidth[b] = width(b);
    for (int b = 0; b < nb; b++) scrunchdiv += P.binweights[b] * width(b);
  }
  auto weight_and_scale = [&](long long widx, int f, float &w, float &scale, int bin = -1) {
    if (bin >= 0 && binloop > 1) w = (float)(fr[widx] / (ffts * binwidth[bin]));
    else if (bin >= 0 && h->nbins > 0) w = (float)(fr[widx] / (ffts * scrunchdiv));
    else w = (float)(fr[widx] / ffts);
    scale = w > 0.0f ? (float)(1.0 / ((double)w * meansub * (double)chanfactor(f))) : 0.0f;
  };
  // freq and polarisation of total band k (recorded bands, then zoom bands)
  auto total_freq = [&](const gx_station_desc &x, int k) {
    return k < x.nbands ? x.recfreq[x.band_localfreq[k]] : x.zoomfreq[x.zoomband_localfreq[k - x.nbands]];
  };
  auto total_pol = [&](const gx_station_desc &x, int k) {
    return k < x.nbands ? x.band_pol[k] : x.zoomband_pol[k - x.nbands];
  };
  // zoom bandwidth / parent recorded bandwidth of total band k >= nbands of
  // station s, as the reference's FP32 `modifier` (visibility.cpp:355, 532-545, 626-631)
  auto zoom_modifier = [&](int s, int k) {
    const gx_station_desc &x = d.stations[s];
    const int pf = x.recfreq[x.band_localfreq[h->zparent[s][k - x.nbands]]];
    float modifier = 1.0f;
    modifier *= d.freqs[total_freq(x, k)].bw_mhz;
    modifier /= d.freqs[pf].bw_mhz;
    return modifier;
  };
  // A-priori calibration with TSYS > 0 (visibility.cpp:463-484, 505-519,
  // 607-616): the FP32 mean of each band's summed parallel-hand
  // autocorrelation (genericMean_32fc: a sequential sum, then a division) and
  // the autocorrelation weights by band, as writedata forms them.
  const int acwidth = h->maxprod > 2 ? 2 : 1;
  std::vector<std::vector<float>> calib(d.nstations), acw0(d.nstations);
  for (int s = 0; s < d.nstations; s++) {
    const gx_station_desc &x = d.stations[s];
    calib[s].assign(x.nbands + x.nzoombands, 0.0f);
    acw0[s].assign(x.nbands + x.nzoombands, 0.0f);
    long long widx = 2LL * h->acwofs[s];   // the parallel-hand weights come first
    for (int k : h->acbands[s]) acw0[s][k] = (float)(fr[widx++] / ffts);
    if (!(s < (int)M.tsys.size() && M.tsys[s] > 0.0)) continue;
    long long off = h->acofs[s];
    for (int k : h->acbands[s]) {
      const int N = nout(total_freq(x, k));
      float re = 0.0f;
      for (int c = 0; c < N; c++) re += fr[2 * (off + c)];
      calib[s][k] = re / N;
      off += N;
    }
  }
  auto tsys = [&](int s) { return s < (int)M.tsys.size() ? M.tsys[s] : 0.0; };
  // Mode::decorrelationpercentage (mode.cpp:1571), by bits per sample
  static const float kDecorrelation[8] = {0.63662f, 0.88f, 0.94f, 0.96f, 0.98f, 0.99f, 0.996f, 0.998f};
  auto matching_band = [&](const gx_station_desc &x, int b) {   // Configuration::getDMatchingBand
    for (int i = 0; i < x.nbands; i++)
      if (i != b && x.band_localfreq[i] == x.band_localfreq[b]) return i;
    return -1;
  };

  // record table, in writeSWIN order
  struct Rec {
    int baseline, freq;
    char pol[2];
    float weight;
    double uvw[3];
    long long offset;
    int nchan;
    int file;     // phase centre x bins + bin: output file DIFX_..s<centre>.b<bin>
    int source;   // source table index in the header
    int bin;      // pulsar bin in the header
  };
  std::vector<Rec> recs;
  std::vector<VisScale> scales;
  const ModelScan &scn = model.scans[scan];
  const int nph = scn.numphasecentres;
  // shift decorrelation factor of phase centre ph: the interval sums over the
  // integration's nanoseconds, in FP32 (visibility.cpp:428-441)
  auto shiftdecorr = [&](int f, int i, int ph) {
    return (float)(fr[2LL * h->bsdofs[f * nbl + i] + ph] / (1000000000.0 * M.int_time));
  };
  const double scanoffset = sec + ((double)ns) / 1e9 + M.int_time / 2.0;
  for (int i = 0; i < nbl; i++) {
    const gx_baseline_desc &B = d.baselines[i];
    for (int f = 0; f < d.nfreqs; f++) {
      const int lf = gx_bl_localfreq(B, f);
      if (lf < 0) continue;
      const int N = nout(f);
      for (int ph = 0; ph < nph; ph++) {   // records of every phase centre and bin, each to its own file
      for (int bin = 0; bin < binloop; bin++) {
      Rec r{};
      r.baseline = (M.telescope[B.ds1] + 1) * 256 + (M.telescope[B.ds2] + 1);
      r.file = ph * binloop + bin;
      r.bin = bin;
      r.source = scn.phase_centre_sources[ph];
      if (!model.uvw(scan, scanoffset, model.station_of_datastream[B.ds1], model.station_of_datastream[B.ds2], ph + 1,
                     r.uvw))
        return h->fail(GX_ERR_MODEL, "no (u, v, w) model for this integration");
      const long long base = h->blofs[f * nbl + i] + ((long long)ph * binloop + bin) * B.npolprod[lf] * N;
      for (int k = 0; k < B.npolprod[lf]; k++) {
        float w, scale;
        weight_and_scale(2LL * h->bwofs[f * nbl + i] + (long long)bin * B.npolprod[lf] + k, f, w, scale, bin);
        if (w > 0.0f) {   // zoom bands: fewer samples per channel (visibility.cpp:530-545)
          if (B.band1[lf][k] >= d.stations[B.ds1].nbands) scale *= std::sqrt(zoom_modifier(B.ds1, B.band1[lf][k]));
          if (B.band2[lf][k] >= d.stations[B.ds2].nbands) scale *= std::sqrt(zoom_modifier(B.ds2, B.band2[lf][k]));
        }
        if (tsys(B.ds1) > 0.0 && tsys(B.ds2) > 0.0) {
          const int b1 = B.band1[lf][k], b2 = B.band2[lf][k];
          const float divisor = kDecorrelation[d.stations[B.ds1].nbits - 1] * kDecorrelation[d.stations[B.ds2].nbits - 1] *
                                calib[B.ds1][b1] * calib[B.ds2][b2] / (acw0[B.ds1][b1] * acw0[B.ds2][b2]);
          scale = (divisor > 0.0f && w > 0.0f)
                      ? (float)(std::sqrt(tsys(B.ds1) * tsys(B.ds2) / divisor) / w) : 0.0f;
        }
        float sd = 1.0f;
        if (nph > 1) {   // further scaled by the decorrelation of the uv shift (visibility.cpp:554-557)
          sd = shiftdecorr(f, i, ph);
          scale /= sd;
        }
        if (scale > 0.0f) scales.push_back(VisScale{base + (long long)k * N, scale, N});
        if (w > 0.0f) {
          r.freq = f;
          r.pol[0] = total_pol(d.stations[B.ds1], B.band1[lf][k]);
          r.pol[1] = total_pol(d.stations[B.ds2], B.band2[lf][k]);
          r.weight = nph > 1 ? w * sd : w;   // the weight times the decorrelation (visibility.cpp:869-872)
          r.offset = base + (long long)k * N;
          r.nchan = N;
          recs.push_back(r);
        }
      }
      }
      }
    }
  }
  if (d.write_autocorrs) {
    for (int s = 0; s < d.nstations; s++) {
      const gx_station_desc &x = d.stations[s];
      long long off = h->acofs[s], widx = 2LL * h->acwofs[s];
      for (int j = 0; j < acwidth; j++)
        for (int b : h->acbands[s]) {   // recorded bands, then zoom bands
          const int f = total_freq(x, b), N = nout(f);
          float w, scale;
          weight_and_scale(widx++, f, w, scale);
          if (tsys(s) > 0.0) {
            const int m = j == 0 ? b : matching_band(x, b);
            const float divisor = m >= 0 ? std::sqrt(calib[s][b] * calib[s][m]) : 0.0f;
            scale = divisor > 0.0f ? (float)(tsys(s) / divisor) : 0.0f;
          } else if (b >= x.nbands && w > 0.0f) {
            // a zoom band's autocorrelation: times zoom bandwidth / parent
            // bandwidth, in FP32 as the reference forms it (visibility.cpp:624-633)
            scale *= zoom_modifier(s, b);
          }
          if (scale > 0.0f) scales.push_back(VisScale{off, scale, N});
          if (w > 0.0f) {
            Rec r{};
            r.baseline = 257 * (M.telescope[s] + 1);
            r.file = 0;   // the autocorrelations follow the first file's crosses (visibility.cpp:895-948)
            r.source = nph == 1 ? scn.phase_centre_sources[0] : scn.pointing_source;
            r.freq = f;
            r.pol[0] = total_pol(x, b);
            r.pol[1] = j == 0 ? r.pol[0] : opposite_pol(r.pol[0]);
            r.weight = w;
            r.offset = off;
            r.nchan = N;
            recs.push_back(r);
          }
          off += N;
        }
    }
  }

  // normalise on the device, then one copy back
  if (!scales.empty()) {
    if ((int)scales.size() > v->maxrec) return h->fail(GX_ERR_ARG, "record table overflow");
    CKR(h, cudaMemcpyAsync(v->d_rec, scales.data(), sizeof(VisScale) * scales.size(), cudaMemcpyHostToDevice, v->st));
    int maxn = 1;
    for (const VisScale &x : scales) maxn = std::max(maxn, x.nchan);
    dim3 grid((maxn + 255) / 256, (unsigned)scales.size());
    vis_scale_kernel<<<grid, 256, 0, v->st>>>(v->d_int, v->d_rec);
    CKR(h, cudaGetLastError());
  }
  CKR(h, cudaMemcpyAsync(v->h_buf, v->d_int, sizeof(float2) * h->rl, cudaMemcpyDeviceToHost, v->st));
  CKR(h, cudaStreamSynchronize(v->st));

  // SWIN records (appendSWINHeaderBuffered): 74-byte header + nchan complex floats
  const int intsec = M.start_seconds + scanstart + sec;
  const int dumpmjd = M.start_mjd + intsec / 86400;
  const double dumpseconds = double(intsec % 86400) + ((double)ns) / 1000000000.0 + M.int_time / 2.0;
  // one file per phase centre and bin (flushBuffersToDisk, visibility.cpp:1056-1091)
  const int nfiles = nph * binloop;
  std::vector<std::vector<char>> bufs(nfiles);
  {
    std::vector<size_t> bytes(nfiles, 0);
    for (const Rec &r : recs) bytes[r.file] += 74 + sizeof(float2) * (size_t)r.nchan;
    for (int q = 0; q < nfiles; q++) bufs[q].reserve(bytes[q]);
  }
  for (const Rec &r : recs) {
    std::vector<char> &buf = bufs[r.file];
    put(buf, (uint32_t)0xFF00FF00u);   // sync word
    put(buf, (int32_t)1);              // binary header version
    put(buf, (int32_t)r.baseline);
    put(buf, (int32_t)dumpmjd);
    put(buf, dumpseconds);
    put(buf, (int32_t)0);              // configuration index
    put(buf, (int32_t)r.source);
    put(buf, (int32_t)r.freq);
    buf.push_back(r.pol[0]);
    buf.push_back(r.pol[1]);
    put(buf, (int32_t)r.bin);          // pulsar bin
    put(buf, (double)r.weight);
    put(buf, r.uvw[0]);
    put(buf, r.uvw[1]);
    put(buf, r.uvw[2]);
    const char *p = reinterpret_cast<const char *>(v->h_buf + r.offset);
    buf.insert(buf.end(), p, p + sizeof(float2) * (size_t)r.nchan);
  }
  for (int q = 0; q < nfiles; q++) {
    char name[64];
    snprintf(name, sizeof(name), "/DIFX_%05d_%06d.s%04d.b%04d", M.start_mjd, M.start_seconds, q / binloop, q % binloop);
    std::ofstream of(v->outdir + name, std::ios::app | std::ios::binary);
    if (!of) return h->fail(GX_ERR_IO, "cannot open " + v->outdir + name);
    of.write(bufs[q].data(), (std::streamsize)bufs[q].size());
    of.close();
    if (!of) return h->fail(GX_ERR_IO, "write failed: " + v->outdir + name);
  }

  // phase-cal lines (writedata, visibility.cpp:650-675 and 985-1053): each band's
  // tones scaled as its parallel-hand autocorrelation, one line per datastream
  {
    const double pcalmjd = dumpmjd + dumpseconds / 86400.0;
    for (int s = 0; s < d.nstations; s++) {
      const gx_station_desc &x = d.stations[s];
      if (x.phase_cal_interval_hz <= 0) continue;
      const int maxt = h->pc_maxtones[s];
      char str[256];
      snprintf(str, sizeof(str), "%s %17.11f %13.11f %d %d %d", M.telescope_name[M.telescope[s]].c_str(), pcalmjd,
               M.int_time / 86400.0, s, x.nbands, maxt);
      std::string line = str;
      bool nonzero = false;
      long long widx = 2LL * h->acwofs[s];
      for (int b = 0; b < x.nbands; b++) {
        const int f = x.recfreq[x.band_localfreq[b]];
        float w = 0.0f, scale = 0.0f;
        if (std::find(h->acbands[s].begin(), h->acbands[s].end(), b) != h->acbands[s].end())
          weight_and_scale(widx++, f, w, scale);
        if (w == 0.0f && x.nzoombands > 0) {
          // zoom mode with no autocorrelation of the band: data contribution only (visibility.cpp:661-663)
          w = 1.0f;
          scale = (float)(1.0 / ((double)w * meansub * (double)chanfactor(f)));
        }
        const size_t key = (size_t)s * GX_MAX_BANDS + b;
        const int nt = h->pc_ntones[key];
        const long long base = h->pc_off[key];
        for (int t = 0; t < maxt; t++) {
          if (t >= nt) {
            line += " -1 0 0 0";
            continue;
          }
          float2 v2 = v->h_buf[base + t];
          if (w > 0.0f) {
            v2.x *= scale;
            v2.y *= scale;
          }
          const bool lsb = d.freqs[f].lower_sideband != 0;
          snprintf(str, sizeof(str), " %.12g %c %12.5e %12.5e", 1e-6 * h->pc_tone_hz[key][t], x.band_pol[b],
                   (double)v2.x, (double)(lsb ? v2.y : -v2.y));
          if (v2.x != 0.0f && -v2.y != 0.0f) nonzero = true;
          line += str;
        }
      }
      if (nonzero) {
        char pname[256];
        snprintf(pname, sizeof(pname), "/PCAL_%05d_%06d_%s", M.start_mjd, M.start_seconds,
                 M.telescope_name[M.telescope[s]].c_str());
        std::ofstream pf(v->outdir + pname, std::ios::app);
        pf << line << "\n";
        if (!pf) return h->fail(GX_ERR_IO, "write failed: " + v->outdir + pname);
      }
    }
  }

  CKR(h, cudaMemsetAsync(v->d_int, 0, sizeof(float2) * h->rl, v->st));
  v->nsub = 0;
  if (nrecords) *nrecords = (int)recs.size();
  return GX_OK;
}

gx_status gx_vis_pcal_headers(gx_vis *v)
{
  if (!v) return GX_ERR_ARG;
  gx_handle *h = v->h;
  const gx_job_desc &d = h->jd;
  const JobMeta &M = *h->meta;
  std::vector<std::string> done;
  for (int s = 0; s < d.nstations; s++) {
    if (d.stations[s].phase_cal_interval_hz <= 0) continue;
    const std::string &name = M.telescope_name[M.telescope[s]];
    bool seen = false;
    for (const std::string &x : done) seen = seen || x == name;
    if (seen) continue;
    char pname[256];
    snprintf(pname, sizeof(pname), "/PCAL_%05d_%06d_%s", M.start_mjd, M.start_seconds, name.c_str());
    std::ofstream pf(v->outdir + pname, std::ios::app);
    pf << "# DiFX-derived pulse cal data\n# File version = 1\n# Start MJD = " << M.start_mjd
       << "\n# Start seconds = " << M.start_seconds << "\n# Telescope name = " << name << "\n";
    if (!pf) return h->fail(GX_ERR_IO, "cannot write " + v->outdir + pname);
    done.push_back(name);
  }
  return GX_OK;
}

gx_status gx_vis_buffer(gx_vis *v, float **dev, long long *nfloats, int *nsub)
{
  if (!v || !dev || !nfloats) return GX_ERR_ARG;
  *dev = reinterpret_cast<float *>(v->d_int);
  *nfloats = 2 * (long long)v->h->rl;
  if (nsub) *nsub = v->nsub;
  return GX_OK;
}

gx_status gx_vis_set_subints(gx_vis *v, int nsub)
{
  if (!v || nsub < 0) return GX_ERR_ARG;
  v->nsub = nsub;
  return GX_OK;
}

gx_status gx_vis_clear(gx_vis *v)
{
  if (!v) return GX_ERR_ARG;
  gx_handle *h = v->h;
  CKR(h, cudaSetDevice(h->device));
  CKR(h, cudaMemsetAsync(v->d_int, 0, sizeof(float2) * h->rl, v->st));
  v->nsub = 0;
  return GX_OK;
}

gx_status gx_vis_close(gx_vis *v)
{
  if (!v) return GX_ERR_ARG;
  if (v->h && v->h->device >= 0) cudaSetDevice(v->h->device);
  if (v->st) cudaStreamSynchronize(v->st);
  if (v->d_int) cudaFree(v->d_int);
  if (v->d_rec) cudaFree(v->d_rec);
  if (v->h_buf) cudaFreeHost(v->h_buf);
  delete v;
  return GX_OK;
}

gx_status gx_uvw(gx_handle *h, int scan, double offset, int ds1, int ds2, double out[3])
{
  if (!h || !out) return GX_ERR_ARG;
  if (!h->model) return h->fail(GX_ERR_STATE, "handle has no delay model (open it with gx_open_input)");
  if (ds1 < 0 || ds2 < 0 || ds1 >= h->jd.nstations || ds2 >= h->jd.nstations)
    return h->fail(GX_ERR_ARG, "datastream out of range");
  if (!h->model->uvw(scan, offset, h->model->station_of_datastream[ds1], h->model->station_of_datastream[ds2], 1, out))
    return h->fail(GX_ERR_MODEL, "no (u, v, w) model at this time");
  return GX_OK;
}

}  // extern "C"
