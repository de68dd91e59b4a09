/*
 * gxoracle -- CPU restatement of DiFX's FX-correlation hot path.
 * TEST INFRASTRUCTURE ONLY (the checker); see gxoracle.h.
 */
#define _GNU_SOURCE
#include "gxoracle.h"
#include "gxfft.h"
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define TWO_PI 6.283185307179586476925286766559 /* architecture.h.in:434 */
#define FLAGS_PER_INT 30                          /* mpifxcorr.h:29 */
#define INVALID_SUBINT (-99999999)                /* mode.h:222 */
static const float MODE_TINY = 0.000000001f;      /* mode.cpp:26 */
#define FILL_WORD64 0x1122334411223344ULL         /* blanker_mark5.c:35 (little-endian hosts) */

typedef struct { float re, im; } cf;
typedef struct { double re, im; } cd;

/* calcstridelength, configuration.cpp:38-50 */
static int stride_length(int n)
{
  if (n <= 16) return n;
  for (unsigned int g = (unsigned int)sqrt(n + 0.1);; --g)
    if (n % g == 0) return n / (int)g;
}

static int bl_localfreq(const gx_baseline_desc *b, int f)
{
  int r = -1;
  for (int j = 0; j < b->nfreqs; j++) if (b->freq[j] == f) r = j;
  return r;
}

static int freq_used(const gx_job_desc *d, int f)
{
  for (int j = 0; j < d->nbaselines; j++) if (bl_localfreq(&d->baselines[j], f) >= 0) return 1;
  return 0;
}

static int max_products(const gx_job_desc *d)
{
  int m = 0;
  for (int j = 0; j < d->nbaselines; j++)
    for (int k = 0; k < d->baselines[j].nfreqs; k++)
      if (d->baselines[j].npolprod[k] > m) m = d->baselines[j].npolprod[k];
  return m;
}

/* populateResultLengths, configuration.cpp:2348-2630, for one phase centre,
   no pulsar bins, no output-band merging and no channel averaging */
long long gxo_layout(const gx_job_desc *d, int *blofs, int *bwofs, int *acofs, int *acwofs)
{
  long long idx = 0;
  int nb = d->nbaselines;
  int bpa = max_products(d) > 2 ? 2 : 1;
  for (int i = 0; i < d->nfreqs * nb; i++) { blofs[i] = -1; bwofs[i] = -1; }
  for (int f = 0; f < d->nfreqs; f++) {
    if (!freq_used(d, f)) continue;
    for (int j = 0; j < nb; j++) {
      int lf = bl_localfreq(&d->baselines[j], f);
      if (lf < 0) continue;
      blofs[f * nb + j] = (int)idx;
      idx += (long long)d->baselines[j].npolprod[lf] * d->freqs[f].nchan;
    }
  }
  for (int f = 0; f < d->nfreqs; f++) {
    if (!freq_used(d, f)) continue;
    for (int j = 0; j < nb; j++) {
      int lf = bl_localfreq(&d->baselines[j], f);
      if (lf < 0) continue;
      bwofs[f * nb + j] = (int)idx;
      int np = d->baselines[j].npolprod[lf];
      idx += np / 2 + np % 2;
    }
  }
  for (int s = 0; s < d->nstations; s++) {
    const gx_station_desc *st = &d->stations[s];
    acofs[s] = (int)idx;
    for (int b = 0; b < st->nbands; b++) {
      int f = st->recfreq[st->band_localfreq[b]];
      if (freq_used(d, f)) idx += (long long)bpa * d->freqs[f].nchan;
    }
  }
  for (int s = 0; s < d->nstations; s++) {
    const gx_station_desc *st = &d->stations[s];
    acwofs[s] = (int)idx;
    int add = 0;
    for (int b = 0; b < st->nbands; b++)
      if (freq_used(d, st->recfreq[st->band_localfreq[b]])) add += bpa;
    add = (add + 1) / 2;
    if (add == 0) add = 1;
    idx += add;
  }
  return idx;
}

/* ------------------------------------------------------------------ unpack */

/* VDIF decode tables, format_vdif.c:66-146 */
static float lut_level(int nbits, int code)
{
  static const float hi = 3.3359f; /* OPTIMAL_2BIT_HIGH, mark5_stream.h:65 */
  switch (nbits) {
    case 1: return code ? 1.0f : -1.0f;
    case 2: { const float l[4] = {-hi, -1.0f, 1.0f, hi}; return l[code]; }
    case 4: return (float)((code - 7.5) / 2.95f) ; /* lut16level: (-7.5..7.5)/FourBit1sigma */
    case 8: return (float)((code - 128.0) / 3.3);
  }
  return 0.0f;
}

static int frame_valid(const unsigned char *frame, int framebytes, int check_header)
{
  const uint32_t *h = (const uint32_t *)frame;
  if (check_header) {
    if (h[2] == 0) return 0;               /* mark5_format_vdif_validate, format_vdif.c:7625 */
    if ((h[0] >> 31) & 1) return 0;        /* invalid bit, format_vdif.c:7656 */
  }
  uint64_t first, last;                    /* blanker_vdif fill-pattern test, blanker_mark5.c:302 */
  memcpy(&first, frame + 32, 8);
  memcpy(&last, frame + framebytes - 8, 8);
  if (first == FILL_WORD64 || last == FILL_WORD64) return 0;
  return 1;
}

static int station_framesamples(const gx_station_desc *st)
{
  /* configuration.cpp:980-986: payload bits / (bits x bands), halved for complex */
  int fs = (st->framebytes - 32) * 8 / (st->nbits * st->nbands);
  if (st->is_complex) fs /= 2;
  return fs;
}

int gxo_unpack(const gx_station_desc *st, int framesamples, const unsigned char *data, long long datalen,
               int offset, int nsamp, float *out)
{
  int nb = st->nbands, nbits = st->nbits, cplx = st->is_complex;
  int sub = cplx ? 2 : 1;
  int bits_per_ts = nb * nbits * sub;
  int good = 0;
  int curframe = -1, curvalid = 0;
  for (int o = 0; o < nsamp; o++) {
    long long sidx = (long long)offset + o;
    int frame = (int)(sidx / framesamples);
    int within = (int)(sidx % framesamples);
    if (frame != curframe) {
      const unsigned char *fp = data + (long long)frame * st->framebytes;
      /* first frame of a complex unpack: the extra blanker call in
         mark5_unpack_complex_with_offset (mark5_stream_unpacker.c:178)
         re-evaluates only the fill pattern */
      int first = (curframe < 0);
      /* a frame that lies outside the buffer is treated as invalid (the
         reference would read past the buffer, which the caller's guard
         data prevents) */
      if ((long long)(frame + 1) * st->framebytes > datalen || frame < 0) curvalid = 0;
      else curvalid = frame_valid(fp, st->framebytes, !(cplx && first));
      curframe = frame;
    }
    if (!curvalid) {
      for (int b = 0; b < nb; b++) {
        if (cplx) { out[b * 2 * nsamp + 2 * o] = 0.0f; out[b * 2 * nsamp + 2 * o + 1] = 0.0f; }
        else out[b * nsamp + o] = 0.0f;
      }
      continue;
    }
    good++;
    const unsigned char *payload = data + (long long)frame * st->framebytes + 32;
    long long bitbase = (long long)within * bits_per_ts;
    for (int b = 0; b < nb; b++) {
      for (int c = 0; c < sub; c++) {
        long long bit = bitbase + (long long)(b * sub + c) * nbits;
        int code = (payload[bit >> 3] >> (bit & 7)) & ((1 << nbits) - 1);
        float v = lut_level(nbits, code);
        if (cplx) out[b * 2 * nsamp + 2 * o + c] = v;
        else out[b * nsamp + o] = v;
      }
    }
  }
  return good;
}

/* EDV4 per-band blanking of multiplexed VDIF after the unpack (Mk5Mode::unpack,
   mk5mode.cpp:142-163; blank_vdif_EDV4 / _complex, format_vdif.c:8486-8660):
   geometry from the first header of the buffer (samples per header frame =
   payload bits / (channels x bits), twice the complex samples for complex
   data); a header frame with its invalid bit clear and a validity mask other
   than all channels zeroes, in every band whose thread bit (band / (channels /
   mask length)) is clear, the unpacked samples that are not zero, counting
   them per band.  Without EDV4 fields nothing is blanked. */
static void edv4_blank(const gx_station_desc *st, const unsigned char *data, long long datalen, int offset,
                       int nsamp, float *unp, int *invalid)
{
  int nb = st->nbands, cplx = st->is_complex;
  for (int b = 0; b < nb; b++) invalid[b] = 0;
  if (datalen < 32) return;
  const uint32_t *h0 = (const uint32_t *)data;
  int ever = (int)(h0[4] >> 24), mlen = (int)((h0[4] >> 16) & 0xffu);
  if (ever != 4 || mlen < 1 || mlen > 64) return;
  int nchan = 1 << ((h0[2] >> 24) & 0x1f);
  long long flen = (long long)(h0[2] & 0xffffffu) * 8;
  int hbits = (int)((h0[3] >> 26) & 0x1f) + 1;
  long long sph = (flen - 32) * 8 / ((long long)nchan * hbits);
  int dch = nchan / mlen;
  if (sph <= 0 || dch <= 0 || nchan > 62) return;
  unsigned long long good_mask = (1ull << nchan) - 1ull;
  for (long long k = offset / sph; k <= ((long long)offset + nsamp - 1) / sph; k++) {
    if ((k + 1) * flen > datalen) break;
    const uint32_t *hk = (const uint32_t *)(data + k * flen);
    unsigned long long vmask = (unsigned long long)hk[6] | ((unsigned long long)hk[7] << 32);
    if ((hk[0] >> 31) != 0u || vmask == good_mask) continue;
    long long lo = k * sph > offset ? k * sph : offset;
    long long hi = (k + 1) * sph < (long long)offset + nsamp ? (k + 1) * sph : (long long)offset + nsamp;
    for (int b = 0; b < nb; b++) {
      if ((vmask >> (b / dch)) & 1ull) continue;
      for (long long sm = lo; sm < hi; sm++) {
        long long o = sm - offset;
        if (cplx) {
          float *v = unp + (long long)b * 2 * nsamp + 2 * o;
          if (v[0] != 0.0f || v[1] != 0.0f) { v[0] = v[1] = 0.0f; invalid[b]++; }
        } else {
          float *v = unp + (long long)b * nsamp + o;
          if (*v != 0.0f) { *v = 0.0f; invalid[b]++; }
        }
      }
    }
  }
}

/* -------------------------------------------------------------- station F */

typedef struct {
  int nchan, fftchannels, S, nfr, nfrac;
  double bw, sampletime;
  int unpacksamples, framesamples;
  int bytespersample;
  int fractional_lo, deltapol;
  int cplx;
} stn;

static void stn_init(const gx_job_desc *d, int s, stn *o)
{
  const gx_station_desc *st = &d->stations[s];
  const gx_freq_desc *f0 = &d->freqs[st->recfreq[0]];
  o->cplx = st->is_complex;
  o->nchan = f0->nchan;
  o->bw = f0->bw_mhz;
  o->fftchannels = o->cplx ? o->nchan : 2 * o->nchan;
  o->S = d->array_stride ? d->array_stride : stride_length(o->nchan);
  o->nfr = o->fftchannels / o->S;
  o->nfrac = o->cplx ? 2 * o->nfr : o->nfr;
  o->sampletime = 1.0 / (2.0 * o->bw);
  if (o->cplx) o->sampletime *= 2.0;
  o->unpacksamples = o->cplx ? o->nchan : 2 * o->nchan;
  o->framesamples = station_framesamples(st);
  o->bytespersample = st->nbands * st->nbits * (o->cplx ? 2 : 1) / 8;
  o->fractional_lo = 0;
  o->deltapol = 0;
  for (int i = 0; i < st->nrecfreqs; i++) {
    double lo = d->freqs[st->recfreq[i]].freq_mhz;
    if (fabs(lo - (int)(lo + 0.5)) > MODE_TINY) o->fractional_lo = 1;
    if (st->clock_offset_delta_us[i] != 0.0) o->deltapol = 1;
  }
}

static inline cf cmul(cf a, cf b)
{
  cf r;
  r.re = a.re * b.re - a.im * b.im;
  r.im = a.re * b.im + a.im * b.re;
  return r;
}

/* State a reference Mode carries across the blocks it processes in order. */
typedef struct { int unpackstart; } mode_state;

/* Mode::process for one block (mode.cpp:634-1374), fringe rotation orders 0, 1 and 2.
   Writes nbands x nchan spectra; returns the data weight (0 = zeroed block).
   FP32 path: float outputs in spec32; FP64 path: double outputs in spec64. */
static float station_block(const gx_job_desc *d, const gx_subint_desc *s, int si, int index,
                           int fp64, mode_state *ms, cf *spec32, cd *spec64, float *bandw)
{
  if (bandw)   /* per-band weights reset at the start of the block (mode.cpp:646-653) */
    for (int b = 0; b < d->stations[si].nbands; b++) bandw[b] = 0.0f;
  const gx_station_desc *st = &d->stations[si];
  stn o;
  stn_init(d, si, &o);
  int nb = st->nbands, N = o.nchan, F = o.fftchannels, S = o.S;
  if (spec32) memset(spec32, 0, sizeof(cf) * nb * N);
  if (spec64) memset(spec64, 0, sizeof(cd) * nb * N);
  const int32_t *ctrl = s->control[si];
  int datasec = ctrl[1], datans = ctrl[2];
  long long datalen = s->datalen[si];
  const double *interp = s->interp + 3 * si;

  int flagword = ctrl[3 + index / FLAGS_PER_INT];
  if (datalen <= 1 || ((flagword >> (index % FLAGS_PER_INT)) & 1) == 0) return 0.0f;

  double fftcentre = index + 0.5;
  double averagedelay = interp[0] * fftcentre * fftcentre + interp[1] * fftcentre + interp[2];
  double fftstartmicrosec = index * F * o.sampletime;
  double starttime = (s->sec - datasec) * 1000000.0 + ((long long)s->ns - (long long)datans) / 1000.0
                     + fftstartmicrosec - averagedelay;
  int nearestsample = (int)(starttime / o.sampletime + 0.5);
  double walltimesecs = s->scan_start_sec + s->sec + s->ns / 1.0e9 + fftstartmicrosec / 1.0e6;
  int intwalltime = (int)walltimesecs;
  double fracwalltime = walltimesecs - intwalltime;

  /* bytes per block numerator / denominator, mode.cpp:131-143, 688 */
  {
    int bits_ts = st->nbands * st->nbits * (o.cplx ? 2 : 1);
    long long need = bits_ts >= 8 ? (long long)(nearestsample + F) * (bits_ts / 8)
                                  : (long long)(nearestsample + F) / (8 / bits_ts);
    if (nearestsample < -1 || need > datalen) return 0.0f;
  }

  float dataweight = 0.0f;
  float *unp = (float *)malloc(sizeof(float) * nb * o.unpacksamples * 2);
  int do_unpack = 1;
  if (nearestsample == -1) nearestsample = 0;
  else if (!(nearestsample < ms->unpackstart || nearestsample > ms->unpackstart + o.unpacksamples - F)) do_unpack = 0;
  if (!do_unpack) { free(unp); return 0.0f; }   /* dataweight stays 0 (mode.cpp:646) */
  ms->unpackstart = nearestsample;
  int good = gxo_unpack(st, o.framesamples, s->data[si], datalen, nearestsample, o.unpacksamples, unp);
  float goodsamples = (float)good;
  if (st->interlaced) {
    int invalid[GX_MAX_BANDS], totalinvalid = 0;
    edv4_blank(st, s->data[si], datalen, nearestsample, o.unpacksamples, unp, invalid);
    for (int b = 0; b < nb; b++) {
      if (bandw) bandw[b] = (goodsamples - invalid[b]) / (float)o.unpacksamples;
      totalinvalid += invalid[b];
    }
    goodsamples -= (float)totalinvalid / (float)nb;
    if (goodsamples < 0) goodsamples = 0;
  }
  dataweight = goodsamples / (float)o.unpacksamples;
  if (bandw && !st->interlaced)
    for (int b = 0; b < nb; b++) bandw[b] = dataweight;
  if (!(dataweight > 0.0f)) { free(unp); return 0.0f; }

  double nearestsampletime = nearestsample * o.sampletime;
  float fracsampleerror = (float)(starttime - nearestsampletime);
  double fracerr64 = starttime - nearestsampletime;

  /* delay interpolation by FRINGE ROTN ORDER, mode.cpp:776-826 */
  const int order = d->fringe_rotation_order;
  double *subxval = (double *)malloc(sizeof(double) * S);
  double *stepxval = (double *)malloc(sizeof(double) * o.nfr);
  double *quadxval = (double *)malloc(sizeof(double) * S);
  int integerdelay = 0;
  double postf_b = 0.0;   /* post-F: block-centre delay without its integer part */
  if (order == 0) {
    integerdelay = (int)averagedelay;
    postf_b = averagedelay - integerdelay;
    for (int k = 0; k < S; k++) subxval[k] = quadxval[k] = 0.0;
    for (int j = 0; j < o.nfr; j++) stepxval[j] = 0.0;
  } else if (order == 2) {
    double qa = interp[0];
    double qb = interp[1] + index * interp[0] * 2.0;
    double c = interp[2] + index * interp[1] + index * index * interp[0];
    integerdelay = (int)c;
    c -= integerdelay;
    double s1 = (double)S / (double)F;   /* stepxoff[1] */
    for (int k = 0; k < S; k++) {
      subxval[k] = ((double)k / (double)F) * (qb + qa * s1);
      subxval[k] += c;
      quadxval[k] = ((double)k / (double)F) * (2 * qa * s1);
    }
    for (int j = 0; j < o.nfr; j++) {
      double x = (double)(j * S) / (double)F;
      stepxval[j] = x * qb + (x * x) * qa;
    }
  } else {
    double d0 = interp[0] * index * index + interp[1] * index + interp[2];
    double d1 = interp[0] * (index + 0.5) * (index + 0.5) + interp[1] * (index + 0.5) + interp[2];
    double d2 = interp[0] * (index + 1) * (index + 1) + interp[1] * (index + 1) + interp[2];
    double a = d2 - d0;
    double b = d0 + (d1 - (a * 0.5 + d0)) / 3.0;
    integerdelay = (int)b;
    b -= integerdelay;
    for (int k = 0; k < S; k++) { subxval[k] = ((double)k / (double)F) * a; subxval[k] += b; quadxval[k] = 0.0; }
    for (int j = 0; j < o.nfr; j++) stepxval[j] = ((double)(j * S) / (double)F) * a;
  }

  cf *rot = (cf *)malloc(sizeof(cf) * F);
  cd *rot64 = (cd *)malloc(sizeof(cd) * F);
  cf *fracA = (cf *)malloc(sizeof(cf) * N), *fracB = (cf *)malloc(sizeof(cf) * N);
  cd *frac64A = (cd *)malloc(sizeof(cd) * N), *frac64B = (cd *)malloc(sizeof(cd) * N);
  double *buf = (double *)malloc(sizeof(double) * 2 * F);
  float *fbuf = (float *)malloc(sizeof(float) * 2 * F);
  int half = o.nfrac / 2;

  for (int fi = 0; fi < st->nrecfreqs; fi++) {
    const gx_freq_desc *fq = &d->freqs[st->recfreq[fi]];
    int lsb = fq->lower_sideband;
    double looffset = st->lo_offset_hz[fi];
    int looff = (looffset > 0.0 || looffset < 0.0);
    double fraclooffset = 0.0;
    int isfraclooffset = 0;
    if (looff) {
      fraclooffset = fabs(looffset) - (int)fabs(looffset);
      if (fraclooffset > MODE_TINY) isfraclooffset = 1;
      if (looffset < 0) fraclooffset = -fraclooffset;
    }
    double lofreq = fq->freq_mhz;
    if (o.cplx && lsb) lofreq = -lofreq;

    /* post-F fringe phase at the block centre (mode.cpp:1038-1049) */
    double postf_ph = 0.0;
    if (order == 0) {
      postf_ph = postf_b * lofreq;
      if (o.fractional_lo) postf_ph += integerdelay * (lofreq - (int)lofreq);
      postf_ph -= walltimesecs * looffset;
    }
    /* fringe rotator, mode.cpp:831-1005 (none before the FFT for post-F) */
    if (order == 0) {
      for (int n = 0; n < F; n++) { rot[n].re = 1.0f; rot[n].im = 0.0f; rot64[n].re = 1.0; rot64[n].im = 0.0; }
    } else if (!fp64) {
      float *subarg = (float *)malloc(sizeof(float) * S), *steparg = (float *)malloc(sizeof(float) * o.nfr);
      for (int k = 0; k < S; k++) {
        double ph = subxval[k] * lofreq;
        if (o.fractional_lo) ph += (lofreq - (int)lofreq) * (double)integerdelay;
        if (looff) {
          ph += (k * o.sampletime / 1e6) * -looffset;
          ph += -looffset * fracwalltime;
          if (isfraclooffset) ph += -fraclooffset * intwalltime;
        }
        subarg[k] = (float)(-TWO_PI * (ph - (int)ph));
      }
      for (int j = 0; j < o.nfr; j++) {
        double ph = stepxval[j] * lofreq;
        if (looff) ph += (j * S * o.sampletime / 1e6) * -looffset;
        steparg[j] = (float)(-TWO_PI * (ph - (int)ph));
      }
      cf *stepc = (cf *)malloc(sizeof(cf) * o.nfr);
      for (int k = 0; k < S; k++) { rot[k].re = cosf(subarg[k]); rot[k].im = sinf(subarg[k]); }
      for (int j = 0; j < o.nfr; j++) { stepc[j].re = cosf(steparg[j]); stepc[j].im = sinf(steparg[j]); }
      if (order == 2) {
        /* piecewise rotator times step[j], then piecewise *= quad (mode.cpp:996-1005) */
        cf *pw = (cf *)malloc(sizeof(cf) * S), *quad = (cf *)malloc(sizeof(cf) * S);
        for (int k = 0; k < S; k++) {
          double ph = quadxval[k] * lofreq;
          float qarg = (float)(-TWO_PI * (ph - (int)ph));
          quad[k].re = cosf(qarg); quad[k].im = sinf(qarg);
          pw[k] = rot[k];
        }
        for (int j = 0; j < o.nfr; j++)
          for (int k = 0; k < S; k++) {
            rot[j * S + k] = cmul(pw[k], stepc[j]);
            pw[k] = cmul(quad[k], pw[k]);
          }
        free(pw); free(quad);
      } else {
        for (int j = 1; j < o.nfr; j++)
          for (int k = 0; k < S; k++) rot[j * S + k] = cmul(rot[k], stepc[j]);
      }
      free(stepc); free(subarg); free(steparg);
    } else {
      for (int n = 0; n < F; n++) {
        int k = n % S, j = n / S;
        double ph = (subxval[k] + stepxval[j] + quadxval[k] * j) * lofreq;
        if (o.fractional_lo) ph += (lofreq - (int)lofreq) * (double)integerdelay;
        if (looff) {
          ph += (n * o.sampletime / 1e6) * -looffset;
          ph += -looffset * fracwalltime;
          if (isfraclooffset) ph += -fraclooffset * intwalltime;
        }
        double arg = -TWO_PI * (ph - floor(ph));
        rot64[n].re = cos(arg); rot64[n].im = sin(arg);
      }
    }

    /* fractional-sample rotator, mode.cpp:1029-1122 */
    for (int pol = 0; pol < (o.deltapol ? 2 : 1); pol++) {
      double sgn = pol == 0 ? 1.0 : -1.0;
      if (!fp64) {
        float val = (float)(fracsampleerror - st->clock_offset_us[fi] + sgn * st->clock_offset_delta_us[fi] / 2);
        cf *fr = pol == 0 ? fracA : fracB;
        cf *stepc = (cf *)malloc(sizeof(cf) * (half > 0 ? half : 1));
        float prf = order == 0 ? (float)(-TWO_PI * (postf_ph - (int)postf_ph)) : 0.0f;
        for (int k = 0; k < S; k++) {
          float cfreq = (float)((TWO_PI * (k) * o.bw) / N);
          float arg = cfreq * val;
          if (order == 0) arg = arg + prf;
          fr[k].re = cosf(arg); fr[k].im = sinf(arg);
        }
        for (int j = 0; j < half; j++) {
          float sfreq = lsb ? (float)((-TWO_PI * ((half - j) * S) * o.bw) / N)
                            : (float)((TWO_PI * j * S * o.bw) / N);
          float arg = sfreq * val;
          stepc[j].re = cosf(arg); stepc[j].im = sinf(arg);
        }
        for (int j = 1; j < half; j++)
          for (int k = 0; k < S; k++) fr[j * S + k] = cmul(fr[k], stepc[j]);
        for (int k = 0; k < S; k++) fr[k] = cmul(fr[k], stepc[0]);
        free(stepc);
      } else {
        double val = fracerr64 - st->clock_offset_us[fi] + sgn * st->clock_offset_delta_us[fi] / 2;
        cd *fr = pol == 0 ? frac64A : frac64B;
        for (int c = 0; c < N; c++) {
          int k = c % S, j = c / S;
          double cfreq = TWO_PI * k * o.bw / N;
          /* every stride, the first included (mode.cpp:1071), carries step[j] */
          double sfreq = lsb ? (-TWO_PI * ((half - j) * S) * o.bw) / N : (TWO_PI * j * S * o.bw) / N;
          double arg = (cfreq + sfreq) * val;
          if (order == 0) arg += -TWO_PI * (postf_ph - floor(postf_ph));
          fr[c].re = cos(arg); fr[c].im = sin(arg);
        }
      }
    }

    /* every recorded band of this freq, mode.cpp:1124-1285 */
    for (int bd = 0; bd < nb; bd++) {
      if (st->band_localfreq[bd] != fi) continue;
      const float *x = unp + (long long)bd * o.unpacksamples * (o.cplx ? 2 : 1);
      int useB = o.deltapol && st->band_pol[bd] != 'R';
      if (!fp64) {
        for (int n = 0; n < F; n++) {
          cf v;
          if (o.cplx) { cf u = {x[2 * n], x[2 * n + 1]}; v = cmul(rot[n], u); }
          else { v.re = x[n] * rot[n].re - 0.0f * rot[n].im; v.im = x[n] * rot[n].im + 0.0f * rot[n].re; }
          fbuf[2 * n] = v.re; fbuf[2 * n + 1] = v.im;
        }
        gxfft_c2c_f32(fbuf, fbuf, F, -1);
        cf *out = spec32 + (long long)bd * N;
        for (int c = 0; c < N; c++) {
          int src;
          float sg = 1.0f;
          if (!o.cplx) src = lsb ? N + c : c;
          else if (!lsb) src = c;
          else { src = c == 0 ? 0 : F - c; sg = c == 0 ? 1.0f : -1.0f; }
          out[c].re = fbuf[2 * src]; out[c].im = sg * fbuf[2 * src + 1];
          out[c] = cmul(out[c], (useB ? fracB : fracA)[c]);
        }
      } else {
        for (int n = 0; n < F; n++) {
          double ur = o.cplx ? x[2 * n] : x[n], ui = o.cplx ? x[2 * n + 1] : 0.0;
          buf[2 * n] = ur * rot64[n].re - ui * rot64[n].im;
          buf[2 * n + 1] = ur * rot64[n].im + ui * rot64[n].re;
        }
        gxfft_c2c_f64(buf, F, -1);
        cd *out = spec64 + (long long)bd * N;
        for (int c = 0; c < N; c++) {
          int src;
          double sg = 1.0;
          if (!o.cplx) src = lsb ? N + c : c;
          else if (!lsb) src = c;
          else { src = c == 0 ? 0 : F - c; sg = c == 0 ? 1.0 : -1.0; }
          double re = buf[2 * src], im = sg * buf[2 * src + 1];
          cd r = (useB ? frac64B : frac64A)[c];
          out[c].re = re * r.re - im * r.im;
          out[c].im = re * r.im + im * r.re;
        }
      }
    }
  }
  free(subxval); free(stepxval); free(quadxval); free(rot); free(rot64); free(fracA); free(fracB);
  free(frac64A); free(frac64B); free(buf); free(fbuf); free(unp);
  return dataweight;
}

int gxo_station_block(const gx_job_desc *d, const gx_subint_desc *s, int station, int block,
                      const gxo_params *p, double *spectra, double *weight)
{
  const gx_station_desc *st = &d->stations[station];
  int N = d->freqs[st->recfreq[0]].nchan;
  mode_state ms = {-999999999};
  float w;
  if (p->precision == GXO_FP64) {
    cd *sp = (cd *)malloc(sizeof(cd) * st->nbands * N);
    w = station_block(d, s, station, block, 1, &ms, 0, sp, 0);
    memcpy(spectra, sp, sizeof(cd) * st->nbands * N);
    free(sp);
  } else {
    cf *sp = (cf *)malloc(sizeof(cf) * st->nbands * N);
    w = station_block(d, s, station, block, 0, &ms, sp, 0, 0);
    for (int i = 0; i < st->nbands * N; i++) { spectra[2 * i] = sp[i].re; spectra[2 * i + 1] = sp[i].im; }
    free(sp);
  }
  *weight = w;
  return 0;
}

/* ------------------------------------------------------------------ subint */

/* Core::processdata for one thread's block range (core.cpp:657-1129), with
   uvshiftAndAverage / averageAndSendAutocorrs flushes (core.cpp:986-1001,
   1055-1063) and the final baseline-weight copy (core.cpp:1066-1112). */
int gxo_subint(const gx_job_desc *d, const gx_subint_desc *s, const gxo_params *p, double *results)
{
  int nst = d->nstations, nbl = d->nbaselines;
  int *blofs = (int *)malloc(sizeof(int) * d->nfreqs * (nbl ? nbl : 1));
  int *bwofs = (int *)malloc(sizeof(int) * d->nfreqs * (nbl ? nbl : 1));
  int *acofs = (int *)malloc(sizeof(int) * nst), *acwofs = (int *)malloc(sizeof(int) * nst);
  long long rl = gxo_layout(d, blofs, bwofs, acofs, acwofs);
  int fp64 = p->precision == GXO_FP64;
  int maxprod = max_products(d);
  int writecross = d->write_autocorrs && maxprod > 2;
  stn o0;
  stn_init(d, 0, &o0);
  double ffttime_ns = 1000.0 * o0.nchan / o0.bw;
  int bps = (int)(d->subint_ns / ffttime_ns + 0.5);
  double blockns = (double)d->subint_ns / (double)bps;
  int nbuf = p->num_buffered_ffts > 0 ? p->num_buffered_ffts : 1;
  int maxxc = (int)(p->xc_avg_ns / blockns); maxxc -= maxxc % nbuf; if (maxxc == 0) maxxc = nbuf;
  int maxac = (int)(p->ac_avg_ns / blockns); maxac -= maxac % nbuf; if (maxac == 0) maxac = nbuf;
  int nthreads = p->nthreads > 0 ? p->nthreads : 1;

  /* results in float (FP32 path) or double */
  float *r32 = (float *)calloc(2 * rl, sizeof(float));
  double *r64 = (double *)calloc(2 * rl, sizeof(double));

  /* per-station spectra of one block */
  int maxnb = 0, maxN = 0;
  for (int i = 0; i < nst; i++) {
    if (d->stations[i].nbands > maxnb) maxnb = d->stations[i].nbands;
    int n = d->freqs[d->stations[i].recfreq[0]].nchan;
    if (n > maxN) maxN = n;
  }
  cf *sp32 = (cf *)malloc(sizeof(cf) * nst * maxnb * maxN);
  cd *sp64 = (cd *)malloc(sizeof(cd) * nst * maxnb * maxN);
  float *w = (float *)malloc(sizeof(float) * nst);
  float *wb = (float *)calloc((size_t)nst * maxnb, sizeof(float));   /* per-band weights (getDataWeight) */
  /* accumulators: cross [f][bl][p][c]; autos [st][2][band][c]; weights */
  long long crosslen = rl;
  cf *xc32 = (cf *)calloc(crosslen, sizeof(cf));
  cd *xc64 = (cd *)calloc(crosslen, sizeof(cd));
  cf *ac32 = (cf *)calloc((long long)nst * 2 * maxnb * maxN, sizeof(cf));
  cd *ac64 = (cd *)calloc((long long)nst * 2 * maxnb * maxN, sizeof(cd));
  float *acw32 = (float *)calloc(nst * 2 * maxnb, sizeof(float));
  double *acw64 = (double *)calloc(nst * 2 * maxnb, sizeof(double));
  float *bw32 = (float *)calloc(d->nfreqs * nbl * 4 + 1, sizeof(float));
  double *bw64 = (double *)calloc(d->nfreqs * nbl * 4 + 1, sizeof(double));
  mode_state *ms = (mode_state *)malloc(sizeof(mode_state) * nst);

  int startblock = 0, numblocks = 0;
  for (int t = 0; t < nthreads; t++) {
    startblock += numblocks;
    numblocks = bps / nthreads + ((t < bps % nthreads) ? 1 : 0);
    for (int i = 0; i < nst; i++) ms[i].unpackstart = -999999999;
    memset(bw32, 0, sizeof(float) * (d->nfreqs * nbl * 4 + 1));
    memset(bw64, 0, sizeof(double) * (d->nfreqs * nbl * 4 + 1));
    int xccount = 0, account = 0;
    int nloops = numblocks / nbuf + (numblocks % nbuf ? 1 : 0);
    for (int loop = 0; loop < nloops; loop++) {
      int nproc = 0;
      for (int sub = 0; sub < nbuf; sub++) {
        int blk = loop * nbuf + sub + startblock;
        if (blk >= startblock + numblocks) break;
        nproc++;
        for (int i = 0; i < nst; i++) {
          const gx_station_desc *st = &d->stations[i];
          int N = d->freqs[st->recfreq[0]].nchan;
          cf *o32 = sp32 + (long long)i * maxnb * maxN;
          cd *o64 = sp64 + (long long)i * maxnb * maxN;
          w[i] = station_block(d, s, i, blk, fp64, &ms[i], fp64 ? 0 : o32, fp64 ? o64 : 0, wb + i * maxnb);
          if (w[i] > 0.0f) {
            /* autocorrelations and their weights, mode.cpp:1270-1284, 1333-1352 */
            for (int bd = 0; bd < st->nbands; bd++) {
              long long ab = ((long long)i * 2 * maxnb + bd) * maxN;
              for (int c = 0; c < N; c++) {
                if (!fp64) {
                  cf a = o32[bd * maxN + c], cj = {a.re, -a.im};
                  ac32[ab + c].re += a.re * cj.re - a.im * cj.im;
                  ac32[ab + c].im += a.re * cj.im + a.im * cj.re;
                } else {
                  cd a = o64[bd * maxN + c];
                  ac64[ab + c].re += a.re * a.re + a.im * a.im;
                }
              }
              acw32[i * 2 * maxnb + bd] += wb[i * maxnb + bd];
              acw64[i * 2 * maxnb + bd] += wb[i * maxnb + bd];
            }
            if (d->write_autocorrs) {
              for (int fi = 0; fi < st->nrecfreqs; fi++) {
                int idx[8], cnt = 0;
                for (int bd = 0; bd < st->nbands; bd++) if (st->band_localfreq[bd] == fi && cnt < 8) idx[cnt++] = bd;
                if (cnt < 2) continue;
                for (int q = 0; q < 2; q++) {
                  int b0 = idx[q], b1 = idx[1 - q];
                  long long ab = ((long long)i * 2 * maxnb + maxnb + b0) * maxN;
                  for (int c = 0; c < N; c++) {
                    if (!fp64) {
                      cf x0 = o32[b0 * maxN + c], x1 = o32[b1 * maxN + c], cj = {x1.re, -x1.im};
                      ac32[ab + c].re += x0.re * cj.re - x0.im * cj.im;
                      ac32[ab + c].im += x0.re * cj.im + x0.im * cj.re;
                    } else {
                      cd x0 = o64[b0 * maxN + c], x1 = o64[b1 * maxN + c];
                      ac64[ab + c].re += x0.re * x1.re + x0.im * x1.im;
                      ac64[ab + c].im += -x0.re * x1.im + x0.im * x1.re;
                    }
                  }
                  /* interlaced: the product of the two bands' weights */
                  float xw = st->interlaced ? wb[i * maxnb + idx[0]] * wb[i * maxnb + idx[1]] : w[i];
                  acw32[i * 2 * maxnb + maxnb + b0] += xw;
                  acw64[i * 2 * maxnb + maxnb + b0] += xw;
                }
              }
            }
          }
        }
        /* XMAC, core.cpp:884-968: vis1 * conj(vis2) accumulated per block */
        for (int f = 0; f < d->nfreqs; f++) {
          for (int j = 0; j < nbl; j++) {
            const gx_baseline_desc *bl = &d->baselines[j];
            int lf = bl_localfreq(bl, f);
            if (lf < 0) continue;
            int N = d->freqs[f].nchan;
            for (int pp = 0; pp < bl->npolprod[lf]; pp++) {
              long long base = blofs[f * nbl + j] + (long long)pp * N;
              int b1 = bl->band1[lf][pp], b2 = bl->band2[lf][pp];
              for (int c = 0; c < N; c++) {
                if (!fp64) {
                  cf x1 = sp32[((long long)bl->ds1 * maxnb + b1) * maxN + c];
                  cf x2 = sp32[((long long)bl->ds2 * maxnb + b2) * maxN + c];
                  cf v2 = {x2.re, -x2.im};
                  xc32[base + c].re += x1.re * v2.re - x1.im * v2.im;
                  xc32[base + c].im += x1.re * v2.im + x1.im * v2.re;
                } else {
                  cd x1 = sp64[((long long)bl->ds1 * maxnb + b1) * maxN + c];
                  cd x2 = sp64[((long long)bl->ds2 * maxnb + b2) * maxN + c];
                  xc64[base + c].re += x1.re * x2.re + x1.im * x2.im;
                  xc64[base + c].im += -x1.re * x2.im + x1.im * x2.re;
                }
              }
              /* baseline weight, core.cpp:1039-1044 */
              float w1 = wb[bl->ds1 * maxnb + b1], w2 = wb[bl->ds2 * maxnb + b2];
              float bwv = w1 * w2;
              bw32[(f * nbl + j) * 4 + pp] += bwv;
              bw64[(f * nbl + j) * 4 + pp] += (double)w1 * (double)w2;
            }
          }
        }
      }
      xccount += nproc;
      account += nproc;
      int lastloop = (loop == nloops - 1);
      if (xccount == maxxc || (lastloop && xccount != 0)) {
        for (long long e = 0; e < crosslen; e++) {
          r32[2 * e] += xc32[e].re; r32[2 * e + 1] += xc32[e].im;
          r64[2 * e] += xc64[e].re; r64[2 * e + 1] += xc64[e].im;
        }
        memset(xc32, 0, sizeof(cf) * crosslen);
        memset(xc64, 0, sizeof(cd) * crosslen);
        xccount = 0;
      }
      if (account == maxac || (lastloop && account != 0)) {
        for (int i = 0; i < nst; i++) {
          const gx_station_desc *st = &d->stations[i];
          int N = d->freqs[st->recfreq[0]].nchan;
          long long ro = acofs[i];
          for (int bd = 0; bd < st->nbands; bd++, ro += N) {
            long long ab = ((long long)i * 2 * maxnb + bd) * maxN;
            for (int c = 0; c < N; c++) {
              r32[2 * (ro + c)] += ac32[ab + c].re; r32[2 * (ro + c) + 1] += ac32[ab + c].im;
              r64[2 * (ro + c)] += ac64[ab + c].re; r64[2 * (ro + c) + 1] += ac64[ab + c].im;
            }
          }
          if (writecross) {
            for (int bd = 0; bd < st->nbands; bd++, ro += N) {
              long long ab = ((long long)i * 2 * maxnb + maxnb + bd) * maxN;
              for (int c = 0; c < N; c++) {
                r32[2 * (ro + c)] += ac32[ab + c].re; r32[2 * (ro + c) + 1] += ac32[ab + c].im;
                r64[2 * (ro + c)] += ac64[ab + c].re; r64[2 * (ro + c) + 1] += ac64[ab + c].im;
              }
            }
          }
          long long wo = 2LL * acwofs[i];
          for (int bd = 0; bd < st->nbands; bd++, wo++) {
            r32[wo] += acw32[i * 2 * maxnb + bd];
            r64[wo] += acw64[i * 2 * maxnb + bd];
          }
          if (writecross)
            for (int bd = 0; bd < st->nbands; bd++, wo++) {
              r32[wo] += acw32[i * 2 * maxnb + maxnb + bd];
              r64[wo] += acw64[i * 2 * maxnb + maxnb + bd];
            }
        }
        memset(ac32, 0, sizeof(cf) * nst * 2 * maxnb * maxN);
        memset(ac64, 0, sizeof(cd) * nst * 2 * maxnb * maxN);
        memset(acw32, 0, sizeof(float) * nst * 2 * maxnb);
        memset(acw64, 0, sizeof(double) * nst * 2 * maxnb);
        account = 0;
      }
    }
    for (int f = 0; f < d->nfreqs; f++)
      for (int j = 0; j < nbl; j++) {
        int lf = bl_localfreq(&d->baselines[j], f);
        if (lf < 0) continue;
        for (int pp = 0; pp < d->baselines[j].npolprod[lf]; pp++) {
          r32[2LL * bwofs[f * nbl + j] + pp] += bw32[(f * nbl + j) * 4 + pp];
          r64[2LL * bwofs[f * nbl + j] + pp] += bw64[(f * nbl + j) * 4 + pp];
        }
      }
  }
  for (long long e = 0; e < 2 * rl; e++) results[e] = fp64 ? r64[e] : (double)r32[e];
  free(blofs); free(bwofs); free(acofs); free(acwofs); free(r32); free(r64); free(sp32); free(sp64);
  free(w); free(wb); free(xc32); free(xc64); free(ac32); free(ac64); free(acw32); free(acw64); free(bw32); free(bw64); free(ms);
  return 0;
}
