// GpuCore (see gpucore.h): gxcorr jobs built from the Configuration, one
// gx_subint per slot.
#include "gpucore.h"

#include <cmath>
#include <cstring>
#include "alert.h"
#include "model.h"

GpuCore::GpuCore(int id, Configuration *conf, int *dids, MPI_Comm rcomm, int dev, int xs)
    : Core(id, conf, dids, rcomm), device(dev), xstep(xs)
{
  jobs.resize(conf->getNumConfigs());
}

GpuCore::~GpuCore()
{
  for (Job &j : jobs)
    if (j.h) gx_close(j.h);
}

// The descriptor of one configuration: freq table, datastreams (the
// arguments Configuration::getMode passes to a Mk5Mode, configuration.cpp:
// 932-998) and baselines (configuration.cpp:1033-1180).
int GpuCore::build(int ci, Job &job)
{
  Configuration *c = config;
  const Configuration::configdata &cd = c->configs[ci];
  for (int f = 0; f < c->getFreqTableLength(); f++) {
    gx_freq_desc d = {};
    d.freq_mhz = c->getFreqTableFreq(f);
    d.bw_mhz = c->getFreqTableBandwidth(f);
    d.lower_sideband = c->getFreqTableLowerSideband(f) ? 1 : 0;
    d.nchan = c->getFNumChannels(f);
    d.chans_to_average = c->getFChannelsToAverage(f);
    job.fr.push_back(d);
  }
  for (int ds = 0; ds < numdatastreams; ds++) {
    const Configuration::datastreamdata &dd = c->datastreamtable[cd.datastreamindices[ds]];
    gx_station_desc s = {};
    s.nbits = c->getDNumBits(ci, ds);
    s.is_complex = c->getDSampling(ci, ds) == Configuration::COMPLEX ? 1 : 0;
    s.interlaced = c->getDataFormat(ci, ds) == Configuration::INTERLACEDVDIF ? 1 : 0;
    // the frames the Core receives: multiplexed ones for INTERLACEDVDIF (configuration.cpp:980-985)
    s.framebytes = s.interlaced ? c->getMultiplexedFrameBytes(ci, ds) : c->getFrameBytes(ci, ds);
    s.nrecfreqs = c->getDNumRecordedFreqs(ci, ds);
    if (s.nrecfreqs > GX_MAX_LOCAL_FREQS) {
      err = "too many recorded frequencies";
      return GX_ERR_UNSUPPORTED;
    }
    for (int i = 0; i < s.nrecfreqs; i++) {
      s.recfreq[i] = c->getDRecordedFreqFreqTableIndex(ci, ds, i);
      s.clock_offset_us[i] = dd.recordedfreqclockoffsets[i];
      s.clock_offset_delta_us[i] = dd.recordedfreqclockoffsetsdelta[i];
      s.lo_offset_hz[i] = dd.recordedfreqlooffsets[i];
      if (dd.recordedfreqphaseoffset[i] != 0.0) {
        err = "phase offsets between polarisations are not implemented by gxcorr";
        return GX_ERR_UNSUPPORTED;
      }
    }
    s.nbands = c->getDNumRecordedBands(ci, ds);
    s.nzoomfreqs = dd.numzoomfreqs;
    s.nzoombands = c->getDNumZoomBands(ci, ds);
    if (s.nbands + s.nzoombands > GX_MAX_BANDS || s.nzoomfreqs > GX_MAX_LOCAL_FREQS) {
      err = "too many recorded or zoom bands";
      return GX_ERR_UNSUPPORTED;
    }
    for (int b = 0; b < s.nbands; b++) {
      s.band_localfreq[b] = c->getDLocalRecordedFreqIndex(ci, ds, b);
      s.band_pol[b] = c->getDRecordedBandPol(ci, ds, b);
    }
    // zoom freqs and bands (the device finds their parents and offsets as Configuration does)
    for (int i = 0; i < s.nzoomfreqs; i++) s.zoomfreq[i] = dd.zoomfreqtableindices[i];
    for (int b = 0; b < s.nzoombands; b++) {
      s.zoomband_localfreq[b] = c->getDLocalZoomFreqIndex(ci, ds, b);
      s.zoomband_pol[b] = c->getDZoomBandPol(ci, ds, b);
    }
    // the VDIF threads (setDatastreamMuxInfo, configuration.cpp:2632-2651), for a ring's multiplexer
    if (s.interlaced) {
      s.nmuxthreads = c->getDNumMuxThreads(ci, ds);
      if (s.nmuxthreads > GX_MAX_MUX_THREADS) {
        err = "more than 64 VDIF threads";
        return GX_ERR_UNSUPPORTED;
      }
      for (int t = 0; t < s.nmuxthreads; t++) s.muxthread[t] = c->getDMuxThreadMap(ci, ds)[t];
    }
    s.clock_int_seconds = (int)std::floor(c->getDClockCoeff(ci, ds, 0) / 1000000.0 + 0.5);   // mode.cpp:68
    s.phase_cal_interval_hz = c->getDPhaseCalIntervalHz(ci, ds);
    s.phase_cal_base_hz = c->getDPhaseCalBaseHz(ci, ds);
    if (s.phase_cal_interval_hz > 0 && c->getDPhaseCalDenominator(ci, ds) != 1) {
      err = "PHASE CAL DIVISOR other than 1 is not implemented by gxcorr";
      return GX_ERR_UNSUPPORTED;
    }
    job.st.push_back(s);
  }
  for (int b = 0; b < numbaselines; b++) {
    gx_baseline_desc d = {};
    d.ds1 = c->getBOrderedDataStream1Index(ci, b);
    d.ds2 = c->getBOrderedDataStream2Index(ci, b);
    d.nfreqs = c->getBNumFreqs(ci, b);
    for (int f = 0; f < d.nfreqs; f++) {
      d.freq[f] = c->getBFreqIndex(ci, b, f);
      d.npolprod[f] = c->getBNumPolProducts(ci, b, f);
      for (int p = 0; p < d.npolprod[f]; p++) {
        d.band1[f][p] = c->getBDataStream1BandIndex(ci, b, f, p);
        d.band2[f][p] = c->getBDataStream2BandIndex(ci, b, f, p);
      }
    }
    job.bl.push_back(d);
  }
  gx_job_desc jd = {};
  jd.nstations = (int)job.st.size();
  jd.stations = job.st.data();
  jd.nfreqs = (int)job.fr.size();
  jd.freqs = job.fr.data();
  jd.nbaselines = (int)job.bl.size();
  jd.baselines = job.bl.data();
  jd.subint_ns = c->getSubintNS(ci);
  jd.guard_ns = c->getGuardNS(ci);
  jd.fringe_rotation_order = cd.fringerotationorder;
  jd.array_stride = c->getArrayStrideLength(ci, 0);
  jd.xmac_stride = c->getXmacStrideLength(ci);
  jd.write_autocorrs = c->writeAutoCorrs(ci) ? 1 : 0;
  jd.max_data_bytes = databytes;   // the Core's receive buffer per datastream
  jd.xstep = xstep;
  const gx_status s = gx_open(&jd, device, &job.h);
  if (s != GX_OK) {
    err = std::string("gx_open: ") + gx_status_string(s);
    job.h = nullptr;
    return s;
  }
  return GX_OK;
}

gx_handle *GpuCore::handle(int ci)
{
  if (ci < 0 || ci >= (int)jobs.size()) return nullptr;
  if (!jobs[ci].h && build(ci, jobs[ci]) != GX_OK) return nullptr;
  return jobs[ci].h;
}

bool GpuCore::interpolator(int ci, int ds, int scan, int sec, int ns, double out[3])
{
  // Mode::setOffsets: sample time of the datastream's first recorded band,
  // the span of the slot's FFT blocks, the source (1 with one phase centre)
  const Configuration::datastreamdata &dd = config->datastreamtable[config->configs[ci].datastreamindices[ds]];
  const bool cplx = config->getDSampling(ci, ds) == Configuration::COMPLEX;
  const double bw = config->getFreqTableBandwidth(dd.recordedfreqtableindices[0]);
  const int nchan = config->getFNumChannels(dd.recordedfreqtableindices[0]);
  double sampletime = 1.0 / (2.0 * bw);   // us
  if (cplx) sampletime *= 2.0;
  const int bps = config->getBlocksPerSend(ci);
  double timespan = bps * 2 * nchan * sampletime / 1e6;
  if (cplx) timespan /= 2;
  const int srcindex = model->getNumPhaseCentres(scan) == 1 ? 1 : 0;
  const bool ok = model->calculateDelayInterpolator(scan, (double)sec + (double)ns / 1000000000.0, timespan, bps,
                                                    config->getDModelFileIndex(ci, ds), srcindex, 2, out);
  out[2] -= 1000000 * (int)std::floor(config->getDClockCoeff(ci, ds, 0) / 1000000.0 + 0.5);
  return ok;
}

int GpuCore::correlateslot(int index)
{
  Core::processslot &slot = procslots[index];
  const int ci = slot.configindex;
  gx_handle *h = handle(ci);
  if (!h) return GX_ERR_STATE;
  const int nds = numdatastreams;
  std::vector<double> interp(3 * nds);
  std::vector<int64_t> len(nds);
  for (int ds = 0; ds < nds; ds++) {
    if (!interpolator(ci, ds, slot.offsets[0], slot.offsets[1], slot.offsets[2], &interp[3 * ds])) {
      // no model for this subint: Mode::setOffsets torches it (mode.cpp:1528-1531)
      memset(slot.results, 0, sizeof(cf32) * config->getCoreResultLength(ci));
      err = "no delay model for this subint";
      return GX_OK;
    }
    len[ds] = slot.datalengthbytes[ds];
  }
  gx_subint_desc sd = {};
  sd.scan = slot.offsets[0];
  sd.sec = slot.offsets[1];
  sd.ns = slot.offsets[2];
  sd.scan_start_sec = model->getScanStartSec(slot.offsets[0], startmjd, startseconds);
  sd.interp = interp.data();
  sd.data = (const uint8_t *const *)slot.databuffer;
  sd.datalen = len.data();
  sd.control = (const int32_t *const *)slot.controlbuffer;
  sd.controllen = controllength;
  const gx_status s = gx_subint(h, &sd, (float *)slot.results);
  if (s != GX_OK) err = std::string("gx_subint: ") + gx_last_error(h);
  return s;
}

void GpuCore::processdata(int index, int threadid, int, int, Mode **, Polyco *, threadscratchspace *)
{
  if (threadid != 0) return;   // thread 0 correlates the whole slot
  if (correlateslot(index) != GX_OK) csevere << startl << "gxcorr: " << err << endl;
}
