/*
 * gxcorr -- B200-native FX correlation for DiFX's Mode/Core hot path.
 *
 * C ABI.  Plain structs, pointers and sizes; no C++ or CUDA types cross it.
 * One handle = one correlation configuration on one GPU, with its own CUDA
 * stream; calls on one handle are serialised by the caller (the reference
 * gives each Core process thread its own Mode objects in the same way,
 * mpifxcorr/src/core.cpp:2186-2193).  Every call returns a gx_status; no
 * exceptions cross the ABI; gx_last_error() gives the message of the last
 * failure on a handle.
 *
 * What each entry point replaces in the reference:
 *
 *   gx_open            Configuration::getMode for every datastream plus the
 *                      result-layout computation Core relies on
 *                      (configuration.cpp:932-998, populateResultLengths
 *                      2348-2630, setStrides 2701-2734).
 *   gx_open_input      new Configuration(file) (non-MPI ctor,
 *                      configuration.cpp:98) + Model(.calc/.im)
 *                      (model.cpp:20-76) + the same as gx_open.
 *   gx_interpolator    Model::calculateDelayInterpolator as called from
 *                      Mode::setOffsets (model.cpp:219-289, mode.cpp:1502-1532).
 *   gx_subint          one Core slot through Core::processdata (core.cpp:657-1129):
 *                      for every datastream setValidFlags/setData/setOffsets
 *                      (mode.cpp:1534-1550) and Mode::process on every FFT
 *                      block (mode.cpp:634-1374, Mk5Mode::unpack
 *                      mk5mode.cpp:94-174), then the baseline XMAC
 *                      (core.cpp:816-982), baseline weights (core.cpp:1005-1052),
 *                      autocorrelation copy (core.cpp:1166-1376) and
 *                      visibility copy (core.cpp:1605-1884), writing the Core
 *                      result array (procslots[].results) layout.
 *   gx_subint_device   the same with every buffer already in device memory.
 *   gx_spectra         Mode::getFreqs (mode.h:138) for one block, for
 *                      incremental adoption behind a GpuMode.
 */
#ifndef GXCORR_H
#define GXCORR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GX_VERSION_MAJOR 0
#define GX_VERSION_MINOR 1

#define GX_MAX_LOCAL_FREQS 64
#define GX_MAX_BANDS 128
#define GX_MAX_POLPRODUCTS 4
#define GX_MAX_MUX_THREADS 64

typedef enum gx_status {
  GX_OK = 0,
  GX_ERR_ARG = 1,          /* invalid argument or descriptor */
  GX_ERR_UNSUPPORTED = 2,  /* a configuration feature this build does not implement */
  GX_ERR_CUDA = 3,         /* CUDA runtime failure (message has the CUDA error string) */
  GX_ERR_NOMEM = 4,        /* device or host allocation failed */
  GX_ERR_IO = 5,           /* could not read or parse a setup file */
  GX_ERR_MODEL = 6,        /* no delay model for the requested time (Mode torches the subint) */
  GX_ERR_TIMEOUT = 7,      /* a bounded device wait gave up */
  GX_ERR_STATE = 8         /* call out of order */
} gx_status;

/* X-step forms */
typedef enum gx_xstep {
  GX_XSTEP_FP32 = 0,       /* plain FP32 Hermitian cross-multiply-accumulate */
  GX_XSTEP_TC_FP16 = 1,    /* tcgen05 tensor cores, FP16 spectra, FP32 accumulation */
  GX_XSTEP_TC_FP16_HILO = 2, /* as above with a split hi+lo FP16 product (3 MMAs) */
  GX_XSTEP_AUTO = 3          /* TC_FP16_HILO when a freq has at least 48 inputs (station
                                bands; env GX_XSTEP_AUTO_MIN_INPUTS) and at most 128, else FP32:
                                the tensor-core tile costs the same for any input count up to
                                128, the FP32 X-step grows with its square */
} gx_xstep;

/* One frequency-table entry (FREQ TABLE, configuration.cpp:1970-2022). */
typedef struct gx_freq_desc {
  double freq_mhz;         /* FREQ (MHZ): band edge / LO frequency */
  double bw_mhz;           /* BW (MHZ) */
  int lower_sideband;      /* SIDEBAND L */
  int nchan;               /* NUM CHANNELS */
  int chans_to_average;    /* CHANS TO AVG: output channels = nchan / this (0 or 1: none); the
                              same for every freq of a job, dividing nchan */
} gx_freq_desc;

/* One datastream (DATASTREAM TABLE, configuration.cpp:1397-1850).  Only
 * single-thread VDIF is decoded on the device. */
typedef struct gx_station_desc {
  int nbits;               /* QUANTISATION BITS: 1, 2, 4 or 8 */
  int is_complex;          /* DATA SAMPLING: 0 REAL, 1 COMPLEX (single sideband) */
  int framebytes;          /* DATA FRAME SIZE including the 32-byte VDIF header */
  int nrecfreqs;           /* NUM RECORDED FREQS */
  int recfreq[GX_MAX_LOCAL_FREQS];                 /* REC FREQ INDEX -> freq table */
  double clock_offset_us[GX_MAX_LOCAL_FREQS];      /* CLK OFFSET (us) */
  double clock_offset_delta_us[GX_MAX_LOCAL_FREQS];/* second field of CLK OFFSET a:b */
  double lo_offset_hz[GX_MAX_LOCAL_FREQS];         /* FREQ OFFSET (Hz) */
  int nbands;              /* recorded bands = sum of NUM REC POLS */
  int band_localfreq[GX_MAX_BANDS];                /* REC BAND i INDEX */
  char band_pol[GX_MAX_BANDS];                     /* REC BAND i POL */
  int clock_int_seconds;   /* floor(CLOCK COEFF 0 / 1e6 + 0.5), subtracted from the delay (mode.cpp:68,1526) */
  long long phase_cal_interval_hz; /* long(1e6 x PHASE CAL INT (MHZ)); 0: no phase-cal extraction */
  long long phase_cal_base_hz;     /* long(1e6 x PHASE CAL BASE(MHZ)); PHASE CAL DIVISOR must be 1 */
  int interlaced;          /* DATA FORMAT INTERLACEDVDIF: framebytes is the multiplexed frame size and
                              EDV4 validity masks blank absent threads per band (mk5mode.cpp:142-163) */
  /* Zoom bands (configuration.cpp:1701-1753; Mode, mode.cpp:184-196): a zoom
     freq is a channel range of the recorded freq that contains it, found and
     offset as Configuration does.  Baseline band indices nbands + i name zoom
     band i, as in the reference's total band numbering. */
  int nzoomfreqs;          /* NUM ZOOM FREQS */
  int zoomfreq[GX_MAX_LOCAL_FREQS];                /* ZOOM FREQ INDEX -> freq table (after the recorded freqs) */
  int nzoombands;          /* sum of NUM ZOOM POLS */
  int zoomband_localfreq[GX_MAX_BANDS];            /* ZOOM BAND i INDEX */
  char zoomband_pol[GX_MAX_BANDS];                 /* ZOOM BAND i POL */
  /* VDIF threads the station's frames arrive on (DATA FORMAT
     INTERLACEDVDIF/<id>:<id>:..., configuration.cpp:2632-2651); 0: plain
     VDIF, one thread of id 0.  Only gx_ring reads them (its multiplexer). */
  int nmuxthreads;
  int muxthread[GX_MAX_MUX_THREADS];
} gx_station_desc;

/* One baseline (BASELINE TABLE, configuration.cpp:1033-1180). */
typedef struct gx_baseline_desc {
  int ds1, ds2;            /* datastream indices (ds1 is the unconjugated one) */
  int nfreqs;              /* NUM FREQS */
  int freq[GX_MAX_LOCAL_FREQS];                            /* freq-table index of each */
  int npolprod[GX_MAX_LOCAL_FREQS];                        /* POL PRODUCTS */
  int band1[GX_MAX_LOCAL_FREQS][GX_MAX_POLPRODUCTS];       /* D/STREAM A BAND */
  int band2[GX_MAX_LOCAL_FREQS][GX_MAX_POLPRODUCTS];       /* D/STREAM B BAND */
} gx_baseline_desc;

/* One correlation configuration (CONFIGURATIONS section, configuration.cpp:1315). */
typedef struct gx_job_desc {
  int nstations;
  const gx_station_desc *stations;
  int nfreqs;
  const gx_freq_desc *freqs;
  int nbaselines;
  const gx_baseline_desc *baselines;
  int subint_ns;           /* SUBINT NANOSECONDS */
  int guard_ns;            /* GUARD NANOSECONDS */
  int fringe_rotation_order; /* FRINGE ROTN ORDER: 1 (linear), 2 (quadratic) or 0 (post-F, real data) */
  int array_stride;        /* ARRAY STRIDE LEN, 0 = automatic */
  int xmac_stride;         /* XMAC STRIDE LEN, 0 = automatic */
  int write_autocorrs;     /* WRITE AUTOCORRS (also enables cross-pol autocorrelations) */
  int64_t max_data_bytes;  /* largest per-station data buffer one subint will pass */
  int xstep;               /* gx_xstep */
  int block_chunk;         /* FFT blocks per device pass, 0 = automatic */
  int64_t spectra_budget_bytes; /* with block_chunk 0: > 0 caps the spectra buffer and makes passes only as
                                   long as keeps accumulator traffic under a quarter of the spectra
                                   traffic (for many resident jobs); 0 = passes of up to 40 GB of
                                   spectra, at most 30% of the device memory free at open */
} gx_job_desc;

/* One subint: the contents of one Core processslot (core.h:76-98). */
typedef struct gx_subint_desc {
  int scan, sec, ns;       /* procslots[].offsets: subint start, relative to scan start */
  double scan_start_sec;   /* Model::getScanStartSec(scan, startmjd, startseconds): wall-clock base */
  const double *interp;    /* [nstations][3] delay interpolators, us, as Mode::setOffsets leaves them
                              (intclockseconds already removed); NULL: use the handle's own model */
  const uint8_t *const *data;    /* [nstations] raw buffers (whole VDIF frames) */
  const int64_t *datalen;        /* [nstations] bytes */
  const int32_t *const *control; /* [nstations] control words: [0]=scan [1]=sec [2]=ns of the
                                    first sample, [3..] valid flags, 30 per word (FLAGS_PER_INT) */
  int controllen;                /* words per control buffer */
} gx_subint_desc;

typedef struct gx_handle gx_handle;

/* Layout summary of the Core result array (configuration.cpp:2348-2630). */
typedef struct gx_layout_info {
  int64_t result_length;   /* complex floats */
  int nfreqs, nbaselines, nstations;
  int blocks_per_send;
  int xmac_stride;
  int array_stride;
  int fftchannels;
  int nchan;
  int xstep;               /* X-step form in use (GX_XSTEP_AUTO resolved) */
  int block_chunk;         /* FFT blocks per device pass in use */
  int chans_to_average;    /* output channels per record = nchan / chans_to_average */
} gx_layout_info;

/* device < 0 opens a host-only handle: layout, offsets and delay-model
   queries work, no CUDA call is made, and gx_subint* return GX_ERR_STATE. */
gx_status gx_open(const gx_job_desc *desc, int device, gx_handle **out);
gx_status gx_open_input(const char *inputfile, int device, int xstep, gx_handle **out);
gx_status gx_close(gx_handle *h);
const char *gx_last_error(const gx_handle *h);
const char *gx_status_string(gx_status s);

gx_status gx_get_layout(const gx_handle *h, gx_layout_info *info);
/* offsets in complex-float units; arrays sized [nfreqs*nbaselines] and [nstations]; -1 = absent */
gx_status gx_get_offsets(const gx_handle *h, int *baseline_offsets, int *bweight_offsets,
                         int *autocorr_offsets, int *acweight_offsets);

gx_status gx_interpolator(gx_handle *h, int station, int scan, int sec, int ns, double out[3]);
gx_status gx_scan_start_sec(gx_handle *h, int scan, double *out);

/* Host buffers in, host results out (results: result_length complex floats, overwritten). */
gx_status gx_subint(gx_handle *h, const gx_subint_desc *sub, float *results);
/* Device buffers in, device results out, on the handle's stream (or `stream` if non-NULL:
   a cudaStream_t passed as void*).  Does not synchronise. */
gx_status gx_subint_device(gx_handle *h, const gx_subint_desc *sub, float *dev_results, void *stream);
gx_status gx_synchronize(gx_handle *h);

/* Pipelined form of gx_subint (no counterpart in the reference, whose Core
   threads block on each slot): copies the station data to the device on the
   handle's copy stream, enqueues the subint's kernels behind that copy and
   the result copy into `results`, and returns.  gx_subint_wait waits for the
   oldest subint in flight and returns its status.  At most two are in flight
   (GX_ERR_STATE for a third), so one subint's upload overlaps the other's
   kernels; `sub`'s buffers and `results` must stay valid (and be pinned for
   the copies to overlap) until its wait returns.  gx_subint and
   gx_subint_device return GX_ERR_STATE while any is in flight. */
gx_status gx_subint_async(gx_handle *h, const gx_subint_desc *sub, float *results);
gx_status gx_subint_wait(gx_handle *h);

/* No counterpart in the reference.  The same subint work as gx_subint_device
   for callers that cannot allocate device memory (host frameworks that own
   all device memory and only pass buffers in; threads that must not call
   cudaMalloc/cudaFree, which can wait for every stream of the device).  No
   handle: desc is planned on every call; sub->data are device pointers,
   sub->control and sub->interp host pointers (interp is required).
   Everything besides the caller's inputs and dev_results lives in one
   library-wide scratch array of GX_NOALLOC_SCRATCH_BYTES in device global
   memory, which every GPU that loads the library holds until exit; jobs that
   do not fit return GX_ERR_UNSUPPORTED with the bytes needed in err.  The
   call allocates no device memory.  The first call on a device looks up the
   array's device address and keeps it: make that call before any stream
   capture begins, and do not reset the device while using this entry point.
   Per-call tables are copied from pageable host memory, so the call may wait
   for work already queued on `stream`.  All calls share the array: calls
   whose work overlaps on the GPU race, so order them on one stream.  Only the
   FP32 X-step form is available on this path.  err (may be NULL) receives a
   message of at most errlen bytes. */
#define GX_NOALLOC_SCRATCH_BYTES (64u << 20)
gx_status gx_subint_device_noalloc(const gx_job_desc *desc, const gx_subint_desc *sub, float *dev_results,
                                   void *stream, char *err, int errlen);

/* Spectra of one FFT block of one datastream after the last gx_subint* call
   (nbands x nchan complex floats, after fractional-sample correction), and its weight. */
gx_status gx_spectra(gx_handle *h, int station, int block, float *out, float *weight);

/* Device time of the last gx_subint* call per stage, milliseconds: [0] unpack+F, [1] X, [2] finalise. */
gx_status gx_stage_times(gx_handle *h, float ms[3]);

/* Number of kernel launches issued by the last gx_subint* call. */
gx_status gx_launch_count(const gx_handle *h, int *count);

/* ---- Visibility output (mpifxcorr/src/visibility.cpp) -------------------- */

/* An integration buffer and SWIN writer on the handle's device (Visibility,
   visibility.cpp:33-103).  Needs a handle opened with gx_open_input (job
   start, integration time, telescope indices and the .im (u, v, w) model).
   Records are appended to <outdir>/DIFX_<start mjd>_<start seconds>.s0000.b0000
   as Visibility::flushBuffersToDisk names them (visibility.cpp:1056-1091).
   GX_ERR_STATE without a .input job, GX_ERR_UNSUPPORTED for TSYS > 0. */
typedef struct gx_vis gx_vis;
gx_status gx_vis_open(gx_handle *h, const char *outdir, gx_vis **out);

/* Visibility::addData (visibility.cpp:192-205): adds one subint's Core result
   array (device memory, gx_layout_info.result_length complex floats) into the
   integration, on stream (NULL: the handle's stream). */
gx_status gx_vis_add(gx_vis *v, const float *dev_results, void *stream);

/* Visibility::writedata and writeSWIN (visibility.cpp:353-690, 781-960) for
   the integration that started at scan, sec (seconds after the scan start),
   ns: normalises every record by 1 / (weight x subints per integration x
   blocks per send x 2 x nchan), writes the records with positive weight
   (74-byte header + nchan complex floats; cross-correlations, then
   autocorrelations) and clears the buffer.  *nrecords (may be NULL) returns
   the number of records written.  Nothing is written for an integration
   past the end of the job or with no subints added. */
gx_status gx_vis_write(gx_vis *v, int scan, int sec, int ns, int *nrecords);
gx_status gx_vis_close(gx_vis *v);
/* With phase-cal extraction, gx_vis_write also appends each datastream's
   scaled tones as one line to <outdir>/PCAL_<start mjd>_<start seconds>_<station>
   (writedata, visibility.cpp:650-675, 985-1053); gx_vis_pcal_headers writes
   the comment lines FxManager puts at the top of those files once per job
   (Visibility::initialisePcalFiles, visibility.cpp:107-138). */
gx_status gx_vis_pcal_headers(gx_vis *v);

/* Partial integrations on several GPUs (subints shared out over ranks, as the
   FxManager shares them over Cores, fxmanager.cpp:331-336): the device
   integration buffer (2 x result_length floats, on the handle's device) and
   the subints added to it, so that the partial buffers can be summed into the
   writing rank's buffer by a collective (the caller synchronises the
   handle's stream first); gx_vis_set_subints then records how many subints
   the sum holds, and gx_vis_clear empties a buffer without writing it. */
gx_status gx_vis_buffer(gx_vis *v, float **dev, long long *nfloats, int *nsub);
gx_status gx_vis_set_subints(gx_vis *v, int nsub);
gx_status gx_vis_clear(gx_vis *v);

/* Model::interpolateUVW (model.cpp:177-217): (u, v, w) in metres of the
   baseline datastream ds1 - datastream ds2, offset seconds after the start
   of scan, first phase centre. */
gx_status gx_uvw(gx_handle *h, int scan, double offset, int ds1, int ds2, double out[3]);

/* ---- Request loop (continuous batching of subints of resident jobs) ------ */

/* Opened handles are attached as jobs; their device memory (delay model,
   twiddles, tables, accumulators, input buffers) stays resident and counts
   against the server's HBM budget.  Submitted requests -- one subint of one
   job -- are admitted earliest deadline first (submission time plus the job's
   deadline, by default the job's subint duration; requests without a deadline
   in arrival order) by `slots` worker threads as soon as a
   slot is free, no other request of the same job is on the GPU, and the
   memory the request adds keeps the total within the budget (a request is
   always admitted when nothing else is in flight).  Requests of different jobs
   run concurrently, each on its job's stream.  Latency runs from submission to
   results in the caller's buffer.  The buffers a submission points to must
   stay valid until gx_server_wait returns for it.  No counterpart in the
   reference, whose FxManager (fxmanager.cpp:301-529) hands subints to Core
   processes over MPI. */
typedef struct gx_server gx_server;

/* Runs one request; the default is gx_subint (host buffers) or, with
   device_inputs, gx_subint_device followed by a copy of the result array to
   `results`.  h is the attached handle (may be NULL for a custom executor). */
typedef gx_status (*gx_server_executor)(void *ctx, gx_handle *h, int job, const gx_subint_desc *sub,
                                        float *results);

typedef struct gx_latency_stats {
  long long completed, failed;
  double p50_ms, p95_ms, p99_ms, mean_ms, max_ms;   /* latency of completed requests */
} gx_latency_stats;

gx_status gx_server_open(int slots, long long hbm_budget_bytes, int device_inputs, gx_server **out);
/* Replaces the executor (before the first submission). */
gx_status gx_server_set_executor(gx_server *s, gx_server_executor fn, void *ctx);
/* resident_bytes < 0: the handle's own device memory (gx_device_bytes).
   GX_ERR_NOMEM when the resident total would exceed the budget. */
gx_status gx_server_attach(gx_server *s, gx_handle *h, long long resident_bytes, int *job);
/* Relative deadline of the job's requests in ms (default: the subint duration
   of the attached handle; <= 0: none, arrival order). */
gx_status gx_server_set_deadline(gx_server *s, int job, double deadline_ms);
/* request_bytes < 0: the growth of the job's input buffers a host-buffer
   request needs (0 with device inputs).  GX_ERR_NOMEM if it can never fit. */
gx_status gx_server_submit(gx_server *s, int job, const gx_subint_desc *sub, float *results, long long request_bytes,
                           long long *ticket);
/* Blocks until the request has completed; returns its status and latency. */
gx_status gx_server_wait(gx_server *s, long long ticket, double *latency_ms);
/* Latency percentiles of the requests completed so far (reset: start over). */
gx_status gx_server_stats(gx_server *s, int reset, gx_latency_stats *out);
/* Finishes every queued request, then stops the workers. */
gx_status gx_server_close(gx_server *s);
/* Message of the last request that failed (its job and the handle's error). */
const char *gx_server_last_error(gx_server *s);

/* ---- Batches of uneven jobs (one subint of every job per step) ---------- */

/* A batch is a fixed set of opened handles on one device, each with a device
   result array.  Every gx_batch_run correlates one subint of each job, with
   device-resident inputs (sub->data are device pointers, as for
   gx_subint_device), and returns without waiting; gx_batch_synchronize waits.
   Each job's results are bit-identical to what gx_subint_device gives it
   alone.  Modes:
     GX_BATCH_SERIAL   one job after another on one stream (per-job launches)
     GX_BATCH_STREAMS  jobs spread over branch streams, longest first onto the
                       least-loaded branch
     GX_BATCH_GRAPH    that schedule captured once into one CUDA graph and
                       replayed each step (one host launch per step)
   nstreams 0 (STREAMS, GRAPH): the branch count is tuned on the first steps
   (1, 2, 4, 8, 16 branches, two steps each; every step still delivers its
   results).  A handle may be in one batch at a time and must not be used
   elsewhere while a step is in flight.  No counterpart in the reference,
   which runs one job per correlator process. */
typedef struct gx_batch gx_batch;
#define GX_BATCH_SERIAL 0
#define GX_BATCH_STREAMS 1
#define GX_BATCH_GRAPH 2

gx_status gx_batch_open(gx_handle *const *jobs, float *const *dev_results, int njobs, int mode, int nstreams,
                        gx_batch **out);
/* subs[j]: the subint of job j (all njobs entries). */
gx_status gx_batch_run(gx_batch *b, const gx_subint_desc *const *subs);
/* Waits for the step in flight; device_ms (may be NULL) = its device time. */
gx_status gx_batch_synchronize(gx_batch *b, float *device_ms);
/* Branch count in use (0 while tuning), whether tuning is still on, and the
   kernel launches of the last step. */
gx_status gx_batch_info(const gx_batch *b, int *nstreams, int *tuning, int *launches);
/* Tunes the launch shapes (gx_set_tiles) of a batch's jobs per shape class:
   the class's costliest job runs its subint of `subs` under every candidate,
   `reps` times each, timed alone on the device, and the fastest goes to every
   job of the class.  Graphs captured before are dropped (the next graph step
   captures the tuned shapes).  *nclasses: the classes found. */
gx_status gx_batch_tune_tiles(gx_batch *b, const gx_subint_desc *const *subs, int reps, int *nclasses);
const char *gx_batch_last_error(const gx_batch *b);
gx_status gx_batch_close(gx_batch *b);

/* ---- Multi-thread VDIF multiplexing on the device ------------------------ */

/* The reference's vdifmux (vdifio/src/vdifmux.c:496-1033), as the VDIF
   DataStream uses it (vdiffile.cpp:495-565, 700-760): single-thread VDIF
   frames of several threads, in one device buffer, become multi-channel
   frames of one thread, sorted in time, in another device buffer.  Frame
   classification and the corner turn run on the GPU; the sequential
   decisions (duplicates, the out-of-order window nsort, the gap limit ngap,
   the end-of-buffer back-off) run on the host over 16 bytes per frame.  The
   input must be frame-aligned (frame k at byte k x input_frame_bytes): a
   frame that starts but does not end with the fill pattern, or whose header
   has another size, channel count or bit depth, is skipped whole (the
   reference rescans it byte by byte).  Output headers, payloads of the frames
   the reference corner-turns, the statistics and the returned byte count
   then equal the reference's; the payload of a filler frame (invalid bit
   set) is left as the destination held it.  Output slots past nthreads
   (rounded up to a power of two) hold zeros.  One channel per input thread
   (channels_per_thread must be 1: GX_ERR_UNSUPPORTED otherwise); fan-out
   (several threads per channel) and legacy headers are not implemented. */
typedef struct gx_vdifmux gx_vdifmux;
#define GX_VDIFMUX_GOTOEND 0x01             /* VDIF_MUX_FLAG_GOTOEND */
#define GX_VDIFMUX_RESPECTGRANULARITY 0x02  /* VDIF_MUX_FLAG_RESPECTGRANULARITY */
#define GX_VDIFMUX_ENABLEVALIDITY 0x04      /* VDIF_MUX_FLAG_ENABLEVALIDITY */
#define GX_VDIFMUX_COMPLEX 0x20             /* VDIF_MUX_FLAG_COMPLEX */
#define GX_VDIFMUX_PROPAGATEVALIDITY 0x40   /* VDIF_MUX_FLAG_PROPAGATEVALIDITY (EDV4 output) */

/* struct vdif_mux_statistics (vdifio.h:404-432): the first eleven
   accumulate over calls (gx_vdifmux_reset_stats clears them), the rest
   describe the last call; returned_bytes is vdifmux's return value. */
typedef struct gx_vdifmux_stats {
  long long valid_frames, invalid_frames, discarded_frames, wrong_thread_frames, skipped_bytes, fill_bytes,
      duplicate_frames, bytes_processed, good_output_frames, partial_output_frames, filler_output_frames;
  long long calls;
  long long src_bytes, src_used, dest_bytes, dest_used, output_frames, start_frame, returned_bytes;
  int epoch;
} gx_vdifmux_stats;

/* configurevdifmux + setvdifmuxinputchannels (vdifmux.c:107-242).  device < 0:
   host-only (gx_vdifmux_info works, gx_vdifmux_run returns GX_ERR_STATE). */
gx_status gx_vdifmux_open(int input_frame_bytes, int frames_per_second, int bits_per_sample, int nthreads,
                          const int *thread_ids, int channels_per_thread, int nsort, int ngap, int flags, int device,
                          gx_vdifmux **out);
gx_status gx_vdifmux_info(const gx_vdifmux *m, int *output_frame_bytes, int *output_channels, int *frame_granularity);
/* vdifmux(): src and dest are device buffers (4-byte aligned); start_frame < 0
   starts at the lowest frame number among the first nsort usable frames.
   Synchronises `stream` before returning. */
gx_status gx_vdifmux_run(gx_vdifmux *m, const uint8_t *src, long long src_bytes, uint8_t *dest, long long dest_bytes,
                         long long start_frame, gx_vdifmux_stats *stats, void *stream);
gx_status gx_vdifmux_reset_stats(gx_vdifmux *m);
const char *gx_vdifmux_last_error(const gx_vdifmux *m);
gx_status gx_vdifmux_close(gx_vdifmux *m);

/* ---- Station data ring and control words computed on the device ---------- */

/* The DataStream's segmented data buffer (DataStream::initialise and
   updateConfig, datastream.cpp:116-230, 733-763, in the VDIF form of
   vdiffile.cpp:475-493) held in device memory, one per station: DATA BUFFER
   FACTOR x the largest data bytes of a subint, cut into NUM DATA SEGMENTS
   segments, then the overflow region a send runs into when it wraps.
   Segments are filled from raw single-thread VDIF frames by the device
   multiplexer (gx_ring_read, as VDIFDataStream::dataRead, vdiffile.cpp:668-
   860) or described by the caller (gx_ring_set_segment).  gx_ring_subint_device
   then correlates one subint straight out of the rings: one kernel finds each
   station's segment and send start from the device-resident segment table
   and writes the subint's control words (first-sample time and the per-block
   valid flags, DataStream::calculateControlParams, datastream.cpp:368-627,
   aligned to whole multiplexed frames as VDIFDataStream::calculateControlParams
   does, vdiffile.cpp:348-470) and data pointers into the device tables the
   F-step reads; a second copies the wrapped part of a send into the overflow
   region (DataStream::execute, datastream.cpp:296-305).  No host round trip
   sits between the segment table and the F-step.  The only host inputs per
   subint are the geometric delays at the two ends of the data span
   (Model::calculateDelayInterpolator of order 0), from the handle's model.
   A ring belongs to one handle and is used on one stream at a time; a
   segment must not be refilled while a subint that reads it is in flight
   (the reference's segment locks). */
typedef struct gx_ring gx_ring;

/* One segment (readinfo, datastream.h): the time of its first multiplexed
   frame relative to the start of its scan, and how many bytes it holds. */
typedef struct gx_ring_segment {
  int scan, scanseconds, scanns;
  int validbytes;
  int readto;          /* nonzero once filled */
  int configindex;     /* 0; < 0: a segment without configuration (the frame
                          alignment then looks at the next segments) */
} gx_ring_segment;

/* Per-station quantities the DataStream derives from the configuration. */
typedef struct gx_ring_geometry {
  int bufferbytes, readbytes, numsegments, overflowbytes;
  int sendbytes, blockspersend, controllength, blockbytes;
  int bytespersamplenum, bytespersampledenom, bytesbetweenintegerns, nsinc;
  int framebytes;        /* multiplexed frame */
  int payloadbytes;      /* multiplexed frame payload */
  int framespersecond;   /* multiplexed frames per second */
  int framegranularity;  /* frames per integer nanosecond (vdifmux) */
  int intclockseconds;
  double sampletimens;
  long long dataspanns;
} gx_ring_geometry;

/* Rings for every station of a handle opened with a delay model
   (gx_open_input); buffers are zeroed as the reference's are. */
gx_status gx_ring_open(gx_handle *h, int databufferfactor, int numdatasegments, gx_ring **out);
gx_status gx_ring_geometry_get(const gx_ring *r, int station, gx_ring_geometry *g);
/* Device address of a station's buffer (segment k at k x readbytes). */
gx_status gx_ring_buffer(const gx_ring *r, int station, uint8_t **dev_buffer);
/* VDIFDataStream::dataRead for one segment: multiplex raw single-thread
   frames (device memory, frame-aligned) of `scan` into the segment, continuing
   the frame numbering of the station's previous read, and set the segment's
   time and valid bytes from the first output frame.  *consumed: raw bytes
   used (the next read starts there).  Synchronises `stream`. */
gx_status gx_ring_read(gx_ring *r, int station, int segment, int scan, const uint8_t *dev_raw, long long raw_bytes,
                       long long *consumed, void *stream);
gx_status gx_ring_set_segment(gx_ring *r, int station, int segment, const gx_ring_segment *seg);
gx_status gx_ring_get_segment(const gx_ring *r, int station, int segment, gx_ring_segment *seg);
/* The control words and send start of one station for a subint, computed on
   the host from the host copy of the segment table with the host's own
   segment position (the CPU form of the device kernel's bookkeeping).
   control: geometry.controllength words. */
gx_status gx_ring_control_host(gx_ring *r, int station, int scan, int sec, int ns, int32_t *control, int *startpos);
/* One subint of the handle from the rings, results into dev_results as
   gx_subint_device writes them; the segment positions advance on the device. */
gx_status gx_ring_subint_device(gx_handle *h, gx_ring *r, int scan, int sec, int ns, double scan_start_sec,
                                float *dev_results, void *stream);
/* The control words [nstations][controllength] and send starts the last
   gx_ring_subint_device computed (synchronises its stream).  GX_ERR_STATE if
   a station's subint lay past every filled segment. */
gx_status gx_ring_last_control(gx_ring *r, int32_t *control, int *startpos);
/* Both segment positions (host and device) back to segment 0. */
gx_status gx_ring_reset(gx_ring *r);
const char *gx_ring_last_error(const gx_ring *r);
gx_status gx_ring_close(gx_ring *r);

/* ---- Monitoring spectra: spectral kurtosis and STA dumps -------------------- */

/* The reference's Core sends two monitoring products on its message bus when
   an operator asks for them: the spectral kurtosis of every recorded band
   (Mode accumulates |X|^2 and |X|^4 of each channel over its FFT blocks,
   mode.cpp:1237-1254, and turns them into n s2 / s1^2 - 1, debiased and
   averaged to the dump channel count, mode.cpp:1403-1454;
   Core::averageAndSendKurtosis, core.cpp:1378-1430), and the STA dump, each
   band's autocorrelation normalised to power spectral density and averaged
   to the dump channels (Core::averageAndSendAutocorrs, core.cpp:1180-1255).
   Both are given here for one subint (the reference's records of a Core with
   one process thread); sending them is the caller's. */

/* Kurtosis accumulation on (dump_channels > 0, the STA DUMP CHANNELS value)
   or off (0) for the following subints.  The sums read the spectra in
   device memory after each pass of the F-step. */
gx_status gx_set_kurtosis(gx_handle *h, int dump_channels);
/* The kurtosis of the last subint: sk[(station * GX_MAX_BANDS + band) *
   dump_channels + j] for recorded bands, nchan[station * GX_MAX_BANDS + band]
   the channels each holds, valid[station] whether the reference would send
   that station's records (its last band had data; a band without data keeps
   its previous values, as the reference's arrays do).  nchan, valid may be
   NULL.  Synchronises the subint's stream. */
gx_status gx_kurtosis(gx_handle *h, float *sk, int *nchan, int *valid);
/* The STA dump of a subint from its Core result array (host memory, complex
   interleaved): sta[(station * GX_MAX_BANDS + band) * dump_channels + j],
   nchan[...] the channels of each record, sent[...] whether the reference
   sends it (the band's weight reaches a third of a full subint's,
   Core::MINIMUM_FILTERBANK_WEIGHT).  GX_ERR_UNSUPPORTED when the dump needs
   more channels than the averaged records keep. */
gx_status gx_sta(const gx_handle *h, const float *results, int dump_channels, float *sta, int *nchan, int *sent);

/* Launch shapes a tuner may choose per job; results do not depend on them.
   xmac_variant: the FP32 X-step's channel tile and stage depth (0 or 1);
   fstep_items: FFT blocks a station-block F-step group takes per CTA (0: 4). */
gx_status gx_set_tiles(gx_handle *h, int xmac_variant, int fstep_items);
gx_status gx_get_tiles(const gx_handle *h, int *xmac_variant, int *fstep_items);

/* Phase-cal section of the Core result array (configuration.cpp:2612-2620,
   core.cpp:1131-1164): offsets[s * GX_MAX_BANDS + b] is the result index of
   the first tone of recorded band b of datastream s (-1 without phase-cal),
   ntones[...] its number of tones (complex values).  Either may be NULL. */
gx_status gx_get_pcal_layout(const gx_handle *h, int *offsets, int *ntones);

/* Device memory a handle holds, bytes. */
gx_status gx_device_bytes(const gx_handle *h, long long *bytes);

/* Operand scales of the tensor-core X-step for one band of one datastream:
   scales[c] multiplies channel c of that band's spectra before they are
   rounded to FP16 and is divided out of every visibility.  Each value is
   rounded to the nearest power of two, so scaling and unscaling are exact.
   The defaults bring noise spectra to an r.m.s. near 8.  Returns GX_ERR_STATE
   for a handle without the tensor-core X-step, GX_ERR_ARG for a value that is
   not finite and positive.  No counterpart in the reference (its X-step is
   FP32 throughout). */
gx_status gx_set_tc_scales(gx_handle *h, int station, int band, const float *scales);

#ifdef __cplusplus
}
#endif
#endif /* GXCORR_H */
