/* Test infrastructure only: drives the reference's vdifmux (vdifio/src/vdifmux.c,
 * compiled unmodified by `make -C oracle vmux`) through a flat C interface for
 * ctypes, so that the tests can compare the device multiplexer against it. */
#include <stdint.h>
#include <string.h>
#include <time.h>
#include "vdifio.h"

/* out[0..19]: the statistics in the order of gx_vdifmux_stats (accumulated
 * over this one call), out[20]: vdifmux's return value, out[21]: output frame
 * bytes, out[22]: nanoseconds the vdifmux call took. */
int ref_vdifmux_channels(unsigned char *dest, int dest_bytes, const unsigned char *src, int src_bytes,
                         int frame_bytes, int frames_per_second, int bits, int nthreads, const int *thread_ids,
                         int nsort, int ngap, int flags, long long start_frame, int channels_per_thread,
                         long long *out)
{
  struct vdif_mux vm;
  struct vdif_mux_statistics st;
  int rv = configurevdifmux(&vm, frame_bytes, frames_per_second, bits, nthreads, thread_ids, nsort, ngap, flags);
  if (rv < 0) return rv;
  /* several recorded bands per thread, as VDIFDataStream::initialiseFile sets them (vdiffile.cpp:533-546) */
  if (channels_per_thread > 1 && (rv = setvdifmuxinputchannels(&vm, channels_per_thread)) < 0) return rv;
  resetvdifmuxstatistics(&st);
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  rv = vdifmux(dest, dest_bytes, src, src_bytes, &vm, start_frame, &st);
  clock_gettime(CLOCK_MONOTONIC, &t1);
  out[22] = (long long)(t1.tv_sec - t0.tv_sec) * 1000000000LL + (t1.tv_nsec - t0.tv_nsec);
  out[0] = st.nValidFrame;
  out[1] = st.nInvalidFrame;
  out[2] = st.nDiscardedFrame;
  out[3] = st.nWrongThread;
  out[4] = st.nSkippedByte;
  out[5] = st.nFillByte;
  out[6] = st.nDuplicateFrame;
  out[7] = st.bytesProcessed;
  out[8] = st.nGoodFrame;
  out[9] = st.nPartialFrame;
  out[10] = st.nFillerFrame;
  out[11] = st.nCall;
  out[12] = st.srcSize;
  out[13] = st.srcUsed;
  out[14] = st.destSize;
  out[15] = st.destUsed;
  out[16] = st.nOutputFrame;
  out[17] = st.startFrameNumber;
  out[18] = rv;
  out[19] = st.epoch;
  out[20] = rv;
  out[21] = vm.outputFrameSize;
  return rv < 0 ? rv : 0;
}

int ref_vdifmux(unsigned char *dest, int dest_bytes, const unsigned char *src, int src_bytes, int frame_bytes,
                int frames_per_second, int bits, int nthreads, const int *thread_ids, int nsort, int ngap,
                int flags, long long start_frame, long long *out)
{
  return ref_vdifmux_channels(dest, dest_bytes, src, src_bytes, frame_bytes, frames_per_second, bits, nthreads,
                              thread_ids, nsort, ngap, flags, start_frame, 1, out);
}
