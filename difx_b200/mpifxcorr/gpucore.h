// GpuCore: the Core of mpifxcorr with each slot correlated by gxcorr on a GPU.
//
// This file and gpucore.cpp are what a DiFX maintainer adds to mpifxcorr/src.
// Core keeps its MPI receive loop, ring of slots and process threads
// (core.cpp:189-470); only the per-thread work of a slot, Core::processdata
// (core.cpp:657-1129: every Mode::process call, the XMAC loop, the weights
// and the copies into procslots[index].results), is replaced: thread 0 hands
// the whole slot to gx_subint, which writes procslots[index].results in the
// Core result layout (configuration.cpp:2348-2630); the other threads return.
//
// Edits this needs in the reference headers (core.cpp and the rest of
// mpifxcorr stay unchanged):
//   core.h           `friend class GpuCore;` inside class Core, and
//                    `virtual` before `void processdata(...)` (core.h:169)
//   configuration.h  `friend class GpuCore; friend class GpuMode;` inside
//                    class Configuration (the datastream table's clock and LO
//                    offsets and the fringe-rotation order have no getters)
// and in mpifxcorr.cpp `new GpuCore(...)` in place of `new Core(...)`.
#pragma once
#include <string>
#include <vector>
#include "configuration.h"
#include "core.h"
#include "gxcorr.h"

class GpuCore : public Core {
 public:
  // device: CUDA device of the handles; xstep: gx_xstep (GX_XSTEP_FP32 is
  // within 1e-5 of Core::processdata, the tensor-core forms within 1e-3).
  GpuCore(int id, Configuration *conf, int *dids, MPI_Comm rcomm, int device = 0, int xstep = GX_XSTEP_FP32);
  ~GpuCore();

  // Core::processdata's replacement: thread 0 correlates the whole slot.
  void processdata(int index, int threadid, int startblock, int numblocks, Mode **modes, Polyco *currentpolyco,
                   threadscratchspace *scratchspace);

  // The whole slot `index` on the GPU into procslots[index].results; 0 on
  // success, else a gx_status (the reason in lasterror()).
  int correlateslot(int index);

  // The gxcorr job of configuration `configindex` (the CONFIGURATIONS and
  // DATASTREAM tables as gx_job_desc; the arrays it points to live in *this).
  gx_handle *handle(int configindex);
  const std::string &lasterror() const { return err; }

  // Delay interpolators of datastream ds for the slot starting at (scan, sec,
  // ns), as Mode::setOffsets computes them (mode.cpp:1502-1532); false when
  // the model has no interpolator there (the slot is then zeroed).
  bool interpolator(int configindex, int ds, int scan, int sec, int ns, double out[3]);

 private:
  struct Job {
    gx_handle *h = nullptr;
    std::vector<gx_station_desc> st;
    std::vector<gx_freq_desc> fr;
    std::vector<gx_baseline_desc> bl;
  };
  int build(int configindex, Job &job);
  std::vector<Job> jobs;   // per configuration index, opened on first use
  int device, xstep;
  std::string err;
};
