// Host-side plan of one job: every table gx_open computes, without touching
// the device.  Used by entry points that bring their own device memory.
#pragma once
#include <string>
#include <vector>
#include "gx_dev.h"
#include "gx_xstep.h"

namespace gx {

struct JobPlan {
  DevJob J{};                       // J.twiddle is left null: the caller places the table
  int maxnrf = 1, nslots = 1, ks = 1;
  XmacShape xs{};
  long long result_length = 0;
  int ctrlstride = 0;
  std::vector<DevStation> stations;
  std::vector<float2> twiddle;      // twiddle_table(F)
  std::vector<ProdEntry> prods;
  std::vector<WeightEntry> wents;
  std::vector<int2> pairs;
};

gx_status plan_job(const gx_job_desc *desc, JobPlan *plan, std::string &err);

// The device twiddle table of an F-point transform (layout of r16::tw_pass_offset).
std::vector<float2> twiddle_table(int F);

}  // namespace gx
