// Batches of uneven jobs on one GPU: one subint of every job per step.
//
// A step stages each job's per-subint tables on the host (a few KB per job),
// then enqueues the jobs' device work in one of three ways:
//   serial   one job after another on one stream -- the per-job launch
//            sequence a caller looping over gx_subint_device gets;
//   streams  the jobs split over k branch streams forked from and joined
//            back to the batch stream, so that small jobs fill the SMs that
//            large ones leave idle and the HBM-bound F-step of one job runs
//            beside the compute-bound X-step of another;
//   graph    the streams schedule captured once into one CUDA graph and
//            replayed every step: one launch per step from the host instead
//            of several per job (the graph's table copies read the pinned
//            blocks the host rewrote for this step).
// Jobs go to branches longest first onto the least-loaded branch (LPT), by
// an estimate of each job's device time.  With k = 0 the branch count is
// tuned online: the first steps try 1, 2, 4, 8 and 16 branches (twice each,
// every step still producing its results) and the fastest is kept.
#include <algorithm>
#include <cmath>
#include <map>
#include <numeric>
#include <tuple>
#include <string>
#include <vector>
#include "gx_handle.h"
#include "gx_xstep.h"

namespace {

constexpr int kMaxBranches = 16;
const int kCandidates[] = {1, 2, 4, 8, 16};
constexpr int kTuneRepeats = 2;

// Relative device time of one subint of a job: F-step bytes at HBM speed plus
// X-step work at the rate of its form (only the ratios between jobs matter).
double job_cost(const gx_handle *h)
{
  const gx::DevJob &J = h->J;
  const double blocks = (double)J.blocks_per_send;
  const double fbytes = blocks * J.nstations * (J.nbands * (double)J.fftlen * (J.cplx ? 2 : 1) * J.nbits / 8.0 +
                                                J.nbands * (double)J.nchan * 8.0);
  const double ni = (double)J.ninputs;
  const double xflops = blocks * h->jd.nfreqs * 8.0 * ni * (ni + 1) / 2 * J.nchan;
  const double xrate = h->tc ? (h->hilo ? 0.35e15 : 1.0e15) : 0.05e15;
  return fbytes / 6.0e12 + xflops / xrate + 20e-6;
}

}  // namespace

struct gx_batch {
  int mode = GX_BATCH_SERIAL;
  int device = 0;
  std::vector<gx_handle *> jobs;
  std::vector<float2 *> results;
  std::vector<double> cost;
  std::string err;

  cudaStream_t origin = nullptr;
  cudaStream_t branch[kMaxBranches] = {};
  cudaEvent_t fork = nullptr, join[kMaxBranches] = {}, ev0 = nullptr, ev1 = nullptr;

  int nbranch = 1;            // branch count in use
  bool tuning = false;
  int tune_step = 0;          // tuning runs done
  double tune_ms[5] = {1e30, 1e30, 1e30, 1e30, 1e30};
  int run_branches = 1;       // branch count of the run in flight

  cudaGraphExec_t graph[kMaxBranches + 1] = {};   // per branch count
  int graph_launches[kMaxBranches + 1] = {};       // kernel launches inside each graph
  bool pending = false;
  float last_ms = 0.0f;
  int launches = 0;

  gx_status fail(gx_status s, const std::string &m)
  {
    err = m;
    return s;
  }
  gx_status cuda(cudaError_t e, const char *what)
  {
    if (e == cudaSuccess) return GX_OK;
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return GX_ERR_CUDA;
  }

  static int cand_index(int k)
  {
    for (int i = 0; i < 5; i++)
      if (kCandidates[i] == k) return i;
    return -1;
  }

  // LPT: jobs longest first, each onto the branch with the least work so far
  std::vector<std::vector<int>> schedule(int k) const
  {
    std::vector<int> order(jobs.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<std::vector<int>> br(k);
    std::vector<double> load(k, 0.0);
    for (int j : order) {
      const int b = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      br[b].push_back(j);
      load[b] += cost[j];
    }
    return br;
  }

  gx_status enqueue_job(int j, cudaStream_t st)
  {
    gx_handle *h = jobs[j];
    h->untimed = true;
    gx_status r = gx_enqueue_subint(h, results[j], st);
    h->untimed = false;
    if (r != GX_OK) return fail(r, "job " + std::to_string(j) + ": " + h->err);
    launches += h->launches;
    return GX_OK;
  }

  // fork from origin, the jobs of each branch on its stream, join back
  gx_status enqueue_branches(int k)
  {
    const auto br = schedule(k);
    gx_status r;
    if ((r = cuda(cudaEventRecord(fork, origin), "cudaEventRecord")) != GX_OK) return r;
    for (int b = 0; b < k; b++) {
      if ((r = cuda(cudaStreamWaitEvent(branch[b], fork, 0), "cudaStreamWaitEvent")) != GX_OK) return r;
      for (int j : br[b])
        if ((r = enqueue_job(j, branch[b])) != GX_OK) return r;
      if ((r = cuda(cudaEventRecord(join[b], branch[b]), "cudaEventRecord")) != GX_OK) return r;
      if ((r = cuda(cudaStreamWaitEvent(origin, join[b], 0), "cudaStreamWaitEvent")) != GX_OK) return r;
    }
    return GX_OK;
  }

  gx_status capture(int k, cudaGraphExec_t *out)
  {
    gx_status r = cuda(cudaStreamBeginCapture(origin, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture");
    if (r != GX_OK) return r;
    launches = 0;
    r = enqueue_branches(k);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(origin, &g);
    graph_launches[k] = launches;
    if (r != GX_OK) {
      if (g) cudaGraphDestroy(g);
      return r;
    }
    if ((r = cuda(e, "cudaStreamEndCapture")) != GX_OK) return r;
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    return cuda(e, "cudaGraphInstantiate");
  }

  // Waits for the run in flight; books its time for the tuner.
  gx_status finish()
  {
    if (!pending) return GX_OK;
    gx_status r = cuda(cudaEventSynchronize(ev1), "cudaEventSynchronize");
    pending = false;
    if (r != GX_OK) return r;
    if ((r = cuda(cudaEventElapsedTime(&last_ms, ev0, ev1), "cudaEventElapsedTime")) != GX_OK) return r;
    for (size_t j = 0; j < jobs.size(); j++)
      if (jobs[j]->h_err && jobs[j]->h_err[0] != 0)
        return fail(GX_ERR_TIMEOUT, "job " + std::to_string(j) + ": a tensor-core X-step wait expired");
    if (tuning) {
      const int ci = cand_index(run_branches);
      if (ci >= 0) tune_ms[ci] = std::min(tune_ms[ci], (double)last_ms);
      tune_step++;
      if (tune_step >= ncand() * kTuneRepeats) {
        int best = 0;
        for (int i = 1; i < ncand(); i++)
          if (tune_ms[i] < tune_ms[best]) best = i;
        nbranch = kCandidates[best];
        tuning = false;
        for (int i = 0; i <= kMaxBranches; i++)   // keep only the chosen graph
          if (i != nbranch && graph[i]) {
            cudaGraphExecDestroy(graph[i]);
            graph[i] = nullptr;
          }
      }
    }
    return GX_OK;
  }

  int ncand() const
  {
    int n = 0;
    for (int k : kCandidates)
      if (k <= std::max<int>(1, (int)jobs.size())) n++;
    return n;
  }

  gx_status run(const gx_subint_desc *const *subs)
  {
    gx_status r;
    if ((r = cuda(cudaSetDevice(device), "cudaSetDevice")) != GX_OK) return r;
    if ((r = finish()) != GX_OK) return r;
    for (size_t j = 0; j < jobs.size(); j++) {
      const gx_subint_desc *s = subs[j];
      if (!s || !s->data || !s->datalen || !s->control)
        return fail(GX_ERR_ARG, "job " + std::to_string(j) + ": incomplete subint");
      if ((r = gx_stage_subint(jobs[j], s, s->data)) != GX_OK)
        return fail(r, "job " + std::to_string(j) + ": " + jobs[j]->err);
    }
    run_branches = tuning ? kCandidates[(tune_step / kTuneRepeats) % ncand()] : nbranch;
    launches = 0;
    if ((r = cuda(cudaEventRecord(ev0, origin), "cudaEventRecord")) != GX_OK) return r;
    if (mode == GX_BATCH_SERIAL) {
      for (size_t j = 0; j < jobs.size(); j++)
        if ((r = enqueue_job((int)j, origin)) != GX_OK) return r;
    } else if (mode == GX_BATCH_STREAMS) {
      if ((r = enqueue_branches(run_branches)) != GX_OK) return r;
    } else {
      const int k = run_branches;
      if (!graph[k] && (r = capture(k, &graph[k])) != GX_OK) return r;
      launches = graph_launches[k];   // kernel launches inside one replay
      if ((r = cuda(cudaGraphLaunch(graph[k], origin), "cudaGraphLaunch")) != GX_OK) return r;
    }
    if ((r = cuda(cudaEventRecord(ev1, origin), "cudaEventRecord")) != GX_OK) return r;
    pending = true;
    return GX_OK;
  }

  void release()
  {
    if (pending) cudaEventSynchronize(ev1);
    for (auto &g : graph)
      if (g) cudaGraphExecDestroy(g);
    for (int b = 0; b < kMaxBranches; b++) {
      if (branch[b]) cudaStreamDestroy(branch[b]);
      if (join[b]) cudaEventDestroy(join[b]);
    }
    if (fork) cudaEventDestroy(fork);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (origin) cudaStreamDestroy(origin);
  }
};

extern "C" {

gx_status gx_batch_open(gx_handle *const *jobs, float *const *dev_results, int njobs, int mode, int nstreams,
                        gx_batch **out)
{
  if (!jobs || !dev_results || !out || njobs < 1) return GX_ERR_ARG;
  if (mode < GX_BATCH_SERIAL || mode > GX_BATCH_GRAPH) return GX_ERR_ARG;
  if (nstreams < 0 || nstreams > kMaxBranches) return GX_ERR_ARG;
  for (int j = 0; j < njobs; j++) {
    if (!jobs[j] || !dev_results[j]) return GX_ERR_ARG;
    if (jobs[j]->device != jobs[0]->device) return GX_ERR_ARG;
    for (int i = 0; i < j; i++)
      if (jobs[i] == jobs[j]) return GX_ERR_ARG;   // a handle's buffers serve one subint at a time
  }
  for (int j = 0; j < njobs; j++)
    if (jobs[j]->device < 0) return GX_ERR_STATE;   // host-only handle
  gx_batch *b = new gx_batch();
  b->mode = mode;
  b->device = jobs[0]->device;
  b->jobs.assign(jobs, jobs + njobs);
  for (int j = 0; j < njobs; j++) {
    b->results.push_back(reinterpret_cast<float2 *>(dev_results[j]));
    b->cost.push_back(job_cost(jobs[j]));
  }
  gx_status r = GX_OK;
  auto ck = [&](cudaError_t e, const char *w) {
    if (r == GX_OK) r = b->cuda(e, w);
  };
  ck(cudaSetDevice(b->device), "cudaSetDevice");
  ck(cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking), "cudaStreamCreate");
  ck(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "cudaEventCreate");
  ck(cudaEventCreate(&b->ev0), "cudaEventCreate");
  ck(cudaEventCreate(&b->ev1), "cudaEventCreate");
  for (int i = 0; i < kMaxBranches && r == GX_OK; i++) {
    ck(cudaStreamCreateWithFlags(&b->branch[i], cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming), "cudaEventCreate");
  }
  if (r != GX_OK) {
    b->release();
    delete b;
    return r;
  }
  if (mode == GX_BATCH_SERIAL) {
    b->nbranch = 1;
  } else if (nstreams == 0) {
    b->tuning = true;
  } else {
    b->nbranch = nstreams;
  }
  *out = b;
  return GX_OK;
}

gx_status gx_batch_run(gx_batch *b, const gx_subint_desc *const *subs)
{
  if (!b || !subs) return GX_ERR_ARG;
  return b->run(subs);
}

gx_status gx_batch_synchronize(gx_batch *b, float *device_ms)
{
  if (!b) return GX_ERR_ARG;
  if (!b->pending) return b->fail(GX_ERR_STATE, "no batch step in flight");
  gx_status r = b->finish();
  if (device_ms) *device_ms = b->last_ms;
  return r;
}

gx_status gx_batch_info(const gx_batch *b, int *nstreams, int *tuning, int *launches)
{
  if (!b) return GX_ERR_ARG;
  if (nstreams) *nstreams = b->tuning ? 0 : b->nbranch;
  if (tuning) *tuning = b->tuning ? 1 : 0;
  if (launches) *launches = b->launches;
  return GX_OK;
}

// Launch-shape tuner: jobs whose kernels take the same template instances
// (X-step form and register/super-tile shape, transform length, sample
// format, band count) form a class; the class's costliest job runs its
// subint under every candidate (X-step variant x F-step items per group),
// timed alone by events, and the fastest candidate goes to every job of the
// class.  The candidates leave the results unchanged, so tuning steps are
// ordinary steps.
gx_status gx_batch_tune_tiles(gx_batch *b, const gx_subint_desc *const *subs, int reps, int *nclasses)
{
  if (!b || !subs || reps < 1) return GX_ERR_ARG;
  gx_status r;
  if ((r = b->cuda(cudaSetDevice(b->device), "cudaSetDevice")) != GX_OK) return r;
  if ((r = b->finish()) != GX_OK) return r;
  for (auto &g : b->graph)   // graphs hold the launch shapes they captured
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  struct Key {
    int tc, T, ST, F, nbits, cplx, nbands;
    bool operator<(const Key &o) const
    {
      return std::tie(tc, T, ST, F, nbits, cplx, nbands) < std::tie(o.tc, o.T, o.ST, o.F, o.nbits, o.cplx, o.nbands);
    }
  };
  std::map<Key, std::vector<int>> classes;
  for (size_t j = 0; j < b->jobs.size(); j++) {
    const gx_handle *h = b->jobs[j];
    const Key k{h->tc ? 1 : 0, h->tc ? 0 : h->xs.T, h->tc ? 0 : h->xs.ST, h->J.fftlen, h->J.nbits, h->J.cplx, h->J.nbands};
    classes[k].push_back((int)j);
  }
  const int items[] = {2, 4, 8};
  for (auto &kv : classes) {
    const std::vector<int> &members = kv.second;
    int jb = members[0];
    for (int j : members)
      if (b->cost[j] > b->cost[jb]) jb = j;
    gx_handle *h = b->jobs[jb];
    const int nxv = h->tc ? 1 : gx::kXmacVariants;
    double best = 1e30;
    int bx = 0, bf = 4;
    for (int xv = 0; xv < nxv; xv++)
      for (int fi : items) {
        if ((r = gx_set_tiles(h, xv, fi)) != GX_OK) return b->fail(r, h->err);
        float ms = 1e30f;
        for (int rep = 0; rep < reps; rep++) {
          if ((r = gx_stage_subint(h, subs[jb], subs[jb]->data)) != GX_OK) return b->fail(r, h->err);
          if ((r = b->cuda(cudaEventRecord(b->ev0, b->origin), "cudaEventRecord")) != GX_OK) return r;
          if ((r = b->enqueue_job(jb, b->origin)) != GX_OK) return r;
          if ((r = b->cuda(cudaEventRecord(b->ev1, b->origin), "cudaEventRecord")) != GX_OK) return r;
          if ((r = b->cuda(cudaEventSynchronize(b->ev1), "cudaEventSynchronize")) != GX_OK) return r;
          float t = 0.f;
          if ((r = b->cuda(cudaEventElapsedTime(&t, b->ev0, b->ev1), "cudaEventElapsedTime")) != GX_OK) return r;
          ms = std::min(ms, t);
        }
        if (ms < best) {
          best = ms;
          bx = xv;
          bf = fi;
        }
      }
    for (int j : members)
      if ((r = gx_set_tiles(b->jobs[j], bx, bf)) != GX_OK) return b->fail(r, b->jobs[j]->err);
  }
  if (nclasses) *nclasses = (int)classes.size();
  return GX_OK;
}

const char *gx_batch_last_error(const gx_batch *b) { return b ? b->err.c_str() : "null batch"; }

gx_status gx_batch_close(gx_batch *b)
{
  if (!b) return GX_ERR_ARG;
  b->release();
  delete b;
  return GX_OK;
}

}  // extern "C"
