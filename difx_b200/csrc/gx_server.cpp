// Request loop over resident correlation jobs on one GPU (continuous batching).
//
// Jobs are opened handles (their delay models, twiddles, tables and
// accumulators stay on the device between requests) attached to the server;
// the device memory they hold counts against the server's HBM budget.
// Requests -- one subint of one job -- are queued as they arrive and admitted
// earliest deadline first (a request's deadline is its submission time plus
// its job's deadline, by default the job's subint duration: a real-time
// subint must be correlated before the next one has been recorded; requests
// without a deadline follow in arrival order) by `slots` worker threads as
// soon as (a) a slot is free,
// (b) no other request of the same job is on the GPU (a job's device buffers
// serve one subint at a time), and (c) the memory the request adds keeps the
// total within the budget (a request is always admitted when nothing else
// is in flight, so an oversized request cannot stall the loop).  Requests of
// different jobs therefore run concurrently, each on its job's stream, and a
// request that arrives while others are on the GPU starts as soon as a slot
// and memory free up.  With device inputs, a request runs on a stream whose
// CUDA priority follows its deadline's rank among the requests on the GPU
// when it is admitted (the earliest deadline on the highest priority), so
// that the GPU's block scheduler serves urgent requests first when several
// share it.  Each request's latency runs from submission to the moment its
// results are in the caller's buffer.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>
#include "gx_handle.h"

using Clock = std::chrono::steady_clock;

namespace {

struct Request {
  long long ticket;
  int job;
  gx_subint_desc sub;
  float *results;
  long long bytes;
  Clock::time_point t_submit;
  Clock::time_point deadline;   // time_point::max(): none
  gx_status status = GX_OK;
  double latency_ms = 0;
  bool done = false;
};

struct Job {
  gx_handle *h;
  long long resident;
  double deadline_ms;   // relative deadline of its requests; <= 0: none
  bool busy = false;
};

// The default executors: host buffers through gx_subint, or device buffers
// through gx_subint_device with the result array copied to the caller.
gx_status run_host(void *, gx_handle *h, int, const gx_subint_desc *sub, float *results)
{
  return gx_subint(h, sub, results);
}

gx_status run_device_inputs(void *, gx_handle *h, int, const gx_subint_desc *sub, float *results)
{
  gx_status s = gx_subint_device(h, sub, reinterpret_cast<float *>(h->d_results), nullptr);
  if (s != GX_OK) return s;
  CKR(h, cudaMemcpyAsync(results, h->d_results, sizeof(float2) * h->rl, cudaMemcpyDeviceToHost, h->stream));
  return gx_synchronize(h);
}

// The same on a given stream (a priority stream of the loop).
gx_status run_device_inputs_on(gx_handle *h, const gx_subint_desc *sub, float *results, cudaStream_t st)
{
  gx_status s = gx_subint_device(h, sub, reinterpret_cast<float *>(h->d_results), st);
  if (s != GX_OK) return s;
  CKR(h, cudaMemcpyAsync(results, h->d_results, sizeof(float2) * h->rl, cudaMemcpyDeviceToHost, st));
  CKR(h, cudaStreamSynchronize(st));
  return gx_synchronize(h);
}

}  // namespace

struct gx_server {
  int slots = 1;
  long long budget = 0;
  bool device_inputs = false;
  gx_server_executor exec = run_host;
  void *exec_ctx = nullptr;
  bool started = false;

  std::vector<Job> jobs;
  long long resident_total = 0, inflight_bytes = 0;
  int inflight = 0;
  std::deque<Request *> queue;
  std::unordered_map<long long, Request *> reqs;
  long long next_ticket = 1;
  std::vector<double> latencies;
  long long completed = 0, failed = 0;
  std::string last_error;       // message of the last failed request
  std::string last_error_copy;  // the copy gx_server_last_error hands out

  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::vector<std::thread> workers;
  bool stopping = false;
  // priority streams (device inputs): [worker][level], level 0 the highest priority
  std::vector<std::vector<cudaStream_t>> pstreams;
  std::vector<Clock::time_point> running_deadline;   // deadlines of the requests on the GPU
  bool streams_tried = false;

  // per worker, one stream per priority level of the device (the inputs' device)
  void make_streams(const gx_handle *h)
  {
    streams_tried = true;
    if (!h || h->device < 0 || cudaSetDevice(h->device) != cudaSuccess) return;
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) return;
    const int nlev = std::min(4, least - greatest + 1);
    if (nlev < 2) return;
    pstreams.assign(slots, {});
    for (int w = 0; w < slots; w++)
      for (int l = 0; l < nlev; l++) {
        cudaStream_t st = nullptr;
        if (cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, greatest + l) != cudaSuccess) {
          pstreams.clear();
          return;
        }
        pstreams[w].push_back(st);
      }
  }

  // the admissible queued request with the earliest deadline (arrival order
  // among equal deadlines and among requests without one)
  std::deque<Request *>::iterator pick()
  {
    auto best = queue.end();
    for (auto it = queue.begin(); it != queue.end(); ++it) {
      const Request *r = *it;
      if (jobs[r->job].busy) continue;
      if (inflight > 0 && resident_total + inflight_bytes + r->bytes > budget) continue;
      if (best == queue.end() || r->deadline < (*best)->deadline) best = it;
    }
    return best;
  }

  void worker(int wid)
  {
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      std::deque<Request *>::iterator it;
      cv_work.wait(lk, [&] { return (it = pick()) != queue.end() || (stopping && queue.empty()); });
      if (it == queue.end()) return;   // stopping, and everything queued has been taken
      Request *r = *it;
      queue.erase(it);
      Job &J = jobs[r->job];
      J.busy = true;
      inflight++;
      inflight_bytes += r->bytes;
      // the request's priority level: how many requests on the GPU have an earlier deadline
      cudaStream_t pst = nullptr;
      if (exec == run_device_inputs) {
        if (!streams_tried) make_streams(J.h);
        if (!pstreams.empty()) {
          int rank = 0;
          for (const auto &dl : running_deadline)
            if (dl < r->deadline) rank++;
          pst = pstreams[wid][std::min(rank, (int)pstreams[wid].size() - 1)];
        }
      }
      running_deadline.push_back(r->deadline);
      lk.unlock();
      const gx_status st = pst ? run_device_inputs_on(J.h, &r->sub, r->results, pst)
                               : exec(exec_ctx, J.h, r->job, &r->sub, r->results);
      const double ms = std::chrono::duration<double, std::milli>(Clock::now() - r->t_submit).count();
      lk.lock();
      running_deadline.erase(std::find(running_deadline.begin(), running_deadline.end(), r->deadline));
      J.busy = false;
      inflight--;
      inflight_bytes -= r->bytes;
      r->status = st;
      r->latency_ms = ms;
      r->done = true;
      if (st == GX_OK) {
        latencies.push_back(ms);
        completed++;
      } else {
        failed++;
        last_error = "job " + std::to_string(r->job) + ": " + (J.h ? J.h->err : std::string("executor failed"));
      }
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }

  void start()
  {
    if (started) return;
    started = true;
    for (int i = 0; i < slots; i++) workers.emplace_back([this, i] { worker(i); });
  }
};

extern "C" {

gx_status gx_server_open(int slots, long long hbm_budget_bytes, int device_inputs, gx_server **out)
{
  if (!out || slots < 1 || slots > 64 || hbm_budget_bytes <= 0) return GX_ERR_ARG;
  gx_server *s = new gx_server();
  s->slots = slots;
  s->budget = hbm_budget_bytes;
  s->device_inputs = device_inputs != 0;
  s->exec = s->device_inputs ? run_device_inputs : run_host;
  *out = s;
  return GX_OK;
}

gx_status gx_server_set_executor(gx_server *s, gx_server_executor fn, void *ctx)
{
  if (!s || !fn) return GX_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->started) return GX_ERR_STATE;
  s->exec = fn;
  s->exec_ctx = ctx;
  return GX_OK;
}

gx_status gx_server_attach(gx_server *s, gx_handle *h, long long resident_bytes, int *job)
{
  if (!s || !job) return GX_ERR_ARG;
  if (!h && resident_bytes < 0) return GX_ERR_ARG;
  const long long res = resident_bytes >= 0 ? resident_bytes : h->dev_bytes;
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->resident_total + res > s->budget) return GX_ERR_NOMEM;
  // a real-time job's subint must be done within the subint's duration
  s->jobs.push_back(Job{h, res, h ? h->jd.subint_ns / 1e6 : 0.0});
  s->resident_total += res;
  *job = (int)s->jobs.size() - 1;
  return GX_OK;
}

gx_status gx_server_set_deadline(gx_server *s, int job, double deadline_ms)
{
  if (!s) return GX_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  if (job < 0 || job >= (int)s->jobs.size()) return GX_ERR_ARG;
  s->jobs[job].deadline_ms = deadline_ms;
  return GX_OK;
}

gx_status gx_server_submit(gx_server *s, int job, const gx_subint_desc *sub, float *results, long long request_bytes,
                           long long *ticket)
{
  if (!s || !sub || !ticket) return GX_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  if (job < 0 || job >= (int)s->jobs.size()) return GX_ERR_ARG;
  long long bytes = request_bytes;
  if (bytes < 0) {   // what the request adds: growth of the job's input buffers (host inputs only)
    bytes = 0;
    const gx_handle *h = s->jobs[job].h;
    if (h && !s->device_inputs && sub->datalen)
      for (int i = 0; i < h->jd.nstations && i < (int)h->data_cap[0].size(); i++)
        bytes += std::max<long long>(0, (long long)sub->datalen[i] - (long long)h->data_cap[0][i]);
  }
  if (s->resident_total + bytes > s->budget) return GX_ERR_NOMEM;
  Request *r = new Request();
  r->ticket = s->next_ticket++;
  r->job = job;
  r->sub = *sub;
  r->results = results;
  r->bytes = bytes;
  r->t_submit = Clock::now();
  const double dl = s->jobs[job].deadline_ms;
  r->deadline = dl > 0 ? r->t_submit + std::chrono::duration_cast<Clock::duration>(
                                           std::chrono::duration<double, std::milli>(dl))
                       : Clock::time_point::max();
  s->queue.push_back(r);
  s->reqs[r->ticket] = r;
  *ticket = r->ticket;
  s->start();
  s->cv_work.notify_one();
  return GX_OK;
}

gx_status gx_server_wait(gx_server *s, long long ticket, double *latency_ms)
{
  if (!s) return GX_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return GX_ERR_ARG;
  Request *r = it->second;
  s->cv_done.wait(lk, [&] { return r->done; });
  const gx_status st = r->status;
  if (latency_ms) *latency_ms = r->latency_ms;
  s->reqs.erase(it);
  delete r;
  return st;
}

gx_status gx_server_stats(gx_server *s, int reset, gx_latency_stats *out)
{
  if (!s || !out) return GX_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  memset(out, 0, sizeof(*out));
  out->completed = s->completed;
  out->failed = s->failed;
  std::vector<double> v = s->latencies;
  if (!v.empty()) {
    std::sort(v.begin(), v.end());
    // percentile with linear interpolation between order statistics
    auto pct = [&](double p) {
      const double x = p / 100.0 * (double)(v.size() - 1);
      const size_t i = (size_t)x;
      const double f = x - (double)i;
      return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
    };
    out->p50_ms = pct(50);
    out->p95_ms = pct(95);
    out->p99_ms = pct(99);
    double sum = 0;
    for (double x : v) sum += x;
    out->mean_ms = sum / (double)v.size();
    out->max_ms = v.back();
  }
  if (reset) {
    s->latencies.clear();
    s->completed = s->failed = 0;
  }
  return GX_OK;
}

gx_status gx_server_close(gx_server *s)
{
  if (!s) return GX_ERR_ARG;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    s->stopping = true;
    s->cv_work.notify_all();
  }
  for (auto &t : s->workers) t.join();
  for (auto &v : s->pstreams)
    for (cudaStream_t st : v) cudaStreamDestroy(st);
  for (auto &kv : s->reqs) delete kv.second;
  delete s;
  return GX_OK;
}

const char *gx_server_last_error(gx_server *s)
{
  if (!s) return "null server";
  std::lock_guard<std::mutex> lk(s->mu);
  s->last_error_copy = s->last_error;
  return s->last_error_copy.c_str();
}

gx_status gx_device_bytes(const gx_handle *h, long long *bytes)
{
  if (!h || !bytes) return GX_ERR_ARG;
  *bytes = h->dev_bytes;
  return GX_OK;
}

}  // extern "C"
