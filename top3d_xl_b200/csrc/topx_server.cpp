// Continuous-batching job server over the C ABI (topx_server_* in include/topx.h).
//
// Worker threads are the slots.  A free worker takes the oldest queued job, builds its host
// model, estimates its device footprint from the model's grid sizes and waits until that
// footprint fits the HBM budget; then it creates the job's engine (own stream, own graphs,
// own scratch), runs the optimisation loop and frees everything.  Jobs on different workers
// overlap on the device.  Engines here run the coarsest-level solve level by level rather than
// as one persistent launch, which would want all of its CTAs resident at once.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "topx.h"
#include "topx_engine.hpp"
#include "topx_nd.hpp"

namespace {

struct Job {
  int64_t id = 0;
  topx_job spec{};
  std::vector<uint8_t> vox;
  topx_job_result res{};
  std::vector<topx_iter> hist;
  std::vector<double> density;
  std::string error;
  bool ended = false;
};

// Device bytes an engine for this model will hold: dense level-1 grid vectors and element
// arrays, the coarsest level's factor tiles with their plan and solve vectors (planned here for
// the full box of coarsest nodes, an upper bound for a masked domain), and fixed scratch.
// Calibrated to stay above the bytes the engine's buffers report (see the serving test).
int64_t footprint_estimate(const topx_info& in, int precision) {
  const int64_t ny = in.resY[0], nx = in.resX[0], nz = in.resZ[0];
  const int64_t nodes = (ny + 1) * (nx + 1) * (nz + 1), elems = ny * nx * nz;
  const int L = in.numLevels - 1;
  const int nny = in.resY[L] + 1, nnx = in.resX[L] + 1, nnz = in.resZ[L] + 1;
  const std::vector<uint8_t> all(size_t(nny) * nnx * nnz, 1);
  const int64_t stride = (int64_t(nny) * nnx * nnz + 31) / 32 * 32;
  const topx::NDPlan P = topx::nd_plan(nny, nnx, nnz, stride, all, topx::nd_leaf_nodes(int64_t(all.size())));
  const int64_t tile = int64_t(topx::ND_T) * topx::ND_T;
  const int64_t coarsest = P.ntiles * tile * (precision != TOPX_FP64 ? 12 : 8) + int64_t(P.nscr) * tile * 8 +
                           P.npos * (8 + 16) + std::max<int64_t>(P.nsolve_tasks, int64_t(P.flow.size())) * topx::ND_T * 8 + P.npos / topx::ND_T * 4 +
                           int64_t(P.tasks.size()) * 8 + int64_t(P.asmb.size()) * 20 +
                           int64_t(P.pad_diag.size()) * 8 + int64_t(P.upd_map.size()) * 4 +
                           int64_t(P.fronts.size()) * int64_t(sizeof(topx::NDFront));
  const int64_t per_node = precision != TOPX_FP64 ? 584 : 544, per_elem = 200;
  return per_node * nodes + per_elem * elems + coarsest + (int64_t(48) << 20);
}

}  // namespace

struct topx_server {
  topx_server_params params{};
  std::mutex mu;
  std::condition_variable cv_work, cv_mem, cv_done;
  std::map<int64_t, std::unique_ptr<Job>> jobs;
  std::deque<Job*> queue;
  double budget = 0, used = 0, peak = 0;
  int running = 0, max_running = 0;
  int64_t next_id = 1, submitted = 0, done = 0, failed = 0;
  bool stop = false;
  std::vector<std::thread> workers;
  std::string err;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  void worker();
  void run(Job& j);
};

void topx_server::run(Job& j) {
  topx_params p;
  topx_default_params(&p);
  p.precision = params.precision;
  p.device = params.device;
  p.coarse_coop = 0;
  topx_ctx* ctx = nullptr;
  topx_status s = topx_create(&ctx, &p);
  auto finish = [&](topx_status st) {
    j.res.status = st;
    if (st != TOPX_OK && ctx) j.error = topx_last_error(ctx);
    if (ctx) topx_destroy(ctx);
    ctx = nullptr;
  };
  if (s != TOPX_OK) return finish(s);
  const topx_job& q = j.spec;
  s = topx_load_voxels(ctx, j.vox.data(), q.nely, q.nelx, q.nelz);
  if (s != TOPX_OK) return finish(s);
  topx_info info;
  topx_get_info(ctx, &info);
  j.res.numElements = info.numElements;
  const int64_t need = footprint_estimate(info, params.precision);
  j.res.footprint_estimate = need;
  {
    std::unique_lock<std::mutex> lk(mu);
    if (double(need) > budget) {
      j.error = "job footprint exceeds the server's HBM budget";
      j.res.status = TOPX_ERR_ARG;
      topx_destroy(ctx);
      return;
    }
    cv_mem.wait(lk, [&] { return stop || used + double(need) <= budget; });
    if (stop) {
      lk.unlock();
      return finish(TOPX_ERR_STATE);
    }
    used += double(need);
    peak = std::max(peak, used);
    ++running;
    max_running = std::max(max_running, running);
  }
  j.res.t_admit = now();
  const int64_t b0 = topx::devbuf_bytes();
  s = topx_begin(ctx, q.consType, q.V0, q.nLoop, q.rMin, q.rHat, &j.res.cSolid);
  j.res.footprint_bytes = topx::devbuf_bytes() - b0;
  int loops = 0;
  while (s == TOPX_OK) {
    topx_iter it;
    const topx_status st = topx_step(ctx, &it);
    if (st == TOPX_STOP) break;
    s = st;
    if (st != TOPX_OK) break;
    j.hist.push_back(it);
    j.res.c_last = it.c;
    for (int lc = 0; lc < info.numLoadCases && lc < TOPX_MAX_LOAD_CASES; ++lc) j.res.pcg_its += it.its[lc];
    ++loops;
  }
  j.res.loops = loops;
  if (s == TOPX_OK && q.keep_density) {
    j.density.resize(size_t(info.numElements));
    s = topx_get_density(ctx, j.density.data(), j.density.size());
  }
  finish(s);
  std::lock_guard<std::mutex> lk(mu);
  used -= double(need);
  --running;
  cv_mem.notify_all();
}

void topx_server::worker() {
  for (;;) {
    Job* j = nullptr;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_work.wait(lk, [&] { return stop || !queue.empty(); });
      if (stop) return;
      j = queue.front();
      queue.pop_front();
    }
    try {
      run(*j);
    } catch (const std::exception& e) {
      j->res.status = TOPX_ERR_INTERNAL;
      j->error = e.what();
    }
    std::lock_guard<std::mutex> lk(mu);
    j->res.t_end = now();
    j->ended = true;
    if (j->res.status == TOPX_OK)
      ++done;
    else {
      ++failed;
      err = "job " + std::to_string(j->id) + ": " + j->error;
    }
    cv_done.notify_all();
  }
}

extern "C" {

topx_status topx_server_default_params(topx_server_params* p) {
  if (!p) return TOPX_ERR_ARG;
  p->slots = 6;
  p->hbm_budget_bytes = 0;
  p->precision = TOPX_FP64;
  p->device = 0;
  return TOPX_OK;
}

topx_status topx_server_create(topx_server** out, const topx_server_params* p) {
  if (!out) return TOPX_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<topx_server> s(new topx_server());
  if (p)
    s->params = *p;
  else
    topx_server_default_params(&s->params);
  if (s->params.slots < 1 || s->params.slots > 64) return TOPX_ERR_ARG;
  if (s->params.precision != TOPX_FP64 && s->params.precision != TOPX_MIXED &&
      s->params.precision != TOPX_MIXED_F32_FILTER)
    return TOPX_ERR_ARG;
  // worker threads wait on their streams a lot: yield the core instead of spinning on it
  // (takes effect only if this process has not touched the device yet)
  if (cudaSetDeviceFlags(cudaDeviceScheduleYield) != cudaSuccess) cudaGetLastError();
  s->budget = s->params.hbm_budget_bytes;
  if (s->budget <= 0) {
    size_t fr = 0, tot = 0;
    if (cudaSetDevice(s->params.device) != cudaSuccess || cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      cudaGetLastError();
      s->budget = 0;  // no device: every job fails its admission check
    } else {
      s->budget = 0.85 * double(fr);
    }
  }
  for (int i = 0; i < s->params.slots; ++i) s->workers.emplace_back([srv = s.get()] { srv->worker(); });
  *out = s.release();
  return TOPX_OK;
}

topx_status topx_server_destroy(topx_server* s) {
  if (!s) return TOPX_ERR_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    for (Job* j : s->queue) {
      j->res.status = TOPX_ERR_STATE;
      j->error = "server destroyed before the job started";
      j->ended = true;
    }
    s->queue.clear();
  }
  s->cv_work.notify_all();
  s->cv_mem.notify_all();
  for (auto& w : s->workers) w.join();
  delete s;
  return TOPX_OK;
}

topx_status topx_server_submit(topx_server* s, const topx_job* job, int64_t* id) {
  if (!s || !job || !id) return TOPX_ERR_ARG;
  if (job->nely < 3 || job->nelx < 3 || job->nelz < 3) return TOPX_ERR_ARG;
  if (job->consType != TOPX_GLOBAL && job->consType != TOPX_LOCAL) return TOPX_ERR_ARG;
  std::unique_ptr<Job> j(new Job());
  j->spec = *job;
  const size_t n = size_t(job->nely) * job->nelx * job->nelz;
  if (job->voxels)
    j->vox.assign(job->voxels, job->voxels + n);
  else
    j->vox.assign(n, 1);
  j->spec.voxels = nullptr;
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return TOPX_ERR_STATE;
  j->id = s->next_id++;
  j->res.t_submit = s->now();
  *id = j->id;
  s->queue.push_back(j.get());
  s->jobs[j->id] = std::move(j);
  ++s->submitted;
  s->cv_work.notify_one();
  return TOPX_OK;
}

topx_status topx_server_poll(topx_server* s, int64_t id, topx_job_result* out) {
  if (!s) return TOPX_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return TOPX_ERR_ARG;
  if (!it->second->ended) return TOPX_STOP;
  if (out) *out = it->second->res;
  return TOPX_OK;
}

topx_status topx_server_wait(topx_server* s, int64_t id, topx_job_result* out) {
  if (!s) return TOPX_ERR_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return TOPX_ERR_ARG;
  Job* j = it->second.get();
  s->cv_done.wait(lk, [&] { return j->ended; });
  if (out) *out = j->res;
  return TOPX_OK;
}

topx_status topx_server_get_history(topx_server* s, int64_t id, topx_iter* hist, int n, int* loops) {
  if (!s) return TOPX_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return TOPX_ERR_ARG;
  const Job& j = *it->second;
  if (!j.ended) return TOPX_ERR_STATE;
  const int k = int(j.hist.size());
  if (loops) *loops = k;
  if (hist)
    for (int i = 0; i < k && i < n; ++i) hist[i] = j.hist[size_t(i)];
  return TOPX_OK;
}

topx_status topx_server_get_density(topx_server* s, int64_t id, double* out, size_t n) {
  if (!s || !out) return TOPX_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if (it == s->jobs.end()) return TOPX_ERR_ARG;
  const Job& j = *it->second;
  if (!j.ended || j.density.empty()) return TOPX_ERR_STATE;
  if (n != j.density.size()) return TOPX_ERR_ARG;
  std::memcpy(out, j.density.data(), n * sizeof(double));
  return TOPX_OK;
}

topx_status topx_server_get_stats(topx_server* s, topx_server_stats* out) {
  if (!s || !out) return TOPX_ERR_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  out->submitted = s->submitted;
  out->done = s->done;
  out->failed = s->failed;
  out->running = s->running;
  out->queued = int64_t(s->queue.size());
  out->max_running = s->max_running;
  out->budget_bytes = s->budget;
  out->peak_bytes = s->peak;
  return TOPX_OK;
}

const char* topx_server_last_error(topx_server* s) {
  if (!s) return "null server";
  std::lock_guard<std::mutex> lk(s->mu);
  thread_local std::string copy;
  copy = s->err;
  return copy.c_str();
}

}  // extern "C"
