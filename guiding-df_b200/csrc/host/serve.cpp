// serve.cpp -- a guiding server: many resident network instances, requests
// admitted continuously under an HBM budget and batched on the device.
//
// The reference guides one render job at a time (GuidedPathTracer owns one
// LearnedDistribution, integrator.h:206-209); this is the loop that lets
// many jobs share one GPU. One scheduler thread owns all CUDA work:
//   * instances (gdf_ctx, registered by the caller) stay resident; their
//     device footprint counts against the budget;
//   * requests wait in arrival order; per instance, a training step (it
//     writes the networks) is admitted once every earlier request of that
//     instance is done, an inference request (it only reads) once no
//     earlier training step of the instance is pending or running, so the
//     inference requests between two steps may run together; each also
//     needs a free stream slot and transient memory within the budget;
//   * all inference requests admitted in one round run as one grouped
//     launch (gdf_group_infer); each training request runs on its own
//     stream, overlapping the inference;
//   * completions are detected with events; latency = completion - submit.
#include <algorithm>
#include <cmath>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "context.h"

namespace {

using Clock = std::chrono::steady_clock;

gdf_status sfail(gdf_status s, const std::string& msg) {
  gdf::set_last_error(msg.c_str());
  return s;
}

struct Request {
  uint64_t ticket = 0;
  gdf_request r{};
  Clock::time_point t_submit{}, t_done{};
  int state = 0;  // 0 pending, 1 on the device, 2 done
  int slot = -1;
  int job = -1;  // index in its slot's grouped launch (inference)
  int64_t transient = 0;
  gdf_status status = GDF_OK;
  std::string msg;  // what failed, when status is not GDF_OK
  gdf_train_stats stats{};
};

struct SlotOut {  // pinned: a training request's loss sum, squared gradient
                  // norm and dropped records; the slot's device error flag
  double stats[2];
  unsigned long long dropped;
  uint32_t dev_err;
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  SlotOut* out = nullptr;      // read back when the slot's work ends
  gdf_group* group = nullptr;  // grouped inference launches on this slot
  std::vector<Request*> reqs;  // requests whose work ends at `done`
  int64_t held_transient = 0;  // of requests done before `done`: freed with it
  bool busy = false;
};

}  // namespace

struct gdf_server {
  gdf_server_config cfg{};
  std::mutex mu;
  std::condition_variable cv;
  std::thread worker;
  bool stop = false;
  std::vector<gdf_ctx*> instances;
  std::unordered_map<gdf_ctx*, int> busy;        // requests of the instance on the device
  std::unordered_map<gdf_ctx*, int> busy_train;  // ... of which training steps
  int64_t resident = 0, transient = 0;
  int max_train = 1, train_busy = 0;  // slots training may hold / holds
  std::deque<Request*> pending;
  std::unordered_map<uint64_t, Request*> all;
  std::vector<Slot> slots;
  uint64_t next_ticket = 1;
  // statistics since the last reset
  std::vector<double> latency_ms;
  int64_t queries_done = 0, requests_done = 0;
  Clock::time_point t_first{}, t_last{};
  bool have_first = false;
};

namespace {

int64_t transient_bytes(const gdf_request& r) {
  // grouped feature tiles for inference (2 networks x 64 B per query at the
  // full configuration); the training step uses its context's workspace
  return r.kind == GDF_REQ_INFER ? (r.n + 127) / 128 * 128 * 128 : 0;
}

// Copies a device error flag to pinned memory and clears it, in stream order.
void read_and_clear(uint32_t* d_flag, uint32_t* h_flag, cudaStream_t st) {
  cudaMemcpyAsync(h_flag, d_flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
  cudaMemsetAsync(d_flag, 0, sizeof(uint32_t), st);
}

// Issues one round of admitted work. Holds the lock.
void admit(gdf_server* s) {
  std::vector<Request*> infer, train;
  std::vector<int> free_slots;
  for (int i = 0; i < static_cast<int>(s->slots.size()); ++i)
    if (!s->slots[i].busy) free_slots.push_back(i);
  if (free_slots.empty()) return;
  size_t slots_needed = 0;
  int64_t mem = s->resident + s->transient;
  // Per instance, in arrival order: a training step (it writes the
  // networks) runs alone, after every earlier request and before every
  // later one; inference requests (they only read) between two training
  // steps may run together, in one grouped launch or beside each other.
  struct Round {
    bool blocked = false;  // an earlier request of the instance waits: so do the later ones
    bool train = false;    // a training step of the instance was admitted this round
    bool infer = false;    // an inference request of the instance was admitted this round
  };
  std::unordered_map<gdf_ctx*, Round> round;
  for (auto it = s->pending.begin(); it != s->pending.end();) {
    Request* q = *it;
    gdf_ctx* inst = q->r.instance;
    Round& ri = round[inst];
    const bool is_infer = q->r.kind == GDF_REQ_INFER;
    const bool inst_free = !ri.blocked && !ri.train &&
                           (is_infer ? s->busy_train[inst] == 0 : (s->busy[inst] == 0 && !ri.infer));
    const bool mem_ok = mem + q->transient <= s->cfg.hbm_budget_bytes;
    bool ok = inst_free && mem_ok;
    if (ok && is_infer)
      ok = static_cast<int>(infer.size()) < s->cfg.max_batch && (!infer.empty() || slots_needed < free_slots.size());
    if (ok && !is_infer)
      ok = slots_needed < free_slots.size() && s->train_busy + static_cast<int>(train.size()) < s->max_train;
    if (!ok) {
      ri.blocked = true;  // keeps arrival order per instance
      ++it;
      continue;
    }
    if (is_infer) ri.infer = true;
    else ri.train = true;
    if (q->r.kind == GDF_REQ_INFER) {
      if (infer.empty()) ++slots_needed;
      infer.push_back(q);
    } else {
      ++slots_needed;
      train.push_back(q);
    }
    q->state = 1;
    mem += q->transient;
    s->transient += q->transient;
    s->busy[inst] += 1;
    if (!is_infer) s->busy_train[inst] += 1;
    it = s->pending.erase(it);
  }
  size_t used_slots = 0;
  for (Request* q : train) {
    Slot& sl = s->slots[free_slots[used_slots++]];
    q->slot = static_cast<int>(&sl - s->slots.data());
    gdf_ctx* inst = q->r.instance;
    // training's persistent kernels leave train_sm_reserve SMs to inference;
    // the step stays on its slot's stream (the other slots fill the device,
    // and forking every instance's steps over more streams lengthened the
    // latency tail: slowdown p99 127-654 against 74-138)
    inst->c.train_ctas = s->cfg.train_sm_reserve > 0 ? inst->c.num_sms - s->cfg.train_sm_reserve : 0;
    inst->c.train_one_stream = true;
    q->status = gdf_train_step(inst, q->r.in_theta_dev, q->r.in_phi_dev, q->r.target_dev, q->r.n, nullptr, sl.stream);
    inst->c.train_ctas = 0;
    inst->c.train_one_stream = false;
    if (q->status) q->msg = gdf_last_error();
    // the step's FP64 statistics and the instance's device error flag, read
    // back without blocking the scheduler
    cudaMemcpyAsync(sl.out->stats, inst->c.ws.stats, sizeof(sl.out->stats), cudaMemcpyDeviceToHost, sl.stream);
    cudaMemcpyAsync(&sl.out->dropped, inst->c.ws.dropped, sizeof(sl.out->dropped), cudaMemcpyDeviceToHost,
                    sl.stream);
    read_and_clear(inst->c.d_err, &sl.out->dev_err, sl.stream);
    sl.reqs.assign(1, q);
    sl.busy = true;
    s->train_busy += 1;
    cudaEventRecord(sl.done, sl.stream);
  }
  if (!infer.empty()) {
    Slot& sl = s->slots[free_slots[used_slots++]];
    // smallest first: a grouped launch finishes its jobs roughly in table
    // order, and each request is returned as soon as its job is done
    std::stable_sort(infer.begin(), infer.end(), [](const Request* a, const Request* b) { return a->r.n < b->r.n; });
    std::vector<gdf_job> jobs(infer.size());
    for (size_t k = 0; k < infer.size(); ++k) {
      const gdf_request& r = infer[k]->r;
      jobs[k] = gdf_job{r.instance, r.queries_dev, r.guided_dev, r.uniforms_dev, r.philox_seed,
                        r.philox_offset, r.wi_dev, r.n};
      infer[k]->job = static_cast<int>(k);
    }
    // while training runs, inference takes the SMs training leaves free;
    // a grouped launch keeps its CTA count to the end, so later requests get
    // the whole device again once training is done
    gdf_group_set_sm_cap(sl.group, s->cfg.train_sm_reserve > 0 && s->train_busy > 0 ? s->cfg.train_sm_reserve : 0);
    const gdf_status st = gdf_group_infer(sl.group, jobs.data(), static_cast<int32_t>(jobs.size()), sl.stream);
    const std::string msg = st ? gdf_last_error() : "";
    for (Request* q : infer) {
      q->status = st;
      q->msg = msg;
    }
    read_and_clear(gdf::group_err_flag(sl.group), &sl.out->dev_err, sl.stream);
    sl.reqs = infer;
    sl.busy = true;
    cudaEventRecord(sl.done, sl.stream);
  }
}

// Marks a request done at `now` (latency and statistics); its transient
// memory is released by the caller.
void finish(gdf_server* s, Request* q, Clock::time_point now) {
  q->state = 2;
  q->t_done = now;
  s->busy[q->r.instance] -= 1;
  if (q->r.kind == GDF_REQ_TRAIN) s->busy_train[q->r.instance] -= 1;
  s->latency_ms.push_back(std::chrono::duration<double, std::milli>(now - q->t_submit).count());
  s->queries_done += q->r.n;
  s->requests_done += 1;
  s->t_last = now;
}

// Completion of requests whose work has ended: inference requests whose
// job in a still-running grouped launch is done (gdf_group_job_done), then
// whole slots. Holds the lock.
bool complete(gdf_server* s) {
  bool any = false;
  for (Slot& sl : s->slots) {
    if (!sl.busy) continue;
    const cudaError_t e = cudaEventQuery(sl.done);
    if (e == cudaErrorNotReady) {
      if (sl.reqs.empty() || sl.reqs[0]->r.kind != GDF_REQ_INFER) continue;
      const Clock::time_point now = Clock::now();
      std::vector<Request*> rest;
      for (Request* q : sl.reqs) {
        if (q->status == GDF_OK && gdf_group_job_done(sl.group, q->job)) {
          finish(s, q, now);
          sl.held_transient += q->transient;
          any = true;
        } else {
          rest.push_back(q);
        }
      }
      sl.reqs.swap(rest);
      continue;
    }
    const Clock::time_point now = Clock::now();
    s->transient -= sl.held_transient;
    sl.held_transient = 0;
    for (Request* q : sl.reqs) {
      if (e != cudaSuccess && q->status == GDF_OK) {
        q->status = GDF_ERR_CUDA;
        q->msg = cudaGetErrorString(e);
      } else if (sl.out->dev_err != 0u && q->status == GDF_OK) {
        q->status = GDF_ERR_TIMEOUT;
        q->msg = "a bounded device wait gave up (code " + std::to_string(sl.out->dev_err) + ")";
      }
      if (q->r.kind == GDF_REQ_TRAIN) {
        s->train_busy -= 1;
        q->stats.loss = sl.out->stats[0] / static_cast<double>(q->r.n);
        q->stats.grad_norm = std::sqrt(sl.out->stats[1]);
        q->stats.n_records = q->r.n;
        q->stats.n_dropped = static_cast<int64_t>(sl.out->dropped);
      }
      s->transient -= q->transient;
      finish(s, q, now);
    }
    sl.reqs.clear();
    sl.busy = false;
    any = true;
  }
  return any;
}

void run(gdf_server* s) {
  cudaSetDevice(s->cfg.device);
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stop) {
    const bool done = complete(s);
    if (!s->pending.empty()) admit(s);
    const bool idle = s->pending.empty() &&
                      std::none_of(s->slots.begin(), s->slots.end(), [](const Slot& x) { return x.busy; });
    if (done) s->cv.notify_all();
    if (idle) s->cv.wait_for(lk, std::chrono::milliseconds(5));
    else s->cv.wait_for(lk, std::chrono::microseconds(20));
  }
}

}  // namespace

extern "C" {

gdf_status gdf_server_create(const gdf_server_config* cfg, gdf_server** out) {
  if (!cfg || !out) return sfail(GDF_ERR_INVALID_ARG, "null config / output");
  if (cfg->slots < 1 || cfg->slots > 64 || cfg->max_batch < 1 || cfg->max_batch > 4096 ||
      cfg->max_train_slots < 0 || cfg->hbm_budget_bytes <= 0 || cfg->train_sm_reserve < 0)
    return sfail(GDF_ERR_INVALID_ARG,
                 "slots in [1, 64], max_batch in [1, 4096], max_train_slots >= 0, positive budget, "
                 "train_sm_reserve >= 0");
  *out = nullptr;
  gdf_server* s = new (std::nothrow) gdf_server();
  if (!s) return sfail(GDF_ERR_OOM_BUDGET, "host allocation failed");
  s->cfg = *cfg;
  s->max_train = cfg->max_train_slots > 0 ? std::min(cfg->max_train_slots, cfg->slots)
                                          : std::max(1, cfg->slots - 1);
  if (cudaSetDevice(cfg->device) != cudaSuccess) {
    delete s;
    return sfail(GDF_ERR_CUDA, "cudaSetDevice");
  }
  int n_sms = 0;
  cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, cfg->device);
  if (cfg->train_sm_reserve >= n_sms) {
    delete s;
    return sfail(GDF_ERR_INVALID_ARG, "train_sm_reserve must leave training at least one SM");
  }
  s->slots.resize(static_cast<size_t>(cfg->slots));
  for (Slot& sl : s->slots) {
    gdf_status st;
    if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess ||
        cudaMallocHost(&sl.out, sizeof(SlotOut)) != cudaSuccess) {
      gdf_server_destroy(s);
      return sfail(GDF_ERR_CUDA, "server streams");
    }
    if ((st = gdf_group_create(cfg->max_batch, &sl.group)) || (st = gdf_group_set_shape(sl.group, 4, 256)) ||
        (st = gdf_group_track_jobs(sl.group, 1))) {
      gdf_server_destroy(s);
      return st;
    }
  }
  s->worker = std::thread(run, s);
  *out = s;
  return GDF_OK;
}

gdf_status gdf_server_destroy(gdf_server* s) {
  if (!s) return GDF_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv.notify_all();
  if (s->worker.joinable()) s->worker.join();
  for (Slot& sl : s->slots) {
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    if (sl.group) gdf_group_destroy(sl.group);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.stream) cudaStreamDestroy(sl.stream);
    if (sl.out) cudaFreeHost(sl.out);
  }
  for (auto& kv : s->all) delete kv.second;
  delete s;
  return GDF_OK;
}

gdf_status gdf_server_add_instance(gdf_server* s, gdf_ctx* ctx) {
  if (!s || !ctx) return sfail(GDF_ERR_INVALID_ARG, "null server / context");
  int64_t bytes = 0;
  gdf_status st = gdf_ctx_bytes(ctx, &bytes);
  if (st) return st;
  std::lock_guard<std::mutex> lk(s->mu);
  if (std::find(s->instances.begin(), s->instances.end(), ctx) != s->instances.end()) return GDF_OK;
  if (s->resident + bytes > s->cfg.hbm_budget_bytes)
    return sfail(GDF_ERR_OOM_BUDGET, "instance does not fit the server's HBM budget");
  s->resident += bytes;
  s->instances.push_back(ctx);
  return GDF_OK;
}

gdf_status gdf_server_submit(gdf_server* s, const gdf_request* r, uint64_t* ticket) {
  if (!s || !r || !ticket) return sfail(GDF_ERR_INVALID_ARG, "null argument");
  if (r->kind != GDF_REQ_INFER && r->kind != GDF_REQ_TRAIN) return sfail(GDF_ERR_INVALID_ARG, "request kind");
  if (r->n <= 0) return sfail(GDF_ERR_INVALID_ARG, "request with n <= 0");
  Request* q = new (std::nothrow) Request();
  if (!q) return sfail(GDF_ERR_OOM_BUDGET, "host allocation failed");
  q->r = *r;
  q->transient = transient_bytes(*r);
  q->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (std::find(s->instances.begin(), s->instances.end(), r->instance) == s->instances.end()) {
      delete q;
      return sfail(GDF_ERR_INVALID_ARG, "request for an unregistered instance");
    }
    if (q->transient + s->resident > s->cfg.hbm_budget_bytes) {
      delete q;
      return sfail(GDF_ERR_OOM_BUDGET, "request can never fit the HBM budget");
    }
    q->ticket = s->next_ticket++;
    s->all[q->ticket] = q;
    s->pending.push_back(q);
    if (!s->have_first) {
      s->have_first = true;
      s->t_first = q->t_submit;
    }
  }
  s->cv.notify_all();
  *ticket = q->ticket;
  return GDF_OK;
}

gdf_status gdf_server_wait(gdf_server* s, uint64_t ticket, gdf_train_stats* stats, double* latency_ms) {
  if (!s) return sfail(GDF_ERR_INVALID_ARG, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(ticket);
  if (it == s->all.end()) return sfail(GDF_ERR_INVALID_ARG, "unknown ticket");
  Request* q = it->second;
  s->cv.wait(lk, [&] { return q->state == 2 || s->stop; });
  if (q->state != 2) return sfail(GDF_ERR_STATE, "server stopped");
  if (stats) *stats = q->stats;
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(q->t_done - q->t_submit).count();
  const gdf_status st = q->status;
  const std::string msg = q->msg;
  s->all.erase(it);
  delete q;
  if (st) return sfail(st, "request failed: " + msg);
  return GDF_OK;
}

gdf_status gdf_server_get_stats(gdf_server* s, gdf_server_stats* out, int32_t reset) {
  if (!s || !out) return sfail(GDF_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(out, 0, sizeof(*out));
  out->requests = s->requests_done;
  out->queries = s->queries_done;
  out->pending = static_cast<int64_t>(s->pending.size());
  out->resident_bytes = s->resident;
  std::vector<double> l = s->latency_ms;
  if (!l.empty()) {
    std::sort(l.begin(), l.end());
    auto pct = [&](double p) { return l[std::min(l.size() - 1, static_cast<size_t>(p * (l.size() - 1) + 0.5))]; };
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    out->max_ms = l.back();
    const double span = std::chrono::duration<double>(s->t_last - s->t_first).count();
    out->queries_per_s = span > 0 ? static_cast<double>(s->queries_done) / span : 0.0;
  }
  if (reset) {
    s->latency_ms.clear();
    s->queries_done = s->requests_done = 0;
    s->have_first = false;
  }
  return GDF_OK;
}

}  // extern "C"
