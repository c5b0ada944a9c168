// Serving loop: continuous batching of propagation requests on one GPU.
//
// Requests (one scenario each, device-resident inputs and outputs) are
// queued by propag_server_submit from any host thread.  A dispatcher thread
// owns `lanes` CUDA streams, each with its own propagation engine.  Whenever
// a lane is free it takes the requests waiting at that moment (up to
// max_batch, within the device-memory budget), runs their fire passes and one
// persistent propagation launch for all of them on its stream, and goes back
// to watching: requests that arrive while earlier batches are on the GPU are
// admitted as soon as a lane and memory free up, and their kernels run
// alongside the earlier ones (each batch occupies only as many clusters as it
// has jobs).  Completion is detected with an event per lane; the dispatcher
// never blocks on the GPU.
//
// Results do not depend on how requests are batched: every job's propagation
// follows its own fixed schedule, so a request's arrival times are the same
// alone and in any mix.
#include <cuda_runtime.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "propag_b200.h"

namespace propag {
void engine_keep_to_clusters(propag_engine *e);  // api.cpp
int engine_reserve(propag_engine *e, size_t job_bytes, uint32_t max_jobs, size_t slot_bytes,
                   cudaStream_t stream);
}
using propag::engine_keep_to_clusters;
using propag::engine_reserve;

// Slot scratch a lane reserves per job of a batch: dirty bitmaps, update
// arrays and list overflow of one team for tiles up to the default 323 x 323
// (about 9 MB in the worst cluster size).
constexpr size_t kSlotBytesPerJob = 10u << 20;

namespace {

uint64_t now_ns() {
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct Request {
  PropagJob job;
  PropagTerrainPtrs terrain;
  bool has_terrain = false;
  uint64_t bytes = 0;
  PropagServerResult res{};
  std::string message;
};

struct Lane {
  propag_engine *eng = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  uint64_t cap = 0;          // job scratch reserved at start-up (0: grown on demand)
  std::vector<int64_t> ids;  // requests of the batch in flight (empty: free)
};

}  // namespace

struct propag_server {
  std::mutex mu;
  std::condition_variable cv_done;  // a request finished
  std::condition_variable cv_work;  // a request arrived, or stop
  std::deque<int64_t> pending;
  std::unordered_map<int64_t, Request> reqs;
  int64_t next_id = 0;
  uint64_t budget = 0, in_use = 0;
  uint32_t max_batch = 64;
  int device = 0;
  bool stop = false;
  std::vector<Lane> lanes;
  std::thread worker;
  std::string init_error;

  void run();
  void finish(Lane &lane);
  bool dispatch(Lane &lane);
};

// Completed batch: statistics per job, then every request of the batch is done.
void propag_server::finish(Lane &lane) {
  const uint32_t n = (uint32_t)lane.ids.size();
  std::vector<PropagStats> st(n);
  const int rc = propag_engine_last_stats(lane.eng, lane.stream, st.data(), n);
  const std::string msg = rc ? propag_last_error() : std::string();
  const uint64_t t = now_ns();
  std::lock_guard<std::mutex> lk(mu);
  for (uint32_t i = 0; i < n; ++i) {
    Request &r = reqs[lane.ids[i]];
    r.res.stats = st[i];
    r.res.done_ns = t;
    r.res.status = rc ? rc : (st[i].status ? PROPAG_ERR_TIMEOUT : 1);
    if (rc) r.message = msg;
    in_use -= r.bytes;
  }
  lane.ids.clear();
  cv_done.notify_all();
}

// Takes the waiting requests that fit (count and memory) and launches them
// on the lane.  Returns whether a batch was launched.
bool propag_server::dispatch(Lane &lane) {
  std::vector<int64_t> ids;
  std::vector<PropagJob> jobs;
  std::vector<PropagTerrainPtrs> terr;
  std::vector<bool> has;
  {
    std::lock_guard<std::mutex> lk(mu);
    uint64_t lane_bytes = 0;
    while (!pending.empty() && ids.size() < max_batch) {
      Request &r = reqs[pending.front()];
      if ((lane.cap && r.bytes > lane.cap) || (budget && r.bytes > budget)) {
        // can never fit: fail it
        r.res.status = PROPAG_ERR_OOM;
        r.message = "request needs more device memory than the server's budget";
        pending.pop_front();
        cv_done.notify_all();
        continue;
      }
      // a lane's batch fits the scratch it reserved at start-up
      if ((budget && in_use + r.bytes > budget) || (lane.cap && lane_bytes + r.bytes > lane.cap)) break;
      in_use += r.bytes;
      lane_bytes += r.bytes;
      r.res.start_ns = now_ns();
      ids.push_back(pending.front());
      jobs.push_back(r.job);
      terr.push_back(r.terrain);
      has.push_back(r.has_terrain);
      pending.pop_front();
    }
    for (int64_t id : ids) reqs[id].res.batch_size = (uint32_t)ids.size();
  }
  if (ids.empty()) return false;
  int rc = 0;
  for (size_t i = 0; i < ids.size() && !rc; ++i)
    if (has[i])
      rc = propag_fire_simple_device((uint64_t)jobs[i].width * jobs[i].height, &terr[i],
                                     const_cast<float *>(jobs[i].speed_max),
                                     const_cast<float *>(jobs[i].azimuth_max),
                                     const_cast<float *>(jobs[i].eccentricity), lane.stream);
  if (!rc) rc = propag_engine_run(lane.eng, jobs.data(), (uint32_t)jobs.size(), lane.stream, nullptr);
  if (!rc && cudaEventRecord(lane.done, lane.stream) != cudaSuccess) rc = PROPAG_ERR_CUDA;
  if (rc) {
    const std::string msg = propag_last_error();
    std::lock_guard<std::mutex> lk(mu);
    for (int64_t id : ids) {
      Request &r = reqs[id];
      r.res.status = rc;
      r.message = msg;
      r.res.done_ns = now_ns();
      in_use -= r.bytes;
    }
    cv_done.notify_all();
    return false;
  }
  lane.ids = std::move(ids);
  return true;
}

void propag_server::run() {
  cudaSetDevice(device);
  for (;;) {
    bool busy = false;
    for (Lane &lane : lanes) {
      if (!lane.ids.empty() && cudaEventQuery(lane.done) == cudaSuccess) finish(lane);
      if (lane.ids.empty()) dispatch(lane);
      busy |= !lane.ids.empty();
    }
    std::unique_lock<std::mutex> lk(mu);
    if (stop && pending.empty() && !busy) break;
    if (busy)  // poll the lanes' events again shortly
      cv_work.wait_for(lk, std::chrono::microseconds(50));
    else if (pending.empty() && !stop)
      cv_work.wait_for(lk, std::chrono::milliseconds(5));
  }
}

extern "C" propag_server *propag_server_create(const PropagServerOptions *opt) {
  auto *s = new propag_server();
  const uint32_t n_lanes = opt && opt->lanes ? opt->lanes : 4;
  if (opt) {
    s->budget = opt->hbm_budget;
    if (opt->max_batch) s->max_batch = opt->max_batch;
  }
  PropagOptions eo{0, 0, 0, opt ? opt->device : -1};
  for (uint32_t i = 0; i < n_lanes; ++i) {
    Lane lane;
    lane.eng = propag_engine_create(&eo);  // selects the device, fails loudly without one
    if (lane.eng) engine_keep_to_clusters(lane.eng);  // lanes run side by side
    if (!lane.eng ||
        cudaStreamCreateWithFlags(&lane.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&lane.done, cudaEventDisableTiming) != cudaSuccess) {
      if (lane.eng) propag_engine_destroy(lane.eng);
      for (Lane &l : s->lanes) {
        cudaStreamDestroy(l.stream);
        cudaEventDestroy(l.done);
        propag_engine_destroy(l.eng);
      }
      delete s;
      return nullptr;
    }
    s->lanes.push_back(lane);
  }
  cudaGetDevice(&s->device);
  // With a budget, every lane reserves its share of it up front as job
  // scratch, plus slot scratch and staging for max_batch jobs, so that
  // serving allocates and frees no device memory: a cudaFree waits for the
  // whole device and would stall the other lanes' batches.
  if (s->budget) {
    for (Lane &l : s->lanes) {
      l.cap = s->budget / n_lanes;
      if (engine_reserve(l.eng, l.cap, s->max_batch, kSlotBytesPerJob * s->max_batch, l.stream) != PROPAG_OK ||
          cudaStreamSynchronize(l.stream) != cudaSuccess) {
        for (Lane &m : s->lanes) {
          cudaStreamDestroy(m.stream);
          cudaEventDestroy(m.done);
          propag_engine_destroy(m.eng);
        }
        delete s;
        return nullptr;
      }
    }
  }
  s->worker = std::thread([s] { s->run(); });
  return s;
}

extern "C" int64_t propag_server_submit(propag_server *s, const PropagJob *job,
                                        const PropagTerrainPtrs *terrain, uint64_t device_bytes) {
  if (!s || !job) return PROPAG_ERR_INVALID;
  if (job->width == 0 || job->height == 0 || !job->time || !job->speed_max || !job->azimuth_max ||
      !job->eccentricity)
    return PROPAG_ERR_INVALID;
  Request r;
  r.job = *job;
  if (terrain) {
    r.terrain = *terrain;
    r.has_terrain = true;
  }
  // the engine scratch the request takes, when the caller does not say
  r.bytes = device_bytes ? device_bytes : propag_engine_job_bytes(job->width, job->height);
  r.res.submit_ns = now_ns();
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return PROPAG_ERR_INVALID;
  const int64_t id = s->next_id++;
  s->reqs.emplace(id, std::move(r));
  s->pending.push_back(id);
  s->cv_work.notify_one();
  return id;
}

static int copy_result(propag_server *s, int64_t id, PropagServerResult *out, bool &done) {
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return PROPAG_ERR_INVALID;
  Request &r = it->second;
  done = r.res.status != 0;
  if (out) {
    *out = r.res;
    std::strncpy(out->message, r.message.c_str(), sizeof(out->message) - 1);
    out->message[sizeof(out->message) - 1] = '\0';
  }
  return PROPAG_OK;
}

extern "C" int propag_server_poll(propag_server *s, int64_t id, PropagServerResult *out) {
  if (!s) return PROPAG_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  bool done = false;
  const int rc = copy_result(s, id, out, done);
  return rc ? rc : (done ? 1 : 0);
}

extern "C" int propag_server_wait(propag_server *s, int64_t id, PropagServerResult *out,
                                  uint32_t timeout_ms) {
  if (!s) return PROPAG_ERR_INVALID;
  std::unique_lock<std::mutex> lk(s->mu);
  bool done = false;
  const auto until = std::chrono::steady_clock::now() + std::chrono::milliseconds(timeout_ms);
  for (;;) {
    const int rc = copy_result(s, id, out, done);
    if (rc) return rc;
    if (done) return 1;
    if (s->cv_done.wait_until(lk, until) == std::cv_status::timeout) {
      copy_result(s, id, out, done);
      return done ? 1 : 0;
    }
  }
}

extern "C" int propag_server_release(propag_server *s, int64_t id) {
  if (!s) return PROPAG_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return PROPAG_ERR_INVALID;
  if (it->second.res.status == 0) return PROPAG_ERR_INVALID;  // still queued or running
  s->reqs.erase(it);
  return PROPAG_OK;
}

extern "C" void propag_server_destroy(propag_server *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv_work.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();  // runs the queue dry first
  for (Lane &l : s->lanes) {
    cudaStreamSynchronize(l.stream);
    cudaStreamDestroy(l.stream);
    cudaEventDestroy(l.done);
    propag_engine_destroy(l.eng);
  }
  delete s;
  cudaGetLastError();
}
