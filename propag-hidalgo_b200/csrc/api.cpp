// extern "C" surface of libpropag.so: the reference plugin ABI
// (include/propag_host.h) and the B200 entry points (include/propag_b200.h).
//
// Host orchestration follows propagate() (crates/propag/src/propag.rs:323-574):
// terrain -> fire behaviour -> boundaries -> propagation -> post mask ->
// outputs.  All device work is stream-ordered; nothing here computes fire
// behaviour or arrival times on the CPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "engine.cuh"
#include "io.hpp"
#include "noalloc.hpp"
#include "propag_b200.h"

namespace propag {

// launchers (fire.cu, engine_launch.cu)
cudaError_t upload_catalog();
cudaError_t launch_fire(bool full, uint64_t n, const uint8_t *fuel, const float *const m[5],
                        const float *ws, const float *waz, const float *slope,
                        const float *aspect, float *const outs[10], int sm_count,
                        cudaStream_t stream);
cudaError_t launch_prep(const JobDev *jobs, uint32_t n_jobs, uint64_t max_cells, int sms,
                        cudaStream_t stream);
cudaError_t launch_ignite(const JobDev *jobs, uint32_t n_jobs, cudaStream_t stream);
cudaError_t launch_engine(const JobDev *jobs, uint32_t n_jobs, const SlotDev *slots,
                          uint32_t n_slots, int csize, int threads, size_t smem, uint32_t *queue,
                          StatsDev *stats, unsigned long long max_sweeps, const uint32_t *order,
                          uint32_t group, uint32_t phantom, cudaStream_t stream);
cudaError_t engine_max_clusters(int csize, int threads, size_t smem, int *n);
cudaError_t launch_post(const JobDev *jobs, uint32_t n_jobs, uint64_t max_cells, int sms,
                        StatsDev *stats, cudaStream_t stream);
cudaError_t launch_fire_weather(uint64_t n, int hour, int month, const float *t, const float *rh,
                                const float *cc, const float *pp, const uint8_t *fuel,
                                const float *herb, const float *wood, const float *ws,
                                const float *waz, const float *slope, const float *aspect,
                                float *speed_max, float *azimuth_max, float *eccentricity,
                                int sm_count, cudaStream_t stream);
// selftest.cu
cudaError_t launch_time_from(bool refm, uint64_t n, const int32_t *fx, const int32_t *fy,
                             const float *ftime, const int32_t *tx, const int32_t *ty,
                             const float *smax, const float *azmax, const float *ecc, float gdx,
                             float gdy, bool north_up, float *out, cudaStream_t stream);
cudaError_t launch_cosf_table(uint32_t first, uint64_t n, float *out, cudaStream_t stream);
cudaError_t launch_atan2f_table(int32_t ma, int32_t mb, int32_t b0, int32_t nb, float *out,
                                cudaStream_t stream);

namespace {

thread_local std::string g_error;

int fail(int code, const std::string &msg) {
  g_error = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char *what) {
  return fail(e == cudaErrorMemoryAllocation ? PROPAG_ERR_OOM : PROPAG_ERR_CUDA,
              std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(call)                                          \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);   \
  } while (0)

struct DeviceState {
  bool ready = false;
  int sms = 0;
};
std::mutex g_dev_mu;
DeviceState g_dev[64];

// Selects the device (opt device or current), uploads the fuel table once per
// device.  Fails loudly when there is no device: there is no CPU path.
int ensure_device(int want, int *sms_out) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return fail(PROPAG_ERR_NO_DEVICE, "no CUDA device available (libpropag has no CPU path)");
  }
  int dev = want;
  if (dev < 0) CK(cudaGetDevice(&dev));
  if (dev >= count || dev >= 64) return fail(PROPAG_ERR_INVALID, "device ordinal out of range");
  CK(cudaSetDevice(dev));
  std::lock_guard<std::mutex> lk(g_dev_mu);
  DeviceState &d = g_dev[dev];
  if (!d.ready) {
    CK(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev));
    CK(upload_catalog());
    d.ready = true;
  }
  if (sms_out) *sms_out = d.sms;
  return PROPAG_OK;
}

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  // Grows to at least `bytes` (with 1/8 headroom for the next growth unless
  // `exact`).  Growth waits for `stream` first.
  cudaError_t reserve(size_t bytes, cudaStream_t stream, bool exact = false) {
    if (bytes <= cap) return cudaSuccess;
    if (p) {
      cudaError_t e = cudaStreamSynchronize(stream);
      if (e != cudaSuccess) return e;
      cudaFree(p);
      p = nullptr;
      cap = 0;
    }
    const size_t want = exact ? bytes + 256 : bytes + bytes / 8 + 256;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) return e;
    cap = want;
    return cudaSuccess;
  }
  template <typename T>
  T *at(size_t off) const {
    return reinterpret_cast<T *>(static_cast<char *>(p) + off);
  }
};

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Sweeps a job may take before it stops with the sweep-limit status: 2^40
// (no real scenario comes near), or PROPAG_MAX_SWEEPS from the environment
// (used by the tests to make the limit run out).
unsigned long long max_sweeps() {
  const char *v = std::getenv("PROPAG_MAX_SWEEPS");
  if (v && *v) {
    const unsigned long long n = std::strtoull(v, nullptr, 10);
    if (n > 0) return n;
  }
  return 1ull << 40;
}

bool valid_size(uint32_t w, uint32_t h) { return w >= 1 && h >= 1 && w <= 65534 && h <= 65534; }

const char *status_text(uint32_t status) {
  return status == kStatusGroupTimeout ? "a group barrier wait gave up" : "sweep limit reached";
}

}  // namespace
}  // namespace propag

using namespace propag;

// ============================================================ engine ======
struct propag_engine {
  int device = 0;
  int sms = 0;
  int csize = 0;    // 0 = auto, PROPAG_CLUSTER_GROUPS = teams of CTAs without clusters
  bool auto_groups = true;  // auto may choose group mode (needs the whole device)
  uint32_t phantom = 0;     // self-test only: CTAs a group-mode team waits for in vain
  int threads = 512;  // the engine kernel's launch bound
  int default_tile = PROPAG_DEFAULT_TILE;
  size_t smem_budget = 200 * 1024;  // dynamic shared memory per CTA for resident tiles
  int last_cluster = 0;             // cluster size and shared memory of the last run
  uint32_t last_group = 0;          // CTAs per team of the last run (group mode), else 0
  size_t last_smem = 0;
  cudaStream_t stream = nullptr;  // the stream of the last run
  DevBuf job_scratch, slot_scratch, meta;
  JobDev *jobs_pinned = nullptr;
  SlotDev *slots_pinned = nullptr;
  size_t pinned_jobs = 0, pinned_slots = 0;
  cudaEvent_t staged = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // around prep, engine, post
  StatsDev *last_stats = nullptr;  // device statistics of the last run's jobs
};

namespace propag {
// Engines whose runs overlap other engines' runs on the device (the server's
// lanes) keep to clusters: a group-mode launch is cooperative and occupies
// every SM, so its teams would wait for CTAs that other kernels hold.
void engine_keep_to_clusters(propag_engine *e) { e->auto_groups = false; }


// Reserves the engine's device scratch and pinned staging for batches of up
// to max_jobs jobs whose job scratch sums to at most job_bytes, with slot
// scratch of slot_bytes, so that such batches allocate nothing (a later
// larger batch still grows the buffers).
int engine_reserve(propag_engine *e, size_t job_bytes, uint32_t max_jobs, size_t slot_bytes,
                   cudaStream_t stream) {
  CK(cudaSetDevice(e->device));
  CK(e->job_scratch.reserve(job_bytes, stream, true));
  CK(e->slot_scratch.reserve(slot_bytes, stream, true));
  CK(e->meta.reserve(align_up(sizeof(JobDev) * max_jobs, 256) + align_up(sizeof(SlotDev) * max_jobs, 256) +
                         align_up(sizeof(StatsDev) * max_jobs, 256) + 256 +
                         align_up(sizeof(uint32_t) * max_jobs, 256),
                     stream));
  if (e->pinned_jobs < max_jobs) {
    if (e->jobs_pinned) cudaFreeHost(e->jobs_pinned);
    e->jobs_pinned = nullptr;
    CK(cudaMallocHost(&e->jobs_pinned, sizeof(JobDev) * max_jobs + sizeof(uint32_t) * max_jobs));
    e->pinned_jobs = max_jobs;
  }
  if (e->pinned_slots < max_jobs) {
    if (e->slots_pinned) cudaFreeHost(e->slots_pinned);
    e->slots_pinned = nullptr;
    CK(cudaMallocHost(&e->slots_pinned, sizeof(SlotDev) * max_jobs));
    e->pinned_slots = max_jobs;
  }
  return PROPAG_OK;
}
}  // namespace propag

extern "C" uint64_t propag_engine_job_bytes(uint32_t width, uint32_t height) {
  const uint64_t N = (uint64_t)width * height, words = (N + 31) / 32;
  return align_up(N * 4, 256) * 15 + 2 * align_up(words * 4, 256);
}

extern "C" propag_engine *propag_engine_create(const PropagOptions *opt) {
  int sms = 0;
  const int want = opt ? opt->device : -1;
  if (ensure_device(want, &sms) != PROPAG_OK) return nullptr;
  auto *e = new propag_engine();
  cudaGetDevice(&e->device);
  e->sms = sms;
  if (opt) {
    if (opt->cluster < -1024 || opt->cluster > 16) {
      fail(PROPAG_ERR_INVALID, "cluster must be 0..16, PROPAG_CLUSTER_GROUPS or -(team size)");
      delete e;
      return nullptr;
    }
    e->csize = opt->cluster;
    if (opt->threads) {
      if (opt->threads % 32 || opt->threads > 512) {
        fail(PROPAG_ERR_INVALID, "threads must be a multiple of 32, <= 512");
        delete e;
        return nullptr;
      }
      e->threads = opt->threads;
    }
    if (opt->tile) e->default_tile = opt->tile;
  }
  bool ok = cudaEventCreateWithFlags(&e->staged, cudaEventDisableTiming) == cudaSuccess;
  for (int i = 0; i < 4; ++i) ok = ok && cudaEventCreate(&e->ev[i]) == cudaSuccess;
  if (!ok) {
    fail(PROPAG_ERR_CUDA, "cudaEventCreate failed");
    delete e;
    return nullptr;
  }
  return e;
}

extern "C" void propag_engine_destroy(propag_engine *e) {
  if (!e) return;
  cudaSetDevice(e->device);
  if (e->staged) {
    cudaEventSynchronize(e->staged);
    cudaEventDestroy(e->staged);
  }
  for (int i = 0; i < 4; ++i)
    if (e->ev[i]) cudaEventDestroy(e->ev[i]);
  if (e->jobs_pinned) cudaFreeHost(e->jobs_pinned);
  if (e->slots_pinned) cudaFreeHost(e->slots_pinned);
  delete e;
  cudaGetLastError();  // leave no error of the teardown to the caller's next CUDA call
}

static int engine_run(propag_engine *e, const PropagJob *jobs, uint32_t n_jobs, cudaStream_t stream,
                      PropagStats *stats) {
  if (!e) return fail(PROPAG_ERR_INVALID, "null engine");
  if (n_jobs == 0) return PROPAG_OK;
  if (!jobs) return fail(PROPAG_ERR_INVALID, "null jobs");
  CK(cudaSetDevice(e->device));
  // ---- validate and lay out per-job scratch ----
  std::vector<JobDev> jd(n_jobs);
  std::vector<size_t> off(n_jobs);
  std::vector<int> tw(n_jobs), th(n_jobs);
  size_t job_bytes = 0;
  uint64_t max_cells = 1;
  for (uint32_t i = 0; i < n_jobs; ++i) {
    const PropagJob &j = jobs[i];
    if (!valid_size(j.width, j.height))
      return fail(PROPAG_ERR_INVALID, "job " + std::to_string(i) + ": width/height must be 1..65534");
    if (!j.speed_max || !j.azimuth_max || !j.eccentricity || !j.time)
      return fail(PROPAG_ERR_INVALID, "job " + std::to_string(i) + ": null fire/time pointer");
    if (j.n_ignitions && !j.ignitions)
      return fail(PROPAG_ERR_INVALID, "job " + std::to_string(i) + ": null ignitions");
    if (!(j.dx != 0.0f) || !(j.dy != 0.0f) || !std::isfinite(j.dx) || !std::isfinite(j.dy))
      return fail(PROPAG_ERR_INVALID, "job " + std::to_string(i) + ": invalid pixel size");
    if (j.arith != PROPAG_ARITH_REFERENCE && j.arith != PROPAG_ARITH_PORTABLE)
      return fail(PROPAG_ERR_INVALID, "job " + std::to_string(i) + ": arith must be PROPAG_ARITH_REFERENCE or PROPAG_ARITH_PORTABLE");
    const uint64_t N = (uint64_t)j.width * j.height;
    const uint64_t words = (N + 31) / 32;
    int T = j.tile ? j.tile : e->default_tile;
    if (T == PROPAG_TILE_WHOLE_GRID || T <= 0) T = (int)std::max(j.width, j.height);
    JobDev &d = jd[i];
    d.W = (int)j.width;
    d.H = (int)j.height;
    d.gdx = j.dx;
    d.gdy = j.dy;
    d.max_time = j.max_time;
    d.T = T;
    d.TX = (int)((j.width + T - 1) / T);
    d.TY = (int)((j.height + T - 1) / T);
    d.north_up = j.dy < 0 ? 1 : 0;
    d.refm = j.arith == PROPAG_ARITH_REFERENCE ? 1 : 0;
    d.speed = j.speed_max;
    d.az = j.azimuth_max;
    d.ecc = j.eccentricity;
    d.time = j.time;
    d.ignitions = j.ignitions;
    d.n_ignitions = j.n_ignitions;
    d.out_rx = j.refs_x;
    d.out_ry = j.refs_y;
    d.out_bnd = j.boundaries;
    tw[i] = std::min<int>(T, (int)j.width);
    th[i] = std::min<int>(T, (int)j.height);
    off[i] = job_bytes;
    // references, referrer boxes, boundary bits, 8 travel-time planes, the
    // second state copy (time, references) and the pending bitmap of
    // global-memory tiles
    job_bytes += align_up(N * 4, 256) * 15 + (j.boundaries ? 0 : align_up(words * 4, 256)) +
                 align_up(words * 4, 256);
    max_cells = std::max<uint64_t>(max_cells, N);
  }
  CK(e->job_scratch.reserve(job_bytes, stream));
  for (uint32_t i = 0; i < n_jobs; ++i) {
    const uint64_t N = (uint64_t)jd[i].W * jd[i].H;
    size_t o = off[i];
    uint32_t *arr[5];
    for (int k = 0; k < 5; ++k) {
      arr[k] = e->job_scratch.at<uint32_t>(o);
      o += align_up(N * 4, 256);
    }
    jd[i].refs = arr[0];
    jd[i].box_x0 = arr[1];
    jd[i].box_y0 = arr[2];
    jd[i].box_x1 = arr[3];
    jd[i].box_y1 = arr[4];
    jd[i].bnd = jobs[i].boundaries ? jobs[i].boundaries : e->job_scratch.at<uint32_t>(o);
    if (!jobs[i].boundaries) o += align_up(((N + 31) / 32) * 4, 256);
    jd[i].tt = e->job_scratch.at<float>(o);
    jd[i].tt_plane = (int64_t)(align_up(N * 4, 256) / 4);
    o += 8 * align_up(N * 4, 256);
    jd[i].time1 = e->job_scratch.at<float>(o);
    o += align_up(N * 4, 256);
    jd[i].refs1 = e->job_scratch.at<uint32_t>(o);
    o += align_up(N * 4, 256);
    jd[i].pending = e->job_scratch.at<uint32_t>(o);  // kept below for global-memory tiles only
  }
  // ---- cluster size and tile residency ----
  // A tile launch runs in the cluster's shared memory when the tile and its
  // halo fit in the dynamic shared-memory budget of the cluster's CTAs.
  const size_t budget = e->smem_budget;
  auto fits = [&](uint32_t i, int c) { return smem_bytes(tw[i], th[i], c) <= budget; };
  int csize = e->csize;
  if (csize == 0 && e->auto_groups) {
    // Group mode, one team per job of max(4, CTAs / jobs) CTAs.  A scenario
    // runs on one cluster at most in cluster mode (its tiles go one after
    // another), so few scenarios leave most SMs idle, while a group-mode team
    // spreads each sweep over its CTAs with one barrier per sweep.  Measured
    // on B200, 1024^2 ensemble members: 1 member 79 ms in group mode against
    // 120 ms on a 16-CTA cluster; 64 members 408 ms (teams of 8) against
    // 514 (8-CTA clusters); 256 members 1 082 ms (teams of 4) against 1 531.
    int ctas = 0;
    CK(engine_max_clusters(1, e->threads, global_tile_smem(e->threads), &ctas));
    if (ctas >= 8) csize = -std::max(4, ctas / (int)std::max<uint32_t>(n_jobs, 1));
  }
  if (csize == 0) {
    // among the cluster sizes that hold every job's tile, the one that runs
    // the most jobs at once (resident clusters, up to the job count); ties go
    // to the larger cluster, which finishes each job sooner.  When some tile
    // never fits, as many clusters as there are jobs, as large as the
    // machine allows.
    uint32_t best_conc = 0;
    for (int c = 16; c >= 1; c /= 2) {
      bool all = true;
      size_t need = 0;
      for (uint32_t i = 0; i < n_jobs && all; ++i) {
        all = fits(i, c);
        need = std::max(need, smem_bytes(tw[i], th[i], c));
      }
      if (!all) continue;
      int mc = 0;
      CK(engine_max_clusters(c, e->threads, need, &mc));
      const uint32_t conc = std::min<uint32_t>(n_jobs, (uint32_t)std::max(mc, 0));
      if (conc > best_conc) {
        best_conc = conc;
        csize = c;
      }
    }
    if (csize == 0) {
      int ctas = 0;
      CK(engine_max_clusters(1, e->threads, 0, &ctas));
      csize = 1;
      while (csize < 16 && (uint64_t)(csize * 2) * n_jobs <= (uint64_t)std::max(ctas, 1)) csize *= 2;
    }
  }
  size_t smem = 0, tn_max = 1, ovf_cap = 0;
  uint32_t n_slots = 0, group = 0;
  if (csize <= PROPAG_CLUSTER_GROUPS) {
    // group mode: the co-resident CTAs split into teams of at least 32 CTAs
    // (or of -csize CTAs when given), one team per job up to that, tiles in
    // global memory
    smem = global_tile_smem(e->threads);
    int ctas = 0;
    CK(engine_max_clusters(1, e->threads, smem, &ctas));
    if (ctas < 2) return fail(PROPAG_ERR_CUDA, "group mode needs at least 2 resident CTAs");
    const int team = csize == PROPAG_CLUSTER_GROUPS ? 32 : std::max(2, -csize);
    n_slots = std::min<uint32_t>(n_jobs, (uint32_t)std::max(1, ctas / team));
    group = (uint32_t)ctas / n_slots;
    for (uint32_t i = 0; i < n_jobs; ++i) {
      jd[i].smem_tile = kSmemTileGlobal;
      tn_max = std::max<size_t>(tn_max, (size_t)tw[i] * (size_t)th[i]);
    }
    csize = 1;
  } else {
    for (uint32_t i = 0; i < n_jobs; ++i) {
      // exact referrer boxes when they fit, else the coarse ones
      const bool exact = smem_bytes(tw[i], th[i], csize, true) <= budget;
      jd[i].smem_tile = exact ? kSmemTileExact : fits(i, csize) ? kSmemTileCoarse : kSmemTileGlobal;
      if (jd[i].smem_tile != kSmemTileGlobal) {
        smem = std::max(smem, smem_bytes(tw[i], th[i], csize, exact));
        ovf_cap = std::max<size_t>(ovf_cap, (size_t)smem_cap(tw[i], th[i], csize));
      } else {
        tn_max = std::max<size_t>(tn_max, (size_t)tw[i] * (size_t)th[i]);
        smem = std::max(smem, global_tile_smem(e->threads));
      }
    }
    int max_clusters = 0;
    CK(engine_max_clusters(csize, e->threads, smem, &max_clusters));
    if (max_clusters < 1) return fail(PROPAG_ERR_CUDA, "cluster size " + std::to_string(csize) + " cannot be resident");
    n_slots = std::min<uint32_t>(n_jobs, (uint32_t)max_clusters);
  }
  // First sweeps skip unchanged cells (pending bitmap) on global-memory tiles
  // of grids below 2^27 cells (a warp sums 32 referrer-box areas in 32 bits);
  // shared-memory tiles evaluate the whole tile in a launch's first sweep.
  for (uint32_t i = 0; i < n_jobs; ++i)
    if (jd[i].smem_tile != kSmemTileGlobal || (uint64_t)jd[i].W * jd[i].H >= (1ull << 27))
      jd[i].pending = nullptr;
  e->last_cluster = group ? PROPAG_CLUSTER_GROUPS : csize;
  e->last_group = group;
  e->last_smem = smem;
  const size_t words_max = tn_max / 32 + 1;
  // global-memory tiles: each CTA of a team has its own update region
  const size_t team_ctas = group ? group : (size_t)csize;
  const size_t upd_max = tn_max + 32 * (team_ctas + 1);
  const size_t ovf_list_bytes = align_up((size_t)csize * ovf_cap * 2, 256);
  const size_t ovf_upd_bytes = align_up((size_t)csize * ovf_cap * sizeof(Update), 256);
  // three dirty bitmaps (in rotation) and two update arrays (by sweep parity)
  const size_t slot_bytes = 3 * align_up(words_max * 4, 256) + 2 * align_up(upd_max * sizeof(TileUpdate), 256) +
                            256 + ovf_list_bytes + ovf_upd_bytes;
  CK(e->slot_scratch.reserve(slot_bytes * n_slots, stream));
  // meta: jobs, slots, stats, queue
  const size_t meta_jobs = align_up(sizeof(JobDev) * n_jobs, 256);
  const size_t meta_slots = align_up(sizeof(SlotDev) * n_slots, 256);
  const size_t meta_stats = align_up(sizeof(StatsDev) * n_jobs, 256);
  const size_t meta_order = align_up(sizeof(uint32_t) * n_jobs, 256);
  CK(e->meta.reserve(meta_jobs + meta_slots + meta_stats + 256 + meta_order, stream));
  // staging buffers (pinned) may still be read by the previous run's copies
  // (a run being captured into a graph follows a completed uncaptured run)
  cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(stream, &capturing));
  if (capturing == cudaStreamCaptureStatusNone) CK(cudaEventSynchronize(e->staged));
  if (e->pinned_jobs < n_jobs) {
    if (e->jobs_pinned) cudaFreeHost(e->jobs_pinned);
    // the job descriptors, then the queue order
    CK(cudaMallocHost(&e->jobs_pinned, sizeof(JobDev) * n_jobs + sizeof(uint32_t) * n_jobs));
    e->pinned_jobs = n_jobs;
  }
  if (e->pinned_slots < n_slots) {
    if (e->slots_pinned) cudaFreeHost(e->slots_pinned);
    CK(cudaMallocHost(&e->slots_pinned, sizeof(SlotDev) * n_slots));
    e->pinned_slots = n_slots;
  }
  std::copy(jd.begin(), jd.end(), e->jobs_pinned);
  // queue order: largest grids first, so that the longest jobs start first
  // and the batch ends close to its longest job (results do not depend on it)
  uint32_t *order_pinned = reinterpret_cast<uint32_t *>(e->jobs_pinned + n_jobs);
  for (uint32_t i = 0; i < n_jobs; ++i) order_pinned[i] = i;
  std::stable_sort(order_pinned, order_pinned + n_jobs, [&](uint32_t a, uint32_t b) {
    return (uint64_t)jd[a].W * jd[a].H > (uint64_t)jd[b].W * jd[b].H;
  });
  for (uint32_t s = 0; s < n_slots; ++s) {
    size_t o = slot_bytes * s;
    SlotDev &sd = e->slots_pinned[s];
    sd.dirty = e->slot_scratch.at<uint32_t>(o);
    sd.dirty_words = (uint32_t)(align_up(words_max * 4, 256) / 4);
    sd.pad0 = 0;
    o += 3 * align_up(words_max * 4, 256);
    sd.upd = e->slot_scratch.at<TileUpdate>(o);
    o += 2 * align_up(upd_max * sizeof(TileUpdate), 256);
    sd.ctr = e->slot_scratch.at<uint32_t>(o);
    o += 256;
    sd.ovf_list = e->slot_scratch.at<uint16_t>(o);
    o += ovf_list_bytes;
    sd.ovf_upd = e->slot_scratch.at<Update>(o);
    sd.ovf_cap = (uint32_t)ovf_cap;
    sd.pad = 0;
    // the dirty bitmap and counters must start cleared
    CK(cudaMemsetAsync(sd.dirty, 0, 3 * align_up(words_max * 4, 256), stream));
    CK(cudaMemsetAsync(sd.ctr, 0, 64, stream));  // counters and barrier arrivals
  }
  JobDev *d_jobs = e->meta.at<JobDev>(0);
  SlotDev *d_slots = e->meta.at<SlotDev>(meta_jobs);
  StatsDev *d_stats = e->meta.at<StatsDev>(meta_jobs + meta_slots);
  uint32_t *d_queue = e->meta.at<uint32_t>(meta_jobs + meta_slots + meta_stats);
  uint32_t *d_order = e->meta.at<uint32_t>(meta_jobs + meta_slots + meta_stats + 256);
  e->last_stats = d_stats;
  CK(cudaMemcpyAsync(d_jobs, e->jobs_pinned, sizeof(JobDev) * n_jobs, cudaMemcpyHostToDevice, stream));
  CK(cudaMemcpyAsync(d_order, order_pinned, sizeof(uint32_t) * n_jobs, cudaMemcpyHostToDevice, stream));
  CK(cudaMemcpyAsync(d_slots, e->slots_pinned, sizeof(SlotDev) * n_slots, cudaMemcpyHostToDevice, stream));
  // the engine's events time uncaptured runs only (an event recorded into a
  // graph cannot be waited on or timed from the host)
  const bool live = capturing == cudaStreamCaptureStatusNone;
  if (live) CK(cudaEventRecord(e->staged, stream));
  CK(cudaMemsetAsync(d_stats, 0, sizeof(StatsDev) * n_jobs, stream));
  CK(cudaMemsetAsync(d_queue, 0, 8, stream));  // queue position, group error flag
  // ---- kernels ----
  if (live) CK(cudaEventRecord(e->ev[0], stream));
  CK(launch_prep(d_jobs, n_jobs, max_cells, e->sms, stream));
  CK(launch_ignite(d_jobs, n_jobs, stream));
  if (live) CK(cudaEventRecord(e->ev[1], stream));
  CK(launch_engine(d_jobs, n_jobs, d_slots, n_slots, csize, e->threads, smem, d_queue, d_stats,
                   max_sweeps(), d_order, group, group ? e->phantom : 0u, stream));
  if (live) CK(cudaEventRecord(e->ev[2], stream));
  CK(launch_post(d_jobs, n_jobs, max_cells, e->sms, d_stats, stream));
  if (live) CK(cudaEventRecord(e->ev[3], stream));
  e->stream = stream;
  if (stats) {
    std::vector<StatsDev> hs(n_jobs);
    CK(cudaMemcpyAsync(hs.data(), d_stats, sizeof(StatsDev) * n_jobs, cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    for (uint32_t i = 0; i < n_jobs; ++i) {
      PropagStats &o = stats[i];
      o.rounds = hs[i].rounds;
      o.launches = hs[i].launches;
      o.sweeps = hs[i].sweeps;
      o.evaluations = hs[i].evaluations;
      o.improvements = hs[i].improvements;
      o.dda_steps = hs[i].dda_steps;
      o.gathers = hs[i].gathers;
      o.refbox_scans = hs[i].refbox_scans;
      o.burned = hs[i].burned;
      o.cyc_first = hs[i].cyc_first;
      o.cyc_eval = hs[i].cyc_eval;
      o.cyc_commit = hs[i].cyc_commit;
      o.cyc_stage = hs[i].cyc_stage;
      o.status = hs[i].status;
      o.max_walk = hs[i].max_walk;
      o.t_start_ns = hs[i].t_start_ns;
      o.t_done_ns = hs[i].t_done_ns;
      o.scan_cells = hs[i].scan_cells;
      o.cyc_wait = hs[i].cyc_wait;
    }
    for (uint32_t i = 0; i < n_jobs; ++i)
      if (hs[i].status) return fail(PROPAG_ERR_TIMEOUT, "job " + std::to_string(i) + ": " + status_text(hs[i].status));
  }
  return PROPAG_OK;
}

extern "C" int propag_engine_run(propag_engine *e, const PropagJob *jobs, uint32_t n_jobs,
                                 void *stream, PropagStats *stats) {
  return engine_run(e, jobs, n_jobs, (cudaStream_t)stream, stats);
}

extern "C" int propag_selftest_group_wait(uint32_t *status) {
  if (!status) return fail(PROPAG_ERR_INVALID, "null status");
  *status = 0;
  int sms = 0;
  const int rc0 = ensure_device(-1, &sms);  // no device: PROPAG_ERR_NO_DEVICE
  if (rc0) return rc0;
  PropagOptions o{0, PROPAG_CLUSTER_GROUPS, 0, -1};
  propag_engine *e = propag_engine_create(&o);
  if (!e) return PROPAG_ERR_CUDA;  // message set by propag_engine_create
  e->phantom = 1;
  const uint32_t W = 8, H = 8, N = W * H;
  DevBuf buf;
  int rc = PROPAG_OK;
  if (buf.reserve(N * 4 * 4 + N * 2 * 2 + 256, nullptr) != cudaSuccess ||
      cudaMemset(buf.at<char>(0), 0, N * 4 * 4 + N * 2 * 2 + 256) != cudaSuccess) {
    rc = fail(PROPAG_ERR_CUDA, "self-test buffers");
  } else {
    PropagJob j{};
    j.width = W;
    j.height = H;
    j.dx = 5.0;
    j.dy = 5.0;
    j.max_time = 100.0f;
    j.speed_max = buf.at<float>(0);
    j.azimuth_max = buf.at<float>(N * 4);
    j.eccentricity = buf.at<float>(N * 8);
    j.time = buf.at<float>(N * 12);
    j.refs_x = buf.at<uint16_t>(N * 16);
    j.refs_y = buf.at<uint16_t>(N * 18);
    PropagStats st{};
    rc = engine_run(e, &j, 1, nullptr, &st);
    *status = st.status;
  }
  propag_engine_destroy(e);
  return rc;
}

extern "C" int propag_engine_last_times(propag_engine *e, float ms[3]) {
  if (!e || !ms) return fail(PROPAG_ERR_INVALID, "null argument");
  CK(cudaSetDevice(e->device));
  CK(cudaEventSynchronize(e->ev[3]));
  for (int i = 0; i < 3; ++i) CK(cudaEventElapsedTime(&ms[i], e->ev[i], e->ev[i + 1]));
  return PROPAG_OK;
}

// ================================================ batches as CUDA graphs ==
static int fire_device(bool full, uint64_t n, const PropagTerrainPtrs *t, float *const outs[10],
                       cudaStream_t stream);

// The fire passes of the jobs that have a terrain, then the batch's
// propagation (prep, ignition, engine, post), on one stream.
static int batch_step(propag_engine *e, const PropagJob *jobs, const PropagTerrainPtrs *terrains,
                      uint32_t n_jobs, cudaStream_t stream, PropagStats *stats) {
  if (terrains) {
    for (uint32_t i = 0; i < n_jobs; ++i) {
      float *outs[10] = {nullptr, nullptr, nullptr, nullptr,
                         const_cast<float *>(jobs[i].speed_max), const_cast<float *>(jobs[i].azimuth_max),
                         const_cast<float *>(jobs[i].eccentricity), nullptr, nullptr, nullptr};
      const int rc = fire_device(false, (uint64_t)jobs[i].width * jobs[i].height, terrains + i, outs, stream);
      if (rc) return rc;
    }
  }
  return engine_run(e, jobs, n_jobs, stream, stats);
}

struct propag_graph {
  propag_engine *eng = nullptr;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint32_t n_jobs = 0;
};

extern "C" void propag_graph_destroy(propag_graph *g) {
  if (!g) return;
  if (g->eng) cudaSetDevice(g->eng->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  if (g->stream) cudaStreamDestroy(g->stream);
  propag_engine_destroy(g->eng);
  delete g;
  cudaGetLastError();  // leave no error of the teardown to the caller's next CUDA call
}

extern "C" propag_graph *propag_graph_create(const PropagOptions *opt, const PropagJob *jobs,
                                             const PropagTerrainPtrs *terrains, uint32_t n_jobs) {
  if (!jobs || n_jobs == 0) {
    fail(PROPAG_ERR_INVALID, "propag_graph_create: no jobs");
    return nullptr;
  }
  auto *g = new propag_graph();
  g->n_jobs = n_jobs;
  g->eng = propag_engine_create(opt);
  if (!g->eng) {
    delete g;
    return nullptr;
  }
  auto bail = [&](cudaError_t err, const char *what) -> propag_graph * {
    if (err != cudaSuccess) cuda_fail(err, what);
    propag_graph_destroy(g);
    return nullptr;
  };
  cudaError_t err = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
  if (err != cudaSuccess) return bail(err, "cudaStreamCreateWithFlags");
  // an uncaptured run first: it sizes and allocates the engine's scratch, so
  // that the captured run allocates nothing (and checks the jobs)
  if (batch_step(g->eng, jobs, terrains, n_jobs, g->stream, nullptr)) return bail(cudaSuccess, "");
  err = cudaStreamSynchronize(g->stream);
  if (err != cudaSuccess) return bail(err, "cudaStreamSynchronize");
  err = cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal);
  if (err != cudaSuccess) return bail(err, "cudaStreamBeginCapture");
  const int rc = batch_step(g->eng, jobs, terrains, n_jobs, g->stream, nullptr);
  const std::string msg = rc ? g_error : std::string();
  err = cudaStreamEndCapture(g->stream, &g->graph);
  if (rc) {
    g_error = msg;
    return bail(cudaSuccess, "");
  }
  if (err != cudaSuccess) return bail(err, "cudaStreamEndCapture");
  err = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (err != cudaSuccess) return bail(err, "cudaGraphInstantiate");
  return g;
}

extern "C" int propag_graph_launch(propag_graph *g, void *stream) {
  if (!g || !g->exec) return fail(PROPAG_ERR_INVALID, "null graph");
  CK(cudaSetDevice(g->eng->device));
  CK(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
  return PROPAG_OK;
}

static void to_stats(const StatsDev &h, PropagStats &o) {
  o.rounds = h.rounds;
  o.launches = h.launches;
  o.sweeps = h.sweeps;
  o.evaluations = h.evaluations;
  o.improvements = h.improvements;
  o.dda_steps = h.dda_steps;
  o.gathers = h.gathers;
  o.refbox_scans = h.refbox_scans;
  o.burned = h.burned;
  o.cyc_first = h.cyc_first;
  o.cyc_eval = h.cyc_eval;
  o.cyc_commit = h.cyc_commit;
  o.cyc_stage = h.cyc_stage;
  o.status = h.status;
  o.max_walk = h.max_walk;
  o.t_start_ns = h.t_start_ns;
  o.t_done_ns = h.t_done_ns;
  o.scan_cells = h.scan_cells;
  o.cyc_wait = h.cyc_wait;
}

extern "C" int propag_engine_last_stats(propag_engine *e, void *stream, PropagStats *stats,
                                        uint32_t n_jobs) {
  if (!e || !stats) return fail(PROPAG_ERR_INVALID, "null argument");
  if (!e->last_stats) return fail(PROPAG_ERR_INVALID, "the engine has not run");
  CK(cudaSetDevice(e->device));
  std::vector<StatsDev> hs(n_jobs);
  CK(cudaMemcpyAsync(hs.data(), e->last_stats, sizeof(StatsDev) * n_jobs, cudaMemcpyDeviceToHost,
                     (cudaStream_t)stream));
  CK(cudaStreamSynchronize((cudaStream_t)stream));
  for (uint32_t i = 0; i < n_jobs; ++i) to_stats(hs[i], stats[i]);
  return PROPAG_OK;
}

extern "C" int propag_graph_stats(propag_graph *g, void *stream, PropagStats *stats) {
  if (!g || !stats) return fail(PROPAG_ERR_INVALID, "null argument");
  propag_engine *e = g->eng;
  if (!e->last_stats) return fail(PROPAG_ERR_INVALID, "the graph has not run");
  CK(cudaSetDevice(e->device));
  std::vector<StatsDev> hs(g->n_jobs);
  CK(cudaMemcpyAsync(hs.data(), e->last_stats, sizeof(StatsDev) * g->n_jobs, cudaMemcpyDeviceToHost,
                     (cudaStream_t)stream));
  CK(cudaStreamSynchronize((cudaStream_t)stream));
  for (uint32_t i = 0; i < g->n_jobs; ++i) to_stats(hs[i], stats[i]);
  for (uint32_t i = 0; i < g->n_jobs; ++i)
    if (hs[i].status) return fail(PROPAG_ERR_TIMEOUT, "job " + std::to_string(i) + ": " + status_text(hs[i].status));
  return PROPAG_OK;
}

// ============================================================ autotuner ===
extern "C" int propag_autotune(const PropagJob *jobs, const PropagTerrainPtrs *terrains,
                               uint32_t n_jobs, void *stream_ptr, int repeats, PropagOptions *best,
                               float *best_ms) {
  if (!jobs || n_jobs == 0 || !best) return fail(PROPAG_ERR_INVALID, "propag_autotune: no jobs or output");
  int sms = 0;
  int rc = ensure_device(-1, &sms);
  if (rc) return rc;
  cudaStream_t stream = (cudaStream_t)stream_ptr;
  repeats = std::max(repeats, 1);
  // candidates: cluster sizes whose shared memory holds every job's tile
  std::vector<int> cands;
  for (int c = 16; c >= 1; c /= 2) {
    bool all = true;
    for (uint32_t i = 0; i < n_jobs && all; ++i) {
      int T = jobs[i].tile ? jobs[i].tile : PROPAG_DEFAULT_TILE;
      if (T == PROPAG_TILE_WHOLE_GRID || T <= 0) T = (int)std::max(jobs[i].width, jobs[i].height);
      all = smem_bytes(std::min<int>(T, (int)jobs[i].width), std::min<int>(T, (int)jobs[i].height), c) <=
            200 * 1024;
    }
    if (all) cands.push_back(c);
  }
  if (cands.empty()) cands.push_back(16);  // global-memory tiles: the largest cluster
  // group mode: the automatic team size and teams of 24, 16, 8 and 4 CTAs
  // (64 uneven scenarios on B200: 350 ms with teams of 24, 373 with 16,
  // 493 with 32)
  cands.push_back(0);
  for (int t : {24, 16, 8, 4})
    if ((uint32_t)t * n_jobs > (uint32_t)sms) cands.push_back(-t);  // else the automatic one
  cudaEvent_t a = nullptr, b = nullptr;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  float best_t = -1.0f;
  for (int c : cands) {
    PropagOptions o{0, c, 0, -1};
    propag_engine *e = propag_engine_create(&o);
    if (!e) {
      rc = PROPAG_ERR_CUDA;
      break;
    }
    rc = batch_step(e, jobs, terrains, n_jobs, stream, nullptr);  // warm-up, allocations
    float t_min = -1.0f;
    for (int r = 0; r < repeats && !rc; ++r) {
      cudaEventRecord(a, stream);
      rc = batch_step(e, jobs, terrains, n_jobs, stream, nullptr);
      cudaEventRecord(b, stream);
      float ms = 0.0f;
      if (!rc && cudaEventSynchronize(b) == cudaSuccess && cudaEventElapsedTime(&ms, a, b) == cudaSuccess)
        t_min = t_min < 0 ? ms : std::min(t_min, ms);
    }
    propag_engine_destroy(e);
    if (rc) break;
    if (t_min >= 0 && (best_t < 0 || t_min < best_t)) {
      best_t = t_min;
      *best = o;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc) return rc;
  if (best_t < 0) return fail(PROPAG_ERR_CUDA, "propag_autotune: no candidate could be timed");
  if (best_ms) *best_ms = best_t;
  return PROPAG_OK;
}

// ============================================= allocation-free variant ====
// One job, the same kernels as engine_run, scratch in the fixed device array
// of noalloc.cu.  No cudaMalloc/cudaFree/cudaMallocHost, no events, no host
// heap on the success path.
namespace propag {
int engine_threads();  // engine.cu: the engine kernel's launch bound
}
static_assert(PROPAG_STATIC_MAX_CELLS == kStaticMaxCells, "header and scratch disagree");
namespace {
// Device address of the fixed scratch per device ordinal, taken once per
// device.  It belongs to the device's primary context: after a
// cudaDeviceReset the process must not call the allocation-free entry
// points on that device again.
constexpr int kStaticDevices = 64;
std::mutex g_static_mu;
void *g_static_base[kStaticDevices] = {};

void copy_stats(const StatsDev &h, PropagStats &o) {
  o.rounds = h.rounds;
  o.launches = h.launches;
  o.sweeps = h.sweeps;
  o.evaluations = h.evaluations;
  o.improvements = h.improvements;
  o.dda_steps = h.dda_steps;
  o.gathers = h.gathers;
  o.refbox_scans = h.refbox_scans;
  o.burned = h.burned;
  o.cyc_first = h.cyc_first;
  o.cyc_eval = h.cyc_eval;
  o.cyc_commit = h.cyc_commit;
  o.cyc_stage = h.cyc_stage;
  o.status = h.status;
  o.max_walk = h.max_walk;
  o.t_start_ns = h.t_start_ns;
  o.t_done_ns = h.t_done_ns;
  o.scan_cells = h.scan_cells;
  o.cyc_wait = h.cyc_wait;
}
}  // namespace

extern "C" int propag_run_device_static(const PropagJob *job, void *stream_ptr, PropagStats *stats) {
  int sms = 0;
  int rc = ensure_device(-1, &sms);
  if (rc) return rc;
  if (!job) return fail(PROPAG_ERR_INVALID, "null job");
  const PropagJob &j = *job;
  if (!valid_size(j.width, j.height)) return fail(PROPAG_ERR_INVALID, "width/height must be 1..65534");
  const uint64_t N = (uint64_t)j.width * j.height;
  if (N > kStaticMaxCells)
    return fail(PROPAG_ERR_INVALID,
                "propag_run_device_static: grid of " + std::to_string(N) + " cells exceeds its fixed scratch of " +
                    std::to_string(kStaticMaxCells) + " cells (use propag_engine_run)");
  if (!j.speed_max || !j.azimuth_max || !j.eccentricity || !j.time)
    return fail(PROPAG_ERR_INVALID, "null fire/time pointer");
  if (j.n_ignitions && !j.ignitions) return fail(PROPAG_ERR_INVALID, "null ignitions");
  if (!(j.dx != 0.0f) || !(j.dy != 0.0f) || !std::isfinite(j.dx) || !std::isfinite(j.dy))
    return fail(PROPAG_ERR_INVALID, "invalid pixel size");
  if (j.arith != PROPAG_ARITH_REFERENCE && j.arith != PROPAG_ARITH_PORTABLE)
    return fail(PROPAG_ERR_INVALID, "arith must be PROPAG_ARITH_REFERENCE or PROPAG_ARITH_PORTABLE");
  int T = j.tile ? j.tile : PROPAG_DEFAULT_TILE;
  if (T == PROPAG_TILE_WHOLE_GRID || T <= 0) T = (int)std::max(j.width, j.height);
  const int tw = std::min<int>(T, (int)j.width), th = std::min<int>(T, (int)j.height);
  // one job: the largest cluster (16 CTAs), which finishes it soonest
  const size_t budget = 200 * 1024;
  const int csize = 16;
  if (smem_bytes(tw, th, csize) > budget ||
      (size_t)csize * (size_t)smem_cap(tw, th, csize) > kStaticOvfSlots)
    return fail(PROPAG_ERR_INVALID,
                "propag_run_device_static: a " + std::to_string(tw) + " x " + std::to_string(th) +
                    " tile does not fit in a 16-CTA cluster's shared memory (use a tile side <= 323 or "
                    "propag_engine_run)");
  const bool exact = smem_bytes(tw, th, csize, true) <= budget;
  const size_t smem = smem_bytes(tw, th, csize, exact);
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kStaticDevices) return fail(PROPAG_ERR_INVALID, "device ordinal out of range");
  char *base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_static_mu);
    if (!g_static_base[dev]) {  // set-up, once per device
      void *p = nullptr;
      CK(static_scratch_address(&p));
      g_static_base[dev] = p;
    }
    base = static_cast<char *>(g_static_base[dev]);
  }
  int max_clusters = 0;
  CK(engine_max_clusters(csize, engine_threads(), smem, &max_clusters));
  if (max_clusters < 1) return fail(PROPAG_ERR_CUDA, "cluster size " + std::to_string(csize) + " cannot be resident");
  JobDev d{};
  d.W = (int)j.width;
  d.H = (int)j.height;
  d.gdx = j.dx;
  d.gdy = j.dy;
  d.max_time = j.max_time;
  d.T = T;
  d.TX = (int)((j.width + T - 1) / T);
  d.TY = (int)((j.height + T - 1) / T);
  d.north_up = j.dy < 0 ? 1 : 0;
  d.refm = j.arith == PROPAG_ARITH_REFERENCE ? 1 : 0;
  d.smem_tile = exact ? kSmemTileExact : kSmemTileCoarse;
  d.speed = j.speed_max;
  d.az = j.azimuth_max;
  d.ecc = j.eccentricity;
  d.time = j.time;
  d.ignitions = j.ignitions;
  d.n_ignitions = j.n_ignitions;
  d.out_rx = j.refs_x;
  d.out_ry = j.refs_y;
  d.out_bnd = j.boundaries;
  uint32_t *cells = reinterpret_cast<uint32_t *>(base + kStaticCellsOff);
  d.refs = cells;
  d.box_x0 = cells + kStaticMaxCells;
  d.box_y0 = cells + 2 * kStaticMaxCells;
  d.box_x1 = cells + 3 * kStaticMaxCells;
  d.box_y1 = cells + 4 * kStaticMaxCells;
  d.bnd = j.boundaries ? j.boundaries : reinterpret_cast<uint32_t *>(base + kStaticBndOff);
  SlotDev s{};  // shared-memory tiles use the counters and the list overflow
  s.ctr = reinterpret_cast<uint32_t *>(base + kStaticCtrOff);
  s.ovf_list = reinterpret_cast<uint16_t *>(base + kStaticOvfListOff);
  s.ovf_upd = reinterpret_cast<Update *>(base + kStaticOvfUpdOff);
  s.ovf_cap = (uint32_t)smem_cap(tw, th, csize);
  JobDev *d_job = reinterpret_cast<JobDev *>(base + kStaticJobOff);
  SlotDev *d_slot = reinterpret_cast<SlotDev *>(base + kStaticSlotOff);
  StatsDev *d_stats = reinterpret_cast<StatsDev *>(base + kStaticStatsOff);
  uint32_t *d_queue = reinterpret_cast<uint32_t *>(base + kStaticQueueOff);
  cudaStream_t stream = (cudaStream_t)stream_ptr;
  CK(launch_stage_static(d_job, d, d_slot, s, d_stats, d_queue, stream));
  CK(launch_prep(d_job, 1, N, sms, stream));
  CK(launch_ignite(d_job, 1, stream));
  CK(launch_engine(d_job, 1, d_slot, 1, csize, engine_threads(), smem, d_queue, d_stats, max_sweeps(),
                   nullptr, 0u, 0u, stream));
  CK(launch_post(d_job, 1, N, sms, d_stats, stream));
  if (stats) {
    StatsDev h;
    CK(cudaMemcpyAsync(&h, d_stats, sizeof(h), cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
    copy_stats(h, *stats);
    if (h.status) return fail(PROPAG_ERR_TIMEOUT, status_text(h.status));
  }
  return PROPAG_OK;
}

extern "C" int propag_static_last_status(void *stream_ptr, PropagStats *stats) {
  int rc = ensure_device(-1, nullptr);
  if (rc) return rc;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kStaticDevices) return fail(PROPAG_ERR_INVALID, "device ordinal out of range");
  char *base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_static_mu);
    base = static_cast<char *>(g_static_base[dev]);
  }
  if (!base) return fail(PROPAG_ERR_INVALID, "no propag_run_device_static call on this device yet");
  StatsDev h;
  cudaStream_t stream = (cudaStream_t)stream_ptr;
  CK(cudaMemcpyAsync(&h, base + kStaticStatsOff, sizeof(h), cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  if (stats) copy_stats(h, *stats);
  if (h.status) return fail(PROPAG_ERR_TIMEOUT, status_text(h.status));
  return PROPAG_OK;
}

// ======================================================== fire behaviour ==
static int fire_device(bool full, uint64_t n, const PropagTerrainPtrs *t, float *const outs[10],
                       cudaStream_t stream) {
  int sms = 0;
  int rc = ensure_device(-1, &sms);
  if (rc) return rc;
  if (!t) return fail(PROPAG_ERR_INVALID, "null terrain");
  if (n == 0) return PROPAG_OK;
  if (!t->fuel_code || !t->d1hr || !t->d10hr || !t->d100hr || !t->herb || !t->wood ||
      !t->wind_speed || !t->wind_azimuth || !t->slope || !t->aspect)
    return fail(PROPAG_ERR_INVALID, "null terrain raster");
  const float *m[5] = {t->d1hr, t->d10hr, t->d100hr, t->herb, t->wood};
  CK(launch_fire(full, n, t->fuel_code, m, t->wind_speed, t->wind_azimuth, t->slope, t->aspect,
                 outs, sms, stream));
  return PROPAG_OK;
}

extern "C" int propag_fire_simple_device(uint64_t n, const PropagTerrainPtrs *terrain,
                                         float *speed_max, float *azimuth_max,
                                         float *eccentricity, void *stream) {
  float *outs[10] = {nullptr, nullptr, nullptr, nullptr, speed_max, azimuth_max, eccentricity,
                     nullptr, nullptr, nullptr};
  return fire_device(false, n, terrain, outs, (cudaStream_t)stream);
}

extern "C" int propag_fire_full_device(uint64_t n, const PropagTerrainPtrs *terrain,
                                       const PropagFireFields *o, void *stream) {
  if (!o) return fail(PROPAG_ERR_INVALID, "null outputs");
  float *outs[10] = {o->rx_int, o->speed0, o->hpua, o->phi_eff_wind, o->speed_max,
                     o->azimuth_max, o->eccentricity, o->residence_time, o->byrams_max,
                     o->flame_max};
  return fire_device(true, n, terrain, outs, (cudaStream_t)stream);
}

namespace {
// Device copies of a host terrain (+ outputs) for the host-buffer entry points.
struct HostPath {
  DevBuf buf;
  std::mutex mu;
};
HostPath &host_path() {
  static HostPath hp;
  return hp;
}

int upload_terrain(DevBuf &buf, uint64_t n, const PropagTerrainPtrs *t, size_t extra,
                   PropagTerrainPtrs *dev, cudaStream_t s) {
  const size_t fb = align_up(n, 256), ff = align_up(n * 4, 256);
  CK(buf.reserve(fb + 9 * ff + extra, s));
  uint8_t *fuel = buf.at<uint8_t>(0);
  float *f[9];
  for (int k = 0; k < 9; ++k) f[k] = buf.at<float>(fb + k * ff);
  const float *src[9] = {t->d1hr, t->d10hr, t->d100hr, t->herb, t->wood,
                         t->wind_speed, t->wind_azimuth, t->slope, t->aspect};
  CK(cudaMemcpyAsync(fuel, t->fuel_code, n, cudaMemcpyHostToDevice, s));
  for (int k = 0; k < 9; ++k) CK(cudaMemcpyAsync(f[k], src[k], n * 4, cudaMemcpyHostToDevice, s));
  *dev = PropagTerrainPtrs{fuel, f[0], f[1], f[2], f[3], f[4], f[5], f[6], f[7], f[8]};
  return PROPAG_OK;
}
}  // namespace

static int fire_host(bool full, uint64_t n, const PropagTerrainPtrs *t, float *const host_outs[10]) {
  int rc = ensure_device(-1, nullptr);
  if (rc) return rc;
  if (!t) return fail(PROPAG_ERR_INVALID, "null terrain");
  if (n == 0) return PROPAG_OK;
  HostPath &hp = host_path();
  std::lock_guard<std::mutex> lk(hp.mu);
  cudaStream_t s = 0;
  const size_t base = align_up(n, 256) + 9 * align_up(n * 4, 256);
  PropagTerrainPtrs dev{};
  rc = upload_terrain(hp.buf, n, t, 10 * align_up(n * 4, 256), &dev, s);
  if (rc) return rc;
  float *douts[10];
  for (int k = 0; k < 10; ++k) douts[k] = host_outs[k] ? hp.buf.at<float>(base + k * align_up(n * 4, 256)) : nullptr;
  rc = fire_device(full, n, &dev, douts, s);
  if (rc) return rc;
  for (int k = 0; k < 10; ++k)
    if (host_outs[k]) CK(cudaMemcpyAsync(host_outs[k], douts[k], n * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return PROPAG_OK;
}

extern "C" int propag_fire_simple_host(uint64_t n, const PropagTerrainPtrs *terrain,
                                       float *speed_max, float *azimuth_max, float *eccentricity) {
  float *outs[10] = {nullptr, nullptr, nullptr, nullptr, speed_max, azimuth_max, eccentricity,
                     nullptr, nullptr, nullptr};
  return fire_host(false, n, terrain, outs);
}

extern "C" int propag_fire_full_host(uint64_t n, const PropagTerrainPtrs *terrain,
                                     const PropagFireFields *o) {
  if (!o) return fail(PROPAG_ERR_INVALID, "null outputs");
  float *outs[10] = {o->rx_int, o->speed0, o->hpua, o->phi_eff_wind, o->speed_max,
                     o->azimuth_max, o->eccentricity, o->residence_time, o->byrams_max,
                     o->flame_max};
  return fire_host(true, n, terrain, outs);
}

// ================================================== terrain preparation ==
namespace propag {
cudaError_t launch_slope_aspect(int W, int H, double dx, double dy, const float *dem, float *slope,
                                float *aspect, int sm_count, cudaStream_t stream);
}

extern "C" int propag_slope_aspect_device(uint32_t width, uint32_t height, double dx, double dy,
                                          const float *dem, float *slope, float *aspect,
                                          void *stream) {
  int sms = 0;
  int rc = ensure_device(-1, &sms);
  if (rc) return rc;
  if (!valid_size(width, height)) return fail(PROPAG_ERR_INVALID, "width/height must be 1..65534");
  if (!(dx != 0.0) || !(dy != 0.0) || !std::isfinite(dx) || !std::isfinite(dy))
    return fail(PROPAG_ERR_INVALID, "invalid pixel size");
  if (!dem || !slope || !aspect) return fail(PROPAG_ERR_INVALID, "null raster");
  CK(launch_slope_aspect((int)width, (int)height, dx, dy, dem, slope, aspect, sms, (cudaStream_t)stream));
  return PROPAG_OK;
}

// =============================================== moisture + fire behaviour ==
extern "C" int propag_fire_weather_device(uint64_t n, int hour, int month,
                                          const PropagWeatherPtrs *weather,
                                          const PropagTerrainPtrs *terrain, float *speed_max,
                                          float *azimuth_max, float *eccentricity, void *stream) {
  int sms = 0;
  int rc = ensure_device(-1, &sms);
  if (rc) return rc;
  if (!weather || !terrain || !speed_max || !azimuth_max || !eccentricity)
    return fail(PROPAG_ERR_INVALID, "null argument");
  if (hour < 0 || hour > 23 || month < 1 || month > 12)
    return fail(PROPAG_ERR_INVALID, "hour must be 0..23 and month 1..12");
  if (n == 0) return PROPAG_OK;
  if (!weather->temperature || !weather->humidity || !weather->cloud_cover || !weather->precipitation)
    return fail(PROPAG_ERR_INVALID, "null weather raster");
  const PropagTerrainPtrs &t = *terrain;
  if (!t.fuel_code || !t.herb || !t.wood || !t.wind_speed || !t.wind_azimuth || !t.slope || !t.aspect)
    return fail(PROPAG_ERR_INVALID, "null terrain raster");
  CK(launch_fire_weather(n, hour, month, weather->temperature, weather->humidity, weather->cloud_cover,
                         weather->precipitation, t.fuel_code, t.herb, t.wood, t.wind_speed,
                         t.wind_azimuth, t.slope, t.aspect, speed_max, azimuth_max, eccentricity, sms,
                         (cudaStream_t)stream));
  return PROPAG_OK;
}

// ============================================================== dmoist ====
namespace propag {
cudaError_t launch_dmoist(uint64_t n, int hour, int month, const float *t, const float *rh,
                          const float *cc, const float *pp, const float *slope, const float *aspect,
                          const uint8_t *fuel, float scale, float *d1, float *d10, float *d100,
                          int sm_count, cudaStream_t stream);
}

extern "C" int propag_dmoist_device(uint64_t n, int hour, int month, const PropagWeatherPtrs *w,
                                    const float *slope, const float *aspect, const uint8_t *fuel,
                                    float scale, float *d1hr, float *d10hr, float *d100hr,
                                    void *stream) {
  int sms = 0;
  int rc = ensure_device(-1, &sms);
  if (rc) return rc;
  if (hour < 0 || hour > 23) return fail(PROPAG_ERR_INVALID, "hour must be 0..23");
  if (!w || !w->temperature || !w->humidity || !w->cloud_cover || !w->precipitation || !slope ||
      !aspect || !fuel || !d1hr || !d10hr || !d100hr)
    return fail(PROPAG_ERR_INVALID, "null dmoist argument");
  if (n == 0) return PROPAG_OK;
  CK(launch_dmoist(n, hour, month, w->temperature, w->humidity, w->cloud_cover, w->precipitation, slope,
                   aspect, fuel, scale, d1hr, d10hr, d100hr, sms, (cudaStream_t)stream));
  return PROPAG_OK;
}

extern "C" int propag_dmoist_host(uint64_t n, int hour, int month, const PropagWeatherPtrs *w,
                                  const float *slope, const float *aspect, const uint8_t *fuel,
                                  float scale, float *d1hr, float *d10hr, float *d100hr) {
  int rc = ensure_device(-1, nullptr);
  if (rc) return rc;
  if (!w || !w->temperature || !w->humidity || !w->cloud_cover || !w->precipitation || !slope ||
      !aspect || !fuel || !d1hr || !d10hr || !d100hr)
    return fail(PROPAG_ERR_INVALID, "null dmoist argument");
  if (n == 0) return PROPAG_OK;
  HostPath &hp = host_path();
  std::lock_guard<std::mutex> lk(hp.mu);
  cudaStream_t s = 0;
  const size_t f4 = align_up(n * 4, 256), hw = align_up(24 * n * 4, 256), pw = align_up(6 * n * 4, 256);
  CK(hp.buf.reserve(3 * hw + pw + 2 * f4 + align_up(n, 256) + 3 * f4, s));
  size_t o = 0;
  auto take = [&](size_t bytes) { char *p = hp.buf.at<char>(o); o += bytes; return p; };
  float *t = (float *)take(hw), *rh = (float *)take(hw), *cc = (float *)take(hw), *pp = (float *)take(pw);
  float *sl = (float *)take(f4), *as = (float *)take(f4);
  uint8_t *fu = (uint8_t *)take(align_up(n, 256));
  float *o1 = (float *)take(f4), *o10 = (float *)take(f4), *o100 = (float *)take(f4);
  CK(cudaMemcpyAsync(t, w->temperature, 24 * n * 4, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(rh, w->humidity, 24 * n * 4, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(cc, w->cloud_cover, 24 * n * 4, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(pp, w->precipitation, 6 * n * 4, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(sl, slope, n * 4, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(as, aspect, n * 4, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(fu, fuel, n, cudaMemcpyHostToDevice, s));
  PropagWeatherPtrs dw{t, rh, cc, pp};
  rc = propag_dmoist_device(n, hour, month, &dw, sl, as, fu, scale, o1, o10, o100, s);
  if (rc) return rc;
  CK(cudaMemcpyAsync(d1hr, o1, n * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(d10hr, o10, n * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(d100hr, o100, n * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return PROPAG_OK;
}

// ======================================================= plain drop-in ====
namespace {
struct RunHostState {
  std::mutex mu;
  propag_engine *engine = nullptr;
  int engine_tile = 0, engine_cluster = -1, engine_threads = -1, engine_device = -2;
  DevBuf buf;
};
RunHostState &run_state() {
  static RunHostState s;
  return s;
}
}  // namespace

extern "C" int propag_run_host(const Settings *settings, const PropagTerrainPtrs *terrain,
                               const PropagIgnition *ignitions, uint64_t n_ignitions,
                               const PropagOptions *opt, float *time, uint16_t *refs_x,
                               uint16_t *refs_y, uint32_t *boundaries, PropagStats *stats) {
  if (!settings || !terrain || !time) return fail(PROPAG_ERR_INVALID, "null argument");
  const GeoReference &g = settings->geo_ref;
  if (!valid_size(g.width, g.height)) return fail(PROPAG_ERR_INVALID, "width/height must be 1..65534");
  if (n_ignitions && !ignitions) return fail(PROPAG_ERR_INVALID, "null ignitions");
  int rc = ensure_device(opt ? opt->device : -1, nullptr);
  if (rc) return rc;
  RunHostState &st = run_state();
  std::lock_guard<std::mutex> lk(st.mu);
  PropagOptions o = opt ? *opt : PropagOptions{0, 0, 0, -1};
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (!st.engine || st.engine_tile != o.tile || st.engine_cluster != o.cluster ||
      st.engine_threads != o.threads || st.engine_device != dev) {
    if (st.engine) propag_engine_destroy(st.engine);
    st.engine = propag_engine_create(&o);
    if (!st.engine) return PROPAG_ERR_INVALID;
    st.engine_tile = o.tile;
    st.engine_cluster = o.cluster;
    st.engine_threads = o.threads;
    st.engine_device = dev;
  }
  cudaStream_t s = 0;
  const uint64_t N = (uint64_t)g.width * g.height;
  const uint64_t words = (N + 31) / 32;
  const size_t tb = align_up(N, 256) + 9 * align_up(N * 4, 256);
  const size_t ff = align_up(N * 4, 256);
  const size_t extra = 4 * ff + 2 * align_up(N * 2, 256) + align_up(words * 4, 256) +
                       align_up(n_ignitions * sizeof(PropagIgnition) + 16, 256);
  PropagTerrainPtrs dev_t{};
  rc = upload_terrain(st.buf, N, terrain, extra, &dev_t, s);
  if (rc) return rc;
  size_t o2 = tb;
  float *d_speed = st.buf.at<float>(o2); o2 += ff;
  float *d_az = st.buf.at<float>(o2); o2 += ff;
  float *d_ecc = st.buf.at<float>(o2); o2 += ff;
  float *d_time = st.buf.at<float>(o2); o2 += ff;
  uint16_t *d_rx = st.buf.at<uint16_t>(o2); o2 += align_up(N * 2, 256);
  uint16_t *d_ry = st.buf.at<uint16_t>(o2); o2 += align_up(N * 2, 256);
  uint32_t *d_bnd = st.buf.at<uint32_t>(o2); o2 += align_up(words * 4, 256);
  PropagIgnition *d_ign = st.buf.at<PropagIgnition>(o2);
  if (n_ignitions)
    CK(cudaMemcpyAsync(d_ign, ignitions, n_ignitions * sizeof(PropagIgnition), cudaMemcpyHostToDevice, s));
  rc = propag_fire_simple_device(N, &dev_t, d_speed, d_az, d_ecc, s);
  if (rc) return rc;
  PropagJob job{};
  job.width = g.width;
  job.height = g.height;
  job.dx = g.transform.gt.dx;
  job.dy = g.transform.gt.dy;
  job.max_time = settings->max_time;
  job.tile = 0;
  job.speed_max = d_speed;
  job.azimuth_max = d_az;
  job.eccentricity = d_ecc;
  job.ignitions = d_ign;
  job.n_ignitions = (uint32_t)n_ignitions;
  job.arith = (uint32_t)o.arith;
  job.time = d_time;
  job.refs_x = d_rx;
  job.refs_y = d_ry;
  job.boundaries = d_bnd;
  PropagStats js{};
  rc = engine_run(st.engine, &job, 1, s, &js);
  if (rc) return rc;
  CK(cudaMemcpyAsync(time, d_time, N * 4, cudaMemcpyDeviceToHost, s));
  if (refs_x) CK(cudaMemcpyAsync(refs_x, d_rx, N * 2, cudaMemcpyDeviceToHost, s));
  if (refs_y) CK(cudaMemcpyAsync(refs_y, d_ry, N * 2, cudaMemcpyDeviceToHost, s));
  if (boundaries) CK(cudaMemcpyAsync(boundaries, d_bnd, words * 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (stats) *stats = js;
  return PROPAG_OK;
}

// ====================================================== rasterisation ====
extern "C" int64_t propag_rasterize_ignitions(const GeoReference *g, const FFITimeFeature *f,
                                              uint64_t n, PropagIgnition *out, uint64_t max_out) {
  if (!g) return fail(PROPAG_ERR_INVALID, "null geo_ref");
  if (n && !f) return fail(PROPAG_ERR_INVALID, "null features");
  int64_t k = 0;
  for (uint64_t i = 0; i < n; ++i) {
    if (!f[i].geom_wkb || f[i].geom_wkb_len == 0) continue;  // propag.rs:130-141
    Geometry geom;
    if (!parse_wkb(f[i].geom_wkb, f[i].geom_wkb_len, geom)) continue;
    const float t = f[i].time;
    rasterize(*g, geom, [&](int64_t c, int64_t r) {
      if ((uint64_t)k < max_out && out) out[k] = PropagIgnition{(uint32_t)c, (uint32_t)r, t};
      ++k;
    });
  }
  return k;
}

extern "C" int propag_write_geotiff(const GeoReference *g, const float *time, const char *path) {
  if (!g || !time || !path) return fail(PROPAG_ERR_INVALID, "null argument");
  std::string err;
  if (!write_geotiff_f32(path, *g, time, err)) return fail(PROPAG_ERR_INVALID, err);
  return PROPAG_OK;
}

// ======================================================= self-tests =======
extern "C" int propag_selftest_time_from(int arith, uint64_t n, const int32_t *fx, const int32_t *fy,
                                         const float *ftime, const int32_t *tx, const int32_t *ty,
                                         const float *smax, const float *azmax, const float *ecc,
                                         float dx, float dy, float *out) {
  int rc = ensure_device(-1, nullptr);
  if (rc) return rc;
  if (arith != PROPAG_ARITH_REFERENCE && arith != PROPAG_ARITH_PORTABLE)
    return fail(PROPAG_ERR_INVALID, "arith must be PROPAG_ARITH_REFERENCE or PROPAG_ARITH_PORTABLE");
  if (n == 0) return PROPAG_OK;
  if (!fx || !fy || !ftime || !tx || !ty || !smax || !azmax || !ecc || !out)
    return fail(PROPAG_ERR_INVALID, "null argument");
  DevBuf b;
  const size_t a = align_up(n * 4, 256);
  CK(b.reserve(10 * a, nullptr));
  const void *src[9] = {fx, fy, ftime, tx, ty, smax, azmax, ecc};
  for (int k = 0; k < 8; ++k) CK(cudaMemcpy(b.at<char>(k * a), src[k], n * 4, cudaMemcpyHostToDevice));
  CK(launch_time_from(arith == PROPAG_ARITH_REFERENCE, n, b.at<int32_t>(0), b.at<int32_t>(a),
                      b.at<float>(2 * a), b.at<int32_t>(3 * a), b.at<int32_t>(4 * a),
                      b.at<float>(5 * a), b.at<float>(6 * a), b.at<float>(7 * a), dx, dy, dy < 0,
                      b.at<float>(8 * a), nullptr));
  CK(cudaMemcpy(out, b.at<float>(8 * a), n * 4, cudaMemcpyDeviceToHost));
  return PROPAG_OK;
}

extern "C" int propag_selftest_cosf_table(uint32_t first_bits, uint64_t n, float *out) {
  int rc = ensure_device(-1, nullptr);
  if (rc) return rc;
  if (n == 0) return PROPAG_OK;
  if (!out) return fail(PROPAG_ERR_INVALID, "null output");
  if ((uint64_t)first_bits + n > (1ull << 32)) return fail(PROPAG_ERR_INVALID, "bit range past 2^32");
  const uint64_t chunk = 1ull << 26;  // 256 MB of floats per pass
  DevBuf b;
  CK(b.reserve(std::min(n, chunk) * 4, nullptr));
  for (uint64_t o = 0; o < n; o += chunk) {
    const uint64_t m = std::min(chunk, n - o);
    CK(launch_cosf_table(first_bits + (uint32_t)o, m, b.at<float>(0), nullptr));
    CK(cudaMemcpy(out + o, b.at<float>(0), m * 4, cudaMemcpyDeviceToHost));
  }
  return PROPAG_OK;
}

extern "C" int propag_selftest_atan2f_table(int32_t max_a, int32_t max_b, float *out) {
  int rc = ensure_device(-1, nullptr);
  if (rc) return rc;
  if (max_a < 0 || max_b < 0 || max_a > 65535 || max_b > 65535 || !out)
    return fail(PROPAG_ERR_INVALID, "table half-widths must be 0..65535, output non-null");
  const int64_t w = 2 * (int64_t)max_a + 1, h = 2 * (int64_t)max_b + 1;
  const int32_t rows = (int32_t)std::max<int64_t>(1, std::min<int64_t>(h, (1 << 26) / w));
  DevBuf b;
  CK(b.reserve((size_t)(w * rows * 4), nullptr));
  for (int32_t r0 = 0; r0 < h; r0 += rows) {
    const int32_t nb = (int32_t)std::min<int64_t>(rows, h - r0);
    CK(launch_atan2f_table(max_a, max_b, r0, nb, b.at<float>(0), nullptr));
    CK(cudaMemcpy(out + (size_t)r0 * w, b.at<float>(0), (size_t)(w * nb * 4), cudaMemcpyDeviceToHost));
  }
  return PROPAG_OK;
}

// ========================================================= misc ===========
extern "C" const char *propag_last_error(void) { return g_error.c_str(); }

extern "C" int propag_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

extern "C" const char *propag_version(void) { return "propag-b200 0.1.0 (sm_100a)"; }

// ======================================================= plugin ABI =======
extern "C" Settings create_settings(GeoReference geo_ref, float max_time) {
  Settings s;
  s.geo_ref = geo_ref;
  s.max_time = max_time;
  return s;
}

extern "C" FireSimpleCuda create_fire(float speed_max, float azimuth_max, float eccentricity) {
  return FireSimpleCuda{speed_max, azimuth_max, eccentricity};
}

extern "C" uint32_t GeoReference_len(const GeoReference *g) { return g->width * g->height; }
extern "C" float GeoReference_x0(const GeoReference *g) {
  const GT &t = g->transform.gt;
  return t.dx > 0.0f ? t.x0 : t.x0 + t.dx * (float)g->width;
}
extern "C" float GeoReference_x1(const GeoReference *g) {
  const GT &t = g->transform.gt;
  return t.dx > 0.0f ? t.x0 + t.dx * (float)g->width : t.x0;
}
extern "C" float GeoReference_y0(const GeoReference *g) {
  const GT &t = g->transform.gt;
  return t.dy > 0.0f ? t.y0 : t.y0 + t.dy * (float)g->height;
}
extern "C" float GeoReference_y1(const GeoReference *g) {
  const GT &t = g->transform.gt;
  return t.dy > 0.0f ? t.y0 + t.dy * (float)g->height : t.y0;
}

// GT::invert, crates/geometry/src/lib.rs:84-124 (f32 arithmetic).
static bool gt_invert(const GT &a, GT &inv) {
  if (a.rx == 0.0f && a.ry == 0.0f && a.dx != 0.0f && a.dy != 0.0f) {
    inv = GT{-a.x0 / a.dx, 1.0f / a.dx, 0.0f, -a.y0 / a.dy, 0.0f, 1.0f / a.dy};
    return true;
  }
  const float det = a.dx * a.dy - a.rx * a.ry;
  const float mag = std::max(std::max(std::fabs(a.dx), std::fabs(a.rx)),
                             std::max(std::fabs(a.ry), std::fabs(a.dy)));
  if (!(std::fabs(det) > 1e-10f * mag * mag)) return false;
  const float id = 1.0f / det;
  inv = GT{(a.rx * a.y0 - a.x0 * a.dy) * id, a.dy * id, -a.rx * id,
           (-a.dx * a.y0 + a.x0 * a.ry) * id, -a.ry * id, a.dx * id};
  return true;
}

// NumCast f32 -> u32 (fails on NaN, negative, too large).
static bool to_u32(float v, uint32_t &out) {
  if (!(v >= 0.0f) || !(v < 4294967296.0f)) return false;
  out = (uint32_t)v;
  return true;
}

// GeoReference::south_up / north_up, crates/geometry/src/lib.rs:239-276.
static bool make_georef(bool north, float x0, float y0, float x1, float y1, float dx, float dy,
                        const char *proj, GeoReference *result) {
  if (!proj || !result) return false;
  const size_t len = strlen(proj);
  if (len >= sizeof(result->proj)) return false;
  GeoReference g;
  std::memset(&g, 0, sizeof(g));
  g.transform.gt = north ? GT{x0, dx, 0.0f, y1, 0.0f, -dy} : GT{x0, dx, 0.0f, y0, 0.0f, dy};
  if (!gt_invert(g.transform.gt, g.transform.inv)) return false;
  if (!to_u32(std::ceil((x1 - x0) / dx), g.width)) return false;
  if (!to_u32(std::ceil((y1 - y0) / dy), g.height)) return false;
  std::memcpy(g.proj, proj, len);
  *result = g;
  return true;
}

extern "C" bool GeoReference_south_up(float x0, float y0, float x1, float y1, float dx, float dy,
                                      const char *proj, GeoReference *result) {
  return make_georef(false, x0, y0, x1, y1, dx, dy, proj, result);
}
extern "C" bool GeoReference_north_up(float x0, float y0, float x1, float y1, float dx, float dy,
                                      const char *proj, GeoReference *result) {
  return make_georef(true, x0, y0, x1, y1, dx, dy, proj, result);
}

static void copy_err(char *err_msg, uintptr_t err_len, const std::string &msg) {
  if (err_msg && err_len) strncpy(err_msg, msg.c_str(), err_len);  // propag.rs:295-306
}

static std::string norm_crs(const char *s) {
  std::string out;
  bool space = false;
  for (const char *p = s; *p; ++p) {
    if (*p == ' ' || *p == '\t' || *p == '\n') {
      space = !out.empty();
      continue;
    }
    if (space) out.push_back(' ');
    space = false;
    out.push_back(*p);
  }
  return out;
}

extern "C" bool propag_rasterize_fuels(const FFIFuelFeature *fuels, uintptr_t fuels_len,
                                       const char *fuels_crs, const GeoReference *geo_ref,
                                       uint8_t *result, char *err_msg, uintptr_t err_len) {
  if (!geo_ref || !result) {
    copy_err(err_msg, err_len, "null geo_ref or result");
    return false;
  }
  if (!fuels_crs) {
    copy_err(err_msg, err_len, "invalid fuels CRS");
    return false;
  }
  const std::string grid = norm_crs((const char *)geo_ref->proj), src = norm_crs(fuels_crs);
  if (!src.empty() && src != grid) {
    copy_err(err_msg, err_len,
             "fuels CRS differs from the grid CRS; this build does not reproject (pass geometries in the grid CRS)");
    return false;
  }
  const uint64_t N = (uint64_t)geo_ref->width * geo_ref->height;
  std::memset(result, 255, N);  // nodata (propag.rs:941-943)
  for (uintptr_t i = 0; fuels && i < fuels_len; ++i) {
    if (!fuels[i].geom_wkb || fuels[i].geom_wkb_len == 0) continue;
    Geometry geom;
    if (!parse_wkb(fuels[i].geom_wkb, fuels[i].geom_wkb_len, geom)) continue;
    const uint8_t code = fuels[i].code;
    rasterize(*geo_ref, geom, [&](int64_t c, int64_t r) { result[c + r * (int64_t)geo_ref->width] = code; });
  }
  return true;
}

// ========================================== rasterisation on the device ====
namespace propag {
cudaError_t launch_rasterize_winner(const RasterPlanDev &p, int64_t W, int64_t H, int32_t *win,
                                    int sm_count, cudaStream_t stream);
cudaError_t launch_finish_times(float *times, const float *value, int64_t n, int sm_count,
                                cudaStream_t stream);
cudaError_t launch_finish_codes(const int32_t *win, const uint8_t *value, uint8_t *out, int64_t n,
                                int sm_count, cudaStream_t stream);
uint64_t burning_chunks(int64_t n);
cudaError_t launch_burning_list(const float *times, int64_t W, int64_t H, uint32_t *counts,
                                uint64_t *offsets, PropagIgnition *out, uint64_t max_out,
                                int sm_count, cudaStream_t stream);
}  // namespace propag

namespace {

// A stream-ordered device allocation, released on the same stream.
struct StreamBuf {
  void *p = nullptr;
  cudaStream_t s = nullptr;
  ~StreamBuf() {
    if (p) cudaFreeAsync(p, s);
  }
};

size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

// Copies a plan and its features' values (segments | polygons | edges |
// values, each 16-byte aligned) into one device allocation.
int upload_plan(const RasterPlan &plan, const void *values, size_t value_bytes, cudaStream_t s,
                StreamBuf &buf, RasterPlanDev &dev, const void *&dev_values) {
  const size_t bs = align16(plan.segs.size() * sizeof(RasterSeg));
  const size_t bp = align16(plan.polys.size() * sizeof(RasterPoly));
  const size_t be = align16(plan.edges.size() * sizeof(RasterEdge));
  const size_t total = bs + bp + be + align16(value_bytes);
  dev = RasterPlanDev{};
  dev_values = nullptr;
  buf.s = s;
  if (total == 0) return PROPAG_OK;
  std::vector<uint8_t> host(total, 0);
  if (bs) std::memcpy(host.data(), plan.segs.data(), plan.segs.size() * sizeof(RasterSeg));
  if (bp) std::memcpy(host.data() + bs, plan.polys.data(), plan.polys.size() * sizeof(RasterPoly));
  if (be) std::memcpy(host.data() + bs + bp, plan.edges.data(), plan.edges.size() * sizeof(RasterEdge));
  if (value_bytes) std::memcpy(host.data() + bs + bp + be, values, value_bytes);
  CK(cudaMallocAsync(&buf.p, total, s));
  // from pageable memory: returns once the bytes are staged, so `host` may go
  CK(cudaMemcpyAsync(buf.p, host.data(), total, cudaMemcpyHostToDevice, s));
  char *d = static_cast<char *>(buf.p);
  dev.segs = reinterpret_cast<const RasterSeg *>(d);
  dev.nseg = plan.segs.size();
  dev.samples = plan.samples;
  dev.polys = reinterpret_cast<const RasterPoly *>(d + bs);
  dev.npoly = plan.polys.size();
  dev.rows = plan.rows;
  dev.edges = reinterpret_cast<const RasterEdge *>(d + bs + bp);
  dev_values = d + bs + bp + be;
  return PROPAG_OK;
}

// Parses features i (skipping missing and invalid WKB, as the host
// rasterisers do) into a plan, feature index = position in the input.
template <typename GetWkb>
RasterPlan plan_features(const GeoReference &g, uint64_t n, GetWkb &&wkb) {
  RasterPlan plan;
  for (uint64_t i = 0; i < n; ++i) {
    const uint8_t *data = nullptr;
    uintptr_t len = 0;
    wkb(i, data, len);
    if (!data || len == 0) continue;
    Geometry geom;
    if (!parse_wkb(data, len, geom)) continue;
    plan_geometry(g, geom, (int32_t)i, plan);
  }
  return plan;
}

}  // namespace

extern "C" int propag_rasterize_times_device(const GeoReference *g, const FFITimeFeature *f,
                                             uint64_t n, float *times, void *stream) {
  int sms = 0;
  int rc = ensure_device(-1, &sms);
  if (rc) return rc;
  if (!g || !times) return fail(PROPAG_ERR_INVALID, "null geo_ref or times");
  if (n && !f) return fail(PROPAG_ERR_INVALID, "null features");
  if (!valid_size(g->width, g->height)) return fail(PROPAG_ERR_INVALID, "width/height must be 1..65534");
  if (n > 0x7FFFFFFFull) return fail(PROPAG_ERR_INVALID, "too many features");
  if ((uintptr_t)times % alignof(float)) return fail(PROPAG_ERR_INVALID, "times is not 4-byte aligned");
  const cudaStream_t s = (cudaStream_t)stream;
  const RasterPlan plan = plan_features(*g, n, [&](uint64_t i, const uint8_t *&d, uintptr_t &l) {
    d = f[i].geom_wkb;
    l = f[i].geom_wkb_len;
  });
  std::vector<float> value(n);
  for (uint64_t i = 0; i < n; ++i) value[i] = f[i].time;
  StreamBuf buf;
  RasterPlanDev dev;
  const void *dev_value;
  rc = upload_plan(plan, value.data(), n * sizeof(float), s, buf, dev, dev_value);
  if (rc) return rc;
  const int64_t W = g->width, H = g->height;
  CK(launch_rasterize_winner(dev, W, H, reinterpret_cast<int32_t *>(times), sms, s));
  CK(launch_finish_times(times, static_cast<const float *>(dev_value), W * H, sms, s));
  return PROPAG_OK;
}

extern "C" int propag_rasterize_fuels_device(const FFIFuelFeature *fuels, uintptr_t n,
                                             const char *fuels_crs, const GeoReference *g,
                                             uint8_t *result, void *stream) {
  int sms = 0;
  int rc = ensure_device(-1, &sms);
  if (rc) return rc;
  if (!g || !result) return fail(PROPAG_ERR_INVALID, "null geo_ref or result");
  if (n && !fuels) return fail(PROPAG_ERR_INVALID, "null features");
  if (!fuels_crs) return fail(PROPAG_ERR_INVALID, "invalid fuels CRS");
  if (!valid_size(g->width, g->height)) return fail(PROPAG_ERR_INVALID, "width/height must be 1..65534");
  if (n > 0x7FFFFFFFull) return fail(PROPAG_ERR_INVALID, "too many features");
  const std::string grid = norm_crs((const char *)g->proj), src = norm_crs(fuels_crs);
  if (!src.empty() && src != grid)
    return fail(PROPAG_ERR_INVALID,
                "fuels CRS differs from the grid CRS; this build does not reproject (pass geometries in the grid CRS)");
  const cudaStream_t s = (cudaStream_t)stream;
  const RasterPlan plan = plan_features(*g, n, [&](uint64_t i, const uint8_t *&d, uintptr_t &l) {
    d = fuels[i].geom_wkb;
    l = fuels[i].geom_wkb_len;
  });
  std::vector<uint8_t> value(n);
  for (uint64_t i = 0; i < n; ++i) value[i] = fuels[i].code;
  StreamBuf buf, win;
  RasterPlanDev dev;
  const void *dev_value;
  rc = upload_plan(plan, value.data(), n, s, buf, dev, dev_value);
  if (rc) return rc;
  const int64_t W = g->width, H = g->height;
  win.s = s;
  CK(cudaMallocAsync(&win.p, (size_t)(W * H) * sizeof(int32_t), s));
  int32_t *w = static_cast<int32_t *>(win.p);
  CK(launch_rasterize_winner(dev, W, H, w, sms, s));
  CK(launch_finish_codes(w, static_cast<const uint8_t *>(dev_value), result, W * H, sms, s));
  return PROPAG_OK;
}

extern "C" int64_t propag_ignitions_from_times_device(const float *times, uint32_t width,
                                                      uint32_t height, PropagIgnition *out,
                                                      uint64_t max_out, void *stream) {
  int sms = 0;
  int rc = ensure_device(-1, &sms);
  if (rc) return rc;
  if (!times) return fail(PROPAG_ERR_INVALID, "null times");
  if (max_out && !out) return fail(PROPAG_ERR_INVALID, "null out with max_out > 0");
  if (!valid_size(width, height)) return fail(PROPAG_ERR_INVALID, "width/height must be 1..65534");
  if ((uintptr_t)times % alignof(float) || (uintptr_t)out % alignof(PropagIgnition))
    return fail(PROPAG_ERR_INVALID, "times or out is not 4-byte aligned");
  const cudaStream_t s = (cudaStream_t)stream;
  const int64_t W = width, H = height;
  const uint64_t chunks = burning_chunks(W * H);
  const size_t bc = align16(chunks * sizeof(uint32_t));
  StreamBuf buf;
  buf.s = s;
  CK(cudaMallocAsync(&buf.p, bc + (chunks + 1) * sizeof(uint64_t), s));
  uint32_t *counts = static_cast<uint32_t *>(buf.p);
  uint64_t *offsets = reinterpret_cast<uint64_t *>(static_cast<char *>(buf.p) + bc);
  CK(launch_burning_list(times, W, H, counts, offsets, out, max_out, sms, s));
  uint64_t total = 0;
  // into pageable memory: returns when the copy (and the work ahead of it) is done
  CK(cudaMemcpyAsync(&total, offsets + chunks, sizeof(total), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return (int64_t)total;
}

namespace propag {  // gpkg.cpp
bool write_refs_gpkg(const GeoReference &g, const float *time, const uint16_t *rx,
                     const uint16_t *ry, const std::string &path, std::string &err);
bool write_boundaries_gpkg(const GeoReference &g, uint32_t tile, uint32_t block,
                           const std::string &grid_path, const std::string &block_path,
                           std::string &err);
}  // namespace propag

// The reference's launch geometry behind its "grids" and "blocks" layers: a
// super-grid tile of the default side, thread blocks of 19 x 19 cells
// (crates/propag/src/propag.rs:33,392-418).
constexpr uint32_t kOutlineBlock = 19;

extern "C" int propag_write_refs_gpkg(const GeoReference *g, const float *time,
                                      const uint16_t *refs_x, const uint16_t *refs_y,
                                      const char *path) {
  if (!g || !time || !refs_x || !refs_y || !path || !*path) return fail(PROPAG_ERR_INVALID, "null argument");
  std::string err;
  if (!write_refs_gpkg(*g, time, refs_x, refs_y, path, err)) return fail(PROPAG_ERR_INVALID, err);
  return PROPAG_OK;
}

extern "C" int propag_write_boundaries_gpkg(const GeoReference *g, int32_t tile,
                                            const char *grid_path, const char *block_path) {
  if (!g) return fail(PROPAG_ERR_INVALID, "null geo_ref");
  const uint32_t T = tile > 0 ? (uint32_t)tile : PROPAG_DEFAULT_TILE;
  std::string err;
  if (!write_boundaries_gpkg(*g, T, kOutlineBlock, grid_path ? grid_path : "",
                             block_path ? block_path : "", err))
    return fail(PROPAG_ERR_INVALID, err);
  return PROPAG_OK;
}

extern "C" bool FFIPropagation_run(FFIPropagation p, uintptr_t err_len, char *err_msg) {
  try {
    const GeoReference &g = p.settings.geo_ref;
    if (!p.output_path || !*p.output_path) {
      copy_err(err_msg, err_len, "invalid output_path");
      return false;
    }
    if (!valid_size(g.width, g.height)) {
      copy_err(err_msg, err_len, "grid width/height must be 1..65534");
      return false;
    }
    if (!p.initial_ignited_elements_crs) {
      copy_err(err_msg, err_len, "invalid initial_ignited_elements_crs");
      return false;
    }
    const std::string grid = norm_crs((const char *)g.proj), src = norm_crs(p.initial_ignited_elements_crs);
    if (!src.empty() && src != grid) {
      copy_err(err_msg, err_len,
               "ignition CRS differs from the grid CRS; this build does not reproject (pass geometries in the grid CRS)");
      return false;
    }
    // ignitions (invalid WKB silently dropped, propag.rs:213-215)
    std::vector<PropagIgnition> ign;
    const uint64_t nf = p.initial_ignited_elements ? p.initial_ignited_elements_len : 0;
    const int64_t k = propag_rasterize_ignitions(&g, p.initial_ignited_elements, nf, nullptr, 0);
    if (k < 0) {
      copy_err(err_msg, err_len, g_error);
      return false;
    }
    ign.resize((size_t)k);
    propag_rasterize_ignitions(&g, p.initial_ignited_elements, nf, ign.data(), ign.size());
    // terrain through the callback (FFITerrainLoader::load_extent, propag.rs:813-835)
    const uint64_t N = (uint64_t)g.width * g.height;
    std::vector<uint8_t> fuel(N, 0);
    std::vector<std::vector<float>> fl(9, std::vector<float>(N, 0.0f));
    FFITerrain t{fuel.data(), fl[0].data(), fl[1].data(), fl[2].data(), fl[3].data(),
                 fl[4].data(), fl[5].data(), fl[6].data(), fl[7].data(), fl[8].data()};
    if (!p.terrain_loader.load || !p.terrain_loader.load(p.terrain_loader.context, &g, &t)) {
      copy_err(err_msg, err_len, "load_extent_error");
      return false;
    }
    PropagTerrainPtrs tp{fuel.data(), fl[0].data(), fl[1].data(), fl[2].data(), fl[3].data(),
                         fl[4].data(), fl[5].data(), fl[6].data(), fl[7].data(), fl[8].data()};
    std::vector<float> time(N);
    std::vector<uint16_t> rx(N), ry(N);
    std::vector<uint32_t> bnd((N + 31) / 32);
    PropagStats stats{};
    const int rc = propag_run_host(&p.settings, &tp, ign.data(), ign.size(), nullptr, time.data(),
                                   rx.data(), ry.data(), bnd.data(), &stats);
    if (rc) {
      copy_err(err_msg, err_len, g_error);
      return false;
    }
    std::string err;
    if (!write_geotiff_f32(p.output_path, g, time.data(), err)) {
      copy_err(err_msg, err_len, err);
      return false;
    }
    if (p.refs_output_path && *p.refs_output_path &&  // write_refs, propag.rs:699-750
        !write_refs_gpkg(g, time.data(), rx.data(), ry.data(), p.refs_output_path, err)) {
      copy_err(err_msg, err_len, err);
      return false;
    }
    // tile outlines (write_boundaries, propag.rs:601-697): the "grids" layer
    // is the super-grid tiles, the "blocks" layer their 19 x 19 thread blocks
    const bool want_grid = p.grid_boundaries_out_path && *p.grid_boundaries_out_path;
    const bool want_block = p.block_boundaries_out_path && *p.block_boundaries_out_path;
    if ((want_grid || want_block) &&
        !write_boundaries_gpkg(g, PROPAG_DEFAULT_TILE, kOutlineBlock,
                               want_grid ? p.grid_boundaries_out_path : "",
                               want_block ? p.block_boundaries_out_path : "", err)) {
      copy_err(err_msg, err_len, err);
      return false;
    }
    return true;
  } catch (const std::exception &ex) {  // catch_unwind, propag.rs:280-308
    copy_err(err_msg, err_len, ex.what());
    return false;
  } catch (...) {
    copy_err(err_msg, err_len, "unknown error");
    return false;
  }
}

extern "C" PluginT create_plugin(void) {
  PluginT p;
  p.run = FFIPropagation_run;
  p.rasterize_fuels = propag_rasterize_fuels;
  return p;
}
