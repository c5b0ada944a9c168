/*
 * propag_b200.h -- B200 entry points of libpropag.so beyond the reference ABI.
 *
 * Plain C: pointers, sizes and an opaque stream handle (a cudaStream_t passed
 * as void*).  Every function returns PROPAG_OK (0) or a negative status; the
 * message of the last failure on the calling thread is propag_last_error().
 * There is no CPU fallback: without a usable CUDA device every compute entry
 * point fails with PROPAG_ERR_NO_DEVICE.
 *
 * The computations are the reference's hot path (paths relative to the
 * reference project):
 *   fire behaviour   crates/firelib/src/cuda.rs:9-95 (cuda_standard_burn,
 *                    cuda_standard_simple_burn) over firelib.rs:996-1188
 *   propagation      crates/propag/src/propag.cu (pre_propagate, propag,
 *                    post_propagate) driven as crates/propag/src/propag.rs:392-556
 *   input rasters    rasterize_times / rasterize_fuels,
 *                    crates/propag/src/propag.rs:837-890, 929-982; dead fuel
 *                    moisture, crates/dmoist/src/lib.rs:55-137
 *   output layers    write_refs / write_boundaries, propag.rs:576-750
 */
#ifndef PROPAG_B200_H
#define PROPAG_B200_H

#include "propag_host.h"

#ifdef __cplusplus
extern "C" {
#endif

#define PROPAG_OK 0
#define PROPAG_ERR_INVALID (-1)   /* bad argument */
#define PROPAG_ERR_CUDA (-2)      /* a CUDA call failed */
#define PROPAG_ERR_NO_DEVICE (-3) /* no CUDA device */
#define PROPAG_ERR_TIMEOUT (-4)   /* a bounded device-side wait gave up */
#define PROPAG_ERR_OOM (-5)       /* device memory exhausted */
#define PROPAG_ERR_LOADER (-6)    /* the terrain loader callback returned false */

/* Cells per side of one super-grid tile when a caller asks for the default.
 * The reference launches one cooperative grid of w x w blocks of 19 x 19
 * threads per tile, w = floor(sqrt(SMs * max active blocks per SM))
 * (crates/propag/src/propag.rs:392-418); on a 148-SM B200 with two resident
 * blocks per SM that is 17 blocks, 323 cells. */
#define PROPAG_DEFAULT_TILE 323
#define PROPAG_TILE_WHOLE_GRID (-1)

/* Message of the last failed call on this thread ("" if none). */
const char *propag_last_error(void);

/* Number of CUDA devices visible (0 when there is none or no driver). */
int propag_device_count(void);

/* Version string of this library. */
const char *propag_version(void);

/* Terrain structure-of-arrays, FFITerrain order (crates/propag/src/propag.rs:
 * 763-775).  Host or device pointers depending on the entry point. */
typedef struct PropagTerrainPtrs {
  const uint8_t *fuel_code;
  const float *d1hr;
  const float *d10hr;
  const float *d100hr;
  const float *herb;
  const float *wood;
  const float *wind_speed;
  const float *wind_azimuth;
  const float *slope;
  const float *aspect;
} PropagTerrainPtrs;

/* The ten per-cell fire fields, SI units: crates/firelib/src/cuda.rs:20-27
 * (FireCuda) plus Byram's intensity (W/m) and flame length (m) of
 * crates/firelib/src/firelib.rs:424-441.  A NULL pointer skips that field. */
typedef struct PropagFireFields {
  float *rx_int;         /* W/m^2 */
  float *speed0;         /* m/s   */
  float *hpua;           /* J/m^2 */
  float *phi_eff_wind;   /* -     */
  float *speed_max;      /* m/s   */
  float *azimuth_max;    /* rad   */
  float *eccentricity;   /* -     */
  float *residence_time; /* s     */
  float *byrams_max;     /* W/m   */
  float *flame_max;      /* m     */
} PropagFireFields;

/* Fire behaviour of n cells, device pointers, stream-ordered (no sync).
 * Cells without fire (fuel 0 or >= 14) get 0 in every field, as the
 * reference's zero-initialised outputs hold (crates/propag/src/propag.rs:437-439).
 * Replaces cuda_standard_simple_burn, crates/firelib/src/cuda.rs:57-95. */
int propag_fire_simple_device(uint64_t n, const PropagTerrainPtrs *terrain, float *speed_max,
                              float *azimuth_max, float *eccentricity, void *stream);

/* All fields (the FireCuda fields written by cuda_standard_burn,
 * crates/firelib/src/cuda.rs:7-55, plus Byram and flame). */
int propag_fire_full_device(uint64_t n, const PropagTerrainPtrs *terrain,
                            const PropagFireFields *out, void *stream);

/* Same over host buffers: copies in, runs, copies out, synchronises. */
int propag_fire_simple_host(uint64_t n, const PropagTerrainPtrs *terrain, float *speed_max,
                            float *azimuth_max, float *eccentricity);
int propag_fire_full_host(uint64_t n, const PropagTerrainPtrs *terrain,
                          const PropagFireFields *out);

/* Slope (rise/run) and aspect (compass azimuth of the downhill direction,
 * radians in [0, 2 pi), 0 on flat ground) from a DEM of width x height cells,
 * for the terrain rasters.  Central differences inside the grid, one-sided on
 * its edges, in double precision; dx and dy are the signed cell sizes of the
 * geo transform (dy < 0 for north-up).  Device pointers, stream-ordered.  No
 * counterpart in the reference, whose loader supplies slope and aspect. */
int propag_slope_aspect_device(uint32_t width, uint32_t height, double dx, double dy,
                               const float *dem, float *slope, float *aspect, void *stream);

/* Per-cell weather for the dmoist model: temperature (deg C), relative
 * humidity (%) and cloud cover (%) hour-major [24][n] (hour h of cell i at
 * h * n + i); daily precipitation (mm) of the last six days day-major [6][n]
 * (day d = d days before the forecast). */
typedef struct PropagWeatherPtrs {
  const float *temperature;
  const float *humidity;
  const float *cloud_cover;
  const float *precipitation;
} PropagWeatherPtrs;

/* Dead fuel moisture of n cells at one hour (0..23) of a day in `month`
 * (1..12), the dmoist model of crates/dmoist/src/lib.rs:55-137 evaluated per
 * cell: 1-h moisture from the hour's weather, shading by cloud cover,
 * exposure and slope, and the precipitation of the last six days; 10-h and
 * 100-h moisture interpolated from hours 6 and 15.  slope is rise/run,
 * aspect radians (as in the terrain rasters), fuel the NFFL code.  Outputs are
 * the model's percent values times `scale` (0.01 gives the fractions the fire
 * pass takes).  Device pointers, stream-ordered. */
int propag_dmoist_device(uint64_t n, int hour, int month, const PropagWeatherPtrs *weather,
                         const float *slope, const float *aspect, const uint8_t *fuel,
                         float scale, float *d1hr, float *d10hr, float *d100hr, void *stream);
/* Dead fuel moisture and fire behaviour fused into one pass: per cell the
 * dmoist model at `hour` of `month` from the cell's weather (as
 * propag_dmoist_device with scale 0.01), then the three fields the
 * propagation needs (as propag_fire_simple_device), with no moisture
 * rasters written or read in between.  terrain's d1hr/d10hr/d100hr are not
 * read (may be NULL); the other nine rasters are.  Same bits as the two
 * passes in a row.  Device pointers, stream-ordered.  Fuses the moisture
 * of crates/dmoist/src/lib.rs:55-137 ahead of cuda_standard_simple_burn
 * (crates/firelib/src/cuda.rs:57-95), which the reference runs apart (its
 * moisture comes from host scalars). */
int propag_fire_weather_device(uint64_t n, int hour, int month, const PropagWeatherPtrs *weather,
                               const PropagTerrainPtrs *terrain, float *speed_max,
                               float *azimuth_max, float *eccentricity, void *stream);

/* Same over host buffers (copies in and out, synchronises). */
int propag_dmoist_host(uint64_t n, int hour, int month, const PropagWeatherPtrs *weather,
                       const float *slope, const float *aspect, const uint8_t *fuel, float scale,
                       float *d1hr, float *d10hr, float *d100hr);

/* One ignited cell (the result of rasterising a TimeFeature). */
typedef struct PropagIgnition {
  uint32_t x;
  uint32_t y;
  float time;
} PropagIgnition;

/* PropagOptions.cluster: group mode.  The engine's co-resident CTAs split
 * into teams of at least 32 (PROPAG_CLUSTER_GROUPS) or N (cluster = -N) CTAs,
 * one per scenario up to that, launched cooperatively without clusters; a
 * team keeps its tiles in global memory and meets at a counter barrier in
 * global memory whose waits are bounded (a wait that gives up fails the run
 * with PROPAG_ERR_TIMEOUT).  One scenario then runs on the whole device
 * instead of one cluster.  cluster = 0 chooses group mode with teams of
 * max(4, CTAs / scenarios).  Results are identical in every mode. */
#define PROPAG_CLUSTER_GROUPS (-1)

/* Self-test of group mode's bounded wait (no reference counterpart): runs an
 * 8 x 8 scenario in group mode whose team counts one CTA more than the launch
 * holds, so that its first barrier never completes.  Every CTA gives up after
 * the wait limit (2 s); the call returns PROPAG_ERR_TIMEOUT with *status = 2
 * (the job's device status: a group wait gave up), and the device stays
 * usable. */
int propag_selftest_group_wait(uint32_t *status);

/* The float arithmetic of time_from (crates/propag/src/propag.cu:269-294),
 * PropagJob.arith and PropagOptions.arith.
 *   PROPAG_ARITH_REFERENCE (0, the default): the reference's own operations as
 *     nvcc compiles propag.cu with its default flags (crates/propag/build.rs:
 *     48-69): CUDA's atan2f, the __cosf intrinsic, __frcp_rd, __fsqrt_rz, and
 *     the three multiply-adds nvcc contracts (1 - e*cos, dx*dx + dy*dy and
 *     from.time + distance * rcp).  Results are the reference kernel's.
 *   PROPAG_ARITH_PORTABLE (1): a portable cosine and arctangent and every
 *     operation rounded on its own, which a CPU reproduces bit for bit.
 * The propagation's fixpoint depends on the last bit of these values, so the
 * two give different (equally valid) arrival times in about 1 % of the cells
 * of a heterogeneous scenario. */
#define PROPAG_ARITH_REFERENCE 0
#define PROPAG_ARITH_PORTABLE 1

/* Element-wise views of the propagation's device arithmetic, for tests (no
 * counterpart in the reference; host buffers, synchronous).
 *
 * propag_selftest_time_from: out[i] = time_from from cell (fx[i], fy[i]),
 * burning since ftime[i], to cell (tx[i], ty[i]) with the fire
 * (smax[i], azmax[i], ecc[i]) on a grid of pixel size dx, dy (dy < 0:
 * north-up), in the arithmetic `arith` -- the device function the engine
 * evaluates (crates/propag/src/propag.cu:269-294).
 *
 * propag_selftest_cosf_table: out[i] = __cosf(x), x the float whose bits
 * are first_bits + i (the cosine the reference's time_from calls).
 *
 * propag_selftest_atan2f_table: out[(a + max_a) + (b + max_b) (2 max_a + 1)]
 * = atan2f(a, b) for the integers |a| <= max_a, |b| <= max_b (the bearings
 * the reference's time_from computes between cells). */
int propag_selftest_time_from(int arith, uint64_t n, const int32_t *fx, const int32_t *fy,
                              const float *ftime, const int32_t *tx, const int32_t *ty,
                              const float *smax, const float *azmax, const float *ecc, float dx,
                              float dy, float *out);
int propag_selftest_cosf_table(uint32_t first_bits, uint64_t n, float *out);
int propag_selftest_atan2f_table(int32_t max_a, int32_t max_b, float *out);

typedef struct PropagOptions {
  int32_t tile;    /* default super-grid tile side; 0 = PROPAG_DEFAULT_TILE,
                      PROPAG_TILE_WHOLE_GRID = one tile for the whole grid */
  int32_t cluster; /* CTAs (one cluster) cooperating on one scenario, 1..16; 0 = auto;
                      PROPAG_CLUSTER_GROUPS = group mode (below); -N (N > 1):
                      group mode with teams of at least N CTAs */
  int32_t threads; /* threads per CTA, multiple of 32, <= 512; 0 = 512 */
  int32_t device;  /* CUDA device ordinal; -1 = the current device */
  int32_t arith;   /* PROPAG_ARITH_*, for propag_run_host (the engine's jobs carry their own) */
} PropagOptions;

typedef struct PropagStats {
  uint64_t rounds;       /* passes over all tiles (propag.rs:502-536) */
  uint64_t launches;     /* tile launches (one cooperative launch each in the reference) */
  uint64_t sweeps;       /* Jacobi sweeps summed over launches */
  uint64_t evaluations;  /* cells evaluated (find_neighbor_which_reaches_first) */
  uint64_t improvements; /* cells whose time improved (commit_point) */
  uint64_t dda_steps;    /* cells visited by line-of-sight walks */
  uint64_t refbox_scans; /* changed cells that were some cell's reference */
  uint64_t burned;       /* cells with time < FLT_MAX after the post mask */
  uint64_t gathers;      /* time[reference] reads (burning neighbours with a reference) */
  /* SM cycles the cluster leader spent per phase, barrier waits included:
   * first sweeps of tile launches, evaluate, commit (with referrer scans),
   * staging and write-back of shared-memory tiles */
  uint64_t cyc_first, cyc_eval, cyc_commit, cyc_stage;
  uint32_t status;       /* 0 ok; nonzero: device-side error code */
  uint32_t max_walk;     /* longest line-of-sight walk (cells) */
  uint64_t t_start_ns;   /* device clock (ns) when a cluster took the job */
  uint64_t t_done_ns;    /* device clock (ns) when its propagation finished */
  uint64_t scan_cells;   /* cells visited by referrer scans (sum of the scanned box areas) */
  uint64_t cyc_wait;     /* SM cycles the team leader waited at phase barriers (included
                            in the phase cycles above) */
} PropagStats;

/* One scenario of a batch.  All pointers are device pointers; time, refs and
 * boundaries are outputs.  dy < 0 means a north-up transform (propag.cu:274). */
typedef struct PropagJob {
  uint32_t width;
  uint32_t height;
  float dx;
  float dy;
  float max_time;
  int32_t tile; /* 0 = the engine's default */
  const float *speed_max;
  const float *azimuth_max;
  const float *eccentricity;
  const PropagIgnition *ignitions;
  uint32_t n_ignitions;
  uint32_t arith;       /* PROPAG_ARITH_*: 0 = the reference's arithmetic */
  float *time;          /* arrival time, s; FLT_MAX = not burned (post_propagate mask) */
  uint16_t *refs_x;     /* reference cell of each burned cell (0xFFFF: none) */
  uint16_t *refs_y;
  uint32_t *boundaries; /* ceil(width*height/32) words, bit i = cell i is a boundary */
} PropagJob;

/* The batched propagation engine.  It owns the scratch memory of the
 * propagation (work lists, reference boxes) and reuses it across calls. */
typedef struct propag_engine propag_engine;

propag_engine *propag_engine_create(const PropagOptions *opt);

/* Device scratch the engine holds for one job of width x height cells
 * (references, referrer boxes, travel-time planes, second state copy,
 * boundary and pending bitmaps: about 60 bytes per cell), as a run lays it
 * out; the server admits requests by it.  No counterpart in the reference. */
uint64_t propag_engine_job_bytes(uint32_t width, uint32_t height);
void propag_engine_destroy(propag_engine *engine);

/* Propagates n_jobs scenarios in one persistent launch.  Stream-ordered; the
 * call returns once the work is enqueued unless stats is non-NULL, in which
 * case it synchronises and fills stats[n_jobs]. */
int propag_engine_run(propag_engine *engine, const PropagJob *jobs, uint32_t n_jobs, void *stream,
                      PropagStats *stats);

/* Device time of the last propag_engine_run's kernels, from CUDA events
 * recorded on its stream around each launch: ms[0] boundary/initial-state
 * pass + ignition scatter, ms[1] propagation kernel, ms[2] post mask.
 * Waits for the last run to finish. */
int propag_engine_last_times(propag_engine *engine, float ms[3]);

/* Statistics of the jobs of the engine's last propag_engine_run (its first
 * n_jobs jobs; n_jobs at most that run's count), for runs made without
 * `stats`: copies on `stream` and synchronises it. */
int propag_engine_last_stats(propag_engine *engine, void *stream, PropagStats *stats,
                             uint32_t n_jobs);

/* ---- serving: continuous batching ------------------------------------------
 * A server owns `lanes` CUDA streams, each with its own engine, and a
 * dispatcher thread.  propag_server_submit queues one scenario (device
 * pointers, like PropagJob; `terrain` optional: with it the fire pass runs
 * first and writes the job's fire rasters).  Whenever a lane is free the
 * dispatcher takes the requests waiting at that moment, up to max_batch and
 * within hbm_budget bytes of engine scratch in flight (each request counts
 * `device_bytes`, propag_engine_job_bytes when 0), and runs them as one batch
 * on that lane; requests that arrive while batches are on the GPU are
 * admitted as lanes and memory free up, and run alongside them.  With a
 * budget, each lane reserves hbm_budget / lanes of engine scratch when the
 * server is created (plus slot scratch, about 10 MB per job of a batch, and
 * pinned staging), so that serving itself allocates and frees no device
 * memory; a request larger than a lane's share fails with PROPAG_ERR_OOM.
 * A request's results are
 * the same alone and in any batch.  No counterpart in the reference (one
 * synchronous propagation per call, crates/propag/src/propag.rs:323-574). */
typedef struct PropagServerOptions {
  uint64_t hbm_budget; /* bytes of engine scratch in flight, reserved at creation;
                          0 = no limit (scratch grows on demand) */
  uint32_t lanes;      /* batches in flight at once (streams); 0 = 4 */
  uint32_t max_batch;  /* requests per batch; 0 = 64 */
  int32_t device;      /* CUDA device ordinal; -1 = the current device */
  int32_t pad;
} PropagServerOptions;

typedef struct PropagServerResult {
  PropagStats stats;
  uint64_t submit_ns, start_ns, done_ns; /* host steady clock: queued, dispatched, seen done */
  int32_t status;                        /* 0 queued or running, 1 done, < 0 error code */
  uint32_t batch_size;                   /* requests in the batch it ran in */
  char message[128];                     /* error message when status < 0 */
} PropagServerResult;

typedef struct propag_server propag_server;
propag_server *propag_server_create(const PropagServerOptions *opt);
/* Returns the request id (>= 0) or a negative status.  The buffers must stay
 * valid until the request is done. */
int64_t propag_server_submit(propag_server *server, const PropagJob *job,
                             const PropagTerrainPtrs *terrain, uint64_t device_bytes);
/* 1 done (or failed: see out->status), 0 not yet, < 0 unknown id. */
int propag_server_poll(propag_server *server, int64_t id, PropagServerResult *out);
/* As poll, waiting up to timeout_ms for the request to finish. */
int propag_server_wait(propag_server *server, int64_t id, PropagServerResult *out,
                       uint32_t timeout_ms);
/* Forgets a finished request. */
int propag_server_release(propag_server *server, int64_t id);
/* Runs the queue dry, then frees the server. */
void propag_server_destroy(propag_server *server);

/* A batch captured as one CUDA graph: the fire pass of every job whose
 * terrain is given (terrains[i], device pointers; terrains may be NULL to
 * skip the fire pass, the jobs' fire rasters then being inputs), then the
 * propagation of all n_jobs in one persistent launch.  Creating the graph
 * runs the batch once (uncaptured) to size the graph's private scratch, then
 * captures a second run; every launch replays it on `stream`, reading the
 * current contents of the same buffers (so new terrains or ignition times
 * written there take effect; new sizes or pointers need a new graph).  The
 * job array may be freed after creation.  No counterpart in the reference
 * (one cooperative launch per tile from the host, crates/propag/src/propag.rs:482-556). */
typedef struct propag_graph propag_graph;
propag_graph *propag_graph_create(const PropagOptions *opt, const PropagJob *jobs,
                                  const PropagTerrainPtrs *terrains, uint32_t n_jobs);
int propag_graph_launch(propag_graph *graph, void *stream);
/* Statistics of the graph's last completed launch (synchronises `stream`). */
int propag_graph_stats(propag_graph *graph, void *stream, PropagStats *stats);
void propag_graph_destroy(propag_graph *graph);

/* Times the batch (fire passes as in propag_graph_create, then the engine)
 * with each cluster size whose shared memory holds every job's tile, `repeats`
 * runs each after a warm-up run, and writes the fastest options to *best and
 * its time to *best_ms.  Results do not depend on the cluster size (the
 * schedule is fixed), only the speed does.  Runs on `stream` and waits. */
int propag_autotune(const PropagJob *jobs, const PropagTerrainPtrs *terrains, uint32_t n_jobs,
                    void *stream, int repeats, PropagOptions *best, float *best_ms);

/* Allocation-free propagation of one grid.  No counterpart in the reference:
 * its propagation allocates its device buffers on every run
 * (crates/propag/src/propag.rs:420-455).
 *
 * Same kernels, schedule and results as propag_engine_run with one job, but
 * its scratch (references, referrer boxes, boundary bits, job descriptor,
 * counters, statistics, list overflow) lives in one fixed device array of about 25 MiB,
 * reserved by the CUDA driver when the library's module holding it is loaded.
 * The call makes no cudaMalloc, cudaFree or cudaMallocHost, creates no events
 * and uses no caching allocator.  It is meant for callers that cannot
 * allocate device memory while they run:
 *   - a process whose device memory is owned by another allocator (a
 *     framework's caching pool, or a pool sized at start-up), where a
 *     cudaMalloc can fail or fragment that pool;
 *   - a latency-bound serving loop: when a larger job arrives the engine grows
 *     its scratch (stream synchronise, cudaFree, cudaMalloc), and cudaFree
 *     waits for the whole device, stalling every other stream;
 *   - a service that must not fail with out-of-memory after start-up.
 *
 * Limits: width * height <= PROPAG_STATIC_MAX_CELLS (1024 x 1024 cells), and
 * the tile (job->tile; 0 = PROPAG_DEFAULT_TILE, PROPAG_TILE_WHOLE_GRID) with
 * its one-cell halo must fit in the shared memory of a cluster of at most 16
 * CTAs (a tile side up to 323 always fits).  Larger jobs are rejected with
 * PROPAG_ERR_INVALID and a message naming the limit.
 *
 * The scratch is one per device.  Calls that overlap on the same device (from
 * two host threads, or on two streams with no ordering between them) race on
 * it and corrupt each other's results: serialise them (one stream, or an
 * event or lock between calls).  Nothing has to be zero beforehand: each call
 * clears its statistics, job queue and counters and re-initialises the
 * per-cell state in its own first kernels.  The first call on each device does
 * set-up (device attributes, the fuel table upload, the scratch's address
 * through cudaGetSymbolAddress); make that first call outside any stream
 * capture.
 *
 * Stream-ordered: returns once the work is enqueued on `stream`, unless stats
 * is non-NULL, in which case it synchronises the stream and fills *stats
 * (and fails with PROPAG_ERR_TIMEOUT if the job hit the sweep limit); a
 * caller that passes no stats reads the job's outcome with
 * propag_static_last_status before its next call.
 * The job's pointers are device pointers, as in propag_engine_run. */
#define PROPAG_STATIC_MAX_CELLS (1u << 20)
int propag_run_device_static(const PropagJob *job, void *stream, PropagStats *stats);

/* Outcome of the last propag_run_device_static on the current device, for
 * callers that ran it without `stats` (stream-ordered, no synchronisation):
 * waits for `stream` (the stream of that call), copies the job's statistics
 * out of the fixed scratch into *stats (may be NULL) and returns
 * PROPAG_ERR_TIMEOUT when the job ended on a device-side error (the sweep
 * limit), else PROPAG_OK.  Call it before the next propag_run_device_static
 * on the device, which clears the statistics.  Allocates nothing.  No
 * counterpart in the reference (its propagation reports errors synchronously,
 * crates/propag/src/propag.rs:323-574). */
int propag_static_last_status(void *stream, PropagStats *stats);

/* Plain drop-in over host buffers for one grid: fire behaviour (3 fields),
 * boundaries, propagation and post mask, like propagate()
 * (crates/propag/src/propag.rs:323-574) without the file writers.
 * time (W*H), refs_x/refs_y (W*H) and boundaries (ceil(W*H/32)) are host
 * outputs; refs/boundaries may be NULL. */
int propag_run_host(const Settings *settings, const PropagTerrainPtrs *terrain,
                    const PropagIgnition *ignitions, uint64_t n_ignitions,
                    const PropagOptions *opt, float *time, uint16_t *refs_x, uint16_t *refs_y,
                    uint32_t *boundaries, PropagStats *stats);

/* Rasterises TimeFeatures (WKB Point, MultiPoint, LineString, Polygon and
 * their Multi forms; Z/M ignored) onto the grid the way GDALRasterizeGeometries
 * burns them (crates/propag/src/propag.rs:837-890): the cell containing a
 * point, every cell a line passes through, every cell whose centre lies inside
 * a polygon; later features overwrite earlier ones.  Features with invalid
 * WKB are skipped, as the reference's filter_map does (propag.rs:213-215).
 * Writes at most max_out ignitions; returns the number of ignited cells
 * (< 0 on error). */
int64_t propag_rasterize_ignitions(const GeoReference *geo_ref, const FFITimeFeature *features,
                                   uint64_t n_features, PropagIgnition *out, uint64_t max_out);

/* Rasterisation on the device.  The host parses the WKB and maps the vertices
 * to pixel space; the burning runs on the GPU with the same rules as the
 * host rasteriser above, and the rasters are bit-identical to its result.
 * All three are stream-ordered on `stream`; the device scratch they need is
 * allocated and released on that stream (cudaMallocAsync / cudaFreeAsync).
 *
 * propag_rasterize_times_device writes the initial time raster of the
 * reference's rasterize_times (crates/propag/src/propag.rs:837-890):
 * times[width*height] (device, 4-byte aligned) = the time of the last feature
 * that burns the cell, FLT_MAX where none does.  Returns without waiting. */
int propag_rasterize_times_device(const GeoReference *geo_ref, const FFITimeFeature *features,
                                  uint64_t n_features, float *times, void *stream);

/* The fuel raster of propag_rasterize_fuels (crates/propag/src/propag.rs:
 * 892-982) into device memory: result[width*height] = the code of the last
 * feature that burns the cell, 255 (nodata) elsewhere; the same CRS rule.
 * Holds 4 bytes per cell of device scratch while it runs.  Returns without
 * waiting. */
int propag_rasterize_fuels_device(const FFIFuelFeature *fuels, uintptr_t fuels_len,
                                  const char *fuels_crs, const GeoReference *geo_ref,
                                  uint8_t *result, void *stream);

/* The ignition list of a device time raster, for PropagJob.ignitions: one
 * entry per cell whose time is not FLT_MAX, in row-major order.  It starts
 * the same propagation as propag_rasterize_ignitions' list of the same
 * features (a list with repeats, where the last entry of a cell wins).
 * Writes at most max_out entries to out (device; NULL when max_out is 0),
 * waits for the stream and returns the number of such cells (< 0 on error). */
int64_t propag_ignitions_from_times_device(const float *times, uint32_t width, uint32_t height,
                                           PropagIgnition *out, uint64_t max_out, void *stream);

/* GeoPackage layers as the reference's write_refs / write_boundaries write
 * them through GDAL (crates/propag/src/propag.rs:601-750), without GDAL:
 * propag_write_refs_gpkg writes layer "fire_references", one LineString per
 * burned cell (time < FLT_MAX) from its reference cell's centre to its own,
 * cells in the reference's order (columns outer); propag_write_boundaries_gpkg
 * writes layer "grids" (the outlines of the super-grid tiles of side `tile`,
 * 0 = PROPAG_DEFAULT_TILE) to grid_path and layer "blocks" (their 19 x 19
 * thread blocks) to block_path; a NULL or empty path skips that layer.  Each
 * file is a new GeoPackage (an existing one is replaced).  The layer's CRS
 * row holds WKT where it needs no projection library or EPSG database
 * (EPSG:4326, EPSG:326zz / 327zz / 25828-25838, PROJ strings of UTM or
 * longlat on WGS 84 / GRS 1980), "undefined" otherwise, and the grid's
 * projection string in its description.  Needs SQLite's runtime library
 * (libsqlite3.so.0).
 * Host only, no GPU. */
int propag_write_refs_gpkg(const GeoReference *geo_ref, const float *time, const uint16_t *refs_x,
                           const uint16_t *refs_y, const char *path);
int propag_write_boundaries_gpkg(const GeoReference *geo_ref, int32_t tile, const char *grid_path,
                                 const char *block_path);

/* Writes width*height arrival times as a single-band float32 GeoTIFF, tiled
 * 256 x 256, with the geo transform and nodata f32::MAX, as write_times does
 * (crates/propag/src/propag.rs:576-600). */
int propag_write_geotiff(const GeoReference *geo_ref, const float *time, const char *path);

#ifdef __cplusplus
}
#endif

#endif /* PROPAG_B200_H */
