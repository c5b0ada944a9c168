// Arrival-time propagation on B200: boundary/prep pass, ignition scatter,
// the persistent engine and the post mask.

// Reference semantics (paths relative to the reference project):
//   pre_propagate / find_boundaries   crates/propag/src/propag.cu:345-375,410-421
//   propag / Propagator::run          crates/propag/src/propag.cu:62-109,382-394
//   post_propagate                    crates/propag/src/propag.cu:110-117,396-408
//   host tile loop                    crates/propag/src/propag.rs:482-556
//
// Schedule.  The reference covers the grid with super-grid tiles of
// T x T cells (one cooperative launch each), runs the tiles one after another
// in row-major order, each until a sweep improves nothing, and repeats the
// pass until no tile improved.  Inside a tile every sweep is a Jacobi sweep
// (two grid.sync()s separate the reads from the writes).  This engine keeps
// exactly that schedule, so its results are the reference's for the same T,
// but a sweep only evaluates the cells whose inputs changed:
//   * the 3x3 neighbourhood of every cell that improved in the last sweep;
//   * the 3x3 neighbourhood of every cell whose reference improved in the last
//     sweep (a cell reads the current time of its neighbours' references,
//     propag.cu:221-224).  Each cell keeps the bounding box of the cells that
//     ever adopted it as their reference, so those referrers are found by
//     scanning that box only.
// The first sweep of each tile launch evaluates the whole tile.
//
// Mapping.  The engine is one persistent launch whose CTAs form teams; a
// team works on one scenario at a time and pulls scenarios from a queue
// (largest first), so a batch runs concurrently, scenario per team.  Two
// kinds of team:
//   * cluster mode: a thread-block cluster of 1-16 CTAs.  The tile and its
//     halo (time, reference, referrer boxes) are staged into the cluster's
//     distributed shared memory, rows dealt round-robin to the CTAs; a sweep
//     is two phases, evaluate (reads only) and commit (writes the state,
//     marks the next sweep's cells, scans referrer boxes), separated by
//     hardware cluster barriers, and the tile is written back at the end of
//     the launch.  Tiles too large for the cluster's shared memory take the
//     global-memory path below.
//   * group mode: a cooperative launch without clusters whose CTAs form
//     teams of any size (the whole device for one scenario).  The tile state
//     stays in global memory in two copies, so that a sweep is one phase; the
//     team meets at a counter barrier in global memory whose wait is bounded
//     (the engine's only spin-wait; see Team).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "engine.cuh"
#include "propag_device.cuh"

namespace cg = cooperative_groups;

namespace propag {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kEngineThreads = 512;
constexpr uint32_t kEmptyBox = 0xFFFFFFFFu;

// The GPU's global nanosecond clock (comparable across SMs and launches).
__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Per-scenario constants of the eight neighbour directions, in the
// reference's neighbour order (j outer, i inner, centre skipped): the bearing
// from the neighbour to the cell and their distance, computed with the same
// operations as time_from, so using them is bit-identical to recomputing.
struct DirConst {
  float bearing[8];
  float dist[8];
};

__device__ __forceinline__ void dir_consts(const JobDev &j, DirConst &d) {
  const bool nu = j.north_up != 0, refm = j.refm != 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int kk = k < 4 ? k : k + 1;
    const int di = kk % 3 - 1, dj = kk / 3 - 1;
    d.bearing[k] = bearing(di, dj, 0, 0, nu, refm);
    d.dist[k] = cell_distance(di, dj, j.gdx, j.gdy, refm);
  }
}

// Round-down reciprocal of the elliptical speed of a cell with fire f toward
// the cell it is neighbour k of, so that step_time(ftime, dc.dist[k], inv)
// is bit-identical to time_from(neighbour -> cell).
__device__ __forceinline__ float dir_inv_speed(const DirConst &dc, int k, const Fire &f, bool refm) {
  return inv_speed(dc.bearing[k], f, refm);
}

// ---------------------------------------------------------------- prep ----
// Boundary bits (find_boundaries) packed with a warp ballot, plus the initial
// state: time = FLT_MAX, no reference, empty referrer boxes; and the
// reciprocal direct-spread speeds toward the 8 neighbours (when the job has them).
__global__ void __launch_bounds__(256) prep_kernel(const JobDev *__restrict__ jobs) {
  const JobDev j = jobs[blockIdx.y];
  __shared__ DirConst dc;
  if (threadIdx.x == 0) dir_consts(j, dc);
  __syncthreads();
  const bool refm = j.refm != 0;
  const int64_t N = (int64_t)j.W * j.H;
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t w0 = warp * 32; w0 < N; w0 += nwarps * 32) {
    const int64_t i = w0 + lane;
    bool b = false;
    if (i < N) {
      const int x = (int)(i % j.W), y = (int)(i / j.W);
      const Fire me{__ldg(j.speed + i), __ldg(j.az + i), __ldg(j.ecc + i)};
#pragma unroll
      for (int di = -1; di < 2; ++di) {
#pragma unroll
        for (int dj = -1; dj < 2; ++dj) {
          if (di == 0 && dj == 0) continue;
          const int nx = x + di, ny = y + dj;
          if (nx < 0 || ny < 0 || nx >= j.W || ny >= j.H) continue;
          const int64_t n = nx + (int64_t)ny * j.W;
          const Fire nb{__ldg(j.speed + n), __ldg(j.az + n), __ldg(j.ecc + n)};
          b |= !similar_fires(nb, me) && me.speed_max < nb.speed_max;
        }
      }
      if (j.tt && me.speed_max != 0.0f) {
#pragma unroll
        for (int k = 0; k < 8; ++k) j.tt[k * j.tt_plane + i] = dir_inv_speed(dc, k, me, refm);
      }
      j.time[i] = FLT_MAX;
      j.refs[i] = kNoRef;
      if (j.time1) {
        j.time1[i] = FLT_MAX;
        j.refs1[i] = kNoRef;
      }
      j.box_x0[i] = kEmptyBox;
      j.box_y0[i] = kEmptyBox;
      j.box_x1[i] = 0u;
      j.box_y1[i] = 0u;
    }
    const unsigned word = __ballot_sync(kFull, b);
    if (lane == 0) {
      j.bnd[w0 >> 5] = word;
      if (j.pending) j.pending[w0 >> 5] = 0u;
    }
  }
}

// ------------------------------------------------------------- ignition ----
// Later ignitions overwrite earlier ones in the same cell (GDAL burn order);
// every cell whose time is not f32::MAX references itself
// (crates/propag/src/propag.rs:441-449).
__global__ void ignite_kernel(const JobDev *__restrict__ jobs) {
  const JobDev j = jobs[blockIdx.x];
  if (threadIdx.x != 0) return;
  struct Ign {
    uint32_t x, y;
    float t;
  };
  const Ign *ign = (const Ign *)j.ignitions;
  for (uint32_t k = 0; k < j.n_ignitions; ++k) {
    if (ign[k].x >= (uint32_t)j.W || ign[k].y >= (uint32_t)j.H) continue;
    j.time[ign[k].x + (int64_t)ign[k].y * j.W] = ign[k].t;
  }
  for (uint32_t k = 0; k < j.n_ignitions; ++k) {
    if (ign[k].x >= (uint32_t)j.W || ign[k].y >= (uint32_t)j.H) continue;
    const int64_t c = ign[k].x + (int64_t)ign[k].y * j.W;
    if (j.time[c] != FLT_MAX) {
      j.refs[c] = pack_ref(ign[k].x, ign[k].y);
      j.box_x0[c] = j.box_x1[c] = ign[k].x;
      j.box_y0[c] = j.box_y1[c] = ign[k].y;
    }
    if (j.time1) {  // the second state copy starts equal
      j.time1[c] = j.time[c];
      j.refs1[c] = j.refs[c];
    }
  }
  // the neighbours of the burning cells are the cells that can improve first
  if (j.pending) {
    for (uint32_t k = 0; k < j.n_ignitions; ++k) {
      if (ign[k].x >= (uint32_t)j.W || ign[k].y >= (uint32_t)j.H) continue;
      const int64_t c = ign[k].x + (int64_t)ign[k].y * j.W;
      if (!(j.time[c] < j.max_time && j.speed[c] != 0.0f)) continue;
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int ax = (int)ign[k].x + dx, ay = (int)ign[k].y + dy;
          if ((dx || dy) && ax >= 0 && ay >= 0 && ax < j.W && ay < j.H) {
            const int64_t n = ax + (int64_t)ay * j.W;
            j.pending[n >> 5] |= 1u << (n & 31);
          }
        }
    }
  }
}

// ------------------------------------------------------- common pieces ----
struct Best {
  float time;
  uint32_t ref;
};

__device__ __forceinline__ bool line_blocked_call(const uint32_t *__restrict__ bnd, int W, int fx,
                                               int fy, int tx, int ty, uint32_t &steps) {
  return line_blocked(bnd, W, fx, fy, tx, ty, steps);
}

struct Counters {
  uint32_t dda = 0, gat = 0, walk_max = 0;
  unsigned long long evals = 0, scans = 0, scan_cells = 0;
};

// find_neighbor_which_reaches_first (propag.cu:124-190) evaluated by the 8
// lanes of a lane group (lanes 8c .. 8c+7), lane k taking neighbour k in the
// reference's order.  Every neighbour offers a time that does not depend on
// the best found so far -- the candidate through its reference, or its own
// direct time when the line of sight is blocked or the candidate is not
// faster -- and the sequential loop keeps the first strictly smaller offer;
// so the result is the first minimum of the offers when it beats the cell's
// own time.  A lane walks its line of sight whenever the sequential loop
// could (candidate faster than the neighbour's direct time and than the
// cell's own time); only the walks the sequential loop performs (candidate
// also faster than every earlier offer) are counted, so the counters match
// the reference's order exactly.  Called by all 32 lanes.
struct GlobalAcc {
  const JobDev &j;
  const float *time;  // the state copy this sweep reads
  const uint32_t *refs;
  __device__ __forceinline__ void cell(int x, int y, float &t, uint32_t &r) const {
    const int64_t n = x + (int64_t)y * j.W;
    t = __ldcg(time + n);
    r = __ldcg(refs + n);
  }
  __device__ __forceinline__ float time_of(uint32_t r) const {
    return __ldcg(time + ref_x(r) + (int64_t)ref_y(r) * j.W);
  }
};

template <typename Acc>
__device__ __forceinline__ Best evaluate_coop(const JobDev &j, const DirConst &dc, const Acc &acc,
                                              int x, int y, Best own, bool valid, uint32_t lane,
                                              Counters &cnt) {
  const float kInf = __int_as_float(0x7f800000);
  const int k = (int)(lane & 7u);
  const int kk = k < 4 ? k : k + 1;
  const int nx = x + kk % 3 - 1, ny = y + kk / 3 - 1;
  bool act = false;
  float nt = FLT_MAX, rt = FLT_MAX;
  uint32_t nr = kNoRef;
  Fire f{0.0f, 0.0f, 0.0f};
  float tt = 0.0f;
  if (valid && nx >= 0 && ny >= 0 && nx < j.W && ny < j.H) {
    // the fire loads go out together with the state load (one memory
    // round trip), whether or not the neighbour turns out to burn
    const int64_t n = nx + (int64_t)ny * j.W;
    f.speed_max = __ldg(j.speed + n);
    f.azimuth_max = __ldg(j.az + n);
    f.eccentricity = __ldg(j.ecc + n);
    if (j.tt) tt = __ldg(j.tt + k * j.tt_plane + n);
    acc.cell(nx, ny, nt, nr);
    act = nt < j.max_time && f.speed_max != 0.0f && !(ref_x(nr) == x && ref_y(nr) == y);
    if (act) rt = acc.time_of(nr);
  }
  cnt.gat += act ? 1u : 0u;
  float offer = kInf, cand = kInf;
  uint32_t oref = 0, steps = 0;
  bool walked = false;
  if (act) {
    const bool refm = j.refm != 0;
    const float ntime =
        step_time(nt, dc.dist[k], j.tt ? tt : dir_inv_speed(dc, k, f, refm), refm);
    cand = time_from(ref_x(nr), ref_y(nr), rt, x, y, f, j.gdx, j.gdy, j.north_up != 0, refm);
    offer = ntime;
    oref = pack_ref(nx, ny);
    if (cand < ntime) {
      bool blocked = false;
      if (cand < own.time) {
        walked = true;
        blocked = line_blocked_call(j.bnd, j.W, nx, ny, ref_x(nr), ref_y(nr), steps);
      }
      if (!blocked) {
        offer = cand;
        oref = nr;
      }
    }
  }
  // running best of the sequential loop before neighbour k (exclusive min)
  float pm = offer;
#pragma unroll
  for (int o = 1; o < 8; o <<= 1) {
    const float t = __shfl_up_sync(kFull, pm, o);
    if (k >= o && t < pm) pm = t;
  }
  float before = __shfl_up_sync(kFull, pm, 1);
  if (k == 0) before = kInf;
  if (walked && cand < before) {
    cnt.dda += steps;
    cnt.walk_max = max(cnt.walk_max, steps);
  }
  // first minimum of the offers
  float bv = offer;
  uint32_t br = oref;
  int bi = k;
#pragma unroll
  for (int o = 1; o < 8; o <<= 1) {
    const float ov = __shfl_xor_sync(kFull, bv, o);
    const uint32_t orf = __shfl_xor_sync(kFull, br, o);
    const int oi = __shfl_xor_sync(kFull, bi, o);
    if (ov < bv || (ov == bv && oi < bi)) {
      bv = ov;
      br = orf;
      bi = oi;
    }
  }
  return bv < own.time ? Best{bv, br} : own;
}

// Warp-aggregated append: every lane of the (fully active) warp passes its
// count; one atomic per warp reserves the space.  Returns this lane's slot.
__device__ __forceinline__ uint32_t warp_append(uint32_t *counter, uint32_t cnt, uint32_t lane) {
  uint32_t x = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  const uint32_t total = __shfl_sync(kFull, x, 31);
  uint32_t base = 0;
  if (lane == 31 && total) base = atomicAdd(counter, total);
  base = __shfl_sync(kFull, base, 31);
  return base + x - cnt;
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, uint32_t lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, v, o);
    if (lane >= (uint32_t)o) v += y;
  }
  return v;
}

// Referrer box of a changed cell clipped to the tile grown by one cell
// (referrers further out have no neighbour inside the tile).
struct Box {
  int x0, y0, x1, y1;
  __device__ __forceinline__ uint32_t area() const {
    return x0 > x1 || y0 > y1 ? 0u : (uint32_t)(x1 - x0 + 1) * (uint32_t)(y1 - y0 + 1);
  }
};

__device__ __forceinline__ Box clip_box(int bx0, int by0, int bx1, int by1, int tx0, int ty0,
                                        int TW, int TH, int W, int H) {
  Box b;
  b.x0 = max(max(bx0, tx0 - 1), 0);
  b.y0 = max(max(by0, ty0 - 1), 0);
  b.x1 = min(min(bx1, tx0 + TW), W - 1);
  b.y1 = min(min(by1, ty0 + TH), H - 1);
  return b;
}

// One lane's referrer box in a warp's concatenated scan.
struct ScanBox {
  int x0, y0;
  uint32_t bw, want, incl;  // width, packed reference, inclusive end in the concatenation
};

// Walks the concatenation of the warp's boxes, 32 cells per step, so that a
// step is one independent wave of loads; mark_fn(hit, gx, gy) is called once
// per step by every lane.  ref_fn(gx, gy, t) returns a cell's reference and
// time.
template <typename RefFn, typename MarkFn>
__device__ __forceinline__ void warp_scan_boxes(ScanBox *sb, const Box &box, uint32_t want,
                                                const JobDev &j, uint32_t lane, Counters &cnt,
                                                RefFn ref_fn,
                                                MarkFn mark_fn) {
  const uint32_t area = box.area();
  cnt.scans += area ? 1 : 0;
  cnt.scan_cells += area;
  const uint32_t incl = warp_incl_scan(area, lane);
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  if (total == 0) return;
  sb[lane] = ScanBox{box.x0, box.y0, (uint32_t)max(box.x1 - box.x0 + 1, 1), want, incl};
  __syncwarp();
  for (uint32_t q0 = 0; q0 < total; q0 += 32) {
    const uint32_t q = q0 + lane;
    bool hit = false;
    int xx = 0, yy = 0;
    if (q < total) {
      int lo = 0, hi = 31;  // first lane whose inclusive end exceeds q
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (sb[mid].incl > q) hi = mid; else lo = mid + 1;
      }
      const ScanBox o = sb[lo];
      const uint32_t a = q - (lo ? sb[lo - 1].incl : 0u);  // offset in lane lo's box
      xx = o.x0 + (int)(a % o.bw);
      yy = o.y0 + (int)(a / o.bw);
      float t;
      const uint32_t r = ref_fn(xx, yy, t);
      // a referrer that burns (a cell that does not burn is skipped by its
      // neighbours; requiring it makes the marked set independent of the
      // order of this sweep's commits)
      hit = r == o.want && t < j.max_time && __ldg(j.speed + xx + (int64_t)yy * j.W) != 0.0f;
    }
    mark_fn(hit, xx, yy);
  }
  __syncwarp();
}

__device__ __forceinline__ void sync_cluster() {
  __threadfence();
  cg::this_cluster().sync();
}

// ---- team synchronisation ----
// The CTAs that work on one job meet at every phase boundary: at the hardware
// cluster barrier, or in group mode (G CTAs of a cooperative launch without
// clusters, tiles in global memory) at an arrival word in global memory.
// Group mode alternates between two 64-bit arrival words (barrier k uses
// word k & 1): a CTA arrives with one release reduction adding 1 to the low
// half and, when it improved a cell in the sweep that ends there, 1 to the
// high half; the barrier is complete when the low half reaches the team's
// running target, and the high half's growth since the word's last use is
// the number of CTAs that improved.  The count is exact: a CTA can add to
// word k & 1 again only at barrier k + 2, which no CTA reaches before every
// CTA has arrived at barrier k + 1, i.e. has finished reading barrier k.
// (The low half carries into the high half after 2^32 arrivals on one word,
// billions of sweeps.)  A group wait is bounded: when the other CTAs have
// not all arrived after kGroupWaitNs, or once any CTA of the launch has
// given up, it sets the launch's error flag and returns false, and the
// caller abandons the launch.
constexpr unsigned long long kGroupWaitNs = 2000000000ull;  // 2 s; a phase takes < 50 ms

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void red_release_add_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

struct Team {
  unsigned long long *bar;  // group mode: the two arrival words; null = cluster
  uint32_t *err;            // group mode: the launch's error flag
  int *ok;                  // shared: [0] this CTA's outcome of the last wait, [1] improving CTAs
  uint32_t G;               // CTAs in the group
  uint32_t phase = 0;       // thread 0: barriers passed
  uint32_t target[2] = {0u, 0u};  // thread 0: arrivals expected on each word (low half, modular)
  uint32_t seen[2] = {0u, 0u};    // thread 0: the high half of each word at its last use
  unsigned long long waited = 0;  // thread 0: cycles from arrival to release
  // Cluster mode's count of improving CTAs: three counters in global memory
  // used in rotation by the barriers that count (barrier k: counter k % 3).
  // The cluster's leader clears counter (k + 2) % 3 after barrier k: it was
  // last read right after barrier k - 1, and no CTA adds to it before it has
  // passed barrier k + 1, which the leader reaches after the clear.
  uint32_t *cnt3 = nullptr;
  bool cnt_leader = false;
  uint32_t dsweep = 0;  // every thread: sweeps of global-memory tiles (dirty bitmap rotation)
  uint32_t cnt_phase = 0;  // thread 0: counting barriers passed, mod 3
  // global_fence = false: cluster mode orders shared-memory accesses only.
  // improved: this CTA improved a cell in the phase that ends here;
  // *improving receives the number of the team's CTAs that did.
  __device__ bool sync(bool global_fence = true, bool improved = false, uint32_t *improving = nullptr) {
    const long long t0 = threadIdx.x == 0 ? clock64() : 0;
    if (!bar) {
      if (improving && threadIdx.x == 0 && improved) atomicAdd(cnt3 + cnt_phase, 1u);
      if (global_fence || improving) __threadfence();
      cg::this_cluster().sync();
      if (threadIdx.x == 0) {
        if (improving) {
          ok[1] = (int)__ldcg(cnt3 + cnt_phase);
          if (cnt_leader) cnt3[(cnt_phase + 2) % 3] = 0u;
          cnt_phase = (cnt_phase + 1) % 3;
        }
        waited += (unsigned long long)(clock64() - t0);
      }
      if (improving) {
        __syncthreads();
        *improving = (uint32_t)ok[1];
      }
      return true;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const uint32_t w = phase & 1u;
      ++phase;
      target[w] += G;  // every CTA of the group passes the same barriers
      unsigned long long *word = bar + w;
      // the release orders this CTA's writes (made visible to thread 0 by the
      // CTA barrier above) before the arrival
      red_release_add_u64(word, 1ull | ((unsigned long long)(improved ? 1u : 0u) << 32));
      bool good = true;
      const unsigned long long start_ns = globaltimer_ns();
      unsigned long long v = ld_acquire_u64(word);
      while ((int32_t)((uint32_t)v - target[w]) < 0) {
        if (ld_relaxed_u32(err) != 0u || globaltimer_ns() - start_ns > kGroupWaitNs) {
          good = false;
          break;
        }
        __nanosleep(32);
        v = ld_acquire_u64(word);
      }
      if (!good) atomicOr(err, 1u);
      const uint32_t hi = (uint32_t)(v >> 32);
      ok[0] = good ? 1 : 0;
      ok[1] = (int)(hi - seen[w]);
      seen[w] = hi;
      waited += (unsigned long long)(clock64() - t0);
    }
    __syncthreads();
    if (improving) *improving = (uint32_t)ok[1];
    return ok[0] != 0;
  }
};

// Referrer box update for a cell (x, y) that adopted reference r, in the
// global arrays (fire-and-forget reductions).
__device__ __forceinline__ void box_expand_global(const JobDev &j, uint32_t r, int x, int y) {
  const int64_t rc = ref_x(r) + (int64_t)ref_y(r) * j.W;
  atomicMin(j.box_x0 + rc, (uint32_t)x);
  atomicMin(j.box_y0 + rc, (uint32_t)y);
  atomicMax(j.box_x1 + rc, (uint32_t)x);
  atomicMax(j.box_y1 + rc, (uint32_t)y);
}

struct TileDesc {
  int x0, y0, TW, TH;
};

// ================================================ global-memory tiles ====
// The tile's state stays in global memory (L2), in two copies X0 (the job's
// arrays) and X1: sweep s reads X[s & 1] and writes X[(s + 1) & 1], so that a
// sweep is a single phase between two team barriers.  The cells are dealt to
// the team's R CTAs by 32-cell words of the dirty bitmap, word w to CTA
// w % R, and only a cell's owner writes it.  In sweep s a CTA
//   1. compacts the marked cells of its words in bitmap D[s & 1] (all its
//      cells on the first sweep) into a work list in shared memory, a chunk
//      of blockDim.x words at a time, clearing the words;
//   2. evaluates them against X[s & 1] and appends its improvements to its
//      update region of parity s & 1;
//   3. copies its improvements of sweep s - 1 (already in X[s & 1]) into
//      X[(s + 1) & 1], then writes this sweep's improvements there, marks
//      the 3x3 neighbourhoods of the burning ones in D[(s + 1) & 1] and scans
//      their referrer boxes (reading X[s & 1]);
//   4. adds its improvement count to the team's and meets the team.
// After a sweep without improvements both copies hold the same state.  Marks
// are bit reductions without a return value; the improvement count is the
// only global atomic a CTA makes per sweep.  The referrer scans read the
// references as the sweep started: a referrer whose reference changes in this
// sweep improved, so its neighbourhood is marked anyway, and one that did not
// reads the same reference either way -- the marks are those of scans run
// after the commits.

// Marks the 3x3 neighbourhood of tile cell (lx, ly), centre excluded, in the
// dirty bitmap: per row the (up to) three cells are consecutive bits, so a
// row takes one reduction, two where it straddles a word.
__device__ __forceinline__ void mark3x3_bits(uint32_t *dirty, int lx, int ly, int TW, int TH) {
  const int xa = max(lx - 1, 0), xb = min(lx + 1, TW - 1);  // columns of the 3x3 inside the tile
  if (xa > xb) return;
#pragma unroll
  for (int dy = -1; dy <= 1; ++dy) {
    const int ay = ly + dy;
    if (ay < 0 || ay >= TH) continue;
    const uint32_t k0 = (uint32_t)xa + (uint32_t)ay * (uint32_t)TW;
    // bits of columns xa..xb, without the centre on the middle row
    uint32_t run = (1u << (xb - xa + 1)) - 1u;
    if (dy == 0 && lx >= xa && lx <= xb) run &= ~(1u << (lx - xa));
    const uint32_t w = k0 >> 5, b = k0 & 31;
    const uint32_t lo = run << b;
    if (lo) atomicOr(dirty + w, lo);
    if (b + (uint32_t)(xb - xa) >= 32) {
      const uint32_t hi = run >> (32 - b);
      if (hi) atomicOr(dirty + w + 1, hi);
    }
  }
}

// As mark3x3_bits, and the neighbours outside the tile (inside the grid) into
// the grid-wide pending bitmap (one reduction per cell: only cells on or
// beyond the tile's border have such neighbours).  (lx, ly) may lie anywhere
// in the grid, relative to the tile's corner (x0, y0).
__device__ __forceinline__ void mark3x3_pending(uint32_t *dirty, uint32_t *pending, const JobDev &j,
                                                int x0, int y0, int lx, int ly, int TW, int TH) {
  mark3x3_bits(dirty, lx, ly, TW, TH);
  if (lx > 0 && ly > 0 && lx < TW - 1 && ly < TH - 1) return;
#pragma unroll
  for (int t = 0; t < 9; ++t) {
    const int ax = lx + t % 3 - 1, ay = ly + t / 3 - 1;
    if (t == 4 || (ax >= 0 && ay >= 0 && ax < TW && ay < TH)) continue;
    const int gx = x0 + ax, gy = y0 + ay;
    if (gx < 0 || gy < 0 || gx >= j.W || gy >= j.H) continue;
    const int64_t g = gx + (int64_t)gy * j.W;
    atomicOr(pending + (g >> 5), 1u << (g & 31));
  }
}

// Takes (reads and clears) the pending bits of tile cells k0 .. k0 + n - 1
// (n <= 32, tile-linear order) selected by mask (bit i: cell k0 + i) from
// the grid-wide bitmap; bit i of the result is cell k0 + i.  The cells of one tile row are consecutive grid
// cells, so each row segment is a funnel shift of two words.
__device__ __forceinline__ uint32_t take_pending(uint32_t *pending, const JobDev &j, int x0, int y0,
                                                 int TW, uint32_t k0, uint32_t n, uint32_t mask) {
  uint32_t out = 0, done = 0;
  while (done < n) {
    const uint32_t k = k0 + done;
    const uint32_t lx = k % (uint32_t)TW, ly = k / (uint32_t)TW;
    const uint32_t seg = min(n - done, (uint32_t)TW - lx);  // cells left in this row
    const int64_t g = (x0 + (int64_t)lx) + (int64_t)(y0 + (int64_t)ly) * j.W;
    const int64_t wi = g >> 5;
    const uint32_t sh = (uint32_t)(g & 31);
    const bool two = sh + seg > 32;  // the segment reaches the next word (same row)
    const uint64_t w2 =
        (uint64_t)__ldcg(pending + wi) | (two ? (uint64_t)__ldcg(pending + wi + 1) << 32 : 0ull);
    const uint32_t m = seg >= 32 ? 0xFFFFFFFFu : (1u << seg) - 1u;
    const uint32_t bits = (uint32_t)(w2 >> sh) & m & (mask >> done);
    if (bits) {
      const uint64_t cm = (uint64_t)bits << sh;
      if ((uint32_t)cm) atomicAnd(pending + wi, ~(uint32_t)cm);
      if ((uint32_t)(cm >> 32)) atomicAnd(pending + wi + 1, ~(uint32_t)(cm >> 32));
    }
    out |= bits << done;
    done += seg;
  }
  return out;
}

struct SweepCtx {
  bool leader;
  Counters cnt;
  unsigned long long sweeps = 0, improvements = 0, max_sweeps = 0;
  unsigned long long cyc[4] = {0, 0, 0, 0};  // first sweeps, evaluate, commit, staging
  long long t_phase = 0;
  bool abort = false;
  bool failed = false;  // a group wait gave up (implies abort)
  __device__ __forceinline__ void tick(int phase) {
    if (leader) {
      const long long now = clock64();
      cyc[phase] += (unsigned long long)(now - t_phase);
      t_phase = now;
    }
  }
};

// Ownership of a global-memory tile's cells: the tile-linear cells are cut
// into groups of kOwnGroup consecutive cells, and group g belongs to CTA
// g mod R of the team, so that the cells of a front spread over the CTAs
// while a CTA's cells still come in short runs (its neighbour reads share
// L1 lines).  Tile word w (cells 32 w .. 32 w + 31) holds kGroupsPerWord
// groups; CTA `rank` owns those at offsets first, first + R, ... of the word.
// Groups of 4 cells measured fastest on the 4096^2 scenario with 148 CTAs
// (769 ms; 1 cell: 787 ms; whole 32-cell words dealt round-robin, with
// the scan of every word: slower still).
constexpr uint32_t kOwnGroup = 4;  // a power of two, at most 32
constexpr uint32_t kGroupsPerWord = 32u / kOwnGroup;
__device__ __forceinline__ uint32_t owned_first(uint32_t w, uint32_t rank, uint32_t R) {
  return (rank + R - (w * kGroupsPerWord) % R) % R;  // offset of the first owned group of word w
}
__device__ __forceinline__ uint32_t owned_mask(uint32_t first, uint32_t R) {
  constexpr uint32_t g = kOwnGroup == 32u ? 0xFFFFFFFFu : (1u << kOwnGroup) - 1u;
  uint32_t m = 0;
  for (uint32_t i = first; i < kGroupsPerWord; i += R) m |= g << (i * kOwnGroup);
  return m;
}
// Owned cells of one word at most: kOwnGroup per owned group.
__host__ __device__ inline uint32_t owned_per_word(uint32_t R) {
  return kOwnGroup * ((kGroupsPerWord + R - 1) / R);
}
constexpr int kScanBatch = 8;  // dirty words a thread loads at once

// A global-memory tile's update entries of one sweep: this CTA's first
// kTileUpdSmem in shared memory, the rest in its global update region.
__device__ __forceinline__ TileUpdate get_update(const TileUpdate *sm_upd, const TileUpdate *g_upd,
                                                 uint32_t u) {
  if (u < (uint32_t)kTileUpdSmem) return sm_upd[u];
  const uint4 *q = reinterpret_cast<const uint4 *>(g_upd + u);
  const uint4 a = __ldcg(q), b = __ldcg(q + 1);
  return TileUpdate{a.x, __uint_as_float(a.y), a.z, a.w, b.x, b.y, 0u, 0u};
}

// One tile launch with the state in global memory, by a team of R CTAs
// (this one is `rank`).  `list` is shared memory for blockDim.x * 32 u16
// entries, `sm_upd` for two sweeps' kTileUpdSmem update entries, `cta_ctr`
// two shared counters.  Returns whether any sweep improved a cell.
//
// An update entry carries what the commit needs besides the new time and
// reference: whether the cell burns (its neighbours read it) and its
// referrer box, both read while the cell is evaluated, so that the commit
// makes no dependent global reads.  The box read then (before or during
// other CTAs' commits of the sweep) holds every referrer adopted in earlier
// sweeps (their growth happened before the last barrier); referrers that
// adopt the cell in this sweep improved, and mark their neighbourhoods
// themselves.  Concurrent growth can only widen the box (a box created in
// this sweep may show the empty marker in a corner: corners are clamped to
// the grid), which costs scan work, never a mark: a scan hits the cells that
// referenced the cell when the sweep started.  With a pending bitmap the
// scans read referrers outside the launching tile too, from X[p]: a launch
// writes only its tile's cells, and both copies agree everywhere when a
// launch ends, so outside the tile X[0] and X[1] hold the same state.
__device__ bool tile_global(const JobDev &j, const DirConst &dc, const SlotDev &s, const TileDesc &td,
                            ScanBox *scan_boxes, uint32_t *list, TileUpdate *sm_upd, uint32_t *cta_ctr,
                            uint32_t rank, uint32_t R, SweepCtx &cx, Team &team) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int x0 = td.x0, y0 = td.y0, TW = td.TW, TH = td.TH;
  const uint32_t TN = (uint32_t)TW * (uint32_t)TH;
  const uint32_t nwords = (TN + 31) / 32;
  // a chunk of words yields at most the list's capacity of owned cells: the
  // whole tile when this CTA's share fits, else a bounded run of words
  const uint32_t cap = global_tile_upd_cap(TN, R);
  const uint32_t chunk_words = cap <= global_tile_list_cap(blockDim.x)
                                   ? nwords
                                   : global_tile_list_cap(blockDim.x) / owned_per_word(R);
  float *const tm[2] = {j.time, j.time1};
  uint32_t *const rf[2] = {j.refs, j.refs1};
  // the launch's counters in registers (the context may live in local memory)
  Counters cnt = cx.cnt;
  bool first = true, worked = false;
  uint32_t prev_upd = 0;  // this CTA's improvements of the previous sweep
  int p = 0;              // sweep parity: read X[p], write X[p ^ 1]
  for (;;) {
    ++cx.sweeps;  // every thread counts, so the abort below is uniform
    const float *const rt = tm[p];
    const uint32_t *const rr = rf[p];
    float *const wt = tm[p ^ 1];
    uint32_t *const wr = rf[p ^ 1];
    // dirty bitmaps in rotation by the team's sweep count d: read D[d % 3],
    // mark D[(d + 1) % 3], clear D[(d + 2) % 3] (read in sweep d - 1)
    const uint32_t dsw = team.dsweep++;
    uint32_t *const dirty = s.dirty + (size_t)(dsw % 3) * s.dirty_words;
    uint32_t *const dirty_next = s.dirty + (size_t)((dsw + 1) % 3) * s.dirty_words;
    uint32_t *const dirty_old = s.dirty + (size_t)((dsw + 2) % 3) * s.dirty_words;
    TileUpdate *const upd = s.upd + ((size_t)p * R + rank) * cap;
    const TileUpdate *const upd_prev = s.upd + ((size_t)(p ^ 1) * R + rank) * cap;
    TileUpdate *const supd = sm_upd + p * kTileUpdSmem;
    const TileUpdate *const supd_prev = sm_upd + (p ^ 1) * kTileUpdSmem;
    // ---- 1, 2: compact and evaluate (nothing is written to X[p]) ----
    // the bitmap read two sweeps ago is cleared now (its marks come in the
    // next sweep): the words w = rank mod R of the slot's bitmap
    for (uint32_t w = rank + threadIdx.x * R; w < s.dirty_words; w += blockDim.x * R) dirty_old[w] = 0u;
    if (threadIdx.x == 0) cta_ctr[1] = 0;
    for (uint32_t c0 = 0; c0 < nwords; c0 += chunk_words) {
      __syncthreads();  // the previous chunk's list is consumed
      if (threadIdx.x == 0) cta_ctr[0] = 0;
      __syncthreads();
      const uint32_t c1 = min(nwords, c0 + chunk_words);
      // this thread's words w = c0 + threadIdx.x + i blockDim.x, in batches of
      // kScanBatch whose loads all go out before any is used; the offset of
      // the first owned group of word w steps by a constant from one word to
      // the next of the thread
      uint32_t fo = owned_first(c0 + threadIdx.x, rank, R);
      const uint32_t fstep = (R - (kGroupsPerWord * blockDim.x) % R) % R;
      for (uint32_t wb = c0 + threadIdx.x; wb < c1; wb += kScanBatch * blockDim.x) {
        uint32_t v[kScanBatch];
#pragma unroll
        for (int i = 0; i < kScanBatch; ++i) {
          const uint32_t w = wb + (uint32_t)i * blockDim.x;
          v[i] = 0u;
          if (w < c1) {
            if (!first) {
              v[i] = __ldcg(dirty + w);
            } else if (!j.pending) {  // the whole tile
              const uint32_t nb = (w == nwords - 1 && (TN & 31)) ? (TN & 31) : 32u;
              v[i] = nb == 32 ? 0xFFFFFFFFu : (1u << nb) - 1u;
            }
          }
        }
#pragma unroll
        for (int i = 0; i < kScanBatch; ++i) {
          const uint32_t w = wb + (uint32_t)i * blockDim.x;
          const uint32_t own = owned_mask(fo, R);
          fo += fstep;
          if (fo >= R) fo -= R;
          if (w >= c1) continue;
          uint32_t bits = v[i] & own;
          if (first && j.pending) {
            // the cells whose inputs changed since their last evaluation
            const uint32_t nb = (w == nwords - 1 && (TN & 31)) ? (TN & 31) : 32u;
            bits = take_pending(j.pending, j, x0, y0, TW, w * 32, nb, own);
          }
          if (bits) {
            uint32_t at = atomicAdd(cta_ctr + 0, (uint32_t)__popc(bits));
            for (; bits; bits &= bits - 1) list[at++] = w * 32 + (uint32_t)(__ffs(bits) - 1);
          }
        }
      }
      __syncthreads();
      const uint32_t nlist = cta_ctr[0];
      if (threadIdx.x == 0) cnt.evals += nlist;
      // four cells per warp, eight lanes per cell
      for (uint32_t base = warp * 4; base < nlist; base += nwarps * 4) {
        const uint32_t ci = base + (lane >> 3);
        const bool valid = ci < nlist;
        uint32_t k = 0;
        int x = 0, y = 0;
        Best own{FLT_MAX, kNoRef};
        uint32_t bx0 = kEmptyBox, by0 = 0, bx1 = 0, by1 = 0;
        float own_speed = 0.0f;
        if (valid) {
          k = list[ci];
          x = x0 + (int)(k % (uint32_t)TW);
          y = y0 + (int)(k / (uint32_t)TW);
          const int64_t c = x + (int64_t)y * j.W;
          own = Best{__ldcg(rt + c), __ldcg(rr + c)};
          if ((lane & 7) == 0) {  // what the commit needs if the cell improves
            own_speed = __ldg(j.speed + c);
            bx0 = __ldcg(j.box_x0 + c);
            by0 = __ldcg(j.box_y0 + c);
            bx1 = __ldcg(j.box_x1 + c);
            by1 = __ldcg(j.box_y1 + c);
          }
        }
        const Best b = evaluate_coop(j, dc, GlobalAcc{j, rt, rr}, x, y, own, valid, lane, cnt);
        const bool improved = valid && (lane & 7) == 0 && b.time < own.time;
        const uint32_t ai = warp_append(cta_ctr + 1, improved ? 1u : 0u, lane);
        if (improved) {
          Box box{1, 1, 0, 0};
          if (bx0 != kEmptyBox) {
            if (j.pending)  // the whole box: referrers anywhere mark pending cells
              box = Box{max((int)bx0, 0), max((int)by0, 0), min((int)bx1, j.W - 1), min((int)by1, j.H - 1)};
            else
              box = clip_box((int)bx0, (int)by0, (int)bx1, (int)by1, x0, y0, TW, TH, j.W, j.H);
          }
          // corners in 16 bits (grids up to 65534 cells a side); an empty box
          // as x0 = 0xFFFF > x1
          const bool empty = box.x0 > box.x1 || box.y0 > box.y1;
          const uint32_t b01 = empty ? 0xFFFFu : (uint32_t)box.x0 | ((uint32_t)box.y0 << 16);
          const uint32_t b23 = empty ? 0u : (uint32_t)box.x1 | ((uint32_t)box.y1 << 16);
          // only a burning cell is read by its neighbours
          const uint32_t burn = b.time < j.max_time && own_speed != 0.0f ? 1u : 0u;
          if (ai < (uint32_t)kTileUpdSmem) {
            supd[ai] = TileUpdate{k, b.time, b.ref, burn, b01, b23, 0u, 0u};
          } else {
            uint4 *q = reinterpret_cast<uint4 *>(upd + ai);
            q[0] = make_uint4(k, __float_as_uint(b.time), b.ref, burn);
            q[1] = make_uint4(b01, b23, 0u, 0u);
          }
        }
      }
    }
    __syncthreads();
    const uint32_t my_upd = cta_ctr[1];
    // ---- 3a: the previous sweep's improvements into X[p ^ 1] ----
    for (uint32_t u = threadIdx.x; u < prev_upd; u += blockDim.x) {
      const TileUpdate e = get_update(supd_prev, upd_prev, u);
      const int64_t c = (x0 + (int)(e.k % (uint32_t)TW)) + (int64_t)(y0 + (int)(e.k / (uint32_t)TW)) * j.W;
      wt[c] = e.time;
      wr[c] = e.ref;
    }
    __syncthreads();  // this sweep's improvements of the same cells land after
    // ---- 3b: commit (update_point / commit_point), mark, referrer scans.
    // Updates are dealt `per` to a warp, as few as spreads them over the
    // CTA's warps (a warp's referrer scans run one after another).
    const uint32_t per = min(32u, (my_upd + nwarps - 1) / nwarps);
    for (uint32_t base = warp * per; base < my_upd; base += nwarps * per) {
      const uint32_t u = base + lane;
      const bool valid = lane < per && u < my_upd;
      uint32_t want = 0;
      Box box{1, 1, 0, 0};
      if (valid) {
        const TileUpdate e = get_update(supd, upd, u);
        const int lx = (int)(e.k % (uint32_t)TW), ly = (int)(e.k / (uint32_t)TW);
        const int x = x0 + lx, y = y0 + ly;
        const int64_t c = x + (int64_t)y * j.W;
        wt[c] = e.time;
        wr[c] = e.ref;
        box_expand_global(j, e.ref, x, y);
        if (e.burn) {
          if (j.pending)
            mark3x3_pending(dirty_next, j.pending, j, x0, y0, lx, ly, TW, TH);
          else
            mark3x3_bits(dirty_next, lx, ly, TW, TH);
        }
        want = pack_ref(x, y);
        if ((e.b01 & 0xFFFFu) != 0xFFFFu)
          box = Box{(int)(e.b01 & 0xFFFFu), (int)(e.b01 >> 16), (int)(e.b23 & 0xFFFFu), (int)(e.b23 >> 16)};
      }
      warp_scan_boxes(
          scan_boxes + (threadIdx.x & ~31u), box, want, j, lane, cnt,
          [&](int xx, int yy, float &t) {
            const int64_t n = xx + (int64_t)yy * j.W;
            t = __ldcg(rt + n);
            return __ldcg(rr + n);
          },
          [&](bool hit, int xx, int yy) {
            if (!hit) return;
            if (j.pending)
              mark3x3_pending(dirty_next, j.pending, j, x0, y0, xx - x0, yy - y0, TW, TH);
            else
              mark3x3_bits(dirty_next, xx - x0, yy - y0, TW, TH);
          });
    }
    // ---- 4: meet; the barrier reports how many CTAs improved a cell ----
    uint32_t improving = 0;
    if (!team.sync(true, my_upd > 0, &improving)) {
      cx.failed = cx.abort = true;
      break;
    }
    cx.tick(first ? 0 : 1);
    if (threadIdx.x == 0) cx.improvements += my_upd;  // summed over the team at the job's end
    if (improving == 0) break;  // X[p ^ 1] got the last improvements: both copies agree
    worked = true;
    prev_upd = my_upd;
    p ^= 1;
    first = false;
    if (cx.sweeps > cx.max_sweeps) {
      cx.abort = true;
      break;
    }
  }
  cx.cnt = cnt;
  return worked;
}

// ================================================ shared-memory tiles ====
// Cell slots of the tile and its halo: halo coordinates hx in [0, TW + 2),
// hy in [0, TH + 2) (grid x = x0 - 1 + hx, y = y0 - 1 + hy); row hy lives in
// CTA hy % C at local row hy / C.
struct SmemTile {
  float *time;
  uint32_t *ref;
  // referrer box of each slot restricted to the staged region, in the job's
  // codec (BoxCoarse or BoxExact); the codec's kEmpty when no referrer lies
  // inside
  void *box;
  uint16_t *list;   // this sweep's cells to evaluate (local slot index); kSmemListCap
  uint16_t *uidx;   // pending updates: local slot, time, reference; kSmemUpdCap
  float *utime;
  uint32_t *uref;
  uint32_t *dirty;  // bit per local slot: evaluate in the next sweep
  uint32_t *grown;  // bit per local slot: a referrer joined its staged box in this launch
  uint32_t *ctr;    // [0] list size, [1] local updates, [2..3] cluster updates (parity)
  uint16_t *ovf_list;  // this CTA's global overflow of list / updates
  Update *ovf_upd;
};

__device__ __forceinline__ SmemTile carve_smem(char *base, int cap, int box_bytes, const SlotDev &s,
                                              int rank) {
  SmemTile t;
  t.box = base;  // first: 8-byte aligned for BoxExact
  base += (size_t)cap * box_bytes;
  t.time = (float *)base;
  base += (size_t)cap * 4;
  t.ref = (uint32_t *)base;
  base += (size_t)cap * 4;
  t.utime = (float *)base;
  base += (size_t)kSmemUpdCap * 4;
  t.uref = (uint32_t *)base;
  base += (size_t)kSmemUpdCap * 4;
  t.list = (uint16_t *)base;
  base += (size_t)kSmemListCap * 2;
  t.uidx = (uint16_t *)base;
  base += (size_t)kSmemUpdCap * 2;
  t.dirty = (uint32_t *)(((uintptr_t)base + 3) & ~(uintptr_t)3);
  base = (char *)(t.dirty + (cap / 32 + 1));
  t.grown = (uint32_t *)base;
  base = (char *)(t.grown + (cap / 32 + 1));
  t.ctr = (uint32_t *)(((uintptr_t)base + 15) & ~(uintptr_t)15);
  t.ovf_list = s.ovf_list + (size_t)rank * s.ovf_cap;
  t.ovf_upd = s.ovf_upd + (size_t)rank * s.ovf_cap;
  return t;
}

// Work-list and update-list entries: shared memory first, then the overflow.
__device__ __forceinline__ void list_put(const SmemTile &t, uint32_t i, uint32_t slot) {
  if (i < (uint32_t)kSmemListCap)
    t.list[i] = (uint16_t)slot;
  else
    t.ovf_list[i - kSmemListCap] = (uint16_t)slot;
}
__device__ __forceinline__ uint32_t list_get(const SmemTile &t, uint32_t i) {
  return i < (uint32_t)kSmemListCap ? t.list[i] : __ldcg(t.ovf_list + (i - kSmemListCap));
}
__device__ __forceinline__ void upd_put(const SmemTile &t, uint32_t i, uint32_t slot, float time,
                                        uint32_t ref) {
  if (i < (uint32_t)kSmemUpdCap) {
    t.uidx[i] = (uint16_t)slot;
    t.utime[i] = time;
    t.uref[i] = ref;
  } else {
    t.ovf_upd[i - kSmemUpdCap] = Update{slot, time, ref, 0u};
  }
}
__device__ __forceinline__ void upd_get(const SmemTile &t, uint32_t i, uint32_t &slot, float &time,
                                        uint32_t &ref) {
  if (i < (uint32_t)kSmemUpdCap) {
    slot = t.uidx[i];
    time = t.utime[i];
    ref = t.uref[i];
  } else {
    const Update u = t.ovf_upd[i - kSmemUpdCap];
    slot = u.k;
    time = u.time;
    ref = u.ref;
  }
}

// Staged referrer-box codecs.  A box is [hx0, hx1] x [hy0, hy1] in halo-local
// cells; grow() adds one cell with a compare-and-swap loop (per-field min of
// the low corner, max of the high corner).
//   BoxCoarse: one u32, a byte per corner in units of 1 << sh cells, decoded
//              rounded outwards (4 bytes per slot; halo sides up to 510);
//   BoxExact:  one u64, 16 bits per corner (8 bytes per slot).
struct BoxCoarse {
  using T = uint32_t;
  static constexpr T kEmpty = 0x0000FFFFu;  // x0 = y0 = 255, x1 = y1 = 0
  static __device__ __forceinline__ T pack(int hx0, int hy0, int hx1, int hy1, int sh) {
    return (T)(hx0 >> sh) | ((T)(hy0 >> sh) << 8) | ((T)(hx1 >> sh) << 16) | ((T)(hy1 >> sh) << 24);
  }
  static __device__ __forceinline__ void grow(T *w, int hx, int hy, int sh) {
    const uint32_t px = (uint32_t)(hx >> sh), py = (uint32_t)(hy >> sh);
    const uint32_t lo = px | (py << 8) | 0xFFFF0000u;
    const uint32_t hi = (px << 16) | (py << 24);
    T o = *w;
    for (;;) {
      const T nw = (__vminu4(o, lo) & 0x0000FFFFu) | (__vmaxu4(o, hi) & 0xFFFF0000u);
      if (nw == o) return;
      const T pr = atomicCAS(w, o, nw);
      if (pr == o) return;
      o = pr;
    }
  }
  static __device__ __forceinline__ void decode(T v, int sh, int &hx0, int &hy0, int &hx1, int &hy1) {
    const int m = (1 << sh) - 1;
    hx0 = (int)(v & 0xFFu) << sh;
    hy0 = (int)((v >> 8) & 0xFFu) << sh;
    hx1 = ((int)((v >> 16) & 0xFFu) << sh) + m;
    hy1 = ((int)(v >> 24) << sh) + m;
  }
};

struct BoxExact {
  using T = unsigned long long;
  static constexpr T kEmpty = 0x00000000FFFFFFFFull;  // low corner 0xFFFF, high corner 0
  static __device__ __forceinline__ T pack(int hx0, int hy0, int hx1, int hy1, int) {
    return (T)((uint32_t)hx0 | ((uint32_t)hy0 << 16)) | ((T)((uint32_t)hx1 | ((uint32_t)hy1 << 16)) << 32);
  }
  static __device__ __forceinline__ void grow(T *w, int hx, int hy, int) {
    const uint32_t p = (uint32_t)hx | ((uint32_t)hy << 16);
    T o = *w;
    for (;;) {
      const T nw = (T)__vminu2((uint32_t)o, p) | ((T)__vmaxu2((uint32_t)(o >> 32), p) << 32);
      if (nw == o) return;
      const T pr = atomicCAS(w, o, nw);
      if (pr == o) return;
      o = pr;
    }
  }
  static __device__ __forceinline__ void decode(T v, int, int &hx0, int &hy0, int &hx1, int &hy1) {
    hx0 = (int)(v & 0xFFFFu);
    hy0 = (int)((v >> 16) & 0xFFFFu);
    hx1 = (int)((v >> 32) & 0xFFFFu);
    hy1 = (int)(v >> 48);
  }
};

struct SmemGeom {
  int x0, y0, TW, TH, P, HR, C, rank, rows_mine;
  int sh;    // box_shift: 0 when the halo side fits a byte, else 1
  int lc;    // log2 C (cluster sizes are powers of two): row hy -> CTA hy & (C-1), local row hy >> lc
  uint32_t pm;  // ceil(2^32 / P): s / P = umulhi(s, pm), exact for s < 2^16 and P < 2^12
  __device__ __forceinline__ int owner(int hy) const { return hy & (C - 1); }
  __device__ __forceinline__ int lrow(int hy) const { return hy >> lc; }
  uint32_t tm;  // the same for TW
  __device__ __forceinline__ int div_p(int s) const { return (int)__umulhi((uint32_t)s, pm); }
  __device__ __forceinline__ int div_tw(int s) const { return (int)__umulhi((uint32_t)s, tm); }
};

template <typename T>
__device__ __forceinline__ T *rank_ptr(T *local, int r) {
  return cg::this_cluster().map_shared_rank(local, (unsigned)r);
}

// Marks the tile cells of the 3x3 neighbourhood of halo cell (hx, hy) in
// their owners' dirty bitmaps (fire-and-forget reductions on shared memory).
// A row's (up to) three cells are consecutive slots of one owner: one
// reduction, two where they straddle a word.
__device__ __forceinline__ void mark3x3_smem(const SmemTile &sm, const SmemGeom &g, int hx, int hy) {
  const int xa = max(hx - 1, 1), xb = min(hx + 1, g.TW);  // tile columns (halo coordinates)
  if (xa > xb) return;
#pragma unroll
  for (int dy = -1; dy <= 1; ++dy) {
    const int ay = hy + dy;
    if (ay < 1 || ay > g.TH) continue;
    uint32_t run = (1u << (xb - xa + 1)) - 1u;
    if (dy == 0 && hx >= xa && hx <= xb) run &= ~(1u << (hx - xa));
    if (!run) continue;
    const int owner = g.owner(ay);
    const uint32_t l0 = (uint32_t)(g.lrow(ay) * g.P + xa);
    uint32_t *d = owner == g.rank ? sm.dirty : rank_ptr(sm.dirty, owner);
    const uint32_t w = l0 >> 5, b = l0 & 31;
    const uint32_t lo = run << b;
    if (lo) atomicOr(d + w, lo);
    if (b + (uint32_t)(xb - xa) >= 32) {
      const uint32_t hi = run >> (32 - b);
      if (hi) atomicOr(d + w + 1, hi);
    }
  }
}

__device__ __forceinline__ void smem_cell(const SmemTile &sm, const SmemGeom &g, int hx, int hy,
                                          float &t, uint32_t &r) {
  const int owner = g.owner(hy);
  const int li = g.lrow(hy) * g.P + hx;
  if (owner == g.rank) {
    t = sm.time[li];
    r = sm.ref[li];
  } else {
    t = rank_ptr(sm.time, owner)[li];
    r = rank_ptr(sm.ref, owner)[li];
  }
}

__device__ __forceinline__ float smem_time_of(const JobDev &j, const SmemTile &sm,
                                              const SmemGeom &g, uint32_t r) {
  const int hx = ref_x(r) - (g.x0 - 1), hy = ref_y(r) - (g.y0 - 1);
  if (hx >= 0 && hy >= 0 && hx < g.P && hy < g.HR) {
    const int owner = g.owner(hy);
    const int li = g.lrow(hy) * g.P + hx;
    return owner == g.rank ? sm.time[li] : rank_ptr(sm.time, owner)[li];
  }
  return __ldcg(j.time + ref_x(r) + (int64_t)ref_y(r) * j.W);  // outside: static this launch
}

struct SmemAcc {
  const JobDev &j;
  const SmemTile &sm;
  const SmemGeom &g;
  __device__ __forceinline__ void cell(int x, int y, float &t, uint32_t &r) const {
    smem_cell(sm, g, x - (g.x0 - 1), y - (g.y0 - 1), t, r);
  }
  __device__ __forceinline__ float time_of(uint32_t r) const { return smem_time_of(j, sm, g, r); }
};

// One tile launch resident in the cluster's shared memory; B is the staged
// referrer-box codec.
template <class B>
__device__ bool tile_smem(const JobDev &j, const DirConst &dc, char *smem, const SlotDev &slot,
                          const TileDesc &td, ScanBox *scan_boxes, SweepCtx &cx, Team &team) {
  using BoxT = typename B::T;
  cg::cluster_group cluster = cg::this_cluster();
  SmemGeom g;
  g.x0 = td.x0;
  g.y0 = td.y0;
  g.TW = td.TW;
  g.TH = td.TH;
  g.P = td.TW + 2;
  g.HR = td.TH + 2;
  g.C = (int)cluster.num_blocks();
  g.lc = __ffs(g.C) - 1;
  g.pm = (uint32_t)(0xFFFFFFFFu / (uint32_t)g.P) + 1u;
  g.tm = (uint32_t)(0xFFFFFFFFu / (uint32_t)g.TW) + 1u;
  g.rank = (int)cluster.block_rank();
  g.rows_mine = g.HR > g.rank ? (g.HR - g.rank + g.C - 1) / g.C : 0;
  g.sh = (sizeof(BoxT) == 4 && (g.P > 256 || g.HR > 256)) ? 1 : 0;
  const SmemTile sm = carve_smem(smem, smem_cap(td.TW, td.TH, g.C), (int)sizeof(BoxT), slot, g.rank);
  BoxT *const sbox = (BoxT *)sm.box;
  const uint32_t lane = threadIdx.x & 31;
  const int nslots = g.rows_mine * g.P;
  const int nwords = (nslots + 31) / 32;

  // ---- stage the tile and its halo (state; referrer boxes restricted to
  // the staged region, where this launch's scans look) ----
  for (int s = threadIdx.x; s < nslots; s += blockDim.x) {
    const int lr = g.div_p(s), hx = s - lr * g.P;
    const int hy = g.rank + lr * g.C;
    const int gx = g.x0 - 1 + hx, gy = g.y0 - 1 + hy;
    float t = FLT_MAX;
    uint32_t r = kNoRef;
    BoxT box = B::kEmpty;
    if (gx >= 0 && gy >= 0 && gx < j.W && gy < j.H) {
      const int64_t c = gx + (int64_t)gy * j.W;
      t = __ldcg(j.time + c);
      r = __ldcg(j.refs + c);
      const uint32_t bx0 = __ldcg(j.box_x0 + c);
      if (bx0 != kEmptyBox) {
        const Box b = clip_box((int)bx0, (int)__ldcg(j.box_y0 + c), (int)__ldcg(j.box_x1 + c),
                               (int)__ldcg(j.box_y1 + c), g.x0, g.y0, g.TW, g.TH, j.W, j.H);
        if (b.x0 <= b.x1 && b.y0 <= b.y1)
          box = B::pack(b.x0 - (g.x0 - 1), b.y0 - (g.y0 - 1), b.x1 - (g.x0 - 1), b.y1 - (g.y0 - 1),
                        g.sh);
      }
    }
    sm.time[s] = t;
    sm.ref[s] = r;
    sbox[s] = box;
  }
  for (int w = threadIdx.x; w < nwords; w += blockDim.x) {
    sm.dirty[w] = 0u;
    sm.grown[w] = 0u;
  }
  if (threadIdx.x == 0) sm.ctr[0] = sm.ctr[1] = sm.ctr[2] = sm.ctr[3] = 0u;
  team.sync(false);
  cx.tick(3);

  // the launch's counters in registers (the context may live in local memory)
  Counters cnt = cx.cnt;
  bool first = true, worked = false;
  int par = 0;
  for (;;) {
    ++cx.sweeps;
    // ---- evaluate: this CTA's list (all its tile cells, or its marks) ----
    // The first sweep's list is implicit: the in-tile rows of this CTA
    // (local rows lr_first ..), TW cells each.
    const int lr_first = g.rank == 0 ? 1 : 0;
    const int in_rows = g.TH >= g.rank ? max((g.TH - g.rank) / g.C - lr_first + 1, 0) : 0;
    if (!first) {
      for (int w0 = (int)(threadIdx.x & ~31u); w0 < nwords; w0 += blockDim.x) {
        const int w = w0 + (int)lane;
        uint32_t bits = 0;
        if (w < nwords) {
          bits = sm.dirty[w];
          if (bits) sm.dirty[w] = 0u;
        }
        uint32_t at = warp_append(sm.ctr + 0, __popc(bits), lane);
        for (; bits; bits &= bits - 1) list_put(sm, at++, (uint32_t)(w * 32 + __ffs(bits) - 1));
      }
    }
    __syncthreads();
    const uint32_t nlist = first ? (uint32_t)(in_rows * g.TW) : sm.ctr[0];
    if (threadIdx.x == 0) cnt.evals += nlist;
    // four cells per warp, eight lanes per cell
    for (uint32_t base = (threadIdx.x >> 5) * 4; base < nlist; base += (blockDim.x >> 5) * 4) {
      const uint32_t ci = base + (lane >> 3);
      const bool valid = ci < nlist;
      uint32_t s = 0;
      int x = 0, y = 0;
      Best own{FLT_MAX, kNoRef};
      if (valid) {
        s = first ? (uint32_t)((lr_first + g.div_tw((int)ci)) * g.P + 1 + ((int)ci - g.div_tw((int)ci) * g.TW))
                  : list_get(sm, ci);
        const int lr = g.div_p((int)s), hx = (int)s - lr * g.P, hy = g.rank + lr * g.C;
        x = g.x0 - 1 + hx;
        y = g.y0 - 1 + hy;
        own = Best{sm.time[s], sm.ref[s]};
      }
      const Best b = evaluate_coop(j, dc, SmemAcc{j, sm, g}, x, y, own, valid, lane, cnt);
      const bool improved = valid && (lane & 7) == 0 && b.time < own.time;
      const uint32_t at = warp_append(sm.ctr + 1, improved ? 1u : 0u, lane);
      if (improved) upd_put(sm, at, s, b.time, b.ref);
    }
    __syncthreads();
    if (threadIdx.x == 0 && sm.ctr[1]) atomicAdd(rank_ptr(sm.ctr, 0) + 2 + par, sm.ctr[1]);
    team.sync(false);
    cx.tick(first ? 0 : 1);
    const uint32_t total = rank_ptr(sm.ctr, 0)[2 + par];
    if (total == 0) break;
    worked = true;
    // ---- commit, mark, referrer scans (scans may run concurrently with
    // the commits of the same sweep: see tile_global) ----
    if (cx.leader) {
      sm.ctr[2 + (par ^ 1)] = 0u;  // the next sweep's cluster counter
      cx.improvements += total;
    }
    const uint32_t nupd = sm.ctr[1];
    // updates dealt `per` to a warp (see tile_global)
    const uint32_t nwarps = blockDim.x >> 5;
    const uint32_t per = min(32u, (nupd + nwarps - 1) / nwarps);
    for (uint32_t base = (threadIdx.x >> 5) * per; base < nupd; base += nwarps * per) {
      const uint32_t u = base + lane;
      const bool valid = lane < per && u < nupd;
      uint32_t want = 0;
      Box box{1, 1, 0, 0};
      if (valid) {
        uint32_t s, r;
        float t;
        upd_get(sm, u, s, t, r);
        const int lr = g.div_p((int)s), hx = (int)s - lr * g.P, hy = g.rank + lr * g.C;
        const int x = g.x0 - 1 + hx, y = g.y0 - 1 + hy;
        sm.time[s] = t;
        sm.ref[s] = r;
        // referrer box of r: the staged box inside the staged region (merged
        // into the grid-wide box at the end of the launch), else the
        // grid-wide box in global memory
        const int rhx = ref_x(r) - (g.x0 - 1), rhy = ref_y(r) - (g.y0 - 1);
        if (rhx >= 0 && rhy >= 0 && rhx < g.P && rhy < g.HR) {
          const int owner = g.owner(rhy);
          const int li = g.lrow(rhy) * g.P + rhx;
          // the staged box is rounded outwards, so it may hold (x, y) already
          // while the grid-wide box does not: mark the slot for the merge
          // either way
          B::grow((owner == g.rank ? sbox : rank_ptr(sbox, owner)) + li, hx, hy, g.sh);
          atomicOr((owner == g.rank ? sm.grown : rank_ptr(sm.grown, owner)) + (li >> 5),
                   1u << (li & 31));
        } else {
          box_expand_global(j, r, x, y);
        }
        // only a burning cell is read by its neighbours
        if (t < j.max_time && __ldg(j.speed + x + (int64_t)y * j.W) != 0.0f)
          mark3x3_smem(sm, g, hx, hy);
        want = pack_ref(x, y);
        const BoxT pb = sbox[s];
        if (pb != B::kEmpty) {
          // halo-local corners back to grid cells, then clipped to the
          // staged region and the grid
          int bx0, by0, bx1, by1;
          B::decode(pb, g.sh, bx0, by0, bx1, by1);
          box = clip_box(g.x0 - 1 + bx0, g.y0 - 1 + by0, g.x0 - 1 + bx1, g.y0 - 1 + by1, g.x0, g.y0,
                         g.TW, g.TH, j.W, j.H);
        }
      }
      warp_scan_boxes(
          scan_boxes + (threadIdx.x & ~31u), box, want, j, lane, cnt,
          [&](int xx, int yy, float &t) {
            uint32_t r;
            smem_cell(sm, g, xx - (g.x0 - 1), yy - (g.y0 - 1), t, r);
            return r;
          },
          [&](bool hit, int xx, int yy) {
            if (hit) mark3x3_smem(sm, g, xx - (g.x0 - 1), yy - (g.y0 - 1));
          });
    }
    __syncthreads();
    if (threadIdx.x == 0) sm.ctr[0] = sm.ctr[1] = 0u;
    team.sync(false);
    cx.tick(2);
    par ^= 1;
    first = false;
    if (cx.sweeps > cx.max_sweeps) {
      cx.abort = true;
      break;
    }
  }
  // ---- write the tile's state back (halo times and references are
  // unchanged) and merge the staged boxes that grew into the grid-wide boxes
  // (rounded outwards: a box may cover a cell more than its referrers, which
  // costs scan work, never a missed referrer) ----
  for (int s = threadIdx.x; s < nslots; s += blockDim.x) {
    const int lr = g.div_p(s), hx = s - lr * g.P;
    const int hy = g.rank + lr * g.C;
    const int gx = g.x0 - 1 + hx, gy = g.y0 - 1 + hy;
    if (gx < 0 || gy < 0 || gx >= j.W || gy >= j.H) continue;
    const int64_t c = gx + (int64_t)gy * j.W;
    if (hx >= 1 && hx <= g.TW && hy >= 1 && hy <= g.TH) {
      j.time[c] = sm.time[s];
      j.refs[c] = sm.ref[s];
    }
    if (sm.grown[s >> 5] & (1u << (s & 31))) {
      int bx0, by0, bx1, by1;
      B::decode(sbox[s], g.sh, bx0, by0, bx1, by1);
      atomicMin(j.box_x0 + c, (uint32_t)max(g.x0 - 1 + bx0, 0));
      atomicMin(j.box_y0 + c, (uint32_t)max(g.y0 - 1 + by0, 0));
      atomicMax(j.box_x1 + c, (uint32_t)min(g.x0 - 1 + bx1, j.W - 1));
      atomicMax(j.box_y1 + c, (uint32_t)min(g.y0 - 1 + by1, j.H - 1));
    }
  }
  if (threadIdx.x == 0) sm.ctr[0] = sm.ctr[1] = 0u;
  team.sync();
  cx.tick(3);
  cx.cnt = cnt;
  return worked;
}

// ================================================================ engine ====
// Cluster mode (group == 0): every cluster is one team.  Group mode
// (group = G > 1, launched cooperatively without clusters): CTAs
// [g * G, (g + 1) * G) form team g, which keeps its tiles in global memory
// and meets at the bounded counter barrier of its slot.
__global__ void __launch_bounds__(kEngineThreads, 1) engine_kernel(const JobDev *__restrict__ jobs,
                                                         uint32_t n_jobs,
                                                         const SlotDev *__restrict__ slots,
                                                         uint32_t *__restrict__ queue,
                                                         StatsDev *__restrict__ stats,
                                                         unsigned long long max_sweeps,
                                                         const uint32_t *__restrict__ order,
                                                         uint32_t group) {
  extern __shared__ __align__(16) char dyn_smem[];
  cg::cluster_group cluster = cg::this_cluster();
  const bool grouped = group > 1;
  const uint32_t csize = grouped ? group : cluster.num_blocks();
  const uint32_t slot_id = blockIdx.x / csize;
  const SlotDev s = slots[slot_id];
  const uint32_t rank = grouped ? blockIdx.x % csize : cluster.block_rank();
  const uint32_t tid = rank * blockDim.x + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31;
  __shared__ DirConst dc;
  __shared__ JobDev js;
  __shared__ ScanBox scan_boxes[kEngineThreads];
  __shared__ int team_ok[2];
  __shared__ uint32_t cta_ctr[2];  // global-memory tiles: work list and update counts
  Team team{grouped ? reinterpret_cast<unsigned long long *>(s.ctr + 8) : nullptr, queue + 1,
            team_ok, csize};
  team.cnt3 = s.ctr + 5;  // cluster mode: slot counters 5..7
  team.cnt_leader = rank == 0;
  uint32_t taken = 0xFFFFFFFFu;  // tid 0: the queue position it took last

  for (;;) {
    if (tid == 0) {
      taken = atomicAdd(queue, 1u);
      s.ctr[4] = taken;
      s.ctr[0] = s.ctr[1] = s.ctr[2] = s.ctr[3] = 0;
    }
    if (!team.sync()) break;
    // teams take the jobs in queue order; `order` (when given) maps queue
    // positions to jobs, e.g. largest first so that the longest jobs start early
    const uint32_t q = __ldcg(s.ctr + 4);
    if (q >= n_jobs) return;
    const uint32_t jid = order ? __ldg(order + q) : q;
    if (threadIdx.x == 0) {
      js = jobs[jid];
      dir_consts(js, dc);
    }
    __syncthreads();
    const JobDev &j = js;  // shared-memory copy: frees registers
    StatsDev *st = stats + jid;
    if (tid == 0) st->t_start_ns = globaltimer_ns();
    SweepCtx cx;
    cx.leader = tid == 0;
    cx.max_sweeps = max_sweeps;
    cx.t_phase = clock64();
    unsigned long long rounds = 0, launches = 0;
    for (;;) {  // rounds
      ++rounds;
      bool round_worked = false;
      for (int t = 0; t < j.TX * j.TY && !cx.abort; ++t) {  // tiles, row-major
        ++launches;
        TileDesc td;
        td.x0 = (t % j.TX) * j.T;
        td.y0 = (t / j.TX) * j.T;
        td.TW = min(j.T, j.W - td.x0);
        td.TH = min(j.T, j.H - td.y0);
        const bool w = j.smem_tile == kSmemTileExact
                           ? tile_smem<BoxExact>(j, dc, dyn_smem, s, td, scan_boxes, cx, team)
                       : j.smem_tile == kSmemTileCoarse
                           ? tile_smem<BoxCoarse>(j, dc, dyn_smem, s, td, scan_boxes, cx, team)
                           : tile_global(j, dc, s, td, scan_boxes,
                                         reinterpret_cast<uint32_t *>(dyn_smem),
                                         reinterpret_cast<TileUpdate *>(
                                             dyn_smem + global_tile_list_bytes(blockDim.x)),
                                         cta_ctr, rank, csize, cx, team);
        round_worked |= w;
      }
      if (!round_worked || cx.abort) break;
    }
    // per-job statistics
    Counters &cnt = cx.cnt;
    unsigned long long evals = cnt.evals, scans = cnt.scans, scan_cells = cnt.scan_cells;
    for (int o = 16; o > 0; o >>= 1) {
      cnt.dda += __shfl_xor_sync(kFull, cnt.dda, o);
      cnt.gat += __shfl_xor_sync(kFull, cnt.gat, o);
      cnt.walk_max = max(cnt.walk_max, __shfl_xor_sync(kFull, cnt.walk_max, o));
      scans += __shfl_xor_sync(kFull, scans, o);
      scan_cells += __shfl_xor_sync(kFull, scan_cells, o);
      evals += __shfl_xor_sync(kFull, evals, o);
    }
    if (lane == 0) {
      if (cnt.dda) atomicAdd(&st->dda_steps, (unsigned long long)cnt.dda);
      if (cnt.gat) atomicAdd(&st->gathers, (unsigned long long)cnt.gat);
      if (scans) atomicAdd(&st->refbox_scans, scans);
      if (scan_cells) atomicAdd(&st->scan_cells, scan_cells);
      if (evals) atomicAdd(&st->evaluations, evals);
      if (cnt.walk_max) atomicMax(&st->max_walk, cnt.walk_max);
    }
    // every CTA's own improvements (global-memory tiles), or the cluster's
    // total counted by its leader (shared-memory tiles)
    if (threadIdx.x == 0 && cx.improvements) atomicAdd(&st->improvements, cx.improvements);
    if (cx.leader) {
      st->rounds = rounds;
      st->launches = launches;
      st->sweeps = cx.sweeps;
      st->cyc_first = cx.cyc[0];
      st->cyc_eval = cx.cyc[1];
      st->cyc_commit = cx.cyc[2];
      st->cyc_stage = cx.cyc[3];
      if (cx.abort) st->status = cx.failed ? kStatusGroupTimeout : kStatusSweepLimit;
      st->t_done_ns = globaltimer_ns();
      st->cyc_wait = team.waited;
    }
    if (cx.failed || !team.sync()) break;
  }
  // A group wait gave up: this team's job and every job no team has taken
  // yet are reported failed (the other teams stop at their next wait).
  if (tid == 0) {
    for (uint32_t q = taken; q < n_jobs; q = atomicAdd(queue, 1u))
      stats[order ? __ldg(order + q) : q].status = kStatusGroupTimeout;
  }
}

// ---------------------------------------------------------------- post ----
// post_propagate (propag.cu:110-117): time = FLT_MAX where the cell's own fire
// is null or the time is past max_time; references unpacked into the x/y
// outputs; burned cells counted.
__global__ void __launch_bounds__(256) post_kernel(const JobDev *__restrict__ jobs,
                                                   StatsDev *__restrict__ stats) {
  const JobDev j = jobs[blockIdx.y];
  const int64_t N = (int64_t)j.W * j.H;
  unsigned long long burned = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (int64_t)gridDim.x * blockDim.x) {
    float t = j.time[i];
    if (__ldg(j.speed + i) == 0.0f || t > j.max_time) t = FLT_MAX;
    j.time[i] = t;
    burned += t < FLT_MAX;
    const uint32_t r = j.refs[i];
    if (j.out_rx) j.out_rx[i] = (uint16_t)(r & 0xFFFFu);
    if (j.out_ry) j.out_ry[i] = (uint16_t)(r >> 16);
  }
  for (int o = 16; o > 0; o >>= 1) burned += __shfl_xor_sync(kFull, burned, o);
  if ((threadIdx.x & 31) == 0 && burned) atomicAdd(&stats[blockIdx.y].burned, burned);
}

// ------------------------------------------------------------ launchers ----
static unsigned grid_for(uint64_t cells, int sms) {
  uint64_t blocks = (cells + 255) / 256;
  const uint64_t cap = (uint64_t)sms * 8;
  if (blocks > cap) blocks = cap;
  return blocks ? (unsigned)blocks : 1u;
}

cudaError_t launch_prep(const JobDev *jobs, uint32_t n_jobs, uint64_t max_cells, int sms,
                        cudaStream_t stream) {
  dim3 grid(grid_for(max_cells, sms), n_jobs);
  prep_kernel<<<grid, 256, 0, stream>>>(jobs);
  return cudaGetLastError();
}

cudaError_t launch_ignite(const JobDev *jobs, uint32_t n_jobs, cudaStream_t stream) {
  ignite_kernel<<<n_jobs, 32, 0, stream>>>(jobs);
  return cudaGetLastError();
}

static cudaLaunchConfig_t engine_config(int csize, int threads, unsigned blocks, size_t smem,
                                        cudaLaunchAttribute *attr, cudaStream_t stream) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks, 1, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

static cudaError_t engine_attrs(size_t smem) {
  cudaError_t e = cudaFuncSetAttribute(engine_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(engine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

int engine_threads() { return kEngineThreads; }

cudaError_t engine_max_clusters(int csize, int threads, size_t smem, int *n) {
  cudaError_t e = engine_attrs(smem);
  if (e != cudaSuccess) return e;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = engine_config(csize, threads, (unsigned)csize, smem, attr, 0);
  return cudaOccupancyMaxActiveClusters(n, engine_kernel, &cfg);
}

// group == 0: n_slots clusters of csize CTAs.  group > 1: n_slots teams of
// `group` CTAs in one cooperative launch (all CTAs co-resident, which the
// teams' barriers need; the launch fails rather than run otherwise).
// phantom > 0 (self-test of the bounded wait, one slot only): the team counts
// `phantom` CTAs more than the launch holds, so its barriers never complete.
cudaError_t launch_engine(const JobDev *jobs, uint32_t n_jobs, const SlotDev *slots,
                          uint32_t n_slots, int csize, int threads, size_t smem, uint32_t *queue,
                          StatsDev *stats, unsigned long long max_sweeps, const uint32_t *order,
                          uint32_t group, uint32_t phantom, cudaStream_t stream) {
  cudaError_t e = engine_attrs(smem);
  if (e != cudaSuccess) return e;
  cudaLaunchAttribute attr[1];
  if (group > 1) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(n_slots * group, 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (phantom && n_slots != 1) return cudaErrorInvalidValue;
    return cudaLaunchKernelEx(&cfg, engine_kernel, jobs, n_jobs, slots, queue, stats, max_sweeps,
                              order, group + phantom);
  }
  cudaLaunchConfig_t cfg = engine_config(csize, threads, n_slots * (unsigned)csize, smem, attr, stream);
  return cudaLaunchKernelEx(&cfg, engine_kernel, jobs, n_jobs, slots, queue, stats, max_sweeps, order,
                            0u);
}

cudaError_t launch_post(const JobDev *jobs, uint32_t n_jobs, uint64_t max_cells, int sms,
                        StatsDev *stats, cudaStream_t stream) {
  dim3 grid(grid_for(max_cells, sms), n_jobs);
  post_kernel<<<grid, 256, 0, stream>>>(jobs, stats);
  return cudaGetLastError();
}

}  // namespace propag
