// Arrival-time propagation on B200: boundary/prep pass, ignition scatter,
// the persistent cluster engine and the post mask.
//
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
// Mapping.  One thread-block cluster works on one scenario at a time and
// pulls scenarios from a queue, so a batch of scenarios runs concurrently,
// each on its own cluster, in one launch.  A sweep has three phases
// separated by cluster barriers: evaluate (reads only), commit (writes state,
// marks the next sweep's cells), referrer scans (marks more cells).
// Cluster barriers are hardware barriers: there is no spin-wait anywhere.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>

#include "engine.cuh"
#include "propag_device.cuh"

namespace cg = cooperative_groups;

namespace propag {

// ---------------------------------------------------------------- prep ----
// Boundary bits (find_boundaries) packed with a warp ballot, plus the initial
// state: time = FLT_MAX, no reference, empty referrer boxes.
__global__ void __launch_bounds__(256) prep_kernel(const JobDev *__restrict__ jobs) {
  const JobDev j = jobs[blockIdx.y];
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
      j.time[i] = FLT_MAX;
      j.refs[i] = kNoRef;
      j.box_lo[i] = 0xFFFFFFFFu;
      j.box_hi[i] = 0u;
    }
    const unsigned word = __ballot_sync(0xFFFFFFFFu, b);
    if (lane == 0) j.bnd[w0 >> 5] = word;
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
      const uint32_t r = pack_ref(ign[k].x, ign[k].y);
      j.refs[c] = r;
      j.box_lo[c] = r;
      j.box_hi[c] = r;
    }
  }
}

// -------------------------------------------------------------- engine ----
struct Best {
  float time;
  uint32_t ref;
};

constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __noinline__ bool line_blocked_call(const uint32_t *__restrict__ bnd, int W, int fx,
                                               int fy, int tx, int ty, uint32_t &steps) {
  return line_blocked(bnd, W, fx, fy, tx, ty, steps);
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
  const bool nu = j.north_up != 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int kk = k < 4 ? k : k + 1;
    const int di = kk % 3 - 1, dj = kk / 3 - 1;
    d.bearing[k] = bearing(di, dj, 0, 0, nu);
    d.dist[k] = cell_distance(di, dj, j.gdx, j.gdy);
  }
}

// find_neighbor_which_reaches_first (propag.cu:124-190) on the current state.
// All loads are issued in three independent waves (neighbour times and
// speeds; references; reference times and the rest of the neighbours'
// fire) before the reference's sequential decision logic runs over the
// neighbours in its order, in registers.
__device__ __forceinline__ Best evaluate(const JobDev &j, const DirConst &dc, int x, int y,
                                         uint32_t &dda, uint32_t &gat, uint32_t &walk_max) {
  const int W = j.W, H = j.H;
  const int64_t me = x + (int64_t)y * W;
  Best best{__ldcg(j.time + me), __ldcg(j.refs + me)};
  const bool nu = j.north_up != 0;
  float nt[8], rt[8], fs[8], fa[8], fe[8];
  uint32_t nr[8];
  uint32_t act = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int kk = k < 4 ? k : k + 1;
    const int nx = x + kk % 3 - 1, ny = y + kk / 3 - 1;
    const bool inb = nx >= 0 && ny >= 0 && nx < W && ny < H;
    const int64_t n = nx + (int64_t)ny * W;
    nt[k] = inb ? __ldcg(j.time + n) : FLT_MAX;
    fs[k] = inb ? __ldg(j.speed + n) : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < 8; ++k)
    if (nt[k] < j.max_time && fs[k] != 0.0f) act |= 1u << k;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int kk = k < 4 ? k : k + 1;
    const int64_t n = (x + kk % 3 - 1) + (int64_t)(y + kk / 3 - 1) * W;
    const bool a = (act >> k) & 1u;
    nr[k] = a ? __ldcg(j.refs + n) : kNoRef;
    fa[k] = a ? __ldg(j.az + n) : 0.0f;
    fe[k] = a ? __ldg(j.ecc + n) : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < 8; ++k)
    if (ref_x(nr[k]) == x && ref_y(nr[k]) == y) act &= ~(1u << k);  // its reference is me
#pragma unroll
  for (int k = 0; k < 8; ++k)
    rt[k] = (act >> k) & 1u ? __ldcg(j.time + ref_x(nr[k]) + (int64_t)ref_y(nr[k]) * W) : FLT_MAX;
  gat += __popc(act);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if (!((act >> k) & 1u)) continue;
    const int kk = k < 4 ? k : k + 1;
    const int nx = x + kk % 3 - 1, ny = y + kk / 3 - 1;
    const int rx = ref_x(nr[k]), ry = ref_y(nr[k]);
    const Fire f{fs[k], fa[k], fe[k]};
    const float ntime = step_time(nt[k], dc.dist[k], __fmul_rn(f.speed_max, spread_factor(dc.bearing[k], f)));
    float cand = time_from(rx, ry, rt[k], x, y, f, j.gdx, j.gdy, nu);
    if (cand < ntime && cand < best.time) {
      uint32_t cref = nr[k];
      const uint32_t before = dda;
      const bool blocked = line_blocked_call(j.bnd, W, nx, ny, rx, ry, dda);
      walk_max = max(walk_max, dda - before);
      if (blocked) {
        cref = pack_ref(nx, ny);
        cand = ntime;
      }
      if (cand < best.time) {
        best.time = cand;
        best.ref = cref;
      }
    } else if (ntime < best.time) {
      best.time = ntime;
      best.ref = pack_ref(nx, ny);
    }
  }
  return best;
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

// Marks the 3x3 neighbourhood of tile cell (lx, ly) for the next sweep
// (deduplicated through the dirty bitmap) and appends the new cells to work
// list q.  Called by every lane of a warp; `active` selects the lanes.
__device__ __forceinline__ void mark3x3(const SlotDev &s, int q, bool active, int lx, int ly,
                                        int TW, int TH, uint32_t lane) {
  uint32_t fresh = 0;
  if (active) {
#pragma unroll
    for (int t = 0; t < 9; ++t) {
      const int ax = lx + t % 3 - 1, ay = ly + t / 3 - 1;
      if (ax < 0 || ay < 0 || ax >= TW || ay >= TH) continue;
      const uint32_t k = (uint32_t)ax + (uint32_t)ay * (uint32_t)TW;
      const uint32_t bit = 1u << (k & 31);
      if (!(atomicOr(s.dirty + (k >> 5), bit) & bit)) fresh |= 1u << t;
    }
  }
  uint32_t at = warp_append(s.ctr + q, __popc(fresh), lane);
#pragma unroll
  for (int t = 0; t < 9; ++t) {
    if (fresh & (1u << t)) {
      const int ax = lx + t % 3 - 1, ay = ly + t / 3 - 1;
      s.cand[q][at++] = (uint32_t)ax + (uint32_t)ay * (uint32_t)TW;
    }
  }
}

__device__ __forceinline__ void box_min(uint32_t *w, int x, int y) {
  uint32_t old = __ldcg(w);
  for (;;) {
    const uint32_t ox = old & 0xFFFFu, oy = old >> 16;
    const uint32_t nw = min(ox, (uint32_t)x) | (min(oy, (uint32_t)y) << 16);
    if (nw == old) return;
    const uint32_t prev = atomicCAS(w, old, nw);
    if (prev == old) return;
    old = prev;
  }
}
__device__ __forceinline__ void box_max(uint32_t *w, int x, int y) {
  uint32_t old = __ldcg(w);
  for (;;) {
    const uint32_t ox = old & 0xFFFFu, oy = old >> 16;
    const uint32_t nw = max(ox, (uint32_t)x) | (max(oy, (uint32_t)y) << 16);
    if (nw == old) return;
    const uint32_t prev = atomicCAS(w, old, nw);
    if (prev == old) return;
    old = prev;
  }
}

__device__ __forceinline__ void sync_cluster() {
  __threadfence();
  cg::this_cluster().sync();
}

// Referrer box of a changed cell, clipped to the tile grown by one cell
// (referrers further out have no neighbour inside the tile).
struct Box {
  int x0, y0, x1, y1;
  __device__ __forceinline__ uint32_t area() const {
    return x0 > x1 || y0 > y1 ? 0u : (uint32_t)(x1 - x0 + 1) * (uint32_t)(y1 - y0 + 1);
  }
};

__device__ __forceinline__ Box clipped_box(const JobDev &j, uint32_t c, int tx0, int ty0, int TW,
                                           int TH) {
  const uint32_t lo = __ldcg(j.box_lo + c), hi = __ldcg(j.box_hi + c);
  Box b;
  b.x0 = max(max((int)(lo & 0xFFFFu), tx0 - 1), 0);
  b.y0 = max(max((int)(lo >> 16), ty0 - 1), 0);
  b.x1 = min(min((int)(hi & 0xFFFFu), tx0 + TW), j.W - 1);
  b.y1 = min(min((int)(hi >> 16), ty0 + TH), j.H - 1);
  return b;
}

// One cell of a referrer scan: does (xx, yy) reference `want`?
__device__ __forceinline__ bool refers(const JobDev &j, int xx, int yy, uint32_t want) {
  const int64_t n = xx + (int64_t)yy * j.W;
  return __ldcg(j.refs + n) == want && __ldcg(j.time + n) < FLT_MAX;
}

// One lane's referrer box in the warp's concatenated scan.
struct ScanBox {
  int x0, y0;
  uint32_t bw, want, incl;  // width, packed reference, inclusive end in the concatenation
};

constexpr int kEngineThreads = 512;

__global__ void __launch_bounds__(kEngineThreads, 1) engine_kernel(const JobDev *__restrict__ jobs,
                                                         uint32_t n_jobs,
                                                         const SlotDev *__restrict__ slots,
                                                         uint32_t *__restrict__ queue,
                                                         StatsDev *__restrict__ stats,
                                                         unsigned long long max_sweeps) {
  cg::cluster_group cluster = cg::this_cluster();
  const uint32_t csize = cluster.num_blocks();
  const uint32_t slot_id = blockIdx.x / csize;
  const SlotDev s = slots[slot_id];
  const uint32_t nthreads = csize * blockDim.x;
  const uint32_t tid = cluster.block_rank() * blockDim.x + threadIdx.x;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t gwarp = tid >> 5;
  const bool leader = tid == 0;
  __shared__ DirConst dc;
  __shared__ JobDev js;
  __shared__ ScanBox scan_boxes[kEngineThreads];

  for (;;) {
    if (leader) {
      s.ctr[4] = atomicAdd(queue, 1u);
      s.ctr[0] = s.ctr[1] = s.ctr[2] = s.ctr[3] = 0;
    }
    sync_cluster();
    const uint32_t jid = __ldcg(s.ctr + 4);
    if (jid >= n_jobs) return;
    if (threadIdx.x == 0) {
      js = jobs[jid];
      dir_consts(js, dc);
    }
    __syncthreads();
    const JobDev &j = js;  // shared-memory copy: frees registers
    StatsDev *st = stats + jid;
    uint32_t dda = 0, gat = 0, walk_max = 0;
    unsigned long long rounds = 0, launches = 0, sweeps = 0, evals = 0, improvements = 0,
                       scans = 0;
    unsigned long long cyc[3] = {0, 0, 0};  // first sweeps, evaluate, commit
    long long t_phase = clock64();
    bool abort = false;
    for (;;) {  // rounds
      ++rounds;
      bool round_worked = false;
      for (int t = 0; t < j.TX * j.TY && !abort; ++t) {  // tiles, row-major
        ++launches;
        const int x0 = (t % j.TX) * j.T, y0 = (t / j.TX) * j.T;
        const int TW = min(j.T, j.W - x0), TH = min(j.T, j.H - y0);
        const uint32_t TN = (uint32_t)TW * (uint32_t)TH;
        bool first = true;
        int p = 0;
        for (;;) {  // sweeps
          // ---- evaluate (Jacobi: nothing is written to the state) ----
          const uint32_t nitems = first ? TN : __ldcg(s.ctr + p);
          ++sweeps;  // every thread counts, so the abort below is uniform
          if (leader) {
            s.ctr[p ^ 1] = 0;
            evals += nitems;
          }
          for (uint32_t base = gwarp * 32; base < nitems; base += nthreads) {
            const uint32_t i = base + lane;
            bool improved = false;
            Best b{0.0f, 0u};
            uint32_t k = i;
            if (i < nitems) {
              if (!first) {
                k = __ldcg(s.cand[p] + i);
                atomicAnd(s.dirty + (k >> 5), ~(1u << (k & 31)));
              }
              const int x = x0 + (int)(k % (uint32_t)TW), y = y0 + (int)(k / (uint32_t)TW);
              b = evaluate(j, dc, x, y, dda, gat, walk_max);
              improved = b.time < __ldcg(j.time + x + (int64_t)y * j.W);
            }
            const uint32_t at = warp_append(s.ctr + 2, improved ? 1u : 0u, lane);
            if (improved) s.upd[at] = Update{k, b.time, b.ref, 0u};
          }
          sync_cluster();
          if (leader) {
            const long long now = clock64();
            cyc[first ? 0 : 1] += (unsigned long long)(now - t_phase);
            t_phase = now;
          }
          const uint32_t nupd = __ldcg(s.ctr + 2);
          if (nupd == 0) break;
          round_worked = true;
          // ---- commit (update_point / commit_point), mark, referrer scans ----
          // A referrer scan may run while other cells of this sweep commit: a
          // cell whose reference changes in this sweep is itself marked, and a
          // box only grows, so what the scan must find (referrers from earlier
          // sweeps) is unaffected by the concurrent writes.
          for (uint32_t base = gwarp * 32; base < nupd; base += nthreads) {
            const uint32_t u = base + lane;
            const bool valid = u < nupd;
            int lx = 0, ly = 0;
            uint32_t c = 0;
            Box box{1, 1, 0, 0};
            if (valid) {
              const Update up = s.upd[u];
              lx = (int)(up.k % (uint32_t)TW);
              ly = (int)(up.k / (uint32_t)TW);
              const int x = x0 + lx, y = y0 + ly;
              c = (uint32_t)(x + y * j.W);
              j.time[c] = up.time;
              j.refs[c] = up.ref;
              const int64_t rc = ref_x(up.ref) + (int64_t)ref_y(up.ref) * j.W;
              box_min(j.box_lo + rc, x, y);
              box_max(j.box_hi + rc, x, y);
              if (__ldcg(j.box_lo + c) != 0xFFFFFFFFu) box = clipped_box(j, c, x0, y0, TW, TH);
            }
            mark3x3(s, p ^ 1, valid, lx, ly, TW, TH, lane);
            // referrer scans: the warp walks the concatenation of its lanes'
            // boxes, 32 cells per step, one independent load wave per step
            const uint32_t area = box.area();
            scans += area ? 1 : 0;
            uint32_t incl = area;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
              const uint32_t v = __shfl_up_sync(kFull, incl, o);
              if (lane >= (uint32_t)o) incl += v;
            }
            const uint32_t total = __shfl_sync(kFull, incl, 31);
            if (total == 0) continue;
            ScanBox *sb = scan_boxes + (threadIdx.x & ~31u);
            sb[lane] = ScanBox{box.x0, box.y0, (uint32_t)max(box.x1 - box.x0 + 1, 1),
                               pack_ref((int)(c % (uint32_t)j.W), (int)(c / (uint32_t)j.W)), incl};
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
                hit = refers(j, xx, yy, o.want);
              }
              if (__any_sync(kFull, hit)) mark3x3(s, p ^ 1, hit, xx - x0, yy - y0, TW, TH, lane);
            }
            __syncwarp();
          }
          sync_cluster();
          if (leader) {
            const long long now = clock64();
            cyc[2] += (unsigned long long)(now - t_phase);
            t_phase = now;
            improvements += nupd;
            s.ctr[2] = 0;  // the update list was consumed
          }
          p ^= 1;
          first = false;
          if (sweeps > max_sweeps) {
            abort = true;
            break;
          }
        }
      }
      if (!round_worked || abort) break;
    }
    // per-job statistics
    for (int o = 16; o > 0; o >>= 1) {
      dda += __shfl_xor_sync(kFull, dda, o);
      gat += __shfl_xor_sync(kFull, gat, o);
      walk_max = max(walk_max, __shfl_xor_sync(kFull, walk_max, o));
      scans += __shfl_xor_sync(kFull, scans, o);
    }
    if (lane == 0) {
      if (dda) atomicAdd(&st->dda_steps, (unsigned long long)dda);
      if (gat) atomicAdd(&st->gathers, (unsigned long long)gat);
      if (scans) atomicAdd(&st->refbox_scans, scans);
      if (walk_max) atomicMax(&st->max_walk, walk_max);
    }
    if (leader) {
      st->rounds = rounds;
      st->launches = launches;
      st->sweeps = sweeps;
      st->evaluations = evals;
      st->improvements = improvements;
      st->cyc_first = cyc[0];
      st->cyc_eval = cyc[1];
      st->cyc_commit = cyc[2];
      st->cyc_scan = 0;
      if (abort) st->status = kStatusSweepLimit;
    }
    sync_cluster();
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
  for (int o = 16; o > 0; o >>= 1) burned += __shfl_xor_sync(0xFFFFFFFFu, burned, o);
  if ((threadIdx.x & 31) == 0 && burned) atomicAdd(&stats[blockIdx.y].burned, burned);
}

}  // namespace propag

// ------------------------------------------------------------ launchers ----
namespace propag {

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

static cudaLaunchConfig_t engine_config(int csize, int threads, unsigned blocks,
                                        cudaLaunchAttribute *attr, cudaStream_t stream) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks, 1, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = stream;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = csize;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

cudaError_t engine_max_clusters(int csize, int threads, int *n) {
  cudaError_t e = cudaFuncSetAttribute(engine_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = engine_config(csize, threads, (unsigned)csize, attr, 0);
  return cudaOccupancyMaxActiveClusters(n, engine_kernel, &cfg);
}

cudaError_t launch_engine(const JobDev *jobs, uint32_t n_jobs, const SlotDev *slots,
                          uint32_t n_slots, int csize, int threads, uint32_t *queue,
                          StatsDev *stats, unsigned long long max_sweeps, cudaStream_t stream) {
  cudaError_t e = cudaFuncSetAttribute(engine_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  cudaLaunchAttribute attr[1];
  cudaLaunchConfig_t cfg = engine_config(csize, threads, n_slots * (unsigned)csize, attr, stream);
  return cudaLaunchKernelEx(&cfg, engine_kernel, jobs, n_jobs, slots, queue, stats, max_sweeps);
}

cudaError_t launch_post(const JobDev *jobs, uint32_t n_jobs, uint64_t max_cells, int sms,
                        StatsDev *stats, cudaStream_t stream) {
  dim3 grid(grid_for(max_cells, sms), n_jobs);
  post_kernel<<<grid, 256, 0, stream>>>(jobs, stats);
  return cudaGetLastError();
}

}  // namespace propag
