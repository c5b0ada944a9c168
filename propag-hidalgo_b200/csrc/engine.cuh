// Internal interface between the host code and the propagation kernels.
#pragma once

#include <cstdint>

namespace propag {

// One scenario as the device sees it.
struct JobDev {
  int32_t W, H;
  float gdx, gdy, max_time;
  int32_t T;       // tile side in cells (>= max(W, H) means one tile)
  int32_t TX, TY;  // tiles per axis
  int32_t north_up;
  int32_t smem_tile;  // 1: tile launches run resident in the cluster's shared memory
  const float *speed, *az, *ecc;
  float *time;         // state, becomes the output after the post pass
  uint32_t *refs;      // state: packed x | y << 16
  uint32_t *bnd;       // boundary bits (written by the prep pass)
  // referrer box of every cell (the cells that ever adopted it as their
  // reference): min and max corner, 0xFFFFFFFF in box_x0 = empty
  uint32_t *box_x0, *box_y0, *box_x1, *box_y1;
  const void *ignitions;  // PropagIgnition[n_ignitions]
  uint32_t n_ignitions;
  uint32_t pad;
  uint16_t *out_rx, *out_ry;
  uint32_t *out_bnd;   // caller's boundary output (may alias bnd)
};

struct Update {
  uint32_t k;     // cell index inside the tile
  float time;
  uint32_t ref;
  uint32_t pad;
};

// Global-memory scratch of one cluster slot (used by tile launches that do
// not fit in shared memory); capacity = largest such tile area of the batch.
struct SlotDev {
  uint32_t *cand[2];
  uint32_t *dirty;
  uint32_t *scan;
  Update *upd;
  uint32_t *ctr;  // [0..1] ncand, [2] nupd, [3] nscan, [4] job
};

// Per-job statistics accumulated on the device (PropagStats order).
struct StatsDev {
  unsigned long long rounds, launches, sweeps, evaluations, improvements, dda_steps,
      refbox_scans, burned, gathers;
  // SM cycles seen by the cluster leader in each phase (barrier wait
  // included): first sweeps of tile launches, evaluate, commit, staging
  unsigned long long cyc_first, cyc_eval, cyc_commit, cyc_stage;
  uint32_t status, max_walk;
  // device clock (%globaltimer, ns) when a cluster took the job and when its
  // propagation finished
  unsigned long long t_start_ns, t_done_ns;
};

constexpr uint32_t kStatusSweepLimit = 1;

// Shared-memory tile layout: rows of the tile plus its one-cell halo are
// dealt to the cluster's CTAs round-robin (row hy -> CTA hy % C), so that a
// front of any orientation spreads over all CTAs.  Bytes per cell slot:
// time 4, reference 4, referrer box 8, work list 2, pending update 10.
constexpr int kSmemBytesPerCell = 28;
constexpr int kSmemFixedBytes = 256;

__host__ __device__ inline int smem_rows_per_cta(int TH, int C) { return (TH + 2 + C - 1) / C; }
__host__ __device__ inline int smem_cap(int TW, int TH, int C) {
  return smem_rows_per_cta(TH, C) * (TW + 2);
}
__host__ __device__ inline size_t smem_bytes(int TW, int TH, int C) {
  const size_t cap = (size_t)smem_cap(TW, TH, C);
  return cap * kSmemBytesPerCell + (cap / 32 + 1) * 4 + kSmemFixedBytes;
}

}  // namespace propag
