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
  const float *speed, *az, *ecc;
  float *time;         // state, becomes the output after the post pass
  uint32_t *refs;      // state: packed x | y << 16
  uint32_t *bnd;       // boundary bits (written by the prep pass)
  uint32_t *box_lo;    // referrer box min corner (x | y << 16), 0xFFFFFFFF = empty
  uint32_t *box_hi;    // referrer box max corner
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

// Scratch of one cluster slot; capacity = largest tile area of the batch.
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
  // included): first sweeps of tile launches, evaluate, commit, scans
  unsigned long long cyc_first, cyc_eval, cyc_commit, cyc_scan;
  uint32_t status, max_walk;
};

constexpr uint32_t kStatusSweepLimit = 1;

}  // namespace propag
