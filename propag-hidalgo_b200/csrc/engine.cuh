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
  int32_t smem_tile;  // kSmemTile*: where tile launches keep the tile's state
  int32_t refm;       // 1: the reference's arithmetic in time_from, 0: portable
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
  // Round-down reciprocal of every cell's elliptical speed toward each of its
  // 8 neighbours (plane k: toward the cell whose neighbour k it is), written
  // by the prep pass; null = computed per evaluation instead.  Plane stride
  // tt_plane.
  float *tt;
  int64_t tt_plane;
  // Second copy of the state for global-memory tiles (sweeps alternate
  // between the copies); null when every tile is resident in shared memory.
  float *time1;
  uint32_t *refs1;
  // Grid-wide pending bitmap of global-memory tiles (bit x + y W): cells whose
  // inputs changed since they were last evaluated, outside the tile that
  // changed them; a tile launch's first sweep evaluates only its pending
  // cells.  Null: first sweeps evaluate the whole tile.
  uint32_t *pending;
};

struct Update {
  uint32_t k;     // cell index inside the tile
  float time;
  uint32_t ref;
  uint32_t pad;
};
static_assert(sizeof(Update) == 16, "an update is read back as one 16-byte load");

// An improvement of a global-memory tile's sweep, with what its commit needs:
// burn = the cell burns (time < max_time, own fire not null); its referrer
// box as read during the evaluation, corners (x0, y0), (x1, y1) in 16 bits
// each (b01 = x0 | y0 << 16, b23 = x1 | y1 << 16; x0 = 0xFFFF: empty).
struct TileUpdate {
  uint32_t k;  // cell index inside the tile
  float time;
  uint32_t ref;
  uint32_t burn;
  uint32_t b01, b23;
  uint32_t pad[2];
};
static_assert(sizeof(TileUpdate) == 32, "two 16-byte halves");
// Update entries a CTA keeps in shared memory per sweep parity (the rest go
// to its global update region).
constexpr int kTileUpdSmem = 1024;

// Global-memory scratch of one team slot.  dirty/upd serve tile launches
// whose state stays in global memory: the tile's dirty bitmaps (read by
// every CTA of the team: a tile's cells are dealt to the CTAs in groups) and the
// update arrays (one per sweep parity), CTA r of an R-CTA team using entries
// from (parity * R + r) * cap on (cap = global_tile_upd_cap; the first
// kTileUpdSmem of them stay in shared memory); ovf_list/ovf_upd take the
// work-list and update-list entries of shared-memory tiles beyond their
// shared-memory capacity (ovf_cap entries per CTA of the cluster, CTA r at
// offset r * ovf_cap).
struct SlotDev {
  uint32_t *dirty;        // three bitmaps of dirty_words words (in rotation by sweep)
  uint32_t dirty_words;
  uint32_t pad0;
  TileUpdate *upd;
  // [0..3] shared-memory tiles' counters, [4] job, [5..7] cluster mode's
  // improving-CTA counts of global-memory tiles (rotating by barrier),
  // [8..11] group mode's two 64-bit barrier arrival words
  uint32_t *ctr;
  uint16_t *ovf_list;
  Update *ovf_upd;
  uint32_t ovf_cap;
  uint32_t pad;
};

// Update-array entries a CTA of an R-CTA team may need in one sweep of a
// global-memory tile of TN cells (the cells it owns: groups of up to 32
// consecutive cells dealt round-robin); the team needs R times that, at most
// TN + 32 R.
__host__ __device__ inline uint32_t global_tile_upd_cap(uint32_t TN, uint32_t R) {
  return ((TN + 31) / 32 + R - 1) / R * 32;
}

// Shared memory a CTA needs for a global-memory tile launch: the work list
// of one chunk (tile cell indices, 32 per thread), then two sweeps' update
// entries.
__host__ __device__ inline uint32_t global_tile_list_cap(int threads) { return (uint32_t)threads * 32u; }
__host__ __device__ inline size_t global_tile_list_bytes(int threads) {
  return (size_t)global_tile_list_cap(threads) * 4;
}
__host__ __device__ inline size_t global_tile_smem(int threads) {
  return global_tile_list_bytes(threads) + 2 * kTileUpdSmem * sizeof(TileUpdate);
}

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
  unsigned long long scan_cells, cyc_wait;
};

constexpr uint32_t kStatusSweepLimit = 1;
// a group barrier wait gave up (group mode); the job's results are invalid
constexpr uint32_t kStatusGroupTimeout = 2;

// Shared-memory tile layout: rows of the tile plus its one-cell halo are
// dealt to the cluster's CTAs round-robin (row hy -> CTA hy % C), so that a
// front of any orientation spreads over all CTAs.  Bytes per cell slot:
// time 4, reference 4, referrer box 4 (halo-local corners, one byte each,
// in units of 1 << box_shift cells), a dirty bit and a box-grown bit.  The work list and
// the update list hold kSmemListCap / kSmemUpdCap entries in shared memory
// and spill beyond that to the slot's global overflow arrays.
// With exact referrer boxes (BoxExact, 8 bytes) a slot takes 16 bytes.
constexpr int kSmemBytesPerCell = 12;
constexpr int kSmemBytesPerCellExact = 16;
constexpr int kSmemListCap = 4096;  // u16 slot indices
constexpr int kSmemUpdCap = 2048;   // u16 slot + f32 time + u32 reference
constexpr int kSmemFixedBytes = 256;
constexpr int kSmemMaxSide = 510;  // halo side whose corners fit a byte at box_shift 1

// JobDev::smem_tile
constexpr int32_t kSmemTileGlobal = 0;  // state in global memory (two copies), bitmaps and update regions in the slot
constexpr int32_t kSmemTileCoarse = 1;  // shared memory, BoxCoarse referrer boxes
constexpr int32_t kSmemTileExact = 2;   // shared memory, BoxExact referrer boxes

__host__ __device__ inline int smem_rows_per_cta(int TH, int C) { return (TH + 2 + C - 1) / C; }
__host__ __device__ inline int smem_cap(int TW, int TH, int C) {
  return smem_rows_per_cta(TH, C) * (TW + 2);
}
__host__ __device__ inline size_t smem_bytes(int TW, int TH, int C, bool exact = false) {
  if (TW + 2 > kSmemMaxSide || TH + 2 > kSmemMaxSide) return ~(size_t)0;  // never fits
  const size_t cap = (size_t)smem_cap(TW, TH, C);
  return cap * (exact ? kSmemBytesPerCellExact : kSmemBytesPerCell) + (cap / 32 + 1) * 8 +
         (size_t)kSmemListCap * 2 +
         (size_t)kSmemUpdCap * 10 + kSmemFixedBytes;
}

}  // namespace propag
