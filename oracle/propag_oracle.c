/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle for arrival-time propagation.
 *
 * The reference has no CPU propagation; its only implementation is the CUDA
 * kernel crates/propag/src/propag.cu (+ propag.h) driven by the host loop in
 * crates/propag/src/propag.rs:392-556.  This file restates that algorithm on
 * the CPU.  It is the checker for the tests, `__graft_entry__.smoke()` and
 * `bench.py`'s CPU-baseline leg; the product never links or calls it.
 *
 * Restated pieces (paths relative to the reference project):
 *   - find_boundaries / similar_fires / set_boundary  propag.cu:9-13,296-302,345-375
 *   - load_point (snapshot incl. time[ref] gather)    propag.cu:209-229
 *   - find_neighbor_which_reaches_first               propag.cu:124-190
 *   - update_point / commit_point                     propag.cu:192-207
 *   - time_from                                        propag.cu:269-294
 *   - DDA line walk                                    propag.h:91-135
 *   - Propagator::run sweep loop (Jacobi in a tile)    propag.cu:62-109
 *   - super-grid tile loop until no tile works         propag.rs:404-418,502-536
 *   - post_propagate mask                              propag.cu:110-117
 *
 * Schedule: a "tile" is the area one cooperative launch covers
 * (grid_w * block cells per axis, propag.rs:404-418).  Inside a tile every
 * sweep reads the state left by the previous sweep (the two grid.sync()s of
 * propag.cu:80,95 make it a Jacobi sweep); tiles run one after another in
 * row-major order, each until it stops improving; the whole tile pass repeats
 * until no tile improved.  With one tile covering the grid this is a global
 * Jacobi iteration.
 *
 * Work skipping that keeps results identical: after the first sweep of a
 * launch, a cell is re-evaluated only if one of its inputs changed in the
 * previous sweep: a burning neighbour changed, or the reference of a burning
 * neighbour changed (a reference's time is read by cells far away,
 * propag.cu:221-224; every cell keeps the bounding box of the cells that ever
 * adopted it as their reference, and that box is scanned).  `full` = 1
 * evaluates the whole tile in every sweep; the tests check both modes agree.
 * `full` = 2 also skips work in the first sweep of a launch: a grid-wide
 * pending bitmap keeps the marks that fall outside the launching tile
 * (neighbours of changed cells, and neighbours of referrers found by scanning
 * the whole referrer box instead of the tile grown by one cell), starting
 * from the neighbours of the burning cells; a launch's first sweep evaluates
 * only the tile's pending cells.  A cell whose inputs did not change since
 * its last evaluation cannot improve, so the results, improvements and sweep
 * counts are those of the other modes (the evaluation counts are smaller).
 *
 * Intrinsics: __frcp_rd and __fsqrt_rz are emulated exactly (round-down
 * reciprocal, round-toward-zero square root).  The cosine and arctangent are
 * the portable float routines below (trig = 0), which the device kernel's
 * portable arithmetic evaluates with the same float operations, or libm's
 * cosf/atan2f (trig = 1).  trig = 2 follows the reference kernel as nvcc
 * compiles it: libm's cosf/atan2f standing in for CUDA's __cosf/atan2f (which
 * a CPU cannot reproduce bit for bit) and the three multiply-adds of time_from
 * fused; trig = 3 also takes the cosine and arctangent from tables of the
 * GPU's values (ops_set_tables), so that it follows the reference kernel's
 * arithmetic exactly.  Build with -ffp-contract=off: every other float
 * operation is rounded on its own.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  uint32_t width, height;
  float dx, dy; /* geo transform pixel size; dy < 0 means north-up (propag.cu:274) */
  float max_time;
} ops_settings_t;

/* ---- exact emulation of the directed-rounding intrinsics ------------------ */

/* __frcp_rd: 1/x rounded toward -inf.  f*x is exact in double. */
static inline float rcp_rd(float x) {
  if (isnan(x)) return x;
  if (x == 0.0f) return signbit(x) ? -INFINITY : INFINITY;
  if (isinf(x)) return signbit(x) ? -0.0f : 0.0f;
  double q = 1.0 / (double)x;
  if (q > FLT_MAX) return FLT_MAX;
  float f = (float)q;
  if (isinf(f)) return -INFINITY;
  double p = (double)f * (double)x;
  if (x > 0 ? p > 1.0 : p < 1.0) f = nextafterf(f, -INFINITY);
  return f;
}

/* __fsqrt_rz: square root rounded toward zero (x >= 0 here). */
static inline float sqrt_rz(float x) {
  float s = sqrtf(x);
  if (x > 0.0f && isfinite(s) && (double)s * (double)s > (double)x) s = nextafterf(s, 0.0f);
  return s;
}

/* ---- portable float cosine / arctangent ------------------------------------
 * cos: Cody-Waite reduction by pi/2 (three-part constant, fma), Taylor
 * polynomials on [-pi/4, pi/4].  atan2: octant reduction, atan(t) for
 * t = mn/mx in [0,1], above tan(pi/8) as u = (mn-mx)/(mn+mx) (one division either way), Taylor series to
 * u^19.  Accuracy is checked against libm in the tests (<= 2 ulp). */
static const float PIO2_HI = 1.57079637050628662109375f;
static const float PIO2_MID = -4.37113900018624283e-8f;
static const float PIO2_LO = -1.71512451677125e-15f;
static const float TWO_OVER_PI = 0.636619772367581343f;

static inline float pg_sin_poly(float r) {
  float r2 = r * r;
  float p = fmaf(r2, 2.75573192e-6f, -1.98412698e-4f);
  p = fmaf(r2, p, 8.33333333e-3f);
  p = fmaf(r2, p, -1.66666667e-1f);
  return fmaf(r * r2, p, r);
}
static inline float pg_cos_poly(float r) {
  float r2 = r * r;
  float p = fmaf(r2, -2.75573192e-7f, 2.48015873e-5f);
  p = fmaf(r2, p, -1.38888889e-3f);
  p = fmaf(r2, p, 4.16666667e-2f);
  p = fmaf(r2, p, -0.5f);
  return fmaf(r2, p, 1.0f);
}
float pg_cosf(float x) {
  float ax = fabsf(x);
  float k = rintf(ax * TWO_OVER_PI);
  float r = fmaf(-k, PIO2_HI, ax);
  r = fmaf(-k, PIO2_MID, r);
  r = fmaf(-k, PIO2_LO, r);
  int q = ((int)k) & 3;
  switch (q) {
  case 0: return pg_cos_poly(r);
  case 1: return -pg_sin_poly(r);
  case 2: return -pg_cos_poly(r);
  default: return pg_sin_poly(r);
  }
}
static const float TAN_PI_8 = 0.414213562373095049f;
static const float PI_F = 3.14159265358979323846f;
static const float PIO2_F = 1.57079632679489661923f;
static const float PIO4_F = 0.785398163397448309616f;
float pg_atan2f(float y, float x) {
  float ax = fabsf(x), ay = fabsf(y);
  float mx = ax > ay ? ax : ay;
  float mn = ax > ay ? ay : ax;
  if (mx == 0.0f) return 0.0f;
  /* one division: t = mn / mx, or (t - 1) / (t + 1) formed directly as
   * (mn - mx) / (mn + mx) above tan(pi/8) */
  float base = 0.0f;
  float u;
  if (mn > TAN_PI_8 * mx) {
    u = (mn - mx) / (mn + mx);
    base = PIO4_F;
  } else {
    u = mn / mx;
  }
  float u2 = u * u;
  float p = fmaf(u2, 5.26315789e-2f, -5.88235294e-2f); /*  1/19, -1/17 */
  p = fmaf(u2, p, 6.66666667e-2f);                     /*  1/15 */
  p = fmaf(u2, p, -7.69230769e-2f);                    /* -1/13 */
  p = fmaf(u2, p, 9.09090909e-2f);                     /*  1/11 */
  p = fmaf(u2, p, -1.11111111e-1f);                    /* -1/9  */
  p = fmaf(u2, p, 1.42857143e-1f);                     /*  1/7  */
  p = fmaf(u2, p, -2.00000000e-1f);                    /* -1/5  */
  p = fmaf(u2, p, 3.33333333e-1f);                     /*  1/3  */
  float a = fmaf(-(u * u2), p, u) + base;
  if (ay > ax) a = PIO2_F - a;
  if (x < 0.0f) a = PI_F - a;
  if (y < 0.0f) a = -a;
  return a;
}

/* 0: portable cosine/arctangent above; 1: libm's cosf/atan2f; 2: libm's
 * cosf/atan2f and the reference's contracted sums (see time_from); 3: as 2,
 * with the cosine and arctangent looked up in tables of the GPU's own
 * __cosf and atan2f values (ops_set_tables), which makes this restatement
 * follow the reference kernel's arithmetic bit for bit. */
static int g_trig = 0;

/* trig = 3 tables: cos_tab[b - cos_lo] = __cosf(x) for the float x with bits
 * b in [cos_lo, cos_lo + cos_n), and __cosf(x) = cos_below for the bits below
 * cos_lo (the angles are non-negative; the caller checked that the GPU's
 * values are that constant there); atan_tab[(a + ma) + (b + mb) (2 ma + 1)]
 * = atan2f(a, b) for integers |a| <= ma, |b| <= mb.  A look-up outside a
 * table counts a miss and falls back to libm. */
static const float *g_cos_tab = NULL;
static uint64_t g_cos_n = 0;
static uint32_t g_cos_lo = 0;
static float g_cos_below = 1.0f;
static const float *g_atan_tab = NULL;
static int g_atan_ma = -1, g_atan_mb = -1;
static int64_t g_table_misses = 0;

void ops_set_tables(const float *cos_tab, uint32_t cos_lo, uint64_t cos_n, float cos_below,
                    const float *atan_tab, int ma, int mb) {
  g_cos_tab = cos_tab;
  g_cos_lo = cos_lo;
  g_cos_n = cos_tab ? cos_n : 0;
  g_cos_below = cos_below;
  g_atan_tab = atan_tab;
  g_atan_ma = atan_tab ? ma : -1;
  g_atan_mb = atan_tab ? mb : -1;
  g_table_misses = 0;
}

int64_t ops_table_misses(void) { return __atomic_load_n(&g_table_misses, __ATOMIC_RELAXED); }

static inline float t_cos(float x) {
  if (g_trig == 3) {
    uint32_t b;
    memcpy(&b, &x, sizeof b);
    if (g_cos_tab && b < g_cos_lo) return g_cos_below;
    if (b >= g_cos_lo && (uint64_t)(b - g_cos_lo) < g_cos_n) return g_cos_tab[b - g_cos_lo];
    __atomic_fetch_add(&g_table_misses, 1, __ATOMIC_RELAXED);
    return cosf(x);
  }
  return g_trig ? cosf(x) : pg_cosf(x);
}
static inline float t_atan2(float y, float x) {
  if (g_trig == 3) {
    /* the arguments are cell offsets: integers */
    const int a = (int)y, b = (int)x;
    if ((float)a == y && (float)b == x && a >= -g_atan_ma && a <= g_atan_ma && b >= -g_atan_mb &&
        b <= g_atan_mb)
      return g_atan_tab[(int64_t)(a + g_atan_ma) + (int64_t)(b + g_atan_mb) * (2 * g_atan_ma + 1)];
    __atomic_fetch_add(&g_table_misses, 1, __ATOMIC_RELAXED);
    return atan2f(y, x);
  }
  return g_trig ? atan2f(y, x) : pg_atan2f(y, x);
}

/* ---- state ---------------------------------------------------------------- */

typedef struct {
  const ops_settings_t *s;
  const float *speed, *az, *ecc;
  float *time;
  uint16_t *rx, *ry;
  const uint32_t *bnd;
  void *unused;
} world_t;

typedef struct {
  float time;
  uint16_t rx, ry;
} best_t;

static inline int is_boundary(const uint32_t *b, int64_t ix) { return (b[ix >> 5] >> (ix & 31)) & 1u; }

/* time_from, propag.cu:269-294.  The `1.0` literals make the reference
 * evaluate denom and factor in double; that is kept.  With g_trig >= 2 the
 * three sums that nvcc contracts by default (the reference is built without
 * -fmad=false, crates/propag/build.rs:48-69) are fused multiply-adds:
 * 1.0 - e*cos -> fmaf(-e, cos, 1) (nvcc narrows that double subtraction of a
 * float product to float, exactly, then contracts it), dx*dx + dy*dy ->
 * fmaf(dx, dx, dy*dy) and from.time + distance * rcp -> fmaf(distance, rcp,
 * from.time); trig 0 and 1 round every operation on its own. */
static inline float time_from(const world_t *w, int fx, int fy, float ftime, int tx, int ty,
                              float smax, float azmax, float ecc) {
  const ops_settings_t *s = w->s;
  float azimuth;
  if (s->dy < 0)
    azimuth = t_atan2((float)(tx - fx), (float)(fy - ty));
  else
    azimuth = t_atan2((float)(tx - fx), (float)(ty - fy));
  float angle = fabsf(azimuth - azmax);
  float denom = g_trig >= 2 ? fmaf(-ecc, t_cos(angle), 1.0f) : (float)(1.0 - (double)(ecc * t_cos(angle)));
  float factor = (float)((1.0 - (double)ecc) * (double)rcp_rd(denom));
  float speed = smax * factor;
  float dx = (float)(fx - tx) * s->dx;
  float dy = (float)(fy - ty) * s->dy;
  if (g_trig >= 2) {
    const float distance = sqrt_rz(fmaf(dx, dx, dy * dy));
    return fmaf(distance, rcp_rd(speed), ftime);
  }
  float dx2 = dx * dx;
  float dy2 = dy * dy;
  float distance = sqrt_rz(dx2 + dy2);
  float step = distance * rcp_rd(speed);
  return ftime + step;
}

/* DDA walk from `from` to `to` inclusive (propag.h:91-135); returns 1 if a
 * visited cell is a boundary.  The walk is bounded by |dx|+|dy|+2 visits. */
static int line_blocked(const world_t *w, int fx, int fy, int tx, int ty, int64_t *steps) {
  const int W = (int)w->s->width;
  int sx = (tx > fx) - (tx < fx), sy = (ty > fy) - (ty < fy);
  int cx = fx, cy = fy;
  float tmx = (float)(1.0 / (double)(float)abs(tx - fx));
  float tmy = (float)(1.0 / (double)(float)abs(ty - fy));
  const float ddx = tmx, ddy = tmy;
  int64_t limit = (int64_t)abs(tx - fx) + abs(ty - fy) + 2;
  for (int64_t n = 0; n < limit; n++) {
    int px = cx, py = cy;
    if (px == tx && py == ty) {
      cx += sx;
      cy += sy;
    } else {
      int vx = sx > 0 ? cx <= tx : cx >= tx;
      int vy = sy > 0 ? cy <= ty : cy >= ty;
      if (!(vx && vy)) return 0;
      if ((double)fabsf(tmx - tmy) < 1e-9) {
        cx += sx;
        cy += sy;
        tmx += ddx;
        tmy += ddy;
      } else if (tmx < tmy) {
        cx += sx;
        tmx += ddx;
      } else {
        cy += sy;
        tmy += ddy;
      }
    }
    (*steps)++;
    if (is_boundary(w->bnd, (int64_t)px + (int64_t)py * W)) return 1;
  }
  return 0;
}

typedef struct {
  int64_t dda_steps, gathers;
} eval_stats_t;

/* find_neighbor_which_reaches_first, propag.cu:124-190, on the current state. */
static best_t evaluate(const world_t *w, int x, int y, eval_stats_t *st) {
  const ops_settings_t *s = w->s;
  const int W = (int)s->width, H = (int)s->height;
  const int64_t me = (int64_t)x + (int64_t)y * W;
  best_t best = {w->time[me], w->rx[me], w->ry[me]};
  for (int j = -1; j < 2; j++) {
    for (int i = -1; i < 2; i++) {
      if (i == 0 && j == 0) continue;
      const int nx = x + i, ny = y + j;
      if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;
      const int64_t n = (int64_t)nx + (int64_t)ny * W;
      const float ntime = w->time[n];
      const float smax = w->speed[n];
      if (!(ntime < s->max_time && smax != 0.0f)) continue;
      /* load_point: the reference is read only for cells with time < FLT_MAX */
      const uint16_t rx = w->rx[n], ry = w->ry[n];
      if (rx == (uint16_t)x && ry == (uint16_t)y) continue;
      const float rtime = w->time[(int64_t)rx + (int64_t)ry * W];
      st->gathers++;
      const float azm = w->az[n], ecc = w->ecc[n];
      const float neighbor_time = time_from(w, nx, ny, ntime, x, y, smax, azm, ecc);
      float candidate = time_from(w, rx, ry, rtime, x, y, smax, azm, ecc);
      if (candidate < neighbor_time && candidate < best.time) {
        uint16_t crx = rx, cry = ry;
        if (line_blocked(w, nx, ny, rx, ry, &st->dda_steps)) {
          crx = (uint16_t)nx;
          cry = (uint16_t)ny;
          candidate = neighbor_time;
        }
        if (candidate < best.time) {
          best.time = candidate;
          best.rx = crx;
          best.ry = cry;
        }
      } else if (neighbor_time < best.time) {
        best.time = neighbor_time;
        best.rx = (uint16_t)nx;
        best.ry = (uint16_t)ny;
      }
    }
  }
  return best;
}

/* similar_fires, propag.cu:296-302 (float differences compared in double) */
static inline int similar(float s1, float a1, float e1, float s2, float a2, float e2) {
  return fabsf(s1 - s2) < 0.1 && fabsf(a1 - a2) < (5.0 * (2 * M_PI) / 360.0) && fabsf(e1 - e2) < 0.05;
}

/* pre_propagate / find_boundaries, propag.cu:345-375.  Returns set bits. */
int64_t ops_find_boundaries(uint32_t width, uint32_t height, const float *speed, const float *az,
                            const float *ecc, uint32_t *bits) {
  const int W = (int)width, H = (int)height;
  const int64_t N = (int64_t)W * H;
  memset(bits, 0, sizeof(uint32_t) * (size_t)((N + 31) / 32));
  int64_t count = 0;
  for (int y = 0; y < H; y++) {
    for (int x = 0; x < W; x++) {
      const int64_t me = (int64_t)x + (int64_t)y * W;
      int changed = 0;
      for (int i = -1; i < 2; i++) {
        for (int j = -1; j < 2; j++) {
          if (i == 0 && j == 0) continue;
          const int nx = x + i, ny = y + j;
          if (nx < 0 || ny < 0 || nx >= W || ny >= H) continue;
          const int64_t n = (int64_t)nx + (int64_t)ny * W;
          changed |= !similar(speed[n], az[n], ecc[n], speed[me], az[me], ecc[me]) && speed[me] < speed[n];
        }
      }
      if (changed) {
        bits[me >> 5] |= 1u << (me & 31);
        count++;
      }
    }
  }
  return count;
}

/* stats[]: 0 rounds, 1 launches, 2 sweeps (summed over launches), 3 cell
 * evaluations, 4 improvements, 5 reference gathers, 6 DDA steps, 7 referrer
 * box scans (a changed cell that is some cell's reference), 8 cells visited by
 * those scans, 9 tiles per axis x, 10 tiles per axis y */
#define NSTATS 11

typedef struct {
  int32_t idx; /* position in the tile, -1 = no improvement */
  best_t b;
} upd_t;

typedef struct {
  uint16_t x0, y0, x1, y1; /* empty when x0 > x1 */
} box_t;

/* Marks the eight neighbours of tile cell (lx, ly) (a cell's own change does
 * not change its own evaluation). */
static inline void mark(uint8_t *dirty, int32_t *cand, int64_t *ncand, int TW, int TH, int lx,
                        int ly) {
  for (int j = -1; j < 2; j++)
    for (int i = -1; i < 2; i++) {
      if (i == 0 && j == 0) continue;
      int ax = lx + i, ay = ly + j;
      if (ax < 0 || ay < 0 || ax >= TW || ay >= TH) continue;
      int32_t kk = ax + ay * TW;
      if (!dirty[kk]) {
        dirty[kk] = 1;
        cand[(*ncand)++] = kk;
      }
    }
}

/* Marks the eight neighbours of grid cell (gx, gy): inside the tile in the
 * sweep's dirty list, outside it in the grid-wide pending bitmap (full = 2). */
static inline void mark_grid(uint8_t *dirty, int32_t *cand, int64_t *ncand, uint8_t *pending,
                             int W, int H, int x0, int y0, int TW, int TH, int gx, int gy) {
  for (int j = -1; j < 2; j++)
    for (int i = -1; i < 2; i++) {
      if (i == 0 && j == 0) continue;
      const int ax = gx + i, ay = gy + j;
      if (ax < 0 || ay < 0 || ax >= W || ay >= H) continue;
      const int lx = ax - x0, ly = ay - y0;
      if (lx >= 0 && ly >= 0 && lx < TW && ly < TH) {
        const int32_t kk = lx + ly * TW;
        if (!dirty[kk]) {
          dirty[kk] = 1;
          cand[(*ncand)++] = kk;
        }
      } else {
        pending[(int64_t)ax + (int64_t)ay * W] = 1;
      }
    }
}

/* One cooperative launch over the tile [x0,x1) x [y0,y1): Jacobi sweeps until
 * a sweep improves nothing (Propagator::run, propag.cu:62-109).  Returns 1 if
 * any sweep improved a cell (the launch's `worked` flag).  `pending` is the
 * grid-wide bitmap of full = 2 (else NULL). */
static int run_tile(world_t *w, box_t *refbox, int x0, int y0, int x1, int y1, int full,
                    int64_t *stats, uint8_t *dirty, int32_t *cand, upd_t *upd, int32_t *chg,
                    uint8_t *pending) {
  const int W = (int)w->s->width, H = (int)w->s->height;
  const int TW = x1 - x0, TH = y1 - y0;
  const int64_t TN = (int64_t)TW * TH;
  int worked = 0;
  int first = 1; /* the first sweep of a launch evaluates the whole tile */
  int64_t nchg = 0;
  for (;;) {
    int64_t ncand = 0;
    if (first && pending) {
      /* the tile's pending cells (their inputs changed since they were last
       * evaluated) */
      for (int64_t k = 0; k < TN; k++) {
        const int64_t g = (int64_t)(x0 + k % TW) + (int64_t)(y0 + k / TW) * W;
        if (pending[g]) {
          pending[g] = 0;
          cand[ncand++] = (int32_t)k;
        }
      }
    } else if (full == 1 || first) {
      for (int64_t k = 0; k < TN; k++) cand[ncand++] = (int32_t)k;
    } else if (pending) {
      /* as below, with marks outside the tile kept in the pending bitmap and
       * the whole referrer box scanned */
      for (int64_t c = 0; c < nchg; c++) {
        int32_t k = chg[c];
        const int gx = x0 + k % TW, gy = y0 + k / TW;
        const int64_t gc = (int64_t)gx + (int64_t)gy * W;
        if (w->time[gc] < w->s->max_time && w->speed[gc] != 0.0f)
          mark_grid(dirty, cand, &ncand, pending, W, H, x0, y0, TW, TH, gx, gy);
        const box_t b = refbox[gc];
        if (b.x0 > b.x1) continue;
        stats[7]++;
        for (int yy = b.y0; yy <= b.y1; yy++)
          for (int xx = b.x0; xx <= b.x1; xx++) {
            const int64_t n = (int64_t)xx + (int64_t)yy * W;
            stats[8]++;
            if (w->time[n] < w->s->max_time && w->speed[n] != 0.0f && w->rx[n] == (uint16_t)gx &&
                w->ry[n] == (uint16_t)gy)
              mark_grid(dirty, cand, &ncand, pending, W, H, x0, y0, TW, TH, xx, yy);
          }
      }
      for (int64_t c = 0; c < ncand; c++) dirty[cand[c]] = 0;
    } else {
      /* cells whose inputs changed: the neighbours of every changed cell that
       * burns (a cell that does not burn is skipped by its neighbours), and
       * the neighbours of every burning cell whose reference changed (found
       * through the box of cells that ever adopted that reference) */
      for (int64_t c = 0; c < nchg; c++) {
        int32_t k = chg[c];
        int lx = k % TW, ly = k / TW;
        const int gx = x0 + lx, gy = y0 + ly;
        const int64_t gc = (int64_t)gx + (int64_t)gy * W;
        if (w->time[gc] < w->s->max_time && w->speed[gc] != 0.0f)
          mark(dirty, cand, &ncand, TW, TH, lx, ly);
        const box_t b = refbox[(int64_t)gx + (int64_t)gy * W];
        if (b.x0 > b.x1) continue;
        stats[7]++;
        /* referrers outside the tile matter only through their neighbours
         * inside it: clip the scan to the tile grown by one cell */
        int bx0 = b.x0 > x0 - 1 ? b.x0 : x0 - 1, bx1 = b.x1 < x1 ? b.x1 : x1;
        int by0 = b.y0 > y0 - 1 ? b.y0 : y0 - 1, by1 = b.y1 < y1 ? b.y1 : y1;
        if (bx0 < 0) bx0 = 0;
        if (by0 < 0) by0 = 0;
        if (bx1 > W - 1) bx1 = W - 1;
        if (by1 > H - 1) by1 = H - 1;
        for (int yy = by0; yy <= by1; yy++)
          for (int xx = bx0; xx <= bx1; xx++) {
            const int64_t n = (int64_t)xx + (int64_t)yy * W;
            stats[8]++;
            if (w->time[n] < w->s->max_time && w->speed[n] != 0.0f && w->rx[n] == (uint16_t)gx &&
                w->ry[n] == (uint16_t)gy)
              mark(dirty, cand, &ncand, TW, TH, xx - x0, yy - y0);
          }
      }
      for (int64_t c = 0; c < ncand; c++) dirty[cand[c]] = 0;
    }
    stats[2]++;
    if (ncand == 0) break; /* the reference's final sweep, which improves nothing */
    first = 0;
    stats[3] += ncand;
    /* evaluate (Jacobi: all reads see the previous sweep's state) */
    int64_t dda = 0, gat = 0;
#pragma omp parallel
    {
      eval_stats_t st = {0, 0};
#pragma omp for schedule(dynamic, 512)
      for (int64_t c = 0; c < ncand; c++) {
        int32_t k = cand[c];
        int x = x0 + k % TW, y = y0 + k / TW;
        int64_t me = (int64_t)x + (int64_t)y * W;
        best_t b = evaluate(w, x, y, &st);
        upd[c].idx = -1;
        if (b.time < w->time[me]) {
          upd[c].idx = k;
          upd[c].b = b;
        }
      }
#pragma omp atomic
      dda += st.dda_steps;
#pragma omp atomic
      gat += st.gathers;
    }
    stats[5] += gat;
    stats[6] += dda;
    /* commit (update_point / commit_point, propag.cu:192-207) */
    nchg = 0;
    for (int64_t c = 0; c < ncand; c++) {
      if (upd[c].idx < 0) continue;
      int32_t k = upd[c].idx;
      int x = x0 + k % TW, y = y0 + k / TW;
      int64_t me = (int64_t)x + (int64_t)y * W;
      w->time[me] = upd[c].b.time;
      w->rx[me] = upd[c].b.rx;
      w->ry[me] = upd[c].b.ry;
      box_t *rb = &refbox[(int64_t)upd[c].b.rx + (int64_t)upd[c].b.ry * W];
      if (rb->x0 > rb->x1) {
        *rb = (box_t){(uint16_t)x, (uint16_t)y, (uint16_t)x, (uint16_t)y};
      } else {
        if (rb->x0 > x) rb->x0 = (uint16_t)x;
        if (rb->x1 < x) rb->x1 = (uint16_t)x;
        if (rb->y0 > y) rb->y0 = (uint16_t)y;
        if (rb->y1 < y) rb->y1 = (uint16_t)y;
      }
      chg[nchg++] = k;
    }
    if (nchg == 0) break;
    worked = 1;
    stats[4] += nchg;
  }
  return worked;
}

/* Runs the propagation (pre-computed boundaries in `bnd`).  time/rx/ry hold
 * the initial state (ignition times, refs = own position for ignited cells,
 * 0xFFFF otherwise) and receive the result before the post mask.
 * tile = cells per side of one cooperative launch; tile <= 0 means one tile
 * for the whole grid.  full = 1 evaluates every cell of the tile in every
 * sweep (no work skipping); full = 2 skips work in first sweeps too (see the
 * top of this file).  Returns 0 on success. */
int ops_propagate(const ops_settings_t *s, const float *speed, const float *az, const float *ecc,
                  float *time, uint16_t *rx, uint16_t *ry, const uint32_t *bnd, int tile, int full,
                  int trig, int threads, int64_t *stats) {
  const int W = (int)s->width, H = (int)s->height;
  const int64_t N = (int64_t)W * H;
  if (W < 1 || H < 1 || W > 65534 || H > 65534) return -1;
  g_trig = trig;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
  memset(stats, 0, sizeof(int64_t) * NSTATS);
  const int T = tile > 0 ? tile : (W > H ? W : H);
  const int SX = (W + T - 1) / T, SY = (H + T - 1) / T;
  stats[9] = SX;
  stats[10] = SY;
  world_t w = {s, speed, az, ecc, time, rx, ry, bnd, NULL};
  box_t *refbox = (box_t *)malloc(sizeof(box_t) * (size_t)N);
  const int64_t TN = (int64_t)T * T;
  uint8_t *dirty = (uint8_t *)calloc((size_t)TN, 1);
  int32_t *cand = (int32_t *)malloc(sizeof(int32_t) * (size_t)TN);
  int32_t *chg = (int32_t *)malloc(sizeof(int32_t) * (size_t)TN);
  upd_t *upd = (upd_t *)malloc(sizeof(upd_t) * (size_t)TN);
  uint8_t *pending = full == 2 ? (uint8_t *)calloc((size_t)N, 1) : NULL;
  if (!refbox || !dirty || !cand || !chg || !upd || (full == 2 && !pending)) return -2;
  if (pending) /* the neighbours of the burning cells can improve first */
    for (int64_t i = 0; i < N; i++) {
      if (!(time[i] < s->max_time && speed[i] != 0.0f)) continue;
      const int x = (int)(i % W), y = (int)(i / W);
      for (int j = -1; j < 2; j++)
        for (int ii = -1; ii < 2; ii++) {
          const int ax = x + ii, ay = y + j;
          if ((ii || j) && ax >= 0 && ay >= 0 && ax < W && ay < H) pending[ax + (int64_t)ay * W] = 1;
        }
    }
  for (int64_t i = 0; i < N; i++) refbox[i] = (box_t){1, 1, 0, 0};
  for (int64_t i = 0; i < N; i++)
    if (time[i] < FLT_MAX) {
      box_t *rb = &refbox[(int64_t)rx[i] + (int64_t)ry[i] * W];
      int x = (int)(i % W), y = (int)(i / W);
      if (rb->x0 > rb->x1) *rb = (box_t){(uint16_t)x, (uint16_t)y, (uint16_t)x, (uint16_t)y};
    }
  int any;
  do {
    any = 0;
    stats[0]++;
    for (int gy = 0; gy < SY; gy++) {
      for (int gx = 0; gx < SX; gx++) {
        int x0 = gx * T, y0 = gy * T;
        int x1 = x0 + T < W ? x0 + T : W, y1 = y0 + T < H ? y0 + T : H;
        stats[1]++;
        any |= run_tile(&w, refbox, x0, y0, x1, y1, full, stats, dirty, cand, upd, chg, pending);
      }
    }
  } while (any);
  free(pending);
  free(refbox);
  free(dirty);
  free(cand);
  free(chg);
  free(upd);
  return 0;
}

/* post_propagate, propag.cu:110-117.  Returns the number of burned cells. */
int64_t ops_post(int64_t n, const float *speed, float max_time, float *time) {
  int64_t burned = 0;
  for (int64_t i = 0; i < n; i++) {
    if (speed[i] == 0.0f || time[i] > max_time)
      time[i] = FLT_MAX;
    else
      burned++;
  }
  return burned;
}

/* Evaluates time_from for a list of (from, to) pairs; exposed so the tests can
 * compare the device arithmetic with this restatement. */
void ops_time_from_batch(const ops_settings_t *s, int64_t n, const int32_t *fx, const int32_t *fy,
                         const float *ftime, const int32_t *tx, const int32_t *ty, const float *smax,
                         const float *azmax, const float *ecc, int trig, float *out) {
  world_t w = {s, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL};
  g_trig = trig;
  for (int64_t i = 0; i < n; i++)
    out[i] = time_from(&w, fx[i], fy[i], ftime[i], tx[i], ty[i], smax[i], azmax[i], ecc[i]);
}

void ops_trig_batch(int64_t n, const float *a, const float *b, float *cos_out, float *atan2_out) {
  for (int64_t i = 0; i < n; i++) {
    cos_out[i] = pg_cosf(a[i]);
    atan2_out[i] = pg_atan2f(a[i], b[i]);
  }
}

int ops_nstats(void) { return NSTATS; }

/* Exposes the directed-rounding emulation (round-down reciprocal,
 * round-toward-zero square root) for the tests. */
void ops_rounding_batch(int64_t n, const float *x, float *rcp_out, float *sqrt_out) {
  for (int64_t i = 0; i < n; i++) {
    rcp_out[i] = rcp_rd(x[i]);
    sqrt_out[i] = x[i] >= 0.0f ? sqrt_rz(x[i]) : NAN;
  }
}

/* Visits the cells of the line-of-sight walk from (fx, fy) to (tx, ty) the
 * way propag.h:91-135 does; writes up to max_out (x, y) pairs and returns the
 * number of cells visited. */
int64_t ops_dda_cells(int fx, int fy, int tx, int ty, int32_t *out, int64_t max_out) {
  int sx = (tx > fx) - (tx < fx), sy = (ty > fy) - (ty < fy);
  int cx = fx, cy = fy;
  float tmx = (float)(1.0 / (double)(float)abs(tx - fx));
  float tmy = (float)(1.0 / (double)(float)abs(ty - fy));
  const float ddx = tmx, ddy = tmy;
  int64_t limit = (int64_t)abs(tx - fx) + abs(ty - fy) + 2, k = 0;
  for (int64_t n = 0; n < limit; n++) {
    int px = cx, py = cy;
    if (px == tx && py == ty) {
      cx += sx;
      cy += sy;
    } else {
      int vx = sx > 0 ? cx <= tx : cx >= tx;
      int vy = sy > 0 ? cy <= ty : cy >= ty;
      if (!(vx && vy)) break;
      if ((double)fabsf(tmx - tmy) < 1e-9) {
        cx += sx;
        cy += sy;
        tmx += ddx;
        tmy += ddy;
      } else if (tmx < tmy) {
        cx += sx;
        tmx += ddx;
      } else {
        cy += sy;
        tmy += ddy;
      }
    }
    if (k < max_out) {
      out[2 * k] = px;
      out[2 * k + 1] = py;
    }
    k++;
  }
  return k;
}
