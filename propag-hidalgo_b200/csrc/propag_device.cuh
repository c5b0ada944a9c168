// Device-side arithmetic of the arrival-time propagation.
//
// Everything here is written with explicitly rounded operations
// (__fadd_rn, __fmul_rn, __fmaf_rn, ...) so that the compiler can neither
// contract nor reorder them: the result of every cell evaluation is a fixed
// sequence of operations, chosen per scenario between the reference's own
// (CUDA's atan2f and __cosf, nvcc's contracted multiply-adds) and a portable
// IEEE sequence that a CPU reproduces (see time_from).
//
// Semantics follow the reference kernel (paths relative to the reference
// project):
//   time_from                          crates/propag/src/propag.cu:269-294
//   DDA line walk                      crates/propag/src/propag.h:91-135
//   find_neighbor_which_reaches_first  crates/propag/src/propag.cu:124-190
//   similar_fires / find_boundaries    crates/propag/src/propag.cu:296-302,345-375
#pragma once

#include <cfloat>
#include <cstdint>

namespace propag {

constexpr uint32_t kNoRef = 0xFFFFFFFFu;  // refs_x = refs_y = 0xFFFF

__device__ __forceinline__ uint32_t pack_ref(int x, int y) {
  return (uint32_t)(x & 0xFFFF) | ((uint32_t)(y & 0xFFFF) << 16);
}
__device__ __forceinline__ int ref_x(uint32_t r) { return (int)(r & 0xFFFFu); }
__device__ __forceinline__ int ref_y(uint32_t r) { return (int)(r >> 16); }

// ---- portable float cosine / arctangent ------------------------------------
// cos: Cody-Waite reduction by pi/2 with a three-part constant, Taylor
// polynomials on [-pi/4, pi/4].  atan2: octant reduction; atan(t), t in [0,1],
// above tan(pi/8) as u = (mn-mx)/(mn+mx) (one division either way), Taylor to u^19.
// Both are accurate to about 1 ulp and, being plain IEEE operations, give the
// same bits on every IEEE machine.
__device__ __forceinline__ float pg_sin_poly(float r) {
  const float r2 = __fmul_rn(r, r);
  float p = __fmaf_rn(r2, 2.75573192e-6f, -1.98412698e-4f);
  p = __fmaf_rn(r2, p, 8.33333333e-3f);
  p = __fmaf_rn(r2, p, -1.66666667e-1f);
  return __fmaf_rn(__fmul_rn(r, r2), p, r);
}
__device__ __forceinline__ float pg_cos_poly(float r) {
  const float r2 = __fmul_rn(r, r);
  float p = __fmaf_rn(r2, -2.75573192e-7f, 2.48015873e-5f);
  p = __fmaf_rn(r2, p, -1.38888889e-3f);
  p = __fmaf_rn(r2, p, 4.16666667e-2f);
  p = __fmaf_rn(r2, p, -0.5f);
  return __fmaf_rn(r2, p, 1.0f);
}
__device__ __forceinline__ float pg_cosf(float x) {
  const float ax = fabsf(x);
  const float k = rintf(__fmul_rn(ax, 0.636619772367581343f));
  float r = __fmaf_rn(-k, 1.57079637050628662109375f, ax);
  r = __fmaf_rn(-k, -4.37113900018624283e-8f, r);
  r = __fmaf_rn(-k, -1.71512451677125e-15f, r);
  switch (((int)k) & 3) {
    case 0: return pg_cos_poly(r);
    case 1: return -pg_sin_poly(r);
    case 2: return -pg_cos_poly(r);
    default: return pg_sin_poly(r);
  }
}
__device__ __forceinline__ float pg_atan2f(float y, float x) {
  const float ax = fabsf(x), ay = fabsf(y);
  const float mx = ax > ay ? ax : ay;
  const float mn = ax > ay ? ay : ax;
  if (mx == 0.0f) return 0.0f;
  // one division: t = mn / mx, or (t - 1) / (t + 1) formed directly as
  // (mn - mx) / (mn + mx) above tan(pi/8)
  float base = 0.0f;
  float u;
  if (mn > __fmul_rn(0.414213562373095049f, mx)) {
    u = __fdiv_rn(__fsub_rn(mn, mx), __fadd_rn(mn, mx));
    base = 0.785398163397448309616f;
  } else {
    u = __fdiv_rn(mn, mx);
  }
  const float u2 = __fmul_rn(u, u);
  float p = __fmaf_rn(u2, 5.26315789e-2f, -5.88235294e-2f);
  p = __fmaf_rn(u2, p, 6.66666667e-2f);
  p = __fmaf_rn(u2, p, -7.69230769e-2f);
  p = __fmaf_rn(u2, p, 9.09090909e-2f);
  p = __fmaf_rn(u2, p, -1.11111111e-1f);
  p = __fmaf_rn(u2, p, 1.42857143e-1f);
  p = __fmaf_rn(u2, p, -2.00000000e-1f);
  p = __fmaf_rn(u2, p, 3.33333333e-1f);
  float a = __fadd_rn(__fmaf_rn(-__fmul_rn(u, u2), p, u), base);
  if (ay > ax) a = __fsub_rn(1.57079632679489661923f, a);
  if (x < 0.0f) a = __fsub_rn(3.14159265358979323846f, a);
  if (y < 0.0f) a = -a;
  return a;
}

// ---- time_from (propag.cu:269-294) -----------------------------------------
// Arrival time at `to` for a fire that left `from` at `ftime`, spreading with
// the elliptical speed of `fire` along the bearing from -> to.  The reference
// writes `1.0 - ...` with double literals, so denom and factor are formed in
// double and rounded to float; __frcp_rd / __fsqrt_rz as in the reference.
//
// Two arithmetics (`refm`, uniform per scenario):
//   reference (refm = true, the default): the reference's own operations as
//     nvcc compiles propag.cu with its default flags -- CUDA's atan2f and the
//     __cosf intrinsic, and the three sums nvcc contracts into multiply-adds,
//     1.0 - e*cos -> fma(-e, cos, 1) (in float), dx*dx + dy*dy ->
//     fma(dx, dx, dy*dy) and from.time + distance * rcp ->
//     fma(distance, rcp, from.time).  A test compiles the reference's
//     time_from from its source and checks these bits against it.
//   portable (refm = false): the float cosine/arctangent above and every
//     operation rounded on its own, which a CPU reproduces bit for bit (the
//     CPU restatement checks the whole propagation schedule against it).
struct Fire {
  float speed_max, azimuth_max, eccentricity;
};

__device__ __forceinline__ float spread_factor(float azimuth, const Fire &f, bool refm) {
  const float angle = fabsf(__fsub_rn(azimuth, f.azimuth_max));
  // denom = 1.0 - e * cos(angle): nvcc narrows the double subtraction of a
  // float product to float (exact either way) and contracts it, so the
  // reference computes fma(-e, cos, 1); the portable arithmetic rounds the
  // product first
  const float denom =
      refm ? __fmaf_rn(-f.eccentricity, __cosf(angle), 1.0f)
           : __double2float_rn(__dsub_rn(1.0, (double)__fmul_rn(f.eccentricity, pg_cosf(angle))));
  const double one_minus_e = __dsub_rn(1.0, (double)f.eccentricity);
  return __double2float_rn(__dmul_rn(one_minus_e, (double)__frcp_rd(denom)));
}

// Round-down reciprocal of the elliptical speed along `azimuth`.
__device__ __forceinline__ float inv_speed(float azimuth, const Fire &f, bool refm) {
  return __frcp_rd(__fmul_rn(f.speed_max, spread_factor(azimuth, f, refm)));
}

// from.time + distance * __frcp_rd(speed), given the reciprocal.
__device__ __forceinline__ float step_time(float ftime, float distance, float inv, bool refm) {
  return refm ? __fmaf_rn(distance, inv, ftime) : __fadd_rn(ftime, __fmul_rn(distance, inv));
}

__device__ __forceinline__ float cell_distance(int ddx, int ddy, float gdx, float gdy, bool refm) {
  const float dx = __fmul_rn((float)ddx, gdx);
  const float dy = __fmul_rn((float)ddy, gdy);
  return __fsqrt_rz(refm ? __fmaf_rn(dx, dx, __fmul_rn(dy, dy))
                         : __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)));
}

__device__ __forceinline__ float bearing(int fx, int fy, int tx, int ty, bool north_up, bool refm) {
  const float y = (float)(tx - fx);
  const float x = north_up ? (float)(fy - ty) : (float)(ty - fy);
  return refm ? atan2f(y, x) : pg_atan2f(y, x);
}

__device__ __forceinline__ float time_from(int fx, int fy, float ftime, int tx, int ty,
                                           const Fire &f, float gdx, float gdy, bool north_up,
                                           bool refm) {
  const float inv = inv_speed(bearing(fx, fy, tx, ty, north_up, refm), f, refm);
  return step_time(ftime, cell_distance(fx - tx, fy - ty, gdx, gdy, refm), inv, refm);
}

// ---- DDA line-of-sight walk (propag.h:91-135) ------------------------------
// Visits the cells from `from` to `to` inclusive in the reference's order and
// reports whether one of them is a boundary; `steps` counts the cells
// visited up to and including the first boundary.  The t-max accumulators
// are the reference's float arithmetic: start 1/|d| (formed in double), step
// +1/|d|, diagonal step when |tmax.x - tmax.y| < 1e-9 (a double comparison
// in the reference: for a float v, (double)v < 1e-9 exactly when v is at most
// the largest float below 1e-9).  The walk is bounded by |dx| + |dy| + 2
// visits, more than any walk takes.
//
// The cells are generated kWalkBatch at a time by the (load-free) DDA
// arithmetic, their bitmap words are loaded together, and then checked in
// visiting order: one load latency per batch instead of one per cell.
constexpr int kWalkBatch = 8;

__device__ __forceinline__ bool is_boundary(const uint32_t *__restrict__ bnd, int64_t ix) {
  return (__ldg(bnd + (ix >> 5)) >> (ix & 31)) & 1u;
}

__device__ __forceinline__ bool line_blocked(const uint32_t *__restrict__ bnd, int W, int fx,
                                             int fy, int tx, int ty, uint32_t &steps) {
  const int sx = (tx > fx) - (tx < fx), sy = (ty > fy) - (ty < fy);
  const int adx = abs(tx - fx), ady = abs(ty - fy);
  float tmx = __double2float_rn(1.0 / (double)(float)adx);
  float tmy = __double2float_rn(1.0 / (double)(float)ady);
  const float ddx = tmx, ddy = tmy;
  const float kTie = __int_as_float(0x3089705F);  // the largest float below 1e-9
  int cx = fx, cy = fy;
  int left = adx + ady + 2;  // visits the bound still allows
  for (;;) {
    uint32_t ix[kWalkBatch];  // cell index x + y W (grids below 2^32 cells)
    int nv = 0;               // cells of this batch
    bool ended = left <= 0;
#pragma unroll
    for (int i = 0; i < kWalkBatch; ++i) {
      if (!ended && i < left) {
        const int px = cx, py = cy;
        if (px == tx && py == ty) {
          cx += sx;
          cy += sy;
        } else {
          const bool vx = sx > 0 ? cx <= tx : cx >= tx;
          const bool vy = sy > 0 ? cy <= ty : cy >= ty;
          if (!(vx && vy)) {
            ended = true;
          } else if (fabsf(__fsub_rn(tmx, tmy)) <= kTie) {
            cx += sx;
            cy += sy;
            tmx = __fadd_rn(tmx, ddx);
            tmy = __fadd_rn(tmy, ddy);
          } else if (tmx < tmy) {
            cx += sx;
            tmx = __fadd_rn(tmx, ddx);
          } else {
            cy += sy;
            tmy = __fadd_rn(tmy, ddy);
          }
        }
        if (!ended) {
          ix[i] = (uint32_t)px + (uint32_t)py * (uint32_t)W;
          nv = i + 1;
        }
      }
    }
    uint32_t word[kWalkBatch];
#pragma unroll
    for (int i = 0; i < kWalkBatch; ++i) word[i] = i < nv ? __ldg(bnd + (ix[i] >> 5)) : 0u;
#pragma unroll
    for (int i = 0; i < kWalkBatch; ++i) {
      if (i < nv) {
        ++steps;
        if ((word[i] >> (ix[i] & 31)) & 1u) return true;
      }
    }
    if (nv < kWalkBatch) return false;  // the walk ended in this batch
    left -= kWalkBatch;
  }
}

// similar_fires (propag.cu:296-302): float differences compared against the
// reference's double thresholds.
__device__ __forceinline__ bool similar_fires(const Fire &a, const Fire &b) {
  return (double)fabsf(__fsub_rn(a.speed_max, b.speed_max)) < 0.1 &&
         (double)fabsf(__fsub_rn(a.azimuth_max, b.azimuth_max)) < (5.0 * (2 * 3.14159265358979323846) / 360.0) &&
         (double)fabsf(__fsub_rn(a.eccentricity, b.eccentricity)) < 0.05;
}

}  // namespace propag
