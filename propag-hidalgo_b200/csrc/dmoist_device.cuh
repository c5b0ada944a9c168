// Device side of the dmoist moisture model (crates/dmoist/src/lib.rs:55-715):
// the model's tables and per-cell functions, shared by the moisture pass
// (dmoist.cu) and the fused moisture + fire-behaviour pass (fire.cu).  Every
// file that includes it gets its own constant copy of the tables.  Float
// operations follow the reference's order; the including files are compiled
// without FMA contraction (explicit __fmaf_rn where the portable arctangent
// uses fused multiply-adds), so results equal the CPU restatement bit for bit.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace propag {

struct DmoistTables {
  int8_t hcb[6][21];
  uint8_t prob[4][9][18];
  int8_t shade[3][2][8][6];
  int8_t pp[2][4][6];
};

// The model's tables (lib.rs:197-262 base humidity index, daytime table;
// 272-453 ignition probability; 472-614 shading correction; 147-183
// precipitation effect), in DmoistTables order.
static __constant__ DmoistTables c_dm = {
    {
    {1, 2, 2, 3, 4, 5, 5, 6, 7, 8, 8, 8, 9, 9, 10, 11, 12, 12, 13, 13, 14},
    {1, 2, 2, 3, 4, 5, 5, 6, 7, 7, 7, 8, 9, 9, 10, 10, 11, 12, 13, 13, 13},
    {1, 2, 2, 3, 4, 5, 5, 6, 6, 7, 7, 8, 9, 9, 9, 10, 11, 12, 12, 12, 13},
    {1, 1, 2, 2, 3, 4, 5, 5, 6, 7, 7, 8, 8, 8, 9, 10, 10, 11, 12, 12, 13},
    {1, 1, 2, 2, 3, 4, 4, 5, 6, 7, 7, 8, 8, 8, 9, 10, 10, 11, 12, 12, 13},
    {1, 1, 2, 2, 3, 4, 4, 5, 6, 7, 7, 8, 8, 8, 9, 10, 10, 11, 12, 12, 12},
},
    {
    {{100, 100, 100, 90, 80, 70, 60, 50, 40, 40, 30, 30, 30, 20, 20, 20, 10, 10},
     {100, 100, 90, 80, 70, 60, 60, 50, 40, 40, 30, 30, 20, 20, 20, 10, 10, 10},
     {100, 100, 90, 80, 70, 60, 50, 50, 40, 30, 30, 30, 20, 20, 20, 10, 10, 10},
     {100, 100, 90, 80, 70, 60, 50, 40, 40, 30, 30, 20, 20, 20, 20, 10, 10, 10},
     {100, 100, 80, 70, 60, 60, 50, 40, 40, 30, 30, 20, 20, 20, 10, 10, 10, 10},
     {100, 90, 80, 70, 60, 50, 50, 40, 30, 30, 30, 20, 20, 20, 10, 10, 10, 10},
     {100, 90, 80, 70, 60, 50, 40, 40, 30, 30, 20, 20, 20, 20, 10, 10, 10, 10},
     {100, 90, 80, 70, 60, 50, 40, 40, 30, 30, 20, 20, 20, 20, 10, 10, 10, 10},
     {100, 90, 70, 60, 60, 50, 40, 40, 30, 30, 20, 20, 20, 20, 10, 10, 10, 10}},
    {{100, 100, 100, 80, 70, 60, 60, 50, 40, 40, 30, 30, 20, 20, 20, 20, 10, 10},
     {100, 100, 90, 80, 70, 60, 50, 50, 40, 40, 30, 30, 20, 20, 20, 10, 10, 10},
     {100, 100, 90, 80, 70, 60, 50, 40, 40, 30, 30, 30, 20, 20, 20, 10, 10, 10},
     {100, 100, 90, 80, 70, 60, 50, 40, 40, 30, 30, 20, 20, 20, 10, 10, 10, 10},
     {100, 100, 80, 70, 60, 50, 50, 40, 40, 30, 30, 20, 20, 20, 10, 10, 10, 10},
     {100, 90, 80, 70, 60, 50, 50, 40, 30, 30, 20, 20, 20, 20, 10, 10, 10, 10},
     {100, 90, 80, 70, 60, 50, 40, 40, 30, 30, 20, 20, 20, 10, 10, 10, 10, 10},
     {100, 90, 80, 70, 60, 50, 40, 40, 30, 30, 20, 20, 20, 10, 10, 10, 10, 10},
     {100, 80, 70, 60, 50, 50, 40, 30, 30, 20, 20, 20, 10, 10, 10, 10, 10, 10}},
    {{100, 100, 90, 80, 70, 60, 50, 50, 40, 40, 30, 30, 20, 20, 20, 10, 10, 10},
     {100, 100, 90, 80, 70, 60, 50, 50, 40, 30, 30, 30, 20, 20, 20, 10, 10, 10},
     {100, 100, 90, 80, 70, 60, 50, 40, 40, 30, 30, 20, 20, 20, 10, 10, 10, 10},
     {100, 100, 80, 70, 60, 60, 50, 40, 40, 30, 30, 20, 20, 20, 10, 10, 10, 10},
     {100, 90, 80, 70, 60, 50, 50, 40, 30, 30, 30, 20, 20, 20, 10, 10, 10, 10},
     {100, 90, 80, 70, 60, 50, 40, 40, 30, 30, 20, 20, 20, 10, 10, 10, 10, 10},
     {100, 90, 80, 70, 60, 50, 40, 40, 30, 30, 20, 20, 20, 10, 10, 10, 10, 10},
     {100, 90, 70, 60, 50, 50, 40, 30, 30, 30, 20, 20, 20, 10, 10, 10, 10, 10},
     {100, 80, 70, 60, 50, 50, 40, 30, 30, 20, 20, 20, 10, 10, 10, 10, 10, 10}},
    {{100, 100, 90, 80, 70, 60, 50, 50, 40, 30, 30, 30, 20, 20, 20, 10, 10, 10},
     {100, 100, 90, 80, 70, 60, 50, 40, 40, 30, 30, 20, 20, 20, 20, 10, 10, 10},
     {100, 100, 80, 70, 60, 60, 50, 40, 40, 30, 30, 20, 20, 20, 10, 10, 10, 10},
     {100, 90, 80, 70, 60, 50, 50, 40, 30, 30, 30, 20, 20, 20, 10, 10, 10, 10},
     {100, 90, 80, 70, 60, 50, 40, 40, 30, 30, 20, 20, 20, 10, 10, 10, 10, 10},
     {100, 90, 80, 70, 60, 50, 40, 40, 30, 30, 20, 20, 20, 10, 10, 10, 10, 10},
     {100, 90, 70, 60, 60, 50, 40, 40, 30, 30, 20, 20, 20, 10, 10, 10, 10, 10},
     {100, 80, 70, 60, 50, 50, 40, 30, 30, 20, 20, 20, 10, 10, 10, 10, 10, 10},
     {100, 80, 70, 60, 50, 40, 40, 30, 30, 20, 20, 20, 10, 10, 10, 10, 10, 10}},
},
    {
    {{{3, 1, 0, 0, 1, 3}, {4, 2, 1, 1, 2, 4}, {2, 1, 0, 0, 1, 4}, {2, 0, 0, 1, 3, 5},
      {3, 1, 0, 0, 1, 3}, {3, 1, 1, 1, 1, 3}, {3, 1, 0, 0, 1, 3}, {5, 3, 1, 0, 0, 2}},
     {{5, 4, 3, 3, 4, 5}, {5, 4, 3, 3, 4, 5}, {4, 4, 3, 4, 4, 5}, {4, 4, 3, 4, 4, 5},
      {4, 4, 3, 3, 4, 5}, {4, 4, 3, 3, 4, 5}, {5, 4, 3, 3, 4, 4}, {5, 4, 3, 3, 4, 4}}},
    {{{4, 2, 1, 1, 2, 4}, {4, 3, 3, 3, 3, 4}, {4, 2, 1, 1, 2, 4}, {3, 1, 1, 2, 4, 5},
      {4, 2, 1, 1, 2, 4}, {4, 2, 1, 1, 2, 4}, {4, 2, 1, 1, 2, 4}, {5, 4, 2, 1, 1, 3}},
     {{5, 5, 4, 4, 5, 5}, {5, 5, 4, 4, 5, 5}, {5, 4, 4, 4, 5, 5}, {5, 4, 4, 4, 5, 5},
      {5, 4, 4, 4, 4, 5}, {5, 4, 4, 4, 4, 5}, {5, 5, 4, 4, 4, 5}, {5, 5, 4, 4, 4, 5}}},
    {{{5, 4, 3, 3, 4, 5}, {5, 5, 5, 5, 5, 5}, {5, 4, 3, 3, 4, 5}, {5, 4, 3, 2, 5, 5},
      {5, 4, 3, 2, 4, 5}, {5, 3, 1, 1, 3, 5}, {5, 4, 3, 3, 4, 5}, {5, 5, 4, 2, 3, 5}},
     {{5, 5, 5, 5, 5, 5}, {5, 5, 5, 5, 5, 5}, {5, 5, 5, 5, 5, 5}, {5, 5, 5, 5, 5, 5},
      {5, 5, 5, 5, 5, 5}, {5, 5, 5, 5, 5, 5}, {5, 5, 5, 5, 5, 5}, {5, 5, 5, 5, 5, 5}}},
},
    {
    {{-1, -1, 0, 0, 0, 0}, {-1, 5, 1, 0, 0, 0}, {-1, 15, 5, 1, 0, 0}, {-1, 35, 15, 5, 1, 0}},
    {{-1, -1, -1, -1, 1, 0}, {-1, -1, -1, -1, 5, 1}, {-1, -1, -1, 15, 5, 1}, {-1, -1, 35, 15, 5, 1}},
},
};

__device__ __forceinline__ float dm_pp_effect(const DmoistTables &T, int month, float pp, int offset) {
  if (pp > 0.0f) {
    const int mi = (month >= 4 && month <= 10) ? 0 : 1;
    const int pi = (pp >= 1.0f && pp < 5.0f) ? 0 : (pp >= 5.0f && pp < 15.0f) ? 1
                 : (pp >= 15.0f && pp < 35.0f) ? 2 : 3;
    const int e = T.pp[mi][pi][offset];
    if (e > -1) return (float)e;
  }
  return pp;
}

__device__ __forceinline__ int dm_hcb(const DmoistTables &T, float t, float rh) {
  float hf = floorf(rh / 5.0f);
  hf = hf < 0.0f ? 0.0f : (hf > 20.0f ? 20.0f : hf);
  if (hf != hf) hf = 0.0f;  // NaN: class 0, as the reference's saturating cast
  int ti;
  if (t < 0.0f) ti = 0;
  else if (t >= 0.0f && t <= 9.0f) ti = 1;
  else if (t > 9.0f && t <= 20.0f) ti = 2;
  else if (t > 20.0f && t <= 31.0f) ti = 3;
  else if (t > 31.0f && t <= 42.0f) ti = 4;
  else ti = 5;
  return T.hcb[ti][(int)hf];
}

__device__ __forceinline__ float dm_shading(float cloud, int fuel) {
  float s = cloud * 0.75f;
  if (fuel >= 7 && fuel <= 12) s = s < 50.0f ? 75.0f : 100.0f;
  return s;
}

__device__ __forceinline__ float dm_prob(const DmoistTables &T, float t, float cloud, float hcs, int fuel) {
  if (fuel == 0) return 0.0f;
  if (!(hcs > 0.0f && hcs < 18.0f)) return 0.0f;
  const float s = dm_shading(cloud, fuel);
  const int si = (s >= 0.0f && s < 10.0f) ? 0 : (s >= 10.0f && s < 50.0f) ? 1
               : (s >= 50.0f && s < 90.0f) ? 2 : 3;
  float tf = 9.0f - ceilf(t / 5.0f);
  tf = tf < 0.0f ? 0.0f : (tf > 8.0f ? 8.0f : tf);
  if (tf != tf) tf = 0.0f;
  const int hci = (int)floorf(hcs) - 1;
  if (hci < 0) return 0.0f;
  return (float)T.prob[si][(int)tf][hci];
}

__device__ __forceinline__ float dm_corrector(const DmoistTables &T, float orientation, float slope,
                                              float shade, int month, int hour_in) {
  int hour;
  float sh;
  if (!(hour_in >= 6 && hour_in <= 19)) {
    hour = 19;
    sh = 100.0f;
  } else if (hour_in < 8) {
    hour = 8;
    sh = 100.0f;
  } else {
    hour = hour_in;
    sh = shade;
  }
  const int shi = sh < 50.0f ? 0 : 1;
  int hi = (hour - 8) / 2;
  hi = hi < 0 ? 0 : (hi > 5 ? 5 : hi);
  int mi;
  if (month >= 5 && month <= 8) mi = 0;
  else if (month == 2 || month == 3 || month == 4 || month == 9 || month == 10) mi = 1;
  else if (month == 11 || month == 12 || month == 1) mi = 2;
  else return __int_as_float(0x7fc00000);
  const float o = slope == 0.0f ? 180.0f : orientation;
  const int steep = slope <= 30.0f ? 0 : 1;
  int oi;
  if ((o >= 315.0f && o <= 360.0f) || (o >= 0.0f && o < 45.0f)) oi = 0 + steep;
  else if (o >= 45.0f && o < 135.0f) oi = 2 + steep;
  else if (o >= 135.0f && o < 225.0f) oi = 4 + steep;
  else if (o >= 225.0f && o < 315.0f) oi = 6 + steep;
  else return __int_as_float(0x7fc00000);
  return (float)T.shade[mi][shi][oi][hi];
}

__device__ __forceinline__ float dm_prob_precip(float p, float e) {
  float a;
  if (e > 0.0f && e < 5.0f) a = -5.0f;
  else if (e >= 5.0f && e < 15.0f) a = -10.0f;
  else if (e >= 15.0f && e < 35.0f) a = -20.0f;
  else if (e >= 35.0f) a = -30.0f;
  else a = 0.0f;
  const float v = p + a;
  return v < 0.0f ? 0.0f : (v > 100.0f ? 100.0f : v);
}

__device__ __forceinline__ float dm_d1hr(float hcs, float prob_sc, float prob) {
  if (prob <= 0.0f) return hcs > 0.0f ? 30.0f : 0.0f;
  return prob_sc / prob * hcs;
}

__device__ __forceinline__ float dm_by_10hr(int hour, float m, float m6, float m15) {
  if (m == 0.0f) return 0.0f;
  const float at6 = m15 + (0.4142f * (m6 - m15));
  const float at15 = m6 - (0.5571f * (m6 - m15));
  if (fabsf(at6 - at15) < 0.001f) return at6 < 0.001f ? m : at6;
  if (hour >= 0 && hour < 6) return at15 + (((at6 - at15) / 15.0f) * (float)(hour + 15));
  if (hour >= 6 && hour < 15) return at6 + (((at15 - at6) / 9.0f) * (float)(hour - 6));
  if (hour >= 15 && hour < 24) return at15 + (((at6 - at15) / 15.0f) * (float)(hour - 15));
  return m;
}

// Portable arctangent of a non-negative ratio (the propagation code's
// series: octant reduction, odd series to u^19).
__device__ __forceinline__ float dm_atan_pos(float y) {
  const float mx = y > 1.0f ? y : 1.0f;
  const float mn = y > 1.0f ? 1.0f : y;
  const float t = mn / mx;
  float base = 0.0f, u = t;
  if (t > 0.414213562373095049f) {
    u = (t - 1.0f) / (t + 1.0f);
    base = 0.785398163397448309616f;
  }
  const float u2 = u * u;
  float p = __fmaf_rn(u2, 5.26315789e-2f, -5.88235294e-2f);
  p = __fmaf_rn(u2, p, 6.66666667e-2f);
  p = __fmaf_rn(u2, p, -7.69230769e-2f);
  p = __fmaf_rn(u2, p, 9.09090909e-2f);
  p = __fmaf_rn(u2, p, -1.11111111e-1f);
  p = __fmaf_rn(u2, p, 1.42857143e-1f);
  p = __fmaf_rn(u2, p, -2.00000000e-1f);
  p = __fmaf_rn(u2, p, 3.33333333e-1f);
  float a = __fmaf_rn(-(u * u2), p, u) + base;
  if (y > 1.0f) a = 1.57079632679489661923f - a;
  return a;
}

struct DmoistIn {
  const float *t, *rh, *cc;  // [24][n]
  const float *pp;           // [6][n]
  const float *slope, *aspect;
  const uint8_t *fuel;
};

// Dead fuel moisture of cell i at `hour` (percent): the 1-h moisture of that
// hour and of hours 6 and 15, the 10-h class interpolated from those, the
// 100-h class from the 10-h values (lib.rs:109-127).  fuel, slope and aspect
// are the cell's (already loaded by the caller).
__device__ __forceinline__ void dmoist_cell(const DmoistTables &T, const DmoistIn &in, uint64_t n,
                                            uint64_t i, int hour, int month, int fuel, float slope,
                                            float aspect, float &d1, float &d10, float &d100) {
  float ppmax = __int_as_float(0xff800000);  // -inf
#pragma unroll
  for (int d = 0; d < 6; ++d) ppmax = fmaxf(ppmax, dm_pp_effect(T, month, __ldg(in.pp + d * n + i), d));
  const float sdeg = dm_atan_pos(slope) * 180.0f / 3.14159274101257324f;
  const float adeg = aspect * 180.0f / 3.14159274101257324f;
  const int hours[3] = {hour, 6, 15};
  float m1[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int h = hours[k];
    const float t = __ldg(in.t + h * n + i), rh = __ldg(in.rh + h * n + i), cc = __ldg(in.cc + h * n + i);
    const float hcb = (float)dm_hcb(T, t, rh);
    const float hcs = fuel == 0 ? 0.0f : hcb + dm_corrector(T, adeg, sdeg, dm_shading(cc, fuel), month, h);
    const float p0 = dm_prob(T, t, cc, hcs, fuel);
    m1[k] = dm_d1hr(hcs, p0, dm_prob_precip(p0, ppmax));
  }
  const float m10h = dm_by_10hr(hour, m1[0], m1[1], m1[2]);
  const float m10_6 = dm_by_10hr(6, m1[1], m1[1], m1[2]);
  const float m10_15 = dm_by_10hr(15, m1[2], m1[1], m1[2]);
  d1 = m1[0];
  d10 = m10h;
  d100 = dm_by_10hr(hour, m10h, m10_6, m10_15);
}

// The tables in shared memory (per-lane indices would serialise constant
// reads); called by every thread of the block.
__device__ __forceinline__ void load_dmoist_tables(DmoistTables &T) {
  for (int k = threadIdx.x; k < (int)sizeof(DmoistTables); k += blockDim.x)
    reinterpret_cast<char *>(&T)[k] = reinterpret_cast<const char *>(&c_dm)[k];
  __syncthreads();
}

}  // namespace propag
