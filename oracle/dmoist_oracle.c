/*
 * CPU oracle (test infrastructure only) -- restatement of the reference's
 * hourly dead fuel moisture model, crates/dmoist/src/lib.rs.  Plain C, float
 * arithmetic in the reference's operation order (compile with
 * -ffp-contract=off); the look-up tables are the model's data, laid out here
 * as flat arrays.  The device kernel (propag-hidalgo_b200/csrc/dmoist.cu)
 * performs the same operations and is checked against this file bit for bit;
 * this file is pinned to the reference's fixtures (crates/dmoist/fixtures).
 *
 * One deliberate difference: the slope angle atan(slope) uses a portable
 * arctangent (the same code as the device: octant reduction + odd series),
 * not the platform atanf, so that CPU and GPU agree bit for bit; it differs
 * from a correctly rounded atanf by at most a few ulp, which changes the
 * result only for a slope within that distance of tan(30 deg).
 */
#include <math.h>
#include <stdint.h>

/* ---- tables (lib.rs:197-262, 272-453, 472-614) ---------------------------- */

/* Base humidity index by temperature class (6) and relative-humidity class
 * (21, 5 % steps).  The reference always uses its daytime table
 * (lib.rs:242: hora_idx = 0). */
static const int8_t HCB_DAY[6][21] = {
    {1, 2, 2, 3, 4, 5, 5, 6, 7, 8, 8, 8, 9, 9, 10, 11, 12, 12, 13, 13, 14},
    {1, 2, 2, 3, 4, 5, 5, 6, 7, 7, 7, 8, 9, 9, 10, 10, 11, 12, 13, 13, 13},
    {1, 2, 2, 3, 4, 5, 5, 6, 6, 7, 7, 8, 9, 9, 9, 10, 11, 12, 12, 12, 13},
    {1, 1, 2, 2, 3, 4, 5, 5, 6, 7, 7, 8, 8, 8, 9, 10, 10, 11, 12, 12, 13},
    {1, 1, 2, 2, 3, 4, 4, 5, 6, 7, 7, 8, 8, 8, 9, 10, 10, 11, 12, 12, 13},
    {1, 1, 2, 2, 3, 4, 4, 5, 6, 7, 7, 8, 8, 8, 9, 10, 10, 11, 12, 12, 12},
};

/* Ignition probability (%) by shading class (4: 0-10, 10-50, 50-90, 90-100 %),
 * dry-bulb temperature class (9: > 40, 35-40, ..., 0-5 C) and corrected
 * humidity index 1..18. */
static const uint8_t PROB_IGN[4][9][18] = {
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
};

/* Humidity-index correction by month class (3: May-Aug, Feb-Apr + Sep-Oct,
 * Nov-Jan), shading (2: exposed, shaded), exposure/slope (8: N, E, S, W each
 * <= 30 deg / > 30 deg) and hour class (6: 8-10, 10-12, ..., 18-20). */
static const int8_t SHADE_CORR[3][2][8][6] = {
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
};

/* Effect of one day's precipitation by season (2: Apr-Oct, rest), amount
 * class (4: [1,5), [5,15), [15,35), >= 35 mm) and days before the forecast
 * (6); -1 = the amount itself (lib.rs:147-183). */
static const int8_t PP_EFFECT[2][4][6] = {
    {{-1, -1, 0, 0, 0, 0}, {-1, 5, 1, 0, 0, 0}, {-1, 15, 5, 1, 0, 0}, {-1, 35, 15, 5, 1, 0}},
    {{-1, -1, -1, -1, 1, 0}, {-1, -1, -1, -1, 5, 1}, {-1, -1, -1, 15, 5, 1}, {-1, -1, 35, 15, 5, 1}},
};

/* ---- functions -------------------------------------------------------------- */

/* lib.rs:147-183 */
float odm_precipitation_effect(int month, float pp, int offset) {
  if (pp > 0.0f) {
    const int mi = (month >= 4 && month <= 10) ? 0 : 1;
    const int pi = (pp >= 1.0f && pp < 5.0f) ? 0 : (pp >= 5.0f && pp < 15.0f) ? 1
                 : (pp >= 15.0f && pp < 35.0f) ? 2 : 3;
    const int e = PP_EFFECT[mi][pi][offset];
    if (e > -1) return (float)e;
  }
  return pp;
}

/* lib.rs:192-195: maximum over the six days (NEG_INFINITY start) */
float odm_maximum_precipitation_effect(int month, const float pp[6]) {
  float m = -INFINITY;
  for (int i = 0; i < 6; ++i) {
    const float e = odm_precipitation_effect(month, pp[i], i);
    m = fmaxf(m, e);
  }
  return m;
}

/* lib.rs:197-262 */
int odm_humidity_content_base(float t, float rh, int hour) {
  (void)hour;
  float hf = floorf(rh / 5.0f);
  hf = hf < 0.0f ? 0.0f : (hf > 20.0f ? 20.0f : hf);
  if (hf != hf) hf = 0.0f; /* NaN: class 0, as the reference's saturating cast */
  const int hi = (int)hf;
  int ti;
  if (t < 0.0f) ti = 0;
  else if (t >= 0.0f && t <= 9.0f) ti = 1;
  else if (t > 9.0f && t <= 20.0f) ti = 2;
  else if (t > 20.0f && t <= 31.0f) ti = 3;
  else if (t > 31.0f && t <= 42.0f) ti = 4;
  else ti = 5;
  return HCB_DAY[ti][hi];
}

/* lib.rs:264-270 */
float odm_shading(float cloud, int fuel) {
  float s = cloud * 0.75f;
  if (fuel >= 7 && fuel <= 12) s = s < 50.0f ? 75.0f : 100.0f;
  return s;
}

/* lib.rs:272-453 */
float odm_ignition_probability(float t, float cloud, float hcs, int fuel) {
  if (fuel == 0) return 0.0f;
  if (!(hcs > 0.0f && hcs < 18.0f)) return 0.0f;
  const float s = odm_shading(cloud, fuel);
  const int si = (s >= 0.0f && s < 10.0f) ? 0 : (s >= 10.0f && s < 50.0f) ? 1
               : (s >= 50.0f && s < 90.0f) ? 2 : 3;
  float tf = 9.0f - ceilf(t / 5.0f);
  tf = tf < 0.0f ? 0.0f : (tf > 8.0f ? 8.0f : tf);
  if (tf != tf) tf = 0.0f;
  const int ti = (int)tf;
  /* hcs in (0, 1) has no table row (the reference's usize index underflows);
   * the model only produces integer indices >= 1 there */
  const int hci = (int)floorf(hcs) - 1;
  if (hci < 0) return 0.0f;
  return (float)PROB_IGN[si][ti][hci];
}

static int is_north(float o) { return (o >= 315.0f && o <= 360.0f) || (o >= 0.0f && o < 45.0f); }
static int is_east(float o) { return o >= 45.0f && o < 135.0f; }
static int is_south(float o) { return o >= 135.0f && o < 225.0f; }
static int is_west(float o) { return o >= 225.0f && o < 315.0f; }

/* lib.rs:472-614; NaN for a month outside 1..12 or an orientation outside [0, 360] */
float odm_corrector_for_shading(float orientation, float slope, float shade, int month, int hour_in) {
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
  else return NAN;
  const float o = slope == 0.0f ? 180.0f : orientation;
  const int steep = slope <= 30.0f ? 0 : 1;
  int oi;
  if (is_north(o)) oi = 0 + steep;
  else if (is_east(o)) oi = 2 + steep;
  else if (is_south(o)) oi = 4 + steep;
  else if (is_west(o)) oi = 6 + steep;
  else return NAN;
  return (float)SHADE_CORR[mi][shi][oi][hi];
}

/* lib.rs:616-631 */
float odm_correct_hcb_for_shading(float hcb, float cloud, int month, float orientation, float slope,
                                  int fuel, int hour) {
  if (fuel == 0) return 0.0f;
  const float s = odm_shading(cloud, fuel);
  return hcb + odm_corrector_for_shading(orientation, slope, s, month, hour);
}

/* lib.rs:633-650 */
float odm_correct_probability_for_precipitation(float p, float e) {
  float a;
  if (e > 0.0f && e < 5.0f) a = -5.0f;
  else if (e >= 5.0f && e < 15.0f) a = -10.0f;
  else if (e >= 15.0f && e < 35.0f) a = -20.0f;
  else if (e >= 35.0f) a = -30.0f;
  else a = 0.0f;
  const float v = p + a;
  return v < 0.0f ? 0.0f : (v > 100.0f ? 100.0f : v);
}

/* lib.rs:652-663 */
float odm_d1hr(float hcs, float prob_sc, float prob) {
  if (prob <= 0.0f) return hcs > 0.0f ? 30.0f : 0.0f;
  return prob_sc / prob * hcs;
}

/* lib.rs:671-703 */
float odm_moisture_by_10hr(int hour, float m, float m6, float m15) {
  if (m == 0.0f) return 0.0f;
  const float at6 = m15 + (0.4142f * (m6 - m15));
  const float at15 = m6 - (0.5571f * (m6 - m15));
  if (fabsf(at6 - at15) < 0.001f) return at6 < 0.001f ? m : at6;
  if (hour >= 0 && hour < 6) return at15 + (((at6 - at15) / 15.0f) * (float)(hour + 15));
  if (hour >= 6 && hour < 15) return at6 + (((at15 - at6) / 9.0f) * (float)(hour - 6));
  if (hour >= 15 && hour < 24) return at15 + (((at6 - at15) / 15.0f) * (float)(hour - 15));
  return m;
}

/* lib.rs:705-715 */
float odm_live_moisture(int month) {
  switch (month) {
    case 1: case 2: return 100.0f;
    case 3: case 4: case 5: return 200.0f;
    case 6: return 100.0f;
    case 7: case 8: return 80.0f;
    case 9: case 10: return 90.0f;
    case 11: case 12: return 100.0f;
    default: return NAN;
  }
}

/* Portable arctangent for a non-negative ratio: the device code's series
 * (octant reduction, t > tan(pi/8) mapped through (t-1)/(t+1), odd series to
 * u^19), float operations only. */
static float odm_atan_pos(float y) {
  const float mx = y > 1.0f ? y : 1.0f;
  const float mn = y > 1.0f ? 1.0f : y;
  const float t = mn / mx;
  float base = 0.0f, u = t;
  if (t > 0.414213562373095049f) {
    u = (t - 1.0f) / (t + 1.0f);
    base = 0.785398163397448309616f;
  }
  const float u2 = u * u;
  float p = fmaf(u2, 5.26315789e-2f, -5.88235294e-2f);
  p = fmaf(u2, p, 6.66666667e-2f);
  p = fmaf(u2, p, -7.69230769e-2f);
  p = fmaf(u2, p, 9.09090909e-2f);
  p = fmaf(u2, p, -1.11111111e-1f);
  p = fmaf(u2, p, 1.42857143e-1f);
  p = fmaf(u2, p, -2.00000000e-1f);
  p = fmaf(u2, p, 3.33333333e-1f);
  float a = fmaf(-(u * u2), p, u) + base;
  if (y > 1.0f) a = 1.57079632679489661923f - a;
  return a;
}

/* Slope ratio -> degrees, aspect radians -> degrees (lib.rs:81-82). */
static float slope_deg(float slope) { return odm_atan_pos(slope) * 180.0f / 3.14159274101257324f; }
static float aspect_deg(float aspect) { return aspect * 180.0f / 3.14159274101257324f; }

/* One hour's 1-h moisture (lib.rs:72-105). */
static float d1hr_at(int h, const float *t, const float *rh, const float *cc, float sdeg, float adeg,
                     int month, int fuel, float ppmax) {
  const float hcb = (float)odm_humidity_content_base(t[h], rh[h], h);
  const float hcs = odm_correct_hcb_for_shading(hcb, cc[h], month, adeg, sdeg, fuel, h);
  const float p0 = odm_ignition_probability(t[h], cc[h], hcs, fuel);
  const float p1 = odm_correct_probability_for_precipitation(p0, ppmax);
  return odm_d1hr(hcs, p0, p1);
}

/* calculate_hourly_fuel_moisture (lib.rs:55-137) for one site: 24 hours. */
void odm_hourly(const float t[24], const float rh[24], const float cc[24], float slope,
                float aspect, const float pp[6], int month, int fuel, float d1[24], float d10[24],
                float d100[24]) {
  const float ppmax = odm_maximum_precipitation_effect(month, pp);
  const float sd = slope_deg(slope), ad = aspect_deg(aspect);
  for (int h = 0; h < 24; ++h) d1[h] = d1hr_at(h, t, rh, cc, sd, ad, month, fuel, ppmax);
  for (int h = 0; h < 24; ++h) d10[h] = odm_moisture_by_10hr(h, d1[h], d1[6], d1[15]);
  for (int h = 0; h < 24; ++h) d100[h] = odm_moisture_by_10hr(h, d10[h], d10[6], d10[15]);
}

/* Per-cell version over rasters: weather hour-major (t[h * n + i]),
 * precipitation day-major (pp[d * n + i]); one output hour.  Values in the
 * model's percent units. */
void odm_cells(int64_t n, int hour, int month, const float *t, const float *rh, const float *cc,
               const float *slope, const float *aspect, const uint8_t *fuel, const float *pp,
               float *d1, float *d10, float *d100) {
  for (int64_t i = 0; i < n; ++i) {
    float tt[24], rr[24], cl[24], p[6], a1[24], a10[24], a100[24];
    for (int h = 0; h < 24; ++h) {
      tt[h] = t[(int64_t)h * n + i];
      rr[h] = rh[(int64_t)h * n + i];
      cl[h] = cc[(int64_t)h * n + i];
    }
    for (int k = 0; k < 6; ++k) p[k] = pp[(int64_t)k * n + i];
    odm_hourly(tt, rr, cl, slope[i], aspect[i], p, month, fuel[i], a1, a10, a100);
    d1[i] = a1[hour];
    d10[i] = a10[hour];
    d100[i] = a100[hour];
  }
}

/* Wind from its components (fixtures mod_viento.txt / dir_viento.txt): speed
 * and the compass direction the vector points to, degrees in [0, 360). */
double odm_wind_speed(double u, double v) { return sqrt(u * u + v * v); }
double odm_wind_direction(double u, double v) {
  if (u == 0.0 && v == 0.0) return 0.0;
  double d = atan2(u, v) * 180.0 / 3.14159265358979323846;
  return d < 0.0 ? d + 360.0 : d;
}
