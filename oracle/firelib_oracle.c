/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle for the per-cell fire-behaviour pass.
 *
 * This file restates, in IEEE double precision, the Rothermel/BEHAVE fire
 * behaviour of the reference crate `firelib` (Rust).  It is used by the tests,
 * by `__graft_entry__.smoke()` and by `bench.py`'s CPU-baseline leg as the
 * checker; the product path never links or calls it.
 *
 * What is restated (all paths relative to the reference project):
 *   - fuel catalog constants  : crates/firelib/src/firelib.rs:554-979 (ParticleDef,
 *                               Particle::make, FuelDef::*, Fuel::make) and the
 *                               NFFL table in crates/firelib/src/lib.rs:126-268
 *   - unit conversions        : crates/firelib/src/units.rs:28-30,123-210
 *   - per-cell burn           : Fuel::burn / burn_simple (firelib.rs:996-1030),
 *                               rx_int_rbqig (:1031-1058), eta_m (:1060-1076),
 *                               calculate_wind_dependent_vars (:1078-1145),
 *                               wind_slope_situation (:1146-1167),
 *                               eccentricity (:1171-1174), phi_* (:1176-1188)
 *   - Byram / flame extras    : Fire::byrams_max / flame_max / flame_length
 *                               (firelib.rs:424-441)
 *
 * Threshold comparisons of the f32 reference (SMIDGEN = 1e-6 in f32,
 * crates/firelib/src/f32.rs:5) are kept: inputs are compared as the reference
 * device path compares them.  Everything else is evaluated in double.
 *
 * Output fields per cell (SI units, as crates/firelib/src/cuda.rs:9-55 writes
 * them, plus Byram intensity and flame length):
 *   0 rx_int        W/m^2        5 azimuth_max   rad
 *   1 speed0        m/s          6 eccentricity  -
 *   2 hpua          J/m^2        7 residence     s
 *   3 phi_eff_wind  -            8 byrams_max    W/m
 *   4 speed_max     m/s          9 flame_max     m
 * Cells whose fuel code has no particles (0 and >= 14) are all zeros, as the
 * reference leaves them (crates/propag/src/propag.rs:437-439).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#define OFL_MAX_PARTICLES 5
#define OFL_MAX_FUELS 20
#define OFL_NFIELDS 10

static const double FOOT_TO_M = 0.3048;     /* units.rs:28 */
static const double BTU = 1054.35;           /* units.rs:30 */
static const float SMIDGEN_F = 1e-6f;        /* f32.rs:5 */
static const double SMIDGEN = 1e-6;

enum { P_DEAD = 0, P_HERB = 1, P_WOOD = 2 };
enum { LIFE_DEAD = 0, LIFE_ALIVE = 1 };

typedef struct {
  int type;
  double load, savr, density, heat, si_total, si_effective;
} pdef_t;

typedef struct {
  int type, life, size_class;
  double load, savr, density, heat, si_total, si_effective;
  double area_weight, surface_area, sigma_factor, size_class_weight;
} particle_t;

typedef struct {
  int n_particles, n_dead, has_live;
  particle_t p[OFL_MAX_PARTICLES];
  double depth, mext, inv_mext;
  double live_area_weight, dead_area_weight;
  double fine_dead_factor, live_ext_factor, fuel_bed_bulk_dens;
  double residence_time, flux_ratio, slope_k;
  double wind_b, wind_b_inv, wind_e, wind_k, sigma, beta;
  double life_rx_factor_alive, life_rx_factor_dead;
} fuel_t;

/* NFFL standard catalog, crates/firelib/src/lib.rs:126-268:
 * {depth ft, mext, n, {type, load lb/ft2, savr 1/ft} x n} */
typedef struct {
  double depth, mext;
  int n;
  struct { int type; double load, savr; } p[4];
} nffl_t;

static const nffl_t NFFL[14] = {
    {0.1, 0.01, 0, {{0}}},
    {1.0, 0.12, 1, {{P_DEAD, 0.0340, 3500.0}}},
    {1.0, 0.15, 4, {{P_DEAD, 0.0920, 3000.0}, {P_DEAD, 0.0460, 109.0}, {P_DEAD, 0.0230, 30.0}, {P_HERB, 0.0230, 1500.0}}},
    {2.5, 0.25, 1, {{P_DEAD, 0.1380, 1500.0}}},
    {6.0, 0.2, 4, {{P_DEAD, 0.2300, 2000.0}, {P_DEAD, 0.1840, 109.0}, {P_DEAD, 0.0920, 30.0}, {P_WOOD, 0.2300, 1500.0}}},
    {2.0, 0.2, 3, {{P_DEAD, 0.0460, 2000.0}, {P_DEAD, 0.0230, 109.0}, {P_WOOD, 0.0920, 1500.0}}},
    {2.5, 0.25, 3, {{P_DEAD, 0.0690, 1750.0}, {P_DEAD, 0.1150, 109.0}, {P_DEAD, 0.0920, 30.0}}},
    {2.5, 0.40, 4, {{P_DEAD, 0.0520, 1750.0}, {P_DEAD, 0.0860, 109.0}, {P_DEAD, 0.0690, 30.0}, {P_WOOD, 0.0170, 1550.0}}},
    {0.2, 0.30, 3, {{P_DEAD, 0.0690, 2000.0}, {P_DEAD, 0.0460, 109.0}, {P_DEAD, 0.1150, 30.0}}},
    {0.2, 0.25, 3, {{P_DEAD, 0.1340, 2500.0}, {P_DEAD, 0.0190, 109.0}, {P_DEAD, 0.0070, 30.0}}},
    {1.0, 0.25, 4, {{P_DEAD, 0.1380, 2000.0}, {P_DEAD, 0.0920, 109.0}, {P_DEAD, 0.2300, 30.0}, {P_WOOD, 0.0920, 1500.0}}},
    {1.0, 0.15, 3, {{P_DEAD, 0.0690, 1500.0}, {P_DEAD, 0.2070, 109.0}, {P_DEAD, 0.2530, 30.0}}},
    {2.3, 0.20, 3, {{P_DEAD, 0.1840, 1500.0}, {P_DEAD, 0.6440, 109.0}, {P_DEAD, 0.7590, 30.0}}},
    {3.0, 0.25, 3, {{P_DEAD, 0.3220, 1500.0}, {P_DEAD, 0.0580, 109.0}, {P_DEAD, 1.2880, 30.0}}},
};

static double safe_div(double a, double b) { return b > SMIDGEN ? a / b : 0.0; } /* firelib.rs:1191-1197 */

/* ParticleDef::size_class, firelib.rs:577-592 (savr in 1/ft) */
static int size_class(double savr) {
  if (savr > 1200.0) return 0;
  if (savr > 192.0) return 1;
  if (savr > 96.0) return 2;
  if (savr > 48.0) return 3;
  if (savr > 16.0) return 4;
  return 5;
}

static int life_of(int type) { return type == P_DEAD ? LIFE_DEAD : LIFE_ALIVE; }

/* ParticleDef::surface_area, firelib.rs:643-648 */
static double surface_area(const pdef_t *d) { return safe_div(d->load * d->savr, d->density); }

/* ParticleDef::area_weight, firelib.rs:605-616 */
static double area_weight(const pdef_t *d, const pdef_t *all, int n) {
  double total = 0.0;
  for (int i = 0; i < n; i++)
    if (life_of(all[i].type) == life_of(d->type)) total += surface_area(&all[i]);
  return safe_div(surface_area(d), total);
}

/* ParticleDef::size_class_weight, firelib.rs:617-642 */
static double size_class_weight(const pdef_t *d, const pdef_t *all, int n) {
  double r = 0.0;
  for (int i = 0; i < n; i++)
    if (life_of(all[i].type) == life_of(d->type) && size_class(all[i].savr) == size_class(d->savr))
      r += area_weight(&all[i], all, n);
  return r;
}

static fuel_t g_catalog[OFL_MAX_FUELS];
static int g_catalog_ready = 0;

/* Fuel::standard + Fuel::make, firelib.rs:870-979 (imperial internal units). */
static void build_fuel(int code, fuel_t *f) {
  memset(f, 0, sizeof(*f));
  if (code >= 14) return;
  const nffl_t *src = &NFFL[code];
  pdef_t defs[OFL_MAX_PARTICLES];
  int n = src->n;
  for (int i = 0; i < n; i++) {
    /* ParticleDef::standard, firelib.rs:557-573: density 32 lb/ft3, heat 8000
     * BTU/lb, total silica 0.0555, effective silica 0.01 */
    defs[i].type = src->p[i].type;
    defs[i].load = src->p[i].load;
    defs[i].savr = src->p[i].savr;
    defs[i].density = 32.0;
    defs[i].heat = 8000.0;
    defs[i].si_total = 0.0555;
    defs[i].si_effective = 0.01;
  }
  /* dead particles first, then live ones (firelib.rs:883-919) */
  int k = 0;
  for (int pass = 0; pass < 2; pass++) {
    for (int i = 0; i < n; i++) {
      int life = life_of(defs[i].type);
      if ((pass == 0 && life != LIFE_DEAD) || (pass == 1 && life != LIFE_ALIVE)) continue;
      particle_t *p = &f->p[k++];
      p->type = defs[i].type;
      p->life = life;
      p->size_class = size_class(defs[i].savr);
      p->load = defs[i].load;
      p->savr = defs[i].savr;
      p->density = defs[i].density;
      p->heat = defs[i].heat;
      p->si_total = defs[i].si_total;
      p->si_effective = defs[i].si_effective;
      p->area_weight = area_weight(&defs[i], defs, n);
      p->size_class_weight = size_class_weight(&defs[i], defs, n);
      p->surface_area = surface_area(&defs[i]);
      p->sigma_factor = exp(safe_div(-138.0, defs[i].savr)); /* firelib.rs:649-652 */
    }
    if (pass == 0) f->n_dead = k;
  }
  f->n_particles = n;
  f->has_live = n > f->n_dead;
  if (n == 0) return;

  const double depth = src->depth;
  f->depth = depth;
  f->mext = src->mext;
  f->inv_mext = 1.0 / src->mext;

  double total_area = 0.0; /* FuelDef::total_area, :717-722 */
  for (int i = 0; i < n; i++) total_area += f->p[i].surface_area;
  double law[2] = {0, 0}, lsavr[2] = {0, 0}, lheat[2] = {0, 0}, lseff[2] = {0, 0};
  double lload[2] = {0, 0}, lfine[2] = {0, 0};
  double beta_sum = 0.0, bulk = 0.0;
  for (int i = 0; i < n; i++) {
    const particle_t *p = &f->p[i];
    law[p->life] += p->surface_area / total_area;                    /* :723-733 */
    lsavr[p->life] += p->area_weight * p->savr;                       /* :755-763 */
    lheat[p->life] += p->area_weight * p->heat;                       /* :764-772 */
    lseff[p->life] += p->area_weight * p->si_effective;               /* :773-781 */
    lload[p->life] += p->size_class_weight * p->load * (1.0 - p->si_total); /* :746-754 */
    if (p->life == LIFE_ALIVE)                                        /* :734-745 */
      lfine[LIFE_ALIVE] += p->load * exp(-500.0 / p->savr);
    else
      lfine[LIFE_DEAD] += p->load * p->sigma_factor;
    beta_sum += p->load / p->density;                                 /* :809-814 */
    bulk += p->load / depth;                                          /* :840-846 */
  }
  const double sigma = law[LIFE_ALIVE] * lsavr[LIFE_ALIVE] + law[LIFE_DEAD] * lsavr[LIFE_DEAD]; /* :795-798 */
  const double beta = beta_sum / depth;
  const double ratio = beta / (3.348 / pow(sigma, 0.8189));                              /* :799-801 */
  const double flux_ratio = exp((0.792 + 0.681 * sqrt(sigma)) * (beta + 0.1)) / (192.0 + 0.2595 * sigma); /* :802-808 */
  const double sigma15 = pow(sigma, 1.5);                                                /* :815-824 */
  const double gamma_max = sigma15 / (495.0 + 0.0594 * sigma15);
  const double aa = 133.0 / pow(sigma, 0.7913);
  const double gamma = gamma_max * pow(ratio, aa) * exp(aa * (1.0 - ratio));
  double eta_s[2];
  for (int l = 0; l < 2; l++) { /* :782-794 */
    if (lseff[l] > SMIDGEN) {
      double eta = 0.174 / pow(lseff[l], 0.19);
      eta_s[l] = eta < 1.0 ? eta : 1.0;
    } else {
      eta_s[l] = 1.0;
    }
  }
  f->life_rx_factor_alive = lload[LIFE_ALIVE] * lheat[LIFE_ALIVE] * eta_s[LIFE_ALIVE] * gamma; /* :826-831 */
  f->life_rx_factor_dead = lload[LIFE_DEAD] * lheat[LIFE_DEAD] * eta_s[LIFE_DEAD] * gamma;
  f->live_area_weight = law[LIFE_ALIVE];
  f->dead_area_weight = law[LIFE_DEAD];
  f->fine_dead_factor = 1.0 / lfine[LIFE_DEAD];
  f->live_ext_factor = 2.9 * safe_div(lfine[LIFE_DEAD], lfine[LIFE_ALIVE]); /* :833-838 */
  f->fuel_bed_bulk_dens = bulk;
  f->residence_time = 384.0 / sigma; /* :848-850 */
  f->flux_ratio = flux_ratio;
  f->slope_k = 5.275 * pow(beta, -0.3); /* :852-854 */
  /* wind_bke, :856-867 */
  f->wind_b = 0.02526 * pow(sigma, 0.54);
  const double c = 7.47 * exp(-0.133 * pow(sigma, 0.55));
  const double e = 0.715 * exp(-0.000359 * sigma);
  f->wind_k = c * pow(ratio, -e);
  f->wind_e = pow(ratio, e) / c;
  f->wind_b_inv = 1.0 / f->wind_b;
  f->sigma = sigma;
  f->beta = beta;
}

static void ensure_catalog(void) {
  if (g_catalog_ready) return;
  for (int i = 0; i < OFL_MAX_FUELS; i++) build_fuel(i, &g_catalog[i]);
  g_catalog_ready = 1;
}

/* Particle::moisture, firelib.rs:699-713 */
static double moisture(const particle_t *p, const double m[5]) {
  switch (p->type) {
  case P_HERB: return m[3];
  case P_WOOD: return m[4];
  default:
    if (p->size_class <= 1) return m[0];
    if (p->size_class <= 3) return m[1];
    return m[2];
  }
}

/* Fuel::eta_m, firelib.rs:1060-1076 */
static double eta_m(const fuel_t *f, int life, double life_moist, double wfmd) {
  double life_mext;
  if (life == LIFE_DEAD) {
    life_mext = f->mext;
  } else if (f->has_live) {
    double fdmois = wfmd * f->fine_dead_factor;
    double live_mext = f->live_ext_factor * (1.0 - fdmois * f->inv_mext) - 0.226;
    life_mext = live_mext > f->mext ? live_mext : f->mext;
  } else {
    life_mext = 0.0;
  }
  if (life_moist >= life_mext) return 0.0;
  double rt = life_moist / life_mext;
  return 1.0 - 2.59 * rt + 5.11 * rt * rt - 3.52 * rt * rt * rt;
}

enum { NO_SPREAD = 0, NO_SLOPE_NO_WIND, WIND_NO_SLOPE, SLOPE_NO_WIND, UP_SLOPE, CROSS_SLOPE };

/* Burns one cell.  Returns the wind/slope situation or -1 when the fuel has no
 * particles (no fire).  out[] gets the 10 SI fields listed at the top. */
static int burn_cell(uint8_t code, const float in[9], double out[OFL_NFIELDS]) {
  memset(out, 0, sizeof(double) * OFL_NFIELDS);
  if (code >= OFL_MAX_FUELS) return -1;
  const fuel_t *f = &g_catalog[code];
  if (f->n_particles == 0) return -1; /* Catalog::get, firelib.rs:382-387 */
  const double m[5] = {in[0], in[1], in[2], in[3], in[4]};
  const float ws_f = in[5], waz_f = in[6], slope_f = in[7], aspect_f = in[8];

  /* rx_int_rbqig, firelib.rs:1031-1058 */
  double wfmd = 0.0, alive_moist = 0.0, dead_moist = 0.0, rbqig = 0.0;
  for (int i = 0; i < f->n_particles; i++) {
    const particle_t *p = &f->p[i];
    double mo = moisture(p, m);
    double law = p->life == LIFE_ALIVE ? f->live_area_weight : f->dead_area_weight;
    rbqig += (250.0 + 1116.0 * mo) * p->area_weight * law * p->sigma_factor;
    if (p->life == LIFE_ALIVE) {
      alive_moist += p->area_weight * mo;
    } else {
      dead_moist += p->area_weight * mo;
      wfmd += mo * p->sigma_factor * p->load;
    }
  }
  const double rx_int = f->life_rx_factor_alive * eta_m(f, LIFE_ALIVE, alive_moist, wfmd) +
                        f->life_rx_factor_dead * eta_m(f, LIFE_DEAD, dead_moist, wfmd);
  rbqig *= f->fuel_bed_bulk_dens;
  const double speed0 = rx_int * f->flux_ratio / rbqig;

  /* calculate_wind_dependent_vars, firelib.rs:1078-1145 */
  const double slope = slope_f;
  const double phi_slope = f->slope_k * slope * slope;
  const double ws_fpm = (double)ws_f / (FOOT_TO_M / 60.0);
  const double phi_wind = f->wind_k * pow(ws_fpm, f->wind_b);
  const double phi_ew = phi_slope + phi_wind;
  const double speed_max1 = speed0 * (1.0 + phi_ew);
  const double aspect = aspect_f;
  const double upslope = aspect >= M_PI ? aspect - M_PI : aspect + M_PI; /* :400-409 */
  const double wind_az = waz_f;
  const double max_wind = 0.9 * rx_int;

  int situation; /* wind_slope_situation, :1146-1167 */
  if (speed0 < SMIDGEN_F) situation = NO_SPREAD;
  else if (phi_ew < SMIDGEN_F) situation = NO_SLOPE_NO_WIND;
  else if (slope_f < SMIDGEN_F) situation = WIND_NO_SLOPE;
  else if (ws_f < SMIDGEN_F) situation = SLOPE_NO_WIND;
  else if (fabs(upslope - wind_az) < SMIDGEN_F) situation = UP_SLOPE;
  else situation = CROSS_SLOPE;

  double pew, ew, smax, az;
  switch (situation) {
  case NO_SPREAD: pew = phi_ew; ew = 0.0; smax = 0.0; az = 0.0; break;
  case NO_SLOPE_NO_WIND: pew = phi_ew; ew = 0.0; smax = speed0; az = 0.0; break;
  case WIND_NO_SLOPE: pew = phi_ew; ew = ws_fpm; smax = speed_max1; az = wind_az; break;
  case SLOPE_NO_WIND:
  case UP_SLOPE:
    pew = phi_ew; ew = pow(phi_ew * f->wind_e, f->wind_b_inv); smax = speed_max1; az = upslope; break;
  default: {
    const double wind_rate = speed0 * phi_wind;
    const double slope_rate = speed0 * phi_slope;
    const double split = upslope <= wind_az ? wind_az - upslope : 2.0 * M_PI - upslope + wind_az;
    const double x = slope_rate + wind_rate * cos(split);
    const double y = wind_rate * sin(split);
    const double rv = sqrt(x * x + y * y);
    const double speed_max2 = speed0 + rv;
    const double phi_ew2 = speed_max2 / speed0 - 1.0;
    const double eff_wind = pow(phi_ew2 * f->wind_e, f->wind_b_inv);
    const double al = asin(fabs(y) / rv);
    double split2;
    if (x >= 0.0 && y >= 0.0) split2 = al;
    else if (x >= 0.0) split2 = 2.0 * M_PI - al;
    else if (y >= 0.0) split2 = M_PI - al;
    else split2 = M_PI + al;
    double azm = upslope + split2;
    if (azm > 2.0 * M_PI) azm -= 2.0 * M_PI;
    pew = phi_ew2; ew = eff_wind; smax = speed_max2; az = azm;
  }
  }
  /* check_wind_limit, :1091-1099 (not applied to NoSpread / NoSlopeNoWind) */
  if (situation >= WIND_NO_SLOPE && ew > max_wind) {
    pew = f->wind_k * pow(max_wind, f->wind_b);
    ew = max_wind;
    smax = speed0 * (1.0 + pew);
    situation += 10; /* reported: the wind limit applied */
  }
  /* eccentricity, :1171-1174 */
  const double lw = 1.0 + 0.002840909 * ew;
  const double ecc = sqrt(lw * lw - 1.0) / lw;
  /* Byram's intensity and flame length, :424-441 (imperial -> SI below) */
  const double byrams = f->residence_time * smax * rx_int / 60.0; /* BTU/ft/s */
  const double flame = byrams > SMIDGEN ? 0.45 * pow(byrams, 0.46) : 0.0; /* ft */

  out[0] = rx_int * (BTU / (FOOT_TO_M * FOOT_TO_M) / 60.0);
  out[1] = speed0 * (FOOT_TO_M / 60.0);
  out[2] = rx_int * f->residence_time * (BTU / (FOOT_TO_M * FOOT_TO_M));
  out[3] = pew;
  out[4] = smax * (FOOT_TO_M / 60.0);
  out[5] = az;
  out[6] = ecc;
  out[7] = f->residence_time * 60.0;
  out[8] = byrams * (BTU / FOOT_TO_M);
  out[9] = flame * FOOT_TO_M;
  return situation;
}

/* ---- exported API (ctypes) ------------------------------------------------ */

/* Fuel-level constants in imperial units, for cross-checking the product's
 * catalog: per fuel [n_particles, sigma, beta, flux_ratio, slope_k, wind_b,
 * wind_e, wind_k, life_rx_factor_alive, life_rx_factor_dead, residence_time,
 * fuel_bed_bulk_dens, live_ext_factor, fine_dead_factor, mext,
 * live_area_weight, dead_area_weight]. */
int ofl_catalog_f64(double *out, int stride) {
  ensure_catalog();
  if (stride < 17) return -1;
  for (int i = 0; i < OFL_MAX_FUELS; i++) {
    const fuel_t *f = &g_catalog[i];
    double *o = out + (size_t)i * stride;
    o[0] = f->n_particles; o[1] = f->sigma; o[2] = f->beta; o[3] = f->flux_ratio;
    o[4] = f->slope_k; o[5] = f->wind_b; o[6] = f->wind_e; o[7] = f->wind_k;
    o[8] = f->life_rx_factor_alive; o[9] = f->life_rx_factor_dead;
    o[10] = f->residence_time; o[11] = f->fuel_bed_bulk_dens; o[12] = f->live_ext_factor;
    o[13] = f->fine_dead_factor; o[14] = f->mext; o[15] = f->live_area_weight;
    o[16] = f->dead_area_weight;
  }
  return 0;
}

/* Per-cell burn over structure-of-arrays inputs (the TerrainCuda layout,
 * crates/firelib/src/firelib.rs:98-109).  out is n x 10 row-major;
 * situation (may be NULL) gets the wind/slope case or -1. */
int64_t ofl_burn_f64(int64_t n, const uint8_t *fuel, const float *d1, const float *d10,
                     const float *d100, const float *herb, const float *wood,
                     const float *wind_speed, const float *wind_azimuth, const float *slope,
                     const float *aspect, double *out, int32_t *situation) {
  ensure_catalog();
  int64_t burning = 0;
  for (int64_t i = 0; i < n; i++) {
    const float in[9] = {d1[i], d10[i], d100[i], herb[i], wood[i],
                         wind_speed[i], wind_azimuth[i], slope[i], aspect[i]};
    int s = burn_cell(fuel[i], in, out + i * OFL_NFIELDS);
    if (situation) situation[i] = s;
    burning += s >= 0;
  }
  return burning;
}
