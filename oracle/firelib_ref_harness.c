/*
 * TEST INFRASTRUCTURE ONLY -- drives the reference's own C fireLib
 * (crates/firelib-sys/fireLib.c, compiled from the reference sources by
 * oracle/Makefile into oracle/_ref/) exactly as the reference's quickcheck
 * harness does (crates/firelib/src/lib.rs:312-367):
 *   Fire_FuelCatalogCreateStandard("standard", 13)
 *   Fire_SpreadNoWindNoSlope(cat, fuel, [d1, d10, d100, 0, herb, wood])
 *   Fire_SpreadWindSlopeMax(cat, fuel, ws ft/min, wind_az deg, slope, aspect deg)
 *   Fire_SpreadAtAzimuth(cat, fuel, azimuthMax, FIRE_BYRAMS | FIRE_FLAME)
 * and converts the imperial outputs to the same 10 SI fields as the FP64
 * restatement in oracle/firelib_oracle.c.  Fuel codes outside 1..13 produce
 * zeros (the Rust catalog has no fire for them).
 *
 * ref_burn_c_rust_catalog does the same with one entry of the C catalog set
 * to the Rust catalog's value: the 10-h dead load of NFFL13, 1.0580 in
 * fireLib.c (fireLib.c:1316) and 0.0580 in crates/firelib/src/lib.rs:262.
 * The reference's own quickcheck comparison draws fuel codes 0..12 only
 * (lib.rs:417), so it never meets that difference.
 */
#include "fireLib.h"
#include <stdint.h>

static const double FOOT_TO_M = 0.3048;
static const double BTU = 1054.35;

static int64_t burn(int rust_nffl13, int64_t n, const uint8_t *fuel, const float *d1,
                    const float *d10, const float *d100, const float *herb, const float *wood,
                    const float *wind_speed, const float *wind_azimuth, const float *slope,
                    const float *aspect, double *out) {
  FuelCatalogPtr cat = Fire_FuelCatalogCreateStandard("standard", 13);
  if (!cat) return -1;
  /* particle 1 of model 13 is its 10-h dead class; its surface area is set
     from the load when the particle is added (fireLib.c:1719), the
     combustion terms on the model's first spread call */
  if (rust_nffl13) {
    Fuel_Load(cat, 13, 1) = 0.0580;
    Fuel_SurfaceArea(cat, 13, 1) = Fuel_Load(cat, 13, 1) * Fuel_Savr(cat, 13, 1) / Fuel_Density(cat, 13, 1);
  }
  int64_t burning = 0;
  for (int64_t i = 0; i < n; i++) {
    double *o = out + i * 10;
    for (int k = 0; k < 10; k++) o[k] = 0.0;
    int code = fuel[i];
    if (code < 1 || code > 13) continue;
    double m[FIRE_MCLASSES] = {d1[i], d10[i], d100[i], 0.0, herb[i], wood[i]};
    Fire_SpreadNoWindNoSlope(cat, code, m);
    Fire_SpreadWindSlopeMax(cat, code, (double)wind_speed[i] / (FOOT_TO_M / 60.0),
                            (double)wind_azimuth[i] * 180.0 / M_PI, (double)slope[i],
                            (double)aspect[i] * 180.0 / M_PI);
    FuelModelPtr f = cat->modelPtr[code];
    Fire_SpreadAtAzimuth(cat, code, f->azimuthMax, FIRE_BYRAMS | FIRE_FLAME);
    o[0] = f->rxInt * (BTU / (FOOT_TO_M * FOOT_TO_M) / 60.0);
    o[1] = f->spread0 * (FOOT_TO_M / 60.0);
    o[2] = f->hpua * (BTU / (FOOT_TO_M * FOOT_TO_M));
    o[3] = f->phiEw;
    o[4] = f->spreadMax * (FOOT_TO_M / 60.0);
    o[5] = f->azimuthMax * M_PI / 180.0;
    o[6] = f->eccentricity;
    o[7] = f->taur * 60.0;
    o[8] = f->byrams * (BTU / FOOT_TO_M);
    o[9] = f->flame * FOOT_TO_M;
    burning++;
  }
  Fire_FuelCatalogDestroy(cat);
  return burning;
}

int64_t ref_burn_c(int64_t n, const uint8_t *fuel, const float *d1, const float *d10,
                   const float *d100, const float *herb, const float *wood,
                   const float *wind_speed, const float *wind_azimuth, const float *slope,
                   const float *aspect, double *out) {
  return burn(0, n, fuel, d1, d10, d100, herb, wood, wind_speed, wind_azimuth, slope, aspect, out);
}

int64_t ref_burn_c_rust_catalog(int64_t n, const uint8_t *fuel, const float *d1, const float *d10,
                                const float *d100, const float *herb, const float *wood,
                                const float *wind_speed, const float *wind_azimuth,
                                const float *slope, const float *aspect, double *out) {
  return burn(1, n, fuel, d1, d10, d100, herb, wood, wind_speed, wind_azimuth, slope, aspect, out);
}
