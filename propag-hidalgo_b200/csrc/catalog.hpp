// Fuel-model table of the fire-behaviour kernel.
//
// The reference evaluates the constants of each NFFL fuel model at compile
// time (crates/firelib/src/firelib.rs:554-979 over the catalog in
// crates/firelib/src/lib.rs:126-268).  Here they are evaluated once on the
// host in double precision and folded into per-moisture-class linear
// coefficients, then rounded to float for the device table.
#pragma once

#include <cstdint>

namespace propag {

constexpr int kMaxFuels = 20;      // MAX_FUELS, firelib.rs:31
constexpr int kCatalogFuels = 14;  // NoFuel + NFFL01..13

// Moisture inputs in the order the kernel reads them.
enum MoistureClass { kD1 = 0, kD10 = 1, kD100 = 2, kHerb = 3, kWood = 4, kMoistureClasses = 5 };

// Device table entry (float).  Per cell, with m = (d1, d10, d100, herb, wood):
//   rbqig      = R0 + sum R[k] m[k]          (fuel_bed_bulk_dens folded in)
//   dead_moist = sum A[k] m[k]
//   live_moist = sum B[k] m[k]
//   live_mext  = LM0 - sum LM[k] m[k]        (before max(., mext))
struct FuelConst {
  float has_fire;  // 1 when the model has particles (Catalog::get)
  float has_live;
  float R0;
  float R[kMoistureClasses];
  float A[kMoistureClasses];
  float B[kMoistureClasses];
  float LM0;
  float LM[kMoistureClasses];
  float mext;
  float rx_alive, rx_dead;  // life_rx_factor
  float flux_ratio, slope_k, wind_b, wind_b_inv, wind_e, wind_k;
  float residence_time;  // min
  // low parts of the double-float pairs used where the kernel subtracts
  // nearly equal quantities (moisture vs moisture of extinction)
  float A_lo[kMoistureClasses];
  float B_lo[kMoistureClasses];
  float LM_lo[kMoistureClasses];
  float LM0_lo, mext_lo;
  float pad[13];
};
static_assert(sizeof(FuelConst) == 64 * 4, "FuelConst layout");

// Double-precision constants of one fuel model (imperial internal units, as
// the reference keeps them).
struct FuelModel64 {
  int n_particles = 0, n_dead = 0;
  bool has_live = false;
  double sigma = 0, beta = 0, flux_ratio = 0, slope_k = 0;
  double wind_b = 0, wind_e = 0, wind_k = 0;
  double rx_alive = 0, rx_dead = 0, residence_time = 0, bulk_density = 0;
  double live_ext_factor = 0, fine_dead_factor = 0, mext = 0;
  double live_area_weight = 0, dead_area_weight = 0;
  // folded coefficients
  double R0 = 0, R[kMoistureClasses] = {}, A[kMoistureClasses] = {}, B[kMoistureClasses] = {};
  double LM0 = 0, LM[kMoistureClasses] = {};
};

// Builds the catalog (indices 0..19; 14..19 and 0 have no fire).
void build_catalog64(FuelModel64 out[kMaxFuels]);
void build_catalog_table(FuelConst out[kMaxFuels]);

}  // namespace propag
