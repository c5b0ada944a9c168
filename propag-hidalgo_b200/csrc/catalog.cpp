// Host construction of the NFFL fuel catalog, in double precision.
//
// Formulas (paths relative to the reference project):
//   ParticleDef::standard / size_class / surface_area / area_weight /
//   size_class_weight / sigma_factor         crates/firelib/src/firelib.rs:554-653
//   FuelDef::* (sigma, beta, ratio, flux_ratio, gamma, life_*, live_ext_factor,
//   bulk_density, residence_time, slope_k, wind_bke)    firelib.rs:716-868
//   Fuel::standard / Fuel::make (dead particles first) firelib.rs:870-979
//   Particle::moisture (size class -> moisture input)  firelib.rs:699-713
//   rx_int_rbqig / eta_m terms that are linear in the moisture, folded here
//                                                      firelib.rs:1031-1076
//   NFFL catalog                                        crates/firelib/src/lib.rs:126-268
#include "catalog.hpp"

#include <cmath>
#include <vector>

namespace propag {
namespace {

enum class Kind { Dead, Herb, Wood };

struct ParticleSpec {
  Kind kind;
  double load;  // lb/ft^2
  double savr;  // 1/ft
};

struct ModelSpec {
  double depth;  // ft
  double mext;
  std::vector<ParticleSpec> particles;
};

// NFFL standard models 0..13 (crates/firelib/src/lib.rs:126-268).
const ModelSpec &nffl(int code) {
  static const std::vector<ModelSpec> table = {
      {0.1, 0.01, {}},
      {1.0, 0.12, {{Kind::Dead, 0.0340, 3500.0}}},
      {1.0, 0.15, {{Kind::Dead, 0.0920, 3000.0}, {Kind::Dead, 0.0460, 109.0}, {Kind::Dead, 0.0230, 30.0}, {Kind::Herb, 0.0230, 1500.0}}},
      {2.5, 0.25, {{Kind::Dead, 0.1380, 1500.0}}},
      {6.0, 0.20, {{Kind::Dead, 0.2300, 2000.0}, {Kind::Dead, 0.1840, 109.0}, {Kind::Dead, 0.0920, 30.0}, {Kind::Wood, 0.2300, 1500.0}}},
      {2.0, 0.20, {{Kind::Dead, 0.0460, 2000.0}, {Kind::Dead, 0.0230, 109.0}, {Kind::Wood, 0.0920, 1500.0}}},
      {2.5, 0.25, {{Kind::Dead, 0.0690, 1750.0}, {Kind::Dead, 0.1150, 109.0}, {Kind::Dead, 0.0920, 30.0}}},
      {2.5, 0.40, {{Kind::Dead, 0.0520, 1750.0}, {Kind::Dead, 0.0860, 109.0}, {Kind::Dead, 0.0690, 30.0}, {Kind::Wood, 0.0170, 1550.0}}},
      {0.2, 0.30, {{Kind::Dead, 0.0690, 2000.0}, {Kind::Dead, 0.0460, 109.0}, {Kind::Dead, 0.1150, 30.0}}},
      {0.2, 0.25, {{Kind::Dead, 0.1340, 2500.0}, {Kind::Dead, 0.0190, 109.0}, {Kind::Dead, 0.0070, 30.0}}},
      {1.0, 0.25, {{Kind::Dead, 0.1380, 2000.0}, {Kind::Dead, 0.0920, 109.0}, {Kind::Dead, 0.2300, 30.0}, {Kind::Wood, 0.0920, 1500.0}}},
      {1.0, 0.15, {{Kind::Dead, 0.0690, 1500.0}, {Kind::Dead, 0.2070, 109.0}, {Kind::Dead, 0.2530, 30.0}}},
      {2.3, 0.20, {{Kind::Dead, 0.1840, 1500.0}, {Kind::Dead, 0.6440, 109.0}, {Kind::Dead, 0.7590, 30.0}}},
      {3.0, 0.25, {{Kind::Dead, 0.3220, 1500.0}, {Kind::Dead, 0.0580, 109.0}, {Kind::Dead, 1.2880, 30.0}}},
  };
  return table[code];
}

constexpr double kSmidgen = 1e-6;
constexpr double kDensity = 32.0;      // lb/ft^3   (ParticleDef::standard)
constexpr double kHeat = 8000.0;       // BTU/lb
constexpr double kSiTotal = 0.0555;
constexpr double kSiEffective = 0.01;

double safe_div(double a, double b) { return b > kSmidgen ? a / b : 0.0; }

int size_class(double savr) {
  if (savr > 1200.0) return 0;
  if (savr > 192.0) return 1;
  if (savr > 96.0) return 2;
  if (savr > 48.0) return 3;
  if (savr > 16.0) return 4;
  return 5;
}

struct Particle {
  bool live;
  Kind kind;
  double load, savr, area, aw, sw, sigma_factor;
  int sc;
  int moisture;  // MoistureClass read by this particle
};

}  // namespace

void build_catalog64(FuelModel64 out[kMaxFuels]) {
  for (int code = 0; code < kMaxFuels; ++code) {
    FuelModel64 &f = out[code];
    f = FuelModel64{};
    if (code >= kCatalogFuels) continue;
    const ModelSpec &spec = nffl(code);
    if (spec.particles.empty()) continue;

    // per-particle derived values, in definition order
    std::vector<Particle> defs;
    for (const ParticleSpec &ps : spec.particles) {
      Particle p{};
      p.kind = ps.kind;
      p.live = ps.kind != Kind::Dead;
      p.load = ps.load;
      p.savr = ps.savr;
      p.area = safe_div(ps.load * ps.savr, kDensity);
      p.sc = size_class(ps.savr);
      p.sigma_factor = std::exp(safe_div(-138.0, ps.savr));
      defs.push_back(p);
    }
    for (Particle &p : defs) {
      double total = 0;
      for (const Particle &q : defs)
        if (q.live == p.live) total += q.area;
      p.aw = safe_div(p.area, total);
    }
    for (Particle &p : defs) {
      double sw = 0;
      for (const Particle &q : defs)
        if (q.live == p.live && q.sc == p.sc) sw += q.aw;
      p.sw = sw;
      switch (p.kind) {
        case Kind::Herb: p.moisture = kHerb; break;
        case Kind::Wood: p.moisture = kWood; break;
        default: p.moisture = p.sc <= 1 ? kD1 : (p.sc <= 3 ? kD10 : kD100);
      }
    }
    // dead first, then live (Fuel::standard)
    std::vector<Particle> ps;
    for (const Particle &p : defs)
      if (!p.live) ps.push_back(p);
    f.n_dead = (int)ps.size();
    for (const Particle &p : defs)
      if (p.live) ps.push_back(p);
    f.n_particles = (int)ps.size();
    f.has_live = f.n_particles > f.n_dead;

    const double depth = spec.depth;
    double total_area = 0;
    for (const Particle &p : ps) total_area += p.area;
    double law[2] = {}, lsavr[2] = {}, lheat[2] = {}, lseff[2] = {}, lload[2] = {}, lfine[2] = {};
    double beta_sum = 0, bulk = 0;
    for (const Particle &p : ps) {
      const int l = p.live ? 1 : 0;
      law[l] += p.area / total_area;
      lsavr[l] += p.aw * p.savr;
      lheat[l] += p.aw * kHeat;
      lseff[l] += p.aw * kSiEffective;
      lload[l] += p.sw * p.load * (1.0 - kSiTotal);
      lfine[l] += p.live ? p.load * std::exp(-500.0 / p.savr) : p.load * p.sigma_factor;
      beta_sum += p.load / kDensity;
      bulk += p.load / depth;
    }
    const double sigma = law[1] * lsavr[1] + law[0] * lsavr[0];
    const double beta = beta_sum / depth;
    const double ratio = beta / (3.348 / std::pow(sigma, 0.8189));
    const double sigma15 = std::pow(sigma, 1.5);
    const double gamma_max = sigma15 / (495.0 + 0.0594 * sigma15);
    const double aa = 133.0 / std::pow(sigma, 0.7913);
    const double gamma = gamma_max * std::pow(ratio, aa) * std::exp(aa * (1.0 - ratio));
    double eta_s[2];
    for (int l = 0; l < 2; ++l) {
      if (lseff[l] > kSmidgen) {
        const double e = 0.174 / std::pow(lseff[l], 0.19);
        eta_s[l] = e < 1.0 ? e : 1.0;
      } else {
        eta_s[l] = 1.0;
      }
    }
    f.sigma = sigma;
    f.beta = beta;
    f.mext = spec.mext;
    f.rx_alive = lload[1] * lheat[1] * eta_s[1] * gamma;
    f.rx_dead = lload[0] * lheat[0] * eta_s[0] * gamma;
    f.flux_ratio = std::exp((0.792 + 0.681 * std::sqrt(sigma)) * (beta + 0.1)) / (192.0 + 0.2595 * sigma);
    f.slope_k = 5.275 * std::pow(beta, -0.3);
    f.wind_b = 0.02526 * std::pow(sigma, 0.54);
    const double c = 7.47 * std::exp(-0.133 * std::pow(sigma, 0.55));
    const double e = 0.715 * std::exp(-0.000359 * sigma);
    f.wind_k = c * std::pow(ratio, -e);
    f.wind_e = std::pow(ratio, e) / c;
    f.residence_time = 384.0 / sigma;
    f.bulk_density = bulk;
    f.live_ext_factor = 2.9 * safe_div(lfine[0], lfine[1]);
    f.fine_dead_factor = 1.0 / lfine[0];
    f.live_area_weight = law[1];
    f.dead_area_weight = law[0];

    // Fold the moisture-linear sums of rx_int_rbqig and eta_m.
    f.R0 = 0;
    for (const Particle &p : ps) {
      const double lw = p.live ? law[1] : law[0];
      const double w = bulk * p.aw * lw * p.sigma_factor;
      f.R0 += 250.0 * w;
      f.R[p.moisture] += 1116.0 * w;
      if (p.live) {
        f.B[p.moisture] += p.aw;
      } else {
        f.A[p.moisture] += p.aw;
        // fdmois = wfmd * fine_dead_factor, wfmd = sum(m * sigma_factor * load)
        f.LM[p.moisture] += f.live_ext_factor * f.fine_dead_factor / f.mext * p.sigma_factor * p.load;
      }
    }
    f.LM0 = f.live_ext_factor - 0.226;
  }
}

void build_catalog_table(FuelConst out[kMaxFuels]) {
  FuelModel64 m[kMaxFuels];
  build_catalog64(m);
  for (int i = 0; i < kMaxFuels; ++i) {
    FuelConst &c = out[i];
    c = FuelConst{};
    const FuelModel64 &f = m[i];
    if (f.n_particles == 0) continue;
    c.has_fire = 1.0f;
    c.has_live = f.has_live ? 1.0f : 0.0f;
    c.R0 = (float)f.R0;
    auto split = [](double v, float &hi, float &lo) {
      hi = (float)v;
      lo = (float)(v - (double)hi);
    };
    for (int k = 0; k < kMoistureClasses; ++k) {
      c.R[k] = (float)f.R[k];
      split(f.A[k], c.A[k], c.A_lo[k]);
      split(f.B[k], c.B[k], c.B_lo[k]);
      split(f.LM[k], c.LM[k], c.LM_lo[k]);
    }
    split(f.LM0, c.LM0, c.LM0_lo);
    split(f.mext, c.mext, c.mext_lo);
    c.rx_alive = (float)f.rx_alive;
    c.rx_dead = (float)f.rx_dead;
    c.flux_ratio = (float)f.flux_ratio;
    c.slope_k = (float)f.slope_k;
    c.wind_b = (float)f.wind_b;
    c.wind_b_inv = (float)(1.0 / f.wind_b);
    c.wind_e = (float)f.wind_e;
    c.wind_k = (float)f.wind_k;
    c.residence_time = (float)f.residence_time;
  }
}

}  // namespace propag
