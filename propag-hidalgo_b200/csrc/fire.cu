// Per-cell fire behaviour (Rothermel / BEHAVE) as an elementwise FP32 pass
// over structure-of-arrays rasters.
//
// Reference (paths relative to the reference project):
//   cuda_standard_simple_burn / cuda_standard_burn   crates/firelib/src/cuda.rs:7-95
//   Fuel::burn / burn_simple                         crates/firelib/src/firelib.rs:996-1030
//   rx_int_rbqig, eta_m                              firelib.rs:1031-1076
//   calculate_wind_dependent_vars, situations        firelib.rs:1078-1167
//   eccentricity, phi_slope, phi_wind                firelib.rs:1171-1188
//   Terrain::upslope                                 firelib.rs:400-409
//   Byram's intensity, flame length                  firelib.rs:424-441
//
// Layout and mapping: one cell per thread, grid-stride, so that every load
// and store of a warp is one coalesced run (4 bytes per lane, 1 for the fuel
// codes); the grid holds as many CTAs as are resident at once (one wave),
// and 32-bit indices serve every grid below 2^32 cells.  Four cells per thread
// with 128-bit loads measured slower (0.298 against 0.277 ms at 4096^2): the
// pass is bound by instruction issue, and four inlined copies of the cell
// code overflow the instruction cache.  The fuel table sits in shared memory
// with a row stride of 65 words (20 models), so that the lanes of a warp that
// read the same field of different models hit different banks.  Double-float
// moisture sums measured faster here than FP64 ones (0.33-0.35 ms against
// 0.35-0.36 ms at 4096^2).  Compiled without automatic multiply-add
// contraction, so that the 3-field and 10-field instantiations round alike
// (contraction measured no faster).
//
// FP32 formulation.  The arithmetic is the reference's, rearranged where the
// float evaluation of the literal formula loses accuracy against double:
//   * the moisture sums are pre-folded per moisture class; the dead and live
//     sums and the live extinction moisture are double-float (error-free
//     products and sums), because they are subtracted from the moisture of
//     extinction, where float cancellation would dominate the error;
//   * eta_m = 1 - 2.59 rt + 5.11 rt^2 - 3.52 rt^3 is evaluated in
//     u = 1 - rt = (mext - moist) / mext as u (2.93 - 5.45 u + 3.52 u^2),
//     the same cubic expanded at rt = 1 where it vanishes;
//   * the cross-slope direction uses atan2(|y|, |x|) instead of
//     asin(|y| / hypot(x, y)) (same angle, no loss near 90 degrees);
//   * the cross-slope vector is summed in phi units (the reference's rate
//     vectors divided by speed0 > 0), so phi_ew2 is its length instead of
//     (speed0 + rv) / speed0 - 1;
//   * eccentricity sqrt(lw^2 - 1) / lw with lw = 1 + a is sqrt(a (2 + a)) / (1 + a);
//   * pi and 2 pi are added as float pairs (hi + lo).
#include <cuda_runtime.h>

#include <cstdint>

#include "catalog.hpp"
#include "dmoist_device.cuh"

namespace propag {

constexpr float kSmidgenF = 1e-6f;  // SMIDGEN, crates/firelib/src/f32.rs:5
constexpr float kPiHi = 3.14159274101257324f, kPiLo = -8.74227766e-8f;
constexpr float kTwoPiHi = 6.28318548202514648f, kTwoPiLo = -1.74845553e-7f;
// unit conversions (crates/firelib/src/units.rs:28-30: foot 0.3048 m,
// BTU 1054.35 J)
constexpr float kFpmToMps = 0.00508f;             // 0.3048 / 60
constexpr float kMpsToFpm = 196.850393700787402f; // 60 / 0.3048
constexpr float kRxToSI = 189.146876418865f;      // BTU/ft^2/min -> W/m^2
constexpr float kHpuaToSI = 11348.8125851319f;    // BTU/ft^2 -> J/m^2
constexpr float kByramsToSI = 3459.15354330709f;  // BTU/ft/s -> W/m
constexpr float kFootToM = 0.3048f;

__constant__ FuelConst c_catalog[kMaxFuels];

struct FireOut {
  float rx_int, speed0, hpua, phi_eff_wind, speed_max, azimuth_max, eccentricity,
      residence_time, byrams, flame;
};

// Double-float value hi + lo (|lo| <= ulp(hi) / 2).
struct DF {
  float hi, lo;
};

// Error-free sum of two floats (Knuth's two-sum).
__device__ __forceinline__ DF two_sum(float a, float b) {
  const float s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  const float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  return DF{s, e};
}

// sum_{k in [K0, K1)} (chi[k] + clo[k]) * m[k] as a double-float: exact
// products (fma) and sums (two-sum), so that moisture sums keep ~2^-44
// relative accuracy.  The catalog's dead-moisture and live-extinction
// coefficients are zero for the live classes (3, 4) and the live-moisture
// coefficients for the dead classes (0-2); zero terms leave hi and lo
// unchanged, so summing only [K0, K1) gives the same bits.
template <int K0, int K1>
__device__ __forceinline__ DF dot_df(const float *chi, const float *clo, const float m[5]) {
  float hi = 0.0f, lo = 0.0f;
#pragma unroll
  for (int k = K0; k < K1; ++k) {
    const float p = __fmul_rn(chi[k], m[k]);
    const float pe = __fmaf_rn(chi[k], m[k], -p);
    const DF s = two_sum(hi, p);
    hi = s.hi;
    lo = __fadd_rn(lo, __fadd_rn(s.lo, __fmaf_rn(clo[k], m[k], pe)));
  }
  return two_sum(hi, lo);
}

__device__ __forceinline__ DF df_sub(DF a, DF b) {
  const DF s = two_sum(a.hi, -b.hi);
  return two_sum(s.hi, __fadd_rn(s.lo, __fsub_rn(a.lo, b.lo)));
}

// eta_m (firelib.rs:1060-1076) with rt = moist / mext, as
// u (2.93 - 5.45 u + 3.52 u^2), u = 1 - rt = (mext - moist) / mext.
__device__ __forceinline__ float eta_m(DF moist, DF mext) {
  const DF d = df_sub(mext, moist);
  if (!(d.hi > 0.0f)) return 0.0f;  // life_moist >= life_mext
  const float u = __fdividef(d.hi + d.lo, mext.hi + mext.lo);  // 2 ulp; operands in [2^-126, 2^126]
  return u * fmaf(u, fmaf(u, 3.52f, -5.45f), 2.93f);
}

// x^y for x >= 0 (0^y = 0 for y > 0) as 2^(y log2 x): about 1e-6 relative
// (|y log2 x| < 30 here), well inside the fields' 1e-5 budget, at a fraction
// of powf's cost (powf keeps extended precision for < 1 ulp).
__device__ __forceinline__ float pow_pos(float x, float y) { return exp2f(y * log2f(x)); }

__device__ __forceinline__ float dot5(const float *c, const float m[5]) {
  float s = c[0] * m[0];
  s = fmaf(c[1], m[1], s);
  s = fmaf(c[2], m[2], s);
  s = fmaf(c[3], m[3], s);
  return fmaf(c[4], m[4], s);
}

template <bool kFull>
__device__ __forceinline__ void burn_cell(const FuelConst &F, const float m[5], float ws,
                                          float waz, float slope, float aspect, FireOut &o) {
  // rx_int_rbqig
  const DF dead = dot_df<0, 3>(F.A, F.A_lo, m);
  const DF live = dot_df<3, 5>(F.B, F.B_lo, m);
  const float rbqig = F.R0 + dot5(F.R, m);
  const DF mext{F.mext, F.mext_lo};
  const float eta_dead = eta_m(dead, mext);
  DF live_mext{0.0f, 0.0f};
  if (F.has_live != 0.0f) {
    live_mext = df_sub(DF{F.LM0, F.LM0_lo}, dot_df<0, 3>(F.LM, F.LM_lo, m));
    if (!(df_sub(live_mext, mext).hi > 0.0f)) live_mext = mext;  // max(live_mext, mext)
  }
  const float eta_live = eta_m(live, live_mext);
  const float rx = fmaf(F.rx_alive, eta_live, F.rx_dead * eta_dead);
  const float speed0 = __fdividef(rx * F.flux_ratio, rbqig);

  // calculate_wind_dependent_vars
  const float phi_slope = F.slope_k * slope * slope;
  const float ws_fpm = ws * kMpsToFpm;
  const float phi_wind = F.wind_k * pow_pos(ws_fpm, F.wind_b);
  const float phi_ew = phi_slope + phi_wind;
  const float upslope = aspect >= kPiHi ? (aspect - kPiHi) - kPiLo : (aspect + kPiHi) + kPiLo;
  const float max_wind = 0.9f * rx;

  float pew = phi_ew, ew = 0.0f, smax = 0.0f, az = 0.0f;
  bool limit = true;
  if (speed0 < kSmidgenF) {  // NoSpread
    limit = false;
  } else if (phi_ew < kSmidgenF) {  // NoSlopeNoWind
    smax = speed0;
    limit = false;
  } else if (slope < kSmidgenF) {  // WindNoSlope
    ew = ws_fpm;
    smax = speed0 * (1.0f + phi_ew);
    az = waz;
  } else if (ws < kSmidgenF || fabsf(upslope - waz) < kSmidgenF) {  // SlopeNoWind, UpSlope
    ew = pow_pos(phi_ew * F.wind_e, F.wind_b_inv);
    smax = speed0 * (1.0f + phi_ew);
    az = upslope;
  } else {  // CrossSlope
    // The reference sums the rate vectors speed0 * phi; the common factor
    // speed0 > 0 is kept out: (x, y) below are those vectors / speed0, the
    // direction and quadrant are unchanged and phi_ew2 = |(x, y)|.
    const float split = upslope <= waz ? waz - upslope : ((kTwoPiHi - upslope) + waz) + kTwoPiLo;
    // the same angle in [-pi, pi], where the fast sine and cosine are
    // accurate to 2^-21.4 absolute (the vector components are then good to
    // ~4e-7 of phi_wind, inside the fields' 1e-5 budget)
    const float red = split > kPiHi ? (split - kTwoPiHi) - kTwoPiLo : split;
    float sn, cs;
    __sincosf(red, &sn, &cs);
    const float x = fmaf(phi_wind, cs, phi_slope);
    const float y = phi_wind * sn;
    pew = sqrtf(fmaf(x, x, y * y));  // phi values far below 1e18: no overflow to guard
    smax = speed0 * (1.0f + pew);
    ew = pow_pos(pew * F.wind_e, F.wind_b_inv);
    const float al = atan2f(fabsf(y), fabsf(x));
    float split2;
    if (x >= 0.0f && y >= 0.0f) split2 = al;
    else if (x >= 0.0f) split2 = (kTwoPiHi - al) + kTwoPiLo;
    else if (y >= 0.0f) split2 = (kPiHi - al) + kPiLo;
    else split2 = (kPiHi + al) + kPiLo;
    az = upslope + split2;
    if (az > kTwoPiHi) az = (az - kTwoPiHi) - kTwoPiLo;
  }
  if (limit && ew > max_wind) {  // check_wind_limit
    pew = F.wind_k * pow_pos(max_wind, F.wind_b);
    ew = max_wind;
    smax = speed0 * (1.0f + pew);
  }
  const float a = 0.002840909f * ew;
  o.speed_max = smax * kFpmToMps;
  o.azimuth_max = az;
  o.eccentricity = __fdividef(sqrtf(a * (2.0f + a)), 1.0f + a);
  if (kFull) {  // the remaining FireCuda fields, Byram and flame
    o.rx_int = rx * kRxToSI;
    o.speed0 = speed0 * kFpmToMps;
    o.hpua = rx * F.residence_time * kHpuaToSI;
    o.phi_eff_wind = pew;
    o.residence_time = F.residence_time * 60.0f;
    const float byrams = F.residence_time * smax * rx * (1.0f / 60.0f);
    o.byrams = byrams * kByramsToSI;
    o.flame = byrams > kSmidgenF ? 0.45f * pow_pos(byrams, 0.46f) * kFootToM : 0.0f;
  }
}

struct Inputs {
  const uint8_t *fuel;
  const float *m[5];
  const float *ws, *waz, *slope, *aspect;
};
struct Outputs {
  float *f[10];  // PropagFireFields order
};

// kFull: every field whose output is given; else the three the propagation
// needs (the 3-field entry point passes only those).
template <bool kFull, typename Index>
__device__ __forceinline__ void store_cell(const Outputs &out, Index i, const FireOut &o) {
  const float v[10] = {o.rx_int, o.speed0, o.hpua, o.phi_eff_wind, o.speed_max,
                       o.azimuth_max, o.eccentricity, o.residence_time, o.byrams, o.flame};
#pragma unroll
  for (int k = 0; k < 10; ++k)
    if ((kFull || (k >= 4 && k <= 6)) && out.f[k]) out.f[k][i] = v[k];
}

// Shared-memory copy of the fuel table, rows kCatStride words apart (odd:
// the same field of different models lies in different banks).
constexpr int kCatStride = 65;
static_assert(sizeof(FuelConst) / 4 <= kCatStride, "a FuelConst fits a table row");

__device__ __forceinline__ void load_catalog(float *cat) {
  const float *src = reinterpret_cast<const float *>(c_catalog);
  constexpr int kWords = (int)(sizeof(FuelConst) / 4);
  for (int t = threadIdx.x; t < kMaxFuels * kWords; t += blockDim.x)
    cat[(t / kWords) * kCatStride + t % kWords] = src[t];
  __syncthreads();
}

__device__ __forceinline__ const FuelConst &fuel_row(const float *cat, uint32_t code) {
  return *reinterpret_cast<const FuelConst *>(cat + code * kCatStride);
}

template <bool kFull, typename Index>
__device__ __forceinline__ void one_cell(const float *cat, const Inputs &in, const Outputs &out,
                                         Index i) {
  const uint8_t code = __ldg(in.fuel + i);
  FireOut o{};
  if (code < kMaxFuels && fuel_row(cat, code).has_fire != 0.0f) {
    const float m[5] = {__ldg(in.m[0] + i), __ldg(in.m[1] + i), __ldg(in.m[2] + i), __ldg(in.m[3] + i),
                        __ldg(in.m[4] + i)};
    burn_cell<kFull>(fuel_row(cat, code), m, __ldg(in.ws + i), __ldg(in.waz + i),
                     __ldg(in.slope + i), __ldg(in.aspect + i), o);
  }
  store_cell<kFull>(out, i, o);
}

// One cell per thread, grid-stride, cells [first, n): every load and store is
// coalesced (4 or 1 consecutive bytes per lane).  kFull: all ten fields; else
// the three the propagation needs (the shared fields are the same
// operations, so both give the same values for them).
// Index: uint32_t when n + the grid's threads fit in 32 bits (cheaper
// address arithmetic), else uint64_t.
template <bool kFull, typename Index>
__global__ void __launch_bounds__(256) fire_kernel(Inputs in, Outputs out, Index first, Index n) {
  __shared__ float cat[kMaxFuels * kCatStride];
  load_catalog(cat);
  const Index stride = (Index)gridDim.x * blockDim.x;
  for (Index i = first + (Index)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    one_cell<kFull>(cat, in, out, i);
}

// Dead fuel moisture and fire behaviour in one pass (no d1/d10/d100 rasters
// in between): per cell the dmoist model at `hour` from the cell's weather
// (dmoist_cell, percent values scaled to fractions as the moisture pass's
// scale 0.01 does), then the three fields the propagation needs.  The same
// operations as the moisture pass followed by fire_kernel<false>, so the
// same bits.  Cells without fire skip the moisture model (their outputs are
// 0 either way).
template <typename Index>
__global__ void __launch_bounds__(256) fire_weather_kernel(DmoistIn win, int hour, int month,
                                                           Inputs in, Outputs out, Index n) {
  __shared__ float cat[kMaxFuels * kCatStride];
  __shared__ DmoistTables T;
  load_dmoist_tables(T);
  load_catalog(cat);
  const Index stride = (Index)gridDim.x * blockDim.x;
  for (Index i = (Index)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint8_t code = __ldg(in.fuel + i);
    FireOut o{};
    if (code < kMaxFuels && fuel_row(cat, code).has_fire != 0.0f) {
      const float slope = __ldg(in.slope + i), aspect = __ldg(in.aspect + i);
      float m1, m10, m100;
      dmoist_cell(T, win, (uint64_t)n, (uint64_t)i, hour, month, code, slope, aspect, m1, m10, m100);
      const float m[5] = {m1 * 0.01f, m10 * 0.01f, m100 * 0.01f, __ldg(in.m[3] + i), __ldg(in.m[4] + i)};
      burn_cell<false>(fuel_row(cat, code), m, __ldg(in.ws + i), __ldg(in.waz + i), slope, aspect, o);
    }
    store_cell<false>(out, i, o);
  }
}

// CTAs of a fire kernel resident per SM (registers limit it).
template <typename K>
static int ctas_per_sm(K kernel, int threads) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, 0) != cudaSuccess || n < 1)
    n = 1;
  return n;
}

// one wave: as many CTAs as are resident at once, each striding over an
// equal share (a second, partial wave would leave SMs idle at the end)
static unsigned one_wave(uint64_t items, int threads, int sm_count, int per_sm) {
  uint64_t blocks = (items + threads - 1) / threads;
  const uint64_t cap = (uint64_t)sm_count * (uint64_t)per_sm;
  if (blocks > cap) blocks = cap;
  return blocks ? (unsigned)blocks : 1u;
}

template <bool kFull, typename Index>
static cudaError_t launch_fire_t(const Inputs &in, const Outputs &out, uint64_t n, int sm_count,
                                 int threads, cudaStream_t stream) {
  auto k1 = fire_kernel<kFull, Index>;
  k1<<<one_wave(n, threads, sm_count, ctas_per_sm(k1, threads)), threads, 0, stream>>>(in, out, (Index)0,
                                                                                    (Index)n);
  return cudaGetLastError();
}

// ---- host-side launchers (called from api.cpp) ------------------------------
cudaError_t upload_catalog() {
  FuelConst table[kMaxFuels];
  build_catalog_table(table);
  // the kernel's moisture sums skip the classes whose coefficients are zero
  for (int f = 0; f < kMaxFuels; ++f) {
    for (int k = kHerb; k <= kWood; ++k)
      if (table[f].A[k] != 0.0f || table[f].A_lo[k] != 0.0f || table[f].LM[k] != 0.0f ||
          table[f].LM_lo[k] != 0.0f)
        return cudaErrorInvalidValue;
    for (int k = kD1; k <= kD100; ++k)
      if (table[f].B[k] != 0.0f || table[f].B_lo[k] != 0.0f) return cudaErrorInvalidValue;
  }
  return cudaMemcpyToSymbol(c_catalog, table, sizeof(table));
}

cudaError_t launch_fire(bool full, uint64_t n, const uint8_t *fuel, const float *const m[5],
                        const float *ws, const float *waz, const float *slope,
                        const float *aspect, float *const outs[10], int sm_count,
                        cudaStream_t stream) {
  Inputs in{fuel, {m[0], m[1], m[2], m[3], m[4]}, ws, waz, slope, aspect};
  Outputs out{};
  for (int k = 0; k < 10; ++k) out.f[k] = outs[k];
  if (n == 0) return cudaSuccess;
  const int threads = 256;
  // 32-bit indices while the last index plus one grid stride stays below 2^32
  const bool narrow = n + (uint64_t)sm_count * 8 * threads < (1ull << 32);
  if (full)
    return narrow ? launch_fire_t<true, uint32_t>(in, out, n, sm_count, threads, stream)
                  : launch_fire_t<true, uint64_t>(in, out, n, sm_count, threads, stream);
  return narrow ? launch_fire_t<false, uint32_t>(in, out, n, sm_count, threads, stream)
                : launch_fire_t<false, uint64_t>(in, out, n, sm_count, threads, stream);
}

cudaError_t launch_fire_weather(uint64_t n, int hour, int month, const float *t, const float *rh,
                                const float *cc, const float *pp, const uint8_t *fuel,
                                const float *herb, const float *wood, const float *ws,
                                const float *waz, const float *slope, const float *aspect,
                                float *speed_max, float *azimuth_max, float *eccentricity,
                                int sm_count, cudaStream_t stream) {
  if (n == 0) return cudaSuccess;
  DmoistIn win{t, rh, cc, pp, slope, aspect, fuel};
  Inputs in{fuel, {nullptr, nullptr, nullptr, herb, wood}, ws, waz, slope, aspect};
  Outputs out{};
  out.f[4] = speed_max;
  out.f[5] = azimuth_max;
  out.f[6] = eccentricity;
  const int threads = 256;
  const bool narrow = n + (uint64_t)sm_count * 8 * threads < (1ull << 32);
  if (narrow) {
    auto k = fire_weather_kernel<uint32_t>;
    k<<<one_wave(n, threads, sm_count, ctas_per_sm(k, threads)), threads, 0, stream>>>(
        win, hour, month, in, out, (uint32_t)n);
  } else {
    auto k = fire_weather_kernel<uint64_t>;
    k<<<one_wave(n, threads, sm_count, ctas_per_sm(k, threads)), threads, 0, stream>>>(
        win, hour, month, in, out, (uint64_t)n);
  }
  return cudaGetLastError();
}

}  // namespace propag
