// rain_cell.cuh — per-cell warm-rain microphysics shared by the plain column kernel,
// the surrogate's training-sample recorder and the surrogate's per-cell fallback.
#pragma once

#include "common.cuh"

namespace gwmb {

__device__ __forceinline__ float sat_vapor_pressure(float tk) {  // moist_thermo.hpp:23-29
  const float tc = tk - 273.15f;
  const float es_hpa = 6.112f * expf((17.67f * tc) / fmaxf(tc + 243.5f, 1.0e-6f));
  return es_hpa * 100.0f;
}
__device__ __forceinline__ float qsat(float tk, float p) {  // moist_thermo.hpp:31-36
  const float eps = kRd / kRv;
  const float es = sat_vapor_pressure(tk);
  const float denom = fmaxf(p - (1.0f - eps) * es, 1000.0f);
  return fminf(fmaxf(eps * es / denom, 0.0f), 0.05f);
}

struct MicroParams {
  float dt, relax, thr, rate, evap;
  int latent;
};

// State of one cell before/after the microphysics: mixing ratios, theta, the
// latent-heating factor L_v / (c_p pi) of the initial state, temperature, pressure.
struct MicroCell {
  float rho;              // max(rho_d, 1e-6)
  float th, qv, qc, qr;
  float lh, temp, p;
};

// Diagnostics of the initial state: warm_rain.cu:42-62 (dry_temperature_from_conserved,
// moist_thermo.hpp:55-62; mixing ratios clipped at zero).
__device__ __forceinline__ MicroCell micro_state(float rho_d, float rt, float rqv, float rqc, float rqr) {
  MicroCell c;
  c.rho = fmaxf(rho_d, 1.0e-6f);
  c.th = rt / c.rho;
  c.p = eos_pressure(c.rho, rt);
  {
    const float thc = theta_of(c.rho, rt);
    const float pc = eos_pressure(c.rho, rt);
    c.temp = thc * powf(fmaxf(pc / kP0, 1.0e-6f), kKappa);
  }
  const float exner = fmaxf(c.temp / fmaxf(c.th, 1.0e-6f), 1.0e-6f);
  c.qv = fmaxf(rqv / c.rho, 0.0f);
  c.qc = fmaxf(rqc / c.rho, 0.0f);
  c.qr = fmaxf(rqr / c.rho, 0.0f);
  c.lh = kLv / (dry_cp() * fmaxf(exner, 1.0e-6f));
  return c;
}

// A cell the warm-rain step certainly leaves in place: no cloud or rain water, and vapour
// below 0.999 of saturation by a fast-math estimate of the state (its error is ~1e-6).
// With a non-negative autoconversion threshold micro_step takes none of its branches
// for such a cell, so the exact temperature, pressure and saturation are not needed.
// A false answer decides nothing: the cell is then judged on its exact state.
__device__ __forceinline__ bool surely_quiet(float rho_d, float rt, float rqv, float rqc, float rqr) {
  if (rqc > 0.0f || rqr > 0.0f) return false;
  const float rho = fmaxf(rho_d, 1.0e-6f), ir = __fdividef(1.0f, rho);
  const float ratio = fmaxf(rt * (kRd / kP0), 1.0e-6f);
  const float p = kP0 * __powf(ratio, 1.0f / (1.0f - kKappa));
  const float temp = rt * ir * __powf(fmaxf(p * (1.0f / kP0), 1.0e-6f), kKappa);
  const float tc = temp - 273.15f;
  const float es = 611.2f * __expf(__fdividef(17.67f * tc, fmaxf(tc + 243.5f, 1.0e-6f)));
  const float eps = kRd / kRv;
  const float qs = fminf(fmaxf(__fdividef(eps * es, fmaxf(p - (1.0f - eps) * es, 1000.0f)), 0.0f), 0.05f);
  return fmaxf(rqv * ir, 0.0f) < qs * (1.0f - 1.0e-3f);
}

// warm_rain_kernel body: warm_rain.cu:63-120 (saturation adjustment with latent heating,
// autoconversion, rain evaporation, clip at zero).  Updates c.th, c.qv, c.qc, c.qr.
// Process amounts of one micro_step (mixing-ratio units): condensation (vapour -> cloud,
// negative for cloud evaporation), autoconversion (cloud -> rain), rain evaporation
// (rain -> vapour).
struct MicroRates {
  float cond, autoconv, rain_evap;
};

__device__ __forceinline__ void micro_step(MicroCell& c, const MicroParams& m, MicroRates* rates = nullptr) {
  float th = c.th, qv = c.qv, qc = c.qc, qr = c.qr;
  const float rho = c.rho, lh = c.lh;
  float qs = qsat(c.temp, c.p);
  float r_cond = 0.0f, r_auto = 0.0f, r_evap = 0.0f;
  if (qv > qs) {
    const float cond = fminf((qv - qs) * fmaxf(m.relax, 0.0f), qv);
    qv -= cond;
    qc += cond;
    r_cond = cond;
    if (m.latent && cond > 0.0f) th += lh * cond;
  } else if (qv < qs && qc > 0.0f) {
    const float ev = fminf((qs - qv) * fmaxf(m.relax, 0.0f), qc);
    qv += ev;
    qc -= ev;
    r_cond = -ev;
    if (m.latent && ev > 0.0f) th -= lh * ev;
  }
  const float excess = fmaxf(qc - m.thr, 0.0f);
  if (excess > 0.0f && m.rate > 0.0f) {
    const float conv = fminf(excess, m.dt * m.rate * excess);
    qc -= conv;
    qr += conv;
    r_auto = conv;
  }
  // rain evaporation, from the saturation of the adjusted state: only a cell holding
  // rain needs it (the state is re-derived only there, with the same result)
  if (qr > 0.0f && m.evap > 0.0f) {
    const float p = eos_pressure(rho, rho * th);
    const float temp = th * powf(fmaxf(p / kP0, 1.0e-6f), kKappa);
    qs = qsat(temp, p);
    if (qv < qs) {
      const float ev = fminf(qr, m.dt * m.evap * fminf(qs - qv, qr));
      qr -= ev;
      qv += ev;
      r_evap = ev;
      if (m.latent && ev > 0.0f) th -= lh * ev;
    }
  }
  if (rates) *rates = MicroRates{r_cond, r_auto, r_evap};
  c.th = th;
  c.qv = fmaxf(qv, 0.0f);
  c.qc = fmaxf(qc, 0.0f);
  c.qr = fmaxf(qr, 0.0f);
}

// The process amounts of one micro_step as fractions of what bounds them, the
// surrogate's first three targets:
//   f_cond:  |cond| / |qv - qs| (the relaxation efficiency; capped by qv or qc),
//   f_auto:  autoconv / max(qc + cond - thr, 0),
//   f_evap:  rain_evap / (qr + autoconv).
// Where a bound is zero the fraction is the value the scheme's rate gives (relax,
// min(1, dt rate), 0), so the targets stay smooth.
__device__ __forceinline__ void rain_fractions(const MicroCell& c0, const MicroRates& r, const MicroParams& m,
                                               float* f) {
  const float d = c0.qv - qsat(c0.temp, c0.p);
  const bool can = d > 0.0f || (d < 0.0f && c0.qc > 0.0f);
  f[0] = can ? fabsf(r.cond) / fabsf(d) : fmaxf(m.relax, 0.0f);
  const float excess = fmaxf(c0.qc + r.cond - m.thr, 0.0f);
  f[1] = excess > 0.0f ? r.autoconv / excess : (m.rate > 0.0f ? fminf(m.dt * m.rate, 1.0f) : 0.0f);
  const float qr_mid = c0.qr + r.autoconv;
  f[2] = qr_mid > 0.0f ? r.rain_evap / qr_mid : 0.0f;
}

// Surrogate inputs of a cell: (T, p, rho_d, qv, qc, qr, dt).
constexpr int kRainIn = 7, kRainOut = 5;
__device__ __forceinline__ void rain_features(const MicroCell& c, float rho_d, float dt, float* x) {
  x[0] = c.temp;
  x[1] = c.p;
  x[2] = rho_d;
  x[3] = c.qv;
  x[4] = c.qc;
  x[5] = c.qr;
  x[6] = dt;
}

}  // namespace gwmb
