// plan_view.cu — the runtime plan view of a member's state (extract_runtime_plan_view,
// src/io/plan_view_output.cpp:715-834, with the dry bundle of extract_dry_plan_view,
// :630-713), computed on the device.
//
// One thread per column (i, j); a warp covers 32 consecutive i, so every load of a level
// is one coalesced row.  The thread diagnoses the slice level k (pressure, temperature,
// velocities, humidity, dewpoint, mixing ratios) and walks its column once for the
// column integrals (FP64, bottom to top, the reference's order) and the column maximum
// of the synthetic reflectivity.  The formulas and float constants are the reference's
// (include/gwm/core/dry_thermo.hpp:21-33, moist_thermo.hpp:23-74); each operation rounds
// on its own, as the reference's host code evaluates them (no fused multiply-adds).
#include "plan_view.cuh"

namespace gwmb {
namespace {

__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }

constexpr float kMinRho = 1.0e-6f;
constexpr float kEps = kRd / kRv;  // kEpsilon (moist_thermo.hpp:21)

// dry_pressure_from_rho_theta_m (dry_thermo.hpp:26-33)
__device__ float pressure_of(float rho, float rt) {
  const float theta = fdiv(rt, fmaxf(rho, kMinRho));
  const float ratio = fmaxf(fdiv(fmul(fmul(rho, kRd), theta), kP0), 1.0e-6f);
  return fmul(kP0, powf(ratio, 1.0f / (1.0f - kKappa)));
}
// saturation_specific_humidity (moist_thermo.hpp:23-36)
__device__ float qsat_of(float t, float p) {
  const float tc = fsub(t, 273.15f);
  const float es = fmul(fmul(6.112f, expf(fdiv(fmul(17.67f, tc), fmaxf(fadd(tc, 243.5f), 1.0e-6f)))), 100.0f);
  const float denom = fmaxf(fsub(p, fmul(1.0f - kEps, es)), 1000.0f);
  return fminf(fmaxf(fdiv(fmul(kEps, es), denom), 0.0f), 0.05f);
}
// relative_humidity_from_specific_humidity (moist_thermo.hpp:38-44)
__device__ float rh_of(float q, float t, float p) {
  const float qs = qsat_of(t, p);
  return fminf(fmaxf(qs > 0.0f ? fdiv(fmul(100.0f, q), qs) : 0.0f, 0.0f), 100.0f);
}
// dewpoint_from_specific_humidity (moist_thermo.hpp:46-55)
__device__ float dewpoint_of(float q_in, float p) {
  const float q = fminf(fmaxf(q_in, 0.0f), 1.0f);
  const float e = fdiv(fmul(p, q), fmaxf(fadd(kEps, fmul(1.0f - kEps, q)), 1.0e-6f));
  const float e_hpa = fmaxf(fmul(e, 0.01f), 1.0e-6f);
  const float l = logf(fdiv(e_hpa, 6.112f));
  return fadd(fdiv(fmul(243.5f, l), fsub(17.67f, l)), 273.15f);
}
// synthetic_reflectivity_dbz_from_rain (moist_thermo.hpp:66-74)
__device__ float dbz_of(float rho, float qr_in) {
  const float qr = fmaxf(qr_in, 0.0f);
  if (qr <= 1.0e-8f || rho <= 1.0e-8f) return -20.0f;
  const float z = fmul(3.63e9f, powf(fmul(rho, qr), 1.75f));
  return fmul(10.0f, log10f(fmaxf(z, 1.0e-6f)));
}

__global__ void __launch_bounds__(256) k_plan_view(const PlanViewArgs a) {
  const Geom& g = a.g;
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const int k = a.k;
  const size_t plane = (size_t)g.nx * g.ny, o = (size_t)j * g.nx + i;
  auto put = [&](int f, double v) { a.out[(size_t)f * plane + o] = v; };
  auto metric = [&](const float* m, int kk) { return __ldg(m + (a.metric_3d ? gidx(g, i, j, kk) : kk)); };
  const int c = gidx(g, i, j, k);

  // ---- the dry bundle (plan_view_output.cpp:75-224, 630-713)
  const float rho = __ldg(a.rho + c), rr = fmaxf(rho, kMinRho);
  const float theta = fdiv(__ldg(a.rt + c), rr);
  const float p = pressure_of(rho, __ldg(a.rt + c));
  const float t = fmul(theta, powf(fdiv(fmaxf(p, 1.0f), kP0), kKappa));
  const float uc = fdiv(fmul(0.5f, fadd(__ldg(a.u + c), __ldg(a.u + c + 1))), rr);
  const float vc = fdiv(fmul(0.5f, fadd(__ldg(a.v + c), __ldg(a.v + c + g.pitch))), rr);
  const float wc = fdiv(fmul(0.5f, fadd(__ldg(a.w + c), __ldg(a.w + c + g.plane))), rr);
  put(kPvZCenter, metric(a.zc, k));
  put(kPvRho, rho);
  put(kPvTheta, theta);
  put(kPvPressure, p);
  put(kPvTemperature, t);
  put(kPvU, uc);
  put(kPvV, vc);
  put(kPvWind, __fsqrt_rn(fadd(fmul(uc, uc), fmul(vc, vc))));
  put(kPvW, wc);
  if (a.nfields <= kPvDry) return;

  // ---- specific humidity, relative humidity, dewpoint (:226-232, 458-503)
  const float q = fdiv(__ldg(a.qv + c), rr);
  put(kPvQ, q);
  put(kPvRh, rh_of(q, t, p));
  put(kPvDewpoint, dewpoint_of(q, p));
  if (a.nfields <= kPvVapour) return;

  // ---- cloud and rain: slices (:234-280), column maps (:282-416)
  const float qcm = fdiv(__ldg(a.qc + c), rr), qrm = fdiv(__ldg(a.qr + c), rr);
  put(kPvQc, qcm);
  put(kPvQr, qrm);
  put(kPvCondensate, fadd(qcm, qrm));
  double col_c = 0.0, col_r = 0.0;
  float dbz = -20.0f;
  for (int kk = 0; kk < g.nz; ++kk) {
    const int ck = gidx(g, i, j, kk);
    const double dz = (double)fdiv(1.0f, metric(a.idc, kk));
    const float rk = __ldg(a.rho + ck), rqr = __ldg(a.qr + ck);
    col_c = __dadd_rn(col_c, __dmul_rn((double)__ldg(a.qc + ck), dz));
    col_r = __dadd_rn(col_r, __dmul_rn((double)rqr, dz));
    dbz = fmaxf(dbz, dbz_of(rk, fdiv(rqr, fmaxf(rk, kMinRho))));
  }
  const double total = col_c + col_r;
  const double tpos = fmax(total, 0.0);
  put(kPvColCloud, col_c);
  put(kPvColRain, col_r);
  put(kPvColTotal, total);
  put(kPvColRainFraction, tpos <= 0.0 ? 0.0 : fmin(fmax(col_r / tpos, 0.0), 1.0));
  put(kPvReflectivity, dbz);
  if (a.nfields <= kPvWarmRain) return;

  // ---- accumulated surface precipitation and its mean rate (:418-456, 804-830)
  const double pr = a.precip[o] + a.precip_comp[o];
  put(kPvPrecip, pr);
  put(kPvPrecipRate, pr * a.inv_hours);
}

}  // namespace

cudaError_t launch_plan_view(const PlanViewArgs& a, cudaStream_t s) {
  if (a.g.nx <= 0 || a.g.ny <= 0 || a.k < 0 || a.k >= a.g.nz || !a.out) return cudaErrorInvalidValue;
  if (a.nfields > kPvDry && !a.qv) return cudaErrorInvalidValue;
  if (a.nfields > kPvVapour && (!a.qc || !a.qr)) return cudaErrorInvalidValue;
  if (a.nfields > kPvWarmRain && (!a.precip || !a.precip_comp)) return cudaErrorInvalidValue;
  const dim3 block(32, 8), grid((a.g.nx + 31) / 32, (a.g.ny + 7) / 8);
  k_plan_view<<<grid, block, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace gwmb
