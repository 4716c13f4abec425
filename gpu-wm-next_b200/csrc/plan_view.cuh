// plan_view.cuh — launch interface of the runtime plan view (plan_view.cu).
#pragma once

#include "common.cuh"

namespace gwmb {

// Fields of the runtime plan-view bundle in the bundle's order
// (extract_dry_plan_view + extract_runtime_plan_view, src/io/plan_view_output.cpp:630-834).
enum PlanViewField : int {
  kPvTerrain = 0, kPvZCenter, kPvRho, kPvTheta, kPvPressure, kPvTemperature, kPvU, kPvV, kPvWind, kPvW,
  kPvDry,  // fields of the dry bundle
  kPvQ = kPvDry, kPvRh, kPvDewpoint,
  kPvVapour,  // + the specific-humidity fields
  kPvQc = kPvVapour, kPvQr, kPvCondensate, kPvColCloud, kPvColRain, kPvColTotal, kPvColRainFraction,
  kPvReflectivity,
  kPvWarmRain,  // + the cloud and rain fields
  kPvPrecip = kPvWarmRain, kPvPrecipRate,
  kPvAll
};

struct PlanViewArgs {
  Geom g;
  int k;                   // slice level (clamped by the caller)
  int nfields;             // kPvDry, kPvVapour, kPvWarmRain or kPvAll
  const float *rho, *rt, *u, *v, *w;
  const float *zc, *idc;   // metric z_center and inv_dz_cell: padded 3-D fields, or one value per level
  int metric_3d;
  const float *qv, *qc, *qr;          // tracer masses rho*q (qc, qr: nfields > kPvVapour)
  const double *precip, *precip_comp;  // accumulated surface precipitation (nfields == kPvAll)
  double inv_hours;        // 1 / max(elapsed hours, 1e-9)
  double* out;             // nfields x ny x nx, row-major (y, x); field 0 (terrain) is left alone
};

cudaError_t launch_plan_view(const PlanViewArgs& a, cudaStream_t s);

}  // namespace gwmb
