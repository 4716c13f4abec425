// physics.cuh — launch interface of the moist kernels: passive-tracer SSPRK3
// stages and warm-rain microphysics with bounded column fallout.
#pragma once

#include <cuda.h>

#include "common.cuh"

namespace gwmb {

// One SSPRK3 stage of the three warm-rain tracers with frozen dry mass fluxes:
// passive_tracer_stage_kernel (src/dycore/dry_transport.cu:49-125) for all
// tracers in one pass, fused with the blend (:40-47).
struct TracerArgs {
  Geom g;
  const float* rho;                 // frozen dry density (end of the dry step)
  const float *u, *v, *w;           // frozen mass fluxes
  const float* q_in[3];             // stage input rho*q
  const float* q0[3];               // blend partner (null: stage 1)
  float* q_out[3];
  float wa, wb, dt;
  int ntracers;
  const float* idz_c;               // per level (flat) or padded 3-D (terrain)
  int terrain;
  int* err;                         // error word: set to 1 when a bounded wait gave up
};

// TMA descriptors of one tracer stage (flat terrain, k_tracer_tma).
struct TracerMaps {
  CUtensorMap rho, q[3];  // box 40 x 18: cells with the halo ring
  CUtensorMap u, v;       // box 36 x 17: owned faces + the east/north face
  CUtensorMap w;          // box 32 x 16
};

// Warm-rain microphysics (warm_rain.cu:36-120) followed, in the same column
// sweep, by rain fallout (metric :156-191 or nominal :122-154).
struct RainArgs {
  Geom g;
  const float* rho;
  float *rt, *qv, *qc, *qr;
  double *precip, *precip_comp;     // FP64 surface accumulation + Neumaier term, (ny, nx); null: none
  float dt, relax, thr, rate, evap, vt, layer_depth;
  int latent, fallout_mode;         // fallout_mode: 0 none, 1 metric, 2 nominal
  const float* idz_c;
  int terrain;
  unsigned long long* th_acc;       // theta level sums of the result (null: none)
  double inv_count;
};

// tile_rows: CTA rows of the overlapped tracer tile (8 or 16; 32 columns wide).
cudaError_t launch_tracer_stage(const TracerArgs& a, cudaStream_t s, int tile_rows);
// Flat-terrain tracer stage on owned 32 x 16 tiles fed by TMA.
cudaError_t launch_tracer_tma(const TracerArgs& a, const TracerMaps& m, cudaStream_t s);
cudaError_t init_tracer_tma();
// micro = false: fallout (and theta level sums) only, on a state whose microphysics
// was already applied.
cudaError_t launch_warm_rain(const RainArgs& a, cudaStream_t s, bool micro = true);

}  // namespace gwmb
