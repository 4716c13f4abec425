// dycore.cuh — launch interface of the dry-dynamics kernels (slow RK stage and
// acoustic substep) of the time-step hot path.
#pragma once

#include <cuda.h>

#include "common.cuh"

namespace gwmb {

constexpr int kMaxNz = 256;   // level-mean tables live in shared memory

// Arguments of one fused slow RK stage: tendencies of
// src/dycore/dry_core.cu:400-539 (K2, K3, K16-K19, K21, K22) plus the stage
// update (K4, :189-197) and SSPRK3 blend (K5, :199-205), for every owned cell and
// face, in one pass up the columns.
struct SlowArgs {
  Geom g;
  const float* rho;                 // stage input density
  const float* th;                  // rho*theta (th_is_rt=1) or theta (0)
  int th_is_rt;
  const float *u, *v, *w;           // stage input momenta (base part)
  const float *du, *dv, *dw;        // acoustic increments added to u,v,w (may be null)
  const float *rho0, *rt0, *u0, *v0, *w0;  // SSPRK3 blend partner q0 (null: no blend)
  float wa, wb;                     // out = wa*q0 + wb*max(floor, q + dt*L(q))
  float dt, gravity;
  float *o_rho, *o_th, *o_u, *o_v, *o_w;
  int out_rt;                       // o_th receives rho*theta (1) or theta (0)
  int tend_only;                    // write raw tendencies L(q), no update/blend/mirror
  const unsigned long long* th_acc; // theta level sums of the input state
  unsigned long long *acc_a, *acc_b; // level sums of the output (see acc_mode)
  unsigned long long *clr_a, *clr_b; // ring slot cleared by block (0,0)
  int acc_mode;                     // 0 none, 1 rho & p of output, 2 theta of output
  float* p_out;                     // acc_mode 1, TMA kernel only: p' of the output (owned cells
                                    // and periodic halo), for the first substep (may be null)
  double inv_count;                 // 1 / (nx*ny)
  const float *zc, *idz_c, *idz_f;  // metrics: padded 3-D (terrain) or per level (flat)
  const double* base;               // FP64 base state [rt_ref | 1/rt_ref | p_ref] per level
  int* err;                         // error word: set to 1 when a bounded wait gave up
  // Rayleigh damping layer (extension; null: off): per-level rates at cell centres and
  // Z faces, and the momentum profiles u, v relax to
  const float *damp_c, *damp_f, *uref, *vref;
};

// TMA descriptors of one slow stage (flat terrain, k_slow_tma): 3-D tiled maps over the
// padded layout with 40 x 18 boxes (cells, X and Z faces) and 40 x 19 (Y faces).
struct SlowMaps {
  CUtensorMap rho, th, u, v, w, du, dv, dw;
  CUtensorMap z;  // cell-centre heights (terrain form only)
};

// Arguments of one acoustic substep: src/dycore/dry_fast_modes.cu:495-652
// (K9-K15) with momenta carried as increments D = m - m_base.
struct FastArgs {
  Geom g;
  const float* rho_in;
  float* rho_out;
  const float* th;                  // theta frozen for the RK stage
  const float *du_in, *dv_in, *dw_in;   // increments before the substep (null: zero)
  float *du_out, *dv_out, *dw_out;
  // pressure of rho_in from the previous substep, and of rho_out for the next one (TMA
  // paths, inner substeps): the perturbation p' on flat terrain, the full pressure on terrain
  const float* p_in;
  float* p_out;
  const float *bu, *bv, *bw;        // stage base momenta (final_kind == 2)
  float *f_rho, *f_rt, *f_u, *f_v, *f_w;  // step result (final_kind == 2)
  int final_kind;                   // 0 inner substep, 1 last of a stage, 2 last of the step
  int acc_off;                      // skip the output level sums
  float dtf, gravity;
  int hmom, dens;
  const unsigned long long *ref_a, *ref_b;  // level sums of rho_in, p(rho_in) (flat terrain)
  double inv_count;
  unsigned long long *acc_a, *acc_b, *clr_a, *clr_b;
  const float *zc, *idz_c, *idz_f;
  const double* base;
  int* err;                         // error word: set to 1 when a bounded wait gave up
  // terrain: the column hydrostatic reference (K11) of rho_in, pressure and density per
  // cell, written by launch_column_reference before the substep and read by it
  float *col_pref, *col_rref;
};

// TMA descriptors of one acoustic substep (flat terrain, k_fast_tma): 3-D tiled maps
// over the padded field layout (dims pitch x rows x (nz+1), FP32, no swizzle).
struct FastMaps {
  CUtensorMap rho, th;     // first substep of a stage deriving p': box 40 x 18, cells with
                           // the halo ring; otherwise box 32 x 16, owned cells
  CUtensorMap du, dv;      // box 36 x 17: owned faces + the tile's east/north face
  CUtensorMap dw;          // box 32 x 16
  CUtensorMap bu, bv, bw;  // box 32 x 16 (last substep of the step)
  CUtensorMap p;           // box 40 x 18: p'(rho_in) with the halo ring (loaded unless the
                           // first substep derives it)
};
// TMA descriptors of one acoustic substep on terrain (k_fast_terrain_tma), same layout.
struct FastTerrainMaps {
  CUtensorMap rho, th;  // first substep of a stage: box 40 x 18 (cells with the halo
                        // ring); otherwise box 32 x 16 (owned cells)
  CUtensorMap z;        // box 40 x 18: cell-centre heights
  CUtensorMap p;        // box 40 x 18: full pressure of rho_in (not the first substep)
  CUtensorMap du, dv;   // box 36 x 17 (not the first substep)
  CUtensorMap dw;       // box 32 x 16 (not the first substep)
};
// Box extents (x, y) of the maps above.
constexpr int kTmaCellBox[2] = {40, 18};
constexpr int kTmaFaceBox[2] = {36, 17};
constexpr int kTmaOwnBox[2] = {32, 16};
constexpr int kTmaYFaceBox[2] = {40, 19};

// Level sums of a stored state.  mode 0: theta = rt/max(rho,1e-6) (the host loop of
// dry_core.cu:462-476); mode 1: rho and p(rho, rho*theta) (K6 of dry_fast_modes.cu:42-57);
// mode 2: theta of a stage input stored as (rho, theta): theta_of(rho, rho*theta).
struct LevelSumArgs {
  Geom g;
  const float *rho, *rt;
  int mode;
  unsigned long long *acc_a, *acc_b, *clr_a, *clr_b;
  const double* base;
};

// tile_rows: CTA rows of the overlapped slow-stage tile (8 or 16; 32 columns wide).
cudaError_t launch_slow(const SlowArgs& a, bool terrain, cudaStream_t s, int tile_rows);
// tile_rows: CTA rows of the acoustic-substep tile (8 or 16; 32 columns wide).
cudaError_t launch_fast(const FastArgs& a, bool first, bool terrain, cudaStream_t s, int tile_rows);
// Flat-terrain slow stage on owned 32 x 16 tiles fed by TMA (not for tend_only).
cudaError_t launch_slow_tma(const SlowArgs& a, const SlowMaps& m, cudaStream_t s);
cudaError_t init_slow_tma();
// Terrain slow stage on owned 32 x 16 tiles fed by TMA (not for tend_only, no p' level
// sums): the arithmetic of the overlapped-tile terrain kernel; m.z maps the heights.
cudaError_t launch_slow_terrain_tma(const SlowArgs& a, const SlowMaps& m, cudaStream_t s);
cudaError_t init_slow_terrain_tma();
// Flat-terrain acoustic substep fed by TMA tile loads (owned 32 x 16 tiles).
// first: the first substep of a stage (no increments in); p_ready: its p' (with the
// halo ring) is in a.p_in, written by the slow stage, instead of derived from rho, theta
cudaError_t launch_fast_tma(const FastArgs& a, const FastMaps& m, bool first, bool p_ready, cudaStream_t s);
// Acoustic substep on terrain fed by TMA tile loads (owned 32 x 16 tiles): the
// arithmetic of the overlapped-tile terrain kernel.  Needs a.col_pref / a.col_rref
// (launch_column_reference of a.rho_in first); inner substeps (final_kind 0) store the
// full pressure of their result in a.p_out, which the next substep loads as a.p_in.
cudaError_t launch_fast_terrain_tma(const FastArgs& a, const FastTerrainMaps& m, bool first, cudaStream_t s);
cudaError_t init_fast_terrain_tma();
// K11 build_column_hydrostatic_reference_kernel (dry_fast_modes.cu:108-158) of a.rho_in
// and a.th into a.col_pref / a.col_rref: one thread per owned column, bottom to top.
cudaError_t launch_column_reference(const FastArgs& a, cudaStream_t s);
// Consecutive acoustic substeps of one RK stage (flat terrain, TMA path) in one
// cooperative launch: a[q], m[q] as launch_fast_tma takes them for substep q (q = 0 the
// stage's first); count/gen: two device words of the grid barrier (count is zeroed on the
// stream before the launch).  Results equal one launch per substep bit for bit.
constexpr int kFastStageMax = 8;
struct FastStage {
  FastMaps m[kFastStageMax];
  FastArgs a[kFastStageMax];
  unsigned *count, *gen;
  int n;
  int slot_floats;  // set by the launch: the longest ring slot of the substeps
};
cudaError_t launch_fast_stage_tma(FastStage& st, bool p_ready, cudaStream_t s);
// One-time kernel attributes (dynamic shared memory) of the TMA substep.
cudaError_t init_fast_tma();
cudaError_t launch_level_sums(const LevelSumArgs& a, cudaStream_t s);
// FP64 base state of the pressure-perturbation EOS: per level the mean rho_theta of
// the state, its reciprocal and p_ref = EOS(mean rho_theta); one CTA per level.
cudaError_t launch_base_state(const Geom& g, const float* rt, double* base, cudaStream_t s);
// theta = rt/max(rho,1e-6) on owned cells with periodic halo mirroring
// (compute_theta_field_kernel + exchange_scalar, dry_fast_modes.cu:86-95, 453-462).
cudaError_t launch_theta_field(const Geom& g, const float* rho, const float* rt, float* th,
                               cudaStream_t s);

}  // namespace gwmb
