// halo.cuh — layout kernels: owned<->padded packing, virtual-rank halo exchange
// on the reference's per-rank Field3D layout, and FP64 budget reductions.
#pragma once

#include "common.cuh"

namespace gwmb {

constexpr int kMaxRanks = 64;

// Owned global array (fz, fy, fx) -> padded field; aliased periodic faces
// (X face 0 / nx, Y face 0 / ny) receive their average, which is what the
// reference's first interface sync makes of them (halo_exchange.cpp:217-285).
cudaError_t launch_pack(const Geom& g, int orient, const float* src, float* dst, cudaStream_t s);
cudaError_t launch_unpack(const Geom& g, int orient, const float* src, float* dst, cudaStream_t s);

// Per-rank descriptor in the reference layout: include/gwm/domain/subdomain_descriptor.hpp:7-26
struct RankDesc {
  int nxl, nyl;
  int west, east, south, north;
  float* data;   // device pointer, Field3D storage of this rank
};
struct RankTable {
  int n, nz, halo, orient;
  RankDesc r[kMaxRanks];
};
// op 0: HaloExchange::exchange_* (halo_exchange.cpp:148-215, 563-620);
// op 1: synchronize_owned_face_interfaces (:217-285).
cudaError_t launch_rank_halo(const RankTable& t, int op, cudaStream_t s);

// Boundary strips (apply_reference_boundaries, src/dycore/boundary_conditions.cpp:8-208):
// the outermost owned strips of a field, over the field's own storage extents
// (fx, fy, fz) = owned shape of its orientation, stored compactly as
//   [west: fy*fz | east: fy*fz | south: fx*fz | north: fx*fz], k-major within a strip.
// Job modes: 0 apply compact -> padded (open sides only, periodic mirrors written);
// 1 save padded -> compact; 2 extract owned global array -> compact (aliased periodic
// faces averaged, as launch_pack does); 3 apply theta = rt/max(rho, 1e-6) from two
// compact strips (c1 = rho*theta, c2 = rho); 4 zero the padded strips (open sides).
struct StripJob {
  float* padded;        // modes 0, 1, 3, 4
  float* compact;       // modes 0-3 (read for 0, 3; written for 1, 2)
  const float* aux;     // mode 2: owned global array; mode 3: rho strips
  int orient, mode;
};
constexpr int kMaxStripJobs = 8;
struct StripJobs {
  int n;
  StripJob j[kMaxStripJobs];
};
long long strip_len(const Geom& g, int orient);  // compact floats of one field
cudaError_t launch_strips(const Geom& g, const StripJobs& jobs, cudaStream_t s);

// Prepared-case boundary updater (src/ingest/prepared_case_init.cpp:396-645,1006-1078)
// on the device.  A cache of snapshots holds, per snapshot, the compact strips of the
// balanced dry state (rho, rho*theta, u, v, w) and of the tracer mixing ratios; the
// strips applied at an updater call are those of the snapshot interpolated at the
// forecast second lround(step_start + sim_time) (runtime_case.cpp:205-228,
// boundary_cache.hpp:52-76), tracers as rho_d * q (prepared_case_init.cpp:570-645).
// The clock holds the step start time and, per RK stage (sim_time 0, dt, dt/2), the
// bracketing snapshots and the weight; one kernel per step fills the table and
// advances the start time by dt (float, as the driver's sim_time += dt), so a captured
// step replays with the forecast time moving on.
struct BoundaryClock {
  float t_start, dt;
  int lo[3], hi[3];
  float alpha[3];
};
cudaError_t launch_boundary_clock(BoundaryClock* clock, const int* offsets, int n, cudaStream_t s);
// Strips of stage `stage` (per snapshot: dry_len dry floats, then ntr cell strips of
// cell_len floats) into out, laid out like one snapshot.
cudaError_t launch_boundary_interp(const float* cache, long long per_snap, long long dry_len, long long cell_len,
                                   int ntr, const BoundaryClock* clock, int stage, float* out, cudaStream_t s);

// EOS over n values (K20 compute_pressure_kernel, dry_pressure_gradient.cu:27-35).
cudaError_t launch_pressure(const float* rho, const float* rt, float* p, long long n, cudaStream_t s);

// Reductions over owned positions.  mode 0: value; 1: theta = rt/max(rho,1e-12)
// in FP64 (dry_diagnostics.cpp:33-45); 2: column water rho_q*dz with
// dz = 1/inv_dz_cell in FP64 (runtime_summary.cpp:72-81).
struct ReduceOut {
  double sum, mn, mx;
};
// partials: scratch of >= 3*kReduceBlocks doubles; out: device ReduceOut.
constexpr int kReduceBlocks = 296;
cudaError_t launch_reduce(const Geom& g, int orient, int mode, const float* f, const float* rho,
                          const float* idz, int idz_terrain, double* partials, ReduceOut* out,
                          cudaStream_t s);
cudaError_t launch_reduce_2d(const double* a, const double* b, long long n, double* partials,
                             ReduceOut* out, cudaStream_t s, int mode = 0);

}  // namespace gwmb
