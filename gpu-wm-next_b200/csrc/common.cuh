// common.cuh — device layout, thermodynamics and small helpers shared by the
// sm_100a kernels of the time-step hot path.
//
// HBM layout (one array per field per member, all fields share one geometry):
//   idx(i, j, k) = k * plane + (j + 1) * pitch + (i + kXOff)
// with i in [-1, nx+1], j in [-1, ny+1], k in [0, nz]  (cells use i < nx+1,
// j < ny+1, k < nz; X faces use i <= nx+1; Y faces j <= ny+1; Z faces k <= nz).
// kXOff = 32 puts owned column 0 on a 128-byte boundary, so a warp's row load
// of 32 owned cells is exactly one 128-byte line.  pitch is a multiple of 32
// floats and plane = pitch * (ny + 3).  Halo width is 1, as in the reference
// (every stencil of src/dycore/*.cu reaches one cell).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gwmb {

constexpr int kXOff = 32;

struct Geom {
  int nx, ny, nz;
  int pitch;        // floats per row
  int rows;         // ny + 3
  int plane;        // pitch * rows
  int per_x, per_y; // periodic lateral boundaries (else open: zero halos)
  float dx, dy;
};

__host__ __device__ __forceinline__ int gidx(const Geom& g, int i, int j, int k) {
  return k * g.plane + (j + 1) * g.pitch + (i + kXOff);
}

enum Orient : int { kCell = 0, kFaceX = 1, kFaceY = 2, kFaceZ = 3 };

// ---------------------------------------------------------------------------
// Thermodynamics.  Same formulas and float constants as the reference
// (include/gwm/core/dry_thermo.hpp:17-44, moist_thermo.hpp:18-62).
constexpr float kRd = 287.05f;
constexpr float kP0 = 100000.0f;
constexpr float kKappa = 0.2854f;
constexpr float kRv = 461.5f;
constexpr float kLv = 2.5e6f;

__device__ __forceinline__ float theta_of(float rho, float rt) {
  return rt / fmaxf(rho, 1.0e-6f);
}
__device__ __forceinline__ float eos_pressure(float rho, float rt) {
  const float th = theta_of(rho, rt);
  const float ratio = fmaxf(rho * kRd * th / kP0, 1.0e-6f);
  return kP0 * powf(ratio, 1.0f / (1.0f - kKappa));
}
__device__ __forceinline__ float eos_rho(float p, float th) {
  const float ex = powf(fmaxf(p / kP0, 1.0e-6f), kKappa);
  return p / fmaxf(kRd * th * ex, 1.0e-6f);
}
__device__ __forceinline__ float dry_cp() { return kRd / kKappa; }

__device__ __forceinline__ float upwind(float a, float ql, float qr) {
  return a >= 0.0f ? a * ql : a * qr;
}

// ---------------------------------------------------------------------------
// Periodic halo mirroring on store.  A value written at an owned position that
// the reference's halo exchange would copy into a halo slot
// (src/comm/halo_exchange.cpp:32-116 faces, :313-373 cells) is written there
// too, by the same thread.  X faces 0 and nx are both owned positions (they
// alias under periodic wrap and are computed identically); face 1 feeds halo
// face nx+1 and face nx-1 feeds halo face -1.  Open axes leave halos at zero.
__device__ __forceinline__ int mirror_targets(int i, int n, bool periodic, bool face, int* out) {
  int c = 0;
  out[c++] = i;
  if (!periodic) return c;
  if (face) {
    if (i == 1) out[c++] = n + 1;
    if (i == n - 1) out[c++] = -1;
  } else {
    if (i == 0) out[c++] = n;
    if (i == n - 1) out[c++] = -1;
  }
  return c;
}

__device__ __forceinline__ void store_mirrored(float* f, const Geom& g, int o, int i, int j,
                                               int k, float v) {
  int xs[3], ys[3];
  const int cx = mirror_targets(i, g.nx, g.per_x != 0, o == kFaceX, xs);
  const int cy = mirror_targets(j, g.ny, g.per_y != 0, o == kFaceY, ys);
  for (int a = 0; a < cy; ++a)
    for (int b = 0; b < cx; ++b) f[gidx(g, xs[b], ys[a], k)] = v;
}

// ---------------------------------------------------------------------------
// Deterministic level sums.  Each CTA reduces its cells in a fixed order (FP64),
// converts the partial to 64-bit fixed point and adds it with an integer atomic.
// Integer addition is associative, so the result does not depend on CTA
// arrival order: reruns are bitwise identical.  Scales keep the largest sums
// (1.6e7 cells per level) inside int64.
constexpr double kScaleRho = 4294967296.0;    // 2^32
constexpr double kScaleP = 1048576.0;         // 2^20
constexpr double kScaleTheta = 268435456.0;   // 2^28

__device__ __forceinline__ void acc_add(unsigned long long* acc, double v, double scale) {
  const long long q = __double2ll_rn(v * scale);
  atomicAdd(acc, (unsigned long long)q);
}
__device__ __forceinline__ double acc_read(const unsigned long long* acc, double scale) {
  return (double)(long long)(*acc) / scale;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace gwmb
