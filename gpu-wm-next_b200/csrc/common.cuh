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
  float inv_dx, inv_dy;
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
// One-sided / centred dp/dz of a column (terrain pressure gradient):
// dry_pressure_gradient.cu:37-73.
__device__ __forceinline__ float column_dpdz(int k, int nz, float pm, float pc, float pn, float zm,
                                             float zcc, float zn) {
  if (nz == 1) return 0.0f;
  if (k == 0) return (pn - pc) / fmaxf(zn - zcc, 1.0e-6f);
  if (k + 1 == nz) return (pc - pm) / fmaxf(zcc - zm, 1.0e-6f);
  return (pn - pm) / fmaxf(zn - zm, 1.0e-6f);
}

// ---------------------------------------------------------------------------
// Pressure perturbation about an FP64 base state.  The reference EOS
// p = p0 (Rd rho_theta / p0)^g, g = 1/(1-kappa) (dry_thermo.hpp:26-33) depends on
// rho_theta alone, so with a per-level base rt_ref(k), p_ref(k) = EOS(rt_ref):
//   p - p_ref = p_ref ((1 + d)^g - 1),  d = rho_theta / rt_ref - 1.
// For |d| < 1/16 the binomial series to d^7, evaluated in FP64, leaves a relative
// truncation error below 3e-10 of p' (the next term is C(g,8) d^8 / (g d)), far
// below the FP32 rounding of the result; otherwise the full EOS is evaluated and
// the base subtracted.  Horizontal differences of p' equal those of p exactly in
// real arithmetic (the base is constant on a level) but keep ~1e-5 Pa resolution
// instead of the ~1e-2 Pa of an FP32 pressure near 1e5 Pa.
// base layout: [rt_ref(nz) | 1/rt_ref(nz) | p_ref(nz)], FP64.
// Core form with the level's 1/rt_ref and p_ref already at hand.
__device__ __forceinline__ float eos_pprime_ref(float rho, float rt, double inv_rt_ref, double pref) {
  const double d = fma((double)rt, inv_rt_ref, -1.0);
  if (rho >= 1.0e-6f && fabs(d) < 0.0625) {
    // C(g, n), n = 1 .. 7, for g = 1.0f / (1.0f - 0.2854f); Estrin's scheme keeps the
    // dependent FP64 chain three operations deep instead of seven (Horner)
    const double d2 = d * d, d4 = d2 * d2;
    const double a = fma(0.2794461309425813, d, 1.3993843793869019);
    const double b = fma(0.022387238647368683, d, -0.055946570454669185);
    const double c = fma(0.0069876670302162856, d, -0.011644120505748048);
    const double lo = fma(b, d2, a);
    const double hi = fma(-0.0045925100129794545, d2, c);
    const double s = fma(hi, d4, lo);
    return (float)(pref * (s * d));
  }
  return (float)((double)eos_pressure(rho, rt) - pref);
}
__device__ __forceinline__ float eos_pprime(float rho, float rt, const double* __restrict__ base, int k,
                                            int nz) {
  return eos_pprime_ref(rho, rt, __ldg(base + nz + k), __ldg(base + 2 * nz + k));
}

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
// Store for a CTA whose tile may touch a periodic edge (edge=true) or certainly
// does not (edge=false, a plain store).
__device__ __forceinline__ void store_mirrored(float* __restrict__ f, const Geom& g, int o, int i,
                                               int j, int k, float v);
__device__ __forceinline__ void store_tile(float* __restrict__ f, const Geom& g, int o, int i, int j,
                                           int k, float v, bool edge) {
  if (edge) store_mirrored(f, g, o, i, j, k, v);
  else f[gidx(g, i, j, k)] = v;
}

// Mirrors are shifts by +-nx columns and +-ny rows: cell 0 -> nx, cell nx-1 -> -1,
// X face 0 -> nx (its periodic alias), X face 1 -> nx+1, X face nx-1 -> -1 (same
// in y).  Interior positions take one store and a predicated exit; only the edge
// ring takes the extra stores.
__device__ __forceinline__ void store_mirrored(float* __restrict__ f, const Geom& g, int o, int i,
                                               int j, int k, float v) {
  const int at = gidx(g, i, j, k);
  f[at] = v;
  const bool xh = g.per_x && (i == 0 || (o == kFaceX && i == 1));
  const bool xl = g.per_x && i == g.nx - 1;
  const bool yh = g.per_y && (j == 0 || (o == kFaceY && j == 1));
  const bool yl = g.per_y && j == g.ny - 1;
  if (!(xh || xl || yh || yl)) return;
  const int sx = g.nx, sy = g.ny * g.pitch;
  if (xh) f[at + sx] = v;
  if (xl) f[at - sx] = v;
  if (yh) {
    f[at + sy] = v;
    if (xh) f[at + sy + sx] = v;
    if (xl) f[at + sy - sx] = v;
  }
  if (yl) {
    f[at - sy] = v;
    if (xh) f[at - sy + sx] = v;
    if (xl) f[at - sy - sx] = v;
  }
}

// ---------------------------------------------------------------------------
// Deterministic level sums.  Every cell's value is converted to 64-bit fixed point
// on its own (v * 2^s is exact in FP32 for a power-of-two scale; the conversion
// rounds to nearest) and the integers are summed: warp shuffles, a CTA total and one
// integer atomic per CTA and level.  Integer addition is exact and associative, so a
// level sum depends only on the cell values: not on CTA arrival order, tile shape or
// which kernel computed it.  Reruns, and runs with different tile choices, are
// bitwise identical.  Scales keep the largest sums (1.6e7 cells per level) inside
// int64.
constexpr double kScaleRho = 4294967296.0;    // 2^32
constexpr double kScaleP = 16777216.0;        // 2^24 (pressure perturbations)
constexpr double kScaleTheta = 268435456.0;   // 2^28
constexpr float kFxRho = 4294967296.0f;
constexpr float kFxP = 16777216.0f;
constexpr float kFxTheta = 268435456.0f;

__device__ __forceinline__ long long fx(float v, float scale) { return __float2ll_rn(v * scale); }
__device__ __forceinline__ void acc_add(unsigned long long* acc, long long q) {
  atomicAdd(acc, (unsigned long long)q);
}
__device__ __forceinline__ double acc_read(const unsigned long long* acc, double scale) {
  return (double)(long long)(*acc) / scale;
}
// Per-thread fixed-point accumulator for at most 4 cells (the warp's sum of lo
// parts must stay below 2^32), reduced across
// the warp with two 32-bit integer reductions.  A cell's fixed-point value
// x = fx(v, scale) is split as x = hi * 2^24 + lo with 0 <= lo < 2^24 (an arithmetic
// shift and a mask of the int64).  The warp total sum(hi) * 2^24 + sum(lo) therefore
// equals the int64 sum of fx() over the same cells, bit for bit, at a fraction of the
// cost of 64-bit shuffles.
struct FxAcc {
  int hi = 0;
  unsigned lo = 0;
  __device__ __forceinline__ void add(float v, float scale) {
    const long long x = fx(v, scale);
    hi += (int)(x >> 24);
    lo += (unsigned)(x & 0xffffffLL);
  }
  // warp total (all lanes get it); every lane of the warp must call it
  __device__ __forceinline__ long long warp_total() const {
    const int sh = __reduce_add_sync(0xffffffffu, hi);
    const unsigned sl = __reduce_add_sync(0xffffffffu, lo);
    return (long long)sh * 16777216LL + (long long)sl;
  }
};

__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace gwmb
