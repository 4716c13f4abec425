// stencil.cuh — the FP32 formulas of the step's stencils with their rounding written out.
//
// Every kernel variant of an operator (TMA-fed owned tiles, owned tiles, overlapped
// tiles; interior and edge copies of a plane loop) computes each value through these
// functions.  Each operation rounds on its own (__fadd_rn, __fmul_rn, ...) and an FMA is
// used only where written, so the compiler cannot contract the same expression
// differently in two kernels or two copies of a loop: the variants agree bit for bit by
// construction.  The formulas and constants are the reference's (file:line per function);
// the FMAs are placed where a multiply feeds an add, the contraction a CUDA build of the
// reference makes of the same expressions.
#pragma once

#include <cuda_runtime.h>

namespace gwmb {
namespace fp {

__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }

// 0.5 (a + b)
__device__ __forceinline__ float avg(float a, float b) { return mul(0.5f, add(a, b)); }

// First-order upwind flux a * (a >= 0 ? q_upstream_low : q_upstream_high)
// (dry_core.cu:98-120, dry_momentum_flux.cu:79-312, dry_transport.cu:91-114).
__device__ __forceinline__ float upwind(float a, float ql, float qr) { return mul(a, a >= 0.0f ? ql : qr); }

// Divergence (e - w) idx + (n - s) idy + (t - b) idz of face values or fluxes.
__device__ __forceinline__ float divergence(float e, float w, float n, float s, float t, float b, float idx, float idy,
                                            float idz) {
  return fma(sub(t, b), idz, fma(sub(n, s), idy, mul(sub(e, w), idx)));
}

// K4 stage update with a floor (dry_core.cu:189-197): max(lo, q + dt tend).
__device__ __forceinline__ float update(float q, float dt, float tend, float lo) { return fmaxf(lo, fma(dt, tend, q)); }

// K5 blend (dry_core.cu:199-205, dry_transport.cu:40-47): wa q0 + wb q.
__device__ __forceinline__ float blend(float wa, float q0, float wb, float q) { return fma(wa, q0, mul(wb, q)); }

// theta = rho_theta / max(rho, 1e-6) (include/gwm/core/dry_thermo.hpp:21-24).
__device__ __forceinline__ float theta(float rho, float rt) { return div(rt, fmaxf(rho, 1.0e-6f)); }

// Cell-centred velocity 0.5 (m_a + m_b) / max(rho, 1e-6) (dry_momentum_flux.cu:36-73).
__device__ __forceinline__ float centred(float ma, float mb, float rr) { return div(avg(ma, mb), rr); }

// ---- acoustic substep (dry_fast_modes.cu:160-394) --------------------------------
// K12/K13 horizontal momentum increment on flat levels: d - dtf (p_r - p_l) inv_d.
__device__ __forceinline__ float hmom(float d, float pr, float pl, float inv_d, float dtf) {
  return fma(-dtf, mul(sub(pr, pl), inv_d), d);
}
// K12/K13 on terrain: the chain-rule gradient (p_r - p_l) inv_d - dz/dx dp/dz
// (dry_fast_modes.cu:160-301, docs/math/terrain_metric_operators.md:7-14).
__device__ __forceinline__ float hmom_terrain(float d, float pr, float pl, float zr, float zl, float dpdz_l,
                                              float dpdz_r, float inv_d, float dtf) {
  const float dzdx = mul(sub(zr, zl), inv_d);
  const float x = fma(-dzdx, avg(dpdz_l, dpdz_r), mul(sub(pr, pl), inv_d));
  return fma(-dtf, x, d);
}
// K14 vertical momentum increment at a face: dw + dtf (-(p'_u - p'_l) idzf - g rho'_f),
// with p'_u = pn - pru, p'_l = pc - prl and rho'_f = 0.5 ((rc - rrl) + (rn - rru)).
__device__ __forceinline__ float wmom(float dw, float pn, float pru, float pc, float prl, float rc, float rrl, float rn,
                                      float rru, float idzf, float gravity, float dtf) {
  const float dp = sub(sub(pn, pru), sub(pc, prl));
  const float rf = mul(0.5f, add(sub(rc, rrl), sub(rn, rru)));
  const float tend = fma(-dp, idzf, -mul(gravity, rf));
  return fma(dtf, tend, dw);
}
// K15 density from the perturbation mass-flux divergence: max(1e-6, rho - dtf div).
__device__ __forceinline__ float density(float rho, float due, float duw, float dvn, float dvs, float dwt, float dwb,
                                         float idx, float idy, float idzc, float dtf) {
  return fmaxf(1.0e-6f, fma(-dtf, divergence(due, duw, dvn, dvs, dwt, dwb, idx, idy, idzc), rho));
}

// ---- slow tendencies (dry_core.cu:62-187, dry_momentum_flux.cu:79-312,
// dry_pressure_gradient.cu:75-175) ---------------------------------------------------
// Horizontal pressure gradient added to a face tendency: t - (p_r - p_l) inv_d.
__device__ __forceinline__ float add_pgf(float t, float pr, float pl, float inv_d) {
  return fma(-sub(pr, pl), inv_d, t);
}
// The same on terrain: t - ((p_r - p_l) inv_d - dz/dx dp/dz).
__device__ __forceinline__ float add_pgf_terrain(float t, float pr, float pl, float zr, float zl, float dpdz_l,
                                                 float dpdz_r, float inv_d) {
  const float dzdx = mul(sub(zr, zl), inv_d);
  return sub(t, fma(-dzdx, avg(dpdz_l, dpdz_r), mul(sub(pr, pl), inv_d)));
}
// Rayleigh damping of a face tendency (extension): t - rate (q - q_ref).
__device__ __forceinline__ float add_damping(float t, float rate, float q, float qref) {
  return fma(-rate, sub(q, qref), t);
}
// K3 buoyancy at a Z face: t + rho_f g (theta_f - theta_ref_f) / max(theta_ref_f, 1e-6)
// with face means of the two cells and of the two level means.
__device__ __forceinline__ float add_buoyancy(float t, float th_l, float th_u, float tref_l, float tref_u, float rho_l,
                                              float rho_u, float gravity) {
  const float tf = avg(th_l, th_u), trf = avg(tref_l, tref_u);
  const float b = div(mul(gravity, sub(tf, trf)), fmaxf(trf, 1.0e-6f));
  return fma(avg(rho_l, rho_u), b, t);
}

}  // namespace fp
}  // namespace gwmb
