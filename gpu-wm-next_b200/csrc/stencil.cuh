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
//
// Scalar FP32 on purpose: a variant of the TMA slow stage that ran a thread's two cells
// through the packed FP32 instructions (two results per instruction) was 6.6 % faster but
// differed from the one-cell kernels by one ulp in rare cells (one ρθ value in 84,000
// cells per stage on a moist 100 x 70 x 12 case), which breaks the bit-for-bit agreement
// of the tilings.  The formulas stay templates on the value type V.
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace gwmb {
namespace fp {

// ---- primitives ---------------------------------------------------------------------
__device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float neg(float a) { return -a; }
__device__ __forceinline__ float vmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ float select_ge0(float a, float x, float y) { return a >= 0.0f ? x : y; }
__device__ __forceinline__ float splat(float s, float) { return s; }

// scalar operand broadcast to V
template <class V> __device__ __forceinline__ V sc(float s) { return splat(s, V{}); }

// ---- shared formulas ------------------------------------------------------------------
// 0.5 (a + b)
template <class V> __device__ __forceinline__ V avg(V a, V b) { return mul(sc<V>(0.5f), add(a, b)); }

// First-order upwind flux a * (a >= 0 ? q_upstream_low : q_upstream_high)
// (dry_core.cu:98-120, dry_momentum_flux.cu:79-312, dry_transport.cu:91-114).
template <class V> __device__ __forceinline__ V upwind(V a, V ql, V qr) { return mul(a, select_ge0(a, ql, qr)); }

// Divergence (e - w) idx + (n - s) idy + (t - b) idz of face values or fluxes.
template <class V>
__device__ __forceinline__ V divergence(V e, V w, V n, V s, V t, V b, float idx, float idy, float idz) {
  return fma(sub(t, b), sc<V>(idz), fma(sub(n, s), sc<V>(idy), mul(sub(e, w), sc<V>(idx))));
}

// K4 stage update with a floor (dry_core.cu:189-197): max(lo, q + dt tend).
template <class V> __device__ __forceinline__ V update(V q, float dt, V tend, float lo) {
  return vmax(sc<V>(lo), fma(sc<V>(dt), tend, q));
}

// K5 blend (dry_core.cu:199-205, dry_transport.cu:40-47): wa q0 + wb q.
template <class V> __device__ __forceinline__ V blend(float wa, V q0, float wb, V q) {
  return fma(sc<V>(wa), q0, mul(sc<V>(wb), q));
}

// theta = rho_theta / max(rho, 1e-6) (include/gwm/core/dry_thermo.hpp:21-24).
template <class V> __device__ __forceinline__ V theta(V rho, V rt) { return div(rt, vmax(rho, sc<V>(1.0e-6f))); }

// Cell-centred velocity 0.5 (m_a + m_b) / max(rho, 1e-6) (dry_momentum_flux.cu:36-73).
template <class V> __device__ __forceinline__ V centred(V ma, V mb, V rr) { return div(avg(ma, mb), rr); }

// ---- acoustic substep (dry_fast_modes.cu:160-394) --------------------------------
// K12/K13 horizontal momentum increment on flat levels: d - dtf (p_r - p_l) inv_d.
template <class V> __device__ __forceinline__ V hmom(V d, V pr, V pl, float inv_d, float dtf) {
  return fma(sc<V>(-dtf), mul(sub(pr, pl), sc<V>(inv_d)), d);
}
// K12/K13 on terrain: the chain-rule gradient (p_r - p_l) inv_d - dz/dx dp/dz
// (dry_fast_modes.cu:160-301, docs/math/terrain_metric_operators.md:7-14).
template <class V>
__device__ __forceinline__ V hmom_terrain(V d, V pr, V pl, V zr, V zl, V dpdz_l, V dpdz_r, float inv_d, float dtf) {
  const V dzdx = mul(sub(zr, zl), sc<V>(inv_d));
  const V x = fma(neg(dzdx), avg(dpdz_l, dpdz_r), mul(sub(pr, pl), sc<V>(inv_d)));
  return fma(sc<V>(-dtf), x, d);
}
// K14 vertical momentum increment at a face: dw + dtf (-(p'_u - p'_l) idzf - g rho'_f),
// with p'_u = pn - pru, p'_l = pc - prl and rho'_f = 0.5 ((rc - rrl) + (rn - rru)).
template <class V>
__device__ __forceinline__ V wmom(V dw, V pn, V pru, V pc, V prl, V rc, V rrl, V rn, V rru, float idzf, float gravity,
                                  float dtf) {
  const V dp = sub(sub(pn, pru), sub(pc, prl));
  const V rf = mul(sc<V>(0.5f), add(sub(rc, rrl), sub(rn, rru)));
  const V tend = fma(neg(dp), sc<V>(idzf), neg(mul(sc<V>(gravity), rf)));
  return fma(sc<V>(dtf), tend, dw);
}
// K15 density from the perturbation mass-flux divergence: max(1e-6, rho - dtf div).
template <class V>
__device__ __forceinline__ V density(V rho, V due, V duw, V dvn, V dvs, V dwt, V dwb, float idx, float idy, float idzc,
                                     float dtf) {
  return vmax(sc<V>(1.0e-6f), fma(sc<V>(-dtf), divergence(due, duw, dvn, dvs, dwt, dwb, idx, idy, idzc), rho));
}

// ---- slow tendencies (dry_core.cu:62-187, dry_momentum_flux.cu:79-312,
// dry_pressure_gradient.cu:75-175) ---------------------------------------------------
// Horizontal pressure gradient added to a face tendency: t - (p_r - p_l) inv_d.
template <class V> __device__ __forceinline__ V add_pgf(V t, V pr, V pl, float inv_d) {
  return fma(neg(sub(pr, pl)), sc<V>(inv_d), t);
}
// The same on terrain: t - ((p_r - p_l) inv_d - dz/dx dp/dz).
template <class V>
__device__ __forceinline__ V add_pgf_terrain(V t, V pr, V pl, V zr, V zl, V dpdz_l, V dpdz_r, float inv_d) {
  const V dzdx = mul(sub(zr, zl), sc<V>(inv_d));
  return sub(t, fma(neg(dzdx), avg(dpdz_l, dpdz_r), mul(sub(pr, pl), sc<V>(inv_d))));
}
// Rayleigh damping of a face tendency (extension): t - rate (q - q_ref).
template <class V> __device__ __forceinline__ V add_damping(V t, float rate, V q, float qref) {
  return fma(sc<V>(-rate), sub(q, sc<V>(qref)), t);
}
// K3 buoyancy at a Z face: t + rho_f g (theta_f - theta_ref_f) / max(theta_ref_f, 1e-6)
// with face means of the two cells and of the two level means.
template <class V>
__device__ __forceinline__ V add_buoyancy(V t, V th_l, V th_u, float tref_l, float tref_u, V rho_l, V rho_u,
                                          float gravity) {
  const float trf = __fmul_rn(0.5f, __fadd_rn(tref_l, tref_u));
  const V tf = avg(th_l, th_u);
  const V b = div(mul(sc<V>(gravity), sub(tf, sc<V>(trf))), sc<V>(fmaxf(trf, 1.0e-6f)));
  return fma(avg(rho_l, rho_u), b, t);
}

// K11 build_column_hydrostatic_reference_kernel (dry_fast_modes.cu:108-158), one level of
// a column, bottom to top: the reference pressure and density at level k from the cell's
// rho, rho*theta and height z, given those of the level below (pref, rref at height zb);
// updates pref, rref and zb.  Four fixed-point iterations, then the density of the result.
// An iteration that returns its own input is a fixed point that every later iteration
// repeats, and the final density is then the one just evaluated, so the loop stops there
// with the same result (the iterations contract by about g dz / (2 c^2) ~ 1e-2).
__device__ __forceinline__ void column_reference_level(int k, float rho, float rt, float z, float gravity,
                                                       float& pref, float& rref, float& zb) {
  const float thp = theta(rho, rt);
  if (k == 0) {
    pref = eos_pressure(rho, rt);
    rref = eos_rho(pref, thp);
  } else {
    const float dzk = z - zb;
    float pn = fmaxf(1.0f, fma(-mul(gravity, rref), dzk, pref));
    float rn = 0.0f;
    bool fixed = false;
    for (int it = 0; it < 4; ++it) {
      rn = eos_rho(pn, thp);
      const float pq = fmaxf(fma(-mul(mul(gravity, 0.5f), add(rref, rn)), dzk, pref), 1.0f);
      if (pq == pn) {
        fixed = true;
        break;
      }
      pn = pq;
    }
    pref = pn;
    rref = fixed ? rn : eos_rho(pn, thp);
  }
  zb = z;
}

}  // namespace fp
}  // namespace gwmb
