// dycore.cu — sm_100a kernels of the dry dynamics: one fused slow RK stage and
// one fused acoustic substep.
//
// The overlapped-tile kernels share one tiling.  A CTA of BX x R threads owns an
// (BX-2) x (R-2) block of columns plus a one-column ring of halo columns; each
// thread owns one column and marches k = 0..nz-1 keeping k-1, k, k+1 values
// in registers, while the current plane is shared through shared memory for
// the horizontal neighbours.  Halo threads load and derive the same per-column
// quantities (pressure, cell velocities, dp/dz) so interior threads never wait
// on another CTA.  Every owned output is written once, by its owner; values
// that the reference's halo exchange would copy into halo slots are written
// there by the same store (store_mirrored), so no separate halo pass runs.
#include "dycore.cuh"
#include "stencil.cuh"

namespace gwmb {
namespace {

constexpr int BX = 32;

__device__ __forceinline__ float met3(const float* m, const Geom& g, int i, int j, int k) {
  return __ldg(m + gidx(g, i, j, k));
}

// Column values of one plane for the slow stage.
struct SlowCol {
  float rho, rt, th, p, uf, vf, wf;
};
// Raw loads of one plane, issued ahead of use.
struct SlowRaw {
  float rho, t, u, v, w, du, dv, dw, z;
};
// Blend partner (q0) at the thread's own positions.
struct SlowQ0 {
  float rho, rt, u, v, w, wtop;
};

template <bool TERRAIN>
__device__ __forceinline__ SlowRaw slow_raw(const SlowArgs& a, bool valid, int base, int kk) {
  SlowRaw r{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (!valid) return r;
  const int o = base + kk * a.g.plane;
  if (kk < a.g.nz) {
    r.rho = __ldg(a.rho + o);
    r.t = __ldg(a.th + o);
    r.u = __ldg(a.u + o);
    r.v = __ldg(a.v + o);
    if (a.du) { r.du = __ldg(a.du + o); r.dv = __ldg(a.dv + o); }
    if (TERRAIN) r.z = __ldg(a.zc + o);
  }
  if (kk <= a.g.nz) {
    r.w = __ldg(a.w + o);
    if (a.dw) r.dw = __ldg(a.dw + o);
  }
  return r;
}

template <bool TERRAIN>
__device__ __forceinline__ SlowCol slow_derive(const SlowArgs& a, const SlowRaw& r, bool valid, int kk) {
  SlowCol c{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (!valid) return c;
  if (kk < a.g.nz) {
    c.rho = r.rho;
    c.rt = a.th_is_rt ? r.t : fp::mul(c.rho, r.t);
    c.th = fp::theta(c.rho, c.rt);
    c.p = TERRAIN ? eos_pressure(c.rho, c.rt) : eos_pprime(c.rho, c.rt, a.base, kk, a.g.nz);
    c.uf = fp::add(r.u, r.du);
    c.vf = fp::add(r.v, r.dv);
  }
  c.wf = fp::add(r.w, r.dw);
  return c;
}

__device__ __forceinline__ SlowQ0 slow_q0(const SlowArgs& a, int base, int kk, bool own_c, bool own_u,
                                          bool own_v) {
  SlowQ0 q{0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (!a.rho0 || kk >= a.g.nz) return q;
  const int o = base + kk * a.g.plane;
  if (own_c) {
    q.rho = __ldg(a.rho0 + o);
    q.rt = __ldg(a.rt0 + o);
    q.w = __ldg(a.w0 + o);
    if (kk + 1 == a.g.nz) q.wtop = __ldg(a.w0 + o + a.g.plane);
  }
  if (own_u) q.u = __ldg(a.u0 + o);
  if (own_v) q.v = __ldg(a.v0 + o);
  return q;
}

template <bool TERRAIN, int SBY>
__global__ void __launch_bounds__(BX * SBY) k_slow_stage(const SlowArgs a) {
  constexpr int SNT = BX * SBY, SNW = SNT / 32;
  const Geom& g = a.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * BX + tx;
  const int gi = blockIdx.x * (BX - 2) - 1 + tx;
  const int gj = blockIdx.y * (SBY - 2) - 1 + ty;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const bool valid = gi >= -1 && gi <= nx + 1 && gj >= -1 && gj <= ny + 1;
  const bool inner = tx >= 1 && tx <= BX - 2 && ty >= 1 && ty <= SBY - 2;
  const bool own_c = inner && gi >= 0 && gi < nx && gj >= 0 && gj < ny;
  const bool own_u = inner && gi >= 0 && gi <= nx && gj >= 0 && gj < ny;
  const bool own_v = inner && gi >= 0 && gi < nx && gj >= 0 && gj <= ny;
  const bool open_x = !g.per_x, open_y = !g.per_y;
  const int base = valid ? gidx(g, gi, gj, 0) : 0;
  const int ilo = blockIdx.x * (BX - 2), jlo = blockIdx.y * (SBY - 2);
  const bool edge = (g.per_x && (ilo <= 1 || ilo + BX - 3 >= nx - 1)) ||
                    (g.per_y && (jlo <= 1 || jlo + SBY - 3 >= ny - 1));
  const float idx = g.inv_dx, idy = g.inv_dy;

  __shared__ float s_th[2][SBY][BX], s_p[2][SBY][BX], s_u[2][SBY][BX], s_v[2][SBY][BX], s_w[2][SBY][BX];
  __shared__ float s_uc[2][SBY][BX], s_vc[2][SBY][BX], s_wc[2][SBY][BX];
  __shared__ float s_zc[TERRAIN ? 2 : 1][SBY][BX], s_dz[TERRAIN ? 2 : 1][SBY][BX];
  __shared__ float s_thref[kMaxNz];
  __shared__ long long s_red[2][SNW][2];

  if (blockIdx.x == 0 && blockIdx.y == 0 && a.clr_a) {
    for (int q = tid; q < nz; q += SNT) { a.clr_a[q] = 0ull; a.clr_b[q] = 0ull; }
  }
  for (int q = tid; q < nz; q += SNT)
    s_thref[q] = (float)(acc_read(a.th_acc + q, kScaleTheta) * a.inv_count);

  // software pipeline: plane fields two planes ahead, blend partner one plane ahead
  const SlowRaw r0 = slow_raw<TERRAIN>(a, valid, base, 0);
  const SlowRaw r1 = slow_raw<TERRAIN>(a, valid, base, 1);
  SlowRaw r2 = slow_raw<TERRAIN>(a, valid, base, 2);
  SlowQ0 q0c = slow_q0(a, base, 0, own_c, own_u, own_v);
  SlowCol cm{}, cc = slow_derive<TERRAIN>(a, r0, valid, 0), cn = slow_derive<TERRAIN>(a, r1, valid, 1);
  float zm = 0.f, zcc = r0.z, zn = r1.z;
  const bool blend = a.rho0 != nullptr;

  for (int k = 0; k < nz; ++k) {
    const int pb = k & 1;
    const SlowRaw r3 = slow_raw<TERRAIN>(a, valid, base, k + 3);
    const SlowQ0 q0n = slow_q0(a, base, k + 1, own_c, own_u, own_v);
    s_th[pb][ty][tx] = cc.th;
    s_p[pb][ty][tx] = cc.p;
    s_u[pb][ty][tx] = cc.uf;
    s_v[pb][ty][tx] = cc.vf;
    s_w[pb][ty][tx] = cc.wf;
    if (TERRAIN) {
      s_zc[pb][ty][tx] = zcc;
      s_dz[pb][ty][tx] = column_dpdz(k, nz, cm.p, cc.p, cn.p, zm, zcc, zn);
    }
    __syncthreads();
    // level sums of the previous plane (one thread, fixed order)
    if (a.acc_mode && k > 0 && tid == 0) {
      long long sa = 0, sb = 0;
      for (int w = 0; w < SNW; ++w) { sa += s_red[pb ^ 1][w][0]; sb += s_red[pb ^ 1][w][1]; }
      if (a.acc_mode == 1) { acc_add(a.acc_a + k - 1, sa); acc_add(a.acc_b + k - 1, sb); }
      else acc_add(a.acc_a + k - 1, sa);
    }
    // cell-centred velocities of plane k, halo included: dry_momentum_flux.cu:36-73
    {
      const float rr = fmaxf(cc.rho, 1.0e-6f);
      s_uc[pb][ty][tx] = (tx + 1 < BX) ? fp::centred(cc.uf, s_u[pb][ty][tx + 1], rr) : 0.0f;
      s_vc[pb][ty][tx] = (ty + 1 < SBY) ? fp::centred(cc.vf, s_v[pb][ty + 1][tx], rr) : 0.0f;
      s_wc[pb][ty][tx] = fp::centred(cc.wf, cn.wf, rr);
    }
    __syncthreads();

    FxAcc red_a, red_b;
    if (inner && valid) {
      const int o = base + k * g.plane;
      // ---- cell: K2 compute_cell_tendencies_kernel (dry_core.cu:62-144)
      if (own_c) {
        const float fw = cc.uf, fe = s_u[pb][ty][tx + 1], fs = cc.vf, fn = s_v[pb][ty + 1][tx];
        const float fb = cc.wf, ft = cn.wf;
        const float idz = TERRAIN ? met3(a.idz_c, g, gi, gj, k) : __ldg(a.idz_c + k);
        const float t_rho = -fp::divergence(fe, fw, fn, fs, ft, fb, idx, idy, idz);
        const float tc = cc.th;
        const float tw = s_th[pb][ty][tx - 1], te = s_th[pb][ty][tx + 1];
        const float ts = s_th[pb][ty - 1][tx], tn = s_th[pb][ty + 1][tx];
        const float tb = (k > 0) ? cm.th : tc;
        const float tt = (k + 1 < nz) ? cn.th : tc;
        const float gw = fp::upwind(fw, tw, tc), ge = fp::upwind(fe, tc, te);
        const float gs = fp::upwind(fs, ts, tc), gn = fp::upwind(fn, tc, tn);
        const float gb = fp::upwind(fb, tb, tc), gt = fp::upwind(ft, tc, tt);
        const float t_rt = -fp::divergence(ge, gw, gn, gs, gt, gb, idx, idy, idz);
        if (a.tend_only) {
          a.o_rho[o] = t_rho;
          a.o_th[o] = t_rt;
        } else {
          // K4 update (floor 1e-6) and K5 blend
          float r1 = fp::update(cc.rho, a.dt, t_rho, 1.0e-6f);
          float q1 = fp::update(cc.rt, a.dt, t_rt, 1.0e-6f);
          if (blend) {
            r1 = fp::blend(a.wa, q0c.rho, a.wb, r1);
            q1 = fp::blend(a.wa, q0c.rt, a.wb, q1);
          }
          const float th1 = fp::theta(r1, q1);
          store_tile(a.o_rho, g, kCell, gi, gj, k, r1, edge);
          store_tile(a.o_th, g, kCell, gi, gj, k, a.out_rt ? q1 : th1, edge);
          if (a.acc_mode == 1) {
            red_a.add(r1, kFxRho);
            red_b.add(eos_pprime(r1, fp::mul(r1, th1), a.base, k, nz), kFxP);
          } else if (a.acc_mode == 2) {
            red_a.add(th1, kFxTheta);
          }
        }
      }
      // ---- X face: K17 (dry_momentum_flux.cu:79-156) + K21 (dry_pressure_gradient.cu:75-123)
      if (own_u) {
        float t_u = 0.0f;
        if (!((gi == 0 && open_x) || (gi == nx && open_x))) {
          const float qw = s_u[pb][ty][tx - 1], qc = cc.uf, qe = s_u[pb][ty][tx + 1];
          const float qs = s_u[pb][ty - 1][tx], qn = s_u[pb][ty + 1][tx];
          const float qb = (k > 0) ? cm.uf : qc;
          const float qt = (k + 1 < nz) ? cn.uf : qc;
          const float flw = fp::upwind(s_uc[pb][ty][tx - 1], qw, qc);
          const float fle = fp::upwind(s_uc[pb][ty][tx], qc, qe);
          float fls = 0.0f, fln = 0.0f, flb = 0.0f, flt = 0.0f;
          if (!(gj == 0 && open_y)) fls = fp::upwind(fp::avg(s_vc[pb][ty - 1][tx - 1], s_vc[pb][ty - 1][tx]), qs, qc);
          if (!(gj + 1 == ny && open_y)) fln = fp::upwind(fp::avg(s_vc[pb][ty][tx - 1], s_vc[pb][ty][tx]), qc, qn);
          if (k > 0) flb = fp::upwind(fp::avg(s_wc[pb ^ 1][ty][tx - 1], s_wc[pb ^ 1][ty][tx]), qb, qc);
          if (k + 1 < nz) flt = fp::upwind(fp::avg(s_wc[pb][ty][tx - 1], s_wc[pb][ty][tx]), qc, qt);
          const float idz = TERRAIN ? fp::avg(met3(a.idz_c, g, gi - 1, gj, k), met3(a.idz_c, g, gi, gj, k))
                                    : __ldg(a.idz_c + k);
          t_u = -fp::divergence(fle, flw, fln, fls, flt, flb, idx, idy, idz);
          const float pl = s_p[pb][ty][tx - 1], pr = cc.p;
          if (TERRAIN)
            t_u = fp::add_pgf_terrain(t_u, pr, pl, s_zc[pb][ty][tx], s_zc[pb][ty][tx - 1], s_dz[pb][ty][tx - 1],
                                      s_dz[pb][ty][tx], idx);
          else
            t_u = fp::add_pgf(t_u, pr, pl, idx);
          if (a.damp_c) t_u = fp::add_damping(t_u, __ldg(a.damp_c + k), qc, __ldg(a.uref + k));
        }
        if (a.tend_only) {
          a.o_u[o] = t_u;
        } else {
          float u1 = fp::update(cc.uf, a.dt, t_u, -1.0e30f);
          if (blend) u1 = fp::blend(a.wa, q0c.u, a.wb, u1);
          // periodic face nx is written by face 0's mirror store, never read here (the
          // output may be the blend partner's buffer)
          if (!(g.per_x && gi == nx)) store_tile(a.o_u, g, kFaceX, gi, gj, k, u1, edge);
        }
      }
      // ---- Y face: K18 (dry_momentum_flux.cu:158-235) + K22 (dry_pressure_gradient.cu:125-173)
      if (own_v) {
        float t_v = 0.0f;
        if (!((gj == 0 && open_y) || (gj == ny && open_y))) {
          const float qw = s_v[pb][ty][tx - 1], qc = cc.vf, qe = s_v[pb][ty][tx + 1];
          const float qs = s_v[pb][ty - 1][tx], qn = s_v[pb][ty + 1][tx];
          const float qb = (k > 0) ? cm.vf : qc;
          const float qt = (k + 1 < nz) ? cn.vf : qc;
          float flw = 0.0f, fle = 0.0f, flb = 0.0f, flt = 0.0f;
          if (!(gi == 0 && open_x)) flw = fp::upwind(fp::avg(s_uc[pb][ty - 1][tx - 1], s_uc[pb][ty][tx - 1]), qw, qc);
          if (!(gi + 1 == nx && open_x)) fle = fp::upwind(fp::avg(s_uc[pb][ty - 1][tx], s_uc[pb][ty][tx]), qc, qe);
          const float fls = fp::upwind(s_vc[pb][ty - 1][tx], qs, qc);
          const float fln = fp::upwind(s_vc[pb][ty][tx], qc, qn);
          if (k > 0) flb = fp::upwind(fp::avg(s_wc[pb ^ 1][ty - 1][tx], s_wc[pb ^ 1][ty][tx]), qb, qc);
          if (k + 1 < nz) flt = fp::upwind(fp::avg(s_wc[pb][ty - 1][tx], s_wc[pb][ty][tx]), qc, qt);
          const float idz = TERRAIN ? fp::avg(met3(a.idz_c, g, gi, gj - 1, k), met3(a.idz_c, g, gi, gj, k))
                                    : __ldg(a.idz_c + k);
          t_v = -fp::divergence(fle, flw, fln, fls, flt, flb, idx, idy, idz);
          const float ps = s_p[pb][ty - 1][tx], pn = cc.p;
          if (TERRAIN)
            t_v = fp::add_pgf_terrain(t_v, pn, ps, s_zc[pb][ty][tx], s_zc[pb][ty - 1][tx], s_dz[pb][ty - 1][tx],
                                      s_dz[pb][ty][tx], idy);
          else
            t_v = fp::add_pgf(t_v, pn, ps, idy);
          if (a.damp_c) t_v = fp::add_damping(t_v, __ldg(a.damp_c + k), qc, __ldg(a.vref + k));
        }
        if (a.tend_only) {
          a.o_v[o] = t_v;
        } else {
          float v1 = fp::update(cc.vf, a.dt, t_v, -1.0e30f);
          if (blend) v1 = fp::blend(a.wa, q0c.v, a.wb, v1);
          if (!(g.per_y && gj == ny)) store_tile(a.o_v, g, kFaceY, gi, gj, k, v1, edge);
        }
      }
      // ---- Z face k: K19 (dry_momentum_flux.cu:237-312) + K3 buoyancy (dry_core.cu:146-187)
      if (own_c) {
        float t_w = 0.0f;
        if (k > 0) {
          const float qw = s_w[pb][ty][tx - 1], qc = cc.wf, qe = s_w[pb][ty][tx + 1];
          const float qs = s_w[pb][ty - 1][tx], qn = s_w[pb][ty + 1][tx];
          const float qb = cm.wf, qt = cn.wf;
          float flw = 0.0f, fle = 0.0f, fls = 0.0f, fln = 0.0f;
          if (!(gi == 0 && open_x)) flw = fp::upwind(fp::avg(s_uc[pb ^ 1][ty][tx - 1], s_uc[pb][ty][tx - 1]), qw, qc);
          if (!(gi + 1 == nx && open_x)) fle = fp::upwind(fp::avg(s_uc[pb ^ 1][ty][tx], s_uc[pb][ty][tx]), qc, qe);
          if (!(gj == 0 && open_y)) fls = fp::upwind(fp::avg(s_vc[pb ^ 1][ty - 1][tx], s_vc[pb][ty - 1][tx]), qs, qc);
          if (!(gj + 1 == ny && open_y)) fln = fp::upwind(fp::avg(s_vc[pb ^ 1][ty][tx], s_vc[pb][ty][tx]), qc, qn);
          const float flb = fp::upwind(s_wc[pb ^ 1][ty][tx], qb, qc);
          const float flt = fp::upwind(s_wc[pb][ty][tx], qc, qt);
          const float idz = TERRAIN ? met3(a.idz_f, g, gi, gj, k) : __ldg(a.idz_f + k);
          t_w = -fp::divergence(fle, flw, fln, fls, flt, flb, idx, idy, idz);
          t_w = fp::add_buoyancy(t_w, cm.th, cc.th, s_thref[k - 1], s_thref[k], cm.rho, cc.rho, a.gravity);
          if (a.damp_c) t_w = fp::add_damping(t_w, __ldg(a.damp_f + k), qc, 0.0f);
        }
        if (a.tend_only) {
          a.o_w[o] = t_w;
          if (k + 1 == nz) a.o_w[o + g.plane] = 0.0f;
        } else {
          float w1 = fp::update(cc.wf, a.dt, t_w, -1.0e30f);
          if (blend) w1 = fp::blend(a.wa, q0c.w, a.wb, w1);
          store_tile(a.o_w, g, kFaceZ, gi, gj, k, w1, edge);
          if (k + 1 == nz) {  // top face: zero tendency
            float wt = fmaxf(-1.0e30f, cn.wf);
            if (blend) wt = fp::blend(a.wa, q0c.wtop, a.wb, wt);
            store_tile(a.o_w, g, kFaceZ, gi, gj, k + 1, wt, edge);
          }
        }
      }
    }
    if (a.acc_mode) {
      const long long ta = red_a.warp_total(), tb = red_b.warp_total();
      if ((tid & 31) == 0) { s_red[pb][tid >> 5][0] = ta; s_red[pb][tid >> 5][1] = tb; }
    }
    // advance the column window
    cm = cc;
    cc = cn;
    cn = slow_derive<TERRAIN>(a, r2, valid, k + 2);
    zm = zcc;
    zcc = zn;
    zn = r2.z;
    r2 = r3;
    q0c = q0n;
  }
  if (a.acc_mode) {
    __syncthreads();
    if (tid == 0) {
      const int pb = (nz - 1) & 1;
      long long sa = 0, sb = 0;
      for (int w = 0; w < SNW; ++w) { sa += s_red[pb][w][0]; sb += s_red[pb][w][1]; }
      if (a.acc_mode == 1) { acc_add(a.acc_a + nz - 1, sa); acc_add(a.acc_b + nz - 1, sb); }
      else acc_add(a.acc_a + nz - 1, sa);
    }
  }
}

// ---------------------------------------------------------------------------
// Acoustic substep.
struct FastCol {
  float rho, th, thp, p;   // thp: theta recovered from (rho, rho*theta) as the reference does
};
struct FastRaw {
  float rho, th, z;        // plane values loaded ahead of use
};
struct FastInc {
  float du, dv, dw1;       // increments at the plane's own faces (dw1: face k+1)
};

template <bool TERRAIN>
__device__ __forceinline__ FastRaw fast_raw(const FastArgs& a, bool valid, int base, int kk, int gi,
                                            int gj) {
  FastRaw r{0.f, 0.f, 0.f};
  if (!valid || kk >= a.g.nz) return r;
  const int o = base + kk * a.g.plane;
  r.rho = __ldg(a.rho_in + o);
  r.th = __ldg(a.th + o);
  if (TERRAIN) r.z = __ldg(a.zc + o);
  return r;
}

template <bool TERRAIN>
__device__ __forceinline__ FastCol fast_derive(const FastArgs& a, const FastRaw& r, bool valid, int kk) {
  FastCol c{0.f, 0.f, 0.f, 0.f};
  if (!valid || kk >= a.g.nz) return c;
  c.rho = r.rho;
  c.th = r.th;
  const float rt = fp::mul(c.rho, c.th);  // K10 rebuild_rho_theta_from_theta_kernel
  c.thp = fp::theta(c.rho, rt);
  // K20: full pressure for the terrain column reference, perturbation otherwise
  c.p = TERRAIN ? eos_pressure(c.rho, rt) : eos_pprime(c.rho, rt, a.base, kk, a.g.nz);
  return c;
}

// K11 build_column_hydrostatic_reference_kernel (dry_fast_modes.cu:108-158): per column,
// bottom to top, the reference pressure and density the terrain substep takes its
// perturbations about.  A column is a chain of dependent powf evaluations (four
// fixed-point iterations per level), so it runs apart from the substep with every
// column in flight at once; the values are the ones the substep used to build inline
// (one level per call of fp::column_reference_level).
__global__ void __launch_bounds__(128) k_column_reference(const FastArgs a) {
  const Geom& g = a.g;
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 4 + threadIdx.y;
  if (i >= g.nx || j >= g.ny) return;
  const int base = gidx(g, i, j, 0);
  float pref = 0.f, rref = 0.f, zb = 0.f;
  for (int k = 0; k < g.nz; ++k) {
    const int o = base + k * g.plane;
    const float rho = __ldg(a.rho_in + o), th = __ldg(a.th + o), z = __ldg(a.zc + o);
    fp::column_reference_level(k, rho, fp::mul(rho, th), z, a.gravity, pref, rref, zb);
    a.col_pref[o] = pref;
    a.col_rref[o] = rref;
  }
}

template <bool FIRST>
__device__ __forceinline__ FastInc fast_inc(const FastArgs& a, int base, int kk, bool do_u, bool do_v,
                                            bool own_c) {
  FastInc d{0.f, 0.f, 0.f};
  if (FIRST || kk >= a.g.nz) return d;
  const int o = base + kk * a.g.plane;
  if (do_u) d.du = __ldg(a.du_in + o);
  if (do_v) d.dv = __ldg(a.dv_in + o);
  if (own_c && kk + 1 < a.g.nz) d.dw1 = __ldg(a.dw_in + o + a.g.plane);
  return d;
}

template <bool TERRAIN, bool FIRST, int FBY>
__global__ void __launch_bounds__(BX * FBY) k_fast_substep(const FastArgs a) {
  constexpr int FNT = BX * FBY;
  constexpr int FNW = FNT / 32;
  const Geom& g = a.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * BX + tx;
  const int gi = blockIdx.x * (BX - 2) - 1 + tx;
  const int gj = blockIdx.y * (FBY - 2) - 1 + ty;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const bool valid = gi >= -1 && gi <= nx + 1 && gj >= -1 && gj <= ny + 1;
  const bool inner = tx >= 1 && tx <= BX - 2 && ty >= 1 && ty <= FBY - 2;
  const bool own_c = inner && gi >= 0 && gi < nx && gj >= 0 && gj < ny;
  // faces computed by this thread (owned or the tile's far-edge duplicate)
  const bool do_u = tx >= 1 && ty >= 1 && ty <= FBY - 2 && gi >= 0 && gi <= nx && gj >= 0 && gj < ny;
  const bool do_v = ty >= 1 && tx >= 1 && tx <= BX - 2 && gi >= 0 && gi < nx && gj >= 0 && gj <= ny;
  // stored faces: owned ones, except periodic faces nx / ny, which face 0's mirror store
  // writes (in the stand-alone fast modes the step result overwrites the base momenta the
  // substep reads, so face nx must not be read after that store and written again)
  const bool own_u = do_u && tx <= BX - 2 && !(g.per_x && gi == nx);
  const bool own_v = do_v && ty <= FBY - 2 && !(g.per_y && gj == ny);
  const bool skip_u = (gi == 0 || gi == nx) && !g.per_x;
  const bool skip_v = (gj == 0 || gj == ny) && !g.per_y;
  const int base = valid ? gidx(g, gi, gj, 0) : 0;
  const float idx = g.inv_dx, idy = g.inv_dy, dtf = a.dtf;
  const bool final_step = a.final_kind == 2;

  __shared__ float s_p[2][FBY][BX], s_du[2][FBY][BX], s_dv[2][FBY][BX];
  __shared__ float s_zc[TERRAIN ? 2 : 1][FBY][BX], s_dz[TERRAIN ? 2 : 1][FBY][BX];
  __shared__ float s_pref[TERRAIN ? 1 : kMaxNz], s_rref[TERRAIN ? 1 : kMaxNz];
  __shared__ long long s_red[2][FNW][2];

  if (blockIdx.x == 0 && blockIdx.y == 0 && a.clr_a) {
    for (int q = tid; q < nz; q += FNT) { a.clr_a[q] = 0ull; a.clr_b[q] = 0ull; }
  }
  // software pipeline: plane fields two planes ahead, increments one plane ahead
  FastRaw r0 = fast_raw<TERRAIN>(a, valid, base, 0, gi, gj);
  FastRaw r1 = fast_raw<TERRAIN>(a, valid, base, 1, gi, gj);
  FastRaw r2 = fast_raw<TERRAIN>(a, valid, base, 2, gi, gj);
  FastInc d0 = fast_inc<FIRST>(a, base, 0, do_u, do_v, own_c);
  if (!TERRAIN) {  // K6/K7 level means (deterministic sums instead of float atomics)
    for (int q = tid; q < nz; q += FNT) {
      s_rref[q] = (float)(acc_read(a.ref_a + q, kScaleRho) * a.inv_count);
      s_pref[q] = (float)(acc_read(a.ref_b + q, kScaleP) * a.inv_count);
    }
    __syncthreads();
  }
  const int acc_mode = a.acc_off ? 0 : (a.final_kind == 0 ? (TERRAIN ? 0 : 1) : 2);

  float zm = 0.f, zcc = r0.z, zn = r1.z;
  FastCol cm{}, cc = fast_derive<TERRAIN>(a, r0, valid, 0);
  FastCol cn = fast_derive<TERRAIN>(a, r1, valid, 1);
  float dw_c = 0.0f;  // increment at face k (face 0 never changes)
  // terrain: the column reference of the owned column at levels k and k+1
  float pref_c = 0.f, rref_c = 0.f;
  if (TERRAIN && own_c) { pref_c = __ldg(a.col_pref + base); rref_c = __ldg(a.col_rref + base); }

  for (int k = 0; k < nz; ++k) {
    const int pb = k & 1;
    const int o = base + k * g.plane;
    // issue the loads of later planes before any use of this plane
    const FastRaw r3 = fast_raw<TERRAIN>(a, valid, base, k + 3, gi, gj);
    const FastInc d1 = fast_inc<FIRST>(a, base, k + 1, do_u, do_v, own_c);
    float bu0 = 0.f, bv0 = 0.f, bw0 = 0.f, bw1 = 0.f;
    if (final_step) {
      if (own_u) bu0 = __ldg(a.bu + o);
      if (own_v) bv0 = __ldg(a.bv + o);
      if (own_c) { bw1 = __ldg(a.bw + o + g.plane); if (k == 0) bw0 = __ldg(a.bw + o); }
    }
    float pref_n = 0.f, rref_n = 0.f;
    if (TERRAIN && own_c && k + 1 < nz) {
      pref_n = __ldg(a.col_pref + o + g.plane);
      rref_n = __ldg(a.col_rref + o + g.plane);
    }
    float idzf = 0.f, idzc = 0.f;
    if (own_c) {
      idzf = (k + 1 < nz) ? (TERRAIN ? __ldg(a.idz_f + o + g.plane) : __ldg(a.idz_f + k + 1)) : 0.f;
      idzc = TERRAIN ? __ldg(a.idz_c + o) : __ldg(a.idz_c + k);
    }
    s_p[pb][ty][tx] = cc.p;
    if (TERRAIN) {
      s_zc[pb][ty][tx] = zcc;
      s_dz[pb][ty][tx] = column_dpdz(k, nz, cm.p, cc.p, cn.p, zm, zcc, zn);
    }
    __syncthreads();
    if (acc_mode && k > 0 && tid == 0) {
      long long sa = 0, sb = 0;
      for (int w = 0; w < FNW; ++w) { sa += s_red[pb ^ 1][w][0]; sb += s_red[pb ^ 1][w][1]; }
      if (acc_mode == 1) { acc_add(a.acc_a + k - 1, sa); acc_add(a.acc_b + k - 1, sb); }
      else acc_add(a.acc_a + k - 1, sa);
    }
    // K12: X-face momentum (dry_fast_modes.cu:160-229)
    float du_new = d0.du;
    if (do_u && a.hmom && !skip_u) {
      const float pl = s_p[pb][ty][tx - 1], pr = cc.p;
      du_new = TERRAIN ? fp::hmom_terrain(d0.du, pr, pl, s_zc[pb][ty][tx], s_zc[pb][ty][tx - 1], s_dz[pb][ty][tx - 1],
                                          s_dz[pb][ty][tx], idx, dtf)
                       : fp::hmom(d0.du, pr, pl, idx, dtf);
    }
    s_du[pb][ty][tx] = du_new;
    // K13: Y-face momentum (dry_fast_modes.cu:231-301)
    float dv_new = d0.dv;
    if (do_v && a.hmom && !skip_v) {
      const float ps = s_p[pb][ty - 1][tx], pn = cc.p;
      dv_new = TERRAIN ? fp::hmom_terrain(d0.dv, pn, ps, s_zc[pb][ty][tx], s_zc[pb][ty - 1][tx], s_dz[pb][ty - 1][tx],
                                          s_dz[pb][ty][tx], idy, dtf)
                       : fp::hmom(d0.dv, pn, ps, idy, dtf);
    }
    s_dv[pb][ty][tx] = dv_new;
    // K14: Z face k+1 (dry_fast_modes.cu:303-348), perturbations about the reference
    float dw_n = d0.dw1;
    if (own_c && k + 1 < nz) {
      const float prl = TERRAIN ? pref_c : s_pref[k], pru = TERRAIN ? pref_n : s_pref[k + 1];
      const float rrl = TERRAIN ? rref_c : s_rref[k], rru = TERRAIN ? rref_n : s_rref[k + 1];
      dw_n = fp::wmom(d0.dw1, cn.p, pru, cc.p, prl, cc.rho, rrl, cn.rho, rru, idzf, a.gravity, dtf);
    }
    __syncthreads();

    FxAcc red_a, red_b;
    if (own_c) {
      // K15: density from the perturbation mass-flux divergence (dry_fast_modes.cu:350-394)
      float rho_new = cc.rho;
      if (a.dens) {
        rho_new = fp::density(cc.rho, s_du[pb][ty][tx + 1], s_du[pb][ty][tx], s_dv[pb][ty + 1][tx], s_dv[pb][ty][tx],
                              dw_n, dw_c, idx, idy, idzc, dtf);
      }
      const float rt_new = fp::mul(rho_new, cc.th);  // K10 on the state
      if (final_step) {
        store_mirrored(a.f_rho, g, kCell, gi, gj, k, rho_new);
        store_mirrored(a.f_rt, g, kCell, gi, gj, k, rt_new);
        if (k == 0) store_mirrored(a.f_w, g, kFaceZ, gi, gj, 0, bw0);
        store_mirrored(a.f_w, g, kFaceZ, gi, gj, k + 1, fp::add(bw1, dw_n));
      } else {
        store_mirrored(a.rho_out, g, kCell, gi, gj, k, rho_new);
        if (k + 1 < nz) store_mirrored(a.dw_out, g, kFaceZ, gi, gj, k + 1, dw_n);
      }
      if (acc_mode == 1) {
        red_a.add(rho_new, kFxRho);
        red_b.add(eos_pprime(rho_new, rt_new, a.base, k, nz), kFxP);
      } else if (acc_mode == 2) {
        red_a.add(fp::theta(rho_new, rt_new), kFxTheta);
      }
    }
    if (own_u) {
      if (final_step) store_mirrored(a.f_u, g, kFaceX, gi, gj, k, fp::add(bu0, du_new));
      else store_mirrored(a.du_out, g, kFaceX, gi, gj, k, du_new);
    }
    if (own_v) {
      if (final_step) store_mirrored(a.f_v, g, kFaceY, gi, gj, k, fp::add(bv0, dv_new));
      else store_mirrored(a.dv_out, g, kFaceY, gi, gj, k, dv_new);
    }
    if (acc_mode) {
      const long long ta = red_a.warp_total(), tb = red_b.warp_total();
      if ((tid & 31) == 0) { s_red[pb][tid >> 5][0] = ta; s_red[pb][tid >> 5][1] = tb; }
    }
    dw_c = dw_n;
    d0 = d1;
    pref_c = pref_n;
    rref_c = rref_n;
    // advance the column window
    cm = cc;
    cc = cn;
    zm = zcc;
    zcc = zn;
    zn = r2.z;
    cn = fast_derive<TERRAIN>(a, r2, valid, k + 2);
    r2 = r3;
  }
  if (acc_mode) {
    __syncthreads();
    if (tid == 0) {
      const int pb = (nz - 1) & 1;
      long long sa = 0, sb = 0;
      for (int w = 0; w < FNW; ++w) { sa += s_red[pb][w][0]; sb += s_red[pb][w][1]; }
      if (acc_mode == 1) { acc_add(a.acc_a + nz - 1, sa); acc_add(a.acc_b + nz - 1, sb); }
      else acc_add(a.acc_a + nz - 1, sa);
    }
  }
}

// Level sums of a stored (rho, rho*theta) state, one CTA row per level.
__global__ void __launch_bounds__(256) k_level_sums(const LevelSumArgs a) {
  const Geom& g = a.g;
  const int k = blockIdx.y;
  if (blockIdx.x == 0 && k == 0 && a.clr_a)
    for (int q = threadIdx.x; q < g.nz; q += blockDim.x) { a.clr_a[q] = 0ull; a.clr_b[q] = 0ull; }
  __shared__ long long s[8][2];
  long long va = 0, vb = 0;
  const int n = g.nx * g.ny;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int i = q % g.nx, j = q / g.nx;
    const int o = gidx(g, i, j, k);
    const float rho = a.rho[o], rt = a.rt[o];
    if (a.mode == 0) {
      va += fx(theta_of(rho, rt), kFxTheta);
    } else if (a.mode == 2) {  // the field holds theta: the slow stage's theta_of(rho, rho*theta)
      va += fx(theta_of(rho, rho * rt), kFxTheta);
    } else {
      const float rtf = rho * theta_of(rho, rt);
      va += fx(rho, kFxRho);
      vb += fx(eos_pprime(rho, rtf, a.base, k, g.nz), kFxP);
    }
  }
  va = warp_sum_ll(va);
  vb = warp_sum_ll(vb);
  if ((threadIdx.x & 31) == 0) { s[threadIdx.x >> 5][0] = va; s[threadIdx.x >> 5][1] = vb; }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long ta = 0, tb = 0;
    for (int w = 0; w < 8; ++w) { ta += s[w][0]; tb += s[w][1]; }
    acc_add(a.acc_a + k, ta);
    if (a.mode == 1) acc_add(a.acc_b + k, tb);
  }
}


// ---------------------------------------------------------------------------
// Acoustic substep, flat terrain.  Owned tile of 32 x 16 columns per CTA of
// 32 x 8 threads, two columns per thread (rows ty and ty+8) for instruction-level
// parallelism.  The pressure perturbation at the 96 halo cells the tile needs
// (west/east columns, south/north rows; no corners) is derived by 96 threads,
// which also compute the tile's east X faces and north Y faces.  No CTA covers
// X face nx or Y face ny: under periodic wrap they are written as the mirror of
// face 0, on open boundaries they never change.
namespace flat {
constexpr int TX = 32, TY = 16, RY = 8, NT = 256, NW = NT / 32;

struct Cell {
  float rho, th, p;  // density, frozen theta, pressure perturbation
};

__device__ __forceinline__ Cell derive(const FastArgs& a, float rho, float th, int k) {
  Cell c;
  c.rho = rho;
  c.th = th;
  c.p = eos_pprime(rho, fp::mul(rho, th), a.base, k, a.g.nz);  // K10 + K20
  return c;
}
}  // namespace flat

template <bool FIRST>
__global__ void __launch_bounds__(flat::NT, 2) k_fast_flat(const FastArgs a) {
  using flat::TX; using flat::TY; using flat::RY; using flat::Cell; using flat::derive;
  constexpr int FT = flat::NT, FW = flat::NW;
  const Geom& g = a.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int w = min(TX, nx - i0), h = min(TY, ny - j0);
  const bool own0 = tx < w && ty < h, own1 = tx < w && ty + RY < h;
  const int gi = i0 + tx, gj0 = j0 + ty, gj1 = j0 + ty + RY;
  const int b0 = own0 ? gidx(g, gi, gj0, 0) : 0, b1 = own1 ? gidx(g, gi, gj1, 0) : 0;
  const bool skip_u = gi == 0 && !g.per_x;         // open west face (never changes)
  const bool skip_v0 = gj0 == 0 && !g.per_y;
  // tiles away from the periodic edge rings store without mirror checks
  const bool edge = (g.per_x && (i0 <= 1 || i0 + w >= nx - 1)) || (g.per_y && (j0 <= 1 || j0 + h >= ny - 1));
  // halo role: 0 west column, 1 east column, 2 south row, 3 north row.  The 96 halo
  // cells go to threads 0-95, i.e. whole warps 0-2: spreading them over all warps
  // balances the barrier but makes every warp execute the divergent halo path, which
  // costs more issue slots than the barrier wait it saves.
  int role = -1, hi = 0, hj = 0;
  const int hq = tid < 2 * TY + 2 * TX ? tid : -1;
  if (hq >= 0 && hq < TY) { if (hq < h) { role = 0; hi = i0 - 1; hj = j0 + hq; } }
  else if (hq >= TY && hq < 2 * TY) { if (hq - TY < h) { role = 1; hi = i0 + w; hj = j0 + hq - TY; } }
  else if (hq >= 2 * TY && hq < 2 * TY + TX) { if (hq - 2 * TY < w) { role = 2; hi = i0 + hq - 2 * TY; hj = j0 - 1; } }
  else if (hq >= 2 * TY + TX && hq < 2 * TY + 2 * TX) { if (hq - 2 * TY - TX < w) { role = 3; hi = i0 + hq - 2 * TY - TX; hj = j0 + h; } }
  const int hb = role >= 0 ? gidx(g, hi, hj, 0) : 0;
  const int hr = hj - j0 + 1, hc = hi - i0 + 1;    // smem coordinates of the halo cell
  const bool h_skip = (role == 1 && hi == nx && !g.per_x) || (role == 3 && hj == ny && !g.per_y);
  const float idx = g.inv_dx, idy = g.inv_dy, dtf = a.dtf;
  const bool final_step = a.final_kind == 2;
  const int acc_mode = a.acc_off ? 0 : (a.final_kind == 0 ? 1 : 2);
  const int P = g.plane;
  const bool hm = a.hmom != 0, dn = a.dens != 0;

  __shared__ float s_p[2][TY + 2][TX + 2];
  __shared__ float s_du[2][TY][TX + 1];
  __shared__ float s_dv[2][TY + 1][TX];
  __shared__ float s_pref[kMaxNz], s_rref[kMaxNz];
  __shared__ long long s_red[2][FW][2];

  if (blockIdx.x == 0 && blockIdx.y == 0 && a.clr_a)
    for (int q = tid; q < nz; q += FT) { a.clr_a[q] = 0ull; a.clr_b[q] = 0ull; }
  // K6/K7: level means of rho and p' (deterministic sums instead of float atomics)
  for (int q = tid; q < nz; q += FT) {
    s_rref[q] = (float)(acc_read(a.ref_a + q, kScaleRho) * a.inv_count);
    s_pref[q] = (float)(acc_read(a.ref_b + q, kScaleP) * a.inv_count);
  }

  // pipeline: own cells two planes ahead, increments and halo one plane ahead
  auto ld2 = [&](int b, bool own, int kk, float& r, float& t) {
    r = 0.f; t = 0.f;
    if (own && kk < nz) { r = __ldg(a.rho_in + b + kk * P); t = __ldg(a.th + b + kk * P); }
  };
  float ra0, ta0, ra1, ta1;  // raw plane k+2
  ld2(b0, own0, 0, ra0, ta0);
  ld2(b1, own1, 0, ra1, ta1);
  Cell c0 = derive(a, ra0, ta0, 0), c1 = derive(a, ra1, ta1, 0);
  ld2(b0, own0, 1, ra0, ta0);
  ld2(b1, own1, 1, ra1, ta1);
  Cell n0 = derive(a, ra0, ta0, 1), n1 = derive(a, ra1, ta1, 1);
  ld2(b0, own0, 2, ra0, ta0);
  ld2(b1, own1, 2, ra1, ta1);
  // increments of plane k: du, dv at own faces, dw at face k+1
  float du0 = 0.f, dv0 = 0.f, dw0 = 0.f, du1 = 0.f, dv1 = 0.f, dw1 = 0.f;
  if (!FIRST) {
    if (own0) { du0 = __ldg(a.du_in + b0); dv0 = __ldg(a.dv_in + b0); if (nz > 1) dw0 = __ldg(a.dw_in + b0 + P); }
    if (own1) { du1 = __ldg(a.du_in + b1); dv1 = __ldg(a.dv_in + b1); if (nz > 1) dw1 = __ldg(a.dw_in + b1 + P); }
  }
  // halo: p' of plane k and the edge-face increment of plane k
  float hp = 0.f, hd = 0.f;
  if (role >= 0) {
    hp = eos_pprime(__ldg(a.rho_in + hb), fp::mul(__ldg(a.rho_in + hb), __ldg(a.th + hb)), a.base, 0, nz);
    if (!FIRST && role == 1) hd = __ldg(a.du_in + hb);
    if (!FIRST && role == 3) hd = __ldg(a.dv_in + hb);
  }
  // state carried from the faces of plane k to its density update one iteration later
  float pun0 = 0.f, pvn0 = 0.f, pwn0 = 0.f, pwc0 = 0.f, prho0 = 0.f, pth0 = 0.f;
  float pun1 = 0.f, pvn1 = 0.f, pwn1 = 0.f, pwc1 = 0.f, prho1 = 0.f, pth1 = 0.f;
  float pbu0 = 0.f, pbv0 = 0.f, pbw0 = 0.f, pbwz0 = 0.f, pbu1 = 0.f, pbv1 = 0.f, pbw1 = 0.f, pbwz1 = 0.f;
  float pidzc = 0.f;
  float dwc0 = 0.f, dwc1 = 0.f;  // increment at face k (face 0 never changes)
  __syncthreads();

  // K15 density, K10 rho*theta and the stores of plane kk, from the faces computed
  // one iteration earlier (their tiles are published by this iteration's barrier)
  auto finish_plane = [&](int kk, int pbk, FxAcc& sa, FxAcc& sb) {
    if (own0) {
      float rn = prho0;
      if (dn) {
        rn = fp::density(prho0, s_du[pbk][ty][tx + 1], pun0, s_dv[pbk][ty + 1][tx], pvn0, pwn0, pwc0, idx, idy,
                         pidzc, dtf);
      }
      const float rt = fp::mul(rn, pth0);
      if (final_step) {
        store_tile(a.f_rho, g, kCell, gi, gj0, kk, rn, edge);
        store_tile(a.f_rt, g, kCell, gi, gj0, kk, rt, edge);
        store_tile(a.f_u, g, kFaceX, gi, gj0, kk, fp::add(pbu0, pun0), edge);
        store_tile(a.f_v, g, kFaceY, gi, gj0, kk, fp::add(pbv0, pvn0), edge);
        if (kk == 0) store_tile(a.f_w, g, kFaceZ, gi, gj0, 0, pbwz0, edge);
        store_tile(a.f_w, g, kFaceZ, gi, gj0, kk + 1, fp::add(pbw0, pwn0), edge);
      } else {
        store_tile(a.rho_out, g, kCell, gi, gj0, kk, rn, edge);
        store_tile(a.du_out, g, kFaceX, gi, gj0, kk, pun0, edge);
        store_tile(a.dv_out, g, kFaceY, gi, gj0, kk, pvn0, edge);
        if (kk + 1 < nz) store_tile(a.dw_out, g, kFaceZ, gi, gj0, kk + 1, pwn0, edge);
      }
      if (acc_mode == 1) { sa.add(rn, kFxRho); sb.add(eos_pprime(rn, rt, a.base, kk, nz), kFxP); }
      else if (acc_mode == 2) { sa.add(fp::theta(rn, rt), kFxTheta); }
    }
    if (own1) {
      float rn = prho1;
      if (dn) {
        rn = fp::density(prho1, s_du[pbk][ty + RY][tx + 1], pun1, s_dv[pbk][ty + RY + 1][tx], pvn1, pwn1, pwc1, idx,
                         idy, pidzc, dtf);
      }
      const float rt = fp::mul(rn, pth1);
      if (final_step) {
        store_tile(a.f_rho, g, kCell, gi, gj1, kk, rn, edge);
        store_tile(a.f_rt, g, kCell, gi, gj1, kk, rt, edge);
        store_tile(a.f_u, g, kFaceX, gi, gj1, kk, fp::add(pbu1, pun1), edge);
        store_tile(a.f_v, g, kFaceY, gi, gj1, kk, fp::add(pbv1, pvn1), edge);
        if (kk == 0) store_tile(a.f_w, g, kFaceZ, gi, gj1, 0, pbwz1, edge);
        store_tile(a.f_w, g, kFaceZ, gi, gj1, kk + 1, fp::add(pbw1, pwn1), edge);
      } else {
        store_tile(a.rho_out, g, kCell, gi, gj1, kk, rn, edge);
        store_tile(a.du_out, g, kFaceX, gi, gj1, kk, pun1, edge);
        store_tile(a.dv_out, g, kFaceY, gi, gj1, kk, pvn1, edge);
        if (kk + 1 < nz) store_tile(a.dw_out, g, kFaceZ, gi, gj1, kk + 1, pwn1, edge);
      }
      if (acc_mode == 1) { sa.add(rn, kFxRho); sb.add(eos_pprime(rn, rt, a.base, kk, nz), kFxP); }
      else if (acc_mode == 2) { sa.add(fp::theta(rn, rt), kFxTheta); }
    }
  };

  for (int k = 0; k <= nz; ++k) {
    const int pb = k & 1;
    const bool active = k < nz;
    // ---- issue the loads of later planes
    float nr0 = 0.f, nt0 = 0.f, nr1 = 0.f, nt1 = 0.f;
    float ndu0 = 0.f, ndv0 = 0.f, ndw0 = 0.f, ndu1 = 0.f, ndv1 = 0.f, ndw1 = 0.f;
    float hrho = 0.f, hth = 0.f, hdn = 0.f;
    float bu0 = 0.f, bv0 = 0.f, bw0 = 0.f, bu1 = 0.f, bv1 = 0.f, bw1 = 0.f, bwz0 = 0.f, bwz1 = 0.f;
    float idzc = 0.f, idzf = 0.f;
    if (active) {
      ld2(b0, own0, k + 3, nr0, nt0);
      ld2(b1, own1, k + 3, nr1, nt1);
      if (!FIRST && k + 1 < nz) {
        const int o = (k + 1) * P;
        if (own0) { ndu0 = __ldg(a.du_in + b0 + o); ndv0 = __ldg(a.dv_in + b0 + o); if (k + 2 < nz) ndw0 = __ldg(a.dw_in + b0 + o + P); }
        if (own1) { ndu1 = __ldg(a.du_in + b1 + o); ndv1 = __ldg(a.dv_in + b1 + o); if (k + 2 < nz) ndw1 = __ldg(a.dw_in + b1 + o + P); }
      }
      if (role >= 0 && k + 1 < nz) {
        const int o = hb + (k + 1) * P;
        hrho = __ldg(a.rho_in + o);
        hth = __ldg(a.th + o);
        if (!FIRST && role == 1) hdn = __ldg(a.du_in + o);
        if (!FIRST && role == 3) hdn = __ldg(a.dv_in + o);
      }
      if (final_step) {
        const int o = k * P;
        if (own0) { bu0 = __ldg(a.bu + b0 + o); bv0 = __ldg(a.bv + b0 + o); bw0 = __ldg(a.bw + b0 + o + P); if (k == 0) bwz0 = __ldg(a.bw + b0); }
        if (own1) { bu1 = __ldg(a.bu + b1 + o); bv1 = __ldg(a.bv + b1 + o); bw1 = __ldg(a.bw + b1 + o + P); if (k == 0) bwz1 = __ldg(a.bw + b1); }
      }
      idzc = __ldg(a.idz_c + k);
      idzf = (k + 1 < nz) ? __ldg(a.idz_f + k + 1) : 0.f;
      // ---- plane k pressure perturbation into shared memory (owners and halo only:
      // on partial edge tiles the slot next to the last owned column/row is a halo slot)
      if (own0) s_p[pb][ty + 1][tx + 1] = c0.p;
      if (own1) s_p[pb][ty + RY + 1][tx + 1] = c1.p;
      if (role >= 0) s_p[pb][hr][hc] = hp;
    }
    __syncthreads();
    // ---- plane k-1: density update and stores (its face tiles are now published)
    if (k > 0) {
      FxAcc sa, sb;
      finish_plane(k - 1, pb ^ 1, sa, sb);
      if (acc_mode) {
        const long long wa = sa.warp_total(), wb = sb.warp_total();
        if (tx == 0) { s_red[pb ^ 1][ty][0] = wa; s_red[pb ^ 1][ty][1] = wb; }
      }
    }
    // level sums of plane k-2, whose warp partials the previous barrier published
    if (acc_mode && k > 1 && tid == 0) {
      long long sa = 0, sb = 0;
      for (int q = 0; q < FW; ++q) { sa += s_red[pb][q][0]; sb += s_red[pb][q][1]; }
      if (acc_mode == 1) { acc_add(a.acc_a + k - 2, sa); acc_add(a.acc_b + k - 2, sb); }
      else acc_add(a.acc_a + k - 2, sa);
    }
    if (!active) break;
    // ---- plane k faces: K12/K13 horizontal momenta, K14 vertical momentum at face k+1
    float un0 = du0, vn0 = dv0, un1 = du1, vn1 = dv1;
    if (hm) {
      if (!skip_u) {
        un0 = fp::hmom(du0, c0.p, s_p[pb][ty + 1][tx], idx, dtf);
        un1 = fp::hmom(du1, c1.p, s_p[pb][ty + RY + 1][tx], idx, dtf);
      }
      if (!skip_v0) vn0 = fp::hmom(dv0, c0.p, s_p[pb][ty][tx + 1], idy, dtf);
      vn1 = fp::hmom(dv1, c1.p, s_p[pb][ty + RY][tx + 1], idy, dtf);
    }
    if (own0) { s_du[pb][ty][tx] = un0; s_dv[pb][ty][tx] = vn0; }
    if (own1) { s_du[pb][ty + RY][tx] = un1; s_dv[pb][ty + RY][tx] = vn1; }
    if (role == 1) {  // tile's east X face
      float d = hd;
      if (hm && !h_skip) d = fp::hmom(hd, hp, s_p[pb][hr][hc - 1], idx, dtf);
      s_du[pb][hr - 1][hc - 1] = d;
      // open east boundary: face nx belongs to no tile; its step value is base + 0
      if (final_step && h_skip) a.f_u[hb + k * P] = fp::add(__ldg(a.bu + hb + k * P), d);
    } else if (role == 3) {  // tile's north Y face
      float d = hd;
      if (hm && !h_skip) d = fp::hmom(hd, hp, s_p[pb][hr - 1][hc], idy, dtf);
      s_dv[pb][hr - 1][hc - 1] = d;
      if (final_step && h_skip) a.f_v[hb + k * P] = fp::add(__ldg(a.bv + hb + k * P), d);
    }
    float wn0 = dw0, wn1 = dw1;
    if (k + 1 < nz) {
      const float prl = s_pref[k], pru = s_pref[k + 1], rrl = s_rref[k], rru = s_rref[k + 1];
      wn0 = fp::wmom(dw0, n0.p, pru, c0.p, prl, c0.rho, rrl, n0.rho, rru, idzf, a.gravity, dtf);
      wn1 = fp::wmom(dw1, n1.p, pru, c1.p, prl, c1.rho, rrl, n1.rho, rru, idzf, a.gravity, dtf);
    }
    // ---- hand plane k to the next iteration's density update, advance the pipeline
    pun0 = un0; pvn0 = vn0; pwn0 = wn0; pwc0 = dwc0; prho0 = c0.rho; pth0 = c0.th;
    pun1 = un1; pvn1 = vn1; pwn1 = wn1; pwc1 = dwc1; prho1 = c1.rho; pth1 = c1.th;
    pbu0 = bu0; pbv0 = bv0; pbw0 = bw0; pbwz0 = bwz0; pbu1 = bu1; pbv1 = bv1; pbw1 = bw1; pbwz1 = bwz1;
    pidzc = idzc;
    dwc0 = wn0; dwc1 = wn1;
    c0 = n0; c1 = n1;
    n0 = derive(a, ra0, ta0, k + 2 < nz ? k + 2 : 0);
    n1 = derive(a, ra1, ta1, k + 2 < nz ? k + 2 : 0);
    ra0 = nr0; ta0 = nt0; ra1 = nr1; ta1 = nt1;
    du0 = ndu0; dv0 = ndv0; dw0 = ndw0; du1 = ndu1; dv1 = ndv1; dw1 = ndw1;
    if (role >= 0 && k + 1 < nz) {
      hp = eos_pprime(hrho, fp::mul(hrho, hth), a.base, k + 1, nz);
      hd = hdn;
    }
  }
  // level sums of the last plane
  if (acc_mode) {
    __syncthreads();
    if (tid == 0) {
      const int pb = (nz - 1) & 1;
      long long sa = 0, sb = 0;
      for (int q = 0; q < FW; ++q) { sa += s_red[pb][q][0]; sb += s_red[pb][q][1]; }
      if (acc_mode == 1) { acc_add(a.acc_a + nz - 1, sa); acc_add(a.acc_b + nz - 1, sb); }
      else acc_add(a.acc_a + nz - 1, sa);
    }
  }
}

// Per-level mean of rho_theta (FP64, fixed order) and the EOS of that mean.
__global__ void __launch_bounds__(256) k_base_state(const Geom g, const float* rt, double* base) {
  const int k = blockIdx.x;
  __shared__ double sh[8];
  double v = 0.0;
  const int n = g.nx * g.ny;
  for (int q = threadIdx.x; q < n; q += blockDim.x) {
    const int i = q % g.nx, j = q / g.nx;
    v += (double)rt[gidx(g, i, j, k)];
  }
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += sh[w];
    const double rt_ref = t / (double)n;
    const double gamma = (double)(1.0f / (1.0f - kKappa));
    base[k] = rt_ref;
    base[g.nz + k] = 1.0 / rt_ref;
    base[2 * g.nz + k] = (double)kP0 * pow((double)kRd * rt_ref / (double)kP0, gamma);
  }
}

__global__ void k_theta_field(const Geom g, const float* rho, const float* rt, float* th) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n;
       q += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(q % g.nx);
    const long long r = q / g.nx;
    const int j = (int)(r % g.ny), k = (int)(r / g.ny);
    const int o = gidx(g, i, j, k);
    store_mirrored(th, g, kCell, i, j, k, theta_of(rho[o], rt[o]));
  }
}

}  // namespace

template <int SBY>
cudaError_t launch_slow_tile(const SlowArgs& a, bool terrain, cudaStream_t s) {
  const dim3 block(BX, SBY);
  const dim3 grid((a.g.nx + 1 + BX - 3) / (BX - 2), (a.g.ny + 1 + SBY - 3) / (SBY - 2));
  if (terrain) k_slow_stage<true, SBY><<<grid, block, 0, s>>>(a);
  else k_slow_stage<false, SBY><<<grid, block, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_slow(const SlowArgs& a, bool terrain, cudaStream_t s, int tile_rows) {
  if (a.g.nz > kMaxNz) return cudaErrorInvalidValue;
  if (tile_rows == 16) return launch_slow_tile<16>(a, terrain, s);
  return launch_slow_tile<8>(a, terrain, s);
}

template <int FBY>
cudaError_t launch_fast_tile(const FastArgs& a, bool first, bool terrain, cudaStream_t s) {
  const dim3 block(BX, FBY);
  const dim3 grid((a.g.nx + 1 + BX - 3) / (BX - 2), (a.g.ny + 1 + FBY - 3) / (FBY - 2));
  if (terrain) {
    if (first) k_fast_substep<true, true, FBY><<<grid, block, 0, s>>>(a);
    else k_fast_substep<true, false, FBY><<<grid, block, 0, s>>>(a);
  } else {
    if (first) k_fast_substep<false, true, FBY><<<grid, block, 0, s>>>(a);
    else k_fast_substep<false, false, FBY><<<grid, block, 0, s>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t launch_fast(const FastArgs& a, bool first, bool terrain, cudaStream_t s, int tile_rows) {
  if (a.g.nz > kMaxNz) return cudaErrorInvalidValue;
  if (!terrain && tile_rows == 0) {  // flat-terrain kernel with owned 32 x 16 tiles
    const dim3 block(flat::TX, flat::RY);
    const dim3 grid((a.g.nx + flat::TX - 1) / flat::TX, (a.g.ny + flat::TY - 1) / flat::TY);
    if (first) k_fast_flat<true><<<grid, block, 0, s>>>(a);
    else k_fast_flat<false><<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
  }
  if (tile_rows == 16) return launch_fast_tile<16>(a, first, terrain, s);
  return launch_fast_tile<8>(a, first, terrain, s);
}

cudaError_t launch_column_reference(const FastArgs& a, cudaStream_t s) {
  if (!a.col_pref || !a.col_rref || !a.zc || a.g.nx <= 0 || a.g.ny <= 0) return cudaErrorInvalidValue;
  const dim3 block(32, 4), grid((a.g.nx + 31) / 32, (a.g.ny + 3) / 4);
  k_column_reference<<<grid, block, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_level_sums(const LevelSumArgs& a, cudaStream_t s) {
  const int n = a.g.nx * a.g.ny;
  const int bx = (n + 255) / 256 < 64 ? (n + 255) / 256 : 64;
  k_level_sums<<<dim3(bx, a.g.nz), 256, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_base_state(const Geom& g, const float* rt, double* base, cudaStream_t s) {
  k_base_state<<<g.nz, 256, 0, s>>>(g, rt, base);
  return cudaGetLastError();
}

cudaError_t launch_theta_field(const Geom& g, const float* rho, const float* rt, float* th,
                               cudaStream_t s) {
  const long long n = (long long)g.nx * g.ny * g.nz;
  long long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  k_theta_field<<<(int)b, 256, 0, s>>>(g, rho, rt, th);
  return cudaGetLastError();
}

}  // namespace gwmb
