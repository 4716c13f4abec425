// physics.cu — sm_100a kernels for the moist part of the step: the fused
// three-tracer SSPRK3 stage and the warm-rain column kernel.
#include "dycore.cuh"
#include "physics.cuh"
#include "stencil.cuh"
#include "rain_cell.cuh"

namespace gwmb {
namespace {

constexpr int BX = 32;
constexpr int NTR = 3;

struct TrCol {
  float rho, uf, vf, wf;
  float rq[NTR], q[NTR];
};

__device__ __forceinline__ TrCol tr_load(const TracerArgs& a, bool valid, int base, int kk) {
  TrCol c{};
  if (!valid) return c;
  const int o = base + kk * a.g.plane;
  if (kk < a.g.nz) {
    c.rho = __ldg(a.rho + o);
    c.uf = __ldg(a.u + o);
    c.vf = __ldg(a.v + o);
#pragma unroll
    for (int t = 0; t < NTR; ++t)
      if (t < a.ntracers) c.rq[t] = __ldg(a.q_in[t] + o);
  }
  if (kk <= a.g.nz) c.wf = __ldg(a.w + o);
  return c;
}

__device__ __forceinline__ void tr_mix(TrCol& c) {
  const float rr = fmaxf(c.rho, 1.0e-6f);
#pragma unroll
  for (int t = 0; t < NTR; ++t) c.q[t] = c.rq[t] / rr;  // mixing ratio: dry_transport.cu:91-94
}

template <int TBY>
__global__ void __launch_bounds__(BX * TBY) k_tracer_stage(const TracerArgs a) {
  const Geom& g = a.g;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int gi = blockIdx.x * (BX - 2) - 1 + tx;
  const int gj = blockIdx.y * (TBY - 2) - 1 + ty;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const bool valid = gi >= -1 && gi <= nx + 1 && gj >= -1 && gj <= ny + 1;
  const bool inner = tx >= 1 && tx <= BX - 2 && ty >= 1 && ty <= TBY - 2;
  const bool own_c = inner && gi >= 0 && gi < nx && gj >= 0 && gj < ny;
  const int base = valid ? gidx(g, gi, gj, 0) : 0;
  const int ilo = blockIdx.x * (BX - 2), jlo = blockIdx.y * (TBY - 2);
  const bool edge = (g.per_x && (ilo <= 1 || ilo + BX - 3 >= nx - 1)) ||
                    (g.per_y && (jlo <= 1 || jlo + TBY - 3 >= ny - 1));
  const float idx = g.inv_dx, idy = g.inv_dy;
  const bool blend = a.q0[0] != nullptr;

  __shared__ float s_q[NTR][2][TBY][BX];
  __shared__ float s_u[2][TBY][BX], s_v[2][TBY][BX];

  TrCol cm{}, cc = tr_load(a, valid, base, 0), cn = tr_load(a, valid, base, 1);
  TrCol c2 = tr_load(a, valid, base, 2);
  tr_mix(cc);
  tr_mix(cn);
  for (int k = 0; k < nz; ++k) {
    const int pb = k & 1;
    const TrCol c3 = tr_load(a, valid, base, k + 3);
    float q0v[NTR] = {0.f, 0.f, 0.f};
    const int o = base + k * g.plane;
    if (own_c && blend) {
#pragma unroll
      for (int t = 0; t < NTR; ++t)
        if (t < a.ntracers) q0v[t] = __ldg(a.q0[t] + o);
    }
    const float idz = own_c ? (a.terrain ? __ldg(a.idz_c + o) : __ldg(a.idz_c + k)) : 0.f;
#pragma unroll
    for (int t = 0; t < NTR; ++t) s_q[t][pb][ty][tx] = cc.q[t];
    s_u[pb][ty][tx] = cc.uf;
    s_v[pb][ty][tx] = cc.vf;
    __syncthreads();
    if (own_c) {
      const float fw = cc.uf, fe = s_u[pb][ty][tx + 1], fs = cc.vf, fn = s_v[pb][ty + 1][tx];
      const float fb = cc.wf, ft = cn.wf;
#pragma unroll
      for (int t = 0; t < NTR; ++t) {
        if (t >= a.ntracers) break;
        const float qc = cc.q[t];
        const float qw = s_q[t][pb][ty][tx - 1], qe = s_q[t][pb][ty][tx + 1];
        const float qs = s_q[t][pb][ty - 1][tx], qn = s_q[t][pb][ty + 1][tx];
        const float qb = (k > 0) ? cm.q[t] : qc;
        const float qt = (k + 1 < nz) ? cn.q[t] : qc;
        const float gw = fp::upwind(fw, qw, qc), ge = fp::upwind(fe, qc, qe);
        const float gs = fp::upwind(fs, qs, qc), gn = fp::upwind(fn, qc, qn);
        const float gb = fp::upwind(fb, qb, qc), gt = fp::upwind(ft, qc, qt);
        const float div = fp::divergence(ge, gw, gn, gs, gt, gb, idx, idy, idz);
        float out = fp::update(cc.rq[t], -a.dt, div, 0.0f);
        if (blend) out = fp::blend(a.wa, q0v[t], a.wb, out);
        store_tile(a.q_out[t], g, kCell, gi, gj, k, out, edge);
      }
    }
    cm = cc;
    cc = cn;
    cn = c2;
    tr_mix(cn);
    c2 = c3;
  }
}


constexpr int RB = 128;  // columns per warm-rain block (one row segment)

// MICRO = false: fallout only, on a state whose microphysics was already applied
// (the surrogate's network kernel); the reference applies each cell's microphysics
// before the rain from above arrives, so the split is exact.
template <bool MICRO>
__global__ void __launch_bounds__(RB) k_warm_rain(const RainArgs a) {
  const Geom& g = a.g;
  const int gi = blockIdx.x * RB + threadIdx.x;
  const int gj = blockIdx.y;
  const bool active = gi < g.nx && gj < g.ny;
  const int ilo = blockIdx.x * RB;
  const bool edge = (g.per_x && (ilo <= 1 || ilo + RB - 1 >= g.nx - 1)) ||
                    (g.per_y && (gj <= 1 || gj >= g.ny - 1));
  __shared__ long long s_th[kMaxNz][RB / 32];
  float incoming = 0.0f;
  // one-cell-ahead prefetch down the column
  float n_rho = 0.f, n_rt = 0.f, n_qv = 0.f, n_qc = 0.f, n_qr = 0.f;
  const bool need_rt = MICRO || a.th_acc;
  if (active) {
    const int o = gidx(g, gi, gj, g.nz - 1);
    n_rho = __ldg(a.rho + o); n_qr = a.qr[o];
    if (need_rt) n_rt = a.rt[o];
    if (MICRO) { n_qv = a.qv[o]; n_qc = a.qc[o]; }
  }
  for (int k = g.nz - 1; k >= 0; --k) {
    FxAcc th_sum;
    const float c_rho = n_rho, c_rt = n_rt, c_qv = n_qv, c_qc = n_qc, c_qr = n_qr;
    if (active && k > 0) {
      const int o1 = gidx(g, gi, gj, k - 1);
      n_rho = __ldg(a.rho + o1); n_qr = a.qr[o1];
      if (need_rt) n_rt = a.rt[o1];
      if (MICRO) { n_qv = a.qv[o1]; n_qc = a.qc[o1]; }
    }
    if (active) {
      const int o = gidx(g, gi, gj, k);
      const float rho_d = c_rho;
      float rho = 0.0f, th = 0.0f, qv = 0.0f, qc = 0.0f, rqr = c_qr;
      if (MICRO) {  // warm_rain_kernel: warm_rain.cu:36-120
        MicroCell mc;
        if (a.thr >= 0.0f && surely_quiet(rho_d, c_rt, c_qv, c_qc, c_qr)) {
          // micro_step leaves the cell as micro_state derives it: only the mixing ratios
          // and theta are needed, not the temperature, pressure or saturation
          mc.rho = fmaxf(rho_d, 1.0e-6f);
          mc.th = c_rt / mc.rho;
          mc.qv = fmaxf(c_qv / mc.rho, 0.0f);
          mc.qc = fmaxf(c_qc / mc.rho, 0.0f);
          mc.qr = fmaxf(c_qr / mc.rho, 0.0f);
        } else {
          mc = micro_state(rho_d, c_rt, c_qv, c_qc, c_qr);
          micro_step(mc, MicroParams{a.dt, a.relax, a.thr, a.rate, a.evap, a.latent});
        }
        rho = mc.rho; th = mc.th; qv = mc.qv; qc = mc.qc;
        rqr = rho * mc.qr;
      }
      // fallout of this cell, fed by the cell above
      if (a.fallout_mode == 1) {  // rain_fallout_metric_kernel: warm_rain.cu:156-191
        const float idz = fmaxf(a.terrain ? __ldg(a.idz_c + o) : __ldg(a.idz_c + k), 1.0e-6f);
        const float dz = 1.0f / idz;
        const float frac = fminf(fmaxf(a.vt * a.dt * idz, 0.0f), 1.0f);
        const float old_a = fmaxf(rqr, 0.0f) * dz;
        const float out = frac * old_a;
        rqr = ((old_a - out) + incoming) * idz;
        incoming = out;
      } else if (a.fallout_mode == 2) {  // rain_fallout_nominal_kernel: warm_rain.cu:122-154
        const float dz = fmaxf(a.layer_depth, 1.0e-3f);
        const float frac = fminf(fmaxf(a.vt * a.dt / dz, 0.0f), 1.0f);
        if (frac > 0.0f) {
          const float old_a = fmaxf(rqr, 0.0f) * dz;
          const float out = frac * old_a;
          rqr = ((old_a - out) + incoming) / dz;
          incoming = out;
        }
      }
      const float rt_new = MICRO ? rho * th : c_rt;
      if (MICRO) {
        store_tile(a.qv, g, kCell, gi, gj, k, rho * qv, edge);
        store_tile(a.qc, g, kCell, gi, gj, k, rho * qc, edge);
        store_tile(a.rt, g, kCell, gi, gj, k, rt_new, edge);
      }
      if (MICRO || a.fallout_mode) store_tile(a.qr, g, kCell, gi, gj, k, rqr, edge);
      if (a.th_acc) th_sum.add(theta_of(rho_d, rt_new), kFxTheta);
    }
    if (a.th_acc) {
      const long long t = th_sum.warp_total();
      if ((threadIdx.x & 31) == 0) s_th[k][threadIdx.x >> 5] = t;
    }
  }
  if (active && a.fallout_mode && a.precip) {  // compensated FP64 surface accumulation
    const int q = gj * g.nx + gi;
    const double s = a.precip[q], x = (double)incoming, t = s + x;
    a.precip_comp[q] += (fabs(s) >= fabs(x)) ? (s - t) + x : (x - t) + s;
    a.precip[q] = t;
  }
  if (a.th_acc) {
    __syncthreads();
    for (int k = threadIdx.x; k < g.nz; k += RB) {
      long long t = 0;
      for (int w = 0; w < RB / 32; ++w) t += s_th[k][w];
      acc_add(a.th_acc + k, t);
    }
  }
}

}  // namespace

cudaError_t launch_tracer_stage(const TracerArgs& a, cudaStream_t s, int tile_rows) {
  if (tile_rows == 16) {
    const dim3 grid((a.g.nx + BX - 3) / (BX - 2), (a.g.ny + 16 - 3) / (16 - 2));
    k_tracer_stage<16><<<grid, dim3(BX, 16), 0, s>>>(a);
  } else {
    const dim3 grid((a.g.nx + BX - 3) / (BX - 2), (a.g.ny + 8 - 3) / (8 - 2));
    k_tracer_stage<8><<<grid, dim3(BX, 8), 0, s>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t launch_warm_rain(const RainArgs& a, cudaStream_t s, bool micro) {
  if (a.g.nz > kMaxNz) return cudaErrorInvalidValue;
  const dim3 grid((a.g.nx + RB - 1) / RB, a.g.ny);
  if (micro) k_warm_rain<true><<<grid, RB, 0, s>>>(a);
  else if (a.fallout_mode || a.th_acc) k_warm_rain<false><<<grid, RB, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace gwmb
