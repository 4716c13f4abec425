// surrogate_rain.cu — warm rain with the learned microphysics (inference).
//
// The column sweep of k_warm_rain (warm_rain.cu:36-191 with metric or nominal fallout),
// with the per-cell microphysics replaced by the trained network on the tensor cores.
// A warp owns 32 columns and marches down k; at each level its 32 cells are two 16-row
// tiles of mma.sync.m16n8k16 (BF16 inputs, FP32 accumulation): 7 (padded to 16) -> 64
// -> 64 -> 64 -> 5 (padded to 8), 76 MMAs per tile.  The weights sit in shared memory
// as per-lane B fragments; each layer's accumulator fragments become the next layer's
// A fragments in registers (the C layout of two adjacent 8-column tiles is the A
// layout of one 16-column k-step), so activations never leave the registers.
// GELU is the tanh form with the hardware tanh approximation.
//
// Per cell the network gives the condensation, autoconversion and rain-evaporation
// amounts as fractions of their bounds (the saturation deficit |qv - qs|, the cloud
// water above the autoconversion threshold, the rain present) and, redundantly, dtheta
// and dqv.  The fractions are held to their intervals widened by tol_water and turned
// into amounts c (negative for cloud evaporation), a, e with the caps the plain scheme
// applies (no more vapour condensed or cloud evaporated than there is), then applied: qv -= c - e, qc += c - a, qr += a - e,
// theta += L_v/(c_p pi) (c - e); water and energy close by construction.  The cell takes
// the plain scheme instead when an input lies outside the training range, when a raw
// fraction lies outside its interval by more than tol_water, or when the network's dqv
// or dtheta disagree with the amounts by more than tol_water or tol_energy of the
// cell's exchange plus the output's training spread.  Quiet cells (no condensate, not
// supersaturated), which the plain scheme leaves unchanged, skip the network.  Fallout
// is the scheme's explicit flux in both paths, and the column accumulation (what leaves
// a cell enters the one below, the bottom flux is precipitation) is exact.
#include <cstring>

#include <cuda_bf16.h>

#include "surrogate.cuh"
#include "surrogate_rain.cuh"

namespace gwmb {
namespace {

constexpr int kRB = 128;  // columns per CTA (4 warps)

__device__ __forceinline__ void mma_bf16(float& c0, float& c1, float& c2, float& c3, unsigned a0, unsigned a1,
                                         unsigned a2, unsigned a3, unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c0), "+f"(c1), "+f"(c2), "+f"(c3)
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const unsigned*>(&v);
}

__device__ __forceinline__ float tanh_approx(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu_fast(float z) {
  return 0.5f * z * (1.0f + tanh_approx(0.7978845608028654f * (z + 0.044715f * z * z * z)));
}

// One 16-cell tile through the network.  p[q] (q = 0..3) are this lane's own cell
// features 2q, 2q+1 packed as BF16 pairs; srcA/srcB the lanes holding rows g and g+8 of
// the tile.  Returns the output fragment (c0..c3) of the last layer.
__device__ __forceinline__ void mlp_tile(const uint2* __restrict__ fr, const float* __restrict__ bias,
                                         const unsigned p[4], int srcA, int srcB, int t, float y[4]) {
  // layer 1 input fragment: row g features 2t, 2t+1 (k 0..7); k 8..15 are padding
  unsigned a0 = 0, a1 = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const unsigned va = __shfl_sync(0xffffffffu, p[q], srcA);
    const unsigned vb = __shfl_sync(0xffffffffu, p[q], srcB);
    if (q == t) { a0 = va; a1 = vb; }
  }
  const int lane = threadIdx.x & 31;
  const int c2 = 2 * t;
  float acc[8][4];
  // layer 1: 8 output tiles
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float b0 = bias[8 * nt + c2], b1 = bias[8 * nt + c2 + 1];
    acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
    const uint2 w = fr[nt * 32 + lane];
    mma_bf16(acc[nt][0], acc[nt][1], acc[nt][2], acc[nt][3], a0, a1, 0u, 0u, w.x, w.y);
  }
  // layers 2 and 3
#pragma unroll
  for (int L = 0; L < 2; ++L) {
    unsigned a[4][4];
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
      a[kt][0] = pack_bf16(gelu_fast(acc[2 * kt][0]), gelu_fast(acc[2 * kt][1]));
      a[kt][1] = pack_bf16(gelu_fast(acc[2 * kt][2]), gelu_fast(acc[2 * kt][3]));
      a[kt][2] = pack_bf16(gelu_fast(acc[2 * kt + 1][0]), gelu_fast(acc[2 * kt + 1][1]));
      a[kt][3] = pack_bf16(gelu_fast(acc[2 * kt + 1][2]), gelu_fast(acc[2 * kt + 1][3]));
    }
    const uint2* f = fr + (8 + L * 32) * 32;
    const float* bb = bias + 64 * (L + 1);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const float b0 = bb[8 * nt + c2], b1 = bb[8 * nt + c2 + 1];
      acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
#pragma unroll
      for (int kt = 0; kt < 4; ++kt) {
        const uint2 w = f[(kt * 8 + nt) * 32 + lane];
        mma_bf16(acc[nt][0], acc[nt][1], acc[nt][2], acc[nt][3], a[kt][0], a[kt][1], a[kt][2], a[kt][3], w.x, w.y);
      }
    }
  }
  // output layer (5 outputs in one 8-column tile)
  unsigned a[4][4];
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    a[kt][0] = pack_bf16(gelu_fast(acc[2 * kt][0]), gelu_fast(acc[2 * kt][1]));
    a[kt][1] = pack_bf16(gelu_fast(acc[2 * kt][2]), gelu_fast(acc[2 * kt][3]));
    a[kt][2] = pack_bf16(gelu_fast(acc[2 * kt + 1][0]), gelu_fast(acc[2 * kt + 1][1]));
    a[kt][3] = pack_bf16(gelu_fast(acc[2 * kt + 1][2]), gelu_fast(acc[2 * kt + 1][3]));
  }
  const float b0 = bias[192 + c2], b1 = bias[192 + c2 + 1];
  y[0] = b0; y[1] = b1; y[2] = b0; y[3] = b1;
  const uint2* f = fr + 72 * 32;
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    const uint2 w = f[kt * 32 + lane];
    mma_bf16(y[0], y[1], y[2], y[3], a[kt][0], a[kt][1], a[kt][2], a[kt][3], w.x, w.y);
  }
}

__global__ void __launch_bounds__(kRB) k_warm_rain_surrogate(const RainArgs a, const SurrogateArgs s) {
  __shared__ uint2 s_fr[kSurFrags * 32];
  __shared__ float s_bias[kSurBias];
  __shared__ float s_norm[kMlpNorm + kMlpRange];
  __shared__ long long s_th[kMaxNz][kRB / 32];
  __shared__ unsigned long long s_st[kSurStats];
  for (int q = threadIdx.x; q < kSurFrags * 32; q += kRB) s_fr[q] = s.frags[q];
  for (int q = threadIdx.x; q < kSurBias; q += kRB) s_bias[q] = s.bias[q];
  for (int q = threadIdx.x; q < kMlpNorm; q += kRB) s_norm[q] = s.norm[q];
  for (int q = threadIdx.x; q < kMlpRange; q += kRB) s_norm[kMlpNorm + q] = s.range[q];
  if (threadIdx.x < kSurStats) s_st[threadIdx.x] = 0ull;
  __syncthreads();

  const Geom& g = a.g;
  const int gi = blockIdx.x * kRB + threadIdx.x;
  const int gj = blockIdx.y;
  const bool active = gi < g.nx && gj < g.ny;
  const int ilo = blockIdx.x * kRB;
  const bool edge = (g.per_x && (ilo <= 1 || ilo + kRB - 1 >= g.nx - 1)) || (g.per_y && (gj <= 1 || gj >= g.ny - 1));
  const int lane = threadIdx.x & 31, gq = lane >> 2, t = lane & 3;
  const MicroParams mp{a.dt, a.relax, a.thr, a.rate, a.evap, a.latent};
  const float* xm = s_norm;
  const float* xs = s_norm + kMlpIn;
  const float* ym = s_norm + 2 * kMlpIn;
  const float* ys = s_norm + 2 * kMlpIn + kMlpOut;
  const float* xmin = s_norm + kMlpNorm;
  const float* xmax = s_norm + kMlpNorm + kMlpIn;
  float incoming = 0.0f;
  unsigned st[kSurStats] = {0u, 0u, 0u, 0u, 0u, 0u};
  for (int k = g.nz - 1; k >= 0; --k) {
    const int o = active ? gidx(g, gi, gj, k) : 0;
    const float rho_d = active ? __ldg(a.rho + o) : 1.0f;
    const float rt = active ? a.rt[o] : 300.0f;
    const float rqv = active ? a.qv[o] : 0.0f, rqc = active ? a.qc[o] : 0.0f, rqr = active ? a.qr[o] : 0.0f;
    MicroCell mc = micro_state(rho_d, rt, rqv, rqc, rqr);
    // activity gate: with no cloud or rain water and no supersaturation the plain scheme
    // leaves the cell exactly as it is (micro_step takes none of its branches), so the
    // network is not consulted; a warp whose cells are all quiet skips the MMAs
    const float qs = qsat(mc.temp, mc.p);
    const bool quiet = mc.qc == 0.0f && mc.qr == 0.0f && !(mc.qv > qs);
    const bool net = active && !quiet;
    float x[kMlpIn];
    rain_features(mc, rho_d, a.dt, x);
    bool in_range = true;
    float xn[8];
#pragma unroll
    for (int f = 0; f < kMlpIn; ++f) {
      in_range = in_range && x[f] >= xmin[f] && x[f] <= xmax[f];
      xn[f] = (x[f] - xm[f]) / xs[f];
    }
    xn[7] = 0.0f;
    unsigned p[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) p[q] = pack_bf16(xn[2 * q], xn[2 * q + 1]);
    // the warp's two tiles: lanes 0-15 and 16-31
    float y0[4] = {0.0f, 0.0f, 0.0f, 0.0f}, y1[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if (__any_sync(0xffffffffu, net)) {  // warp-uniform
      mlp_tile(s_fr, s_bias, p, gq, gq + 8, t, y0);
      mlp_tile(s_fr, s_bias, p, 16 + gq, 24 + gq, t, y1);
    }
    // gather this lane's 5 outputs: row r of its tile sits in lanes 4 (r % 8) + o/2
    const int r = lane & 15;
    const int src = 4 * (r & 7);
    float out[6];
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float u0 = __shfl_sync(0xffffffffu, y0[0], src + j), u1 = __shfl_sync(0xffffffffu, y0[1], src + j);
      const float u2 = __shfl_sync(0xffffffffu, y0[2], src + j), u3 = __shfl_sync(0xffffffffu, y0[3], src + j);
      const float v0 = __shfl_sync(0xffffffffu, y1[0], src + j), v1 = __shfl_sync(0xffffffffu, y1[1], src + j);
      const float v2 = __shfl_sync(0xffffffffu, y1[2], src + j), v3 = __shfl_sync(0xffffffffu, y1[3], src + j);
      const bool hi = r >= 8, t1 = lane >= 16;
      out[2 * j] = t1 ? (hi ? v2 : v0) : (hi ? u2 : u0);
      out[2 * j + 1] = t1 ? (hi ? v3 : v1) : (hi ? u3 : u1);
    }
    float dq[kMlpOut];
#pragma unroll
    for (int q = 0; q < kMlpOut; ++q) dq[q] = out[q] * ys[q] + ym[q];
    // network step from the fractions, or the plain scheme (lanes past the domain edge
    // take part in the warp's MMAs and reductions but store nothing)
    const float lat = a.latent ? mc.lh : 0.0f;
    // The fractions are used inside [-tol_water, hi + tol_water], not clipped to
    // [0, hi]: the plain scheme's efficiency often sits on an end of its interval (full
    // adjustment, no rain evaporation in saturated air), and clipping the network's
    // noise there would bias the amounts.  Small reverse amounts stay bounded by the caps
    // below, which keep every mixing ratio non-negative.
    const float tw = s.tol_water, te = s.tol_energy;
    const float fc_hi = fmaxf(fmaxf(a.relax, 0.0f), 1.0f);
    const float fc = fminf(fmaxf(dq[0], -tw), fc_hi + tw);
    const float fa = fminf(fmaxf(dq[1], 0.0f), 1.0f);
    const float fe = fminf(fmaxf(dq[2], -tw), 1.0f);
    const float d = mc.qv - qs;
    const float c_p = (d > 0.0f || mc.qc > 0.0f) ? fminf(fmaxf(fc * d, -mc.qc), mc.qv) : 0.0f;
    const float qc_mid = mc.qc + c_p;
    const float a_p = a.rate > 0.0f ? fa * fmaxf(qc_mid - a.thr, 0.0f) : 0.0f;
    const float qr_mid = mc.qr + a_p;
    const float e_p = a.evap > 0.0f ? fe * qr_mid : 0.0f;
    const float qv1 = mc.qv - c_p + e_p;
    const bool frac_ok = dq[0] >= -tw && dq[0] <= fc_hi + tw && dq[1] >= -tw && dq[1] <= 1.0f + tw &&
                         dq[2] >= -tw && dq[2] <= 1.0f + tw && qv1 >= 0.0f;
    const bool water_ok = fabsf(dq[4] - (e_p - c_p)) <= tw * (fabsf(c_p) + fabsf(e_p) + ys[4]);
    const bool energy_ok = fabsf(dq[3] - lat * (c_p - e_p)) <= te * (lat * fabsf(c_p - e_p) + ys[3]);
    const bool ok = net && in_range && frac_ok && water_ok && energy_ok;
    if (net) {
      st[1] += 1u;
      st[0] += ok ? 0u : 1u;
      st[2] += in_range ? 0u : 1u;
      st[3] += frac_ok ? 0u : 1u;
      st[4] += water_ok ? 0u : 1u;
      st[5] += energy_ok ? 0u : 1u;
    }
    float dz = 1.0f, idz = 1.0f;
    if (a.fallout_mode == 1) {
      idz = fmaxf(a.terrain ? __ldg(a.idz_c + o) : __ldg(a.idz_c + k), 1.0e-6f);
      dz = 1.0f / idz;
    } else if (a.fallout_mode == 2) {
      dz = fmaxf(a.layer_depth, 1.0e-3f);
    }
    float th, qv, qc, qr;
    const float rho = mc.rho;
    if (ok) {
      th = mc.th + lat * (c_p - e_p);
      qv = qv1;
      qc = fmaxf(qc_mid - a_p, 0.0f);
      qr = fmaxf(qr_mid - e_p, 0.0f);
    } else {
      micro_step(mc, mp);
      th = mc.th;
      qv = mc.qv;
      qc = mc.qc;
      qr = mc.qr;
    }
    float rqr_new = rho * qr, flux = 0.0f;
    if (a.fallout_mode == 1) {
      const float frac = fminf(fmaxf(a.vt * a.dt * idz, 0.0f), 1.0f);
      flux = frac * (fmaxf(rqr_new, 0.0f) * dz);
    } else if (a.fallout_mode == 2) {
      const float frac = fminf(fmaxf(a.vt * a.dt / dz, 0.0f), 1.0f);
      flux = frac > 0.0f ? frac * (fmaxf(rqr_new, 0.0f) * dz) : 0.0f;
    }
    if (a.fallout_mode) {  // column accumulation: warm_rain.cu:122-191
      const float old_a = fmaxf(rqr_new, 0.0f) * dz;
      rqr_new = a.fallout_mode == 1 ? ((old_a - flux) + incoming) * idz : ((old_a - flux) + incoming) / dz;
      incoming = flux;
    }
    const float rt_new = rho * th;
    FxAcc th_sum;
    if (active) {
      store_tile(a.qv, g, kCell, gi, gj, k, rho * qv, edge);
      store_tile(a.qc, g, kCell, gi, gj, k, rho * qc, edge);
      store_tile(a.qr, g, kCell, gi, gj, k, rqr_new, edge);
      store_tile(a.rt, g, kCell, gi, gj, k, rt_new, edge);
      th_sum.add(theta_of(rho_d, rt_new), kFxTheta);
    }
    if (a.th_acc) {
      const long long tw = th_sum.warp_total();
      if (lane == 0) s_th[k][threadIdx.x >> 5] = tw;
    }
  }
  if (active && a.fallout_mode && a.precip) {  // compensated FP64 surface accumulation
    const int q = gj * g.nx + gi;
    const double sp = a.precip[q], xp = (double)incoming, tp = sp + xp;
    a.precip_comp[q] += (fabs(sp) >= fabs(xp)) ? (sp - tp) + xp : (xp - tp) + sp;
    a.precip[q] = tp;
  }
#pragma unroll
  for (int q = 0; q < kSurStats; ++q) {
    const unsigned w = __reduce_add_sync(0xffffffffu, st[q]);
    if (lane == 0 && w) atomicAdd(&s_st[q], (unsigned long long)w);
  }
  __syncthreads();
  if (threadIdx.x < kSurStats && s_st[threadIdx.x] && s.stats) atomicAdd(s.stats + threadIdx.x, s_st[threadIdx.x]);
  if (a.th_acc) {
    for (int k = threadIdx.x; k < g.nz; k += kRB) {
      long long tt = 0;
      for (int w = 0; w < kRB / 32; ++w) tt += s_th[k][w];
      acc_add(a.th_acc + k, tt);
    }
  }
}

}  // namespace

namespace {
uint16_t bf16_rne(float f) {  // round to nearest even (finite inputs)
  uint32_t u;
  std::memcpy(&u, &f, 4);
  const uint32_t rounding = ((u >> 16) & 1u) + 0x7FFFu;
  return (uint16_t)((u + rounding) >> 16);
}
}  // namespace

void surrogate_fragments(const float* params, uint2* frags, float* bias) {
  // W (nout x nin, row-major) at off -> B fragments of mma.m16n8k16 (B[k][n] = W[n][k]):
  // lane (g, t): b0 = (B[16kt+2t][8nt+g], B[16kt+2t+1][8nt+g]), b1 = rows 2t+8, 2t+9
  auto frag = [&](int off, int nout, int nin, int kt, int nt, int lane) {
    const int gq = lane >> 2, t = lane & 3, n = 8 * nt + gq;
    auto w = [&](int k) { return (n < nout && k < nin) ? params[off + n * nin + k] : 0.0f; };
    const int k0 = 16 * kt + 2 * t;
    uint2 v;
    v.x = (uint32_t)bf16_rne(w(k0)) | ((uint32_t)bf16_rne(w(k0 + 1)) << 16);
    v.y = (uint32_t)bf16_rne(w(k0 + 8)) | ((uint32_t)bf16_rne(w(k0 + 9)) << 16);
    return v;
  };
  for (int lane = 0; lane < 32; ++lane) {
    for (int nt = 0; nt < 8; ++nt) frags[nt * 32 + lane] = frag(kOffW1, kMlpHid, kMlpIn, 0, nt, lane);
    for (int L = 0; L < 2; ++L)
      for (int kt = 0; kt < 4; ++kt)
        for (int nt = 0; nt < 8; ++nt)
          frags[(8 + L * 32 + kt * 8 + nt) * 32 + lane] = frag(L == 0 ? kOffW2 : kOffW3, kMlpHid, kMlpHid, kt, nt, lane);
    for (int kt = 0; kt < 4; ++kt) frags[(72 + kt) * 32 + lane] = frag(kOffW4, kMlpOut, kMlpHid, kt, 0, lane);
  }
  for (int q = 0; q < kMlpHid; ++q) {
    bias[q] = params[kOffB1 + q];
    bias[64 + q] = params[kOffB2 + q];
    bias[128 + q] = params[kOffB3 + q];
  }
  for (int q = 0; q < 8; ++q) bias[192 + q] = q < kMlpOut ? params[kOffB4 + q] : 0.0f;
}

cudaError_t launch_warm_rain_surrogate(const RainArgs& a, const SurrogateArgs& s, cudaStream_t st) {
  if (a.g.nz > kMaxNz) return cudaErrorInvalidValue;
  const dim3 grid((a.g.nx + kRB - 1) / kRB, a.g.ny);
  k_warm_rain_surrogate<<<grid, kRB, 0, st>>>(a, s);
  return cudaGetLastError();
}

}  // namespace gwmb
