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
#include <algorithm>
#include <cstring>

#include <cuda_bf16.h>

#include "surrogate.cuh"
#include "surrogate_rain.cuh"

namespace gwmb {
namespace {

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

// Two 16-cell tiles (the warp's 32 slots) through the network, interleaved: every
// weight fragment is loaded once for both tiles and the two tiles' MMA chains are
// independent.  p[q] (q = 0..3) are this lane's own slot features 2q, 2q+1 packed as
// BF16 pairs; rows g and g+8 of tile 0 are slots g and g+8, of tile 1 slots 16+g and
// 24+g.  Returns the output fragments (c0..c3) of the last layer for both tiles.
__device__ __forceinline__ void mlp_tiles(const uint2* __restrict__ fr, const float* __restrict__ bias,
                                          const unsigned p[4], int gq, int t, float y0[4], float y1[4]) {
  unsigned a00 = 0, a01 = 0, a10 = 0, a11 = 0;  // layer 1 A fragments (k 8..15 are padding)
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const unsigned v0 = __shfl_sync(0xffffffffu, p[q], gq), v1 = __shfl_sync(0xffffffffu, p[q], gq + 8);
    const unsigned v2 = __shfl_sync(0xffffffffu, p[q], 16 + gq), v3 = __shfl_sync(0xffffffffu, p[q], 24 + gq);
    if (q == t) { a00 = v0; a01 = v1; a10 = v2; a11 = v3; }
  }
  const int lane = threadIdx.x & 31;
  const int c2 = 2 * t;
  float acc[2][8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float b0 = bias[8 * nt + c2], b1 = bias[8 * nt + c2 + 1];
    const uint2 w = fr[nt * 32 + lane];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      acc[h][nt][0] = b0; acc[h][nt][1] = b1; acc[h][nt][2] = b0; acc[h][nt][3] = b1;
    }
    mma_bf16(acc[0][nt][0], acc[0][nt][1], acc[0][nt][2], acc[0][nt][3], a00, a01, 0u, 0u, w.x, w.y);
    mma_bf16(acc[1][nt][0], acc[1][nt][1], acc[1][nt][2], acc[1][nt][3], a10, a11, 0u, 0u, w.x, w.y);
  }
  auto act = [&](unsigned a[2][4][4]) {
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
      for (int kt = 0; kt < 4; ++kt) {
        a[h][kt][0] = pack_bf16(gelu_fast(acc[h][2 * kt][0]), gelu_fast(acc[h][2 * kt][1]));
        a[h][kt][1] = pack_bf16(gelu_fast(acc[h][2 * kt][2]), gelu_fast(acc[h][2 * kt][3]));
        a[h][kt][2] = pack_bf16(gelu_fast(acc[h][2 * kt + 1][0]), gelu_fast(acc[h][2 * kt + 1][1]));
        a[h][kt][3] = pack_bf16(gelu_fast(acc[h][2 * kt + 1][2]), gelu_fast(acc[h][2 * kt + 1][3]));
      }
  };
#pragma unroll
  for (int L = 0; L < 2; ++L) {
    unsigned a[2][4][4];
    act(a);
    const uint2* f = fr + (8 + L * 32) * 32;
    const float* bb = bias + 64 * (L + 1);
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      const float b0 = bb[8 * nt + c2], b1 = bb[8 * nt + c2 + 1];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        acc[h][nt][0] = b0; acc[h][nt][1] = b1; acc[h][nt][2] = b0; acc[h][nt][3] = b1;
      }
#pragma unroll
      for (int kt = 0; kt < 4; ++kt) {
        const uint2 w = f[(kt * 8 + nt) * 32 + lane];
#pragma unroll
        for (int h = 0; h < 2; ++h)
          mma_bf16(acc[h][nt][0], acc[h][nt][1], acc[h][nt][2], acc[h][nt][3], a[h][kt][0], a[h][kt][1],
                   a[h][kt][2], a[h][kt][3], w.x, w.y);
      }
    }
  }
  unsigned a[2][4][4];
  act(a);
  const float b0 = bias[192 + c2], b1 = bias[192 + c2 + 1];
  y0[0] = b0; y0[1] = b1; y0[2] = b0; y0[3] = b1;
  y1[0] = b0; y1[1] = b1; y1[2] = b0; y1[3] = b1;
  const uint2* f = fr + 72 * 32;
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    const uint2 w = f[kt * 32 + lane];
    mma_bf16(y0[0], y0[1], y0[2], y0[3], a[0][kt][0], a[0][kt][1], a[0][kt][2], a[0][kt][3], w.x, w.y);
    mma_bf16(y1[0], y1[1], y1[2], y1[3], a[1][kt][0], a[1][kt][1], a[1][kt][2], a[1][kt][3], w.x, w.y);
  }
}

// Microphysics of every cell with the network (the first of the two kernels of the
// surrogate warm rain; the fallout sweep is k_warm_rain without microphysics).
// A warp walks chunks of 32 consecutive cells of one (j, k) row.  Each lane builds its
// cell's state and features and applies the activity gate; quiet cells are left as
// they are (no store).  The active cells of successive chunks are packed into the
// warp's 32 slots (shared memory); whenever the slots fill, the warp runs them through
// the network as two 16-row MMA tiles and every lane applies the result of its slot.
// The network therefore runs on active cells only, in dense tiles, and the work has no
// dependence between levels.
constexpr int kNW = 4, kNT = 32 * kNW;

__global__ void __launch_bounds__(kNT, 3) k_rain_net(const RainArgs a, const SurrogateArgs s) {
  __shared__ uint2 s_fr[kSurFrags * 32];
  __shared__ float s_bias[kSurBias];
  __shared__ float s_norm[kMlpNorm + kMlpRange];
  __shared__ int s_ij[kNW][32], s_kf[kNW][32];
  __shared__ unsigned s_pk[kNW][4][32];
  __shared__ unsigned long long s_st[kSurStats];
  for (int q = threadIdx.x; q < kSurFrags * 32; q += kNT) s_fr[q] = s.frags[q];
  for (int q = threadIdx.x; q < kSurBias; q += kNT) s_bias[q] = s.bias[q];
  for (int q = threadIdx.x; q < kMlpNorm; q += kNT) s_norm[q] = s.norm[q];
  for (int q = threadIdx.x; q < kMlpRange; q += kNT) s_norm[kMlpNorm + q] = s.range[q];
  if (threadIdx.x < kSurStats) s_st[threadIdx.x] = 0ull;
  __syncthreads();

  const Geom& g = a.g;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, gq = lane >> 2, t = lane & 3;
  const unsigned lt = (1u << lane) - 1u;
  const MicroParams mp{a.dt, a.relax, a.thr, a.rate, a.evap, a.latent};
  const float* xm = s_norm;
  const float* xs = s_norm + kMlpIn;
  const float* ym = s_norm + 2 * kMlpIn;
  const float* ys = s_norm + 2 * kMlpIn + kMlpOut;
  const float* xmin = s_norm + kMlpNorm;
  const float* xmax = s_norm + kMlpNorm + kMlpIn;

  // the slots' cells through the network; lane L applies slot L (L < count)
  auto run = [&](int count) {
    __syncwarp();
    const bool mine = lane < count;
    unsigned p[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) p[q] = mine ? s_pk[wid][q][lane] : 0u;
    const int ij = s_ij[wid][lane], kf = s_kf[wid][lane];
    __syncwarp();
    // tile 0 holds slots 0-15, tile 1 slots 16-31; row r of a tile sits in lanes
    // 4 (r % 8) + o/2 of its output fragment, and each lane gathers its own row
    float y0[4], y1[4];
    mlp_tiles(s_fr, s_bias, p, gq, t, y0, y1);
    float out[6];
    {
      const int r = lane & 15;
      const int src = 4 * (r & 7);
      const bool hi = r >= 8, t1 = lane >= 16;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const float u0 = __shfl_sync(0xffffffffu, y0[0], src + j), u1 = __shfl_sync(0xffffffffu, y0[1], src + j);
        const float u2 = __shfl_sync(0xffffffffu, y0[2], src + j), u3 = __shfl_sync(0xffffffffu, y0[3], src + j);
        const float v0 = __shfl_sync(0xffffffffu, y1[0], src + j), v1 = __shfl_sync(0xffffffffu, y1[1], src + j);
        const float v2 = __shfl_sync(0xffffffffu, y1[2], src + j), v3 = __shfl_sync(0xffffffffu, y1[3], src + j);
        out[2 * j] = t1 ? (hi ? v2 : v0) : (hi ? u2 : u0);
        out[2 * j + 1] = t1 ? (hi ? v3 : v1) : (hi ? u3 : u1);
      }
    }
    unsigned fl = 0u;  // this cell's check failures: bit 0 fallback, 2 range, 3 fraction, 4 water, 5 energy
    if (mine) {
    const int i = ij & 0xffff, jj = ij >> 16, k = kf & 0xffff;
    const bool in_range = (kf >> 16) != 0;
    const int o = gidx(g, i, jj, k);
    const float rho_d = __ldg(a.rho + o);
    MicroCell mc = micro_state(rho_d, a.rt[o], a.qv[o], a.qc[o], a.qr[o]);
    const float qs = qsat(mc.temp, mc.p);
    float dq[kMlpOut];
#pragma unroll
    for (int q = 0; q < kMlpOut; ++q) dq[q] = out[q] * ys[q] + ym[q];
    // The fractions are used inside [-tol_water, hi + tol_water], not clipped to
    // [0, hi]: the plain scheme's efficiency often sits on an end of its interval (full
    // adjustment, no rain evaporation in saturated air), and clipping the network's
    // noise there would bias the amounts.  Small reverse amounts stay bounded by the caps
    // below, which keep every mixing ratio non-negative.
    const float lat = a.latent ? mc.lh : 0.0f;
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
    const bool ok = in_range && frac_ok && water_ok && energy_ok;
    fl = (ok ? 0u : 1u) | (in_range ? 0u : 4u) | (frac_ok ? 0u : 8u) | (water_ok ? 0u : 16u) |
         (energy_ok ? 0u : 32u);
    float th, qv, qc, qr;
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
    const float rho = mc.rho;
    const bool edge = (g.per_x && (i <= 1 || i >= g.nx - 2)) || (g.per_y && (jj <= 1 || jj >= g.ny - 2));
    store_tile(a.qv, g, kCell, i, jj, k, rho * qv, edge);
    store_tile(a.qc, g, kCell, i, jj, k, rho * qc, edge);
    store_tile(a.qr, g, kCell, i, jj, k, rho * qr, edge);
    store_tile(a.rt, g, kCell, i, jj, k, rho * th, edge);
    }
    if (lane == 0) atomicAdd(&s_st[1], (unsigned long long)count);
#pragma unroll
    for (int q = 0; q < kSurStats; ++q) {
      if (q == 1) continue;
      const unsigned b = __ballot_sync(0xffffffffu, (fl >> q) & 1u);
      if (lane == 0 && b) atomicAdd(&s_st[q], (unsigned long long)__popc(b));
    }
  };

  // a warp takes whole (j, k) rows and walks their 32-cell chunks in x, loading the next
  // chunk's five fields while the current one is processed
  const int cx = (g.nx + 31) >> 5;
  const int rows = g.ny * g.nz;
  int cnt = 0;  // filled slots (warp-uniform)
  for (;;) {
    // rows are taken from a shared counter: the active cells cluster in a few levels, and
    // a static split would leave the warps that drew cloudy rows working alone at the end
    int row = 0;
    if (lane == 0) row = atomicAdd(s.work, 1);
    row = __shfl_sync(0xffffffffu, row, 0);
    if (row >= rows) break;
    const int j = row % g.ny, k = row / g.ny;
    const int obase = gidx(g, 0, j, k);
    float f_rho = 0.f, f_rt = 0.f, f_qv = 0.f, f_qc = 0.f, f_qr = 0.f;
    auto fetch = [&](int ci) {
      const int ii = ci * 32 + lane;
      if (ci < cx && ii < g.nx) {
        const int o = obase + ii;
        f_rho = __ldg(a.rho + o); f_rt = a.rt[o]; f_qv = a.qv[o]; f_qc = a.qc[o]; f_qr = a.qr[o];
      }
    };
    fetch(0);
    for (int ci = 0; ci < cx; ++ci) {
      const int i = ci * 32 + lane;
      const float rho_d = f_rho, rt = f_rt, rqv = f_qv, rqc = f_qc, rqr = f_qr;
      fetch(ci + 1);
      bool net = false, in_range = true;
      unsigned p[4] = {0u, 0u, 0u, 0u};
      if (i < g.nx) {
        // activity gate: with no cloud or rain water and no supersaturation the plain
        // scheme leaves the cell exactly as it is (micro_step takes none of its branches).
        // A cell without condensate that a fast-math estimate finds clearly subsaturated
        // (vapour below 0.999 of saturation; the estimate's error is ~1e-6) is quiet
        // without the exact state; every other cell is decided on the exact state.
        bool exact = rqc > 0.0f || rqr > 0.0f;
        if (!exact) {
          const float rho = fmaxf(rho_d, 1.0e-6f), ir = __fdividef(1.0f, rho);
          const float ratio = fmaxf(rt * (kRd / kP0), 1.0e-6f);
          const float p_ = kP0 * __powf(ratio, 1.0f / (1.0f - kKappa));
          const float temp = rt * ir * __powf(fmaxf(p_ * (1.0f / kP0), 1.0e-6f), kKappa);
          const float tc = temp - 273.15f;
          const float es = 611.2f * __expf(__fdividef(17.67f * tc, fmaxf(tc + 243.5f, 1.0e-6f)));
          const float eps = kRd / kRv;
          const float qs = fminf(fmaxf(__fdividef(eps * es, fmaxf(p_ - (1.0f - eps) * es, 1000.0f)), 0.0f), 0.05f);
          exact = !(fmaxf(rqv * ir, 0.0f) < qs * (1.0f - 1.0e-3f));
        }
        if (exact) {
          const MicroCell mc = micro_state(rho_d, rt, rqv, rqc, rqr);
          net = !(mc.qc == 0.0f && mc.qr == 0.0f && !(mc.qv > qsat(mc.temp, mc.p)));
          if (net) {
            float x[kMlpIn];
            rain_features(mc, rho_d, a.dt, x);
            float xn[8];
  #pragma unroll
            for (int f = 0; f < kMlpIn; ++f) {
              in_range = in_range && x[f] >= xmin[f] && x[f] <= xmax[f];
              xn[f] = (x[f] - xm[f]) / xs[f];
            }
            xn[7] = 0.0f;
  #pragma unroll
            for (int q = 0; q < 4; ++q) p[q] = pack_bf16(xn[2 * q], xn[2 * q + 1]);
          }
        }
      }
      const unsigned m = __ballot_sync(0xffffffffu, net);
      if (m == 0u) continue;
      const int r = __popc(m & lt), n = __popc(m);
      auto put = [&](int slot) {
  #pragma unroll
        for (int q = 0; q < 4; ++q) s_pk[wid][q][slot] = p[q];
        s_ij[wid][slot] = i | (j << 16);
        s_kf[wid][slot] = k | (in_range ? 0x10000 : 0);
      };
      if (net && cnt + r < 32) put(cnt + r);
      if (cnt + n >= 32) {
        run(32);
        if (net && cnt + r >= 32) put(cnt + r - 32);
        cnt = cnt + n - 32;
      } else {
        cnt += n;
      }
    }
  }
  if (cnt > 0) run(cnt);

  __syncthreads();
  if (threadIdx.x < kSurStats && s_st[threadIdx.x] && s.stats) atomicAdd(s.stats + threadIdx.x, s_st[threadIdx.x]);
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
  if (a.g.nz > kMaxNz || a.g.nx > 0xffff || a.g.ny > 0x7fff || a.g.nz > 0xffff) return cudaErrorInvalidValue;
  static int blocks = 0;  // resident CTAs of the whole device (the work loop is grid-strided)
  if (blocks == 0) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_rain_net, kNT, 0);
    if (e != cudaSuccess) return e;
    blocks = sms * (per_sm > 0 ? per_sm : 1);
  }
  if (!s.work) return cudaErrorInvalidValue;
  const long long rows = (long long)a.g.ny * a.g.nz;
  const int grid = (int)std::min<long long>(blocks, (rows + kNW - 1) / kNW);
  cudaError_t e = cudaMemsetAsync(s.work, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  k_rain_net<<<grid, kNT, 0, st>>>(a, s);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_warm_rain(a, st, /*micro=*/false);
}

}  // namespace gwmb
