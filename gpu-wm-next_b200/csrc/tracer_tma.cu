// tracer_tma.cu — one SSPRK3 stage of up to three passive tracers on owned tiles fed by
// TMA (flat terrain, and terrain with the per-cell inverse layer depth).
//
// Same operator and per-cell arithmetic as k_tracer_stage: the upwind mixing-ratio
// flux divergence with frozen end-of-step dry mass fluxes
// (passive_tracer_stage_kernel, src/dycore/dry_transport.cu:49-125; clip at zero) and
// the SSPRK3 blend of advance_passive_tracers_ssprk3 (:440-518).  A CTA owns a
// 32 x 16 tile, two columns per thread; one elected thread fetches each plane's boxes
// with cp.async.bulk.tensor.3d into a three-slot shared-memory ring:
//   rho, rho*q (three tracers)   40 x 18 boxes: the tile and its halo ring
//   u, v                         36 x 17 boxes: owned faces + the east/north face
//   w                            32 x 16 box: owned Z faces (plane nz: w only)
// Per plane the mixing ratios of the tile and its ring (no corners) go to shared
// memory; one barrier per plane publishes them.
#include <type_traits>

#include "physics.cuh"
#include "stencil.cuh"
#include "tma.cuh"

namespace gwmb {
namespace {

namespace tt {
constexpr int TX = 32, TY = 16, RY = 8, NT = 256, NTR = 3;
// the thread that issues the TMA loads: lane 0 of the last warp, which has no halo-ring
// role (warps 0-2 carry those)
constexpr int ISSUER = NT - 32;
constexpr int CBW = 40, CBH = 18, FBW = 36, FBH = 17, OBW = 32, OBH = 16;
constexpr int O_RHO = 0, O_Q = 736, O_U = 2944, O_V = 3584, O_W = 4224, SLOT = 4736, NSLOT = 3;
constexpr unsigned B_CELL = CBW * CBH * 4, B_FACE = FBW * FBH * 4, B_OWN = OBW * OBH * 4;
constexpr int QW = TX + 2, QH = TY + 2;  // mixing-ratio plane: 34 x 18
constexpr size_t kDynSmem = size_t(SLOT) * NSLOT * sizeof(float) + 128;
static_assert(O_Q % 32 == 0 && O_U % 32 == 0 && O_V % 32 == 0 && O_W % 32 == 0 && SLOT % 32 == 0,
              "128-byte aligned sub-buffers");
static_assert(O_Q - O_RHO >= CBW * CBH && O_U - O_Q >= NTR * 736 && O_V - O_U >= FBW * FBH &&
                  O_W - O_V >= FBW * FBH && SLOT - O_W >= OBW * OBH,
              "boxes fit their sub-buffers");
}  // namespace tt

template <bool TERRAIN>
__global__ void __launch_bounds__(tt::NT, 3) k_tracer_tma(const TracerArgs a, const __grid_constant__ TracerMaps m) {
  using namespace tt;
  extern __shared__ unsigned char s_dyn[];
  __shared__ float s_q[NTR][2][QH][QW];
  __shared__ __align__(8) uint64_t s_bar[NSLOT];
  __shared__ int s_abort[2];
  float* const ring = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(s_dyn) + 127) & ~uintptr_t(127));

  const Geom& g = a.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int w = min(TX, nx - i0), h = min(TY, ny - j0);
  const bool own0 = tx < w && ty < h, own1 = tx < w && ty + RY < h;
  const int gi = i0 + tx, gj0 = j0 + ty, gj1 = j0 + ty + RY;
  const bool edge = (g.per_x && (i0 <= 1 || i0 + w >= nx - 1)) || (g.per_y && (j0 <= 1 || j0 + h >= ny - 1));
  const float idx = g.inv_dx, idy = g.inv_dy;
  const bool blend = a.q0[0] != nullptr;
  // halo ring (threads 0-95, whole warps): west, east columns, south, north rows;
  // (hr, hc) are mixing-ratio plane coordinates (row 0 = j0-1, column 0 = i0-1)
  int hr = -1, hc = 0;
  if (tid < TY) { if (tid < h) { hr = tid + 1; hc = 0; } }
  else if (tid < 2 * TY) { if (tid - TY < h) { hr = tid - TY + 1; hc = w + 1; } }
  else if (tid < 2 * TY + TX) { if (tid - 2 * TY < w) { hr = 0; hc = tid - 2 * TY + 1; } }
  else if (tid < 2 * TY + 2 * TX) { if (tid - 2 * TY - TX < w) { hr = h + 1; hc = tid - 2 * TY - TX + 1; } }

  if (tid == 0) {
    for (int s = 0; s < NSLOT; ++s) mbar_init(&s_bar[s], 1);
    mbar_fence_init();
    s_abort[0] = 0;
    s_abort[1] = 0;
  }
  __syncthreads();

  // err[1] > 0 (set only by failure-path tests): the first CTA to see it leaves the loads
  // of plane err[1] - 1 unissued, so that CTA's bounded wait runs out
  int stall = -1;
  if (tid == ISSUER && *(volatile int*)(a.err + 1) > 0) stall = atomicExch(a.err + 1, 0) - 1;
  auto issue = [&](int kk) {  // plane kk in [0, nz]; plane nz holds the top faces only
    float* st = ring + (kk % NSLOT) * SLOT;
    uint64_t* bar = &s_bar[kk % NSLOT];
    const bool cells = kk < nz;
    unsigned bytes = B_OWN;
    if (cells) bytes += (1 + a.ntracers) * B_CELL + 2 * B_FACE;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(bar, bytes);
    if (kk == stall) return;  // failure-path testing: this plane's loads stay unissued
    tma_load_3d(st + O_W, &m.w, i0 + kXOff, j0 + 1, kk, bar);
    if (cells) {
      tma_load_3d(st + O_RHO, &m.rho, i0 + kXOff - 4, j0, kk, bar);
      for (int t = 0; t < a.ntracers; ++t) tma_load_3d(st + O_Q + t * 736, &m.q[t], i0 + kXOff - 4, j0, kk, bar);
      tma_load_3d(st + O_U, &m.u, i0 + kXOff, j0 + 1, kk, bar);
      tma_load_3d(st + O_V, &m.v, i0 + kXOff, j0 + 1, kk, bar);
    }
  };
  int issued = -1, waited = -1;
  auto wait_plane = [&](int kk, int epoch) {
    if (!mbar_wait(&s_bar[kk % NSLOT], (kk / NSLOT) & 1)) {
      s_abort[epoch & 1] = 1;
      atomicExch(a.err, 1);
    } else {
      waited = kk;  // a plane whose wait gave up stays in the drain below
    }
  };
  // mixing ratios of plane kk (dry_transport.cu:91-94) at the owned cells and the ring
  auto mix = [&](int kk) {
    const float* st = ring + (kk % NSLOT) * SLOT;
    auto one = [&](int r, int c) {
      const int b = r * CBW + c + 3;
      const float rr = fmaxf(st[O_RHO + b], 1.0e-6f);
#pragma unroll
      for (int t = 0; t < NTR; ++t)
        if (t < a.ntracers) s_q[t][kk & 1][r][c] = st[O_Q + t * 736 + b] / rr;
    };
    if (own0) one(ty + 1, tx + 1);
    if (own1) one(ty + RY + 1, tx + 1);
    if (hr >= 0) one(hr, hc);
  };

  if (tid == ISSUER) {
    issue(0);
    issue(1);
    issued = 1;
    if (nz >= 2) { issue(2); issued = 2; }
  }
  wait_plane(0, 0);
  mix(0);
  float qb0[NTR] = {0.f, 0.f, 0.f}, qb1[NTR] = {0.f, 0.f, 0.f};  // own mixing ratios at k-1
  __syncthreads();

  // blend partner of plane kk at the thread's owned cells (prefetched a plane ahead)
  auto load_q0 = [&](int gj, bool own, int kk, float* q0v) {
#pragma unroll
    for (int t = 0; t < NTR; ++t) q0v[t] = 0.f;
    if (!own || !blend || kk >= nz) return;
    const int o = gidx(g, gi, gj, kk);
#pragma unroll
    for (int t = 0; t < NTR; ++t)
      if (t < a.ntracers) q0v[t] = __ldg(a.q0[t] + o);
  };
  float q0a[NTR], q0b[NTR];
  load_q0(gj0, own0, 0, q0a);
  load_q0(gj1, own1, 0, q0b);

  // one owned column of plane k
  auto column = [&](auto tile_class, int k, int r, int gj, bool own_rt, float* qb, const float* q0v, float idz) {
    constexpr bool IN = decltype(tile_class)::value;  // interior tile: plain stores
    const bool own = IN || own_rt;
    const float* st = ring + (k % NSLOT) * SLOT;
    const float* sn = ring + ((k + 1) % NSLOT) * SLOT;
    const int c = tx + 1;
    const int pb = k & 1;
    const float fw = st[O_U + (r - 1) * FBW + tx], fe = st[O_U + (r - 1) * FBW + tx + 1];
    const float fs = st[O_V + (r - 1) * FBW + tx], fn = st[O_V + r * FBW + tx];
    const float fb = st[O_W + (r - 1) * OBW + tx], ft = sn[O_W + (r - 1) * OBW + tx];
#pragma unroll
    for (int t = 0; t < NTR; ++t) {
      if (t >= a.ntracers) break;
      const float qc = s_q[t][pb][r][c];
      const float qw = s_q[t][pb][r][c - 1], qe = s_q[t][pb][r][c + 1];
      const float qs = s_q[t][pb][r - 1][c], qn = s_q[t][pb][r + 1][c];
      const float qbt = (k > 0) ? qb[t] : qc;
      const float qt = (k + 1 < nz) ? s_q[t][pb ^ 1][r][c] : qc;
      const float gw = fp::upwind(fw, qw, qc), ge = fp::upwind(fe, qc, qe);
      const float gs = fp::upwind(fs, qs, qc), gn = fp::upwind(fn, qc, qn);
      const float gb = fp::upwind(fb, qbt, qc), gt = fp::upwind(ft, qc, qt);
      const float div = fp::divergence(ge, gw, gn, gs, gt, gb, idx, idy, idz);
      float out = fp::update(st[O_Q + t * 736 + r * CBW + c + 3], -a.dt, div, 0.0f);
      if (blend) out = fp::blend(a.wa, q0v[t], a.wb, out);
      if (own) {
        if (IN) a.q_out[t][gidx(g, gi, gj, k)] = out;
        else store_tile(a.q_out[t], g, kCell, gi, gj, k, out, edge);
      }
      qb[t] = qc;
    }
  };

  // Interior tiles (full, away from every periodic edge ring) run a copy of the plane
  // loop with plain stores instead of the periodic mirror stores; the arithmetic is the same.
  const bool interior = !edge && i0 + TX <= nx && j0 + TY <= ny;
  auto plane_loop = [&](auto tile_class) -> bool {  // true when a bounded wait gave up
    [[maybe_unused]] constexpr bool IN = decltype(tile_class)::value;
    for (int k = 0; k < nz; ++k) {
      // mixing ratios of plane k+1 (the own ones are this thread's, the ring published
      // by the barrier below for the next plane)
      // inverse layer depth (per level on flat terrain, per cell on terrain), loaded ahead
      // of the mixing-ratio work
      float idz0, idz1;
      if constexpr (TERRAIN) {
        idz0 = (IN || own0) ? __ldg(a.idz_c + gidx(g, gi, gj0, k)) : 0.f;
        idz1 = (IN || own1) ? __ldg(a.idz_c + gidx(g, gi, gj1, k)) : 0.f;
      } else {
        idz0 = idz1 = __ldg(a.idz_c + k);
      }
      float n0a[NTR], n0b[NTR];
      load_q0(gj0, own0, k + 1, n0a);
      load_q0(gj1, own1, k + 1, n0b);
      wait_plane(k + 1, k);
      if (k + 1 < nz) mix(k + 1);
      column(tile_class, k, ty + 1, gj0, own0, qb0, q0a, idz0);
      column(tile_class, k, ty + RY + 1, gj1, own1, qb1, q0b, idz1);
  #pragma unroll
      for (int t = 0; t < NTR; ++t) { q0a[t] = n0a[t]; q0b[t] = n0b[t]; }
      __syncthreads();  // publishes plane k+1's ring; slot k is free
      if (s_abort[k & 1]) return true;
      if (tid == ISSUER && k + 3 <= nz) { issue(k + 3); issued = k + 3; }
    }
    return false;
  };
  const bool aborted = interior ? plane_loop(std::true_type{}) : plane_loop(std::false_type{});
  if (aborted && tid == ISSUER)
    for (int kk = waited + 1; kk <= issued; ++kk) mbar_wait(&s_bar[kk % NSLOT], (kk / NSLOT) & 1);
}

}  // namespace

cudaError_t init_tracer_tma() {
  const cudaError_t e =
      cudaFuncSetAttribute(k_tracer_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tt::kDynSmem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_tracer_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tt::kDynSmem);
}

cudaError_t launch_tracer_tma(const TracerArgs& a, const TracerMaps& m, cudaStream_t s) {
  if (a.g.nz < 1 || !a.err || a.ntracers < 1 || a.ntracers > tt::NTR) return cudaErrorInvalidValue;
  const dim3 block(tt::TX, tt::RY);
  const dim3 grid((a.g.nx + tt::TX - 1) / tt::TX, (a.g.ny + tt::TY - 1) / tt::TY);
  if (a.terrain) k_tracer_tma<true><<<grid, block, tt::kDynSmem, s>>>(a, m);
  else k_tracer_tma<false><<<grid, block, tt::kDynSmem, s>>>(a, m);
  return cudaGetLastError();
}

}  // namespace gwmb
