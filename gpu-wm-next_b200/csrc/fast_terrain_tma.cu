// fast_terrain_tma.cu — acoustic substep on terrain fed by TMA tile loads.
//
// Same operator and per-cell arithmetic as k_fast_substep<TERRAIN = true> (K9-K15 of
// LocalSplitExplicitFastMode::apply, src/dycore/dry_fast_modes.cu:160-394: the
// chain-rule horizontal pressure gradient of :160-301, perturbations about the column
// hydrostatic reference of :108-158, which k_column_reference builds before the
// substep), with the data path of k_fast_tma: one elected thread per CTA fetches every
// plane's tiles with cp.async.bulk.tensor.3d into a five-slot shared-memory ring, and a
// CTA owns a 32 x 16 tile, two rows per thread.  Per plane kk the slot holds
//   rho(kk), theta(kk)   first substep of a stage: 40 x 18 boxes (the tile and its halo
//                        ring, from which the full pressure is derived); otherwise the
//                        owned 32 x 16 box
//   z(kk)                40 x 18: cell-centre heights of the tile and its ring
//   p(kk)                40 x 18, not in a first substep: the full pressure of the input
//                        with its ring, stored by the previous substep, so the EOS runs
//                        once per owned cell instead of at every position of a tile
//   du(kk), dv(kk)       36 x 17, not in a first substep: owned faces plus the tile's
//                        east/north face
//   dw(kk+1)             32 x 16, not in a first substep
// The vertical pressure derivative of the tile and its ring takes p at three levels; it
// is derived one plane ahead (plane k+1 while plane k's faces are computed, from the
// slots of planes k, k+1, k+2), so one barrier per plane publishes it together with the
// new face increments.  The owned cells' metric columns, column reference and (last
// substep of the step) stage base momenta are per-thread coalesced loads issued one
// plane ahead.
#include <type_traits>

#include "dycore.cuh"
#include "stencil.cuh"
#include "tma.cuh"

namespace gwmb {
namespace {

namespace fz {
constexpr int TX = 32, TY = 16, RY = 8, NT = 256, NW = NT / 32;
constexpr int CBW = 40, CBH = 18;  // cell box: tile + halo ring, x from i0-4 (16-byte aligned)
constexpr int FBW = 36, FBH = 17;  // face box: owned faces + the tile's east/north face
constexpr int OBW = 32, OBH = 16;  // owned box
constexpr unsigned B_CELL = CBW * CBH * 4, B_FACE = FBW * FBH * 4, B_OWN = OBW * OBH * 4;
// ring: planes k, k+1, k+2 are read while plane k is computed; plane k+4 is issued into
// the slot of plane k-1 after the plane's barrier
constexpr int NSLOT = 5, AHEAD = NSLOT - 1;
constexpr int ISSUER = NT - 32;  // lane 0 of the last warp: no halo role (warps 0-2 carry those)
constexpr int PW = TX + 2, PH = TY + 2;  // derived planes: tile + ring, 34 x 18
// Slot layouts in floats; every sub-buffer starts on a 128-byte boundary.
template <bool FIRST> struct Slot;
template <> struct Slot<true> {  // rho, theta with the ring (pressure derived), heights
  static constexpr int O_RHO = 0, O_TH = 736, O_Z = 1472, O_P = 0, O_DU = 0, O_DV = 0, O_DW = 0, SIZE = 2208,
                       RW = CBW, R0 = 1, C0 = 4;
};
template <> struct Slot<false> {  // owned rho, theta; heights and pressure with the ring; increments
  static constexpr int O_RHO = 0, O_TH = 512, O_Z = 1024, O_P = 1760, O_DU = 2496, O_DV = 3136, O_DW = 3776,
                       SIZE = 4288, RW = OBW, R0 = 0, C0 = 0;
};
template <bool FIRST>
constexpr bool slot_ok() {
  using L = Slot<FIRST>;
  constexpr int rb = FIRST ? CBW * CBH : OBW * OBH;
  return L::O_TH % 32 == 0 && L::O_Z % 32 == 0 && L::SIZE % 32 == 0 && L::O_TH - L::O_RHO >= rb &&
         L::O_Z - L::O_TH >= rb &&
         (FIRST ? L::SIZE - L::O_Z >= CBW * CBH
                : (L::O_P % 32 == 0 && L::O_DU % 32 == 0 && L::O_DV % 32 == 0 && L::O_DW % 32 == 0 &&
                   L::O_P - L::O_Z >= CBW * CBH && L::O_DU - L::O_P >= CBW * CBH && L::O_DV - L::O_DU >= FBW * FBH &&
                   L::O_DW - L::O_DV >= FBW * FBH && L::SIZE - L::O_DW >= OBW * OBH));
}
static_assert(slot_ok<true>() && slot_ok<false>(), "128-byte aligned sub-buffers that fit their boxes");
template <bool FIRST>
constexpr size_t dyn_smem() {
  return size_t(Slot<FIRST>::SIZE) * NSLOT * sizeof(float) + 128;
}
}  // namespace fz

// Derived planes and per-CTA state besides the ring.  p: the full pressure of the tile
// and its ring, three planes (first substep only; later substeps read it from the ring).
template <bool FIRST>
struct TerrainShared {
  float p[FIRST ? 3 : 1][fz::PH][fz::PW];
  float dz[2][fz::PH][fz::PW];     // dp/dz of the tile and its ring (column_dpdz)
  float du[2][fz::TY][fz::TX + 1];  // new X-face increments (own + east face)
  float dv[2][fz::TY + 1][fz::TX];  // new Y-face increments (own + north face)
  long long red[2][fz::NW][2];
  __align__(8) uint64_t bar[fz::NSLOT];
  int abort[2];
};

// Owned-cell columns of one plane, loaded a plane ahead of their use.
struct TerrainCol {
  float idzc, idzf, pref, rref, bu, bv, bw;  // idzf, bw: face k+1; pref, rref: level k+1
};

template <bool FIRST>
__global__ void __launch_bounds__(fz::NT, 2)
    k_fast_terrain_tma(const FastArgs a, const __grid_constant__ FastTerrainMaps m) {
  using namespace fz;
  using L = Slot<FIRST>;
  constexpr int O_RHO = L::O_RHO, O_TH = L::O_TH, O_Z = L::O_Z, O_P = L::O_P, O_DU = L::O_DU, O_DV = L::O_DV,
                O_DW = L::O_DW, RW = L::RW, R0 = L::R0, C0 = L::C0, SLOT = L::SIZE;
  extern __shared__ unsigned char s_dyn[];
  __shared__ TerrainShared<FIRST> S;
  float* const ring = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(s_dyn) + 127) & ~uintptr_t(127));

  const Geom& g = a.g;
  const int nz = g.nz;
  const bool final_step = a.final_kind == 2;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int nx = g.nx, ny = g.ny;
  const int w = min(TX, nx - i0), h = min(TY, ny - j0);
  const bool own0 = tx < w && ty < h, own1 = tx < w && ty + RY < h;
  const int gi = i0 + tx, gj0 = j0 + ty, gj1 = j0 + ty + RY;
  const bool skip_u = gi == 0 && !g.per_x;  // open west face (never changes)
  const bool skip_v0 = gj0 == 0 && !g.per_y;
  const bool edge = (g.per_x && (i0 <= 1 || i0 + w >= nx - 1)) || (g.per_y && (j0 <= 1 || j0 + h >= ny - 1));
  // halo roles (threads 0-95, whole warps): 0 west column, 1 east column, 2 south row,
  // 3 north row; (hr, hc) in derived-plane coordinates (row 0 = j0-1, column 0 = i0-1)
  int role = -1, hr = 0, hc = 0;
  if (tid < TY) { if (tid < h) { role = 0; hr = tid + 1; hc = 0; } }
  else if (tid < 2 * TY) { if (tid - TY < h) { role = 1; hr = tid - TY + 1; hc = w + 1; } }
  else if (tid < 2 * TY + TX) { if (tid - 2 * TY < w) { role = 2; hr = 0; hc = tid - 2 * TY + 1; } }
  else if (tid < 2 * TY + 2 * TX) { if (tid - 2 * TY - TX < w) { role = 3; hr = h + 1; hc = tid - 2 * TY - TX + 1; } }
  const int hi = i0 + hc - 1, hj = j0 + hr - 1;  // global cell of the halo role
  const bool h_skip = (role == 1 && hi == nx && !g.per_x) || (role == 3 && hj == ny && !g.per_y);
  const float idx = g.inv_dx, idy = g.inv_dy, dtf = a.dtf;
  // terrain: no reference level sums; theta level sums of a stage's result
  const int acc_mode = (a.acc_off || a.final_kind == 0) ? 0 : 2;
  const bool hm = a.hmom != 0, dn = a.dens != 0;

  if (tid == 0) {
    for (int s = 0; s < NSLOT; ++s) mbar_init(&S.bar[s], 1);
    mbar_fence_init();
    S.abort[0] = 0;
    S.abort[1] = 0;
  }
  if (blockIdx.x == 0 && blockIdx.y == 0 && a.clr_a)
    for (int q = tid; q < nz; q += NT) { a.clr_a[q] = 0ull; a.clr_b[q] = 0ull; }
  __syncthreads();

  // err[1] > 0 (set only by failure-path tests): the first CTA to see it leaves the loads
  // of plane err[1] - 1 unissued, so that CTA's bounded wait runs out
  int stall = -1;
  if (tid == ISSUER && *(volatile int*)(a.err + 1) > 0) stall = atomicExch(a.err + 1, 0) - 1;
  auto issue = [&](int kk) {
    float* st = ring + (kk % NSLOT) * SLOT;
    uint64_t* bar = &S.bar[kk % NSLOT];
    const bool wface = kk + 1 < nz;
    unsigned bytes = FIRST ? 3 * B_CELL : 2 * B_OWN + 2 * B_CELL + 2 * B_FACE + (wface ? B_OWN : 0u);
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(bar, bytes);
    if (kk == stall) return;  // failure-path testing: this plane's loads stay unissued
    if (FIRST) {
      tma_load_3d(st + O_RHO, &m.rho, i0 + kXOff - 4, j0, kk, bar);
      tma_load_3d(st + O_TH, &m.th, i0 + kXOff - 4, j0, kk, bar);
    } else {
      tma_load_3d(st + O_RHO, &m.rho, i0 + kXOff, j0 + 1, kk, bar);
      tma_load_3d(st + O_TH, &m.th, i0 + kXOff, j0 + 1, kk, bar);
      tma_load_3d(st + O_P, &m.p, i0 + kXOff - 4, j0, kk, bar);
      tma_load_3d(st + O_DU, &m.du, i0 + kXOff, j0 + 1, kk, bar);
      tma_load_3d(st + O_DV, &m.dv, i0 + kXOff, j0 + 1, kk, bar);
      if (wface) tma_load_3d(st + O_DW, &m.dw, i0 + kXOff, j0 + 1, kk + 1, bar);
    }
    tma_load_3d(st + O_Z, &m.z, i0 + kXOff - 4, j0, kk, bar);
  };
  int issued = -1, waited = -1;
  auto wait_plane = [&](int kk, int epoch) {
    if (!mbar_wait(&S.bar[kk % NSLOT], (kk / NSLOT) & 1)) {
      S.abort[epoch & 1] = 1;
      atomicExch(a.err, 1);
    } else {
      waited = kk;  // a plane whose wait gave up stays in the drain below
    }
  };
  auto slot_of = [&](int kk) { return ring + (kk % NSLOT) * SLOT; };
  // values of plane kk at derived-plane position (r, c)
  auto Pv = [&](int kk, int r, int c) {
    if constexpr (FIRST) return S.p[kk % 3][r][c];
    else return slot_of(kk)[O_P + r * CBW + c + 3];
  };
  auto Zv = [&](int kk, int r, int c) { return slot_of(kk)[O_Z + r * CBW + c + 3]; };
  // K10 + K20 (first substep): the full pressure of plane kk at the thread's positions
  auto derive_p = [&](int kk) {
    if constexpr (FIRST) {
      const float* st = slot_of(kk);
      auto one = [&](int r, int c) {
        const float rho = st[O_RHO + r * CBW + c + 3], th = st[O_TH + r * CBW + c + 3];
        S.p[kk % 3][r][c] = eos_pressure(rho, fp::mul(rho, th));
      };
      if (own0) one(ty + 1, tx + 1);
      if (own1) one(ty + RY + 1, tx + 1);
      if (role >= 0) one(hr, hc);
    }
  };
  // dp/dz of plane kk at the thread's positions (planes kk-1 .. kk+1 resident)
  auto derive_dz = [&](int kk) {
    auto one = [&](int r, int c) {
      const float pc = Pv(kk, r, c), zc = Zv(kk, r, c);
      const float pm = kk > 0 ? Pv(kk - 1, r, c) : 0.f, zm = kk > 0 ? Zv(kk - 1, r, c) : 0.f;
      const float pn = kk + 1 < nz ? Pv(kk + 1, r, c) : 0.f, zn = kk + 1 < nz ? Zv(kk + 1, r, c) : 0.f;
      S.dz[kk & 1][r][c] = column_dpdz(kk, nz, pm, pc, pn, zm, zc, zn);
    };
    if (own0) one(ty + 1, tx + 1);
    if (own1) one(ty + RY + 1, tx + 1);
    if (role >= 0) one(hr, hc);
  };
  // owned-cell columns of plane kk (zeros above the top)
  auto load_col = [&](bool own, int gj, int kk) {
    TerrainCol c{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (!own || kk >= nz) return c;
    const int o = gidx(g, gi, gj, kk);
    c.idzc = __ldg(a.idz_c + o);
    if (kk + 1 < nz) {
      c.idzf = __ldg(a.idz_f + o + g.plane);
      c.pref = __ldg(a.col_pref + o + g.plane);
      c.rref = __ldg(a.col_rref + o + g.plane);
    }
    if (final_step) {
      c.bu = __ldg(a.bu + o);
      c.bv = __ldg(a.bv + o);
      c.bw = __ldg(a.bw + o + g.plane);
    }
    return c;
  };

  if (tid == ISSUER) {
    for (int kk = 0; kk < AHEAD && kk < nz; ++kk) { issue(kk); issued = kk; }
  }
  // the column reference at level 0 and the step's bottom face
  float prc0 = 0.f, rrc0 = 0.f, prc1 = 0.f, rrc1 = 0.f, bwz0 = 0.f, bwz1 = 0.f;
  if (own0) {
    const int o = gidx(g, gi, gj0, 0);
    prc0 = __ldg(a.col_pref + o); rrc0 = __ldg(a.col_rref + o);
    if (final_step) bwz0 = __ldg(a.bw + o);
  }
  if (own1) {
    const int o = gidx(g, gi, gj1, 0);
    prc1 = __ldg(a.col_pref + o); rrc1 = __ldg(a.col_rref + o);
    if (final_step) bwz1 = __ldg(a.bw + o);
  }
  TerrainCol c0 = load_col(own0, gj0, 0), c1 = load_col(own1, gj1, 0);
  wait_plane(0, 0);
  derive_p(0);
  if (nz > 1) {
    wait_plane(1, 0);
    derive_p(1);
  }
  derive_dz(0);
  float dwc0 = 0.f, dwc1 = 0.f;  // increment at face k (face 0 never changes)
  __syncthreads();

  // Interior tiles (full, away from every periodic edge ring and open side) run a copy
  // of the plane loop compiled without the edge logic; both copies do the same arithmetic.
  const bool interior = !edge && (g.per_x || (i0 > 0 && i0 + TX < nx)) && (g.per_y || (j0 > 0 && j0 + TY < ny));
  auto plane_loop = [&](auto tile_class) -> bool {  // true when a bounded wait gave up
    constexpr bool IN = decltype(tile_class)::value;
    const bool o0 = IN || own0, o1 = IN || own1;
    const bool su = !IN && skip_u, sv = !IN && skip_v0, hs = !IN && h_skip;
    auto put = [&](float* f, const Geom& gg, int o, int i, int j, int kk, float v) {
      if (IN) f[gidx(gg, i, j, kk)] = v;
      else store_tile(f, gg, o, i, j, kk, v, edge);
    };
    for (int k = 0; k < nz; ++k) {
      const int pb = k & 1;
      const float* st = slot_of(k);
      const float* stn = slot_of(k + 1);
      const TerrainCol n0 = load_col(o0, gj0, k + 1), n1 = load_col(o1, gj1, k + 1);
      // ---- dp/dz of plane k+1 (plane k+2 arrives first)
      if (k + 2 < nz) {
        wait_plane(k + 2, k);
        derive_p(k + 2);
      }
      if (k + 1 < nz) derive_dz(k + 1);
      // ---- faces of plane k: K12/K13 horizontal momenta, K14 vertical momentum at face k+1
      auto P0 = [&](int r, int c) { return Pv(k, r, c); };
      auto Z0 = [&](int r, int c) { return st[O_Z + r * CBW + c + 3]; };
      auto D0 = [&](int r, int c) { return S.dz[pb][r][c]; };
      float du0 = 0.f, dv0 = 0.f, du1 = 0.f, dv1 = 0.f, dw0 = 0.f, dw1 = 0.f;
      if (!FIRST) {
        du0 = st[O_DU + ty * FBW + tx];
        dv0 = st[O_DV + ty * FBW + tx];
        du1 = st[O_DU + (ty + RY) * FBW + tx];
        dv1 = st[O_DV + (ty + RY) * FBW + tx];
        if (k + 1 < nz) { dw0 = st[O_DW + ty * OBW + tx]; dw1 = st[O_DW + (ty + RY) * OBW + tx]; }
      }
      const int r0 = ty + 1, r1 = ty + RY + 1, cc = tx + 1;
      const float pc0 = P0(r0, cc), pc1 = P0(r1, cc);
      float un0 = du0, vn0 = dv0, un1 = du1, vn1 = dv1;
      if (hm) {
        if (!su) {
          un0 = fp::hmom_terrain(du0, pc0, P0(r0, cc - 1), Z0(r0, cc), Z0(r0, cc - 1), D0(r0, cc - 1), D0(r0, cc), idx,
                                 dtf);
          un1 = fp::hmom_terrain(du1, pc1, P0(r1, cc - 1), Z0(r1, cc), Z0(r1, cc - 1), D0(r1, cc - 1), D0(r1, cc), idx,
                                 dtf);
        }
        if (!sv)
          vn0 = fp::hmom_terrain(dv0, pc0, P0(r0 - 1, cc), Z0(r0, cc), Z0(r0 - 1, cc), D0(r0 - 1, cc), D0(r0, cc), idy,
                                 dtf);
        vn1 = fp::hmom_terrain(dv1, pc1, P0(r1 - 1, cc), Z0(r1, cc), Z0(r1 - 1, cc), D0(r1 - 1, cc), D0(r1, cc), idy,
                               dtf);
      }
      if (o0) { S.du[pb][ty][tx] = un0; S.dv[pb][ty][tx] = vn0; }
      if (o1) { S.du[pb][ty + RY][tx] = un1; S.dv[pb][ty + RY][tx] = vn1; }
      if (role == 1) {  // the tile's east X face
        float d = FIRST ? 0.f : st[O_DU + (hr - 1) * FBW + w];
        if (hm && !hs)
          d = fp::hmom_terrain(d, P0(hr, hc), P0(hr, hc - 1), Z0(hr, hc), Z0(hr, hc - 1), D0(hr, hc - 1), D0(hr, hc),
                               idx, dtf);
        S.du[pb][hr - 1][w] = d;
        // open east boundary: face nx belongs to no tile; its step value is base + increment
        if (final_step && hs) {
          const int o = gidx(g, hi, hj, k);
          a.f_u[o] = fp::add(__ldg(a.bu + o), d);
        }
      } else if (role == 3) {  // the tile's north Y face
        float d = FIRST ? 0.f : st[O_DV + h * FBW + hc - 1];
        if (hm && !hs)
          d = fp::hmom_terrain(d, P0(hr, hc), P0(hr - 1, hc), Z0(hr, hc), Z0(hr - 1, hc), D0(hr - 1, hc), D0(hr, hc),
                               idy, dtf);
        S.dv[pb][h][hc - 1] = d;
        if (final_step && hs) {
          const int o = gidx(g, hi, hj, k);
          a.f_v[o] = fp::add(__ldg(a.bv + o), d);
        }
      }
      const float rc0 = st[O_RHO + (ty + R0) * RW + tx + C0], rc1 = st[O_RHO + (ty + RY + R0) * RW + tx + C0];
      float wn0 = dw0, wn1 = dw1;
      if (k + 1 < nz) {
        const float pn0 = Pv(k + 1, r0, cc), pn1 = Pv(k + 1, r1, cc);
        const float rn0 = stn[O_RHO + (ty + R0) * RW + tx + C0], rn1 = stn[O_RHO + (ty + RY + R0) * RW + tx + C0];
        wn0 = fp::wmom(dw0, pn0, c0.pref, pc0, prc0, rc0, rrc0, rn0, c0.rref, c0.idzf, a.gravity, dtf);
        wn1 = fp::wmom(dw1, pn1, c1.pref, pc1, prc1, rc1, rrc1, rn1, c1.rref, c1.idzf, a.gravity, dtf);
      }
      __syncthreads();  // publishes dz(k+1), p(k+2), du(k), dv(k); the slot of plane k-1 is free
      if (S.abort[pb]) return true;
      if (tid == ISSUER) {
        if (acc_mode && k > 0) {  // level sums of plane k-1 (warp totals published above)
          long long sa = 0;
          for (int q = 0; q < NW; ++q) sa += S.red[pb ^ 1][q][0];
          acc_add(a.acc_a + k - 1, sa);
        }
        if (k + AHEAD < nz) { issue(k + AHEAD); issued = k + AHEAD; }
      }
      // ---- K15 density of plane k, K10 rho*theta, stores
      FxAcc sa;
      auto cell = [&](bool o, int row, int gj, float rc, float un, float vn, float wn, float dwc, const TerrainCol& cl,
                      float bwz) {
        if (!o) return;
        float rn = rc;
        if (dn) rn = fp::density(rc, S.du[pb][row][tx + 1], un, S.dv[pb][row + 1][tx], vn, wn, dwc, idx, idy, cl.idzc, dtf);
        const float rt = fp::mul(rn, st[O_TH + (row + R0) * RW + tx + C0]);
        if (final_step) {
          put(a.f_rho, g, kCell, gi, gj, k, rn);
          put(a.f_rt, g, kCell, gi, gj, k, rt);
          put(a.f_u, g, kFaceX, gi, gj, k, fp::add(cl.bu, un));
          put(a.f_v, g, kFaceY, gi, gj, k, fp::add(cl.bv, vn));
          if (k == 0) put(a.f_w, g, kFaceZ, gi, gj, 0, bwz);
          put(a.f_w, g, kFaceZ, gi, gj, k + 1, fp::add(cl.bw, wn));
        } else {
          put(a.rho_out, g, kCell, gi, gj, k, rn);
          put(a.du_out, g, kFaceX, gi, gj, k, un);
          put(a.dv_out, g, kFaceY, gi, gj, k, vn);
          if (k + 1 < nz) put(a.dw_out, g, kFaceZ, gi, gj, k + 1, wn);
          // the next substep's pressure, loaded with its ring
          if (a.final_kind == 0) put(a.p_out, g, kCell, gi, gj, k, eos_pressure(rn, rt));
        }
        if (acc_mode == 2) sa.add(fp::theta(rn, rt), kFxTheta);
      };
      cell(o0, ty, gj0, rc0, un0, vn0, wn0, dwc0, c0, bwz0);
      cell(o1, ty + RY, gj1, rc1, un1, vn1, wn1, dwc1, c1, bwz1);
      if (acc_mode) {
        const long long ta = sa.warp_total();
        if (tx == 0) S.red[pb][ty][0] = ta;
      }
      dwc0 = wn0;
      dwc1 = wn1;
      prc0 = c0.pref; rrc0 = c0.rref;
      prc1 = c1.pref; rrc1 = c1.rref;
      c0 = n0;
      c1 = n1;
    }
    return false;
  };
  const bool aborted = interior ? plane_loop(std::true_type{}) : plane_loop(std::false_type{});
  if (aborted) {
    // drain the tiles still in flight (bounded) before the CTA's shared memory goes away
    if (tid == ISSUER)
      for (int kk = waited + 1; kk <= issued; ++kk) mbar_wait(&S.bar[kk % NSLOT], (kk / NSLOT) & 1);
    return;
  }
  if (acc_mode) {
    __syncthreads();  // the last plane's warp totals
    if (tid == ISSUER) {
      const int pb = (nz - 1) & 1;
      long long sa = 0;
      for (int q = 0; q < NW; ++q) sa += S.red[pb][q][0];
      acc_add(a.acc_a + nz - 1, sa);
    }
  }
}

}  // namespace

cudaError_t init_fast_terrain_tma() {
  cudaError_t e = cudaFuncSetAttribute(k_fast_terrain_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)fz::dyn_smem<true>());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_fast_terrain_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)fz::dyn_smem<false>());
  return e;
}

cudaError_t launch_fast_terrain_tma(const FastArgs& a, const FastTerrainMaps& m, bool first, cudaStream_t s) {
  if (a.g.nz > kMaxNz || a.g.nz < 1 || !a.err || !a.col_pref || !a.col_rref || !a.idz_c || !a.idz_f ||
      (a.final_kind == 0 && !a.p_out) || (a.final_kind == 2 && (!a.bu || !a.bv || !a.bw)))
    return cudaErrorInvalidValue;
  const dim3 block(fz::TX, fz::RY);
  const dim3 grid((a.g.nx + fz::TX - 1) / fz::TX, (a.g.ny + fz::TY - 1) / fz::TY);
  if (first) k_fast_terrain_tma<true><<<grid, block, fz::dyn_smem<true>(), s>>>(a, m);
  else k_fast_terrain_tma<false><<<grid, block, fz::dyn_smem<false>(), s>>>(a, m);
  return cudaGetLastError();
}

}  // namespace gwmb
