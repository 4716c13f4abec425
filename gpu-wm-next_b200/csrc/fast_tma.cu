// fast_tma.cu — acoustic substep (flat terrain) fed by TMA tile loads.
//
// Same operator as k_fast_flat (LocalSplitExplicitFastMode::apply,
// dry_fast_modes.cu:400-656, K9-K15 on one substep) and the same per-cell
// arithmetic, with a different data path: one elected thread per CTA fetches every
// plane's tiles with cp.async.bulk.tensor.3d into a four-slot shared-memory ring,
// three planes ahead of the compute, and the 256 threads work from shared memory.
// Per plane k the ring slot holds
//   rho(k), theta(k)        first substep of a stage deriving p': 40 x 18 boxes, columns
//                           i0-4 .. i0+35, rows j0-1 .. j0+16 (the owned 32 x 16 tile and
//                           its one-cell halo ring, from which p' is derived; the box starts
//                           4 columns left so x stays 16-byte aligned); otherwise the owned
//                           32 x 16 box (p' comes with its halo below)
//   du(k), dv(k)            36 x 17 box: owned faces plus the tile's east/north face
//   dw(k+1)                 32 x 16 box: owned Z faces above the plane
//   p'(k)                   40 x 18 box like the first substep's rho: the pressure
//                           perturbation the previous substep computed for its level sums
//                           (the slow stage, for the first substep of a stage, when it ran
//                           on the TMA path), so the EOS runs once per cell per substep
//   bu(k), bv(k), bw(k+1)   32 x 16 boxes, last substep of the step only (m = B + D)
// so the kernel issues no per-thread global loads on the main path, holds no load
// pipeline in registers and needs no halo threads reading global memory.  The level
// tables (reference means, metric columns, EOS base state) follow the ring in dynamic
// shared memory, sized by nz.
#include <algorithm>
#include <type_traits>

#include "dycore.cuh"
#include "stencil.cuh"
#include "tma.cuh"

namespace gwmb {
namespace {

namespace ft {
constexpr int TX = 32, TY = 16, RY = 8, NT = 256, NW = NT / 32;
constexpr int CBW = 40, CBH = 18;  // cell box
constexpr int FBW = 36, FBH = 17;  // face box (owned faces + east/north face)
constexpr int OBW = 32, OBH = 16;  // owned box
constexpr unsigned B_CELL = CBW * CBH * 4, B_FACE = FBW * FBH * 4, B_OWN = OBW * OBH * 4;
constexpr int NSLOT = 4, AHEAD = NSLOT - 1;  // ring slots; planes in flight beyond the one computed
// the thread that issues the TMA loads and folds the level sums: lane 0 of the last warp,
// which has no halo role (warps 0-2 carry those), so the per-plane serial work does not
// land on a warp that is already the slowest
constexpr int ISSUER = NT - 32;
// Slot layouts in floats; every sub-buffer starts on a 128-byte boundary.  The
// base-momentum boxes are only present, and the slot only that long, in the last
// substep of the step.  RW, R0, C0: row width of the rho/theta boxes and the box
// position of owned cell (0, 0).
template <bool FIRST, bool PIN> struct Slot;  // PIN: p' loaded (with its ring) by TMA
template <> struct Slot<true, false> {  // first substep deriving p': rho, theta with the halo ring
  static constexpr int O_RHO = 0, O_TH = 736, O_DU = 0, O_DV = 0, O_DW = 0, O_P = 0, O_BU = 1472, O_BV = 1984,
                       O_BW = 2496, LONG = 3008, SHORT = 1472, RW = CBW, R0 = 1, C0 = 4;
};
template <> struct Slot<true, true> {  // first substep with p' from the slow stage: owned rho, theta; p'
  static constexpr int O_RHO = 0, O_TH = 512, O_DU = 0, O_DV = 0, O_DW = 0, O_P = 1024, O_BU = 1760,
                       O_BV = 2272, O_BW = 2784, LONG = 3296, SHORT = 1760, RW = OBW, R0 = 0, C0 = 0;
};
template <> struct Slot<false, true> {  // inner substeps: owned rho, theta; increments; p' with its ring
  static constexpr int O_RHO = 0, O_TH = 512, O_DU = 1024, O_DV = 1664, O_DW = 2304, O_P = 2816, O_BU = 3552,
                       O_BV = 4064, O_BW = 4576, LONG = 5088, SHORT = 3552, RW = OBW, R0 = 0, C0 = 0;
};
template <bool FIRST, bool PIN>
constexpr bool slot_ok() {
  using L = Slot<FIRST, PIN>;
  constexpr int rb = (FIRST && !PIN) ? CBW * CBH : OBW * OBH;  // rho, theta boxes
  constexpr int after_th = !FIRST ? L::O_DU : (PIN ? L::O_P : L::O_BU);
  return L::O_TH % 32 == 0 && L::O_BU % 32 == 0 && L::O_BV % 32 == 0 && L::O_BW % 32 == 0 &&
         L::LONG % 32 == 0 && L::SHORT % 32 == 0 && L::SHORT == L::O_BU && L::O_TH - L::O_RHO >= rb &&
         after_th - L::O_TH >= rb &&
         (FIRST || (L::O_DU % 32 == 0 && L::O_DV % 32 == 0 && L::O_DW % 32 == 0 &&
                    L::O_DV - L::O_DU >= FBW * FBH && L::O_DW - L::O_DV >= FBW * FBH &&
                    L::O_P - L::O_DW >= OBW * OBH)) &&
         (!PIN || (L::O_P % 32 == 0 && L::O_BU - L::O_P >= CBW * CBH)) &&
         L::O_BV - L::O_BU >= OBW * OBH && L::O_BW - L::O_BV >= OBW * OBH && L::LONG - L::O_BW >= OBW * OBH;
}
static_assert(slot_ok<true, false>() && slot_ok<true, true>() && slot_ok<false, true>(),
              "128-byte aligned sub-buffers that fit their boxes");
// dynamic shared memory: the ring, then the level tables (2 double + 4 float per level)
constexpr size_t kLevelBytes = 2 * sizeof(double) + 4 * sizeof(float);
template <bool FIRST, bool PIN>
constexpr size_t dyn_smem(bool final_step, int nz) {
  return size_t(final_step ? Slot<FIRST, PIN>::LONG : Slot<FIRST, PIN>::SHORT) * NSLOT * sizeof(float) + 128 +
         kLevelBytes * size_t(nz);
}
}  // namespace ft

// Per-CTA shared state of the substep kernels besides the dynamic ring and level tables.
struct FastShared {
  float p[2][ft::TY + 2][ft::TX + 2];  // pressure perturbation, tile + halo ring (first substep)
  float du[2][ft::TY][ft::TX + 1];     // new X-face increments (own + east face)
  float dv[2][ft::TY + 1][ft::TX];     // new Y-face increments (own + north face)
  long long red[2][ft::NW][2];
  __align__(8) uint64_t bar[ft::NSLOT];
  int abort[2];  // per plane parity: set before barrier k, read after it
};

// Level tables of a substep in dynamic shared memory, after the ring.
struct FastTables {
  double *binv, *bpr;  // EOS base state: 1/rt_ref, p_ref
  float *pref, *rref;  // K6/K7 level means
  float *idzc, *idzf;  // metric columns
};

__device__ __forceinline__ FastTables fast_tables(float* ring, int slot_floats, int nz) {
  FastTables t;
  t.binv = reinterpret_cast<double*>(ring + slot_floats * ft::NSLOT);
  t.bpr = t.binv + nz;
  t.pref = reinterpret_cast<float*>(t.bpr + nz);
  t.rref = t.pref + nz;
  t.idzc = t.rref + nz;
  t.idzf = t.idzc + nz;
  return t;
}

// Start of a substep in a CTA: block 0 clears the level-sum slot of the substep after
// next, every CTA loads the level tables.  Ends with a block barrier.
__device__ __forceinline__ void fast_substep_setup(const FastArgs& a, const FastTables& T, bool first_cta) {
  using namespace ft;
  const int tid = threadIdx.y * TX + threadIdx.x, nz = a.g.nz;
  if (first_cta && a.clr_a)
    for (int q = tid; q < nz; q += NT) { a.clr_a[q] = 0ull; a.clr_b[q] = 0ull; }
  for (int q = tid; q < nz; q += NT) {  // K6/K7 level means; metric columns
    T.rref[q] = (float)(acc_read(a.ref_a + q, kScaleRho) * a.inv_count);
    T.pref[q] = (float)(acc_read(a.ref_b + q, kScaleP) * a.inv_count);
    T.idzc[q] = __ldg(a.idz_c + q);
    T.idzf[q] = __ldg(a.idz_f + q);
    T.binv[q] = __ldg(a.base + nz + q);
    T.bpr[q] = __ldg(a.base + 2 * nz + q);
  }
  __syncthreads();
}

// One tile (bx, by) of one acoustic substep: K9-K15 plane by plane over the TMA ring.
// FIRST: the first substep of a stage (no increments in).  PIN: p' of the input (with its
// ring) is loaded; otherwise (first substep only) it is derived from rho and theta.
// The ring's planes are counted across the tiles a CTA runs: plane kk of this tile is
// ring plane base + kk (its slot and barrier phase).  stall >= 0 (failure-path tests
// only) leaves that plane's loads unissued.  Returns true when a bounded wait gave up;
// the tile's loads in flight are drained first.
template <bool FIRST, bool PIN>
__device__ __forceinline__ bool fast_tile(const FastArgs& a, const FastMaps& m, int bx, int by, FastShared& S,
                                          float* ring, const FastTables& T, unsigned base, int stall) {
  using namespace ft;
  using L = Slot<FIRST, PIN>;
  constexpr int O_RHO = L::O_RHO, O_TH = L::O_TH, O_DU = L::O_DU, O_DV = L::O_DV, O_DW = L::O_DW, O_P = L::O_P,
                O_BU = L::O_BU, O_BV = L::O_BV, O_BW = L::O_BW, RW = L::RW, R0 = L::R0, C0 = L::C0;
  const int nz = a.g.nz;
  const bool final_step = a.final_kind == 2;
  const int slot = final_step ? L::LONG : L::SHORT;

  const Geom& g = a.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = bx * TX, j0 = by * TY;
  const int nx = g.nx, ny = g.ny;
  const int w = min(TX, nx - i0), h = min(TY, ny - j0);
  const bool own0 = tx < w && ty < h, own1 = tx < w && ty + RY < h;
  const int gi = i0 + tx, gj0 = j0 + ty, gj1 = j0 + ty + RY;
  const bool skip_u = gi == 0 && !g.per_x;  // open west face (never changes)
  const bool skip_v0 = gj0 == 0 && !g.per_y;
  const bool edge = (g.per_x && (i0 <= 1 || i0 + w >= nx - 1)) || (g.per_y && (j0 <= 1 || j0 + h >= ny - 1));
  // halo roles (threads 0-95, whole warps): 0 west column, 1 east column, 2 south row,
  // 3 north row; (hr, hc) are s_p coordinates (row 0 = j0-1, column 0 = i0-1)
  int role = -1, hr = 0, hc = 0;
  if (tid < TY) { if (tid < h) { role = 0; hr = tid + 1; hc = 0; } }
  else if (tid < 2 * TY) { if (tid - TY < h) { role = 1; hr = tid - TY + 1; hc = w + 1; } }
  else if (tid < 2 * TY + TX) { if (tid - 2 * TY < w) { role = 2; hr = 0; hc = tid - 2 * TY + 1; } }
  else if (tid < 2 * TY + 2 * TX) { if (tid - 2 * TY - TX < w) { role = 3; hr = h + 1; hc = tid - 2 * TY - TX + 1; } }
  const int hi = i0 + hc - 1, hj = j0 + hr - 1;  // global cell of the halo role
  const bool h_skip = (role == 1 && hi == nx && !g.per_x) || (role == 3 && hj == ny && !g.per_y);
  const float idx = g.inv_dx, idy = g.inv_dy, dtf = a.dtf;
  const int acc_mode = a.acc_off ? 0 : (a.final_kind == 0 ? 1 : 2);
  const bool hm = a.hmom != 0, dn = a.dens != 0;

  // producer: all tiles of plane kk into slot (base + kk) % NSLOT, completing on its barrier
  auto issue = [&](int kk) {
    float* st = ring + ((base + kk) % NSLOT) * slot;
    uint64_t* bar = &S.bar[(base + kk) % NSLOT];
    const bool wface = kk + 1 < nz;
    unsigned bytes = (FIRST && !PIN) ? 2 * B_CELL : 2 * B_OWN;
    if (!FIRST) bytes += 2 * B_FACE + (wface ? B_OWN : 0u);
    if (PIN) bytes += B_CELL;
    if (final_step) bytes += 3 * B_OWN;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(bar, bytes);
    if (kk == stall) return;  // failure-path testing: this plane's loads stay unissued
    if (FIRST && !PIN) {  // with the halo ring
      tma_load_3d(st + O_RHO, &m.rho, i0 + kXOff - 4, j0, kk, bar);
      tma_load_3d(st + O_TH, &m.th, i0 + kXOff - 4, j0, kk, bar);
    } else {  // owned cells
      tma_load_3d(st + O_RHO, &m.rho, i0 + kXOff, j0 + 1, kk, bar);
      tma_load_3d(st + O_TH, &m.th, i0 + kXOff, j0 + 1, kk, bar);
    }
    if (!FIRST) {
      tma_load_3d(st + O_DU, &m.du, i0 + kXOff, j0 + 1, kk, bar);
      tma_load_3d(st + O_DV, &m.dv, i0 + kXOff, j0 + 1, kk, bar);
      if (wface) tma_load_3d(st + O_DW, &m.dw, i0 + kXOff, j0 + 1, kk + 1, bar);
    }
    if (PIN) tma_load_3d(st + O_P, &m.p, i0 + kXOff - 4, j0, kk, bar);
    if (final_step) {
      tma_load_3d(st + O_BU, &m.bu, i0 + kXOff, j0 + 1, kk, bar);
      tma_load_3d(st + O_BV, &m.bv, i0 + kXOff, j0 + 1, kk, bar);
      tma_load_3d(st + O_BW, &m.bw, i0 + kXOff, j0 + 1, kk + 1, bar);
    }
  };
  int issued = -1, waited = -1;  // planes issued / waited for (producer bookkeeping)
  auto wait_plane = [&](int kk, int epoch) {
    if (!mbar_wait(&S.bar[(base + kk) % NSLOT], ((base + kk) / NSLOT) & 1)) {
      S.abort[epoch & 1] = 1;
      atomicExch(a.err, 1);
    } else {
      waited = kk;  // a plane whose wait gave up stays in the drain below
    }
  };
  // K10 + K20: pressure perturbation of plane kk at the owned cells and the halo ring
  auto cell_p = [&](const float* st, int r, int c, int kk) {
    const float rho = st[O_RHO + r * CBW + c + 3], th = st[O_TH + r * CBW + c + 3];
    return eos_pprime_ref(rho, fp::mul(rho, th), T.binv[kk], T.bpr[kk]);
  };
  auto plane_p = [&](int kk) {
    const float* st = ring + ((base + kk) % NSLOT) * slot;
    float(*sp)[TX + 2] = S.p[kk & 1];
    if (own0) sp[ty + 1][tx + 1] = cell_p(st, ty + 1, tx + 1, kk);
    if (own1) sp[ty + RY + 1][tx + 1] = cell_p(st, ty + RY + 1, tx + 1, kk);
    if (role >= 0) sp[hr][hc] = cell_p(st, hr, hc, kk);
  };

  if (tid == ISSUER) {
    issue(0);
    issued = 0;
    for (int kk = 1; kk < AHEAD && kk < nz; ++kk) { issue(kk); issued = kk; }
  }
  wait_plane(0, 0);
  if (FIRST && !PIN) plane_p(0);
  float dwc0 = 0.f, dwc1 = 0.f;  // increment at face k (face 0 never changes)
  float bwz0 = 0.f, bwz1 = 0.f;  // base momentum at face 0 (last substep of the step)
  if (final_step) {
    if (own0) bwz0 = __ldg(a.bw + gidx(g, gi, gj0, 0));
    if (own1) bwz1 = __ldg(a.bw + gidx(g, gi, gj1, 0));
  }
  __syncthreads();

  // Interior tiles (full, away from every periodic edge ring and open side) run a copy
  // of the plane loop compiled without the edge logic: plain stores instead of the
  // periodic mirror stores, and none of the open-boundary face tests.  Both copies do
  // the same arithmetic on the same values.
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
      const float* st = ring + ((base + k) % NSLOT) * slot;
      const float* stn = ring + ((base + k + 1) % NSLOT) * slot;
      // ---- pressure perturbation of plane k+1 (its tiles were issued a plane ago)
      if (k + 1 < nz) {
        wait_plane(k + 1, k);
        if (FIRST && !PIN) plane_p(k + 1);
      }
      // ---- faces of plane k: K12/K13 horizontal momenta, K14 vertical momentum at face k+1
      // p'(r, c) of plane k (P0) and k+1 (P1) in s_p coordinates (row 0 = j0-1, column
      // 0 = i0-1): loaded with the tiles, or derived above in a first substep
      auto P0 = [&](int r, int c) { return PIN ? st[O_P + r * CBW + c + 3] : S.p[pb][r][c]; };
      auto P1 = [&](int r, int c) { return PIN ? stn[O_P + r * CBW + c + 3] : S.p[pb ^ 1][r][c]; };
      float du0 = 0.f, dv0 = 0.f, du1 = 0.f, dv1 = 0.f, dw0 = 0.f, dw1 = 0.f;
      if (!FIRST) {
        du0 = st[O_DU + ty * FBW + tx];
        dv0 = st[O_DV + ty * FBW + tx];
        du1 = st[O_DU + (ty + RY) * FBW + tx];
        dv1 = st[O_DV + (ty + RY) * FBW + tx];
        if (k + 1 < nz) { dw0 = st[O_DW + ty * OBW + tx]; dw1 = st[O_DW + (ty + RY) * OBW + tx]; }
      }
      const float pc0 = P0(ty + 1, tx + 1), pc1 = P0(ty + RY + 1, tx + 1);
      float un0 = du0, vn0 = dv0, un1 = du1, vn1 = dv1;
      if (hm) {
        if (!su) {
          un0 = fp::hmom(du0, pc0, P0(ty + 1, tx), idx, dtf);
          un1 = fp::hmom(du1, pc1, P0(ty + RY + 1, tx), idx, dtf);
        }
        if (!sv) vn0 = fp::hmom(dv0, pc0, P0(ty, tx + 1), idy, dtf);
        vn1 = fp::hmom(dv1, pc1, P0(ty + RY, tx + 1), idy, dtf);
      }
      if (o0) { S.du[pb][ty][tx] = un0; S.dv[pb][ty][tx] = vn0; }
      if (o1) { S.du[pb][ty + RY][tx] = un1; S.dv[pb][ty + RY][tx] = vn1; }
      if (role == 1) {  // the tile's east X face
        float d = FIRST ? 0.f : st[O_DU + (hr - 1) * FBW + w];
        if (hm && !hs) d = fp::hmom(d, P0(hr, hc), P0(hr, hc - 1), idx, dtf);
        S.du[pb][hr - 1][w] = d;
        // open east boundary: face nx belongs to no tile; its step value is base + increment
        if (final_step && hs) {
          const int o = gidx(g, hi, hj, k);
          a.f_u[o] = fp::add(__ldg(a.bu + o), d);
        }
      } else if (role == 3) {  // the tile's north Y face
        float d = FIRST ? 0.f : st[O_DV + h * FBW + hc - 1];
        if (hm && !hs) d = fp::hmom(d, P0(hr, hc), P0(hr - 1, hc), idy, dtf);
        S.dv[pb][h][hc - 1] = d;
        if (final_step && hs) {
          const int o = gidx(g, hi, hj, k);
          a.f_v[o] = fp::add(__ldg(a.bv + o), d);
        }
      }
      const float rc0 = st[O_RHO + (ty + R0) * RW + tx + C0], rc1 = st[O_RHO + (ty + RY + R0) * RW + tx + C0];
      float wn0 = dw0, wn1 = dw1;
      if (k + 1 < nz) {
        const float prl = T.pref[k], pru = T.pref[k + 1], rrl = T.rref[k], rru = T.rref[k + 1];
        const float idzf = T.idzf[k + 1];
        const float pn0 = P1(ty + 1, tx + 1), pn1 = P1(ty + RY + 1, tx + 1);
        const float rn0 = stn[O_RHO + (ty + R0) * RW + tx + C0], rn1 = stn[O_RHO + (ty + RY + R0) * RW + tx + C0];
        wn0 = fp::wmom(dw0, pn0, pru, pc0, prl, rc0, rrl, rn0, rru, idzf, a.gravity, dtf);
        wn1 = fp::wmom(dw1, pn1, pru, pc1, prl, rc1, rrl, rn1, rru, idzf, a.gravity, dtf);
      }
      __syncthreads();  // publishes s_p(k+1), s_du(k), s_dv(k); the slot of plane k-1 is free
      if (S.abort[pb]) return true;
      if (tid == ISSUER) {
        if (acc_mode && k > 0) {  // level sums of plane k-1 (warp totals published above)
          long long sa = 0, sb = 0;
          for (int q = 0; q < NW; ++q) { sa += S.red[pb ^ 1][q][0]; sb += S.red[pb ^ 1][q][1]; }
          acc_add(a.acc_a + k - 1, sa);
          if (acc_mode == 1) acc_add(a.acc_b + k - 1, sb);
        }
        if (k + AHEAD < nz) { issue(k + AHEAD); issued = k + AHEAD; }
      }
      // ---- K15 density of plane k, K10 rho*theta, stores
      const float idzc = T.idzc[k];
      FxAcc sa, sb;
      if (o0) {
        float rn = rc0;
        if (dn) {
          rn = fp::density(rc0, S.du[pb][ty][tx + 1], un0, S.dv[pb][ty + 1][tx], vn0, wn0, dwc0, idx, idy, idzc, dtf);
        }
        const float rt = fp::mul(rn, st[O_TH + (ty + R0) * RW + tx + C0]);
        if (final_step) {
          put(a.f_rho, g, kCell, gi, gj0, k, rn);
          put(a.f_rt, g, kCell, gi, gj0, k, rt);
          put(a.f_u, g, kFaceX, gi, gj0, k, fp::add(st[O_BU + ty * OBW + tx], un0));
          put(a.f_v, g, kFaceY, gi, gj0, k, fp::add(st[O_BV + ty * OBW + tx], vn0));
          if (k == 0) put(a.f_w, g, kFaceZ, gi, gj0, 0, bwz0);
          put(a.f_w, g, kFaceZ, gi, gj0, k + 1, fp::add(st[O_BW + ty * OBW + tx], wn0));
        } else {
          put(a.rho_out, g, kCell, gi, gj0, k, rn);
          put(a.du_out, g, kFaceX, gi, gj0, k, un0);
          put(a.dv_out, g, kFaceY, gi, gj0, k, vn0);
          if (k + 1 < nz) put(a.dw_out, g, kFaceZ, gi, gj0, k + 1, wn0);
        }
        if (acc_mode == 1) {
          const float pv = eos_pprime_ref(rn, rt, T.binv[k], T.bpr[k]);
          sa.add(rn, kFxRho);
          sb.add(pv, kFxP);
          put(a.p_out, g, kCell, gi, gj0, k, pv);
        }
        else if (acc_mode == 2) sa.add(fp::theta(rn, rt), kFxTheta);
      }
      if (o1) {
        float rn = rc1;
        if (dn) {
          rn = fp::density(rc1, S.du[pb][ty + RY][tx + 1], un1, S.dv[pb][ty + RY + 1][tx], vn1, wn1, dwc1, idx, idy,
                           idzc, dtf);
        }
        const float rt = fp::mul(rn, st[O_TH + (ty + RY + R0) * RW + tx + C0]);
        if (final_step) {
          put(a.f_rho, g, kCell, gi, gj1, k, rn);
          put(a.f_rt, g, kCell, gi, gj1, k, rt);
          put(a.f_u, g, kFaceX, gi, gj1, k, fp::add(st[O_BU + (ty + RY) * OBW + tx], un1));
          put(a.f_v, g, kFaceY, gi, gj1, k, fp::add(st[O_BV + (ty + RY) * OBW + tx], vn1));
          if (k == 0) put(a.f_w, g, kFaceZ, gi, gj1, 0, bwz1);
          put(a.f_w, g, kFaceZ, gi, gj1, k + 1, fp::add(st[O_BW + (ty + RY) * OBW + tx], wn1));
        } else {
          put(a.rho_out, g, kCell, gi, gj1, k, rn);
          put(a.du_out, g, kFaceX, gi, gj1, k, un1);
          put(a.dv_out, g, kFaceY, gi, gj1, k, vn1);
          if (k + 1 < nz) put(a.dw_out, g, kFaceZ, gi, gj1, k + 1, wn1);
        }
        if (acc_mode == 1) {
          const float pv = eos_pprime_ref(rn, rt, T.binv[k], T.bpr[k]);
          sa.add(rn, kFxRho);
          sb.add(pv, kFxP);
          put(a.p_out, g, kCell, gi, gj1, k, pv);
        }
        else if (acc_mode == 2) sa.add(fp::theta(rn, rt), kFxTheta);
      }
      if (acc_mode) {
        const long long ta = sa.warp_total(), tb = sb.warp_total();
        if (tx == 0) { S.red[pb][ty][0] = ta; S.red[pb][ty][1] = tb; }
      }
      dwc0 = wn0;
      dwc1 = wn1;
    }
    return false;
  };
  const bool aborted = interior ? plane_loop(std::true_type{}) : plane_loop(std::false_type{});
  if (aborted) {
    // drain the tiles still in flight (bounded) before the CTA's shared memory goes away
    if (tid == ISSUER)
      for (int kk = waited + 1; kk <= issued; ++kk)
        mbar_wait(&S.bar[(base + kk) % NSLOT], ((base + kk) / NSLOT) & 1);
    return true;
  }
  __syncthreads();  // the last plane's warp totals; every thread is done with the tile
  if (acc_mode && tid == ISSUER) {  // level sums of the last plane
    const int pb = (nz - 1) & 1;
    long long sa = 0, sb = 0;
    for (int q = 0; q < NW; ++q) { sa += S.red[pb][q][0]; sb += S.red[pb][q][1]; }
    acc_add(a.acc_a + nz - 1, sa);
    if (acc_mode == 1) acc_add(a.acc_b + nz - 1, sb);
  }
  return false;
}

// CTA start: the ring's barriers, the abort flags.
__device__ __forceinline__ void fast_cta_init(FastShared& S) {
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    for (int s = 0; s < ft::NSLOT; ++s) mbar_init(&S.bar[s], 1);
    mbar_fence_init();
    S.abort[0] = 0;
    S.abort[1] = 0;
  }
}

// err[1] > 0 (set only by failure-path tests): the first CTA to see it leaves the loads
// of plane err[1] - 1 unissued, so that CTA's bounded wait runs out
__device__ __forceinline__ int fast_stall_plane(const FastArgs& a) {
  const int tid = threadIdx.y * ft::TX + threadIdx.x;
  if (tid == ft::ISSUER && *(volatile int*)(a.err + 1) > 0) return atomicExch(a.err + 1, 0) - 1;
  return -1;
}

// One acoustic substep: one CTA per tile.
template <bool FIRST, bool PIN>
__global__ void __launch_bounds__(ft::NT, 3) k_fast_tma(const FastArgs a, const __grid_constant__ FastMaps m) {
  extern __shared__ unsigned char s_dyn[];
  __shared__ FastShared S;
  using L = ft::Slot<FIRST, PIN>;
  const int slot = a.final_kind == 2 ? L::LONG : L::SHORT;
  float* const ring = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(s_dyn) + 127) & ~uintptr_t(127));
  const FastTables T = fast_tables(ring, slot, a.g.nz);
  fast_cta_init(S);
  fast_substep_setup(a, T, blockIdx.x == 0 && blockIdx.y == 0);
  fast_tile<FIRST, PIN>(a, m, blockIdx.x, blockIdx.y, S, ring, T, 0u, fast_stall_plane(a));
}

// Grid-wide barrier of a cooperative launch: arrive on count, the last arrival resets it
// and advances gen; the others wait for gen to move, bounded by WaitDeadline.  Returns
// false (err set) when the wait gave up.
__device__ __forceinline__ bool fast_grid_barrier(unsigned* count, unsigned* gen, int* err) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    ok = 1;
    const unsigned nblocks = gridDim.x * gridDim.y;
    const unsigned g0 = *(volatile unsigned*)gen;
    __threadfence();  // this CTA's stores before its arrival
    if (atomicAdd(count, 1u) == nblocks - 1) {
      atomicExch(count, 0u);
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      WaitDeadline d;
      while (*(volatile unsigned*)gen == g0) {
        if (d.expired()) { ok = 0; atomicExch(err, 1); break; }
        __nanosleep(64);
      }
    }
    __threadfence();  // the other CTAs' stores before this CTA's later loads
  }
  __syncthreads();
  // those stores feed this CTA's next TMA loads (async proxy), issued by another thread
  asm volatile("fence.proxy.async.global;" ::: "memory");
  return ok != 0;
}

// All acoustic substeps of one RK stage in one cooperative launch: each CTA runs tiles
// blockIdx.x, blockIdx.x + gridDim.x, ... of every substep; a grid barrier separates the
// substeps (the next one reads the level sums and the halos the previous one wrote).
// Every tile's arithmetic is the one-launch-per-substep kernel's.
template <bool PIN_FIRST>
__global__ void __launch_bounds__(ft::NT, 3) k_fast_stage_tma(const __grid_constant__ FastStage st) {
  using namespace ft;
  extern __shared__ unsigned char s_dyn[];
  __shared__ FastShared S;
  float* const ring = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(s_dyn) + 127) & ~uintptr_t(127));
  const int nz = st.a[0].g.nz;
  const int ntx = (st.a[0].g.nx + TX - 1) / TX, nty = (st.a[0].g.ny + TY - 1) / TY, ntiles = ntx * nty;
  fast_cta_init(S);
  unsigned base = 0;
  for (int q = 0; q < st.n; ++q) {
    const FastArgs& a = st.a[q];
    if (q > 0 && !fast_grid_barrier(st.count, st.gen, a.err)) return;
    // the tables follow the longest ring of the launch, so no substep's ring overlaps them
    const FastTables T = fast_tables(ring, st.slot_floats, nz);
    fast_substep_setup(a, T, blockIdx.x == 0);
    const int stall = fast_stall_plane(a);
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      const int bx = t % ntx, by = t / ntx;
      bool aborted;
      if (q > 0) aborted = fast_tile<false, true>(a, st.m[q], bx, by, S, ring, T, base, t == blockIdx.x ? stall : -1);
      else if (PIN_FIRST) aborted = fast_tile<true, true>(a, st.m[q], bx, by, S, ring, T, base, t == blockIdx.x ? stall : -1);
      else aborted = fast_tile<true, false>(a, st.m[q], bx, by, S, ring, T, base, t == blockIdx.x ? stall : -1);
      if (aborted) {
        // the other CTAs find out at the next grid barrier, which this CTA never reaches
        return;
      }
      base += nz;
    }
  }
}

}  // namespace

cudaError_t init_fast_tma() {
  cudaError_t e = cudaFuncSetAttribute(k_fast_tma<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)ft::dyn_smem<true, false>(true, kMaxNz));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_fast_tma<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ft::dyn_smem<true, true>(true, kMaxNz));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_fast_tma<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)ft::dyn_smem<false, true>(true, kMaxNz));
  const int stage_max = (int)std::max({ft::dyn_smem<true, false>(true, kMaxNz), ft::dyn_smem<true, true>(true, kMaxNz),
                                       ft::dyn_smem<false, true>(true, kMaxNz)});
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_fast_stage_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, stage_max);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_fast_stage_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, stage_max);
  return e;
}

cudaError_t launch_fast_tma(const FastArgs& a, const FastMaps& m, bool first, bool p_ready, cudaStream_t s) {
  if (a.g.nz > kMaxNz || a.g.nz < 1 || !a.err) return cudaErrorInvalidValue;
  const dim3 block(ft::TX, ft::RY);
  const dim3 grid((a.g.nx + ft::TX - 1) / ft::TX, (a.g.ny + ft::TY - 1) / ft::TY);
  const bool fin = a.final_kind == 2;
  if (first && p_ready) k_fast_tma<true, true><<<grid, block, ft::dyn_smem<true, true>(fin, a.g.nz), s>>>(a, m);
  else if (first) k_fast_tma<true, false><<<grid, block, ft::dyn_smem<true, false>(fin, a.g.nz), s>>>(a, m);
  else k_fast_tma<false, true><<<grid, block, ft::dyn_smem<false, true>(fin, a.g.nz), s>>>(a, m);
  return cudaGetLastError();
}

cudaError_t launch_fast_stage_tma(FastStage& st, bool p_ready, cudaStream_t s) {
  if (st.n < 1 || st.n > kFastStageMax || !st.count || !st.gen) return cudaErrorInvalidValue;
  const Geom& g = st.a[0].g;
  if (g.nz > kMaxNz || g.nz < 1) return cudaErrorInvalidValue;
  size_t slot = 0;  // the longest ring slot of the launch's substeps
  for (int q = 0; q < st.n; ++q) {
    const FastArgs& a = st.a[q];
    if (!a.err || a.g.nx != g.nx || a.g.ny != g.ny || a.g.nz != g.nz) return cudaErrorInvalidValue;
    const bool fin = a.final_kind == 2;
    size_t f;
    if (q > 0) f = fin ? ft::Slot<false, true>::LONG : ft::Slot<false, true>::SHORT;
    else if (p_ready) f = fin ? ft::Slot<true, true>::LONG : ft::Slot<true, true>::SHORT;
    else f = fin ? ft::Slot<true, false>::LONG : ft::Slot<true, false>::SHORT;
    slot = std::max(slot, f);
  }
  st.slot_floats = (int)slot;
  const size_t smem = slot * ft::NSLOT * sizeof(float) + 128 + ft::kLevelBytes * size_t(g.nz);
  const void* fn = p_ready ? (const void*)k_fast_stage_tma<true> : (const void*)k_fast_stage_tma<false>;
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, ft::NT, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const int tiles = ((g.nx + ft::TX - 1) / ft::TX) * ((g.ny + ft::TY - 1) / ft::TY);
  // every CTA resident at once (the grid barrier needs it; the cooperative launch checks it)
  const unsigned blocks = (unsigned)std::min(tiles, per_sm * sms);
  e = cudaMemsetAsync(st.count, 0, sizeof(unsigned), s);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(ft::TX, ft::RY);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (p_ready) return cudaLaunchKernelEx(&cfg, k_fast_stage_tma<true>, st);
  return cudaLaunchKernelEx(&cfg, k_fast_stage_tma<false>, st);
}

}  // namespace gwmb
