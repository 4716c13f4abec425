// slow_terrain_tma.cu — one fused slow RK stage on terrain on owned tiles fed by TMA.
//
// Same operator and per-cell arithmetic as k_slow_stage<true, R> (the K2/K3/K16-K19/
// K21/K22 tendencies of compute_slow_tendencies, src/dycore/dry_core.cu:400-539, with
// the terrain pressure gradient of dry_pressure_gradient.cu:37-240 and the hybrid-height
// metric columns; the update K4 and blend K5 of :189-205), with the data path of
// k_slow_tma: a CTA owns a 32 x 16 tile, two columns per thread, and one elected thread
// fetches each plane's boxes with cp.async.bulk.tensor.3d into a three-slot shared-memory
// ring two planes ahead:
//   rho, theta (or rho*theta), u, w, z (+ du, dw)   40 x 18 boxes: tile, halo ring, corners
//   v (+ dv)                                        40 x 19 (one more Y-face row)
// Plane nz carries only w (+ dw), the top faces.  Per plane the CTA derives, at all 34 x 18
// positions of the tile and its ring, theta, the cell velocities uc, vc, wc, the full
// pressure of the plane above (three pressure planes are kept) and dp/dz of the plane; one
// barrier publishes them, every thread computes its cells and faces, and a second barrier
// frees the derived planes for the next one (the terrain planes would not fit a CTA pair
// per SM double-buffered).  The owned columns' metric values (the cell and face inverse
// layer depths) and the blend partner q0 are per-thread coalesced loads a plane ahead.
#include <type_traits>

#include "dycore.cuh"
#include "stencil.cuh"
#include "tma.cuh"

namespace gwmb {
namespace {

namespace st {
constexpr int TX = 32, TY = 16, RY = 8, NT = 256, NW = NT / 32;
// the thread that issues the TMA loads and folds the level sums: lane 0 of the last warp
constexpr int ISSUER = NT - 32;
constexpr int BW = 40, BH = 18, BHV = 19;  // boxes: cells, X and Z faces / Y faces
constexpr int DW = TX + 2, DH = TY + 2, DN = DW * DH;  // derived plane: 34 x 18
// raw slot (floats; sub-buffers on 128-byte boundaries)
constexpr int R_RHO = 0, R_TH = 736, R_U = 1472, R_W = 2208, R_V = 2944, R_Z = 3712, R_DU = 4448, R_DW = 5184,
              R_DV = 5920, SLOT = 6688, SLOT_SHORT = 4448, NSLOT = 3;
constexpr unsigned B_BOX = BW * BH * 4, B_BOXV = BW * BHV * 4;
// derived arrays (floats): uc, vc, wc [2][DN] (planes k-1, k); theta, dp/dz [DN]; p [3][DN]
constexpr int D_UC = 0, D_VC = 2 * DN, D_WC = 4 * DN, D_TH = 6 * DN, D_DZ = 7 * DN, D_P = 8 * DN, DERIVED = 11 * DN;
static_assert(R_TH % 32 == 0 && R_U % 32 == 0 && R_W % 32 == 0 && R_V % 32 == 0 && R_Z % 32 == 0 &&
                  R_DU % 32 == 0 && R_DW % 32 == 0 && R_DV % 32 == 0 && SLOT % 32 == 0 && SLOT_SHORT == R_DU,
              "128-byte aligned sub-buffers");
static_assert(R_TH - R_RHO >= BW * BH && R_U - R_TH >= BW * BH && R_W - R_U >= BW * BH &&
                  R_V - R_W >= BW * BH && R_Z - R_V >= BW * BHV && R_DU - R_Z >= BW * BH &&
                  R_DW - R_DU >= BW * BH && R_DV - R_DW >= BW * BH && SLOT - R_DV >= BW * BHV,
              "boxes fit their sub-buffers");
constexpr size_t smem_bytes(bool inc) {
  return size_t((inc ? SLOT : SLOT_SHORT) * NSLOT + DERIVED) * sizeof(float) + 128;
}
}  // namespace st

// Values of one owned column carried from plane k-1 to plane k.
struct TerrCarry {
  float rho, th, uf, vf, wf;
};
// Blend partner q0 at a column's owned positions of one plane.
struct TerrBlend {
  float rho, rt, u, v, w;
};
// Metric values of one owned column at one plane: inverse layer depth of the cell, of its
// west and south neighbours (the X and Y faces average two cells) and of the Z face.
struct TerrMetric {
  float c, w, s, f;
};

template <bool INC>
__global__ void __launch_bounds__(st::NT, 2)
    k_slow_terrain_tma(const SlowArgs a, const __grid_constant__ SlowMaps m) {
  using namespace st;
  extern __shared__ unsigned char s_dyn[];
  __shared__ float s_thref[kMaxNz];
  __shared__ long long s_red[2][NW];
  __shared__ __align__(8) uint64_t s_bar[NSLOT];
  __shared__ int s_abort[2];
  constexpr int slot = INC ? SLOT : SLOT_SHORT;
  float* const ring = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(s_dyn) + 127) & ~uintptr_t(127));
  float* const der = ring + NSLOT * slot;

  const Geom& g = a.g;
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  const int w = min(TX, nx - i0), h = min(TY, ny - j0);
  const bool own0 = tx < w && ty < h, own1 = tx < w && ty + RY < h;
  const int gi = i0 + tx, gj0 = j0 + ty, gj1 = j0 + ty + RY;
  const bool open_x = !g.per_x, open_y = !g.per_y;
  const bool edge = (g.per_x && (i0 <= 1 || i0 + w >= nx - 1)) || (g.per_y && (j0 <= 1 || j0 + h >= ny - 1));
  const float idx = g.inv_dx, idy = g.inv_dy, dt = a.dt;
  const bool blend = a.rho0 != nullptr;
  // open boundaries: X face nx and Y face ny belong to the last tiles; their tendency
  // is zero (dry_momentum_flux.cu:79-235 skips them), so they are blends of the stage value
  const bool xf = open_x && i0 + w == nx && ty == 0 && tx < h;  // X face nx, row j0+tx
  const bool yf = open_y && j0 + h == ny && ty == 1 && tx < w;  // Y face ny, column i0+tx

  if (tid == 0) {
    for (int s = 0; s < NSLOT; ++s) mbar_init(&s_bar[s], 1);
    mbar_fence_init();
    s_abort[0] = 0;
    s_abort[1] = 0;
  }
  if (blockIdx.x == 0 && blockIdx.y == 0 && a.clr_a)
    for (int q = tid; q < nz; q += NT) { a.clr_a[q] = 0ull; a.clr_b[q] = 0ull; }
  for (int q = tid; q < nz; q += NT) s_thref[q] = (float)(acc_read(a.th_acc + q, kScaleTheta) * a.inv_count);
  __syncthreads();

  // err[1] > 0 (set only by failure-path tests): the first CTA to see it leaves the loads
  // of plane err[1] - 1 unissued, so that CTA's bounded wait runs out
  int stall = -1;
  if (tid == ISSUER && *(volatile int*)(a.err + 1) > 0) stall = atomicExch(a.err + 1, 0) - 1;
  auto issue = [&](int kk) {  // plane kk in [0, nz] into slot kk % NSLOT
    float* sr = ring + (kk % NSLOT) * slot;
    uint64_t* bar = &s_bar[kk % NSLOT];
    const bool cells = kk < nz;
    unsigned bytes = (INC ? 2u : 1u) * B_BOX;
    if (cells) bytes += 4 * B_BOX + B_BOXV + (INC ? B_BOX + B_BOXV : 0u);
    const int x = i0 + kXOff - 4, y = j0;
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(bar, bytes);
    if (kk == stall) return;  // failure-path testing: this plane's loads stay unissued
    tma_load_3d(sr + R_W, &m.w, x, y, kk, bar);
    if (INC) tma_load_3d(sr + R_DW, &m.dw, x, y, kk, bar);
    if (cells) {
      tma_load_3d(sr + R_RHO, &m.rho, x, y, kk, bar);
      tma_load_3d(sr + R_TH, &m.th, x, y, kk, bar);
      tma_load_3d(sr + R_U, &m.u, x, y, kk, bar);
      tma_load_3d(sr + R_V, &m.v, x, y, kk, bar);
      tma_load_3d(sr + R_Z, &m.z, x, y, kk, bar);
      if (INC) {
        tma_load_3d(sr + R_DU, &m.du, x, y, kk, bar);
        tma_load_3d(sr + R_DV, &m.dv, x, y, kk, bar);
      }
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
  // raw accessors: box index of derived position (r, c) is r * BW + c + 3
  auto U = [&](const float* sr, int b) { return INC ? fp::add(sr[R_U + b], sr[R_DU + b]) : sr[R_U + b]; };
  auto V = [&](const float* sr, int b) { return INC ? fp::add(sr[R_V + b], sr[R_DV + b]) : sr[R_V + b]; };
  auto W = [&](const float* sr, int b) { return INC ? fp::add(sr[R_W + b], sr[R_DW + b]) : sr[R_W + b]; };
  auto RT = [&](const float* sr, int b) {
    const float t = sr[R_TH + b];
    return a.th_is_rt ? t : fp::mul(sr[R_RHO + b], t);
  };

  // blend partner of plane kk at the thread's owned positions
  auto load_q0 = [&](int gj, bool own, int kk) {
    TerrBlend q{0.f, 0.f, 0.f, 0.f, 0.f};
    if (!blend || !own || kk >= nz) return q;
    const int o = gidx(g, gi, gj, kk);
    q.rho = __ldg(a.rho0 + o);
    q.rt = __ldg(a.rt0 + o);
    q.u = __ldg(a.u0 + o);
    q.v = __ldg(a.v0 + o);
    q.w = __ldg(a.w0 + o);
    return q;
  };
  // metric values of plane kk at the thread's owned positions
  auto load_metric = [&](int gj, bool own, int kk) {
    TerrMetric t{0.f, 0.f, 0.f, 0.f};
    if (!own || kk >= nz) return t;
    const int o = gidx(g, gi, gj, kk);
    t.c = __ldg(a.idz_c + o);
    t.w = __ldg(a.idz_c + o - 1);
    t.s = __ldg(a.idz_c + o - g.pitch);
    t.f = __ldg(a.idz_f + o);
    return t;
  };

  if (tid == ISSUER) {
    issue(0);
    issue(1);
    issued = 1;
  }
  TerrBlend q0a = load_q0(gj0, own0, 0), q0b = load_q0(gj1, own1, 0);
  TerrMetric m0a = load_metric(gj0, own0, 0), m0b = load_metric(gj1, own1, 0);
  TerrCarry ca{0.f, 0.f, 0.f, 0.f, 0.f}, cb{0.f, 0.f, 0.f, 0.f, 0.f};
  wait_plane(0, 0);

  // store of an owned value: a plain store in interior tiles, else with the periodic mirrors
  auto put = [&](bool in, float* f, const Geom& gg, int o, int i, int j, int kk, float v) {
    if (in) f[gidx(gg, i, j, kk)] = v;
    else store_tile(f, gg, o, i, j, kk, v, edge);
  };
  // one owned column: cell, X face, Y face and Z face of plane k (+ the top face)
  auto column = [&](auto tile_class, int k, int r, int gj, bool own_rt, TerrCarry& cy, const TerrBlend& q0,
                    const TerrMetric& mt, FxAcc& ra) {
    constexpr bool IN = decltype(tile_class)::value;  // an interior tile
    const bool own = IN || own_rt;
    const float* sr = ring + (k % NSLOT) * slot;
    const float* sn = ring + ((k + 1) % NSLOT) * slot;
    const float* uc = der + D_UC + (k & 1) * DN;
    const float* vc = der + D_VC + (k & 1) * DN;
    const float* wc = der + D_WC + (k & 1) * DN;
    const float* ucm = der + D_UC + ((k + 1) & 1) * DN;  // plane k-1
    const float* vcm = der + D_VC + ((k + 1) & 1) * DN;
    const float* wcm = der + D_WC + ((k + 1) & 1) * DN;
    const float* th = der + D_TH;
    const float* dz = der + D_DZ;
    const float* pp = der + D_P + (k % 3) * DN;
    const int c = tx + 1;
    const int d = r * DW + c;   // derived index
    const int b = r * BW + c + 3;  // raw box index
    const bool top = k + 1 == nz;
    // values of the column at planes k and k+1
    const float rho = sr[R_RHO + b], rt = RT(sr, b);
    const float tc = th[d], pc = pp[d];
    const float uf = U(sr, b), vf = V(sr, b), wf = W(sr, b);
    const float wft = W(sn, b);  // face k+1 (plane nz holds the top faces)
    float uft = uf, vft = vf, tt = tc;
    if (!top) {
      uft = U(sn, b);
      vft = V(sn, b);
      tt = fp::theta(sn[R_RHO + b], RT(sn, b));
    }
    const float tb = k > 0 ? cy.th : tc;
    // ---- cell: K2 compute_cell_tendencies_kernel (dry_core.cu:62-144)
    {
      const float fw = uf, fe = U(sr, b + 1), fs = vf, fn = V(sr, b + BW);
      const float fb = wf, ft = wft;
      const float t_rho = -fp::divergence(fe, fw, fn, fs, ft, fb, idx, idy, mt.c);
      const float tw = th[d - 1], te = th[d + 1], ts = th[d - DW], tn = th[d + DW];
      const float gw = fp::upwind(fw, tw, tc), ge = fp::upwind(fe, tc, te);
      const float gs = fp::upwind(fs, ts, tc), gn = fp::upwind(fn, tc, tn);
      const float gb = fp::upwind(fb, tb, tc), gt = fp::upwind(ft, tc, tt);
      const float t_rt = -fp::divergence(ge, gw, gn, gs, gt, gb, idx, idy, mt.c);
      float r1 = fp::update(rho, dt, t_rho, 1.0e-6f);
      float q1 = fp::update(rt, dt, t_rt, 1.0e-6f);
      if (blend) {
        r1 = fp::blend(a.wa, q0.rho, a.wb, r1);
        q1 = fp::blend(a.wa, q0.rt, a.wb, q1);
      }
      const float th1 = fp::theta(r1, q1);
      if (own) {
        put(IN, a.o_rho, g, kCell, gi, gj, k, r1);
        put(IN, a.o_th, g, kCell, gi, gj, k, a.out_rt ? q1 : th1);
        if (a.acc_mode == 2) ra.add(th1, kFxTheta);
      }
    }
    // ---- X face: K17 (dry_momentum_flux.cu:79-156) + K21 (dry_pressure_gradient.cu:75-123)
    {
      float t_u = 0.0f;
      if ((IN || !(gi == 0 && open_x))) {
        const float qw = U(sr, b - 1), qc = uf, qe = U(sr, b + 1);
        const float qs = U(sr, b - BW), qn = U(sr, b + BW);
        const float qb = k > 0 ? cy.uf : qc;
        const float qt = top ? qc : uft;
        const float flw = fp::upwind(uc[d - 1], qw, qc);
        const float fle = fp::upwind(uc[d], qc, qe);
        float fls = 0.0f, fln = 0.0f, flb = 0.0f, flt = 0.0f;
        if ((IN || !(gj == 0 && open_y))) fls = fp::upwind(fp::avg(vc[d - DW - 1], vc[d - DW]), qs, qc);
        if ((IN || !(gj + 1 == ny && open_y))) fln = fp::upwind(fp::avg(vc[d - 1], vc[d]), qc, qn);
        if (k > 0) flb = fp::upwind(fp::avg(wcm[d - 1], wcm[d]), qb, qc);
        if (!top) flt = fp::upwind(fp::avg(wc[d - 1], wc[d]), qc, qt);
        t_u = -fp::divergence(fle, flw, fln, fls, flt, flb, idx, idy, fp::avg(mt.w, mt.c));
        t_u = fp::add_pgf_terrain(t_u, pc, pp[d - 1], sr[R_Z + b], sr[R_Z + b - 1], dz[d - 1], dz[d], idx);
        if (a.damp_c) t_u = fp::add_damping(t_u, __ldg(a.damp_c + k), qc, __ldg(a.uref + k));
      }
      float u1 = fp::update(uf, dt, t_u, -1.0e30f);
      if (blend) u1 = fp::blend(a.wa, q0.u, a.wb, u1);
      if (own) put(IN, a.o_u, g, kFaceX, gi, gj, k, u1);
    }
    // ---- Y face: K18 (dry_momentum_flux.cu:158-235) + K22 (dry_pressure_gradient.cu:125-173)
    {
      float t_v = 0.0f;
      if ((IN || !(gj == 0 && open_y))) {
        const float qw = V(sr, b - 1), qc = vf, qe = V(sr, b + 1);
        const float qs = V(sr, b - BW), qn = V(sr, b + BW);
        const float qb = k > 0 ? cy.vf : qc;
        const float qt = top ? qc : vft;
        float flw = 0.0f, fle = 0.0f, flb = 0.0f, flt = 0.0f;
        if ((IN || !(gi == 0 && open_x))) flw = fp::upwind(fp::avg(uc[d - DW - 1], uc[d - 1]), qw, qc);
        if ((IN || !(gi + 1 == nx && open_x))) fle = fp::upwind(fp::avg(uc[d - DW], uc[d]), qc, qe);
        const float fls = fp::upwind(vc[d - DW], qs, qc);
        const float fln = fp::upwind(vc[d], qc, qn);
        if (k > 0) flb = fp::upwind(fp::avg(wcm[d - DW], wcm[d]), qb, qc);
        if (!top) flt = fp::upwind(fp::avg(wc[d - DW], wc[d]), qc, qt);
        t_v = -fp::divergence(fle, flw, fln, fls, flt, flb, idx, idy, fp::avg(mt.s, mt.c));
        t_v = fp::add_pgf_terrain(t_v, pc, pp[d - DW], sr[R_Z + b], sr[R_Z + b - BW], dz[d - DW], dz[d], idy);
        if (a.damp_c) t_v = fp::add_damping(t_v, __ldg(a.damp_c + k), qc, __ldg(a.vref + k));
      }
      float v1 = fp::update(vf, dt, t_v, -1.0e30f);
      if (blend) v1 = fp::blend(a.wa, q0.v, a.wb, v1);
      if (own) put(IN, a.o_v, g, kFaceY, gi, gj, k, v1);
    }
    // ---- Z face k: K19 (dry_momentum_flux.cu:237-312) + K3 buoyancy (dry_core.cu:146-187)
    {
      float t_w = 0.0f;
      if (k > 0) {
        const float qw = W(sr, b - 1), qc = wf, qe = W(sr, b + 1);
        const float qs = W(sr, b - BW), qn = W(sr, b + BW);
        const float qb = cy.wf, qt = wft;
        float flw = 0.0f, fle = 0.0f, fls = 0.0f, fln = 0.0f;
        if ((IN || !(gi == 0 && open_x))) flw = fp::upwind(fp::avg(ucm[d - 1], uc[d - 1]), qw, qc);
        if ((IN || !(gi + 1 == nx && open_x))) fle = fp::upwind(fp::avg(ucm[d], uc[d]), qc, qe);
        if ((IN || !(gj == 0 && open_y))) fls = fp::upwind(fp::avg(vcm[d - DW], vc[d - DW]), qs, qc);
        if ((IN || !(gj + 1 == ny && open_y))) fln = fp::upwind(fp::avg(vcm[d], vc[d]), qc, qn);
        const float flb = fp::upwind(wcm[d], qb, qc);
        const float flt = fp::upwind(wc[d], qc, qt);
        t_w = -fp::divergence(fle, flw, fln, fls, flt, flb, idx, idy, mt.f);
        t_w = fp::add_buoyancy(t_w, cy.th, tc, s_thref[k - 1], s_thref[k], cy.rho, rho, a.gravity);
        if (a.damp_c) t_w = fp::add_damping(t_w, __ldg(a.damp_f + k), qc, 0.0f);
      }
      float w1 = fp::update(wf, dt, t_w, -1.0e30f);
      if (blend) w1 = fp::blend(a.wa, q0.w, a.wb, w1);
      if (own) {
        put(IN, a.o_w, g, kFaceZ, gi, gj, k, w1);
        if (top) {  // top face: zero tendency
          float wt = fmaxf(-1.0e30f, wft);
          if (blend) wt = fp::blend(a.wa, __ldg(a.w0 + gidx(g, gi, gj, nz)), a.wb, wt);
          put(IN, a.o_w, g, kFaceZ, gi, gj, nz, wt);
        }
      }
    }
    cy.rho = rho;
    cy.th = tc;
    cy.uf = uf;
    cy.vf = vf;
    cy.wf = wf;
  };

  // Interior tiles (full, away from every periodic edge ring and open side) run a copy of
  // the plane loop compiled without the edge logic; both copies do the same arithmetic.
  const bool interior = !edge && (g.per_x || (i0 > 0 && i0 + TX < nx)) && (g.per_y || (j0 > 0 && j0 + TY < ny));
  auto plane_loop = [&](auto tile_class) -> bool {  // true when a bounded wait gave up
    constexpr bool IN = decltype(tile_class)::value;
    for (int k = 0; k < nz; ++k) {
      const int pb = k & 1;
      // ---- derive plane k at the 34 x 18 positions: theta, uc, vc, wc, the pressure of
      // plane k+1 (and of plane 0 at the start) and dp/dz of plane k
      wait_plane(k + 1, k);
      {
        const float* sm = ring + ((k + NSLOT - 1) % NSLOT) * slot;  // plane k-1 (its slot is intact)
        const float* sr = ring + (k % NSLOT) * slot;
        const float* sn = ring + ((k + 1) % NSLOT) * slot;
        float* uc = der + D_UC + pb * DN;
        float* vc = der + D_VC + pb * DN;
        float* wc = der + D_WC + pb * DN;
        float* th = der + D_TH;
        float* dz = der + D_DZ;
        float* pm = der + D_P + ((k + 2) % 3) * DN;
        float* pc = der + D_P + (k % 3) * DN;
        float* pn = der + D_P + ((k + 1) % 3) * DN;
        for (int q = tid; q < DN; q += NT) {
          const int r = q / DW, c = q - r * DW;
          const int b = r * BW + c + 3;
          const float rho = sr[R_RHO + b], rt = RT(sr, b);
          th[q] = fp::theta(rho, rt);
          // K20: the full pressure (dry_pressure_gradient.cu:27-35)
          if (k == 0) pc[q] = eos_pressure(rho, rt);
          if (k + 1 < nz) pn[q] = eos_pressure(sn[R_RHO + b], RT(sn, b));
          dz[q] = column_dpdz(k, nz, k > 0 ? pm[q] : 0.f, pc[q], k + 1 < nz ? pn[q] : 0.f,
                              k > 0 ? sm[R_Z + b] : 0.f, sr[R_Z + b], k + 1 < nz ? sn[R_Z + b] : 0.f);
          // cell-centred velocities: dry_momentum_flux.cu:36-73
          const float rr = fmaxf(rho, 1.0e-6f);
          uc[q] = fp::centred(U(sr, b), U(sr, b + 1), rr);
          vc[q] = fp::centred(V(sr, b), V(sr, b + BW), rr);
          wc[q] = fp::centred(W(sr, b), W(sn, b), rr);
        }
      }
      const TerrBlend n0a = load_q0(gj0, own0, k + 1), n0b = load_q0(gj1, own1, k + 1);
      const TerrMetric nma = load_metric(gj0, own0, k + 1), nmb = load_metric(gj1, own1, k + 1);
      __syncthreads();  // publishes plane k's derived values; slot (k-1) is free
      if (s_abort[pb]) return true;
      if (tid == ISSUER) {
        if (a.acc_mode && k > 0) {
          long long sa = 0;
          for (int q = 0; q < NW; ++q) sa += s_red[pb ^ 1][q];
          acc_add(a.acc_a + k - 1, sa);
        }
        if (k + 2 <= nz) { issue(k + 2); issued = k + 2; }
      }
      // ---- cells and faces of plane k
      FxAcc ra;
      column(tile_class, k, ty + 1, gj0, own0, ca, q0a, m0a, ra);
      column(tile_class, k, ty + RY + 1, gj1, own1, cb, q0b, m0b, ra);
      if (!IN && xf) {  // open east boundary: X face nx of row j0+tx
        const float* sr = ring + (k % NSLOT) * slot;
        const float uf = U(sr, (tx + 1) * BW + w + 4);
        float u1 = fp::update(uf, dt, 0.0f, -1.0e30f);
        if (blend) u1 = fp::blend(a.wa, __ldg(a.u0 + gidx(g, nx, j0 + tx, k)), a.wb, u1);
        put(false, a.o_u, g, kFaceX, nx, j0 + tx, k, u1);
      }
      if (!IN && yf) {  // open north boundary: Y face ny of column i0+tx
        const float* sr = ring + (k % NSLOT) * slot;
        const float vf = V(sr, (h + 1) * BW + tx + 4);
        float v1 = fp::update(vf, dt, 0.0f, -1.0e30f);
        if (blend) v1 = fp::blend(a.wa, __ldg(a.v0 + gidx(g, i0 + tx, ny, k)), a.wb, v1);
        put(false, a.o_v, g, kFaceY, i0 + tx, ny, k, v1);
      }
      if (a.acc_mode) {
        const long long ta = ra.warp_total();
        if (tx == 0) s_red[pb][ty] = ta;
      }
      q0a = n0a;
      q0b = n0b;
      m0a = nma;
      m0b = nmb;
      __syncthreads();  // every thread is done with plane k's derived values
    }
    return false;
  };
  const bool aborted = interior ? plane_loop(std::true_type{}) : plane_loop(std::false_type{});
  if (aborted) {
    if (tid == ISSUER)
      for (int kk = waited + 1; kk <= issued; ++kk) mbar_wait(&s_bar[kk % NSLOT], (kk / NSLOT) & 1);
    return;
  }
  if (a.acc_mode && tid == ISSUER) {  // the last plane's warp totals (published by the loop's last barrier)
    const int pb = (nz - 1) & 1;
    long long sa = 0;
    for (int q = 0; q < NW; ++q) sa += s_red[pb][q];
    acc_add(a.acc_a + nz - 1, sa);
  }
}

}  // namespace

cudaError_t init_slow_terrain_tma() {
  cudaError_t e = cudaFuncSetAttribute(k_slow_terrain_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)st::smem_bytes(true));
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_slow_terrain_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)st::smem_bytes(false));
}

cudaError_t launch_slow_terrain_tma(const SlowArgs& a, const SlowMaps& m, cudaStream_t s) {
  if (a.g.nz > kMaxNz || a.g.nz < 1 || !a.err || a.tend_only || a.acc_mode == 1 || !a.idz_c || !a.idz_f)
    return cudaErrorInvalidValue;
  const dim3 block(st::TX, st::RY);
  const dim3 grid((a.g.nx + st::TX - 1) / st::TX, (a.g.ny + st::TY - 1) / st::TY);
  if (a.du) k_slow_terrain_tma<true><<<grid, block, st::smem_bytes(true), s>>>(a, m);
  else k_slow_terrain_tma<false><<<grid, block, st::smem_bytes(false), s>>>(a, m);
  return cudaGetLastError();
}

}  // namespace gwmb
