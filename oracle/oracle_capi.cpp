#include <algorithm>
// oracle_capi.cpp — C entry points of the CPU ORACLE (test infrastructure only).
//
// Wraps gwm_oracle.hpp for the Python test-suite.  All field I/O goes through
// global owned arrays in double precision: cells (nz,ny,nx), X faces (nz,ny,nx+1),
// Y faces (nz,ny+1,nx), Z faces (nz+1,ny,nx).  Internally the fields are scattered
// onto the reference's virtual-rank layout (src/comm/virtual_rank_layout.cpp:7-47,
// scatter_scalar :49-71) and gathered back (gather_scalar/gather_face :73-137),
// then the restated operators run on the per-rank arrays exactly as the
// reference does.  precision selects the arithmetic type: 32 or 64.
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "gwm_oracle.hpp"

extern "C" {

typedef struct {
  int nx, ny, nz, halo, ranks_x, ranks_y, periodic_x, periodic_y;
  double dx, dy, z_top, terrain_taper_eta;
  const double* terrain;         // ny*nx, or NULL for flat
  const double* eta_interfaces;  // nz+1, or NULL for uniform levels
} gwo_grid;

typedef struct {
  double dt;
  int fast_substeps;
  double gravity;
  int fast_hmom, fast_density, fast_modes;
  // Rayleigh damping layer (extension): rate <= 0 disables; u_ref/v_ref: nz values or NULL
  double damp_z_bottom, damp_rate;
  const double *damp_u_ref, *damp_v_ref;
} gwo_step;

typedef struct {
  double dt, condensation_relaxation, autoconv_threshold, autoconv_rate, rain_evap_rate,
      terminal_velocity, layer_depth;
  int latent_heating;
} gwo_rain;

typedef struct {
  double *rho, *rho_theta, *u, *v, *w;
  double *qv, *qc, *qr;
  double* precip;  // ny*nx accumulated surface precipitation (kg m-2)
} gwo_fields;

typedef struct {
  double p_surface, theta_ref, theta_lapse_k_per_m, relative_humidity, rh_top_m;
  double qv_scale_height_m, qv_floor, noise_rms_k, noise_depth_m;
  unsigned long long seed;
} gwo_sounding;

typedef struct {
  double rho_background, theta_background, u_background, v_background, w_background;
  double center_x_fraction, center_y_fraction, center_z_fraction;
  double radius_x_fraction, radius_y_fraction, radius_z_fraction, theta_perturbation;
  double rho_surface, theta_ref;
} gwo_case_params;

}  // extern "C"

namespace {

thread_local std::string g_err;

struct Ctx {
  std::vector<gwo::Desc> L;
};

template <class T>
gwo::Metrics<T> metrics_from(const gwo_grid* g) {
  std::vector<double> terr((size_t)g->nx * g->ny, 0.0);
  if (g->terrain) std::memcpy(terr.data(), g->terrain, terr.size() * sizeof(double));
  return gwo::make_hybrid_height<T>(g->nx, g->ny, g->nz, g->dx, g->dy, g->z_top, terr,
                                    g->terrain_taper_eta, g->periodic_x != 0,
                                    g->periodic_y != 0, g->eta_interfaces);
}

std::vector<gwo::Desc> layout_from(const gwo_grid* g) {
  gwo::require(g->nx > 0 && g->ny > 0 && g->nz > 0, "grid dimensions must be positive");
  gwo::require(g->ranks_x > 0 && g->ranks_y > 0, "rank counts must be positive");
  return gwo::build_layout(g->nx, g->ny, g->nz, g->halo, g->ranks_x, g->ranks_y,
                           g->periodic_x != 0, g->periodic_y != 0);
}

// Global owned-array shapes per orientation.
inline size_t gidx(int o, const gwo_grid* g, int i, int j, int k) {
  const int gx = g->nx + (o == gwo::FX), gy = g->ny + (o == gwo::FY);
  return ((size_t)k * gy + j) * gx + i;
}

template <class T>
void scatter(const double* src, std::vector<gwo::Field<T>*> F, const std::vector<gwo::Desc>& L,
             const gwo_grid* g) {
  if (!src) return;
  for (size_t r = 0; r < L.size(); ++r) {
    gwo::Field<T>& f = *F[r];
    for (int k = 0; k < f.nz; ++k)
      for (int j = 0; j < f.ny; ++j)
        for (int i = 0; i < f.nx; ++i)
          f(i, j, k) = (T)src[gidx(f.o, g, L[r].i0 + i, L[r].j0 + j, k)];
  }
}

template <class T>
void gather(double* dst, std::vector<gwo::Field<T>*> F, const std::vector<gwo::Desc>& L,
            const gwo_grid* g) {
  if (!dst) return;
  for (size_t r = 0; r < L.size(); ++r) {
    gwo::Field<T>& f = *F[r];
    for (int k = 0; k < f.nz; ++k)
      for (int j = 0; j < f.ny; ++j)
        for (int i = 0; i < f.nx; ++i)
          dst[gidx(f.o, g, L[r].i0 + i, L[r].j0 + j, k)] = (double)f(i, j, k);
  }
}

template <class T>
gwo::States<T> make_states(const std::vector<gwo::Desc>& L) {
  gwo::States<T> S;
  for (const auto& d : L) S.emplace_back(d.nxl(), d.nyl(), d.nz, d.halo);
  return S;
}

template <class T>
void states_in(gwo::States<T>& S, const gwo_fields* io, const std::vector<gwo::Desc>& L,
               const gwo_grid* g) {
  std::vector<gwo::Field<T>*> a, b, c, d, e;
  for (auto& s : S) { a.push_back(&s.rho); b.push_back(&s.rt); c.push_back(&s.mu); d.push_back(&s.mv); e.push_back(&s.mw); }
  scatter(io->rho, a, L, g); scatter(io->rho_theta, b, L, g);
  scatter(io->u, c, L, g); scatter(io->v, d, L, g); scatter(io->w, e, L, g);
}

template <class T>
void states_out(gwo::States<T>& S, gwo_fields* io, const std::vector<gwo::Desc>& L,
                const gwo_grid* g) {
  std::vector<gwo::Field<T>*> a, b, c, d, e;
  for (auto& s : S) { a.push_back(&s.rho); b.push_back(&s.rt); c.push_back(&s.mu); d.push_back(&s.mv); e.push_back(&s.mw); }
  gather(io->rho, a, L, g); gather(io->rho_theta, b, L, g);
  gather(io->u, c, L, g); gather(io->v, d, L, g); gather(io->w, e, L, g);
}

template <class T> gwo::StepCfg<T> step_from(const gwo_step* s, const gwo::Metrics<T>* M = nullptr) {
  gwo::StepCfg<T> c;
  c.dt = (T)(float)s->dt;
  c.fast_substeps = s->fast_substeps;
  c.gravity = (T)(float)s->gravity;
  c.fast_hmom = s->fast_hmom != 0;
  c.fast_density = s->fast_density != 0;
  c.fast_modes = s->fast_modes != 0;
  if (M && s->damp_rate > 0.0) {
    const int nz = M->nz;
    c.damp_c.resize(nz);
    c.damp_f.resize(nz + 1);
    c.u_ref.assign(nz, T(0));
    c.v_ref.assign(nz, T(0));
    for (int k = 0; k < nz; ++k)
      c.damp_c[k] = (T)(float)gwo::rayleigh_rate(M->eta_c[k] * M->z_top, s->damp_z_bottom, M->z_top, s->damp_rate);
    for (int k = 0; k <= nz; ++k)
      c.damp_f[k] = (T)(float)gwo::rayleigh_rate(M->eta_i[k] * M->z_top, s->damp_z_bottom, M->z_top, s->damp_rate);
    for (int k = 0; k < nz; ++k) {
      if (s->damp_u_ref) c.u_ref[k] = (T)(float)s->damp_u_ref[k];
      if (s->damp_v_ref) c.v_ref[k] = (T)(float)s->damp_v_ref[k];
    }
  }
  return c;
}

template <class T> gwo::RainCfg<T> rain_from(const gwo_rain* r) {
  gwo::RainCfg<T> c;
  c.dt = (T)(float)r->dt;
  c.condensation_relaxation = (T)(float)r->condensation_relaxation;
  c.autoconv_threshold = (T)(float)r->autoconv_threshold;
  c.autoconv_rate = (T)(float)r->autoconv_rate;
  c.rain_evap_rate = (T)(float)r->rain_evap_rate;
  c.terminal_velocity = (T)(float)r->terminal_velocity;
  c.layer_depth = (T)(float)r->layer_depth;
  c.latent_heating = r->latent_heating != 0;
  return c;
}

// Prepared-case boundary cache (test restatement of prepared_case_init.cpp:396-645,
// 1006-1078, runtime_case.cpp:205-228, boundary_cache.hpp:52-76): snapshots of balanced
// states (tracers as mixing ratios) at integer forecast offsets; the boundary of an
// updater call is the snapshot interpolated at lround(step_start + sim_time).
struct BoundaryCacheIn {
  int n = 0;
  const int* offsets = nullptr;
  const gwo_fields* snapshots = nullptr;
  float t_start = 0.0f;
};

template <class T>
int run_impl(const gwo_grid* g, const gwo_step* st, const gwo_rain* rn, int phases, int nsteps,
             gwo_fields* io, const gwo_fields* bnd, const BoundaryCacheIn* cache = nullptr) {
  const auto L = layout_from(g);
  const auto M = metrics_from<T>(g);
  auto S = make_states<T>(L);
  states_in(S, io, L, g);
  // reference boundary state (apply_reference_boundaries at every stage start), or none
  gwo::States<T> B;
  std::vector<std::vector<gwo::Field<T>>> QB;
  if (bnd) {
    B = make_states<T>(L);
    states_in(B, bnd, L, g);
    if (bnd->qv && bnd->qc && bnd->qr) {
      for (const auto& d : L) {
        std::vector<gwo::Field<T>> q;
        for (int t = 0; t < 3; ++t) q.emplace_back(d.nxl(), d.nyl(), d.nz, d.halo);
        QB.push_back(std::move(q));
      }
      double* src[3] = {bnd->qv, bnd->qc, bnd->qr};
      for (int t = 0; t < 3; ++t) {
        std::vector<gwo::Field<T>*> f;
        for (auto& q : QB) f.push_back(&q[t]);
        scatter(src[t], f, L, g);
      }
    }
  }
  const bool moist = (phases & 6) != 0;
  std::vector<std::vector<gwo::Field<T>>> Q;
  std::vector<std::vector<T>> P;
  if (moist || (phases & 8)) {
    for (const auto& d : L) {
      std::vector<gwo::Field<T>> q;
      for (int t = 0; t < 3; ++t) q.emplace_back(d.nxl(), d.nyl(), d.nz, d.halo);
      Q.push_back(std::move(q));
      P.emplace_back((size_t)d.nxl() * d.nyl(), T(0));
    }
    double* src[3] = {io->qv, io->qc, io->qr};
    for (int t = 0; t < 3; ++t) {
      std::vector<gwo::Field<T>*> f;
      for (auto& q : Q) f.push_back(&q[t]);
      scatter(src[t], f, L, g);
    }
    if (io->precip)
      for (size_t r = 0; r < L.size(); ++r)
        for (int j = 0; j < L[r].nyl(); ++j)
          for (int i = 0; i < L[r].nxl(); ++i)
            P[r][(size_t)j * L[r].nxl() + i] = (T)io->precip[(size_t)(L[r].j0 + j) * g->nx + L[r].i0 + i];
  }
  const auto cfg = step_from<T>(st, &M);
  gwo::RainCfg<T> rc;
  if (rn) rc = rain_from<T>(rn);
  // boundary cache: the snapshots on the rank layout, and per stage the interpolated state
  std::vector<gwo::States<T>> CS;
  std::vector<std::vector<std::vector<gwo::Field<T>>>> CQ;  // [snapshot][rank][tracer] mixing ratios
  gwo::States<T> BS[3];
  std::vector<std::vector<gwo::Field<T>>> QS[3];
  bool cache_tracers = false;
  if (cache && cache->n > 0) {
    cache_tracers = moist;
    for (int q = 0; q < cache->n; ++q) {
      const gwo_fields& f = cache->snapshots[q];
      CS.push_back(make_states<T>(L));
      states_in(CS.back(), &f, L, g);
      cache_tracers = cache_tracers && f.qv && f.qc && f.qr;
    }
    if (cache_tracers)
      for (int q = 0; q < cache->n; ++q) {
        std::vector<std::vector<gwo::Field<T>>> per_rank;
        for (const auto& d : L) {
          std::vector<gwo::Field<T>> tq;
          for (int t = 0; t < 3; ++t) tq.emplace_back(d.nxl(), d.nyl(), d.nz, d.halo);
          per_rank.push_back(std::move(tq));
        }
        double* src[3] = {cache->snapshots[q].qv, cache->snapshots[q].qc, cache->snapshots[q].qr};
        for (int t = 0; t < 3; ++t) {
          std::vector<gwo::Field<T>*> fp;
          for (auto& rq : per_rank) fp.push_back(&rq[t]);
          scatter(src[t], fp, L, g);
        }
        CQ.push_back(std::move(per_rank));
      }
  }
  float t_start = cache ? std::max(cache->t_start, 0.0f) : 0.0f;
  for (int s = 0; s < nsteps; ++s) {  // gwm_prepared_case_driver.cpp:427-463
    const gwo::States<T>* Bs[3] = {&B, &B, &B};
    const std::vector<std::vector<gwo::Field<T>>>* QBs[3] = {&QB, &QB, &QB};
    if (!CS.empty()) {
      const float dtf = (float)st->dt;
      const float sim[3] = {0.0f, dtf, 0.5f * dtf};
      for (int k = 0; k < 3; ++k) {
        const int t = (int)std::lround(t_start + sim[k]);
        int lo = -1, hi = -1;
        for (int q = 0; q < cache->n; ++q) {
          if (cache->offsets[q] <= t) lo = q;
          if (cache->offsets[q] >= t) { hi = q; break; }
        }
        if (lo < 0) lo = 0;
        if (hi < 0) hi = cache->n - 1;
        const bool one = lo == hi || cache->offsets[lo] == cache->offsets[hi];
        const float alpha = one ? 0.0f : (float)(t - cache->offsets[lo]) / (float)(cache->offsets[hi] - cache->offsets[lo]);
        const T a = (T)alpha, b = T(1) - (T)alpha;
        auto lerp = [&](const gwo::Field<T>& x, const gwo::Field<T>& y, gwo::Field<T>& out) {
          out = x;
          if (!one)
            for (size_t e = 0; e < out.d.size(); ++e) out.d[e] = b * x.d[e] + a * y.d[e];
        };
        BS[k] = CS[lo];
        for (size_t r = 0; r < L.size(); ++r) {
          lerp(CS[lo][r].rho, CS[hi][r].rho, BS[k][r].rho);
          lerp(CS[lo][r].rt, CS[hi][r].rt, BS[k][r].rt);
          lerp(CS[lo][r].mu, CS[hi][r].mu, BS[k][r].mu);
          lerp(CS[lo][r].mv, CS[hi][r].mv, BS[k][r].mv);
          lerp(CS[lo][r].mw, CS[hi][r].mw, BS[k][r].mw);
        }
        QS[k].clear();
        if (cache_tracers)
          for (size_t r = 0; r < L.size(); ++r) {
            std::vector<gwo::Field<T>> tq(3);
            for (int t2 = 0; t2 < 3; ++t2) {
              lerp(CQ[lo][r][t2], CQ[hi][r][t2], tq[t2]);
              for (size_t e = 0; e < tq[t2].d.size(); ++e) tq[t2].d[e] *= BS[k][r].rho.d[e];  // rho_d * q
            }
            QS[k].push_back(std::move(tq));
          }
        Bs[k] = &BS[k];
        QBs[k] = cache_tracers ? &QS[k] : nullptr;
      }
      t_start = t_start + dtf;  // the driver's sim_time += dt (float)
    }
    const bool dry_bnd = bnd || !CS.empty();
    const bool tr_bnd = !CS.empty() ? cache_tracers : !QB.empty();
    if (phases & 1) gwo::advance_dry_ssprk3(S, L, M, cfg, dry_bnd ? Bs : nullptr);
    if (phases & 2) gwo::advance_tracers_ssprk3(Q, S, L, M, cfg, tr_bnd ? QBs : nullptr);
    if (phases & 4) gwo::apply_warm_rain(S, Q, L, &M, rc, io->precip ? &P : nullptr);
    if (phases & 8) gwo::apply_warm_rain<T>(S, Q, L, nullptr, rc, io->precip ? &P : nullptr);
  }
  states_out(S, io, L, g);
  if (!Q.empty()) {
    double* dst[3] = {io->qv, io->qc, io->qr};
    for (int t = 0; t < 3; ++t) {
      std::vector<gwo::Field<T>*> f;
      for (auto& q : Q) f.push_back(&q[t]);
      gather(dst[t], f, L, g);
    }
    if (io->precip)
      for (size_t r = 0; r < L.size(); ++r)
        for (int j = 0; j < L[r].nyl(); ++j)
          for (int i = 0; i < L[r].nxl(); ++i)
            io->precip[(size_t)(L[r].j0 + j) * g->nx + L[r].i0 + i] = (double)P[r][(size_t)j * L[r].nxl() + i];
  }
  return 0;
}

template <class T>
int slow_impl(const gwo_grid* g, const gwo_step* st, const gwo_fields* in, gwo_fields* out) {
  const auto L = layout_from(g);
  const auto M = metrics_from<T>(g);
  auto S = make_states<T>(L);
  states_in(S, in, L, g);
  gwo::States<T> tend;
  gwo::compute_slow_tendencies(S, L, M, step_from<T>(st, &M), tend);
  states_out(tend, out, L, g);
  return 0;
}

template <class T>
int fast_impl(const gwo_grid* g, const gwo_step* st, gwo_fields* io) {
  const auto L = layout_from(g);
  const auto M = metrics_from<T>(g);
  auto S = make_states<T>(L);
  states_in(S, io, L, g);
  gwo::fast_modes(S, L, M, step_from<T>(st, &M));
  states_out(S, io, L, g);
  return 0;
}

template <class T>
int metrics_impl(const gwo_grid* g, double* zc, double* zi, double* idc, double* idf) {
  const auto M = metrics_from<T>(g);
  for (size_t q = 0; q < M.zc.size(); ++q) { if (zc) zc[q] = M.zc[q]; if (idc) idc[q] = M.inv_dz_cell[q]; }
  for (size_t q = 0; q < M.zi.size(); ++q) { if (zi) zi[q] = M.zi[q]; if (idf) idf[q] = M.inv_dz_face[q]; }
  return 0;
}

// idealized_cases.cpp:14-20
template <class T> T bubble_weight(T dx, T dy, T dz) {
  const T r2 = dx * dx + dy * dy + dz * dz;
  if (r2 >= T(1)) return T(0);
  return T(0.5f) * (T(1) + std::cos(T(3.14159265358979323846f) * std::sqrt(r2)));
}

// Initial states.  kind: 0 warm_bubble, 1 density_current (idealized_cases.cpp:105-180),
// 2 hydrostatic_rest (dry_core.cu:363-398), 3 mountain_wave_background
// (idealized_cases.cpp:182-223, set_background_face_momenta :36-103),
// 4 constant (DryState::fill_constant, dry_core.cu:299-306),
// 5 warm bubble composed on the hydrostatic base (theta = theta_ref + dtheta*weight,
//   rho_theta = rho_hydrostatic*theta; a composition of the two reference functions).
template <class T>
int case_impl(int kind, const gwo_grid* g, const gwo_case_params* c, gwo_fields* io) {
  const auto L = layout_from(g);
  const auto M = metrics_from<T>(g);
  auto S = make_states<T>(L);
  const T pi = T(3.14159265358979323846f);
  (void)pi;
  for (size_t r = 0; r < L.size(); ++r) {
    const gwo::Desc& d = L[r];
    gwo::DryState<T>& s = S[r];
    auto fill_const = [&](T rho, T th, T u, T v, T w) {
      s.rho.fill(rho); s.rt.fill(rho * th); s.mu.fill(rho * u); s.mv.fill(rho * v); s.mw.fill(rho * w);
    };
    if (kind == 0 || kind == 1 || kind == 5) {
      const T sign = (kind == 1) ? T(-1) : T(1);
      const T dth = sign * std::abs((T)(float)c->theta_perturbation);
      const T x0 = (T)(float)c->center_x_fraction * (T)(M.nx - 1) * (T)(float)M.dx;
      const T y0 = (T)(float)c->center_y_fraction * (T)(M.ny - 1) * (T)(float)M.dy;
      const T z0 = (T)(float)c->center_z_fraction * (T)(float)M.z_top;
      const T rx = std::max((T)(float)c->radius_x_fraction * (T)M.nx * (T)(float)M.dx, T(1));
      const T ry = std::max((T)(float)c->radius_y_fraction * (T)M.ny * (T)(float)M.dy, T(1));
      const T rz = std::max((T)(float)c->radius_z_fraction * (T)(float)M.z_top, T(1));
      if (kind == 5) fill_const(T(0), (T)(float)c->theta_ref, (T)(float)c->u_background,
                                (T)(float)c->v_background, (T)(float)c->w_background);
      else fill_const((T)(float)c->rho_background, (T)(float)c->theta_background,
                      (T)(float)c->u_background, (T)(float)c->v_background, (T)(float)c->w_background);
      for (int k = 0; k < d.nz; ++k)
        for (int j = 0; j < d.nyl(); ++j)
          for (int i = 0; i < d.nxl(); ++i) {
            const int gi = d.i0 + i, gj = d.j0 + j;
            const T x = (T)gi * (T)(float)M.dx, y = (T)gj * (T)(float)M.dy;
            const T z = M.zc[M.m(gi, gj, k)];
            const T wgt = bubble_weight((x - x0) / rx, (y - y0) / ry, (z - z0) / rz);
            if (kind == 5) {
              const T rho = gwo::hydrostatic_rho_at_height((T)(float)c->rho_surface, (T)(float)c->theta_ref, z);
              s.rho(i, j, k) = rho;
              s.rt(i, j, k) = rho * ((T)(float)c->theta_ref + dth * wgt);
            } else {
              s.rt(i, j, k) = (T)(float)c->rho_background * ((T)(float)c->theta_background + dth * wgt);
            }
          }
      if (kind == 5) { s.mu.fill(T(0)); s.mv.fill(T(0)); s.mw.fill(T(0)); }
    } else if (kind == 2) {
      fill_const(T(0), (T)(float)c->theta_ref, T(0), T(0), T(0));
      for (int k = 0; k < d.nz; ++k)
        for (int j = 0; j < d.nyl(); ++j)
          for (int i = 0; i < d.nxl(); ++i) {
            const T rho = gwo::hydrostatic_rho_at_height((T)(float)c->rho_surface, (T)(float)c->theta_ref,
                                                         M.zc[M.m(d.i0 + i, d.j0 + j, k)]);
            s.rho(i, j, k) = rho;
            s.rt(i, j, k) = rho * (T)(float)c->theta_ref;
          }
      s.mu.fill(T(0)); s.mv.fill(T(0)); s.mw.fill(T(0));
    } else if (kind == 3) {
      const T ub = (T)(float)c->u_background, vb = (T)(float)c->v_background, wb = (T)(float)c->w_background;
      fill_const(T(0), (T)(float)c->theta_ref, ub, vb, wb);
      for (int k = 0; k < d.nz; ++k)
        for (int j = 0; j < d.nyl(); ++j)
          for (int i = 0; i < d.nxl(); ++i) {
            const double terr = (double)M.terrain[(size_t)(d.j0 + j) * M.nx + d.i0 + i];
            const double z = M.z_c[k] + M.bw_c[k] * terr;
            const T rho = gwo::hydrostatic_rho_at_height((T)(float)c->rho_surface, (T)(float)c->theta_ref, (T)z);
            s.rho(i, j, k) = rho;
            s.rt(i, j, k) = rho * (T)(float)c->theta_ref;
          }
      const int nx = d.nxl(), ny = d.nyl(), nz = d.nz;
      auto fdx = [&](int i, int j, int k) -> T {
        if (nx == 1 || i <= 0) return s.rho(0, j, k);
        if (i >= nx) return s.rho(nx - 1, j, k);
        return T(0.5f) * (s.rho(i - 1, j, k) + s.rho(i, j, k));
      };
      auto fdy = [&](int i, int j, int k) -> T {
        if (ny == 1 || j <= 0) return s.rho(i, 0, k);
        if (j >= ny) return s.rho(i, ny - 1, k);
        return T(0.5f) * (s.rho(i, j - 1, k) + s.rho(i, j, k));
      };
      auto fdz = [&](int i, int j, int k) -> T {
        if (nz == 1 || k <= 0) return s.rho(i, j, 0);
        if (k >= nz) return s.rho(i, j, nz - 1);
        return T(0.5f) * (s.rho(i, j, k - 1) + s.rho(i, j, k));
      };
      for (int k = 0; k < s.mu.nz; ++k) for (int j = 0; j < s.mu.ny; ++j) for (int i = 0; i < s.mu.nx; ++i) s.mu(i, j, k) = fdx(i, j, k) * ub;
      for (int k = 0; k < s.mv.nz; ++k) for (int j = 0; j < s.mv.ny; ++j) for (int i = 0; i < s.mv.nx; ++i) s.mv(i, j, k) = fdy(i, j, k) * vb;
      for (int k = 0; k < s.mw.nz; ++k) for (int j = 0; j < s.mw.ny; ++j) for (int i = 0; i < s.mw.nx; ++i) s.mw(i, j, k) = fdz(i, j, k) * wb;
    } else if (kind == 4) {
      fill_const((T)(float)c->rho_background, (T)(float)c->theta_background, (T)(float)c->u_background,
                 (T)(float)c->v_background, (T)(float)c->w_background);
    } else {
      gwo::require(false, "unknown case kind");
    }
  }
  states_out(S, io, L, g);
  return 0;
}

template <class F> int guard(F&& f) {
  try {
    return f();
  } catch (const std::exception& e) {
    g_err = e.what();
    return -1;
  }
}

}  // namespace

extern "C" {

const char* gwo_last_error(void) { return g_err.c_str(); }

void gwo_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int gwo_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int gwo_run(const gwo_grid* g, const gwo_step* st, const gwo_rain* rn, int phases, int nsteps,
            int precision, gwo_fields* io) {
  return guard([&] {
    return precision == 32 ? run_impl<float>(g, st, rn, phases, nsteps, io, nullptr)
                           : run_impl<double>(g, st, rn, phases, nsteps, io, nullptr);
  });
}

// gwo_run with a reference boundary state (global owned arrays; tracers optional)
// applied by apply_reference_boundaries at every stage start.
int gwo_run_boundary(const gwo_grid* g, const gwo_step* st, const gwo_rain* rn, int phases, int nsteps,
                     int precision, gwo_fields* io, const gwo_fields* bnd) {
  return guard([&] {
    return precision == 32 ? run_impl<float>(g, st, rn, phases, nsteps, io, bnd)
                           : run_impl<double>(g, st, rn, phases, nsteps, io, bnd);
  });
}

// gwo_run with a prepared-case boundary cache: n snapshots (balanced states; tracers as
// mixing ratios, optional) at strictly increasing forecast offsets (s); t_start is the
// first step's start time.
int gwo_run_boundary_cache(const gwo_grid* g, const gwo_step* st, const gwo_rain* rn, int phases, int nsteps,
                           int precision, gwo_fields* io, int n, const int* offsets, const gwo_fields* snapshots,
                           double t_start) {
  return guard([&] {
    BoundaryCacheIn c;
    c.n = n; c.offsets = offsets; c.snapshots = snapshots; c.t_start = (float)t_start;
    return precision == 32 ? run_impl<float>(g, st, rn, phases, nsteps, io, nullptr, &c)
                           : run_impl<double>(g, st, rn, phases, nsteps, io, nullptr, &c);
  });
}

// MLP of the learned warm-rain surrogate, FP64: loss = mean over samples and the 5
// outputs of (y_hat - (y - y_mean)/y_std)^2 (0 for y_std = 0) with inputs (x - x_mean)/x_std, three
// 64-wide hidden layers with GELU 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))).
// params: W1 (64x7) b1 W2 (64x64) b2 W3 (64x64) b3 W4 (5x64) b4; grad has the same layout.
int gwo_mlp_loss_grad(const double* params, const double* norm, const double* x, const double* y, int n,
                      double* grad, double* loss) {
  return guard([&] {
    const int I = 7, H = 64, O = 5;
    const int oW1 = 0, oB1 = oW1 + H * I, oW2 = oB1 + H, oB2 = oW2 + H * H, oW3 = oB2 + H,
              oB3 = oW3 + H * H, oW4 = oB3 + H, oB4 = oW4 + O * H, np = oB4 + O;
    std::fill(grad, grad + np, 0.0);
    const double c = std::sqrt(2.0 / 3.14159265358979323846);
    auto gelu = [&](double z, double& dg) {
      const double u = c * (z + 0.044715 * z * z * z), t = std::tanh(u);
      dg = 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * c * (1.0 + 3.0 * 0.044715 * z * z);
      return 0.5 * z * (1.0 + t);
    };
    double total = 0.0;
    std::vector<double> x0(I), z1(H), a1(H), g1(H), z2(H), a2(H), g2(H), z3(H), a3(H), g3(H);
    std::vector<double> d1(H), d2(H), d3(H), d4(O);
    for (int b = 0; b < n; ++b) {
      for (int f = 0; f < I; ++f) x0[f] = (x[b * I + f] - norm[f]) / norm[I + f];
      auto layer = [&](const double* W, const double* B, const std::vector<double>& in, int nin,
                       std::vector<double>& z, std::vector<double>& a, std::vector<double>& g) {
        for (int j = 0; j < H; ++j) {
          double s = B[j];
          for (int f = 0; f < nin; ++f) s += W[j * nin + f] * in[f];
          z[j] = s;
          a[j] = gelu(s, g[j]);
        }
      };
      layer(params + oW1, params + oB1, x0, I, z1, a1, g1);
      layer(params + oW2, params + oB2, a1, H, z2, a2, g2);
      layer(params + oW3, params + oB3, a2, H, z3, a3, g3);
      for (int o = 0; o < O; ++o) {
        double s = params[oB4 + o];
        for (int f = 0; f < H; ++f) s += params[oW4 + o * H + f] * a3[f];
        const double sd = norm[2 * I + O + o];  // 0: a constant target, normalised to 0
        const double t = sd > 0.0 ? (y[b * O + o] - norm[2 * I + o]) / sd : 0.0;
        total += (s - t) * (s - t);
        d4[o] = 2.0 * (s - t) / ((double)n * O);
      }
      for (int o = 0; o < O; ++o) {
        for (int f = 0; f < H; ++f) grad[oW4 + o * H + f] += d4[o] * a3[f];
        grad[oB4 + o] += d4[o];
      }
      auto back = [&](const double* W, int nout, const std::vector<double>& dout, const std::vector<double>& g,
                      std::vector<double>& din) {
        for (int f = 0; f < H; ++f) {
          double s = 0.0;
          for (int j = 0; j < nout; ++j) s += W[j * H + f] * dout[j];
          din[f] = s * g[f];
        }
      };
      back(params + oW4, O, d4, g3, d3);
      for (int j = 0; j < H; ++j) {
        for (int f = 0; f < H; ++f) grad[oW3 + j * H + f] += d3[j] * a2[f];
        grad[oB3 + j] += d3[j];
      }
      back(params + oW3, H, d3, g2, d2);
      for (int j = 0; j < H; ++j) {
        for (int f = 0; f < H; ++f) grad[oW2 + j * H + f] += d2[j] * a1[f];
        grad[oB2 + j] += d2[j];
      }
      back(params + oW2, H, d2, g1, d1);
      for (int j = 0; j < H; ++j) {
        for (int f = 0; f < I; ++f) grad[oW1 + j * I + f] += d1[j] * x0[f];
        grad[oB1 + j] += d1[j];
      }
    }
    *loss = total / ((double)n * O);
    return 0;
  });
}

int gwo_slow_tendencies(const gwo_grid* g, const gwo_step* st, int precision, const gwo_fields* in,
                        gwo_fields* out) {
  return guard([&] {
    return precision == 32 ? slow_impl<float>(g, st, in, out) : slow_impl<double>(g, st, in, out);
  });
}

int gwo_fast_modes(const gwo_grid* g, const gwo_step* st, int precision, gwo_fields* io) {
  return guard([&] {
    return precision == 32 ? fast_impl<float>(g, st, io) : fast_impl<double>(g, st, io);
  });
}

int gwo_metrics(const gwo_grid* g, int precision, double* zc, double* zi, double* inv_dz_cell,
                double* inv_dz_face) {
  return guard([&] {
    return precision == 32 ? metrics_impl<float>(g, zc, zi, inv_dz_cell, inv_dz_face)
                           : metrics_impl<double>(g, zc, zi, inv_dz_cell, inv_dz_face);
  });
}

int gwo_case(int kind, const gwo_grid* g, const gwo_case_params* c, int precision, gwo_fields* io) {
  return guard([&] {
    return precision == 32 ? case_impl<float>(kind, g, c, io) : case_impl<double>(kind, g, c, io);
  });
}

// Synthetic moist sounding (gwo::moist_sounding) on a flat grid: rho, rho_theta and qv
// (as rho*qv) written; momenta, cloud, rain and precipitation left to the caller (zero).
int gwo_moist_sounding(const gwo_grid* g, const gwo_sounding* c, gwo_fields* io) {
  return guard([&] {
    gwo::require(g->nx > 0 && g->ny > 0 && g->nz > 0 && !g->terrain, "flat grid with positive dimensions");
    gwo::Sounding s;
    s.p_surface = (float)c->p_surface; s.theta_ref = (float)c->theta_ref; s.lapse = (float)c->theta_lapse_k_per_m;
    s.rh = (float)c->relative_humidity; s.rh_top = (float)c->rh_top_m; s.qv_scale = (float)c->qv_scale_height_m;
    s.qv_floor = (float)c->qv_floor; s.noise_rms = (float)c->noise_rms_k; s.noise_depth = (float)c->noise_depth_m;
    s.seed = c->seed;
    std::vector<float> rho, rt, qv;
    gwo::moist_sounding(g->nx, g->ny, g->nz, g->z_top, g->eta_interfaces, s, rho, rt, qv);
    for (size_t q = 0; q < rho.size(); ++q) {
      io->rho[q] = rho[q];
      io->rho_theta[q] = rt[q];
      if (io->qv) io->qv[q] = qv[q];
    }
    return 0;
  });
}

// nsteps of advance_scalar_ssprk3 on q (nz, ny, nx) in place.
int gwo_scalar_ssprk3(int nx, int ny, int nz, int px, int py, double u, double v, double dt, double dx, double dy,
                      int nsteps, int precision, double* q) {
  return guard([&] {
    const size_t n = (size_t)nx * ny * nz;
    if (precision == 32) {
      std::vector<float> f(q, q + n);
      for (int s = 0; s < nsteps; ++s)
        gwo::scalar_ssprk3<float>(f, nx, ny, nz, px != 0, py != 0, (float)u, (float)v, (float)dt, (float)dx,
                                  (float)dy);
      std::copy(f.begin(), f.end(), q);
    } else {
      std::vector<double> f(q, q + n);
      for (int s = 0; s < nsteps; ++s)
        gwo::scalar_ssprk3<double>(f, nx, ny, nz, px != 0, py != 0, u, v, dt, dx, dy);
      std::copy(f.begin(), f.end(), q);
    }
    return 0;
  });
}

// Runtime plan view (gwo::plan_view) of a state given as global float64 arrays (the
// values are FP32 state values; they are rounded to float first).  Metrics from the grid
// in FP32.  qv/qc/qr/precip may be NULL as nfields allows.
int gwo_plan_view(const gwo_grid* g, int level, int nfields, int steps, double dt, const double* rho,
                  const double* rt, const double* u, const double* v, const double* w, const double* qv,
                  const double* qc, const double* qr, const double* precip, double* out) {
  return guard([&] {
    gwo::require(nfields == 10 || nfields == 13 || nfields == 21 || nfields == 23, "plan-view field count");
    const int nx = g->nx, ny = g->ny, nz = g->nz;
    const size_t nc = (size_t)nx * ny * nz;
    auto f32 = [](const double* p, size_t n) {
      std::vector<float> v(p ? n : 0);
      for (size_t q = 0; p && q < n; ++q) v[q] = (float)p[q];
      return v;
    };
    const auto M = metrics_from<float>(g);
    const auto r = f32(rho, nc), t = f32(rt, nc), fu = f32(u, (size_t)(nx + 1) * ny * nz),
               fv = f32(v, (size_t)nx * (ny + 1) * nz), fw = f32(w, nc + (size_t)nx * ny), fqv = f32(qv, nc),
               fqc = f32(qc, nc), fqr = f32(qr, nc), fp = f32(precip, (size_t)nx * ny),
               ter = f32(g->terrain, (size_t)nx * ny);
    std::vector<float> zc(M.zc.begin(), M.zc.end()), idc(M.inv_dz_cell.begin(), M.inv_dz_cell.end());
    gwo::PlanViewIn a{};
    a.nx = nx; a.ny = ny; a.nz = nz; a.k = std::clamp(level, 0, nz - 1); a.nfields = nfields;
    a.steps = steps; a.dt = (float)dt;
    a.terrain = g->terrain ? ter.data() : nullptr; a.zc = zc.data(); a.idc = idc.data();
    a.rho = r.data(); a.rt = t.data(); a.u = fu.data(); a.v = fv.data(); a.w = fw.data();
    a.qv = qv ? fqv.data() : nullptr; a.qc = qc ? fqc.data() : nullptr; a.qr = qr ? fqr.data() : nullptr;
    a.precip = precip ? fp.data() : nullptr;
    gwo::require(nfields <= 10 || a.qv, "specific humidity required");
    gwo::require(nfields <= 13 || (a.qc && a.qr), "cloud and rain water required");
    gwo::require(nfields <= 21 || a.precip, "precipitation required");
    gwo::plan_view(a, out);
    return 0;
  });
}

int gwo_pressure(long n, const double* rho, const double* rt, double* p, int precision) {
  for (long q = 0; q < n; ++q)
    p[q] = precision == 32 ? (double)gwo::pressure_from_rho_theta<float>((float)rho[q], (float)rt[q])
                           : gwo::pressure_from_rho_theta<double>(rho[q], rt[q]);
  return 0;
}

// Layout table: per rank 12 ints {rank, cx, cy, i0, i1, j0, j1, west, east, south, north, nz}.
int gwo_layout(int gnx, int gny, int nz, int halo, int rx, int ry, int px, int py, int* out) {
  return guard([&] {
    const auto L = gwo::build_layout(gnx, gny, nz, halo, rx, ry, px != 0, py != 0);
    for (size_t r = 0; r < L.size(); ++r) {
      const auto nb = gwo::neighbors(L, L[r]);
      int* o = out + 12 * r;
      o[0] = L[r].rank; o[1] = L[r].cx; o[2] = L[r].cy; o[3] = L[r].i0; o[4] = L[r].i1;
      o[5] = L[r].j0; o[6] = L[r].j1; o[7] = nb.w; o[8] = nb.e; o[9] = nb.s; o[10] = nb.n; o[11] = L[r].nz;
    }
    return (int)L.size();
  });
}

// Halo operations on per-rank padded arrays (reference Field3D layout).
// orient: 0 cell, 1 X face, 2 Y face, 3 Z face.  op: 0 exchange, 1 interface sync.
int gwo_halo(int gnx, int gny, int nz, int halo, int rx, int ry, int px, int py, int orient, int op,
             double** rank_fields) {
  return guard([&] {
    const auto L = gwo::build_layout(gnx, gny, nz, halo, rx, ry, px != 0, py != 0);
    std::vector<gwo::Field<double>> F;
    for (const auto& d : L) {
      gwo::Field<double> f = orient == 0 ? gwo::Field<double>(d.nxl(), d.nyl(), d.nz, d.halo)
                                         : gwo::make_face<double>(d.nxl(), d.nyl(), d.nz, d.halo, (gwo::Orient)orient);
      F.push_back(std::move(f));
    }
    for (size_t r = 0; r < L.size(); ++r)
      std::memcpy(F[r].d.data(), rank_fields[r], F[r].d.size() * sizeof(double));
    if (orient == 0) {
      gwo::require(op == 0, "interface sync applies to face fields only");
      gwo::exchange_scalar(F, L);
    } else {
      auto p = gwo::ptrs(F);
      if (op == 0) gwo::exchange_face(p, L); else gwo::sync_face_interfaces(p, L);
    }
    for (size_t r = 0; r < L.size(); ++r)
      std::memcpy(rank_fields[r], F[r].d.data(), F[r].d.size() * sizeof(double));
    return 0;
  });
}

}  // extern "C"
