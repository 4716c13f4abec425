// cases.cpp — host-side initial states and terrain (C++, run once per case).
//
// Restates the reference's idealized initialisers (src/dycore/idealized_cases.cpp,
// src/dycore/dry_core.cu:22-35,363-398, src/domain/idealized_domain_builder.cpp:14-35)
// and adds the synthetic cases the benchmark configurations name:
//  * hydrostatic_warm_bubble: the cos^2 bubble of idealized_cases.cpp:14-20,105-154
//    applied as theta perturbation on the constant-theta hydrostatic base of
//    dry_core.cu:363-398 (the reference puts its bubble on a constant-rho background);
//  * moist_sounding: theta 300 K to 1 km then +4 K/km, qv at 90 % RH below 2 km
//    decaying with a 1.5 km scale height to 1e-5, seeded Gaussian theta noise in
//    the lowest 1 km, balanced with the column recipe of
//    src/ingest/prepared_case_init.cpp:39-53,320-385;
//  * Witch-of-Agnesi terrain h / (1 + r^2/a^2)^1.5.
// All arithmetic that the reference does in float is done in float here.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/gwm_b200.h"
#include "../../include/gwm_b200_cases.h"

namespace {

constexpr float kRd = 287.05f, kP0 = 100000.0f, kKappa = 0.2854f, kRv = 461.5f;
constexpr float kG = 9.81f;

float theta_of(float rho, float rt) { return rt / std::max(rho, 1.0e-6f); }
float eos_p(float rho, float rt) {
  const float th = theta_of(rho, rt);
  const float ratio = std::max(rho * kRd * th / kP0, 1.0e-6f);
  return kP0 * std::pow(ratio, 1.0f / (1.0f - kKappa));
}
float eos_rho(float p, float th) {
  const float ex = std::pow(std::max(p / kP0, 1.0e-6f), kKappa);
  return p / std::max(kRd * th * ex, 1.0e-6f);
}
float cp() { return kRd / kKappa; }

// idealized_cases.cpp:22-34
float hydrostatic_rho_at_height(float rho_s, float theta, float z) {
  const float ps = eos_p(rho_s, rho_s * theta);
  const float exs = std::pow(std::max(ps / kP0, 1.0e-6f), kKappa);
  const float ex = std::max(1.0e-4f, exs - kG * z / (cp() * theta));
  const float p = kP0 * std::pow(ex, 1.0f / kKappa);
  return eos_rho(p, theta);
}

// prepared_case_init.cpp:39-53
float rho_theta_from_pressure(float p) {
  float rt = (kP0 / kRd) * std::pow(std::max(p / kP0, 1.0e-6f), 1.0f - kKappa);
  for (int it = 0; it < 2; ++it) {
    const float pe = eos_p(1.0f, rt);
    const float ratio = std::max(p / std::max(pe, 1.0f), 1.0e-6f);
    rt *= std::pow(ratio, 1.0f - kKappa);
  }
  return rt;
}

// moist_thermo.hpp:23-36
float qsat(float tk, float p) {
  const float eps = kRd / kRv;
  const float tc = tk - 273.15f;
  const float es = 6.112f * std::exp((17.67f * tc) / std::max(tc + 243.5f, 1.0e-6f)) * 100.0f;
  const float denom = std::max(p - (1.0f - eps) * es, 1000.0f);
  return std::min(std::max(eps * es / denom, 0.0f), 0.05f);
}

float bubble_weight(float dx, float dy, float dz) {  // idealized_cases.cpp:14-20
  const float r2 = dx * dx + dy * dy + dz * dz;
  if (r2 >= 1.0f) return 0.0f;
  return 0.5f * (1.0f + std::cos(3.14159265358979323846f * std::sqrt(r2)));
}

// Counter-based normal deviate: splitmix64 of (seed, index), Box-Muller.
uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
double unit_open(uint64_t bits) { return ((double)(bits >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

// Hybrid-height column heights: grid_metrics.hpp:126-161,224-229.
double weight(double eta, double taper) {
  if (eta <= 0.0) return 1.0;
  if (eta >= 1.0) return 0.0;
  if (taper <= 0.0) { const double s = std::clamp(eta, 0.0, 1.0); return 1.0 - s * s * (3.0 - 2.0 * s); }
  if (eta <= taper) return 1.0;
  const double s = std::clamp((eta - taper) / std::max(1.0e-9, 1.0 - taper), 0.0, 1.0);
  return 1.0 - s * s * (3.0 - 2.0 * s);
}
float z_center(const gwm_b200_grid_desc& g, int i, int j, int k) {
  const double ec = g.eta_interfaces ? 0.5 * (g.eta_interfaces[k] + g.eta_interfaces[k + 1])
                                     : ((double)k + 0.5) / (double)g.nz;
  const double th = g.terrain ? (double)g.terrain[(size_t)j * g.nx + i] : 0.0;
  return (float)(ec * g.z_top + weight(ec, g.terrain_taper_eta) * th);
}

inline size_t cidx(const gwm_b200_grid_desc& g, int i, int j, int k) { return ((size_t)k * g.ny + j) * g.nx + i; }

void fill(float* a, size_t n, float v) { if (a) std::fill(a, a + n, v); }

}  // namespace

extern "C" {

int gwm_b200_build_case(const char* kind_c, const gwm_b200_grid_desc* g, const gwm_b200_case_params* c,
                        gwm_b200_fields* out) {
  if (!kind_c || !g || !c || !out || g->nx <= 0 || g->ny <= 0 || g->nz <= 0) return GWM_B200_ERR_ARG;
  const std::string kind(kind_c);
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  const size_t nc = (size_t)nx * ny * nz;
  const size_t nu = (size_t)(nx + 1) * ny * nz, nv = (size_t)nx * (ny + 1) * nz, nw = (size_t)nx * ny * (nz + 1);
  float *rho = out->rho_d, *rt = out->rho_theta_m;
  if (!rho || !rt) return GWM_B200_ERR_ARG;
  auto fill_const = [&](float r, float th, float u, float v, float w) {  // DryState::fill_constant
    fill(rho, nc, r); fill(rt, nc, r * th);
    fill(out->mom_u, nu, r * u); fill(out->mom_v, nv, r * v); fill(out->mom_w, nw, r * w);
  };
  fill(out->qv, nc, 0.0f); fill(out->qc, nc, 0.0f); fill(out->qr, nc, 0.0f);
  if (out->precip) std::fill(out->precip, out->precip + (size_t)nx * ny, 0.0);

  if (kind == "constant") {
    fill_const(c->rho_background, c->theta_background, c->u_background, c->v_background, c->w_background);
    return GWM_B200_OK;
  }
  if (kind == "warm_bubble" || kind == "density_current" || kind == "hydrostatic_warm_bubble") {
    // make_bubble_like_state: idealized_cases.cpp:105-154
    const float sign = kind == "density_current" ? -1.0f : 1.0f;
    const float dth = sign * std::fabs(c->theta_perturbation);
    const float x0 = c->center_x_fraction * (float)(nx - 1) * (float)g->dx;
    const float y0 = c->center_y_fraction * (float)(ny - 1) * (float)g->dy;
    const float z0 = c->center_z_fraction * (float)g->z_top;
    const float rx = std::max(c->radius_x_fraction * (float)nx * (float)g->dx, 1.0f);
    const float ry = std::max(c->radius_y_fraction * (float)ny * (float)g->dy, 1.0f);
    const float rz = std::max(c->radius_z_fraction * (float)g->z_top, 1.0f);
    const bool hydro = kind == "hydrostatic_warm_bubble";
    if (hydro) fill_const(0.0f, c->theta_ref, c->u_background, c->v_background, c->w_background);
    else fill_const(c->rho_background, c->theta_background, c->u_background, c->v_background, c->w_background);
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const float x = (float)i * (float)g->dx, y = (float)j * (float)g->dy;
          const float z = z_center(*g, i, j, k);
          const float wgt = bubble_weight((x - x0) / rx, (y - y0) / ry, (z - z0) / rz);
          if (hydro) {
            const float r = hydrostatic_rho_at_height(c->rho_surface, c->theta_ref, z);
            rho[cidx(*g, i, j, k)] = r;
            rt[cidx(*g, i, j, k)] = r * (c->theta_ref + dth * wgt);
          } else {
            rt[cidx(*g, i, j, k)] = c->rho_background * (c->theta_background + dth * wgt);
          }
        }
    if (hydro) { fill(out->mom_u, nu, 0.0f); fill(out->mom_v, nv, 0.0f); fill(out->mom_w, nw, 0.0f); }
    return GWM_B200_OK;
  }
  if (kind == "hydrostatic_rest" || kind == "mountain_wave_background") {
    // make_hydrostatic_rest_state (dry_core.cu:363-398) / make_mountain_wave_background_state
    // (idealized_cases.cpp:182-223)
    const bool mw = kind == "mountain_wave_background";
    const float ub = mw ? c->u_background : 0.0f, vb = mw ? c->v_background : 0.0f, wb = mw ? c->w_background : 0.0f;
    fill_const(0.0f, c->theta_ref, ub, vb, wb);
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const float r = hydrostatic_rho_at_height(c->rho_surface, c->theta_ref, z_center(*g, i, j, k));
          rho[cidx(*g, i, j, k)] = r;
          rt[cidx(*g, i, j, k)] = r * c->theta_ref;
        }
    auto R = [&](int i, int j, int k) { return rho[cidx(*g, i, j, k)]; };
    if (out->mom_u)  // set_background_face_momenta: idealized_cases.cpp:36-103
      for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i <= nx; ++i) {
            const float fd = (nx == 1 || i <= 0) ? R(0, j, k) : (i >= nx ? R(nx - 1, j, k) : 0.5f * (R(i - 1, j, k) + R(i, j, k)));
            out->mom_u[((size_t)k * ny + j) * (nx + 1) + i] = fd * ub;
          }
    if (out->mom_v)
      for (int k = 0; k < nz; ++k)
        for (int j = 0; j <= ny; ++j)
          for (int i = 0; i < nx; ++i) {
            const float fd = (ny == 1 || j <= 0) ? R(i, 0, k) : (j >= ny ? R(i, ny - 1, k) : 0.5f * (R(i, j - 1, k) + R(i, j, k)));
            out->mom_v[((size_t)k * (ny + 1) + j) * nx + i] = fd * vb;
          }
    if (out->mom_w)
      for (int k = 0; k <= nz; ++k)
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i < nx; ++i) {
            const float fd = (nz == 1 || k <= 0) ? R(i, j, 0) : (k >= nz ? R(i, j, nz - 1) : 0.5f * (R(i, j, k - 1) + R(i, j, k)));
            out->mom_w[((size_t)k * ny + j) * nx + i] = fd * wb;
          }
    return GWM_B200_OK;
  }
  if (kind == "stratified_mountain_wave") {
    // constant N: theta(z) = theta0 exp(N^2 z / g); hydrostatic Exner function
    // pi(z) = pi_s - g^2 / (cp theta0 N^2) (1 - exp(-N^2 z / g)), p = p0 pi^(1/kappa)
    const double n2 = (double)c->brunt_vaisala * (double)c->brunt_vaisala;
    if (n2 <= 0.0) return GWM_B200_ERR_ARG;
    const double th0 = c->theta_ref, gg = kG, cpd = (double)cp();
    const double pis = std::pow((double)c->p_surface / kP0, (double)kKappa);
    fill(out->mom_w, nw, 0.0f);
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const double z = z_center(*g, i, j, k);
          const double th = th0 * std::exp(n2 * z / gg);
          const double pi = std::max(1.0e-4, pis - gg * gg / (cpd * th0 * n2) * (1.0 - std::exp(-n2 * z / gg)));
          const float p = (float)(kP0 * std::pow(pi, 1.0 / kKappa));
          const float r = eos_rho(p, (float)th);
          rho[cidx(*g, i, j, k)] = r;
          rt[cidx(*g, i, j, k)] = r * (float)th;
        }
    auto R = [&](int i, int j, int k) { return rho[cidx(*g, i, j, k)]; };
    const float ub = c->u_background, vb = c->v_background;
    if (out->mom_u)  // face-averaged density times the background wind (idealized_cases.cpp:36-103)
      for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i <= nx; ++i) {
            const float fd = (nx == 1 || i <= 0) ? R(0, j, k) : (i >= nx ? R(nx - 1, j, k) : 0.5f * (R(i - 1, j, k) + R(i, j, k)));
            out->mom_u[((size_t)k * ny + j) * (nx + 1) + i] = fd * ub;
          }
    if (out->mom_v)
      for (int k = 0; k < nz; ++k)
        for (int j = 0; j <= ny; ++j)
          for (int i = 0; i < nx; ++i) {
            const float fd = (ny == 1 || j <= 0) ? R(i, 0, k) : (j >= ny ? R(i, ny - 1, k) : 0.5f * (R(i, j - 1, k) + R(i, j, k)));
            out->mom_v[((size_t)k * (ny + 1) + j) * nx + i] = fd * vb;
          }
    return GWM_B200_OK;
  }
  if (kind == "moist_sounding") {
    fill(out->mom_u, nu, 0.0f); fill(out->mom_v, nv, 0.0f); fill(out->mom_w, nw, 0.0f);
    const float th0 = c->theta_ref;
    auto theta_env = [&](float z) { return z <= 1000.0f ? th0 : th0 + c->theta_lapse_k_per_m * (z - 1000.0f); };
    // surface (z = 0) pressure p_surface, constant theta below the first level
    std::vector<float> p(nz), r(nz), th(nz);
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        for (int k = 0; k < nz; ++k) {
          const float z = z_center(*g, i, j, k);
          float t = theta_env(z);
          if (z < c->noise_depth_m && c->noise_rms_k > 0.0f) {
            const uint64_t q = cidx(*g, i, j, k);
            const uint64_t h1 = splitmix64(c->seed * 0x100000001B3ull ^ (2 * q));
            const uint64_t h2 = splitmix64(c->seed * 0x100000001B3ull ^ (2 * q + 1));
            const double u1 = unit_open(h1), u2 = unit_open(h2);
            const double n = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * 3.14159265358979323846 * u2);
            t += (float)(c->noise_rms_k * n);
          }
          th[k] = t;
        }
        // first level from the surface with an isentropic (constant theta) layer
        const float z0 = z_center(*g, i, j, 0);
        const float exs = std::pow(c->p_surface / kP0, kKappa);
        const float ex0 = std::max(1.0e-4f, exs - kG * z0 / (cp() * th[0]));
        p[0] = kP0 * std::pow(ex0, 1.0f / kKappa);
        r[0] = eos_rho(p[0], th[0]);
        for (int k = 1; k < nz; ++k) {  // prepared_case_init.cpp:357-377
          const float dz = z_center(*g, i, j, k) - z_center(*g, i, j, k - 1);
          float pn = std::max(1.0f, p[k - 1] - kG * r[k - 1] * dz);
          for (int it = 0; it < 4; ++it) {
            const float rn = eos_rho(pn, th[k]);
            pn = std::max(p[k - 1] - kG * 0.5f * (r[k - 1] + rn) * dz, 1.0f);
          }
          p[k] = pn;
          r[k] = eos_rho(pn, th[k]);
        }
        // qv: relative humidity below rh_top, then exponential decay from the last
        // level below rh_top, floored at qv_floor
        float qv_last = -1.0f, z_last = 0.0f;
        for (int k = 0; k < nz; ++k) {
          const float z = z_center(*g, i, j, k);
          const float ex = std::pow(std::max(p[k] / kP0, 1.0e-6f), kKappa);
          float qv;
          if (z < c->rh_top_m || k == 0) {
            qv = c->relative_humidity * qsat(th[k] * ex, p[k]);
            if (z < c->rh_top_m || qv_last < 0.0f) { qv_last = qv; z_last = z; }
          } else {
            qv = std::max(c->qv_floor, qv_last * std::exp(-(z - z_last) / c->qv_scale_height_m));
          }
          const size_t q = cidx(*g, i, j, k);
          rho[q] = r[k];
          rt[q] = rho_theta_from_pressure(p[k]);
          if (out->qv) out->qv[q] = r[k] * std::max(qv, 0.0f);
        }
      }
    return GWM_B200_OK;
  }
  return GWM_B200_ERR_ARG;
}

int gwm_b200_build_terrain(const char* kind_c, int nx, int ny, double dx, double dy,
                           const gwm_b200_terrain_params* t, float* out) {
  if (!kind_c || !t || !out || nx <= 0 || ny <= 0) return GWM_B200_ERR_ARG;
  const std::string kind(kind_c);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      float h = 0.0f;
      if (kind == "cosine_mountain") {  // idealized_domain_builder.cpp:14-35
        if (t->height > 0.0) {
          const double x = nx > 1 ? (double)i / (double)(nx - 1) : 0.0;
          const double y = ny > 1 ? (double)j / (double)(ny - 1) : 0.0;
          const double ddx = (x - t->center_x_fraction) / t->half_width_x;
          const double ddy = (y - t->center_y_fraction) / t->half_width_y;
          if (std::abs(ddx) < 1.0 && std::abs(ddy) < 1.0)
            h = (float)(t->height * 0.5 * (1.0 + std::cos(3.14159265358979323846 * ddx)) * 0.5 *
                        (1.0 + std::cos(3.14159265358979323846 * ddy)));
        }
      } else if (kind == "agnesi") {  // 3-D Witch of Agnesi
        const double xc = t->center_x_fraction * (double)(nx - 1) * dx;
        const double yc = t->center_y_fraction * (double)(ny - 1) * dy;
        const double rx = ((double)i * dx - xc) / t->half_width_x;
        const double ry = ((double)j * dy - yc) / t->half_width_y;
        h = (float)(t->height / std::pow(1.0 + rx * rx + ry * ry, 1.5));
      } else if (kind != "flat") {
        return GWM_B200_ERR_ARG;
      }
      out[(size_t)j * nx + i] = h;
    }
  return GWM_B200_OK;
}

}  // extern "C"
