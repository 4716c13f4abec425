// gwm_oracle.hpp — CPU ORACLE (test infrastructure only).
//
// This header is a plain C++ restatement of the reference's time-step hot path
// (FahrenheitResearch/gpu-wm-next), templated on the arithmetic type T so the
// same code runs as an FP32 replay of the reference arithmetic and as the FP64
// standard that both are measured against.  It is NEVER linked into the product:
// only tests/, the smoke() check and bench.py's CPU-baseline leg load it, always
// as the checker.
//
// Every function cites the reference file:line it restates.  The data layout
// is the reference's own: one halo-padded array per virtual rank, x fastest,
// storage_index = (k*pitch_y + j+h)*pitch_x + i+h (include/gwm/state/field3d.hpp:49-54),
// face fields one longer along their orientation (include/gwm/state/face_field.hpp:16-23).
//
// Deliberate differences from the reference, all of them ordering-only:
//  * the per-level rho/p means of the flat-terrain fast mode use float atomics in
//    the reference (src/dycore/dry_fast_modes.cu:42-57, order nondeterministic);
//    here they are sequential sums in (rank,k,j,i) order, in T.
//  * constants are the reference's float literals promoted to T, so the FP64
//    oracle computes with the same constant values as the FP32 code.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace gwo {

inline void require(bool ok, const char* msg) {
  if (!ok) throw std::runtime_error(msg);
}

// ---------------------------------------------------------------------------
// Constants: include/gwm/core/dry_thermo.hpp:17-19, moist_thermo.hpp:18-21,
// src/dycore/dry_core.cu:20.
template <class T> struct K {
  static constexpr T Rd = T(287.05f);
  static constexpr T p0 = T(100000.0f);
  static constexpr T kappa = T(0.2854f);
  static constexpr T Rv = T(461.5f);
  static constexpr T Lv = T(2.5e6f);
};

template <class T> inline T fmx(T a, T b) { return std::fmax(a, b); }
template <class T> inline T fmn(T a, T b) { return std::fmin(a, b); }

// dry_thermo.hpp:21-24
template <class T> inline T theta_from_conserved(T rho, T rt) {
  return rt / fmx(rho, T(1.0e-6f));
}
// dry_thermo.hpp:26-33
template <class T> inline T pressure_from_rho_theta(T rho, T rt) {
  const T theta = theta_from_conserved(rho, rt);
  const T ratio = fmx(rho * K<T>::Rd * theta / K<T>::p0, T(1.0e-6f));
  return K<T>::p0 * std::pow(ratio, T(1) / (T(1) - K<T>::kappa));
}
// dry_thermo.hpp:35-40
template <class T> inline T rho_from_pressure_theta(T p, T theta) {
  const T exner = std::pow(fmx(p / K<T>::p0, T(1.0e-6f)), K<T>::kappa);
  return p / fmx(K<T>::Rd * theta * exner, T(1.0e-6f));
}
// dry_thermo.hpp:42-44
template <class T> inline T dry_cp() { return K<T>::Rd / K<T>::kappa; }

// moist_thermo.hpp:23-29
template <class T> inline T sat_vapor_pressure(T tk) {
  const T tc = tk - T(273.15f);
  const T es_hpa = T(6.112f) * std::exp((T(17.67f) * tc) / fmx(tc + T(243.5f), T(1.0e-6f)));
  return es_hpa * T(100.0f);
}
// moist_thermo.hpp:31-36
template <class T> inline T qsat(T tk, T p) {
  const T eps = K<T>::Rd / K<T>::Rv;
  const T es = sat_vapor_pressure(tk);
  const T denom = fmx(p - (T(1) - eps) * es, T(1000.0f));
  return fmn(fmx(eps * es / denom, T(0)), T(0.05f));
}
// moist_thermo.hpp:55-62
template <class T> inline T temperature_from_conserved(T rho, T rt) {
  const T theta = theta_from_conserved(rho, rt);
  const T p = pressure_from_rho_theta(rho, rt);
  const T exner = std::pow(fmx(p / K<T>::p0, T(1.0e-6f)), K<T>::kappa);
  return theta * exner;
}

// ---------------------------------------------------------------------------
// Layout: src/comm/virtual_rank_layout.cpp:7-47, include/gwm/domain/subdomain_descriptor.hpp:7-26
struct Desc {
  int rank = 0, cx = 0, cy = 0, rx = 1, ry = 1, gnx = 0, gny = 0, nz = 0, halo = 0;
  int i0 = 0, i1 = 0, j0 = 0, j1 = 0;
  bool px = true, py = true;
  int nxl() const { return i1 - i0; }
  int nyl() const { return j1 - j0; }
};

inline std::vector<Desc> build_layout(int gnx, int gny, int nz, int halo, int rx, int ry,
                                      bool px, bool py) {
  std::vector<Desc> out;
  const int bnx = gnx / rx, rnx = gnx % rx, bny = gny / ry, rny = gny % ry;
  int jb = 0;
  for (int y = 0; y < ry; ++y) {
    const int nyl = bny + (y < rny ? 1 : 0);
    int ib = 0;
    for (int x = 0; x < rx; ++x) {
      const int nxl = bnx + (x < rnx ? 1 : 0);
      Desc d;
      d.rank = (int)out.size(); d.cx = x; d.cy = y; d.rx = rx; d.ry = ry;
      d.gnx = gnx; d.gny = gny; d.nz = nz; d.halo = halo;
      d.i0 = ib; d.i1 = ib + nxl; d.j0 = jb; d.j1 = jb + nyl; d.px = px; d.py = py;
      out.push_back(d);
      ib += nxl;
    }
    jb += nyl;
  }
  return out;
}

struct Nbr { int w = -1, e = -1, s = -1, n = -1; };

// src/comm/cartesian_topology.cpp:17-74
inline int rank_at(const std::vector<Desc>& L, int cx, int cy, bool px, bool py) {
  if (L.empty()) return -1;
  const int rx = L.front().rx, ry = L.front().ry;
  auto wrap = [](int v, int n) { int w = v % n; return w < 0 ? w + n : w; };
  if (px) cx = wrap(cx, rx); else if (cx < 0 || cx >= rx) return -1;
  if (py) cy = wrap(cy, ry); else if (cy < 0 || cy >= ry) return -1;
  for (const auto& c : L) if (c.cx == cx && c.cy == cy) return c.rank;
  return -1;
}
inline Nbr neighbors(const std::vector<Desc>& L, const Desc& d) {
  Nbr n;
  n.w = rank_at(L, d.cx - 1, d.cy, d.px, d.py);
  n.e = rank_at(L, d.cx + 1, d.cy, d.px, d.py);
  n.s = rank_at(L, d.cx, d.cy - 1, d.px, d.py);
  n.n = rank_at(L, d.cx, d.cy + 1, d.px, d.py);
  return n;
}

// ---------------------------------------------------------------------------
// Fields: include/gwm/state/field3d.hpp:11-132, face_field.hpp:11-32
enum Orient { CELL = 0, FX = 1, FY = 2, FZ = 3 };

template <class T> struct Field {
  int nx = 0, ny = 0, nz = 0, h = 0;
  Orient o = CELL;
  std::vector<T> d;
  Field() = default;
  Field(int nx_, int ny_, int nz_, int h_, Orient o_ = CELL)
      : nx(nx_), ny(ny_), nz(nz_), h(h_), o(o_),
        d((size_t)(nx_ + 2 * h_) * (ny_ + 2 * h_) * nz_, T(0)) {}
  int px() const { return nx + 2 * h; }
  int py() const { return ny + 2 * h; }
  size_t idx(int i, int j, int k) const {
    return ((size_t)k * py() + (size_t)(j + h)) * px() + (size_t)(i + h);
  }
  T& operator()(int i, int j, int k) { return d[idx(i, j, k)]; }
  const T& operator()(int i, int j, int k) const { return d[idx(i, j, k)]; }
  void fill(T v) { std::fill(d.begin(), d.end(), v); }
  double owned_sum() const {  // field3d.hpp:82-92
    double s = 0.0;
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) s += (double)(*this)(i, j, k);
    return s;
  }
};

// FaceField(nx,ny,nz,halo,orientation): face_field.hpp:16-23
template <class T> Field<T> make_face(int nx, int ny, int nz, int h, Orient o) {
  return Field<T>(nx + (o == FX), ny + (o == FY), nz + (o == FZ), h, o);
}

// DryState: include/gwm/dycore/dry_core.hpp:14-34
template <class T> struct DryState {
  Field<T> rho, rt, mu, mv, mw;
  DryState() = default;
  DryState(int nx, int ny, int nz, int h)
      : rho(nx, ny, nz, h), rt(nx, ny, nz, h), mu(make_face<T>(nx, ny, nz, h, FX)),
        mv(make_face<T>(nx, ny, nz, h, FY)), mw(make_face<T>(nx, ny, nz, h, FZ)) {}
};

// ---------------------------------------------------------------------------
// Halo exchange over virtual ranks: src/comm/halo_exchange.cpp
// Absent neighbours deliver zeros (fresh buffers, :289-301, :593-600).
template <class T>
void exchange_scalar(std::vector<Field<T>>& F, const std::vector<Desc>& L) {
  // halo_exchange.cpp:563-620 with pack/unpack :313-373
  const size_t n = L.size();
  require(F.size() == n, "Field/layout size mismatch in exchange_scalar");
  std::vector<Nbr> nb(n);
  for (size_t r = 0; r < n; ++r) nb[r] = neighbors(L, L[r]);
  std::vector<std::vector<T>> ws(n), es(n), ss(n), ns(n);
  for (size_t r = 0; r < n; ++r) {
    const Desc& d = L[r];
    for (int k = 0; k < d.nz; ++k)
      for (int j = 0; j < d.nyl(); ++j)
        for (int hh = 0; hh < d.halo; ++hh) {
          ws[r].push_back(F[r](hh, j, k));
          es[r].push_back(F[r](d.nxl() - d.halo + hh, j, k));
        }
  }
  for (size_t r = 0; r < n; ++r) {
    const Desc& d = L[r];
    const size_t cnt = (size_t)d.halo * d.nyl() * d.nz;
    std::vector<T> wr(cnt, T(0)), er(cnt, T(0));
    if (nb[r].w >= 0) wr = es[nb[r].w];
    if (nb[r].e >= 0) er = ws[nb[r].e];
    size_t a = 0, b = 0;
    for (int k = 0; k < d.nz; ++k)
      for (int j = 0; j < d.nyl(); ++j)
        for (int hh = 0; hh < d.halo; ++hh) {
          F[r](-d.halo + hh, j, k) = wr[a++];
          F[r](d.nxl() + hh, j, k) = er[b++];
        }
  }
  for (size_t r = 0; r < n; ++r) {
    const Desc& d = L[r];
    for (int k = 0; k < d.nz; ++k)
      for (int hh = 0; hh < d.halo; ++hh)
        for (int i = -d.halo; i < d.nxl() + d.halo; ++i) {
          ss[r].push_back(F[r](i, hh, k));
          ns[r].push_back(F[r](i, d.nyl() - d.halo + hh, k));
        }
  }
  for (size_t r = 0; r < n; ++r) {
    const Desc& d = L[r];
    const size_t cnt = (size_t)d.halo * (d.nxl() + 2 * d.halo) * d.nz;
    std::vector<T> sr(cnt, T(0)), nr(cnt, T(0));
    if (nb[r].s >= 0) sr = ns[nb[r].s];
    if (nb[r].n >= 0) nr = ss[nb[r].n];
    size_t a = 0, b = 0;
    for (int k = 0; k < d.nz; ++k)
      for (int hh = 0; hh < d.halo; ++hh)
        for (int i = -d.halo; i < d.nxl() + d.halo; ++i) {
          F[r](i, -d.halo + hh, k) = sr[a++];
          F[r](i, d.nyl() + hh, k) = nr[b++];
        }
  }
}

template <class T>
void exchange_face(std::vector<Field<T>*>& F, const std::vector<Desc>& L) {
  // halo_exchange.cpp:148-215 with pack/unpack :32-116
  const size_t n = L.size();
  require(F.size() == n, "Field/layout size mismatch in exchange_face");
  if (n == 0) return;
  const Orient o = F[0]->o;
  std::vector<Nbr> nb(n);
  for (size_t r = 0; r < n; ++r) nb[r] = neighbors(L, L[r]);
  std::vector<std::vector<T>> ws(n), es(n), ss(n), ns(n);
  for (size_t r = 0; r < n; ++r) {
    const Desc& d = L[r];
    Field<T>& s = *F[r];
    for (int k = 0; k < s.nz; ++k)
      for (int j = 0; j < s.ny; ++j)
        for (int hh = 0; hh < d.halo; ++hh) {
          int wi = hh, ei = s.nx - d.halo + hh;
          if (o == FX) { wi = 1 + hh; ei = d.nxl() - d.halo + hh; }
          ws[r].push_back(s(wi, j, k));
          es[r].push_back(s(ei, j, k));
        }
  }
  for (size_t r = 0; r < n; ++r) {
    const Desc& d = L[r];
    Field<T>& s = *F[r];
    const size_t cnt = (size_t)d.halo * s.ny * s.nz;
    std::vector<T> wr(cnt, T(0)), er(cnt, T(0));
    if (nb[r].w >= 0) wr = es[nb[r].w];
    if (nb[r].e >= 0) er = ws[nb[r].e];
    size_t a = 0, b = 0;
    for (int k = 0; k < s.nz; ++k)
      for (int j = 0; j < s.ny; ++j)
        for (int hh = 0; hh < d.halo; ++hh) {
          s(-d.halo + hh, j, k) = wr[a++];
          s(s.nx + hh, j, k) = er[b++];
        }
  }
  for (size_t r = 0; r < n; ++r) {
    const Desc& d = L[r];
    Field<T>& s = *F[r];
    for (int k = 0; k < s.nz; ++k)
      for (int hh = 0; hh < d.halo; ++hh)
        for (int i = -d.halo; i < s.nx + d.halo; ++i) {
          int sj = hh, nj = s.ny - d.halo + hh;
          if (o == FY) { sj = 1 + hh; nj = d.nyl() - d.halo + hh; }
          ss[r].push_back(s(i, sj, k));
          ns[r].push_back(s(i, nj, k));
        }
  }
  for (size_t r = 0; r < n; ++r) {
    const Desc& d = L[r];
    Field<T>& s = *F[r];
    const size_t cnt = (size_t)d.halo * (s.nx + 2 * d.halo) * s.nz;
    std::vector<T> sr(cnt, T(0)), nr(cnt, T(0));
    if (nb[r].s >= 0) sr = ns[nb[r].s];
    if (nb[r].n >= 0) nr = ss[nb[r].n];
    size_t a = 0, b = 0;
    for (int k = 0; k < s.nz; ++k)
      for (int hh = 0; hh < d.halo; ++hh)
        for (int i = -d.halo; i < s.nx + d.halo; ++i) {
          s(i, -d.halo + hh, k) = sr[a++];
          s(i, s.ny + hh, k) = nr[b++];
        }
  }
}

template <class T>
void sync_face_interfaces(std::vector<Field<T>*>& F, const std::vector<Desc>& L) {
  // halo_exchange.cpp:217-285 (virtual-rank path)
  const size_t n = L.size();
  if (n == 0) return;
  const Orient o = F[0]->o;
  if (o == FZ) return;
  for (size_t r = 0; r < n; ++r) {
    Field<T>& s = *F[r];
    const Desc& d = L[r];
    const Nbr nb = neighbors(L, d);
    if (o == FX && nb.e >= 0 && ((int)r < nb.e || nb.e == (int)r)) {
      Field<T>& p = *F[nb.e];
      for (int k = 0; k < s.nz; ++k)
        for (int j = 0; j < d.nyl(); ++j) {
          const T avg = T(0.5f) * (s(d.nxl(), j, k) + p(0, j, k));
          s(d.nxl(), j, k) = avg;
          p(0, j, k) = avg;
        }
    }
    if (o == FY && nb.n >= 0 && ((int)r < nb.n || nb.n == (int)r)) {
      Field<T>& p = *F[nb.n];
      for (int k = 0; k < s.nz; ++k)
        for (int i = 0; i < d.nxl(); ++i) {
          const T avg = T(0.5f) * (s(i, d.nyl(), k) + p(i, 0, k));
          s(i, d.nyl(), k) = avg;
          p(i, 0, k) = avg;
        }
    }
  }
}

template <class T>
std::vector<Field<T>*> ptrs(std::vector<Field<T>>& v) {
  std::vector<Field<T>*> p;
  for (auto& f : v) p.push_back(&f);
  return p;
}

// The exchange sequence used before every face-field consumer:
// src/dycore/dry_core.cu:451-457, dry_fast_modes.cu:463-469, 614-620, dry_transport.cu:223-229
template <class T>
void exchange_momenta(std::vector<Field<T>*>& U, std::vector<Field<T>*>& V,
                      std::vector<Field<T>*>& W, const std::vector<Desc>& L) {
  exchange_face(U, L);
  exchange_face(V, L);
  exchange_face(W, L);
  sync_face_interfaces(U, L);
  sync_face_interfaces(V, L);
  exchange_face(U, L);
  exchange_face(V, L);
}

// ---------------------------------------------------------------------------
// Metrics: include/gwm/domain/grid_metrics.hpp:87-239.  Metric arrays are
// unpadded global fields indexed (k*ny + j)*nx + i.  Computed in double, stored
// in T.  Extension (not in the reference): caller-supplied eta interfaces for
// stretched levels; eta centres are then interface midpoints (for uniform
// levels this equals the reference's (k+0.5)/nz).
template <class T> struct Metrics {
  int nx = 0, ny = 0, nz = 0;
  double dx = 0, dy = 0, z_top = 0, taper = 0.25;
  bool px = true, py = true;
  std::vector<double> eta_i, eta_c, bw_i, bw_c, z_i, z_c;
  std::vector<T> terrain, zc, zi, inv_dz_cell, inv_dz_face;
  size_t m(int i, int j, int k) const { return ((size_t)k * ny + j) * nx + i; }
};

template <class T>
Metrics<T> make_hybrid_height(int nx, int ny, int nz, double dx, double dy, double z_top,
                              const std::vector<double>& terrain, double taper, bool px,
                              bool py, const double* eta_interfaces = nullptr) {
  Metrics<T> M;
  M.nx = nx; M.ny = ny; M.nz = nz; M.dx = dx; M.dy = dy; M.z_top = z_top; M.taper = taper;
  M.px = px; M.py = py;
  M.eta_i.resize(nz + 1); M.eta_c.resize(nz); M.bw_i.resize(nz + 1); M.bw_c.resize(nz);
  M.z_i.resize(nz + 1); M.z_c.resize(nz);
  auto weight = [taper](double eta) {  // grid_metrics.hpp:126-144
    if (eta <= 0.0) return 1.0;
    if (eta >= 1.0) return 0.0;
    if (taper <= 0.0) {
      const double s = std::clamp(eta, 0.0, 1.0);
      return 1.0 - s * s * (3.0 - 2.0 * s);
    }
    if (eta <= taper) return 1.0;
    const double s = std::clamp((eta - taper) / std::max(1.0e-9, 1.0 - taper), 0.0, 1.0);
    return 1.0 - s * s * (3.0 - 2.0 * s);
  };
  for (int k = 0; k <= nz; ++k) {  // grid_metrics.hpp:146-161
    M.eta_i[k] = eta_interfaces ? eta_interfaces[k] : (double)k / (double)nz;
    M.bw_i[k] = weight(M.eta_i[k]);
    M.z_i[k] = M.eta_i[k] * z_top;
  }
  for (int k = 0; k < nz; ++k) {
    M.eta_c[k] = eta_interfaces ? 0.5 * (eta_interfaces[k] + eta_interfaces[k + 1])
                                : ((double)k + 0.5) / (double)nz;
    M.bw_c[k] = weight(M.eta_c[k]);
    M.z_c[k] = M.eta_c[k] * z_top;
  }
  const size_t plane = (size_t)nx * ny;
  M.terrain.assign(plane, T(0));
  M.zc.assign(plane * nz, T(0));
  M.zi.assign(plane * (nz + 1), T(0));
  M.inv_dz_cell.assign(plane * nz, T(0));
  M.inv_dz_face.assign(plane * (nz + 1), T(0));
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const double th = terrain[(size_t)j * nx + i];
      M.terrain[(size_t)j * nx + i] = (T)th;
      for (int k = 0; k <= nz; ++k) {  // grid_metrics.hpp:204-222
        M.zi[M.m(i, j, k)] = (T)(M.z_i[k] + M.bw_i[k] * th);
        if (k == 0 || k == nz) {
          M.inv_dz_face[M.m(i, j, k)] = T(0);
        } else {
          const double dzf = (M.z_c[k] + M.bw_c[k] * th) - (M.z_c[k - 1] + M.bw_c[k - 1] * th);
          M.inv_dz_face[M.m(i, j, k)] = (T)(1.0 / std::max(dzf, 1.0e-6));
        }
      }
      for (int k = 0; k < nz; ++k) {  // grid_metrics.hpp:224-234
        M.zc[M.m(i, j, k)] = (T)(M.z_c[k] + M.bw_c[k] * th);
        const double dzc = (double)M.zi[M.m(i, j, k + 1)] - (double)M.zi[M.m(i, j, k)];
        M.inv_dz_cell[M.m(i, j, k)] = (T)(1.0 / std::max(dzc, 1.0e-6));
      }
    }
  return M;
}

inline int wrap_metric(int idx, int n, bool periodic) {  // dry_fast_modes.cu:24-30
  if (!periodic) return idx;
  const int m = idx % n;
  return m < 0 ? m + n : m;
}

// ---------------------------------------------------------------------------
// Step configuration: include/gwm/dycore/dry_core.hpp:50-56
template <class T> struct StepCfg {
  T dt = T(2.0f);
  int fast_substeps = 1;
  T gravity = T(9.81f);
  bool fast_hmom = true;
  bool fast_density = true;
  bool fast_modes = true;
  // Rayleigh damping layer (extension; not in the reference): per-level rates at cell
  // centres and Z faces, and the per-level momentum profiles u, v relax to (empty: off)
  std::vector<T> damp_c, damp_f, u_ref, v_ref;
};

// Rayleigh damping rate tau(z) = rate * sin^2(pi/2 (z - z_d)/(z_top - z_d)) above z_d,
// evaluated at a level's terrain-free height eta * z_top.
inline double rayleigh_rate(double z, double z_d, double z_top, double rate) {
  if (rate <= 0.0 || z <= z_d || z_top <= z_d) return 0.0;
  const double s = std::sin(0.5 * 3.14159265358979323846 * std::min(1.0, (z - z_d) / (z_top - z_d)));
  return rate * s * s;
}

template <class T> using States = std::vector<DryState<T>>;

template <class T>
void copy_state(DryState<T>& dst, const DryState<T>& src) { dst = src; }

// ---------------------------------------------------------------------------
// Slow tendencies: src/dycore/dry_core.cu:400-539 and the kernels it launches.
template <class T>
void compute_slow_tendencies(const States<T>& S, const std::vector<Desc>& L,
                             const Metrics<T>& M, const StepCfg<T>& cfg, States<T>& out) {
  const size_t n = S.size();
  require(n == L.size(), "State/layout size mismatch in compute_slow_tendencies");
  std::vector<Field<T>> R(n), RT(n), U(n), V(n), W(n), P(n);
  for (size_t r = 0; r < n; ++r) {
    R[r] = S[r].rho; RT[r] = S[r].rt; U[r] = S[r].mu; V[r] = S[r].mv; W[r] = S[r].mw;
  }
  exchange_scalar(R, L);  // dry_core.cu:449-457
  exchange_scalar(RT, L);
  auto Up = ptrs(U), Vp = ptrs(V), Wp = ptrs(W);
  exchange_momenta(Up, Vp, Wp, L);
  for (size_t r = 0; r < n; ++r) {  // compute_dry_pressure_fields, dry_pressure_gradient.cu:177-202
    P[r] = R[r];
    for (size_t q = 0; q < P[r].d.size(); ++q)
      P[r].d[q] = pressure_from_rho_theta(R[r].d[q], RT[r].d[q]);
  }
  // theta level mean over owned cells, FP64 accumulate: dry_core.cu:462-490
  std::vector<double> tsum(M.nz, 0.0);
  std::vector<uint64_t> tcnt(M.nz, 0);
  for (size_t r = 0; r < n; ++r)
    for (int k = 0; k < S[r].rho.nz; ++k)
      for (int j = 0; j < S[r].rho.ny; ++j)
        for (int i = 0; i < S[r].rho.nx; ++i) {
          const T rho = S[r].rho(i, j, k);
          const T th = S[r].rt(i, j, k) / std::max(rho, T(1.0e-6f));
          tsum[k] += (double)th;
          tcnt[k] += 1;
        }
  std::vector<T> theta_ref(M.nz);
  for (int k = 0; k < M.nz; ++k)
    theta_ref[k] = (T)(tsum[k] / (double)std::max<uint64_t>(1, tcnt[k]));

  out.resize(n);
  const T dx = (T)M.dx, dy = (T)M.dy;
  for (size_t r = 0; r < n; ++r) {
    const Desc& d = L[r];
    const int nx = d.nxl(), ny = d.nyl(), nz = d.nz;
    const Nbr nb = neighbors(L, d);
    const bool ow = nb.w < 0, oe = nb.e < 0, os = nb.s < 0, on = nb.n < 0;
    out[r] = DryState<T>(nx, ny, nz, d.halo);  // fill_zero: dry_core.cu:327-334
    DryState<T>& o = out[r];
    const Field<T>&rho = R[r], &rt = RT[r], &u = U[r], &v = V[r], &w = W[r], &p = P[r];
    // K2 compute_cell_tendencies_kernel: dry_core.cu:62-144
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const T fw = u(i, j, k), fe = u(i + 1, j, k), fs = v(i, j, k), fn = v(i, j + 1, k);
          const T fb = w(i, j, k), ft = w(i, j, k + 1);
          const T idz = M.inv_dz_cell[M.m(d.i0 + i, d.j0 + j, k)];
          const T div = (fe - fw) / dx + (fn - fs) / dy + (ft - fb) * idz;
          o.rho(i, j, k) = -div;
          const T tc = theta_from_conserved(rho(i, j, k), rt(i, j, k));
          const T tw = theta_from_conserved(rho(i - 1, j, k), rt(i - 1, j, k));
          const T te = theta_from_conserved(rho(i + 1, j, k), rt(i + 1, j, k));
          const T ts = theta_from_conserved(rho(i, j - 1, k), rt(i, j - 1, k));
          const T tn = theta_from_conserved(rho(i, j + 1, k), rt(i, j + 1, k));
          const T tb = (k > 0) ? theta_from_conserved(rho(i, j, k - 1), rt(i, j, k - 1)) : tc;
          const T tt = (k + 1 < nz) ? theta_from_conserved(rho(i, j, k + 1), rt(i, j, k + 1)) : tc;
          const T gw = fw * (fw >= T(0) ? tw : tc);
          const T ge = fe * (fe >= T(0) ? tc : te);
          const T gs = fs * (fs >= T(0) ? ts : tc);
          const T gn = fn * (fn >= T(0) ? tc : tn);
          const T gb = fb * (fb >= T(0) ? tb : tc);
          const T gt = ft * (ft >= T(0) ? tc : tt);
          o.rt(i, j, k) = -((ge - gw) / dx + (gn - gs) / dy + (gt - gb) * idz);
        }
    // K16 cell velocities incl. halo: dry_momentum_flux.cu:36-73
    Field<T> uc(nx, ny, nz, d.halo), vc(nx, ny, nz, d.halo), wc(nx, ny, nz, d.halo);
    for (int k = 0; k < nz; ++k)
      for (int j = -d.halo; j < ny + d.halo; ++j)
        for (int i = -d.halo; i < nx + d.halo; ++i) {
          const T rr = std::max(rho(i, j, k), T(1.0e-6f));
          uc(i, j, k) = T(0.5f) * (u(i, j, k) + u(i + 1, j, k)) / rr;
          vc(i, j, k) = T(0.5f) * (v(i, j, k) + v(i, j + 1, k)) / rr;
          wc(i, j, k) = T(0.5f) * (w(i, j, k) + w(i, j, k + 1)) / rr;
        }
    auto upw = [](T a, T ql, T qr) { return a >= T(0) ? a * ql : a * qr; };
    // K17 u momentum flux: dry_momentum_flux.cu:79-156
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i <= nx; ++i) {
          if ((i == 0 && ow) || (i == nx && oe)) continue;
          const T qw = u(i - 1, j, k), qc = u(i, j, k), qe = u(i + 1, j, k);
          const T qs = u(i, j - 1, k), qn = u(i, j + 1, k);
          const T qb = (k > 0) ? u(i, j, k - 1) : qc;
          const T qt = (k + 1 < nz) ? u(i, j, k + 1) : qc;
          const T flw = upw(uc(i - 1, j, k), qw, qc);
          const T fle = upw(uc(i, j, k), qc, qe);
          T fls = 0, fln = 0, flb = 0, flt = 0;
          if (!(j == 0 && os)) fls = upw(T(0.5f) * (vc(i - 1, j - 1, k) + vc(i, j - 1, k)), qs, qc);
          if (!(j + 1 == ny && on)) fln = upw(T(0.5f) * (vc(i - 1, j, k) + vc(i, j, k)), qc, qn);
          if (k > 0) flb = upw(T(0.5f) * (wc(i - 1, j, k - 1) + wc(i, j, k - 1)), qb, qc);
          if (k + 1 < nz) flt = upw(T(0.5f) * (wc(i - 1, j, k) + wc(i, j, k)), qc, qt);
          const int gj = wrap_metric(d.j0 + j, M.ny, M.py);
          const int gl = wrap_metric(d.i0 + i - 1, M.nx, M.px);
          const int gr = wrap_metric(d.i0 + i, M.nx, M.px);
          const T idz = T(0.5f) * (M.inv_dz_cell[M.m(gl, gj, k)] + M.inv_dz_cell[M.m(gr, gj, k)]);
          o.mu(i, j, k) += -((fle - flw) / dx + (fln - fls) / dy + (flt - flb) * idz);
        }
    // K18 v momentum flux: dry_momentum_flux.cu:158-235
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j <= ny; ++j)
        for (int i = 0; i < nx; ++i) {
          if ((j == 0 && os) || (j == ny && on)) continue;
          const T qw = v(i - 1, j, k), qc = v(i, j, k), qe = v(i + 1, j, k);
          const T qs = v(i, j - 1, k), qn = v(i, j + 1, k);
          const T qb = (k > 0) ? v(i, j, k - 1) : qc;
          const T qt = (k + 1 < nz) ? v(i, j, k + 1) : qc;
          T flw = 0, fle = 0, flb = 0, flt = 0;
          if (!(i == 0 && ow)) flw = upw(T(0.5f) * (uc(i - 1, j - 1, k) + uc(i - 1, j, k)), qw, qc);
          if (!(i + 1 == nx && oe)) fle = upw(T(0.5f) * (uc(i, j - 1, k) + uc(i, j, k)), qc, qe);
          const T fls = upw(vc(i, j - 1, k), qs, qc);
          const T fln = upw(vc(i, j, k), qc, qn);
          if (k > 0) flb = upw(T(0.5f) * (wc(i, j - 1, k - 1) + wc(i, j, k - 1)), qb, qc);
          if (k + 1 < nz) flt = upw(T(0.5f) * (wc(i, j - 1, k) + wc(i, j, k)), qc, qt);
          const int gi = wrap_metric(d.i0 + i, M.nx, M.px);
          const int gs_ = wrap_metric(d.j0 + j - 1, M.ny, M.py);
          const int gn_ = wrap_metric(d.j0 + j, M.ny, M.py);
          const T idz = T(0.5f) * (M.inv_dz_cell[M.m(gi, gs_, k)] + M.inv_dz_cell[M.m(gi, gn_, k)]);
          o.mv(i, j, k) += -((fle - flw) / dx + (fln - fls) / dy + (flt - flb) * idz);
        }
    // K19 w momentum flux: dry_momentum_flux.cu:237-312
#pragma omp parallel for schedule(static)
    for (int kf = 1; kf < nz; ++kf)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const int kl = kf - 1, ku = kf;
          const T qw = w(i - 1, j, kf), qc = w(i, j, kf), qe = w(i + 1, j, kf);
          const T qs = w(i, j - 1, kf), qn = w(i, j + 1, kf);
          const T qb = w(i, j, kf - 1), qt = w(i, j, kf + 1);
          T flw = 0, fle = 0, fls = 0, fln = 0;
          if (!(i == 0 && ow)) flw = upw(T(0.5f) * (uc(i - 1, j, kl) + uc(i - 1, j, ku)), qw, qc);
          if (!(i + 1 == nx && oe)) fle = upw(T(0.5f) * (uc(i, j, kl) + uc(i, j, ku)), qc, qe);
          if (!(j == 0 && os)) fls = upw(T(0.5f) * (vc(i, j - 1, kl) + vc(i, j - 1, ku)), qs, qc);
          if (!(j + 1 == ny && on)) fln = upw(T(0.5f) * (vc(i, j, kl) + vc(i, j, ku)), qc, qn);
          const T flb = upw(wc(i, j, kl), qb, qc);
          const T flt = upw(wc(i, j, ku), qc, qt);
          const T idz = M.inv_dz_face[M.m(wrap_metric(d.i0 + i, M.nx, M.px),
                                          wrap_metric(d.j0 + j, M.ny, M.py), kf)];
          o.mw(i, j, kf) += -((fle - flw) / dx + (fln - fls) / dy + (flt - flb) * idz);
        }
    // K21/K22 horizontal pressure gradient: dry_pressure_gradient.cu:37-175
    auto vgrad = [&](int gi, int gj, int k, int li, int lj) -> T {
      if (nz == 1) return T(0);
      if (k == 0) {
        const T dz = M.zc[M.m(gi, gj, 1)] - M.zc[M.m(gi, gj, 0)];
        return (p(li, lj, 1) - p(li, lj, 0)) / std::max(dz, T(1.0e-6f));
      }
      if (k + 1 == nz) {
        const T dz = M.zc[M.m(gi, gj, k)] - M.zc[M.m(gi, gj, k - 1)];
        return (p(li, lj, k) - p(li, lj, k - 1)) / std::max(dz, T(1.0e-6f));
      }
      const T dz = M.zc[M.m(gi, gj, k + 1)] - M.zc[M.m(gi, gj, k - 1)];
      return (p(li, lj, k + 1) - p(li, lj, k - 1)) / std::max(dz, T(1.0e-6f));
    };
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i <= nx; ++i) {
          if ((i == 0 && ow) || (i == nx && oe)) continue;
          const T pl = p(i - 1, j, k), pr = p(i, j, k);
          const int gj = wrap_metric(d.j0 + j, M.ny, M.py);
          const int gl = wrap_metric(d.i0 + i - 1, M.nx, M.px);
          const int gr = wrap_metric(d.i0 + i, M.nx, M.px);
          const T dzdx = (M.zc[M.m(gr, gj, k)] - M.zc[M.m(gl, gj, k)]) / dx;
          const T dpdz = T(0.5f) * (vgrad(gl, gj, k, i - 1, j) + vgrad(gr, gj, k, i, j));
          o.mu(i, j, k) += -((pr - pl) / dx - dzdx * dpdz);
        }
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j <= ny; ++j)
        for (int i = 0; i < nx; ++i) {
          if ((j == 0 && os) || (j == ny && on)) continue;
          const T ps = p(i, j - 1, k), pn = p(i, j, k);
          const int gi = wrap_metric(d.i0 + i, M.nx, M.px);
          const int gs_ = wrap_metric(d.j0 + j - 1, M.ny, M.py);
          const int gn_ = wrap_metric(d.j0 + j, M.ny, M.py);
          const T dzdy = (M.zc[M.m(gi, gn_, k)] - M.zc[M.m(gi, gs_, k)]) / dy;
          const T dpdz = T(0.5f) * (vgrad(gi, gs_, k, i, j - 1) + vgrad(gi, gn_, k, i, j));
          o.mv(i, j, k) += -((pn - ps) / dy - dzdy * dpdz);
        }
    // K3 buoyancy: dry_core.cu:146-187
#pragma omp parallel for schedule(static)
    for (int kf = 1; kf < nz; ++kf)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          const int kl = kf - 1, ku = kf;
          const T rl = rho(i, j, kl), ru = rho(i, j, ku);
          const T tl = rt(i, j, kl) / std::max(rl, T(1.0e-6f));
          const T tu = rt(i, j, ku) / std::max(ru, T(1.0e-6f));
          const T tf = T(0.5f) * (tl + tu);
          const T trf = T(0.5f) * (theta_ref[kl] + theta_ref[ku]);
          const T rf = T(0.5f) * (rl + ru);
          const T b = cfg.gravity * (tf - trf) / std::max(trf, T(1.0e-6f));
          o.mw(i, j, kf) += rf * b;
        }
    // Rayleigh damping layer (extension): relaxation of the momenta on the faces whose
    // tendency the reference computes (open-boundary faces and Z faces 0, nz excluded)
    if (!cfg.damp_c.empty()) {
      const Field<T>& u = S[r].mu;
      const Field<T>& v = S[r].mv;
      const Field<T>& w = S[r].mw;
      for (int k = 0; k < nz; ++k) {
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i <= nx; ++i) {
            if ((i == 0 && ow) || (i == nx && oe)) continue;
            o.mu(i, j, k) += -cfg.damp_c[k] * (u(i, j, k) - cfg.u_ref[k]);
          }
        for (int j = 0; j <= ny; ++j)
          for (int i = 0; i < nx; ++i) {
            if ((j == 0 && os) || (j == ny && on)) continue;
            o.mv(i, j, k) += -cfg.damp_c[k] * (v(i, j, k) - cfg.v_ref[k]);
          }
      }
      for (int kf = 1; kf < nz; ++kf)
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i < nx; ++i) o.mw(i, j, kf) += -cfg.damp_f[kf] * w(i, j, kf);
    }
  }
}

// ---------------------------------------------------------------------------
// Split-explicit fast modes: src/dycore/dry_fast_modes.cu:400-656
template <class T>
void fast_modes(States<T>& S, const std::vector<Desc>& L, const Metrics<T>& M,
                const StepCfg<T>& cfg) {
  const size_t n = S.size();
  require(n == L.size(), "State/layout size mismatch in fast modes");
  if (n == 0) return;
  const int ns = std::max(1, cfg.fast_substeps);
  const T dtf = cfg.dt / (T)ns;
  std::vector<Field<T>> TH(n), RH(n), RTF(n), P(n), RREF(n), PREF(n), UB(n), VB(n), WB(n);
  for (size_t r = 0; r < n; ++r) {
    TH[r] = S[r].rt;  // K9 over whole padded array: :86-95, :453-461
    for (size_t q = 0; q < TH[r].d.size(); ++q)
      TH[r].d[q] = theta_from_conserved(S[r].rho.d[q], S[r].rt.d[q]);
    UB[r] = S[r].mu; VB[r] = S[r].mv; WB[r] = S[r].mw;
    RREF[r] = Field<T>(S[r].rho.nx, S[r].rho.ny, S[r].rho.nz, S[r].rho.h);
    PREF[r] = RREF[r];
  }
  exchange_scalar(TH, L);  // :462-469
  {
    auto a = ptrs(UB), b = ptrs(VB), c = ptrs(WB);
    exchange_momenta(a, b, c, L);
  }
  int hcount = 0;
  for (const auto& d : L) hcount += d.nxl() * d.nyl();
  const T inv_hcount = T(1) / (T)std::max(1, hcount);  // :477-482
  bool terrain_active = false;  // :484-492
  for (int j = 0; j < M.ny && !terrain_active; ++j)
    for (int i = 0; i < M.nx; ++i)
      if (std::abs((double)M.terrain[(size_t)j * M.nx + i]) > 1.0e-6) { terrain_active = true; break; }

  std::vector<T> rref_lev(M.nz), pref_lev(M.nz);
  const T dx = (T)M.dx, dy = (T)M.dy, g = cfg.gravity;
  for (int sub = 0; sub < ns; ++sub) {
    for (size_t r = 0; r < n; ++r) RH[r] = S[r].rho;  // :496-499
    exchange_scalar(RH, L);
    for (size_t r = 0; r < n; ++r) {  // K10 + K20: :500-509
      RTF[r] = RH[r];
      P[r] = RH[r];
      for (size_t q = 0; q < RH[r].d.size(); ++q) {
        RTF[r].d[q] = RH[r].d[q] * TH[r].d[q];
        P[r].d[q] = pressure_from_rho_theta(RH[r].d[q], RTF[r].d[q]);
      }
    }
    if (!terrain_active) {  // K6 + K7: :511-533 (sequential sum instead of atomics)
      std::fill(rref_lev.begin(), rref_lev.end(), T(0));
      std::fill(pref_lev.begin(), pref_lev.end(), T(0));
      for (size_t r = 0; r < n; ++r)
        for (int k = 0; k < L[r].nz; ++k)
          for (int j = 0; j < L[r].nyl(); ++j)
            for (int i = 0; i < L[r].nxl(); ++i) {
              rref_lev[k] += RH[r](i, j, k);
              pref_lev[k] += P[r](i, j, k);
            }
      for (int k = 0; k < M.nz; ++k) { rref_lev[k] *= inv_hcount; pref_lev[k] *= inv_hcount; }
    }
    for (size_t r = 0; r < n; ++r) {
      const Desc& d = L[r];
      const int nx = d.nxl(), ny = d.nyl(), nz = d.nz;
      const Nbr nb = neighbors(L, d);
      Field<T>&rh = RH[r], &rtf = RTF[r], &p = P[r], &rref = RREF[r], &pref = PREF[r];
      if (terrain_active) {  // K11 build_column_hydrostatic_reference_kernel: :108-158
#pragma omp parallel for schedule(static)
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i < nx; ++i) {
            auto mi = [&](int kk) {
              return M.m(wrap_metric(d.i0 + i, M.nx, M.px), wrap_metric(d.j0 + j, M.ny, M.py), kk);
            };
            const T th0 = theta_from_conserved(rh(i, j, 0), rtf(i, j, 0));
            pref(i, j, 0) = p(i, j, 0);
            rref(i, j, 0) = rho_from_pressure_theta(pref(i, j, 0), th0);
            for (int k = 1; k < nz; ++k) {
              const T thk = theta_from_conserved(rh(i, j, k), rtf(i, j, k));
              const T dz = M.zc[mi(k)] - M.zc[mi(k - 1)];
              T pn = std::max(T(1.0f), pref(i, j, k - 1) - g * rref(i, j, k - 1) * dz);
              for (int it = 0; it < 4; ++it) {
                const T rn = rho_from_pressure_theta(pn, thk);
                pn = pref(i, j, k - 1) - g * T(0.5f) * (rref(i, j, k - 1) + rn) * dz;
                pn = std::max(pn, T(1.0f));
              }
              pref(i, j, k) = pn;
              rref(i, j, k) = rho_from_pressure_theta(pn, thk);
            }
          }
      } else {  // K8: :69-84
        for (int k = 0; k < nz; ++k)
          for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) { rref(i, j, k) = rref_lev[k]; pref(i, j, k) = pref_lev[k]; }
      }
      auto vgrad = [&](int gi, int gj, int k, int li, int lj) -> T {  // :194-219
        if (nz == 1) return T(0);
        if (k == 0) {
          const T dz = M.zc[M.m(gi, gj, 1)] - M.zc[M.m(gi, gj, 0)];
          return (p(li, lj, 1) - p(li, lj, 0)) / std::max(dz, T(1.0e-6f));
        }
        if (k + 1 == nz) {
          const T dz = M.zc[M.m(gi, gj, k)] - M.zc[M.m(gi, gj, k - 1)];
          return (p(li, lj, k) - p(li, lj, k - 1)) / std::max(dz, T(1.0e-6f));
        }
        const T dz = M.zc[M.m(gi, gj, k + 1)] - M.zc[M.m(gi, gj, k - 1)];
        return (p(li, lj, k + 1) - p(li, lj, k - 1)) / std::max(dz, T(1.0e-6f));
      };
      if (cfg.fast_hmom) {
        // K12: :160-229
#pragma omp parallel for schedule(static)
        for (int k = 0; k < nz; ++k)
          for (int j = 0; j < ny; ++j)
            for (int i = 0; i <= nx; ++i) {
              if ((i == 0 && nb.w < 0) || (i == nx && nb.e < 0)) continue;
              const T pl = p(i - 1, j, k), pr = p(i, j, k);
              const int gj = wrap_metric(d.j0 + j, M.ny, M.py);
              const int gl = wrap_metric(d.i0 + i - 1, M.nx, M.px);
              const int gr = wrap_metric(d.i0 + i, M.nx, M.px);
              const T dzdx = (M.zc[M.m(gr, gj, k)] - M.zc[M.m(gl, gj, k)]) / dx;
              const T dpdz = T(0.5f) * (vgrad(gl, gj, k, i - 1, j) + vgrad(gr, gj, k, i, j));
              S[r].mu(i, j, k) += -dtf * ((pr - pl) / dx - dzdx * dpdz);
            }
        // K13: :231-301
#pragma omp parallel for schedule(static)
        for (int k = 0; k < nz; ++k)
          for (int j = 0; j <= ny; ++j)
            for (int i = 0; i < nx; ++i) {
              if ((j == 0 && nb.s < 0) || (j == ny && nb.n < 0)) continue;
              const T ps = p(i, j - 1, k), pn = p(i, j, k);
              const int gi = wrap_metric(d.i0 + i, M.nx, M.px);
              const int gs_ = wrap_metric(d.j0 + j - 1, M.ny, M.py);
              const int gn_ = wrap_metric(d.j0 + j, M.ny, M.py);
              const T dzdy = (M.zc[M.m(gi, gn_, k)] - M.zc[M.m(gi, gs_, k)]) / dy;
              const T dpdz = T(0.5f) * (vgrad(gi, gs_, k, i, j - 1) + vgrad(gi, gn_, k, i, j));
              S[r].mv(i, j, k) += -dtf * ((pn - ps) / dy - dzdy * dpdz);
            }
      }
      // K14: :303-348
#pragma omp parallel for schedule(static)
      for (int kf = 1; kf < nz; ++kf)
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i < nx; ++i) {
            const int kl = kf - 1, ku = kf;
            const T ppl = p(i, j, kl) - pref(i, j, kl);
            const T ppu = p(i, j, ku) - pref(i, j, ku);
            const T rpf = T(0.5f) * ((rh(i, j, kl) - rref(i, j, kl)) + (rh(i, j, ku) - rref(i, j, ku)));
            const T idz = M.inv_dz_face[M.m(wrap_metric(d.i0 + i, M.nx, M.px),
                                            wrap_metric(d.j0 + j, M.ny, M.py), kf)];
            const T tend = -(ppu - ppl) * idz - g * rpf;
            S[r].mw(i, j, kf) += dtf * tend;
          }
    }
    {  // :614-620
      std::vector<Field<T>*> a, b, c;
      for (size_t r = 0; r < n; ++r) { a.push_back(&S[r].mu); b.push_back(&S[r].mv); c.push_back(&S[r].mw); }
      exchange_momenta(a, b, c, L);
    }
    for (size_t r = 0; r < n; ++r) {
      const Desc& d = L[r];
      const int nx = d.nxl(), ny = d.nyl(), nz = d.nz;
      if (cfg.fast_density) {  // K15: :350-394
        DryState<T>& s = S[r];
#pragma omp parallel for schedule(static)
        for (int k = 0; k < nz; ++k)
          for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
              const T div =
                  ((s.mu(i + 1, j, k) - UB[r](i + 1, j, k)) - (s.mu(i, j, k) - UB[r](i, j, k))) / dx +
                  ((s.mv(i, j + 1, k) - VB[r](i, j + 1, k)) - (s.mv(i, j, k) - VB[r](i, j, k))) / dy +
                  ((s.mw(i, j, k + 1) - WB[r](i, j, k + 1)) - (s.mw(i, j, k) - WB[r](i, j, k))) *
                      M.inv_dz_cell[M.m(wrap_metric(d.i0 + i, M.nx, M.px),
                                        wrap_metric(d.j0 + j, M.ny, M.py), k)];
              s.rho(i, j, k) = std::max(T(1.0e-6f), s.rho(i, j, k) - dtf * div);
            }
      }
    }
    for (size_t r = 0; r < n; ++r)  // K10 on the state: :643-651
      for (size_t q = 0; q < S[r].rho.d.size(); ++q) S[r].rt.d[q] = S[r].rho.d[q] * TH[r].d[q];
  }
}

// K4 update_cell_field_kernel over the whole padded array: dry_core.cu:189-197
template <class T> void update_field(Field<T>& out, const Field<T>& base, const Field<T>& tend,
                                     T dt, T floor) {
  for (size_t q = 0; q < out.d.size(); ++q) out.d[q] = std::max(floor, base.d[q] + dt * tend.d[q]);
}
// K5 blend_cell_field_kernel: dry_core.cu:199-205
template <class T> void blend_field(Field<T>& out, const Field<T>& a, const Field<T>& b, T wa, T wb) {
  for (size_t q = 0; q < out.d.size(); ++q) out.d[q] = wa * a.d[q] + wb * b.d[q];
}

template <class T> void update_state(DryState<T>& out, const DryState<T>& base,
                                     const DryState<T>& tend, T dt) {
  update_field(out.rho, base.rho, tend.rho, dt, T(1.0e-6f));
  update_field(out.rt, base.rt, tend.rt, dt, T(1.0e-6f));
  update_field(out.mu, base.mu, tend.mu, dt, T(-1.0e30f));
  update_field(out.mv, base.mv, tend.mv, dt, T(-1.0e30f));
  update_field(out.mw, base.mw, tend.mw, dt, T(-1.0e30f));
}
template <class T> void blend_state(DryState<T>& out, const DryState<T>& a, const DryState<T>& b,
                                    T wa, T wb) {
  blend_field(out.rho, a.rho, b.rho, wa, wb);
  blend_field(out.rt, a.rt, b.rt, wa, wb);
  blend_field(out.mu, a.mu, b.mu, wa, wb);
  blend_field(out.mv, a.mv, b.mv, wa, wb);
  blend_field(out.mw, a.mw, b.mw, wa, wb);
}

// ---------------------------------------------------------------------------
// Reference boundaries: src/dycore/boundary_conditions.cpp:8-99 (strip copies),
// :95-109 (touches_*), :111-161 (dry state), :163-208 (tracers).  On an open side the
// outermost owned strip of every field (cells and faces, over the field's own storage
// extents) is copied from the boundary state.
inline bool touches_west(const Desc& d) { return !d.px && d.cx == 0; }
inline bool touches_east(const Desc& d) { return !d.px && d.cx == d.rx - 1; }
inline bool touches_south(const Desc& d) { return !d.py && d.cy == 0; }
inline bool touches_north(const Desc& d) { return !d.py && d.cy == d.ry - 1; }

template <class T> void copy_strips(Field<T>& dst, const Field<T>& src, const Desc& d) {
  if (touches_west(d))
    for (int k = 0; k < dst.nz; ++k)
      for (int j = 0; j < dst.ny; ++j) dst(0, j, k) = src(0, j, k);
  if (touches_east(d))
    for (int k = 0; k < dst.nz; ++k)
      for (int j = 0; j < dst.ny; ++j) dst(dst.nx - 1, j, k) = src(dst.nx - 1, j, k);
  if (touches_south(d))
    for (int k = 0; k < dst.nz; ++k)
      for (int i = 0; i < dst.nx; ++i) dst(i, 0, k) = src(i, 0, k);
  if (touches_north(d))
    for (int k = 0; k < dst.nz; ++k)
      for (int i = 0; i < dst.nx; ++i) dst(i, dst.ny - 1, k) = src(i, dst.ny - 1, k);
}

template <class T>
void apply_reference_boundaries(std::vector<DryState<T>>& S, const std::vector<DryState<T>>& B,
                                const std::vector<Desc>& L) {
  for (size_t r = 0; r < S.size(); ++r) {
    copy_strips(S[r].rho, B[r].rho, L[r]);
    copy_strips(S[r].rt, B[r].rt, L[r]);
    copy_strips(S[r].mu, B[r].mu, L[r]);
    copy_strips(S[r].mv, B[r].mv, L[r]);
    copy_strips(S[r].mw, B[r].mw, L[r]);
  }
}

// advance_dry_state_ssprk3: dry_core.cu:541-651.  With boundary states the updater
// applies apply_reference_boundaries at the three stage starts (:568, :591, :620), with
// Bs[0], Bs[1], Bs[2] (the boundary at sim_time 0, dt, dt/2); the blend partner q0 is the
// state before the first application.
template <class T>
void advance_dry_ssprk3(States<T>& S, const std::vector<Desc>& L, const Metrics<T>& M,
                        const StepCfg<T>& cfg, const States<T>* const* Bs = nullptr) {
  const size_t n = S.size();
  States<T> q0 = S, q1 = S, q2 = S, tmp = S, tend;
  const States<T>* B = Bs ? Bs[0] : nullptr;
  if (B) apply_reference_boundaries(S, *B, L);
  compute_slow_tendencies(S, L, M, cfg, tend);
  for (size_t r = 0; r < n; ++r) update_state(q1[r], S[r], tend[r], cfg.dt);
  if (cfg.fast_modes) fast_modes(q1, L, M, cfg);
  if (Bs) B = Bs[1];
  if (B) apply_reference_boundaries(q1, *B, L);
  compute_slow_tendencies(q1, L, M, cfg, tend);
  for (size_t r = 0; r < n; ++r) {
    update_state(tmp[r], q1[r], tend[r], cfg.dt);
    blend_state(q2[r], q0[r], tmp[r], T(0.75f), T(0.25f));
  }
  if (cfg.fast_modes) fast_modes(q2, L, M, cfg);
  if (Bs) B = Bs[2];
  if (B) apply_reference_boundaries(q2, *B, L);
  compute_slow_tendencies(q2, L, M, cfg, tend);
  for (size_t r = 0; r < n; ++r) {
    update_state(tmp[r], q2[r], tend[r], cfg.dt);
    blend_state(S[r], q0[r], tmp[r], T(1.0f / 3.0f), T(2.0f / 3.0f));
  }
  if (cfg.fast_modes) fast_modes(S, L, M, cfg);
}

// ---------------------------------------------------------------------------
// Passive tracers: src/dycore/dry_transport.cu:49-125 (K25), 189-230, 440-518
template <class T>
void tracer_stage(const Field<T>& qin, const Field<T>& rho, const Field<T>& u, const Field<T>& v,
                  const Field<T>& w, Field<T>& qout, const Desc& d, const Metrics<T>& M, T dt) {
  const int nx = d.nxl(), ny = d.nyl(), nz = d.nz;
  const T dx = (T)M.dx, dy = (T)M.dy;
  auto mr = [&](int i, int j, int k) { return qin(i, j, k) / std::max(rho(i, j, k), T(1.0e-6f)); };
#pragma omp parallel for schedule(static)
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const T qc = mr(i, j, k), qw = mr(i - 1, j, k), qe = mr(i + 1, j, k);
        const T qs = mr(i, j - 1, k), qn = mr(i, j + 1, k);
        const T qb = (k > 0) ? mr(i, j, k - 1) : qc;
        const T qt = (k + 1 < nz) ? mr(i, j, k + 1) : qc;
        const T fw = u(i, j, k), fe = u(i + 1, j, k), fs = v(i, j, k), fn = v(i, j + 1, k);
        const T fb = w(i, j, k), ft = w(i, j, k + 1);
        const T idz = M.inv_dz_cell[M.m(d.i0 + i, d.j0 + j, k)];
        const T gw = fw * (fw >= T(0) ? qw : qc);
        const T ge = fe * (fe >= T(0) ? qc : qe);
        const T gs = fs * (fs >= T(0) ? qs : qc);
        const T gn = fn * (fn >= T(0) ? qc : qn);
        const T gb = fb * (fb >= T(0) ? qb : qc);
        const T gt = ft * (ft >= T(0) ? qc : qt);
        const T div = (ge - gw) / dx + (gn - gs) / dy + (gt - gb) * idz;
        qout(i, j, k) = std::max(T(0), qin(i, j, k) - dt * div);
      }
}

// tracers[r][t] is tracer t of rank r (registry order).  With boundary tracers QBs the
// tracer updater applies apply_reference_boundaries to each stage input
// (dry_transport.cu:254-276, 484-517): a copy of the state (QBs[0], sim_time 0), then q1
// (QBs[1], dt), then q2 (QBs[2], dt/2).
template <class T>
void advance_tracers_ssprk3(std::vector<std::vector<Field<T>>>& Q, const States<T>& S,
                            const std::vector<Desc>& L, const Metrics<T>& M, const StepCfg<T>& cfg,
                            const std::vector<std::vector<Field<T>>>* const* QBs = nullptr) {
  const size_t n = S.size();
  if (n == 0 || Q.empty() || Q[0].empty()) return;
  std::vector<Field<T>> R(n), U(n), V(n), W(n);
  for (size_t r = 0; r < n; ++r) { R[r] = S[r].rho; U[r] = S[r].mu; V[r] = S[r].mv; W[r] = S[r].mw; }
  exchange_scalar(R, L);  // prepare_dry_transport_halos: :189-230
  {
    auto a = ptrs(U), b = ptrs(V), c = ptrs(W);
    exchange_momenta(a, b, c, L);
  }
  const size_t nt = Q[0].size();
  for (size_t t = 0; t < nt; ++t) {
    std::vector<Field<T>> q0(n), q1(n), q2(n), tmp(n), st(n);
    for (size_t r = 0; r < n; ++r) { q0[r] = Q[r][t]; st[r] = Q[r][t]; q1[r] = q2[r] = tmp[r] = Q[r][t]; }
    auto bnd = [&](std::vector<Field<T>>& F, int stage) {
      if (QBs && QBs[stage])
        for (size_t r = 0; r < n; ++r) copy_strips(F[r], (*QBs[stage])[r][t], L[r]);
    };
    bnd(st, 0);
    exchange_scalar(st, L);
    for (size_t r = 0; r < n; ++r) tracer_stage(st[r], R[r], U[r], V[r], W[r], q1[r], L[r], M, cfg.dt);
    bnd(q1, 1);
    exchange_scalar(q1, L);
    for (size_t r = 0; r < n; ++r) {
      tracer_stage(q1[r], R[r], U[r], V[r], W[r], tmp[r], L[r], M, cfg.dt);
      blend_field(q2[r], q0[r], tmp[r], T(0.75f), T(0.25f));
    }
    bnd(q2, 2);
    exchange_scalar(q2, L);
    for (size_t r = 0; r < n; ++r) {
      tracer_stage(q2[r], R[r], U[r], V[r], W[r], tmp[r], L[r], M, cfg.dt);
      blend_field(Q[r][t], q0[r], tmp[r], T(1.0f / 3.0f), T(2.0f / 3.0f));
    }
  }
}

// ---------------------------------------------------------------------------
// Warm rain: include/gwm/physics/warm_rain.hpp:14-23, src/physics/warm_rain.cu
template <class T> struct RainCfg {
  T dt = T(2.0f);
  T condensation_relaxation = T(1.0f);
  T autoconv_threshold = T(1.0e-4f);
  T autoconv_rate = T(1.0e-3f);
  T rain_evap_rate = T(5.0e-3f);
  T terminal_velocity = T(0.0f);
  T layer_depth = T(0.0f);
  bool latent_heating = true;
};

// warm_rain_kernel (K26): warm_rain.cu:36-120, one cell
template <class T>
void warm_rain_cell(T rho_in, T& rt, T& rqv, T& rqc, T& rqr, const RainCfg<T>& c) {
  const T rho = std::max(rho_in, T(1.0e-6f));
  T th = rt / rho;
  T p = pressure_from_rho_theta(rho, rt);
  T temp = temperature_from_conserved(rho, rt);
  const T exner = std::max(temp / std::max(th, T(1.0e-6f)), T(1.0e-6f));
  T qv = std::max(rqv / rho, T(0)), qc = std::max(rqc / rho, T(0)), qr = std::max(rqr / rho, T(0));
  const T lh = K<T>::Lv / (dry_cp<T>() * std::max(exner, T(1.0e-6f)));
  T qs = qsat(temp, p);
  if (qv > qs) {
    const T cond = std::min((qv - qs) * std::max(c.condensation_relaxation, T(0)), qv);
    qv -= cond; qc += cond;
    if (c.latent_heating && cond > T(0)) th += lh * cond;
  } else if (qv < qs && qc > T(0)) {
    const T ev = std::min((qs - qv) * std::max(c.condensation_relaxation, T(0)), qc);
    qv += ev; qc -= ev;
    if (c.latent_heating && ev > T(0)) th -= lh * ev;
  }
  const T excess = std::max(qc - c.autoconv_threshold, T(0));
  if (excess > T(0) && c.autoconv_rate > T(0)) {
    const T conv = std::min(excess, c.dt * c.autoconv_rate * excess);
    qc -= conv; qr += conv;
  }
  p = pressure_from_rho_theta(rho, rho * th);
  temp = th * std::pow(std::max(p / K<T>::p0, T(1.0e-6f)), K<T>::kappa);
  qs = qsat(temp, p);
  if (qr > T(0) && qv < qs && c.rain_evap_rate > T(0)) {
    const T ev = std::min(qr, c.dt * c.rain_evap_rate * std::min(qs - qv, qr));
    qr -= ev; qv += ev;
    if (c.latent_heating && ev > T(0)) th -= lh * ev;
  }
  qv = std::max(qv, T(0)); qc = std::max(qc, T(0)); qr = std::max(qr, T(0));
  rqv = rho * qv; rqc = rho * qc; rqr = rho * qr; rt = rho * th;
}

// Both overloads of apply_warm_rain_microphysics (warm_rain.cu:214-271 nominal,
// :273-353 metric).  metric==nullptr selects the nominal overload (K27), else K28.
// precip[r] is the rank's (nxl*nyl) accumulation, may be null (no fallout).
template <class T>
void apply_warm_rain(States<T>& S, std::vector<std::vector<Field<T>>>& Q,
                     const std::vector<Desc>& L, const Metrics<T>* M, const RainCfg<T>& c,
                     std::vector<std::vector<T>>* precip) {
  const size_t n = S.size();
  for (size_t r = 0; r < n; ++r) {
    DryState<T>& s = S[r];
    Field<T>&qv = Q[r][0], &qc = Q[r][1], &qr = Q[r][2];
    const int nx = s.rho.nx, ny = s.rho.ny, nz = s.rho.nz;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i)
          warm_rain_cell(s.rho(i, j, k), s.rt(i, j, k), qv(i, j, k), qc(i, j, k), qr(i, j, k), c);
    if (precip == nullptr) continue;
    std::vector<T>& acc = (*precip)[r];
    if (M == nullptr) {
      if (!(c.terminal_velocity > T(0) && c.layer_depth > T(0))) continue;
      // K27 rain_fallout_nominal_kernel: warm_rain.cu:122-154
      const T dz = std::max(c.layer_depth, T(1.0e-3f));
      const T frac = std::min(std::max(c.terminal_velocity * c.dt / dz, T(0)), T(1));
      if (frac <= T(0)) continue;
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          T incoming = T(0);
          for (int k = nz - 1; k >= 0; --k) {
            const T old_v = std::max(qr(i, j, k), T(0));
            const T old_a = old_v * dz;
            const T out = frac * old_a;
            const T kept = old_a - out;
            qr(i, j, k) = (kept + incoming) / dz;
            incoming = out;
          }
          acc[(size_t)j * nx + i] += incoming;
        }
    } else {
      if (!(c.terminal_velocity > T(0))) continue;
      // K28 rain_fallout_metric_kernel: warm_rain.cu:156-191 (reads a copy of qr)
      const Field<T> qr_old = qr;
      const Desc& d = L[r];
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
          T incoming = T(0);
          for (int k = nz - 1; k >= 0; --k) {
            const T idz = std::max(M->inv_dz_cell[M->m(d.i0 + i, d.j0 + j, k)], T(1.0e-6f));
            const T dz = T(1) / idz;
            const T frac = std::min(std::max(c.terminal_velocity * c.dt * idz, T(0)), T(1));
            const T old_v = std::max(qr_old(i, j, k), T(0));
            const T old_a = old_v * dz;
            const T out = frac * old_a;
            const T kept = old_a - out;
            qr(i, j, k) = (kept + incoming) * idz;
            incoming = out;
          }
          acc[(size_t)j * nx + i] += incoming;
        }
    }
  }
}

// ---------------------------------------------------------------------------
// Idealized initial states: src/dycore/idealized_cases.cpp, src/dycore/dry_core.cu:22-35,363-398

// hydrostatic_rho_at_height: idealized_cases.cpp:22-34 (dup. dry_core.cu:22-35)
template <class T> T hydrostatic_rho_at_height(T rho_s, T theta, T z, T g = T(9.81f)) {
  const T ps = pressure_from_rho_theta(rho_s, rho_s * theta);
  const T exs = std::pow(std::max(ps / K<T>::p0, T(1.0e-6f)), K<T>::kappa);
  const T ex = std::max(T(1.0e-4f), exs - g * z / (dry_cp<T>() * theta));
  const T p = K<T>::p0 * std::pow(ex, T(1) / K<T>::kappa);
  return rho_from_pressure_theta(p, theta);
}

// rho*theta that reproduces pressure p through the dry EOS: prepared_case_init.cpp:39-53
// (an isentropic first guess refined by two ratio corrections).
template <class T> T rho_theta_for_pressure(T p) {
  T rt = (K<T>::p0 / K<T>::Rd) * std::pow(std::max(p / K<T>::p0, T(1.0e-6f)), T(1) - K<T>::kappa);
  for (int it = 0; it < 2; ++it) {
    const T pe = pressure_from_rho_theta(T(1), rt);
    rt *= std::pow(std::max(p / std::max(pe, T(1)), T(1.0e-6f)), T(1) - K<T>::kappa);
  }
  return rt;
}

// ---------------------------------------------------------------------------
// Synthetic moist sounding of the moist warm-rain benchmark, built independently of the
// library (input generator of the CPU baseline and of the parity tests).  Arithmetic in
// float, as the reference's initialisers.  Per column:
//   theta(z) = theta_ref for z <= 1 km, theta_ref + lapse (z - 1 km) above, plus a
//     Gaussian deviate of rms noise_rms below noise_depth: Box-Muller of two uniforms
//     from a splitmix64 counter hash of (seed, 2q) and (seed, 2q + 1), q = (k ny + j) nx + i;
//   the first level from p_surface over an isentropic layer (Exner drop g z / (cp theta));
//   the levels above balanced as prepared_case_init.cpp:357-377 (trapezoidal hydrostatic
//     step, four density refinements, pressure floored at 1 Pa);
//   rho*theta from the balanced pressure (prepared_case_init.cpp:39-53);
//   qv = RH qsat(T, p) below rh_top (and at k = 0), above it exponential decay with
//     scale height qv_scale from the last level below rh_top, floored at qv_floor.
struct Sounding {
  float p_surface = 100000.0f, theta_ref = 300.0f, lapse = 0.004f, rh = 0.9f, rh_top = 2000.0f;
  float qv_scale = 1500.0f, qv_floor = 1.0e-5f, noise_rms = 0.5f, noise_depth = 1000.0f;
  uint64_t seed = 1;
};

inline uint64_t mix64(uint64_t x) {  // splitmix64 finaliser
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Outputs (global owned arrays, float): rho, rt, qv as rho*qv; flat terrain only.
// Compiled without floating-point contraction, so the values do not depend on the
// target's FMA support.
#pragma GCC push_options
#pragma GCC optimize("fp-contract=off")
inline void moist_sounding(int nx, int ny, int nz, double z_top, const double* eta_interfaces, const Sounding& s,
                           std::vector<float>& rho, std::vector<float>& rt, std::vector<float>& qv) {
  using F = float;
  const size_t n = (size_t)nx * ny * nz;
  rho.assign(n, 0.0f); rt.assign(n, 0.0f); qv.assign(n, 0.0f);
  std::vector<F> zc(nz);
  for (int k = 0; k < nz; ++k) {
    const double ec = eta_interfaces ? 0.5 * (eta_interfaces[k] + eta_interfaces[k + 1]) : ((double)k + 0.5) / nz;
    zc[k] = (F)(ec * z_top);
  }
  const F g = 9.81f, cp = dry_cp<F>();
  const uint64_t key = s.seed * 0x100000001B3ull;
#pragma omp parallel for schedule(static)
  for (int col = 0; col < nx * ny; ++col) {
    std::vector<F> th(nz), p(nz), r(nz);
    for (int k = 0; k < nz; ++k) {
      const size_t q = (size_t)k * nx * ny + col;
      F t = zc[k] <= 1000.0f ? s.theta_ref : s.theta_ref + s.lapse * (zc[k] - 1000.0f);
      if (zc[k] < s.noise_depth && s.noise_rms > 0.0f) {
        const double u1 = ((double)(mix64(key ^ (2 * q)) >> 11) + 0.5) / 9007199254740992.0;
        const double u2 = ((double)(mix64(key ^ (2 * q + 1)) >> 11) + 0.5) / 9007199254740992.0;
        t += (F)(s.noise_rms * (std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * 3.14159265358979323846 * u2)));
      }
      th[k] = t;
    }
    const F ex0 = std::max(1.0e-4f, std::pow(s.p_surface / K<F>::p0, K<F>::kappa) - g * zc[0] / (cp * th[0]));
    p[0] = K<F>::p0 * std::pow(ex0, 1.0f / K<F>::kappa);
    r[0] = rho_from_pressure_theta(p[0], th[0]);
    for (int k = 1; k < nz; ++k) {
      const F dz = zc[k] - zc[k - 1];
      F pk = std::max(1.0f, p[k - 1] - g * r[k - 1] * dz);
      for (int it = 0; it < 4; ++it)
        pk = std::max(p[k - 1] - g * 0.5f * (r[k - 1] + rho_from_pressure_theta(pk, th[k])) * dz, 1.0f);
      p[k] = pk;
      r[k] = rho_from_pressure_theta(pk, th[k]);
    }
    F q_anchor = -1.0f, z_anchor = 0.0f;
    for (int k = 0; k < nz; ++k) {
      const size_t q = (size_t)k * nx * ny + col;
      F v;
      if (zc[k] < s.rh_top || k == 0) {
        const F tk = th[k] * std::pow(std::max(p[k] / K<F>::p0, 1.0e-6f), K<F>::kappa);
        v = s.rh * qsat(tk, p[k]);
        if (zc[k] < s.rh_top || q_anchor < 0.0f) { q_anchor = v; z_anchor = zc[k]; }
      } else {
        v = std::max(s.qv_floor, q_anchor * std::exp(-(zc[k] - z_anchor) / s.qv_scale));
      }
      rho[q] = r[k];
      rt[q] = rho_theta_for_pressure(p[k]);
      qv[q] = r[k] * std::max(v, 0.0f);
    }
  }
}
#pragma GCC pop_options

// ---------------------------------------------------------------------------
// Runtime plan view: extract_runtime_plan_view (src/io/plan_view_output.cpp:715-834)
// over extract_dry_plan_view (:630-713) on global owned arrays (float, the state's
// storage type), with the FP32 formulas of dry_thermo.hpp:21-33 and
// moist_thermo.hpp:23-74 and the FP64 column integrals of :282-416.  nfields is 10
// (dry), 13 (+ specific humidity), 21 (+ cloud and rain) or 23 (+ the surface
// precipitation and its mean rate); out holds nfields x ny x nx doubles in the
// bundle's field order.  Field 0 (terrain height) and 1 (z_center) come from the
// caller's metric arrays (terrain (ny, nx), zc and idc (nz, ny, nx), FP32).
#pragma GCC push_options
#pragma GCC optimize("fp-contract=off")
struct PlanViewIn {
  int nx, ny, nz, k, nfields, steps;
  float dt;
  const float *terrain, *zc, *idc;
  const float *rho, *rt, *u, *v, *w;   // cells, X faces (nz, ny, nx+1), Y faces (nz, ny+1, nx), Z faces
  const float *qv, *qc, *qr;           // tracer masses rho*q
  const float* precip;                 // liquid_precipitation_kg_m2 (ny, nx)
};

inline float pv_pressure(float rho, float rt) {  // dry_pressure_from_rho_theta_m
  const float theta = rt / std::max(rho, 1.0e-6f);
  const float ratio = std::max(rho * 287.05f * theta / 100000.0f, 1.0e-6f);
  return 100000.0f * std::pow(ratio, 1.0f / (1.0f - 0.2854f));
}
inline float pv_qsat(float t, float p) {  // saturation_specific_humidity
  const float eps = 287.05f / 461.5f;
  const float tc = t - 273.15f;
  const float es = 6.112f * std::exp((17.67f * tc) / std::max(tc + 243.5f, 1.0e-6f)) * 100.0f;
  const float denom = std::max(p - (1.0f - eps) * es, 1000.0f);
  return std::min(std::max(eps * es / denom, 0.0f), 0.05f);
}
inline float pv_rh(float q, float t, float p) {  // relative_humidity_from_specific_humidity
  const float qs = pv_qsat(t, p);
  return std::min(std::max((qs > 0.0f) ? (100.0f * q / qs) : 0.0f, 0.0f), 100.0f);
}
inline float pv_dewpoint(float q_in, float p) {  // dewpoint_from_specific_humidity
  const float eps = 287.05f / 461.5f;
  const float q = std::min(std::max(q_in, 0.0f), 1.0f);
  const float e = p * q / std::max(eps + (1.0f - eps) * q, 1.0e-6f);
  const float e_hpa = std::max(e * 0.01f, 1.0e-6f);
  const float l = std::log(e_hpa / 6.112f);
  return (243.5f * l) / (17.67f - l) + 273.15f;
}
inline float pv_dbz(float rho, float qr_in) {  // synthetic_reflectivity_dbz_from_rain
  const float qr = std::max(qr_in, 0.0f);
  if (qr <= 1.0e-8f || rho <= 1.0e-8f) return -20.0f;
  const float z = 3.63e9f * std::pow(rho * qr, 1.75f);
  return 10.0f * std::log10(std::max(z, 1.0e-6f));
}

inline void plan_view(const PlanViewIn& a, double* out) {
  const int nx = a.nx, ny = a.ny, nz = a.nz, k = a.k;
  const size_t plane = (size_t)nx * ny;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const size_t o = (size_t)j * nx + i, c = (size_t)k * plane + o;
      auto put = [&](int f, double v) { out[(size_t)f * plane + o] = v; };
      const float rho = a.rho[c], rr = std::max(rho, 1.0e-6f);
      const float theta = a.rt[c] / rr;
      const float p = pv_pressure(rho, a.rt[c]);
      const float t = theta * std::pow(std::max(p, 1.0f) / 100000.0f, 0.2854f);
      const size_t cu = ((size_t)k * ny + j) * (nx + 1) + i, cv = ((size_t)k * (ny + 1) + j) * nx + i;
      const float uc = 0.5f * (a.u[cu] + a.u[cu + 1]) / rr;
      const float vc = 0.5f * (a.v[cv] + a.v[cv + nx]) / rr;
      const float wc = 0.5f * (a.w[c] + a.w[c + plane]) / rr;
      const double vals[10] = {a.terrain ? (double)a.terrain[o] : 0.0, (double)a.zc[c], rho, theta, p, t, uc, vc,
                               std::sqrt(uc * uc + vc * vc), wc};
      for (int f = 0; f < 10; ++f) put(f, vals[f]);
      if (a.nfields <= 10) continue;
      const float q = a.qv[c] / rr;
      put(10, q);
      put(11, pv_rh(q, t, p));
      put(12, pv_dewpoint(q, p));
      if (a.nfields <= 13) continue;
      const float qcm = a.qc[c] / rr, qrm = a.qr[c] / rr;
      put(13, qcm);
      put(14, qrm);
      put(15, qcm + qrm);
      double col_c = 0.0, col_r = 0.0;
      float dbz = -20.0f;
      for (int kk = 0; kk < nz; ++kk) {
        const size_t ck = (size_t)kk * plane + o;
        const double dz = (double)(1.0f / a.idc[ck]);
        col_c += (double)a.qc[ck] * dz;
        col_r += (double)a.qr[ck] * dz;
        dbz = std::max(dbz, pv_dbz(a.rho[ck], a.qr[ck] / std::max(a.rho[ck], 1.0e-6f)));
      }
      const double total = col_c + col_r, tpos = std::max(total, 0.0);
      put(16, col_c);
      put(17, col_r);
      put(18, total);
      put(19, tpos <= 0.0 ? 0.0 : std::clamp(col_r / tpos, 0.0, 1.0));
      put(20, dbz);
      if (a.nfields <= 21) continue;
      const double hours = std::max((double)a.steps * (double)a.dt / 3600.0, 1.0e-9);
      put(21, (double)a.precip[o]);
      put(22, (double)a.precip[o] / hours);
    }
}
#pragma GCC pop_options

// ---------------------------------------------------------------------------
// Scalar advection: advance_scalar_ssprk3 (src/dycore/dry_transport.cu:285-325) with
// upwind_stage_kernel (:13-37) and blend_stage_kernel (:39-46) on the global owned array
// (nz, ny, nx).  Halo values are the periodic image, or zero beyond an open side (the
// halo exchange's absent neighbour, src/comm/halo_exchange.cpp:563-620), which is what
// the virtual-rank exchange gives the stencil.
template <class T>
void scalar_upwind_stage(const std::vector<T>& in, std::vector<T>& out, int nx, int ny, int nz, bool px, bool py,
                         T u, T v, T dt, T dx, T dy) {
  auto at = [&](int i, int j, int k) -> T {
    if (i < 0 || i >= nx) {
      if (!px) return T(0);
      i = (i + nx) % nx;
    }
    if (j < 0 || j >= ny) {
      if (!py) return T(0);
      j = (j + ny) % ny;
    }
    return in[((size_t)k * ny + j) * nx + i];
  };
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const T q = at(i, j, k);
        const T dqx = (u >= T(0)) ? (q - at(i - 1, j, k)) / dx : (at(i + 1, j, k) - q) / dx;
        const T dqy = (v >= T(0)) ? (q - at(i, j - 1, k)) / dy : (at(i, j + 1, k) - q) / dy;
        // q - dt*(u*dqx + v*dqy) with the reference build's contractions
        out[((size_t)k * ny + j) * nx + i] = std::fma(-dt, std::fma(u, dqx, v * dqy), q);
      }
}

template <class T>
void scalar_ssprk3(std::vector<T>& q, int nx, int ny, int nz, bool px, bool py, T u, T v, T dt, T dx, T dy) {
  const std::vector<T> q0 = q;
  std::vector<T> q1(q.size()), q2(q.size()), tmp(q.size());
  scalar_upwind_stage(q, q1, nx, ny, nz, px, py, u, v, dt, dx, dy);
  scalar_upwind_stage(q1, tmp, nx, ny, nz, px, py, u, v, dt, dx, dy);
  // wa*a + wb*b as fma(wa, a, wb*b), the reference build's contraction
  for (size_t n = 0; n < q.size(); ++n) q2[n] = std::fma(T(0.75f), q0[n], T(0.25f) * tmp[n]);
  scalar_upwind_stage(q2, tmp, nx, ny, nz, px, py, u, v, dt, dx, dy);
  for (size_t n = 0; n < q.size(); ++n) q[n] = std::fma(T(1.0f / 3.0f), q0[n], T(2.0f / 3.0f) * tmp[n]);
}

}  // namespace gwo
