// gwm_b200_idealized_driver — the command-line contract of the reference's
// gwm_idealized_driver (src/core/gwm_idealized_driver.cpp:69-276) on top of the C-ABI
// of libgwm_b200.so: the same flags with the same defaults, the same four idealized
// cases, `steps` calls of advance_dry_state_ssprk3 with NullBoundaryUpdater and
// LocalSplitExplicitFastMode, and the same summary JSON (case, steps, dt, initial and
// final DryStateSummary; src/dycore/dry_diagnostics.cpp:11-125) on stdout and, with
// --summary-json, in a file.  The step runs on the GPU; the summaries are taken on the
// host from the state in the reference's own virtual-rank order, so multi-rank layouts
// count shared faces once per rank exactly as summarize_dry_states does.
//
// --plan-view-json writes the dry plan-view bundle of the final state
// (extract_dry_plan_view + plan_view_bundle_to_json, src/io/plan_view_output.cpp:630-713,
// 950-1003): terrain height, z_center and the diagnosed cell-centre fields at
// --plan-view-level, computed on the host with the reference's formulas.
//
// One difference is reported as an error rather than run differently: --halo other than
// 1 (every stencil of the step reaches one cell; the device layout has a one-cell halo).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <iomanip>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <limits>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "gwm_b200.h"
#include "gwm_b200_cases.h"

namespace {

struct Domain {  // RectilinearDomainConfig (include/gwm/domain/idealized_domain_builder.hpp:12-31)
  int nx = 0, ny = 0, nz = 0, halo = 1, ranks_x = 1, ranks_y = 1;
  double dx = 1000.0, dy = 1000.0, z_top = 16000.0, terrain_taper_eta = 0.25;
  std::string terrain_kind = "flat";
  double center_x = 0.5, center_y = 0.5, half_width_x = 0.15, half_width_y = 0.15, height = 0.0;
  bool periodic_x = true, periodic_y = true;
};

struct Bubble {  // ThermoBubbleConfig (include/gwm/dycore/idealized_cases.hpp:11-24)
  float rho_background = 1.0f, theta_background = 300.0f;
  float u_background = 0.0f, v_background = 0.0f, w_background = 0.0f;
  float center_x = 0.5f, center_y = 0.5f, center_z = 0.5f;
  float radius_x = 0.1f, radius_y = 0.1f, radius_z = 0.1f, theta_perturbation = 2.0f;
};

struct Mountain {  // MountainWaveBackgroundConfig (idealized_cases.hpp:26-35)
  float rho_surface = 1.18f, theta_ref = 300.0f, density_scale_height = 8200.0f;
  float u_background = 15.0f, v_background = 0.0f, w_background = 0.0f;
};

struct Options {
  std::string case_kind = "density_current";
  Domain domain;
  Bubble bubble;
  Mountain mountain;
  gwm_b200_step_config step{2.0f, 1, 9.81f, 1, 1, 1};  // DryStepperConfig defaults
  int steps = 10;
  std::string summary_json_path, plan_view_json_path;
  int plan_view_level = 0;
};

bool to_bool(const std::string& v) {
  if (v == "true" || v == "1") return true;
  if (v == "false" || v == "0") return false;
  throw std::runtime_error("Invalid boolean value: " + v);
}

void parse(int argc, char** argv, Options& o) {
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto next = [&]() -> std::string {
      if (i + 1 >= argc) throw std::runtime_error("Missing value for " + a);
      return argv[++i];
    };
    auto f = [&]() { return std::stof(next()); };
    auto d = [&]() { return std::stod(next()); };
    auto n = [&]() { return std::stoi(next()); };
    Domain& D = o.domain;
    if (a == "--case") o.case_kind = next();
    else if (a == "--nx") D.nx = n();
    else if (a == "--ny") D.ny = n();
    else if (a == "--nz") D.nz = n();
    else if (a == "--halo") D.halo = n();
    else if (a == "--ranks-x") D.ranks_x = n();
    else if (a == "--ranks-y") D.ranks_y = n();
    else if (a == "--dx") D.dx = d();
    else if (a == "--dy") D.dy = d();
    else if (a == "--z-top") D.z_top = d();
    else if (a == "--periodic-x") D.periodic_x = to_bool(next());
    else if (a == "--periodic-y") D.periodic_y = to_bool(next());
    else if (a == "--terrain-kind") {
      D.terrain_kind = next();
      if (D.terrain_kind != "flat" && D.terrain_kind != "cosine_mountain")
        throw std::runtime_error("Unsupported terrain kind: " + D.terrain_kind);
    } else if (a == "--terrain-center-x") D.center_x = d();
    else if (a == "--terrain-center-y") D.center_y = d();
    else if (a == "--terrain-half-width-x") D.half_width_x = d();
    else if (a == "--terrain-half-width-y") D.half_width_y = d();
    else if (a == "--terrain-height") D.height = d();
    else if (a == "--rho-background") o.bubble.rho_background = f();
    else if (a == "--theta-background") o.bubble.theta_background = f();
    else if (a == "--u-background") o.bubble.u_background = o.mountain.u_background = f();
    else if (a == "--v-background") o.bubble.v_background = o.mountain.v_background = f();
    else if (a == "--w-background") o.bubble.w_background = o.mountain.w_background = f();
    else if (a == "--theta-perturbation") o.bubble.theta_perturbation = f();
    else if (a == "--center-x-fraction") o.bubble.center_x = f();
    else if (a == "--center-y-fraction") o.bubble.center_y = f();
    else if (a == "--center-z-fraction") o.bubble.center_z = f();
    else if (a == "--radius-x-fraction") o.bubble.radius_x = f();
    else if (a == "--radius-y-fraction") o.bubble.radius_y = f();
    else if (a == "--radius-z-fraction") o.bubble.radius_z = f();
    else if (a == "--rho-surface") o.mountain.rho_surface = f();
    else if (a == "--theta-ref") o.mountain.theta_ref = f();
    else if (a == "--density-scale-height") o.mountain.density_scale_height = f();
    else if (a == "--steps") o.steps = n();
    else if (a == "--dt") o.step.dt = f();
    else if (a == "--fast-substeps") o.step.fast_substeps = n();
    else if (a == "--gravity") o.step.gravity = f();
    else if (a == "--summary-json") o.summary_json_path = next();
    else if (a == "--plan-view-json") o.plan_view_json_path = next();
    else if (a == "--plan-view-level") o.plan_view_level = n();
    else throw std::runtime_error("Unknown argument: " + a);
  }
}

// The initialiser parameters of one case kind in the library's case-builder block.
gwm_b200_case_params case_params(const Options& o) {
  gwm_b200_case_params p{};
  const std::string& k = o.case_kind;
  if (k == "warm_bubble" || k == "density_current") {
    const Bubble& b = o.bubble;
    p.rho_background = b.rho_background;
    p.theta_background = b.theta_background;
    p.u_background = b.u_background;
    p.v_background = b.v_background;
    p.w_background = b.w_background;
    p.center_x_fraction = b.center_x;
    p.center_y_fraction = b.center_y;
    p.center_z_fraction = b.center_z;
    p.radius_x_fraction = b.radius_x;
    p.radius_y_fraction = b.radius_y;
    p.radius_z_fraction = b.radius_z;
    p.theta_perturbation = b.theta_perturbation;
  } else if (k == "hydrostatic_rest" || k == "mountain_wave_background") {
    const Mountain& m = o.mountain;  // density_scale_height is ignored, as in the reference
    p.rho_surface = m.rho_surface;
    p.theta_ref = m.theta_ref;
    p.u_background = m.u_background;
    p.v_background = m.v_background;
    p.w_background = m.w_background;
  } else {
    throw std::runtime_error("Unsupported case kind: " + k);
  }
  return p;
}

struct Range {
  double min = std::numeric_limits<double>::max(), max = -std::numeric_limits<double>::max();
  void add(double v) {
    min = std::min(min, v);
    max = std::max(max, v);
  }
};

struct Summary {  // DryStateSummary (include/gwm/dycore/dry_diagnostics.hpp:15-26)
  double mass = 0.0, rho_theta = 0.0, mom_x = 0.0, mom_y = 0.0, mom_z = 0.0;
  Range rho, theta, u, v, w;
};

struct State {
  std::vector<float> rho, rt, u, v, w;
};

// summarize_dry_states over the virtual ranks of the layout (row-major, remainder to
// the low ranks: src/comm/virtual_rank_layout.cpp:7-47).  Each rank sums its own cells
// and its own faces (shared faces belong to both neighbours) in k, j, i order in FP64,
// and the rank totals are added in rank order, as owned_sum does per state.
Summary summarize(const State& s, const Domain& D) {
  Summary out;
  const int nx = D.nx, ny = D.ny, nz = D.nz;
  auto cell = [&](int i, int j, int k) { return ((size_t)k * ny + j) * nx + i; };
  auto xface = [&](int i, int j, int k) { return ((size_t)k * ny + j) * (nx + 1) + i; };
  auto yface = [&](int i, int j, int k) { return ((size_t)k * (ny + 1) + j) * nx + i; };
  int jb = 0;
  for (int ry = 0; ry < D.ranks_y; ++ry) {
    const int nyl = ny / D.ranks_y + (ry < ny % D.ranks_y ? 1 : 0);
    int ib = 0;
    for (int rx = 0; rx < D.ranks_x; ++rx) {
      const int nxl = nx / D.ranks_x + (rx < nx % D.ranks_x ? 1 : 0);
      double m = 0.0, rt = 0.0, mu = 0.0, mv = 0.0, mw = 0.0;
      for (int k = 0; k < nz; ++k)
        for (int j = jb; j < jb + nyl; ++j)
          for (int i = ib; i < ib + nxl; ++i) m += (double)s.rho[cell(i, j, k)];
      for (int k = 0; k < nz; ++k)
        for (int j = jb; j < jb + nyl; ++j)
          for (int i = ib; i < ib + nxl; ++i) rt += (double)s.rt[cell(i, j, k)];
      for (int k = 0; k < nz; ++k)
        for (int j = jb; j < jb + nyl; ++j)
          for (int i = ib; i <= ib + nxl; ++i) mu += (double)s.u[xface(i, j, k)];
      for (int k = 0; k < nz; ++k)
        for (int j = jb; j <= jb + nyl; ++j)
          for (int i = ib; i < ib + nxl; ++i) mv += (double)s.v[yface(i, j, k)];
      for (int k = 0; k <= nz; ++k)
        for (int j = jb; j < jb + nyl; ++j)
          for (int i = ib; i < ib + nxl; ++i) mw += (double)s.w[cell(i, j, k)];
      out.mass += m;
      out.rho_theta += rt;
      out.mom_x += mu;
      out.mom_y += mv;
      out.mom_z += mw;
      for (int k = 0; k < nz; ++k)
        for (int j = jb; j < jb + nyl; ++j)
          for (int i = ib; i < ib + nxl; ++i) {
            const double r = s.rho[cell(i, j, k)];
            out.rho.add(r);
            out.theta.add((double)s.rt[cell(i, j, k)] / std::max(r, 1.0e-12));
          }
      for (int k = 0; k < nz; ++k)
        for (int j = jb; j < jb + nyl; ++j)
          for (int i = ib; i <= ib + nxl; ++i) out.u.add(s.u[xface(i, j, k)]);
      for (int k = 0; k < nz; ++k)
        for (int j = jb; j <= jb + nyl; ++j)
          for (int i = ib; i < ib + nxl; ++i) out.v.add(s.v[yface(i, j, k)]);
      for (int k = 0; k <= nz; ++k)
        for (int j = jb; j < jb + nyl; ++j)
          for (int i = ib; i < ib + nxl; ++i) out.w.add(s.w[cell(i, j, k)]);
      ib += nxl;
    }
    jb += nyl;
  }
  return out;
}

std::string summary_json(const Summary& s, const std::string& ind) {
  std::ostringstream o;
  auto range = [&](const char* name, const Range& r, bool last) {
    o << ind << "\"" << name << "\": {\"min\": " << r.min << ", \"max\": " << r.max << "}" << (last ? "\n" : ",\n");
  };
  o << "{\n";
  o << ind << "\"total_dry_mass\": " << s.mass << ",\n";
  o << ind << "\"total_rho_theta_m\": " << s.rho_theta << ",\n";
  o << ind << "\"total_horizontal_momentum_x\": " << s.mom_x << ",\n";
  o << ind << "\"total_horizontal_momentum_y\": " << s.mom_y << ",\n";
  o << ind << "\"total_vertical_momentum\": " << s.mom_z << ",\n";
  range("rho_d", s.rho, false);
  range("theta_m", s.theta, false);
  range("u_face", s.u, false);
  range("v_face", s.v, false);
  range("w_face", s.w, true);
  o << "}";
  return o.str();
}

std::string json_string(const std::string& v) {
  std::string o = "\"";
  for (char ch : v) {
    if (ch == '"' || ch == '\\') o += '\\';
    o += ch;
  }
  return o + "\"";
}

// The dry plan-view bundle at level k of the final state (global owned arrays).
std::string plan_view_json(const Options& o, const State& s, const std::vector<float>& terrain,
                           const std::vector<float>& zc, int level) {
  const Domain& D = o.domain;
  const int nx = D.nx, ny = D.ny, k = std::clamp(level, 0, D.nz - 1);
  const size_t plane = (size_t)nx * ny;
  struct Field {
    const char* name;
    const char* units;
    std::vector<double> v;
  };
  std::vector<Field> f = {{"terrain_height", "m", {}}, {"z_center", "m", {}}, {"rho_d", "kg m^-3", {}},
                          {"theta_m", "K", {}}, {"air_pressure", "Pa", {}}, {"air_temperature", "K", {}},
                          {"u_velocity", "m s^-1", {}}, {"v_velocity", "m s^-1", {}},
                          {"wind_speed", "m s^-1", {}}, {"w_velocity", "m s^-1", {}}};
  double zsum = 0.0;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      const size_t c = (size_t)k * plane + (size_t)j * nx + i;
      const float rho = s.rho[c], rt = s.rt[c], rr = std::max(rho, 1.0e-6f);
      const float theta = rt / rr;  // dry_theta_from_conserved (dry_thermo.hpp:21-24)
      const float ratio = std::max(rho * 287.05f * theta / 100000.0f, 1.0e-6f);
      const float p = 100000.0f * std::pow(ratio, 1.0f / (1.0f - 0.2854f));
      const float temp = theta * std::pow(std::max(p, 1.0f) / 100000.0f, 0.2854f);
      const float uc = 0.5f * (s.u[((size_t)k * ny + j) * (nx + 1) + i] + s.u[((size_t)k * ny + j) * (nx + 1) + i + 1]);
      const float vc = 0.5f * (s.v[((size_t)k * (ny + 1) + j) * nx + i] + s.v[((size_t)k * (ny + 1) + j + 1) * nx + i]);
      const float wc = 0.5f * (s.w[c] + s.w[c + plane]);
      const float u = uc / rr, v = vc / rr, w = wc / rr;
      const float z = zc[c];
      zsum += (double)z;
      const double vals[10] = {terrain.empty() ? 0.0 : (double)terrain[(size_t)j * nx + i], z, rho, theta, p, temp,
                               u, v, std::sqrt(u * u + v * v), w};
      for (int q = 0; q < 10; ++q) f[q].v.push_back(vals[q]);
    }
  std::ostringstream js;
  js << std::setprecision(10);
  js << "{\n  \"schema_version\": " << json_string("gwm-next-plan-view/v1") << ",\n";
  js << "  \"case\": " << json_string(o.case_kind) << ",\n";
  js << "  \"steps\": " << o.steps << ",\n  \"dt\": " << o.step.dt << ",\n  \"slice_k\": " << k << ",\n";
  js << "  \"grid\": {\n    \"nx\": " << nx << ",\n    \"ny\": " << ny << ",\n    \"dx\": " << D.dx
     << ",\n    \"dy\": " << D.dy << ",\n    \"slice_mean_height_m\": " << zsum / (double)(nx * ny) << "\n  },\n";
  js << "  \"fields\": [\n";
  for (size_t n = 0; n < f.size(); ++n) {
    js << "    {\n      \"name\": " << json_string(f[n].name) << ",\n      \"units\": " << json_string(f[n].units)
       << ",\n      \"location\": \"cell_center\",\n      \"nx\": " << nx << ",\n      \"ny\": " << ny
       << ",\n      \"storage\": \"row_major_yx\",\n      \"values\": [";
    for (size_t q = 0; q < f[n].v.size(); ++q) js << (q ? ", " : "") << f[n].v[q];
    js << "]\n    }" << (n + 1 < f.size() ? "," : "") << "\n";
  }
  js << "  ]\n}";
  return js.str();
}

void check(int rc, gwm_b200_ctx* ctx, const char* what) {
  if (rc == GWM_B200_OK) return;
  std::string msg = std::string(what) + " failed with status " + std::to_string(rc);
  if (ctx) msg += ": " + std::string(gwm_b200_last_error(ctx));
  throw std::runtime_error(msg);
}

}  // namespace

int main(int argc, char** argv) {
  gwm_b200_ctx* ctx = nullptr;
  try {
    Options o;
    parse(argc, argv, o);
    const Domain& D = o.domain;
    if (D.nx <= 0 || D.ny <= 0 || D.nz <= 0) throw std::runtime_error("--nx, --ny and --nz must be positive");
    if (D.halo != 1) throw std::runtime_error("only --halo 1 is supported (every stencil of the step reaches one cell)");

    std::vector<float> terrain((size_t)D.nx * D.ny, 0.0f);
    if (D.terrain_kind == "cosine_mountain") {
      gwm_b200_terrain_params tp{D.height, D.center_x, D.center_y, D.half_width_x, D.half_width_y};
      check(gwm_b200_build_terrain("cosine_mountain", D.nx, D.ny, D.dx, D.dy, &tp, terrain.data()), nullptr,
            "terrain");
    }
    gwm_b200_grid_desc grid{D.nx, D.ny, D.nz, 1, D.ranks_x, D.ranks_y, D.periodic_x ? 1 : 0, D.periodic_y ? 1 : 0,
                            D.dx, D.dy, D.z_top, D.terrain_taper_eta,
                            D.terrain_kind == "flat" ? nullptr : terrain.data(), nullptr};
    gwm_b200_member_desc member{};
    member.step = o.step;

    State s;
    const size_t cells = (size_t)D.nx * D.ny * D.nz;
    s.rho.resize(cells);
    s.rt.resize(cells);
    s.u.resize((size_t)(D.nx + 1) * D.ny * D.nz);
    s.v.resize((size_t)D.nx * (D.ny + 1) * D.nz);
    s.w.resize((size_t)D.nx * D.ny * (D.nz + 1));
    gwm_b200_fields f{s.rho.data(), s.rt.data(), s.u.data(), s.v.data(), s.w.data(), nullptr, nullptr, nullptr, nullptr};
    const gwm_b200_case_params cp = case_params(o);
    check(gwm_b200_build_case(o.case_kind.c_str(), &grid, &cp, &f), nullptr, "case setup");
    const Summary initial = summarize(s, D);

    check(gwm_b200_create(&grid, &member, 1, &ctx), nullptr, "context creation");
    check(gwm_b200_upload(ctx, 0, &f), ctx, "upload");
    if (o.steps > 0) check(gwm_b200_advance_dry(ctx, o.steps), ctx, "advance_dry_state_ssprk3");
    check(gwm_b200_download(ctx, 0, &f), ctx, "download");
    gwm_b200_destroy(ctx);
    ctx = nullptr;
    const Summary final_ = summarize(s, D);

    std::ostringstream js;
    js << "{\n";
    js << "  \"case\": \"" << o.case_kind << "\",\n";
    js << "  \"steps\": " << o.steps << ",\n";
    js << "  \"dt\": " << o.step.dt << ",\n";
    js << "  \"initial\": " << summary_json(initial, "    ") << ",\n";
    js << "  \"final\": " << summary_json(final_, "    ") << "\n";
    js << "}";
    std::cout << js.str() << "\n";
    if (!o.summary_json_path.empty()) {
      std::ofstream out(o.summary_json_path, std::ios::binary);
      if (!out) throw std::runtime_error("Failed to open summary path: " + o.summary_json_path);
      out << js.str() << "\n";
    }
    if (!o.plan_view_json_path.empty()) {
      std::vector<float> zc(cells);
      check(gwm_b200_grid_z_center(&grid, zc.data()), nullptr, "grid metrics");
      const std::string pv = plan_view_json(o, s, D.terrain_kind == "flat" ? std::vector<float>() : terrain, zc,
                                            o.plan_view_level);
      std::ofstream out(o.plan_view_json_path, std::ios::binary);
      if (!out) throw std::runtime_error("Failed to open plan-view output path: " + o.plan_view_json_path);
      out << pv << "\n";
    }
    return EXIT_SUCCESS;
  } catch (const std::exception& ex) {
    if (ctx) gwm_b200_destroy(ctx);
    std::cerr << "gwm_b200_idealized_driver error: " << ex.what() << "\n";
    return EXIT_FAILURE;
  }
}
