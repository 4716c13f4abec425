// ref_golden.cpp — runs the reference's own step operators on one case file and
// writes the resulting fields.  Test infrastructure only: it produces golden
// vectors that pin the oracle restatement and the CUDA path to the reference
// implementation itself.  Built against the reference sources by oracle/Makefile
// (target `ref`); nothing in the product links it.
//
// The step sequence is the prepared-case driver loop
// (src/core/gwm_prepared_case_driver.cpp:427-463): advance_dry_state_ssprk3
// (include/gwm/dycore/dry_core.hpp:106-110) with NullBoundaryUpdater and
// LocalSplitExplicitFastMode (or no fast modes), then
// advance_passive_tracers_ssprk3 (passive_tracer.hpp:44-49) and
// apply_warm_rain_microphysics (warm_rain.hpp:57-68; metric or nominal overload).
//
// A second case kind (ScalarHeader, magic "GWMSCAL1") runs advance_scalar_ssprk3.
//
// Case file (little endian): CaseHeader, then float arrays in global C order
// (k, j, i): terrain (ny, nx), rho (nz, ny, nx), rho_theta (nz, ny, nx),
// u (nz, ny, nx+1), v (nz, ny+1, nx), w (nz+1, ny, nx) and, when moist, the
// tracer masses rho*qv, rho*qc, rho*qr (nz, ny, nx).
// Output file: "GWMOUT01", then the same state arrays after `steps` steps and,
// when moist, the surface precipitation (ny, nx).
// Each step's wall time (host clock around the step and a device synchronisation) goes
// to stderr as "step <n> ms <t>", so the reference's own GPU step can be timed too.
// With a third and fourth argument (path, level) the reference's runtime plan view of the
// final state (extract_runtime_plan_view, src/io/plan_view_output.cpp:715-834, with the
// warm-rain accumulation of a moist case) is written there by plan_view_bundle_to_json.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "gwm/comm/virtual_rank_layout.hpp"
#include "gwm/domain/grid_metrics.hpp"
#include "gwm/dycore/dry_core.hpp"
#include "gwm/dycore/dry_transport.hpp"
#include "gwm/dycore/passive_tracer.hpp"
#include "gwm/io/plan_view_output.hpp"
#include "gwm/physics/warm_rain.hpp"
#include "gwm/state/tracer_registry.hpp"

namespace {

struct CaseHeader {
  char magic[8];  // "GWMCASE1"
  int nx, ny, nz, ranks_x, ranks_y, periodic_x, periodic_y;
  int fast_substeps, fast_hmom, fast_density, fast_modes, steps;
  int moist, rain_mode, latent_heating, pad;
  double dx, dy, z_top, taper, dt, gravity;
  double relax, autoconv_threshold, autoconv_rate, evap_rate, terminal_velocity, layer_depth;
};

class NoFastModes final : public gwm::dycore::FastModeIntegrator {
 public:
  void apply(std::vector<gwm::dycore::DryState>&, const std::vector<gwm::domain::SubdomainDescriptor>&,
             const gwm::domain::GridMetrics&, const gwm::dycore::DryStepperConfig&) override {}
};

std::vector<float> read_floats(std::FILE* f, size_t n) {
  std::vector<float> v(n);
  if (std::fread(v.data(), sizeof(float), n, f) != n) throw std::runtime_error("short case file");
  return v;
}

void write_floats(std::FILE* f, const std::vector<float>& v) {
  if (std::fwrite(v.data(), sizeof(float), v.size(), f) != v.size()) throw std::runtime_error("write failed");
}

// Global array extents of a field: ox/oy/oz = 1 along the face orientation.
struct Ext {
  int ox, oy, oz;
};

void scatter(const std::vector<float>& g, const Ext& e, int gnx, int gny,
             const std::vector<gwm::domain::SubdomainDescriptor>& layout,
             const std::vector<gwm::state::Field3D<gwm::real>*>& fields) {
  for (size_t r = 0; r < layout.size(); ++r) {
    const auto& d = layout[r];
    auto& f = *fields[r];
    for (int k = 0; k < d.nz + e.oz; ++k)
      for (int j = 0; j < d.ny_local() + e.oy; ++j)
        for (int i = 0; i < d.nx_local() + e.ox; ++i) {
          const size_t gi = d.i_begin + i, gj = d.j_begin + j;
          f(i, j, k) = g[(k * size_t(gny + e.oy) + gj) * size_t(gnx + e.ox) + gi];
        }
  }
}

// Owned positions of each rank; a face shared by two ranks is taken from the rank
// that owns the cell on its high side (the low rank's last face is skipped).
std::vector<float> gather(const Ext& e, int gnx, int gny, int gnz,
                          const std::vector<gwm::domain::SubdomainDescriptor>& layout,
                          const std::vector<const gwm::state::Field3D<gwm::real>*>& fields) {
  std::vector<float> g(size_t(gnx + e.ox) * (gny + e.oy) * (gnz + e.oz), 0.0f);
  for (size_t r = 0; r < layout.size(); ++r) {
    const auto& d = layout[r];
    const auto& f = *fields[r];
    const int xe = d.nx_local() + ((e.ox && d.i_end == gnx) ? 1 : 0);
    const int ye = d.ny_local() + ((e.oy && d.j_end == gny) ? 1 : 0);
    for (int k = 0; k < d.nz + e.oz; ++k)
      for (int j = 0; j < ye; ++j)
        for (int i = 0; i < xe; ++i) {
          const size_t gi = d.i_begin + i, gj = d.j_begin + j;
          g[(k * size_t(gny + e.oy) + gj) * size_t(gnx + e.ox) + gi] = f(i, j, k);
        }
  }
  return g;
}

int run(const char* in_path, const char* out_path, const char* plan_view_path, int plan_view_level) {
  std::FILE* in = std::fopen(in_path, "rb");
  if (!in) throw std::runtime_error(std::string("cannot open ") + in_path);
  CaseHeader h{};
  if (std::fread(&h, sizeof(h), 1, in) != 1 || std::memcmp(h.magic, "GWMCASE1", 8) != 0)
    throw std::runtime_error("bad case header");
  const int nx = h.nx, ny = h.ny, nz = h.nz;
  const size_t nc = size_t(nx) * ny * nz;
  const auto terrain = read_floats(in, size_t(nx) * ny);
  const auto rho = read_floats(in, nc);
  const auto rt = read_floats(in, nc);
  const auto u = read_floats(in, size_t(nx + 1) * ny * nz);
  const auto v = read_floats(in, size_t(nx) * (ny + 1) * nz);
  const auto w = read_floats(in, size_t(nx) * ny * (nz + 1));
  std::vector<float> qm[3];
  if (h.moist)
    for (auto& q : qm) q = read_floats(in, nc);
  std::fclose(in);

  const auto layout = gwm::comm::VirtualRankLayout::build(nx, ny, nz, 1, h.ranks_x, h.ranks_y,
                                                          h.periodic_x != 0, h.periodic_y != 0);
  std::vector<gwm::real> terrain_r(terrain.begin(), terrain.end());
  const auto metrics = gwm::domain::GridMetrics::make_hybrid_height(
      nx, ny, nz, h.dx, h.dy, h.z_top, terrain_r, h.taper, h.periodic_x != 0, h.periodic_y != 0);

  std::vector<gwm::dycore::DryState> states;
  for (const auto& d : layout)
    states.emplace_back(d.nx_local(), d.ny_local(), nz, d.halo, "golden_rank_" + std::to_string(d.rank));
  for (auto& s : states) s.fill_constant(0.0f, 0.0f, 0.0f, 0.0f, 0.0f);
  auto pick = [&](auto fn) {
    std::vector<gwm::state::Field3D<gwm::real>*> p;
    for (auto& s : states) p.push_back(&fn(s));
    return p;
  };
  using DS = gwm::dycore::DryState;
  scatter(rho, {0, 0, 0}, nx, ny, layout, pick([](DS& s) -> gwm::state::Field3D<gwm::real>& { return s.rho_d; }));
  scatter(rt, {0, 0, 0}, nx, ny, layout, pick([](DS& s) -> gwm::state::Field3D<gwm::real>& { return s.rho_theta_m; }));
  scatter(u, {1, 0, 0}, nx, ny, layout, pick([](DS& s) -> gwm::state::Field3D<gwm::real>& { return s.mom_u.storage(); }));
  scatter(v, {0, 1, 0}, nx, ny, layout, pick([](DS& s) -> gwm::state::Field3D<gwm::real>& { return s.mom_v.storage(); }));
  scatter(w, {0, 0, 1}, nx, ny, layout, pick([](DS& s) -> gwm::state::Field3D<gwm::real>& { return s.mom_w.storage(); }));

  const char* names[3] = {gwm::state::kSpecificHumidityTracerName, gwm::state::kCloudWaterTracerName,
                          gwm::state::kRainWaterTracerName};
  std::vector<gwm::state::TracerState> tracers;
  std::vector<gwm::physics::WarmRainSurfaceAccumulation> accum(layout.size());
  if (h.moist) {
    const std::vector<gwm::real> zeros(nc, 0.0f);
    tracers = gwm::dycore::make_warm_rain_tracers_from_global_fields(states, layout, nx, ny, zeros);
    for (int t = 0; t < 3; ++t) {
      std::vector<gwm::state::Field3D<gwm::real>*> p;
      for (auto& tr : tracers) p.push_back(&tr.mass(names[t]));
      scatter(qm[t], {0, 0, 0}, nx, ny, layout, p);
    }
    for (size_t r = 0; r < layout.size(); ++r)
      accum[r].reset(layout[r].nx_local(), layout[r].ny_local(), h.dx * h.dy);
  }

  gwm::dycore::DryStepperConfig cfg;
  cfg.dt = static_cast<gwm::real>(h.dt);
  cfg.fast_substeps = h.fast_substeps;
  cfg.gravity = static_cast<gwm::real>(h.gravity);
  cfg.fast_update_horizontal_momentum = h.fast_hmom != 0;
  cfg.fast_update_density = h.fast_density != 0;
  gwm::physics::WarmRainConfig rc;
  rc.dt = static_cast<gwm::real>(h.dt);
  rc.condensation_relaxation = static_cast<gwm::real>(h.relax);
  rc.cloud_autoconversion_threshold = static_cast<gwm::real>(h.autoconv_threshold);
  rc.cloud_autoconversion_rate = static_cast<gwm::real>(h.autoconv_rate);
  rc.rain_evaporation_rate = static_cast<gwm::real>(h.evap_rate);
  rc.rain_terminal_velocity = static_cast<gwm::real>(h.terminal_velocity);
  rc.sedimentation_layer_depth_m = static_cast<gwm::real>(h.layer_depth);
  rc.enable_latent_heating = h.latent_heating != 0;

  gwm::dycore::NullBoundaryUpdater boundary;
  gwm::dycore::NullTracerBoundaryUpdater tracer_boundary;
  gwm::dycore::LocalSplitExplicitFastMode fast;
  NoFastModes no_fast;
  gwm::dycore::FastModeIntegrator& fm = h.fast_modes ? static_cast<gwm::dycore::FastModeIntegrator&>(fast)
                                                     : static_cast<gwm::dycore::FastModeIntegrator&>(no_fast);
  for (int step = 0; step < h.steps; ++step) {
    if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("device error before a step");
    const auto t0 = std::chrono::steady_clock::now();
    gwm::dycore::advance_dry_state_ssprk3(states, layout, metrics, cfg, boundary, fm);
    if (h.moist) {
      gwm::dycore::advance_passive_tracers_ssprk3(tracers, states, layout, metrics, cfg, tracer_boundary);
      if (h.rain_mode == 1)
        gwm::physics::apply_warm_rain_microphysics(states, tracers, layout, metrics, rc, &accum);
      else if (h.rain_mode == 2)
        gwm::physics::apply_warm_rain_microphysics(states, tracers, rc, &accum);
    }
    if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("device error in a step");
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::fprintf(stderr, "step %d ms %.3f\n", step, ms);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("device error after the steps");

  std::FILE* out = std::fopen(out_path, "wb");
  if (!out) throw std::runtime_error(std::string("cannot write ") + out_path);
  std::fwrite("GWMOUT01", 1, 8, out);
  auto cpick = [&](auto fn) {
    std::vector<const gwm::state::Field3D<gwm::real>*> p;
    for (const auto& s : states) p.push_back(&fn(s));
    return p;
  };
  using CF = const gwm::state::Field3D<gwm::real>&;
  write_floats(out, gather({0, 0, 0}, nx, ny, nz, layout, cpick([](const DS& s) -> CF { return s.rho_d; })));
  write_floats(out, gather({0, 0, 0}, nx, ny, nz, layout, cpick([](const DS& s) -> CF { return s.rho_theta_m; })));
  write_floats(out, gather({1, 0, 0}, nx, ny, nz, layout, cpick([](const DS& s) -> CF { return s.mom_u.storage(); })));
  write_floats(out, gather({0, 1, 0}, nx, ny, nz, layout, cpick([](const DS& s) -> CF { return s.mom_v.storage(); })));
  write_floats(out, gather({0, 0, 1}, nx, ny, nz, layout, cpick([](const DS& s) -> CF { return s.mom_w.storage(); })));
  if (h.moist) {
    for (int t = 0; t < 3; ++t) {
      std::vector<const gwm::state::Field3D<gwm::real>*> p;
      for (const auto& tr : tracers) p.push_back(&tr.mass(names[t]));
      write_floats(out, gather({0, 0, 0}, nx, ny, nz, layout, p));
    }
    std::vector<const gwm::state::Field3D<gwm::real>*> p;
    for (const auto& a : accum) p.push_back(&a.liquid_precipitation_kg_m2);
    // the accumulation fields are halo-free (nx_local, ny_local, 1)
    std::vector<float> pr(size_t(nx) * ny, 0.0f);
    for (size_t r = 0; r < layout.size(); ++r)
      for (int j = 0; j < layout[r].ny_local(); ++j)
        for (int i = 0; i < layout[r].nx_local(); ++i)
          pr[size_t(layout[r].j_begin + j) * nx + layout[r].i_begin + i] = (*p[r])(i, j, 0);
    write_floats(out, pr);
  }
  std::fclose(out);
  if (plan_view_path) {
    const auto bundle = gwm::io::extract_runtime_plan_view(states, tracers, layout, metrics, "golden", h.steps,
                                                           cfg.dt, plan_view_level, h.moist ? &accum : nullptr);
    std::FILE* pv = std::fopen(plan_view_path, "wb");
    if (!pv) throw std::runtime_error(std::string("cannot write ") + plan_view_path);
    const std::string js = gwm::io::plan_view_bundle_to_json(bundle);
    std::fwrite(js.data(), 1, js.size(), pv);
    std::fclose(pv);
  }
  return 0;
}

// Scalar-advection case (magic "GWMSCAL1"): ScalarHeader, then q (nz, ny, nx) floats.
// `steps` calls of advance_scalar_ssprk3 (include/gwm/dycore/dry_transport.hpp:19-21)
// on the virtual-rank fields; output "GWMSCA01" + q.
struct ScalarHeader {
  char magic[8];  // "GWMSCAL1"
  int nx, ny, nz, ranks_x, ranks_y, periodic_x, periodic_y, steps;
  float u_adv, v_adv, dt, dx, dy, pad;
};

int run_scalar(const char* in_path, const char* out_path) {
  std::FILE* in = std::fopen(in_path, "rb");
  if (!in) throw std::runtime_error(std::string("cannot open ") + in_path);
  ScalarHeader h{};
  if (std::fread(&h, sizeof(h), 1, in) != 1 || std::memcmp(h.magic, "GWMSCAL1", 8) != 0)
    throw std::runtime_error("bad scalar case header");
  const auto q = read_floats(in, size_t(h.nx) * h.ny * h.nz);
  std::fclose(in);
  const auto layout = gwm::comm::VirtualRankLayout::build(h.nx, h.ny, h.nz, 1, h.ranks_x, h.ranks_y,
                                                          h.periodic_x != 0, h.periodic_y != 0);
  std::vector<gwm::state::Field3D<gwm::real>> fields;
  for (const auto& d : layout) {
    fields.emplace_back(d.nx_local(), d.ny_local(), h.nz, d.halo, "golden_scalar_" + std::to_string(d.rank));
    fields.back().fill(0.0f);
  }
  std::vector<gwm::state::Field3D<gwm::real>*> p;
  for (auto& f : fields) p.push_back(&f);
  scatter(q, {0, 0, 0}, h.nx, h.ny, layout, p);
  gwm::dycore::DryTransportConfig cfg;
  cfg.u_adv = h.u_adv;
  cfg.v_adv = h.v_adv;
  cfg.dt = h.dt;
  cfg.dx = h.dx;
  cfg.dy = h.dy;
  for (int step = 0; step < h.steps; ++step) gwm::dycore::advance_scalar_ssprk3(fields, layout, cfg);
  if (cudaDeviceSynchronize() != cudaSuccess) throw std::runtime_error("device error after the steps");
  std::vector<const gwm::state::Field3D<gwm::real>*> cp;
  for (const auto& f : fields) cp.push_back(&f);
  std::FILE* out = std::fopen(out_path, "wb");
  if (!out) throw std::runtime_error(std::string("cannot write ") + out_path);
  std::fwrite("GWMSCA01", 1, 8, out);
  write_floats(out, gather({0, 0, 0}, h.nx, h.ny, h.nz, layout, cp));
  std::fclose(out);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3 && argc != 5) {
    std::fprintf(stderr, "usage: %s <case.bin> <out.bin> [<plan_view.json> <level>]\n", argv[0]);
    return 2;
  }
  try {
    char magic[8] = {};
    if (std::FILE* f = std::fopen(argv[1], "rb")) {
      if (std::fread(magic, 1, 8, f) != 8) magic[0] = 0;
      std::fclose(f);
    }
    if (std::memcmp(magic, "GWMSCAL1", 8) == 0) return run_scalar(argv[1], argv[2]);
    return run(argv[1], argv[2], argc == 5 ? argv[3] : nullptr, argc == 5 ? std::atoi(argv[4]) : 0);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_golden error: %s\n", e.what());
    return 1;
  }
}
