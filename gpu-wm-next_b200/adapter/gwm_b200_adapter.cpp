// gwm_b200_adapter.cpp — drop-in definitions of gpu-wm-next's step operators over the
// libgwm_b200 C-ABI, with the reference's own signatures.
//
// A gwm-next build that compiles this file in place of its CUDA step sources runs the
// step on the B200 path while its drivers, tests and state types stay as they are:
//   advance_dry_state_ssprk3        include/gwm/dycore/dry_core.hpp:106-110
//   LocalSplitExplicitFastMode::apply (FastModeIntegrator)  dry_core.hpp:73-88
//   B200FastModes, the same integrator as a class of its own
//   advance_passive_tracers_ssprk3  include/gwm/dycore/passive_tracer.hpp:44-49
//   advance_scalar_ssprk3           include/gwm/dycore/dry_transport.hpp:19-21
//   apply_warm_rain_microphysics    include/gwm/physics/warm_rain.hpp:57-68 (both overloads)
// Each call gathers the per-rank Field3D storage into global owned arrays
// (gwm_b200_ranks_to_global), uploads it into a context, runs the operator on the device
// and scatters the result back (gwm_b200_global_to_ranks).  States are host-visible
// (the reference's managed memory), so no staging beyond those arrays is needed.  A long
// run keeps one context and its state on the device instead (gwm_b200_step): this file
// favours a faithful per-call contract over speed.
//
// Errors: a non-zero status becomes std::runtime_error through gwm::require, as the
// reference reports failures (include/gwm/core/types.hpp:24-28).
//
// With GWM_B200_ADAPTER_REPORT set in the environment, the process prints at exit how many
// times each operator ran here ("gwm_b200 adapter: <operator> <calls>"), which shows a
// linked program which definitions it used.
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "gwm/dycore/dry_core.hpp"
#include "gwm/dycore/dry_transport.hpp"
#include "gwm/dycore/passive_tracer.hpp"
#include "gwm/physics/warm_rain.hpp"
#include "gwm/state/tracer_registry.hpp"

extern "C" {
#include "gwm_b200.h"
}

namespace gwm::b200 {

enum Op { kDry, kFast, kTracers, kScalar, kRainBox, kRainMetric, kOps };
inline std::atomic<long>& calls(int op) {
  static std::atomic<long> c[kOps];
  return c[op];
}
struct CallReport {
  ~CallReport() {
    if (!std::getenv("GWM_B200_ADAPTER_REPORT")) return;
    const char* names[kOps] = {"advance_dry_state_ssprk3", "fast_modes", "advance_passive_tracers_ssprk3",
                               "advance_scalar_ssprk3", "apply_warm_rain_microphysics(box)",
                               "apply_warm_rain_microphysics(metric)"};
    for (int op = 0; op < kOps; ++op) std::fprintf(stderr, "gwm_b200 adapter: %s %ld\n", names[op], calls(op).load());
  }
};
inline void count(int op) {
  static CallReport report;  // printed when the program exits
  ++calls(op);
}

using dycore::DryState;
using domain::GridMetrics;
using domain::SubdomainDescriptor;

// Field orientations of the C-ABI: 0 cell, 1 X face, 2 Y face, 3 Z face.
enum { kCell = 0, kFaceX = 1, kFaceY = 2, kFaceZ = 3 };

inline void check(int rc, gwm_b200_ctx* ctx, const char* what) {
  gwm::require(rc == GWM_B200_OK, std::string("gwm_b200 ") + what + ": " +
                                      (ctx ? gwm_b200_last_error(ctx) : "status " + std::to_string(rc)));
}

inline gwm_b200_layout_desc layout_desc(const std::vector<SubdomainDescriptor>& L) {
  const auto& d = L.front();
  return {d.global_nx, d.global_ny, d.nz, d.halo, d.ranks_x, d.ranks_y, d.periodic_x ? 1 : 0,
          d.periodic_y ? 1 : 0};
}

inline size_t global_count(const gwm_b200_layout_desc& ld, int orient) {
  return size_t(ld.global_nx + (orient == kFaceX)) * (ld.global_ny + (orient == kFaceY)) *
         (ld.nz + (orient == kFaceZ));
}

// Owned parts of the ranks' storage gathered onto the global grid, and back.
template <class Pick>
std::vector<float> gather(const gwm_b200_layout_desc& ld, int orient, size_t nranks, Pick pick) {
  std::vector<const float*> ranks;
  for (size_t r = 0; r < nranks; ++r) ranks.push_back(pick(r).data());
  std::vector<float> g(global_count(ld, orient));
  check(gwm_b200_ranks_to_global(&ld, orient, ranks.data(), g.data()), nullptr, "ranks_to_global");
  return g;
}
template <class Pick>
void scatter(const gwm_b200_layout_desc& ld, int orient, const std::vector<float>& g, size_t nranks, Pick pick) {
  std::vector<float*> ranks;
  for (size_t r = 0; r < nranks; ++r) ranks.push_back(pick(r).data());
  check(gwm_b200_global_to_ranks(&ld, orient, g.data(), ranks.data()), nullptr, "global_to_ranks");
}

// The dry state of every rank as global owned arrays.
struct GlobalDry {
  std::vector<float> rho, rt, u, v, w;
  void gather_from(const std::vector<DryState>& s, const gwm_b200_layout_desc& ld) {
    const size_t n = s.size();
    rho = gather(ld, kCell, n, [&](size_t r) -> const state::Field3D<real>& { return s[r].rho_d; });
    rt = gather(ld, kCell, n, [&](size_t r) -> const state::Field3D<real>& { return s[r].rho_theta_m; });
    u = gather(ld, kFaceX, n, [&](size_t r) -> const state::Field3D<real>& { return s[r].mom_u.storage(); });
    v = gather(ld, kFaceY, n, [&](size_t r) -> const state::Field3D<real>& { return s[r].mom_v.storage(); });
    w = gather(ld, kFaceZ, n, [&](size_t r) -> const state::Field3D<real>& { return s[r].mom_w.storage(); });
  }
  void scatter_to(std::vector<DryState>& s, const gwm_b200_layout_desc& ld) const {
    const size_t n = s.size();
    scatter(ld, kCell, rho, n, [&](size_t r) -> state::Field3D<real>& { return s[r].rho_d; });
    scatter(ld, kCell, rt, n, [&](size_t r) -> state::Field3D<real>& { return s[r].rho_theta_m; });
    scatter(ld, kFaceX, u, n, [&](size_t r) -> state::Field3D<real>& { return s[r].mom_u.storage(); });
    scatter(ld, kFaceY, v, n, [&](size_t r) -> state::Field3D<real>& { return s[r].mom_v.storage(); });
    scatter(ld, kFaceZ, w, n, [&](size_t r) -> state::Field3D<real>& { return s[r].mom_w.storage(); });
  }
  gwm_b200_fields fields() {
    gwm_b200_fields f{};
    f.rho_d = rho.data(); f.rho_theta_m = rt.data(); f.mom_u = u.data(); f.mom_v = v.data(); f.mom_w = w.data();
    return f;
  }
};

// One context for the grid of `metrics` (terrain, eta levels, periodicity and rank layout
// taken from the reference's GridMetrics and layout).
class Context {
 public:
  Context(const GridMetrics& m, const std::vector<SubdomainDescriptor>& L, const gwm_b200_member_desc& member) {
    terrain_.resize(size_t(m.nx) * m.ny);
    for (int j = 0; j < m.ny; ++j)
      for (int i = 0; i < m.nx; ++i) terrain_[size_t(j) * m.nx + i] = m.terrain_height(i, j);
    gwm_b200_grid_desc g{};
    g.nx = m.nx; g.ny = m.ny; g.nz = m.nz; g.halo = 1;
    g.ranks_x = L.front().ranks_x; g.ranks_y = L.front().ranks_y;
    g.periodic_x = L.front().periodic_x ? 1 : 0; g.periodic_y = L.front().periodic_y ? 1 : 0;
    g.dx = m.dx; g.dy = m.dy; g.z_top = m.z_top; g.terrain_taper_eta = m.terrain_taper_eta;
    g.terrain = terrain_.data();
    g.eta_interfaces = m.eta_interfaces.size() == size_t(m.nz) + 1 ? m.eta_interfaces.data() : nullptr;
    check(gwm_b200_create(&g, &member, 1, &ctx_), nullptr, "create");
  }
  // a single-rank box of nx x ny x nz cells (the warm-rain overload without metrics)
  Context(int nx, int ny, int nz, const gwm_b200_member_desc& member) {
    gwm_b200_grid_desc g{};
    g.nx = nx; g.ny = ny; g.nz = nz; g.halo = 1; g.ranks_x = 1; g.ranks_y = 1;
    g.periodic_x = 1; g.periodic_y = 1; g.dx = 1000.0; g.dy = 1000.0; g.z_top = 1000.0 * nz;
    g.terrain_taper_eta = 0.25;
    check(gwm_b200_create(&g, &member, 1, &ctx_), nullptr, "create");
  }
  ~Context() { gwm_b200_destroy(ctx_); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  gwm_b200_ctx* get() { return ctx_; }
  void ok(int rc, const char* what) { check(rc, ctx_, what); }

 private:
  std::vector<float> terrain_;
  gwm_b200_ctx* ctx_ = nullptr;
};

inline gwm_b200_step_config step_config(const dycore::DryStepperConfig& c, bool fast_modes) {
  gwm_b200_step_config s{};
  s.dt = c.dt;
  s.fast_substeps = c.fast_substeps;
  s.gravity = c.gravity;
  s.fast_update_horizontal_momentum = c.fast_update_horizontal_momentum ? 1 : 0;
  s.fast_update_density = c.fast_update_density ? 1 : 0;
  s.enable_fast_modes = fast_modes ? 1 : 0;
  return s;
}

inline gwm_b200_warm_rain_config rain_config(const physics::WarmRainConfig& c) {
  gwm_b200_warm_rain_config r{};
  r.dt = c.dt;
  r.condensation_relaxation = c.condensation_relaxation;
  r.cloud_autoconversion_threshold = c.cloud_autoconversion_threshold;
  r.cloud_autoconversion_rate = c.cloud_autoconversion_rate;
  r.rain_evaporation_rate = c.rain_evaporation_rate;
  r.rain_terminal_velocity = c.rain_terminal_velocity;
  r.sedimentation_layer_depth_m = c.sedimentation_layer_depth_m;
  r.enable_latent_heating = c.enable_latent_heating ? 1 : 0;
  return r;
}

}  // namespace gwm::b200

namespace gwm::dycore {

namespace {
// The split-explicit acoustic subcycle (dry_fast_modes.cu:400-656) of the states on the device.
void device_fast_modes(std::vector<DryState>& states, const std::vector<domain::SubdomainDescriptor>& layout,
                     const domain::GridMetrics& metrics, const DryStepperConfig& config) {
  b200::count(b200::kFast);
  const auto ld = b200::layout_desc(layout);
  gwm_b200_member_desc mem{};
  mem.step = b200::step_config(config, true);
  b200::Context ctx(metrics, layout, mem);
  b200::GlobalDry g;
  g.gather_from(states, ld);
  auto f = g.fields();
  ctx.ok(gwm_b200_upload(ctx.get(), 0, &f), "upload");
  ctx.ok(gwm_b200_fast_modes(ctx.get()), "fast_modes");
  ctx.ok(gwm_b200_download(ctx.get(), 0, &f), "download");
  g.scatter_to(states, ld);
}
}  // namespace

// The reference's fast-mode integrator class, its apply now on the device.
void LocalSplitExplicitFastMode::apply(std::vector<DryState>& states,
                                       const std::vector<domain::SubdomainDescriptor>& layout,
                                       const domain::GridMetrics& metrics, const DryStepperConfig& config) {
  device_fast_modes(states, layout, metrics, config);
}

// The same integrator under a name of its own, for code that adds it beside the reference's.
class B200FastModes final : public FastModeIntegrator {
 public:
  void apply(std::vector<DryState>& states, const std::vector<domain::SubdomainDescriptor>& layout,
             const domain::GridMetrics& metrics, const DryStepperConfig& config) override {
    device_fast_modes(states, layout, metrics, config);
  }
};

// advance_scalar_ssprk3 (dry_transport.cu:285-325) on the device: the ranks' fields gathered
// onto the global grid, advanced by gwm_b200_scalar_ssprk3 (the reference's roundings), and
// scattered back.
void advance_scalar_ssprk3(std::vector<state::Field3D<real>>& fields,
                           const std::vector<domain::SubdomainDescriptor>& layout, const DryTransportConfig& config) {
  b200::count(b200::kScalar);
  gwm::require(fields.size() == layout.size(), "Field/layout size mismatch in advance_scalar_ssprk3");
  if (fields.empty()) return;
  const auto ld = b200::layout_desc(layout);
  auto q = b200::gather(ld, b200::kCell, fields.size(), [&](size_t r) -> const state::Field3D<real>& { return fields[r]; });
  gwm_b200_scalar_desc d{ld.global_nx, ld.global_ny, ld.nz, ld.periodic_x, ld.periodic_y,
                         config.u_adv, config.v_adv, config.dt, config.dx, config.dy};
  float* dq = nullptr;
  gwm::require(cudaMalloc(&dq, q.size() * sizeof(float)) == cudaSuccess, "gwm_b200 adapter: device buffer");
  const bool ok = cudaMemcpy(dq, q.data(), q.size() * sizeof(float), cudaMemcpyHostToDevice) == cudaSuccess &&
                  gwm_b200_scalar_ssprk3(&d, dq, 1, nullptr) == GWM_B200_OK &&
                  cudaMemcpy(q.data(), dq, q.size() * sizeof(float), cudaMemcpyDeviceToHost) == cudaSuccess;
  cudaFree(dq);
  gwm::require(ok, "gwm_b200 adapter: scalar transport");
  b200::scatter(ld, b200::kCell, q, fields.size(), [&](size_t r) -> state::Field3D<real>& { return fields[r]; });
}

// advance_dry_state_ssprk3 (dry_core.cu:541-651) on the device.  The boundary updater must
// be the Null one and the fast modes the reference's split-explicit scheme (or this
// file's B200FastModes), or absent (NullFastModeIntegrator-like: any other integrator is
// rejected, since its code cannot run inside the device step).
void advance_dry_state_ssprk3(std::vector<DryState>& states, const std::vector<domain::SubdomainDescriptor>& layout,
                              const domain::GridMetrics& metrics, const DryStepperConfig& config,
                              BoundaryUpdater& boundary_updater, FastModeIntegrator& fast_modes) {
  b200::count(b200::kDry);
  gwm::require(!states.empty() && states.size() == layout.size(), "State/layout size mismatch");
  gwm::require(dynamic_cast<NullBoundaryUpdater*>(&boundary_updater) != nullptr,
               "gwm_b200 adapter: only the Null boundary updater runs inside the device step");
  const bool split_explicit = dynamic_cast<LocalSplitExplicitFastMode*>(&fast_modes) != nullptr ||
                              dynamic_cast<B200FastModes*>(&fast_modes) != nullptr;
  const auto ld = b200::layout_desc(layout);
  gwm_b200_member_desc mem{};
  mem.step = b200::step_config(config, split_explicit);
  b200::Context ctx(metrics, layout, mem);
  b200::GlobalDry g;
  g.gather_from(states, ld);
  auto f = g.fields();
  ctx.ok(gwm_b200_upload(ctx.get(), 0, &f), "upload");
  ctx.ok(gwm_b200_advance_dry(ctx.get(), 1), "advance_dry");
  ctx.ok(gwm_b200_download(ctx.get(), 0, &f), "download");
  g.scatter_to(states, ld);
}

// advance_passive_tracers_ssprk3 (dry_transport.cu:440-518) on the device: every tracer of
// the registry, with the dry states' frozen mass fluxes.  Null tracer boundary updater only.
void advance_passive_tracers_ssprk3(std::vector<state::TracerState>& tracers, const std::vector<DryState>& dry_states,
                                    const std::vector<domain::SubdomainDescriptor>& layout,
                                    const domain::GridMetrics& metrics, const DryStepperConfig& config,
                                    TracerBoundaryUpdater& boundary_updater) {
  b200::count(b200::kTracers);
  gwm::require(tracers.size() == dry_states.size() && dry_states.size() == layout.size(),
               "Tracer/state/layout size mismatch");
  if (tracers.empty() || tracers.front().size() == 0) return;
  gwm::require(dynamic_cast<NullTracerBoundaryUpdater*>(&boundary_updater) != nullptr,
               "gwm_b200 adapter: only the Null tracer boundary updater runs inside the device step");
  const auto ld = b200::layout_desc(layout);
  gwm_b200_member_desc mem{};
  mem.step = b200::step_config(config, true);
  mem.enable_tracer_transport = 1;
  b200::Context ctx(metrics, layout, mem);
  b200::GlobalDry g;
  g.gather_from(dry_states, ld);
  auto f = g.fields();
  ctx.ok(gwm_b200_upload(ctx.get(), 0, &f), "upload");
  const auto& reg = tracers.front().registry();
  const size_t nt = reg.size(), n = tracers.size();
  std::vector<std::vector<float>> mass(nt);
  for (size_t t = 0; t < nt; ++t) {
    const auto& spec = reg.at(int(t));
    const int idx = gwm_b200_tracer_add(ctx.get(), 0, spec.name.c_str(), spec.units.c_str(), spec.positive ? 1 : 0);
    gwm::require(idx == int(t), "gwm_b200 adapter: tracer registration");
    mass[t] = b200::gather(ld, b200::kCell, n, [&](size_t r) -> const state::Field3D<real>& {
      return tracers[r].mass(int(t));
    });
    ctx.ok(gwm_b200_tracer_upload(ctx.get(), 0, int(t), mass[t].data()), "tracer_upload");
  }
  ctx.ok(gwm_b200_advance_tracers(ctx.get()), "advance_tracers");
  for (size_t t = 0; t < nt; ++t) {
    ctx.ok(gwm_b200_tracer_download(ctx.get(), 0, int(t), mass[t].data()), "tracer_download");
    b200::scatter(ld, b200::kCell, mass[t], n, [&](size_t r) -> state::Field3D<real>& {
      return tracers[r].mass(int(t));
    });
  }
}

}  // namespace gwm::dycore

namespace gwm::physics {

namespace {

// The warm-rain tracers of a state, by registry name (warm_rain.cu:236-240).
struct RainIdx {
  int qv, qc, qr;
};
RainIdx rain_indices(const state::TracerState& t) {
  const auto qv = t.find(state::kSpecificHumidityTracerName);
  const auto qc = t.find(state::kCloudWaterTracerName);
  const auto qr = t.find(state::kRainWaterTracerName);
  gwm::require(qv && qc && qr, "Warm-rain microphysics requires qv, qc and qr tracers");
  return {*qv, *qc, *qr};
}

}  // namespace

// Unit-test overload (warm_rain.cu:214-271): every state is its own box; the fallout, when
// accumulations are given, uses the nominal layer depth.
void apply_warm_rain_microphysics(std::vector<dycore::DryState>& states, std::vector<state::TracerState>& tracers,
                                  const WarmRainConfig& config,
                                  std::vector<WarmRainSurfaceAccumulation>* accumulations) {
  b200::count(b200::kRainBox);
  gwm::require(states.size() == tracers.size(), "State/tracer size mismatch in warm-rain microphysics");
  if (accumulations) {
    gwm::require(accumulations->size() == states.size(), "Warm-rain accumulation/state size mismatch");
    for (size_t n = 0; n < states.size(); ++n)
      if (!(*accumulations)[n].matches(states[n].rho_d.nx(), states[n].rho_d.ny()))
        (*accumulations)[n].reset(states[n].rho_d.nx(), states[n].rho_d.ny());
  }
  for (size_t n = 0; n < states.size(); ++n) {
    auto& s = states[n];
    const int nx = s.rho_d.nx(), ny = s.rho_d.ny(), nz = s.rho_d.nz();
    gwm_b200_member_desc mem{};
    mem.moist = 1;
    mem.enable_warm_rain = 1;
    mem.step.dt = config.dt;
    mem.step.fast_substeps = 1;
    mem.rain = b200::rain_config(config);
    b200::Context ctx(nx, ny, nz, mem);
    const std::vector<domain::SubdomainDescriptor> one{[&] {
      domain::SubdomainDescriptor d{};
      d.global_nx = nx; d.global_ny = ny; d.nz = nz; d.halo = s.rho_d.halo();
      d.i_end = nx; d.j_end = ny;
      return d;
    }()};
    const auto ld = b200::layout_desc(one);
    b200::GlobalDry g;
    g.rho = b200::gather(ld, b200::kCell, 1, [&](size_t) -> const state::Field3D<real>& { return s.rho_d; });
    g.rt = b200::gather(ld, b200::kCell, 1, [&](size_t) -> const state::Field3D<real>& { return s.rho_theta_m; });
    g.u = b200::gather(ld, b200::kFaceX, 1, [&](size_t) -> const state::Field3D<real>& { return s.mom_u.storage(); });
    g.v = b200::gather(ld, b200::kFaceY, 1, [&](size_t) -> const state::Field3D<real>& { return s.mom_v.storage(); });
    g.w = b200::gather(ld, b200::kFaceZ, 1, [&](size_t) -> const state::Field3D<real>& { return s.mom_w.storage(); });
    const RainIdx ix = rain_indices(tracers[n]);
    auto pick = [&](int t) {
      return b200::gather(ld, b200::kCell, 1, [&](size_t) -> const state::Field3D<real>& { return tracers[n].mass(t); });
    };
    std::vector<float> qv = pick(ix.qv), qc = pick(ix.qc), qr = pick(ix.qr);
    std::vector<double> precip(size_t(nx) * ny, 0.0);
    const bool fall = accumulations && config.rain_terminal_velocity > 0.0f && config.sedimentation_layer_depth_m > 0.0f;
    if (fall) {
      const auto& acc = (*accumulations)[n].liquid_precipitation_kg_m2;
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) precip[size_t(j) * nx + i] = acc(i, j, 0);
    }
    auto f = g.fields();
    f.qv = qv.data(); f.qc = qc.data(); f.qr = qr.data(); f.precip = precip.data();
    ctx.ok(gwm_b200_upload(ctx.get(), 0, &f), "upload");
    ctx.ok(gwm_b200_warm_rain(ctx.get(), fall ? 2 : 0), "warm_rain");
    ctx.ok(gwm_b200_download(ctx.get(), 0, &f), "download");
    b200::scatter(ld, b200::kCell, g.rho, 1, [&](size_t) -> state::Field3D<real>& { return s.rho_d; });
    b200::scatter(ld, b200::kCell, g.rt, 1, [&](size_t) -> state::Field3D<real>& { return s.rho_theta_m; });
    auto put = [&](int t, const std::vector<float>& q) {
      b200::scatter(ld, b200::kCell, q, 1, [&](size_t) -> state::Field3D<real>& { return tracers[n].mass(t); });
    };
    put(ix.qv, qv); put(ix.qc, qc); put(ix.qr, qr);
    if (fall) {
      auto& acc = (*accumulations)[n].liquid_precipitation_kg_m2;
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) acc(i, j, 0) = float(precip[size_t(j) * nx + i]);
    }
  }
}

// Metric overload (warm_rain.cu:273-353): the ranks' states on the global grid, fallout
// with the metric layer depths when accumulations are given.
void apply_warm_rain_microphysics(std::vector<dycore::DryState>& states, std::vector<state::TracerState>& tracers,
                                  const std::vector<domain::SubdomainDescriptor>& layout,
                                  const domain::GridMetrics& metrics, const WarmRainConfig& config,
                                  std::vector<WarmRainSurfaceAccumulation>* accumulations) {
  b200::count(b200::kRainMetric);
  gwm::require(states.size() == tracers.size() && states.size() == layout.size() && !layout.empty(),
               "State/tracer/layout size mismatch in warm-rain microphysics");
  if (accumulations) {
    gwm::require(accumulations->size() == states.size(), "Warm-rain accumulation/state size mismatch");
    for (size_t n = 0; n < states.size(); ++n)
      if (!(*accumulations)[n].matches(states[n].rho_d.nx(), states[n].rho_d.ny()))
        (*accumulations)[n].reset(states[n].rho_d.nx(), states[n].rho_d.ny(), metrics.dx * metrics.dy);
  }
  const auto ld = b200::layout_desc(layout);
  gwm_b200_member_desc mem{};
  mem.moist = 1;
  mem.enable_warm_rain = 1;
  mem.step.dt = config.dt;
  mem.step.fast_substeps = 1;
  mem.rain = b200::rain_config(config);
  b200::Context ctx(metrics, layout, mem);
  b200::GlobalDry g;
  g.gather_from(states, ld);
  const size_t n = states.size();
  const RainIdx ix = rain_indices(tracers.front());
  auto pick = [&](int t) {
    return b200::gather(ld, b200::kCell, n, [&](size_t r) -> const state::Field3D<real>& { return tracers[r].mass(t); });
  };
  std::vector<float> qv = pick(ix.qv), qc = pick(ix.qc), qr = pick(ix.qr);
  const int gnx = metrics.nx, gny = metrics.ny;
  std::vector<double> precip(size_t(gnx) * gny, 0.0);
  const bool fall = accumulations && config.rain_terminal_velocity > 0.0f;
  if (fall)
    for (size_t r = 0; r < n; ++r) {
      const auto& d = layout[r];
      const auto& acc = (*accumulations)[r].liquid_precipitation_kg_m2;
      for (int j = 0; j < d.ny_local(); ++j)
        for (int i = 0; i < d.nx_local(); ++i)
          precip[size_t(d.j_begin + j) * gnx + d.i_begin + i] = acc(i, j, 0);
    }
  auto f = g.fields();
  f.qv = qv.data(); f.qc = qc.data(); f.qr = qr.data(); f.precip = precip.data();
  ctx.ok(gwm_b200_upload(ctx.get(), 0, &f), "upload");
  ctx.ok(gwm_b200_warm_rain(ctx.get(), fall ? 1 : 0), "warm_rain");
  ctx.ok(gwm_b200_download(ctx.get(), 0, &f), "download");
  g.scatter_to(states, ld);
  auto put = [&](int t, const std::vector<float>& q) {
    b200::scatter(ld, b200::kCell, q, n, [&](size_t r) -> state::Field3D<real>& { return tracers[r].mass(t); });
  };
  put(ix.qv, qv); put(ix.qc, qc); put(ix.qr, qr);
  if (fall)
    for (size_t r = 0; r < n; ++r) {
      const auto& d = layout[r];
      auto& acc = (*accumulations)[r].liquid_precipitation_kg_m2;
      for (int j = 0; j < d.ny_local(); ++j)
        for (int i = 0; i < d.nx_local(); ++i) acc(i, j, 0) = float(precip[size_t(d.j_begin + j) * gnx + d.i_begin + i]);
    }
}

}  // namespace gwm::physics
