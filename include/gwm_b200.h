/* gwm_b200.h — C-ABI of the B200 time-step hot path (libgwm_b200.so).
 *
 * Drop-in boundary for the dry SSPRK3 + split-explicit step, passive-tracer
 * transport, warm-rain microphysics with fallout, C-grid halo fill and the
 * budget reductions of FahrenheitResearch/gpu-wm-next.  Plain C types only:
 * host pointers for field I/O, device pointers where stated, and an opaque
 * context that owns all device buffers of one or more independent members.
 *
 * Field I/O layout ("global owned arrays", x fastest, float32):
 *   cells       (nz,   ny,   nx)      rho_d, rho_theta_m, tracer masses rho*q
 *   X faces     (nz,   ny,   nx+1)    mom_u
 *   Y faces     (nz,   ny+1, nx)      mom_v
 *   Z faces     (nz+1, ny,   nx)      mom_w
 *   surface     (ny,   nx)            accumulated precipitation, float64
 * These are the owned parts of the reference's Field3D / FaceField storage
 * (include/gwm/state/field3d.hpp:49-54, face_field.hpp:16-23) gathered onto
 * the global grid as VirtualRankLayout::gather_scalar / gather_face do
 * (src/comm/virtual_rank_layout.cpp:73-137).  gwm_b200_ranks_to_global and
 * gwm_b200_global_to_ranks convert per-rank halo-padded buffers.
 *
 * Every call returns GWM_B200_OK (0) or a negative status; no C++ exception
 * crosses the boundary (the reference throws std::runtime_error from
 * gwm::require, include/gwm/core/types.hpp:24-28).  Calls are synchronous
 * unless a stream was set with gwm_b200_set_stream.
 */
#ifndef GWM_B200_H
#define GWM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define GWM_B200_OK 0
#define GWM_B200_ERR_ARG (-1)          /* invalid argument / unsupported shape */
#define GWM_B200_ERR_CUDA (-2)         /* CUDA runtime error; see gwm_b200_last_error */
#define GWM_B200_ERR_STATE (-3)        /* non-finite or non-positive density detected */
#define GWM_B200_ERR_NO_DEVICE (-4)    /* no CUDA device visible */
#define GWM_B200_ERR_TIMEOUT (-5)      /* a bounded device wait gave up; the step's result is invalid */

typedef struct gwm_b200_ctx gwm_b200_ctx;

/* Grid of one member.  Mirrors RectilinearDomainConfig + GridMetrics::make_hybrid_height
 * (include/gwm/domain/idealized_domain_builder.hpp:12-31, grid_metrics.hpp:87-92). */
typedef struct {
  int nx, ny, nz;              /* global owned cells */
  int halo;                    /* must be 1 (every reference stencil reaches one cell) */
  int ranks_x, ranks_y;        /* virtual-rank layout of per-rank host buffers */
  int periodic_x, periodic_y;  /* else open boundaries: halos read zero */
  double dx, dy, z_top;
  double terrain_taper_eta;    /* reference default 0.25 */
  const float* terrain;        /* (ny, nx) terrain height in m, NULL = flat */
  const double* eta_interfaces;/* (nz+1) eta levels, NULL = uniform k/nz (extension) */
} gwm_b200_grid_desc;

/* DryStepperConfig (include/gwm/dycore/dry_core.hpp:50-56) plus the fast-mode switch
 * of the prepared-case driver (src/core/gwm_prepared_case_driver.cpp:37-41). */
typedef struct {
  float dt;
  int fast_substeps;
  float gravity;
  int fast_update_horizontal_momentum;
  int fast_update_density;
  int enable_fast_modes;
} gwm_b200_step_config;

/* WarmRainConfig (include/gwm/physics/warm_rain.hpp:14-23). */
typedef struct {
  float dt;
  float condensation_relaxation;
  float cloud_autoconversion_threshold;
  float cloud_autoconversion_rate;
  float rain_evaporation_rate;
  float rain_terminal_velocity;
  float sedimentation_layer_depth_m;
  int enable_latent_heating;
} gwm_b200_warm_rain_config;

/* One member: the dry state, and for moist members the warm-rain registry
 * (specific_humidity, cloud_water_mixing_ratio, rain_water_mixing_ratio;
 * include/gwm/state/tracer_registry.hpp:18-23,56-62) and surface precipitation. */
typedef struct {
  int moist;
  int enable_tracer_transport;
  int enable_warm_rain;
  gwm_b200_step_config step;
  gwm_b200_warm_rain_config rain;
} gwm_b200_member_desc;

/* Host field set for upload / download; NULL members are skipped. */
typedef struct {
  float* rho_d;
  float* rho_theta_m;
  float* mom_u;
  float* mom_v;
  float* mom_w;
  float* qv;     /* rho_d * specific_humidity */
  float* qc;     /* rho_d * cloud water */
  float* qr;     /* rho_d * rain water */
  double* precip;/* accumulated surface precipitation, kg m-2 */
} gwm_b200_fields;

/* summarize_dry_states (src/dycore/dry_diagnostics.cpp:11-96) and the moisture part
 * of summarize_runtime_state / summarize_warm_rain (src/core/runtime_summary.cpp:27-178,
 * src/physics/warm_rain.cpp:355-403), reduced on the device in FP64. */
typedef struct {
  double total_dry_mass, total_rho_theta_m;
  double total_horizontal_momentum_x, total_horizontal_momentum_y, total_vertical_momentum;
  double rho_min, rho_max, theta_min, theta_max;
  double u_min, u_max, v_min, v_max, w_min, w_max;
  double vapor_water_path_sum_kg_m2, cloud_water_path_sum_kg_m2, rain_water_path_sum_kg_m2;
  double accumulated_surface_precipitation_sum_mm, mean_surface_precipitation_mm,
      max_surface_precipitation_mm;
} gwm_b200_budget;

/* ---- context ------------------------------------------------------------ */
/* Allocates device buffers for n_members independent members (grids[i], members[i]),
 * builds the hybrid-height metrics (FP64 compute, FP32 store: grid_metrics.hpp:87-239). */
int gwm_b200_create(const gwm_b200_grid_desc* grids, const gwm_b200_member_desc* members,
                    int n_members, gwm_b200_ctx** out);
void gwm_b200_destroy(gwm_b200_ctx* ctx);
const char* gwm_b200_last_error(const gwm_b200_ctx* ctx);
/* cudaStream_t passed as void*; NULL restores the context's own stream. */
int gwm_b200_set_stream(gwm_b200_ctx* ctx, void* stream);
int gwm_b200_synchronize(gwm_b200_ctx* ctx);
/* Replay multi-step calls from a captured CUDA graph (1) or launch directly (0). */
int gwm_b200_use_graph(gwm_b200_ctx* ctx, int enable);

/* ---- state I/O ------------------------------------------------------------ */
int gwm_b200_upload(gwm_b200_ctx* ctx, int member, const gwm_b200_fields* host);
int gwm_b200_download(gwm_b200_ctx* ctx, int member, gwm_b200_fields* host);

/* ---- time step -------------------------------------------------------------- */
/* nsteps of the prepared-case driver loop (gwm_prepared_case_driver.cpp:427-463):
 * dry SSPRK3 step, then (moist members) tracer transport and warm rain. */
int gwm_b200_step(gwm_b200_ctx* ctx, int nsteps);
/* One step of a single-member context from host buffers to host buffers: every field of
 * the state (and the precipitation of a moist member) copied in from `in`, one
 * gwm_b200_step, every field copied out to `out` (`in` and `out` may be the same
 * buffers).  The copies overlap the step on two copy streams: the moisture fields go up
 * during the dry step, rho and the momenta come down during the tracers and warm rain.
 * The result equals gwm_b200_upload + gwm_b200_step(1) + gwm_b200_download.  Pinned host
 * memory gives full PCIe bandwidth.  Returns after the outputs are in `out`.  The first call
 * allocates one device staging buffer per field (together about the state's owned size,
 * 2.2 GB at 1024 x 1024 x 64) and two copy streams, kept until gwm_b200_destroy. */
int gwm_b200_step_host(gwm_b200_ctx* ctx, const gwm_b200_fields* in, gwm_b200_fields* out);
/* advance_dry_state_ssprk3 with NullBoundaryUpdater and LocalSplitExplicitFastMode
 * (include/gwm/dycore/dry_core.hpp:106-110, src/dycore/dry_core.cu:541-651). */
int gwm_b200_advance_dry(gwm_b200_ctx* ctx, int nsteps);
/* advance_passive_tracers_ssprk3 with NullTracerBoundaryUpdater
 * (include/gwm/dycore/passive_tracer.hpp:44-49, src/dycore/dry_transport.cu:440-518). */
int gwm_b200_advance_tracers(gwm_b200_ctx* ctx);
/* apply_warm_rain_microphysics: fallout 1 = metric overload (warm_rain.hpp:63-68,
 * warm_rain.cu:273-353), 2 = nominal-depth overload (:57-61, :214-271), 0 = none. */
int gwm_b200_warm_rain(gwm_b200_ctx* ctx, int fallout);
/* FastModeIntegrator::apply of LocalSplitExplicitFastMode on the current state
 * (dry_core.hpp:73-88, dry_core.cu:341-346, dry_fast_modes.cu:400-656). */
int gwm_b200_fast_modes(gwm_b200_ctx* ctx);
/* compute_slow_tendencies of the current state (dry_core.hpp:100-104, dry_core.cu:400-539);
 * the five tendency fields are written to host arrays in the field I/O layout
 * (rho_theta_m receives the rho*theta tendency). */
int gwm_b200_slow_tendencies(gwm_b200_ctx* ctx, int member, gwm_b200_fields* host_out);
/* Reference boundary state of a member (host arrays in the field I/O layout; tracers
 * optional, used when the member is moist).  While set, every step applies
 * apply_reference_boundaries (src/dycore/boundary_conditions.cpp:111-208) on the open
 * sides at the reference's BoundaryUpdater points: the dry stage starts
 * (dry_core.cu:568, 591, 620) and the tracer stage inputs (dry_transport.cu:259-276, called at 489-508),
 * leaving the SSPRK3 blend partner q0 as it was before the first application.  The
 * strips are kept on the device (perimeter x nz floats per field); aliased periodic
 * faces of the boundary state are averaged as on upload.  NULL removes it (the Null
 * updaters).  Periodic sides are never touched. */
int gwm_b200_set_boundary_state(gwm_b200_ctx* ctx, int member, const gwm_b200_fields* boundary);
/* PreparedCaseBoundaryUpdater + PreparedCaseTracerBoundaryUpdater
 * (src/ingest/prepared_case_init.cpp:396-645,1006-1078) on the device, for open sides.
 * snapshots[q] (host arrays, field I/O layout) is the balanced state of boundary-cache
 * entry q at forecast offset offsets[q] seconds (strictly increasing): rho_d,
 * rho_theta_m and the three momenta, and for moist members the tracer MIXING RATIOS
 * (kg/kg) in qv, qc, qr (all three, or none).  Only the outermost strips are kept (per
 * snapshot: perimeter x nz floats per field).  At every updater call of a step (the dry
 * stage starts, dry_core.cu:568, 591, 620, and the tracer stage inputs,
 * dry_transport.cu:488-508, at sim_time 0, dt and dt/2) the strips applied are those of
 * the cache interpolated at the forecast second lround(step_start + sim_time): the
 * bracketing entries of BoundaryCacheIR::bracket (include/gwm/ingest/boundary_cache.hpp:
 * 52-76) weighted as interpolate_boundary_snapshot (src/ingest/runtime_case.cpp:205-228),
 * tracers as rho_d * q (prepared_case_init.cpp:570-645).  The reference interpolates the
 * raw analysis fields and rebalances them on the host (hydrostatic columns, SOR face
 * projection: ingest code); here the caller supplies each entry already balanced and the
 * device interpolates the balanced strips.  The step start time starts at 0 and every
 * step advances it by dt on the device (float, as the driver's sim_time += dt), also
 * inside a replayed CUDA graph.  n = 0 removes the cache (the Null updaters); setting a
 * fixed boundary state (gwm_b200_set_boundary_state) replaces it. */
int gwm_b200_set_boundary_cache(gwm_b200_ctx* ctx, int member, int n, const int* offsets,
                                const gwm_b200_fields* snapshots);
/* PreparedCaseBoundaryUpdater::set_step_start_time (max(t, 0)) / the current value. */
int gwm_b200_set_step_start_time(gwm_b200_ctx* ctx, int member, float t);
int gwm_b200_get_step_start_time(gwm_b200_ctx* ctx, int member, float* t);
/* Rayleigh damping layer (an extension: the reference has none).  Above z_bottom the
 * slow tendencies gain -tau(z) (u - u_ref(k)), -tau(z) (v - v_ref(k)) and -tau(z) w,
 * with tau(z) = rate * sin^2(pi/2 (z - z_bottom)/(z_top - z_bottom)) at each level's
 * terrain-free height eta * z_top, on the faces whose tendency the reference computes.
 * u_ref, v_ref: nz momenta per level (NULL: 0).  rate <= 0 removes the layer. */
int gwm_b200_set_damping(gwm_b200_ctx* ctx, int member, double z_bottom, double rate,
                         const double* u_ref, const double* v_ref);
/* apply_reference_boundaries once on the current state (dry fields and, when set, tracers). */
int gwm_b200_apply_reference_boundaries(gwm_b200_ctx* ctx, int member);
/* ---- tracer registry ----------------------------------------------------------
 * TracerRegistry / TracerState of a member (include/gwm/state/tracer_registry.hpp:23-49,
 * tracer_state.hpp:12-119).  A moist member starts with make_warm_rain_registry
 * (tracer_registry.hpp:56-62): specific_humidity, cloud_water_mixing_ratio and
 * rain_water_mixing_ratio at indices 0-2 (the qv, qc, qr of gwm_b200_fields); a dry member
 * starts empty.  Every registered tracer's mass rho*q is carried by
 * advance_passive_tracers_ssprk3 in each step (dry_transport.cu:440-518); warm rain acts
 * on indices 0-2 only, and the reference boundary state (gwm_b200_set_boundary_state)
 * covers those three.
 * TracerRegistry::add: a new name (duplicates are rejected, as the reference requires);
 * returns the tracer's index (>= 0) or a negative status.  Its mass starts at zero. */
int gwm_b200_tracer_add(gwm_b200_ctx* ctx, int member, const char* name, const char* units, int positive);
/* TracerRegistry::find: the index of name, or GWM_B200_ERR_ARG when it is not registered. */
int gwm_b200_tracer_find(const gwm_b200_ctx* ctx, int member, const char* name);
/* TracerRegistry::size (or a negative status). */
int gwm_b200_tracer_count(const gwm_b200_ctx* ctx, int member);
/* TracerRegistry::at(index).name, or NULL for an index out of range. */
const char* gwm_b200_tracer_name(const gwm_b200_ctx* ctx, int member, int index);
/* TracerState::mass(index) in and out: host array (nz, ny, nx) of rho*q, float32. */
int gwm_b200_tracer_upload(gwm_b200_ctx* ctx, int member, int index, const float* host);
int gwm_b200_tracer_download(gwm_b200_ctx* ctx, int member, int index, float* host);
/* TracerState::total_mass: FP64 sum of rho*q over the owned cells (Field3D::owned_sum). */
int gwm_b200_tracer_total(gwm_b200_ctx* ctx, int member, int index, double* total);
/* ---- learned warm-rain microphysics (training side) ----
 * Cell samples of the plain scheme at the member's current state (no state change):
 * x (capacity x 7, device) = (T, p, rho_d, qv, qc, qr, dt), y (capacity x 5, device) =
 * (f_cond, f_auto, f_evap, dtheta, dqv): condensation as a fraction of the saturation
 * deficit |qv - qs|, autoconversion as a fraction of the cloud water above the
 * threshold, rain evaporation as a fraction of the rain present (each the scheme's
 * nominal value where its bound is zero), and the step's theta and vapour changes.
 * Cells with a non-zero tendency are kept with probability p_active, the others with
 * p_inactive (seeded hash of the cell index); *n_out = samples written. */
int gwm_b200_rain_record(gwm_b200_ctx* ctx, int member, float* x, float* y, long long capacity,
                         unsigned long long seed, float p_active, float p_inactive, long long* n_out);
typedef struct {
  int epochs, batch;
  float lr;                 /* Adam learning rate */
  unsigned long long seed;  /* initialisation and shuffling */
  int init;                 /* 1: initialise params (Xavier uniform), 0: start from params */
} gwm_b200_mlp_train_config;
/* Trains the 7-64-64-64-5 GELU network on n device samples (x, y as above) with the
 * project's FP32 forward/backward kernels and Adam; params (host, 9157 floats) in/out,
 * norm (host, 24 floats) out: input mean/std (std 1 for a constant input), target
 * mean/std (std 0 for a constant target: it is reproduced exactly); range (host, 14 floats,
 * may be NULL) out: input min/max; loss_per_epoch (host, epochs) out: mean squared
 * error of the normalised targets. */
int gwm_b200_mlp_train(const float* x, const float* y, long long n, const gwm_b200_mlp_train_config* cfg,
                       float* params, float* norm, float* range, double* loss_per_epoch);
/* The trained network evaluated by the warm-rain surrogate's tensor-core inference (BF16
 * operands, FP32 accumulation in tensor memory, GELU in FP32) on n feature rows: x (n x 7,
 * device) -> y (n x 5, device), de-normalised outputs (f_cond, f_auto, f_evap, dtheta,
 * dqv) before any check.  params (9157) and norm (24) are host arrays as for
 * gwm_b200_set_rain_surrogate.  For validating the inference (no counterpart in the
 * reference, which has no learned part).  Returns when done. */
int gwm_b200_mlp_infer(const float* params, const float* norm, const float* x, float* y, long long n, void* stream);
/* Warm rain of a member with the trained network (params 9157, norm 24, range 14
 * floats, host) instead of the plain per-cell microphysics; NULL params restores the
 * plain scheme.  The network gives condensation, autoconversion and rain evaporation as
 * fractions of their bounds (saturation deficit, cloud water above the threshold, rain
 * present) plus dtheta and dqv; the amounts move water between vapour, cloud and rain,
 * so water and energy close by construction (qv -= c - e, qc += c - a, qr += a - e,
 * theta += L/(cp pi)(c - e)).  Quiet cells (no cloud or rain water, not supersaturated),
 * which the plain scheme leaves unchanged, are left unchanged without the network.  A
 * cell takes the plain scheme when its inputs leave the training range, a raw fraction
 * leaves its interval by more than tol_water, |dqv_net - (e - c)| > tol_water (|c| + |e|
 * + dqv spread) or |dtheta_net - L/(cp pi)(c - e)| > tol_energy (L/(cp pi)|c - e| +
 * dtheta spread), the spreads being the training targets' standard deviations. */
int gwm_b200_set_rain_surrogate(gwm_b200_ctx* ctx, int member, const float* params, const float* norm,
                                const float* range, float tol_water, float tol_energy);
/* Cumulative surrogate counters (reset != 0 clears them): stats[0] cells that fell back
 * to the plain scheme, [1] cells the network ran on, [2..5] cells failing the input
 * range, fraction range, water and energy checks (a cell can fail several). */
#define GWM_B200_SURROGATE_STATS 6
int gwm_b200_surrogate_stats(gwm_b200_ctx* ctx, int member, long long* stats, int reset);
/* stats[0] alone. */
int gwm_b200_surrogate_fallbacks(gwm_b200_ctx* ctx, int member, long long* count, int reset);
/* Loss and gradient of the network on n host samples (gradient check). */
int gwm_b200_mlp_loss_grad(const float* params, const float* norm, const float* x, const float* y, int n,
                           float* grad, double* loss);
/* Failure-path testing (no counterpart in the reference): the next TMA-fed stencil
 * launch of the member (slow stage, acoustic substep or tracer stage on flat terrain)
 * leaves the tile loads of `plane` unissued in one CTA, so that CTA's bounded wait runs
 * out; the step call then returns GWM_B200_ERR_TIMEOUT and the context stays usable.
 * The request is kept until a TMA-fed kernel takes it. */
int gwm_b200_test_stall_tile_load(gwm_b200_ctx* ctx, int member, int plane);
/* FP64 budgets of the current state. */
int gwm_b200_budgets(gwm_b200_ctx* ctx, int member, gwm_b200_budget* out);
/* summarize_runtime_state + runtime_state_summary_to_json (src/core/runtime_summary.cpp:
 * 27-247): the dry summary, every registered tracer's column integral sum(rho q dz) and
 * mixing-ratio range (rho q / max(rho, 1e-12)), and the moisture budget (water paths of the
 * warm-rain tracers, surface precipitation sum, mean, maximum and precipitating cells),
 * reduced in FP64 on the device over the member's global fields (the reference's
 * per-rank sums for a one-rank layout), written as the reference's JSON (17 digits) with
 * `indent` (NULL: two spaces) into buf (cap bytes, NUL-terminated).  *len (may be NULL)
 * receives the bytes needed.  A state with a non-finite or non-positive density is
 * written and reported as GWM_B200_ERR_STATE. */
int gwm_b200_runtime_summary_json(gwm_b200_ctx* ctx, int member, const char* indent, char* buf, long long cap,
                                  long long* len);
/* The phase summary of maybe_write_phase_summary (src/core/gwm_prepared_case_driver.cpp:
 * 97-131): step, step start time, phase name and the runtime summary (indent "    ") of
 * the member's current state; buf/cap/len as gwm_b200_runtime_summary_json. */
int gwm_b200_phase_summary_json(gwm_b200_ctx* ctx, int member, int step, float step_start_seconds,
                                const char* phase, char* buf, long long cap, long long* len);
/* nsteps of the prepared-case driver's step loop (gwm_prepared_case_driver.cpp:427-463)
 * over every member, with its phase summaries.  A step whose summaries are not wanted is
 * gwm_b200_step (one CUDA graph when graphs are on).  When phase_summary_dir is non-empty
 * and the step is selected (step == only_step when only_step >= 0, else step_min <= step
 * <= step_max, a negative bound being absent: the GWM_PHASE_SUMMARY_STEP/_MIN/_MAX rules
 * of :71-88), the step runs as its three phases (dry step; tracer transport; warm rain,
 * the same kernels in the same order, so the state is the same bit for bit) and after
 * each phase step_<n>_<phase>.json is written into the directory (which must exist) for
 * member 0, step_<n>_<phase>_member<m>.json for member m > 0.  *sim_time (may be NULL:
 * 0) is the first step's start time and receives the time after the last step; it
 * advances by member 0's dt in FP32, as the driver's sim_time does. */
int gwm_b200_prepared_steps(gwm_b200_ctx* ctx, int nsteps, float* sim_time, const char* phase_summary_dir,
                            int only_step, int step_min, int step_max);
/* What the prepared-case summary reports beyond the member's own configuration: the
 * analysis' identity, the boundary switch, the surface runtime's extents and the startup
 * balance diagnostics (ingest and the surface layer stay with the caller). */
typedef struct {
  const char* source;                   /* to_string(analysis.source), e.g. "HRRR" */
  const char* cycle_time_utc;
  const char* analysis_valid_time_utc;
  int enable_boundaries;
  int surface_ntile, surface_nsoil;
  double max_rel_eos, max_rel_hydrostatic, max_rel_fast_vertical, max_abs_mass_divergence,
      max_rel_mass_divergence, max_abs_mom_w_bottom, max_abs_mom_w_top, max_abs_tracer_closure;
  int has_max_abs_z_src_minus_metric;
  double max_abs_z_src_minus_metric;
} gwm_b200_prepared_meta;
/* prepared_summary_json (gwm_prepared_case_driver.cpp:252-350) after `steps` steps: the
 * member's step and warm-rain configuration and grid, meta, the caller's initial runtime
 * summary (initial_json, as gwm_b200_runtime_summary_json wrote it with indent "    ")
 * and the final summary of the member's current state. */
int gwm_b200_prepared_summary_json(gwm_b200_ctx* ctx, int member, const gwm_b200_prepared_meta* meta, int steps,
                                   const char* initial_json, char* buf, long long cap, long long* len);
/* Runtime plan view of a member's current state at level `level` (clamped to [0, nz-1]),
 * computed on the device: extract_runtime_plan_view (src/io/plan_view_output.cpp:715-834)
 * over extract_dry_plan_view (:630-713), with the reference's FP32 diagnostics and FP64
 * column integrals.  The field list follows the member's tracers as the reference's
 * branches do: without tracers the dry bundle's 10 fields; with a specific_humidity
 * tracer + specific humidity, relative humidity and dewpoint (13; any other tracer state
 * without it is GWM_B200_ERR_ARG, as the reference's require is); with the cloud and rain
 * water tracers too + their mixing ratios, total condensate, the column cloud, rain and
 * total condensate, the column rain fraction and the synthetic reflectivity (21); for a
 * moist member + the accumulated surface precipitation and its mean rate over steps * dt
 * (23).  out (host, may be NULL): *nfields x ny x nx doubles, row-major (y, x); cap is the
 * number of doubles out holds.  gwm_b200_plan_view_field names field n (0-based, the
 * bundle's order) and gives its units. */
int gwm_b200_plan_view(gwm_b200_ctx* ctx, int member, int level, int steps, double dt, double* out, long long cap,
                       int* nfields);
int gwm_b200_plan_view_field(int field, const char** name, const char** units);
/* The same bundle as plan_view_bundle_to_json writes it (plan_view_output.cpp:950-1003),
 * with case_kind, steps and dt as the bundle's metadata; buf/cap/len as
 * gwm_b200_runtime_summary_json. */
int gwm_b200_plan_view_json(gwm_b200_ctx* ctx, int member, int level, const char* case_kind, int steps, double dt,
                            char* buf, long long cap, long long* len);
/* Tile shape of a kernel.  kernel 0 = slow stage: rows 3 = owned 32x16 tiles fed by
 * TMA tile loads (flat terrain and terrain; the stand-alone slow tendencies use 16),
 * 8 or 16 = overlapped 32-wide tiles (default 16).  kernel 2 = tracer stage: rows 3 =
 * owned 32x16 tiles fed by TMA (flat terrain and terrain), 8 or 16 (overlapped,
 * default 16).  kernel 1 = acoustic substep: rows 0 = owned 32x16 tiles
 * (flat terrain; terrain falls back to 8), 3 = owned 32x16 tiles fed by TMA tile loads
 * (flat terrain and terrain), 4 = the same tiles with all the substeps of an RK stage in
 * one persistent cooperative launch (a bounded grid barrier between substeps; the
 * step's last substep keeps its own launch; terrain runs one launch per substep), 8 or
 * 16 = overlapped 32-wide tiles of that many rows.  The environment variable GWM_B200_FAST_TILE_ROWS sets the
 * acoustic default at context creation.  The choice changes speed only: every tiling
 * computes the same values.  gwm_b200_get_tile returns the current rows (or < 0). */
int gwm_b200_set_tile(gwm_b200_ctx* ctx, int kernel, int rows);
int gwm_b200_get_tile(const gwm_b200_ctx* ctx, int kernel);
/* Members of a context advance concurrently (default 1): each on its own stream,
 * forked from and joined back to the context stream, so a captured step is one graph
 * with a branch per member; 0 runs them one after another on the context stream.
 * Either way every member's result is the same bit for bit. */
int gwm_b200_set_concurrent(gwm_b200_ctx* ctx, int enable);
/* Kernel launches issued by the last step call (for accounting). */
long long gwm_b200_launch_count(const gwm_b200_ctx* ctx);
/* Per-kernel CUDA-event timing on the context's stream (no graph while enabled).
 * Enabling resets the accumulators; gwm_b200_profile_read returns the number of
 * kernel kinds and, for kind, the accumulated device time, launch count and name. */
int gwm_b200_profile(gwm_b200_ctx* ctx, int enable);
int gwm_b200_profile_read(const gwm_b200_ctx* ctx, int kind, double* total_ms,
                          long long* launches, const char** name);

/* ---- halo operators on the reference per-rank layout (device pointers) ---- */
/* Field orientation: 0 cell, 1 X face, 2 Y face, 3 Z face. */
typedef struct {
  int global_nx, global_ny, nz, halo, ranks_x, ranks_y, periodic_x, periodic_y;
} gwm_b200_layout_desc;
/* VirtualRankLayout::build + find_cartesian_neighbors (virtual_rank_layout.cpp:7-47,
 * cartesian_topology.cpp:57-74): 12 ints per rank {rank, coord_x, coord_y, i_begin,
 * i_end, j_begin, j_end, west, east, south, north, nz}.  Returns the rank count. */
int gwm_b200_layout(const gwm_b200_layout_desc* d, int* out, int capacity);
/* op 0: HaloExchange::exchange_scalar / exchange_face (halo_exchange.cpp:563-637);
 * op 1: synchronize_owned_face_interfaces (:639-654).  rank_fields[r] is rank r's
 * Field3D storage on the device (halo-padded, reference layout). */
int gwm_b200_halo_exchange(const gwm_b200_layout_desc* d, int orientation, int op,
                           float* const* rank_fields, void* stream);
/* compute_dry_pressure_fields on n device values (dry_pressure_gradient.cu:177-202). */
int gwm_b200_dry_pressure(const float* rho_d, const float* rho_theta_m, float* pressure,
                          long long n, void* stream);

/* Allocation-free FP64 statistics of n device floats: out (3 doubles, device memory)
 * receives {sum, minimum, maximum}, reduced in a fixed order (bitwise reproducible).
 * No counterpart in the reference.  For callers that must not allocate device memory
 * at the point of the call: code that owns every device allocation through its own
 * pool, code running where cudaMalloc would synchronise the device or is not allowed,
 * and callers without a gwm_b200_ctx.  The scratch is a fixed 24 KiB array inside the
 * library (1024 blocks of partials), held on every device that loads the library until
 * process exit; n must lie in [1, 2^31-1].  The first call on a device resolves that
 * array's device address, so make it before any stream capture on that device; after
 * the device's context is re-created (cudaDeviceReset), the next call resolves it
 * again, and the same applies to that call.  A CUDA error already pending from other
 * code is left in place and the call returns GWM_B200_ERR_CUDA without launching.  All
 * calls share the array: calls that can overlap on the GPU (different streams, or
 * threads without ordering) race and must be serialised by the caller. */
int gwm_b200_field_stats_noalloc(const float* x, long long n, double* out, void* stream);

/* ---- scalar transport -------------------------------------------------------- */
/* DryTransportConfig (include/gwm/dycore/dry_transport.hpp:11-17) with the grid of the
 * advected field. */
typedef struct {
  int nx, ny, nz;
  int periodic_x, periodic_y;  /* else zero beyond the open side, as the halo exchange gives */
  float u_adv, v_adv, dt, dx, dy;
} gwm_b200_scalar_desc;
/* nsteps of advance_scalar_ssprk3 (include/gwm/dycore/dry_transport.hpp:19-21,
 * src/dycore/dry_transport.cu:285-325) on q, a device array (nz, ny, nx) in the global
 * owned layout, in place; the arithmetic is the reference's, so results match it bit
 * for bit.  Two scratch copies of q are taken from the stream-ordered allocator for the
 * call.  stream: cudaStream_t as void* (NULL: the default stream); returns when done. */
int gwm_b200_scalar_ssprk3(const gwm_b200_scalar_desc* desc, float* q, int nsteps, void* stream);

/* ---- host layout helpers (no device work) --------------------------------- */
/* Cell-centre heights GridMetrics::z_center (include/gwm/domain/grid_metrics.hpp:87-239:
 * FP64 compute, FP32 result) of a grid into out (nz, ny, nx), host memory. */
int gwm_b200_grid_z_center(const gwm_b200_grid_desc* grid, float* out);
/* Per-rank halo-padded host buffers <-> global owned arrays.  Faces shared by two
 * ranks (and periodic aliases) take the average of both copies on the way in, as the
 * reference's first interface sync does. */
int gwm_b200_ranks_to_global(const gwm_b200_layout_desc* d, int orientation,
                             const float* const* rank_fields, float* global);
int gwm_b200_global_to_ranks(const gwm_b200_layout_desc* d, int orientation,
                             const float* global, float* const* rank_fields);

#ifdef __cplusplus
}
#endif

#endif /* GWM_B200_H */
