/* gwm_b200_cases.h — host-side case setup of libgwm_b200.so (initial states and
 * terrain, C++ run once per case).  Replaces the reference's idealized initialisers
 * (src/dycore/idealized_cases.cpp:105-223, src/dycore/dry_core.cu:363-398) and the
 * cosine-mountain terrain of src/domain/idealized_domain_builder.cpp:14-35, and adds
 * the synthetic soundings of the benchmark configurations. */
#ifndef GWM_B200_CASES_H
#define GWM_B200_CASES_H

#include <stdint.h>

#include "gwm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ThermoBubbleConfig + MountainWaveBackgroundConfig
 * (include/gwm/dycore/idealized_cases.hpp:12-37) + the moist sounding. */
typedef struct {
  float rho_background, theta_background, u_background, v_background, w_background;
  float center_x_fraction, center_y_fraction, center_z_fraction;
  float radius_x_fraction, radius_y_fraction, radius_z_fraction, theta_perturbation;
  float rho_surface, theta_ref;
  /* moist_sounding */
  float p_surface;            /* Pa at z = 0 */
  float theta_lapse_k_per_m;  /* above 1 km */
  float relative_humidity;    /* below rh_top_m */
  float rh_top_m;
  float qv_scale_height_m;
  float qv_floor;
  float noise_rms_k;          /* Gaussian theta noise below noise_depth_m */
  float noise_depth_m;
  /* stratified_mountain_wave: Brunt-Vaisala frequency N (1/s) of the background */
  float brunt_vaisala;
  uint64_t seed;
} gwm_b200_case_params;

typedef struct {
  double height;
  double center_x_fraction, center_y_fraction;
  double half_width_x, half_width_y; /* cosine_mountain: fraction of the domain; agnesi: metres */
} gwm_b200_terrain_params;

/* kind: "constant", "warm_bubble", "density_current", "hydrostatic_rest",
 * "mountain_wave_background", "hydrostatic_warm_bubble", "moist_sounding",
 * "stratified_mountain_wave" (an extension: constant-N background
 * theta = theta_ref exp(N^2 z / g) in hydrostatic balance from p_surface, with the
 * mountain-wave face momenta of u_background, v_background).
 * Fills host arrays in the field I/O layout of gwm_b200.h (NULL members skipped;
 * rho_d and rho_theta_m required). */
int gwm_b200_build_case(const char* kind, const gwm_b200_grid_desc* grid,
                        const gwm_b200_case_params* params, gwm_b200_fields* out);
/* kind: "flat", "cosine_mountain", "agnesi"; out is (ny, nx). */
int gwm_b200_build_terrain(const char* kind, int nx, int ny, double dx, double dy,
                           const gwm_b200_terrain_params* params, float* out);

#ifdef __cplusplus
}
#endif

#endif /* GWM_B200_CASES_H */
