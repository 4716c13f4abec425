"""gwm-b200: B200-native time-step hot path of the gpu-wm-next weather model.

Python front-end of ``libgwm_b200.so`` (CUDA kernels for sm_100a behind the C-ABI
declared in ``include/gwm_b200.h``).  The object model mirrors the reference's
operator API: a :class:`Model` owns the device state of one or more members and
exposes ``advance_dry_state_ssprk3``, ``advance_passive_tracers_ssprk3``,
``apply_warm_rain_microphysics``, ``compute_slow_tendencies``, the fast-mode
integrator and the budget summaries; module functions expose the halo operators
on the reference's per-rank layout.  Errors raise ``RuntimeError`` with the
library's message, as the reference throws ``std::runtime_error``
(include/gwm/core/types.hpp:24-28).

There is no CPU fallback: every call runs the CUDA library, and importing the
bindings fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field
from typing import Dict, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)
_LIB_PATH = os.path.join(_HERE, "_build", "libgwm_b200.so")
# the reference's gwm_idealized_driver command line over the C-ABI (C++, links the library)
DRIVER_PATH = os.path.join(_HERE, "_build", "gwm_b200_idealized_driver")
_DRIVER_SRC = os.path.join(_HERE, "drivers", "gwm_b200_idealized_driver.cpp")
_SOURCES = ["capi.cu", "dycore.cu", "fast_tma.cu", "fast_terrain_tma.cu", "slow_tma.cu", "slow_terrain_tma.cu",
            "tracer_tma.cu",
            "physics.cu", "halo.cu", "plan_view.cu", "surrogate.cu", "surrogate_rain.cu", "scalar.cu", "cases.cpp"]
_HEADERS = ["common.cuh", "stencil.cuh", "dycore.cuh", "physics.cuh", "halo.cuh", "tma.cuh", "plan_view.cuh", "rain_cell.cuh", "surrogate.cuh", "surrogate_rain.cuh"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]

OK, ERR_ARG, ERR_CUDA, ERR_STATE, ERR_NO_DEVICE, ERR_TIMEOUT = 0, -1, -2, -3, -4, -5
CELL, FACE_X, FACE_Y, FACE_Z = 0, 1, 2, 3


def _stale() -> bool:
    if not os.path.exists(_LIB_PATH):
        return True
    t = os.path.getmtime(_LIB_PATH)
    deps = [os.path.join(_HERE, "csrc", f) for f in _SOURCES + _HEADERS]
    deps += [os.path.join(_ROOT, "include", f) for f in ("gwm_b200.h", "gwm_b200_cases.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the CUDA library in-tree for sm_100a (nvcc cross-compiles without a GPU),
    then the idealized-driver executable that links it."""
    if force or _stale():
        os.makedirs(os.path.dirname(_LIB_PATH), exist_ok=True)
        srcs = [os.path.join(_HERE, "csrc", f) for f in _SOURCES]
        cmd = ["nvcc", *NVCC_FLAGS, "-o", _LIB_PATH + ".tmp", *srcs]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
        os.replace(_LIB_PATH + ".tmp", _LIB_PATH)
    if force or not os.path.exists(DRIVER_PATH) or os.path.getmtime(DRIVER_PATH) < max(
            os.path.getmtime(_LIB_PATH), os.path.getmtime(_DRIVER_SRC)):
        cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-I", os.path.join(_ROOT, "include"), "-o", DRIVER_PATH + ".tmp",
               _DRIVER_SRC, "-L", os.path.dirname(_LIB_PATH), "-lgwm_b200", "-Wl,-rpath,$ORIGIN"]
        subprocess.run(cmd, check=True)
        os.replace(DRIVER_PATH + ".tmp", DRIVER_PATH)
    return _LIB_PATH


# ---------------------------------------------------------------------------
# C structures (include/gwm_b200.h, include/gwm_b200_cases.h)
class _Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("halo", C.c_int),
                ("ranks_x", C.c_int), ("ranks_y", C.c_int), ("periodic_x", C.c_int),
                ("periodic_y", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
                ("z_top", C.c_double), ("terrain_taper_eta", C.c_double),
                ("terrain", C.POINTER(C.c_float)), ("eta_interfaces", C.POINTER(C.c_double))]


class _Step(C.Structure):
    _fields_ = [("dt", C.c_float), ("fast_substeps", C.c_int), ("gravity", C.c_float),
                ("fast_update_horizontal_momentum", C.c_int), ("fast_update_density", C.c_int),
                ("enable_fast_modes", C.c_int)]


class _Rain(C.Structure):
    _fields_ = [("dt", C.c_float), ("condensation_relaxation", C.c_float),
                ("cloud_autoconversion_threshold", C.c_float),
                ("cloud_autoconversion_rate", C.c_float), ("rain_evaporation_rate", C.c_float),
                ("rain_terminal_velocity", C.c_float), ("sedimentation_layer_depth_m", C.c_float),
                ("enable_latent_heating", C.c_int)]


class _Member(C.Structure):
    _fields_ = [("moist", C.c_int), ("enable_tracer_transport", C.c_int),
                ("enable_warm_rain", C.c_int), ("step", _Step), ("rain", _Rain)]


class _ScalarDesc(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("periodic_x", C.c_int),
                ("periodic_y", C.c_int), ("u_adv", C.c_float), ("v_adv", C.c_float), ("dt", C.c_float),
                ("dx", C.c_float), ("dy", C.c_float)]


class _PreparedMeta(C.Structure):
    _fields_ = [("source", C.c_char_p), ("cycle_time_utc", C.c_char_p), ("analysis_valid_time_utc", C.c_char_p),
                ("enable_boundaries", C.c_int), ("surface_ntile", C.c_int), ("surface_nsoil", C.c_int)] + [
                (n, C.c_double) for n in ("max_rel_eos", "max_rel_hydrostatic", "max_rel_fast_vertical",
                                          "max_abs_mass_divergence", "max_rel_mass_divergence",
                                          "max_abs_mom_w_bottom", "max_abs_mom_w_top", "max_abs_tracer_closure")] + [
                ("has_max_abs_z_src_minus_metric", C.c_int), ("max_abs_z_src_minus_metric", C.c_double)]


class _Fields(C.Structure):
    _fields_ = [("rho_d", C.POINTER(C.c_float)), ("rho_theta_m", C.POINTER(C.c_float)),
                ("mom_u", C.POINTER(C.c_float)), ("mom_v", C.POINTER(C.c_float)),
                ("mom_w", C.POINTER(C.c_float)), ("qv", C.POINTER(C.c_float)),
                ("qc", C.POINTER(C.c_float)), ("qr", C.POINTER(C.c_float)),
                ("precip", C.POINTER(C.c_double))]


_BUDGET_KEYS = ("total_dry_mass", "total_rho_theta_m", "total_horizontal_momentum_x",
                "total_horizontal_momentum_y", "total_vertical_momentum", "rho_min", "rho_max",
                "theta_min", "theta_max", "u_min", "u_max", "v_min", "v_max", "w_min", "w_max",
                "vapor_water_path_sum_kg_m2", "cloud_water_path_sum_kg_m2",
                "rain_water_path_sum_kg_m2", "accumulated_surface_precipitation_sum_mm",
                "mean_surface_precipitation_mm", "max_surface_precipitation_mm")


class _Budget(C.Structure):
    _fields_ = [(k, C.c_double) for k in _BUDGET_KEYS]


class _LayoutDesc(C.Structure):
    _fields_ = [(k, C.c_int) for k in ("global_nx", "global_ny", "nz", "halo", "ranks_x",
                                       "ranks_y", "periodic_x", "periodic_y")]


class _CaseParams(C.Structure):
    _fields_ = [(k, C.c_float) for k in (
        "rho_background", "theta_background", "u_background", "v_background", "w_background",
        "center_x_fraction", "center_y_fraction", "center_z_fraction", "radius_x_fraction",
        "radius_y_fraction", "radius_z_fraction", "theta_perturbation", "rho_surface",
        "theta_ref", "p_surface", "theta_lapse_k_per_m", "relative_humidity", "rh_top_m",
        "qv_scale_height_m", "qv_floor", "noise_rms_k", "noise_depth_m", "brunt_vaisala")] + [
        ("seed", C.c_uint64)]


class _MlpTrain(C.Structure):
    _fields_ = [("epochs", C.c_int), ("batch", C.c_int), ("lr", C.c_float), ("seed", C.c_ulonglong),
                ("init", C.c_int)]


class _TerrainParams(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("height", "center_x_fraction", "center_y_fraction",
                                          "half_width_x", "half_width_y")]


_lib = None


def lib():
    """Load libgwm_b200.so (building it first when sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    if _stale():
        build()
    if not os.path.exists(_LIB_PATH):
        raise RuntimeError(f"gwm-b200: CUDA library missing at {_LIB_PATH}; run build()")
    L = C.CDLL(_LIB_PATH)
    vp = C.c_void_p
    L.gwm_b200_create.argtypes = [C.POINTER(_Grid), C.POINTER(_Member), C.c_int, C.POINTER(vp)]
    L.gwm_b200_destroy.argtypes = [vp]
    L.gwm_b200_destroy.restype = None
    L.gwm_b200_last_error.argtypes = [vp]
    L.gwm_b200_last_error.restype = C.c_char_p
    for name in ("gwm_b200_step", "gwm_b200_advance_dry"):
        getattr(L, name).argtypes = [vp, C.c_int]
    L.gwm_b200_warm_rain.argtypes = [vp, C.c_int]
    L.gwm_b200_advance_tracers.argtypes = [vp]
    L.gwm_b200_fast_modes.argtypes = [vp]
    L.gwm_b200_synchronize.argtypes = [vp]
    L.gwm_b200_use_graph.argtypes = [vp, C.c_int]
    L.gwm_b200_set_stream.argtypes = [vp, vp]
    L.gwm_b200_upload.argtypes = [vp, C.c_int, C.POINTER(_Fields)]
    L.gwm_b200_download.argtypes = [vp, C.c_int, C.POINTER(_Fields)]
    L.gwm_b200_step_host.argtypes = [vp, C.POINTER(_Fields), C.POINTER(_Fields)]
    L.gwm_b200_slow_tendencies.argtypes = [vp, C.c_int, C.POINTER(_Fields)]
    L.gwm_b200_budgets.argtypes = [vp, C.c_int, C.POINTER(_Budget)]
    L.gwm_b200_profile.argtypes = [vp, C.c_int]
    L.gwm_b200_set_tile.argtypes = [vp, C.c_int, C.c_int]
    L.gwm_b200_set_boundary_state.argtypes = [vp, C.c_int, C.POINTER(_Fields)]
    L.gwm_b200_set_concurrent.argtypes = [vp, C.c_int]
    L.gwm_b200_apply_reference_boundaries.argtypes = [vp, C.c_int]
    L.gwm_b200_set_damping.argtypes = [vp, C.c_int, C.c_double, C.c_double, C.POINTER(C.c_double),
                                       C.POINTER(C.c_double)]
    L.gwm_b200_rain_record.argtypes = [vp, C.c_int, vp, vp, C.c_longlong, C.c_ulonglong, C.c_float,
                                       C.c_float, C.POINTER(C.c_longlong)]
    L.gwm_b200_mlp_train.argtypes = [vp, vp, C.c_longlong, C.POINTER(_MlpTrain), C.POINTER(C.c_float),
                                     C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_double)]
    L.gwm_b200_mlp_loss_grad.argtypes = [C.POINTER(C.c_float)] * 4 + [C.c_int, C.POINTER(C.c_float),
                                                                      C.POINTER(C.c_double)]
    L.gwm_b200_set_rain_surrogate.argtypes = [vp, C.c_int] + [C.POINTER(C.c_float)] * 3 + [C.c_float, C.c_float]
    L.gwm_b200_surrogate_fallbacks.argtypes = [vp, C.c_int, C.POINTER(C.c_longlong), C.c_int]
    L.gwm_b200_surrogate_stats.argtypes = [vp, C.c_int, C.POINTER(C.c_longlong), C.c_int]
    L.gwm_b200_get_tile.argtypes = [vp, C.c_int]
    L.gwm_b200_profile_read.argtypes = [vp, C.c_int, C.POINTER(C.c_double),
                                        C.POINTER(C.c_longlong), C.POINTER(C.c_char_p)]
    L.gwm_b200_launch_count.argtypes = [vp]
    L.gwm_b200_launch_count.restype = C.c_longlong
    L.gwm_b200_layout.argtypes = [C.POINTER(_LayoutDesc), C.POINTER(C.c_int), C.c_int]
    L.gwm_b200_halo_exchange.argtypes = [C.POINTER(_LayoutDesc), C.c_int, C.c_int,
                                         C.POINTER(C.c_void_p), vp]
    L.gwm_b200_dry_pressure.argtypes = [vp, vp, vp, C.c_longlong, vp]
    L.gwm_b200_test_stall_tile_load.argtypes = [vp, C.c_int, C.c_int]
    L.gwm_b200_set_boundary_cache.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(_Fields)]
    L.gwm_b200_runtime_summary_json.argtypes = [vp, C.c_int, C.c_char_p, C.c_char_p, C.c_longlong,
                                                 C.POINTER(C.c_longlong)]
    L.gwm_b200_phase_summary_json.argtypes = [vp, C.c_int, C.c_int, C.c_float, C.c_char_p, C.c_char_p,
                                              C.c_longlong, C.POINTER(C.c_longlong)]
    L.gwm_b200_prepared_steps.argtypes = [vp, C.c_int, C.POINTER(C.c_float), C.c_char_p, C.c_int, C.c_int,
                                          C.c_int]
    L.gwm_b200_prepared_summary_json.argtypes = [vp, C.c_int, C.POINTER(_PreparedMeta), C.c_int, C.c_char_p,
                                                 C.c_char_p, C.c_longlong, C.POINTER(C.c_longlong)]
    L.gwm_b200_plan_view.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_double, vp, C.c_longlong,
                                     C.POINTER(C.c_int)]
    L.gwm_b200_plan_view_field.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_char_p)]
    L.gwm_b200_plan_view_json.argtypes = [vp, C.c_int, C.c_int, C.c_char_p, C.c_int, C.c_double, C.c_char_p,
                                          C.c_longlong, C.POINTER(C.c_longlong)]
    L.gwm_b200_mlp_infer.argtypes = [C.POINTER(C.c_float), C.POINTER(C.c_float), vp, vp, C.c_longlong, vp]
    L.gwm_b200_set_step_start_time.argtypes = [vp, C.c_int, C.c_float]
    L.gwm_b200_get_step_start_time.argtypes = [vp, C.c_int, C.POINTER(C.c_float)]
    L.gwm_b200_tracer_add.argtypes = [vp, C.c_int, C.c_char_p, C.c_char_p, C.c_int]
    L.gwm_b200_tracer_find.argtypes = [vp, C.c_int, C.c_char_p]
    L.gwm_b200_tracer_count.argtypes = [vp, C.c_int]
    L.gwm_b200_tracer_name.argtypes = [vp, C.c_int, C.c_int]
    L.gwm_b200_tracer_name.restype = C.c_char_p
    L.gwm_b200_tracer_upload.argtypes = [vp, C.c_int, C.c_int, vp]
    L.gwm_b200_tracer_download.argtypes = [vp, C.c_int, C.c_int, vp]
    L.gwm_b200_tracer_total.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.gwm_b200_field_stats_noalloc.argtypes = [vp, C.c_longlong, vp, vp]
    L.gwm_b200_scalar_ssprk3.argtypes = [C.POINTER(_ScalarDesc), vp, C.c_int, vp]
    L.gwm_b200_grid_z_center.argtypes = [C.POINTER(_Grid), vp]
    L.gwm_b200_ranks_to_global.argtypes = [C.POINTER(_LayoutDesc), C.c_int,
                                           C.POINTER(C.c_void_p), vp]
    L.gwm_b200_global_to_ranks.argtypes = [C.POINTER(_LayoutDesc), C.c_int, vp,
                                           C.POINTER(C.c_void_p)]
    L.gwm_b200_build_case.argtypes = [C.c_char_p, C.POINTER(_Grid), C.POINTER(_CaseParams),
                                      C.POINTER(_Fields)]
    L.gwm_b200_build_terrain.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_double,
                                         C.POINTER(_TerrainParams), C.POINTER(C.c_float)]
    _lib = L
    return L


# C-ABI symbols the header declares (checked by the CPU test-suite).
EXPORTED = ("gwm_b200_create", "gwm_b200_destroy", "gwm_b200_last_error", "gwm_b200_set_stream",
            "gwm_b200_synchronize", "gwm_b200_use_graph", "gwm_b200_upload", "gwm_b200_download",
            "gwm_b200_step", "gwm_b200_step_host", "gwm_b200_advance_dry", "gwm_b200_advance_tracers",
            "gwm_b200_warm_rain", "gwm_b200_fast_modes", "gwm_b200_slow_tendencies",
            "gwm_b200_budgets", "gwm_b200_launch_count", "gwm_b200_profile", "gwm_b200_profile_read", "gwm_b200_set_tile", "gwm_b200_get_tile", "gwm_b200_set_boundary_state", "gwm_b200_set_concurrent",
            "gwm_b200_apply_reference_boundaries", "gwm_b200_set_damping", "gwm_b200_rain_record",
            "gwm_b200_mlp_train", "gwm_b200_mlp_loss_grad", "gwm_b200_set_rain_surrogate",
            "gwm_b200_surrogate_fallbacks", "gwm_b200_surrogate_stats", "gwm_b200_layout",
            "gwm_b200_halo_exchange", "gwm_b200_dry_pressure", "gwm_b200_field_stats_noalloc", "gwm_b200_test_stall_tile_load", "gwm_b200_set_boundary_cache", "gwm_b200_runtime_summary_json", "gwm_b200_mlp_infer",
            "gwm_b200_plan_view", "gwm_b200_plan_view_field", "gwm_b200_plan_view_json",
            "gwm_b200_phase_summary_json", "gwm_b200_prepared_steps", "gwm_b200_prepared_summary_json",
            "gwm_b200_set_step_start_time", "gwm_b200_get_step_start_time", "gwm_b200_tracer_add",
            "gwm_b200_tracer_find", "gwm_b200_tracer_count", "gwm_b200_tracer_name", "gwm_b200_tracer_upload",
            "gwm_b200_tracer_download", "gwm_b200_tracer_total", "gwm_b200_scalar_ssprk3", "gwm_b200_grid_z_center", "gwm_b200_ranks_to_global",
            "gwm_b200_global_to_ranks", "gwm_b200_build_case", "gwm_b200_build_terrain")


# ---------------------------------------------------------------------------
@dataclass
class GridSpec:
    """RectilinearDomainConfig / GridMetrics inputs (idealized_domain_builder.hpp:12-31)."""
    nx: int
    ny: int
    nz: int
    dx: float = 1000.0
    dy: float = 1000.0
    z_top: float = 16000.0
    periodic_x: bool = True
    periodic_y: bool = True
    ranks_x: int = 1
    ranks_y: int = 1
    halo: int = 1
    terrain_taper_eta: float = 0.25
    terrain: Optional[np.ndarray] = None
    eta_interfaces: Optional[np.ndarray] = None

    def c(self) -> _Grid:
        g = _Grid(self.nx, self.ny, self.nz, self.halo, self.ranks_x, self.ranks_y,
                  int(self.periodic_x), int(self.periodic_y), self.dx, self.dy, self.z_top,
                  self.terrain_taper_eta, None, None)
        if self.terrain is not None:
            self._t = np.ascontiguousarray(self.terrain, dtype=np.float32)
            assert self._t.shape == (self.ny, self.nx)
            g.terrain = self._t.ctypes.data_as(C.POINTER(C.c_float))
        if self.eta_interfaces is not None:
            self._e = np.ascontiguousarray(self.eta_interfaces, dtype=np.float64)
            assert self._e.shape == (self.nz + 1,)
            g.eta_interfaces = self._e.ctypes.data_as(C.POINTER(C.c_double))
        return g

    def shapes(self) -> Dict[str, tuple]:
        nx, ny, nz = self.nx, self.ny, self.nz
        return {"rho": (nz, ny, nx), "rho_theta": (nz, ny, nx), "u": (nz, ny, nx + 1),
                "v": (nz, ny + 1, nx), "w": (nz + 1, ny, nx), "qv": (nz, ny, nx),
                "qc": (nz, ny, nx), "qr": (nz, ny, nx), "precip": (ny, nx)}


@dataclass
class StepConfig:
    """DryStepperConfig (include/gwm/dycore/dry_core.hpp:50-56)."""
    dt: float = 2.0
    fast_substeps: int = 1
    gravity: float = 9.81
    fast_update_horizontal_momentum: bool = True
    fast_update_density: bool = True
    enable_fast_modes: bool = True

    def c(self) -> _Step:
        return _Step(self.dt, self.fast_substeps, self.gravity,
                     int(self.fast_update_horizontal_momentum), int(self.fast_update_density),
                     int(self.enable_fast_modes))


@dataclass
class WarmRainConfig:
    """WarmRainConfig (include/gwm/physics/warm_rain.hpp:14-23)."""
    dt: float = 2.0
    condensation_relaxation: float = 1.0
    cloud_autoconversion_threshold: float = 1.0e-4
    cloud_autoconversion_rate: float = 1.0e-3
    rain_evaporation_rate: float = 5.0e-3
    rain_terminal_velocity: float = 0.0
    sedimentation_layer_depth_m: float = 0.0
    enable_latent_heating: bool = True

    def c(self) -> _Rain:
        return _Rain(self.dt, self.condensation_relaxation, self.cloud_autoconversion_threshold,
                     self.cloud_autoconversion_rate, self.rain_evaporation_rate,
                     self.rain_terminal_velocity, self.sedimentation_layer_depth_m,
                     int(self.enable_latent_heating))


@dataclass
class MemberSpec:
    step: StepConfig = field(default_factory=StepConfig)
    rain: WarmRainConfig = field(default_factory=WarmRainConfig)
    moist: bool = False
    enable_tracer_transport: bool = True
    enable_warm_rain: bool = True

    def c(self) -> _Member:
        return _Member(int(self.moist), int(self.enable_tracer_transport),
                       int(self.enable_warm_rain), self.step.c(), self.rain.c())


STATE_KEYS = ("rho", "rho_theta", "u", "v", "w")
TRACER_KEYS = ("qv", "qc", "qr")
_C_NAMES = {"rho": "rho_d", "rho_theta": "rho_theta_m", "u": "mom_u", "v": "mom_v",
            "w": "mom_w", "qv": "qv", "qc": "qc", "qr": "qr"}


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Model:
    """Device state of one or more independent members behind ``gwm_b200_ctx``."""

    def __init__(self, grids, members):
        if isinstance(grids, GridSpec):
            grids = [grids]
        if isinstance(members, MemberSpec):
            members = [members]
        if len(grids) != len(members):
            raise ValueError("one MemberSpec per GridSpec")
        self.grids = list(grids)
        self.members = list(members)
        L = lib()
        gs = (_Grid * len(grids))(*[g.c() for g in grids])
        ms = (_Member * len(members))(*[m.c() for m in members])
        h = C.c_void_p()
        rc = L.gwm_b200_create(gs, ms, len(grids), C.byref(h))
        if rc == ERR_NO_DEVICE:
            raise RuntimeError("gwm-b200: no CUDA device visible (the library has no CPU path)")
        if rc != OK:
            raise RuntimeError(f"gwm-b200: create failed with status {rc}")
        self._h = h

    # -- lifetime
    def close(self):
        if getattr(self, "_h", None):
            lib().gwm_b200_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int, what: str):
        if rc != OK:
            msg = lib().gwm_b200_last_error(self._h).decode()
            raise RuntimeError(f"gwm-b200 {what}: status {rc}: {msg}")

    # -- I/O
    def upload(self, state: Dict[str, np.ndarray], member: int = 0):
        g = self.grids[member]
        sh = g.shapes()
        f = _Fields()
        keep = []
        for k, cname in _C_NAMES.items():
            if state.get(k) is not None:
                a = np.ascontiguousarray(state[k], dtype=np.float32)
                if a.shape != sh[k]:
                    raise ValueError(f"{k}: shape {a.shape} != {sh[k]}")
                keep.append(a)
                setattr(f, cname, _fptr(a))
        if state.get("precip") is not None:
            p = np.ascontiguousarray(state["precip"], dtype=np.float64)
            keep.append(p)
            f.precip = p.ctypes.data_as(C.POINTER(C.c_double))
        self._check(lib().gwm_b200_upload(self._h, member, C.byref(f)), "upload")

    def set_boundary_state(self, boundary: Optional[Dict[str, np.ndarray]], member: int = 0):
        """Reference boundary state applied on the open sides at every stage start
        (apply_reference_boundaries); ``None`` removes it (the Null updaters)."""
        if boundary is None:
            self._check(lib().gwm_b200_set_boundary_state(self._h, member, None), "set_boundary_state")
            return
        sh = self.grids[member].shapes()
        f = _Fields()
        keep = []
        for k, cname in _C_NAMES.items():
            if boundary.get(k) is not None:
                a = np.ascontiguousarray(boundary[k], dtype=np.float32)
                if a.shape != sh[k]:
                    raise ValueError(f"{k}: shape {a.shape} != {sh[k]}")
                keep.append(a)
                setattr(f, cname, _fptr(a))
        self._check(lib().gwm_b200_set_boundary_state(self._h, member, C.byref(f)), "set_boundary_state")

    def runtime_summary(self, member: int = 0, indent: str = "  ") -> dict:
        """summarize_runtime_state as the reference's JSON (runtime_state_summary_to_json),
        reduced on the device; returned parsed, with the text under "_json"."""
        import json
        need = C.c_longlong()
        lib().gwm_b200_runtime_summary_json(self._h, member, indent.encode(), None, 0, C.byref(need))
        buf = C.create_string_buffer(int(need.value))
        rc = lib().gwm_b200_runtime_summary_json(self._h, member, indent.encode(), buf, len(buf), None)
        text = buf.value.decode()
        if rc not in (OK, ERR_STATE):
            self._check(rc, "runtime_summary")
        out = json.loads(text.replace("nan", "NaN").replace("inf", "Infinity"))
        out["_json"] = text
        out["_status"] = rc
        return out

    def _text(self, fn, what, *args):
        need = C.c_longlong()
        rc = fn(self._h, *args, None, 0, C.byref(need))
        if rc not in (OK, ERR_STATE):
            self._check(rc, what)
        buf = C.create_string_buffer(int(need.value))
        rc = fn(self._h, *args, buf, len(buf), None)
        if rc not in (OK, ERR_STATE):
            self._check(rc, what)
        return buf.value.decode()

    def phase_summary(self, step: int, step_start_seconds: float, phase: str, member: int = 0) -> str:
        """maybe_write_phase_summary's JSON document for the current state."""
        return self._text(lib().gwm_b200_phase_summary_json, "phase_summary", member, step, step_start_seconds,
                          phase.encode())

    def prepared_steps(self, nsteps: int, sim_time: float = 0.0, phase_summary_dir: Optional[str] = None,
                       step: Optional[int] = None, step_min: Optional[int] = None,
                       step_max: Optional[int] = None) -> float:
        """The prepared-case driver's step loop with its phase summaries; unset arguments
        take GWM_PHASE_SUMMARY_DIR / _STEP / _STEP_MIN / _STEP_MAX from the environment,
        as the driver does.  Returns the start time after the last step."""
        env = os.environ

        def opt(v, name):
            if v is not None:
                return int(v)
            e = env.get(name, "")
            return int(e) if e else -1
        d = phase_summary_dir if phase_summary_dir is not None else env.get("GWM_PHASE_SUMMARY_DIR", "")
        if d:
            os.makedirs(d, exist_ok=True)
        t = C.c_float(sim_time)
        self._check(lib().gwm_b200_prepared_steps(self._h, nsteps, C.byref(t), d.encode() if d else None,
                                                  opt(step, "GWM_PHASE_SUMMARY_STEP"),
                                                  opt(step_min, "GWM_PHASE_SUMMARY_STEP_MIN"),
                                                  opt(step_max, "GWM_PHASE_SUMMARY_STEP_MAX")), "prepared_steps")
        return t.value

    def prepared_summary(self, steps: int, initial_json: str, member: int = 0, **meta) -> str:
        """prepared_summary_json: keyword arguments fill gwm_b200_prepared_meta (strings for
        source / cycle_time_utc / analysis_valid_time_utc, the startup-balance numbers;
        max_abs_z_src_minus_metric given sets its presence flag)."""
        m = _PreparedMeta()
        for k, v in meta.items():
            if k == "max_abs_z_src_minus_metric":
                m.has_max_abs_z_src_minus_metric = 1
            setattr(m, k, v.encode() if isinstance(v, str) else v)
        return self._text(lib().gwm_b200_prepared_summary_json, "prepared_summary", member, C.byref(m), steps,
                          initial_json.encode())

    def plan_view(self, level: int, steps: int = 0, dt: float = 0.0, member: int = 0) -> dict:
        """extract_runtime_plan_view of the current state at ``level``, computed on the
        device: {field name: (ny, nx) float64 array} in the bundle's order, with the units
        under "_units"."""
        nf = C.c_int()
        self._check(lib().gwm_b200_plan_view(self._h, member, level, steps, dt, None, 0, C.byref(nf)), "plan_view")
        g = self.grids[member]
        out = np.empty((nf.value, g.ny, g.nx), np.float64)
        self._check(lib().gwm_b200_plan_view(self._h, member, level, steps, dt, out.ctypes.data_as(C.c_void_p),
                                             out.size, C.byref(nf)),
                    "plan_view")
        res, units = {}, {}
        for q in range(nf.value):
            name, unit = C.c_char_p(), C.c_char_p()
            lib().gwm_b200_plan_view_field(q, C.byref(name), C.byref(unit))
            res[name.value.decode()] = out[q]
            units[name.value.decode()] = unit.value.decode()
        res["_units"] = units
        return res

    def plan_view_json(self, level: int, case_kind: str, steps: int, dt: float, member: int = 0) -> str:
        """The runtime plan-view bundle as plan_view_bundle_to_json writes it."""
        need = C.c_longlong()
        self._check(lib().gwm_b200_plan_view_json(self._h, member, level, case_kind.encode(), steps, dt, None, 0,
                                                  C.byref(need)), "plan_view_json")
        buf = C.create_string_buffer(int(need.value))
        self._check(lib().gwm_b200_plan_view_json(self._h, member, level, case_kind.encode(), steps, dt, buf,
                                                  len(buf), None), "plan_view_json")
        return buf.value.decode()

    def set_boundary_cache(self, offsets, snapshots, member: int = 0):
        """The prepared-case boundary updater: ``snapshots`` are balanced states (dicts of the
        state keys; tracers qv, qc, qr as mixing ratios, kg/kg) at forecast ``offsets``
        (seconds, strictly increasing).  Each updater call applies the strips interpolated at
        the forecast second of the call; the step start time advances by dt per step.  An
        empty list removes the cache."""
        n = len(snapshots)
        if n != len(offsets):
            raise ValueError("one offset per snapshot")
        if n == 0:
            self._check(lib().gwm_b200_set_boundary_cache(self._h, member, 0, None, None), "set_boundary_cache")
            return
        sh = self.grids[member].shapes()
        arr = (_Fields * n)()
        keep = []
        for q, snap in enumerate(snapshots):
            for k, cname in _C_NAMES.items():
                if snap.get(k) is not None:
                    a = np.ascontiguousarray(snap[k], dtype=np.float32)
                    if a.shape != sh[k]:
                        raise ValueError(f"{k}: shape {a.shape} != {sh[k]}")
                    keep.append(a)
                    setattr(arr[q], cname, _fptr(a))
        off = (C.c_int * n)(*[int(t) for t in offsets])
        self._check(lib().gwm_b200_set_boundary_cache(self._h, member, n, off, arr), "set_boundary_cache")

    def set_step_start_time(self, t: float, member: int = 0):
        self._check(lib().gwm_b200_set_step_start_time(self._h, member, float(t)), "set_step_start_time")

    def step_start_time(self, member: int = 0) -> float:
        t = C.c_float()
        self._check(lib().gwm_b200_get_step_start_time(self._h, member, C.byref(t)), "step_start_time")
        return t.value

    def set_damping(self, z_bottom: float, rate: float, u_ref=None, v_ref=None, member: int = 0):
        """Rayleigh damping layer above ``z_bottom`` (extension); rate <= 0 removes it."""
        nz = self.grids[member].nz
        ptrs = []
        for ref in (u_ref, v_ref):
            if ref is None:
                ptrs.append(None)
            else:
                a = np.ascontiguousarray(ref, dtype=np.float64)
                if a.shape != (nz,):
                    raise ValueError(f"reference profile shape {a.shape} != ({nz},)")
                ptrs.append(a)
        args = [p.ctypes.data_as(C.POINTER(C.c_double)) if p is not None else None for p in ptrs]
        self._check(lib().gwm_b200_set_damping(self._h, member, float(z_bottom), float(rate), *args),
                    "set_damping")

    def rain_samples(self, x, y, seed: int = 1, p_active: float = 1.0, p_inactive: float = 0.05,
                     member: int = 0) -> int:
        """Cell samples of the plain warm-rain scheme at the current state into device
        buffers ``x`` (capacity, 7) and ``y`` (capacity, 5) (float32 tensors or device
        pointers); returns the number written."""
        xp, cap = _dev_ptr(x), _rows(x)
        yp = _dev_ptr(y)
        n = C.c_longlong()
        self._check(lib().gwm_b200_rain_record(self._h, member, xp, yp, cap, seed, p_active, p_inactive,
                                               C.byref(n)), "rain_samples")
        return int(n.value)

    def set_rain_surrogate(self, params=None, norm=None, rng=None, tol_water: float = 0.1,
                           tol_energy: float = 0.1, member: int = 0):
        """Warm rain with the trained network (BF16 tensor-core inference of process
        fractions, amounts bounded as in the plain scheme, plain-scheme fallback per cell
        when the inputs leave the training range, a fraction leaves its interval by more
        than ``tol_water``, or the redundant dqv / dtheta outputs disagree with the amounts
        by more than ``tol_water`` / ``tol_energy`` of the exchange plus the output's
        spread); ``params=None`` restores the plain scheme."""
        if params is None:
            self._check(lib().gwm_b200_set_rain_surrogate(self._h, member, None, None, None, 0.0, 0.0),
                        "set_rain_surrogate")
            return
        f = lambda a: np.ascontiguousarray(a, np.float32)
        p, n_, r_ = f(params), f(norm), f(rng)
        ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        self._check(lib().gwm_b200_set_rain_surrogate(self._h, member, ptr(p), ptr(n_), ptr(r_), tol_water,
                                                      tol_energy), "set_rain_surrogate")

    def surrogate_fallbacks(self, reset: bool = False, member: int = 0) -> int:
        n = C.c_longlong()
        self._check(lib().gwm_b200_surrogate_fallbacks(self._h, member, C.byref(n), int(reset)),
                    "surrogate_fallbacks")
        return int(n.value)

    def surrogate_stats(self, reset: bool = False, member: int = 0) -> dict:
        """Cumulative counters of the network warm rain: cells that fell back, cells the
        network ran on, and per check the cells that failed it."""
        st = (C.c_longlong * 6)()
        self._check(lib().gwm_b200_surrogate_stats(self._h, member, st, int(reset)), "surrogate_stats")
        keys = ("fallbacks", "network_cells", "out_of_range", "fraction", "water", "energy")
        return dict(zip(keys, (int(v) for v in st)))

    # -- tracer registry (TracerRegistry / TracerState)
    def add_tracer(self, name: str, units: str = "kg/kg", positive: bool = True, member: int = 0) -> int:
        """TracerRegistry::add: registers a passive tracer (mass rho*q, starting at zero)
        that every step transports; returns its index."""
        rc = lib().gwm_b200_tracer_add(self._h, member, name.encode(), units.encode(), int(positive))
        if rc < 0:
            self._check(rc, "add_tracer")
        return rc

    def find_tracer(self, name: str, member: int = 0) -> Optional[int]:
        """TracerRegistry::find: the tracer's index, or None."""
        rc = lib().gwm_b200_tracer_find(self._h, member, name.encode())
        return rc if rc >= 0 else None

    def tracer_names(self, member: int = 0) -> list:
        n = lib().gwm_b200_tracer_count(self._h, member)
        return [lib().gwm_b200_tracer_name(self._h, member, i).decode() for i in range(max(n, 0))]

    def _tracer_index(self, tracer, member):
        if isinstance(tracer, str):
            i = self.find_tracer(tracer, member)
            if i is None:
                raise KeyError(f"Tracer not found in TracerState: {tracer}")
            return i
        return int(tracer)

    def upload_tracer(self, tracer, mass: np.ndarray, member: int = 0):
        """TracerState::mass(tracer) from a host array (nz, ny, nx) of rho*q."""
        g = self.grids[member]
        a = np.ascontiguousarray(mass, dtype=np.float32)
        if a.shape != (g.nz, g.ny, g.nx):
            raise ValueError(f"tracer field shape {a.shape}, expected {(g.nz, g.ny, g.nx)}")
        self._check(lib().gwm_b200_tracer_upload(self._h, member, self._tracer_index(tracer, member),
                                                 a.ctypes.data), "upload_tracer")

    def download_tracer(self, tracer, member: int = 0) -> np.ndarray:
        g = self.grids[member]
        out = np.empty((g.nz, g.ny, g.nx), dtype=np.float32)
        self._check(lib().gwm_b200_tracer_download(self._h, member, self._tracer_index(tracer, member),
                                                   out.ctypes.data), "download_tracer")
        return out

    def tracer_total(self, tracer, member: int = 0) -> float:
        """TracerState::total_mass: FP64 sum of rho*q over the owned cells."""
        t = C.c_double()
        self._check(lib().gwm_b200_tracer_total(self._h, member, self._tracer_index(tracer, member),
                                                C.byref(t)), "tracer_total")
        return t.value

    def test_stall_tile_load(self, plane: int, member: int = 0):
        """Failure-path testing: the next TMA-fed stencil launch leaves one CTA's tile
        loads of ``plane`` unissued, so its bounded wait runs out (the step call then
        fails with GWM_B200_ERR_TIMEOUT)."""
        self._check(lib().gwm_b200_test_stall_tile_load(self._h, member, plane), "test_stall_tile_load")

    def apply_reference_boundaries(self, member: int = 0):
        """apply_reference_boundaries once on the current state."""
        self._check(lib().gwm_b200_apply_reference_boundaries(self._h, member), "apply_reference_boundaries")

    def download(self, member: int = 0, keys: Optional[Sequence[str]] = None,
                 out: Optional[Dict[str, np.ndarray]] = None) -> Dict[str, np.ndarray]:
        """Copy the state to host arrays (new ones, or the given ``out`` arrays)."""
        g = self.grids[member]
        sh = g.shapes()
        moist = self.members[member].moist
        if keys is None:
            keys = list(out) if out else STATE_KEYS + ((TRACER_KEYS + ("precip",)) if moist else ())
        out = {} if out is None else out
        f = _Fields()
        for k in keys:
            dtype = np.float64 if k == "precip" else np.float32
            if k not in out:
                out[k] = np.zeros(sh[k], dtype=dtype)
            a = out[k]
            if a.shape != sh[k] or a.dtype != dtype or not a.flags["C_CONTIGUOUS"]:
                raise ValueError(f"download target {k} must be a C-contiguous {dtype} array of {sh[k]}")
            if k == "precip":
                f.precip = a.ctypes.data_as(C.POINTER(C.c_double))
            else:
                setattr(f, _C_NAMES[k], _fptr(a))
        self._check(lib().gwm_b200_download(self._h, member, C.byref(f)), "download")
        return out

    # -- operators
    def step(self, nsteps: int = 1):
        """The prepared-case driver loop (gwm_prepared_case_driver.cpp:427-463)."""
        self._check(lib().gwm_b200_step(self._h, nsteps), "step")

    def step_host(self, state: Dict[str, np.ndarray], out: Optional[Dict[str, np.ndarray]] = None
                  ) -> Dict[str, np.ndarray]:
        """One step from host arrays to host arrays (single-member models): the full state
        in, one ``step``, the full state out, with the copies overlapping the step's phases.
        ``out`` may be ``state`` itself; pinned (page-locked) arrays copy at full PCIe rate."""
        if len(self.grids) != 1:
            raise ValueError("step_host takes a single-member model")
        g = self.grids[0]
        sh = g.shapes()
        keys = STATE_KEYS + ((TRACER_KEYS + ("precip",)) if self.members[0].moist else ())
        out = {} if out is None else out
        fin, fout, keep = _Fields(), _Fields(), []
        for k in keys:
            dtype = np.float64 if k == "precip" else np.float32
            if k not in state:
                raise ValueError(f"step_host needs {k}")
            a = np.ascontiguousarray(state[k], dtype=dtype)
            if a.shape != sh[k]:
                raise ValueError(f"{k}: shape {a.shape} != {sh[k]}")
            keep.append(a)
            if k not in out:
                out[k] = np.empty(sh[k], dtype=dtype)
            o = out[k]
            if o.shape != sh[k] or o.dtype != dtype or not o.flags["C_CONTIGUOUS"]:
                raise ValueError(f"step_host target {k} must be a C-contiguous {dtype} array of {sh[k]}")
            if k == "precip":
                fin.precip = a.ctypes.data_as(C.POINTER(C.c_double))
                fout.precip = o.ctypes.data_as(C.POINTER(C.c_double))
            else:
                setattr(fin, _C_NAMES[k], _fptr(a))
                setattr(fout, _C_NAMES[k], _fptr(o))
        self._check(lib().gwm_b200_step_host(self._h, C.byref(fin), C.byref(fout)), "step_host")
        return out

    def advance_dry_state_ssprk3(self, nsteps: int = 1):
        self._check(lib().gwm_b200_advance_dry(self._h, nsteps), "advance_dry_state_ssprk3")

    def advance_passive_tracers_ssprk3(self):
        self._check(lib().gwm_b200_advance_tracers(self._h), "advance_passive_tracers_ssprk3")

    def apply_warm_rain_microphysics(self, fallout: Optional[str] = "metric"):
        mode = {None: 0, "none": 0, "metric": 1, "nominal": 2}[fallout]
        self._check(lib().gwm_b200_warm_rain(self._h, mode), "apply_warm_rain_microphysics")

    def fast_modes(self):
        """LocalSplitExplicitFastMode::apply on the current state."""
        self._check(lib().gwm_b200_fast_modes(self._h), "fast_modes")

    def compute_slow_tendencies(self, member: int = 0) -> Dict[str, np.ndarray]:
        sh = self.grids[member].shapes()
        out = {k: np.zeros(sh[k], dtype=np.float32) for k in STATE_KEYS}
        f = _Fields()
        for k in STATE_KEYS:
            setattr(f, _C_NAMES[k], _fptr(out[k]))
        self._check(lib().gwm_b200_slow_tendencies(self._h, member, C.byref(f)),
                    "compute_slow_tendencies")
        return out

    def budgets(self, member: int = 0) -> Dict[str, float]:
        b = _Budget()
        self._check(lib().gwm_b200_budgets(self._h, member, C.byref(b)), "budgets")
        return {k: getattr(b, k) for k in _BUDGET_KEYS}

    def use_graph(self, enable: bool = True):
        self._check(lib().gwm_b200_use_graph(self._h, int(enable)), "use_graph")

    def set_stream(self, stream_handle: Optional[int]):
        self._check(lib().gwm_b200_set_stream(self._h, stream_handle), "set_stream")

    def synchronize(self):
        self._check(lib().gwm_b200_synchronize(self._h), "synchronize")

    @property
    def launch_count(self) -> int:
        return int(lib().gwm_b200_launch_count(self._h))

    _TILE_KERNELS = {"slow_stage": 0, "fast_substep": 1, "tracer_stage": 2}

    def set_tile(self, kernel: str, rows: int):
        """CTA tile rows of a kernel: "slow_stage" 3 (owned tiles fed by TMA, flat terrain
        and terrain), 8 or 16; "tracer_stage" 3 (owned tiles fed by TMA, flat terrain and
        terrain), 8 or 16;
        "fast_substep" 0 (owned flat tiles), 3 (owned tiles fed by TMA, flat terrain and
        terrain), 4 (the same, all substeps of a flat RK stage in one persistent launch),
        8 or 16 (overlapped tiles)."""
        self._check(lib().gwm_b200_set_tile(self._h, self._TILE_KERNELS[kernel], rows), "set_tile")

    def get_tile(self, kernel: str) -> int:
        r = lib().gwm_b200_get_tile(self._h, self._TILE_KERNELS[kernel])
        if r < 0:
            raise ValueError(kernel)
        return r

    def autotune(self, steps: int = 1, whole_step: bool = False) -> Dict[str, int]:
        """Pick the fastest tile of each stencil kernel by timing real steps.

        Every tiling computes the same values, so the tuning steps are ordinary
        model steps: the state advances by ``steps`` per candidate (10 candidates
        per pass; one more step each with ``whole_step``).  Re-upload the initial state
        afterwards to start from it.  Returns the chosen rows per kernel.

        By default each candidate is timed per kernel launch with the profiling events,
        which run the members one after another; an acoustic substep on terrain is
        charged the column reference kernel that precedes it.  ``whole_step`` times
        whole steps instead, replayed from the captured graph with the members running
        side by side as they do in a timed run (the right measure for an ensemble of small
        members, whose kernels share the GPU); it leaves graph replay on."""
        import time
        candidates = {"slow_stage": (3, 8, 16), "fast_substep": (0, 3, 8, 16), "tracer_stage": (3, 8, 16)}
        kinds = {"slow_stage": ("k_slow_stage",), "fast_substep": ("k_fast_substep", "k_column_reference"),
                 "tracer_stage": ("k_tracer_stage",)}
        best = {k: self.get_tile(k) for k in candidates}
        self.tile_times = {}
        if whole_step:
            self.use_graph(True)
        for kernel, rows_list in candidates.items():
            times = {}
            self.tile_times[kernel] = times
            for rows in rows_list:
                self.set_tile(kernel, rows)
                if whole_step:
                    self.step(1)            # captures the step graph of this tiling
                    self.synchronize()
                    t0 = time.perf_counter()
                    self.step(steps)
                    self.synchronize()
                    times[rows] = (time.perf_counter() - t0) * 1e3 / steps
                    continue
                self.profile(True)
                self.step(steps)
                rep = self.profile_report()
                self.profile(False)
                main = rep.get(kinds[kernel][0])
                if main:
                    times[rows] = sum(rep[k]["total_ms"] for k in kinds[kernel] if k in rep) / main["launches"]
            if times:
                best[kernel] = min(times, key=times.get)
            self.set_tile(kernel, best[kernel])
        return best

    def set_concurrent(self, enable: bool = True):
        """Members advance concurrently on their own streams (one graph branch each)."""
        self._check(lib().gwm_b200_set_concurrent(self._h, int(enable)), "set_concurrent")

    def profile(self, enable: bool = True):
        """Per-kernel CUDA-event timing of subsequent direct (non-graph) launches."""
        self._check(lib().gwm_b200_profile(self._h, int(enable)), "profile")

    def profile_report(self) -> Dict[str, Dict[str, float]]:
        rep = {}
        n = lib().gwm_b200_profile_read(self._h, 0, None, None, None)
        for kind in range(n):
            ms, cnt, name = C.c_double(), C.c_longlong(), C.c_char_p()
            lib().gwm_b200_profile_read(self._h, kind, C.byref(ms), C.byref(cnt), C.byref(name))
            if cnt.value:
                rep[name.value.decode()] = {"total_ms": ms.value, "launches": cnt.value,
                                            "avg_ms": ms.value / cnt.value}
        return rep


# ---------------------------------------------------------------------------
def _layout_desc(nx, ny, nz, halo, rx, ry, px, py) -> _LayoutDesc:
    return _LayoutDesc(nx, ny, nz, halo, rx, ry, int(px), int(py))


def layout(nx, ny, nz, halo=1, ranks_x=1, ranks_y=1, periodic_x=True, periodic_y=True) -> np.ndarray:
    """VirtualRankLayout::build + neighbours: rows of 12 ints per rank."""
    d = _layout_desc(nx, ny, nz, halo, ranks_x, ranks_y, periodic_x, periodic_y)
    out = np.zeros(12 * ranks_x * ranks_y, dtype=np.int32)
    n = lib().gwm_b200_layout(C.byref(d), out.ctypes.data_as(C.POINTER(C.c_int)), ranks_x * ranks_y)
    if n < 0:
        raise RuntimeError(f"layout: status {n}")
    return out.reshape(n, 12)


def halo_exchange(rank_ptrs: Sequence[int], nx, ny, nz, halo, ranks_x, ranks_y, periodic_x,
                  periodic_y, orientation: int, op: str = "exchange", stream: Optional[int] = None):
    """HaloExchange::exchange_* / synchronize_owned_face_interfaces on device buffers."""
    d = _layout_desc(nx, ny, nz, halo, ranks_x, ranks_y, periodic_x, periodic_y)
    arr = (C.c_void_p * len(rank_ptrs))(*rank_ptrs)
    rc = lib().gwm_b200_halo_exchange(C.byref(d), orientation, 0 if op == "exchange" else 1, arr,
                                      stream)
    if rc != OK:
        raise RuntimeError(f"halo_exchange: status {rc}")


def dry_pressure(rho_ptr: int, rho_theta_ptr: int, p_ptr: int, n: int, stream: Optional[int] = None):
    rc = lib().gwm_b200_dry_pressure(rho_ptr, rho_theta_ptr, p_ptr, n, stream)
    if rc != OK:
        raise RuntimeError(f"dry_pressure: status {rc}")


def grid_z_center(grid: "GridSpec") -> np.ndarray:
    """Cell-centre heights of a grid (GridMetrics::z_center, grid_metrics.hpp:87-239: FP64
    compute, FP32 result), shape (nz, ny, nx); host code, no device needed."""
    out = np.empty((grid.nz, grid.ny, grid.nx), dtype=np.float32)
    gc = grid.c()
    rc = lib().gwm_b200_grid_z_center(C.byref(gc), out.ctypes.data_as(C.c_void_p))
    if rc != OK:
        raise RuntimeError(f"grid_z_center: status {rc}")
    return out


def scalar_ssprk3(q, u_adv: float = 20.0, v_adv: float = 0.0, dt: float = 10.0, dx: float = 1000.0,
                  dy: float = 1000.0, periodic_x: bool = True, periodic_y: bool = True, nsteps: int = 1):
    """nsteps of advance_scalar_ssprk3 (dry_transport.cu:285-325) on the GPU.

    q: (nz, ny, nx) float32, a contiguous torch CUDA tensor (advanced in place and
    returned) or an array (copied to the device and back; the result is returned).
    Defaults are DryTransportConfig's (dry_transport.hpp:11-17)."""
    import torch
    on_device = isinstance(q, torch.Tensor)
    t = q if on_device else torch.from_numpy(np.ascontiguousarray(q, dtype=np.float32)).cuda()
    if t.dtype != torch.float32 or not t.is_cuda or not t.is_contiguous() or t.dim() != 3:
        raise ValueError("scalar_ssprk3: q must be a contiguous (nz, ny, nx) float32 CUDA tensor")
    nz, ny, nx = t.shape
    d = _ScalarDesc(nx, ny, nz, int(periodic_x), int(periodic_y), u_adv, v_adv, dt, dx, dy)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib().gwm_b200_scalar_ssprk3(C.byref(d), t.data_ptr(), nsteps, stream)
    if rc != OK:
        raise RuntimeError(f"scalar_ssprk3: status {rc}")
    return t if on_device else t.cpu().numpy()


def field_stats_noalloc(x_ptr: int, n: int, out_ptr: int, stream: Optional[int] = None):
    """FP64 {sum, min, max} of n device floats into 3 device doubles, allocating nothing.

    For callers that cannot allocate device memory at the call site (their own memory
    pool owns the device, or cudaMalloc's implicit synchronisation is not allowed
    there).  The scratch is a fixed 24 KiB device array inside the library; concurrent
    calls that can overlap on the GPU race.  Make the first call on a device before
    any stream capture (it resolves the array's device address)."""
    rc = lib().gwm_b200_field_stats_noalloc(x_ptr, n, out_ptr, stream)
    if rc != OK:
        raise RuntimeError(f"field_stats_noalloc: status {rc}")


def ranks_to_global(rank_arrays: Sequence[np.ndarray], nx, ny, nz, halo, ranks_x, ranks_y,
                    periodic_x, periodic_y, orientation: int) -> np.ndarray:
    d = _layout_desc(nx, ny, nz, halo, ranks_x, ranks_y, periodic_x, periodic_y)
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in rank_arrays]
    shp = (nz + (orientation == 3), ny + (orientation == 2), nx + (orientation == 1))
    out = np.zeros(shp, dtype=np.float32)
    ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    rc = lib().gwm_b200_ranks_to_global(C.byref(d), orientation, ptrs, out.ctypes.data)
    if rc != OK:
        raise RuntimeError(f"ranks_to_global: status {rc}")
    return out


def global_to_ranks(glob: np.ndarray, rank_arrays: Sequence[np.ndarray], nx, ny, nz, halo,
                    ranks_x, ranks_y, periodic_x, periodic_y, orientation: int):
    d = _layout_desc(nx, ny, nz, halo, ranks_x, ranks_y, periodic_x, periodic_y)
    g = np.ascontiguousarray(glob, dtype=np.float32)
    for a in rank_arrays:
        assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    ptrs = (C.c_void_p * len(rank_arrays))(*[a.ctypes.data for a in rank_arrays])
    rc = lib().gwm_b200_global_to_ranks(C.byref(d), orientation, g.ctypes.data, ptrs)
    if rc != OK:
        raise RuntimeError(f"global_to_ranks: status {rc}")


@dataclass
class CaseParams:
    """ThermoBubbleConfig + MountainWaveBackgroundConfig + moist sounding parameters."""
    rho_background: float = 1.0
    theta_background: float = 300.0
    u_background: float = 0.0
    v_background: float = 0.0
    w_background: float = 0.0
    center_x_fraction: float = 0.5
    center_y_fraction: float = 0.5
    center_z_fraction: float = 0.5
    radius_x_fraction: float = 0.1
    radius_y_fraction: float = 0.1
    radius_z_fraction: float = 0.1
    theta_perturbation: float = 2.0
    rho_surface: float = 1.18
    theta_ref: float = 300.0
    p_surface: float = 100000.0
    theta_lapse_k_per_m: float = 0.004
    relative_humidity: float = 0.9
    rh_top_m: float = 2000.0
    qv_scale_height_m: float = 1500.0
    qv_floor: float = 1.0e-5
    noise_rms_k: float = 0.0
    noise_depth_m: float = 1000.0
    brunt_vaisala: float = 0.01
    seed: int = 0

    def c(self) -> _CaseParams:
        vals = [getattr(self, n) for n, _ in _CaseParams._fields_]
        return _CaseParams(*vals)


def build_case(kind: str, grid: GridSpec, params: CaseParams, moist: bool = False) -> Dict[str, np.ndarray]:
    """Initial state in the field I/O layout (C++ case builders of the library)."""
    sh = grid.shapes()
    keys = STATE_KEYS + ((TRACER_KEYS + ("precip",)) if moist else ())
    out = {k: np.zeros(sh[k], dtype=np.float64 if k == "precip" else np.float32) for k in keys}
    f = _Fields()
    for k in keys:
        if k == "precip":
            f.precip = out[k].ctypes.data_as(C.POINTER(C.c_double))
        else:
            setattr(f, _C_NAMES[k], _fptr(out[k]))
    gc, pc = grid.c(), params.c()
    rc = lib().gwm_b200_build_case(kind.encode(), C.byref(gc), C.byref(pc), C.byref(f))
    if rc != OK:
        raise RuntimeError(f"build_case({kind}): status {rc}")
    return out


def build_terrain(kind: str, nx: int, ny: int, dx: float, dy: float, height: float = 0.0,
                  center_x_fraction: float = 0.5, center_y_fraction: float = 0.5,
                  half_width_x: float = 0.15, half_width_y: float = 0.15) -> np.ndarray:
    out = np.zeros((ny, nx), dtype=np.float32)
    p = _TerrainParams(height, center_x_fraction, center_y_fraction, half_width_x, half_width_y)
    rc = lib().gwm_b200_build_terrain(kind.encode(), nx, ny, dx, dy, C.byref(p), _fptr(out))
    if rc != OK:
        raise RuntimeError(f"build_terrain({kind}): status {rc}")
    return out


# ---------------------------------------------------------------------------
# Learned warm-rain microphysics: training side
MLP_PARAMS = 64 * 7 + 64 + 2 * (64 * 64 + 64) + 5 * 64 + 5
MLP_NORM = 24


def _dev_ptr(t):
    """Device pointer of a CUDA tensor (or an int pointer)."""
    return t if isinstance(t, int) else t.data_ptr()


def _rows(t):
    return t.shape[0]


def mlp_train(x, y, n: int, epochs: int = 10, batch: int = 65536, lr: float = 1e-3, seed: int = 1,
              params: Optional[np.ndarray] = None):
    """Train the 7-64-64-64-5 network on ``n`` device samples with the library's own
    forward/backward kernels and Adam.  Returns (params, norm, input range, loss per epoch)."""
    p = np.zeros(MLP_PARAMS, np.float32) if params is None else np.array(params, np.float32)
    norm = np.zeros(MLP_NORM, np.float32)
    rng = np.zeros(14, np.float32)
    loss = np.zeros(epochs, np.float64)
    cfg = _MlpTrain(epochs, batch, lr, seed, 1 if params is None else 0)
    f32 = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    rc = lib().gwm_b200_mlp_train(_dev_ptr(x), _dev_ptr(y), n, C.byref(cfg), f32(p), f32(norm), f32(rng),
                                  loss.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != OK:
        raise RuntimeError(f"mlp_train: status {rc}")
    return p, norm, rng, loss


def mlp_infer(params, norm, x_ptr: int, y_ptr: int, n: int, stream: Optional[int] = None):
    """The network through the warm-rain surrogate's tensor-core inference on n device
    feature rows (x: n x 7 float32 at x_ptr) into y (n x 5 float32 at y_ptr), outputs
    de-normalised; params and norm are host arrays."""
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    p, nm = f32(params), f32(norm)
    rc = lib().gwm_b200_mlp_infer(_fptr(p), _fptr(nm), x_ptr, y_ptr, int(n), stream)
    if rc != OK:
        raise RuntimeError(f"mlp_infer: status {rc}")


def mlp_loss_grad(params, norm, x, y):
    """Loss and gradient of the network on host samples (the GPU kernels of training)."""
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    p, nm, xx, yy = f32(params), f32(norm), f32(x), f32(y)
    g = np.zeros(MLP_PARAMS, np.float32)
    loss = C.c_double()
    ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    rc = lib().gwm_b200_mlp_loss_grad(ptr(p), ptr(nm), ptr(xx), ptr(yy), xx.shape[0], ptr(g), C.byref(loss))
    if rc != OK:
        raise RuntimeError(f"mlp_loss_grad: status {rc}")
    return loss.value, g
