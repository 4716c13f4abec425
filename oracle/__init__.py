"""CPU ORACLE — test infrastructure only.

ctypes front-end of ``oracle/_build/liboracle.so`` (built from ``gwm_oracle.hpp``
by ``oracle/Makefile``), a C++ restatement of the reference's time-step hot path
in FP32 and FP64.  Only the tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module, and only as the checker or
the timed CPU baseline; the product never links or calls it.

Field arrays are numpy float64 arrays in global owned layout:
cells (nz, ny, nx), X faces (nz, ny, nx+1), Y faces (nz, ny+1, nx),
Z faces (nz+1, ny, nx), surface precipitation (ny, nx).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

DP = C.POINTER(C.c_double)


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("halo", C.c_int),
                ("ranks_x", C.c_int), ("ranks_y", C.c_int), ("periodic_x", C.c_int),
                ("periodic_y", C.c_int), ("dx", C.c_double), ("dy", C.c_double),
                ("z_top", C.c_double), ("terrain_taper_eta", C.c_double),
                ("terrain", DP), ("eta_interfaces", DP)]


class Step(C.Structure):
    _fields_ = [("dt", C.c_double), ("fast_substeps", C.c_int), ("gravity", C.c_double),
                ("fast_hmom", C.c_int), ("fast_density", C.c_int), ("fast_modes", C.c_int),
                ("damp_z_bottom", C.c_double), ("damp_rate", C.c_double),
                ("damp_u_ref", C.POINTER(C.c_double)), ("damp_v_ref", C.POINTER(C.c_double))]


class Rain(C.Structure):
    _fields_ = [("dt", C.c_double), ("condensation_relaxation", C.c_double),
                ("autoconv_threshold", C.c_double), ("autoconv_rate", C.c_double),
                ("rain_evap_rate", C.c_double), ("terminal_velocity", C.c_double),
                ("layer_depth", C.c_double), ("latent_heating", C.c_int)]


class Fields(C.Structure):
    _fields_ = [("rho", DP), ("rho_theta", DP), ("u", DP), ("v", DP), ("w", DP),
                ("qv", DP), ("qc", DP), ("qr", DP), ("precip", DP)]


class CaseParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "rho_background", "theta_background", "u_background", "v_background", "w_background",
        "center_x_fraction", "center_y_fraction", "center_z_fraction",
        "radius_x_fraction", "radius_y_fraction", "radius_z_fraction", "theta_perturbation",
        "rho_surface", "theta_ref")]


class Sounding(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "p_surface", "theta_ref", "theta_lapse_k_per_m", "relative_humidity", "rh_top_m",
        "qv_scale_height_m", "qv_floor", "noise_rms_k", "noise_depth_m")] + [("seed", C.c_ulonglong)]


def build() -> str:
    """Compile the oracle library (gcc, OpenMP) if it is missing or stale."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.gwo_last_error.restype = C.c_char_p
        L.gwo_max_threads.restype = C.c_int
        L.gwo_run.argtypes = [C.POINTER(Grid), C.POINTER(Step), C.POINTER(Rain), C.c_int, C.c_int,
                              C.c_int, C.POINTER(Fields)]
        L.gwo_run_boundary.argtypes = [C.POINTER(Grid), C.POINTER(Step), C.POINTER(Rain), C.c_int,
                                       C.c_int, C.c_int, C.POINTER(Fields), C.POINTER(Fields)]
        L.gwo_run_boundary_cache.argtypes = [C.POINTER(Grid), C.POINTER(Step), C.POINTER(Rain), C.c_int,
                                             C.c_int, C.c_int, C.POINTER(Fields), C.c_int,
                                             C.POINTER(C.c_int), C.POINTER(Fields), C.c_double]
        L.gwo_mlp_loss_grad.argtypes = [DP, DP, DP, DP, C.c_int, DP, DP]
        L.gwo_slow_tendencies.argtypes = [C.POINTER(Grid), C.POINTER(Step), C.c_int,
                                          C.POINTER(Fields), C.POINTER(Fields)]
        L.gwo_fast_modes.argtypes = [C.POINTER(Grid), C.POINTER(Step), C.c_int, C.POINTER(Fields)]
        L.gwo_metrics.argtypes = [C.POINTER(Grid), C.c_int, DP, DP, DP, DP]
        L.gwo_case.argtypes = [C.c_int, C.POINTER(Grid), C.POINTER(CaseParams), C.c_int,
                               C.POINTER(Fields)]
        L.gwo_moist_sounding.argtypes = [C.POINTER(Grid), C.POINTER(Sounding), C.POINTER(Fields)]
        L.gwo_pressure.argtypes = [C.c_long, DP, DP, DP, C.c_int]
        L.gwo_plan_view.argtypes = [C.POINTER(Grid), C.c_int, C.c_int, C.c_int, C.c_double] + [DP] * 10
        L.gwo_scalar_ssprk3.argtypes = [C.c_int] * 5 + [C.c_double] * 5 + [C.c_int, C.c_int, DP]
        L.gwo_layout.argtypes = [C.c_int] * 8 + [C.POINTER(C.c_int)]
        L.gwo_halo.argtypes = [C.c_int] * 10 + [C.POINTER(DP)]
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc < 0:
        raise RuntimeError("oracle: " + lib().gwo_last_error().decode())


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(DP)


@dataclass
class GridSpec:
    nx: int
    ny: int
    nz: int
    dx: float = 1000.0
    dy: float = 1000.0
    z_top: float = 16000.0
    ranks_x: int = 1
    ranks_y: int = 1
    periodic_x: bool = True
    periodic_y: bool = True
    halo: int = 1
    terrain_taper_eta: float = 0.25
    terrain: Optional[np.ndarray] = None          # (ny, nx) metres
    eta_interfaces: Optional[np.ndarray] = None   # (nz+1,)

    def c(self) -> Grid:
        g = Grid(self.nx, self.ny, self.nz, self.halo, self.ranks_x, self.ranks_y,
                 int(self.periodic_x), int(self.periodic_y), self.dx, self.dy, self.z_top,
                 self.terrain_taper_eta, None, None)
        if self.terrain is not None:
            self._t = np.ascontiguousarray(self.terrain, dtype=np.float64)
            g.terrain = _ptr(self._t)
        if self.eta_interfaces is not None:
            self._e = np.ascontiguousarray(self.eta_interfaces, dtype=np.float64)
            g.eta_interfaces = _ptr(self._e)
        return g


@dataclass
class StepSpec:
    dt: float = 2.0
    fast_substeps: int = 1
    gravity: float = 9.81
    fast_hmom: bool = True
    fast_density: bool = True
    fast_modes: bool = True
    damp_z_bottom: float = 0.0        # Rayleigh damping layer (extension): bottom height (m)
    damp_rate: float = 0.0            # maximum rate (1/s); <= 0: off
    damp_u_ref: Optional[np.ndarray] = None  # (nz,) momentum profiles the layer relaxes to
    damp_v_ref: Optional[np.ndarray] = None

    def c(self) -> Step:
        st = Step(self.dt, self.fast_substeps, self.gravity, int(self.fast_hmom),
                  int(self.fast_density), int(self.fast_modes), self.damp_z_bottom, self.damp_rate,
                  None, None)
        if self.damp_u_ref is not None:
            self._u = np.ascontiguousarray(self.damp_u_ref, dtype=np.float64)
            st.damp_u_ref = _ptr(self._u)
        if self.damp_v_ref is not None:
            self._v = np.ascontiguousarray(self.damp_v_ref, dtype=np.float64)
            st.damp_v_ref = _ptr(self._v)
        return st


@dataclass
class RainSpec:
    dt: float = 2.0
    condensation_relaxation: float = 1.0
    autoconv_threshold: float = 1.0e-4
    autoconv_rate: float = 1.0e-3
    rain_evap_rate: float = 5.0e-3
    terminal_velocity: float = 0.0
    layer_depth: float = 0.0
    latent_heating: bool = True

    def c(self) -> Rain:
        return Rain(self.dt, self.condensation_relaxation, self.autoconv_threshold,
                    self.autoconv_rate, self.rain_evap_rate, self.terminal_velocity,
                    self.layer_depth, int(self.latent_heating))


STATE_KEYS = ("rho", "rho_theta", "u", "v", "w")
TRACER_KEYS = ("qv", "qc", "qr")


def shapes(g: GridSpec) -> dict:
    nx, ny, nz = g.nx, g.ny, g.nz
    return {"rho": (nz, ny, nx), "rho_theta": (nz, ny, nx), "u": (nz, ny, nx + 1),
            "v": (nz, ny + 1, nx), "w": (nz + 1, ny, nx), "qv": (nz, ny, nx),
            "qc": (nz, ny, nx), "qr": (nz, ny, nx), "precip": (ny, nx)}


def zeros(g: GridSpec, moist: bool = False) -> dict:
    sh = shapes(g)
    keys = STATE_KEYS + ((TRACER_KEYS + ("precip",)) if moist else ())
    return {k: np.zeros(sh[k]) for k in keys}


def _fields(d: dict) -> Fields:
    f = Fields()
    for k in STATE_KEYS + TRACER_KEYS + ("precip",):
        a = d.get(k)
        if a is not None:
            d[k] = np.ascontiguousarray(a, dtype=np.float64)
            setattr(f, k, _ptr(d[k]))
    return f


PHASE_DRY, PHASE_TRACERS, PHASE_RAIN, PHASE_RAIN_NOMINAL = 1, 2, 4, 8


def run(g: GridSpec, step: StepSpec, state: dict, nsteps: int = 1, phases: int = PHASE_DRY,
        rain: Optional[RainSpec] = None, precision: int = 64, boundary: Optional[dict] = None,
        boundary_cache: Optional[tuple] = None) -> dict:
    """Advance copies of ``state`` by ``nsteps`` steps; returns the new fields.
    ``boundary`` (same keys as a state; tracers optional) is a reference boundary state
    applied by apply_reference_boundaries at every stage start.  ``boundary_cache`` =
    (offsets, snapshots, t_start) is the prepared-case updater: balanced snapshot states
    (tracers qv, qc, qr as mixing ratios) at integer forecast offsets, interpolated at
    lround(step start + stage time); t_start is the first step's start time."""
    out = {k: np.array(v, dtype=np.float64, copy=True) for k, v in state.items() if v is not None}
    gc, sc = g.c(), step.c()
    rc = rain.c() if rain is not None else None
    f = _fields(out)
    rcp = C.byref(rc) if rc is not None else None
    if boundary_cache is not None:
        offsets, snaps, t_start = boundary_cache
        keep = [{k: np.array(v, dtype=np.float64, copy=True) for k, v in sn.items() if v is not None} for sn in snaps]
        arr = (Fields * len(keep))(*[_fields(d) for d in keep])
        off = (C.c_int * len(keep))(*[int(t) for t in offsets])
        _check(lib().gwo_run_boundary_cache(C.byref(gc), C.byref(sc), rcp, phases, nsteps, precision, C.byref(f),
                                            len(keep), off, arr, float(t_start)))
    elif boundary is None:
        _check(lib().gwo_run(C.byref(gc), C.byref(sc), rcp, phases, nsteps, precision, C.byref(f)))
    else:
        bnd = {k: np.array(v, dtype=np.float64, copy=True) for k, v in boundary.items() if v is not None}
        fb = _fields(bnd)
        _check(lib().gwo_run_boundary(C.byref(gc), C.byref(sc), rcp, phases, nsteps, precision,
                                      C.byref(f), C.byref(fb)))
    return out


def slow_tendencies(g: GridSpec, step: StepSpec, state: dict, precision: int = 64) -> dict:
    inp = {k: np.array(state[k], dtype=np.float64, copy=True) for k in STATE_KEYS}
    out = zeros(g)
    gc, sc = g.c(), step.c()
    fi, fo = _fields(inp), _fields(out)
    _check(lib().gwo_slow_tendencies(C.byref(gc), C.byref(sc), precision, C.byref(fi), C.byref(fo)))
    return out


def fast_modes(g: GridSpec, step: StepSpec, state: dict, precision: int = 64) -> dict:
    out = {k: np.array(state[k], dtype=np.float64, copy=True) for k in STATE_KEYS}
    gc, sc = g.c(), step.c()
    f = _fields(out)
    _check(lib().gwo_fast_modes(C.byref(gc), C.byref(sc), precision, C.byref(f)))
    return out


def metrics(g: GridSpec, precision: int = 64) -> dict:
    nx, ny, nz = g.nx, g.ny, g.nz
    zc, idc = np.zeros((nz, ny, nx)), np.zeros((nz, ny, nx))
    zi, idf = np.zeros((nz + 1, ny, nx)), np.zeros((nz + 1, ny, nx))
    gc = g.c()
    _check(lib().gwo_metrics(C.byref(gc), precision, _ptr(zc), _ptr(zi), _ptr(idc), _ptr(idf)))
    return {"z_centers": zc, "z_interfaces": zi, "inv_dz_cell": idc, "inv_dz_face": idf}


CASE_KINDS = {"warm_bubble": 0, "density_current": 1, "hydrostatic_rest": 2,
              "mountain_wave_background": 3, "constant": 4, "hydrostatic_warm_bubble": 5}


@dataclass
class CaseSpec:
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

    def c(self) -> CaseParams:
        return CaseParams(*[getattr(self, n) for n, _ in CaseParams._fields_])


def case(kind: str, g: GridSpec, params: CaseSpec, precision: int = 32) -> dict:
    out = zeros(g)
    gc, pc = g.c(), params.c()
    f = _fields(out)
    _check(lib().gwo_case(CASE_KINDS[kind], C.byref(gc), C.byref(pc), precision, C.byref(f)))
    return out


def moist_sounding(g: GridSpec, p_surface: float = 100000.0, theta_ref: float = 300.0,
                   theta_lapse_k_per_m: float = 0.004, relative_humidity: float = 0.9, rh_top_m: float = 2000.0,
                   qv_scale_height_m: float = 1500.0, qv_floor: float = 1e-5, noise_rms_k: float = 0.5,
                   noise_depth_m: float = 1000.0, seed: int = 1) -> dict:
    """The moist warm-rain benchmark's initial state (FP32 values as float64 arrays), built
    by the oracle itself: the seeded sounding balanced column by column, at rest, with no
    cloud or rain water (flat grid)."""
    out = zeros(g, moist=True)
    gc = g.c()
    sc = Sounding(p_surface, theta_ref, theta_lapse_k_per_m, relative_humidity, rh_top_m, qv_scale_height_m,
                  qv_floor, noise_rms_k, noise_depth_m, seed)
    f = _fields(out)
    _check(lib().gwo_moist_sounding(C.byref(gc), C.byref(sc), C.byref(f)))
    return out


def scalar_ssprk3(q: np.ndarray, u_adv: float, v_adv: float, dt: float, dx: float = 1000.0, dy: float = 1000.0,
                  periodic_x: bool = True, periodic_y: bool = True, nsteps: int = 1,
                  precision: int = 64) -> np.ndarray:
    """nsteps of advance_scalar_ssprk3 (dry_transport.cu:285-325) on q (nz, ny, nx)."""
    out = np.array(q, dtype=np.float64, copy=True, order="C")
    nz, ny, nx = out.shape
    _check(lib().gwo_scalar_ssprk3(nx, ny, nz, int(periodic_x), int(periodic_y), float(u_adv), float(v_adv),
                                   float(dt), float(dx), float(dy), nsteps, precision, _ptr(out)))
    return out


def pressure(rho: np.ndarray, rho_theta: np.ndarray, precision: int = 64) -> np.ndarray:
    r = np.ascontiguousarray(rho, dtype=np.float64)
    t = np.ascontiguousarray(rho_theta, dtype=np.float64)
    p = np.zeros_like(r)
    _check(lib().gwo_pressure(r.size, _ptr(r), _ptr(t), _ptr(p), precision))
    return p


# Fields of the runtime plan-view bundle, in its order (plan_view_output.cpp:630-834).
PLAN_VIEW_FIELDS = ("terrain_height", "z_center", "rho_d", "theta_m", "air_pressure", "air_temperature",
                    "u_velocity", "v_velocity", "wind_speed", "w_velocity", "specific_humidity",
                    "relative_humidity", "dewpoint", "cloud_water_mixing_ratio", "rain_water_mixing_ratio",
                    "total_condensate", "column_cloud_water", "column_rain_water", "column_total_condensate",
                    "column_rain_fraction", "synthetic_reflectivity", "accumulated_surface_precipitation",
                    "mean_surface_precipitation_rate")


def plan_view(g: GridSpec, state: dict, level: int, steps: int = 0, dt: float = 0.0,
              nfields: Optional[int] = None) -> dict:
    """extract_runtime_plan_view of a state (global arrays; the warm-rain tracers as
    masses rho*q, "precip" the surface accumulation) at ``level``: {field: (ny, nx)}.
    nfields defaults to what the state holds (10 dry, 21 with qv/qc/qr, 23 with precip)."""
    if nfields is None:
        nfields = 10 if "qv" not in state else (21 if "precip" not in state else 23)
    arr = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in state.items()}
    out = np.zeros((nfields, g.ny, g.nx), np.float64)
    gc = g.c()
    _check(lib().gwo_plan_view(C.byref(gc), level, nfields, steps, dt, *[_ptr(arr.get(k)) for k in (
        "rho", "rho_theta", "u", "v", "w", "qv", "qc", "qr", "precip")], _ptr(out)))
    return {PLAN_VIEW_FIELDS[q]: out[q] for q in range(nfields)}


def layout(nx, ny, nz, halo, rx, ry, px=True, py=True) -> np.ndarray:
    out = np.zeros(12 * rx * ry, dtype=np.int32)
    _check(lib().gwo_layout(nx, ny, nz, halo, rx, ry, int(px), int(py),
                            out.ctypes.data_as(C.POINTER(C.c_int))))
    return out.reshape(rx * ry, 12)


ORIENT = {"cell": 0, "x": 1, "y": 2, "z": 3}


def rank_field_shape(desc_row, nz: int, halo: int, orient: str):
    nxl = int(desc_row[4] - desc_row[3])
    nyl = int(desc_row[6] - desc_row[5])
    fx = nxl + (orient == "x")
    fy = nyl + (orient == "y")
    fz = nz + (orient == "z")
    return (fz, fy + 2 * halo, fx + 2 * halo)


def halo(fields: list, nx, ny, nz, halo_w, rx, ry, px, py, orient: str, op: str = "exchange"):
    """Apply the reference halo exchange (or interface sync) in place on per-rank arrays."""
    arrs = [np.ascontiguousarray(f, dtype=np.float64) for f in fields]
    ptrs = (DP * len(arrs))(*[_ptr(a) for a in arrs])
    _check(lib().gwo_halo(nx, ny, nz, halo_w, rx, ry, int(px), int(py), ORIENT[orient],
                          0 if op == "exchange" else 1, ptrs))
    for f, a in zip(fields, arrs):
        if f is not a:
            f[...] = a
    return arrs


def set_threads(n: int) -> None:
    lib().gwo_set_threads(int(n))


def max_threads() -> int:
    return int(lib().gwo_max_threads())


MLP_PARAMS = 64 * 7 + 64 + 2 * (64 * 64 + 64) + 5 * 64 + 5


def mlp_loss_grad(params: np.ndarray, norm: np.ndarray, x: np.ndarray, y: np.ndarray):
    """FP64 loss and gradient of the warm-rain surrogate MLP (checker of the GPU kernels)."""
    p = np.ascontiguousarray(params, dtype=np.float64)
    nm = np.ascontiguousarray(norm, dtype=np.float64)
    xx = np.ascontiguousarray(x, dtype=np.float64)
    yy = np.ascontiguousarray(y, dtype=np.float64)
    g = np.zeros(MLP_PARAMS)
    loss = C.c_double()
    _check(lib().gwo_mlp_loss_grad(_ptr(p), _ptr(nm), _ptr(xx), _ptr(yy), xx.shape[0], _ptr(g), C.byref(loss)))
    return loss.value, g
