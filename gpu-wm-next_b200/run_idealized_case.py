"""Run an idealized case described by a case file (YAML), as a regression harness.

The case-file schema is the reference's idealized one (cases/idealized/*.yaml read by
tools/casebuilder/run_idealized_case.py): a `grid` section (nx, ny, nz, dx, dy, z_top),
an optional `terrain` section (kind, center_x_fraction, center_y_fraction,
half_width_x_fraction, half_width_y_fraction, height) and an `initialization` section
(kind plus the ThermoBubbleConfig / MountainWaveBackgroundConfig keys).  Such a case
runs through gwm_b200_idealized_driver, the reference driver's command line over this
library, and its summary JSON is written next to the case file (or to
--summary-json).

A case file with a `transport` section (u_adv, v_adv) and a `time` section (dt, t_end)
runs scalar advection instead: t_end / dt steps of advance_scalar_ssprk3 on the GPU,
from the field sin(0.2 i) + cos(0.3 j) of the reference's virtual-rank equivalence test,
with a summary of the field's mass and range before and after.

Usage:
    python gpu-wm-next_b200/run_idealized_case.py case.yaml [--steps N] [--dt S]
        [--fast-substeps N] [--summary-json PATH] [--plan-view-json PATH] [--plan-view-level K]
        [--driver PATH] [--print-command]
"""
import argparse
import importlib
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

# case-file key -> driver flag, per section
GRID_KEYS = {"nx": "--nx", "ny": "--ny", "nz": "--nz", "dx": "--dx", "dy": "--dy", "z_top": "--z-top"}
TERRAIN_KEYS = {"center_x_fraction": "--terrain-center-x", "center_y_fraction": "--terrain-center-y",
                "half_width_x_fraction": "--terrain-half-width-x",
                "half_width_y_fraction": "--terrain-half-width-y", "height": "--terrain-height"}
INIT_KEYS = ("rho_background", "theta_background", "u_background", "v_background", "w_background",
             "theta_perturbation", "center_x_fraction", "center_y_fraction", "center_z_fraction",
             "radius_x_fraction", "radius_y_fraction", "radius_z_fraction", "rho_surface", "theta_ref",
             "density_scale_height")


def load_case(path):
    import yaml
    with open(path, encoding="utf-8") as f:
        data = yaml.safe_load(f) or {}
    if not isinstance(data, dict):
        raise ValueError(f"{path}: expected a mapping at the top level")
    for sec in ("grid", "terrain", "initialization", "transport", "time"):
        if sec in data and not isinstance(data[sec], dict):
            raise ValueError(f"{path}: section {sec!r} must be a mapping")
    return data


def driver_command(case, driver, summary_json, steps=None, dt=None, fast_substeps=None, plan_view_json=None,
                   plan_view_level=None):
    """The gwm_b200_idealized_driver command line of a dry idealized case file."""
    grid, terrain, init = case.get("grid", {}), case.get("terrain", {}), case.get("initialization", {})
    cmd = [driver, "--case", str(init.get("kind", "density_current"))]
    cmd += [x for k, flag in GRID_KEYS.items() if k in grid for x in (flag, str(grid[k]))]
    if "kind" in terrain:
        cmd += ["--terrain-kind", str(terrain["kind"])]
        cmd += [x for k, flag in TERRAIN_KEYS.items() if k in terrain for x in (flag, str(terrain[k]))]
    cmd += [x for k in INIT_KEYS if k in init for x in ("--" + k.replace("_", "-"), str(init[k]))]
    for flag, value in (("--steps", steps), ("--dt", dt), ("--fast-substeps", fast_substeps),
                        ("--plan-view-json", plan_view_json), ("--plan-view-level", plan_view_level)):
        if value is not None:
            cmd += [flag, str(value)]
    return cmd + ["--summary-json", summary_json]


def run_scalar_case(case, summary_json, steps=None, dt=None):
    """t_end / dt steps of advance_scalar_ssprk3 from the equivalence-test field."""
    import numpy as np
    gwm = importlib.import_module("gpu-wm-next_b200")
    grid, tr, tm = case.get("grid", {}), case["transport"], case.get("time", {})
    nx, ny, nz = int(grid.get("nx", 32)), int(grid.get("ny", 32)), int(grid.get("nz", 1))
    dt = float(dt if dt is not None else tm.get("dt", 10.0))
    n = int(steps if steps is not None else round(float(tm.get("t_end", dt)) / dt))
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    q0 = np.broadcast_to((np.sin(0.2 * i) + np.cos(0.3 * j)).astype(np.float32), (nz, ny, nx)).copy()
    q = gwm.scalar_ssprk3(q0, u_adv=float(tr.get("u_adv", 20.0)), v_adv=float(tr.get("v_adv", 0.0)), dt=dt,
                          dx=float(grid.get("dx", 1000.0)), dy=float(grid.get("dy", 1000.0)), nsteps=n)
    stat = lambda a: {"mass": float(a.astype(np.float64).sum()), "min": float(a.min()), "max": float(a.max())}
    summary = {"case": str(case.get("name", "scalar_advection")), "steps": n, "dt": dt,
               "initial": stat(q0), "final": stat(q)}
    text = json.dumps(summary, indent=2)
    print(text)
    with open(summary_json, "w") as f:
        f.write(text + "\n")
    return summary


def main(argv=None):
    ap = argparse.ArgumentParser(description="Run an idealized case file through this library.")
    ap.add_argument("case_file")
    ap.add_argument("--driver", default=None, help="gwm_b200_idealized_driver path (default: the built one)")
    ap.add_argument("--summary-json", default=None)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--dt", type=float, default=None)
    ap.add_argument("--fast-substeps", type=int, default=None)
    ap.add_argument("--plan-view-json", default=None, help="also write the dry plan-view bundle here")
    ap.add_argument("--plan-view-level", type=int, default=None)
    ap.add_argument("--print-command", action="store_true", help="print the driver command and stop")
    args = ap.parse_args(argv)
    case = load_case(args.case_file)
    summary_json = args.summary_json or os.path.splitext(args.case_file)[0] + ".summary.json"
    if "transport" in case:
        if args.print_command:
            print("scalar advection (advance_scalar_ssprk3 through the library)")
            return 0
        run_scalar_case(case, summary_json, args.steps, args.dt)
        return 0
    driver = args.driver
    if driver is None:
        gwm = importlib.import_module("gpu-wm-next_b200")
        gwm.build()
        driver = gwm.DRIVER_PATH
    cmd = driver_command(case, driver, summary_json, args.steps, args.dt, args.fast_substeps, args.plan_view_json,
                         args.plan_view_level)
    print(" ".join(cmd), flush=True)
    if args.print_command:
        return 0
    return subprocess.run(cmd).returncode


if __name__ == "__main__":
    sys.exit(main())
