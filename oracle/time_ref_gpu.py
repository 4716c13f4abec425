"""Time the reference's own GPU step on the bench workload, for the baseline record.

Measurement infrastructure beside the oracle, not part of the product: it drives
oracle/_ref/gwm_ref_golden (the reference's own step operators compiled from its sources
by oracle/Makefile, target `ref`) on the moist C3 sounding of bench.py (3 km spacing, 64
levels to 16 km, dt 1 s, 6 acoustic substeps, three tracers, warm rain with metric
fallout at 12 m/s) at the horizontal sizes given, and prints one JSON line per size with
the reference's per-step wall times (host clock around each step with a device
synchronisation on both sides, as the reference's operators return synchronised).  The
first step is reported but not used: it includes the reference's first-touch page
migration of its managed memory.

Two further workloads of the baseline table (--case):
  c1   the dry warm bubble: 32 x 32 x 40, dx 500 m, 10 km top, +2 K cos^2 bubble of 2 km
       radius at 2 km on a neutral hydrostatic 300 K base, dt 2 s, 3 acoustic substeps;
  c2p  the mountain wave in the form the reference supports: a cosine hill (400 m) on
       uniform levels to 20 km, constant theta, 10 m/s, no damping layer, dx 1 km,
       dt 0.5 s, 6 acoustic substeps, at the sizes given (512 for the benchmark grid).

Usage (on a machine with the GPU and the built checker):
    python oracle/time_ref_gpu.py --sizes 128,256,512 --steps 3 [--timeout 1200]
    python oracle/time_ref_gpu.py --case c1 --steps 5
    python oracle/time_ref_gpu.py --case c2p --sizes 512 --steps 2
"""
import argparse
import importlib
import json
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "gwm_ref_golden")


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--sizes", default="128,256")
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--timeout", type=float, default=1200.0, help="seconds per size")
    ap.add_argument("--case", default="c3", choices=("c3", "c1", "c2p"))
    args = ap.parse_args(argv)
    if not os.path.exists(DRIVER):
        raise SystemExit(f"{DRIVER} missing: build it with `make -C oracle ref` where the reference tree is")
    import bench
    import make_golden
    gwm = importlib.import_module("gpu-wm-next_b200")
    sizes = [32] if args.case == "c1" else [int(x) for x in args.sizes.split(",")]
    for n in sizes:
        nz, terrain = bench.NZ, np.zeros((n, n), np.float32)
        if args.case == "c1":
            nz = 40
            g = gwm.GridSpec(n, n, nz, dx=500.0, dy=500.0, z_top=10000.0)
            p = gwm.CaseParams(rho_surface=np.float32(1e5 / (287.05 * 300.0)), theta_ref=300.0,
                               theta_perturbation=2.0, center_z_fraction=0.2, radius_x_fraction=2000.0 / (n * 500.0),
                               radius_y_fraction=2000.0 / (n * 500.0), radius_z_fraction=0.2)
            state = gwm.build_case("hydrostatic_warm_bubble", g, p)
            spec = dict(grid=dict(nx=n, ny=n, nz=nz, dx=500.0, dy=500.0, z_top=10000.0),
                        step=dict(dt=2.0, fast_substeps=3), moist=False, steps=args.steps)
        elif args.case == "c2p":
            nz = 80
            terrain = gwm.build_terrain("cosine_mountain", n, n, 1000.0, 1000.0, height=400.0,
                                        half_width_x=0.1, half_width_y=0.1)
            g = gwm.GridSpec(n, n, nz, dx=1000.0, dy=1000.0, z_top=20000.0, terrain=terrain)
            state = gwm.build_case("mountain_wave_background", g,
                                   gwm.CaseParams(theta_ref=288.0, p_surface=100000.0, u_background=10.0))
            spec = dict(grid=dict(nx=n, ny=n, nz=nz, dx=1000.0, dy=1000.0, z_top=20000.0),
                        step=dict(dt=0.5, fast_substeps=6), moist=False, steps=args.steps)
        else:
            g = bench.grid_spec(gwm, n, n, bench.NZ)
            state = gwm.build_case("moist_sounding", g, bench.case_params(gwm), moist=True)
            spec = dict(grid=dict(nx=n, ny=n, nz=bench.NZ, dx=bench.DX, dy=bench.DX, z_top=bench.ZTOP),
                        step=dict(dt=bench.DT, fast_substeps=bench.NS), moist=True,
                        rain=dict(mode=1, terminal_velocity=bench.VT), steps=args.steps)
        with tempfile.TemporaryDirectory() as tmp:
            cpath, opath = os.path.join(tmp, "case.bin"), os.path.join(tmp, "out.bin")
            make_golden.write_case(cpath, spec, state, terrain)
            r = subprocess.run([DRIVER, cpath, opath], capture_output=True, text=True, timeout=args.timeout)
        if r.returncode != 0:
            raise SystemExit(f"reference run failed at {n}x{n}: {r.stderr[-500:]}")
        ms = [float(m.group(1)) for m in re.finditer(r"step \d+ ms ([0-9.]+)", r.stderr)]
        cells = n * n * nz
        timed = ms[1:] if len(ms) > 1 else ms
        med = float(np.median(timed))
        print(json.dumps({"impl": "reference GPU step (oracle/_ref)", "case": args.case, "nx": n, "ny": n, "nz": nz,
                          "cells": cells, "step_ms": ms, "median_ms_after_first": med,
                          "cell_updates_per_s": cells / (med * 1e-3)}), flush=True)


if __name__ == "__main__":
    main()
