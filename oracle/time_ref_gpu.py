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

Usage (on a machine with the GPU and the built checker):
    python oracle/time_ref_gpu.py --sizes 128,256,512 --steps 3 [--timeout 1200]
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
    args = ap.parse_args(argv)
    if not os.path.exists(DRIVER):
        raise SystemExit(f"{DRIVER} missing: build it with `make -C oracle ref` where the reference tree is")
    import bench
    import make_golden
    gwm = importlib.import_module("gpu-wm-next_b200")
    for n in (int(x) for x in args.sizes.split(",")):
        g = bench.grid_spec(gwm, n, n, bench.NZ)
        state = gwm.build_case("moist_sounding", g, bench.case_params(gwm), moist=True)
        spec = dict(grid=dict(nx=n, ny=n, nz=bench.NZ, dx=bench.DX, dy=bench.DX, z_top=bench.ZTOP),
                    step=dict(dt=bench.DT, fast_substeps=bench.NS), moist=True,
                    rain=dict(mode=1, terminal_velocity=bench.VT), steps=args.steps)
        with tempfile.TemporaryDirectory() as tmp:
            cpath, opath = os.path.join(tmp, "case.bin"), os.path.join(tmp, "out.bin")
            make_golden.write_case(cpath, spec, state, np.zeros((n, n), np.float32))
            r = subprocess.run([DRIVER, cpath, opath], capture_output=True, text=True, timeout=args.timeout)
        if r.returncode != 0:
            raise SystemExit(f"reference run failed at {n}x{n}: {r.stderr[-500:]}")
        ms = [float(m.group(1)) for m in re.finditer(r"step \d+ ms ([0-9.]+)", r.stderr)]
        cells = n * n * bench.NZ
        timed = ms[1:] if len(ms) > 1 else ms
        med = float(np.median(timed))
        print(json.dumps({"impl": "reference GPU step (oracle/_ref)", "nx": n, "ny": n, "nz": bench.NZ,
                          "cells": cells, "step_ms": ms, "median_ms_after_first": med,
                          "cell_updates_per_s": cells / (med * 1e-3)}), flush=True)


if __name__ == "__main__":
    main()
