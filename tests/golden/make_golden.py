"""Generate golden vectors from the reference implementation itself.

Each case builds an initial state with the library's case builders (host code),
writes it as a case file, runs ``oracle/_ref/gwm_ref_golden`` (the reference's own
step operators compiled from its sources by ``make -C oracle ref``; it needs a
GPU because the reference runs its kernels on managed memory) and stores inputs,
parameters and outputs in ``ref_<case>.npz``.  The reference's level-mean
reduction uses float atomics, so its output is reproducible only to rounding;
the tests compare against it with tolerances, never bitwise.  The scalar-advection
cases (advance_scalar_ssprk3, no atomics) are exact and compared bit for bit.
The plan-view cases (``ref_pv_<case>.npz``) also keep the reference's runtime plan view
of its final state (extract_runtime_plan_view + plan_view_bundle_to_json, as JSON text)
beside that state, so the diagnostics are compared on exactly the state they describe.

Usage (on a machine with a GPU and the built driver):
    python tests/golden/make_golden.py --out tests/golden
"""
import argparse
import importlib
import json
import os
import struct
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "gwm_ref_golden")

# name -> (grid, case kind, case params, terrain, step, moist/rain, steps)
CASES = {
    "bubble_periodic": dict(
        grid=dict(nx=24, ny=20, nz=16, dx=500.0, dy=500.0, z_top=8000.0),
        kind="hydrostatic_warm_bubble",
        params=dict(rho_surface=1.16123, theta_ref=300.0, center_z_fraction=0.25,
                    radius_x_fraction=0.2, radius_y_fraction=0.2, radius_z_fraction=0.2,
                    theta_perturbation=2.0),
        step=dict(dt=1.0, fast_substeps=3), steps=3),
    "ranks_open_wind": dict(
        grid=dict(nx=22, ny=18, nz=12, dx=1000.0, dy=1000.0, z_top=10000.0,
                  periodic_x=False, periodic_y=False, ranks_x=2, ranks_y=2),
        kind="hydrostatic_warm_bubble",
        params=dict(rho_surface=1.16123, theta_ref=300.0, center_x_fraction=0.4, center_z_fraction=0.3, radius_x_fraction=0.2,
                    radius_y_fraction=0.25, radius_z_fraction=0.25, theta_perturbation=1.5),
        wind=(4.0, -2.0), step=dict(dt=1.0, fast_substeps=4), steps=3),
    "terrain_cosine": dict(
        grid=dict(nx=32, ny=12, nz=14, dx=1000.0, dy=1000.0, z_top=12000.0, periodic_y=True),
        kind="mountain_wave_background",
        params=dict(rho_surface=1.16123, theta_ref=300.0, u_background=8.0),
        terrain=dict(kind="cosine_mountain", height=400.0, half_width_x=0.2, half_width_y=0.5),
        step=dict(dt=1.0, fast_substeps=4), steps=2),
    "fast_off": dict(
        grid=dict(nx=16, ny=16, nz=12, dx=500.0, dy=500.0, z_top=6000.0),
        kind="hydrostatic_warm_bubble",
        params=dict(rho_surface=1.16123, theta_ref=300.0, radius_x_fraction=0.25,
                    radius_y_fraction=0.25, radius_z_fraction=0.25, theta_perturbation=1.0),
        step=dict(dt=0.5, fast_substeps=2, fast_modes=False), steps=2),
    "moist_metric": dict(
        grid=dict(nx=20, ny=16, nz=16, dx=2000.0, dy=2000.0, z_top=8000.0),
        kind="moist_sounding",
        params=dict(theta_ref=300.0, relative_humidity=1.03, noise_rms_k=0.5, seed=3),
        step=dict(dt=2.0, fast_substeps=4), moist=True,
        rain=dict(mode=1, terminal_velocity=12.0), steps=3),
    "moist_nominal": dict(
        grid=dict(nx=16, ny=12, nz=12, dx=2000.0, dy=2000.0, z_top=6000.0),
        kind="moist_sounding",
        params=dict(theta_ref=300.0, relative_humidity=1.05, noise_rms_k=0.3, seed=7),
        step=dict(dt=2.0, fast_substeps=3), moist=True,
        rain=dict(mode=2, terminal_velocity=5.0, layer_depth=500.0), steps=2),
}

# Plan-view cases: a step case whose final state's runtime plan view (at `level`) is
# kept.  The moist case starts with a seeded cloud and rain bump reaching the ground, so
# every moist field, the column maps and the surface precipitation are non-trivial.
PLAN_VIEW_CASES = {
    "pv_moist_rain": dict(
        grid=dict(nx=20, ny=16, nz=12, dx=2000.0, dy=2000.0, z_top=8000.0, ranks_x=2),
        kind="moist_sounding",
        params=dict(theta_ref=300.0, relative_humidity=1.02, noise_rms_k=0.5, seed=5),
        step=dict(dt=2.0, fast_substeps=3), moist=True,
        rain=dict(mode=1, terminal_velocity=12.0), steps=3,
        bump=dict(qc=1.5e-3, qr=8.0e-4, sigma=3.0, depth=6), level=2),
    "pv_dry_terrain": dict(CASES["terrain_cosine"], level=3),
}

RAIN_DEFAULTS = dict(mode=1, relax=1.0, autoconv_threshold=1.0e-4, autoconv_rate=1.0e-3,
                     evap_rate=5.0e-3, terminal_velocity=0.0, layer_depth=0.0, latent=True)
STEP_DEFAULTS = dict(dt=2.0, fast_substeps=1, gravity=9.81, fast_hmom=True, fast_density=True,
                     fast_modes=True)


def case_state(gwm, spec):
    """Initial fields (float32, global C order) and terrain for a case spec."""
    gkw = dict(spec["grid"])
    terrain = np.zeros((gkw["ny"], gkw["nx"]), dtype=np.float32)
    if "terrain" in spec:
        t = dict(spec["terrain"])
        kind = t.pop("kind")
        terrain = gwm.build_terrain(kind, gkw["nx"], gkw["ny"], gkw["dx"], gkw["dy"], **t)
        gkw["terrain"] = terrain
    g = gwm.GridSpec(**gkw)
    moist = spec.get("moist", False)
    s = gwm.build_case(spec["kind"], g, gwm.CaseParams(**spec["params"]), moist=moist)
    if "wind" in spec:  # uniform wind on the bubble: face momentum = face-mean density * wind
        ub, vb = spec["wind"]
        r = s["rho"]
        ru = np.concatenate([r[:, :, :1], 0.5 * (r[:, :, 1:] + r[:, :, :-1]), r[:, :, -1:]], axis=2)
        rv = np.concatenate([r[:, :1, :], 0.5 * (r[:, 1:, :] + r[:, :-1, :]), r[:, -1:, :]], axis=1)
        s["u"] = (ru * ub).astype(np.float32)
        s["v"] = (rv * vb).astype(np.float32)
    if "bump" in spec:  # cloud and rain mass in a Gaussian column over the lowest levels
        b = spec["bump"]
        nz, ny, nx = s["rho"].shape
        j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
        f = np.exp(-((i - 0.5 * nx) ** 2 + (j - 0.5 * ny) ** 2) / (2.0 * b["sigma"] ** 2))
        col = (np.arange(nz) < b["depth"]).astype(np.float64)[:, None, None] * f[None]
        s["qc"] = (s["qc"] + s["rho"] * b["qc"] * col).astype(np.float32)
        s["qr"] = (s["qr"] + s["rho"] * b["qr"] * col).astype(np.float32)
    return s, terrain


def write_case(path, spec, state, terrain):
    g = spec["grid"]
    st = dict(STEP_DEFAULTS, **spec["step"])
    rn = dict(RAIN_DEFAULTS, **spec.get("rain", {}))
    moist = spec.get("moist", False)
    hdr = struct.pack("<8s16i12d", b"GWMCASE1", g["nx"], g["ny"], g["nz"], g.get("ranks_x", 1),
                      g.get("ranks_y", 1), int(g.get("periodic_x", True)), int(g.get("periodic_y", True)),
                      st["fast_substeps"], int(st["fast_hmom"]), int(st["fast_density"]),
                      int(st["fast_modes"]), spec["steps"], int(moist), rn["mode"] if moist else 0,
                      int(rn["latent"]), 0,
                      g["dx"], g["dy"], g["z_top"], g.get("terrain_taper_eta", 0.25), st["dt"],
                      st["gravity"], rn["relax"], rn["autoconv_threshold"], rn["autoconv_rate"],
                      rn["evap_rate"], rn["terminal_velocity"], rn["layer_depth"])
    keys = ("rho", "rho_theta", "u", "v", "w") + (("qv", "qc", "qr") if moist else ())
    with open(path, "wb") as f:
        f.write(hdr)
        f.write(np.ascontiguousarray(terrain, dtype=np.float32).tobytes())
        for k in keys:
            f.write(np.ascontiguousarray(state[k], dtype=np.float32).tobytes())


def read_out(path, spec, shapes):
    moist = spec.get("moist", False)
    keys = ("rho", "rho_theta", "u", "v", "w") + (("qv", "qc", "qr", "precip") if moist else ())
    raw = open(path, "rb").read()
    assert raw[:8] == b"GWMOUT01", "bad output header"
    off, out = 8, {}
    for k in keys:
        n = int(np.prod(shapes[k]))
        out[k] = np.frombuffer(raw, dtype=np.float32, count=n, offset=off).reshape(shapes[k]).copy()
        off += 4 * n
    assert off == len(raw), "output size mismatch"
    return out


# Scalar advection cases (advance_scalar_ssprk3): name -> grid, ranks, periodicity,
# DryTransportConfig, steps and the initial field q(i, j, k).  The first three take the
# configurations of the reference's own tests (test_constant_state.cpp,
# test_scalar_mass_conservation.cpp, test_virtual_rank_equivalence.cpp); the wave runs
# the scalar_advection case file's 300 s (60 steps); the last has an open side.
SCALAR_CASES = {
    "scalar_constant": dict(nx=24, ny=24, nz=3, rx=2, ry=2, px=True, py=True, u=20.0, v=-10.0, dt=4.0, steps=1,
                            init="constant"),
    "scalar_mass": dict(nx=32, ny=20, nz=1, rx=2, ry=2, px=True, py=True, u=12.0, v=7.0, dt=2.0, steps=1,
                        init="stripes"),
    "scalar_wave": dict(nx=32, ny=32, nz=2, rx=2, ry=2, px=True, py=True, u=15.0, v=-5.0, dt=5.0, steps=60,
                        init="wave"),
    "scalar_open": dict(nx=40, ny=24, nz=3, rx=2, ry=1, px=False, py=True, u=-18.0, v=6.0, dt=3.0, steps=5,
                        init="random"),
}


def scalar_field(c):
    nz, ny, nx = c["nz"], c["ny"], c["nx"]
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    if c["init"] == "constant":
        q = np.full((nz, ny, nx), 7.5)
    elif c["init"] == "stripes":
        q = 1.0 + 0.1 * ((i + 2 * j) % 7)
    elif c["init"] == "wave":
        q = np.sin(0.2 * i) + np.cos(0.3 * j)
    else:
        q = np.random.default_rng(17).uniform(0.5, 2.0, (nz, ny, nx))
    return np.asarray(q, dtype=np.float32)


def write_scalar_case(path, c, q):
    hdr = struct.pack("<8s8i6f", b"GWMSCAL1", c["nx"], c["ny"], c["nz"], c["rx"], c["ry"], int(c["px"]),
                      int(c["py"]), c["steps"], c["u"], c["v"], c["dt"], 1000.0, 1000.0, 0.0)
    with open(path, "wb") as f:
        f.write(hdr)
        f.write(np.ascontiguousarray(q, dtype=np.float32).tobytes())


def read_scalar_out(path, c):
    raw = open(path, "rb").read()
    assert raw[:8] == b"GWMSCA01", "bad scalar output header"
    n = c["nx"] * c["ny"] * c["nz"]
    assert len(raw) == 8 + 4 * n, "scalar output size mismatch"
    return np.frombuffer(raw, dtype=np.float32, offset=8).reshape(c["nz"], c["ny"], c["nx"]).copy()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--cases", nargs="*", default=list(CASES) + list(SCALAR_CASES) + list(PLAN_VIEW_CASES))
    args = ap.parse_args()
    if not os.path.exists(DRIVER):
        sys.exit(f"{DRIVER} missing: build it with `make -C oracle ref`")
    sys.path.insert(0, ROOT)
    gwm = importlib.import_module("gpu-wm-next_b200")
    os.makedirs(args.out, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        for name in args.cases:
            if name in SCALAR_CASES:
                c = SCALAR_CASES[name]
                q = scalar_field(c)
                cpath, opath = os.path.join(tmp, name + ".case"), os.path.join(tmp, name + ".out")
                write_scalar_case(cpath, c, q)
                subprocess.run([DRIVER, cpath, opath], check=True, timeout=600)
                out = read_scalar_out(opath, c)
                np.savez_compressed(os.path.join(args.out, f"ref_{name}.npz"),
                                    spec=np.frombuffer(json.dumps(c).encode(), dtype=np.uint8), in_q=q, out_q=out)
                print(f"{name}: wrote ref_{name}.npz (finite={np.isfinite(out).all()})", flush=True)
                continue
            spec = CASES[name] if name in CASES else PLAN_VIEW_CASES[name]
            state, terrain = case_state(gwm, spec)
            cpath, opath = os.path.join(tmp, name + ".case"), os.path.join(tmp, name + ".out")
            write_case(cpath, spec, state, terrain)
            cmd = [DRIVER, cpath, opath]
            pv_path = os.path.join(tmp, name + ".pv.json")
            if name in PLAN_VIEW_CASES:
                cmd += [pv_path, str(spec["level"])]
            subprocess.run(cmd, check=True, timeout=600)
            shapes = gwm.GridSpec(**{k: v for k, v in spec["grid"].items()}).shapes()
            out = read_out(opath, spec, shapes)
            arrays = {"in_" + k: np.asarray(v, dtype=np.float32) for k, v in state.items() if k != "precip"}
            arrays.update({"out_" + k: v for k, v in out.items()})
            arrays["terrain"] = terrain
            if name in PLAN_VIEW_CASES:
                arrays["plan_view_json"] = np.frombuffer(open(pv_path, "rb").read(), dtype=np.uint8)
            np.savez_compressed(os.path.join(args.out, f"ref_{name}.npz"),
                                spec=np.frombuffer(json.dumps(spec).encode(), dtype=np.uint8), **arrays)
            fin = all(np.isfinite(v).all() for v in out.values())
            print(f"{name}: wrote ref_{name}.npz (finite={fin})", flush=True)


if __name__ == "__main__":
    main()
