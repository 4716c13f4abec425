"""gwm_b200_idealized_driver: the reference's gwm_idealized_driver command line
(src/core/gwm_idealized_driver.cpp:69-276) over the C-ABI.

CPU: the executable is built with the library and reports argument errors the way the
reference does (message on stderr, exit status 1).  GPU: its summary JSON (keys and
layout of driver_summary_json / summary_to_json, src/dycore/dry_diagnostics.cpp:98-125)
matches the library's own step, run through the Python binding, and the FP64 oracle;
with a 2 x 2 virtual-rank layout the totals count shared faces once per rank, as
summarize_dry_states does.
"""
import json
import os
import subprocess

import numpy as np
import pytest


def _driver(gwm):
    gwm.build()
    assert os.path.exists(gwm.DRIVER_PATH)
    return gwm.DRIVER_PATH


@pytest.mark.parametrize("args, message", [
    (["--nx", "8", "--ny", "8", "--nz", "4", "--bogus", "1"], "Unknown argument: --bogus"),
    (["--nx", "8", "--ny", "8", "--nz", "4", "--periodic-x", "maybe"], "Invalid boolean value: maybe"),
    (["--nx", "8", "--ny", "8", "--nz", "4", "--terrain-kind", "agnesi"], "Unsupported terrain kind: agnesi"),
    (["--nx", "8", "--ny", "8", "--nz", "4", "--case", "squall_line"], "Unsupported case kind: squall_line"),
    (["--nx", "8", "--ny", "8", "--nz", "4", "--halo", "2"], "only --halo 1"),
    (["--nx"], "Missing value for --nx"),
])
def test_driver_argument_errors(gwm, args, message):
    r = subprocess.run([_driver(gwm), *args], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1
    assert r.stderr.startswith("gwm_b200_idealized_driver error: ") and message in r.stderr, r.stderr


def _ranks(n, parts):
    """Row-major virtual-rank split, remainder to the low ranks (virtual_rank_layout.cpp:7-47)."""
    out, b = [], 0
    for r in range(parts):
        m = n // parts + (1 if r < n % parts else 0)
        out.append((b, m))
        b += m
    return out


def _summary(s, rx=1, ry=1):
    """summarize_dry_states over the virtual ranks of the global arrays (FP64)."""
    nz, ny, nx = s["rho"].shape
    tot = dict(total_dry_mass=0.0, total_rho_theta_m=0.0, total_horizontal_momentum_x=0.0,
               total_horizontal_momentum_y=0.0, total_vertical_momentum=0.0)
    rng = {k: [np.inf, -np.inf] for k in ("rho_d", "theta_m", "u_face", "v_face", "w_face")}
    f64 = {k: np.asarray(v, np.float64) for k, v in s.items()}
    for jb, nyl in _ranks(ny, ry):
        for ib, nxl in _ranks(nx, rx):
            rho = f64["rho"][:, jb:jb + nyl, ib:ib + nxl]
            rt = f64["rho_theta"][:, jb:jb + nyl, ib:ib + nxl]
            u = f64["u"][:, jb:jb + nyl, ib:ib + nxl + 1]
            v = f64["v"][:, jb:jb + nyl + 1, ib:ib + nxl]
            w = f64["w"][:, jb:jb + nyl, ib:ib + nxl]
            tot["total_dry_mass"] += rho.sum()
            tot["total_rho_theta_m"] += rt.sum()
            tot["total_horizontal_momentum_x"] += u.sum()
            tot["total_horizontal_momentum_y"] += v.sum()
            tot["total_vertical_momentum"] += w.sum()
            for key, a in (("rho_d", rho), ("theta_m", rt / np.maximum(rho, 1e-12)), ("u_face", u),
                           ("v_face", v), ("w_face", w)):
                rng[key] = [min(rng[key][0], a.min()), max(rng[key][1], a.max())]
    for k, (lo, hi) in rng.items():
        tot[k] = {"min": lo, "max": hi}
    return tot


def _compare(got, want, rel):
    for k, v in want.items():
        if isinstance(v, dict):
            for m in ("min", "max"):
                assert got[k][m] == pytest.approx(v[m], rel=rel, abs=rel), (k, m, got[k][m], v[m])
        else:
            assert got[k] == pytest.approx(v, rel=rel, abs=rel), (k, got[k], v)


CASE = dict(nx=32, ny=24, nz=20, dx=1000.0, dy=1000.0, z_top=10000.0)
ARGS = ["--case", "density_current", "--nx", "32", "--ny", "24", "--nz", "20", "--dx", "1000", "--dy", "1000",
        "--z-top", "10000", "--dt", "1", "--fast-substeps", "2", "--steps", "3", "--theta-perturbation", "3",
        "--radius-x-fraction", "0.2", "--radius-y-fraction", "0.25", "--radius-z-fraction", "0.3",
        "--center-z-fraction", "0.3"]


def _run_driver(gwm, extra, tmp_path):
    path = tmp_path / "summary.json"
    r = subprocess.run([_driver(gwm), *ARGS, *extra, "--summary-json", str(path)], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    printed = json.loads(r.stdout)
    assert json.loads(path.read_text()) == printed
    assert list(printed) == ["case", "steps", "dt", "initial", "final"]
    assert list(printed["final"]) == ["total_dry_mass", "total_rho_theta_m", "total_horizontal_momentum_x",
                                      "total_horizontal_momentum_y", "total_vertical_momentum", "rho_d",
                                      "theta_m", "u_face", "v_face", "w_face"]
    assert printed["case"] == "density_current" and printed["steps"] == 3 and printed["dt"] == 1
    return printed


def _library_state(gwm, rx=1, ry=1):
    g = gwm.GridSpec(**CASE, ranks_x=rx, ranks_y=ry)
    p = gwm.CaseParams(rho_background=1.0, theta_background=300.0, theta_perturbation=3.0,
                       radius_x_fraction=0.2, radius_y_fraction=0.25, radius_z_fraction=0.3,
                       center_z_fraction=0.3)
    s0 = gwm.build_case("density_current", g, p)
    with gwm.Model(g, gwm.MemberSpec(step=gwm.StepConfig(dt=1.0, fast_substeps=2))) as m:
        m.upload(s0)
        m.advance_dry_state_ssprk3(3)
        s1 = m.download()
    return g, s0, s1


@pytest.mark.gpu
def test_driver_summary_matches_library_and_oracle(gwm, orc, tmp_path):
    js = _run_driver(gwm, [], tmp_path)
    g, s0, s1 = _library_state(gwm)
    # JSON numbers carry 6 significant digits (the reference's default stream format)
    _compare(js["initial"], _summary(s0), rel=5e-6)
    _compare(js["final"], _summary(s1), rel=5e-6)
    og = orc.GridSpec(CASE["nx"], CASE["ny"], CASE["nz"], dx=CASE["dx"], dy=CASE["dy"], z_top=CASE["z_top"])
    ref = orc.run(og, orc.StepSpec(dt=1.0, fast_substeps=2), s0, 3, precision=64)
    want = _summary(ref)
    _compare({k: js["final"][k] for k in ("total_dry_mass", "total_rho_theta_m", "rho_d", "theta_m")},
             {k: want[k] for k in ("total_dry_mass", "total_rho_theta_m", "rho_d", "theta_m")}, rel=2e-5)
    for k in ("u_face", "v_face", "w_face"):  # momenta after 3 steps: within 1e-4 of their range
        scale = max(abs(want[k]["min"]), abs(want[k]["max"]))
        assert abs(js["final"][k]["max"] - want[k]["max"]) <= 1e-4 * scale + 1e-6
        assert abs(js["final"][k]["min"] - want[k]["min"]) <= 1e-4 * scale + 1e-6


@pytest.mark.gpu
def test_driver_virtual_rank_totals(gwm, tmp_path):
    one = _run_driver(gwm, [], tmp_path)
    four = _run_driver(gwm, ["--ranks-x", "2", "--ranks-y", "2"], tmp_path)
    _, s0, s1 = _library_state(gwm, 2, 2)
    _compare(four["final"], _summary(s1, 2, 2), rel=5e-6)
    # the cell totals do not depend on the layout; the face totals gain the shared faces
    assert four["final"]["total_dry_mass"] == pytest.approx(one["final"]["total_dry_mass"], rel=2e-6)
    shared_u = np.asarray(s1["u"], np.float64)[:, :, CASE["nx"] // 2].sum()
    assert four["final"]["total_horizontal_momentum_x"] == pytest.approx(
        one["final"]["total_horizontal_momentum_x"] + shared_u, rel=5e-6, abs=5e-6)


CASES_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "gpu-wm-next_b200", "cases")


def _harness():
    import importlib.util
    path = os.path.join(os.path.dirname(CASES_DIR), "run_idealized_case.py")
    spec = importlib.util.spec_from_file_location("run_idealized_case", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_case_file_maps_to_driver_flags():
    h = _harness()
    case = h.load_case(os.path.join(CASES_DIR, "mountain_wave.yaml"))
    cmd = h.driver_command(case, "drv", "out.json", steps=5, dt=2.0)
    flags = dict(zip(cmd[1::2], cmd[2::2]))
    assert cmd[0] == "drv" and flags["--case"] == "mountain_wave_background"
    assert flags["--nx"] == "96" and flags["--z-top"] == "16000.0"
    assert flags["--terrain-kind"] == "cosine_mountain" and flags["--terrain-half-width-x"] == "0.12"
    assert flags["--terrain-height"] == "800.0" and flags["--u-background"] == "10.0"
    assert flags["--steps"] == "5" and flags["--dt"] == "2.0" and flags["--summary-json"] == "out.json"
    assert "--fast-substeps" not in flags and "--theta-background" not in flags


@pytest.mark.gpu
def test_case_files_run(gwm, tmp_path):
    h = _harness()
    out = tmp_path / "bubble.json"
    assert h.main([os.path.join(CASES_DIR, "warm_bubble.yaml"), "--steps", "3", "--dt", "1",
                   "--fast-substeps", "2", "--summary-json", str(out)]) == 0
    js = json.loads(out.read_text())
    assert js["case"] == "warm_bubble" and js["steps"] == 3
    assert js["final"]["theta_m"]["max"] > 300.0 and js["final"]["w_face"]["max"] > 0.0
    out = tmp_path / "scalar.json"
    s = h.run_scalar_case(h.load_case(os.path.join(CASES_DIR, "scalar_advection.yaml")), str(out))
    assert s["steps"] == 50 and json.loads(out.read_text()) == s
    # upwind SSPRK3 on a periodic grid conserves mass and does not create new extrema
    assert abs(s["final"]["mass"] - s["initial"]["mass"]) <= 1e-3 * abs(s["initial"]["mass"]) + 1e-3
    assert s["initial"]["min"] - 1e-6 <= s["final"]["min"] and s["final"]["max"] <= s["initial"]["max"] + 1e-6


@pytest.mark.gpu
def test_driver_plan_view_bundle(gwm, orc, tmp_path):
    # extract_dry_plan_view + plan_view_bundle_to_json (plan_view_output.cpp:630-713,
    # 950-1003) of the final state: the schema, the field list, and every value against
    # the library's own state diagnosed with the reference's formulas
    nx, ny, nz, level = 32, 16, 12, 3
    args = ["--case", "mountain_wave_background", "--nx", str(nx), "--ny", str(ny), "--nz", str(nz),
            "--z-top", "12000", "--terrain-kind", "cosine_mountain", "--terrain-height", "600",
            "--terrain-half-width-x", "0.2", "--terrain-half-width-y", "0.4", "--u-background", "8",
            "--dt", "1", "--fast-substeps", "2", "--steps", "2", "--plan-view-level", str(level)]
    path = tmp_path / "pv.json"
    r = subprocess.run([_driver(gwm), *args, "--plan-view-json", str(path)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    pv = json.loads(path.read_text())
    assert pv["schema_version"] == "gwm-next-plan-view/v1" and pv["case"] == "mountain_wave_background"
    assert pv["steps"] == 2 and pv["slice_k"] == level and pv["grid"]["nx"] == nx and pv["grid"]["ny"] == ny
    names = [f["name"] for f in pv["fields"]]
    assert names == ["terrain_height", "z_center", "rho_d", "theta_m", "air_pressure", "air_temperature",
                     "u_velocity", "v_velocity", "wind_speed", "w_velocity"]
    f = {x["name"]: np.asarray(x["values"]).reshape(ny, nx) for x in pv["fields"]}
    assert all(x["storage"] == "row_major_yx" and x["location"] == "cell_center" for x in pv["fields"])
    terrain = gwm.build_terrain("cosine_mountain", nx, ny, 1000.0, 1000.0, height=600.0, half_width_x=0.2,
                                half_width_y=0.4)
    g = gwm.GridSpec(nx, ny, nz, dx=1000.0, dy=1000.0, z_top=12000.0, terrain=terrain)
    s0 = gwm.build_case("mountain_wave_background", g, gwm.CaseParams(rho_surface=1.18, theta_ref=300.0,
                                                                      u_background=8.0))
    with gwm.Model(g, gwm.MemberSpec(step=gwm.StepConfig(dt=1.0, fast_substeps=2))) as m:
        m.upload(s0)
        m.advance_dry_state_ssprk3(2)
        s = m.download()
    zc = orc.metrics(orc.GridSpec(nx, ny, nz, dx=1000.0, dy=1000.0, z_top=12000.0,
                                  terrain=terrain))["z_centers"]
    rho = s["rho"][level].astype(np.float64)
    rr = np.maximum(rho, 1e-6)
    th = s["rho_theta"][level] / rr
    p = 1e5 * np.maximum(rho * 287.05 * th / 1e5, 1e-6) ** (1.0 / (1.0 - 0.2854))
    u = 0.5 * (s["u"][level, :, :-1] + s["u"][level, :, 1:]) / rr
    v = 0.5 * (s["v"][level, :-1, :] + s["v"][level, 1:, :]) / rr
    w = 0.5 * (s["w"][level] + s["w"][level + 1]) / rr
    want = {"terrain_height": terrain, "z_center": zc[level], "rho_d": rho, "theta_m": th, "air_pressure": p,
            "air_temperature": th * (np.maximum(p, 1.0) / 1e5) ** 0.2854, "u_velocity": u, "v_velocity": v,
            "wind_speed": np.sqrt(u * u + v * v), "w_velocity": w}
    for k, v_ in want.items():
        scale = max(np.abs(v_).max(), 1e-3)
        assert np.abs(f[k] - v_).max() <= 2e-6 * scale, k
    assert pv["grid"]["slice_mean_height_m"] == pytest.approx(zc[level].mean(), rel=1e-6)
