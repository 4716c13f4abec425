"""The runtime-state summary (summarize_runtime_state + runtime_state_summary_to_json,
src/core/runtime_summary.cpp:27-247) reduced on the device, against host sums of the
downloaded fields: the same keys in the reference's order, FP64 values."""
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ["total_dry_mass", "total_rho_theta_m", "total_horizontal_momentum_x", "total_horizontal_momentum_y",
        "total_vertical_momentum", "rho_d", "theta_m", "u_face", "v_face", "w_face", "moisture", "tracers"]
MOISTURE = ["vapor_water_path_sum_kg_m2", "cloud_water_path_sum_kg_m2", "rain_water_path_sum_kg_m2",
            "condensed_water_path_sum_kg_m2", "total_water_path_sum_kg_m2",
            "accumulated_surface_precipitation_sum_mm", "mean_surface_precipitation_mm",
            "max_surface_precipitation_mm", "total_surface_cell_count", "precipitating_surface_cell_count",
            "precipitating_surface_fraction", "mean_precipitating_surface_precipitation_mm"]


def test_runtime_summary_matches_host_sums(gwm, orc):
    g = gwm.GridSpec(40, 32, 16, dx=2000.0, dy=2000.0, z_top=6000.0)
    p = gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=2, relative_humidity=1.04)
    s = gwm.build_case("moist_sounding", g, p, moist=True)
    spec = gwm.MemberSpec(step=gwm.StepConfig(dt=1.0, fast_substeps=3),
                          rain=gwm.WarmRainConfig(dt=1.0, rain_terminal_velocity=40.0), moist=True)
    with gwm.Model(g, spec) as m:
        m.upload(s)
        smoke = m.add_tracer("smoke", units="kg/kg", positive=False)
        m.upload_tracer(smoke, s["rho"] * np.float32(1e-3))
        m.step(30)
        summ = m.runtime_summary()
        out = m.download()
        smoke_mass = m.download_tracer("smoke")
    assert summ["_status"] == 0
    # key order of runtime_state_summary_to_json
    assert list(json.loads(summ["_json"]).keys()) == KEYS
    assert list(summ["moisture"].keys()) == MOISTURE
    assert list(summ["tracers"].keys()) == ["specific_humidity", "cloud_water_mixing_ratio",
                                            "rain_water_mixing_ratio", "smoke"]
    d = {k: v.astype(np.float64) for k, v in out.items()}
    assert summ["total_dry_mass"] == pytest.approx(d["rho"].sum(), rel=1e-13)
    assert summ["rho_d"] == {"min": d["rho"].min(), "max": d["rho"].max()}
    # dz = 1 / inv_dz_cell with the metric in FP32, as runtime_summary.cpp:72-81 takes it
    idz = orc.metrics(orc.GridSpec(g.nx, g.ny, g.nz, dx=g.dx, dy=g.dy, z_top=g.z_top), precision=32)["inv_dz_cell"]
    dz = 1.0 / np.asarray(idz, np.float64).reshape(g.nz, g.ny, g.nx)
    rho = np.maximum(d["rho"], 1e-12)
    for name, key in (("specific_humidity", "qv"), ("cloud_water_mixing_ratio", "qc"),
                      ("rain_water_mixing_ratio", "qr")):
        t = summ["tracers"][name]
        assert t["units"] == "kg/kg" and t["positive"] is True
        assert t["column_integrated_sum_kg_m2"] == pytest.approx((d[key] * dz).sum(), rel=1e-12)
        assert t["mixing_ratio"]["min"] == (d[key] / rho).min()
        assert t["mixing_ratio"]["max"] == (d[key] / rho).max()
    assert summ["tracers"]["smoke"]["positive"] is False
    assert summ["tracers"]["smoke"]["column_integrated_sum_kg_m2"] == pytest.approx(
        (smoke_mass.astype(np.float64) * dz).sum(), rel=1e-12)
    mo = summ["moisture"]
    assert mo["condensed_water_path_sum_kg_m2"] == pytest.approx(
        mo["cloud_water_path_sum_kg_m2"] + mo["rain_water_path_sum_kg_m2"], rel=1e-15)
    pr = d["precip"]
    assert pr.max() > 0                                  # the case precipitates
    assert mo["accumulated_surface_precipitation_sum_mm"] == pytest.approx(pr.sum(), rel=1e-12)
    assert mo["max_surface_precipitation_mm"] == pytest.approx(pr.max(), rel=1e-15)
    assert mo["total_surface_cell_count"] == g.nx * g.ny
    assert mo["precipitating_surface_cell_count"] == int((pr > 0).sum())
    assert mo["mean_precipitating_surface_precipitation_mm"] == pytest.approx(pr[pr > 0].mean(), rel=1e-12)


PREPARED_KEYS = ["case", "source", "cycle_time_utc", "analysis_valid_time_utc", "steps", "dt", "fast_substeps",
                 "enable_boundaries", "enable_fast_modes", "enable_tracer_transport", "enable_warm_rain",
                 "fast_update_horizontal_momentum", "fast_update_density", "warm_rain", "elapsed_seconds",
                 "elapsed_hours", "grid", "surface_runtime", "startup_balance", "initial", "final"]


def _moist_member(gwm, seed=4):
    g = gwm.GridSpec(32, 24, 14, dx=2000.0, dy=2000.0, z_top=7000.0)
    s = gwm.build_case("moist_sounding", g, gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=seed,
                                                           relative_humidity=1.04), moist=True)
    spec = gwm.MemberSpec(step=gwm.StepConfig(dt=1.5, fast_substeps=3),
                          rain=gwm.WarmRainConfig(dt=1.5, rain_terminal_velocity=20.0), moist=True)
    return g, s, spec


def test_prepared_steps_phase_summaries(gwm, tmp_path):
    """gwm_prepared_case_driver.cpp:427-463 with maybe_write_phase_summary (:97-131): the
    selected steps run phase by phase and leave step_<n>_<phase>.json; the state equals
    the graph-replayed step bit for bit."""
    g, s, spec = _moist_member(gwm)
    with gwm.Model(g, spec) as m:
        m.use_graph(True)
        m.upload(s)
        m.step(6)
        want = m.download()
    with gwm.Model(g, spec) as m:
        m.use_graph(True)
        m.upload(s)
        t = m.prepared_steps(6, phase_summary_dir=str(tmp_path), step_min=2, step_max=3)
        got = m.download()
        final = m.runtime_summary(indent="    ")
    for k in want:
        assert np.array_equal(got[k], want[k]), k
    assert t == np.float32(np.float32(1.5) * 6)
    names = sorted(p.name for p in tmp_path.iterdir())
    assert names == sorted(f"step_{n}_{ph}.json" for n in (2, 3) for ph in ("dry", "tracers", "warm_rain"))
    for n in (2, 3):
        for ph in ("dry", "tracers", "warm_rain"):
            text = (tmp_path / f"step_{n}_{ph}.json").read_text()
            doc = json.loads(text)
            assert list(doc) == ["step", "step_start_seconds", "phase", "summary"]
            assert doc["step"] == n and doc["phase"] == ph
            assert doc["step_start_seconds"] == pytest.approx(1.5 * n)
            assert list(doc["summary"]) == KEYS
            assert text.startswith('{\n  "step": ') and text.endswith("\n}\n")
    # the phase summary after the last selected step's rain is the state's summary then;
    # a run to step 4 reproduces it
    with gwm.Model(g, spec) as m:
        m.upload(s)
        m.prepared_steps(4)
        at4 = m.runtime_summary(indent="    ")
    doc = json.loads((tmp_path / "step_3_warm_rain.json").read_text())
    assert doc["summary"] == json.loads(at4["_json"])
    assert final["_status"] == 0


def test_prepared_steps_single_step_selection(gwm, tmp_path):
    g, s, spec = _moist_member(gwm, seed=6)
    with gwm.Model(g, spec) as m:
        m.upload(s)
        m.prepared_steps(3, phase_summary_dir=str(tmp_path), step=1)
    assert sorted(p.name for p in tmp_path.iterdir()) == ["step_1_dry.json", "step_1_tracers.json",
                                                         "step_1_warm_rain.json"]


def test_prepared_summary_layout(gwm):
    g, s, spec = _moist_member(gwm, seed=8)
    with gwm.Model(g, spec) as m:
        m.upload(s)
        initial = m.runtime_summary(indent="    ")["_json"]
        m.prepared_steps(5)
        text = m.prepared_summary(5, initial, source="HRRR", cycle_time_utc="2026-04-04T00:00:00Z",
                                  analysis_valid_time_utc="2026-04-04T01:00:00Z", enable_boundaries=1,
                                  surface_ntile=3, surface_nsoil=4, max_rel_eos=1.5e-7,
                                  max_abs_tracer_closure=2.0e-9)
        final = m.runtime_summary(indent="    ")["_json"]
    doc = json.loads(text)
    assert list(doc) == PREPARED_KEYS
    assert doc["case"] == "prepared_case" and doc["source"] == "HRRR" and doc["steps"] == 5
    assert doc["dt"] == 1.5 and doc["fast_substeps"] == 3 and doc["enable_boundaries"] is True
    assert doc["enable_warm_rain"] is True and doc["warm_rain"]["rain_terminal_velocity"] == 20.0
    assert doc["elapsed_seconds"] == 7.5 and doc["elapsed_hours"] == pytest.approx(7.5 / 3600.0, rel=1e-15)
    assert doc["grid"] == {"nx": 32, "ny": 24, "nz": 14, "dx": 2000.0, "dy": 2000.0, "z_top": 7000.0}
    assert doc["surface_runtime"] == {"ntile": 3, "nsoil": 4}
    assert "max_abs_z_src_minus_metric" not in doc["startup_balance"]
    assert doc["startup_balance"]["max_rel_eos"] == 1.5e-7
    assert doc["initial"] == json.loads(initial) and doc["final"] == json.loads(final)
    assert doc["initial"] != doc["final"]


def test_runtime_summary_reference_kats(gwm):
    """tests/unit/test_runtime_summary.cpp: a 2 x 1 x 1 column pair (1 km deep), rho 1,
    theta 300, qv masses 0.010 / 0.012, qc 0.001 in the first column, qr 0.002 in the
    second, 0.75 mm accumulated over the second."""
    g = gwm.GridSpec(2, 1, 1, dx=1000.0, dy=1000.0, z_top=1000.0)
    s = gwm.build_case("constant", g, gwm.CaseParams(rho_background=1.0, theta_background=300.0), moist=True)
    s["qv"][0, 0, :] = np.float32([0.010, 0.012])
    s["qc"][0, 0, :] = np.float32([0.001, 0.0])
    s["qr"][0, 0, :] = np.float32([0.0, 0.002])
    s["precip"] = np.array([[0.0, np.float32(0.75)]])
    with gwm.Model(g, gwm.MemberSpec(step=gwm.StepConfig(dt=1.0, fast_substeps=1), moist=True)) as m:
        m.upload(s)
        summ = m.runtime_summary()
    mo = summ["moisture"]
    assert mo["vapor_water_path_sum_kg_m2"] == pytest.approx(0.010 * 1000 + 0.012 * 1000, abs=1e-5)
    assert mo["cloud_water_path_sum_kg_m2"] == pytest.approx(1.0, abs=1e-5)
    assert mo["rain_water_path_sum_kg_m2"] == pytest.approx(2.0, abs=1e-5)
    assert mo["condensed_water_path_sum_kg_m2"] == pytest.approx(3.0, abs=1e-5)
    assert mo["total_water_path_sum_kg_m2"] == pytest.approx(25.0, abs=1e-5)
    assert mo["accumulated_surface_precipitation_sum_mm"] == pytest.approx(0.75, abs=1e-6)
    assert mo["mean_surface_precipitation_mm"] == pytest.approx(0.375, abs=1e-6)
    assert mo["max_surface_precipitation_mm"] == pytest.approx(0.75, abs=1e-6)
    tr = summ["tracers"]
    assert len(tr) == 3
    for name, lo, hi in (("specific_humidity", 0.010, 0.012), ("cloud_water_mixing_ratio", 0.0, 0.001),
                         ("rain_water_mixing_ratio", 0.0, 0.002)):
        assert tr[name]["mixing_ratio"]["min"] == pytest.approx(lo, abs=1e-6)
        assert tr[name]["mixing_ratio"]["max"] == pytest.approx(hi, abs=1e-6)
        assert tr[name]["positive"] is True
    for key in ('"specific_humidity"', '"total_water_path_sum_kg_m2"', '"accumulated_surface_precipitation_sum_mm"',
                '"mixing_ratio"'):
        assert key in summ["_json"]


def test_dry_summary_reference_kats(gwm):
    """tests/unit/test_dry_diagnostics.cpp: summarize_dry_states of a constant 4 x 3 x 2
    state (rho 1.5, theta 300, velocities 2, -1, 0.25), face totals over every storage face
    (5 X faces per row, 4 Y faces per column, 3 Z faces per column)."""
    g = gwm.GridSpec(4, 3, 2, dx=1000.0, dy=1000.0, z_top=2000.0)
    s = gwm.build_case("constant", g, gwm.CaseParams(rho_background=1.5, theta_background=300.0, u_background=2.0,
                                                     v_background=-1.0, w_background=0.25))
    with gwm.Model(g, gwm.MemberSpec(step=gwm.StepConfig(dt=1.0, fast_substeps=1))) as m:
        m.upload(s)
        b = m.budgets()
    assert b["total_dry_mass"] == pytest.approx(4 * 3 * 2 * 1.5, abs=1e-6)
    assert b["total_rho_theta_m"] == pytest.approx(4 * 3 * 2 * 1.5 * 300.0, abs=1e-6)
    assert b["total_horizontal_momentum_x"] == pytest.approx(5 * 3 * 2 * 1.5 * 2.0, abs=1e-6)
    assert b["total_horizontal_momentum_y"] == pytest.approx(4 * 4 * 2 * 1.5 * -1.0, abs=1e-6)
    assert b["total_vertical_momentum"] == pytest.approx(4 * 3 * 3 * 1.5 * 0.25, abs=1e-6)
    for key, val in (("rho", 1.5), ("theta", 300.0), ("u", 3.0), ("v", -1.5), ("w", 0.375)):
        assert b[f"{key}_min"] == pytest.approx(val, abs=1e-6) and b[f"{key}_max"] == pytest.approx(val, abs=1e-6)
