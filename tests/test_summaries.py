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
