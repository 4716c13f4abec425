"""The runtime plan view (extract_runtime_plan_view over extract_dry_plan_view,
src/io/plan_view_output.cpp:630-834, and plan_view_bundle_to_json :950-1003).

* The oracle's restatement against the known answers of the reference's own unit test
  (tests/unit/test_plan_view_output.cpp:54-214: a constant 6 x 4 x 3 state on 2 x 1
  virtual ranks; the dry, specific-humidity and warm-rain bundles) and against the
  reference's plan view of its own stepped states (``tests/golden/ref_pv_*.npz``).
* The device computation (``gwm_b200_plan_view``) on the same inputs, on a stepped moist
  member against the oracle, and the JSON writer's layout.

Tolerances: values without a transcendental function are equal bit for bit; pressure,
temperature, relative humidity, dewpoint and reflectivity go through powf/expf/logf/log10f,
whose device and host implementations may differ in the last bits, so those compare to
4e-6 relative (a few FP32 ulps, amplified at most by the dewpoint's logarithm)."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
TRANSCENDENTAL = {"air_pressure", "air_temperature", "relative_humidity", "dewpoint", "synthetic_reflectivity"}
KEYS = ("rho", "rho_theta", "u", "v", "w", "qv", "qc", "qr")


def _constant_state(nx=6, ny=4, nz=3, rho=1.2, theta=300.0, u=10.0, v=-4.0, w=0.5, q=None, precip=None):
    """make_constant_dry_state (momenta = rho * velocity) plus tracer masses rho * q."""
    f32 = np.float32
    s = {"rho": np.full((nz, ny, nx), rho, f32), "rho_theta": np.full((nz, ny, nx), f32(rho) * f32(theta), f32),
         "u": np.full((nz, ny, nx + 1), f32(rho) * f32(u), f32), "v": np.full((nz, ny + 1, nx), f32(rho) * f32(v), f32),
         "w": np.full((nz + 1, ny, nx), f32(rho) * f32(w), f32)}
    if q is not None:
        for k, val in zip(("qv", "qc", "qr"), q):
            s[k] = (s["rho"] * f32(val)).astype(f32)
    if precip is not None:
        s["precip"] = precip
    return s


def _pressure(rho, rt):  # dry_pressure_from_rho_theta_m in FP32
    f32 = np.float32
    th = f32(rt) / max(f32(rho), f32(1e-6))
    ratio = max(f32(rho) * f32(287.05) * th / f32(100000.0), f32(1e-6))
    return float(f32(100000.0) * np.power(ratio, f32(1.0) / (f32(1.0) - f32(0.2854)), dtype=f32))


def _kats(pv, nfields):
    """test_plan_view_output.cpp:85-214 on a bundle (first value of each field)."""
    assert len(pv) == nfields
    first = {k: float(np.asarray(v).ravel()[0]) for k, v in pv.items() if not k.startswith("_")}
    assert first["rho_d"] == pytest.approx(1.2, abs=1e-6)
    assert first["theta_m"] == pytest.approx(300.0, abs=1e-4)
    assert first["u_velocity"] == pytest.approx(10.0, abs=1e-5)
    assert first["v_velocity"] == pytest.approx(-4.0, abs=1e-5)
    assert first["w_velocity"] == pytest.approx(0.5, abs=1e-6)
    assert first["wind_speed"] == pytest.approx(np.sqrt(116.0), abs=1e-5)
    assert first["terrain_height"] == 0.0
    assert first["z_center"] == pytest.approx(4500.0, abs=1e-6)
    p = _pressure(1.2, np.float32(1.2) * np.float32(300.0))
    assert first["air_pressure"] == pytest.approx(p, abs=1e-4 * p)
    assert first["air_temperature"] == pytest.approx(300.0 * (p / 1e5) ** 0.2854, abs=1e-3)
    if nfields >= 13:
        assert first["specific_humidity"] == pytest.approx(0.004, abs=1e-6)
        assert 0.0 < first["relative_humidity"] <= 100.0
        assert first["dewpoint"] < first["air_temperature"]
    if nfields >= 21:
        assert first["cloud_water_mixing_ratio"] == pytest.approx(0.001, abs=1e-6)
        assert first["rain_water_mixing_ratio"] == pytest.approx(0.0005, abs=1e-6)
        assert first["total_condensate"] == pytest.approx(0.0015, abs=1e-6)
        assert first["column_cloud_water"] == pytest.approx(10.8, abs=1e-5)
        assert first["column_rain_water"] == pytest.approx(5.4, abs=1e-5)
        assert first["column_total_condensate"] == pytest.approx(16.2, abs=1e-5)
        assert first["column_rain_fraction"] == pytest.approx(1.0 / 3.0, abs=1e-6)
        assert first["synthetic_reflectivity"] <= 75.0
    if nfields >= 23:
        assert first["accumulated_surface_precipitation"] == pytest.approx(0.25, abs=1e-6)
        assert first["mean_surface_precipitation_rate"] == pytest.approx(112.5, abs=1e-6)


def _kat_precip():
    pr = np.zeros((4, 6))
    pr[0, 0] = pr[0, 3] = np.float32(0.25)  # (0, 0) of each of the 2 x 1 ranks
    return pr


# the reference (and the oracle restating it) holds the surface accumulation in FP32;
# this path keeps it in FP64 with a compensation term
PRECIP = {"accumulated_surface_precipitation", "mean_surface_precipitation_rate"}


def _compare(got, want, tag=""):
    for name, w in want.items():
        g = np.asarray(got[name], np.float64)
        w = np.asarray(w, np.float64)
        if name in PRECIP:
            assert np.allclose(g, w, rtol=6e-8, atol=0.0), f"{tag} {name}: max |diff| {np.abs(g - w).max():.3e}"
        elif name in TRANSCENDENTAL:
            scale = np.maximum(np.abs(w), 1e-30)
            err = float((np.abs(g - w) / scale).max())
            assert err <= 4e-6, f"{tag} {name}: relative {err:.3e}"
        else:
            assert np.array_equal(g, w), f"{tag} {name}: max |diff| {np.abs(g - w).max():.3e}"


def _fixtures():
    return sorted(f for f in os.listdir(GOLDEN) if f.startswith("ref_pv_") and f.endswith(".npz"))


def _fixture(name):
    z = np.load(os.path.join(GOLDEN, name))
    spec = json.loads(bytes(z["spec"]).decode())
    bundle = json.loads(bytes(z["plan_view_json"]).decode())
    return z, spec, bundle


def _bundle_fields(bundle):
    return {f["name"]: np.asarray(f["values"], np.float64).reshape(f["ny"], f["nx"]) for f in bundle["fields"]}


# ---------------------------------------------------------------------------- CPU
def test_oracle_plan_view_reference_kats(orc):
    g = orc.GridSpec(6, 4, 3, dx=1000.0, dy=1000.0, z_top=9000.0, ranks_x=2)
    dry = orc.plan_view(g, {k: v.astype(np.float64) for k, v in _constant_state().items()}, 1, 4, 2.0)
    _kats(dry, 10)
    s = {k: v.astype(np.float64) for k, v in _constant_state(q=(0.004, 0.0, 0.0)).items()}
    _kats(orc.plan_view(g, s, 1, 4, 2.0, nfields=13), 13)
    s = {k: np.asarray(v, np.float64) for k, v in _constant_state(q=(0.004, 0.001, 0.0005),
                                                                  precip=_kat_precip()).items()}
    _kats(orc.plan_view(g, s, 1, 4, 2.0), 23)


@pytest.mark.parametrize("name", _fixtures())
def test_oracle_plan_view_matches_reference(orc, name):
    z, spec, bundle = _fixture(name)
    gk = spec["grid"]
    terrain = z["terrain"].astype(np.float64) if "terrain" in spec else None
    g = orc.GridSpec(gk["nx"], gk["ny"], gk["nz"], dx=gk["dx"], dy=gk["dy"], z_top=gk["z_top"],
                     periodic_x=gk.get("periodic_x", True), periodic_y=gk.get("periodic_y", True), terrain=terrain)
    state = {k: z["out_" + k].astype(np.float64) for k in KEYS + ("precip",) if "out_" + k in z.files}
    ref = _bundle_fields(bundle)
    got = orc.plan_view(g, state, spec["level"], spec["steps"], spec["step"]["dt"])
    assert list(got) == [f["name"] for f in bundle["fields"]]
    # the reference's JSON holds 10 significant digits
    for k, w in ref.items():
        assert np.allclose(got[k], w, rtol=2e-9, atol=1e-300), k
    assert bundle["slice_k"] == spec["level"] and bundle["steps"] == spec["steps"]


# ---------------------------------------------------------------------------- GPU
def _member(gwm, s, nz=3, nx=6, ny=4, z_top=9000.0, moist=True):
    g = gwm.GridSpec(nx, ny, nz, dx=1000.0, dy=1000.0, z_top=z_top)
    return g, gwm.MemberSpec(step=gwm.StepConfig(dt=2.0, fast_substeps=2), moist=moist)


@pytest.mark.gpu
def test_plan_view_reference_kats_on_device(gwm, orc):
    g, spec = _member(gwm, None, moist=False)
    with gwm.Model(g, spec) as m:
        m.upload(_constant_state())
        pv = m.plan_view(1, 4, 2.0)
    _kats({k: v for k, v in pv.items() if k != "_units"}, 10)
    g, spec = _member(gwm, None, moist=True)
    s = _constant_state(q=(0.004, 0.001, 0.0005), precip=_kat_precip())
    with gwm.Model(g, spec) as m:
        m.upload(s)
        pv = m.plan_view(1, 4, 2.0)
    _kats({k: v for k, v in pv.items() if k != "_units"}, 23)
    assert pv["_units"]["synthetic_reflectivity"] == "dBZ" and pv["_units"]["relative_humidity"] == "%"
    og = orc.GridSpec(6, 4, 3, dx=1000.0, dy=1000.0, z_top=9000.0)
    _compare(pv, orc.plan_view(og, {k: np.asarray(v, np.float64) for k, v in s.items()}, 1, 4, 2.0), "kat")


@pytest.mark.gpu
def test_plan_view_vapour_only_and_missing_humidity(gwm):
    g, spec = _member(gwm, None, moist=False)
    with gwm.Model(g, spec) as m:
        m.upload(_constant_state())
        t = m.add_tracer("smoke")
        m.upload_tracer(t, np.full((3, 4, 6), 1e-3, np.float32))
        with pytest.raises(RuntimeError, match="specific_humidity"):
            m.plan_view(1)
    with gwm.Model(g, spec) as m:
        m.upload(_constant_state())
        t = m.add_tracer("specific_humidity")
        m.upload_tracer(t, np.full((3, 4, 6), np.float32(1.2) * np.float32(0.004), np.float32))
        pv = m.plan_view(1, 4, 2.0)
    _kats({k: v for k, v in pv.items() if k != "_units"}, 13)


@pytest.mark.gpu
@pytest.mark.parametrize("name", _fixtures())
def test_plan_view_matches_reference_on_device(gwm, orc, name):
    z, spec, bundle = _fixture(name)
    gk = dict(spec["grid"])
    gk.pop("ranks_x", None), gk.pop("ranks_y", None)
    if "terrain" in spec:
        gk["terrain"] = z["terrain"]
    g = gwm.GridSpec(**gk)
    moist = spec.get("moist", False)
    state = {k: z["out_" + k] for k in KEYS if "out_" + k in z.files}
    if moist:
        state["precip"] = z["out_precip"].astype(np.float64)
    with gwm.Model(g, gwm.MemberSpec(step=gwm.StepConfig(dt=spec["step"]["dt"]), moist=moist)) as m:
        m.upload(state)
        pv = m.plan_view(spec["level"], spec["steps"], spec["step"]["dt"])
        text = m.plan_view_json(spec["level"], "golden", spec["steps"], spec["step"]["dt"])
    ref = _bundle_fields(bundle)
    assert [k for k in pv if k != "_units"] == list(ref)
    for k, w in ref.items():  # the reference's JSON holds 10 significant digits
        tol = 4e-6 if k in TRANSCENDENTAL else 2e-9
        assert np.allclose(pv[k], w, rtol=tol, atol=1e-300), k
    # the writer's layout and metadata equal the reference's bundle
    mine = json.loads(text)
    assert {k: v for k, v in mine.items() if k != "fields"} == {k: v for k, v in bundle.items() if k != "fields"}
    for a, b in zip(mine["fields"], bundle["fields"]):
        assert {k: v for k, v in a.items() if k != "values"} == {k: v for k, v in b.items() if k != "values"}
    assert text.count('"storage": "row_major_yx"') == len(ref)


@pytest.mark.gpu
def test_plan_view_of_a_raining_member_vs_oracle(gwm, orc):
    """A moist member stepped until rain reaches the ground; the device plan view of
    its state against the oracle's on the downloaded state."""
    nx, ny, nz = 48, 40, 20
    g = gwm.GridSpec(nx, ny, nz, dx=2000.0, dy=2000.0, z_top=8000.0)
    s = gwm.build_case("moist_sounding", g, gwm.CaseParams(theta_ref=300.0, relative_humidity=1.04,
                                                           noise_rms_k=0.5, seed=11), moist=True)
    j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    bump = np.exp(-((i - nx / 2) ** 2 + (j - ny / 2) ** 2) / 50.0)[None] * (np.arange(nz) < 8)[:, None, None]
    s["qr"] = (s["qr"] + s["rho"] * np.float32(1e-3) * bump).astype(np.float32)
    # dt 1 s on 400 m levels (c dt / dz = 0.85, inside the acoustic limit of the scheme)
    spec = gwm.MemberSpec(step=gwm.StepConfig(dt=1.0, fast_substeps=3),
                          rain=gwm.WarmRainConfig(dt=1.0, rain_terminal_velocity=10.0), moist=True)
    with gwm.Model(g, spec) as m:
        m.upload(s)
        m.step(20)
        out = m.download()
        pv = m.plan_view(4, 20, 1.0)
    assert out["precip"].max() > 0 and len(pv) - 1 == 23
    og = orc.GridSpec(nx, ny, nz, dx=2000.0, dy=2000.0, z_top=8000.0)
    assert all(np.isfinite(v).all() for v in out.values())
    want = orc.plan_view(og, {k: np.asarray(v, np.float64) for k, v in out.items()}, 4, 20, 1.0)
    _compare(pv, want, "raining")
