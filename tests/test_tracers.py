"""The tracer registry (TracerRegistry / TracerState) and the transport of any number of
passive tracers, through the C-ABI.

Reference semantics (include/gwm/state/tracer_registry.hpp:23-62): names are unique,
add returns the new index, find returns the index or nothing, a moist state starts with
the warm-rain registry.  advance_passive_tracers_ssprk3 (src/dycore/dry_transport.cu:
440-518) advances every tracer of the state on its own, so a tracer added by name must be
transported exactly as the warm-rain tracers are, whatever group of the kernel it lands in.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _moist_member(gwm, rain=True, nx=48, ny=40, nz=14, terrain=False):
    kw = {}
    if terrain:  # a cosine hill: the tracer stage takes the per-cell inverse layer depth
        kw["terrain"] = gwm.build_terrain("cosine_mountain", nx, ny, 2000.0, 2000.0, height=600.0,
                                          half_width_x=0.3, half_width_y=0.3)
    g = gwm.GridSpec(nx, ny, nz, dx=2000.0, dy=2000.0, z_top=8000.0, **kw)
    p = gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=8, relative_humidity=1.02)
    s = gwm.build_case("moist_sounding", g, p, moist=True)
    s["u"][:] = np.float32(3.0)
    s["v"][:] = np.float32(-2.0)
    spec = gwm.MemberSpec(step=gwm.StepConfig(dt=1.0, fast_substeps=3),
                          rain=gwm.WarmRainConfig(dt=1.0, rain_terminal_velocity=12.0), moist=True,
                          enable_warm_rain=rain)
    return g, s, spec


def test_registry_names_add_find(gwm):
    g, s, spec = _moist_member(gwm)
    with gwm.Model(g, spec) as m:
        assert m.tracer_names() == ["specific_humidity", "cloud_water_mixing_ratio", "rain_water_mixing_ratio"]
        assert m.find_tracer("rain_water_mixing_ratio") == 2
        assert m.find_tracer("smoke") is None
        assert m.add_tracer("smoke") == 3
        assert m.add_tracer("dust", units="kg/kg") == 4
        with pytest.raises(RuntimeError, match="already exists"):
            m.add_tracer("smoke")
        assert m.find_tracer("dust") == 4 and m.tracer_names()[3:] == ["smoke", "dust"]
        assert not m.download_tracer("dust").any()          # a new tracer starts at zero
    with gwm.Model(g, gwm.MemberSpec(step=spec.step)) as dry:
        assert dry.tracer_names() == []
        assert dry.add_tracer("smoke") == 0


@pytest.mark.parametrize("tile,terrain", [(3, False), (16, False), (3, True), (16, True)])
def test_added_tracers_move_like_the_warm_rain_tracers(gwm, tile, terrain):
    # warm rain off, so qv, qc and qr are passive too: tracers added by name and started
    # from the same fields must come out bit-identical, in the second kernel group (3-5)
    # and in a partial third group (6), on flat levels and over terrain
    g, s, spec = _moist_member(gwm, rain=False, terrain=terrain)
    with gwm.Model(g, spec) as m:
        m.set_tile("tracer_stage", tile)
        m.upload(s)
        for name, key in (("a", "qv"), ("b", "qc"), ("c", "qr"), ("d", "qv")):
            i = m.add_tracer(name)
            m.upload_tracer(i, s[key])
        total0 = m.tracer_total("a")
        m.step(3)
        out = m.download()
        for name, key in (("a", "qv"), ("b", "qc"), ("c", "qr"), ("d", "qv")):
            assert np.array_equal(m.download_tracer(name), out[key]), name
        # periodic domain on flat levels: the transport conserves each tracer's mass (the
        # total is the plain sum of rho*q over cells, which over terrain would need the
        # cells' depths as weights)
        if not terrain:
            assert m.tracer_total("a") == pytest.approx(total0, rel=2e-6)
        assert m.tracer_total(0) == pytest.approx(float(out["qv"].astype(np.float64).sum()), rel=1e-12)


def test_dry_member_with_four_tracers_vs_oracle(gwm, orc):
    # a dry member with four registered tracers (groups of three and one) against the
    # oracle's passive-tracer transport of the same fields
    g = gwm.GridSpec(40, 32, 12, dx=2000.0, dy=2000.0, z_top=8000.0)
    p = gwm.CaseParams(rho_background=1.0, theta_background=300.0, theta_perturbation=3.0,
                       center_z_fraction=0.35, radius_x_fraction=0.2, radius_y_fraction=0.2,
                       radius_z_fraction=0.3)
    s = gwm.build_case("density_current", g, p)
    s["u"][:] = np.float32(4.0)
    rng = np.random.default_rng(3)
    zz, yy, xx = np.meshgrid(np.arange(g.nz), np.arange(g.ny), np.arange(g.nx), indexing="ij")
    fields = [(s["rho"] * np.exp(-((xx - 12) ** 2 + (yy - 10) ** 2 + (zz - 4) ** 2) / 20.0)).astype(np.float32),
              (s["rho"] * rng.uniform(0, 1e-3, s["rho"].shape)).astype(np.float32),
              (s["rho"] * (zz / g.nz) * 1e-2).astype(np.float32)]
    step = gwm.StepConfig(dt=1.0, fast_substeps=3)
    with gwm.Model(g, gwm.MemberSpec(step=step)) as m:
        m.upload(s)
        for n, f in zip(("t0", "t1", "t2", "t3"), fields + [fields[0]]):
            m.upload_tracer(m.add_tracer(n), f)
        m.step(2)
        got = [m.download_tracer(n) for n in ("t0", "t1", "t2", "t3")]
        dry = m.download()
    st = {k: v.astype(np.float64) for k, v in s.items()}
    st.update(qv=fields[0].astype(np.float64), qc=fields[1].astype(np.float64), qr=fields[2].astype(np.float64),
              precip=np.zeros((g.ny, g.nx)))
    og = orc.GridSpec(g.nx, g.ny, g.nz, dx=g.dx, dy=g.dy, z_top=g.z_top)
    ost = orc.StepSpec(dt=1.0, fast_substeps=3)
    ref = orc.run(og, ost, st, 2, phases=orc.PHASE_DRY | orc.PHASE_TRACERS, precision=64)
    ref32 = orc.run(og, ost, st, 2, phases=orc.PHASE_DRY | orc.PHASE_TRACERS, precision=32)
    assert np.array_equal(got[3], got[0])
    for out, key in zip(got[:3], ("qv", "qc", "qr")):
        e = np.abs(out - ref[key]).max() / np.abs(ref[key]).max()
        e32 = np.abs(ref32[key] - ref[key]).max() / np.abs(ref[key]).max()
        assert e <= max(2.0 * e32, 1e-6), (key, e, e32)
    assert np.abs(dry["rho"] - ref["rho"]).max() / ref["rho"].max() < 1e-5
