"""GPU parity: the CUDA path (through the C-ABI) against the CPU oracle.

Integer/index work (halo maps) must match bit-exactly.  Floating-point fields
are compared with the FP64 oracle of the same discretisation; the tolerance is
stated per test as a maximum error relative to the field's largest magnitude
(the dynamic fields carry FP32 rounding, the oracle none).
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STATE = ("rho", "rho_theta", "u", "v", "w")


def rel_err(a, b, floor=1e-12):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), floor))


def perturbation_err(a, b, base):
    """max |a-b| relative to the largest departure of b from a base field."""
    a, b, base = (np.asarray(x, dtype=np.float64) for x in (a, b, base))
    return float(np.abs(a - b).max() / max(np.abs(b - base).max(), 1e-12))


def to64(d):
    return {k: np.asarray(v, dtype=np.float64) for k, v in d.items()}


def assert_envelope(out, ref64, ref32, keys, base=None, floor=1e-6, factor=2.0, tag=""):
    """The CUDA result must sit inside the FP32 rounding envelope of the reference
    discretisation: its error against the FP64 oracle may not exceed ``factor``
    times the error of the FP32 oracle (the reference arithmetic replayed on the
    CPU) against the same FP64 oracle, nor ``floor`` when that envelope is smaller.
    Errors are maxima relative to the field's largest magnitude, or to its largest
    departure from ``base`` when a base state is given."""
    report = {}
    for k in keys:
        if base is not None and k in base:
            e_gpu = perturbation_err(out[k], ref64[k], base[k])
            e_32 = perturbation_err(ref32[k], ref64[k], base[k])
        else:
            e_gpu = rel_err(out[k], ref64[k], floor=1e-12)
            e_32 = rel_err(ref32[k], ref64[k], floor=1e-12)
        report[k] = (e_gpu, e_32)
        assert np.all(np.isfinite(out[k])), f"{tag} {k}: non-finite values"
        assert e_gpu <= max(factor * e_32, floor), f"{tag} {k}: gpu {e_gpu:.3e} vs fp32 envelope {e_32:.3e}"
    return report


def ogrid(orc, g):
    return orc.GridSpec(g.nx, g.ny, g.nz, dx=g.dx, dy=g.dy, z_top=g.z_top, ranks_x=g.ranks_x,
                        ranks_y=g.ranks_y, periodic_x=g.periodic_x, periodic_y=g.periodic_y,
                        terrain=None if g.terrain is None else g.terrain.astype(np.float64),
                        eta_interfaces=g.eta_interfaces)


def ostep(orc, s):
    return orc.StepSpec(dt=s.dt, fast_substeps=s.fast_substeps, gravity=s.gravity,
                        fast_hmom=s.fast_update_horizontal_momentum,
                        fast_density=s.fast_update_density, fast_modes=s.enable_fast_modes)


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


def test_native_library_loaded(gwm, torch_cuda):
    gwm.lib()
    maps = open("/proc/self/maps").read()
    assert "libgwm_b200.so" in maps


# ---------------------------------------------------------------------------
LAYOUTS = [(8, 8, 2, 1, 2, 2, True, True), (13, 7, 3, 1, 3, 2, False, True),
           (10, 9, 2, 1, 1, 3, True, False), (6, 5, 2, 1, 1, 1, False, False),
           (9, 9, 2, 2, 2, 2, True, True), (7, 6, 2, 1, 1, 1, True, True)]


@pytest.mark.parametrize("lay", LAYOUTS)
@pytest.mark.parametrize("orient", [0, 1, 2, 3])
@pytest.mark.parametrize("op", ["exchange", "sync"])
def test_halo_ops_bit_exact(gwm, orc, torch_cuda, lay, orient, op):
    if op == "sync" and orient in (0, 3):
        pytest.skip("interface sync is defined for X and Y faces")
    torch = torch_cuda
    nx, ny, nz, h, rx, ry, px, py = lay
    rows = orc.layout(nx, ny, nz, h, rx, ry, px, py)
    name = {0: "cell", 1: "x", 2: "y", 3: "z"}[orient]
    host, dev = [], []
    rng = np.random.default_rng(orient * 7 + len(rows))
    for row in rows:
        shape = orc.rank_field_shape(row, nz, h, name)
        a = np.full(shape, -999.0)
        fz, fy, fx = shape
        i0, j0 = int(row[3]), int(row[5])
        for k in range(fz):
            for j in range(fy - 2 * h):
                for i in range(fx - 2 * h):
                    a[k, j + h, i + h] = 1000 * k + 100 * (j0 + j) + (i0 + i) + rng.integers(0, 3) * 0.25
        host.append(a)
        dev.append(torch.tensor(a.astype(np.float32), device="cuda"))
    ref = orc.halo([x.copy() for x in host], nx, ny, nz, h, rx, ry, px, py, name, op=op)
    gwm.halo_exchange([t.data_ptr() for t in dev], nx, ny, nz, h, rx, ry, px, py, orient, op=op)
    torch.cuda.synchronize()
    for r, (t, b) in enumerate(zip(dev, ref)):
        got = t.cpu().numpy().astype(np.float64)
        assert np.array_equal(got, b), f"rank {r}: {np.argwhere(got != b)[:5]}"


def test_dry_pressure_matches_reference_formula(gwm, orc, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(1)
    rho = rng.uniform(0.05, 1.3, 100000).astype(np.float32)
    rt = (rho * rng.uniform(280.0, 500.0, rho.size)).astype(np.float32)
    r, t = torch.tensor(rho, device="cuda"), torch.tensor(rt, device="cuda")
    p = torch.empty_like(r)
    gwm.dry_pressure(r.data_ptr(), t.data_ptr(), p.data_ptr(), rho.size)
    torch.cuda.synchronize()
    ref = orc.pressure(rho, rt, precision=64)
    # FP32 powf against the FP64 formula: a few ulp
    assert rel_err(p.cpu().numpy(), ref) < 1e-6
    assert np.max(np.abs(p.cpu().numpy() / ref - 1.0)) < 2e-6


# ---------------------------------------------------------------------------
def bubble_grid(gwm, nx=32, ny=32, nz=40, **kw):
    return gwm.GridSpec(nx, ny, nz, dx=500.0, dy=500.0, z_top=10000.0, **kw)


def c1_state(gwm, g, u=0.0, v=0.0):
    # C1 warm bubble: +2 K cos^2 bubble (2 km radius, z = 2 km) on a 300 K hydrostatic base
    p = gwm.CaseParams(rho_surface=np.float32(1e5 / (287.05 * 300.0)), theta_ref=300.0,
                       theta_perturbation=2.0, center_x_fraction=0.5, center_y_fraction=0.5,
                       center_z_fraction=0.2, radius_x_fraction=2000.0 / (g.nx * g.dx),
                       radius_y_fraction=2000.0 / (g.ny * g.dy), radius_z_fraction=0.2,
                       u_background=u, v_background=v)
    s = gwm.build_case("hydrostatic_warm_bubble", g, p)
    if u or v:
        s["u"] = (np.full_like(s["u"], u) * 1.1).astype(np.float32)
        s["v"] = (np.full_like(s["v"], v) * 1.1).astype(np.float32)
    return s


@pytest.mark.parametrize("variant", ["flat", "terrain", "open"])
def test_slow_tendencies_vs_oracle(gwm, orc, variant):
    kw = {}
    if variant == "terrain":
        kw["terrain"] = gwm.build_terrain("cosine_mountain", 24, 20, 500.0, 500.0, height=500.0,
                                          half_width_x=0.3, half_width_y=0.3)
    if variant == "open":
        kw.update(periodic_x=False, periodic_y=False)
    g = bubble_grid(gwm, 24, 20, 16, **kw)
    s = c1_state(gwm, g, u=3.0, v=-2.0)
    rng = np.random.default_rng(5)
    s["w"] = (rng.standard_normal(s["w"].shape) * 0.2).astype(np.float32)
    s["w"][0] = 0.0
    s["w"][-1] = 0.0
    step = gwm.StepConfig(dt=2.0, fast_substeps=3)
    with gwm.Model(g, gwm.MemberSpec(step=step)) as m:
        m.upload(s)
        t = m.compute_slow_tendencies()
    ref = orc.slow_tendencies(ogrid(orc, g), ostep(orc, step), to64(s), precision=64)
    ref32 = orc.slow_tendencies(ogrid(orc, g), ostep(orc, step), to64(s), precision=32)
    # the pressure-gradient part differences FP32 pressures of ~1e5 Pa: the FP32
    # envelope, not 1e-7, bounds these tendencies (reference arithmetic included)
    rep = assert_envelope(t, ref, ref32, STATE, floor=2e-5, tag=variant)
    assert max(v[0] for v in rep.values()) < 5e-4, rep


def test_fast_modes_reference_kats(gwm):
    # tests/unit/test_dry_fast_modes.cpp:65-192 through the CUDA path
    g = gwm.GridSpec(20, 20, 8)
    const = gwm.build_case("constant", g, gwm.CaseParams(rho_background=1.1, theta_background=300.0,
                                                         u_background=12.0, v_background=-6.0))
    with gwm.Model(g, gwm.MemberSpec(step=gwm.StepConfig(dt=2.0, fast_substeps=4))) as m:
        m.upload(const)
        b0 = m.budgets()
        m.fast_modes()
        b1 = m.budgets()
    assert abs(b1["total_dry_mass"] - b0["total_dry_mass"]) < 1e-4
    assert abs(b1["u_max"] - b0["u_max"]) < 1e-5 and abs(b1["v_min"] - b0["v_min"]) < 1e-5

    def pulse():
        s = gwm.build_case("constant", g, gwm.CaseParams(rho_background=1.0, theta_background=300.0))
        s["rho"][4, 10, 10] += np.float32(0.02)
        s["rho_theta"][4, 10, 10] = s["rho"][4, 10, 10] * np.float32(300.0)
        return s

    def run(step, n=1):
        with gwm.Model(g, gwm.MemberSpec(step=step)) as m:
            m.upload(pulse())
            b0 = m.budgets()
            for _ in range(n):
                m.fast_modes()
            return b0, m.budgets(), m.download()

    b0, b1, _ = run(gwm.StepConfig(dt=1.0, fast_substeps=4), 3)
    assert abs(b1["total_dry_mass"] - b0["total_dry_mass"]) < 1e-3
    for hmom in (True, False):
        b0, b1, out = run(gwm.StepConfig(dt=1.0, fast_substeps=1, fast_update_horizontal_momentum=hmom,
                                         fast_update_density=False))
        assert abs(b1["total_dry_mass"] - b0["total_dry_mass"]) < 1e-5
        mag = max(abs(b1["u_min"]), abs(b1["u_max"]))
        assert (mag > 1e-5) if hmom else (mag < 1e-8)
        assert abs(b1["rho_max"] - 1.02) < 1e-6 and abs(b1["rho_min"] - 1.0) < 1e-6
    b0, b1, _ = run(gwm.StepConfig(dt=1.0, fast_substeps=1, fast_update_horizontal_momentum=False,
                                   fast_update_density=True))
    assert abs(b1["total_dry_mass"] - b0["total_dry_mass"]) < 1e-5
    assert abs(b1["rho_max"] - 1.02) > 1e-5


@pytest.mark.parametrize("terrain", [False, True])
def test_fast_modes_vs_oracle(gwm, orc, terrain):
    kw = {}
    if terrain:
        kw["terrain"] = gwm.build_terrain("cosine_mountain", 20, 18, 1000.0, 1000.0, height=800.0,
                                          half_width_x=0.3, half_width_y=0.3)
    g = gwm.GridSpec(20, 18, 12, dx=1000.0, dy=1000.0, z_top=12000.0, **kw)
    s = gwm.build_case("mountain_wave_background", g, gwm.CaseParams(rho_surface=1.18, theta_ref=300.0,
                                                                     u_background=10.0))
    s["rho"][5, 9, 10] *= np.float32(1.01)
    s["rho_theta"][5, 9, 10] = s["rho"][5, 9, 10] * np.float32(300.0)
    step = gwm.StepConfig(dt=4.0, fast_substeps=4)
    with gwm.Model(g, gwm.MemberSpec(step=step)) as m:
        m.upload(s)
        m.fast_modes()
        out = m.download()
    ref = orc.fast_modes(ogrid(orc, g), ostep(orc, step), to64(s), precision=64)
    ref32 = orc.fast_modes(ogrid(orc, g), ostep(orc, step), to64(s), precision=32)
    base = to64(s)
    assert rel_err(out["rho"], ref["rho"]) < 1e-6
    assert rel_err(out["rho_theta"], ref["rho_theta"]) < 1e-6
    assert_envelope(out, ref, ref32, ("u", "v", "w"), base=base, floor=1e-4, tag=f"terrain={terrain}")


# ---------------------------------------------------------------------------
def run_both(gwm, orc, g, step, state, nsteps, graph=False):
    with gwm.Model(g, gwm.MemberSpec(step=step)) as m:
        m.use_graph(graph)
        m.upload(state)
        m.advance_dry_state_ssprk3(nsteps)
        out = m.download()
    ref = orc.run(ogrid(orc, g), ostep(orc, step), to64(state), nsteps, precision=64)
    ref32 = orc.run(ogrid(orc, g), ostep(orc, step), to64(state), nsteps, precision=32)
    return out, ref, ref32


@pytest.mark.parametrize("dt,nsteps", [(2.0, 1), (0.5, 4)])
def test_c1_warm_bubble_vs_fp64_oracle(gwm, orc, dt, nsteps):
    # C1 grid and state: 32x32x40, 500 m, dz 250 m, 3 acoustic substeps.
    # At the configured dt = 2 s the reference discretisation is unstable from the
    # second step on (c*dt/dz = 2.8 in the slow stage; the FP64 oracle reaches
    # |w| ~ 1e19 at step 2), so the exact configuration is compared over one step
    # and the 4-step comparison runs at dt = 0.5 s.
    g = bubble_grid(gwm)
    step = gwm.StepConfig(dt=dt, fast_substeps=3)
    s = c1_state(gwm, g)
    out, ref, ref32 = run_both(gwm, orc, g, step, s, nsteps)
    base = to64(s)
    assert_envelope(out, ref, ref32, ("rho", "rho_theta"), floor=1e-6, tag="c1")
    rep = assert_envelope(out, ref, ref32, ("u", "v", "w", "rho"), base=base, floor=1e-4, tag="c1")
    if dt == 0.5:  # the stable run stays inside the north-star bound outright
        assert max(rep[k][0] for k in ("u", "v", "w")) < 1e-3, rep


@pytest.mark.parametrize("variant", ["terrain", "open", "ranks"])
def test_dry_step_variants_vs_oracle(gwm, orc, variant):
    kw = {}
    if variant == "terrain":
        kw["terrain"] = gwm.build_terrain("cosine_mountain", 24, 20, 1000.0, 1000.0, height=600.0,
                                          half_width_x=0.3, half_width_y=0.3)
    if variant == "open":
        kw.update(periodic_x=False, periodic_y=True)
    if variant == "ranks":
        kw.update(ranks_x=2, ranks_y=2)
    g = gwm.GridSpec(24, 20, 16, dx=1000.0, dy=1000.0, z_top=12000.0, **kw)
    if variant == "terrain":
        s = gwm.build_case("mountain_wave_background", g, gwm.CaseParams(rho_surface=1.18, theta_ref=300.0,
                                                                         u_background=10.0))
    else:
        s = gwm.build_case("density_current", g, gwm.CaseParams(rho_background=1.0, theta_background=300.0,
                                                                theta_perturbation=3.0, center_z_fraction=0.35,
                                                                radius_x_fraction=0.15, radius_y_fraction=0.15,
                                                                radius_z_fraction=0.2))
    step = gwm.StepConfig(dt=2.0, fast_substeps=3)
    out, ref, ref32 = run_both(gwm, orc, g, step, s, 3)
    base = to64(s)
    assert_envelope(out, ref, ref32, ("rho", "rho_theta"), floor=1e-6, tag=variant)
    assert_envelope(out, ref, ref32, ("u", "v", "w"), base=base, floor=1e-4, tag=variant)


def test_fast_modes_off_path(gwm, orc):
    g = bubble_grid(gwm, 16, 16, 12)
    step = gwm.StepConfig(dt=1.0, fast_substeps=2, enable_fast_modes=False)
    s = c1_state(gwm, g)
    out, ref, ref32 = run_both(gwm, orc, g, step, s, 2)
    base = to64(s)
    assert_envelope(out, ref, ref32, ("u", "v", "w"), base=base, floor=1e-4, tag="no-fast")


def test_determinism_and_graph_replay(gwm):
    g = bubble_grid(gwm, 32, 24, 20)
    step = gwm.StepConfig(dt=2.0, fast_substeps=3)
    s = c1_state(gwm, g, u=2.0)
    outs = []
    for graph in (False, False, True):
        with gwm.Model(g, gwm.MemberSpec(step=step)) as m:
            m.use_graph(graph)
            m.upload(s)
            m.advance_dry_state_ssprk3(1)
            m.step(2)
            outs.append(m.download())
    for k in STATE:
        assert np.array_equal(outs[0][k], outs[1][k]), k
        assert np.array_equal(outs[0][k], outs[2][k]), k


def test_budgets_match_host_sums(gwm):
    g = bubble_grid(gwm, 20, 16, 10)
    s = c1_state(gwm, g, u=1.0)
    with gwm.Model(g, gwm.MemberSpec(step=gwm.StepConfig(dt=2.0, fast_substeps=2))) as m:
        m.upload(s)
        m.advance_dry_state_ssprk3(1)
        b = m.budgets()
        out = m.download()
    d = to64(out)
    assert b["total_dry_mass"] == pytest.approx(d["rho"].sum(), rel=1e-13)
    assert b["total_rho_theta_m"] == pytest.approx(d["rho_theta"].sum(), rel=1e-13)
    assert b["total_horizontal_momentum_x"] == pytest.approx(d["u"].sum(), rel=1e-12, abs=1e-9)
    assert b["rho_min"] == d["rho"].min() and b["w_max"] == d["w"].max()
    th = d["rho_theta"] / np.maximum(d["rho"], 1e-12)
    assert b["theta_max"] == pytest.approx(th.max(), rel=1e-15)


# ---------------------------------------------------------------------------
def moist_setup(gwm, nx=16, ny=12, nz=24, seed=7):
    g = gwm.GridSpec(nx, ny, nz, dx=3000.0, dy=3000.0, z_top=18000.0)
    p = gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=seed, relative_humidity=1.02)
    s = gwm.build_case("moist_sounding", g, p, moist=True)
    return g, s


def test_moist_step_vs_fp64_oracle(gwm, orc):
    # supersaturated moist sounding (RH 1.02) so condensation, autoconversion and
    # fallout all act within a few steps; dt keeps the scheme inside its stable range
    g, s = moist_setup(gwm)
    step = gwm.StepConfig(dt=2.0, fast_substeps=4)
    rain = gwm.WarmRainConfig(dt=2.0, rain_terminal_velocity=12.0)
    ms = gwm.MemberSpec(step=step, rain=rain, moist=True)
    with gwm.Model(g, ms) as m:
        m.upload(s)
        m.step(3)
        out = m.download()
        bud = m.budgets()
    orain = orc.RainSpec(dt=2.0, terminal_velocity=12.0)
    ref = orc.run(ogrid(orc, g), ostep(orc, step), to64(s), 3,
                  phases=orc.PHASE_DRY | orc.PHASE_TRACERS | orc.PHASE_RAIN, rain=orain, precision=64)
    assert rel_err(out["rho"], ref["rho"]) < 1e-5
    assert rel_err(out["rho_theta"], ref["rho_theta"]) < 1e-5
    for k in ("qv", "qc", "qr"):
        assert rel_err(out[k], ref[k], floor=1e-9) < 1e-3, k
    assert rel_err(out["precip"], ref["precip"], floor=1e-12) < 1e-3
    assert ref["qc"].max() > 0 and ref["qr"].max() > 0  # the case rains
    assert bud["accumulated_surface_precipitation_sum_mm"] == pytest.approx(out["precip"].sum(), rel=1e-12)


@pytest.mark.parametrize("fallout", ["nominal", "metric"])
def test_warm_rain_kats_gpu(gwm, fallout):
    # tests/unit/test_warm_rain_microphysics.cpp:41-161 through the CUDA path
    def one(rho, theta, qv, qc, qr, nz=1, z_top=1000.0, rain=None):
        g = gwm.GridSpec(1, 1, nz, dx=1000.0, dy=1000.0, z_top=z_top)
        s = gwm.build_case("constant", g, gwm.CaseParams(rho_background=rho, theta_background=theta), moist=True)
        s["qv"][:] = np.asarray(qv, dtype=np.float32).reshape(nz, 1, 1) * np.float32(rho)
        s["qc"][:] = np.asarray(qc, dtype=np.float32).reshape(nz, 1, 1) * np.float32(rho)
        s["qr"][:] = np.asarray(qr, dtype=np.float32).reshape(nz, 1, 1) * np.float32(rho)
        with gwm.Model(g, gwm.MemberSpec(rain=rain, moist=True)) as m:
            m.upload(s)
            m.apply_warm_rain_microphysics(fallout)
            return m.download()

    if fallout == "nominal":
        o = one(1.0, 300.0, 0.030, 0.0, 0.0, rain=gwm.WarmRainConfig(dt=2.0, cloud_autoconversion_rate=0.0))
        assert o["qv"][0, 0, 0] < 0.030 and o["qc"][0, 0, 0] > 0 and abs(o["qr"][0, 0, 0]) < 1e-6
        assert abs(o["qv"].sum() + o["qc"].sum() + o["qr"].sum() - 0.030) < 1e-5
        assert o["rho_theta"][0, 0, 0] / o["rho"][0, 0, 0] > 300.0
        o = one(1.0, 295.0, [0, 0], [0, 0], [0.004, 0.010], nz=2, z_top=2000.0,
                rain=gwm.WarmRainConfig(dt=1.0, cloud_autoconversion_rate=0.0, rain_evaporation_rate=0.0,
                                        rain_terminal_velocity=250.0, sedimentation_layer_depth_m=1000.0,
                                        enable_latent_heating=False))
        assert abs(o["qr"][1, 0, 0] - 0.0075) < 1e-6 and abs(o["qr"][0, 0, 0] - 0.0055) < 1e-6
        assert abs(o["precip"][0, 0] - 1.0) < 1e-6
        o = one(1.0, 295.0, 0.006, 0.002, 0.001,
                rain=gwm.WarmRainConfig(dt=2.0, cloud_autoconversion_threshold=1e-4, cloud_autoconversion_rate=1.0,
                                        rain_evaporation_rate=0.0, enable_latent_heating=False))
        assert o["qc"][0, 0, 0] < 0.002 and o["qr"][0, 0, 0] > 0.001
        assert abs(o["qv"].sum() + o["qc"].sum() + o["qr"].sum() - 0.009) < 1e-5
    else:
        o = one(1.0, 295.0, 0.0, 0.0, 0.010,
                rain=gwm.WarmRainConfig(dt=1.0, cloud_autoconversion_rate=0.0, rain_evaporation_rate=0.0,
                                        rain_terminal_velocity=1500.0, enable_latent_heating=False))
        assert abs(o["qr"][0, 0, 0]) < 1e-6
        assert abs(o["precip"][0, 0] - 10.0) < 1e-6


def test_interior_tiles_vs_oracle(gwm, orc):
    # a grid wide enough that every kernel has CTAs away from the periodic edge ring
    # (those take plain stores; edge CTAs also write the mirrored halo slots)
    g = gwm.GridSpec(160, 96, 10, dx=2000.0, dy=2000.0, z_top=12000.0)
    p = gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=11, relative_humidity=1.02)
    s = gwm.build_case("moist_sounding", g, p, moist=True)
    step = gwm.StepConfig(dt=2.0, fast_substeps=3)
    rain = gwm.WarmRainConfig(dt=2.0, rain_terminal_velocity=12.0)
    with gwm.Model(g, gwm.MemberSpec(step=step, rain=rain, moist=True)) as m:
        m.upload(s)
        m.step(2)
        out = m.download()
    kw = dict(phases=orc.PHASE_DRY | orc.PHASE_TRACERS | orc.PHASE_RAIN, rain=orc.RainSpec(dt=2.0, terminal_velocity=12.0))
    ref = orc.run(ogrid(orc, g), ostep(orc, step), to64(s), 2, precision=64, **kw)
    ref32 = orc.run(ogrid(orc, g), ostep(orc, step), to64(s), 2, precision=32, **kw)
    base = to64(s)
    assert_envelope(out, ref, ref32, ("rho", "rho_theta"), floor=1e-6, tag="interior")
    assert_envelope(out, ref, ref32, ("u", "v", "w"), base=base, floor=1e-4, tag="interior")
    for k in ("qv", "qc", "qr"):
        assert rel_err(out[k], ref[k], floor=1e-9) < 1e-3, k


@pytest.mark.parametrize("rows", [0, 3, 8, 16])
def test_substep_tilings_agree(gwm, rows):
    g = gwm.GridSpec(100, 70, 12, dx=2000.0, dy=2000.0, z_top=12000.0)
    s = c1_state(gwm, g, u=2.0, v=1.0)
    step = gwm.StepConfig(dt=1.0, fast_substeps=4)
    outs = {}
    for r in (0, rows):
        with gwm.Model(g, gwm.MemberSpec(step=step)) as m:
            m.set_tile("fast_substep", r)
            m.upload(s)
            m.advance_dry_state_ssprk3(2)
            outs[r] = m.download()
    base = to64(s)
    for k in ("rho", "rho_theta"):
        assert rel_err(outs[rows][k], outs[0][k]) < 1e-6, k
    for k in ("u", "v", "w"):
        assert perturbation_err(outs[rows][k], outs[0][k], base[k]) < 1e-4, k


@pytest.mark.parametrize("kernel", ["slow_stage", "tracer_stage"])
@pytest.mark.parametrize("periodic", [True, False])
def test_stage_tilings_bit_exact(gwm, kernel, periodic):
    # the slow and tracer stages compute each cell from the same inputs in the same
    # order whatever the tile: 8- and 16-row tiles must agree bit for bit
    g = gwm.GridSpec(100, 70, 12, dx=2000.0, dy=2000.0, z_top=12000.0,
                     periodic_x=periodic, periodic_y=periodic)
    p = gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=5, relative_humidity=1.02)
    s = gwm.build_case("moist_sounding", g, p, moist=True)
    step = gwm.StepConfig(dt=1.0, fast_substeps=4)
    rain = gwm.WarmRainConfig(dt=1.0, rain_terminal_velocity=12.0)
    outs = {}
    choices = (3, 8, 16)  # 3: owned tiles fed by TMA
    for r in choices:
        with gwm.Model(g, gwm.MemberSpec(step=step, rain=rain, moist=True)) as m:
            m.set_tile(kernel, r)
            assert m.get_tile(kernel) == r
            m.upload(s)
            m.step(2)
            outs[r] = m.download()
    for r in choices[1:]:
        for k in outs[16]:
            assert np.array_equal(outs[choices[0]][k], outs[r][k]), (r, k)


@pytest.mark.parametrize("periodic", [True, False])
def test_tma_substep_bit_exact(gwm, periodic):
    # the TMA-fed kernels run the per-thread-load kernels' arithmetic on the same values.
    # All three stencil kernels switch together, so the slow stage hands p' to the first
    # substep of every stage (the benchmark's path): a full moist step with every substep
    # kind (first with the handoff, inner, stage end, step end) must agree bit for bit;
    # 100 x 70 leaves partial tiles on both axes
    g = gwm.GridSpec(100, 70, 12, dx=2000.0, dy=2000.0, z_top=12000.0,
                     periodic_x=periodic, periodic_y=periodic)
    p = gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=9, relative_humidity=1.02)
    s = gwm.build_case("moist_sounding", g, p, moist=True)
    step = gwm.StepConfig(dt=1.0, fast_substeps=4)
    rain = gwm.WarmRainConfig(dt=1.0, rain_terminal_velocity=12.0)
    outs = {}
    for tiles in ((0, 16, 16), (3, 3, 3), (3, 16, 16)):
        with gwm.Model(g, gwm.MemberSpec(step=step, rain=rain, moist=True)) as m:
            for kernel, r in zip(("fast_substep", "slow_stage", "tracer_stage"), tiles):
                m.set_tile(kernel, r)
            m.upload(s)
            m.step(3)
            outs[tiles] = m.download()
    ref = outs[(0, 16, 16)]
    for tiles in ((3, 3, 3), (3, 16, 16)):
        for k in ref:
            assert np.array_equal(ref[k], outs[tiles][k]), (tiles, k)


@pytest.mark.parametrize("periodic,moist,bnd,ns,fast_modes", [(True, False, False, 4, True), (False, False, False, 6, True),
                                                              (True, True, False, 3, True), (False, True, True, 4, True),
                                                              (False, False, True, 1, True), (True, False, False, 2, False),
                                                              (False, True, True, 2, False)])
def test_terrain_tma_substep_bit_exact(gwm, periodic, moist, bnd, ns, fast_modes):
    # on terrain, tiles 3 select the TMA-fed acoustic substep (full pressure handed from
    # substep to substep, dp/dz derived a plane ahead), slow stage and tracer stage; they
    # run the overlapped-tile kernels' arithmetic on the same values: full steps with every
    # substep kind (first, inner, stage end, step end; one substep that is first and last
    # at once), stage inputs with and without acoustic increments, fast modes off (theta
    # level sums from the slow stage), the stand-alone fast modes, periodic and open sides
    # with the reference boundary strips, moist members (theta level sums left to the
    # rain), and 100 x 70 leaves partial tiles
    g, s = _c2_case(gwm, nx=100, ny=70, nz=12, periodic=periodic)
    if moist:
        p = gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=5, relative_humidity=1.02)
        s = gwm.build_case("moist_sounding", g, p, moist=True)
    b = _boundary_of(s, g, factor=1.002) if bnd else None
    step = gwm.StepConfig(dt=1.0 if fast_modes else 0.25, fast_substeps=ns, enable_fast_modes=fast_modes)
    rain = gwm.WarmRainConfig(dt=step.dt, rain_terminal_velocity=12.0)
    outs, fm = {}, {}
    tilings = ((8, 16, 16), (8, 3, 16), (3, 3, 3))   # (acoustic substep, slow stage, tracer stage)
    for t in tilings:
        with gwm.Model(g, gwm.MemberSpec(step=step, rain=rain, moist=moist)) as m:
            for kernel, rows in zip(("fast_substep", "slow_stage", "tracer_stage"), t):
                m.set_tile(kernel, rows)
            m.upload(s)
            if b is not None:
                m.set_boundary_state(b)
            m.step(3)
            outs[t] = m.download()
            if fast_modes:
                m.upload(s)
                m.fast_modes()
                fm[t] = m.download()
    ref = tilings[0]
    for t in tilings[1:]:
        for k in outs[ref]:
            assert np.array_equal(outs[ref][k], outs[t][k]), ("step", t, k)
            if fast_modes:
                assert np.array_equal(fm[ref][k], fm[t][k]), ("fast_modes", t, k)
    assert all(np.isfinite(v).all() for v in outs[3, 3, 3].values())


@pytest.mark.parametrize("periodic,slow,ns", [(True, 3, 4), (False, 3, 6), (True, 16, 9), (False, 16, 4)])
def test_persistent_stage_substeps_bit_exact(gwm, periodic, slow, ns):
    # all substeps of an RK stage in one cooperative launch with a grid barrier between
    # them (acoustic tiles 4) against one launch per substep (tiles 3), graph replay on:
    # with and without the slow stage's p' handoff, partial tiles on both axes, and more
    # substeps than one launch takes (9: eight in the launch, then one on its own)
    g = gwm.GridSpec(100, 70, 12, dx=2000.0, dy=2000.0, z_top=12000.0,
                     periodic_x=periodic, periodic_y=periodic)
    p = gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=13, relative_humidity=1.02)
    s = gwm.build_case("moist_sounding", g, p, moist=True)
    step = gwm.StepConfig(dt=1.0, fast_substeps=ns)
    rain = gwm.WarmRainConfig(dt=1.0, rain_terminal_velocity=12.0)
    outs = {}
    for fast in (3, 4):
        with gwm.Model(g, gwm.MemberSpec(step=step, rain=rain, moist=True)) as m:
            m.set_tile("fast_substep", fast)
            m.set_tile("slow_stage", slow)
            m.use_graph(True)
            m.upload(s)
            m.step(3)
            outs[fast] = m.download()
    for k in outs[3]:
        assert np.array_equal(outs[3][k], outs[4][k]), k


@pytest.mark.parametrize("nz", [12, 40])
def test_tma_kernels_with_open_boundary_state(gwm, nz):
    # open x with a reference boundary state (strips written at every stage start), deep
    # and shallow columns: the TMA-fed kernels with the slow-stage p' handoff against the
    # per-thread-load kernels, bit for bit
    g = gwm.GridSpec(72, 40, nz, dx=2000.0, dy=2000.0, z_top=500.0 * nz, periodic_x=False, periodic_y=True)
    p = gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=6, relative_humidity=1.02)
    s = gwm.build_case("moist_sounding", g, p, moist=True)
    s["u"][:] = np.float32(2.0)
    b = _boundary_of(s, g, factor=1.004)
    step = gwm.StepConfig(dt=1.0, fast_substeps=4)
    rain = gwm.WarmRainConfig(dt=1.0, rain_terminal_velocity=12.0)
    outs = {}
    for tiles in ((0, 16, 16), (3, 3, 3)):
        with gwm.Model(g, gwm.MemberSpec(step=step, rain=rain, moist=True)) as m:
            for kernel, r in zip(("fast_substep", "slow_stage", "tracer_stage"), tiles):
                m.set_tile(kernel, r)
            m.upload(s)
            m.set_boundary_state(b)
            m.step(2)
            outs[tiles[0]] = m.download()
    for k in outs[0]:
        assert np.isfinite(outs[3][k]).all(), k
        assert np.array_equal(outs[0][k], outs[3][k]), k


@pytest.mark.parametrize("nz", [1, 2, 3, 5])
def test_tma_kernels_on_shallow_columns(gwm, nz):
    # columns with fewer planes than the TMA rings hold ahead (the substep keeps three
    # planes in flight, the slow and tracer stages two): every TMA kernel must agree bit
    # for bit with its per-thread-load counterpart
    g = gwm.GridSpec(40, 20, nz, dx=2000.0, dy=2000.0, z_top=1500.0 * nz)
    p = gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=4, relative_humidity=1.02)
    s = gwm.build_case("moist_sounding", g, p, moist=True)
    step = gwm.StepConfig(dt=1.0, fast_substeps=4)
    rain = gwm.WarmRainConfig(dt=1.0, rain_terminal_velocity=12.0)
    outs = {}
    for tiles in ((0, 16, 16), (3, 3, 3)):
        with gwm.Model(g, gwm.MemberSpec(step=step, rain=rain, moist=True)) as m:
            for kernel, r in zip(("fast_substep", "slow_stage", "tracer_stage"), tiles):
                m.set_tile(kernel, r)
            m.upload(s)
            m.step(2)
            outs[tiles[0]] = m.download()
    for k in outs[0]:
        assert np.isfinite(outs[3][k]).all(), k
        assert np.array_equal(outs[0][k], outs[3][k]), k


@pytest.mark.parametrize("periodic", [True, False])
def test_tma_slow_stage_without_fast_modes(gwm, periodic):
    # the TMA slow stage on stage inputs without acoustic increments (fast modes off)
    # and with the last stage writing rho*theta straight into the state
    g = gwm.GridSpec(72, 40, 10, dx=1000.0, dy=1000.0, z_top=10000.0,
                     periodic_x=periodic, periodic_y=periodic)
    s = c1_state(gwm, g, u=3.0, v=-1.0)
    step = gwm.StepConfig(dt=0.5, fast_substeps=2, enable_fast_modes=False)
    outs = {}
    for r in (3, 16):
        with gwm.Model(g, gwm.MemberSpec(step=step)) as m:
            m.set_tile("slow_stage", r)
            m.upload(s)
            m.advance_dry_state_ssprk3(2)
            outs[r] = m.download()
    for k in outs[16]:
        assert np.array_equal(outs[3][k], outs[16][k]), k


def _boundary_of(state, g, factor=1.01):
    """A reference boundary state: the state scaled, with aliased periodic faces equal."""
    b = {k: (np.asarray(v, np.float64) * factor).astype(np.float32) for k, v in state.items() if k != "precip"}
    if g.periodic_x:
        b["u"][:, :, -1] = b["u"][:, :, 0]
    if g.periodic_y:
        b["v"][:, -1, :] = b["v"][:, 0, :]
    return b


@pytest.mark.parametrize("slow_tile", [16, 3])
def test_reference_boundaries_dry_vs_oracle(gwm, orc, slow_tile):
    # apply_reference_boundaries at every stage start (open x, periodic y): the CUDA path
    # against the oracle's restatement of boundary_conditions.cpp + dry_core.cu:568-620
    g = gwm.GridSpec(40, 24, 10, dx=1000.0, dy=1000.0, z_top=10000.0, periodic_x=False, periodic_y=True)
    s = c1_state(gwm, g, u=3.0, v=1.0)
    s["v"][:, -1, :] = s["v"][:, 0, :]
    b = _boundary_of(s, g)
    step = gwm.StepConfig(dt=1.0, fast_substeps=3)
    with gwm.Model(g, gwm.MemberSpec(step=step)) as m:
        m.set_tile("slow_stage", slow_tile)
        m.upload(s)
        m.set_boundary_state(b)
        m.advance_dry_state_ssprk3(3)
        out = m.download()
    kw = dict(boundary={k: v.astype(np.float64) for k, v in b.items()})
    ref = orc.run(ogrid(orc, g), ostep(orc, step), to64(s), 3, precision=64, **kw)
    ref32 = orc.run(ogrid(orc, g), ostep(orc, step), to64(s), 3, precision=32, **kw)
    plain = orc.run(ogrid(orc, g), ostep(orc, step), to64(s), 3, precision=64)
    base = to64(s)
    # the boundary must matter at all (guards against a no-op on both sides)
    assert np.abs(ref["rho"] - plain["rho"]).max() > 1e-4
    assert_envelope(out, ref, ref32, ("rho", "rho_theta"), floor=2e-6, factor=3.0, tag="bnd")
    assert_envelope(out, ref, ref32, ("u", "v", "w"), base=base, floor=2e-4, factor=3.0, tag="bnd")


def test_reference_boundaries_moist_vs_oracle(gwm, orc):
    # moist step with dry and tracer boundary states, open on both axes
    g = gwm.GridSpec(36, 28, 12, dx=2000.0, dy=2000.0, z_top=8000.0, periodic_x=False, periodic_y=False)
    p = gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=4, relative_humidity=1.03)
    s = gwm.build_case("moist_sounding", g, p, moist=True)
    b = _boundary_of(s, g, factor=1.005)
    step = gwm.StepConfig(dt=2.0, fast_substeps=4)
    rain = gwm.WarmRainConfig(dt=2.0, rain_terminal_velocity=12.0)
    with gwm.Model(g, gwm.MemberSpec(step=step, rain=rain, moist=True)) as m:
        m.upload(s)
        m.set_boundary_state(b)
        m.step(2)
        out = m.download()
    kw = dict(phases=orc.PHASE_DRY | orc.PHASE_TRACERS | orc.PHASE_RAIN,
              rain=orc.RainSpec(dt=2.0, terminal_velocity=12.0),
              boundary={k: v.astype(np.float64) for k, v in b.items()})
    ref = orc.run(ogrid(orc, g), ostep(orc, step), to64(s), 2, precision=64, **kw)
    ref32 = orc.run(ogrid(orc, g), ostep(orc, step), to64(s), 2, precision=32, **kw)
    base = to64(s)
    assert_envelope(out, ref, ref32, ("rho", "rho_theta"), floor=2e-6, factor=3.0, tag="bnd-moist")
    assert_envelope(out, ref, ref32, ("u", "v", "w"), base=base, floor=2e-4, factor=3.0, tag="bnd-moist")
    for k in ("qv", "qc", "qr"):
        assert rel_err(out[k], ref[k], floor=1e-9) < 1e-3, k


def test_apply_reference_boundaries_strips(gwm):
    # the stand-alone operator copies exactly the outermost owned strips of open sides
    g = gwm.GridSpec(20, 14, 6, dx=1000.0, dy=1000.0, z_top=6000.0, periodic_x=False, periodic_y=True)
    s = c1_state(gwm, g, u=2.0)
    s["v"][:, -1, :] = s["v"][:, 0, :]
    b = _boundary_of(s, g, factor=1.5)
    with gwm.Model(g, gwm.MemberSpec()) as m:
        m.upload(s)
        before = m.download()
        m.set_boundary_state(b)
        m.apply_reference_boundaries()
        out = m.download()
    for k in ("rho", "rho_theta", "u", "v", "w"):
        exp = before[k].copy()
        exp[:, :, 0] = b[k][:, :, 0]      # west strip (open x); periodic y untouched
        exp[:, :, -1] = b[k][:, :, -1]    # east strip
        assert np.array_equal(out[k], exp), k


def _c2_case(gwm, nx=40, ny=28, nz=20, periodic=True):
    """C2-style case on a small grid: Agnesi hill, stretched hybrid-height levels, constant-N
    stratified background with a 10 m/s wind (extensions of the reference's cases)."""
    a = 1.2
    eta = (np.exp(a * np.arange(nz + 1) / nz) - 1.0) / (np.exp(a) - 1.0)
    terrain = gwm.build_terrain("agnesi", nx, ny, 1000.0, 1000.0, height=400.0, half_width_x=6000.0,
                                half_width_y=6000.0)
    g = gwm.GridSpec(nx, ny, nz, dx=1000.0, dy=1000.0, z_top=20000.0, terrain=terrain,
                     eta_interfaces=eta, periodic_x=periodic, periodic_y=periodic)
    p = gwm.CaseParams(theta_ref=288.0, p_surface=100000.0, u_background=10.0, brunt_vaisala=0.01)
    s = gwm.build_case("stratified_mountain_wave", g, p)
    if periodic:
        s["u"][:, :, -1] = s["u"][:, :, 0]
    return g, s


def test_c2_stratified_damped_terrain_vs_oracle(gwm, orc):
    g, s = _c2_case(gwm)
    uref = s["u"].astype(np.float64).mean(axis=(1, 2))
    step = gwm.StepConfig(dt=1.0, fast_substeps=6)   # c dt / dz_min = 0.64 (stable window)
    with gwm.Model(g, gwm.MemberSpec(step=step)) as m:
        m.upload(s)
        m.set_damping(14000.0, 0.05, u_ref=uref)
        m.advance_dry_state_ssprk3(3)
        out = m.download()
    ost = ostep(orc, step)
    ost.damp_z_bottom, ost.damp_rate, ost.damp_u_ref, ost.damp_v_ref = 14000.0, 0.05, uref, np.zeros(g.nz)
    ref = orc.run(ogrid(orc, g), ost, to64(s), 3, precision=64)
    ref32 = orc.run(ogrid(orc, g), ost, to64(s), 3, precision=32)
    base = to64(s)
    assert_envelope(out, ref, ref32, ("rho", "rho_theta"), floor=2e-6, factor=3.0, tag="c2")
    assert_envelope(out, ref, ref32, ("u", "v", "w"), base=base, floor=2e-4, factor=3.0, tag="c2")


def test_damping_tma_and_overlapped_slow_agree(gwm):
    # flat terrain with the damping layer: the TMA slow stage and the overlapped tiles agree
    nz = 16
    g = gwm.GridSpec(72, 40, nz, dx=1000.0, dy=1000.0, z_top=16000.0)
    p = gwm.CaseParams(theta_ref=288.0, u_background=10.0, v_background=-3.0, brunt_vaisala=0.01)
    s = gwm.build_case("stratified_mountain_wave", g, p)
    s["u"][:, :, -1] = s["u"][:, :, 0]
    s["v"][:, -1, :] = s["v"][:, 0, :]
    s["w"][8:] = 0.3
    uref = s["u"].astype(np.float64).mean(axis=(1, 2))
    vref = s["v"].astype(np.float64).mean(axis=(1, 2))
    outs = {}
    for r in (3, 16):
        with gwm.Model(g, gwm.MemberSpec(step=gwm.StepConfig(dt=1.0, fast_substeps=3))) as m:
            m.set_tile("slow_stage", r)
            m.upload(s)
            m.set_damping(10000.0, 0.1, u_ref=uref, v_ref=vref)
            m.advance_dry_state_ssprk3(2)
            outs[r] = m.download()
    for k in outs[16]:
        assert np.array_equal(outs[3][k], outs[16][k]), k
