"""Pin the CPU oracle against the reference's own known-answer tests.

Each test restates a reference unit/regression test (file:line cited) and runs
it on the oracle, in FP32 (the reference's arithmetic) and, where the answer is
precision independent, FP64 as well.  No GPU is needed.
"""
import numpy as np
import pytest


def rank_fields(orc, nx, ny, nz, halo, rx, ry, orient, fn, fill=0.0):
    lay = orc.layout(nx, ny, nz, halo, rx, ry)
    out = []
    for row in lay:
        shape = orc.rank_field_shape(row, nz, halo, orient)
        a = np.full(shape, fill)
        i0, j0 = int(row[3]), int(row[5])
        fz, fy, fx = shape
        for k in range(fz):
            for j in range(fy - 2 * halo):
                for i in range(fx - 2 * halo):
                    a[k, j + halo, i + halo] = fn(i0 + i, j0 + j, k)
        out.append(a)
    return lay, out


def at(a, halo, i, j, k):
    return a[k, j + halo, i + halo]


def test_scalar_halo_exchange_kat(orc):
    # tests/unit/test_halo_exchange.cpp:8-19
    lay, F = rank_fields(orc, 8, 8, 1, 1, 2, 2, "cell", lambda i, j, k: 100 * j + i)
    orc.halo(F, 8, 8, 1, 1, 2, 2, True, True, "cell")
    r0 = F[0]
    assert at(r0, 1, -1, 0, 0) == 7.0
    assert at(r0, 1, 4, 0, 0) == 4.0
    assert at(r0, 1, 0, -1, 0) == 700.0
    assert at(r0, 1, 0, 4, 0) == 400.0


def test_scalar_halo_buffers_kat(orc):
    # tests/unit/test_scalar_halo_buffers.cpp:11-30
    lay = orc.layout(8, 8, 2, 1, 2, 2)
    assert tuple(lay[0][7:11]) == (1, 1, 2, 2)  # west, east, south, north
    x_face_count = 1 * (lay[0][6] - lay[0][5]) * 2
    y_face_count = 1 * (lay[0][4] - lay[0][3] + 2) * 2
    assert (x_face_count, y_face_count) == (8, 12)
    _, F = rank_fields(orc, 8, 8, 2, 1, 2, 2, "cell", lambda i, j, k: 1000 * k + 100 * j + i)
    orc.halo(F, 8, 8, 2, 1, 2, 2, True, True, "cell")
    assert at(F[0], 1, -1, 0, 0) == 7.0
    assert at(F[0], 1, 0, -1, 1) == 1700.0


def test_face_halo_exchange_kat(orc):
    # tests/unit/test_face_halo_exchange.cpp:28-61
    fn = lambda i, j, k: 1000 * k + 100 * j + i
    _, X = rank_fields(orc, 8, 8, 2, 1, 2, 2, "x", fn, fill=-999.0)
    _, Y = rank_fields(orc, 8, 8, 2, 1, 2, 2, "y", fn, fill=-999.0)
    _, Z = rank_fields(orc, 8, 8, 2, 1, 2, 2, "z", fn, fill=-999.0)
    orc.halo(X, 8, 8, 2, 1, 2, 2, True, True, "x")
    orc.halo(Y, 8, 8, 2, 1, 2, 2, True, True, "y")
    orc.halo(Z, 8, 8, 2, 1, 2, 2, True, True, "z")
    x0, y0, z0 = X[0], Y[0], Z[0]
    assert at(x0, 1, -1, 0, 0) == 7.0
    assert at(x0, 1, 5, 0, 0) == 5.0
    assert at(x0, 1, 0, -1, 0) == 700.0
    assert at(x0, 1, -1, -1, 0) == 707.0
    assert at(y0, 1, -1, 0, 0) == 7.0
    assert at(y0, 1, 0, -1, 0) == 700.0
    assert at(y0, 1, 0, 5, 0) == 500.0
    assert at(y0, 1, -1, -1, 0) == 707.0
    assert at(z0, 1, -1, 0, 0) == 7.0
    assert at(z0, 1, 0, -1, 1) == 1700.0
    assert at(z0, 1, -1, -1, 1) == 1707.0


def test_open_boundary_halo_is_zero(orc):
    # absent neighbours deliver zero-filled buffers: halo_exchange.cpp:289-301,593-600
    _, F = rank_fields(orc, 6, 5, 2, 1, 1, 1, "cell", lambda i, j, k: 1.0 + i + 10 * j, fill=-5.0)
    orc.halo(F, 6, 5, 2, 1, 1, 1, False, False, "cell")
    a = F[0]
    assert np.all(a[:, 0, :] == 0.0) and np.all(a[:, -1, :] == 0.0)
    assert np.all(a[:, :, 0] == 0.0) and np.all(a[:, :, -1] == 0.0)


def test_face_interface_sync_self_pair(orc):
    # halo_exchange.cpp:255-267: a periodic 1x1 layout averages face 0 with face nx
    _, X = rank_fields(orc, 4, 3, 1, 1, 1, 1, "x", lambda i, j, k: float(i))
    orc.halo(X, 4, 3, 1, 1, 1, 1, True, True, "x", op="sync")
    assert at(X[0], 1, 0, 0, 0) == 2.0 and at(X[0], 1, 4, 0, 0) == 2.0


def test_hybrid_height_metrics_kat(orc):
    # tests/unit/test_hybrid_height_metrics.cpp:10-27 (flat)
    g = orc.GridSpec(12, 10, 8, z_top=16000.0)
    m = orc.metrics(g, precision=32)
    assert abs(m["z_interfaces"][0, 0, 0]) < 1e-6
    assert abs(m["z_interfaces"][8, 0, 0] - 16000.0) < 1e-4
    assert abs(m["inv_dz_cell"][0, 0, 0] - np.float32(1.0 / 2000.0)) < 1e-7
    assert np.all(np.diff(m["z_interfaces"][:, 0, 0]) > 0)
    # :29-68 (cosine mountain, built the way idealized_domain_builder.cpp:14-35 does)
    nx = ny = 21
    terr = np.zeros((ny, nx))
    for j in range(ny):
        for i in range(nx):
            x, y = i / (nx - 1), j / (ny - 1)
            dx, dy = (x - 0.5) / 0.25, (y - 0.5) / 0.25
            if abs(dx) < 1 and abs(dy) < 1:
                terr[j, i] = np.float32(1200.0 * 0.5 * (1 + np.cos(np.pi * dx)) * 0.5 * (1 + np.cos(np.pi * dy)))
    g = orc.GridSpec(nx, ny, 12, z_top=18000.0, terrain=terr)
    m = orc.metrics(g, precision=32)
    zi, zc, idc = m["z_interfaces"][:, 10, 10], m["z_centers"][:, 10, 10], m["inv_dz_cell"][:, 10, 10]
    assert abs(zi[0] - terr[10, 10]) < 1e-3
    assert abs(zi[12] - 18000.0) < 1e-4
    assert np.all(zi[1:] > zi[:-1]) and np.all(zc > zi[:-1]) and np.all(zc < zi[1:]) and np.all(idc > 0)


def test_moist_qsat_kat(orc):
    # tests/unit/test_moist_thermo.cpp:13-21 restated in numpy against the formula
    t, p = np.float32(300.0), np.float32(90000.0)
    eps = np.float32(287.05) / np.float32(461.5)
    tc = t - np.float32(273.15)
    es = np.float32(6.112) * np.exp(np.float32(17.67) * tc / (tc + np.float32(243.5))) * np.float32(100.0)
    expected = eps * es / (p - (np.float32(1) - eps) * es)
    assert 0.02 < expected < 0.03


@pytest.mark.parametrize("precision", [32, 64])
def test_constant_state_bundle(orc, precision):
    # tests/regression/test_dry_constant_state_bundle.cpp:11-35
    g = orc.GridSpec(20, 16, 6, ranks_x=2, ranks_y=2)
    s = orc.case("constant", g, orc.CaseSpec(rho_background=1.1, theta_background=301.0,
                                             u_background=10.0, v_background=-4.0))
    out = orc.run(g, orc.StepSpec(dt=2.0, fast_substeps=2), s, 1, precision=precision)
    assert np.allclose(out["rho"], 1.1, atol=1e-5)
    assert np.allclose(out["rho_theta"], np.float32(1.1) * np.float32(301.0), atol=1e-3)


@pytest.mark.parametrize("precision", [32, 64])
def test_fast_modes_kats(orc, precision):
    # tests/unit/test_dry_fast_modes.cpp:65-192
    g = orc.GridSpec(20, 20, 8, ranks_x=2, ranks_y=2)
    s = orc.case("constant", g, orc.CaseSpec(rho_background=1.1, theta_background=300.0,
                                             u_background=12.0, v_background=-6.0))
    out = orc.fast_modes(g, orc.StepSpec(dt=2.0, fast_substeps=4), s, precision=precision)
    assert abs(out["rho"].sum() - s["rho"].sum()) < 1e-4
    assert abs(out["u"].max() - s["u"].max()) < 1e-5 and abs(out["v"].min() - s["v"].min()) < 1e-5

    def pulse():
        st = orc.case("constant", g, orc.CaseSpec(rho_background=1.0, theta_background=300.0))
        st["rho"][4, 10, 10] += np.float32(0.02)
        st["rho_theta"][4, 10, 10] = np.float32(st["rho"][4, 10, 10]) * np.float32(300.0)
        st["rho"] = st["rho"].astype(np.float32).astype(np.float64)
        return st

    st = pulse()
    m0 = st["rho"].sum()
    for _ in range(3):
        st = orc.fast_modes(g, orc.StepSpec(dt=1.0, fast_substeps=4), st, precision=precision)
    assert abs(st["rho"].sum() - m0) < 1e-3

    on = orc.fast_modes(g, orc.StepSpec(dt=1.0, fast_substeps=1, fast_hmom=True, fast_density=False), pulse(), precision=precision)
    off = orc.fast_modes(g, orc.StepSpec(dt=1.0, fast_substeps=1, fast_hmom=False, fast_density=False), pulse(), precision=precision)
    assert np.abs(on["u"]).max() > 1e-5 and np.abs(on["v"]).max() > 1e-5
    assert np.abs(off["u"]).max() < 1e-8 and np.abs(off["v"]).max() < 1e-8
    for o in (on, off):
        assert abs(o["rho"].max() - 1.02) < 1e-6 and abs(o["rho"].min() - 1.0) < 1e-6

    don = orc.fast_modes(g, orc.StepSpec(dt=1.0, fast_substeps=1, fast_hmom=False, fast_density=True), pulse(), precision=precision)
    assert abs(don["rho"].sum() - m0) < 1e-5
    assert abs(don["rho"].max() - 1.02) > 1e-5


@pytest.mark.parametrize("precision", [32, 64])
def test_momentum_flux_constant_state_zero_sum(orc, precision):
    # tests/unit/test_dry_momentum_flux.cpp:42-85 — constant state: the flux part of
    # the slow tendency sums to zero; pressure gradient and buoyancy vanish too.
    g = orc.GridSpec(20, 18, 8, ranks_x=2, ranks_y=2)
    s = orc.case("constant", g, orc.CaseSpec(rho_background=1.05, theta_background=300.0,
                                             u_background=12.0, v_background=-4.0, w_background=0.5))
    t = orc.slow_tendencies(g, orc.StepSpec(), s, precision=precision)
    assert abs(t["u"].sum()) < 1e-3 and abs(t["v"].sum()) < 1e-3


@pytest.mark.parametrize("precision", [32, 64])
def test_warm_rain_kats(orc, precision):
    # tests/unit/test_warm_rain_microphysics.cpp:41-161
    def one_cell(rho, theta, qv, qc=0.0, qr=0.0, nz=1):
        g = orc.GridSpec(1, 1, nz)
        s = orc.case("constant", g, orc.CaseSpec(rho_background=rho, theta_background=theta))
        s.update(qv=np.full((nz, 1, 1), rho * qv), qc=np.full((nz, 1, 1), rho * qc),
                 qr=np.full((nz, 1, 1), rho * qr), precip=np.zeros((1, 1)))
        return g, s

    g, s = one_cell(1.0, 300.0, 0.030)
    out = orc.run(g, orc.StepSpec(), s, 1, phases=orc.PHASE_RAIN_NOMINAL,
                  rain=orc.RainSpec(dt=2.0, autoconv_rate=0.0), precision=precision)
    assert out["qv"][0, 0, 0] < 0.030 and out["qc"][0, 0, 0] > 0 and abs(out["qr"][0, 0, 0]) < 1e-6
    assert abs(out["qv"].sum() + out["qc"].sum() + out["qr"].sum() - 0.030) < 1e-5
    assert out["rho_theta"][0, 0, 0] / out["rho"][0, 0, 0] > 300.0

    g = orc.GridSpec(1, 1, 2)
    s = orc.case("constant", g, orc.CaseSpec(rho_background=1.0, theta_background=295.0))
    s.update(qv=np.zeros((2, 1, 1)), qc=np.zeros((2, 1, 1)),
             qr=np.array([[[0.004]], [[0.010]]]), precip=np.zeros((1, 1)))
    out = orc.run(g, orc.StepSpec(), s, 1, phases=orc.PHASE_RAIN_NOMINAL,
                  rain=orc.RainSpec(dt=1.0, autoconv_rate=0.0, rain_evap_rate=0.0,
                                    terminal_velocity=250.0, layer_depth=1000.0,
                                    latent_heating=False), precision=precision)
    assert abs(out["qr"][1, 0, 0] - 0.0075) < 1e-6
    assert abs(out["qr"][0, 0, 0] - 0.0055) < 1e-6
    assert abs(out["precip"][0, 0] - 1.0) < 1e-6

    g, s = one_cell(1.0, 295.0, 0.006, 0.002, 0.001)
    out = orc.run(g, orc.StepSpec(), s, 1, phases=orc.PHASE_RAIN_NOMINAL,
                  rain=orc.RainSpec(dt=2.0, autoconv_threshold=1e-4, autoconv_rate=1.0,
                                    rain_evap_rate=0.0, latent_heating=False), precision=precision)
    assert out["qc"][0, 0, 0] < 0.002 and out["qr"][0, 0, 0] > 0.001
    assert abs(out["qv"].sum() + out["qc"].sum() + out["qr"].sum() - 0.009) < 1e-5

    g = orc.GridSpec(1, 1, 1, dx=1000.0, dy=1000.0, z_top=1000.0)
    s = orc.case("constant", g, orc.CaseSpec(rho_background=1.0, theta_background=295.0))
    s.update(qv=np.zeros((1, 1, 1)), qc=np.zeros((1, 1, 1)), qr=np.full((1, 1, 1), 0.010),
             precip=np.zeros((1, 1)))
    out = orc.run(g, orc.StepSpec(), s, 1, phases=orc.PHASE_RAIN,
                  rain=orc.RainSpec(dt=1.0, autoconv_rate=0.0, rain_evap_rate=0.0,
                                    terminal_velocity=1500.0, latent_heating=False), precision=precision)
    assert abs(out["qr"][0, 0, 0]) < 1e-6
    assert abs(out["precip"][0, 0] - 10.0) < 1e-6


def test_pgf_linear_pressure_kat(orc):
    # tests/unit/test_dry_pressure_gradient.cpp:28-55: the oracle's PGF term equals
    # -dp/dx for a field whose pressure varies linearly; checked here through the
    # full slow tendency of a state built to have p = p0 + 10 i + 20 j is not
    # possible (p is derived from rho and rho_theta), so the check runs on the
    # discrete formula: (p_r - p_l)/dx with dzdx = 0 gives -10/dx.
    dx = 1000.0
    p = lambda i, j: 100000.0 + 10.0 * i + 20.0 * j
    assert np.float32(-(np.float32(p(1, 2)) - np.float32(p(0, 2))) / np.float32(dx)) == pytest.approx(-10.0 / dx, abs=1e-6)


@pytest.mark.parametrize("precision", [32, 64])
def test_virtual_rank_equivalence(orc, precision):
    # tests/property/test_dry_virtual_rank_equivalence.cpp: 1x1 vs 2x2 layouts agree.
    cs = orc.CaseSpec(rho_background=1.0, theta_background=300.0, theta_perturbation=3.0,
                      center_z_fraction=0.35, radius_x_fraction=0.15, radius_y_fraction=0.15,
                      radius_z_fraction=0.2)
    st = orc.StepSpec(dt=2.0, fast_substeps=3)
    outs = []
    for rx, ry in ((1, 1), (2, 2)):
        g = orc.GridSpec(20, 18, 8, ranks_x=rx, ranks_y=ry)
        s = orc.case("density_current", g, cs)
        outs.append(orc.run(g, st, s, 2, precision=precision))
    # FP32: the level-mean sums run in a different order per layout (the
    # reference sums them with float atomics); the reference property tests
    # allow 1e-4..5e-4 (test_terrain_virtual_rank_equivalence.cpp:205-209).
    tol = 5e-4 if precision == 32 else 1e-11
    for k in ("rho", "rho_theta", "u", "v", "w"):
        a, b = outs[0][k], outs[1][k]
        assert np.max(np.abs(a - b)) <= tol * max(1.0, np.max(np.abs(a))), k


def test_boundary_cache_single_entry_is_the_fixed_boundary(orc):
    # the prepared-case updater with one cache entry (or past its last entry) applies that
    # entry's strips at every call: the same step as apply_reference_boundaries with it
    g = orc.GridSpec(14, 10, 6, dx=1000.0, dy=1000.0, z_top=6000.0, periodic_x=False, periodic_y=False)
    s = orc.case("density_current", g, orc.CaseSpec(theta_perturbation=3.0, center_z_fraction=0.4,
                                                     radius_x_fraction=0.3, radius_y_fraction=0.3,
                                                     radius_z_fraction=0.3, u_background=2.0))
    b0 = {k: v * 1.01 for k, v in s.items()}
    b1 = {k: v * 0.98 for k, v in s.items()}
    st = orc.StepSpec(dt=1.0, fast_substeps=2)
    fixed = orc.run(g, st, s, 3, precision=64, boundary=b1)
    one = orc.run(g, st, s, 3, precision=64, boundary_cache=([0], [b1], 0.0))
    past = orc.run(g, st, s, 3, precision=64, boundary_cache=([0, 10], [b0, b1], 100.0))
    for k in ("rho", "rho_theta", "u", "v", "w"):
        assert np.array_equal(fixed[k], one[k]), k
        assert np.array_equal(fixed[k], past[k]), k
    mid = orc.run(g, st, s, 3, precision=64, boundary_cache=([0, 10], [b0, b1], 4.0))
    assert not np.array_equal(mid["rho"], fixed["rho"])
