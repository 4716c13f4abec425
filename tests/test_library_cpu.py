"""CPU-side checks of the product library: it builds, loads without a GPU,
exports every symbol its headers declare, and its host-side code (layout table,
rank<->global conversion, case builders, terrain) agrees with the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in ("gwm_b200.h", "gwm_b200_cases.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"\b(gwm_b200_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol(gwm):
    L = gwm.lib()
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert set(gwm.EXPORTED) <= set(syms)


def test_create_fails_loudly_without_device(gwm):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    with pytest.raises(RuntimeError, match="no CUDA device"):
        gwm.Model(gwm.GridSpec(8, 8, 4), gwm.MemberSpec())


@pytest.mark.parametrize("args", [(8, 8, 2, 1, 2, 2, True, True), (13, 7, 3, 1, 3, 2, False, True),
                                  (10, 9, 2, 1, 1, 3, True, False), (5, 5, 1, 2, 2, 2, False, False)])
def test_layout_matches_oracle(gwm, orc, args):
    nx, ny, nz, h, rx, ry, px, py = args
    a = gwm.layout(nx, ny, nz, h, rx, ry, px, py)
    b = orc.layout(nx, ny, nz, h, rx, ry, px, py)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("orient", [0, 1, 2, 3])
def test_rank_global_round_trip(gwm, orient):
    nx, ny, nz, h, rx, ry = 11, 9, 3, 1, 3, 2
    lay = gwm.layout(nx, ny, nz, h, rx, ry)
    rng = np.random.default_rng(orient)
    shp = (nz + (orient == 3), ny + (orient == 2), nx + (orient == 1))
    glob = rng.standard_normal(shp).astype(np.float32)
    ranks = []
    for row in lay:
        nxl, nyl = row[4] - row[3], row[6] - row[5]
        ranks.append(np.zeros((nz + (orient == 3), nyl + (orient == 2) + 2 * h, nxl + (orient == 1) + 2 * h),
                              dtype=np.float32))
    gwm.global_to_ranks(glob, ranks, nx, ny, nz, h, rx, ry, True, True, orient)
    back = gwm.ranks_to_global(ranks, nx, ny, nz, h, rx, ry, True, True, orient)
    assert np.array_equal(back, glob)


CASES = [
    ("constant", dict(rho_background=1.1, theta_background=301.0, u_background=10.0, v_background=-4.0)),
    ("warm_bubble", dict(theta_perturbation=2.0, center_z_fraction=0.3)),
    ("density_current", dict(theta_perturbation=15.0, center_z_fraction=0.35, radius_x_fraction=0.15)),
    ("hydrostatic_rest", dict(rho_surface=1.16, theta_ref=300.0)),
    ("mountain_wave_background", dict(rho_surface=1.18, theta_ref=300.0, u_background=15.0)),
    ("hydrostatic_warm_bubble", dict(rho_surface=1.16, theta_ref=300.0, theta_perturbation=2.0,
                                     center_z_fraction=0.2, radius_x_fraction=0.25, radius_z_fraction=0.2)),
]


@pytest.mark.parametrize("kind,kw", CASES)
def test_case_builders_match_oracle(gwm, orc, kind, kw):
    terr = gwm.build_terrain("cosine_mountain", 16, 12, 1000.0, 1000.0, height=600.0,
                             half_width_x=0.3, half_width_y=0.3)
    g = gwm.GridSpec(16, 12, 10, dx=1000.0, dy=1000.0, z_top=10000.0, terrain=terr)
    og = orc.GridSpec(16, 12, 10, dx=1000.0, dy=1000.0, z_top=10000.0, terrain=terr.astype(np.float64))
    mine = gwm.build_case(kind, g, gwm.CaseParams(**kw))
    ref = orc.case(kind, og, orc.CaseSpec(**{k: v for k, v in kw.items()}), precision=32)
    for k in ("rho", "rho_theta", "u", "v", "w"):
        np.testing.assert_allclose(mine[k], ref[k], rtol=2e-6, atol=1e-6, err_msg=f"{kind}:{k}")


def test_cosine_terrain_kat(gwm):
    # tests/unit/test_hybrid_height_metrics.cpp:29-41: the cosine hill peaks at the centre
    t = gwm.build_terrain("cosine_mountain", 21, 21, 1000.0, 1000.0, height=1200.0,
                          half_width_x=0.25, half_width_y=0.25)
    assert t[10, 10] == pytest.approx(1200.0)
    assert t[0, 0] == 0.0 and t.max() == t[10, 10]
    a = gwm.build_terrain("agnesi", 64, 64, 1000.0, 1000.0, height=400.0,
                          half_width_x=10000.0, half_width_y=10000.0)
    assert a.max() <= 400.0 and a.max() > 390.0


def test_moist_sounding_properties(gwm):
    g = gwm.GridSpec(8, 6, 32, dx=3000.0, dy=3000.0, z_top=24000.0)
    p = gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=3)
    s = gwm.build_case("moist_sounding", g, p, moist=True)
    th = s["rho_theta"] / s["rho"]
    zc = (np.arange(32) + 0.5) * 750.0
    qv = s["qv"] / s["rho"]
    # theta: noisy below 1 km, 300 K + 4 K/km above (within FP32 of the EOS inversion)
    upper = zc > 1500.0
    np.testing.assert_allclose(th[upper, 0, 0], 300.0 + 0.004 * (zc[upper] - 1000.0), rtol=2e-5)
    low = zc < 1000.0
    assert np.std(th[low]) > 0.1
    # hydrostatic: pressure decreases with height, density positive
    assert np.all(s["rho"] > 0) and np.all(np.diff(s["rho"][:, 0, 0]) < 0)
    assert np.all(qv >= 1e-5 * 0.999) and qv[0].mean() > 0.005
    # same seed -> same state; another seed -> different noise
    s2 = gwm.build_case("moist_sounding", g, p, moist=True)
    assert np.array_equal(s["rho_theta"], s2["rho_theta"])
    s3 = gwm.build_case("moist_sounding", g, gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=4), moist=True)
    assert not np.array_equal(s["rho_theta"], s3["rho_theta"])


def test_stratified_mountain_wave_background(gwm):
    # constant-N background (an extension of the reference's constant-theta mountain-wave
    # case): N^2 = g/theta dtheta/dz recovered from the cell values, hydrostatic residual
    # small, face momenta = face-mean density x wind
    nz = 40
    g = gwm.GridSpec(16, 12, nz, dx=1000.0, dy=1000.0, z_top=20000.0)
    p = gwm.CaseParams(theta_ref=288.0, p_surface=100000.0, u_background=10.0, brunt_vaisala=0.01)
    s = gwm.build_case("stratified_mountain_wave", g, p)
    rho = s["rho"][:, 5, 7].astype(np.float64)
    th = (s["rho_theta"][:, 5, 7] / s["rho"][:, 5, 7]).astype(np.float64)
    z = (np.arange(nz) + 0.5) * 20000.0 / nz
    n2 = 9.81 * np.diff(np.log(th)) / np.diff(z)   # exact for theta0 exp(N^2 z / g)
    assert np.allclose(n2, 1.0e-4, rtol=2e-3)
    # hydrostatic: (p_{k+1} - p_k)/dz = -g * mean density, to discretisation accuracy
    pres = 1.0e5 * (287.05 * rho * th / 1.0e5) ** (1.0 / (1.0 - 0.2854))
    resid = np.diff(pres) / np.diff(z) + 9.81 * 0.5 * (rho[1:] + rho[:-1])
    assert np.abs(resid).max() < 2e-3 * 9.81 * rho.max()
    u = s["u"][:, 5, 7].astype(np.float64)
    assert np.allclose(u, 10.0 * 0.5 * (s["rho"][:, 5, 6] + s["rho"][:, 5, 7]), rtol=1e-6)
    assert np.all(s["w"] == 0.0)


def test_rayleigh_layer_in_oracle(orc, gwm):
    # the damping layer (extension) acts only above its bottom and pulls w to zero there
    g = gwm.GridSpec(16, 12, 20, dx=1000.0, dy=1000.0, z_top=20000.0)
    p = gwm.CaseParams(theta_ref=288.0, u_background=10.0, brunt_vaisala=0.01)
    s = gwm.build_case("stratified_mountain_wave", g, p)
    s["w"][10:, :, :] = 0.5  # an upper-level vertical motion to be damped
    st = {k: v.astype(np.float64) for k, v in s.items()}
    og = orc.GridSpec(16, 12, 20, dx=1000.0, dy=1000.0, z_top=20000.0)
    uref = s["u"].astype(np.float64).mean(axis=(1, 2))
    free = orc.run(og, orc.StepSpec(dt=1.0, fast_substeps=2), st, 1)
    damp = orc.run(og, orc.StepSpec(dt=1.0, fast_substeps=2, damp_z_bottom=14000.0, damp_rate=0.2,
                                    damp_u_ref=uref, damp_v_ref=np.zeros(20)), st, 1)
    top = slice(16, 20)   # faces above 16 km
    assert np.abs(damp["w"][top]).mean() < np.abs(free["w"][top]).mean() * 0.95
    low = slice(1, 10)    # below the layer the two runs agree to rounding at one step
    assert np.abs(damp["w"][low] - free["w"][low]).max() < 1e-3 * max(np.abs(free["w"][low]).max(), 1e-3)


@pytest.mark.parametrize("kind", ["flat", "cosine_mountain", "agnesi_stretched"])
def test_grid_z_center_matches_oracle(gwm, orc, kind):
    # GridMetrics::z_center through the C-ABI (host code, no device): the FP64 heights of
    # the oracle's metric builder, rounded once to FP32
    nx, ny, nz = 24, 18, 12
    kw, okw = {}, {}
    if kind != "flat":
        shape = "cosine_mountain" if kind == "cosine_mountain" else "agnesi"
        t = gwm.build_terrain(shape, nx, ny, 1000.0, 1000.0, height=700.0)
        kw["terrain"] = okw["terrain"] = t
    if kind == "agnesi_stretched":
        eta = (np.linspace(0.0, 1.0, nz + 1) ** 1.4).astype(np.float64)
        kw["eta_interfaces"] = okw["eta_interfaces"] = eta
    g = gwm.GridSpec(nx, ny, nz, dx=1000.0, dy=1000.0, z_top=15000.0, **kw)
    og = orc.GridSpec(nx, ny, nz, dx=1000.0, dy=1000.0, z_top=15000.0, **okw)
    zc = gwm.grid_z_center(g)
    ref = orc.metrics(og)["z_centers"]
    assert zc.shape == ref.shape
    assert np.array_equal(zc, ref.astype(np.float32))


def test_host_entry_points_reject_bad_arguments(gwm):
    # argument checks come before any device work, so they answer without a GPU
    L = gwm.lib()
    assert L.gwm_b200_grid_z_center(None, None) == gwm.ERR_ARG
    g = gwm.GridSpec(8, 8, 0, dx=1000.0, dy=1000.0, z_top=1000.0)
    out = np.empty(8, np.float32)
    assert L.gwm_b200_grid_z_center(ctypes.byref(g.c()), out.ctypes.data_as(ctypes.c_void_p)) == gwm.ERR_ARG
    assert L.gwm_b200_scalar_ssprk3(None, None, 1, None) == gwm.ERR_ARG
    assert L.gwm_b200_field_stats_noalloc(None, 10, None, None) == gwm.ERR_ARG
    buf, res = np.zeros(4, np.float32), np.zeros(3, np.float64)
    assert L.gwm_b200_field_stats_noalloc(buf.ctypes.data_as(ctypes.c_void_p), 0,
                                          res.ctypes.data_as(ctypes.c_void_p), None) == gwm.ERR_ARG


D, F, LL, ULL = ctypes.c_double, ctypes.c_float, ctypes.c_longlong, ctypes.c_ulonglong
NULL_CONTEXT_CALLS = [
    ("gwm_b200_set_concurrent", (1,)), ("gwm_b200_set_stream", (None,)), ("gwm_b200_synchronize", ()),
    ("gwm_b200_use_graph", (1,)), ("gwm_b200_set_tile", (1, 3)), ("gwm_b200_upload", (0, None)),
    ("gwm_b200_set_boundary_state", (0, None)), ("gwm_b200_set_damping", (0, D(1000.0), D(0.1), None, None)),
    ("gwm_b200_apply_reference_boundaries", (0,)),
    ("gwm_b200_rain_record", (0, None, None, LL(0), ULL(1), F(1.0), F(0.0), None)),
    ("gwm_b200_set_rain_surrogate", (0, None, None, None, F(0.1), F(0.1))),
    ("gwm_b200_download", (0, None)), ("gwm_b200_profile", (1,)), ("gwm_b200_step", (1,)),
    ("gwm_b200_advance_dry", (1,)), ("gwm_b200_advance_tracers", ()), ("gwm_b200_warm_rain", (1,)),
    ("gwm_b200_fast_modes", ()), ("gwm_b200_slow_tendencies", (0, None)), ("gwm_b200_budgets", (0, None)),
]


@pytest.mark.parametrize("name,args", NULL_CONTEXT_CALLS, ids=[c[0] for c in NULL_CONTEXT_CALLS])
def test_null_context_is_an_argument_error(gwm, name, args):
    # every context call answers a NULL context with the invalid-argument status (the
    # reference's require() failures become status codes; nothing is dereferenced)
    assert getattr(gwm.lib(), name)(None, *args) == gwm.ERR_ARG


def test_null_context_counters_and_destroy(gwm):
    L = gwm.lib()
    count = ctypes.c_longlong(7)
    stats = (ctypes.c_longlong * 6)()
    assert L.gwm_b200_surrogate_stats(None, 0, stats, 0) == gwm.ERR_ARG
    assert L.gwm_b200_surrogate_fallbacks(None, 0, ctypes.byref(count), 0) == gwm.ERR_ARG
    assert count.value == 0
    L.gwm_b200_destroy(None)  # a no-op


@pytest.mark.parametrize("nx,ny,nz,seed", [(16, 12, 24, 7), (40, 33, 64, 3)])
def test_moist_sounding_oracle_builder_matches_library(gwm, orc, nx, ny, nz, seed):
    # the CPU baseline builds the benchmark's initial state with the oracle's own builder;
    # it must be the state the library builds, bit for bit
    sounding = dict(theta_ref=300.0, theta_lapse_k_per_m=0.004, relative_humidity=0.9, rh_top_m=2000.0,
                    qv_scale_height_m=1500.0, qv_floor=1e-5, noise_rms_k=0.5, noise_depth_m=1000.0)
    g = gwm.GridSpec(nx, ny, nz, dx=3000.0, dy=3000.0, z_top=16000.0)
    a = gwm.build_case("moist_sounding", g, gwm.CaseParams(seed=seed, **sounding), moist=True)
    b = orc.moist_sounding(orc.GridSpec(nx, ny, nz, dx=3000.0, dy=3000.0, z_top=16000.0), seed=seed, **sounding)
    for k in a:
        assert np.array_equal(a[k].astype(np.float64), b[k]), k
    assert b["qv"].max() > 0 and np.ptp(b["rho_theta"][0]) > 0  # moist, with noise
