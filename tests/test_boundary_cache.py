"""The prepared-case boundary updater on the device, against the oracle.

PreparedCaseBoundaryUpdater / PreparedCaseTracerBoundaryUpdater
(src/ingest/prepared_case_init.cpp:396-645,1006-1078): at every updater call of a step
(sim_time 0, dt, dt/2 of the dry stages and of the tracer stages) the open-side strips
come from the boundary cache interpolated at the forecast second
lround(step_start + sim_time), tracers as rho_d times the interpolated mixing ratio; the
step start advances by dt each step.  The device keeps the cache's strips and a clock
that a captured CUDA graph advances on every replay.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

STATE = ("rho", "rho_theta", "u", "v", "w")


def _case(gwm, moist=True):
    g = gwm.GridSpec(36, 28, 12, dx=2000.0, dy=2000.0, z_top=8000.0, periodic_x=False, periodic_y=False)
    p = gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=4, relative_humidity=1.03)
    s = gwm.build_case("moist_sounding", g, p, moist=True)
    s["u"][:] = np.float32(2.5)
    if not moist:
        s = {k: s[k] for k in STATE}
    return g, s


def _snapshots(s, moist):
    """Three cache entries: the state scaled slightly, tracers as mixing ratios."""
    snaps = []
    for f in (1.004, 0.997, 1.009):
        d = {k: (s[k].astype(np.float64) * f).astype(np.float32) for k in STATE}
        if moist:
            for k in ("qv", "qc", "qr"):
                d[k] = (s[k].astype(np.float64) / s["rho"].astype(np.float64) * (2.0 - f)).astype(np.float32)
        snaps.append(d)
    return [0, 3, 7], snaps


def _ogrid(orc, g):
    return orc.GridSpec(g.nx, g.ny, g.nz, dx=g.dx, dy=g.dy, z_top=g.z_top, periodic_x=g.periodic_x,
                        periodic_y=g.periodic_y)


@pytest.mark.parametrize("tiles", [(0, 16, 16), (3, 3, 3)])
def test_boundary_cache_moist_vs_oracle(gwm, orc, tiles):
    g, s = _case(gwm)
    offsets, snaps = _snapshots(s, True)
    step = gwm.StepConfig(dt=1.0, fast_substeps=3)
    rain = gwm.WarmRainConfig(dt=1.0, rain_terminal_velocity=12.0)
    with gwm.Model(g, gwm.MemberSpec(step=step, rain=rain, moist=True)) as m:
        for kernel, r in zip(("fast_substep", "slow_stage", "tracer_stage"), tiles):
            m.set_tile(kernel, r)
        m.use_graph(True)
        m.upload(s)
        m.set_boundary_cache(offsets, snaps)
        m.set_step_start_time(1.0)
        m.step(5)                         # forecast seconds 1 .. 6: inside both brackets
        assert m.step_start_time() == 6.0
        out = m.download()
    st64 = {k: v.astype(np.float64) for k, v in s.items()}
    kw = dict(phases=orc.PHASE_DRY | orc.PHASE_TRACERS | orc.PHASE_RAIN,
              rain=orc.RainSpec(dt=1.0, terminal_velocity=12.0), boundary_cache=(offsets, snaps, 1.0))
    ost = orc.StepSpec(dt=1.0, fast_substeps=3)
    ref = orc.run(_ogrid(orc, g), ost, st64, 5, precision=64, **kw)
    ref32 = orc.run(_ogrid(orc, g), ost, st64, 5, precision=32, **kw)
    plain = orc.run(_ogrid(orc, g), ost, st64, 5, precision=64, phases=kw["phases"], rain=kw["rain"])
    assert np.abs(ref["rho"] - plain["rho"]).max() > 1e-4   # the boundary matters
    for k in STATE:
        base = st64 if k in ("u", "v", "w") else None
        if base is None:
            e = np.abs(out[k] - ref[k]).max() / np.abs(ref[k]).max()
            e32 = np.abs(ref32[k] - ref[k]).max() / np.abs(ref[k]).max()
            assert e <= max(3.0 * e32, 2e-6), (k, e, e32)
        else:
            d = np.abs(ref[k] - base[k]).max()
            e = np.abs(out[k] - ref[k]).max() / d
            e32 = np.abs(ref32[k] - ref[k]).max() / d
            assert e <= max(3.0 * e32, 2e-4), (k, e, e32)
    for k in ("qv", "qc", "qr"):
        e = np.abs(out[k] - ref[k]).max() / max(np.abs(ref[k]).max(), 1e-9)
        assert e < 1e-3, (k, e)


def test_boundary_cache_graph_replay_advances_time(gwm):
    # the clock lives on the device: replays of the captured step and direct launches
    # see the same forecast seconds and give the same state bit for bit
    g, s = _case(gwm)
    offsets, snaps = _snapshots(s, True)
    spec = gwm.MemberSpec(step=gwm.StepConfig(dt=1.5, fast_substeps=3),
                          rain=gwm.WarmRainConfig(dt=1.5, rain_terminal_velocity=12.0), moist=True)
    outs = []
    for graph in (False, True):
        with gwm.Model(g, spec) as m:
            m.use_graph(graph)
            m.upload(s)
            m.set_boundary_cache(offsets, snaps)
            m.step(2)
            m.step(3)
            assert m.step_start_time() == pytest.approx(7.5)
            outs.append(m.download())
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k]), k


def test_boundary_cache_past_the_last_entry_is_the_fixed_boundary(gwm):
    # beyond the last entry the bracket is that entry alone: the same strips as the fixed
    # reference boundary state
    g, s = _case(gwm, moist=False)
    offsets, snaps = _snapshots(s, False)
    step = gwm.StepConfig(dt=1.0, fast_substeps=3)
    outs = []
    for mode in ("cache", "fixed"):
        with gwm.Model(g, gwm.MemberSpec(step=step)) as m:
            m.upload(s)
            if mode == "cache":
                m.set_boundary_cache(offsets, snaps)
                m.set_step_start_time(50.0)
            else:
                m.set_boundary_state(snaps[-1])
            m.step(3)
            outs.append(m.download())
    for k in STATE:
        assert np.array_equal(outs[0][k], outs[1][k]), k
