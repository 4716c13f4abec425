"""gwm_b200_step_host: one step from host buffers to host buffers, with the copies
overlapping the step's phases on two copy streams, against upload + step + download."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pinned_copy(state):
    import torch
    out = {}
    for k, v in state.items():
        t = torch.empty(v.shape, dtype=torch.float64 if k == "precip" else torch.float32, pin_memory=True)
        a = t.numpy()
        a[...] = v
        out[k] = a
    return out


@pytest.mark.parametrize("moist,periodic,terrain", [(True, True, False), (True, False, False), (False, True, False),
                                                   (False, False, True)])
def test_step_host_equals_upload_step_download(gwm, moist, periodic, terrain):
    kw = {}
    if terrain:  # Agnesi hill on stretched levels (the terrain TMA substep and its column reference)
        eta = (np.exp(1.2 * np.arange(13) / 12) - 1.0) / (np.exp(1.2) - 1.0)
        kw = dict(terrain=gwm.build_terrain("agnesi", 100, 70, 2000.0, 2000.0, height=400.0,
                                            half_width_x=12000.0, half_width_y=12000.0), eta_interfaces=eta)
    g = gwm.GridSpec(100, 70, 12, dx=2000.0, dy=2000.0, z_top=12000.0, periodic_x=periodic, periodic_y=periodic,
                     **kw)
    p = gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=21, relative_humidity=1.02, u_background=5.0)
    s = gwm.build_case("moist_sounding" if moist else "warm_bubble", g, p, moist=moist)
    if moist:
        s["precip"][...] = np.linspace(0.0, 1.5, s["precip"].size).reshape(s["precip"].shape)
    step = gwm.StepConfig(dt=1.0, fast_substeps=4)
    rain = gwm.WarmRainConfig(dt=1.0, rain_terminal_velocity=12.0)
    spec = gwm.MemberSpec(step=step, rain=rain, moist=moist)
    with gwm.Model(g, spec) as m:
        m.set_tile("fast_substep", 3)
        m.set_tile("slow_stage", 3)
        m.set_tile("tracer_stage", 3)
        ref = s
        for _ in range(2):
            m.upload(ref)
            m.step(1)
            ref = m.download()
        host = _pinned_copy(s)
        for _ in range(2):
            m.step_host(host, out=host)      # the same buffers in and out
        fresh = m.step_host(s)               # pageable input, new output arrays
        m.upload(s)
        m.step(1)
        one = m.download()
    for k in ref:
        assert np.array_equal(ref[k], host[k]), k
        assert np.array_equal(one[k], fresh[k]), k


def test_step_host_arguments(gwm):
    g = gwm.GridSpec(20, 16, 6, dx=1000.0, dy=1000.0, z_top=6000.0)
    s = gwm.build_case("moist_sounding", g, gwm.CaseParams(), moist=True)
    with gwm.Model(g, gwm.MemberSpec(moist=True)) as m:
        partial = {k: v for k, v in s.items() if k != "qr"}
        with pytest.raises(ValueError):
            m.step_host(partial)
    with gwm.Model([g, g], [gwm.MemberSpec(), gwm.MemberSpec()]) as m2:
        with pytest.raises(ValueError):
            m2.step_host(s)
