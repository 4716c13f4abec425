"""Failure paths through the C-ABI, made without faulting or hanging the GPU.

* A non-finite value or a non-positive density in an uploaded state is reported as
  GWM_B200_ERR_STATE (-3) by the budget reduction, and a good state uploaded into the same
  context afterwards is accepted.
* A tile load that is never issued (a test-only request through
  gwm_b200_test_stall_tile_load: the wait is on a barrier nothing completes) makes the
  kernel's bounded wait run out: the step call returns GWM_B200_ERR_TIMEOUT (-5), the
  CTA drains the loads it did issue and exits, and the context stays usable: the next
  step from the same state matches a fresh context bit for bit.  In the persistent
  acoustic launch (all substeps of a stage in one cooperative kernel) the other CTAs
  find out at the grid barrier, whose wait is bounded the same way.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _moist(gwm, nx=72, ny=40, nz=16):
    g = gwm.GridSpec(nx, ny, nz, dx=2000.0, dy=2000.0, z_top=8000.0)
    p = gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=3, relative_humidity=1.02)
    s = gwm.build_case("moist_sounding", g, p, moist=True)
    spec = gwm.MemberSpec(step=gwm.StepConfig(dt=1.0, fast_substeps=3),
                          rain=gwm.WarmRainConfig(dt=1.0, rain_terminal_velocity=12.0), moist=True)
    return g, s, spec


@pytest.mark.parametrize("field,value", [("rho_theta", np.nan), ("rho", -0.5), ("rho", np.inf)])
def test_bad_uploaded_state_is_a_state_error(gwm, field, value):
    g, s, spec = _moist(gwm)
    bad = {k: v.copy() for k, v in s.items()}
    bad[field][3, 7, 11] = np.float32(value)
    with gwm.Model(g, spec) as m:
        m.upload(bad)
        with pytest.raises(RuntimeError, match="status -3"):
            m.budgets()
        m.upload(s)                      # the context takes a good state afterwards
        b = m.budgets()
        assert b["rho_min"] > 0 and np.isfinite(b["total_rho_theta_m"])


# (acoustic, slow, tracer) tiles per stalled kernel; "fast_stage": the substeps of a stage
# in one persistent launch, whose other CTAs then give up at the grid barrier
TILES = {"slow_stage": (0, 3, 16), "fast_substep": (3, 16, 16), "tracer_stage": (0, 16, 3),
         "fast_stage": (4, 3, 16)}


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("kernel", list(TILES))
def test_stalled_tile_load_times_out_and_context_recovers(gwm, kernel, graph):
    g, s, spec = _moist(gwm)

    def tiles(m):
        for name, r in zip(("fast_substep", "slow_stage", "tracer_stage"), TILES[kernel]):
            m.set_tile(name, r)

    with gwm.Model(g, spec) as ref:
        tiles(ref)
        ref.upload(s)
        ref.step(1)
        expect = ref.download()
    with gwm.Model(g, spec) as m:
        tiles(m)
        m.use_graph(graph)
        m.upload(s)
        m.test_stall_tile_load(plane=2)
        with pytest.raises(RuntimeError, match="status -5"):
            m.step(1)
        m.upload(s)
        m.step(1)                        # no request pending: a normal step
        got = m.download()
    for k in expect:
        assert np.array_equal(got[k], expect[k]), k
