"""Parity at the benchmarked sizes, and the error growth of the benchmark case over time.

* The moist warm-rain member exactly as ``bench.py`` builds and runs it (1024 x 1024 x 64,
  3 km, 16 km top, the seeded sounding, TMA-fed slow/acoustic/tracer kernels, warm rain
  with fallout, CUDA-graph replay) advanced two steps, against the FP64 and FP32 oracles.
* The mountain-wave configuration at its full size (512 x 512 x 80, Agnesi hill,
  stretched hybrid-height levels to 20 km, constant N = 0.01, Rayleigh layer above
  14 km, 6 acoustic substeps) advanced two steps.
* The error of the moist benchmark case against the FP64 oracle every 50 steps over its
  first 300 s (64 x 64 x 64, dt 1 s), beside the error of the reference's FP32 arithmetic
  (the FP32 oracle) on the same trajectory.  The discretisation is unstable at the
  configured 12 s step and goes convective within minutes, so "1e-4 after one simulated
  hour" is replaced by this record over the stable window.

The oracle runs on the host cores (OpenMP); the 1024^2 case needs about 40 GB of host
memory for the FP64 oracle and skips itself where the host has less.
"""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _rel(a, b, floor=1e-12):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), floor))


def _pert(a, b, base):
    a, b, base = (np.asarray(x, np.float64) for x in (a, b, base))
    return float(np.abs(a - b).max() / max(np.abs(b - base).max(), 1e-12))


def _envelope(out, ref64, ref32, keys, base=None, floor=1e-6, factor=2.0, tag=""):
    rep = {}
    for k in keys:
        if base is not None:
            e, e32 = _pert(out[k], ref64[k], base[k]), _pert(ref32[k], ref64[k], base[k])
        else:
            e, e32 = _rel(out[k], ref64[k]), _rel(ref32[k], ref64[k])
        rep[k] = (e, e32)
        assert np.isfinite(out[k]).all(), f"{tag} {k}: non-finite"
        assert e <= max(factor * e32, floor), f"{tag} {k}: gpu {e:.3e} vs fp32 envelope {e32:.3e}"
    return rep


def _host_gb():
    try:
        import psutil
        return psutil.virtual_memory().available / 2**30
    except Exception:
        return float("inf")


def _oracle(orc):
    orc.set_threads(orc.max_threads())
    return orc


def test_c3_bench_member_vs_oracles(gwm, orc):
    import bench
    if _host_gb() < 48:
        pytest.skip(f"the FP64 oracle at 1024x1024x64 needs ~40 GB of host memory ({_host_gb():.0f} GB free)")
    _oracle(orc)
    g = bench.grid_spec(gwm)
    state = gwm.build_case("moist_sounding", g, bench.case_params(gwm), moist=True)
    with gwm.Model(g, bench.member_spec(gwm)) as m:
        for kernel in ("slow_stage", "fast_substep", "tracer_stage"):
            m.set_tile(kernel, 3)
        m.use_graph(True)
        m.upload(state)
        m.step(2)
        out = m.download()
    og = orc.GridSpec(g.nx, g.ny, g.nz, dx=g.dx, dy=g.dy, z_top=g.z_top)
    kw = dict(phases=orc.PHASE_DRY | orc.PHASE_TRACERS | orc.PHASE_RAIN,
              rain=orc.RainSpec(dt=bench.DT, terminal_velocity=bench.VT))
    step = orc.StepSpec(dt=bench.DT, fast_substeps=bench.NS)
    st64 = {k: v.astype(np.float64) for k, v in state.items()}
    ref = orc.run(og, step, st64, 2, precision=64, **kw)
    ref32 = orc.run(og, step, st64, 2, precision=32, **kw)
    _envelope(out, ref, ref32, ("rho", "rho_theta"), floor=1e-6, tag="c3")
    _envelope(out, ref, ref32, ("u", "v", "w"), base=st64, floor=1e-4, tag="c3")
    for k in ("qv", "qc", "qr"):
        assert _rel(out[k], ref[k], floor=1e-9) < 1e-3, k
    assert _rel(out["precip"], ref["precip"], floor=1e-12) < 1e-3


def test_c2_full_size_vs_oracles(gwm, orc):
    if _host_gb() < 24:
        pytest.skip(f"the FP64 oracle at 512x512x80 needs ~12 GB of host memory ({_host_gb():.0f} GB free)")
    _oracle(orc)
    import bench
    g, s = bench.c2_grid_and_state(gwm)
    uref = s["u"].astype(np.float64).mean(axis=(1, 2))
    # dt 0.5 s: c dt / dz = 0.95 on the 183 m bottom levels (the slow step is bounded by
    # the acoustic CFL of the reference discretisation, about 1.4)
    step = gwm.StepConfig(dt=0.5, fast_substeps=6)
    with gwm.Model(g, gwm.MemberSpec(step=step)) as m:
        m.use_graph(True)
        m.upload(s)
        m.set_damping(14000.0, 0.05, u_ref=uref)
        m.advance_dry_state_ssprk3(2)
        out = m.download()
    og = orc.GridSpec(g.nx, g.ny, g.nz, dx=g.dx, dy=g.dy, z_top=g.z_top, terrain=g.terrain.astype(np.float64),
                      eta_interfaces=g.eta_interfaces)
    ost = orc.StepSpec(dt=0.5, fast_substeps=6, damp_z_bottom=14000.0, damp_rate=0.05, damp_u_ref=uref,
                       damp_v_ref=np.zeros(g.nz))
    st64 = {k: v.astype(np.float64) for k, v in s.items()}
    ref = orc.run(og, ost, st64, 2, precision=64)
    ref32 = orc.run(og, ost, st64, 2, precision=32)
    _envelope(out, ref, ref32, ("rho", "rho_theta"), floor=2e-6, factor=3.0, tag="c2")
    _envelope(out, ref, ref32, ("u", "v", "w"), base=st64, floor=2e-4, factor=3.0, tag="c2")


def test_c3_error_growth_over_the_stable_window(gwm, orc):
    """Relative L2 error per field against the FP64 oracle every 50 steps over 300 s,
    for this path and for the reference's FP32 arithmetic; written as JSON to
    $GWM_B200_RECORD (when set)."""
    import bench
    _oracle(orc)
    n, every, total = 64, 50, 300
    g = bench.grid_spec(gwm, n, n)
    state = gwm.build_case("moist_sounding", g, bench.case_params(gwm), moist=True)
    og = orc.GridSpec(n, n, bench.NZ, dx=g.dx, dy=g.dy, z_top=g.z_top)
    kw = dict(phases=orc.PHASE_DRY | orc.PHASE_TRACERS | orc.PHASE_RAIN,
              rain=orc.RainSpec(dt=bench.DT, terminal_velocity=bench.VT))
    ostep = orc.StepSpec(dt=bench.DT, fast_substeps=bench.NS)
    keys = ("rho", "rho_theta", "u", "v", "w", "qv", "qc", "qr", "precip")

    def l2(a, b):
        a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
        return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))

    rec = []
    s64 = s32 = {k: v.astype(np.float64) for k, v in state.items()}
    with gwm.Model(g, bench.member_spec(gwm)) as m:
        for kernel in ("slow_stage", "fast_substep", "tracer_stage"):
            m.set_tile(kernel, 3)
        m.use_graph(True)
        m.upload(state)
        for t in range(every, total + 1, every):
            m.step(every)
            out = m.download()
            s64 = orc.run(og, ostep, s64, every, precision=64, **kw)
            s32 = orc.run(og, ostep, s32, every, precision=32, **kw)
            rec.append({"t_s": t * bench.DT,
                        "gpu_vs_fp64": {k: l2(out[k], s64[k]) for k in keys},
                        "fp32_oracle_vs_fp64": {k: l2(s32[k], s64[k]) for k in keys}})
    path = os.environ.get("GWM_B200_RECORD")
    if path:
        with open(path, "w") as f:
            json.dump({"case": f"moist warm-rain benchmark case, {n}x{n}x{bench.NZ}, dt {bench.DT} s, "
                               f"{bench.NS} substeps", "relative_l2": rec}, f, indent=1)
    for r in rec:
        for k in keys:
            e, e32 = r["gpu_vs_fp64"][k], r["fp32_oracle_vs_fp64"][k]
            assert np.isfinite(e), (r["t_s"], k)
            # this path carries FP64 level sums and the perturbation EOS: it stays at least
            # as close to the FP64 discretisation as the reference's own FP32 arithmetic
            assert e <= max(2.0 * e32, 1e-6), (r["t_s"], k, e, e32)
