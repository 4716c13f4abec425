"""Parity against golden vectors produced by the reference implementation itself.

``tests/golden/ref_<case>.npz`` hold an initial state, the case parameters and the
fields after N steps of the reference's own operators (advance_dry_state_ssprk3
with LocalSplitExplicitFastMode, advance_passive_tracers_ssprk3 and
apply_warm_rain_microphysics, built from the reference sources and run on a B200 by
tests/golden/make_golden.py).  The reference reduces its level means with float
atomics, so its FP32 output carries rounding of unspecified order; the checks below
are therefore envelopes, stated per field:

* the CPU oracle (FP64) must reproduce the reference to within a small multiple of
  the FP32 oracle's own rounding error, which pins the restatement to the reference;
* the CUDA path (through the C-ABI) must sit as close to the FP64 oracle as the
  reference itself does, and within the same bound of the reference's output.
"""
import glob
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
# step cases (the scalar-advection fixtures, ref_scalar_*, are tests/test_scalar.py's)
FILES = sorted(f for f in glob.glob(os.path.join(HERE, "golden", "ref_*.npz"))
               if not os.path.basename(f).startswith("ref_scalar_"))
NAMES = [os.path.basename(f)[4:-4] for f in FILES]
STATE = ("rho", "rho_theta", "u", "v", "w")
TRACERS = ("qv", "qc", "qr")
FACTOR = 3.0   # allowed ratio to the FP32 oracle's own rounding error
FLOORS = {"rho": 2e-6, "rho_theta": 2e-6, "u": 2e-4, "v": 2e-4, "w": 2e-4}


def load(name):
    z = np.load(os.path.join(HERE, "golden", f"ref_{name}.npz"))
    spec = json.loads(bytes(z["spec"]).decode())
    inp = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    out = {k[4:]: z[k] for k in z.files if k.startswith("out_")}
    return spec, inp, out, z["terrain"]


def err(a, b, base=None):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    scale = np.abs(b - base).max() if base is not None else np.abs(b).max()
    return float(np.abs(a - b).max() / max(scale, 1e-12))


def oracle_specs(orc, spec, terrain):
    g = spec["grid"]
    has_t = "terrain" in spec
    grid = orc.GridSpec(g["nx"], g["ny"], g["nz"], dx=g["dx"], dy=g["dy"], z_top=g["z_top"],
                        ranks_x=g.get("ranks_x", 1), ranks_y=g.get("ranks_y", 1),
                        periodic_x=g.get("periodic_x", True), periodic_y=g.get("periodic_y", True),
                        terrain=terrain.astype(np.float64) if has_t else None)
    st = spec["step"]
    step = orc.StepSpec(dt=st["dt"], fast_substeps=st["fast_substeps"],
                        fast_modes=st.get("fast_modes", True))
    phases, rain = orc.PHASE_DRY, None
    if spec.get("moist"):
        r = spec["rain"]
        phases |= orc.PHASE_TRACERS | (orc.PHASE_RAIN if r["mode"] == 1 else orc.PHASE_RAIN_NOMINAL)
        rain = orc.RainSpec(dt=st["dt"], terminal_velocity=r.get("terminal_velocity", 0.0),
                            layer_depth=r.get("layer_depth", 0.0))
    return grid, step, phases, rain


def oracle_runs(orc, name):
    spec, inp, ref, terrain = load(name)
    grid, step, phases, rain = oracle_specs(orc, spec, terrain)
    state = {k: np.asarray(v, np.float64) for k, v in inp.items()}
    if spec.get("moist"):
        state["precip"] = np.zeros((spec["grid"]["ny"], spec["grid"]["nx"]))
    o64 = orc.run(grid, step, state, spec["steps"], phases=phases, rain=rain, precision=64)
    o32 = orc.run(grid, step, state, spec["steps"], phases=phases, rain=rain, precision=32)
    return spec, inp, ref, o64, o32


def check_envelope(cand, ref, o64, o32, inp, tag):
    """cand within FACTOR x the FP32 envelope of the FP64 oracle, per field."""
    for k in STATE:
        base = None if k in ("rho", "rho_theta") else np.asarray(inp[k], np.float64)
        e_c, e_32 = err(cand[k], o64[k], base), err(o32[k], o64[k], base)
        assert np.isfinite(cand[k]).all(), f"{tag} {k}: non-finite"
        assert e_c <= max(FACTOR * e_32, FLOORS[k]), f"{tag} {k}: {e_c:.3e} vs fp32 envelope {e_32:.3e}"
    for k in TRACERS:
        if k in ref:
            e_c = err(cand[k], o64[k])
            assert e_c <= max(FACTOR * err(o32[k], o64[k]), 1e-4), f"{tag} {k}: {e_c:.3e}"
    if "precip" in ref:
        e_c = err(cand["precip"], o64["precip"])
        assert e_c <= max(FACTOR * err(o32["precip"], o64["precip"]), 1e-4), f"{tag} precip: {e_c:.3e}"


@pytest.mark.skipif(not FILES, reason="no golden vectors")
@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_reference(orc, name):
    spec, inp, ref, o64, o32 = oracle_runs(orc, name)
    check_envelope(ref, ref, o64, o32, inp, f"reference[{name}]")


@pytest.mark.gpu
@pytest.mark.skipif(not FILES, reason="no golden vectors")
@pytest.mark.parametrize("name", NAMES)
def test_cuda_path_matches_reference(gwm, orc, name):
    spec, inp, ref, o64, o32 = oracle_runs(orc, name)
    g = spec["grid"]
    gkw = dict(g)
    if "terrain" in spec:
        gkw["terrain"] = load(name)[3]
    grid = gwm.GridSpec(**gkw)
    st = spec["step"]
    step = gwm.StepConfig(dt=st["dt"], fast_substeps=st["fast_substeps"],
                          enable_fast_modes=st.get("fast_modes", True))
    moist = bool(spec.get("moist"))
    kw = {}
    if moist:
        r = spec["rain"]
        kw["rain"] = gwm.WarmRainConfig(dt=st["dt"], rain_terminal_velocity=r.get("terminal_velocity", 0.0),
                                        sedimentation_layer_depth_m=r.get("layer_depth", 0.0))
    state = {k: np.ascontiguousarray(v, np.float32) for k, v in inp.items()}
    if moist:
        state["precip"] = np.zeros((g["ny"], g["nx"]))
    with gwm.Model(grid, gwm.MemberSpec(step=step, moist=moist, **kw)) as m:
        m.upload(state)
        if not moist:
            m.advance_dry_state_ssprk3(spec["steps"])
        elif spec["rain"]["mode"] == 1:
            m.step(spec["steps"])          # the prepared-case driver step (metric fallout)
        else:
            for _ in range(spec["steps"]):  # the same sequence with the nominal overload
                m.advance_dry_state_ssprk3(1)
                m.advance_passive_tracers_ssprk3()
                m.apply_warm_rain_microphysics("nominal")
        out = m.download()
    check_envelope(out, ref, o64, o32, inp, f"cuda[{name}]")
    # and directly against the reference's own output
    for k in STATE:
        base = None if k in ("rho", "rho_theta") else np.asarray(inp[k], np.float64)
        e_ref = err(ref[k], o64[k], base)
        assert err(out[k], ref[k], base) <= max(2 * FACTOR * err(o32[k], o64[k], base), e_ref, FLOORS[k]) * 2, k
