"""The reference's own regression tests, run through the drop-in adapter.

`make -C oracle adapter-tests` (run by build() where the reference tree is present) links
each of gpu-wm-next's tests/regression programs against
gpu-wm-next_b200/adapter/gwm_b200_adapter.cpp, which defines advance_dry_state_ssprk3,
LocalSplitExplicitFastMode::apply, advance_passive_tracers_ssprk3, advance_scalar_ssprk3
and both apply_warm_rain_microphysics overloads over libgwm_b200 with the reference's
signatures.  The programs keep the reference's state types, initialisers, summaries and
assertions; their step operators run on the device path.  Each must exit 0, and the
adapter's call report must show that the operators it exercises ran in the adapter.
"""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "adapter")

# program -> adapter operators it must have called
PROGRAMS = {
    "test_dry_constant_state_bundle": ["advance_dry_state_ssprk3"],
    "test_hydrostatic_rest": ["advance_dry_state_ssprk3"],
    "test_terrain_hydrostatic_rest": ["advance_dry_state_ssprk3"],
    "test_acoustic_pulse": ["fast_modes"],
    "test_buoyancy_response": ["advance_dry_state_ssprk3"],
    "test_density_current_evolution": ["advance_dry_state_ssprk3"],
    "test_horizontal_pressure_response": ["advance_dry_state_ssprk3"],
    "test_mountain_wave_evolution": ["advance_dry_state_ssprk3"],
    "test_constant_state": ["advance_scalar_ssprk3"],
    "test_scalar_mass_conservation": ["advance_scalar_ssprk3", "advance_passive_tracers_ssprk3"],
    "test_warm_rain_closed_box": ["apply_warm_rain_microphysics(box)"],
    "test_warm_rain_summary_closure": ["apply_warm_rain_microphysics(metric)"],
}


@pytest.mark.parametrize("program", list(PROGRAMS))
def test_reference_regression_through_adapter(program):
    exe = os.path.join(BIN, program)
    if not os.path.exists(exe):
        pytest.skip("adapter programs not built (the reference tree was absent at build time)")
    env = dict(os.environ, GWM_B200_ADAPTER_REPORT="1")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, (r.stdout + r.stderr)[-3000:]
    calls = {}
    for line in r.stderr.splitlines():
        if line.startswith("gwm_b200 adapter: "):
            name, n = line[len("gwm_b200 adapter: "):].rsplit(" ", 1)
            calls[name] = int(n)
    for op in PROGRAMS[program]:
        assert calls.get(op, 0) > 0, (op, calls)
