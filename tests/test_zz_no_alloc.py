"""The allocation-free statistics entry point, checked against the budget reduction.

Some callers cannot allocate device memory where they call us (their own pool owns
the device, or cudaMalloc's implicit synchronisation is forbidden there), so
gwm_b200_field_stats_noalloc keeps its scratch in a fixed device array inside the
library.  This test calls it through the C-ABI twice in a row, on two fields of
different sizes, and compares each result with the context-based budget reduction
of the same field.  The file is named to be collected last.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_field_stats_noalloc_matches_budgets(gwm):
    import torch
    assert torch.cuda.is_available(), "GPU test"
    g = gwm.GridSpec(40, 36, 24, dx=1000.0, dy=1000.0, z_top=12000.0)
    p = gwm.CaseParams(rho_surface=1.16, theta_ref=300.0, theta_perturbation=2.0, center_z_fraction=0.3,
                       radius_x_fraction=0.2, radius_y_fraction=0.2, radius_z_fraction=0.25)
    s = gwm.build_case("hydrostatic_warm_bubble", g, p)
    with gwm.Model(g, gwm.MemberSpec(step=gwm.StepConfig(dt=1.0, fast_substeps=2))) as m:
        m.upload(s)
        m.advance_dry_state_ssprk3(1)
        b = m.budgets()
        f = m.download(keys=["rho", "u"])
    cases = [(f["rho"], b["total_dry_mass"], b["rho_min"], b["rho_max"]),
             (f["u"], b["total_horizontal_momentum_x"], b["u_min"], b["u_max"])]
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    for field, total, mn, mx in cases:  # two calls in a row, different sizes
        x = torch.tensor(np.ascontiguousarray(field).ravel(), device="cuda")
        out.fill_(np.nan)
        gwm.field_stats_noalloc(x.data_ptr(), x.numel(), out.data_ptr())
        torch.cuda.synchronize()
        got_sum, got_min, got_max = out.cpu().tolist()
        # both reductions are FP64 in a fixed order; only the summation order differs
        assert got_sum == pytest.approx(total, rel=1e-12, abs=1e-9)
        assert got_min == mn and got_max == mx
    with pytest.raises(RuntimeError):
        gwm.field_stats_noalloc(x.data_ptr(), 0, out.data_ptr())


def test_field_stats_noalloc_large_input_allocates_nothing(gwm):
    # 3,000,000 values: more than the 1024 blocks x 2048 values one pass covers, so each
    # thread of the first pass strides over several chunks (the capped branch).  Device
    # free memory is the same before and after the calls that follow the first one.
    import torch
    rng = np.random.default_rng(12)
    n = 3_000_000
    host = rng.normal(5.0, 3.0, n).astype(np.float32)
    host[1234567] = np.float32(-40.0)
    host[2999999] = np.float32(77.0)
    x = torch.tensor(host, device="cuda")
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    gwm.field_stats_noalloc(x.data_ptr(), n, out.data_ptr())   # first call on the device
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        out.fill_(np.nan)
        gwm.field_stats_noalloc(x.data_ptr(), n, out.data_ptr())
        torch.cuda.synchronize()
        s, mn, mx = out.cpu().tolist()
        exact = host.astype(np.float64)
        assert s == pytest.approx(exact.sum(), rel=1e-12)
        assert mn == -40.0 and mx == 77.0
    assert torch.cuda.mem_get_info()[0] == free0
