"""Scalar advection: advance_scalar_ssprk3 (src/dycore/dry_transport.cu:285-325).

The golden vectors come from the reference itself (tests/golden/make_golden.py runs
its advance_scalar_ssprk3 on virtual-rank layouts): four cases, three in the
configurations of the reference's own tests.  CPU: the oracle restatement meets the
reference's known answers (test_constant_state.cpp: a constant stays within 1e-5;
test_scalar_mass_conservation.cpp: mass within 1e-3) and the golden vectors.  GPU:
gwm_b200_scalar_ssprk3 reproduces the golden vectors bit for bit, the virtual-rank
layouts included (test_virtual_rank_equivalence.cpp asks 1e-5), and the FP64 oracle to
rounding.
"""
import glob
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "ref_scalar_*.npz")))


def _load(path):
    z = np.load(path)
    return json.loads(bytes(z["spec"]).decode()), z["in_q"], z["out_q"]


def _args(c):
    return dict(u_adv=c["u"], v_adv=c["v"], dt=c["dt"], dx=1000.0, dy=1000.0, periodic_x=c["px"],
                periodic_y=c["py"], nsteps=c["steps"])


def test_golden_scalar_fixtures_present():
    assert len(FIXTURES) == 4, FIXTURES


def test_oracle_scalar_reference_kats(orc):
    q = np.full((3, 24, 24), 7.5)
    assert np.abs(orc.scalar_ssprk3(q, 20.0, -10.0, 4.0, precision=32) - 7.5).max() <= 1e-5
    j, i = np.meshgrid(np.arange(20), np.arange(32), indexing="ij")
    q = (1.0 + 0.1 * ((i + 2 * j) % 7)).astype(np.float32)[None]
    out = orc.scalar_ssprk3(q, 12.0, 7.0, 2.0, precision=32)
    assert abs(out.sum() - q.astype(np.float64).sum()) <= 1e-3


@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p))
def test_oracle_scalar_matches_reference(orc, path):
    c, q, ref = _load(path)
    a = _args(c)
    out32 = orc.scalar_ssprk3(q, a["u_adv"], a["v_adv"], a["dt"], periodic_x=c["px"], periodic_y=c["py"],
                              nsteps=c["steps"], precision=32)
    assert np.array_equal(out32.astype(np.float32), ref)  # FP32 restatement: the reference's roundings


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=lambda p: os.path.basename(p))
def test_scalar_ssprk3_bit_exact_vs_reference(gwm, orc, path):
    c, q, ref = _load(path)
    out = gwm.scalar_ssprk3(q, **_args(c))
    assert out.dtype == np.float32 and out.shape == ref.shape
    assert np.array_equal(out, ref), np.abs(out - ref).max()
    # and the FP64 restatement, to FP32 rounding accumulated over the steps
    a = _args(c)
    out64 = orc.scalar_ssprk3(q, a["u_adv"], a["v_adv"], a["dt"], periodic_x=c["px"], periodic_y=c["py"],
                              nsteps=c["steps"], precision=64)
    assert np.abs(out - out64).max() <= 1e-6 * np.abs(out64).max() * c["steps"]


@pytest.mark.gpu
def test_scalar_ssprk3_device_tensor_in_place(gwm):
    import torch
    c, q, ref = _load(os.path.join(GOLDEN, "ref_scalar_wave.npz"))
    t = torch.from_numpy(q).cuda()
    a = _args(c)
    a["nsteps"] = 20
    for _ in range(3):  # 3 calls of 20 steps = the 60-step golden run
        assert gwm.scalar_ssprk3(t, **a) is t
    assert np.array_equal(t.cpu().numpy(), ref)
    with pytest.raises(ValueError):
        gwm.scalar_ssprk3(t.double(), **a)
