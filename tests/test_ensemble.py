"""Uneven ensemble members in one context: concurrent graph branches, sequential
execution and each member on its own give the same result bit for bit."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_ensemble_branches_bit_exact(gwm):
    ens = importlib.import_module("gpu-wm-next_b200.ensemble")
    grids, specs, states, damping, kinds = ens.c5_members(8, seed=3, size_range=(40, 120), nz_choices=(16, 24))
    assert set(kinds) == set(ens.CASES)
    outs = {}
    for mode in ("concurrent", "sequential"):
        with ens.build_model(grids, specs, states, damping, concurrent=(mode == "concurrent")) as m:
            m.use_graph(True)
            m.step(3)
            outs[mode] = [m.download(member=i) for i in range(len(grids))]
    for i in (0, 2, 3):   # a dry flat, the terrain and a moist member on their own
        with ens.build_model([grids[i]], [specs[i]], [states[i]], [damping[i]]) as m:
            m.use_graph(True)
            m.step(3)
            alone = m.download()
        for k in alone:
            assert np.array_equal(alone[k], outs["concurrent"][i][k]), (i, k)
    for i in range(len(grids)):
        for k in outs["sequential"][i]:
            assert np.array_equal(outs["sequential"][i][k], outs["concurrent"][i][k]), (i, k)
            assert np.isfinite(outs["concurrent"][i][k]).all(), (i, k)
