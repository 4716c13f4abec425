"""Model.autotune's selection on the host, no GPU: the device calls of a Model are replaced
by a fake whose step time depends on the tiles set, so the candidates, the greedy choice
per kernel (slow stage, then acoustic substep, then tracer stage) and the two timing modes
(per-launch profiling events; whole graph-replayed steps) can be checked exactly."""
import time

import pytest

SLOW = {3: 1.0, 8: 2.0, 16: 1.5}
FAST = {0: 2.0, 3: 0.5, 8: 1.2, 16: 1.1}
COLREF = {0: 0.3, 3: 0.3, 8: 0.3, 16: 0.3}   # terrain: a column reference before each substep
TRACER = {3: 0.3, 8: 0.4, 16: 0.2}


def _fake(gwm, monkeypatch, terrain=False):
    m = gwm.Model.__new__(gwm.Model)  # no context: every device call below is a fake
    st = {"tiles": {"slow_stage": 16, "fast_substep": 0, "tracer_stage": 16}, "graph": False,
          "steps": 0, "clock": 0.0, "prof": False, "rep": {}}

    def step_cost(t):
        c = 3 * SLOW[t["slow_stage"]] + 6 * FAST[t["fast_substep"]] + 3 * TRACER[t["tracer_stage"]]
        return c + (6 * COLREF[t["fast_substep"]] if terrain else 0.0)

    def step(n=1):
        t = st["tiles"]
        st["steps"] += n
        st["clock"] += n * step_cost(t) * 1e-3
        if st["prof"]:
            rep = st["rep"]
            for name, per, count in (("k_slow_stage", SLOW[t["slow_stage"]], 3),
                                     ("k_fast_substep", FAST[t["fast_substep"]], 6),
                                     ("k_tracer_stage", TRACER[t["tracer_stage"]], 3)) + \
                    ((("k_column_reference", COLREF[t["fast_substep"]], 6),) if terrain else ()):
                e = rep.setdefault(name, {"total_ms": 0.0, "launches": 0})
                e["total_ms"] += n * per * count
                e["launches"] += n * count

    def profile(on=True):
        st["prof"] = on
        if on:
            st["rep"] = {}

    monkeypatch.setattr(m, "set_tile", lambda k, r: st["tiles"].__setitem__(k, r), raising=False)
    monkeypatch.setattr(m, "get_tile", lambda k: st["tiles"][k], raising=False)
    monkeypatch.setattr(m, "use_graph", lambda on=True: st.__setitem__("graph", on), raising=False)
    monkeypatch.setattr(m, "synchronize", lambda: None, raising=False)
    monkeypatch.setattr(m, "step", step, raising=False)
    monkeypatch.setattr(m, "profile", profile, raising=False)
    monkeypatch.setattr(m, "profile_report",
                        lambda: {k: dict(v, avg_ms=v["total_ms"] / v["launches"]) for k, v in st["rep"].items()},
                        raising=False)
    monkeypatch.setattr(time, "perf_counter", lambda: st["clock"])
    return m, st


def test_autotune_per_launch_picks_the_fastest_tiles(gwm, monkeypatch):
    m, st = _fake(gwm, monkeypatch)
    best = m.autotune(1)
    assert best == {"slow_stage": 3, "fast_substep": 3, "tracer_stage": 16}
    assert st["tiles"] == best
    assert m.tile_times["fast_substep"] == pytest.approx(FAST)   # per substep launch
    assert st["steps"] == 10 and not st["graph"]


def test_autotune_charges_a_terrain_substep_its_column_reference(gwm, monkeypatch):
    m, _ = _fake(gwm, monkeypatch, terrain=True)
    m.autotune(1)
    assert m.tile_times["fast_substep"] == pytest.approx({r: FAST[r] + COLREF[r] for r in FAST})


def test_autotune_whole_step_times_graph_replayed_steps(gwm, monkeypatch):
    m, st = _fake(gwm, monkeypatch)
    best = m.autotune(2, whole_step=True)
    assert best == {"slow_stage": 3, "fast_substep": 3, "tracer_stage": 16}
    assert st["graph"]                       # graph replay left on
    assert st["steps"] == 10 * (1 + 2)       # one warm-up step per candidate, then two timed
    # whole-step times: the slow stage was tuned first, with the other kernels at their tiles then
    slow_times = m.tile_times["slow_stage"]
    assert slow_times[3] < slow_times[16] < slow_times[8]
    assert slow_times[3] == pytest.approx(3 * SLOW[3] + 6 * FAST[0] + 3 * TRACER[16], rel=1e-9)
