"""Autotuner host logic on CPU: the launch-shape knobs of the C ABI (set,
get, rejection of unknown knobs and out-of-range values), and the tuner's
choice of the fastest candidate, its on-disk cache and cache reuse, with an
injected timer (no GPU)."""

import json

import pytest

from dequantizer_b200 import _lib, autotune


@pytest.fixture(autouse=True)
def _reset_knobs():
    yield
    autotune.set_knobs({k: 0 for k in autotune.KNOBS})


def test_knobs_roundtrip_and_validation():
    lib = _lib.lib()
    cfg = {"gauge_edge_warps": 4, "gauge_dist_warps": 2, "gauge_path": 1, "su_grid": 100, "su_onchip": 1,
           "sweep_onecta": 2}
    autotune.set_knobs(cfg)
    assert autotune.get_knobs() == cfg
    assert lib.dqz_set_tuning(autotune.KNOBS["su_onchip"], 5) == _lib.DQZ_ERR_ARG
    assert lib.dqz_set_tuning(autotune.KNOBS["sweep_onecta"], 3) == _lib.DQZ_ERR_ARG
    assert lib.dqz_set_tuning(autotune.KNOBS["gauge_edge_warps"], 9) == _lib.DQZ_ERR_ARG
    assert lib.dqz_set_tuning(autotune.KNOBS["gauge_path"], 3) == _lib.DQZ_ERR_ARG
    assert lib.dqz_set_tuning(99, 1) == _lib.DQZ_ERR_ARG
    assert lib.dqz_set_tuning(0, -1) == _lib.DQZ_ERR_ARG
    assert lib.dqz_get_tuning(99) == -1


def test_tuner_picks_fastest_and_reuses_cache(tmp_path):
    path = str(tmp_path / "tune.json")
    cost = {1: 3.0, 2: 1.0, 4: 2.0}
    calls = []

    def timer(run):
        run()
        w = autotune.get_knobs()["gauge_edge_warps"]
        calls.append(w)
        return cost[w]

    t = autotune.Tuner(path, timer=timer)
    key = t.key("gauge", "dev", chi=8, deg=3)
    best = t.tune(key, [{"gauge_edge_warps": w} for w in (1, 2, 4)], lambda: None)
    assert best == {"gauge_edge_warps": 2} and calls == [1, 2, 4]
    assert autotune.get_knobs()["gauge_edge_warps"] == 2
    assert json.load(open(path))[key] == {"gauge_edge_warps": 2}
    autotune.set_knobs({"gauge_edge_warps": 0})
    t2 = autotune.Tuner(path, timer=timer)
    assert t2.tune(key, [{"gauge_edge_warps": w} for w in (1, 2, 4)], lambda: None) == {"gauge_edge_warps": 2}
    assert calls == [1, 2, 4] and t2.timed_keys == []  # cache hit: nothing timed
    assert autotune.get_knobs()["gauge_edge_warps"] == 2
