"""bench.learned_setup's choice of the learned configuration, on a fake
layout (no GPU): each hub-target candidate runs at its own largest theta
whose error is not above the plain walk's, the fastest candidate that
reaches theta 1.2 wins (the fastest of all when none does), a fixed
--hub-targets count is kept, and layouts up to 2^20 vertices are judged on
every vertex (a 65,536-vertex sample above)."""
import types

import numpy as np
import pytest

import bench


class _Model:
    def __init__(self, seed=0):
        pass

    def train(self, *a, **k):
        return [1.0, 0.5]

    def attach(self, lay):
        pass


class _Layout:
    """Repulsion error grows with theta and shrinks with hub targets; a
    step's time falls with theta and rises with hub targets."""

    def __init__(self, V):
        self.V = V
        self.p = {}
        self.judged = None

    def step(self):
        pass

    def set_params(self, **kw):
        self.p.update(kw)

    def _err(self):
        th = self.p.get("theta", 0.5)
        if not self.p.get("farField"):
            return 0.003 * th / 0.5
        k = self.p.get("farHubTargets", 0)
        return 0.0025 * (th / 1.1) ** 4 * (1.0 - 0.2 * (k > 0) - 0.05 * (k > self.V // 1024))

    def exact_repulsion(self, t):
        self.judged = (self.judged or 0) + len(t)
        return np.ones((len(t), 2))

    def repulsion(self):
        return np.ones((self.V, 2)) * (1.0 + self._err())

    def positions(self):
        return np.zeros(2 * self.V)

    def fa2_state(self):
        return np.zeros(2 * self.V), 1.0, 1.0

    def set_positions(self, x):
        pass

    def set_fa2_state(self, *a):
        pass

    def time_steps(self, n):
        th = self.p.get("theta", 0.5)
        k = self.p.get("farHubTargets", 0)
        return n * (3.0 - th + 0.3 * k / self.V)


@pytest.fixture
def fake_training(monkeypatch):
    import grapher_b200.farfield as ff
    monkeypatch.setattr(ff, "FarFieldModel", _Model)
    monkeypatch.setattr(ff, "harvest_training_set",
                        lambda lay, th, t: (np.zeros((4, 10), np.float32),
                                            np.zeros((4, 2), np.float32),
                                            np.ones(4, np.float32)))


def _setup(V, hub_targets="auto"):
    lay = _Layout(V)
    w = types.SimpleNamespace(V=V, spec={"theta": 0.5})
    _, info = bench.learned_setup(lay, w, lambda x: x, hub_targets)
    return lay, info


def test_candidates_take_their_largest_qualifying_theta(fake_training):
    lay, info = _setup(1 << 16)
    counts = [c["hub_targets"] for c in info["candidates"]]
    assert counts == [0, (1 << 16) // 1024, (1 << 16) // 256]
    plain = info["plain_rms_err"]
    for c in info["candidates"]:
        table = info["learned_errors_by_hub_targets"][str(c["hub_targets"])]
        ok = [float(t) for t, e in table.items() if e["rms_err"] <= plain]
        assert c["theta"] == max(ok)
        assert c["rms_err"] <= plain
        assert set(table[str(c["theta"])]) == {"rms_err", "rms_rel_err_per_vertex",
                                               "max_err_over_rms_force"}


def test_fastest_candidate_wins(fake_training):
    _, info = _setup(1 << 16)
    at_target = [c for c in info["candidates"] if c["theta"] >= bench.TARGET_THETA]
    assert at_target
    best = min(at_target, key=lambda c: c["ms_per_step"])
    assert info["hub_targets"] == best["hub_targets"]
    assert info["learned_theta"] == best["theta"]
    p = bench.learned_params(info)
    assert p["farHubTargets"] == best["hub_targets"] and p["theta"] == best["theta"]


def test_fixed_hub_count_is_kept(fake_training):
    _, info = _setup(1 << 16, "100")
    assert info["hub_choice"] == "fixed" and info["hub_targets"] == 100
    _, info = _setup(1 << 16, "0")
    assert info["hub_targets"] == 0 and len(info["candidates"]) == 1


def test_every_vertex_judged_up_to_2_pow_20(fake_training):
    lay, info = _setup(1 << 20)
    assert info["judge_vertices"] == 1 << 20 and lay.judged == 1 << 20
    lay, info = _setup((1 << 20) + 1)
    assert info["judge_vertices"] == bench.JUDGE_VERTICES == lay.judged


def test_candidates_reaching_the_target_theta_are_preferred():
    c = [{"hub_targets": 0, "theta": 1.1, "ms_per_step": 1.70},
         {"hub_targets": 1024, "theta": 1.175, "ms_per_step": 1.72},
         {"hub_targets": 4096, "theta": 1.2, "ms_per_step": 1.74},
         {"hub_targets": 16384, "theta": 1.25, "ms_per_step": 1.80}]
    assert bench.pick_candidate(c) == 4096
    assert bench.pick_candidate(c[:2]) == 0  # none reaches it: the fastest
