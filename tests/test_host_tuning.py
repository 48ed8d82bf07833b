"""Host logic of the measurement tools, on CPU: the launch-shape tuner's choice (every
candidate timed on the handle, the fastest set last, only the knobs that apply to the
handle's systems), and the roofline's per-workload DRAM traffic lookup."""
import pytest

from nuvort_b200.abi import make_params


class _FakeHandle:
    """Stands in for a handle: the setters record the shape, and a velocity pass 'takes' the
    time the table gives for the current shapes (no GPU)."""

    def __init__(self, params, cost):
        self.params = params
        self.cost = cost  # (walk_parts, direct_split) -> ms
        self.parts, self.split = 0, 0
        self.set_calls = []
        self.now = 0.0

    def set_walk_parts(self, c):
        self.parts = c
        self.set_calls.append(("parts", c))

    def set_direct_split(self, c):
        self.split = c
        self.set_calls.append(("split", c))

    def calc_velocity(self, sys=0):
        self.now += self.cost(self.parts, self.split) * 1e-3


@pytest.fixture
def fake_clock(monkeypatch):
    import time
    box = {}

    def perf_counter():
        return box["h"].now
    monkeypatch.setattr(time, "perf_counter", perf_counter)
    return box


def test_mixed_tree_handle_tunes_walk_parts_only(fake_clock):
    from nuvort_b200.autotune import tune_launch_shapes
    p = make_params(velocity="Tree", tree_theta=0.4, precision="mixed")
    q = make_params(velocity="BS", precision="mixed")  # a mixed direct sum has no split knob
    h = _FakeHandle([p, q], lambda parts, split: {1: 5.0, 2: 4.0, 4: 3.0, 8: 3.5}[parts])
    fake_clock["h"] = h
    r = tune_launch_shapes(h, repeats=2)
    assert r["walk_parts"]["choice"] == 4
    assert r["walk_parts"]["ms"] == pytest.approx({1: 5.0, 2: 4.0, 4: 3.0, 8: 3.5})
    assert "direct_split" not in r
    assert h.set_calls[-1] == ("parts", 4) and h.parts == 4


def test_plain_handle_tunes_both_knobs(fake_clock):
    from nuvort_b200.autotune import tune_launch_shapes
    p = make_params(velocity="Tree", tree_theta=0.4)
    q = make_params(velocity="BS")
    cost = lambda parts, split: (2.0 if parts == 2 else 3.0) + {64: 4.0, 8: 1.0, 4: 2.0, 2: 3.0, 1: 5.0}.get(split, 9.0)
    h = _FakeHandle([p, q], cost)
    fake_clock["h"] = h
    r = tune_launch_shapes(h, repeats=1)
    assert set(r["walk_parts"]["ms"]) == {1, 2} and r["walk_parts"]["choice"] == 2
    assert set(r["direct_split"]["ms"]) == {64, 8, 4, 2, 1} and r["direct_split"]["choice"] == 8
    assert (h.parts, h.split) == (2, 8)


def test_traffic_lookup_is_per_workload():
    import bench
    t = bench.profile_traffic("k_tree_walk_mixed", "ensemble512")
    assert t["workload"] == "ensemble512" and t["bytes_per_launch"] > 1e9
    assert t["source"].startswith("profiles/")
    assert bench.profile_traffic("k_tree_walk_mixed", "tangle1m")["bytes_per_launch"] > 1e9
    assert bench.profile_traffic("k_tree_walk_fp64", "ensemble512") is None  # no capture: no figure
    assert bench.profile_traffic("k_no_such_kernel", "tangle32k") is None
