"""The autotuner's search (mjolnir_b200/autotune.py) on a fake engine, on the
CPU: which launch shapes it tries, that half lists are tried only in the
mixed form, and that it applies the fastest shape it measured."""
import pytest

from mjolnir_b200 import autotune


class FakeEngine:
    """Records the knobs set and times each launch shape from a table."""

    def __init__(self, precision, cost):
        self.precision = precision
        self.cost = cost                      # (schedule, tpp, unroll, half) -> ms
        self.state = {"schedule": 0, "tpp": 1, "unroll": 1, "half": False}
        self.tried = []

    def set_half_lists(self, term, on):
        if self.precision != "mixed":
            raise RuntimeError("half lists need the mixed form")
        self.state["half"] = bool(on)

    def set_pair_schedule(self, term, s):
        self.state["schedule"] = s

    def set_threads_per_particle(self, term, p):
        self.state["tpp"] = p

    def set_pair_unroll(self, term, u):
        self.state["unroll"] = u

    def get_threads_per_particle(self, term):
        return self.state["tpp"]

    def time_kernel(self, term, reps=10):
        key = (self.state["schedule"], self.state["tpp"], self.state["unroll"], self.state["half"])
        self.tried.append(key)
        return self.cost(key)


def test_shapes_tried_in_the_mixed_form():
    e = FakeEngine("mixed", lambda k: 1.0)
    autotune._tune_shape(e, "exv", (1, 2, 4, 8, 16, 32), (1, 2, 4), (0, 1, 2, 3, 4, 5))
    tried = set(e.tried)
    assert len(tried) == len(e.tried)                       # no shape timed twice
    for half in (False, True):
        assert (0, 32, 4, half) in tried and (1, 16, 2, half) in tried
        # block-vector schedules: one partner batch, no 1- or 32-word blocks
        assert not any(k[0] in (2, 3) and (k[1] in (1, 32) or k[2] != 1) for k in tried)
        assert (3, 16, 1, half) in tried
        # slot-major lists: whole 32-byte sectors per group
        assert not any(k[0] == 5 and k[1] < 8 for k in tried)
        assert (5, 32, 1, half) in tried


def test_half_lists_only_in_the_mixed_form():
    e = FakeEngine("fp64", lambda k: 1.0)
    autotune._tune_shape(e, "dh", (1, 2, 4, 8, 16, 32), (1, 2, 4), (0, 2, 3, 4, 5))
    assert e.tried and not any(k[3] for k in e.tried)


@pytest.mark.parametrize("best", [(3, 2, 1, True), (4, 32, 2, False), (5, 8, 1, True)])
def test_the_fastest_measured_shape_is_applied(best):
    e = FakeEngine("mixed", lambda k: 0.5 if k == best else 1.0 + 0.01 * k[1])
    shape = autotune._tune_shape(e, "exv", (1, 2, 4, 8, 16, 32), (1, 2, 4), (0, 1, 2, 3, 4, 5))
    assert shape == best
    autotune._apply(e, "exv", shape)
    assert (e.state["schedule"], e.state["tpp"], e.state["unroll"], e.state["half"]) == best


def test_margin_choice_prefers_the_narrowest_within_one_percent(monkeypatch):
    """Whole-step times per margin (a fake clock): the fastest is 0.5, but
    0.3 is within 1 % of it and narrower, so 0.3 is kept; the build lanes
    are then chosen at that margin."""
    step_ms = {0.1: 1.0, 0.2: 0.8, 0.3: 0.795, 0.5: 0.79}
    lanes_ms = {4: 0.71, 8: 0.70, 16: 0.69, 32: 0.72}

    class Eng(FakeEngine):
        def __init__(self):
            super().__init__("mixed", lambda k: 1.0)
            self.margin, self.lanes, self.timing_lanes = None, None, False

        def set_margin(self, term, m):
            self.margin = m

        def set_build_lanes(self, term, lanes):
            self.lanes, self.timing_lanes = lanes, True

        def step(self, n):
            pass

    e = Eng()
    monkeypatch.setattr(autotune, "_time_steps",
                        lambda eng, n: lanes_ms[eng.lanes] if eng.timing_lanes else step_ms[eng.margin])
    choice = autotune.tune(e, terms=("exv",), margins=tuple(step_ms))
    assert choice["exv"]["margin"] == 0.3 and e.margin == 0.3
    assert choice["exv"]["build_lanes"] == 16 and e.lanes == 16
