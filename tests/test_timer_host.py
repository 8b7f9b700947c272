"""Host logic of the Timer facade (opentimer_b200.timer.Timer) over a fake
device design: the operation queue (runs of resizes as one batch, change
SPEFs in order between them, queries applying what is pending), the
argument checks of repower_gate, and the endpoint reductions of
report_wns / report_tns (Timer::_update_endpoints, report_wns/tns:
minimum slack; sum of negative slacks in float32, per corner, then over
the corners asked for)."""
import numpy as np
import pytest

from opentimer_b200.timer import MAX, MIN, RISE, FALL, Timer


class FakeDesign:
    def __init__(self):
        self.calls = []
        self.names = ["a", "b", "c", "d"]
        self.endpoints = np.array([1, 3], np.int64)
        self.slack = np.array([[1, 1, 1, 1],
                               [-2.0, 0.5, -1.0, np.nan],
                               [9, 9, 9, 9],
                               [-3.0, -0.25, 4.0, -1.5]], np.float32)

    def resize(self, batch):
        self.calls.append(("resize", list(batch)))

    def change_spef(self, path):
        self.calls.append(("spef", path))

    def result(self):
        at = np.zeros((4, 4), np.float32)
        at[0, 0] = np.nan
        return {"at": at, "slew": at + 1, "rat": at + 2, "slack": self.slack.copy()}


def make_timer():
    t = Timer.__new__(Timer)
    t._d = FakeDesign()
    t._pin = {n: i for i, n in enumerate(t._d.names)}
    t._net = {}
    t._gate_cell = {"u1": "NAND2_X1", "u2": "INV_X1", "u3": "DFF_X1"}
    t._pending, t._res, t._rc, t._pg, t._pg_fresh = [], None, None, None, False
    return t


def test_queue_applies_runs_of_resizes_and_spefs_in_order():
    t = make_timer()
    t.repower_gate("u1", "NAND2_X2").repower_gate("u2", "INV_X4")
    t.read_spef("c1.spef")
    t.repower_gate("u1", "NAND2_X4")
    t.read_spef("c2.spef").read_spef("c3.spef")
    assert t._d.calls == []  # queued until an update or a query
    t.report_at("b", MAX, RISE)
    assert t._d.calls == [("resize", [("u1", "NAND2_X2"), ("u2", "INV_X4")]),
                          ("spef", "c1.spef"), ("resize", [("u1", "NAND2_X4")]),
                          ("spef", "c2.spef"), ("spef", "c3.spef")]
    t.update_timing()  # nothing pending: no device work
    assert len(t._d.calls) == 5


def test_repower_gate_checks():
    t = make_timer()
    with pytest.raises(KeyError):
        t.repower_gate("nope", "INV_X2")
    with pytest.raises(ValueError):
        t.repower_gate("u2", "NAND2_X2")  # another function
    t.repower_gate("u2", "INV_X2")
    with pytest.raises(ValueError):
        t.repower_gate("u2", "DFF_X1")  # checked against the queued cell
    assert t._pending == [("resize", ("u2", "INV_X2"))]


def test_pin_queries_and_empty_values():
    t = make_timer()
    assert t.report_at("a", MIN, RISE) is None  # NaN: the reference's empty optional
    assert t.report_rat("a", MIN, RISE) is None  # rat blanked where at is empty
    assert t.report_slew("b", MAX, FALL) == 1.0
    assert t.report_slack("zz", MIN, RISE) is None  # unknown pin
    assert t.report_load("no-net", MAX, RISE) is None


def test_wns_tns_over_endpoints():
    t = make_timer()
    # corner c = split * 2 + transition; endpoints are pins 1 and 3
    assert t.report_wns(MIN, RISE) == -3.0
    assert t.report_wns(MAX, FALL) == -1.5  # pin 1 has no slack there
    assert t.report_wns() == -3.0
    assert t.report_wns(MAX) == -1.5  # min over MAX RISE (-1.0) and MAX FALL (-1.5)
    assert t.report_tns(MIN, FALL) == -0.25  # 0.5 is not negative
    assert t.report_tns(MIN) == np.float32(-5.0) + np.float32(-0.25)
    assert t.report_tns() == pytest.approx(-5.0 - 0.25 - 1.0 - 1.5)


def test_rc_slew_formula():
    t = make_timer()
    imp = np.full((2, 2), 7.0, np.float32)
    t.rc_node = lambda net, pin: {"impulse": imp}
    assert t.rc_slew("n", "p", MAX, RISE, 3.0) == pytest.approx(4.0)
    assert t.rc_slew("n", "p", MAX, RISE, -3.0) == pytest.approx(-4.0)
    t.rc_node = lambda net, pin: None
    assert t.rc_slew("n", "p", MAX, RISE, 3.0) is None
