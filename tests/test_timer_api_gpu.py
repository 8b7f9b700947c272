"""The Timer-style host layer (opentimer_b200.timer.Timer) against the
reference Timer (oracle/_ref/ot_run_ref, its CPU path) on the same design,
after the first full update, after a batch of repower_gate calls, and
after a change SPEF followed by a resize batch, and report_timing (the K
worst paths) against the reference's, before and after a resize batch:

* report_at / report_slew / report_rat / report_slack of every pin within
  the pin tolerance of tests/helpers.pin_err;
* report_wns and report_tns of every corner: WNS within the tolerance of
  the worst endpoint, TNS within the sum of the endpoints' tolerances (the
  two sum the same terms in different orders);
* report_load of every net and rc_node values of the pins' RC nodes within
  the RC tolerance (1e-5 relative, floor 1e-6 x the net's max |value|).
"""
import os
import subprocess

import numpy as np
import pytest

from helpers import pin_err, read_ref_pins
from opentimer_b200 import designgen

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE_REF = os.path.join(ROOT, "oracle", "_ref", "ot_run_ref")


def read_ref(path):
    N, L, R = {}, {}, {}
    with open(path) as f:
        for line in f:
            t = line.split()
            if t[0] == "N":
                N[(int(t[1]), int(t[2]))] = (float(t[3]), float(t[4]))
            elif t[0] == "L":
                L[t[1]] = np.array([float(x) for x in t[2:]])
            elif t[0] == "R":
                R[(t[1], t[2])] = np.array([float(x) for x in t[3:]]).reshape(4, 4)
    return read_ref_pins(path), N, L, R


def check_against(t, ref):
    from opentimer_b200.timer import MAX, MIN
    pins, N, L, R = ref
    ours = {}
    for name in pins:
        v = np.full((4, 4), np.nan)
        for c, (el, rf) in enumerate([(0, 0), (0, 1), (1, 0), (1, 1)]):
            for q, f in enumerate((t.report_at, t.report_slew, t.report_rat, t.report_slack)):
                x = f(name, el, rf)
                v[q, c] = np.nan if x is None else x
        ours[name] = v
    assert pin_err(ours, pins) <= 1.0
    # endpoints: the facade's set, tolerances from the reference's pins
    d = t._d
    for (el, rf), (wns, tns) in N.items():
        c = el * 2 + rf
        tol = []
        for i in d.endpoints:
            r = pins[d.names[i]]
            if not np.isnan(r[3][c]):
                tol.append(1e-5 * max(abs(r[3][c]), abs(np.nan_to_num(r[0][c]))) + 1e-5)
        assert abs(t.report_wns(el, rf) - wns) <= max(tol), (el, rf)
        assert abs(t.report_tns(el, rf) - tns) <= sum(tol), (el, rf)
    assert t.report_wns() == min(t.report_wns(a, b) for a in (MIN, MAX) for b in (0, 1))
    # net loads and RC nodes
    loads = 0
    for net, l in L.items():
        if t.report_load(net, 0, 0) is None:  # a net without parasitics (no RC tree here)
            continue
        got = np.array([t.report_load(net, el, rf) for el in (0, 1) for rf in (0, 1)])
        assert np.all(np.abs(got - l) <= 1e-5 * np.abs(l) + 1e-6 * np.abs(l).max()), net
        loads += 1
    assert loads > 0.9 * len(L)
    nets = {}
    for (net, node), v in R.items():
        nets.setdefault(net, []).append((node, v))
    checked = 0
    for net, rows in nets.items():
        mx = np.abs(np.stack([v for _, v in rows])).max(axis=0)
        for node, v in rows:
            got = t.rc_node(net, node)
            if got is None:  # an internal node: the facade answers by pin name
                continue
            g = np.stack([got[k].reshape(4) for k in ("load", "delay", "ldelay", "impulse")])
            assert np.all(np.abs(g - v) <= 1e-5 * np.abs(v) + 1e-6 * mx), (net, node)
            if checked % 97 == 0:  # RctNode::slew from the node's impulse
                for si in (-40.0, 25.0):
                    want = np.copysign(np.sqrt(np.float32(si * si + v[3][3])), si)
                    assert abs(t.rc_slew(net, node, 1, 1, si) - want) <= 1e-5 * abs(want) + 1e-4
            checked += 1
    assert checked > 1000


@pytest.fixture(scope="module")
def design(tmp_path_factory, cuda):
    if not os.path.exists(EXE_REF):
        pytest.skip("the reference Timer harness (oracle/_ref) is not built")
    d = str(tmp_path_factory.mktemp("timer_api"))
    keep = {}
    designgen.write_design(d, seed=2041, gates=1500, keep=keep)
    return d, keep


def test_reports_match_the_reference(design):
    from opentimer_b200.sizing import resize_trace, write_ops
    from opentimer_b200.timer import Timer
    d, keep = design
    steps = resize_trace(keep, seed=11, steps=1, per_step=40)
    out0 = os.path.join(d, "ref0.txt")
    p = subprocess.run([EXE_REF, d, "cpu", out0], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    ops = os.path.join(d, "ops.txt")
    write_ops(ops, steps)
    out1 = os.path.join(d, "ref1.txt")
    p = subprocess.run([EXE_REF, d, "cpu", out1, f"repower={ops}"], capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    t = Timer(d, keep)
    check_against(t, read_ref(out0))
    for gate, cell in steps[0]:
        t.repower_gate(gate, cell)
    check_against(t, read_ref(out1))  # the queries apply the queued resizes first
    with pytest.raises(ValueError):
        t.repower_gate(steps[0][0][0], "DFF_X1")


def test_change_spef_then_resizes(design):
    """read_spef of a change SPEF (5% of the nets get new trees), then a
    resize batch on the new layout: every report against the reference
    Timer after the same two updates."""
    from opentimer_b200.sizing import resize_trace, write_ops
    from opentimer_b200.timer import Timer
    d, keep = design
    change = os.path.join(d, "change.spef")
    changed = designgen.change_spef(keep, change, frac=0.05, seed=5)
    steps = resize_trace(keep, seed=12, steps=1, per_step=40)
    ops = os.path.join(d, "ops_after_change.txt")
    write_ops(ops, steps)
    out1 = os.path.join(d, "ref_change.txt")
    p = subprocess.run([EXE_REF, d, "cpu", out1, f"change={change}"], capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    out2 = os.path.join(d, "ref_change_repower.txt")
    p = subprocess.run([EXE_REF, d, "cpu", out2, f"change={change}", f"repower={ops}"],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    t = Timer(d, keep)
    before = {n: t.report_load(n, 1, 0) for n in changed}
    t.read_spef(change)
    check_against(t, read_ref(out1))
    after = {n: t.report_load(n, 1, 0) for n in changed}
    assert sum(before[n] != after[n] for n in changed) > 0.9 * len(changed)
    for gate, cell in steps[0]:
        t.repower_gate(gate, cell)
    check_against(t, read_ref(out2))


def read_ref_paths(path):
    paths = []
    with open(path) as f:
        for line in f:
            t = line.split()
            if t[0] == "T":
                paths.append({"slack": float(t[2]), "el": int(t[3]), "points": []})
            elif t[0] == "Q":
                paths[int(t[1])]["points"].append((t[2], int(t[3]), float(t[4])))
    return paths


def check_paths(ours, ref, tol=1e-3):
    """Same count; slacks pairwise within tol (ps) in ascending order; where
    a path's slack is more than 2 tol from its neighbours' the path itself
    (pins, transitions) is the reference's and its arrivals within tol."""
    assert len(ours) == len(ref) and len(ref) > 0
    s_ours = [p.slack for p in ours]
    s_ref = [p["slack"] for p in ref]
    assert s_ours == sorted(s_ours)
    assert np.all(np.abs(np.array(s_ours) - np.array(s_ref)) <= tol), (s_ours[:5], s_ref[:5])
    checked = 0
    for i, r in enumerate(ref):
        near = [abs(r["slack"] - ref[j]["slack"]) for j in (i - 1, i + 1) if 0 <= j < len(ref)]
        if near and min(near) <= 2 * tol:
            continue
        o = ours[i]
        assert [(p.pin, p.transition) for p in o.points] == [(n, t) for n, t, _ in r["points"]]
        assert np.all(np.abs(np.array([p.at for p in o.points]) -
                             np.array([a for _, _, a in r["points"]])) <= tol)
        assert o.endpoint[1] == r["el"] and o.endpoint[0] == r["points"][-1][0]
        checked += 1
    return checked


def test_report_timing_matches_the_reference(design):
    """report_timing(K) against Timer::report_timing(K) on the same design,
    after the first update and after a resize batch."""
    from opentimer_b200.sizing import resize_trace, write_ops
    from opentimer_b200.timer import Timer
    d, keep = design
    steps = resize_trace(keep, seed=13, steps=1, per_step=40)
    ops = os.path.join(d, "ops_paths.txt")
    write_ops(ops, steps)
    t = Timer(d, keep)
    for tag, extra in (("0", []), ("1", [f"repower={ops}"])):
        if tag == "1":
            for gate, cell in steps[0]:
                t.repower_gate(gate, cell)
        for K in (1, 40):
            out = os.path.join(d, f"ref_paths_{tag}_{K}.txt")
            p = subprocess.run([EXE_REF, d, "cpu", out, *extra, f"paths={K}"],
                               capture_output=True, text=True, timeout=600)
            assert p.returncode == 0, p.stderr[-2000:]
            ref = read_ref_paths(out)
            ours = t.report_timing(K)
            n = check_paths(ours, ref)
            assert n >= (1 if K == 1 else 10), (tag, K, n)
            if K == 1:
                assert len(ours[0].points) > 10
