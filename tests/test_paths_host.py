"""The path search (opentimer_b200.paths) on the reference Timer's own
values: the harness (oracle/_ref/ot_run_ref, CPU path) dumps its timing
graph with every arc's delays and the data-path sources, and its pins'
arrival/required times and slacks; fed those, PathGraph.report_timing must
return the paths Timer::report_timing returns -- the same slacks, the same
endpoints and the same (pin, transition, arrival) points, bit for bit,
paths of equal slack compared as sets."""
import os
import subprocess

import numpy as np
import pytest

from opentimer_b200 import designgen
from opentimer_b200.paths import PathGraph

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE_REF = os.path.join(ROOT, "oracle", "_ref", "ot_run_ref")


def parse(out, graph):
    pins, paths = {}, []
    with open(out) as f:
        for line in f:
            t = line.split()
            if t[0] == "P":
                pins[t[1]] = np.array([float(x) for x in t[2:]], np.float32).reshape(4, 4)
            elif t[0] == "T":
                paths.append({"slack": np.float32(t[2]), "el": int(t[3]), "points": []})
            elif t[0] == "Q":
                paths[int(t[1])]["points"].append((t[2], int(t[3]), np.float32(t[4])))
    names, arcs, delays, tests, src, po = {}, [], {}, [], [], []
    with open(graph) as f:
        for line in f:
            t = line.split()
            if t[0] == "p":
                names[int(t[1])] = t[2]
                if any(not np.isnan(float(x)) for x in t[12:16]):
                    po.append(int(t[1]))
            elif t[0] == "a":
                arcs.append((int(t[2]), int(t[3])))
            elif t[0] == "d":
                delays[int(t[1])] = [float(x) for x in t[2:10]]
            elif t[0] == "s":
                tests.append(int(t[1]))
            elif t[0] == "z":
                src.append(int(t[1]))
    return pins, paths, names, arcs, delays, tests, src, po


def run_ref(d, K, extra=()):
    out, graph = os.path.join(d, f"ref_paths{K}.txt"), os.path.join(d, f"graph{K}.txt")
    # a paths= argument in `extra` overrides this one (the harness keeps the last)
    p = subprocess.run([EXE_REF, d, "cpu", out, graph, f"paths={K}", *extra],
                       capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    return parse(out, graph)


def path_graph(pins, names, arcs, delays, tests, src, po):
    P = max(names) + 1
    nm = [names.get(i, f"?{i}") for i in range(P)]
    arc = np.array(arcs, np.int64).reshape(-1, 2)
    dl = np.array([delays[k] for k in range(len(arcs))], np.float32).reshape(-1, 2, 2, 2)
    source = np.zeros(P, bool)
    source[src] = True
    # endpoints: primary outputs and the tests' constrained pins
    ends = np.unique(np.array(po + [int(arc[a, 1]) for a in tests], np.int64))
    vals = np.full((P, 4, 4), np.nan, np.float32)
    for i, n in enumerate(nm):
        if n in pins:
            vals[i] = pins[n]
    g = PathGraph(nm, arc[:, 0], arc[:, 1], tests, source, ends)
    return g.values(dl, vals[:, 0], vals[:, 2], vals[:, 3])


def same_paths(ours, ref):
    assert len(ours) == len(ref)
    key = lambda pts: tuple((n, r, float(a)) for n, r, a in pts)  # noqa: E731
    got = sorted((float(p.slack), p.endpoint[1], key(p.points)) for p in ours)
    want = sorted((float(p["slack"]), p["el"], key(p["points"])) for p in ref)
    assert got == want


@pytest.fixture(scope="module")
def design(tmp_path_factory):
    if not os.path.exists(EXE_REF):
        pytest.skip("the reference Timer harness (oracle/_ref) is not built")
    d = str(tmp_path_factory.mktemp("paths"))
    keep = {}
    designgen.write_design(d, seed=77, gates=1200, keep=keep)
    return d, keep


@pytest.mark.parametrize("K", [1, 5, 60, 400])
def test_paths_equal_reference_on_its_values(design, K):
    d, _ = design
    pins, ref, *rest = run_ref(d, K)
    g = path_graph(pins, *rest)
    ours = g.report_timing(K)
    assert len(ref) > 0 and ours[0].points, "no path to compare"
    if K == 1:
        # the worst endpoint's path, reported with the endpoint's slack
        assert float(ours[0].slack) == float(ref[0]["slack"])
    same_paths(ours, ref)


@pytest.mark.parametrize("el,rf", [(1, None), (0, None), (None, 1), (1, 0)])
def test_split_and_transition_forms(design, el, rf):
    """report_timing(K, el), (K, rf) and (K, el, rf) against the
    reference's forms of the same name."""
    d, _ = design
    K = 8
    arg = f"paths={K},{-1 if el is None else el}" + ("" if rf is None else f",{rf}")
    pins, ref, *rest = run_ref(d, K, extra=(arg,))
    g = path_graph(pins, *rest)
    ours = g.report_timing(K, el, rf)
    assert len(ref) > 0
    same_paths(ours, ref)
    for p in ours:
        assert el is None or p.endpoint[1] == el
        assert rf is None or p.endpoint[2] == rf


def test_worst_endpoints_follow_slack_order(design):
    d, _ = design
    pins, _, *rest = run_ref(d, 1)
    g = path_graph(pins, *rest)
    e = g.worst_endpoints(40)
    s = [float(g.slack[p, 2 * el + rf]) for p, el, rf in e]
    assert s == sorted(s) and len(e) == 40
    # per split / transition the lists are restricted to that corner
    assert all(el == 1 for _, el, _ in g.worst_endpoints(10, el=1))
    assert all((el, rf) == (0, 1) for _, el, rf in g.worst_endpoints(10, el=0, rf=1))


def test_native_search_on_a_hand_built_graph():
    """0 (a primary input, a source) -> 1 -> 2 (an endpoint): a net arc
    (rise->rise 1, fall->fall 2) then a negative-unate cell arc (rise->fall
    3, fall->rise 4), late split only.  The worst late path ends at 2 rising:
    from 0 falling, 5 + 2 + 4 = 11 against a required time of 10."""
    import ctypes
    from opentimer_b200 import _lib
    nan = np.nan
    delay = np.full((2, 2, 2, 2), nan, np.float32)  # [arc][el][frf][trf]
    delay[0, 1, 0, 0], delay[0, 1, 1, 1] = 1.0, 2.0
    delay[1, 1, 0, 1], delay[1, 1, 1, 0] = 3.0, 4.0
    at = np.full((3, 4), nan, np.float32)
    at[0, 2:] = [4.0, 5.0]
    at[1, 2:] = [5.0, 7.0]
    at[2, 2:] = [11.0, 8.0]
    rat = np.full((3, 4), nan, np.float32)
    rat[2, 2:] = 10.0
    slack = np.full((3, 4), nan, np.float32)
    slack[2, 2:] = rat[2, 2:] - at[2, 2:]
    g = PathGraph(["i", "u:A", "u:ZN"], [0, 1], [1, 2], [], [True, False, False], [2])
    g.values(delay, at, rat, slack)
    (p,) = g.report_timing(1)
    assert p.slack == -1.0 and p.endpoint == ("u:ZN", 1, 0)
    assert [(q.pin, q.transition, float(q.at)) for q in p.points] == \
        [("i", 1, 5.0), ("u:A", 1, 7.0), ("u:ZN", 0, 11.0)]
    # K > 1: only the negative-slack path (the other ends at 8 <= 10)
    assert [x.slack for x in g.report_timing(5)] == [-1.0]
    assert g.report_timing(0) == [] and g.report_timing(3, el=0) == []
    # the C ABI: a result larger than max_points, then bad arguments
    L = _lib.lib()
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    cg = _lib.PathGraph(3, 2, 1, ptr(g._from32), ptr(g._to32), ptr(g._test8), ptr(g._src8),
                        ptr(g._ends32), ptr(g._delay8), ptr(g.at), ptr(g.rat), ptr(g.slack))
    n, need = ctypes.c_int32(), ctypes.c_int32()
    sl, ep, st = np.zeros(1, np.float32), np.zeros(3, np.int32), np.zeros(2, np.int32)
    pin, tr, pa = np.zeros(1, np.int32), np.zeros(1, np.int32), np.zeros(1, np.float32)
    code = L.otg_report_paths(ctypes.byref(cg), 1, -1, -1, ctypes.byref(n), ptr(sl), ptr(ep),
                              ptr(st), 1, ptr(pin), ptr(tr), ptr(pa), ctypes.byref(need))
    assert code == 8 and need.value == 3 and n.value == 1  # OTG_ERR_WORKSPACE
    assert L.otg_report_paths(ctypes.byref(cg), 1, 2, -1, ctypes.byref(n), ptr(sl), ptr(ep),
                              ptr(st), 1, ptr(pin), ptr(tr), ptr(pa), ctypes.byref(need)) == 1
    bad = np.array([0, 7], np.int32)  # an arc to a pin that does not exist
    cg.arc_to = ptr(bad)
    assert L.otg_report_paths(ctypes.byref(cg), 1, -1, -1, ctypes.byref(n), ptr(sl), ptr(ep),
                              ptr(st), 1, ptr(pin), ptr(tr), ptr(pa), ctypes.byref(need)) == 1
