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
