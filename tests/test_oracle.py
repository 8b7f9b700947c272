"""The CPU oracle is pinned against the reference: the committed fixtures
(made by the reference's own Rct::update_rc_timing / SPEF parser, see
tests/golden/make_golden.py) and, where the reference tree was compiled
here, oracle/_ref/libotref.so directly."""
import os

import numpy as np
import pytest

import oracle as O
import rcgen
from helpers import levels_as_sets

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_fixture(name):
    d = np.load(os.path.join(GOLD, name))
    f = O.Forest(d["nodes_start"], d["edges"], d["roots"], d["res"], d["cap"])
    return f, d


@pytest.mark.parametrize("name", ["rc_cpu_small.npz", "rc_cpu_c17.npz", "rc_cpu_s27.npz"])
def test_cpu_restatement_bitexact_vs_reference_fixture(name):
    f, d = load_fixture(name)
    st, outs = O.elmore_cpu_f32(f)
    assert st == 0
    for q, got in zip(["load", "delay", "ldelay", "impulse"], outs):
        assert np.array_equal(got.view(np.int32), d[q].view(np.int32)), q


@pytest.mark.skipif(not O.ref_available(), reason="reference harness not built")
def test_cpu_restatement_bitexact_vs_reference_live():
    f = rcgen.random_forest(3, 150, 2, 700)
    st, outs = O.elmore_cpu_f32(f)
    st2, ref = O.ref_rct_update(f, 2)
    assert st == 0 and st2 == 0
    for got, r in zip(outs, ref):
        assert np.array_equal(got.view(np.int32), r.view(np.int32))


def test_f64_close_to_f32_reference():
    f, d = load_fixture("rc_cpu_small.npz")
    st, outs = O.elmore_f64(f)
    assert st == 0
    for q, x in zip(["load", "delay", "ldelay"], outs):
        r = d[q].astype(np.float64)
        assert np.max(np.abs(x - r) / np.maximum(np.abs(x), 1e-30)) < 1e-4


def _bfs_slots_by_definition(f):
    """(distance asc, local id desc) by brute force per net."""
    out = np.zeros(f.total_nodes, np.int32)
    for i in range(f.num_nets):
        b, e = int(f.nodes_start[i]), int(f.nodes_start[i + 1])
        n = e - b
        adj = [[] for _ in range(n)]
        for s, t in f.edges[b - i:e - i - 1]:
            adj[s].append(t)
            adj[t].append(s)
        dist = [-1] * n
        dist[f.roots[i]] = 0
        q = [int(f.roots[i])]
        for v in q:
            for w in adj[v]:
                if dist[w] < 0:
                    dist[w] = dist[v] + 1
                    q.append(w)
        order = sorted(range(n), key=lambda v: (dist[v], -v))
        for k, v in enumerate(order):
            out[b + v] = k
    return out


def test_bfs_tie_rule():
    f = rcgen.forest(5, [1, 2, 5, 17, 40, 90], ["rrt", "rrt", "star", "rrt", "chain", "rrt"])
    st, e, n2b, pid, depth = O.bfs(f)
    assert st == 0
    assert np.array_equal(n2b, _bfs_slots_by_definition(f))
    # pid: parent of slot i is i - pid[i]; parents precede children
    for i in range(f.num_nets):
        b, en = int(f.nodes_start[i]), int(f.nodes_start[i + 1])
        assert pid[b] == 0
        assert np.all(pid[b + 1:en] >= 1)
        assert n2b[b + f.roots[i]] == 0
    # edges are directed parent -> child: depth(child) = depth(parent)+1
    eb = np.repeat(f.nodes_start[:-1], np.diff(f.nodes_start) - 1)
    assert np.all(depth[eb + e[:, 1]] == depth[eb + e[:, 0]] + 1)


def test_bfs_rejects_non_tree():
    f = rcgen.forest(1, [6], ["path"])
    f.edges[2] = f.edges[0]  # duplicate edge -> a node becomes unreachable
    st, *_ = O.bfs(f)
    assert st == 4


def test_levelize_oracle_definition():
    fs, fi, od, f0 = rcgen.pin_dag(2, 500, 1200, 12)
    order, ends, level = O.levelize(len(od), fs, fi, od, f0)
    n = len(od)
    # level(v) = 1 + max level over fanouts, 0 without fanout
    fanout = [[] for _ in range(n)]
    for v in range(n):
        for u in fi[fs[v]:fs[v + 1]]:
            fanout[u].append(v)
    memo = {}

    def lv(v):
        if v not in memo:
            memo[v] = 0 if not fanout[v] else 1 + max(lv(w) for w in fanout[v])
        return memo[v]
    import sys
    sys.setrecursionlimit(10000)
    assert all(level[v] == lv(v) for v in range(n))
    assert len(ends) == max(level) + 2
    sets = levels_as_sets(order, ends)
    for k, s in enumerate(sets):
        assert all(level[v] == k for v in s)
    # levels after the seed are emitted in ascending pin order
    for k in range(1, len(ends) - 1):
        seg = order[ends[k]:ends[k + 1]]
        assert np.all(np.diff(seg) > 0)


def test_host_generator_matches_product_generator():
    """The reference arm of bench.py builds its inputs with the oracle's host
    generator (so the product library is not loaded there); it must give
    the very nets the product library's generator gives, including a slice
    that starts in the middle of the workload."""
    import opentimer_b200 as otg
    ns = otg.workloads.net_sizes(77, 400, 2, 600)
    g = otg.synth_forest_host(77, ns)
    f, slew, cnt = O.synth_forest(77, ns, threads=3)
    assert np.array_equal(f.edges, g["edges"])
    assert np.array_equal(f.roots, g["roots"])
    assert np.array_equal(f.res.view(np.int32), g["res"].view(np.int32))
    assert np.array_equal(f.cap.view(np.int32), g["cap"].view(np.int32))
    assert np.array_equal(slew.view(np.int32), g["driver_slew"].view(np.int32))
    assert np.array_equal(cnt, g["sink_count"])
    # nets 150..299 as a slice of their own
    k0, k1 = 150, 300
    fs, slew_s, cnt_s = O.synth_forest(77, ns[k0:k1 + 1], first_net=k0, threads=2)
    v0, v1 = int(ns[k0]), int(ns[k1])
    assert np.array_equal(fs.edges, g["edges"][v0 - k0:v1 - k1])
    assert np.array_equal(fs.roots, g["roots"][k0:k1])
    assert np.array_equal(fs.cap.view(np.int32), g["cap"][v0:v1].view(np.int32))
    assert np.array_equal(slew_s.view(np.int32), g["driver_slew"][k0:k1].view(np.int32))
