"""Seeded generators of RC forests and pin DAGs for the CPU-side tests.

Forests follow the batched-Elmore workload: net sizes log-uniform, 70%
random recursive trees and 30% chains with side branches, edges shuffled
with random orientation and local ids assigned by first appearance while
scanning the edges (the id rule of OpenTimer's Net::_make_flat_rct,
ot/timer/net.cpp:392-410), R ~ U(0.1, 50), ground C ~ U(0.05, 5) plus a
per-corner pin cap on leaves so the four corners differ.
"""
import numpy as np

import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "oracle"))
from oracle import Forest  # noqa: E402


def net_sizes(rng, num_nets, lo=2, hi=4096):
    u = rng.random(num_nets)
    n = np.floor(np.exp(np.log(lo) + u * (np.log(hi + 1) - np.log(lo)))).astype(np.int64)
    return np.clip(n, lo, hi)


def make_tree(rng, n, kind):
    """Canonical parent array (node 0 = root)."""
    par = np.full(n, -1, np.int64)
    if n <= 1:
        return par
    if kind == "chain":
        s = max(1, (n * 4) // 5)
        par[1:s] = np.arange(0, s - 1)
        if n > s:
            par[s:] = rng.integers(0, s, n - s)
    elif kind == "star":
        par[1:] = 0
    elif kind == "path":
        par[1:] = np.arange(0, n - 1)
    else:  # random recursive tree
        par[1:] = (rng.random(n - 1) * np.arange(1, n)).astype(np.int64)
    return par


def forest(seed, sizes, kinds=None, chain_frac=0.3, pin_jitter=True):
    """Build a Forest from a list of node counts."""
    rng = np.random.default_rng(seed)
    sizes = [int(x) for x in sizes]
    N = len(sizes)
    V = int(sum(sizes))
    nodes_start = np.zeros(N + 1, np.int64)
    nodes_start[1:] = np.cumsum(sizes)
    edges = np.zeros((V - N, 2), np.int32)
    res = np.zeros(V - N, np.float32)
    cap = np.zeros((V, 4), np.float32)
    roots = np.zeros(N, np.int32)
    for i, n in enumerate(sizes):
        kind = kinds[i] if kinds is not None else ("chain" if rng.random() < chain_frac else "rrt")
        par = make_tree(rng, n, kind)
        b = int(nodes_start[i])
        eb = b - i
        m = n - 1
        if m > 0:
            ch = np.arange(1, n)
            pa = par[1:]
            perm = rng.permutation(m)
            ch, pa = ch[perm], pa[perm]
            flip = rng.random(m) < 0.5
            a = np.where(flip, ch, pa)
            c = np.where(flip, pa, ch)
            seq = np.stack([a, c], 1).reshape(-1)
            # first-appearance local ids over the edge scan
            _, first = np.unique(seq, return_index=True)
            order = np.argsort(first, kind="stable")
            uniq = np.unique(seq)[order]
            lid = np.empty(n, np.int64)
            lid[uniq] = np.arange(n)
            edges[eb:eb + m] = lid[seq].reshape(-1, 2)
            roots[i] = lid[0]
            res[eb:eb + m] = rng.uniform(0.1, 50.0, m).astype(np.float32)
            nchild = np.bincount(par[1:], minlength=n)
            leaf = (nchild == 0)
            leaf[0] = False
            leaf_l = np.zeros(n, bool)
            leaf_l[lid] = leaf
        else:
            roots[i] = 0
            leaf_l = np.zeros(n, bool)
        g = rng.uniform(0.05, 5.0, n).astype(np.float32)
        cap[b:b + n] = g[:, None]
        if pin_jitter:
            pins = rng.uniform(0.5, 2.0, (n, 4)).astype(np.float32)
            cap[b:b + n] += np.where(leaf_l[:, None], pins, 0.0).astype(np.float32)
    return Forest(nodes_start.astype(np.int32), edges, roots, res, cap)


def random_forest(seed, num_nets, lo=2, hi=4096):
    rng = np.random.default_rng(seed + 7777)
    return forest(seed, net_sizes(rng, num_nets, lo, hi))


def sinks_of(f):
    """Leaf (degree-1, non-root) nodes of each net, ascending local id."""
    starts = [0]
    nodes = []
    for i in range(f.num_nets):
        b, e = int(f.nodes_start[i]), int(f.nodes_start[i + 1])
        n = e - b
        eb = b - i
        deg = np.bincount(f.edges[eb:eb + n - 1].reshape(-1), minlength=n)
        lv = np.nonzero((deg == 1) & (np.arange(n) != f.roots[i]))[0]
        nodes.extend(lv.tolist())
        starts.append(len(nodes))
    return np.array(starts, np.int32), np.array(nodes, np.int32)


def pin_dag(seed, n_pins, n_edges, n_levels, hf_frac=0.0):
    """Random levelled pin DAG.  Returns (fanin_start, fanin, out_deg,
    frontier0) in the layout of Timer::_build_prop_tasks_cuda: fanin CSR
    over all pins, out_deg = fanout count, frontier0 = pins without fanout
    in index order."""
    rng = np.random.default_rng(seed)
    lvl = np.sort(rng.integers(0, n_levels, n_pins))
    lvl[:n_levels] = np.arange(n_levels)  # every level populated
    perm = rng.permutation(n_pins)
    level_of = np.empty(n_pins, np.int64)
    level_of[perm] = lvl
    by_level = [perm[lvl == k] for k in range(n_levels)]
    src, dst = [], []
    # one edge from level k-1 to each pin of level k guarantees the depth
    for k in range(1, n_levels):
        prev = by_level[k - 1]
        cur = by_level[k]
        src.append(prev[rng.integers(0, len(prev), len(cur))])
        dst.append(cur)
    extra = n_edges - sum(len(d) for d in dst)
    if extra > 0:
        a = rng.integers(0, n_pins, extra * 2)
        b = rng.integers(0, n_pins, extra * 2)
        ok = level_of[a] < level_of[b]
        a, b = a[ok][:extra], b[ok][:extra]
        src.append(a)
        dst.append(b)
    src = np.concatenate(src) if src else np.zeros(0, np.int64)
    dst = np.concatenate(dst) if dst else np.zeros(0, np.int64)
    # dedupe (u,v)
    key = np.unique(src * n_pins + dst)
    src, dst = key // n_pins, key % n_pins
    order = np.lexsort((src, dst))
    src, dst = src[order], dst[order]
    fanin_start = np.zeros(n_pins + 1, np.int64)
    np.add.at(fanin_start, dst + 1, 1)
    fanin_start = np.cumsum(fanin_start)
    fanin = src
    out_deg = np.bincount(src, minlength=n_pins)
    frontier0 = np.nonzero(out_deg == 0)[0]
    return (fanin_start.astype(np.int32), fanin.astype(np.int32), out_deg.astype(np.int32),
            frontier0.astype(np.int32))
