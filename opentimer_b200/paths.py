"""Path reports over a propagated timing graph: the K worst data paths, as
Timer::report_timing gives them (ot/timer/path.cpp:365-420).

The graph's values come from the device -- arrival and required times and
slacks of every pin, and the delay of every arc at every (split, from
transition, to transition) that the propagation computed
(otg_prop_arc_delays) -- and the search runs on the host, as the
reference's does on its CPU.  Nodes are (pin, transition), encoded
2 * pin + transition.

* Endpoints (Timer::_worst_endpoints, ot/timer/endpoint.cpp:33-127): per
  (split, transition) the primary outputs and the timing tests' constrained
  pins whose slack is defined, sorted by slack; K of them by repeatedly
  taking the smallest head of those lists, ties to the first list in the
  order (MIN, RISE), (MIN, FALL), (MAX, RISE), (MAX, FALL).
* Suffix tree of an endpoint T at split el (Timer::_sfxt_cache, _spdp,
  _topologize, ot/timer/sfxt.cpp:52-246): the nodes of T's fanin cone in
  topological order (a depth-first post-order from T that stops at the
  data-path sources: pins without fanin, clock pins of cells, primary
  inputs), dist(T) = +rat (late) or -rat (early), and dist(u) = the
  smallest dist(v) + w over arcs u -> v, w = -delay (late) or +delay
  (early), keeping the first minimum (a strict comparison) and its arc; a
  super source S takes dist(S) = min over sources s of dist(s) + (-at(s)
  late, +at(s) early).  dist(S) is the slack of the worst path.
* K = 1 (Timer::_report_timing): the worst endpoint's suffix tree path,
  reported with the endpoint's slack.
* K > 1 (Timer::_spur, _pfxt_cache, ot/timer/pfxt.cpp:67-149): per
  endpoint, deviations from the suffix tree are ranked in a min-heap of
  prefix-tree nodes (slack, from, to, arc, parent): first the sources,
  then, for each popped path, every arc that leaves it into the cone other
  than the tree's own, at slack dist(v) + w - dist(u) + the path's slack;
  only negative slacks enter.  The K smallest over all endpoints are kept
  and returned by ascending slack.
* A path's points are (pin, transition, arrival): the source's arrival
  time, then the previous point's plus each arc's delay
  (Timer::_recover_datapath, path.cpp:460-537).

The arithmetic is float32, as the reference's.  Paths with equal slack
may come out in another order than the reference's, whose endpoint and
source orders follow hash maps.
"""
import heapq
from typing import NamedTuple

import numpy as np

F32 = np.float32
SUPER = -1  # the super source's node id


class Point(NamedTuple):
    pin: str
    transition: int
    at: float


class Path(NamedTuple):
    slack: float
    endpoint: tuple  # (pin name, split, transition)
    points: list


class _Sfxt:
    __slots__ = ("el", "t", "dist", "tree", "link", "srcs")

    def __init__(self, el, t):
        self.el, self.t = el, t
        self.dist, self.tree, self.link = {}, {}, {}
        self.srcs = []  # (source node, offset)

    def relax(self, u, v, link, d):
        cur = self.dist.get(u)
        if cur is None or d < cur:
            self.dist[u] = d
            self.tree[u] = v
            self.link[u] = link


class _Node:
    __slots__ = ("slack", "frm", "to", "arc", "parent")

    def __init__(self, slack, frm, to, arc, parent):
        self.slack, self.frm, self.to, self.arc, self.parent = slack, frm, to, arc, parent


class PathGraph:
    """The static part of a timing graph for path queries: pin names, arcs,
    data-path sources and endpoints.  `values(...)` attaches one update's
    results; report_timing then answers from them."""

    def __init__(self, names, arc_from, arc_to, test_arcs, source, endpoints):
        self.names = list(names)
        P = len(self.names)
        self.arc_from = np.asarray(arc_from, np.int64)
        self.arc_to = np.asarray(arc_to, np.int64)
        test = np.zeros(len(self.arc_from), bool)
        test[np.asarray(test_arcs, np.int64)] = True
        # fanin / fanout arcs per pin in arc order; constraint arcs carry no
        # delay and are left out
        self.fanin = [[] for _ in range(P)]
        self.fanout = [[] for _ in range(P)]
        for a in np.nonzero(~test)[0].tolist():
            self.fanin[int(self.arc_to[a])].append(a)
            self.fanout[int(self.arc_from[a])].append(a)
        self.source = np.asarray(source, bool)
        self.endpoints = np.asarray(endpoints, np.int64)
        self.delay = self.at = self.rat = self.slack = None

    def values(self, delay, at, rat, slack):
        """delay [A][2][2][2] (split, from, to transition), at / rat / slack
        [P][4] (corner = split * 2 + transition), NaN for empty values."""
        self.delay = np.asarray(delay, np.float32)
        self.at = np.asarray(at, np.float32)
        self.rat = np.asarray(rat, np.float32)
        self.slack = np.asarray(slack, np.float32)
        return self

    # ------------------------------------------------------------ endpoints
    def worst_endpoints(self, K, el=None, rf=None):
        lists = {}
        for e in (0, 1):
            for r in (0, 1):
                if el not in (None, e) or rf not in (None, r):
                    continue
                s = self.slack[self.endpoints, 2 * e + r]
                ok = ~np.isnan(s)
                pins, ss = self.endpoints[ok], s[ok]
                o = np.argsort(ss, kind="stable")
                lists[(e, r)] = [(ss[i], int(pins[i])) for i in o.tolist()]
        head = {k: 0 for k in lists}
        out = []
        for _ in range(K):
            best = None
            for k in sorted(lists):
                i = head[k]
                if i < len(lists[k]) and (best is None or
                                          lists[k][i][0] < lists[best][head[best]][0]):
                    best = k
            if best is None:
                break
            out.append((lists[best][head[best]][1], best[0], best[1]))
            head[best] += 1
        return out

    # ---------------------------------------------------------- suffix tree
    def _fanin_nodes(self, v, el):
        pin, vrf = v >> 1, v & 1
        out = []
        if self.source[pin]:
            return out
        for a in self.fanin[pin]:
            for urf in (0, 1):
                if not np.isnan(self.delay[a, el, urf, vrf]):
                    out.append(2 * int(self.arc_from[a]) + urf)
        return out

    def sfxt(self, T, el, rf):
        t = 2 * T + rf
        # the cone's depth-first post-order (Timer::_topologize)
        seen = {t}
        post = []
        stack = [(t, iter(self._fanin_nodes(t, el)))]
        while stack:
            v, it = stack[-1]
            for u in it:
                if u not in seen:
                    seen.add(u)
                    stack.append((u, iter(self._fanin_nodes(u, el))))
                    break
            else:
                stack.pop()
                post.append(v)
        sf = _Sfxt(el, t)
        rat = self.rat[T, 2 * el + rf]
        sf.dist[t] = -rat if el == 0 else rat
        for v in reversed(post):
            pin, vrf = v >> 1, v & 1
            if self.source[pin]:
                off = self.at[pin, 2 * el + vrf]
                sf.srcs.append((v, None if np.isnan(off) else (off if el == 0 else -off)))
                continue
            dv = sf.dist[v]
            for a in self.fanin[pin]:
                for urf in (0, 1):
                    d = self.delay[a, el, urf, vrf]
                    if np.isnan(d):
                        continue
                    u = 2 * int(self.arc_from[a]) + urf
                    sf.relax(u, v, (a, urf, vrf), F32(dv + (d if el == 0 else -d)))
        for s, off in sf.srcs:
            if off is not None:
                sf.relax(SUPER, s, None, F32(sf.dist[s] + off))
        return sf

    def _recover(self, sf, u, v, pts):
        """Follows the suffix tree from u to v, appending the points."""
        while u != v:
            a, frf, trf = sf.link[u]
            u = sf.tree[u]
            pts.append(Point(self.names[u >> 1], u & 1,
                             F32(pts[-1].at + self.delay[a, sf.el, frf, trf])))

    def _source_point(self, sf, s):
        return Point(self.names[s >> 1], s & 1, self.at[s >> 1, 2 * sf.el + (s & 1)])

    def _recover_node(self, sf, node, v, pts):
        """The path of prefix-tree node `node` up to v: its ancestors'
        segments from the source on, each up to where the next deviates
        (iterative: a chain of deviations can be K long)."""
        chain = []
        while node is not None:
            chain.append(node)
            node = node.parent
        for k in range(len(chain) - 1, -1, -1):
            nd = chain[k]
            end = chain[k - 1].frm if k > 0 else v
            u = nd.to
            if nd.frm == SUPER:
                pts.append(self._source_point(sf, u))
            else:
                d = self.delay[nd.arc, sf.el, pts[-1].transition, u & 1]
                pts.append(Point(self.names[u >> 1], u & 1, F32(pts[-1].at + d)))
            self._recover(sf, u, end, pts)

    def _spur(self, sf, pf, pfx, seq):
        u = pfx.to
        el = sf.el
        while u != sf.t:
            pin, urf = u >> 1, u & 1
            du = sf.dist[u]
            for a in self.fanout[pin]:
                for vrf in (0, 1):
                    d = self.delay[a, el, urf, vrf]
                    if np.isnan(d):
                        continue
                    v = 2 * int(self.arc_to[a]) + vrf
                    dv = sf.dist.get(v)
                    if dv is None or (a, urf, vrf) == sf.link[u]:
                        continue
                    w = d if el == 0 else -d
                    s = F32(F32(F32(dv + w) - du) + pfx.slack)
                    if s < 0.0:
                        heapq.heappush(pf, (s, next(seq), _Node(s, u, v, a, pfx)))
            u = sf.tree[u]

    # --------------------------------------------------------------- report
    def report_timing(self, K, el=None, rf=None):
        """The K worst paths (Timer::report_timing(K[, el][, rf]))."""
        epts = self.worst_endpoints(K, el, rf)
        if K == 0 or not epts:
            return []
        if K == 1:
            T, e, r = epts[0]
            sf = self.sfxt(T, e, r)
            pts = []
            if SUPER in sf.tree:
                pts.append(self._source_point(sf, sf.tree[SUPER]))
                self._recover(sf, sf.tree[SUPER], sf.t, pts)
            return [Path(float(self.slack[T, 2 * e + r]), (self.names[T], e, r), pts)]
        seq = iter(range(1 << 62))
        heap = []  # the K best paths so far, a max-heap by slack
        for T, e, r in epts:
            sf = self.sfxt(T, e, r)
            pf = []
            for s, off in sf.srcs:
                if off is None:
                    continue
                sl = F32(sf.dist[s] + off)
                if sl < 0.0:
                    heapq.heappush(pf, (sl, next(seq), _Node(sl, SUPER, s, None, None)))
            for _ in range(K):
                if not pf:
                    break
                node = heapq.heappop(pf)[2]
                if len(heap) >= K and -heap[0][0] <= node.slack:
                    break
                pts = []
                self._recover_node(sf, node, sf.t, pts)
                heapq.heappush(heap, (-float(node.slack), next(seq),
                                      Path(float(node.slack), (self.names[T], e, r), pts)))
                if len(heap) > K:
                    heapq.heappop(heap)
                self._spur(sf, pf, node, seq)
        return [p for _, _, p in sorted(heap, key=lambda x: (-x[0], x[1]))]
