"""Path reports over a propagated timing graph: the K worst data paths, as
Timer::report_timing gives them (ot/timer/path.cpp:365-420).

The graph's values come from the device -- arrival and required times and
slacks of every pin, and the delay of every arc at every (split, from
transition, to transition) that the propagation computed
(otg_prop_arc_delays) -- and the search runs on the host, as the
reference's does on its CPU, in native code (otg_report_paths,
opentimer_b200/csrc/otg_paths.cpp, which states the algorithm: the worst
endpoints, a suffix tree per endpoint down to the data-path sources, and
for K > 1 the prefix-tree search over deviations from it, in float32 in
the reference's order of operations).  Paths with equal slack may come out
in another order than the reference's, whose endpoint and source orders
follow hash maps.
"""
import ctypes
from typing import NamedTuple

import numpy as np


class Point(NamedTuple):
    pin: str
    transition: int
    at: float


class Path(NamedTuple):
    slack: float
    endpoint: tuple  # (pin name, split, transition)
    points: list


class PathGraph:
    """The static part of a timing graph for path queries: pin names, arcs,
    data-path sources and endpoints.  `values(...)` attaches one update's
    results; report_timing then answers from them."""

    def __init__(self, names, arc_from, arc_to, test_arcs, source, endpoints):
        self.names = list(names)
        self.arc_from = np.ascontiguousarray(arc_from, np.int32)
        self.arc_to = np.ascontiguousarray(arc_to, np.int32)
        self._test8 = np.zeros(len(self.arc_from), np.uint8)  # constraint arcs: no delay
        self._test8[np.asarray(test_arcs, np.int64)] = 1
        self.source = np.ascontiguousarray(source, bool)
        self._src8 = self.source.astype(np.uint8)
        self.endpoints = np.ascontiguousarray(endpoints, np.int32)
        self._from32, self._to32, self._ends32 = self.arc_from, self.arc_to, self.endpoints
        self.delay = self.at = self.rat = self.slack = None

    def values(self, delay, at, rat, slack):
        """delay [A][2][2][2] (split, from, to transition), at / rat / slack
        [P][4] (corner = split * 2 + transition), NaN for empty values."""
        self.delay = np.ascontiguousarray(delay, np.float32).reshape(-1, 2, 2, 2)
        self._delay8 = self.delay.reshape(-1, 8)
        self.at = np.ascontiguousarray(at, np.float32)
        self.rat = np.ascontiguousarray(rat, np.float32)
        self.slack = np.ascontiguousarray(slack, np.float32)
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

    # --------------------------------------------------------------- report
    def report_timing(self, K, el=None, rf=None):
        """The K worst paths (Timer::report_timing(K[, el][, rf])), by
        ascending slack: Path(slack, endpoint (pin name, split, tran),
        points [Point(pin name, tran, arrival)])."""
        from ._lib import PathGraph as CGraph
        from ._lib import check, lib
        K = int(K)
        if K <= 0:
            return []
        P, A = len(self.names), len(self.arc_from)
        ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p) if a.size else None  # noqa: E731
        cg = CGraph(P, A, len(self._ends32), ptr(self._from32), ptr(self._to32),
                    ptr(self._test8), ptr(self._src8), ptr(self._ends32), ptr(self._delay8),
                    ptr(self.at), ptr(self.rat), ptr(self.slack))
        n = ctypes.c_int32(0)
        need = ctypes.c_int32(0)
        slack = np.zeros(K, np.float32)
        ept = np.zeros((K, 3), np.int32)
        start = np.zeros(K + 1, np.int32)
        cap = 256 * K
        while True:
            pin, tr, at = (np.zeros(cap, np.int32), np.zeros(cap, np.int32),
                           np.zeros(cap, np.float32))
            code = lib().otg_report_paths(
                ctypes.byref(cg), K, -1 if el is None else int(el), -1 if rf is None else int(rf),
                ctypes.byref(n), ptr(slack), ptr(ept), ptr(start), cap, ptr(pin), ptr(tr),
                ptr(at), ctypes.byref(need))
            if code == 8 and need.value > cap:  # OTG_ERR_WORKSPACE: room for every point
                cap = need.value
                continue
            check("otg_report_paths", code)
            break
        out = []
        for i in range(n.value):
            a, b = int(start[i]), int(start[i + 1])
            pts = [Point(self.names[int(pin[q])], int(tr[q]), at[q]) for q in range(a, b)]
            out.append(Path(float(slack[i]), (self.names[int(ept[i, 0])], int(ept[i, 1]),
                                              int(ept[i, 2])), pts))
        return out
