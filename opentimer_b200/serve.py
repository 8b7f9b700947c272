"""Device-resident designs and incremental re-timing (otg_server_* in
include/otg.h).

A design is an RC forest with sinks (one net per driver pin).  The server
keeps it on the device, times it once in full, then applies requests:
each request is a set of node-capacitance updates (a resized sink gate
changes its pin cap) and driver-slew updates (a resized driver).  Only the
nets a request touches are re-timed -- the device-side counterpart of the
dirty-net skip in Net::_update_rc_timing (ot/timer/net.cpp:536-540).

    srv = TimingServer(budget_bytes=8 << 30)
    d, nbytes = srv.add_design(synth_design(7, nodes_start))
    t = srv.submit(d, cap=(nets, nodes, vals), slew=(nets2, vals2))
    r = srv.wait(t)          # worst sink slew / delay of the dirty nets
    out = srv.read(d)        # full per-node state, BFS order

submit/wait batch requests of different designs into shared launches
(CUDA graphs, continuous batching); update_sync is the same request applied
and timed alone (one set of launches and a synchronization each).
"""
import ctypes

import numpy as np

from ._lib import STATUS, OtgError, RcForest, RcResult, check, lib

NC = 4


def synth_design(seed, nodes_start):
    """Seeded synthetic design on the host: the RC forest of
    otg_synth_rc_forest_host plus its sinks (degree-1 nodes other than the
    root, ascending local id).  Returns a dict of numpy arrays."""
    from . import synth_forest_host
    f = synth_forest_host(seed, nodes_start)
    ns = f["nodes_start"].astype(np.int64)
    N = len(ns) - 1
    V = int(ns[-1])
    net_of_edge = np.repeat(np.arange(N), np.diff(ns) - 1)
    base = ns[:-1][net_of_edge]
    deg = np.bincount((f["edges"] + base[:, None]).reshape(-1), minlength=V)
    is_root = np.zeros(V, bool)
    is_root[ns[:-1] + f["roots"]] = True
    leaf = (deg == 1) & ~is_root
    net_of_node = np.repeat(np.arange(N), np.diff(ns))
    sinks_start = np.zeros(N + 1, np.int32)
    sinks_start[1:] = np.cumsum(np.bincount(net_of_node[leaf], minlength=N))
    sink_nodes = (np.nonzero(leaf)[0] - ns[net_of_node[leaf]]).astype(np.int32)
    f["sinks_start"] = sinks_start
    f["sink_nodes"] = sink_nodes
    return f


def _forest(d):
    a = {k: np.ascontiguousarray(v) for k, v in d.items()}
    f = RcForest(len(a["roots"]), int(a["nodes_start"][-1]), a["nodes_start"].ctypes.data,
                 a["edges"].ctypes.data, a["roots"].ctypes.data, a["res"].ctypes.data,
                 a["cap"].ctypes.data, None, None, None, None, None, None,
                 a["sinks_start"].ctypes.data, a["sink_nodes"].ctypes.data,
                 a["driver_slew"].ctypes.data, None)
    return f, a


def _result(r):
    if r.status not in (0,):
        raise OtgError("otg_server request", r.status)
    return {"worst_slew": np.array(r.worst_slew[:], np.float32),
            "worst_delay": np.array(r.worst_delay[:], np.float32),
            "dirty_nets": int(r.dirty_nets),
            "latency_s": (r.t_done_ns - r.t_submit_ns) * 1e-9}


def _updates(cap, slew):
    if cap is None:
        cap = (np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros((0, NC), np.float32))
    if slew is None:
        slew = (np.zeros(0, np.int32), np.zeros((0, NC), np.float32))
    cn = np.ascontiguousarray(cap[0], np.int32)
    cv = np.ascontiguousarray(cap[1], np.int32)
    cval = np.ascontiguousarray(cap[2], np.float32).reshape(-1, NC)
    sn = np.ascontiguousarray(slew[0], np.int32)
    sval = np.ascontiguousarray(slew[1], np.float32).reshape(-1, NC)
    assert len(cn) == len(cv) == len(cval) and len(sn) == len(sval)
    return cn, cv, cval, sn, sval


class TimingServer:
    """Host handle of an otg_server on the current CUDA device.

    budget_bytes: device memory the designs may hold (0: no limit);
    slots: batches in flight; max_requests / max_updates: one batch's
    capacity (a request with more updates than max_updates is refused).
    """

    def __init__(self, budget_bytes=0, slots=4, max_requests=64, max_updates=1 << 16):
        self._h = ctypes.c_void_p()
        check("otg_server_create", lib().otg_server_create(
            budget_bytes, slots, max_requests, max_updates, ctypes.byref(self._h)))
        self._designs = {}

    def close(self):
        if self._h:
            lib().otg_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add_design(self, design):
        """Uploads and fully times a design (dict of numpy arrays as from
        synth_design).  Returns (design_id, footprint_bytes); raises
        OtgError(OTG_ERR_ADMISSION) when the budget has no room."""
        f, keep = _forest(design)
        did = ctypes.c_int32()
        fp = ctypes.c_size_t()
        check("otg_server_add_design", lib().otg_server_add_design(
            self._h, ctypes.byref(f), ctypes.byref(did), ctypes.byref(fp)))
        self._designs[did.value] = (int(f.total_nodes), len(keep["sink_nodes"]))
        return did.value, fp.value

    def remove_design(self, d):
        check("otg_server_remove_design", lib().otg_server_remove_design(self._h, d))
        self._designs.pop(d, None)

    def submit(self, d, cap=None, slew=None):
        """Queues a request: cap = (net, local node, [k,4] values), slew =
        (net, [k,4] values).  Returns a ticket for wait()."""
        cn, cv, cval, sn, sval = _updates(cap, slew)
        t = ctypes.c_int64()
        check("otg_server_submit", lib().otg_server_submit(
            self._h, d, len(cn), cn.ctypes.data, cv.ctypes.data, cval.ctypes.data, len(sn),
            sn.ctypes.data, sval.ctypes.data, ctypes.byref(t)))
        return t.value

    def wait(self, ticket, timeout_ms=-1):
        r = RcResult()
        check("otg_server_wait", lib().otg_server_wait(self._h, ticket, timeout_ms,
                                                       ctypes.byref(r)))
        return _result(r)

    def update_sync(self, d, cap=None, slew=None):
        """The same request, applied and timed by itself (blocking)."""
        cn, cv, cval, sn, sval = _updates(cap, slew)
        r = RcResult()
        check("otg_server_update_sync", lib().otg_server_update_sync(
            self._h, d, len(cn), cn.ctypes.data, cv.ctypes.data, cval.ctypes.data, len(sn),
            sn.ctypes.data, sval.ctypes.data, ctypes.byref(r)))
        return _result(r)

    def replay(self, trace, plain=False):
        """Open-loop replay of a request trace (dict from request_trace):
        returns (latency_s per request, makespan_s).  plain=True applies
        the requests one at a time with update_sync instead of batching."""
        t = {k: np.ascontiguousarray(v) for k, v in trace.items()}
        lat = np.zeros(len(t["arrival_ns"]), np.int64)
        span = ctypes.c_int64()
        check("otg_server_replay", lib().otg_server_replay(
            self._h, len(lat), t["arrival_ns"].ctypes.data, t["design"].ctypes.data,
            t["cap_start"].ctypes.data, t["cap_net"].ctypes.data, t["cap_node"].ctypes.data,
            t["cap_val"].ctypes.data, t["slew_start"].ctypes.data, t["slew_net"].ctypes.data,
            t["slew_val"].ctypes.data, 1 if plain else 0, lat.ctypes.data, ctypes.byref(span)))
        return lat * 1e-9, span.value * 1e-9

    def stats(self):
        """(batches launched, requests they carried) since creation."""
        b, r = ctypes.c_int64(), ctypes.c_int64()
        check("otg_server_stats", lib().otg_server_stats(self._h, ctypes.byref(b), ctypes.byref(r)))
        return b.value, r.value

    def read(self, d):
        """A design's per-node outputs (BFS order) and sink slews."""
        V, S = self._designs[d]
        out = {"node2bfs": np.empty(V, np.int32)}
        for k in ("load", "delay", "ldelay", "impulse"):
            out[k] = np.empty((V, NC), np.float32)
        out["sink_slew"] = np.empty((S, NC), np.float32)
        check("otg_server_read", lib().otg_server_read(
            self._h, d, out["node2bfs"].ctypes.data, out["load"].ctypes.data,
            out["delay"].ctypes.data, out["ldelay"].ctypes.data, out["impulse"].ctypes.data,
            out["sink_slew"].ctypes.data))
        return out


__all__ = ["TimingServer", "synth_design", "STATUS"]
