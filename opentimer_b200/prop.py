"""Levelized timing propagation on the GPU (otg_propagate in include/otg.h).

    g = TimingGraph(arrays)          # numpy arrays of the otg_prop_graph layout
    out = g.propagate(rc_batch)      # at / slew / rat / slack [P][4], numpy

The graph is flat: pins, arcs (net arcs onto RC nodes of the RcBatch's
forest, cell arcs with a timing record per split), timing records, look-up
tables, timing tests and primary-input/-output assertions.  The pin order
comes from otg_levelize over the graph's fanin CSR.
"""
import ctypes

from itertools import compress

import numpy as np

from . import LevelizeBatch, _ptr, _stream, check, fanin_csr, lib

NC = 4


class PropGraph(ctypes.Structure):
    _fields_ = [("num_pins", ctypes.c_int32), ("num_arcs", ctypes.c_int32),
                ("num_tests", ctypes.c_int32)] + [
        (k, ctypes.c_void_p) for k in
        ["arc_from", "arc_to", "arc_kind", "arc_timing", "arc_net", "arc_node", "fanin_start",
         "fanin", "fanout_start", "fanout", "test_arc", "test_start", "test_of_pin", "pi_at",
         "pi_slew", "po_rat", "timing", "lut_meta", "lut_data"]] + [
        ("period", ctypes.c_float), ("num_lut_data", ctypes.c_int32)]


class PropRc(ctypes.Structure):
    _fields_ = [(k, ctypes.c_void_p) for k in
                ["nodes_start", "node2bfs", "load", "delay", "impulse"]]


def _csr(keys, n):
    """CSR of item indices grouped by key (stable)."""
    keys = np.asarray(keys, np.int64)
    start = np.zeros(n + 1, np.int32)
    start[1:] = np.cumsum(np.bincount(keys, minlength=n))
    return start, np.argsort(keys, kind="stable").astype(np.int32)


class TimingGraph:
    """arrays: arc_from, arc_to, arc_kind, arc_timing [A,2], arc_net,
    arc_node, test_arc, pi_at, pi_slew, po_rat [P,4], timing [R,9],
    lut_meta [L,4], lut_data, period; num_pins.  order: a pin order to use
    instead of levelizing (every pin after all of its fanouts); it is not
    checked, and one that breaks the rule ends in OTG_ERR_TIMEOUT.
    forward: the forward pass's pin order, "sinks" (the backward order
    reversed) or "sources" (a second levelization, by distance from the
    sources: pins start in about the order they become ready, a few percent
    faster per propagation for one more levelization per topology change);
    results are the same."""

    def __init__(self, arrays, device="cuda", order=None, forward="sinks"):
        import torch
        a = arrays
        P = int(a["num_pins"])
        A = len(a["arc_from"])
        self.P, self.A = P, A
        t = lambda x, dt: torch.from_numpy(  # noqa: E731
            np.ascontiguousarray(x, dt).reshape(-1) if np.size(x) else np.zeros(1, dt)).to(device)
        self.dev = {k: t(a[k], np.int32) for k in
                    ("arc_from", "arc_to", "arc_kind", "arc_timing", "arc_net", "arc_node",
                     "timing", "lut_meta")}
        test_arc = np.asarray(a["test_arc"], np.int32)
        self.dev["test_arc"] = t(test_arc, np.int32)
        self.T = len(test_arc)
        # the CSRs of the graph, built on the device (otg_fanin_csr): arcs into
        # and out of every pin, tests at every constrained pin
        self.build_csr()
        # what the host side of an incremental change reads
        self.arc_to = np.asarray(a["arc_to"], np.int32)
        self.net_arcs = net_arc_index(a["arc_kind"], a["arc_net"])
        for k in ("pi_at", "pi_slew", "po_rat", "lut_data"):
            self.dev[k] = t(a[k], np.float32)
        self.graph = PropGraph(P, A, len(test_arc),
                               *[self.dev[k].data_ptr() for k in
                                 ["arc_from", "arc_to", "arc_kind", "arc_timing", "arc_net",
                                  "arc_node", "fanin_start", "fanin", "fanout_start", "fanout",
                                  "test_arc", "test_start", "test_of_pin", "pi_at", "pi_slew",
                                  "po_rat", "timing", "lut_meta", "lut_data"]],
                               float(a["period"]), int(np.size(a["lut_data"])))
        ws = ctypes.c_size_t()
        check("otg_prop_workspace_size", lib().otg_prop_workspace_size(P, A, len(test_arc),
                                                                       ctypes.byref(ws)))
        self.workspace = torch.empty(max(ws.value, 256), dtype=torch.uint8, device=device)
        self.out = {k: torch.empty(P, NC, dtype=torch.float32, device=device)
                    for k in ("at", "slew", "rat", "slack")}
        self.fwd_order, self.fwd_levelizer = None, None
        if order is not None:
            assert len(order) == P
            self.order, self.levelizer, self.num_levels = t(order, np.int32), None, None
            return
        # levels over the pin graph: a pin's level is its longest path to a pin
        # without fanout (otg_levelize, the reference's frontier rule), on the
        # levelization input built on the device
        lb = LevelizeBatch(*self.levelize_input())
        lb.run()
        lb.check()
        self.levelizer = lb  # re-run after a topology change (otg_levelize)
        order, ends, _ = lb.result()
        assert len(order) == P, "the timing graph has a cycle"
        self.order = t(order, np.int32)
        self.level_ends = t(ends, np.int32)
        self.num_levels = len(ends) - 1
        if forward == "sources":
            # the same levelization over the reversed arcs: a pin after all of
            # its fanins, sources first
            fl = LevelizeBatch(*fanin_csr(P, self.dev["arc_to"][:A], self.dev["arc_from"][:A]))
            fl.run()
            fl.check()
            self.fwd_levelizer = fl  # re-run with levelizer after a topology change
            fwd, _, _ = fl.result()
            assert len(fwd) == P, "the timing graph has a cycle"
            self.fwd_order = t(fwd, np.int32)

    def build_csr(self):
        """Fanin and fanout arc lists of every pin and the tests constrained
        at every pin, on the device (otg_fanin_csr, arc order within a pin)."""
        import torch
        P, A = self.P, self.A
        frm, to = self.dev["arc_from"][:A], self.dev["arc_to"][:A]
        self.dev["fanin_start"], fi, _, _ = fanin_csr(P, frm, to, as_arcs=True)
        self.dev["fanout_start"], fo, _, _ = fanin_csr(P, to, frm, as_arcs=True)
        ta = self.dev["test_arc"][:self.T]
        keys = to[ta.long()] if self.T else torch.zeros(0, dtype=torch.int32, device=to.device)
        self.dev["test_start"], tp, _, _ = fanin_csr(P, keys, keys, as_arcs=True)

        def pad(x):
            return x if x.numel() else torch.zeros(1, dtype=torch.int32, device=to.device)
        self.dev["fanin"], self.dev["fanout"], self.dev["test_of_pin"] = pad(fi), pad(fo), pad(tp)

    def levelize_input(self):
        """otg_levelize's input for this graph, built on the device: per pin
        its fanin source pins, fanout counts and the pins without fanout
        (Timer::_build_prop_tasks_cuda steps 1-2)."""
        return fanin_csr(self.P, self.dev["arc_from"][:self.A], self.dev["arc_to"][:self.A])

    def propagate(self, batch, stream=None):
        """Forward and backward propagation on the RC outputs of `batch`
        (an RcBatch whose forest the graph's net arcs refer to)."""
        rc = PropRc(_ptr(batch.nodes_start).value, _ptr(batch.node2bfs).value,
                    _ptr(batch.load).value, _ptr(batch.delay).value, _ptr(batch.impulse).value)
        o = self.out
        check("otg_propagate", lib().otg_propagate(
            ctypes.byref(self.graph), ctypes.byref(rc), _ptr(self.order), _ptr(self.fwd_order),
            _ptr(o["at"]), _ptr(o["slew"]),
            _ptr(o["rat"]), _ptr(o["slack"]), _ptr(self.workspace), self.workspace.numel(),
            _stream(stream)))
        return self

    def propagate_items(self, batch, items, stream=None):
        """Propagation of the listed pins only (items: a CUDA int32 tensor
        in backward level order holding, with each pin, every pin it reads
        that is not final -- e.g. whole designs of a union, see
        otg_propagate_items); every other pin keeps its values."""
        rc = PropRc(_ptr(batch.nodes_start).value, _ptr(batch.node2bfs).value,
                    _ptr(batch.load).value, _ptr(batch.delay).value, _ptr(batch.impulse).value)
        o = self.out
        check("otg_propagate_items", lib().otg_propagate_items(
            ctypes.byref(self.graph), ctypes.byref(rc), _ptr(items), int(items.numel()),
            _ptr(o["at"]), _ptr(o["slew"]), _ptr(o["rat"]), _ptr(o["slack"]),
            _ptr(self.workspace), self.workspace.numel(), _stream(stream)))
        return self

    def change_nets(self, nets, node_of, pin_names):
        """After RcBatch.replace_nets(nets, ...) with change_nets' output:
        points the net arcs into those nets at their sinks' new local ids.
        Returns (arcs, nodes)."""
        arcs, nodes = change_arcs(self.net_arcs, self.arc_to, pin_names, nets, node_of)
        if len(arcs):
            self.set_arc_nodes(arcs, nodes)
        return arcs, nodes

    def set_arc_nodes(self, arcs, nodes):
        """New sink node ids (local to their nets) for some net arcs, as
        after an incremental SPEF replaced their nets' trees."""
        import torch
        arcs = torch.as_tensor(np.asarray(arcs, np.int64), device=self.dev["arc_node"].device)
        self.dev["arc_node"][arcs] = torch.as_tensor(np.asarray(nodes, np.int32),
                                                     device=arcs.device)

    def arc_delays(self):
        """The arc delays of the last propagation on the host, [A][2][2][2]
        by (split, from transition, to transition) -- Arc::_delay, NaN where
        the reference's value is empty (otg_prop_arc_delays)."""
        import torch
        self.check()
        ptr = ctypes.c_void_p()
        check("otg_prop_arc_delays", lib().otg_prop_arc_delays(
            _ptr(self.workspace), self.workspace.numel(), self.A, ctypes.byref(ptr)))
        off = ptr.value - self.workspace.data_ptr()
        raw = self.workspace[off:off + 32 * self.A]
        return raw.view(torch.float32).cpu().numpy().reshape(self.A, 2, 2, 2)

    def check(self, stream=None):
        """Synchronizes; raises if a bounded wait of the last propagation
        gave up (OTG_ERR_TIMEOUT)."""
        check("otg_prop_status", lib().otg_prop_status(_ptr(self.workspace), _stream(stream)))

    def result(self):
        self.check()
        return {k: v.cpu().numpy() for k, v in self.out.items()}


def rc_inputs(spef, pin_caps, net_ids=None):
    """Flat RC inputs from read_spef's output plus each non-root pin's cap
    (pin_caps: name -> [4]), as the flat path adds them (ot/timer/
    net.cpp:433-446).  Returns (cap [V,4], node_of {(net, pin name): the
    pin's local node id in the net}).  With net_ids (an index per net of
    the file, -1 for none), node_of is keyed by those indices and leaves
    out the nets without one."""
    ns, ps = np.asarray(spef["nodes_start"], np.int64), np.asarray(spef["pins_start"])
    cap = spef["cap"].copy()
    names = spef["pin_names"]
    net = np.repeat(np.arange(len(ns) - 1), np.diff(ps))
    node = np.asarray(spef["pin_node"], np.int64)
    on = np.nonzero(node >= 0)[0]
    on_names = [names[q] for q in on.tolist()]
    if net_ids is None:
        node_of = dict(zip(zip(net[on].tolist(), on_names), node[on].tolist()))
    else:
        key = np.asarray(net_ids, np.int64)[net[on]]
        m = key >= 0
        node_of = dict(zip(zip(key[m].tolist(), compress(on_names, m.tolist())),
                           node[on][m].tolist()))
    nonroot = (node[on] != np.asarray(spef["roots"])[net[on]]).tolist()
    rows, vals = [], []
    for row, name, add in zip((ns[net[on]] + node[on]).tolist(), on_names, nonroot):
        c = pin_caps.get(name) if add else None
        if c is not None:
            rows.append(row)
            vals.append(c)
    if rows:  # float32 adds, in pin order (np.add.at is unbuffered)
        np.add.at(cap, np.asarray(rows, np.int64), np.asarray(vals, np.float32))
    return cap, node_of


def _ranges(starts, sizes):
    """Concatenated aranges [starts[k], starts[k] + sizes[k])."""
    sizes = np.asarray(sizes, np.int64)
    total = int(sizes.sum())
    off = np.zeros(len(sizes), np.int64)
    np.cumsum(sizes[:-1], out=off[1:])
    return np.arange(total, dtype=np.int64) - np.repeat(off, sizes) + \
        np.repeat(np.asarray(starts, np.int64), sizes)


def change_nets(spef_change, net_index, pin_caps, with_ground=False):
    """Reads a change SPEF (read_spef output) against a design whose forest
    nets are named by net_index {name: forest net}.  Returns (nets, forest,
    node_of): the forest indices of the nets it names (unknown names are
    skipped, as Timer::_read_spef does, ot/timer/spef.cpp:40-53), their new
    trees as a forest in file order (nodes_start, edges, roots, res, cap
    with the pin caps added) for RcBatch.replace_nets, and node_of
    {(forest net, pin name): local node} for the arcs into them.  With
    with_ground, a fourth item: the trees' SPEF ground caps alone [V', 4]
    (the forest's cap before the pin caps were added)."""
    f = spef_change
    ns = np.asarray(f["nodes_start"], np.int64)
    keep = np.array([i for i, n in enumerate(f["net_names"]) if n in net_index], np.int64)
    nets = np.array([net_index[f["net_names"][i]] for i in keep.tolist()], np.int64)
    net_ids = np.full(len(ns) - 1, -1, np.int64)
    net_ids[keep] = nets
    cap, node_of = rc_inputs(f, pin_caps, net_ids)
    sizes = ns[keep + 1] - ns[keep] if len(keep) else np.zeros(0, np.int64)
    sub_ns = np.zeros(len(keep) + 1, np.int64)
    np.cumsum(sizes, out=sub_ns[1:])
    node_rows = _ranges(ns[keep], sizes)
    edge_rows = _ranges(ns[keep] - keep, sizes - 1)
    forest = (sub_ns.astype(np.int32), f["edges"][edge_rows].copy(),
              np.asarray(f["roots"])[keep].astype(np.int32), f["res"][edge_rows].copy(),
              cap[node_rows].copy())
    if with_ground:
        return nets, forest, node_of, np.asarray(f["cap"], np.float32)[node_rows].copy()
    return nets, forest, node_of


def net_arc_index(arc_kind, arc_net):
    """The graph's net arcs grouped by their forest net, for change_arcs:
    (arcs, nets), both sorted by net (arcs ascending within a net)."""
    arc_net = np.asarray(arc_net)
    na = np.nonzero((np.asarray(arc_kind) == 0) & (arc_net >= 0))[0]
    by = np.argsort(arc_net[na], kind="stable")
    return na[by], arc_net[na][by]


def change_arcs(index, arc_to, pin_names, nets, node_of):
    """The net arcs into the nets a change SPEF replaced (`nets`, forest
    indices), ascending, and their sinks' new local ids from change_nets'
    node_of (-1: the sink is not in the new tree): (arcs, nodes) for
    TimingGraph.set_arc_nodes.  index is net_arc_index's output and arc_to
    the graph's per-arc sink pins, both kept with the design."""
    arcs_by_net, net_of = index
    nets = np.asarray(nets, np.int64)
    if len(nets) == 0:
        return np.zeros(0, np.int64), []
    lo = np.searchsorted(net_of, nets, side="left")
    hi = np.searchsorted(net_of, nets, side="right")
    rows = _ranges(lo, hi - lo)
    by_id = np.argsort(arcs_by_net[rows], kind="stable")
    arcs, arc_nets = arcs_by_net[rows][by_id], net_of[rows][by_id]
    get = node_of.get
    return arcs, [get((i, pin_names[t]), -1)
                  for i, t in zip(arc_nets.tolist(), np.asarray(arc_to)[arcs].tolist())]


def attach_nets(arrays, pin_names, pin_net_names, spef, node_of):
    """Fills arc_net / arc_node of a graph whose net arcs name their net
    (arrays["arc_net_name"]): a net arc gets its forest net and its sink's
    RC node, a cell arc the forest net of the pin it drives (its load)."""
    net_idx = {n: i for i, n in enumerate(spef["net_names"])}
    A = len(arrays["arc_from"])
    arc_net = np.full(A, -1, np.int32)
    arc_node = np.full(A, -1, np.int32)
    for k in range(A):
        to = int(arrays["arc_to"][k])
        if arrays["arc_kind"][k] == 0:
            i = net_idx[arrays["arc_net_name"][k]]
            arc_net[k] = i
            arc_node[k] = node_of.get((i, pin_names[to]), -1)
        else:
            arc_net[k] = net_idx.get(pin_net_names[to], -1)
    out = dict(arrays)
    out["arc_net"], out["arc_node"] = arc_net, arc_node
    return out


def _main():
    """python -m opentimer_b200.prop [--gates N] [--seed S] [--reps R]: a
    seeded design (designgen) through the SPEF reader, the RC pass,
    levelization and R propagations on cuda:0; prints one JSON line with
    the CUDA-event times (the last propagation's)."""
    import argparse
    import json
    import os
    import tempfile
    import torch
    from . import RcBatch, designgen
    from .spef import read_spef
    ap = argparse.ArgumentParser()
    ap.add_argument("--gates", type=int, default=10000)
    ap.add_argument("--seed", type=int, default=77)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()
    with tempfile.TemporaryDirectory() as d:
        keep = {}
        designgen.write_design(d, seed=args.seed, gates=args.gates, keep=keep)
        arrays, names, nets = designgen.timing_graph(keep)
        f = read_spef(os.path.join(d, "design.spef"), r_scale=np.float32(1e-3))
    cap, node_of = rc_inputs(f, designgen.pin_caps(keep))
    g = TimingGraph(attach_nets(arrays, names, nets, f, node_of))
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    b = RcBatch(t(f["nodes_start"]), t(f["edges"].copy()), t(f["roots"]), t(f["res"]), t(cap))
    b.run()
    b.check()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for _ in range(max(args.reps, 1)):
        ev[0].record()
        g.propagate(b)
        ev[1].record()
    g.check()
    out = g.result()
    print(json.dumps({"gates": args.gates, "pins": g.P, "arcs": g.A, "levels": g.num_levels,
                      "propagation_ms": ev[0].elapsed_time(ev[1]),
                      "pins_with_slack": int(np.isfinite(out["slack"]).any(axis=1).sum())}))


if __name__ == "__main__":
    _main()
