"""Served incremental timing of gate-level designs: several designs resident
on the device as one union, requests that resize gates and ask for the
design's worst slack, batched across designs.

    ds = DesignSet([build_design(dir, keep) for ...])   # device-resident union
    srv = GateServer(ds)
    lat, span, results = srv.replay(trace)                # continuous batching
    lat, span, results = srv.replay(trace, plain=True)    # one request at a time

A request (design d, [(gate, cell), ...]) is Timer::repower_gate for each
gate followed by update_timing and report_wns on design d
(ot/timer/timer.cpp:57-118, 1239-1334).  The designs share one cell
library, so the union's timing records and look-up tables are the
library's once.  A batch takes at most one request per design -- the
oldest pending one -- so every request sees exactly the state its design's
earlier requests left, whatever else is in the batch: its result is the
same alone and in the mix.  A batch is one launch set on one stream:
otg_apply_updates (all its resizes), otg_rc_timing_subset (all their dirty
nets), otg_propagate_items over only the batch's designs' pins (the union's
level order filtered to them, so their level chains run side by side), and
otg_worst_slack_groups (one row per design), copied back into pinned host
memory.  Requests that arrive while batches run are taken into the next
batch (continuous batching); two batches can be in flight, queued in
order on the stream.
"""
import ctypes
import os
import time

import numpy as np

from . import RcBatch, _ptr, _stream, check, designgen, lib
from .prop import TimingGraph, attach_nets, rc_inputs
from .sizing import ResizeTable
from .spef import read_spef

NC = 4


def build_design(dirpath, keep):
    """Host side of one design: its attached timing graph arrays, pin names,
    RC forest (with pin caps) and resize table."""
    arrays, names, pin_net = designgen.timing_graph(keep)
    f = read_spef(os.path.join(dirpath, "design.spef"), r_scale=np.float32(1e-3))
    cap, node_of = rc_inputs(f, designgen.pin_caps(keep))
    attached = attach_nets(arrays, names, pin_net, f, node_of)
    table = ResizeTable(keep, arrays, f, node_of)
    forest = {k: np.asarray(f[k]) for k in ("nodes_start", "edges", "roots", "res")}
    forest["cap"] = cap
    return {"arrays": attached, "names": names, "forest": forest, "table": table,
            "gates": [g for g, _, _ in keep["gates"]]}


def union_arrays(designs):
    """The union of the designs' timing graphs in the otg_prop_graph
    layout, over the first design's timing records and tables (the library
    they share): (arrays, pins per design, pin / arc / net / node offsets,
    per design the map of its record ids to the first design's)."""
    base = designs[0]["arrays"]
    canon = base["records"]
    P = [int(d["arrays"]["num_pins"]) for d in designs]
    A = [len(d["arrays"]["arc_from"]) for d in designs]
    N = [len(d["forest"]["roots"]) for d in designs]
    V = [int(d["forest"]["nodes_start"][-1]) for d in designs]
    off = lambda x: np.concatenate([[0], np.cumsum(x)]).astype(np.int64)  # noqa: E731
    p_off, a_off, n_off, v_off = off(P), off(A), off(N), off(V)
    rec_map = []
    for d in designs:
        inv = np.full(len(d["arrays"]["timing"]), -1, np.int64)
        for key, r in d["arrays"]["records"].items():
            inv[r] = canon[key]
        rec_map.append(inv)

    def cat(k, f):
        return np.concatenate([f(i, d["arrays"][k]) for i, d in enumerate(designs)])
    u = {"num_pins": int(p_off[-1]), "period": base["period"], "timing": base["timing"],
         "lut_meta": base["lut_meta"], "lut_data": base["lut_data"]}
    u["arc_from"] = cat("arc_from", lambda i, x: x + p_off[i])
    u["arc_to"] = cat("arc_to", lambda i, x: x + p_off[i])
    u["arc_kind"] = cat("arc_kind", lambda i, x: x)
    u["arc_node"] = cat("arc_node", lambda i, x: x)
    u["arc_net"] = cat("arc_net", lambda i, x: np.where(x >= 0, x + n_off[i], -1))
    u["arc_timing"] = cat("arc_timing", lambda i, x: np.where(
        x >= 0, rec_map[i][np.maximum(x, 0)], -1))
    u["test_arc"] = cat("test_arc", lambda i, x: x + a_off[i])
    for k in ("pi_at", "pi_slew", "po_rat"):
        u[k] = cat(k, lambda i, x: x)
    for k in ("arc_from", "arc_to", "arc_kind", "arc_node", "arc_net", "arc_timing", "test_arc"):
        u[k] = u[k].astype(np.int32)
    return u, P, p_off, a_off, n_off, v_off, rec_map


class DesignSet:
    """Designs (build_design outputs over one shared library) as one union on
    the device: pins, arcs, nets and RC nodes of design d follow those of
    design d-1; pin_group gives each pin its design."""

    def __init__(self, designs, device="cuda"):
        import torch
        self.designs = designs
        for d in designs:  # the device state is built with the initial cells
            d["table"].reset()
        G = len(designs)
        u, P, self.p_off, self.a_off, self.n_off, self.v_off, self.rec_map = union_arrays(designs)
        self.graph = TimingGraph(u, device=device)
        fz = [d["forest"] for d in designs]
        ns = np.concatenate([[0]] + [f["nodes_start"][1:].astype(np.int64) + self.v_off[i]
                                     for i, f in enumerate(fz)])
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
        self.batch = RcBatch(t(ns.astype(np.int32)),
                             t(np.concatenate([f["edges"] for f in fz]).astype(np.int32)),
                             t(np.concatenate([f["roots"] for f in fz]).astype(np.int32)),
                             t(np.concatenate([f["res"] for f in fz]).astype(np.float32)),
                             t(np.concatenate([f["cap"] for f in fz]).astype(np.float32)))
        group = np.repeat(np.arange(G, dtype=np.int32), P)
        self.pin_group = t(group)
        self.G, self.P, self.device = G, int(self.p_off[-1]), device
        # the union's level order regrouped design by design (stable, so each
        # design keeps its level order): design d's pins are the slice
        # seg[d]:seg[d+1], which one design alone propagates.  Several
        # designs take the union's order filtered to their pins instead, so
        # their level chains run side by side (consecutive slices would run
        # one design's chain after another's).
        order = self.graph.order.cpu().numpy()
        by_design = order[np.argsort(group[order], kind="stable")]
        self.dorder = t(by_design.astype(np.int32))
        self.order_group = t(group[order].astype(np.int64))
        self.seg = np.concatenate([[0], np.cumsum(np.bincount(group[order], minlength=G))]
                                  ).astype(np.int64)
        self.status = torch.zeros(1, dtype=torch.int32, device=device)
        self.batch.run()
        self.graph.propagate(self.batch)
        self.check()

    def updates(self, d, resizes):
        """Union-space update arrays of one request on design d (advances
        that design's record of its cells)."""
        cap_row, cap_val, arc_slot, arc_rec, nets = self.designs[d]["table"].updates(resizes)
        return (cap_row + np.int32(self.v_off[d]), cap_val,
                arc_slot + np.int32(2 * self.a_off[d]),
                self.rec_map[d][arc_rec].astype(np.int32), nets + np.int32(self.n_off[d]))

    def check(self, stream=None):
        self.batch.check(stream)
        self.graph.check(stream)
        if int(self.status.item()) != 0:
            from ._lib import OtgError
            raise OtgError("otg_apply_updates", int(self.status.item()))

    def pins(self, d):
        """{pin name: [4,4] at/slew/rat/slack by corner} of design d (rat
        blanked where the pin has no arrival, as the reference reports)."""
        r = self.graph.result()
        p0, p1 = int(self.p_off[d]), int(self.p_off[d + 1])
        r = {k: v[p0:p1] for k, v in r.items()}
        r["rat"] = np.where(np.isnan(r["at"]), np.nan, r["rat"])
        return {n: np.stack([r[k][i] for k in ("at", "slew", "rat", "slack")])
                for i, n in enumerate(self.designs[d]["names"])}


class _Slot:
    """Device and pinned buffers of one batch in flight."""

    def __init__(self, ds, max_updates, max_arcs, max_nets):
        import torch
        dev, G = ds.device, ds.G
        pin = lambda shape, dt: torch.empty(shape, dtype=dt).pin_memory()  # noqa: E731
        self.h = {"cap_row": pin(max_updates, torch.int32), "cap_val": pin((max_updates, NC),
                                                                           torch.float32),
                  "arc_slot": pin(max_arcs, torch.int32), "arc_rec": pin(max_arcs, torch.int32),
                  "nets": pin(max_nets, torch.int32), "num": pin(1, torch.int32),
                  "active": pin(G, torch.uint8), "wns": pin((G, NC), torch.float32)}
        self.d = {k: torch.empty(v.shape, dtype=v.dtype, device=dev)
                  for k, v in self.h.items() if k != "wns"}
        self.d["wns"] = torch.empty((G, NC), dtype=torch.float32, device=dev)
        self.items = torch.empty(int(ds.seg[-1]) + 1, dtype=torch.int32, device=dev)
        self.scratch = torch.empty(4 * G, dtype=torch.int32, device=dev)
        self.event = torch.cuda.Event()
        self.reqs = None


class GateServer:
    """Continuous batching over a DesignSet (see the module docstring)."""

    def __init__(self, ds, max_updates=1 << 16, max_arcs=1 << 17, max_nets=1 << 16, slots=2):
        import torch
        self.ds = ds
        self.stream = torch.cuda.Stream(device=ds.device)
        self.slots = [_Slot(ds, max_updates, max_arcs, max_nets) for _ in range(slots)]
        self.max = (max_updates, max_arcs, max_nets)

    def _launch(self, slot, reqs):
        """Enqueues one batch (reqs: [(k, design, resizes)], designs distinct)."""
        import torch
        ds = self.ds
        parts = [ds.updates(d, rz) for _, d, rz in reqs]
        cr = np.concatenate([p[0] for p in parts])
        cv = np.concatenate([p[1] for p in parts]).reshape(-1, NC)
        asl = np.concatenate([p[2] for p in parts])
        ar = np.concatenate([p[3] for p in parts])
        nets = np.concatenate([p[4] for p in parts])
        if len(cr) > self.max[0] or len(asl) > self.max[1] or len(nets) > self.max[2]:
            raise ValueError("batch larger than the server's buffers")
        h, dv = slot.h, slot.d
        h["cap_row"][:len(cr)].numpy()[:] = cr
        h["cap_val"][:len(cr)].numpy()[:] = cv
        h["arc_slot"][:len(asl)].numpy()[:] = asl
        h["arc_rec"][:len(ar)].numpy()[:] = ar
        h["nets"][:len(nets)].numpy()[:] = nets
        h["num"].numpy()[0] = len(nets)
        act = h["active"].numpy()
        act[:] = 0
        for _, d, _ in reqs:
            act[d] = 1
        s = self.stream
        with torch.cuda.stream(s):
            for k, n in (("cap_row", len(cr)), ("cap_val", len(cr)), ("arc_slot", len(asl)),
                         ("arc_rec", len(ar)), ("nets", len(nets)), ("num", 1),
                         ("active", ds.G)):
                if n:
                    dv[k][:n].copy_(h[k][:n], non_blocking=True)
        # the pins to propagate: one design's slice of the grouped order, or
        # the union's order filtered to the batch's designs (an
        # order-preserving compaction on the device; its size is known here)
        designs = sorted(d for _, d, _ in reqs)
        if len(designs) == 1:
            d0 = designs[0]
            items = ds.dorder[int(ds.seg[d0]):int(ds.seg[d0 + 1])]
        else:
            k = int(sum(ds.seg[d + 1] - ds.seg[d] for d in designs))
            with torch.cuda.stream(s):
                keep = dv["active"][ds.order_group].to(torch.int32)
                pos = torch.cumsum(keep, 0, dtype=torch.int32) - 1
                idx = torch.where(keep.bool(), pos, k).long()  # the rest to the spare slot k
                slot.items.scatter_(0, idx, ds.graph.order)
            items = slot.items[:k]
        L, b, g = lib(), ds.batch, ds.graph
        st = _stream(s)
        check("otg_apply_updates", L.otg_apply_updates(
            len(cr), _ptr(dv["cap_row"]), _ptr(dv["cap_val"]), _ptr(b.cap), b.total_nodes,
            len(asl), _ptr(dv["arc_slot"]), _ptr(dv["arc_rec"]), _ptr(g.dev["arc_timing"]), g.A,
            _ptr(ds.status), st))
        if len(nets):
            check("otg_rc_timing_subset", L.otg_rc_timing_subset(
                ctypes.byref(b._forest), b.max_net_nodes, _ptr(dv["nets"]), _ptr(dv["num"]),
                len(nets), _ptr(b.workspace), b.workspace.numel(), st))
        from .prop import PropRc
        rc = PropRc(_ptr(b.nodes_start).value, _ptr(b.node2bfs).value, _ptr(b.load).value,
                    _ptr(b.delay).value, _ptr(b.impulse).value)
        o = g.out
        check("otg_propagate_items", L.otg_propagate_items(
            ctypes.byref(g.graph), ctypes.byref(rc), _ptr(items), int(items.numel()),
            _ptr(o["at"]), _ptr(o["slew"]), _ptr(o["rat"]), _ptr(o["slack"]),
            _ptr(g.workspace), g.workspace.numel(), st))
        check("otg_worst_slack_groups", L.otg_worst_slack_groups(
            _ptr(o["slack"]), ds.P, _ptr(ds.pin_group), _ptr(dv["active"]), ds.G,
            _ptr(slot.scratch), _ptr(dv["wns"]), st))
        with torch.cuda.stream(s):
            h["wns"].copy_(dv["wns"], non_blocking=True)
        slot.event.record(s)
        slot.reqs = reqs

    def replay(self, trace, plain=False):
        """Serves a trace: arrival [R] (seconds from the start), design [R],
        resizes [R] (lists).  Latency counts from each request's scheduled
        arrival to the moment its batch is seen complete.  Returns
        (latency seconds [R], span seconds, worst slack [R][4])."""
        arr = np.asarray(trace["arrival"], np.float64)
        des = np.asarray(trace["design"], np.int64)
        rz = trace["resizes"]
        R = len(arr)
        lat = np.zeros(R)
        res = np.zeros((R, NC), np.float32)
        queues = [[] for _ in range(self.ds.G)]  # per design, pending request ids
        nxt, done = 0, 0
        free = list(self.slots)
        busy = []
        t0 = time.perf_counter()
        while done < R:
            now = time.perf_counter() - t0
            while nxt < R and arr[nxt] <= now:
                queues[des[nxt]].append(nxt)
                nxt += 1
            # completions
            for slot in list(busy):
                if slot.event.query():
                    tdone = time.perf_counter() - t0
                    w = slot.h["wns"].numpy()
                    for k, d, _ in slot.reqs:
                        lat[k] = tdone - arr[k]
                        res[k] = w[d]
                    done += len(slot.reqs)
                    busy.remove(slot)
                    free.append(slot)
            if free and (not plain or not busy):
                # the oldest pending request of every design not in flight...
                # (in flight is fine too: batches run in order on the stream)
                heads = [(q[0], d) for d, q in enumerate(queues) if q]
                if heads:
                    heads.sort()
                    if plain:
                        heads = heads[:1]
                    reqs = [(k, d, rz[k]) for k, d in heads]
                    for _, d in heads:
                        queues[d].pop(0)
                    slot = free.pop(0)
                    self._launch(slot, reqs)
                    busy.append(slot)
                    continue
            if not busy and nxt < R and not any(queues):
                time.sleep(max(0.0, min(arr[nxt] - now, 1e-3)))
        span = time.perf_counter() - t0
        self.ds.check()
        return lat, span, res


def request_trace(designs, seed, num, rate, lo=1, hi=64, at_zero=False):
    """A seeded request stream: Poisson arrivals at `rate` per second (or all
    at time 0), a uniformly chosen design each, resizing lo..hi distinct
    random combinational gates of it to another drive strength.  designs:
    the designs' keep dicts (designgen.write_design), in the DesignSet's
    order."""
    from .sizing import cell_family
    rng = np.random.default_rng(seed)
    arrival = np.zeros(num) if at_zero else np.cumsum(rng.exponential(1.0 / rate, num))
    design = rng.integers(0, len(designs), num)
    cur = [{g: c for g, c, _ in keep["gates"]} for keep in designs]
    names = [[g for g, c, _ in keep["gates"] if cell_family(c) != "DFF"] for keep in designs]
    fam = {}
    for c in sorted(designs[0]["libs"]["late"]):
        fam.setdefault(cell_family(c), []).append(c)
    resizes = []
    for d in design.tolist():
        k = int(rng.integers(lo, hi + 1))
        pick = rng.choice(len(names[d]), size=min(k, len(names[d])), replace=False)
        step = []
        for i in pick.tolist():
            g = names[d][i]
            options = [c for c in fam[cell_family(cur[d][g])] if c != cur[d][g]]
            c = options[int(rng.integers(len(options)))]
            cur[d][g] = c
            step.append((g, c))
        resizes.append(step)
    return {"arrival": arrival, "design": design, "resizes": resizes}
