"""Incremental gate sizing on a device-resident design: the GPU form of
Timer::repower_gate + update_timing (ot/timer/timer.cpp:57-118, 1239-1334).

    d = SizingDesign(dirpath, keep)       # designgen.write_design's files + keep
    d.resize([(gate, "NAND2_X2"), ...])   # one batch of resizes, then re-time
    d.worst_slack()                       # per corner [4]
    d.result()                            # at / slew / rat / slack [P][4]

A resize remaps the gate's pins to the new cell (Pin::_remap_cellpin,
ot/timer/pin.cpp:382-399): each input pin's node in its net's RC tree takes
the new cell pin's capacitance (the SPEF ground cap plus the pin cap, as
the flat RC path adds it, ot/timer/net.cpp:433-446) and its net becomes
dirty; the gate's cell arcs take the new cell's timing records.  A batch
is applied on the device by otg_apply_updates, the dirty nets are re-timed
by otg_rc_timing_subset and the timing graph is propagated again by
otg_propagate; otg_worst_slack reduces the slack.  Nothing of the design
goes back to the host except what is asked for.

prepare() turns a sequence of batches into device arrays once, so a timed
loop (run_prepared) issues only launches: each batch's launch set is
queued behind the previous one on one stream, and its worst slack lands in
a device row of its own.
"""
import ctypes
import os

import numpy as np

from . import RcBatch, _ptr, _stream, check, designgen, lib
from .prop import TimingGraph, attach_nets, change_nets, rc_inputs
from .spef import read_spef

NC = 4


def cell_family(cell):
    """NAND2_X2 -> NAND2."""
    return cell.rsplit("_X", 1)[0]


class ResizeTable:
    """What a resize changes, host side: for every gate its input pins' flat
    RC rows and nets, its cell arcs (arc, split, cell pin, timing group),
    the timing record of every (cell, split, cell pin, group), the cells'
    pin capacitances and the SPEF ground capacitance of every RC node."""

    def __init__(self, keep, arrays, spef, node_of):
        self.gcap = np.asarray(spef["cap"], np.float32)  # SPEF ground caps [V,4]
        self.records = arrays["records"]
        self.gate_arcs = arrays["gate_arcs"]
        self.lib = keep["libs"]["late"]  # pin caps (the same in both libraries)
        self.gates = [g for g, _, _ in keep["gates"]]
        self.gate_index = {g: i for i, g in enumerate(self.gates)}
        self.cell_of = [c for _, c, _ in keep["gates"]]
        self.cell0 = list(self.cell_of)
        ns = np.asarray(spef["nodes_start"], np.int64)
        net_idx = {n: i for i, n in enumerate(spef["net_names"])}
        self.gate_inputs = []  # per gate: (cell pin, flat RC row, net) of its inputs
        for inst, cell, conn in keep["gates"]:
            ins = []
            for cp, net in conn.items():
                if cp not in self.lib[cell]["caps"]:
                    continue  # an output pin
                i = net_idx.get(net)
                node = node_of.get((i, f"{inst}:{cp}")) if i is not None else None
                if node is not None:
                    ins.append((cp, int(ns[i] + node), i))
            self.gate_inputs.append(ins)

    def reset(self):
        """Every gate back at the cell the design was built with."""
        self.cell_of = list(self.cell0)

    def current_pin_caps(self, design):
        """pin_caps (designgen.pin_caps) for the gates' current cells."""
        return designgen.pin_caps(dict(design, gates=[
            (g, c, conn) for (g, _, conn), c in zip(design["gates"], self.cell_of)]))

    def relayout(self, ns_old, ns_new, nets, ground, node_of_new):
        """After a change SPEF replaced the trees of forest nets `nets`
        (RcBatch.replace_nets: every net moves to the new layout ns_new;
        the replaced ones have new local ids, node_of_new {(net, pin name):
        node}, and new ground caps `ground`, their trees' rows in `nets`
        order): the ground caps and the gate input pins' rows follow."""
        ns_old, ns_new = np.asarray(ns_old, np.int64), np.asarray(ns_new, np.int64)
        nets = np.asarray(nets, np.int64)
        N = len(ns_old) - 1
        changed = np.zeros(N, bool)
        changed[nets] = True
        net_of = np.repeat(np.arange(N), np.diff(ns_old))
        keep = ~changed[net_of]
        rows = np.arange(int(ns_old[-1]))[keep]
        gcap = np.zeros((int(ns_new[-1]), NC), np.float32)
        gcap[ns_new[net_of[keep]] + (rows - ns_old[net_of[keep]])] = self.gcap[rows]
        g0 = 0
        for i in nets.tolist():
            n = int(ns_new[i + 1] - ns_new[i])
            gcap[ns_new[i]:ns_new[i] + n] = ground[g0:g0 + n]
            g0 += n
        self.gcap = gcap
        for gi, ins in enumerate(self.gate_inputs):
            moved = []
            for cp, row, net in ins:
                if changed[net]:
                    node = node_of_new.get((net, f"{self.gates[gi]}:{cp}"))
                    if node is not None:
                        moved.append((cp, int(ns_new[net] + node), net))
                else:
                    moved.append((cp, int(ns_new[net] + row - ns_old[net]), net))
            self.gate_inputs[gi] = moved

    def updates(self, resizes):
        """Host arrays of one batch of resizes [(gate name or index, cell),
        ...], applied in order (a gate resized twice keeps the last cell):
        (cap_row [U], cap_val [U,4], arc_slot [K], arc_rec [K], nets [D]).
        Advances the table's record of each gate's cell."""
        rows, arcs = {}, {}
        for g, cell in resizes:
            gi = self.gate_index[g] if isinstance(g, str) else int(g)
            old = self.cell_of[gi]
            if cell_family(old) != cell_family(cell):
                raise ValueError(f"{self.gates[gi]}: {old} -> {cell} changes the function")
            self.cell_of[gi] = cell
            caps = self.lib[cell]["caps"]
            for cp, row, net in self.gate_inputs[gi]:
                # float32 add, as the flat path adds the pin cap to the node
                rows[row] = (self.gcap[row] + np.float32(caps[cp]), net)
            for arc, el, cp, k in self.gate_arcs[gi]:
                arcs[2 * arc + el] = self.records[(cell, el, cp, k)]
        cap_row = np.fromiter(rows.keys(), np.int32, len(rows))
        cap_val = np.array([v for v, _ in rows.values()], np.float32).reshape(-1, NC)
        nets = np.unique(np.fromiter((n for _, n in rows.values()), np.int32, len(rows)))
        arc_slot = np.fromiter(arcs.keys(), np.int32, len(arcs))
        arc_rec = np.fromiter(arcs.values(), np.int32, len(arcs))
        return cap_row, cap_val, arc_slot, arc_rec, nets


class SizingDesign:
    """A designgen design (its files in `dirpath` and the in-memory `keep`)
    resident on the device, with the metadata of every gate's resize."""

    def __init__(self, dirpath, keep, device="cuda", stream=None):
        import torch
        self.keep = keep
        arrays, names, pin_net = designgen.timing_graph(keep)
        f = read_spef(os.path.join(dirpath, "design.spef"), r_scale=np.float32(1e-3))
        self.names = names
        cap, node_of = rc_inputs(f, designgen.pin_caps(keep))
        self.table = ResizeTable(keep, arrays, f, node_of)
        attached = attach_nets(arrays, names, pin_net, f, node_of)
        self.graph = TimingGraph(attached, device=device)
        # what the Timer-style queries need: endpoints (primary outputs and
        # the constrained pins of the timing tests), nets by name, pin nodes
        po = np.where(np.any(~np.isnan(np.asarray(attached["po_rat"])), axis=1))[0]
        tests = np.asarray(attached["arc_to"])[np.asarray(attached["test_arc"], np.int64)]
        self.endpoints = np.unique(np.concatenate([po, tests]).astype(np.int64))
        self.net_names = list(f["net_names"])
        self.nodes_start = np.asarray(f["nodes_start"], np.int64)
        self.node_of = node_of  # (net index, pin name) -> local RC node
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(device)  # noqa: E731
        self.batch = RcBatch(t(f["nodes_start"]), t(f["edges"].copy()), t(f["roots"]),
                             t(f["res"]), t(cap))
        self.P = self.graph.P
        self.status = torch.zeros(1, dtype=torch.int32, device=device)
        self.scratch = torch.zeros(4, dtype=torch.int32, device=device)
        self.wns = torch.zeros(NC, dtype=torch.float32, device=device)
        self.device = device
        self.batch.run(stream)
        self.graph.propagate(self.batch, stream)

    def updates(self, resizes):
        return self.table.updates(resizes)

    def change_spef(self, path, stream=None):
        """A change SPEF (Timer::read_spef + update_timing on the nets it
        names, ot/timer/spef.cpp:40-53): the named nets get their new trees,
        with the pin caps of the gates' current cells; every other net keeps
        its tree and results (RcBatch.replace_nets); the net arcs into the
        changed nets, the resize table's rows and the queries' node map
        follow the new layout; then the design is propagated again.
        Returns the forest indices of the changed nets."""
        f = read_spef(path, r_scale=np.float32(1e-3))
        net_index = {n: i for i, n in enumerate(self.net_names)}
        nets, forest, node_of_c, ground = change_nets(
            f, net_index, self.table.current_pin_caps(self.keep), with_ground=True)
        if len(nets) == 0:
            return nets
        ns_old = self.nodes_start
        self.batch = self.batch.replace_nets(nets, *forest, stream=stream)
        ns_new = self.batch.nodes_start.cpu().numpy().astype(np.int64)
        self.graph.change_nets(nets, node_of_c, self.names)
        self.table.relayout(ns_old, ns_new, nets, ground, node_of_c)
        changed = set(np.asarray(nets).tolist())
        self.node_of = {k: v for k, v in self.node_of.items() if k[0] not in changed}
        self.node_of.update(node_of_c)
        self.nodes_start = ns_new
        self.graph.propagate(self.batch, stream)
        g = self.graph
        check("otg_worst_slack", lib().otg_worst_slack(_ptr(g.out["slack"]), self.P,
                                                       _ptr(self.scratch), _ptr(self.wns),
                                                       _stream(stream)))
        return nets

    # -------------------------------------------------------------- device
    def _launch(self, cap_row, cap_val, n_cap, arc_slot, arc_rec, n_arc, nets, n_nets_dev,
                max_nets, wns_out, stream):
        L = lib()
        s = _stream(stream)
        b, g = self.batch, self.graph
        check("otg_apply_updates", L.otg_apply_updates(
            n_cap, cap_row, cap_val, _ptr(b.cap), b.total_nodes, n_arc, arc_slot, arc_rec,
            _ptr(g.dev["arc_timing"]), g.A, _ptr(self.status), s))
        if max_nets:
            check("otg_rc_timing_subset", L.otg_rc_timing_subset(
                ctypes.byref(b._forest), b.max_net_nodes, nets, n_nets_dev, max_nets,
                _ptr(b.workspace), b.workspace.numel(), s))
        g.propagate(b, stream)
        check("otg_worst_slack", L.otg_worst_slack(_ptr(g.out["slack"]), self.P,
                                                   _ptr(self.scratch), wns_out, s))

    def resize(self, resizes, stream=None):
        """Applies one batch of resizes and re-times the design (enqueued
        on `stream`; read the results with worst_slack() or result())."""
        import torch
        cap_row, cap_val, arc_slot, arc_rec, nets = self.updates(resizes)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)  # noqa: E731
        keep = [t(cap_row), t(cap_val), t(arc_slot), t(arc_rec), t(nets),
                torch.tensor([len(nets)], dtype=torch.int32, device=self.device)]
        self._keep = keep  # alive until the stream has used them
        self._launch(_ptr(keep[0]), _ptr(keep[1]), len(cap_row), _ptr(keep[2]), _ptr(keep[3]),
                     len(arc_slot), _ptr(keep[4]), _ptr(keep[5]), len(nets), _ptr(self.wns),
                     stream)
        return self

    def prepare(self, steps):
        """Device arrays for a sequence of resize batches (steps: list of
        resize lists).  Advances the design's cell record through all of
        them; run_prepared then applies them on the device."""
        import torch
        parts = [self.updates(r) for r in steps]
        cat = lambda k, dt, shape=(-1,): np.concatenate(  # noqa: E731
            [np.asarray(p[k], dt).reshape(shape) for p in parts]) if parts else \
            np.zeros(0, dt)
        off = lambda k: np.concatenate(  # noqa: E731
            [[0], np.cumsum([len(p[k]) for p in parts])]).astype(np.int64)
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(self.device)  # noqa: E731
        prep = {"cap_row": t(cat(0, np.int32)), "cap_val": t(cat(1, np.float32, (-1, NC))),
                "arc_slot": t(cat(2, np.int32)), "arc_rec": t(cat(3, np.int32)),
                "nets": t(cat(4, np.int32)),
                "num_nets": t(np.array([len(p[4]) for p in parts], np.int32)),
                "o_cap": off(0), "o_arc": off(2), "o_net": off(4),
                "wns": torch.zeros((len(parts), NC), dtype=torch.float32, device=self.device),
                "steps": len(parts)}
        for k in ("cap_row", "arc_slot", "nets"):
            if prep[k].numel() == 0:
                prep[k] = torch.zeros(1, dtype=torch.int32, device=self.device)
        if prep["cap_val"].numel() == 0:
            prep["cap_val"] = torch.zeros((1, NC), dtype=torch.float32, device=self.device)
        prep["arc_rec"] = prep["arc_rec"] if prep["arc_rec"].numel() else \
            torch.zeros(1, dtype=torch.int32, device=self.device)
        return prep

    def run_prepared(self, prep, first=0, count=None, stream=None, sync_each=False):
        """Applies prepared batches first..first+count-1 in order, each one's
        worst slack into prep["wns"][k].  sync_each: wait for every batch
        and read its worst slack to the host before issuing the next (the
        plain path); otherwise all batches are queued back to back."""
        count = prep["steps"] - first if count is None else count
        base = lambda x: x.data_ptr()  # noqa: E731
        out = []
        for k in range(first, first + count):
            oc, oa, on = prep["o_cap"], prep["o_arc"], prep["o_net"]
            nc, na, nn = int(oc[k + 1] - oc[k]), int(oa[k + 1] - oa[k]), int(on[k + 1] - on[k])
            self._launch(ctypes.c_void_p(base(prep["cap_row"]) + 4 * int(oc[k])),
                         ctypes.c_void_p(base(prep["cap_val"]) + 16 * int(oc[k])), nc,
                         ctypes.c_void_p(base(prep["arc_slot"]) + 4 * int(oa[k])),
                         ctypes.c_void_p(base(prep["arc_rec"]) + 4 * int(oa[k])), na,
                         ctypes.c_void_p(base(prep["nets"]) + 4 * int(on[k])),
                         ctypes.c_void_p(base(prep["num_nets"]) + 4 * k), nn,
                         ctypes.c_void_p(base(prep["wns"]) + 16 * k), stream)
            if sync_each:
                out.append(prep["wns"][k].cpu().numpy())
        return out

    # ------------------------------------------------------------- results
    def check(self, stream=None):
        """Synchronizes; raises on a device-side error of the last batches."""
        self.batch.check(stream)
        self.graph.check(stream)
        if int(self.status.item()) != 0:
            from ._lib import OtgError
            raise OtgError("otg_apply_updates", int(self.status.item()))

    def worst_slack(self):
        self.check()
        return self.wns.cpu().numpy()

    def result(self):
        self.check()
        return self.graph.result()

    def pins(self):
        """{pin name: [4,4] at/slew/rat/slack by corner} (rat blanked where
        the pin has no arrival, as the reference reports it)."""
        r = self.result()
        r["rat"] = np.where(np.isnan(r["at"]), np.nan, r["rat"])
        return {n: np.stack([r[k][i] for k in ("at", "slew", "rat", "slack")])
                for i, n in enumerate(self.names)}


def resize_trace(keep, seed, steps, per_step, exclude=("DFF",)):
    """A seeded sequence of resize batches: each step picks `per_step`
    distinct gates (not flops) and gives each another drive strength of
    its function.  Returns [[(gate, cell), ...], ...]; the cells follow
    the gates' current cells step by step."""
    rng = np.random.default_rng(seed)
    cells = sorted(keep["libs"]["late"])
    fam = {}
    for c in cells:
        fam.setdefault(cell_family(c), []).append(c)
    gates = [(g, c) for g, c, _ in keep["gates"] if cell_family(c) not in exclude]
    cur = {g: c for g, c in gates}
    names = [g for g, _ in gates]
    out = []
    for _ in range(steps):
        pick = rng.choice(len(names), size=min(per_step, len(names)), replace=False)
        step = []
        for i in pick.tolist():
            g = names[i]
            options = [c for c in fam[cell_family(cur[g])] if c != cur[g]]
            c = options[int(rng.integers(len(options)))]
            cur[g] = c
            step.append((g, c))
        out.append(step)
    return out


def write_ops(path, steps):
    """The repower ops file of oracle/ot_run.cpp: "<gate> <cell>" lines,
    steps separated by "=" lines."""
    with open(path, "w") as f:
        for step in steps:
            for g, c in step:
                f.write(f"{g} {c}\n")
            f.write("=\n")
